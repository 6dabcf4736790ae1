"""Element colouring (color_mesh, generate_element_groups; src/mesh/coloring.jl).

The colouring runs on the host inside libfemtools_b200 and needs no GPU; the
groups feed the conflict-free coloured thermal assembly
(`solver.assemble_diffusion_matrices_colored`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi as abi


def color_mesh(mesh_or_el2n, nnodes: int | None = None) -> np.ndarray:
    """color_mesh_greedy (coloring.jl:26-50): colours 1..n, one per element.

    Accepts a MixedMesh or an nels × nv 1-based connectivity (plus `nnodes`).
    """
    el2n = getattr(mesh_or_el2n, "el2n", mesh_or_el2n)
    el2n = np.ascontiguousarray(el2n, dtype=np.int32)
    nels, nv = el2n.shape
    nn = int(nnodes if nnodes is not None else getattr(mesh_or_el2n, "nnodes", el2n.max(initial=0)))
    colors = np.zeros(nels, dtype=np.int32)
    nc = C.c_int32(0)
    lib = abi.load_library()
    rc = lib.femb200_color_mesh(el2n.ctypes.data, nv, nels, nn, colors.ctypes.data, C.byref(nc))
    if rc != abi.OK:
        raise abi.FemB200Error(rc, "color_mesh: invalid connectivity")
    return colors


@dataclass
class ElementGroups:
    """generate_element_groups (coloring.jl:77-81) as CSR: the 1-based elements of
    colour c are elements[offsets[c-1]:offsets[c]]."""
    offsets: np.ndarray      # int64, ncolors + 1
    elements: np.ndarray     # int32, nels

    @property
    def ncolors(self) -> int:
        return len(self.offsets) - 1

    def group(self, c: int) -> np.ndarray:
        return self.elements[self.offsets[c - 1]:self.offsets[c]]


def generate_element_groups(colors: np.ndarray) -> ElementGroups:
    colors = np.ascontiguousarray(colors, dtype=np.int32)
    nc = int(colors.max(initial=0))
    offsets = np.zeros(nc + 1, dtype=np.int64)
    elements = np.zeros(len(colors), dtype=np.int32)
    lib = abi.load_library()
    rc = lib.femb200_color_groups(colors.ctypes.data, len(colors), nc, offsets.ctypes.data, elements.ctypes.data)
    if rc != abi.OK:
        raise abi.FemB200Error(rc, "generate_element_groups: colours must lie in 1..maximum")
    return ElementGroups(offsets, elements)
