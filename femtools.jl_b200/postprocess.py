"""Post-processing: element-averaged strain-rate and stress diagnostics on the device,
their projection back to nodal old stresses, and the legacy ASCII VTK writer
(src/postprocess/postprocess.jl).

The diagnostics run on the GPU through `femb200_strain_rate_stress`; the projection and
the writer are host code, as in the reference (plain loops over CPU arrays there).
"""
from __future__ import annotations

import collections
import ctypes as C
from typing import Mapping, Optional

import numpy as np

DIAGNOSTIC_FIELDS_2D = ("εxx", "εyy", "εzz", "εxy", "εII", "τxx", "τyy", "τzz", "τxy", "tauII")
DIAGNOSTIC_FIELDS_3D = ("εxx", "εyy", "εzz", "εxy", "εxz", "εyz", "εII",
                        "τxx", "τyy", "τzz", "τxy", "τxz", "τyz", "tauII")
Diagnostics2D = collections.namedtuple("Diagnostics2D", DIAGNOSTIC_FIELDS_2D)
Diagnostics3D = collections.namedtuple("Diagnostics3D", DIAGNOSTIC_FIELDS_3D)


def compute_strain_rate_stress_postprocess(dr, tau=None):
    """compute_strain_rate_stress_postprocess(v, el2n_v, geo_v, τ_ip, element_v)
    (postprocess.jl:84-105 in 2-D, :168-215 in 3-D) for a StokesDR state: per element the
    dΩ-weighted averages of the strain rate of `dr.v`, of the integration-point stress
    `tau` (default `dr.tau`, the current stress; (xx, yy, zz, xy, xz, yz) in 3-D,
    (xx, yy, xy) in 2-D with τzz = −(τxx + τyy)) and of their second invariants. Returns a
    named tuple of device arrays (one value per element) with the reference's field names."""
    import torch
    from . import solver
    tau = dr.tau if tau is None else tau
    dim = dr.mesh.dim
    nt, fields = (6, Diagnostics3D) if dim == 3 else (3, Diagnostics2D)
    if tau is None or len(tau) != nt:
        raise ValueError(f"tau must hold {nt} integration-point components")
    n = dr.mesh.nels * dr.mesh.nq
    tau = [t if isinstance(t, torch.Tensor) else torch.as_tensor(np.asarray(t), dtype=dr.dtype) for t in tau]
    tau = [t.to(device=dr.device, dtype=dr.dtype).reshape(-1).contiguous() for t in tau]
    if any(t.numel() != n for t in tau):
        raise ValueError(f"every stress component must hold nq·nels = {n} values")
    out = [torch.empty(dr.mesh.nels, dtype=dr.dtype, device=dr.device) for _ in fields._fields]
    lib, h = solver._Handle.get()
    p = dr.problem()
    tp = (C.c_void_p * 6)(*([solver._ptr(t) for t in tau] + [0] * (6 - nt)))
    op = (C.c_void_p * 14)(*([solver._ptr(o) for o in out] + [0] * (14 - len(out))))
    solver._check(lib, h, lib.femb200_strain_rate_stress(h, C.byref(p), tp, op))
    return fields(*out)


def update_old_stress_from_cells(tau_old, post, el2n, nnodes):
    """update_old_stress_from_cells!(τ_old, post, el2n_v, nnodes_v) (postprocess.jl:229-256):
    each node takes the mean of the cell-averaged stresses of the elements that contain
    it (3 components in plane strain, 6 in 3-D); nodes in no element keep zero. `tau_old`
    is a list of host arrays (numpy, filled in place) or device tensors (copied into)."""
    nt = len(tau_old)
    names = ("τxx", "τyy", "τxy") if nt == 3 else ("τxx", "τyy", "τzz", "τxy", "τxz", "τyz")
    el2n = np.asarray(el2n, dtype=np.int64) - 1                 # nels × nv
    counts = np.bincount(el2n.ravel(), minlength=nnodes).astype(np.float64)
    for c, name in enumerate(names):
        cells = getattr(post, name)
        cells = cells.detach().cpu().numpy() if hasattr(cells, "detach") else np.asarray(cells)
        nodal = np.bincount(el2n.ravel(), weights=np.repeat(cells, el2n.shape[1]), minlength=nnodes)
        nodal = np.divide(nodal, counts, out=np.zeros(nnodes), where=counts > 0)
        dst = tau_old[c]
        if hasattr(dst, "copy_"):
            import torch
            dst.copy_(torch.as_tensor(nodal, dtype=dst.dtype))
        else:
            dst[...] = nodal
    return tau_old


# ---- legacy ASCII VTK --------------------------------------------------------------

class VtkMesh:
    """Connectivity for the writer: coords (nnodes × dim), el2n (nels × nv, 1-based)."""

    def __init__(self, coords, el2n, dim: Optional[int] = None):
        self.coords = np.asarray(coords, dtype=np.float64)
        if self.coords.ndim == 1:
            self.coords = self.coords[:, None]
        self.el2n = np.atleast_2d(np.asarray(el2n, dtype=np.int64))
        self.dim = dim or self.coords.shape[1]
        self.nels = self.el2n.shape[0]


def vtk_corner_rows(dim: int, nlocal: int):
    """Local rows (0-based) of the corner nodes the writer keeps (postprocess.jl:360-378)."""
    if dim == 1:
        if nlocal == 2:
            return [0, 1]
        if nlocal == 3:
            return [0, 2]
        raise ValueError(f"cannot write VTK line cells with {nlocal} local nodes")
    if dim == 2:
        if nlocal in (3, 6, 7):
            return [0, 1, 2]
        if nlocal in (4, 8, 9):
            return [0, 1, 2, 3]
        raise ValueError(f"cannot write VTK 2D cells with {nlocal} local nodes")
    if nlocal in (4, 10, 11):
        return [0, 1, 2, 3]
    if nlocal in (8, 27):
        return list(range(8))
    raise ValueError(f"cannot write VTK 3D cells with {nlocal} local nodes")


def _vtk_cell_type(dim, ncorner):
    if dim == 1:
        return 3
    if dim == 2:
        return 5 if ncorner == 3 else 9
    return 10 if ncorner == 4 else 12


def _vtk_arrays(mesh):
    """(coords, el2n, dim) of the topology the reference writes (postprocess.jl:318-330):
    the velocity connectivity, except for a 2-D mixed mesh with a continuous P1
    pressure, whose pressure triangles are written. The structured meshes here carry a
    discontinuous P1 pressure, whose DoF nodes are interpolation points, not a geometric
    cell, so they write the velocity cells (as the reference does in 3-D)."""
    if isinstance(mesh, VtkMesh):
        return mesh.coords, mesh.el2n, mesh.dim
    coords = np.asarray(mesh.coords, dtype=np.float64)
    el2n = np.asarray(mesh.el2n, dtype=np.int64)
    el2nP = getattr(mesh, "el2nP", None)
    if mesh.dim == 2 and el2nP is not None and getattr(mesh, "pressure_continuous", False):
        el2n = np.asarray(el2nP, dtype=np.int64)
    return coords, el2n, mesh.dim


def _vtk_topology(mesh, coords_override=None):
    mesh_coords, el2n, dim = _vtk_arrays(mesh)
    coords = mesh_coords if coords_override is None else np.asarray(coords_override, dtype=np.float64)
    if coords.ndim == 1:
        coords = coords[:, None]
    if len(coords) != len(mesh_coords):
        raise ValueError(f"coords has length {len(coords)}; expected {len(mesh_coords)}")
    rows = vtk_corner_rows(dim, el2n.shape[1])
    corner = el2n[:, rows]
    nodes = np.unique(corner.ravel())                 # sorted, 1-based
    if nodes.size and (nodes[0] < 1 or nodes[-1] > len(coords)):
        raise IndexError("connectivity refers to a node outside the coordinates")
    node_map = np.zeros(len(coords) + 1, dtype=np.int64)
    node_map[nodes] = np.arange(1, nodes.size + 1)
    return dict(coords=coords, el2n=corner, nodes=nodes, node_map=node_map, nels=el2n.shape[0],
                cell_type=_vtk_cell_type(dim, len(rows)))


def _fmt(x):
    """Float text as the reference prints it (shortest round-trip repr)."""
    return repr(float(x))


def _values(field, topo, name, where):
    vals = field.detach().cpu().numpy() if hasattr(field, "detach") else np.asarray(field)
    vals = np.asarray(vals, dtype=np.float64).ravel()
    if where == "point":
        if len(vals) == len(topo["nodes"]):
            return vals
        if len(vals) == len(topo["coords"]):
            return vals[topo["nodes"] - 1]
        raise ValueError(f"point_data[{name}] has length {len(vals)}; expected {len(topo['nodes'])} or "
                         f"{len(topo['coords'])}")
    if len(vals) == topo["nels"]:
        return vals
    raise ValueError(f"cell_data[{name}] has length {len(vals)}; expected {topo['nels']}")


# row-major 3 × 3 positions of (xx, yy, zz, xy, xz, yz) (postprocess.jl:459-461)
_SYM_LAYOUT = (0, 3, 4, 3, 1, 5, 4, 5, 2)


def _write_field(lines, name, field, topo, where):
    if isinstance(field, tuple):
        comps = [_values(c, topo, name, where) for c in field]
        n = len(comps)
        if n in (2, 3):
            lines.append(f"VECTORS {name} float")
            for i in range(len(comps[0])):
                third = comps[2][i] if n == 3 else 0.0
                lines.append(f"{_fmt(comps[0][i])} {_fmt(comps[1][i])} {_fmt(third)}")
            return
        if n in (6, 9):
            layout = _SYM_LAYOUT if n == 6 else tuple(range(9))
            lines.append(f"TENSORS {name} float")
            for i in range(len(comps[0])):
                for r in range(3):
                    lines.append(" ".join(_fmt(comps[layout[3 * r + c]][i]) for c in range(3)))
            return
        raise ValueError(f"field {name} has {n} components; a tuple field must hold 2 or 3 (vector), "
                         "6 (symmetric tensor), or 9 (full tensor) of them")
    vals = _values(field, topo, name, where)
    lines.append(f"SCALARS {name} float 1")
    lines.append("LOOKUP_TABLE default")
    lines.extend(_fmt(x) for x in vals)


def write_vtk(path, mesh, point_data: Optional[Mapping] = None, cell_data: Optional[Mapping] = None,
              title: str = "FEMTools", coords=None):
    """write_vtk(path, mesh; point_data, cell_data, title, coords) (postprocess.jl:273-316):
    a legacy ASCII VTK unstructured grid. High-order cells are written by their corner
    nodes; a point field holds one value per mesh node or per written point, a cell field
    one per element; a tuple (a list is one scalar field) of 2–3 components is a vector, of 6 a symmetric tensor
    (xx, yy, zz, xy, xz, yz), of 9 a full row-major tensor. `coords` replaces the written
    coordinates (same node count)."""
    topo = _vtk_topology(mesh, coords)
    lines = ["# vtk DataFile Version 3.0", title, "ASCII", "DATASET UNSTRUCTURED_GRID",
             f"POINTS {len(topo['nodes'])} float"]
    for i in topo["nodes"]:
        c = topo["coords"][i - 1]
        pad = [_fmt(x) for x in c[:3]] + ["0.0"] * (3 - min(3, len(c)))
        lines.append(" ".join(pad))
    nc = topo["el2n"].shape[1]
    lines.append(f"CELLS {topo['nels']} {(nc + 1) * topo['nels']}")
    nm = topo["node_map"]
    for e in range(topo["nels"]):
        lines.append(" ".join([str(nc)] + [str(nm[n] - 1) for n in topo["el2n"][e]]))
    lines.append(f"CELL_TYPES {topo['nels']}")
    lines.extend([str(topo["cell_type"])] * topo["nels"])
    # validate every field before writing
    body = []
    if point_data:
        body.append(f"POINT_DATA {len(topo['nodes'])}")
        for name, field in point_data.items():
            _write_field(body, name, field, topo, "point")
    if cell_data:
        body.append(f"CELL_DATA {topo['nels']}")
        for name, field in cell_data.items():
            _write_field(body, name, field, topo, "cell")
    with open(path, "w") as f:
        f.write("\n".join(lines + body) + "\n")


def write_stokes_vtk(path, mesh, coords, el2nP, dofsP, P, v, post, title=None, cell_data=None, Q=None):
    """write_stokes_vtk (postprocess.jl:488-602). 2-D (`v` = (vx, vy)): P averaged from the
    pressure DoFs onto the written points, Vx, Vy and the vector V, and the diagnostics
    as scalar cell fields (strain_xx … tau_II; `Q` averaged per cell when given). 3-D
    (`v` = (vx, vy, vz)): the velocity vector, the point elevation z, the cell-centre
    pressure (the first P1-disc DoF of a Hex27 cell; the mean of four on tetrahedra) and
    the strain-rate and stress tensors with their invariants."""
    v = [x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x, dtype=np.float64) for x in v]
    P = P.detach().cpu().numpy() if hasattr(P, "detach") else np.asarray(P, dtype=np.float64)
    post_np = {k: (x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)) for k, x in post._asdict().items()} \
        if hasattr(post, "_asdict") else {k: np.asarray(x) for k, x in dict(post).items()}
    el2nP = np.asarray(el2nP, dtype=np.int64)
    dofsP = np.asarray(dofsP, dtype=np.int64)
    topo = _vtk_topology(mesh, coords)
    nodes = topo["nodes"]
    extra = dict(cell_data or {})
    if len(v) == 2:
        nm = topo["node_map"]
        vtk_P = np.zeros(len(nodes))
        cnt = np.zeros(len(nodes))
        for e in range(el2nP.shape[0]):
            for a in range(el2nP.shape[1]):
                i = nm[el2nP[e, a]] - 1
                if i < 0:
                    continue
                vtk_P[i] += P[dofsP[e, a] - 1]
                cnt[i] += 1
        vtk_P = np.divide(vtk_P, cnt, out=np.zeros_like(vtk_P), where=cnt > 0)
        vx, vy = v[0][nodes - 1], v[1][nodes - 1]
        cells = dict(extra)
        cells.update(strain_xx=post_np["εxx"], strain_yy=post_np["εyy"], strain_zz=post_np["εzz"],
                     strain_xy=post_np["εxy"], strain_II=post_np["εII"], tau_xx=post_np["τxx"],
                     tau_yy=post_np["τyy"], tau_zz=post_np["τzz"], tau_xy=post_np["τxy"],
                     tau_II=post_np["tauII"])
        if Q is not None:
            Qa = np.asarray(Q, dtype=np.float64)
            cells["Q"] = Qa[dofsP - 1].mean(axis=1)
        return write_vtk(path, mesh, point_data={"P": vtk_P, "Vx": vx, "Vy": vy, "V": (vx, vy)},
                         cell_data=cells, coords=coords, title=title or "FEMTools Stokes 2D")
    vel = tuple(x[nodes - 1] for x in v)
    nv = np.asarray(mesh.el2n).shape[1]
    cell_P = P[dofsP[:, :4] - 1].mean(axis=1) if nv in (10, 11) else P[dofsP[:, 0] - 1]
    cells = dict(extra)
    cells.update(P=cell_P,
                 strain=tuple(post_np[k] for k in ("εxx", "εyy", "εzz", "εxy", "εxz", "εyz")),
                 strain_II=post_np["εII"],
                 tau=tuple(post_np[k] for k in ("τxx", "τyy", "τzz", "τxy", "τxz", "τyz")),
                 tau_II=post_np["tauII"])
    zc = topo["coords"][nodes - 1][:, 2]
    return write_vtk(path, mesh, point_data={"velocity": vel, "z": zc}, cell_data=cells, coords=coords,
                     title=title or "FEMTools Stokes 3D")
