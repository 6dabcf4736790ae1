"""Host-side mesh setup mirroring FEMTools.jl's structured generators.

Builds the arrays the device kernels consume, in the reference's layouts:
coordinates on the refined tensor grid (x fastest), 1-based int32 column-major
connectivity, P1-discontinuous pressure DoFs and the precomputed geometry
(inverse Jacobian + |det J|·ω per quadrature point). This is set-up work done
once per mesh, as in the reference (`Mesh(backend, Ω, element, nels)`,
src/mesh/mesh.jl:68-100; `MixedMesh(mesh_v, element_P)`, src/mesh/mixed_mesh.jl:173).
"""
from __future__ import annotations

from dataclasses import dataclass, field
import numpy as np

# Hex27 local node reference coordinates (src/elements/shape_functions.jl:414-442).
HEX27_NODES = np.array([
    (-1, -1, -1), (+1, -1, -1), (+1, +1, -1), (-1, +1, -1),
    (-1, -1, +1), (+1, -1, +1), (+1, +1, +1), (-1, +1, +1),
    (0, -1, -1), (+1, 0, -1), (0, +1, -1), (-1, 0, -1),
    (0, -1, +1), (+1, 0, +1), (0, +1, +1), (-1, 0, +1),
    (-1, -1, 0), (+1, -1, 0), (+1, +1, 0), (-1, +1, 0),
    (0, 0, -1), (0, -1, 0), (+1, 0, 0), (0, +1, 0), (-1, 0, 0), (0, 0, +1), (0, 0, 0),
], dtype=np.int64)
# Q9 local node reference coordinates (shape_functions.jl:268-278).
Q9_NODES = np.array([(-1, -1), (+1, -1), (+1, +1), (-1, +1), (0, -1), (+1, 0), (0, +1), (-1, 0), (0, 0)],
                    dtype=np.int64)
# Local velocity nodes carrying the P1-disc pressure DoFs (mixed_mesh.jl:408-417), 0-based.
PRESSURE_ROWS = {3: (26, 22, 23, 25), 2: (8, 5, 6)}


def _line_N(x, node):
    return np.where(node == -1, x * (x - 1) * 0.5, np.where(node == 0, 1 - x * x, x * (x + 1) * 0.5))


def _line_dN(x, node):
    return np.where(node == -1, x - 0.5, np.where(node == 0, -2 * x, x + 0.5))


@dataclass
class ElementTables:
    """Shape-function tables at the velocity quadrature points."""
    dim: int
    N: np.ndarray    # nq × nv
    dN: np.ndarray   # nq × nv × dim (reference gradients)
    NP: np.ndarray   # nq × np (pressure basis at the velocity points)
    w: np.ndarray    # nq

    @property
    def nv(self):
        return self.N.shape[1]

    @property
    def nq(self):
        return self.N.shape[0]

    @property
    def np_(self):
        return self.NP.shape[1]


def element_tables(dim: int) -> ElementTables:
    """Hex27 + 3×3×3 Gauss (integration_points.jl:321) or Q9 + 3×3 Gauss (:223),
    with the P1 pressure basis of LinearElement{dim, dim+1} at those points."""
    a = np.sqrt(3.0 / 5.0)
    pts = np.array([-a, 0.0, a])
    wts = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
    nodes = HEX27_NODES if dim == 3 else Q9_NODES
    nq = 3 ** dim
    q = np.arange(nq)
    qi = np.stack([(q // 3 ** d) % 3 for d in range(dim)], axis=1)  # ξ fastest
    X = pts[qi]                                                     # nq × dim
    if dim == 3:
        w = wts[qi[:, 0]] * wts[qi[:, 1]] * wts[qi[:, 2]]
    else:
        w = np.array([25, 40, 25, 40, 64, 40, 25, 40, 25], dtype=np.float64) / 81.0
    L = np.stack([_line_N(X[:, None, d], nodes[None, :, d]) for d in range(dim)], axis=-1)   # nq×nv×dim
    dL = np.stack([_line_dN(X[:, None, d], nodes[None, :, d]) for d in range(dim)], axis=-1)
    N = np.prod(L, axis=-1)
    dN = np.empty(L.shape)
    for j in range(dim):
        f = np.ones(L.shape[:2])
        for d in range(dim):
            f = f * (dL[..., d] if d == j else L[..., d])
        dN[..., j] = f
    NP = np.concatenate([1 - X.sum(axis=1, keepdims=True), X], axis=1)
    return ElementTables(dim, N, dN, NP, w)


@dataclass
class MixedMesh:
    """Structured Q2–P1-discontinuous mesh (Hex27 in 3-D, Q9 in 2-D)."""
    dim: int
    nel: tuple
    coords: np.ndarray      # nnodes × dim
    el2n: np.ndarray        # nels × nv (C order) == nv × nels column-major, 1-based
    dofsP: np.ndarray       # nels × np
    el2nP: np.ndarray       # nels × np
    geo_v: np.ndarray       # nels × nq × (dim² + 1)
    geo_P: np.ndarray       # nels × nq
    boundary_nodes: np.ndarray = field(default=None)  # 1-based Γnodes

    @property
    def nels(self):
        return self.el2n.shape[0]

    @property
    def nnodes(self):
        return self.coords.shape[0]

    @property
    def nnodesP(self):
        return self.dofsP.size

    @property
    def nv(self):
        return self.el2n.shape[1]

    @property
    def np_(self):
        return self.dofsP.shape[1]

    @property
    def nq(self):
        return self.geo_P.shape[1]


def _grid_axis(lo, hi, n):
    """LinRange(lo, hi, n) of Julia: ((n-1-i)·lo + i·hi)/(n-1); exact i/(n-1)·hi for lo = 0."""
    i = np.arange(n, dtype=np.float64)
    d = float(n - 1)
    if lo == 0.0:
        return i / d * hi
    return ((d - i) / d) * lo + (i / d) * hi


def structured_connectivity(dim: int, nel) -> np.ndarray:
    """generate_element2node for Hex27 (src/mesh/connectivity.jl:273) or Q9 (:201); 1-based."""
    nodes = HEX27_NODES if dim == 3 else Q9_NODES
    if dim == 3:
        nx, ny, nz = nel
        sy, sz = 2 * nx + 1, (2 * nx + 1) * (2 * ny + 1)
        ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
        ix = 2 * ex[:, None] + 1 + nodes[None, :, 0]
        iy = 2 * ey[:, None] + 1 + nodes[None, :, 1]
        iz = 2 * ez[:, None] + 1 + nodes[None, :, 2]
        return (iz * sz + iy * sy + ix + 1).astype(np.int32)
    nx, ny = nel
    sy = 2 * nx + 1
    ey, ex = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ex, ey = ex.ravel(), ey.ravel()
    ix = 2 * ex[:, None] + 1 + nodes[None, :, 0]
    iy = 2 * ey[:, None] + 1 + nodes[None, :, 1]
    return (iy * sy + ix + 1).astype(np.int32)


def precompute_geometry(coords: np.ndarray, el2n: np.ndarray, tables: ElementTables, chunk: int = 65536):
    """precompute_geometry_kernel! (src/mesh/mesh.jl:674-682): J = Σ_a x_a ∂N_a/∂ξ,
    stores J⁻¹ (column-major) and |det J|·ω per quadrature point."""
    dim, nq = tables.dim, tables.nq
    nels = el2n.shape[0]
    geo_v = np.empty((nels, nq, dim * dim + 1))
    geo_P = np.empty((nels, nq))
    for s in range(0, nels, chunk):
        e = slice(s, min(s + chunk, nels))
        X = coords[el2n[e] - 1]                                  # ne × nv × dim
        J = np.einsum("ean,qaj->eqnj", X, tables.dN)             # J[n=i, j]: ∂x_i/∂ξ_j
        det = np.linalg.det(J)
        inv = np.linalg.inv(J)                                   # inv[r, c]
        geo_v[e, :, : dim * dim] = np.swapaxes(inv, -1, -2).reshape(inv.shape[0], nq, dim * dim)
        geo_v[e, :, dim * dim] = np.abs(det) * tables.w[None, :]
        geo_P[e] = np.abs(det) * tables.w[None, :]
    return geo_v, geo_P


def structured_mixed_mesh(dim: int, nel, lo=None, hi=None) -> MixedMesh:
    """Mesh(CPU(), box, element, nel) + MixedMesh(mesh_v, element_P) for Hex27/P1 or Q9/P1."""
    nel = tuple(int(n) for n in nel)
    lo = [0.0] * dim if lo is None else [float(x) for x in lo]
    hi = [1.0] * dim if hi is None else [float(x) for x in hi]
    axes = [_grid_axis(lo[d], hi[d], 2 * nel[d] + 1) for d in range(dim)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")
    coords = np.stack([g.ravel() for g in grids[::-1]], axis=1)   # x fastest
    el2n = structured_connectivity(dim, nel)
    tables = element_tables(dim)
    nels = el2n.shape[0]
    npd = tables.np_
    dofsP = (np.arange(nels * npd, dtype=np.int64).reshape(nels, npd) + 1).astype(np.int32)
    el2nP = el2n[:, list(PRESSURE_ROWS[dim])].copy()
    geo_v, geo_P = precompute_geometry(coords, el2n, tables)
    on_b = np.zeros(coords.shape[0], dtype=bool)
    for d in range(dim):
        on_b |= (coords[:, d] == lo[d]) | (coords[:, d] == hi[d])
    bnodes = (np.nonzero(on_b)[0] + 1).astype(np.int32)
    return MixedMesh(dim, nel, coords, el2n, dofsP, el2nP, geo_v, geo_P, bnodes)


def cell_centroids(mesh: MixedMesh) -> np.ndarray:
    """Element centroid from the corner nodes (the first 2^dim local nodes)."""
    ncorner = 8 if mesh.dim == 3 else 4
    return mesh.coords[mesh.el2n[:, :ncorner] - 1].mean(axis=1)


def wall_nodes(mesh: MixedMesh, axis: int, lo=0.0, hi=1.0, atol=None) -> np.ndarray:
    """1-based nodes on the two walls normal to `axis` (the free-slip sets of the examples)."""
    tol = 32 * np.finfo(np.float64).eps * max(abs(hi), 1.0) if atol is None else atol
    x = mesh.coords[:, axis]
    return (np.nonzero((np.abs(x - lo) <= tol) | (np.abs(x - hi) <= tol))[0] + 1).astype(np.int32)
