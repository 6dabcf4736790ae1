"""Sparse Q2/P1-disc saddle-point system of the StokesDR residual, assembled directly
from the element integrals: the pin the reference applies to its own matrix-free
Stokes residuals (test/test_stokes_3d_reference.jl:34-97, 155: A·x − rhs equals the
assembled residual to rtol 1e-11), restated for the StokesDR element.

Without plasticity the StokesDR residual is affine in (v, P), so it is A·x − b for
one sparse matrix. Per Hex27 element and Gauss point q, with ∂N_a/∂x = ∂N/∂ξ·J⁻¹,
dΩ from geo_v and dΩ_P from geo_P (momentum_residuals.jl:209-258,
pressure_residual.jl:132-158, rheology.jl:413-439, eos_density :11-16):

  momentum row (a, i):
    K   (b, j): ηve dΩ (δ_ij ∇N_a·∇N_b + ∂_j N_a ∂_i N_b − ⅔ ∂_i N_a ∂_j N_b)
    B   (p)   : −∂_i N_a N^P_p dΩ                       (pressure and Pnum)
    E   (p)   : −N_a ρ0 β g_i N^P_p dΩ                  (EOS: ρ = ρ0(1 − α(T−Tref) + βP))
    c_v       : Σ_k ∂_k N_a 2ηve τold_ki/(2GΔt) dΩ − N_a ρ0(1 − α(T−Tref)) g_i dΩ
  continuity row p:
    G   (b, j): −N^P_p ∂_j N_b dΩ_P
    S   (r)   : N^P_p N^P_r dΩ_P / (ηb Δt)              (zero when every ηb is ∞)
    c_P       : N^P_p dΩ_P (P0_q/(ηb Δt) + α_P (T − T0)_q / Δt)

with the phase tables interpolated at q as the residual does (utils.jl:37-44: the
velocity shape functions for η, 1/G, ρ0, α, β; the pressure basis for ηb and α_P),
ηve = 1/(1/η + (1/G)/Δt). Then RP = G v − S P + c_P, Pnum = D RP with
D = diag(γP/M_P) (DR.jl:674), and Rv = K v + (B + E) P + B Pnum + c_v. The augmented
operator of the fused sweep is therefore

  A = [[K + B D G, B + E − B D S], [G, −S]],   b = −[c_v + B D c_P, c_P].

Velocity DoFs are numbered c·nnodes + node (the SoA component arrays), pressure
DoFs after them.
"""
import numpy as np
import scipy.sparse as sp

from conftest import fem

abi = fem._abi


def _phases(layout, table, e, ids, n):
    if table is None:
        return np.zeros(n, dtype=np.int64)
    if layout == abi.PHASE_CELL:
        return np.full(n, table[e] - 1, dtype=np.int64)
    if layout == abi.PHASE_ELEMENT_NODE:
        return np.asarray(table[e], dtype=np.int64) - 1
    return np.asarray(table[ids - 1], dtype=np.int64) - 1


def assemble(case, dt, gammaP, M_P, P0, T, T0, tau_old):
    """The blocks of the StokesDR residual of `case` (no plasticity) at time step `dt`."""
    assert case.plastic is None
    mesh, mat = case.mesh, case.material
    t = fem.element_tables(3)
    nn, nP, ne = mesh.nnodes, mesh.nnodesP, mesh.nels
    nv = 3 * nn
    eta, invG = np.asarray(mat.eta), 1.0 / np.asarray(mat.G)
    rho0, alpha, beta = np.asarray(mat.rho0), np.asarray(mat.alpha), 1.0 / np.asarray(mat.K)
    bulk = np.asarray(mat.eta_b)
    all_inf = bool(np.all(np.isinf(bulk)))
    g = np.asarray(mat.g)
    I3 = np.eye(3)
    kr, kc, kv = [], [], []          # velocity × velocity
    br, bc, bv = [], [], []          # velocity × pressure, B
    er, ec, ev = [], [], []          # velocity × pressure, E
    gr, gc, gv = [], [], []          # pressure × velocity
    sr, sc, svals = [], [], []       # pressure × pressure
    c_v = np.zeros(nv)
    c_P = np.zeros(nP)
    for e in range(ne):
        nodes = mesh.el2n[e]
        dofs = mesh.dofsP[e]
        phv = _phases(case.phases_v_layout, case.phases_v, e, nodes, 27)
        php = _phases(case.phases_P_layout, case.phases_P, e, dofs, 4)
        vd = (np.arange(3)[:, None] * nn + (nodes - 1)[None, :])       # [i, a]
        pd = dofs - 1
        Ke = np.zeros((3, 27, 3, 27))
        Be = np.zeros((3, 27, 4))
        Ee = np.zeros((3, 27, 4))
        Ge = np.zeros((4, 3, 27))
        Se = np.zeros((4, 4))
        cve = np.zeros((3, 27))
        cPe = np.zeros(4)
        for q in range(27):
            geo = mesh.geo_v[e, q]
            Jinv = geo[:9].reshape(3, 3, order="F")
            dO, dOP = geo[9], mesh.geo_P[e, q]
            Nq, NPq = t.N[q], t.NP[q]
            Gq = t.dN[q] @ Jinv                                         # ∂N_a/∂x_k
            etaq = Nq @ eta[phv]
            invGq = Nq @ invG[phv]
            etave = 1.0 / (1.0 / etaq + invGq / dt)
            inv2Gdt = invGq / (2 * dt)
            Tq = NPq @ T[pd]
            rhoq0 = (Nq @ rho0[phv]) * (1 - (Nq @ alpha[phv]) * (Tq - mat.Tref))
            betaq = (Nq @ rho0[phv]) * (Nq @ beta[phv])                 # ρ0·β of the EOS
            Ke += etave * dO * (np.einsum("ab,ij->iajb", Gq @ Gq.T, I3) + np.einsum("aj,bi->iajb", Gq, Gq)
                                - (2.0 / 3.0) * np.einsum("ai,bj->iajb", Gq, Gq))
            Be += -dO * np.einsum("ai,p->iap", Gq, NPq)
            Ee += -dO * betaq * np.einsum("a,i,p->iap", Nq, g, NPq)
            Ge += -dOP * np.einsum("p,bj->pjb", NPq, Gq)
            told = np.array([[tau_old[0][27 * e + q], tau_old[3][27 * e + q], tau_old[4][27 * e + q]],
                             [tau_old[3][27 * e + q], tau_old[1][27 * e + q], tau_old[5][27 * e + q]],
                             [tau_old[4][27 * e + q], tau_old[5][27 * e + q], tau_old[2][27 * e + q]]])
            cve += dO * 2 * etave * inv2Gdt * np.einsum("ak,ki->ia", Gq, told)
            cve -= dO * rhoq0 * np.einsum("a,i->ia", Nq, g)
            aP = NPq @ alpha[php]
            src = aP * (NPq @ (T[pd] - T0[pd])) / dt
            if not all_inf:
                ebq = NPq @ bulk[php]
                Se += dOP * np.outer(NPq, NPq) / (ebq * dt)
                src += (NPq @ P0[pd]) / (ebq * dt)
            cPe += dOP * NPq * src
        r, c = np.meshgrid(vd.ravel(), vd.ravel(), indexing="ij")
        kr.append(r.ravel()); kc.append(c.ravel()); kv.append(Ke.reshape(81, 81).ravel())
        r, c = np.meshgrid(vd.ravel(), pd, indexing="ij")
        br.append(r.ravel()); bc.append(c.ravel()); bv.append(Be.reshape(81, 4).ravel())
        er.append(r.ravel()); ec.append(c.ravel()); ev.append(Ee.reshape(81, 4).ravel())
        r, c = np.meshgrid(pd, vd.ravel(), indexing="ij")
        gr.append(r.ravel()); gc.append(c.ravel()); gv.append(Ge.reshape(4, 81).ravel())
        r, c = np.meshgrid(pd, pd, indexing="ij")
        sr.append(r.ravel()); sc.append(c.ravel()); svals.append(Se.ravel())
        np.add.at(c_v, vd.ravel(), cve.ravel())
        np.add.at(c_P, pd, cPe)
    mk = lambda r, c, v, shape: sp.csr_matrix((np.concatenate(v), (np.concatenate(r), np.concatenate(c))), shape=shape)
    K = mk(kr, kc, kv, (nv, nv))
    B = mk(br, bc, bv, (nv, nP))
    E = mk(er, ec, ev, (nv, nP))
    G = mk(gr, gc, gv, (nP, nv))
    S = mk(sr, sc, svals, (nP, nP))
    M = np.asarray(M_P, dtype=float)
    D = sp.diags(np.divide(np.asarray(gammaP, dtype=float), M, out=np.zeros_like(M), where=M != 0))
    return {"K": K, "B": B, "E": E, "G": G, "S": S, "D": D, "c_v": c_v, "c_P": c_P}


def augmented_system(blk, with_pnum=True):
    """(A, b) with R(x) = A·x − b, x = [v (component-major); P]."""
    K, B, E, G, S, D = blk["K"], blk["B"], blk["E"], blk["G"], blk["S"], blk["D"]
    if with_pnum:
        top = sp.hstack([K + B @ D @ G, B + E - B @ D @ S])
        b_v = -(blk["c_v"] + B @ (D @ blk["c_P"]))
    else:
        top = sp.hstack([K, B + E])
        b_v = -blk["c_v"]
    A = sp.vstack([top, sp.hstack([G, -S])]).tocsr()
    return A, np.concatenate([b_v, -blk["c_P"]])


def linear_vep_case(n=3, seed=0, distort=True, phases="nodal"):
    """A visco-elastic StokesDR case without plasticity (the residual is then affine):
    random v, P, P0, T, T0, τ_old, γP, M_P, finite G, ηb and K, thermal expansion, on
    a distorted (or affinely sheared) Hex27 mesh, phases in the given layout."""
    return fem.configs.random_state_case(dim=3, n=n, seed=seed, phases=phases, plastic=False, distort=distort)


def layered_solve_case(n=2, seed=0, distort=True):
    """The layered visco-elastic case of the benchmark without plasticity, with a
    random stress history and old pressure: a well-posed linear problem to solve to
    convergence; on a mesh whose interior nodes are perturbed (non-affine cells) when
    `distort`, else on the box itself (affine cells, as the mixed-precision solve needs)."""
    case = fem.configs.vep_layers_case(n=n, seed=seed, plastic=False)
    rng = np.random.default_rng(seed + 50)
    mesh = case.mesh
    if distort:
        h = 1.0 / (2 * n)
        coords = mesh.coords.copy()
        interior = np.all((coords > 1e-12) & (coords < 1 - 1e-12), axis=1)
        coords[interior] += rng.uniform(-0.15 * h, 0.15 * h, size=(interior.sum(), 3))
        mesh.coords = coords
        mesh.geo_v, mesh.geo_P = fem.mesh.precompute_geometry(coords, mesh.el2n, fem.element_tables(3))
    case.tau_old = [0.3 * rng.standard_normal(mesh.nq * mesh.nels) for _ in range(6)]
    case.P0 = 0.3 * rng.standard_normal(mesh.nnodesP)
    return case


def sparse_solution(case, blk):
    """The sparse direct solution with the case's Dirichlet velocities (no gauge: a
    finite bulk viscosity fixes the pressure)."""
    import scipy.sparse.linalg as spla
    A, b = augmented_system(blk, with_pnum=False)
    nn = case.mesh.nnodes
    nv = 3 * nn
    x = np.zeros(A.shape[0])
    fixed = np.zeros(A.shape[0], dtype=bool)
    for c, (dofs, vals) in enumerate(case.bc):
        x[c * nn + dofs - 1] = vals
        fixed[c * nn + dofs - 1] = True
    free = np.flatnonzero(~fixed)
    rhs = b[free] - A[free][:, fixed] @ x[fixed]
    x[free] = spla.spsolve(A[free][:, free].tocsc(), rhs)
    return x[:nv], x[nv:]
