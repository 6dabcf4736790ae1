"""Benchmark: time to a 1e-8 DR solve of 3-D Hex27/Q2–P1-disc visco-elasto-plastic Stokes at 64³.

One step = one `solve` (solve! of the reference, src/stokes/solvers/DR.jl:302) of the
layered visco-elasto-plastic configuration from the same initial state to
min(err_abs, err_rel) < 1e-8, with M_P/γP assembly, the Jacobian diagnostics every
check and the Powell–Hestenes/DYREL loop, all inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 64] [--impl ours|reference]

Prints one JSON line (rank 0). Multi-GPU runs are independent replicas (the path has
no exchange step on one mesh): value = slowest rank's time per solve, scaling "weak".
`--impl reference` times the CPU restatement of the reference's algorithm (the
oracle, all host cores) on the same workload by a bounded sample.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "time-to-1e-8 residual, 3D Q2 Stokes 64³: chosen vs plain FP64 DR; HBM GB/s"

# DR path of the 64³ solve of this workload, measured by this file's plain FP64 arm on
# a B200: the CPU reference time is extrapolated along it (the oracle and the device
# take the same path: equal iteration counts at 32³, `--mode parity`).
PATH_64 = {"iterations": 12300, "itPH": 89, "jacobian_assemblies": 124, "check_interval": 100}
# DRAM bytes read + written by one launch of the chosen method's hot kernel at 64³,
# from the ncu capture summarised in profiles/hex27_incr_kernel_vep64.md.
TRAFFIC = {(64, "mixed"): 133528576}


def load_package():
    import importlib.util
    if "femtools_b200" in sys.modules:
        return sys.modules["femtools_b200"]
    pkg_dir = os.path.join(ROOT, "femtools.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "femtools_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["femtools_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def mesh_is_affine(mesh, tol=1e-12):
    """Every element carries one J⁻¹ and |det J| at all quadrature points (the test the
    library applies before it takes the compressed-geometry sweep)."""
    g = mesh.geo_v
    w = __import__("femtools_b200").mesh.element_tables(mesh.dim).w
    c = g[:, 13:14, :]
    sc = np.abs(c[:, :, :9]).max(axis=2, keepdims=True)
    ok = np.all(np.abs(g[:, :, :9] - c[:, :, :9]) <= tol * sc)
    d = g[:, :, 9] / w[None, :]
    ok = ok and np.all(np.abs(d - d[:, 13:14]) <= tol * np.abs(d[:, 13:14]))
    ok = ok and np.all(np.abs(mesh.geo_P - g[:, :, 9]) <= tol * np.abs(g[:, :, 9]))
    return bool(ok)


def incremental_kernel_bytes(case, stress_reads=None):
    """Algorithmic bytes of one FP32 incremental sweep of the mixed-precision solve
    (hex27_incr_kernel): δv, the tiled connectivity, FP32 affine geometry, the two
    element phases, δP, the Pnum scale γP/M_P of the element's DoFs, the base yield
    value of every integration point (27 FP32), the base trial stress (6 FP32) of the
    points the elastic bound does not settle (`stress_reads` per launch, measured by
    the library's counter; every point when None), the RP increment written and the
    Rv read-modify-write (FP32). The pressure DoFs are numbered 4e + p on the
    structured mesh, so no DoF table is read."""
    m = case.mesh
    nels, nn, nP = m.nels, m.nnodes, m.nnodesP
    b = 3 * nn * 4                         # δv
    b += 27 * 4 * nels                     # el2n (tiled)
    b += 10 * 4 * nels                     # J⁻¹ and |det J| per element
    b += 2 * 4 * nels                      # phases of the velocity nodes and of the pressure DoFs
    b += nP * 4                            # δP
    b += 4 * 4 * nels                      # γP/M_P
    b += 27 * 4 * nels                     # base yield value
    b += 6 * 4 * (27 * nels if stress_reads is None else stress_reads)   # base trial stress where read
    b += nP * 4                            # RP increment written
    b += 2 * 3 * nn * 4                    # Rv atomic read-modify-write
    return b


def residual_kernel_bytes(case, itemsize=8, geo_itemsize=8, affine=None):
    """Algorithmic bytes of one fused residual-sweep launch: every array the sweep
    must touch, once, at its stored precision (Rv read-modify-write counted twice).
    On affine meshes the sweep reads one J⁻¹ and |det J| per element (80 B) instead
    of the reference layout's per-point J⁻¹, dΩ and dΩ_P (2376 B), and the figure
    counts what it reads."""
    m = case.mesh
    nels, nn, nP = m.nels, m.nnodes, m.nnodesP
    if affine is None:
        affine = m.dim == 3 and mesh_is_affine(m)
    b = 0
    b += 3 * nn * itemsize                 # v
    b += 27 * 4 * nels + 4 * 4 * nels      # el2n, dofsP
    if affine:
        b += 10 * itemsize * nels          # per-element J⁻¹ and |det J|
    else:
        b += 27 * 10 * geo_itemsize * nels     # geo_v (J⁻¹ + dΩ per point)
        b += 27 * geo_itemsize * nels          # geo_P
    b += 4 * nP * itemsize                 # P, P_old, γP, M_P
    b += 4 * nels                          # cell phase
    b += 6 * 27 * itemsize * nels          # τ_old at integration points
    b += 2 * nP * itemsize                 # RP, Pnum written
    b += 2 * 3 * nn * itemsize             # Rv atomic read-modify-write
    return b


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.proc = None
        self.index = index
        # the raw samples go to FEMB_CLOCKS_DIR when set (a folder the caller keeps), else
        # to the system temporary directory; the JSON line carries their summary
        import tempfile
        out_dir = os.environ.get("FEMB_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_rank{index}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x, world, device="cuda"):
    """The largest of a per-rank value over all ranks (every multi-GPU time is the max over
    ranks); the value itself on one rank. Every rank must call it, in the same order."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def cpu_model():
    """The host CPU's model name (first /proc/cpuinfo entry) and logical core count."""
    name = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                name = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return name, os.cpu_count()


class CpuSample:
    """Timed sample of the CPU restatement of the reference (the oracle, OpenMP on all
    host cores) on one workload, for extrapolating its time to solution.

    Setup (untimed): the host state, M_P/γP and one full Jacobian assembly (the
    preconditioner of the iterations and their Chebyshev steps). One `step()` then
    times, on the full mesh, `block` whole inner DR iterations of the solve's own loop
    (pressure residual, Pnum, momentum residual, Dirichlet pins, velocity update), one
    more iteration with a check's work (Rv → Rv0, velocity error, λmin; no Jacobian)
    and the Jacobian assembly of one of `parts` equal blocks of the elements into the
    full-size arrays; successive steps take the blocks in turn. `estimate()` prices a
    solve's path with the step's figures:
    iterations·t_iter + checks·t_check + assemblies·parts·t_part + itPH·t_iter."""

    def __init__(self, case, block=8, parts=8, threads=None):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_host as oh
        L = oh.lib()
        if threads:
            L.orc_set_num_threads(threads)
        self.cores = L.orc_num_threads()
        self.case, self.block, self.parts = case, block, parts
        self.hs = case.host_state(oh)
        self.hs.pressure_scaling(50.0, case.dt)
        self.hs.jacobian_diagnostics(case.dt)
        lmax = [float(np.max(self.hs.dRdv[c] / self.hs.PC[c])) for c in range(case.mesh.dim)]
        dtau = [2.0 / math.sqrt(x) * 0.98 for x in lmax]
        self.alpha = [d * d for d in dtau]      # Chebyshev step with λmin = 0 (c = 0)
        self.beta = [1.0] * case.mesh.dim
        self.v0 = [x.copy() for x in self.hs.v]
        self.k = 0

    def step(self):
        hs, dt, m = self.hs, self.case.dt, self.case.mesh
        for c in range(m.dim):          # every step samples the same state
            hs.v[c][:] = self.v0[c]
            hs.rate[c][:] = 0.0
        t0 = time.perf_counter()
        hs.dr_iterations(dt, self.alpha, self.beta, self.block)
        t1 = time.perf_counter()
        hs.dr_iterations(dt, self.alpha, self.beta, 1, check_norms=True)
        t2 = time.perf_counter()
        e0 = m.nels * (self.k % self.parts) // self.parts
        e1 = m.nels * (self.k % self.parts + 1) // self.parts
        hs.jacobian_range(dt, e0, e1)
        t3 = time.perf_counter()
        self.k += 1
        t_iter = (t1 - t0) / self.block
        return {"t_iter": t_iter, "t_check": max(t2 - t1 - t_iter, 0.0), "t_jacobian": (t3 - t2) * self.parts,
                "sampled_s": t3 - t0}

    @staticmethod
    def estimate(fig, path):
        checks = path["iterations"] // path["check_interval"]
        return (path["iterations"] * fig["t_iter"] + checks * fig["t_check"]
                + path["jacobian_assemblies"] * fig["t_jacobian"] + path["itPH"] * fig["t_iter"])

    def describe(self, fig):
        return (f"oracle (C++ FP64 restatement of the reference CPU path, {self.cores} threads) on the full "
                f"{self.case.mesh.nel} mesh: {self.block} whole DR iterations ({fig['t_iter']:.3f} s each), one "
                f"check ({fig['t_check']:.3f} s) and 1/{self.parts} of a Jacobian assembly "
                f"({fig['t_jacobian']:.2f} s per full assembly) per step")


def cpu_baseline_estimate(case, path, steps=1, threads=None):
    """Time to solution of the oracle along `path`, from `steps` CpuSample steps."""
    smp = CpuSample(case, threads=threads)
    figs = [smp.step() for _ in range(steps)]
    fig = {k: statistics.mean(f[k] for f in figs) for k in figs[0]}
    return CpuSample.estimate(fig, path), smp.cores, smp.describe(fig) + f", extrapolated along {path}"


def sweep_mode(args, fem, case, dr, lib, h):
    """Kernel-level timing: K fused residual sweeps and K Jacobian assemblies."""
    import torch
    fem.assemble_viscosity_weighted_pressure_scaling(dr, 50.0, case.dt)
    for _ in range(args.warmup):
        fem.assemble_stokes_residuals(dr, case.dt)
    fem.assemble_augmented_momentum_jacobian(dr, case.dt)
    torch.cuda.synchronize()
    lib.femb200_profile(h, 1)
    for _ in range(args.steps):
        fem.assemble_stokes_residuals(dr, case.dt)
    for _ in range(max(1, args.steps // 10)):
        fem.assemble_augmented_momentum_jacobian(dr, case.dt)
    prof_ms = (C.c_double * fem._abi.PROF_COUNT)()
    prof_n = (C.c_int64 * fem._abi.PROF_COUNT)()
    lib.femb200_profile_read(h, prof_ms, prof_n)
    lib.femb200_profile(h, 0)
    nbytes = residual_kernel_bytes(case)
    res_ms = prof_ms[0] / max(prof_n[0], 1)
    peak, kind = measured_peaks()
    print(json.dumps({"mode": "sweep", "n": args.n, "residual_ms": res_ms, "residual_launches": prof_n[0],
                      "achieved_GBs": nbytes / (res_ms / 1e3) / 1e9, "frac": nbytes / (res_ms / 1e3) / 1e9 / peak,
                      "bytes_per_launch": nbytes, "jacobian_ms": prof_ms[1] / max(prof_n[1], 1),
                      "jacobian_launches": prof_n[1]}), flush=True)
    return 0


def scatter_order_mode(args, fem, case, dr, lib, h):
    """The FP32 sweep's ordered scatter (one launch per tile colour) against its atomic
    scatter on the mixed-precision solve: per-sweep time, whole-solve time, iterations, and
    whether two solves of each kind repeat each other's path and fields."""
    import torch
    stream = torch.cuda.current_stream()
    init = {"v": [x.clone() for x in dr.v], "P": dr.P.clone(), "P0": dr.P0.clone(),
            "tau_old": [x.clone() for x in dr.tau_old]}

    def reset():
        for c in range(3):
            dr.v[c].copy_(init["v"][c])
        dr.P.copy_(init["P"])
        dr.P0.copy_(init["P0"])
        for c in range(6):
            dr.tau_old[c].copy_(init["tau_old"][c])

    kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=args.check_interval, throw_on_failure=False,
              max_iterations=args.max_iterations, iter_max=args.max_iterations, precision="mixed")
    bc = case.bc_device()
    out = {"mode": "scatter-order", "n": args.n, "tolerance": args.tolerance}
    fields = {}

    def rel(x, y):
        return _rel(x.double().cpu().numpy(), y.double().cpu().numpy())

    try:
        for ordered in (0, 1):
            assert lib.femb200_set_ordered_scatter(h, ordered) == fem._abi.OK
            name = "ordered" if ordered else "atomic"
            reset()
            fem.solve(dr, bc, **kw)   # warm-up
            runs = []
            for rep in range(2):
                reset()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ev0.record(stream)
                st = fem.solve(dr, bc, **kw)
                ev1.record(stream)
                torch.cuda.synchronize()
                fem.update_stokes_current_stress(dr, case.dt)
                f = {"v": torch.cat([x.clone() for x in dr.v]), "P": dr.P.clone(),
                     "tau": torch.cat([x.clone() for x in dr.tau])}
                fields[(name, rep)] = f
                runs.append({"s": ev0.elapsed_time(ev1) / 1e3, "iterations": st["iter"], "itPH": st["itPH"],
                             "err": st["err"]})
            # per-sweep time from one more solve with events around every sweep
            lib.femb200_profile(h, 1)
            reset()
            fem.solve(dr, bc, **kw)
            prof_ms = (C.c_double * fem._abi.PROF_COUNT)()
            prof_n = (C.c_int64 * fem._abi.PROF_COUNT)()
            lib.femb200_profile_read(h, prof_ms, prof_n)
            lib.femb200_profile(h, 0)
            same = all(torch.equal(fields[(name, 0)][k], fields[(name, 1)][k]) for k in ("v", "P", "tau"))
            out[name] = {"runs": runs, "sweep_ms": prof_ms[0] / max(prof_n[0], 1), "sweeps": int(prof_n[0]),
                         "residual_ms_total": prof_ms[0], "jacobian_ms": prof_ms[1], "node_update_ms": prof_ms[2],
                         "outer_fp64_ms": prof_ms[4], "two_runs_bitwise_equal": bool(same),
                         "two_runs_rel_diff": {k: rel(fields[(name, 0)][k], fields[(name, 1)][k])
                                                   for k in ("v", "P", "tau")}}
    finally:
        lib.femb200_set_ordered_scatter(h, 0)
    out["ordered_vs_atomic_rel_diff"] = {k: rel(fields[("ordered", 0)][k], fields[("atomic", 0)][k])
                                         for k in ("v", "P", "tau")}
    out["sweep_cost"] = out["ordered"]["sweep_ms"] / out["atomic"]["sweep_ms"] - 1.0
    print(json.dumps(out), flush=True)
    return 0


def adjoint_mode(args, fem):
    """Adjoint workload (coupled thermal–Stokes forward with shear heating on a Hex27 n³
    mesh, T-dependent viscosity η = exp(−0.1·T)·exp(δ_e)): the coupled forward solve,
    then with the temperature frozen at its converged value the device adjoint solve
    and the per-element log-viscosity gradient, checked against central differences
    of Stokes solves on `--fd-elements` random elements. Prints one JSON line."""
    import torch
    n = args.n
    ac = fem.configs.adjoint_case(n=n, seed=args.seed)
    case = ac.case
    mesh = case.mesh
    dt = args.adjoint_dt
    rng = np.random.default_rng(args.seed + 100)
    # thermal state on the Hex27 nodes: T linear from 1 at the bottom to 0 at the top, plus noise
    z = mesh.coords[:, 2]
    T0n = 1.0 - z + rng.normal(0.0, 0.01, size=mesh.nnodes)
    bot = (np.nonzero(np.abs(z) < 1e-12)[0] + 1).astype(np.int32)
    topn = (np.nonzero(np.abs(z - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    T0n[bot - 1] = 1.0
    T0n[topn - 1] = 0.0
    bcT = fem.DirichletBoundaryCondition(np.concatenate([bot, topn]),
                                         np.concatenate([np.ones(len(bot)), np.zeros(len(topn))]))
    th = fem.ThermalDiffusionDR(mesh, k=(1.0,), Cp=(1.0,), rho0=(1.0,), alpha=(case.material.alpha[0],), eps=1e-8)
    th.T.copy_(torch.as_tensor(T0n, device="cuda"))
    th.T0.copy_(th.T)
    dr = case.device_state(fem)
    Tq = (T0n[mesh.el2n - 1] @ fem.element_tables(3).N.T).reshape(-1)   # initial T at the integration points
    eta0 = dr.tensor(np.exp(-0.1 * Tq))
    dr.viscosity_ip = (eta0 * torch.repeat_interleave(dr.tensor(np.exp(ac.delta)), mesh.nq)).contiguous()
    bc = case.bc_device()
    lib, h = fem.solver._Handle.get()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    e0, e1, e2, e3, e4 = ev(), ev(), ev(), ev(), ev()
    e0.record()
    stf, _phi = fem.solve_coupled(th, dr, bcT, bc, dt, Tref=0.0, shear_heating=True, tolerance=args.tolerance,
                                  max_iterations=2_000_000, iter_max=2_000_000, throw_on_failure=False)
    e1.record()
    J, obj = ac.objective(dr.v)
    lam_v, lam_P, sta = fem.solve_adjoint(dr, bc, dt, [dr.tensor(o) for o in obj], tolerance=args.tolerance,
                                          max_iterations=2_000_000, iter_max=2_000_000, max_ph_iterations=1000,
                                          throw_on_failure=False)
    e2.record()
    torch.cuda.synchronize()
    # the gradient once untimed (first launches load their modules), then timed
    (dr.viscosity_ip * fem.viscosity_sensitivity(dr, dt, lam_v, lam_P)).reshape(mesh.nels, mesh.nq).sum(dim=1)
    e2b = ev()
    e2b.record()
    sens = fem.viscosity_sensitivity(dr, dt, lam_v, lam_P)
    grad = (dr.viscosity_ip * sens).reshape(mesh.nels, mesh.nq).sum(dim=1)
    e3.record()
    torch.cuda.synchronize()
    grad = grad.cpu().numpy()
    # central differences with T frozen at the converged coupled state
    ck = fem.DRCheckpoint(dr)
    kfd = min(args.fd_elements, mesh.nels)
    els = rng.choice(mesh.nels, size=kfd, replace=False)
    scale = float(np.abs(grad).max())
    fd_out = []
    fd_iters = 0
    for hh in [float(x) for x in str(args.fd_h).split(",")]:
        errs, fds = [], []
        for k in els:
            vals = []
            for sgn in (1.0, -1.0):
                ck.restore(dr)
                d = ac.delta.copy()
                d[k] += sgn * hh
                dr.viscosity_ip = (eta0 * torch.repeat_interleave(dr.tensor(np.exp(d)), mesh.nq)).contiguous()
                st = fem.solve(dr, bc, dt, tolerance=args.fd_tolerance, max_iterations=2_000_000,
                               iter_max=2_000_000, throw_on_failure=False)
                fd_iters += st["iter"]
                vals.append(ac.objective(dr.v)[0])
            fd = (vals[0] - vals[1]) / (2 * hh)
            fds.append(fd)
            errs.append(abs(fd - grad[k]) / max(abs(fd), 1e-300))
        fd_out.append({"h": hh, "max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs)),
                       "max_abs_err_over_max_grad": float(max(abs(f - grad[k]) for f, k in zip(fds, els)) / scale)})
    e4.record()
    torch.cuda.synchronize()
    line = {
        "mode": "adjoint", "workload": f"coupled-thermal-stokes-adjoint-hex27-{n}^3", "n": n, "dt": dt,
        "forward": {"ms": e0.elapsed_time(e1), "iterations": stf["iter"], "itPH": stf["itPH"],
                    "converged": bool(stf["converged"]), "thermal_iterations": stf["thermal_iterations"]},
        "adjoint": {"ms": e1.elapsed_time(e2), "iterations": sta["iter"], "itPH": sta["itPH"],
                    "converged": bool(sta["converged"]), "err": sta["err"]},
        "gradient_ms": e2b.elapsed_time(e3), "J": J,
        "fd": {"elements": int(kfd), "tolerance": args.fd_tolerance, "ms": e3.elapsed_time(e4),
               "iterations": fd_iters, "per_h": fd_out},
        "scope": "T frozen at the converged coupled state in the adjoint and the differences",
    }
    print(json.dumps(line), flush=True)
    return 0


def warmstart_mode(args, fem):
    """Learned-warm-start workload (2-D Q9/P1-disc shear band, n², `--ws-steps` steps,
    trained on the first `--ws-train`): DR iterations and time to the tolerance per step
    from the plain start, from linear extrapolation and from extrapolation + the network,
    each over the same states. Prints one JSON line."""
    import torch
    rows_out = []
    res = fem.warmstart.shear_band_warm_start(n=args.n, nsteps=args.ws_steps, ntrain=args.ws_train,
                                              epochs=args.ws_epochs, seed=args.seed, tolerance=args.tolerance,
                                              check_interval=args.check_interval, online_steps=args.ws_online,
                                              online_batch=args.ws_online_batch,
                                              log=(lambda r: rows_out.append(r)))
    test = [r for r in res["rows"] if "learned_iter" in r]
    mean = lambda k: float(np.mean([r[k] for r in test])) if test else None
    tot = lambda k: float(np.sum([r[k] for r in test])) if test else None
    line = {
        "mode": "warmstart", "workload": f"shear-band-q9-{args.n}^2", "n": args.n, "steps": args.ws_steps,
        "check_interval": args.check_interval, "online_adam_steps": args.ws_online, "online_batch": args.ws_online_batch,
        "online_train_ms_mean": mean("online_train_ms") if args.ws_online else 0.0,
        "train_steps": args.ws_train, "epochs": args.ws_epochs, "train_ms": res["train_ms"],
        "train_loss_first_last": [res["train_loss"][0], res["train_loss"][-1]] if res["train_loss"] else None,
        "gain": res["gain"], "test_steps": len(test),
        "gain_trace": [r.get("gain") for r in test][::10],
        "iterations_mean": {"plain": mean("plain_iter"), "extrapolation": mean("extrap_iter"),
                            "learned": mean("learned_iter")},
        "time_ms_total": {"plain": tot("plain_ms"), "extrapolation": tot("extrap_ms"), "learned": tot("learned_ms")},
        "inference_ms_mean": mean("infer_ms"),
        "learned_vs_plain_max_rel": max(r["learned_vs_plain_rel"] for r in test) if test else None,
        "all_converged": all(r["plain_converged"] for r in res["rows"]) and all(r["learned_converged"] for r in test),
        "per_step": [{k: r.get(k) for k in ("step", "plain_iter", "extrap_iter", "learned_iter")} for r in test],
    }
    print(json.dumps(line), flush=True)
    return 0


def cellpressure_mode(args, fem):
    """Cell-pressure Hex27 Stokes (CellPressureStokesDR): the sinking block on an n³
    structured mesh (configs.cell_pressure_case), solved from rest to the reference's
    default absolute tolerance 1e-5 with its default steps. Prints one JSON line: the
    solve time and iteration count, the per-launch time and algorithmic HBM bandwidth of
    the momentum and pressure residual kernels, and the oracle's time per iteration on
    all host cores (a bounded sample of 20 iterations) extrapolated to the GPU run's count."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_host as oh
    case = fem.configs.cell_pressure_case(n=args.n, seed=args.seed, distort=False)
    mesh = case.mesh
    dr = fem.CellPressureStokesDR(mesh, case.material, phases=case.phases)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # per-launch kernel times on the zero state (inputs larger than L2 at 64³: geometry 566 MB)
    for _ in range(args.warmup):
        fem.assemble_stokes_momentum_residual_3d(dr)
        fem.assemble_stokes_pressure_residual_3d(dr)
    k = max(args.steps, 5)
    e0, e1, e2 = ev(), ev(), ev()
    e0.record()
    for _ in range(k):
        fem.assemble_stokes_momentum_residual_3d(dr)
    e1.record()
    for _ in range(k):
        fem.assemble_stokes_pressure_residual_3d(dr)
    e2.record()
    torch.cuda.synchronize()
    t_mom = e0.elapsed_time(e1) / k     # includes the launch's Rv zero-fill and the device phase check
    t_pres = e1.elapsed_time(e2) / k
    ne, nn = mesh.nels, mesh.nnodes
    # algorithmic bytes per launch: geometry (J⁻¹ + dΩ per point), connectivity, velocities
    # gathered once per node, phase and pressure per cell, Rv read-modify-write / RP write
    geo = ne * 27 * 10 * 8 + ne * 27 * 4
    b_mom = geo + 3 * nn * 8 + ne * (4 + 32) + 3 * nn * 8 * 2
    b_pres = geo + 3 * nn * 8 + ne * 32
    peak, kind = measured_peaks()
    # the solve
    torch.cuda.synchronize()
    s0, s1 = ev(), ev()
    s0.record()
    st = fem.solve_cell_pressure(dr, case.bc, tolerance=1e-5, max_iterations=args.max_iterations,
                                 check_interval=100, throw_on_failure=False)
    s1.record()
    torch.cuda.synchronize()
    t_solve = s0.elapsed_time(s1) / 1e3
    cpu = None
    if not args.no_cpu_baseline:
        hs = oh.HostCellPressure(mesh, case.material.eta, case.material.rho0, case.material.g, case.phases)
        sample = 20
        t0 = time.perf_counter()
        hs.solve(case.bc, tolerance=1e-300, max_iterations=sample, check_interval=sample, throw_on_failure=False)
        per_it = (time.perf_counter() - t0) / sample
        cpu = {"value": per_it * st["iterations"], "unit": "s", "cores": 1, "kind": "port",
               "sample": f"{sample} oracle iterations at {mesh.nel} ({per_it:.3f} s each, serial), "
                         f"extrapolated to {st['iterations']} iterations"}
    print(json.dumps({
        "mode": "cellpressure", "workload": f"sinking-block-hex27-cell-pressure-{args.n}^3", "nels": ne,
        "nnodes": nn, "value": t_solve, "unit": "s", "iterations": st["iterations"],
        "per_iteration_ms": t_solve * 1e3 / max(st["iterations"], 1), "converged": st["converged"],
        "residual": st["residual"],
        "kernels": {"momentum_ms": t_mom, "momentum_GBs": b_mom / (t_mom / 1e3) / 1e9,
                    "momentum_frac": b_mom / (t_mom / 1e3) / 1e9 / peak, "momentum_bytes": b_mom,
                    "pressure_ms": t_pres, "pressure_GBs": b_pres / (t_pres / 1e3) / 1e9,
                    "pressure_frac": b_pres / (t_pres / 1e3) / 1e9 / peak, "pressure_bytes": b_pres,
                    "peak_GBs": peak, "peak_kind": kind},
        "cpu_baseline": cpu}), flush=True)
    return 0


def cap_mode(args, fem):
    """Tensile-cap local updates (femb200_cap_update, ncomp 6): one 3-D cap_local_update
    per integration point of an n³ Hex27 mesh (27·n³ points; 7.1 M at n = 64) with random
    trial stresses, pressures and per-point materials around the cap (elastic, shear and
    cap branches mixed in every warp). Prints one JSON line: points per second, the
    per-launch time and its algorithmic HBM bandwidth (14 FP64 inputs, 9 FP64 outputs and
    the converged flag per point), and the serial oracle on a 100 000-point sample."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_host as oh
    n = 27 * args.n ** 3
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    u = lambda lo, hi: torch.rand(n, generator=g, device="cuda", dtype=torch.float64) * (hi - lo) + lo
    phi = u(math.radians(10), math.radians(40))
    psi = u(0.0, 1.0) * phi * (u(0.0, 1.0) < 0.8)
    k, kq = torch.sin(phi), torch.sin(psi)
    c = u(0.5, 3.0) * torch.cos(phi)
    pT = -u(0.05, 0.9) * c / k
    tau = torch.randn(n, 6, generator=g, device="cuda", dtype=torch.float64) * 1.5
    P, eve, kdt = u(-3.0, 4.0), u(0.2, 3.0), u(0.5, 8.0)
    ereg = u(0.0, 0.5) * (u(0.0, 1.0) < 0.7)
    out_tau = torch.empty_like(tau)
    out = [torch.empty(n, device="cuda", dtype=torch.float64) for _ in range(3)]
    conv = torch.empty(n, device="cuda", dtype=torch.int32)
    del phi, psi
    lib, h = fem.solver._Handle.get()
    pr = fem._abi.CapProblemC()
    pr.n, pr.ncomp, pr.maxiter = n, 6, 40
    pr.tau_trial, pr.P_trial, pr.eta_ve, pr.K_dt = tau.data_ptr(), P.data_ptr(), eve.data_ptr(), kdt.data_ptr()
    pr.k, pr.kq, pr.c, pr.pT, pr.eta_reg = k.data_ptr(), kq.data_ptr(), c.data_ptr(), pT.data_ptr(), ereg.data_ptr()
    pr.tau, pr.P, pr.gamma_dot, pr.theta_dot = out_tau.data_ptr(), out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr()
    pr.converged = conv.data_ptr()
    call = lambda: fem.solver._check(lib, h, lib.femb200_cap_update(h, C.byref(pr)))
    for _ in range(args.warmup):
        call()
    k_steps = max(args.steps, 5)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record()
    for _ in range(k_steps):
        call()                    # inputs (1.3 GB at n = 64) exceed L2 between launches
    ev[1].record()
    torch.cuda.synchronize()
    t = ev[0].elapsed_time(ev[1]) / k_steps / 1e3
    nbytes = n * (14 * 8 + 9 * 8 + 4)
    peak, kind = measured_peaks()
    cv = conv.bool()
    cpu = None
    if not args.no_cpu_baseline:
        m = 100_000
        host = lambda x: x[:m].cpu().numpy().copy()
        args_h = [host(x) for x in (tau, P, eve, kdt, k, kq, c, pT, ereg)]
        t0 = time.perf_counter()
        oh.cap_update(6, *args_h)
        per = (time.perf_counter() - t0) / m
        cpu = {"value": 1.0 / per, "unit": "points/s", "cores": 1, "kind": "port",
               "sample": f"{m} points of the same batch through the serial oracle ({per * 1e6:.2f} us each)"}
    print(json.dumps({
        "mode": "cap", "workload": f"tensile-cap-local-update-3d-{n}-points", "points": n,
        "value": n / t, "unit": "points/s", "ms_per_launch": t * 1e3, "steps": k_steps, "warmup": args.warmup,
        "converged_frac": float(cv.double().mean()),
        "plastic_frac": float(((out[1] > 0) & cv).double().mean()),
        "roofline": {"bound": "hbm", "achieved": nbytes / t / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": nbytes / t / 1e9 / peak, "bytes_per_launch": nbytes, "peak_kind": kind},
        "cpu_baseline": cpu}), flush=True)
    return 0


def lithostatic_mode(args, fem):
    """Lithostatic pressure (LithostaticPressureDR) on a structured Hex27 n³ mesh: two
    phases in horizontal layers, a temperature that falls with height, the EOS with a
    finite bulk modulus, P = 0 on the top; solved from zero to the reference's default
    relative tolerance 1e-6. Prints one JSON line: solve time and iterations, the
    residual kernel's per-launch time (with and without the Jacobian diagnostics), and
    the oracle's time per iteration on a bounded sample extrapolated to the GPU count."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_host as oh
    n = args.n
    mesh = fem.structured_mixed_mesh(3, (n, n, n))
    z = mesh.coords[:, 2]
    ph = np.where(z < 0.5, 1, 2).astype(np.int32)
    mat = dict(rho0=(3.3, 2.8), alpha=(3e-2, 3e-2), K=(100.0, 80.0))
    T = 1.0 - z
    top = (np.nonzero(np.abs(z - 1.0) < 1e-12)[0] + 1).astype(np.int32)
    bc = (top, np.zeros(len(top)))
    g = (0.0, 0.0, -1.0)
    dr = fem.LithostaticPressureDR(mesh, phases=ph, **mat)
    dr.T.copy_(torch.as_tensor(T, device="cuda"))
    ev = lambda: torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        fem.assemble_lithostatic_pressure(dr, Tref=0.0, g=g, compute_jacobian=True)
    k = max(args.steps, 5)
    e0, e1, e2 = ev(), ev(), ev()
    e0.record()
    for _ in range(k):
        fem.assemble_lithostatic_pressure(dr, Tref=0.0, g=g)
    e1.record()
    for _ in range(k):
        fem.assemble_lithostatic_pressure(dr, Tref=0.0, g=g, compute_jacobian=True)
    e2.record()
    torch.cuda.synchronize()
    t_res, t_jac = e0.elapsed_time(e1) / k, e1.elapsed_time(e2) / k
    dr.P.zero_()
    dr.rate.zero_()
    s0, s1 = ev(), ev()
    s0.record()
    st = fem.solve_lithostatic(dr, bc, Tref=0.0, g=g, tolerance=1e-6, max_iterations=args.max_iterations,
                               throw_on_failure=False)
    s1.record()
    torch.cuda.synchronize()
    t_solve = s0.elapsed_time(s1) / 1e3
    ne, nn = mesh.nels, mesh.nnodes
    nbytes = ne * 27 * 10 * 8 + ne * 27 * 4 + nn * 8 * 3 + nn * 4 + nn * 8 * 2   # geometry, el2n, P/T + phase, R RMW
    peak, kind = measured_peaks()
    cpu = None
    if not args.no_cpu_baseline:
        # the oracle's first iteration assembles the Jacobian diagnostics; the next ones do not
        hs = oh.HostLithostatic(mesh, phases=ph, T=T, **mat)
        t0 = time.perf_counter()
        hs.solve(bc, Tref=0.0, g=g, tolerance=0.0, max_iterations=1, check_interval=1000, throw_on_failure=False)
        t_jac_it = time.perf_counter() - t0
        hs = oh.HostLithostatic(mesh, phases=ph, T=T, **mat)
        sample = 10
        t0 = time.perf_counter()
        hs.solve(bc, Tref=0.0, g=g, tolerance=0.0, max_iterations=sample + 1, check_interval=1000,
                 throw_on_failure=False)
        t_it = max(time.perf_counter() - t0 - t_jac_it, 0.0) / sample
        n_jac = st["iterations"] // 100 + 1
        cpu = {"value": n_jac * t_jac_it + (st["iterations"] - n_jac) * t_it, "unit": "s", "cores": 1,
               "kind": "port",
               "sample": f"oracle at {mesh.nel}, serial: one iteration with the Jacobian diagnostics "
                         f"({t_jac_it:.3f} s) and {sample} without ({t_it:.4f} s each), extrapolated to "
                         f"{st['iterations']} iterations with {n_jac} Jacobian assemblies"}
    print(json.dumps({
        "mode": "lithostatic", "workload": f"layered-lithostatic-hex27-{n}^3", "nels": ne, "nnodes": nn,
        "value": t_solve, "unit": "s", "iterations": st["iterations"], "converged": st["converged"],
        "residual": st["residual"],
        "kernels": {"residual_ms": t_res, "residual_GBs": nbytes / (t_res / 1e3) / 1e9,
                    "residual_frac": nbytes / (t_res / 1e3) / 1e9 / peak, "residual_bytes": nbytes,
                    "residual_with_jacobian_ms": t_jac, "peak_GBs": peak, "peak_kind": kind},
        "cpu_baseline": cpu}), flush=True)
    return 0


def conv_mode(args, fem):
    """The learned warm start's network on its own: the (2n+1)² node grid of an n² Q9 mesh,
    `--conv-batch` images; CUDA-event times of the 6-layer forward and of one training step
    (forward, MSE, backward through the ReLU masks, Adam), after `--warmup` untimed repetitions,
    averaged over `--steps`. Prints one JSON line."""
    import torch
    ws = fem.warmstart
    B, H = args.conv_batch, 2 * args.n + 1
    net = ws.WarmStartNet(seed=args.seed)
    g = torch.Generator(device="cuda").manual_seed(args.seed)
    x = torch.randn(B * H * H * ws.IN_CH, device="cuda", generator=g).to(torch.bfloat16)
    tgt = torch.randn(B * H * H * 3, device="cuda", generator=g)
    npix = B * H * H

    def forward():
        net.forward(x, B, H, H)

    def train_step():
        net.zero_grad()
        out, acts = net.forward(x, B, H, H, keep=True)
        _, dy = net.loss_grad(out, tgt, npix, 1.0 / npix)
        net.backward(acts, dy, B, H, H)
        net.adam()

    line = {"mode": "conv", "workload": f"warm-start-net-{B}x{H}^2", "batch": B, "grid": [H, H],
            "layers": len(net.layers), "steps": args.steps, "warmup": args.warmup,
            "kernels": "conv3x3_tc_kernel / conv3x3_wgrad_tc_kernel (tcgen05.mma kind::f16, FP32 in TMEM)"}
    for name, fn in (("forward_ms", forward), ("train_step_ms", train_step)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        line[name] = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps(line))


def timeloop_mode(args, fem):
    """Time loop of the layered visco-elasto-plastic case (BASELINE config 2 shape): each
    step P0 ← P, solve to the tolerance, τ_old ← τ. Arms, each on its own trajectory:
    plain FP64 DR from the previous step's solution; mixed precision from the previous
    solution; mixed precision from the linearly extrapolated state 2x_t − x_{t−1}
    (steps ≥ 3). Prints one JSON line with per-step iterations and times."""
    import torch
    case = fem.configs.vep_layers_case(n=args.n, seed=args.seed)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    lib, h = fem.solver._Handle.get()

    def run(precision, extrapolate, profile=False):
        dr = case.device_state()
        bc = case.bc_device()
        hist, rows = [], []
        for step in range(1, args.tl_steps + 1):
            dr.P0.copy_(dr.P)
            torch.cuda.synchronize()
            if profile:
                lib.femb200_profile(h, 1)
            ev0.record()
            if extrapolate and len(hist) == 2:
                fem.warmstart.extrapolate_state(dr, bc, hist[0][0], hist[1][0], hist[0][1], hist[1][1])
            st = fem.solve(dr, bc, dt=case.dt, tolerance=args.tolerance, check_interval=args.check_interval,
                           throw_on_failure=False, max_iterations=2_000_000, iter_max=2_000_000, precision=precision)
            ev1.record()
            torch.cuda.synchronize()
            rows.append({"step": step, "iter": st["iter"], "ms": ev0.elapsed_time(ev1), "converged": bool(st["converged"])})
            if profile:
                pm = (C.c_double * fem._abi.PROF_COUNT)()
                pn = (C.c_int64 * fem._abi.PROF_COUNT)()
                lib.femb200_profile_read(h, pm, pn)
                cnt = (C.c_int64 * fem._abi.COUNTER_COUNT)()
                lib.femb200_profile_counters(h, cnt, fem._abi.COUNTER_COUNT)
                lib.femb200_profile(h, 0)
                rows[-1]["kernel_ms"] = {"sweep": pm[0], "jacobian": pm[1], "node_update": pm[2], "outer_fp64": pm[4]}
                rows[-1]["sweep_avg_us"] = pm[0] / max(pn[0], 1) * 1e3
                rows[-1]["jacobian_assemblies"] = st["jacobian_assemblies"]
                rows[-1]["stress_reads_per_sweep"] = cnt[fem._abi.COUNTER_STRESS_READS] / max(pn[0], 1)
                rows[-1]["shared_jacobian_elements"] = int(cnt[fem._abi.COUNTER_SHARED_JACOBIANS])
            fem.update_stokes_current_stress(dr, case.dt)
            for c in range(6):
                dr.tau_old[c].copy_(dr.tau[c])
            hist.append(([x.clone() for x in dr.v], dr.P.clone()))
            hist = hist[-2:]
        return rows, torch.cat(list(dr.v)), dr.P.clone()

    arms = {"plain_fp64": run("fp64", False), "mixed": run("mixed", False), "mixed_extrapolated": run("mixed", True)}
    ref_v, ref_P = arms["plain_fp64"][1], arms["plain_fp64"][2]
    out = {"mode": "timeloop", "workload": f"vep-layers-hex27-{args.n}^3 x {args.tl_steps} steps", "n": args.n,
           "steps": args.tl_steps, "tolerance": args.tolerance, "arms": {}}
    for name, (rows, v, P) in arms.items():
        out["arms"][name] = {
            "total_s": sum(r["ms"] for r in rows) / 1e3, "iterations": [r["iter"] for r in rows],
            "all_converged": all(r["converged"] for r in rows),
            "final_rel_err_vs_plain": {"v": float(torch.linalg.norm(v - ref_v) / torch.linalg.norm(ref_v)),
                                       "P": float(torch.linalg.norm(P - ref_P) / torch.linalg.norm(ref_P))}}
    tp = out["arms"]["plain_fp64"]["total_s"]
    out["speedup_vs_plain_fp64"] = {k: tp / a["total_s"] for k, a in out["arms"].items()}
    if args.tl_profile:
        # the mixed arm once more with CUDA events around every launch: the per-step split
        out["mixed_profiled_steps"] = run("mixed", False, profile=True)[0]
    print(json.dumps(out), flush=True)
    return 0


def _rel(a, b):
    """Relative L2 difference ‖a − b‖ / ‖b‖ of two numpy arrays."""
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def _mean_free(P, M):
    """P without its M_P-weighted mean (pressure is compared up to a constant)."""
    return P - float(np.sum(P * M) / np.sum(M))


def field_subsample(case, seed=1234):
    """Seeded index sets into the concatenated v (3·nnodes), P (nnodesP) and τ (6·27·nels)
    of a 3-D case: up to 50 000, 50 000 and 100 000 entries, the same on every host."""
    m = case.mesh
    rng = np.random.default_rng(seed)
    pick = lambda n, k: np.sort(rng.choice(n, size=min(n, k), replace=False))
    return {"v": pick(3 * m.nnodes, 50_000), "P": pick(m.nnodesP, 50_000), "tau": pick(6 * m.nq * m.nels, 100_000)}


def oracle_time_loop(args, fem):
    """The oracle's time loop of the layered case (P0 ← P, τ_old ← τ between steps), saved
    after every step to --oracle3d: per-step statistics and wall time, and the fields on the
    seeded subsample (P also without its M_P-weighted mean)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_host as oh
    case = fem.configs.vep_layers_case(n=args.n, seed=args.seed)
    hs = case.host_state(oh)
    sub = field_subsample(case)
    kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=args.check_interval, throw_on_failure=False,
              max_iterations=args.max_iterations, iter_max=args.max_iterations)
    name, nproc = cpu_model()
    meta = {"n": args.n, "seed": args.seed, "tolerance": args.tolerance, "check_interval": args.check_interval,
            "host": {"cpu_model": name, "nproc": nproc, "oracle_threads": oh.lib().orc_num_threads()}, "steps": []}
    arrays = {}
    for step in range(args.tl_steps):
        t0 = time.perf_counter()
        st = hs.solve(**kw)
        sec = time.perf_counter() - t0
        hs.store_stress(case.dt)
        v, P, tau = np.concatenate(hs.v), hs.P.copy(), np.concatenate(hs.tau)
        Pmf = P - float(np.sum(P * hs.M_P) / np.sum(hs.M_P))
        meta["steps"].append({"stats": {k: st[k] for k in ("iter", "itPH", "jacobian_assemblies", "converged", "err")},
                              "seconds": sec})
        arrays.update({f"v{step}": v[sub["v"]], f"P{step}": P[sub["P"]], f"Pmf{step}": Pmf[sub["P"]],
                       f"tau{step}": tau[sub["tau"]]})
        np.savez(args.oracle3d, meta=json.dumps(meta), **arrays)
        print(json.dumps({"oracle_step": step + 1, **meta["steps"][-1]}), flush=True)
        hs.P0[:] = hs.P
        for c in range(6):
            hs.tau_old[c][:] = hs.tau[c]
    return 0


def load_oracle_steps(args):
    z = np.load(args.oracle3d, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    if meta["n"] != args.n or meta["tolerance"] != args.tolerance or meta["check_interval"] != args.check_interval:
        raise SystemExit(f"{args.oracle3d} holds another configuration: {meta}")
    if len(meta["steps"]) < args.tl_steps:
        raise SystemExit(f"{args.oracle3d} holds {len(meta['steps'])} steps, {args.tl_steps} asked")
    steps = [dict(m, v=z[f"v{k}"], P=z[f"P{k}"], P_mean_free=z[f"Pmf{k}"], tau=z[f"tau{k}"])
             for k, m in enumerate(meta["steps"])]
    return {"steps": steps, "host": meta["host"]}


def parity_mode(args, fem):
    """Parity at the configurations' own sizes, against the FP64 oracle on all host cores.

    3-D (the layered visco-elasto-plastic case, --n, `--tl-steps` time steps with
    P0 ← P and τ_old ← τ): the device FP64 solve, the device mixed-precision solve and
    the oracle's solve, each from the same state to min(err_abs, err_rel) < tol
    (src/stokes/solvers/DR.jl:568-586); reported per step: iteration counts, relative
    L2 errors of v, P (also without its M_P-weighted mean) and τ against the oracle,
    and the wall times. The oracle's measured time is compared with the CpuSample
    extrapolation along the oracle's own path (the model the 64³ reference figure uses).
    2-D (the inclusion case at --n2d, FP64): the device solve against the oracle's.
    Prints one JSON line."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_host as oh
    out = {"mode": "parity", "tolerance": args.tolerance, "check_interval": args.check_interval}
    name, nproc = cpu_model()
    out["host"] = {"cpu_model": name, "nproc": nproc, "oracle_threads": oh.lib().orc_num_threads()}
    stream = torch.cuda.current_stream()

    def gpu_solve(dr, bc, **kw):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        st = fem.solve(dr, bc, **kw)
        ev1.record(stream)
        torch.cuda.synchronize()
        return st, ev0.elapsed_time(ev1) / 1e3

    keys = ("iter", "itPH", "jacobian_assemblies", "converged", "err")
    if args.n > 0:
        case = fem.configs.vep_layers_case(n=args.n, seed=args.seed)
        bc = case.bc_device()
        d64, dmx = case.device_state(), case.device_state()
        kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=args.check_interval, throw_on_failure=False,
                  max_iterations=args.max_iterations, iter_max=args.max_iterations)
        saved = load_oracle_steps(args) if args.oracle3d else None
        hs = None if saved else case.host_state(oh)
        sub = field_subsample(case) if saved else None
        # warm-up of the device code paths on a copy, so the timed solves carry no first-launch costs
        warm = case.device_state()
        fem.solve(warm, bc, **dict(kw, max_iterations=200, iter_max=200))
        fem.solve(warm, bc, **dict(kw, max_iterations=200, iter_max=200, precision="mixed"))
        del warm
        steps = []
        for step in range(args.tl_steps):
            s64, t64 = gpu_solve(d64, bc, **kw)
            smx, tmx = gpu_solve(dmx, bc, precision="mixed", **kw)
            fem.update_stokes_current_stress(d64, case.dt)
            fem.update_stokes_current_stress(dmx, case.dt)
            torch.cuda.synchronize()
            host = lambda dr: {"v": np.concatenate([x.cpu().numpy() for x in dr.v]), "P": dr.P.cpu().numpy(),
                               "tau": np.concatenate([x.cpu().numpy() for x in dr.tau])}
            if saved:
                o = saved["steps"][step]
                row = {"step": step + 1, "oracle": o["stats"], "oracle_s": o["seconds"],
                       "compared_on": {k: int(len(v)) for k, v in sub.items()}}
            else:
                t0 = time.perf_counter()
                sor = hs.solve(**kw)
                tor = time.perf_counter() - t0
                hs.store_stress(case.dt)
                ref = {"v": np.concatenate(hs.v), "P": hs.P.copy(), "tau": np.concatenate(hs.tau)}
                row = {"step": step + 1, "oracle": {k: sor[k] for k in keys}, "oracle_s": tor}
            for label, dr, st, t in (("gpu_fp64", d64, s64, t64), ("gpu_mixed", dmx, smx, tmx)):
                f = host(dr)
                row[label] = {k: st[k] for k in keys}
                row[label]["seconds"] = t
                if saved:
                    o = saved["steps"][step]
                    M = dr.M_P.cpu().numpy()
                    Pmf = f["P"] - float(np.sum(f["P"] * M) / np.sum(M))
                    row[label]["rel_err_vs_oracle"] = {
                        "v": _rel(f["v"][sub["v"]], o["v"]), "P": _rel(f["P"][sub["P"]], o["P"]),
                        "P_mean_free": _rel(Pmf[sub["P"]], o["P_mean_free"]), "tau": _rel(f["tau"][sub["tau"]], o["tau"])}
                else:
                    row[label]["rel_err_vs_oracle"] = {
                        "v": _rel(f["v"], ref["v"]), "P": _rel(f["P"], ref["P"]),
                        "P_mean_free": _rel(_mean_free(f["P"], hs.M_P), _mean_free(ref["P"], hs.M_P)),
                        "tau": _rel(f["tau"], ref["tau"])}
            steps.append(row)
            print(json.dumps({"parity_step": row}), flush=True)
            # the time-step driver: P0 ← P, τ_old ← τ
            for dr in (d64, dmx):
                dr.P0.copy_(dr.P)
                for c in range(6):
                    dr.tau_old[c].copy_(dr.tau[c])
            if hs is not None:
                hs.P0[:] = hs.P
                for c in range(6):
                    hs.tau_old[c][:] = hs.tau[c]
        out["vep3d"] = {"workload": f"vep-layers-hex27-{args.n}^3 x {args.tl_steps} steps", "steps": steps}
        if saved:
            out["vep3d"]["oracle_host"] = saved["host"]
            out["vep3d"]["comparison"] = "relative L2 on seeded subsamples of the fields (field_subsample)"
        else:
            first = steps[0]["oracle"]
            path = {"iterations": first["iter"], "itPH": first["itPH"],
                    "jacobian_assemblies": first["jacobian_assemblies"], "check_interval": args.check_interval}
            # the extrapolation model on the same workload, priced along the oracle's own path of step 1
            est, cores, sample = cpu_baseline_estimate(fem.configs.vep_layers_case(n=args.n, seed=args.seed), path,
                                                       steps=3)
            out["vep3d"]["cpu_model_check"] = {"measured_s": steps[0]["oracle_s"], "extrapolated_s": est,
                                               "model_error": est / steps[0]["oracle_s"] - 1.0, "sample": sample}
    if args.n2d > 0:
        case = fem.configs.inclusion_2d_case(n=args.n2d)
        kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=50, throw_on_failure=False,
                  max_iterations=args.max_iterations, iter_max=args.max_iterations)
        ref = inclusion_oracle(args, case, oh, kw)
        dr = case.device_state()
        st, tg = gpu_solve(dr, case.bc_device(), **kw)
        f = {"v": np.concatenate([x.cpu().numpy() for x in dr.v]), "P": dr.P.cpu().numpy()}
        out["inclusion2d"] = {
            "workload": f"inclusion-q9-{args.n2d}^2", "check_interval": 50,
            "oracle": ref["stats"], "oracle_s": ref["seconds"], "oracle_host": ref["host"],
            "gpu_fp64": dict({k: st[k] for k in ("iter", "itPH", "converged", "err")}, seconds=tg),
            "rel_err_vs_oracle": {"v": _rel(f["v"], ref["v"]), "P": _rel(f["P"], ref["P"]),
                                  "P_mean_free": _rel(_mean_free(f["P"], ref["M_P"]), _mean_free(ref["P"], ref["M_P"]))}}
    print(json.dumps(out), flush=True)
    return 0


def inclusion_oracle(args, case, oh, kw):
    """The oracle's solve of the 2-D inclusion case: loaded from --oracle2d (an .npz
    this function wrote with --oracle-only, possibly on another host), or run here."""
    if args.oracle2d and os.path.exists(args.oracle2d) and not args.oracle_only:
        z = np.load(args.oracle2d, allow_pickle=False)
        meta = json.loads(str(z["meta"]))
        if meta["n"] != args.n2d or meta["tolerance"] != args.tolerance:
            raise SystemExit(f"{args.oracle2d} holds n={meta['n']}, tolerance={meta['tolerance']}")
        return {"v": z["v"], "P": z["P"], "M_P": z["M_P"], "stats": meta["stats"], "seconds": meta["seconds"],
                "host": meta["host"]}
    hs = case.host_state(oh)
    t0 = time.perf_counter()
    sor = hs.solve(**kw)
    sec = time.perf_counter() - t0
    name, nproc = cpu_model()
    res = {"v": np.concatenate(hs.v), "P": hs.P.copy(), "M_P": hs.M_P.copy(),
           "stats": {k: sor[k] for k in ("iter", "itPH", "converged", "err")}, "seconds": sec,
           "host": {"cpu_model": name, "nproc": nproc, "oracle_threads": oh.lib().orc_num_threads()}}
    if args.oracle2d:
        meta = {"n": args.n2d, "tolerance": args.tolerance, "stats": res["stats"], "seconds": sec, "host": res["host"]}
        np.savez(args.oracle2d, v=res["v"], P=res["P"], M_P=res["M_P"], meta=json.dumps(meta))
    return res


def workload_config(args, case, world=1):
    """The `config` object of both arms' JSON lines: the workload only, no run results."""
    m = case.mesh
    return {"workload": f"vep-layers-hex27-{args.n}^3", "nel": [args.n] * 3, "seed": args.seed,
            "tolerance": args.tolerance, "check_interval": args.check_interval, "dt": case.dt,
            "nels": m.nels, "nnodes": m.nnodes, "nnodesP": m.nnodesP,
            "l2": "inputs larger than L2 (geometry alone %.0f MB)" % (m.geo_v.nbytes / 1e6),
            "parallelism": f"replicas{world}"}


def run_reference(args):
    """--impl reference: the reference's CPU path on this host (the oracle, its C++ FP64
    restatement, all host cores) on the same workload. Julia cannot run here, so this is
    the stand-in the reference's CPU KernelAbstractions path is timed by. Every step is
    one bounded CpuSample step on the full mesh; the value is the solve's time
    extrapolated along the measured DR path (PATH_64, or --ref-* for other sizes)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    fem = load_package()
    case = fem.configs.vep_layers_case(n=args.n, seed=args.seed)
    if args.ref_iterations > 0:
        path = {"iterations": args.ref_iterations, "itPH": args.ref_itph, "jacobian_assemblies": args.ref_jacobians,
                "check_interval": args.check_interval}
    elif args.n == 64 and args.seed == 0 and args.check_interval == PATH_64["check_interval"]:
        path = dict(PATH_64)
    else:
        print(json.dumps({"impl": "reference", "unavailable": "no measured DR path for this size; pass --ref-iterations, "
                          "--ref-itph and --ref-jacobians"}))
        return 0
    smp = CpuSample(case)
    figs = []
    for i in range(args.warmup + args.steps):
        f = smp.step()
        if i >= args.warmup:
            figs.append(f)
    fig = {k: statistics.mean(f[k] for f in figs) for k in figs[0]}
    t = CpuSample.estimate(fig, path)
    name, nproc = cpu_model()
    line = {
        "impl": "reference", "metric": METRIC, "value": t, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "method": "oracle: C++ FP64 restatement of the reference's CPU path (Julia is not available here)",
        "config": workload_config(args, case),
        "value_kind": "extrapolated: the timed per-step sample priced along the measured DR path",
        "path": path,
        "sample_figures_s": fig,
        "cpu_baseline": {"value": t, "unit": "s", "cores": smp.cores, "kind": "port", "sample": smp.describe(fig),
                         "cpu_model": name, "nproc": nproc},
        "e2e": {"value": t, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", "--size", dest="n", type=int, default=64,
                    help="elements per direction (--size spells it under torchrun, whose own options --n abbreviates)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="the chosen method (mixed: FP32 increments inside FP64 outer steps)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison solve")
    ap.add_argument("--check-interval", type=int, default=100)
    ap.add_argument("--tolerance", type=float, default=1e-8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-iterations", type=int, default=0,
                    help="DR iterations of the path the reference sample is priced along (default: PATH_64)")
    ap.add_argument("--ref-jacobians", type=int, default=0)
    ap.add_argument("--ref-itph", type=int, default=0)
    ap.add_argument("--max-iterations", type=int, default=2_000_000,
                    help="cap on DR iterations per solve (profiling runs of a few sweeps)")
    ap.add_argument("--adjoint-dt", type=float, default=1e-2)
    ap.add_argument("--fd-elements", type=int, default=20)
    ap.add_argument("--fd-h", default="1e-6,1e-4", help="central-difference steps, comma-separated")
    ap.add_argument("--fd-tolerance", type=float, default=1e-13)
    ap.add_argument("--ws-steps", type=int, default=200)
    ap.add_argument("--ws-train", type=int, default=50)
    ap.add_argument("--ws-epochs", type=int, default=300)
    ap.add_argument("--ws-online", type=int, default=0, help="Adam steps on the newest converged pairs per solved step")
    ap.add_argument("--ws-online-batch", type=int, default=4)
    ap.add_argument("--tl-steps", type=int, default=10)
    ap.add_argument("--tl-profile", action="store_true", help="timeloop mode: per-step kernel split of the mixed arm")
    ap.add_argument("--n2d", type=int, default=0, help="parity mode: size of the 2-D inclusion case (0: skip)")
    ap.add_argument("--oracle2d", default="", help="parity mode: .npz of the 2-D oracle solve (read, or written "
                    "with --oracle-only)")
    ap.add_argument("--oracle-only", action="store_true", help="parity mode: run and save the oracle's solves only")
    ap.add_argument("--oracle3d", default="", help="parity mode: .npz of the 3-D oracle time loop (read, or written "
                    "with --oracle-only)")
    ap.add_argument("--conv-batch", type=int, default=8, help="conv mode: images per batch")
    ap.add_argument("--mode", default="solve", choices=["solve", "sweep", "adjoint", "warmstart", "timeloop", "cellpressure", "lithostatic", "cap",
                             "parity", "scatter-order", "conv"],
                    help="sweep: time K fused residual sweeps and K Jacobian assemblies on the initial state")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "parity" and args.oracle_only and args.oracle3d:
        # the CPU half of the 3-D time-loop parity check, on a host without a GPU
        return oracle_time_loop(args, load_package())
    if args.mode == "parity" and args.oracle_only:
        # the CPU half of the 2-D parity check, on a host without a GPU
        fem = load_package()
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_host as oh
        case = fem.configs.inclusion_2d_case(n=args.n2d)
        kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=50, throw_on_failure=False,
                  max_iterations=args.max_iterations, iter_max=args.max_iterations)
        ref = inclusion_oracle(args, case, oh, kw)
        print(json.dumps({"mode": "parity-oracle-2d", "n": args.n2d, "stats": ref["stats"], "seconds": ref["seconds"],
                          "host": ref["host"]}), flush=True)
        return 0

    import torch
    import torch.distributed as dist
    fem = load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    if args.mode == "adjoint":
        return adjoint_mode(args, fem)
    if args.mode == "warmstart":
        return warmstart_mode(args, fem)
    if args.mode == "conv":
        return conv_mode(args, fem)
    if args.mode == "timeloop":
        return timeloop_mode(args, fem)
    if args.mode == "cellpressure":
        return cellpressure_mode(args, fem)
    if args.mode == "lithostatic":
        return lithostatic_mode(args, fem)
    if args.mode == "cap":
        return cap_mode(args, fem)
    if args.mode == "parity":
        return parity_mode(args, fem)
    case = fem.configs.vep_layers_case(n=args.n, seed=args.seed)
    dr = case.device_state()
    bc = case.bc_device()
    lib, h = fem.solver._Handle.get()
    if args.mode == "sweep":
        return sweep_mode(args, fem, case, dr, lib, h)
    if args.mode == "scatter-order":
        return scatter_order_mode(args, fem, case, dr, lib, h)
    # device-resident initial state of every step
    init = {"v": [x.clone() for x in dr.v], "P": dr.P.clone(), "P0": dr.P0.clone(),
            "tau_old": [x.clone() for x in dr.tau_old]}

    def reset():
        for c in range(3):
            dr.v[c].copy_(init["v"][c])
        dr.P.copy_(init["P"])
        dr.P0.copy_(init["P0"])
        for c in range(6):
            dr.tau_old[c].copy_(init["tau_old"][c])

    kw = dict(dt=case.dt, tolerance=args.tolerance, check_interval=args.check_interval, throw_on_failure=False,
              max_iterations=args.max_iterations, iter_max=args.max_iterations, precision=args.precision)
    stats = None
    for _ in range(args.warmup):
        reset()
        stats = fem.solve(dr, bc, **kw)
    barrier()

    # ---- timed region: inputs resident in HBM ----
    sampler = ClockSampler(local)
    sampler.start()
    # launch counter reset; no per-kernel events inside the timed region
    lib.femb200_profile(h, 0)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    step_stats = []
    for _ in range(args.steps):
        reset()
        step_stats.append(fem.solve(dr, bc, **kw))
    ev1.record(stream)
    barrier()
    ms_total = ev0.elapsed_time(ev1)
    prof_ms = (C.c_double * fem._abi.PROF_COUNT)()
    prof_n = (C.c_int64 * fem._abi.PROF_COUNT)()
    lib.femb200_profile_read(h, prof_ms, prof_n)
    launches_timed = int(prof_n[3])
    clocks = sampler.stop()
    # the kernel split and the hot kernel's launch times: one more solve with CUDA events
    # around every launch (kept out of the timed steps: the events cost host time)
    lib.femb200_profile(h, 1)
    reset()
    ev0.record(stream)
    fem.solve(dr, bc, **kw)
    ev1.record(stream)
    barrier()
    ms_profiled = ev0.elapsed_time(ev1)
    lib.femb200_profile_read(h, prof_ms, prof_n)
    counters = (C.c_int64 * fem._abi.COUNTER_COUNT)()
    lib.femb200_profile_counters(h, counters, fem._abi.COUNTER_COUNT)
    lib.femb200_profile(h, 0)
    stress_reads = counters[fem._abi.COUNTER_STRESS_READS] / max(prof_n[0], 1)
    t_step = ms_total / 1e3 / args.steps
    t_step = max_over_ranks(t_step, world)

    # ---- end to end: host inputs in pinned memory, copies inside the timed region ----
    host_in = {k: ([x.cpu().pin_memory() for x in v] if isinstance(v, list) else v.cpu().pin_memory())
               for k, v in init.items()}
    out_v = [torch.empty(dr.mesh.nnodes, dtype=dr.dtype).pin_memory() for _ in range(3)]
    out_P = torch.empty(dr.mesh.nnodesP, dtype=dr.dtype).pin_memory()
    h2d = sum(x.numel() * x.element_size() for v in host_in.values() for x in (v if isinstance(v, list) else [v]))
    d2h = sum(x.numel() * x.element_size() for x in out_v) + out_P.numel() * out_P.element_size()
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    ev0.record(stream)
    for _ in range(e2e_steps):
        for c in range(3):
            dr.v[c].copy_(host_in["v"][c], non_blocking=True)
        dr.P.copy_(host_in["P"], non_blocking=True)
        dr.P0.copy_(host_in["P0"], non_blocking=True)
        for c in range(6):
            dr.tau_old[c].copy_(host_in["tau_old"][c], non_blocking=True)
        fem.solve(dr, bc, **kw)
        for c in range(3):
            out_v[c].copy_(dr.v[c], non_blocking=True)
        out_P.copy_(dr.P, non_blocking=True)
    ev1.record(stream)
    barrier()
    t_e2e = ev0.elapsed_time(ev1) / 1e3 / e2e_steps
    t_e2e = max_over_ranks(t_e2e, world)

    st = step_stats[-1]
    iters = st["iter"]
    jacs = st["jacobian_assemblies"]

    def snapshot():
        fem.update_stokes_current_stress(dr, case.dt)
        return {"v": torch.cat([x.clone() for x in dr.v]), "P": dr.P.clone(),
                "tau": torch.cat([x.clone() for x in dr.tau])}

    # ---- the plain FP64 DR solve of the same workload, and the chosen method's field error ----
    plain = None
    if args.precision == "mixed" and not args.no_plain:
        chosen_fields = snapshot()
        kw64 = dict(kw, precision="fp64")
        # warm-up solve with per-kernel events (the split), then the timed solve without
        lib.femb200_profile(h, 1)
        reset()
        fem.solve(dr, bc, **kw64)
        barrier()
        pm = (C.c_double * fem._abi.PROF_COUNT)()
        pn = (C.c_int64 * fem._abi.PROF_COUNT)()
        lib.femb200_profile_read(h, pm, pn)
        lib.femb200_profile(h, 0)
        reset()
        ev0.record(stream)
        st64 = fem.solve(dr, bc, **kw64)
        ev1.record(stream)
        barrier()
        t64 = ev0.elapsed_time(ev1) / 1e3
        t64 = max_over_ranks(t64, world)
        f64 = snapshot()
        err = {k: float(torch.linalg.norm(chosen_fields[k] - f64[k]) / torch.linalg.norm(f64[k])) for k in f64}
        plain = {"value": t64, "unit": "s", "iterations": st64["iter"], "itPH": st64["itPH"],
                 "jacobian_assemblies": st64["jacobian_assemblies"], "converged": bool(st64["converged"]),
                 "err": st64["err"],
                 "kernel_ms": {"residual": pm[0], "jacobian": pm[1], "node_update": pm[2]},
                 "residual_avg_ms": pm[0] / max(pn[0], 1),
                 "field_rel_err_chosen_vs_fp64": err}
    if plain:
        path = {"iterations": plain["iterations"], "itPH": plain["itPH"],
                "jacobian_assemblies": plain["jacobian_assemblies"], "check_interval": args.check_interval}
    else:
        path = {"iterations": iters, "itPH": st["itPH"], "jacobian_assemblies": jacs,
                "check_interval": args.check_interval}

    peak, peak_kind = measured_peaks()
    mixed = args.precision == "mixed"
    # the survey's counting rule for one fused element pass (every array the sweep must touch,
    # once, at its stored precision): FP32 for the chosen method's sweep, FP64 for the plain one
    nbytes = residual_kernel_bytes(case, itemsize=4 if mixed else 8, geo_itemsize=4 if mixed else 8)
    res_avg_ms = prof_ms[0] / max(prof_n[0], 1)
    achieved = nbytes / (res_avg_ms / 1e3) / 1e9
    traffic = TRAFFIC.get((args.n, args.precision))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # a bounded sample: two CpuSample steps (about 20 s of CPU work at 64³)
        est, cores, sample = cpu_baseline_estimate(case, path, steps=2)
        name, nproc = cpu_model()
        cpu = {"value": est, "unit": "s", "cores": cores, "kind": "port", "sample": sample, "cpu_model": name,
               "nproc": nproc}

    if rank == 0:
        if mixed:
            kernel = "hex27_incr_kernel (thread-per-element FP32 incremental sweep: RP, Pnum, Rv increments)"
        elif mesh_is_affine(case.mesh):
            kernel = "hex27_residual_pipe_kernel<double> (fused RP + Pnum + Rv sweep, affine geometry)"
        else:
            kernel = "hex27_residual_kernel (fused RP + Pnum + Rv sweep)"
        line = {
            "metric": METRIC, "value": t_step, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "method": "mixed precision (FP32 increments, FP64 outer steps)" if mixed else "plain FP64 DR",
            "config": workload_config(args, case, world),
            "path": {"iterations": iters, "itPH": st["itPH"], "jacobian_assemblies": jacs,
                     "fp64_outer_sweeps": st.get("defect_corrections", 0), "converged": bool(st["converged"]),
                     "err": st["err"]},
            "plain_fp64": plain,
            "speedup_vs_plain_fp64": (plain["value"] / t_step) if plain else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                         "algorithmic_bytes_per_launch": nbytes, "avg_launch_ms": res_avg_ms,
                         "launches": int(prof_n[0]), "peak_kind": peak_kind,
                         "bytes_rule": "fused element pass, stored precision, affine geometry (SURVEY 8d rule)",
                         "kernel_read_bytes_per_launch": incremental_kernel_bytes(case, stress_reads) if mixed else None,
                         "base_stress_reads_per_launch": stress_reads if mixed else None},
            "kernel_ms": {"residual": prof_ms[0], "jacobian": prof_ms[1], "node_update": prof_ms[2],
                          "outer_fp64_sweeps": prof_ms[4], "profiled_solve": ms_profiled},
            "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_timed,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
