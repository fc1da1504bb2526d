#!/usr/bin/env python
"""Benchmark of the GeoFLOW spectral-element hot path on B200.

Headline workload (one GPU): the 3-d Helmholtz solve (alpha M + nu K) u = f
on the unit cube, 32^3 hexahedral elements at p = 7 (16.8 M element-local
nodes), homogeneous Dirichlet boundaries, alpha = nu = 1, right-hand side a
seeded sum of 8 sinusoidal modes (wavenumbers 1..8, N(0,1) amplitudes),
b = M_L f.  CG to a relative residual of 1e-10 (||r||_2 <= 1e-10 ||b||_2 on
the assembled, masked FP64 residual).  One "step" is one complete solve
from x = 0.  Three solvers are timed on the same problem: plain FP64
Jacobi-PCG (the reference algorithm), FP32 PCG with FP64 reliable updates,
and FP64 CG preconditioned by one FP32 p/h-multigrid V-cycle (its hierarchy
is built by a first, separately timed solve and reused); `value` is the
time to solution of the fastest, with inputs resident in HBM.

Also reported: RK-stage throughput (GDOF/s) of 3-d Burgers with SSP-RK3 on
a periodic 64^3-element p = 5 box in FP32 and FP64 (per kernel, and the
FP32 state's difference from FP64), the roofline of the fused Helmholtz
apply, an end-to-end solve through the host-buffer C ABI entry point, the
2-d advection case's error against the reference's own run, and the CPU
port timed on a bounded sample.

Reference arm (--impl reference): the oracle port of the reference's FP64
Jacobi-PCG (GCG + GHelmholtz + GGFX, bit-identical to the reference's own
compiled code on the pinned cases) built with OpenMP on every host core,
on the full headline problem: bounded samples of CG iterations as the
steps, then one complete solve to the same stop rule, whose measured time
is the value.

Usage: python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU (torchrun): every rank solves its own replica (the path does not
partition across GPUs in this build); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GDOF/s per RK stage and CG time-to-1e-10: FP32+refine vs plain FP64, same B200"
SEED = 20261203
L2_BYTES = 126 * 2 ** 20


def profile_traffic(name):
    """DRAM bytes (read + write) per launch recorded by the ncu capture that
    profiles/<name>.md summarises (its `traffic_bytes_per_launch:` line), or
    None."""
    try:
        for line in (ROOT / "profiles" / f"{name}.md").read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ne", type=int, default=32)
    ap.add_argument("--p", type=int, default=7)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--rk-ne", type=int, default=64)
    ap.add_argument("--rk-p", type=int, default=5)
    ap.add_argument("--no-rk", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample-ne", type=int, default=16)
    ap.add_argument("--inner", type=float, default=None,
                    help="mixed: relative drop per restarted FP32 run (0: reliable updates)")
    ap.add_argument("--ru", type=int, default=32,
                    help="FP32 iterations between FP64 residual replacements (mixed solve)")
    ap.add_argument("--mixed-apply", type=int, default=0,
                    help="mixed solve: 1 = FP64 arithmetic in the FP32-stored applies")
    ap.add_argument("--poly", type=int, default=2,
                    help="FP32 applies per Chebyshev preconditioner application")
    ap.add_argument("--poly-ratio", type=float, default=0.0,
                    help="b/a of the Chebyshev interval (0: library default)")
    ap.add_argument("--mg-degree", type=int, default=1,
                    help="multigrid: Chebyshev smoothing degree per level and side")
    ap.add_argument("--mg-ratio", type=float, default=0.0,
                    help="multigrid: lmax/lmin of the smoothing interval (0: library default)")
    ap.add_argument("--ens-members", type=int, default=16,
                    help="ensemble: members of each kind (the first ones drawn)")
    ap.add_argument("--ens-max-level", type=int, default=5,
                    help="ensemble: icosahedral levels above this are lowered to it")
    ap.add_argument("--ens-fixed-shape", action="store_true",
                    help="ensemble: a fixed launch shape instead of the autotuner's (profiling)")
    ap.add_argument("--only", choices=["fp64", "mixed", "cheb", "pmg", "pmg64", "pmgkern", "apply",
                                       "adjoint", "graphs", "ensemble", "rk", "maps"],
                    default=None,
                    help="time only one CG path (for profiling runs)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """Samples SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms",
                 "200", "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


# ---------------------------------------------------------------------------
def make_helmholtz_problem(ctx, ne, p):
    import torch
    from geoflow_b200 import GGFX, GMass, GridBox, Problem
    from geoflow_b200 import workloads as W
    g = GridBox(3, [ne] * 3, p)
    prob = Problem(ctx, g)
    k, a = W.helmholtz_rhs_modes()
    dev = ctx.torch_device
    x, y, z = (torch.from_numpy(c).to(dev) for c in g.xyz)
    f = torch.zeros_like(x)
    for m in range(len(a)):
        f += a[m] * torch.sin(np.pi * k[m, 0] * x) * torch.sin(np.pi * k[m, 1] * y) * \
            torch.sin(np.pi * k[m, 2] * z)
    del x, y, z
    b = prob.zeros()
    GMass(prob).opVec_prod(f, None, b)
    return g, prob, b


def time_solves(ctx, prob, H, b, traits, steps, warmup):
    import torch
    from geoflow_b200 import GCG
    cg = GCG(traits, prob)
    xb = prob.zeros()
    x = prob.zeros()
    for _ in range(warmup):
        x.zero_()
        rc = cg.solve(H, b, xb, x)
    torch.cuda.synchronize()
    times, iters = [], []
    for _ in range(steps):
        x.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        rc = cg.solve(H, b, xb, x)
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e) / 1e3)
        iters.append(cg.iter_)
    return times, iters, rc, x


def cold_solve(ctx, prob, H, b, traits):
    """Device time of a solve on a problem without a cached multigrid
    hierarchy: the set-up (levels, Jacobi diagonals, eigenvalue estimates)
    plus the solve."""
    import torch
    from geoflow_b200 import GCG
    cg = GCG(traits, prob)
    x = prob.zeros()
    xb = prob.zeros()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    cg.solve(H, b, xb, x)
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / 1e3


class L2Flush:
    """Between timed launches: write a buffer twice the L2 (126 MB), then
    read another of the same size, so the timed launch starts with a cold
    L2 that holds no dirty lines (the write alone would leave ~126 MB of
    dirty lines for the timed kernel to write back)."""

    def __init__(self, device):
        import torch
        self.w = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)
        self.r = torch.ones(2 * L2_BYTES // 4, dtype=torch.float32, device=device)

    def __call__(self, clean=True):
        self.w.zero_()
        if clean:
            return self.r.sum()
        return None


def kernel_roofline(ctx, prob, peaks, reps=20):
    """Average duration of the fused 3-d Helmholtz applies on the headline
    grid, each launch timed alone after an L2 flush (L2Flush): FP32 in both
    line-contraction forms (FP32x2 FMA, 3xTF32 tensor cores) and FP64.
    `ms_dirty_flush` times the same launches after the write alone."""
    import torch
    from geoflow_b200 import _abi as A
    lib = A.load()
    flush = L2Flush(ctx.torch_device)
    res = {}
    g = prob.grid
    prev = lib.gf_set_fp32_apply(A.GF_FP32_APPLY_FMA)
    for name, dt, code, mode in (("f32", torch.float32, A.GF_F32, A.GF_FP32_APPLY_FMA),
                                 ("f32_tf32", torch.float32, A.GF_F32, A.GF_FP32_APPLY_TF32),
                                 ("f64", torch.float64, A.GF_F64, A.GF_FP32_APPLY_FMA)):
        lib.gf_set_fp32_apply(mode)
        u = torch.randn(prob.nlocal, dtype=dt, device=ctx.torch_device)
        uo = torch.empty_like(u)
        for _ in range(3):
            ctx.check(lib.gf_helmholtz_apply(prob.handle, code, 1.0, None, 1.0, None, 1, A.ptr(u),
                                             A.ptr(uo)))
        times = {}
        for clean in (True, False):
            ts = []
            for _ in range(reps):
                flush(clean)
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record()
                ctx.check(lib.gf_helmholtz_apply(prob.handle, code, 1.0, None, 1.0, None, 1,
                                                 A.ptr(u), A.ptr(uo)))
                e.record()
                torch.cuda.synchronize()
                ts.append(s.elapsed_time(e) / 1e3)
            times[clean] = statistics.mean(ts)
        t = times[True]
        s_ = 4 if dt == torch.float32 else 8
        alg = prob.nlocal * 2 * s_ + g.nelems * (3 + 1) * s_
        res[name] = {"ms": t * 1e3, "alg_bytes": alg, "gbs": alg / t / 1e9,
                     "gdofs": prob.nlocal / t / 1e9, "ms_dirty_flush": times[False] * 1e3}
    lib.gf_set_fp32_apply(prev)
    return res


def pmg_launches_per_iteration(m):
    """Launches of each finest-level kernel per multigrid-preconditioned CG
    iteration at smoothing degree m: m pre-smoothing steps, the residual,
    the first post-smoothing term and m more steps, each step after an
    apply; plus the outer FP64 apply."""
    return {"apply_fp64": 1, "apply_vcycle": 2 * m + 2, "smoother_step": 2 * m + 1,
            "residual": 1, "restrict": 1, "prolong": 1}


def pmg_kernel_roofline(ctx, prob, traits, peaks, reps=10):
    """The finest-level kernels of a multigrid-preconditioned solve (the
    instances the solve runs inside its graph), each launched alone through
    gf_pmg_launch after an L2 flush and timed with CUDA events on the
    context's stream: the outer FP64 lattice -> element apply, the V-cycle's
    lattice -> element apply, a smoother step pass and the residual pass.
    Algorithmic bytes per launch: apply = lattice in + element out +
    element geometry; step = q_E + b, dinv, x, d in + x, d out + the 1-byte
    lattice mask; residual = q_E + b in + res out + mask."""
    import ctypes as C
    import torch
    from geoflow_b200 import _abi as A
    lib = A.load()
    flush = L2Flush(ctx.torch_device)
    g = prob.grid
    tr = traits.to_c()
    ctx.check(lib.gf_pmg_launch(prob.handle, C.byref(tr), 1.0, 1.0, 1, 1, A.GF_PMG_PREPARE),
              "gf_pmg_launch")
    nL, nE, ne, dim = g.nclass, prob.nlocal, g.nelems, g.dim
    sm = 8 if traits.precond == A.GF_PRECOND_PMG64 else 4
    # the next level: order ceil(p/2) on the same elements (its lattice and
    # its element-local size)
    pc = (g.p + 1) // 2
    nLc = int(np.prod([g.ne[d] * pc + (0 if g.periodic[d] else 1) for d in range(dim)]))
    nEc = ne * (pc + 1) ** dim
    kinds = {
        "apply_fp64": (A.GF_PMG_APPLY64, nL * 8 + nE * 8 + ne * (dim + 1) * 8),
        "apply_vcycle": (A.GF_PMG_APPLY, nL * sm + nE * sm + ne * (dim + 1) * sm),
        "smoother_step": (A.GF_PMG_STEP, nE * sm + 6 * nL * sm + nL),
        "residual": (A.GF_PMG_RESID, nE * sm + 2 * nL * sm + nL),
        # fine residual in, coarse E-vector out; coarse x in, fine x updated
        "restrict": (A.GF_PMG_RESTRICT, nL * sm + nEc * sm),
        "prolong": (A.GF_PMG_PROLONG, nLc * sm + 2 * nL * sm),
    }
    hbm = peaks.get("hbm_gbs") or 6650.0
    out = {}
    for name, (which, alg) in kinds.items():
        for _ in range(3):
            ctx.check(lib.gf_pmg_launch(prob.handle, C.byref(tr), 1.0, 1.0, 1, 1, which),
                      "gf_pmg_launch")
        ts = []
        for _ in range(reps):
            flush(True)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            ctx.check(lib.gf_pmg_launch(prob.handle, C.byref(tr), 1.0, 1.0, 1, 1, which),
                      "gf_pmg_launch")
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
        t = statistics.mean(ts)
        out[name] = {"ms": t * 1e3, "alg_bytes": alg, "gbs": alg / t / 1e9,
                     "frac": alg / t / 1e9 / hbm}
    return out


def dss_timing(ctx, prob, reps=10):
    import torch
    from geoflow_b200 import _abi as A
    lib = A.load()
    out = {}
    for name, dt, code in (("f32", torch.float32, A.GF_F32), ("f64", torch.float64, A.GF_F64)):
        u = torch.randn(prob.nlocal, dtype=dt, device=ctx.torch_device)
        ctx.check(lib.gf_dss(prob.handle, code, A.GF_DSS_SUM, A.ptr(u)))
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            ctx.check(lib.gf_dss(prob.handle, code, A.GF_DSS_SUM, A.ptr(u)))
        e.record()
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3 / reps
        s_ = 4 if dt == torch.float32 else 8
        # box lattice (k_dss_box): every E-node read and written once, no
        # index arrays; CSR (k_dss_csr): plus members and class_ptr
        box = getattr(prob, "structured", True)
        alg = prob.nlocal * 2 * s_ + (0 if box else prob.nlocal * 4 + prob.grid.nclass * 4)
        out[name] = {"ms": t * 1e3, "alg_bytes": alg, "gbs": alg / t / 1e9,
                     "kernel": "k_dss_box" if box else "k_dss_csr"}
    return out


def e2e_solve(ctx, prob, H, b, traits, reps=2):
    """Solve through gf_cg_solve_host with pinned host buffers."""
    import ctypes as C
    import torch
    from geoflow_b200 import _abi as A
    lib = A.load()
    bh = b.cpu().pin_memory()
    xh = torch.zeros_like(bh).pin_memory()
    xbh = torch.zeros_like(bh).pin_memory()
    tr = traits.to_c()
    P = A.P_double
    times = []
    for i in range(reps + 1):
        xh.zero_()
        it, rn = C.c_int(), C.c_double()
        t0 = time.perf_counter()
        rc = lib.gf_cg_solve_host(prob.handle, C.byref(tr), 1.0, 1.0, 1,
                                  C.cast(bh.data_ptr(), P), C.cast(xbh.data_ptr(), P),
                                  C.cast(xh.data_ptr(), P), C.byref(it), C.byref(rn))
        t1 = time.perf_counter()
        ctx.check(rc, "gf_cg_solve_host")
        if i > 0:
            times.append(t1 - t0)
    n = prob.nlocal * 8
    return statistics.mean(times), 3 * n, n


# ---------------------------------------------------------------------------
def rk_stage_bench(ctx, ne, p, steps=3, warmup=2):
    """SSP-RK3 Burgers on a periodic box: GDOF/s per stage in FP32 and FP64,
    the stage split into its two kernels (the fused RHS k_dudt3d, timed
    alone through gf_dudt, and the rest of the stage: the stage update and
    Smooth pass; in FP32 the stage's RHS kernel carries the update as its
    epilogue, so there the RHS-alone figure is the kernel without it) with
    their GB/s, and the FP32 state's difference from the FP64 state after
    the same steps."""
    import torch
    from geoflow_b200 import GBurgers, GridBox, Problem, workloads as W
    from geoflow_b200 import _abi as A
    g = GridBox(3, [ne] * 3, p, length=[2 * np.pi] * 3, periodic=[1, 1, 1])
    prob = Problem(ctx, g, dirichlet_mask=False)
    dev = ctx.torch_device
    xyz = [torch.from_numpy(c).to(dev) for c in g.xyz]
    u = W.burgers_velocity(xyz, W.burgers_modes(), xp=torch)
    del xyz
    umax = max(float(t.abs().max()) for t in u)
    dt_cfl = W.burgers_dt(umax, ne, p, g.xi)
    n = prob.nlocal
    out = {"workload": f"3d Burgers, periodic {ne}^3 elements p={p}, SSP-RK3, nu=1e-3",
           "n_local": n, "dt": dt_cfl, "steps_timed": steps}
    final = {}
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, dtp in (("f32", torch.float32), ("f64", torch.float64)):
        sz = 4 if dtp == torch.float32 else 8
        uu = [t.to(dtp).contiguous() for t in u]
        B = GBurgers(prob, GBurgers.BURGERS, 1e-3, scheme=A.GF_SSP33)
        for _ in range(warmup):
            B.step(uu, None, dt=dt_cfl, nsteps=1)
        uu = [t.to(dtp).contiguous() for t in u]
        torch.cuda.synchronize()
        s.record()
        B.step(uu, None, dt=dt_cfl, nsteps=steps)
        e.record()
        torch.cuda.synchronize()
        t_stage = s.elapsed_time(e) / 1e3 / (3 * steps)
        final[name] = [t.double() for t in uu]
        # the RHS kernel alone (3 components in, 3 out, inverse mass)
        K = [torch.empty_like(t) for t in uu]
        B.dudt(uu, None, K)
        reps = 5
        torch.cuda.synchronize()
        s.record()
        for _ in range(reps):
            B.dudt(uu, None, K)
        e.record()
        torch.cuda.synchronize()
        t_rhs = s.elapsed_time(e) / 1e3 / reps
        t_upd = max(t_stage - t_rhs, 1e-9)
        rhs_bytes = n * sz * (3 + 3 + 1)
        # SSP33 stage update + Smooth: reads the RHS and one or two stage
        # vectors per component, writes the result (stage 1: 2 reads, 2-3: 3)
        upd_bytes = n * sz * 3 * (1 + (2 + 3 + 3) / 3.0)
        del K
        out[name] = {"ms_per_stage": t_stage * 1e3,
                     "gdofs_per_stage": 3 * n / t_stage / 1e9,
                     "stage_kernels": ("k_dudt3d with the SSP update epilogue, then the "
                                       "Smooth k_dss_smooth_box_n" if name == "f32" else
                                       "k_dudt3d, then the stage update and Smooth "
                                       "k_dss_rk_box_n"),
                     "kernels": {
                         "k_dudt3d": {"ms": t_rhs * 1e3, "alg_bytes": rhs_bytes,
                                      "gbs": rhs_bytes / t_rhs / 1e9},
                         "k_dss_rk_box_n (stage - rhs)": {"ms": t_upd * 1e3,
                                                          "alg_bytes": upd_bytes,
                                                          "gbs": upd_bytes / t_upd / 1e9}}}
        del uu
    d = max(float((a - b).abs().max()) for a, b in zip(final["f32"], final["f64"]))
    m = max(float(b.abs().max()) for b in final["f64"])
    out["f32_rel_diff_vs_f64"] = d / m
    prob.close()
    return out


# ---------------------------------------------------------------------------
def adjoint_bench(ctx, ne=16, p=6, nsteps=50, ck=10, reps=3):
    """Adjoint workload: gradient of J = 1/2 ||u(T) - u_obs||_M^2 with
    respect to u(0) through 50 RK4 steps of 3d Burgers (16^3 elements,
    p = 6, FP64), checkpoint every 10 steps, against the forward run alone."""
    import torch
    from geoflow_b200 import GBurgers, GridBox, Problem
    from geoflow_b200 import _abi as A
    g = GridBox(3, [ne] * 3, p, periodic=[1, 1, 1])
    prob = Problem(ctx, g, dirichlet_mask=False)
    dev = ctx.torch_device
    rng = np.random.default_rng(SEED + 4)
    first = g.members[g.class_ptr[:-1]][g.node_class]

    def fourier(amp):
        u = np.zeros(g.ndof())
        for _ in range(8):
            k = rng.integers(-4, 5, 3)
            u += rng.standard_normal() * np.cos(2 * np.pi * (k[0] * g.xyz[0] + k[1] * g.xyz[1]
                                                             + k[2] * g.xyz[2])
                                                + rng.uniform(0, 2 * np.pi))
        u = u[first]
        return torch.from_numpy(amp * u / np.abs(u).max()).to(dev)

    dt, nu = 1e-3, 1e-3
    B = GBurgers(prob, GBurgers.BURGERS, nu, scheme=A.GF_RK4)
    u0 = [fourier(0.5) for _ in range(3)]
    obs = [a + fourier(0.1) for a in u0]
    B.step(obs, None, dt=dt, nsteps=nsteps)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reset=None):
        if reset:
            reset()
        fn()  # warm-up (allocates the work buffers once)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            if reset:
                reset()
            torch.cuda.synchronize()
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
        return statistics.median(ts)

    u = [a.clone() for a in u0]

    def reset():  # every timed forward run starts from u0 (50 steps, not 200)
        for a, b in zip(u, u0):
            a.copy_(b)

    t_fwd = timed(lambda: B.step(u, None, dt=dt, nsteps=nsteps), reset)
    t_adj = timed(lambda: B.adjoint_gradient(u0, None, obs, dt, nsteps, ck))
    prob.close()
    return {"workload": (f"3d Burgers, periodic {ne}^3 elements p={p}, RK4, {nsteps} steps, "
                         f"nu={nu:g}, dt={dt:g}, FP64, checkpoint every {ck}"),
            "n_local": prob.nlocal, "forward_s": t_fwd, "gradient_s": t_adj,
            "gradient_over_forward": t_adj / t_fwd}


# ---------------------------------------------------------------------------
def graph_bench(ctx, reps=3):
    """The small, launch-bound CPU-runnable case: 2-d periodic
    advection-diffusion on 16^2 elements p = 4 (c = (1, 0.5), nu = 0.01,
    dt = 1e-4, RK4, 200 steps) by direct calls vs one CUDA graph, each
    against the reference's own run of it."""
    import torch
    from geoflow_b200 import GBurgers, Graph, GridBox, Problem, workloads as W
    from geoflow_b200 import _abi as A
    dev = ctx.torch_device
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
        return statistics.median(ts)

    def box(ne, p, seed):
        g = GridBox(2, [ne, ne], p, periodic=[1, 1])
        prob = Problem(ctx, g, dirichlet_mask=False)
        u0 = W.advection2d_initial(g.xyz, g.node_class, g.nclass, seed=seed)
        u = [torch.from_numpy(u0).to(dev)]
        c = [torch.ones(g.ndof(), dtype=torch.float64, device=dev),
             torch.full((g.ndof(),), 0.5, dtype=torch.float64, device=dev)]
        return g, prob, GBurgers(prob, A.GF_EQN_ADVECT, 0.01, scheme=A.GF_RK4), u, c

    out = {}
    g, prob, B, u, c = box(16, 4, SEED + 1)
    u0 = u[0].clone()
    nsteps = 200
    t_direct = timed(lambda: B.step(u, c, dt=1e-4, nsteps=nsteps))
    u[0].copy_(u0)
    B.step(u, c, dt=1e-4, nsteps=nsteps)
    u_direct = u[0].cpu().numpy()
    G = B.capture(u, c, dt=1e-4, nsteps=nsteps)
    t_graph = timed(G.launch)
    u[0].copy_(u0)
    G.launch()
    torch.cuda.synchronize()
    u_graph = u[0].cpu().numpy()
    stages = 4 * nsteps
    # the reference's own run of this case (tests/golden/make_path_golden.py)
    ref = np.load(ROOT / "tests" / "golden" / "ref_path.npz")
    same_ic = bool(np.array_equal(ref["cfg1_u0"], u0.cpu().numpy()))
    r200 = ref["cfg1_u200"]
    out["config1"] = {
        "workload": "2d periodic advection-diffusion, 16^2 elements p=4, RK4, 200 steps, FP64",
        "n_local": prob.nlocal, "direct_s": t_direct, "graph_s": t_graph,
        "gdofs_per_stage_direct": prob.nlocal * stages / t_direct / 1e9,
        "gdofs_per_stage_graph": prob.nlocal * stages / t_graph / 1e9,
        "graph_nodes": G.nodes(),
        "rel_err_vs_reference": {
            "direct": float(np.max(np.abs(u_direct - r200)) / np.max(np.abs(r200))),
            "graph": float(np.max(np.abs(u_graph - r200)) / np.max(np.abs(r200))),
            "same_initial_state": same_ic}}
    G.close()
    return out


# ---------------------------------------------------------------------------
def ensemble_bench(ctx, steps=10, reps=3, members=16, max_level=5, fixed_shape=False):
    """The batched ensemble: (1) 16 icosahedral-sphere advection members
    (level 3..5, p 4..8, cosine bell with seeded centre, solid-body wind,
    RK4, dt at CFL 0.25) as one gf_ensemble, one persistent launch per stage,
    FP32, against the same members stepped one by one by gf_rk_advance
    (every member bit-identical), with the FP32-vs-FP64 difference; (2) 16
    2-d Dirichlet box Helmholtz solves (8^2..64^2 elements, p 3..8, seeded
    sinusoidal RHS, (M + K)x = b to 1e-10 relative EUC residual), one
    persistent launch per CG iteration (FP32 PCG, FP64 refinement), against
    the members solved one by one (gf_cg_solve, mixed and FP64), each
    member's FP64 residual recomputed by the FP64 apply.  Launch shapes
    from the autotuner (or, with fixed_shape, 512 threads and 2 blocks per SM,
    timed by the tuner without a search).  members / max_level shrink the
    ensemble for profiling runs."""
    import torch
    from geoflow_b200 import (CGTraits, Ensemble, GBurgers, GCG, GGFX, GHelmholtz, GMass,
                              GridBox, IcosGrid, Problem, workloads as W)
    from geoflow_b200 import _abi as A
    dev = ctx.torch_device
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, prep=None):
        ts = []
        for _ in range(reps):
            if prep:
                prep()
            torch.cuda.synchronize()
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e) / 1e3)
        return statistics.median(ts)

    out = {}
    # ---- (1) icosahedral advection members ----
    t0 = time.perf_counter()
    mem = []
    for level, p, lat0, lon0 in W.icos_members()[:members]:
        g = IcosGrid(min(level, max_level), p, ctx=ctx)
        prob = g.problem(ctx)
        u0 = W.icos_cosine_bell(g.xyz, lat0, lon0)
        c = W.icos_solid_body_wind(g.xyz)
        cmax = float(np.max(np.sqrt(sum(a * a for a in c))))
        mem.append((g, prob, u0, c, 0.25 * g.minnodedist / cmax))
    setup_s = time.perf_counter() - t0
    probs = [m[1] for m in mem]
    dts = [m[4] for m in mem]
    ndof = sum(p.nlocal for p in probs)

    def state(dtype):
        us = [torch.from_numpy(m[2]).to(dev, dtype) for m in mem]
        cs = [[torch.from_numpy(a).to(dev, dtype) for a in m[3]] for m in mem]
        return us, cs

    E = Ensemble(ctx, probs)
    us, cs = state(torch.float32)
    u0s = [u.clone() for u in us]

    def reset():
        for u, v in zip(us, u0s):
            u.copy_(v)

    E.advance(us, cs, dt=dts, nsteps=1)
    t1 = time.perf_counter()
    if fixed_shape:
        E.set_shape(512, 2, {n: (8 if n <= 7 else 16) for n in range(3, 11)}, dtype=torch.float32)
        E.tune(torch.float32, reps=-3)
    else:
        E.tune(torch.float32, reps=3)
    tune_s = time.perf_counter() - t1
    shape = E.shape(torch.float32)

    l0 = E.launches()
    t_ens = timed(lambda: E.advance(us, cs, dt=dts, nsteps=steps), reset)
    launches_per_run = (E.launches() - l0) // reps
    reset()
    E.advance(us, cs, dt=dts, nsteps=steps)
    got32 = [u.cpu().numpy() for u in us]
    Bs = [GBurgers(m[1], A.GF_EQN_ADVECT, 0.0, scheme=A.GF_RK4) for m in mem]

    def seq():
        for k, B in enumerate(Bs):
            B.step([us[k]], cs[k], dt=dts[k], nsteps=steps)

    t_seq = timed(seq, reset)
    reset()
    seq()
    same = sum(int(np.array_equal(got32[k], us[k].cpu().numpy())) for k in range(len(mem)))
    us64, cs64 = state(torch.float64)
    E.advance(us64, cs64, dt=dts, nsteps=steps)
    err32 = max(float(np.max(np.abs(got32[k] - us64[k].cpu().numpy())) /
                      np.max(np.abs(us64[k].cpu().numpy()))) for k in range(len(mem)))
    stages = 4 * steps
    # algorithmic bytes per node and stage (FP32): stage input u + the mean
    # 1.5 earlier slopes, 3 velocity, 6 dXi/dX, 3 metric, Jac, inverse mass
    # read and the slope written by the element phase; the fold reads and
    # writes the slope and the output state (8 words)
    alg_b = 4 * (1 + 1.5 + 3 + 6 + 3 + 1 + 1 + 1 + 4)
    out["icos_advection"] = {
        "workload": ("16 icosahedral-sphere advection members (level 3..5, p 4..8, cosine bell, "
                     "solid-body wind), RK4, dt at CFL 0.25, FP32, %d steps" % steps),
        "members": [[m[0].level, m[0].p] for m in mem], "n_local_total": ndof,
        "setup_s": setup_s, "tune_s": tune_s, "shape": shape,
        "ensemble_s": t_ens, "sequential_s": t_seq, "speedup_vs_sequential": t_seq / t_ens,
        "gdofs_per_stage_ensemble": ndof * stages / t_ens / 1e9,
        "gdofs_per_stage_sequential": ndof * stages / t_seq / 1e9,
        "alg_bytes_per_node_stage": alg_b,
        "hbm_gbs_ensemble": ndof * stages * alg_b / t_ens / 1e9,
        "launches_per_run": launches_per_run,
        "members_bit_identical_to_single": f"{same}/{len(mem)}",
        "f32_rel_diff_vs_f64": err32}
    del E, us, cs, us64, cs64, u0s, Bs
    # ---- (2) box Helmholtz members ----
    bm = []
    for k, (ne, p) in enumerate(W.box_members()[:members]):
        g = GridBox(2, [ne, ne], p)
        prob = Problem(ctx, g)
        f = torch.from_numpy(W.helmholtz2d_rhs(g.xyz, seed=SEED + 20 + k)).to(dev)
        b = prob.zeros()
        GMass(prob).opVec_prod(f, None, b)
        bm.append((g, prob, b))
    E2 = Ensemble(ctx, [m[1] for m in bm])
    bs = [m[2] for m in bm]
    xs = [torch.zeros_like(b) for b in bs]

    def zero():
        for x in xs:
            x.zero_()

    def traits(**kw):
        t = CGTraits()
        t.maxit, t.normtype, t.tol, t.relative = 50000, A.GF_NORM_EUC, 1e-10, 1
        t.precond, t.precision, t.check_every = A.GF_PRECOND_JACOBI, A.GF_CG_MIXED, 16
        for k, v in kw.items():
            setattr(t, k, v)
        return t

    def fp64_residual():
        """each member's mask*DSS_Sum(b - A x) relative to b (EUC), FP64 apply"""
        worst = 0.0
        for (g, prob, b), x in zip(bm, xs):
            H = GHelmholtz(prob)
            H.set_Lap_scalar(1.0)
            H.set_mass_scalar(1.0)
            r = prob.zeros()
            H.opVec_prod(x, None, r)
            r = b - r
            GGFX(prob).doOp(r, GGFX.Sum)
            r *= torch.from_numpy(g.mask).to(dev)
            worst = max(worst, float(torch.sqrt((r * r).mean()) / torch.sqrt((b * b).mean())))
        return worst

    E2.solve(bs, xs, traits(precision=A.GF_CG_FP64))
    t1 = time.perf_counter()
    if fixed_shape:
        E2.set_shape(512, 2)
        E2.tune(reps=-3)
    else:
        E2.tune(reps=3)
    tune2_s = time.perf_counter() - t1
    modes = {"mixed": {"inner_tol": 1e-4}, "fp64": {"precision": A.GF_CG_FP64}}
    runs = {}
    for name, kw in modes.items():
        tr = traits(**kw)
        zero()
        E2.solve(bs, xs, tr)
        l0 = E2.launches()
        t_m = timed(lambda: E2.solve(bs, xs, tr), zero)
        nl = (E2.launches() - l0) // reps
        zero()
        rc, its, nrm, st = E2.solve(bs, xs, tr)
        runs[name] = {"s": t_m, "iterations": [int(i) for i in its], "rc": int(rc),
                      "statuses": [int(v) for v in st], "launches_per_solve": nl,
                      "member_iterations_per_s": float(sum(its)) / t_m,
                      "max_rel_fp64_residual": fp64_residual(),
                      "x": [x.clone() for x in xs]}
    seqs = {}
    xseq = [torch.zeros_like(b) for b in bs]
    diff = 0.0
    for name, prec, ce in (("mixed", A.GF_CG_MIXED, 16), ("fp64", A.GF_CG_FP64, 32)):
        t2 = CGTraits()
        t2.maxit, t2.normtype, t2.tol, t2.relative = 50000, A.GF_NORM_EUC, 1e-10, 1
        t2.precond, t2.precision, t2.check_every = A.GF_PRECOND_JACOBI, prec, ce
        solvers = []
        for g, prob, b in bm:
            H = GHelmholtz(prob)
            H.set_Lap_scalar(1.0)
            H.set_mass_scalar(1.0)
            solvers.append((GCG(t2, prob), H))

        zb = [torch.zeros_like(b) for b in bs]

        def run():  # solve_impl (2), xb = 0: the masked (Dirichlet) solve
            for (cg, H), b, xb, x in zip(solvers, bs, zb, xseq):
                cg.solve(H, b, xb, x)

        seqs[name] = timed(run, lambda: [x.zero_() for x in xseq])
        if name == "fp64":
            for x in xseq:
                x.zero_()
            run()
    for r in runs.values():
        r["max_rel_diff_vs_sequential_fp64"] = max(
            float((a - c).abs().max() / c.abs().max()) for a, c in zip(r.pop("x"), xseq))
    nL = sum(m[1].nlocal for m in bm)
    head = min(runs.values(), key=lambda r: r["s"] if r["rc"] == 0 else float("inf"))
    head_name = [k for k, v in runs.items() if v is head][0]
    out["box_helmholtz"] = {
        "workload": ("16 2d Dirichlet box Helmholtz solves (M+K)x=b (8^2..64^2 elements, "
                     "p 3..8), Jacobi PCG to 1e-10 relative EUC residual"),
        "members": [[m[0].ne[0], m[0].p] for m in bm], "n_local_total": nL,
        "tune_s": tune2_s, "shape": E2.shape(),
        "ensemble_s": head["s"], "scheme": head_name,
        "modes": runs,
        "sequential_mixed_s": seqs["mixed"], "sequential_fp64_s": seqs["fp64"],
        "speedup_mixed_ensemble_vs_sequential_mixed": seqs["mixed"] / runs["mixed"]["s"],
        "speedup_fp64_ensemble_vs_sequential_fp64": seqs["fp64"] / runs["fp64"]["s"],
        "speedup_vs_fastest_sequential": min(seqs.values()) / head["s"]}
    return out


# ---------------------------------------------------------------------------
def index_map_bench(ctx):
    """Gather-scatter class construction (GGFX::init's job) on the host and
    on the device: box lattice classes at 32^3 p=7 and coordinate matching
    at 16^3 and 32^3 p=7 (16.8 M nodes; the host matching is timed at 16^3)."""
    import ctypes as C
    import torch
    from geoflow_b200 import GridBox, _abi as A
    lib = A.load()
    out = {}

    def dev_time(fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()  # warm-up (allocations, module load)
        torch.cuda.synchronize()
        s.record()
        k = fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / 1e3, k

    ne3 = (C.c_int * 3)(32, 32, 32)
    per3 = (C.c_int * 3)(0, 0, 0)
    n = 32 ** 3 * 8 ** 3
    nc, cp, mem = np.zeros(n, np.int32), np.zeros(n + 1, np.int32), np.zeros(n, np.int32)
    t0 = time.perf_counter()
    k = lib.gf_box_classes(3, ne3, 7, per3, A.ptr(nc), A.ptr(cp), A.ptr(mem))
    th = time.perf_counter() - t0
    dn = torch.zeros(n, dtype=torch.int32, device="cuda")
    dc = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    dm = torch.zeros(n, dtype=torch.int32, device="cuda")
    td, kd = dev_time(lambda: lib.gf_box_classes_device(
        ctx.handle, 3, ne3, 7, per3, C.c_void_p(dn.data_ptr()), C.c_void_p(dc.data_ptr()),
        C.c_void_p(dm.data_ptr())))
    same = kd == k and bool((dm.cpu().numpy() == mem).all())
    out["box_32cube_p7"] = {"nodes": n, "host_s": th, "device_s": td, "identical": same}
    for ne in (16, 32):
        g = GridBox(3, [ne] * 3, 7)
        N = g.ndof()
        tol = 0.25 * float(np.min(np.diff(g.xi))) * 0.5 / ne
        dx = [torch.from_numpy(a).cuda() for a in g.xyz]
        darr = (C.c_void_p * 3)(*[a.data_ptr() for a in dx])
        dn = torch.zeros(N, dtype=torch.int32, device="cuda")
        dc = torch.zeros(N + 1, dtype=torch.int32, device="cuda")
        dm = torch.zeros(N, dtype=torch.int32, device="cuda")
        td, kd = dev_time(lambda: lib.gf_classes_from_coords_device(
            ctx.handle, 3, N, darr, tol, C.c_void_p(dn.data_ptr()), C.c_void_p(dc.data_ptr()),
            C.c_void_p(dm.data_ptr())))
        rec = {"nodes": N, "device_s": td, "classes": int(kd)}
        if ne == 16:
            nc, cp, mem = np.zeros(N, np.int32), np.zeros(N + 1, np.int32), np.zeros(N, np.int32)
            arr = (A.P_double * 3)(*[A.ptr(a) for a in g.xyz])
            t0 = time.perf_counter()
            k = lib.gf_classes_from_coords(3, N, arr, tol, A.ptr(nc), A.ptr(cp), A.ptr(mem))
            rec["host_s"] = time.perf_counter() - t0
            rec["identical"] = kd == k and bool((dm.cpu().numpy() == mem).all())
        out[f"coords_{ne}cube_p7"] = rec
    return out


class CPUPort:
    """The oracle port of the reference's FP64 Jacobi-PCG (GCG::solve_impl
    with GHelmholtz::reg_prod and GGFX::doOp, bit-identical to the
    reference's own compiled code on the pinned cases) built with OpenMP,
    on every host core, on the headline problem itself: the same box, the
    same right-hand side b = M f and the same relative stop rule
    ||r||_EUC <= tol ||b||_EUC (an absolute tolerance of tol ||b||_EUC, since
    ||b||_EUC < 1 here).  Set-up (grid, classes, diagonal, b) is untimed."""

    def __init__(self, ne, p, tol):
        os.environ["GFO_OPENMP"] = "1"
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        from geoflow_b200 import workloads as W
        self.O = O
        self.cores = len(os.sched_getaffinity(0))
        t0 = time.perf_counter()
        g = self.g = O.OracleBox(3, [ne] * 3, p)
        k, a = W.helmholtz_rhs_modes()
        x, y, z = g.xyz
        f = np.zeros(g.N)
        for m in range(len(a)):
            f += a[m] * np.sin(np.pi * k[m, 0] * x) * np.sin(np.pi * k[m, 1] * y) * \
                np.sin(np.pi * k[m, 2] * z)
        self.b = g.mass * f
        self.q = np.ones(g.N)
        self.zb = np.zeros(g.N)
        self.dinv = 1.0 / g.helmholtz_diag(1.0, self.q)
        self.tol_abs = tol * float(np.sqrt(np.mean(self.b * self.b)))
        self.setup_s = time.perf_counter() - t0

    def iterations(self, n):
        """Seconds for n CG iterations (a tolerance no residual reaches)."""
        x = np.zeros(self.g.N)
        t0 = time.perf_counter()
        self.g.cg_solve(self.b, x, p=1.0, q_vec=self.q, xb=self.zb, maxit=n, tol=1e-300,
                        normtype=self.O.NORM_EUC, dinv=self.dinv)
        return time.perf_counter() - t0

    def solve(self, maxit=5000):
        """A complete solve to the stop rule: (seconds, iterations, rc)."""
        x = np.zeros(self.g.N)
        t0 = time.perf_counter()
        rc, it, _ = self.g.cg_solve(self.b, x, p=1.0, q_vec=self.q, xb=self.zb, maxit=maxit,
                                    tol=self.tol_abs, normtype=self.O.NORM_EUC, dinv=self.dinv)
        return time.perf_counter() - t0, it, rc


def run_reference(args, ws, rank):
    """The reference arm: the CPU port on every host core (rank 0 only).
    Each step is a bounded sample, SAMPLE_ITERS + 1 CG iterations on the full
    problem; after the timed steps one complete solve to the stop rule gives
    the port's own iteration count and the measured time to solution, which
    is `value` (the steps' per-iteration time x that count is reported next
    to it as a consistency check)."""
    if rank != 0:
        return
    SAMPLE_ITERS = 5
    port = CPUPort(args.ne, args.p, args.tol)
    port.iterations(1)
    for _ in range(args.warmup):
        port.iterations(SAMPLE_ITERS)
    steps = [port.iterations(SAMPLE_ITERS + 1) for _ in range(args.steps)]
    t_first = port.iterations(1)  # the set-up part of every call (residual, norms)
    per_iter = (statistics.mean(steps) - t_first) / SAMPLE_ITERS
    full_s, iters, rc = port.solve()
    value = full_s
    n_full = port.g.N
    cfg = {"workload": f"3d Helmholtz (M+K)u=f, unit cube {args.ne}^3 hex p={args.p}, Dirichlet, "
                       f"Jacobi-PCG to {args.tol:g} relative residual",
           "n_local": n_full, "l2": "CPU run"}
    sample = (f"each step {SAMPLE_ITERS + 1} FP64 Jacobi-PCG iterations of the OpenMP port of "
              f"GCG/GHelmholtz/GGFX on the full {args.ne}^3 p={args.p} problem ({n_full} nodes, "
              f"{port.cores} threads); value = one complete solve to the stop rule, measured "
              f"({iters} iterations, rc {rc}); per-iteration time of the steps x {iters} = "
              f"{per_iter * iters:.2f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(steps) * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg, "seconds_per_cg_iteration": per_iter, "iterations": iters,
            "projected_from_steps_s": per_iter * iters, "setup_s": port.setup_s,
            "cpu_baseline": {"value": value, "unit": "s", "cores": port.cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(p, fp64_iters, sample_ne=16, sample_iters=10):
    """The GPU arm's cpu_baseline: the OpenMP port (see CPUPort) timed on a
    bounded sample, sample_iters iterations on a sample_ne^3-element box at
    the same p, per node, scaled to the full problem and to the iteration
    count of the same algorithm on it (the device FP64 Jacobi-PCG's count;
    the reference arm measures the port's own count on the full problem)."""
    port = CPUPort(sample_ne, p, 1e-10)
    port.iterations(1)
    t = port.iterations(sample_iters + 1) - port.iterations(1)
    per_node_iter = t / sample_iters / port.g.N
    return per_node_iter, port.cores, port.g.N


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch
    import torch.distributed as dist
    from geoflow_b200 import CGTraits, Context, GHelmholtz
    from geoflow_b200 import _abi as A
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    ctx = Context(local)
    peaks = measured_peaks()
    g, prob, b = make_helmholtz_problem(ctx, args.ne, args.p)
    H = GHelmholtz(prob)
    H.set_Lap_scalar(1.0)
    H.set_mass_scalar(1.0)
    common = dict(maxit=50000, normtype=A.GF_NORM_EUC, tol=args.tol, precond=A.GF_PRECOND_JACOBI,
                  relative=1)
    # mixed: FP64 residual replacement every args.ru FP32 iterations
    mix_kw = {} if args.inner is None else {"inner_tol": args.inner}
    tr_mix = CGTraits(precision=A.GF_CG_MIXED, check_every=args.ru, mixed_apply=args.mixed_apply,
                      **mix_kw, **common)
    tr_64 = CGTraits(precision=A.GF_CG_FP64, check_every=32, **common)
    # FP64 flexible CG with the FP32 Chebyshev polynomial preconditioner
    tr_cheb = CGTraits(precision=A.GF_CG_MIXED, check_every=4, poly_degree=args.poly,
                       poly_ratio=args.poly_ratio,
                       **dict(common, precond=A.GF_PRECOND_CHEBYSHEV))
    # FP64 flexible CG with one FP32 p/h-multigrid V-cycle as preconditioner
    tr_pmg = CGTraits(precision=A.GF_CG_MIXED, check_every=4, poly_degree=args.mg_degree,
                      poly_ratio=args.mg_ratio, **dict(common, precond=A.GF_PRECOND_PMG))
    # the same multigrid with an FP64 V-cycle: what the FP32 V-cycle saves
    tr_pmg64 = CGTraits(precision=A.GF_CG_FP64, check_every=4, poly_degree=args.mg_degree,
                        poly_ratio=args.mg_ratio, **dict(common, precond=A.GF_PRECOND_PMG64))
    if args.only == "rk":
        print(json.dumps({"only": "rk", "rk_stage": rk_stage_bench(ctx, args.rk_ne, args.rk_p,
                                                                  steps=args.steps,
                                                                  warmup=args.warmup)}), flush=True)
        return
    if args.only == "graphs":
        print(json.dumps({"only": "graphs", "graphs": graph_bench(ctx)}), flush=True)
        return
    if args.only == "ensemble":
        print(json.dumps({"only": "ensemble", "ensemble": ensemble_bench(
            ctx, steps=args.steps, members=args.ens_members, max_level=args.ens_max_level,
            fixed_shape=args.ens_fixed_shape)}), flush=True)
        return
    if args.only == "maps":
        print(json.dumps({"only": "maps", "index_maps": index_map_bench(ctx)}), flush=True)
        return
    if args.only == "adjoint":
        print(json.dumps({"only": "adjoint", "adjoint": adjoint_bench(ctx)}), flush=True)
        return
    if args.only == "apply":
        roof = kernel_roofline(ctx, prob, measured_peaks(), reps=args.steps)
        print(json.dumps({"only": "apply", "helm3d": roof}), flush=True)
        return
    if args.only == "pmgkern":
        out = {"fp32_vcycle": pmg_kernel_roofline(ctx, prob, tr_pmg, peaks, reps=args.steps),
               "fp64_vcycle": pmg_kernel_roofline(ctx, prob, tr_pmg64, peaks, reps=args.steps)}
        print(json.dumps({"only": "pmgkern", "pmg_finest_level": out}), flush=True)
        return
    if args.only:
        tr = {"fp64": tr_64, "mixed": tr_mix, "cheb": tr_cheb, "pmg": tr_pmg,
              "pmg64": tr_pmg64}[args.only]
        cold = cold_solve(ctx, prob, H, b, tr) if args.only in ("pmg", "pmg64") else None
        t, it, rc, x = time_solves(ctx, prob, H, b, tr, args.steps, args.warmup)
        out = {"only": args.only, "s_per_solve": statistics.mean(t), "iterations": it[-1],
               "rc": rc, "first_solve_s": cold}
        if args.only != "fp64":
            _, _, _, x64 = time_solves(ctx, prob, H, b, tr_64, 1, 0)
            out["rel_diff_vs_fp64"] = float((x - x64).abs().max() / x64.abs().max())
        print(json.dumps(out), flush=True)
        return

    def barrier():
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()

    def max_over_ranks(v):
        if ws == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=ctx.torch_device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up of both paths, then the timed region of the headline (mixed)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    l0 = C_stats(prob)
    t_64, it_64, rc_64, x_64 = time_solves(ctx, prob, H, b, tr_64, args.steps, args.warmup)
    l1 = C_stats(prob)
    t_mix, it_mix, rc_mix, x_mix = time_solves(ctx, prob, H, b, tr_mix, args.steps, args.warmup)
    l2 = C_stats(prob)
    # multigrid-preconditioned CG: the first solve builds the hierarchy
    # (timed apart as `first_solve_s`), the timed solves reuse it
    t_cold = cold_solve(ctx, prob, H, b, tr_pmg)
    l3 = C_stats(prob)
    t_pmg, it_pmg, rc_pmg, x_pmg = time_solves(ctx, prob, H, b, tr_pmg, args.steps, args.warmup)
    l4 = C_stats(prob)
    t_cold64 = cold_solve(ctx, prob, H, b, tr_pmg64)
    l5 = C_stats(prob)
    t_pmg64, it_pmg64, rc_pmg64, x_pmg64 = time_solves(ctx, prob, H, b, tr_pmg64, args.steps,
                                                       args.warmup)
    l6 = C_stats(prob)
    barrier()
    clk = clocks.stop()
    t64 = max_over_ranks(statistics.mean(t_64))
    tmix = max_over_ranks(statistics.mean(t_mix))
    tpmg = max_over_ranks(statistics.mean(t_pmg))
    tpmg64 = max_over_ranks(statistics.mean(t_pmg64))
    diff = float((x_mix - x_64).abs().max() / x_64.abs().max())
    diff_pmg = float((x_pmg - x_64).abs().max() / x_64.abs().max())
    diff_pmg64 = float((x_pmg64 - x_64).abs().max() / x_64.abs().max())
    # headline: the fastest complete solver (same problem, same 1e-10
    # relative-residual stop test on the FP64 residual)
    times = {"fp64": t64, "mixed": tmix, "pmg": tpmg, "pmg64": tpmg64}
    trs = {"fp64": tr_64, "mixed": tr_mix, "pmg": tr_pmg, "pmg64": tr_pmg64}
    path = min(times, key=times.get)
    fp64_wins = path in ("fp64", "pmg64")
    value = times[path]
    launches = {"fp64": l1 - l0, "mixed": l2 - l1, "pmg": l4 - l3, "pmg64": l6 - l5}[path]
    per_step_launches = launches // (args.steps + args.warmup)
    roof = kernel_roofline(ctx, prob, peaks)
    pmg_roof = {"fp32_vcycle": pmg_kernel_roofline(ctx, prob, tr_pmg, peaks),
                "fp64_vcycle": pmg_kernel_roofline(ctx, prob, tr_pmg64, peaks)}
    dss = dss_timing(ctx, prob)
    e2e_t, h2d, d2h = e2e_solve(ctx, prob, H, b, trs[path], reps=args.steps)
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    rk = adj = graphs = maps = ens = None
    if not args.no_rk:
        rk = rk_stage_bench(ctx, args.rk_ne, args.rk_p, steps=100)  # config 3's full 100 steps
        adj = adjoint_bench(ctx)
        graphs = graph_bench(ctx)
        maps = index_map_bench(ctx)
        ens = ensemble_bench(ctx)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        t_node, cores, nsample = cpu_baseline_sample(args.p, it_64[-1], args.cpu_sample_ne)
        t_cpu = t_node * prob.nlocal * it_64[-1]
        cpu = {"value": t_cpu, "unit": "s", "cores": cores, "kind": "port",
               "sample": (f"OpenMP port of GCG/GHelmholtz/GGFX ({cores} threads), 10 FP64 "
                          f"Jacobi-PCG iterations on a {args.cpu_sample_ne}^3-element p={args.p} "
                          f"box ({nsample} nodes), per node scaled to {prob.nlocal} nodes and "
                          f"{it_64[-1]} iterations (the device FP64 count of the same "
                          f"algorithm)")}
    if path in ("pmg", "pmg64"):
        # the multigrid solve's dominant kernel: per iteration its finest
        # level runs PMG_PER_ITER launches of each timed kernel; the most
        # device time goes to the Chebyshev smoother's step pass
        kk = pmg_roof["fp32_vcycle" if path == "pmg" else "fp64_vcycle"]
        per_iter = pmg_launches_per_iteration(args.mg_degree)
        share = {k: per_iter[k] * v["ms"] for k, v in kk.items()}
        top = max(share, key=share.get)
        head = kk[top]
        tname = "float" if path == "pmg" else "double"
        kname = {"smoother_step": f"k_mg_pass_lat<{args.p + 1},MG_STEP,{tname}> (finest-level "
                                  "Chebyshev smoother step: fold of q_E, residual, x and d update)",
                 "apply_vcycle": f"k_helm3d_k1<{tname},{args.p + 1},LoadBox> (finest-level "
                                 "apply, lattice in, element-local out)",
                 "residual": f"k_mg_pass_lat<{args.p + 1},MG_RESID,{tname}> (finest-level "
                             "residual pass)",
                 "apply_fp64": f"k_helm3d_k1<double,{args.p + 1},LoadBox> (outer FP64 apply)",
                 "restrict": f"k_pxfer_restrict<{args.p + 1},{tname}> (finest-level restriction)",
                 "prolong": f"k_pxfer_prolong<{args.p + 1},{tname}> (finest-level prolongation)",
                 }[top]
        prof = f"mg_pass_{top}_{'f32' if path == 'pmg' else 'f64'}_{args.ne}cube_p{args.p}"
    else:
        head = roof["f64" if fp64_wins else "f32"]
        kname = (f"k_helm3d_k1<{'double' if fp64_wins else 'float'},{args.p + 1}> "
                 "(3-d Helmholtz apply, element-local in/out)")
        prof = f"helm3d_k1_{'f64' if fp64_wins else 'f32'}_{args.ne}cube_p{args.p}"
    traffic = profile_traffic(prof)
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64_wins else "f32+f64",
        "data": "synthetic",
        "config": {"workload": (f"3d Helmholtz (M+K)u=f, unit cube {args.ne}^3 hex p={args.p}, "
                                f"Dirichlet, CG to {args.tol:g} relative residual"),
                   "path": path, "n_local": prob.nlocal, "n_unique": g.nclass,
                   "parallelism": f"replicas x{ws}",
                   "l2": ("inputs larger than L2 (16.8M-node vectors); the apply timings "
                          "write then read a 252 MB buffer before each launch (L2 cold, clean)")},
        "fp64_plain": {"value": t64, "unit": "s", "iterations": it_64[-1], "rc": rc_64},
        "mixed": {"value": tmix, "unit": "s", "iterations": it_mix[-1], "rc": rc_mix,
                  "scheme": "FP32 PCG with FP64 reliable updates"},
        "pmg": {"value": tpmg, "unit": "s", "iterations": it_pmg[-1], "rc": rc_pmg,
                "first_solve_s": t_cold,
                "scheme": (f"FP64 CG, preconditioner one FP32 p/h-multigrid V-cycle "
                           f"(Chebyshev-Jacobi degree {args.mg_degree}, dense coarsest solve); "
                           "hierarchy built by the first solve and reused")},
        "pmg_fp64": {"value": tpmg64, "unit": "s", "iterations": it_pmg64[-1], "rc": rc_pmg64,
                     "first_solve_s": t_cold64,
                     "scheme": ("the same FP64 CG and multigrid with every level of the "
                                "V-cycle in FP64")},
        "speedup_mixed_vs_fp64": t64 / tmix,
        "speedup_pmg_vs_fp64": t64 / tpmg,
        "speedup_pmg_fp64_vs_fp64": t64 / tpmg64,
        "speedup_fp32_vcycle_vs_fp64_vcycle": tpmg64 / tpmg,
        "solution_rel_diff_mixed_vs_fp64": diff,
        "solution_rel_diff_pmg_vs_fp64": diff_pmg,
        "solution_rel_diff_pmg_fp64_vs_fp64": diff_pmg64,
        "cg_iterations_per_s": {"fp64": it_64, "mixed": it_mix, "pmg": it_pmg,
                                "pmg64": it_pmg64}[path][-1] / value,
        "roofline": {"kernel": kname, "bound": "hbm", "achieved": head["gbs"], "peak": hbm,
                     "unit": "GB/s", "frac": head["gbs"] / hbm, "peak_source": peak_src,
                     "alg_bytes_per_launch": head["alg_bytes"], "ms_per_launch": head["ms"],
                     "traffic": traffic,
                     "traffic_source": f"profiles/{prof}.md" if traffic else None},
        "kernels": {"helm3d": roof, "dss_sum": dss, "pmg_finest_level": pmg_roof,
                    "pmg_launches_per_iteration": pmg_launches_per_iteration(args.mg_degree)},
        "rk_stage": rk,
        "adjoint": adj,
        "graphs": graphs,
        "ensemble": ens,
        "index_maps": maps,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_t, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": per_step_launches * args.steps,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def C_stats(prob):
    import ctypes as C
    from geoflow_b200 import _abi as A
    v = C.c_int64()
    A.load().gf_problem_stats(prob.handle, C.byref(v))
    return v.value


if __name__ == "__main__":
    main()
