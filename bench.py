"""Benchmark of the weakly-compressible SPH time step (libsph_b200).

Workload: the 2048 x 2048 Taylor-Green vortex (4,194,304 particles), MUSCL
linear-Riemann + delta-SPH + SPS solver, Wendland C2 (h = 1.3 dx), true 2x2
renormalisation, periodic images, RK4 with K1 reuse (3 RHS per step after the
first), particle shifting.  A "step" is one time step of that integrator over
all particles.  Synthetic data: the analytic Taylor-Green initial field on the
lattice jittered by a seeded uniform +/-0.1 dx (seed 1) -- the state on which
the mixed path meets the 1e-5 velocity bound; on the exact lattice the MUSCL
limiter sits on ties that round-off decides, and that lattice is timed as a
side report (lattice_exact).

Headline value: particle-steps/s of the mixed-precision step (FP32 pair
arithmetic, compensated sums, FP64 state), inputs resident on the device,
device-timed with CUDA events on the library's stream; the FP64 step is
reported beside it.  e2e: the same step through the C-ABI with host buffers:
every step uploads x, v, rho (sph_update_state), advances (sph_step) and
downloads x, v, rho (sph_get_state).

Side reports in the same line (skipped with --skip-accuracy / --skip-adjoint):
accuracy (mixed vs FP64 velocity L2), adjoint and adjoint_moving_square
(cost against a forward step, central-difference checks), moving_square (the
D/100 moving square, mixed and FP64), plain_method (the 100 x 100 plain
delta-SPH Taylor-Green case to t = 0.5 against the analytic decay) and
output_streaming (snapshot overhead).

Multi-GPU: the path does not shard (one GPU holds all particles), so
--gpus N runs N independent replicas (weak scaling, no collective on the data
path); value = particles x steps of all ranks / max-over-ranks time.

--impl reference: the CPU restatement of the reference (oracle/, OpenMP over
particles) on the host cores, on bounded samples of the same workload (512^2
and 256^2 of the same jittered case, --steps steps each) and a serial leg.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sph-2d_b200"))

METRIC = "particle-steps/s at 4.2M TGV: mixed vs FP64 GPU at <=1e-5 L2; adjoint/fwd cost"
UNIT = "particle-steps/s"
N_SIDE = 2048
JITTER, JITTER_SEED = 0.1, 1
WORKLOAD = ("Taylor-Green vortex 2048x2048 (4,194,304 particles) on the lattice jittered +-0.1dx (seed 1), "
            "MUSCL linear-Riemann + delta-SPH + SPS, Wendland C2 h=1.3dx, rho0=1, c0=10, Re=100, "
            "RK4 with K1 reuse (3 RHS/step), shifting, periodic images")


def bench_config(n_side: int, world: int) -> dict:
    """The `config` object of both arms (the native step and the CPU reference)."""
    import sph_b200 as S
    cfg = S.tgv_baseline_config(n_side, S.SOLVER_MUSCL_DELTA_SPS, S.PREC_MIXED)
    return {"workload": WORKLOAD, "particles": n_side * n_side, "rhs_per_step": 3, "dt": S.baseline_dt(cfg),
            "lattice": f"jittered +-{JITTER}dx, seed {JITTER_SEED}",
            "l2": "state (~1.4 GB) larger than L2 (126 MB), no flush needed",
            "parallelism": f"replicas x{world}"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--n-side", type=int, default=N_SIDE)
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_env():
    import replicas
    return replicas.dist_env()


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def roofline_traffic():
    """Measured DRAM bytes per particle of the pass-C kernel (ncu capture summarised
    in profiles/), or None when no capture has been committed."""
    path = os.path.join(ROOT, "profiles", "pass_c_dram_bytes_per_particle.txt")
    try:
        for line in open(path):
            line = line.strip()
            if line and not line.startswith("#"):
                return float(line.split()[0])
    except OSError:
        return None
    return None


def pass_c_instructions():
    """Measured warp instructions per slot of the pass-C kernel (ncu capture
    summarised in profiles/), or None."""
    path = os.path.join(ROOT, "profiles", "pass_c_warp_instructions_per_slot.txt")
    try:
        for line in open(path):
            line = line.strip()
            if line and not line.startswith("#"):
                return float(line.split()[0])
    except OSError:
        return None
    return None


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# Algorithmic bytes per particle of mixed pass C (the dominant kernel): its own
# records read once (hi/lo position 16 B, hi/lo kinematic record 32, aux 16,
# nb1..nb3 48, B^-1 16, flags 1) and its outputs written once (drhodt 4, acc 8,
# avg 8).  The mixed path forms the shifting sum in a separate gather
# (k_shift_gather, timed with the update).
PASS_C_BYTES_MIXED = 16 + 32 + 16 + 48 + 16 + 1 + 4 + 8 + 8
PASS_C_BYTES_FP64 = 16 + 32 + 32 + 96 + 32 + 1 + 8 + 16 + 16 + 16


def passes(tm, steps: int) -> dict:
    """Device time per step of each phase of the step (sph_timings)."""
    return {"images": tm.images_ms / steps, "sort_lists": tm.sort_ms / steps, "pass_a": tm.pass_a_ms / steps,
            "surface": tm.surface_ms / steps, "pass_c": tm.pass_c_ms / steps, "update": tm.update_ms / steps}


def run_native(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    import sph_b200 as S
    import build_lib as pkg_build
    if rank == 0:
        pkg_build.build()
    if world > 1:
        torch.distributed.barrier()
    S.load()

    import replicas

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, world, device=f"cuda:{local}")

    def barrier():
        replicas.barrier(world, sync=torch.cuda.synchronize)

    n_side = args.n_side
    results = {}
    clocks_info = None
    for prec in (S.PREC_MIXED, S.PREC_FP64):
        case = S.make_tgv(n_side, solver=S.SOLVER_MUSCL_DELTA_SPS, precision=prec, jitter=JITTER, seed=JITTER_SEED)
        dt = S.baseline_dt(case.cfg)
        sim = S.Simulation(case.cfg, case.n)
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        # the clock sampler starts before the warm-up so that it is running
        # (nvidia-smi needs a moment to start) when the timed region begins
        clk = Clocks(local) if prec == S.PREC_MIXED else None
        if clk:
            clk.start()
        sim.time_iteration(args.warmup, dt)           # includes the 4-RHS first step
        barrier()
        sim.reset_timings()
        barrier()
        t0 = time.perf_counter()
        diag = sim.time_iteration(args.steps, dt)
        tm = sim.timings()
        barrier()
        wall = time.perf_counter() - t0
        if clk:
            clocks_info = clk.stop()
        dev_ms = max_over_ranks(tm.total_ms)
        # the velocity of the state that was timed (warm-up + timed steps)
        vel_end = sim.get_state()[1] if rank == 0 else None
        results[prec] = dict(sim=sim, case=case, dt=dt, dev_ms=dev_ms, wall_s=wall, tm=tm, diag=diag, vel=vel_end)
        if prec == S.PREC_FP64:
            sim.close()

    mixed = results[S.PREC_MIXED]
    fp64 = results[S.PREC_FP64]
    n = mixed["case"].n
    steps = args.steps
    value = replicas.aggregate_rate(n * steps, world, mixed["dev_ms"] / 1e3)
    value64 = replicas.aggregate_rate(n * steps, world, fp64["dev_ms"] / 1e3)
    tm = mixed["tm"]

    # ---- e2e through the C-ABI with pinned host buffers ---------------------
    sim = mixed["sim"]
    pos_h = torch.empty(2 * n, dtype=torch.float64).pin_memory().numpy()
    vel_h = torch.empty(2 * n, dtype=torch.float64).pin_memory().numpy()
    rho_h = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    lib = S.load()
    dp = ctypes.POINTER(ctypes.c_double)
    P = lambda a: a.ctypes.data_as(dp)  # noqa: E731
    rc = lib.sph_get_state(sim.h, n, P(pos_h), P(vel_h), P(rho_h), None)
    assert rc == 0
    e2e_steps = max(2, min(steps, 10))
    diag = S.SphDiag()
    barrier()
    t0 = time.perf_counter()
    launches0 = sim.timings().kernel_launches
    for _ in range(e2e_steps):
        assert lib.sph_update_state(sim.h, n, P(pos_h), P(vel_h), P(rho_h)) == 0
        assert lib.sph_step(sim.h, 1, ctypes.c_double(mixed["dt"]), ctypes.byref(diag)) == 0
        assert lib.sph_get_state(sim.h, n, P(pos_h), P(vel_h), P(rho_h), None) == 0
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = replicas.aggregate_rate(n * e2e_steps, world, e2e_s)
    h2d = 40 * n
    d2h = 40 * n

    # ---- output streaming: snapshots overlapped with the steps (rank 0) -------
    streaming = None
    if rank == 0 and not args.skip_accuracy:
        streaming = streaming_report(S, sim, n, mixed["dt"])

    # ---- accuracy: mixed vs FP64 on the timed state -----------------------------
    accuracy = None
    if rank == 0:
        vm, vd = mixed["vel"], fp64["vel"]
        accuracy = {"timed_state": {
            "velocity_l2_mixed_vs_fp64": float(np.linalg.norm(vm - vd) / np.linalg.norm(vd)),
            "steps": args.warmup + steps,
            "case": "the timed runs themselves: the same jittered initial state, warm-up + timed steps"}}
    if not args.skip_accuracy and rank == 0:
        # the same initial state over 100 steps (the horizon of the 1e-5 bound);
        # on the exact lattice the MUSCL limiter sits on ties that round-off
        # decides, and FP64 runs one ulp apart already differ by 2.5e-4 there
        acc_steps = 100
        v = {}
        for prec in (S.PREC_FP64, S.PREC_MIXED):
            c = S.make_tgv(n_side, solver=S.SOLVER_MUSCL_DELTA_SPS, precision=prec, jitter=JITTER, seed=JITTER_SEED)
            with S.Simulation(c.cfg, c.n) as s2:
                s2.set_state(c.pos, c.vel, c.rho, c.mass, c.type)
                s2.time_iteration(acc_steps, S.baseline_dt(c.cfg))
                v[prec] = s2.get_state()[1]
        l2 = float(np.linalg.norm(v[S.PREC_MIXED] - v[S.PREC_FP64]) / np.linalg.norm(v[S.PREC_FP64]))
        accuracy.update({"velocity_l2_mixed_vs_fp64": l2, "steps": acc_steps,
                         "case": f"TGV {n_side}x{n_side}, the timed initial state (lattice jittered "
                                 f"+-{JITTER}dx, seed {JITTER_SEED}), same solver"})

    # ---- roofline of the dominant kernel (pass C) ----------------------------
    pk, pk_kind = peaks()
    passc_ms = tm.pass_c_ms / max(tm.rhs_evaluations, 1)
    n_tot = n + mixed["diag"].n_images
    alg = PASS_C_BYTES_MIXED * n_tot
    achieved = alg / (passc_ms / 1e3) / 1e9
    tr = roofline_traffic()
    roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "traffic": (tr * n_tot if tr else None),
            "kernel": "k_pass_c<float,MUSCL>", "launch_ms": passc_ms, "algorithmic_bytes": alg,
            "peak_kind": pk_kind + " (burst copy)"}
    # pass C is bound by instruction issue, not bytes: the same launch against the
    # issue limit of 4 warp instructions per SM per clock (148 SMs, sampled clock)
    ipb = pass_c_instructions()
    if ipb:
        mhz = (clocks_info or {}).get("sm_mhz") or 1965.0
        issue_peak = 4.0 * 148 * mhz * 1e6
        issue_ach = ipb * n_tot / (passc_ms / 1e3)
        roof["issue"] = {"achieved": issue_ach, "peak": issue_peak, "unit": "warp-instructions/s",
                         "frac": issue_ach / issue_peak, "instructions_per_slot": ipb, "sm_mhz": mhz,
                         "source": "ncu smsp__inst_executed.sum per slot (profiles/) x slots / live launch time"}

    # ---- adjoint cost (rank 0) -------------------------------------------------
    adj = adj_ms = None
    if rank == 0 and not args.skip_adjoint:
        adj = adjoint_report(S)
        adj_ms = adjoint_ms_report(S)
    ms = plain = exact = None
    if rank == 0 and not args.skip_accuracy:
        exact = exact_lattice_report(S, n_side)
        ms = moving_square_report(S)
        plain = plain_method_report(S)

    # ---- CPU baseline (rank 0 only, N = 1) ----------------------------------
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_reference(steps=steps, warmup=1, sides=(256,), serial=True)

    mixed["sim"].close()
    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": mixed["dev_ms"] / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 pair arithmetic + f64 state (mixed)", "data": "synthetic",
        "config": bench_config(n_side, world),
        "images": int(mixed["diag"].n_images),
        "fp64": {"value": value64, "unit": UNIT, "ms_per_step": fp64["dev_ms"] / steps,
                 "passes_ms_per_step": passes(fp64["tm"], steps),
                 "mixed_over_fp64": value / value64},
        "accuracy": accuracy,
        "adjoint_over_forward": adj["adjoint_over_forward"] if adj else None,
        "adjoint": adj,
        "adjoint_moving_square": adj_ms,
        "moving_square": ms,
        "plain_method": plain,
        "lattice_exact": exact,
        "output_streaming": streaming,
        "passes_ms_per_step": passes(tm, steps),
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps, "api": "sph_update_state + sph_step(1) + sph_get_state, pinned host buffers"},
        "gpu_launches": int(tm.kernel_launches),
        "clocks": clocks_info,
        "wall_s_timed": mixed["wall_s"],
    }


ADJ_SIDE, ADJ_STEPS, ADJ_EVERY = 256, 500, 32


def adjoint_leg(S, precision, solver=None):
    """Cost of the discrete adjoint on the adjoint Taylor-Green case: 256 x 256
    particles, 500 steps, a checkpoint every 32 steps, loss = squared velocity
    misfit at the end against a target from a forward run whose initial
    velocity carries 8 seeded Fourier modes of amplitude 0.05 U0.  Solver:
    modified linear Riemann + delta-SPH + SPS (or the MUSCL linear Riemann
    solver), Wendland C2, renormalised, no
    shifting: with shifting this solver amplifies lattice-scale perturbations
    (the mixed and FP64 runs of the same start drift apart e-fold every few
    steps until they saturate), so over 500 steps the exact gradient is
    dominated by that growth and no difference check can confirm it; the
    shifting reverse is checked on short horizons by the tests.  Both calls
    return only when their device work is done, so the
    host clock around each is its cost; the device-event sums are beside it."""
    solver = S.SOLVER_MODLR_DELTA_SPS if solver is None else solver
    case = S.make_tgv(ADJ_SIDE, solver=solver, precision=precision)
    case.cfg.shifting = 0
    case.cfg.mls_order = 0      # density re-initialisation is outside the adjoint's scope
    dt = S.baseline_dt(case.cfg)
    dv = S.fourier_perturbation(case.pos, n_modes=8, amp=0.05, seed=2024)
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel + dv, case.rho, case.mass, case.type)
        sim.time_iteration(ADJ_STEPS, dt)
        target = sim.get_state()[1]
    out = {}
    with S.Simulation(case.cfg, case.n) as sim:
        for rep in range(2):         # the first round warms up allocations and module loading
            sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
            sim.reset_timings()
            t0 = time.perf_counter()
            sim.time_iteration(ADJ_STEPS, dt)
            t_fwd = time.perf_counter() - t0
            dev_fwd = sim.timings().total_ms
            sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
            sim.reset_timings()
            t0 = time.perf_counter()
            loss = sim.adjoint_forward(ADJ_STEPS, dt, checkpoint_every=ADJ_EVERY, target_vel=target)
            t_fck = time.perf_counter() - t0
            sim.reset_timings()
            t0 = time.perf_counter()
            g = sim.adjoint_backward(1.0)
            t_bwd = time.perf_counter() - t0
            tb = sim.timings()
        out = {"loss": loss, "forward_s": t_fwd, "forward_checkpointed_s": t_fck, "backward_s": t_bwd,
               "adjoint_over_forward": t_bwd / t_fwd,
               "forward_device_ms": dev_fwd, "backward_device_ms": tb.total_ms,
               "adjoint_over_forward_device": tb.total_ms / dev_fwd,
               "backward_reverse_kernels_ms": tb.adjoint_ms, "grad": g}
    return case, dt, target, out


ADJ_FD_DIRECTIONS = 16


def adjoint_report(S):
    """The adjoint leg in both precisions, checked by central differences of
    the FP64 forward along 16 seeded directions of the initial velocity
    (eps = 1e-6) and in the viscosity (relative step 1e-5; at 1e-4 the
    quotient's own truncation error is 1.6e-4).  The MUSCL solver's adjoint is
    timed on the same case without a difference check: its limiter switches
    branch (and its large-jump branch jumps in value) at slope-ratio
    thresholds, which the exact Taylor-Green lattice meets everywhere, so the
    500-step loss is a dense staircase whose difference quotient does not
    converge at any step; the tests check that adjoint on jittered lattices
    over short horizons."""
    _, _, _, m = adjoint_leg(S, S.PREC_MIXED)
    # the differences use the FP64 leg's own target (the mixed forward's target
    # differs from it by the mixed path's error)
    case, dt, target, d = adjoint_leg(S, S.PREC_FP64)

    def loss_at(vel, cfg=None):
        with S.Simulation(case.cfg if cfg is None else cfg, case.n) as sim:
            sim.set_state(case.pos, vel, case.rho, case.mass, case.type)
            return sim.adjoint_forward(ADJ_STEPS, dt, checkpoint_every=ADJ_STEPS, target_vel=target)

    t0 = time.perf_counter()
    fd_err = []
    for k in range(ADJ_FD_DIRECTIONS):
        dirv = np.random.default_rng(300 + k).standard_normal(2 * case.n)
        eps = 1e-6
        fd = (loss_at(case.vel + eps * dirv) - loss_at(case.vel - eps * dirv)) / (2 * eps)
        fd_err.append(abs(float(d["grad"]["vel0"] @ dirv) - fd) / abs(fd))
    nu, e = case.cfg.nu, 1e-5 * case.cfg.nu
    ls = []
    for sgn in (1.0, -1.0):
        c = case.cfg.copy()
        c.nu = nu + sgn * e
        ls.append(loss_at(case.vel, c))
    fd_nu = (ls[0] - ls[1]) / (2 * e)
    t_fd = time.perf_counter() - t0
    _, _, _, mm = adjoint_leg(S, S.PREC_MIXED, S.SOLVER_MUSCL_DELTA_SPS)
    _, _, _, md = adjoint_leg(S, S.PREC_FP64, S.SOLVER_MUSCL_DELTA_SPS)
    gm, g64 = m["grad"]["vel0"], d["grad"]["vel0"]
    keep = ("loss", "forward_s", "forward_checkpointed_s", "backward_s", "adjoint_over_forward",
            "forward_device_ms", "backward_device_ms", "adjoint_over_forward_device", "backward_reverse_kernels_ms")
    return {
        "case": f"TGV {ADJ_SIDE}x{ADJ_SIDE} ({case.n} particles), {ADJ_STEPS} steps, checkpoint every {ADJ_EVERY}, "
                "velocity-misfit loss vs a target from 8 seeded Fourier modes (0.05 U0); modified linear Riemann "
                "+ delta-SPH + SPS, Wendland C2, renormalised, no shifting",
        "mixed": {k: m[k] for k in keep}, "fp64": {k: d[k] for k in keep},
        "adjoint_over_forward": m["adjoint_over_forward"],
        "grad_vel0_l2_mixed_vs_fp64": float(np.linalg.norm(gm - g64) / np.linalg.norm(g64)),
        "dnu_mixed": m["grad"]["nu"], "dnu_fp64": d["grad"]["nu"],
        "fd_rel_err_fp64": fd_err, "fd_rel_err_fp64_max": max(fd_err),
        "fd_nu_rel_err_fp64": abs(d["grad"]["nu"] - fd_nu) / abs(fd_nu),
        "fd": f"central differences of the FP64 forward: {ADJ_FD_DIRECTIONS} seeded initial-velocity directions "
              f"(eps=1e-6) and the viscosity (step 1e-5 nu); {t_fd:.1f} s",
        "muscl": {"mixed": {k: mm[k] for k in keep}, "fp64": {k: md[k] for k in keep},
                  "adjoint_over_forward": mm["adjoint_over_forward"],
                  "note": "same case with the MUSCL linear Riemann solver; cost only (the limiter's branch "
                          "switches make long-horizon difference quotients meaningless; checked in the tests)"},
    }


def streaming_report(S, sim, n, dt, chunks: int = 4, every: int = 5):
    """Output every `every` steps on the benchmark state: wall time per step of
    the same step calls with no output, with sph_snapshot_begin into page-locked
    buffers before each chunk (the transfer of x, v, rho, p runs on the copy
    stream while the next steps compute), and with a synchronous sph_get_state
    before each chunk."""
    import torch
    bufs = [torch.empty(m * n, dtype=torch.float64).pin_memory().numpy() for m in (2, 2, 1, 1)]
    res = {}
    for mode in ("none", "snapshot", "get_state"):
        sim.time_iteration(1, dt)
        t0 = time.perf_counter()
        for _ in range(chunks):
            if mode == "snapshot":
                sim.snapshot_begin(*bufs)
            elif mode == "get_state":
                sim.get_state()
            sim.time_iteration(every, dt)
        sim.snapshot_wait()
        res[mode] = (time.perf_counter() - t0) * 1e3 / (chunks * every)
    return {"ms_per_step": res, "every": every, "bytes_per_snapshot": 48 * n,
            "snapshot_overhead_pct": 100.0 * (res["snapshot"] / res["none"] - 1.0),
            "get_state_overhead_pct": 100.0 * (res["get_state"] / res["none"] - 1.0),
            "note": "wall clock, mixed 2048^2 step; sph_step calls of `every` steps each"}


MS_DX, MS_STEPS, MS_EVERY, MS_FD_STEPS, MS_FD_STEPS_WENDLAND = 0.02, 2000, 64, 200, 1000
MS_COEFFS = (1.0, 0.2, -0.1, 0.05, 0.02)


def adjoint_ms_report(S):
    """Cost and check of the moving-square adjoint: square of side D = 1 in a
    [0,10] x [0,5] tank of still water, dx = D/50 (~125k particles with 4 ghost
    layers), Re = 100, modified linear Riemann + delta-SPH (the adjoint's
    moving-square solver), ghost assignment every RHS, Euler predictor-corrector,
    FP64; 2,000 steps with a checkpoint every 64.  Motion u(t) = a0 + sum_k a_k
    sin(2 pi k t / T) over the run time T; loss = time-averaged drag coefficient
    sum_s dt F_x / (T F0), F0 = rho0 U^2 D / 2.  Forward = time_iteration over
    the same number of steps with the body at its mean speed a0 (the same work
    per step: translation, ghost assignment, RHS, body force).  The
    gradient with respect to a0 and the four Fourier coefficients is checked by
    central differences on the
    first 200 steps of the same case, and on 1,000 steps of the case with the
    Wendland C2 kernel, whose gradient vanishes at its cut-off: the improved
    Gaussian's gradient does not
    vanish at its 3h cut-off, so the right-hand side jumps whenever a pair
    crosses the support, and over thousands of steps so many crossings move by
    a step inside any difference interval that the difference quotient no
    longer measures the derivative (the adjoint's is that of the taken pair
    sets)."""
    case, ity = S.make_moving_square(dx=MS_DX, lx=10.0, ly=5.0, D=1.0, U=1.0, solver=S.SOLVER_MS_MODLR_DELTA)
    cfg = case.cfg
    cfg.ghost_assign, cfg.shifting, cfg.mls_order = 1, 0, 0
    lab = S.moving_square_labels(case, ity)
    dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
    T = MS_STEPS * dt
    scale = 1.0 / (T * 0.5 * cfg.rho0 * 1.0 * 1.0)
    coeffs = np.array(MS_COEFFS)
    motion, jac = S.body_motion_schedule(coeffs, MS_STEPS, dt, period=T)

    def reset(sim):
        # sph_set_state clears the body marks, the wall labels and the time
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        sim.set_initial_type(ity)
        sim.set_boundary_labels(lab)
        sim.set_time(0.0)

    def new_sim():
        sim = S.Simulation(cfg, case.n)
        reset(sim)
        return sim

    def loss_of(mo, nsteps):
        with new_sim() as sim:
            return scale * sim.adjoint_forward(nsteps, dt, checkpoint_every=MS_EVERY, loss=S.LOSS_DRAG,
                                               body_motion=mo)

    out = {}
    with new_sim() as sim:
        for rep in range(2):          # the first round warms up allocations
            reset(sim)
            sim.set_body_motion((coeffs[0], 0.0))
            sim.reset_timings()
            t0 = time.perf_counter()
            sim.time_iteration(MS_STEPS, dt)
            t_fwd = time.perf_counter() - t0
            dev_fwd = sim.timings().total_ms
            reset(sim)
            t0 = time.perf_counter()
            L = sim.adjoint_forward(MS_STEPS, dt, checkpoint_every=MS_EVERY, loss=S.LOSS_DRAG, body_motion=motion)
            t_fck = time.perf_counter() - t0
            sim.reset_timings()
            t0 = time.perf_counter()
            g = sim.adjoint_backward(scale)
            gm = sim.adjoint_motion_gradient()
            t_bwd = time.perf_counter() - t0
            tb = sim.timings()
    gc = np.einsum("sq,sqk->k", gm, jac)
    # the check on the first MS_FD_STEPS steps (same schedule, same scale)
    nf = MS_FD_STEPS
    with new_sim() as sim:
        sim.adjoint_forward(nf, dt, checkpoint_every=MS_EVERY, loss=S.LOSS_DRAG, body_motion=motion[:nf])
        sim.adjoint_backward(scale)
        gcf = np.einsum("sq,sqk->k", sim.adjoint_motion_gradient(), jac[:nf])
    fd = []
    for k in range(len(coeffs)):
        # the improved Gaussian's RHS jumps where a pair crosses the 3h cut-off; at
        # 1e-7 on a0 the difference interval shifts one such crossing by a step
        # (2.8e-4 off), at 1e-8 none (8e-7; at 1e-9 rounding gives 1e-5)
        eps = 1e-8
        cp, cm = coeffs.copy(), coeffs.copy()
        cp[k] += eps
        cm[k] -= eps
        f = (loss_of(S.body_motion_schedule(cp, MS_STEPS, dt, period=T)[0][:nf], nf)
             - loss_of(S.body_motion_schedule(cm, MS_STEPS, dt, period=T)[0][:nf], nf)) / (2 * eps)
        fd.append({"coefficient": k, "adjoint": float(gcf[k]), "fd": f, "rel_err": abs(gcf[k] - f) / abs(f)})
    # half the run's length with the Wendland C2 kernel (h = 1.3 dx, support 2h): its
    # gradient is zero at the cut-off, so pairs crossing it put no jumps into the
    # right-hand side and the difference quotient keeps measuring the derivative
    cfg_w = cfg.copy()
    cfg_w.kernel_model, cfg_w.kernel_scale, cfg_w.h = S.KERNEL_WENDLAND2, 2.0, 1.3 * cfg.dx
    dt_w = 0.25 * cfg_w.h / np.sqrt(cfg_w.c0sq)
    nw = MS_FD_STEPS_WENDLAND
    mo_w, jac_w = S.body_motion_schedule(coeffs, MS_STEPS, dt_w, period=MS_STEPS * dt_w)
    scale_w = 1.0 / (MS_STEPS * dt_w * 0.5 * cfg.rho0)

    def loss_w(c):
        with S.Simulation(cfg_w, case.n) as sim:
            reset(sim)
            mo = S.body_motion_schedule(c, MS_STEPS, dt_w, period=MS_STEPS * dt_w)[0][:nw]
            return scale_w * sim.adjoint_forward(nw, dt_w, checkpoint_every=MS_EVERY, loss=S.LOSS_DRAG, body_motion=mo)

    with S.Simulation(cfg_w, case.n) as sim:
        reset(sim)
        sim.adjoint_forward(nw, dt_w, checkpoint_every=MS_EVERY, loss=S.LOSS_DRAG, body_motion=mo_w[:nw])
        sim.adjoint_backward(scale_w)
        gw = np.einsum("sq,sqk->k", sim.adjoint_motion_gradient(), jac_w[:nw])
    fd_w = []
    for k in (0, 2):
        eps = 1e-6
        cp, cm = coeffs.copy(), coeffs.copy()
        cp[k] += eps
        cm[k] -= eps
        f = (loss_w(cp) - loss_w(cm)) / (2 * eps)
        fd_w.append({"coefficient": k, "adjoint": float(gw[k]), "fd": f, "rel_err": abs(gw[k] - f) / abs(f)})
    return {
        "case": f"moving square D=1 in [0,10]x[0,5], dx=D/50 ({case.n} particles incl. ghosts), Re=100, "
                f"MS modified linear Riemann + delta-SPH, ghost assignment, Euler PC, FP64, {MS_STEPS} steps, "
                f"checkpoint every {MS_EVERY}, motion a0 + 4 Fourier coefficients {list(MS_COEFFS)}",
        "loss": "time-averaged drag coefficient", "mean_drag_coefficient": scale * L,
        "forward_s": t_fwd, "forward_checkpointed_s": t_fck, "backward_s": t_bwd,
        "adjoint_over_forward": t_bwd / t_fwd,
        "forward_particle_steps_per_s": case.n * MS_STEPS / t_fwd,
        "adjoint_particle_steps_per_s": case.n * MS_STEPS / t_bwd,
        "forward_device_ms": dev_fwd, "backward_device_ms": tb.total_ms,
        "adjoint_over_forward_device": tb.total_ms / dev_fwd, "backward_reverse_kernels_ms": tb.adjoint_ms,
        "dC_d_coeffs": [float(x) for x in gc], "dC_dnu": g["nu"], "fd": fd,
        "fd_note": f"central differences eps=1e-8 of the FP64 forward over the first {MS_FD_STEPS} steps",
        "fd_wendland": fd_w,
        "fd_wendland_note": (f"the same case with the Wendland C2 kernel (h = 1.3 dx), {MS_FD_STEPS_WENDLAND} steps, "
                             "central differences eps=1e-6 of coefficients 0 and 2"),
    }


def plain_method_report(S, t_end: float = 0.5):
    """The 100 x 100 Taylor-Green case of the plain method, as the reference runs it
    on its CPU: Solver_Normalized_Delta_SPH_SPS (normalised delta-SPH + SPS, no
    Riemann state), Wendland C2 h = 1.3 dx, rho0 = 1, U0 = 1, c0 = 10, Re = 100,
    Tait gamma 7, dt = 0.25 h / c0, shifting, RK4 with K1 reuse, to t = 0.5
    (1,539 steps), FP64 on the GPU.  Device-timed particle-steps/s and KE/KE0 at
    t = 0.5 against the analytic decay exp(-16 pi^2 nu t)."""
    case = S.make_tgv(100, solver=S.SOLVER_DELTA_SPS, precision=S.PREC_FP64)
    dt = S.baseline_dt(case.cfg)
    nsteps = int(round(t_end / dt))
    with S.Simulation(case.cfg, case.n) as sim:
        sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
        ke0 = sim.diagnostics().kinetic_energy
        sim.reset_timings()
        d = sim.time_iteration(nsteps, dt)
        tm = sim.timings()
    t = nsteps * dt
    ratio = d.kinetic_energy / ke0
    analytic = float(np.exp(-16 * np.pi ** 2 * case.cfg.nu * t))
    return {"case": "TGV 100x100, Solver_Normalized_Delta_SPH_SPS, Wendland C2, FP64, dt = 0.25 h/c0",
            "steps": nsteps, "t_end": t, "particle_steps_per_s": case.n * nsteps / (tm.total_ms / 1e3),
            "ms_per_step": tm.total_ms / nsteps, "ke_over_ke0": ratio, "ke_analytic": analytic,
            "ke_rel_err_vs_analytic": (ratio - analytic) / analytic}


def moving_square_report(S, steps: int = 200, warmup: int = 3):
    """The moving-square forward: square of side D = 1 in a [0,10] x [0,5] tank,
    dx = D/100 (about 500k fluid particles, 4 ghost layers), HLLC + delta-SPH,
    Re = 100, the square started impulsively at U = 1, ghost assignment and the
    body force every step, Euler predictor-corrector with shifting and MLS
    density re-initialisation every 40 steps (the shipped moving-square
    settings).  Mixed and FP64 from the same state: device-timed particle-steps/s,
    the velocity L2 difference after the run and the drag coefficient of the
    last step (F0 = rho0 U^2 D / 2)."""
    out = {}
    vel = {}
    for name, prec in (("mixed", S.PREC_MIXED), ("fp64", S.PREC_FP64)):
        case, ity = S.make_moving_square(dx=0.01, lx=10.0, ly=5.0, D=1.0, U=1.0, solver=S.SOLVER_MS_HLLC_DELTA,
                                         precision=prec)
        cfg = case.cfg
        cfg.ghost_assign = 1
        lab = S.moving_square_labels(case, ity)
        dt = 0.25 * cfg.h / np.sqrt(cfg.c0sq)
        with S.Simulation(cfg, case.n) as sim:
            sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
            sim.set_initial_type(ity)
            sim.set_boundary_labels(lab)
            sim.set_body_motion((1.0, 0.0))
            sim.set_time(0.0)
            sim.time_iteration(warmup, dt)
            sim.reset_timings()
            sim.time_iteration(steps // 2, dt)
            vel[name + "_half"] = sim.get_state()[1]
            d = sim.time_iteration(steps - steps // 2, dt)
            tm = sim.timings()
            vel[name] = sim.get_state()[1]
        out[name] = {"particle_steps_per_s": case.n * steps / (tm.total_ms / 1e3),
                     "ms_per_step": tm.total_ms / steps,
                     "drag_coefficient": d.body_force[4] / (0.5 * cfg.rho0)}
        n = case.n
    water = np.r_[case.type, case.type] == S.TYPE_WATER
    dv = vel["mixed"][water] - vel["fp64"][water]
    out["mixed_over_fp64"] = out["mixed"]["particle_steps_per_s"] / out["fp64"]["particle_steps_per_s"]
    out["velocity_l2_mixed_vs_fp64"] = float(np.linalg.norm(dv) / np.linalg.norm(vel["fp64"][water]))
    dvh = vel["mixed_half"][water] - vel["fp64_half"][water]
    out["velocity_l2_mixed_vs_fp64_half"] = float(np.linalg.norm(dvh) / np.linalg.norm(vel["fp64_half"][water]))
    out["velocity_l2_steps"] = [warmup + steps // 2, warmup + steps]
    out["case"] = (f"moving square D=1 in [0,10]x[0,5], dx=D/100 ({n} particles incl. ghosts), HLLC + delta-SPH, "
                   f"Re=100, impulsive U=1, ghost assignment, body force every step, Euler PC, shifting, MLS every "
                   f"40 steps; {steps} steps after {warmup}, device-timed")
    return out


def cpu_reference(steps: int, warmup: int, sides=(256,), serial: bool = True):
    """The oracle (CPU restatement of the reference) on bounded samples of the
    workload: the same solver, physics and jittered lattice at `sides` x `sides`
    particles (h = 1.3 dx at every size, so the work per particle is that of the
    2048^2 case), `steps` timed steps after `warmup` (at least the 4-RHS first
    step) with OpenMP over particles on all host threads, and a serial leg
    (1 thread, 128^2, a few steps).  The value is the rate of the largest sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_api as O
    import sph_b200 as S
    O.build()
    threads = O.threads(os.cpu_count() or 1)

    def leg(n_side, nsteps):
        case = S.make_tgv(n_side, solver=S.SOLVER_MUSCL_DELTA_SPS, jitter=JITTER, seed=JITTER_SEED)
        dt = S.baseline_dt(case.cfg)
        sim = O.OracleSim(case.cfg, case.pos, case.vel, case.rho, case.mass, case.type)
        sim.run(max(warmup, 1), dt)        # the first step has 4 RHS: keep it out of the timing
        t0 = time.perf_counter()
        sim.run(nsteps, dt)
        el = time.perf_counter() - t0
        return {"n_side": n_side, "particles": case.n, "steps": nsteps, "seconds": el,
                "particle_steps_per_s": case.n * nsteps / el}

    legs = [leg(ns, steps) for ns in sides]
    out = {"value": legs[-1]["particle_steps_per_s"], "unit": UNIT, "cores": threads, "kind": "port",
           "sample": (f"TGV {legs[-1]['n_side']}^2 ({legs[-1]['particles']} particles) on the jittered lattice "
                      f"(+-{JITTER}dx, seed {JITTER_SEED}), {steps} steps after {max(warmup, 1)} warm-up, same solver, "
                      f"FP64, {threads} OpenMP threads"),
           "seconds": legs[-1]["seconds"], "sizes": legs,
           "per_particle_note": "the rate per particle at each sample size in `sizes` (h = 1.3 dx everywhere)"}
    if serial:
        O.threads(1)
        try:
            out["serial"] = dict(leg(128, min(steps, 3)), cores=1)
        finally:
            O.threads(threads)
    return out


def exact_lattice_report(S, n_side: int, steps: int = 20, warmup: int = 3):
    """The same benchmark step on the exact (unjittered) lattice: device-timed
    particle-steps/s of the mixed and FP64 paths and their velocity difference
    after warm-up + timed steps (MUSCL limiter ties there are decided by
    round-off, so that difference is not bounded by 1e-5)."""
    out, vel = {}, {}
    for name, prec in (("mixed", S.PREC_MIXED), ("fp64", S.PREC_FP64)):
        case = S.make_tgv(n_side, solver=S.SOLVER_MUSCL_DELTA_SPS, precision=prec)
        dt = S.baseline_dt(case.cfg)
        with S.Simulation(case.cfg, case.n) as sim:
            sim.set_state(case.pos, case.vel, case.rho, case.mass, case.type)
            sim.time_iteration(warmup, dt)
            sim.reset_timings()
            sim.time_iteration(steps, dt)
            tm = sim.timings()
            vel[name] = sim.get_state()[1]
        out[name] = {"particle_steps_per_s": case.n * steps / (tm.total_ms / 1e3), "ms_per_step": tm.total_ms / steps}
    out["mixed_over_fp64"] = out["mixed"]["particle_steps_per_s"] / out["fp64"]["particle_steps_per_s"]
    out["velocity_l2_mixed_vs_fp64"] = float(np.linalg.norm(vel["mixed"] - vel["fp64"]) / np.linalg.norm(vel["fp64"]))
    out["case"] = f"TGV {n_side}x{n_side} exact lattice, same solver, {steps} steps after {warmup}, device-timed"
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return 0
        steps = max(1, args.steps)
        t0 = time.perf_counter()
        # bounded samples of the workload (512^2 gives the value, 256^2 shows the
        # rate per particle does not depend on the sample size) and a serial leg
        cpu = cpu_reference(steps=steps, warmup=1, sides=(256, 512), serial=True)
        el = time.perf_counter() - t0
        line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world, "steps": steps,
                "warmup": args.warmup, "ms_per_step": cpu["seconds"] / steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": bench_config(args.n_side, world),
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "wall_s": el}
        print(json.dumps(line))
        return 0
    import replicas
    if world > 1:
        import torch
        torch.cuda.set_device(local)
    replicas.init(world, "nccl")
    out = run_native(args, rank, world, local)
    replicas.shutdown(world)
    if rank == 0 and out is not None:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
