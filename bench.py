#!/usr/bin/env python
"""Benchmark of the PonD step on B200: D3Q27, 256^3 spherical Riemann problem.

Workload (the MLUPS metric's configuration): unit box at 256^3, inside r < 0.2
(rho = 1, p = 1), outside (rho = 0.125, p = 0.1), u = 0, lattice time step
dt/dx = 0.25 (so T_lattice = 0.0625 p/rho), tau = 0.52, cubic Lagrange
interpolation (the reference's propagate<4>), float32 populations with float64
moments and convergence test at |delta| < 1e-8 + 1e-6 |value|.  One "step" is
one PonD time step of the whole box.  The state (2.1 GB per buffer) is far
larger than L2, so no flush is needed between steps.  Before the warm-up,
--spinup steps (default 150, untimed) advance the blast until its shock has
crossed most of the box: right after the initial condition almost every node
sits in a uniform region and converges in one iteration, which is not
representative of the 1500-step run.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line.  With --gpus N > 1 (under torchrun) every rank advances
its own independent box (replicas: the step has no exchange on one GPU per
problem) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lbmpond_b200 import configs  # noqa: E402  (initial conditions; loads no library)

METRIC = "MLUPS D3Q27 256^3: learned-gauge vs plain PonD at equal L1 error vs FP64"
LAMBDA = 0.25            # dt/dx of the lattice
TAU = 0.52
TOL_ABS, TOL_REL = 1e-7, 1e-6  # float32 floor: 1e-8 sits below the accumulation noise at rho ~ 1
BYTES_PER_NODE = (27 + 5) * 4 * 2   # f, rho, u, T read once and written once (float32)
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 lanes x FMA at the max SM clock


def sphere_params():
    # cx, cy, cz, radius, rho_in, T_in, rho_out, T_out  (T = lambda^2 p/rho)
    return configs.sphere_params(LAMBDA)


def sphere_state(n):
    """The same initial condition on the host (for the oracle's sample)."""
    return configs.sphere_state(n, LAMBDA)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(n_gpus):
    from lbmpond_b200 import replicas
    return replicas.setup("nccl")


def barrier(pg):
    from lbmpond_b200 import replicas
    replicas.barrier(pg)


def allmax(pg, v):
    from lbmpond_b200 import replicas
    return replicas.max_over_ranks(pg, v)


# ------------------------------------------------------------------ CPU baseline (oracle)
def _oracle_sample(m, spin, warmup, steps):
    """The FP64 oracle (restated reference step, all host threads) on an m^3
    sample of the sphere problem: `spin` + `warmup` untimed steps (spin = the
    benchmark's spin-up scaled to the sample, so the blast has crossed the
    same fraction of the box), then `steps` timed steps."""
    from oracle import oracle as O
    O.build()
    rho, g = sphere_state(m)
    st = O.base_state(1, rho, *g)
    for _ in range(spin + warmup):
        st, _, _ = O.step(st, 1, (m, m, m), tau=TAU, tol_abs=TOL_ABS, tol_rel=TOL_REL)
    t0 = time.perf_counter()
    it = []
    for _ in range(steps):
        st, niter, _ = O.step(st, 1, (m, m, m), tau=TAU, tol_abs=TOL_ABS, tol_rel=TOL_REL)
        it.append(float(niter.mean()))
    dt = (time.perf_counter() - t0) / steps
    return m ** 3 / dt / 1e6, dt, float(np.mean(it)), O.max_threads()


SAMPLE = os.path.join(ROOT, "tests", "golden", "bench", "sphere256_blocks.npz")


def _oracle_blocks(warmup, steps):
    """The FP64 oracle (restated reference step, all host threads) on blocks
    cut out of the benchmark's own spun-up 256^3 state (tests/golden/bench,
    made by tests/golden/make_cpu_sample.py): every pass steps each block
    once from the stored state (zero-gradient block faces, the benchmark's
    tau and tolerance), so each timed pass does the per-node work of the
    timed GPU steps.  Returns (MLUPS, s per pass, iterations per node, the
    GPU's iterations on the same nodes, threads, description)."""
    from oracle import oracle as O
    O.build()
    z = np.load(SAMPLE)
    e = int(z["edge"])
    blocks = [O.State(z["f"][:, b].astype(np.float64), z["rho"][b].astype(np.float64),
                      z["g"][:, b].astype(np.float64)) for b in range(z["rho"].shape[0])]
    nodes = len(blocks) * e ** 3

    def one_pass():
        it = 0
        for st in blocks:
            _, niter, _ = O.step(st, 1, (e, e, e), tau=TAU, tol_abs=TOL_ABS, tol_rel=TOL_REL,
                                 bc=(O.BC_CLAMP,) * 3)
            it += int(niter.sum())
        return it / nodes

    for _ in range(warmup):
        one_pass()
    t0 = time.perf_counter()
    its = [one_pass() for _ in range(steps)]
    dt = (time.perf_counter() - t0) / max(steps, 1)
    desc = (f"{len(blocks)} blocks of {e}^3 nodes cut from the 256^3 state after {int(z['spinup'])} spin-up "
            f"steps (seeded positions; the GPU iterates {float(z['niter_gpu'].mean()):.2f} times per node on them, "
            f"{float(z['niter_mean_domain']):.2f} over the whole box), each block stepped once per pass with "
            f"zero-gradient faces")
    return nodes / dt / 1e6, dt, float(np.mean(its)), float(z["niter_gpu"].mean()), O.max_threads(), desc


def cpu_baseline(spinup=150, m=24):
    """FP64 oracle on a bounded sample of the same workload at the same stage
    of the run (about 10-30 s of host time): the blocks of the spun-up state
    when their file is present, else a coarse re-simulation."""
    if os.path.exists(SAMPLE):
        v, dt, it, it_gpu, cores, desc = _oracle_blocks(1, 3)
        return {"value": v, "unit": "MLUPS", "cores": cores, "kind": "port",
                "sample": f"{desc}; 3 timed passes of {dt:.2f} s on the FP64 oracle, {it:.2f} iterations per node",
                "niter_mean": it, "niter_mean_gpu_same_nodes": it_gpu}
    spin = round(spinup * m / 256)
    v, dt, it, cores = _oracle_sample(m, spin, 0, 2)
    return {"value": v, "unit": "MLUPS", "cores": cores, "kind": "port",
            "sample": f"{m}^3 sample of the sphere problem after {spin} spin-up steps (the 256^3 spin-up scaled), "
                      f"2 timed steps of {dt:.2f} s on the FP64 oracle, {it:.2f} iterations per node"}


# ------------------------------------------------------------------ reference kernels on the GPU
REF_TOL = (1e-12, 1e-10)  # isConv of the reference's build (steps.cu:62-63), both precisions
# (precision, grid, steps, timed steps): the reference's USE_DOUBLE build on the sphere
# problem at 64^3 from the initial condition through the benchmark's spin-up scaled to
# the grid (round(150 * 64 / 256) = 38 steps), timing the last two; its USE_FLOAT
# build at 32^3, one step from the initial condition (it never meets its tolerance in
# float32, so every node runs the 100-iteration cap whatever the state)
SAME_STATE = (("double", 64, 40, 2), ("float", 32, 1, 1))


def reference_cuda():
    """Reference arm: the reference's own PonDstep (built for sm_100a from its
    sources by oracle/build_ref.sh), kernel time by CUDA events, on the
    SAME_STATE runs; this library's arm times its kernels on the same runs."""
    from oracle import oracle as O
    from tests.golden.make_golden import read_niter_mean, read_state, write_state
    out = {}
    for prec, n, nsteps, timed in SAME_STATE:
        binary = os.path.join(ROOT, "oracle", "_ref", f"ref_pond_D3Q27_{prec}_{n}x{n}x{n}")
        if not os.path.exists(binary):
            out[prec] = None
            continue
        rho, g = sphere_state(n)
        f = O.tables(1).w[:, None] * rho[None, :]
        with tempfile.TemporaryDirectory() as td:
            fin, fout = os.path.join(td, "in"), os.path.join(td, "out")
            write_state(fin, f, rho, g, (n, n, n))
            r = subprocess.run([binary, fin, fout, str(nsteps), repr(TAU)], capture_output=True, text=True,
                               timeout=900)
            if r.returncode != 0:
                out[prec] = {"error": r.stderr[-300:]}
                continue
            _, _, _, nmax, ms = read_state(fout, 27, (n, n, n))
            im = read_niter_mean(fout, 27, (n, n, n))
        t = float(np.mean(ms[-timed:]))
        out[prec] = {"build": "USE_DOUBLE" if prec == "double" else "USE_FLOAT", "grid": f"{n}^3",
                     "steps": nsteps, "timed_steps": timed, "tolerance": list(REF_TOL), "ms_per_step": t,
                     "MLUPS": n ** 3 / t / 1e3, "niter_mean_last_step": im, "niter_max_last_step": nmax,
                     "node_iterations_per_s": n ** 3 * im / (t / 1e3) if im else None}
    return out


def ours_same_state(local=0):
    """This library's kernels on reference_cuda's runs: the same initial state
    and step counts, float64 at the reference's tolerance, float32 at the
    reference's tolerance and at the benchmark's."""
    import lbmpond_b200 as pond
    out = {}
    for prec, n, nsteps, timed in SAME_STATE:
        rho, g = sphere_state(n)
        runs = [("fp64", REF_TOL)] if prec == "double" else [("fp32", REF_TOL)]
        runs.append(("fp32", (TOL_ABS, TOL_REL)))
        rec = {"grid": f"{n}^3", "steps": nsteps, "timed_steps": timed}
        for p, tol in runs:
            with pond.Solver(lattice="D3Q27", shape=(n, n, n), interp=pond.LAGR4, precision=p, tau=TAU,
                             tol_abs=tol[0], tol_rel=tol[1], device=local) as s:
                s.set_state(rho, g)
                s.step(nsteps - timed)
                ms = []
                for _ in range(timed):
                    s.step(1)
                    ms.append(s.last_step_ms())
                d = s.diagnostics()
            t = float(np.mean(ms))
            key = p + ("_reference_tolerance" if tol == REF_TOL else "_bench_tolerance")
            rec[key] = {"tolerance": list(tol), "ms_per_step": t, "MLUPS": n ** 3 / t / 1e3,
                        "niter_mean_last_step": d["niter_mean"], "niter_max_last_step": d["niter_max"],
                        "node_iterations_per_s": n ** 3 * d["niter_mean"] / (t / 1e3)}
        out[prec] = rec
    return out


# ------------------------------------------------------------------ our arm
def _timed_window(s, pg, steps, warmup):
    """W untimed warm-up steps, then K steps timed with CUDA events on the
    library's stream, bracketed by a barrier and a synchronisation."""
    import torch
    s.step(warmup)
    s.last_step_ms()
    barrier(pg)
    torch.cuda.synchronize()
    d0 = s.diagnostics()
    s.step(steps)
    ms = s.last_step_ms()
    torch.cuda.synchronize()
    barrier(pg)
    d1 = s.diagnostics()
    return ms / steps, d0, d1


def _l1(a, b):
    return float(np.abs(a - b).mean() / np.abs(b).mean())


def run_ours(args, rank, local, world, pg):
    import torch

    import lbmpond_b200 as pond
    from lbmpond_b200.learned import Predictor, attach, calibrate_gate, collect_pairs, keep_history
    n = args.size
    N = n ** 3
    mk = lambda prec="fp32": pond.Solver(lattice="D3Q27", shape=(n, n, n), interp=pond.LAGR4,  # noqa: E731
                                        precision=prec, tau=TAU,
                                        tol_abs=TOL_ABS if prec == "fp32" else None,
                                        tol_rel=TOL_REL if prec == "fp32" else None, device=local)
    s = mk()
    s.init("sphere", *sphere_params())
    # spin-up (untimed), collecting training pairs over its last steps
    cap = args.pair_capacity
    X = torch.empty((cap, 39), dtype=torch.float32, device="cuda")
    Y = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
    rows = 0
    t0 = time.perf_counter()
    for k in range(args.spinup):
        collect = args.learned and k >= args.spinup - args.collect_steps and rows < cap
        if collect:
            keep_history(s, True)
        s.step(1)
        if collect:
            rows += collect_pairs(s, X, Y, offset_rows=rows, stride=args.pair_stride, seed=k)
    keep_history(s, False)
    torch.cuda.synchronize()
    t_spin = time.perf_counter() - t0
    snap = mk()
    snap.copy_state_from(s)

    # plain path
    ms_plain, p0, p1 = _timed_window(s, pg, args.steps, args.warmup)
    ms_plain = allmax(pg, ms_plain)
    work = s.last_step_work()
    plain = {"value": world * N / (ms_plain / 1e3) / 1e6, "ms_per_step": ms_plain,
             "iterations_mean": p1["niter_mean"], "iterations_max": p1["niter_max"],
             "nonconverged": p1["nonconverged"]}

    # iterations per node of one more plain step, and what a perfect starting
    # gauge could save: the first convergence test compares the new
    # populations with the previous time level's (steps.cu:360-510), so a node
    # whose populations change needs two iterations whatever its start and an
    # unchanged node one
    s.keep_niter(True)
    s.step(1)
    ni = s.niter()
    s.keep_niter(False)
    hist = np.bincount(np.minimum(ni, 12), minlength=13)[1:].tolist()
    ceiling = {"histogram_1_to_12plus": hist, "plain_mean": float(ni.mean()),
               "perfect_start_mean": float(np.minimum(ni, 2).mean()),
               "iteration_ratio": float(ni.mean() / np.minimum(ni, 2).mean())}

    # the same plain path with the convergence test of u and T at an absolute
    # 1e-8 (float64 gauge residual), the populations' test at the float32 floor
    gauge_tight = None
    if args.gauge_tol > 0:
        t = mk()
        t.copy_state_from(snap)
        t.set_gauge_tolerance(args.gauge_tol, 0.0)
        ms_g, _, g1 = _timed_window(t, pg, args.steps, args.warmup)
        ms_g = allmax(pg, ms_g)
        t.close()
        gauge_tight = {"value": world * N / (ms_g / 1e3) / 1e6, "ms_per_step": ms_g,
                       "iterations_mean": g1["niter_mean"], "iterations_max": g1["niter_max"],
                       "nonconverged": g1["nonconverged"],
                       "tolerance": {"gauge": [args.gauge_tol, 0.0], "populations": [TOL_ABS, TOL_REL]}}

    # learned path from the same state
    learned = None
    net = None
    if args.learned:
        t0 = time.perf_counter()
        net = Predictor(64, seed=0, device=local)
        net.fit_stats(X[:rows], Y[:rows])
        loss = net.train(X[:rows], Y[:rows], steps=args.train_steps, batch=8192, lr=2e-3)
        gate, _ = calibrate_gate(net, X[:rows], Y[:rows])
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        s.copy_state_from(snap)
        attach(s, net, gate=gate)
        with ClockSampler(local) as clk:
            ms_learned, l0, l1d = _timed_window(s, pg, args.steps, args.warmup)
        ms_learned = allmax(pg, ms_learned)
        work = s.last_step_work()
        learned = {"value": world * N / (ms_learned / 1e3) / 1e6, "ms_per_step": ms_learned,
                   "iterations_mean": l1d["niter_mean"], "iterations_max": l1d["niter_max"],
                   "nonconverged": l1d["nonconverged"],
                   "training": {"pairs": rows, "adam_steps": args.train_steps, "batch": 8192,
                                "loss_first": float(loss[:10].mean()), "loss_last": float(loss[-50:].mean()),
                                "seconds": t_train, "network": "39-64-64-4 tanh, bf16 tensor cores, fp32 accumulate",
                                "start": "previous gauge + predicted increment on nodes whose last increment >= gate",
                                "gate": gate}}
        d_first, d_last = l0, l1d
    else:
        with ClockSampler(local) as clk:
            pass
        d_first, d_last = p0, p1
    clocks = clk.summary()
    path = "learned" if learned else "plain"
    head = learned if learned else plain
    ms_step = head["ms_per_step"]
    value = head["value"]

    # equal L1 error: a few steps from the snapshot on the float64 path (the
    # reference-precision result) against the float32 plain and learned paths
    l1 = None
    if not args.no_l1 and world == 1:
        def drift(obj, d0):
            d1 = obj.diagnostics()
            return {"mass": (d1["mass"] - d0["mass"]) / d0["mass"] / args.l1_steps,
                    "energy": (d1["enrg"] - d0["enrg"]) / d0["enrg"] / args.l1_steps}

        ref64 = mk("fp64")
        ref64.copy_state_from(snap)
        d0 = ref64.diagnostics()
        ref64.step(args.l1_steps)
        fr = ref64.fields()
        l1 = {"steps": args.l1_steps, "reference": "float64 GPU path (tolerance 1e-12 + 1e-10|v|)",
              "drift_per_step": {"fp64": drift(ref64, d0)}}
        ref64.close()
        for name, use in (("plain", None), ("learned", net)):
            if name == "learned" and net is None:
                continue
            t = mk()
            t.copy_state_from(snap)
            if use is not None:
                attach(t, use, gate=learned["training"]["gate"])
            d0 = t.diagnostics()
            t.step(args.l1_steps)
            ft = t.fields()
            l1["drift_per_step"][name] = drift(t, d0)
            t.close()
            l1[name] = {"rho": _l1(ft["rho"], fr["rho"]), "T": _l1(ft["T"], fr["T"])}

    # e2e through the C ABI with host buffers on the timed path: every step
    # uploads its full input state from pinned host memory and reads rho, u, T
    # (the drop() fields) back, through pond_step_host, which overlaps one
    # step's copies with the neighbouring steps on two copy streams.  Timed by
    # the host clock between synchronisations (what a caller observes).
    e2e = None
    if not args.no_e2e:
        f_h = torch.empty((27, N), dtype=torch.float32, pin_memory=True)
        r_h = torch.empty(N, dtype=torch.float32, pin_memory=True)
        g_h = torch.empty((4, N), dtype=torch.float32, pin_memory=True)
        s.download_native(f_h.data_ptr(), r_h.data_ptr(), g_h.data_ptr())
        ro_h = torch.empty(N, dtype=torch.float32, pin_memory=True)
        go_h = torch.empty((4, N), dtype=torch.float32, pin_memory=True)
        attach(s, None)  # the pipelined call runs the plain start
        k = max(3, min(3 * args.steps, 32))  # the pipeline's fill and drain stay inside the window
        io = (f_h.data_ptr(), r_h.data_ptr(), g_h.data_ptr(), ro_h.data_ptr(), go_h.data_ptr())
        for _ in range(2):
            s.step_host(*io)
        s.sync()
        barrier(pg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            s.step_host(*io)
        s.sync()
        e2e_ms = allmax(pg, (time.perf_counter() - t0) * 1e3 / k)
        e2e = {"value": world * N / (e2e_ms / 1e3) / 1e6, "unit": "MLUPS", "path": "plain (pond_step_host)",
               "h2d_bytes_per_step": (27 + 5) * N * 4, "d2h_bytes_per_step": 5 * N * 4, "ms_per_step": e2e_ms,
               "steps": k, "timing": "host clock around the calls, synchronised on both sides (the first "
                                     "upload and the last read-back, which nothing overlaps, included)"}

    achieved_gbs = BYTES_PER_NODE * N / (ms_step / 1e3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get("pull_d3q27_lagr4_f32")
        if t and t.get("bytes_per_node"):
            traffic = t["bytes_per_node"] * N
    flops = work  # the kernel counts the floating-point operations of its basis contractions (last timed step)
    tflops = flops / (ms_step / 1e3) / 1e12
    drift = {"mass_per_step": (d_last["mass"] - d_first["mass"]) / d_first["mass"] / args.steps,
             "energy_per_step": (d_last["enrg"] - d_first["enrg"]) / d_first["enrg"] / args.steps}
    for obj in (s, snap):
        obj.close()
    if net is not None:
        net.close()
    out = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"D3Q27 {n}^3 spherical Riemann problem, tau {TAU}, cubic Lagrange, "
                               f"tolerance {TOL_ABS:g}+{TOL_REL:g}|v|", "path": path,
                   "grid": [n, n, n], "lattice": "D3Q27", "interp": "lagrange4", "precision": "fp32 (fp64 moments)",
                   "l2": "inputs larger than L2 (2.15 GB state per buffer)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "spinup_steps": args.spinup, "spinup_seconds": t_spin,
                   "timed_steps": f"{args.spinup + args.warmup + 1}..{args.spinup + args.warmup + args.steps}"},
        "plain": plain, "learned": learned, "plain_gauge_residual_1e8": gauge_tight,
        "speedup_learned_vs_plain": (learned["value"] / plain["value"]) if learned else None,
        "learned_start_ceiling": ceiling,
        "l1_vs_fp64": l1, "drift": drift,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved_gbs / hbm_peak, "traffic": traffic, "peak_source": "measured",
                     "algorithmic_bytes_per_node": BYTES_PER_NODE},
        "roofline_fp32": {"bound": "fp32", "achieved": tflops, "peak": NOMINAL_FP32_TFLOPS, "unit": "TFLOP/s",
                          "frac": tflops / NOMINAL_FP32_TFLOPS, "peak_source": "nominal at 1965 MHz",
                          "flops_per_step": flops,
                          "flops_counted": "basis contractions of the D3Q27 kernel (FMA = 2)"},
        "e2e": e2e,
        "gpu_launches": args.steps * (2 if learned else 1),
        "clocks": clocks,
    }
    return out


def _batch_set(lengths, rho, u, T, steps, chunk, pg, world, label):
    """Advance one problem set `steps` steps in graph-replayed launches of
    `chunk` steps, after the autotuner picked the tile; after every launch the
    state is read back (outside the timed launches) to record the step at
    which each problem first holds a non-finite value.  Returns the rates over
    all node updates and over the updates of problems still finite."""
    from lbmpond_b200 import replicas
    from lbmpond_b200.batch import Batch
    with Batch(lengths, interp=8, tau=0.9) as b:
        b.set_state(rho, u, T)
        tile, _ = b.autotune(probe_steps=5)
        b.set_state(rho, u, T)
        replicas.barrier(pg)
        alive = np.full(lengths.size, steps, dtype=np.int64)  # steps each problem stayed finite
        ms = 0.0
        niter = nonconv = 0
        for k0 in range(0, steps, chunk):
            ms += b.run(min(chunk, steps - k0), steps_per_launch=chunk)
            st = b.stats()
            niter += st["niter_sum"]
            nonconv += st["nonconverged"]
            f, r, uu, tt = b.get_state()
            fin = np.isfinite(f).all(0) & np.isfinite(r) & np.isfinite(uu) & np.isfinite(tt)
            for p in np.nonzero(alive == steps)[0]:
                if not fin[b.offsets[p]:b.offsets[p + 1]].all():
                    alive[p] = k0  # diverged within this launch: count the launch as lost
        nodes = b.nodes
    ms = replicas.max_over_ranks(pg, ms)
    upd = replicas.sum_over_ranks(pg, nodes * steps)
    upd_fin = replicas.sum_over_ranks(pg, int((lengths.astype(np.int64) * alive).sum()))
    dead = alive < steps
    out = {"workload": label, "nodes": int(replicas.sum_over_ranks(pg, nodes)), "steps": steps,
           "MLUPS": upd / (ms / 1e3) / 1e6, "MLUPS_finite_updates": upd_fin / (ms / 1e3) / 1e6,
           "ms_per_step": ms / steps, "tile": {"threads": tile[0], "lane_cap": tile[1]},
           "niter_mean": replicas.sum_over_ranks(pg, niter) / upd,
           "nonconverged_frac": replicas.sum_over_ranks(pg, nonconv) / upd,
           "nonfinite_problems": int(replicas.sum_over_ranks(pg, int(dead.sum()))),
           "steps_to_divergence": {"resolution": chunk,
                                   "quartiles": [float(q) for q in np.percentile(alive[dead], [25, 50, 75])]
                                   if dead.any() else None}}
    return out


def run_batch1d(steps=1000, nproblems=4096, pg=None, rank=0, world=1):
    """The batched D1Q5 workload: `nproblems` seeded Riemann problems
    (lengths uniform in [256, 4096], rho and p log-uniform in [0.1, 10], u
    uniform in [-1, 1], jump at the midpoint), WENO5, tau 0.9, float32 with
    float64 moments, `steps` steps in persistent graph-replayed launches of
    50 steps after the autotuner picked the tile.  The reference iteration
    drives most of these problems non-finite (the float64 oracle diverges on
    the same strong jumps), so the line also gives the rate over the node
    updates of problems still finite and the steps to divergence, and the same
    measurement on a well-posed companion set (density ratio <= 4,
    temperature ratio <= 1.5, moderate velocities).  Under several ranks the
    problems are split by node count (strong scaling: the whole set is the
    job) and the time is the slowest rank's."""
    from lbmpond_b200 import replicas
    from lbmpond_b200.batch import Batch, riemann_problems, riemann_problems_moderate
    import torch
    out = None
    for which in ("specified", "moderate"):
        gen = riemann_problems if which == "specified" else riemann_problems_moderate
        lengths, rho, u, T = gen(nproblems, seed=0)
        off = np.concatenate([[0], np.cumsum(lengths)])
        mine = replicas.partition_problems(lengths, world)[rank]
        sel = np.concatenate([np.arange(off[p], off[p + 1]) for p in mine])
        lengths, rho, u, T = lengths[mine], rho[sel], u[sel], T[sel]
        label = (f"{nproblems} D1Q5 Riemann problems, lengths U[256,4096] (seed 0), WENO5, {steps} steps"
                 if which == "specified" else
                 f"{nproblems} moderate D1Q5 Riemann problems (density ratio <= 4, temperature ratio <= 1.5, "
                 f"|u| <= 0.06, lattice T ~ 0.09), lengths U[256,4096] (seed 0), WENO5, {steps} steps")
        rec = _batch_set(lengths, rho, u, T, steps, 50, pg, world, label)
        if which == "specified":
            out = rec
            out["n_gpus"] = world
            out["scaling"] = "strong (problems split across ranks)" if world > 1 else None
            # training pairs written by the kernel itself, every 10 steps at every 16th node
            with Batch(lengths, interp=8, tau=0.9) as b:
                cap = 1 << 21
                X = torch.empty((cap, 21), dtype=torch.float32, device="cuda")
                Y = torch.empty((cap, 2), dtype=torch.float32, device="cuda")
                b.set_state(rho, u, T)
                b.set_pairs(X, Y, every=10, stride=16)
                ms_pairs = replicas.max_over_ranks(pg, b.run(100, steps_per_launch=50))
                pairs = b.pairs_written()
            out["pairs"] = {"rows_per_100_steps": int(replicas.sum_over_ranks(pg, pairs)), "every": 10,
                            "stride": 16, "ms_per_step_with_pairs": ms_pairs / 100}
        else:
            out["moderate_set"] = rec
    return out


def _time_steps(s, steps, warmup):
    s.step(warmup)
    ms = []
    for _ in range(steps):
        s.step(1)
        ms.append(s.last_step_ms())
    return float(np.mean(ms)), s.diagnostics()


shock_vortex_state = configs.shock_vortex_state


def run_configs(steps=5, warmup=2, d3q125_size=48):
    """Step throughput of the other workloads: the D1Q5 Sod tube (float64,
    TVD, 500 steps; at gamma 3 with one population and at gamma 1.4 with the
    energy populations, each with its L1 distance to the exact Riemann
    solution; the float64 oracle's own 500-step comparison is a GPU test),
    the D3Q27 Taylor-Green vortex at 128^3 (quadratic, float32) and the D3Q125
    shock-vortex box (fixed-origin quadratic, float32).  Progress goes to
    stderr."""
    import lbmpond_b200 as pond
    from tests.riemann import sample
    out = {}
    t_start = time.perf_counter()

    def note(msg):
        print(f"[configs {time.perf_counter() - t_start:7.1f} s] {msg}", file=sys.stderr, flush=True)

    # config 1: 1000 nodes on [0,1], dt/dx = 0.1 -> T = 0.01 p/rho (at dt/dx >= 0.2 the
    # TVD iteration of the float64 oracle itself goes non-finite within 20 steps)
    # the energy populations with 4 extra degrees of freedom give gamma = 1.4
    n, lam2, nsteps = 1000, 0.01, 500
    left, right = (1.0, 0.0, lam2 * 1.0), (0.125, 0.0, lam2 * 0.1 / 0.125)
    x = (np.arange(n) - (n / 2 - 0.5)) / nsteps
    for key, gamma, dof in (("sod_d1q5_fp64", 3.0, None), ("sod_d1q5_fp64_gamma14", 1.4, 4)):
        with pond.Solver(lattice="D1Q5", shape=(n, 1, 1), precision="fp64", interp=pond.TVD, tau=0.55,
                         bc=("clamp",) * 3, ddf_dof=dof) as s:
            s.init("sod", 0.5, *left, *right)
            t0 = time.perf_counter()
            s.step(nsteps)
            wall = time.perf_counter() - t0
            _, r1, g1 = s.get_state()
            d = s.diagnostics()
        er, eu, ep = sample((left[0], left[1], left[0] * left[2]), (right[0], right[1], right[0] * right[2]), gamma, x)
        out[key] = {"workload": f"D1Q5 Sod, {n} nodes, TVD, tau 0.55, zero-gradient ends, {nsteps} steps, float64, "
                                f"gamma {gamma:g}" + (f" (energy populations, {dof} extra degrees of freedom)" if dof
                                                      else " (one population)"),
                    "ms_per_step_wall": wall / nsteps * 1e3,
                    "l1_vs_exact_riemann": {"rho": float(np.abs(r1 - er).mean() / er.mean()),
                                            "u": float(np.abs(g1[0] - eu).mean() / np.abs(eu).mean()),
                                            "p": float(np.abs(r1 * g1[3] - ep).mean() / ep.mean())},
                    "niter_max_last_step": d["niter_max"]}
        note(f"sod gamma {gamma:g} done")
    # config 2: TGV 128^3, Mach 0.5 with gamma 5/3, T0 = TLat/4 (c = 0.5 node/step)
    T0 = (1.0 / 3.0) / 4
    U0 = 0.5 * np.sqrt(5.0 / 3.0 * T0)
    with pond.Solver(lattice="D3Q27", shape=(128,) * 3, precision="fp32", interp=pond.LAGR3, tau=0.51) as s:
        s.init("tgv", U0, T0, 1.0, 5.0 / 3.0)
        ms, d = _time_steps(s, steps, warmup)
        out["tgv_d3q27_128"] = {"workload": "D3Q27 Taylor-Green 128^3, Mach 0.5, quadratic Lagrange, tau 0.51, float32",
                                "ms_per_step": ms, "MLUPS": 128 ** 3 / ms / 1e3, "niter_mean": d["niter_mean"],
                                "niter_max": d["niter_max"], "steps_timed": f"{warmup + 1}..{warmup + steps}"}
    note("tgv done")
    # the same vortex as a gamma = 1.4 gas: energy populations with 2 extra degrees of freedom
    # (the energy tile kernel: the f and h of each node on two paired warps)
    T14 = (1.0 / 3.0) / 4
    U14 = 0.5 * np.sqrt(1.4 * T14)
    with pond.Solver(lattice="D3Q27", shape=(128,) * 3, precision="fp32", interp=pond.LAGR3, tau=0.51,
                     ddf_dof=2) as s:
        s.init("tgv", U14, T14, 1.0, 1.4)
        ms, d = _time_steps(s, steps, warmup)
        out["tgv_d3q27_128_gamma14"] = {
            "workload": "D3Q27 Taylor-Green 128^3, Mach 0.5, quadratic Lagrange, tau 0.51, float32, gamma 1.4 "
                        "(energy populations, 2 extra degrees of freedom)",
            "ms_per_step": ms, "MLUPS": 128 ** 3 / ms / 1e3, "niter_mean": d["niter_mean"], "niter_max": d["niter_max"],
            "steps_timed": f"{warmup + 1}..{warmup + steps}"}
    note("tgv gamma 1.4 done")
    # config 5: D3Q125 shock + vortex, plain and learned start from the same spun-up state
    import torch
    from lbmpond_b200.learned import Predictor, attach, calibrate_gate, collect_pairs, keep_history
    m = d3q125_size
    kw = dict(lattice="D3Q125", shape=(m,) * 3, precision="fp32", tau=0.9, bc=("clamp", "periodic", "periodic"))
    with pond.Solver(**kw) as s, pond.Solver(**kw) as snap:
        rho, g = shock_vortex_state(m)
        s.set_state(rho, g)
        note(f"d3q125 {m}^3 state set")
        cap = 2_000_000
        X = torch.zeros((cap, 39), dtype=torch.float32, device="cuda")
        Y = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
        rows = 0
        keep_history(s, True)
        for k in range(8):
            s.step(1)
            rows += collect_pairs(s, X, Y, offset_rows=rows, stride=31, seed=k)
        keep_history(s, False)
        snap.copy_state_from(s)
        ms_p, d_p = _time_steps(s, max(1, steps // 2), 1)
        _, rho_p, _ = s.get_state()
        note("d3q125 plain timed")
        net = Predictor(128, seed=0)
        net.fit_stats(X[:rows], Y[:rows])
        loss = net.train(X[:rows], Y[:rows], steps=2000, batch=8192, lr=2e-3)
        gate, _ = calibrate_gate(net, X[:rows], Y[:rows])
        s.copy_state_from(snap)
        attach(s, net, gate=gate)
        ms_l, d_l = _time_steps(s, max(1, steps // 2), 1)
        _, rho_l, _ = s.get_state()
        attach(s, None)
        net.close()
        note("d3q125 learned timed")
        out["shock_vortex_d3q125"] = {
            "workload": f"D3Q125 {m}^3 Mach 1.5 shock + isentropic vortex, fixed-origin quadratic, zero-gradient x "
                        "ends, periodic y/z, float32; 8 spin-up steps feed the training pairs",
            "plain": {"ms_per_step": ms_p, "MLUPS": m ** 3 / ms_p / 1e3, "niter_mean": d_p["niter_mean"],
                      "niter_max": d_p["niter_max"], "nonconverged": d_p["nonconverged"]},
            "learned": {"ms_per_step": ms_l, "MLUPS": m ** 3 / ms_l / 1e3, "niter_mean": d_l["niter_mean"],
                        "niter_max": d_l["niter_max"], "nonconverged": d_l["nonconverged"],
                        "network": "39-128-128-4", "pairs": rows, "loss_first": float(loss[0]),
                        "loss_last": float(loss[-1]), "gate": gate},
            "l1_rho_learned_vs_plain": float(np.abs(rho_l - rho_p).mean() / np.abs(rho_p).mean())}
    # the shock + vortex problem for a gamma = 1.4 gas: energy populations with 2 extra degrees of
    # freedom and the Rankine-Hugoniot states and isentropic vortex of gamma 1.4
    with pond.Solver(**kw, ddf_dof=2) as s:
        rho, g = shock_vortex_state(m, gamma=1.4)
        s.set_state(rho, g)
        s.step(8)
        ms_e, d_e = _time_steps(s, max(1, steps // 2), 1)
    out["shock_vortex_d3q125_energy"] = {
        "workload": f"D3Q125 {m}^3 Mach 1.5 shock + isentropic vortex at gamma 1.4 (energy populations, 2 extra "
                    "degrees of freedom), float32, after 8 steps",
        "ms_per_step": ms_e, "MLUPS": m ** 3 / ms_e / 1e3, "niter_mean": d_e["niter_mean"],
        "niter_max": d_e["niter_max"], "nonconverged": d_e["nonconverged"]}
    note("d3q125 energy populations timed")
    return out


def _chunked(s, steps, chunk=50):
    """Advance `steps` steps in calls of up to `chunk`; returns the summed
    device time of the step kernels (CUDA events, ms)."""
    ms = 0.0
    for k0 in range(0, steps, chunk):
        s.step(min(chunk, steps - k0))
        ms += s.last_step_ms()
    return ms


def _drift(d0, d1, steps):
    """Relative change of mass and energy over the run and per 1000 steps."""
    m, e = (d1["mass"] - d0["mass"]) / d0["mass"], (d1["enrg"] - d0["enrg"]) / d0["enrg"]
    return {"mass": m, "energy": e, "mass_per_1000_steps": m * 1000 / steps, "energy_per_1000_steps": e * 1000 / steps}


def _l1_fields(a, b):
    return {"rho": _l1(a["rho"], b["rho"]), "T": _l1(a["T"], b["T"])}


def run_configs_full(which, d3q125_size=192, l1_size_d3q125=48):
    """Full-length runs of the five configurations, one JSON object each
    (keyed by configuration), every result with its L1 distance in rho and T
    to this library's float64 path on the same run (itself held to the FP64
    oracle by the GPU tests) and its relative mass and energy drift:

      1  D1Q5 Sod, 1000 nodes, TVD, 500 steps, float64 (gamma 3, and gamma 1.4
         with the energy populations): L1 to the exact Riemann solution; the
         float32 path against the float64 one
      2  D3Q27 Taylor-Green 128^3, quadratic, tau 0.51, 2000 steps, float32
         against float64
      3  the batched D1Q5 problems (the benchmark line's batch1d)
      4  D3Q27 sphere 256^3, cubic, tau 0.52, up to 1500 steps: float32 plain
         and learned (pairs from steps 121-150, the network attached from
         step 151), each stopped at its first non-finite check (the
         rarefaction focusing at the centre drives rho and T towards 0 there)
         and held against the float64 path over three steps from its last
         finite checkpoint; and the step by which the float32 and the float64
         path go non-finite at 128^3
      5  D3Q125 shock + vortex at d3q125_size^3, centred WENO5, inflow/outflow
         in x, 1000 steps, float32; L1 against float64 over ten steps from
         the final state (the float64 path at the reference's tolerance);
         learned against plain at d3q125_size^3 after 200 steps.

    Device time by CUDA events on the library's stream, summed over the
    steps.  Progress goes to stderr."""
    import torch

    import lbmpond_b200 as pond
    from lbmpond_b200.learned import Predictor, attach, calibrate_gate, collect_pairs, keep_history
    from tests.riemann import sample
    t_start = time.perf_counter()

    def note(msg):
        print(f"[configs-full {time.perf_counter() - t_start:7.1f} s] {msg}", file=sys.stderr, flush=True)

    out = {}
    if "1" in which:
        n, lam2, nsteps = 1000, configs.SOD_LAMBDA2, 500
        left, right = (1.0, 0.0, lam2 * 1.0), (0.125, 0.0, lam2 * 0.1 / 0.125)
        x = (np.arange(n) - (n / 2 - 0.5)) / nsteps
        for key, gamma, dof in (("sod_d1q5", 3.0, None), ("sod_d1q5_gamma14", 1.4, 4)):
            res = {}
            for prec in ("fp64", "fp32"):
                with pond.Solver(lattice="D1Q5", shape=(n, 1, 1), precision=prec, interp=pond.TVD, tau=0.55,
                                 bc=("clamp",) * 3, ddf_dof=dof) as s:
                    s.init("sod", 0.5, *left, *right)
                    d0 = s.diagnostics()
                    ms = _chunked(s, nsteps)
                    res[prec] = (s.fields(), _drift(d0, s.diagnostics(), nsteps), ms / nsteps)
            er, eu, ep = sample((left[0], left[1], left[0] * left[2]), (right[0], right[1], right[0] * right[2]),
                                gamma, x)
            fr = res["fp64"][0]
            out[key] = {"workload": f"D1Q5 Sod, {n} nodes, TVD, tau 0.55, zero-gradient ends, {nsteps} steps, gamma "
                                    f"{gamma:g}" + (f" (energy populations, {dof} extra degrees of freedom)" if dof else ""),
                        "fp64": {"ms_per_step": res["fp64"][2], "drift": res["fp64"][1],
                                 "l1_vs_exact_riemann": {"rho": float(np.abs(fr["rho"] - er).mean() / er.mean()),
                                                         "p": float(np.abs(fr["rho"] * fr["T"] - ep).mean() / ep.mean())}},
                        "fp32": {"ms_per_step": res["fp32"][2], "drift": res["fp32"][1],
                                 "l1_vs_fp64": _l1_fields(res["fp32"][0], fr)}}
            note(f"{key} done")
    if "2" in which:
        n, nsteps = 128, 2000
        res = {}
        for prec in ("fp32", "fp64"):
            with pond.Solver(lattice="D3Q27", shape=(n,) * 3, precision=prec, interp=pond.LAGR3, tau=0.51) as s:
                s.init("tgv", *configs.tgv_params())
                d0 = s.diagnostics()
                ms, its, ks = 0.0, [], [d0["k"]]
                for k0 in range(0, nsteps, 100):
                    ms += _chunked(s, 100)
                    d = s.diagnostics()
                    its.append(d["niter_mean"])
                    ks.append(d["k"])
                res[prec] = (s.fields(), _drift(d0, d, nsteps), ms / nsteps, float(np.mean(its)), ks)
            note(f"tgv {prec} done")
        out["tgv_d3q27_128"] = {
            "workload": f"D3Q27 Taylor-Green {n}^3, Mach 0.5, quadratic Lagrange, tau 0.51, {nsteps} steps",
            "fp32": {"ms_per_step": res["fp32"][2], "MLUPS": n ** 3 / res["fp32"][2] / 1e3,
                     "niter_mean": res["fp32"][3], "drift": res["fp32"][1],
                     "l1_vs_fp64": _l1_fields(res["fp32"][0], res["fp64"][0]),
                     "kinetic_energy_every_100_steps": res["fp32"][4]},
            "fp64": {"ms_per_step": res["fp64"][2], "MLUPS": n ** 3 / res["fp64"][2] / 1e3,
                     "niter_mean": res["fp64"][3], "drift": res["fp64"][1]}}
    if "3" in which:
        out["batch1d"] = run_batch1d(1000, 4096)
        note("batch done")
    if "4" in which:
        n, nsteps, spin, l1_steps, chunk = 256, 1500, 150, 3, 25
        mk = lambda prec="fp32", m=n: pond.Solver(lattice="D3Q27", shape=(m,) * 3, interp=pond.LAGR4,  # noqa: E731
                                                 precision=prec, tau=TAU,
                                                 tol_abs=TOL_ABS if prec == "fp32" else None,
                                                 tol_rel=TOL_REL if prec == "fp32" else None)
        rec = {"workload": f"D3Q27 {n}^3 spherical Riemann problem, tau {TAU}, cubic Lagrange, up to {nsteps} "
                           f"steps; the state goes non-finite where the rarefaction focuses at the centre, so each "
                           f"run stops at the first non-finite check (every {chunk} steps) and its L1 is taken over "
                           f"{l1_steps} steps from the last finite checkpoint"}

        def finite(s):
            return bool(np.isfinite(s.diagnostics()["mass"]))

        def progress(s, label, k, ms):
            d, fl = s.diagnostics(), s.fields()
            umax = np.sqrt(fl["ux"] ** 2 + fl["uy"] ** 2 + fl["uz"] ** 2).max()
            note(f"{label} step {k}: {ms:.0f} ms so far, niter mean {d['niter_mean']:.3f} max {d['niter_max']} "
                 f"nonconverged {d['nonconverged']}, T {fl['T'].min():.4g}..{fl['T'].max():.4g}, max |u| {umax:.4g}, "
                 f"rho {fl['rho'].min():.4g}..{fl['rho'].max():.4g}")

        def l1_window(snap, k0):
            """float32 against float64 over l1_steps steps from the snapshot taken after step k0."""
            note(f"float64 window from step {k0}")
            with mk("fp64") as r:
                r.copy_state_from(snap)
                d0 = r.diagnostics()
                r.step(l1_steps)
                fr = r.fields()
                dr = _drift(d0, r.diagnostics(), l1_steps)
                ms64 = r.last_step_ms() / l1_steps
            snap.step(l1_steps)
            return {"window": f"steps {k0 + 1}..{k0 + l1_steps}", **_l1_fields(snap.fields(), fr),
                    "fp64_drift_in_window": dr, "fp64_ms_per_step": ms64}

        def run(s, snap, label, k_start, ms0):
            """Steps s from k_start to nsteps in chunks, keeping the last finite
            state in snap; returns (steps run, device ms, first non-finite check)."""
            ms, k, bad = ms0, k_start, None
            snap.copy_state_from(s)
            kept = k
            while k < nsteps:
                ms += _chunked(s, min(chunk, nsteps - k))
                k = min(k + chunk, nsteps)
                progress(s, label, k, ms)
                if not finite(s):
                    bad = k
                    break
                snap.copy_state_from(s)
                kept = k
            return k, ms, bad, kept

        with mk() as s, mk() as snap:
            s.init("sphere", *sphere_params())
            d0 = s.diagnostics()
            done, ms, bad, kept = run(s, snap, "plain", 0, 0.0)
            d = s.diagnostics()
            rec["plain"] = {"steps_run": done, "non_finite_by_step": bad, "last_finite_checkpoint": kept,
                            "ms_per_step": ms / done, "MLUPS": n ** 3 / (ms / done) / 1e3,
                            "drift_to_checkpoint": _drift(d0, snap.diagnostics(), kept),
                            "niter_mean_last_step": d["niter_mean"], "nonconverged_last_step": d["nonconverged"],
                            "l1_vs_fp64": l1_window(snap, kept)}
        note("sphere plain done")
        cap = 4_000_000
        X = torch.empty((cap, 39), dtype=torch.float32, device="cuda")
        Y = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
        with mk() as s, mk() as snap:
            s.init("sphere", *sphere_params())
            d0 = s.diagnostics()
            rows = 0
            ms = _chunked(s, spin - 30)
            keep_history(s, True)
            for k in range(30):
                s.step(1)
                ms += s.last_step_ms()
                rows += collect_pairs(s, X, Y, offset_rows=rows, stride=61, seed=k)
            keep_history(s, False)
            net = Predictor(64, seed=0)
            net.fit_stats(X[:rows], Y[:rows])
            net.train(X[:rows], Y[:rows], steps=10000, batch=8192, lr=2e-3)
            gate, _ = calibrate_gate(net, X[:rows], Y[:rows])
            attach(s, net, gate=gate)
            done, ms_all, bad, kept = run(s, snap, "learned", spin, ms)
            d = s.diagnostics()
            attach(s, None)
            net.close()
            rec["learned"] = {"steps_run": done, "non_finite_by_step": bad, "last_finite_checkpoint": kept,
                              "ms_per_step": ms_all / done, "MLUPS": n ** 3 / (ms_all / done) / 1e3,
                              "MLUPS_after_attach": n ** 3 / ((ms_all - ms) / (done - spin)) / 1e3,
                              "drift_to_checkpoint": _drift(d0, snap.diagnostics(), kept),
                              "niter_mean_last_step": d["niter_mean"], "nonconverged_last_step": d["nonconverged"],
                              "l1_vs_fp64": l1_window(snap, kept)}
        note("sphere learned done")
        # the same problem at 128^3 in both precisions: does the float64 path go non-finite too?
        m = n // 2
        div = {}
        for prec in ("fp32", "fp64"):
            with mk(prec, m) as s:
                s.init("sphere", *sphere_params())
                k, first = 0, None
                while k < nsteps // 2:
                    s.step(min(chunk // 2, nsteps // 2 - k))
                    k = min(k + chunk // 2, nsteps // 2)
                    if not finite(s):
                        first = k
                        break
                div[prec] = {"non_finite_by_step": first, "steps_run": k, "check_every": chunk // 2,
                             "tolerance": [TOL_ABS, TOL_REL] if prec == "fp32" else [1e-12, 1e-10]}
            note(f"sphere {m}^3 {prec}: non-finite by step {first}")
        rec[f"divergence_{m}cube"] = div
        out["sphere_d3q27_256"] = rec
    if "5" in which:
        m, nsteps, l1_steps = d3q125_size, 1000, 10
        rec = {}
        with configs.build("shock_vortex_d3q125", size=m) as s:
            d0 = s.diagnostics()
            ms, its, nmax = 0.0, [], 0
            for k0 in range(0, nsteps, 50):
                ms += _chunked(s, 50)
                d = s.diagnostics()
                its.append(d["niter_mean"])
                nmax = max(nmax, d["niter_max"])
            rec["fp32"] = {"grid": f"{m}^3", "steps": nsteps, "ms_per_step": ms / nsteps,
                           "MLUPS": m ** 3 / (ms / nsteps) / 1e3, "niter_mean": float(np.mean(its)),
                           "niter_max_seen": nmax, "nonconverged_last_step": d["nonconverged"],
                           "drift": _drift(d0, d, nsteps)}
            note("d3q125 fp32 1000 steps done")
            # float32 against float64 over l1_steps steps from the final state
            with configs.build("shock_vortex_d3q125", size=m, precision="fp64") as r:
                r.copy_state_from(s)
                r.set_inflow(*configs.shock_vortex_inflow())
                r.step(l1_steps)
                fr = r.fields()
                rec["fp64_window"] = {"steps": l1_steps, "ms_per_step": r.last_step_ms() / l1_steps}
            s.step(l1_steps)
            rec["fp32"]["l1_vs_fp64"] = {"window": f"steps {nsteps + 1}..{nsteps + l1_steps} from the float32 "
                                                   "state, float64 path at 1e-12 + 1e-10|v|",
                                         **_l1_fields(s.fields(), fr)}
        note("d3q125 l1 done")
        # learned against plain at the full size, from the state after 200 steps
        m = d3q125_size
        with configs.build("shock_vortex_d3q125", size=m) as s, configs.build("shock_vortex_d3q125", size=m) as snap:
            cap = 2_000_000
            X = torch.zeros((cap, 39), dtype=torch.float32, device="cuda")
            Y = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
            s.step(180)
            keep_history(s, True)
            rows = 0
            for k in range(20):
                s.step(1)
                rows += collect_pairs(s, X, Y, offset_rows=rows, stride=31, seed=k)
            keep_history(s, False)
            snap.copy_state_from(s)
            ms_p = _chunked(s, 20, 20) / 20
            dp = s.diagnostics()
            fp = s.fields()
            net = Predictor(128, seed=0)
            net.fit_stats(X[:rows], Y[:rows])
            loss = net.train(X[:rows], Y[:rows], steps=4000, batch=8192, lr=2e-3)
            gate, _ = calibrate_gate(net, X[:rows], Y[:rows])
            s.copy_state_from(snap)
            attach(s, net, gate=gate)
            ms_l = _chunked(s, 20, 20) / 20
            dl = s.diagnostics()
            fl = s.fields()
            attach(s, None)
            net.close()
        rec["learned_vs_plain_after_200_steps"] = {
            "grid": f"{m}^3", "steps": 20, "network": "39-128-128-4",
            "plain": {"ms_per_step": ms_p, "MLUPS": m ** 3 / ms_p / 1e3, "niter_mean": dp["niter_mean"]},
            "learned": {"ms_per_step": ms_l, "MLUPS": m ** 3 / ms_l / 1e3, "niter_mean": dl["niter_mean"],
                        "pairs": rows, "loss_last": float(loss[-1]), "gate": gate},
            "l1_learned_vs_plain": _l1_fields(fl, fp)}
        note("d3q125 learned done")
        rec["workload"] = ("D3Q125 Mach 1.5 shock + isentropic vortex, centred WENO5 (POND_WENO5_ROW), "
                           "inflow/outflow in x, periodic y/z, tau 0.9, float32")
        out["shock_vortex_d3q125"] = rec
    return out


def run_mesh1d(steps=20, warmup=3, n=1 << 24):
    """The one-dimensional mesh path on a Sod tube of n nodes (float32, tau
    0.55, periodic): GAP2 on an AMR mask (every other node active, then one
    refinement around the jumps) and NONUNIFORM3 on stretched positions.  Step
    time by CUDA events on the library's stream; the state (n x 7 floats x 2
    levels, 0.94 GB at 2^24) is far larger than L2.  Algorithmic bytes per
    active node and step: (5 + 2) x 4 x 2 = 56 (populations, rho, u_x, T read
    once and written once).  The AMR calls are timed by the host clock around
    the synchronous call (which includes reading back its counts)."""
    import lbmpond_b200 as pond
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    measured = {}
    try:  # DRAM bytes per grid node of each kernel, from one ncu capture (profiles/pull_1d_mesh_4M.md)
        measured = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except OSError:
        pass
    out = {"workload": f"D1Q5 Sod tube, {n} nodes, float32, tau 0.55, periodic", "steps": steps, "warmup": warmup}
    sod = (0.5, 1.0, 0.0, 0.01, 0.125, 0.0, 0.008)
    for scheme in ("GAP2", "NONUNIFORM3"):
        with pond.Solver(lattice="D1Q5", shape=(n, 1, 1), interp=getattr(pond, scheme), precision="fp32",
                         tau=0.55) as s:
            s.init("sod", *sod)
            rec = {}
            if scheme == "GAP2":
                s.set_mask((np.arange(n) % 2 == 0).astype(np.uint8))
                t0 = time.perf_counter()
                added, _ = s.amr_refine(0.01)
                rec["refine_ms"] = (time.perf_counter() - t0) * 1e3
                rec["refined_nodes"] = added
            else:
                x = np.arange(n, dtype=np.float64)
                s.set_positions(x + 0.3 * np.sin(2 * np.pi * x / n))
            active = int(s.get_mask().sum())
            ms, d = _time_steps(s, steps, warmup)
            if scheme == "GAP2":
                t0 = time.perf_counter()
                removed = s.amr_coarsen(0.01)
                rec["coarsen_ms"] = (time.perf_counter() - t0) * 1e3
                rec["coarsened_nodes"] = removed
            gbs = 56.0 * active / (ms / 1e3) / 1e9
            t = measured.get("pull_1d_mesh_" + ("gap2" if scheme == "GAP2" else "nu3") + "_f32")
            rec.update({"active_nodes": active, "ms_per_step": ms, "MLUPS": active / (ms / 1e3) / 1e6,
                        "niter_mean": d["niter_mean"], "niter_max": d["niter_max"],
                        "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s",
                                     "frac": gbs / hbm_peak, "bytes_per_node": 56,
                                     "traffic": t["bytes_per_node"] * n if t else None}})
            out[scheme.lower()] = rec
    return out


def run_reference(args, rank, world):
    """The reference arm: the reference's step restated on the host (FP64
    oracle; the reference itself has no CPU implementation), all host threads,
    each step a bounded sample of the same problem at the same stage of the
    blast as the timed GPU steps."""
    m = args.ref_size
    spin = round(args.spinup * m / 256)
    if os.path.exists(SAMPLE):
        v, dt, it, it_gpu, cores, desc = _oracle_blocks(args.warmup, args.steps)
        sample = f"{desc}; FP64 oracle, {cores} threads, {it:.2f} iterations per node"
    else:
        v, dt, it, cores = _oracle_sample(m, spin, args.warmup, args.steps)
        sample = (f"{m}^3 sample of the sphere problem after {spin} spin-up steps (the 256^3 spin-up scaled), "
                  f"FP64 oracle, {cores} threads, {it:.2f} iterations per node")
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"D3Q27 {args.size}^3 spherical Riemann problem, tau {TAU}, cubic Lagrange, "
                                   f"tolerance {TOL_ABS:g}+{TOL_REL:g}|v|",
                       "path": "reference step on the host", "sample": sample},
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--spinup", type=int, default=150, help="untimed steps before the warm-up")
    ap.add_argument("--no-learned", dest="learned", action="store_false")
    ap.add_argument("--collect-steps", type=int, default=30, help="spin-up steps that feed training pairs")
    ap.add_argument("--pair-stride", type=int, default=61)
    ap.add_argument("--pair-capacity", type=int, default=4_000_000)
    ap.add_argument("--train-steps", type=int, default=10000)
    ap.add_argument("--no-l1", action="store_true")
    ap.add_argument("--l1-steps", type=int, default=3)
    ap.add_argument("--ref-size", type=int, default=24)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-cuda", dest="ref_cuda", action="store_false",
                    help="skip the same-state comparison with the reference's own kernels (64^3 float64, 32^3 "
                         "float32; the reference arm runs its kernels, this arm its own on the same runs)")
    ap.add_argument("--gauge-tol", type=float, default=1e-8,
                    help="also time the plain path with this absolute gauge tolerance (0: skip)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 1D measurement")
    ap.add_argument("--batch-steps", type=int, default=1000)
    ap.add_argument("--batch-problems", type=int, default=4096)
    ap.add_argument("--configs", default="12345", help="configs-full: which configurations (digits 1-5)")
    ap.add_argument("--cfg5-size", type=int, default=192, help="configs-full: grid edge of configuration 5")
    ap.add_argument("--workload", default="d3q27", choices=["d3q27", "batch1d", "configs", "configs-full", "mesh1d"],
                    help="batch1d: only the batched D1Q5 measurement; configs: the other workloads (one JSON object); "
                         "mesh1d: the 1D mesh path (node mask, AMR, non-uniform positions)")
    ap.add_argument("--d3q125-size", type=int, default=48)
    ap.add_argument("--mesh-size", type=int, default=1 << 24, help="nodes of the mesh1d workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        if rank != 0:
            return
        out = run_reference(args, rank, world)
        if args.ref_cuda:
            out["reference_cuda"] = reference_cuda()
        print(json.dumps(out), flush=True)
        return
    if args.workload == "batch1d":
        rank, local, world, pg = dist_setup(args.gpus)
        out = run_batch1d(args.batch_steps, args.batch_problems, pg, rank, world)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    if args.workload == "mesh1d":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(run_mesh1d(args.steps, args.warmup, args.mesh_size)), flush=True)
        return
    if args.workload == "configs-full":
        if int(os.environ.get("RANK", "0")) == 0:
            for key, rec in run_configs_full(args.configs, args.cfg5_size).items():
                print(json.dumps({key: rec}), flush=True)
        return
    if args.workload == "configs":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(run_configs(args.steps, args.warmup, args.d3q125_size)), flush=True)
        return
    rank, local, world, pg = dist_setup(args.gpus)
    out = run_ours(args, rank, local, world, pg)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(args.spinup)
    if rank == 0 and world == 1 and args.ref_cuda:
        out["same_state_as_reference_kernels"] = ours_same_state(local)
    if rank == 0 and world == 1 and not args.no_batch:
        out["batch1d"] = run_batch1d(args.batch_steps, args.batch_problems)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
