#!/usr/bin/env python
"""bench.py — zone-updates/s of the 2+1D finite-volume stage on B200.

Workload (one GPU): a viscous single event, shear + bulk IS/DNMR (eta/s = 0.16,
C_s = 0.2 so tau_pi = 5 eta/(e+P), delta_pipi = 4/3 tau_pi; zeta/s Gaussian peak
0.05 at 0.180 GeV, width 0.024 GeV), diffusing charm (D_s T = 0.5), LatticeHRG
EOS, 384 x 384 cells on [-15, 15] fm, SSPRK3, CFL 0.2 / CFLtau 0.05, starting
at tau0 = 0.6 fm/c from a seeded MC-Glauber Pb+Pb event (seed 1001 + rank).

A step is one iteration of run_sim_2d!'s loop (main2D.jl:436-513): the CFL dt,
the three SSPRK3 stages (each: BCs, primitive recovery on every cell, MUSCL +
HLLE + sources, combination, floors/bounds/admissibility), the primitive
refresh, the IS/DNMR relaxation and the shear projection. A zone-update is one
interior cell advanced through one accepted step. The event is laid on the edge
state of the reference's production profile (T = 0.12786 GeV, alpha = 1.8878),
so it runs to the configured tau = 10 fm/c.

  value     device-resident: K steps after W warm-up steps, per-step CUDA events on
            the library's stream, L2 flushed (256 MB write) between steps, sum over
            the K steps, max over ranks. Kernel by kernel; --graphs replays each step's
            two launch sequences (the optimistic SSPRK step, then the primitive
            refresh and relaxation) as CUDA graphs instead (fivo_ctx_set_graphs, the
            same bits). The per-kernel times of the roofline come from replaying the
            same K steps (a device copy of the state taken before them) kernel by
            kernel with the library's kernel timing on, so the timed run has no
            profiling events.
  full_run  the whole configured run, tau0 = 0.6 -> 10 fm/c, timed the same way
            from a device copy of the initial state: the figure that does not
            depend on the window.
  e2e       the same steps through the C ABI with the state in pinned host memory:
            every step uploads U, advances, downloads U (the drop-in usage from a
            host driver that keeps U on the host).
  metric_comparison  the metric's own comparison: 256 events of the event-by-event
            sizes (N in {96..400}, dx = 30/384 fm) advanced in plain FP64, in FP32 (faces
            and relaxation sources) and with the learned recovery guess plus FP32, one
            stream per event, then plain FP64 and FP32 in lockstep (each kernel of a
            step launched once over all events, replayed from CUDA graphs, schedule
            tuned on the warm-up steps), on the same events; each form's L2(T) and
            L2(pibar) against the plain run after the window.

`--impl reference` times the reference's CPU path (the C++ restatement in
oracle/, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "fivohydro.jl_b200"))

N_CELLS = 384
BOX = 15.0
TAU0 = 0.6
TAU_END = 10.0          # the configured end of the viscous event's run
CFL, CFLTAU = 0.2, 0.05
SEED = 1001
WORKLOAD = "viscous_event_384x384_ssprk3_lhrg_shear_bulk_diffusion"
METRIC = "zone-updates/s on 1 B200: batched learned+FP32 vs plain FP64, L2(T)<=1e-6"
UNIT = "zone-updates/s"


def model_and_grid():
    import fivo2d
    g = fivo2d.make_grid2d(N_CELLS, N_CELLS, xmax=BOX, ymax=BOX)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                              enable_diff=True, eta_over_s=0.16, tauShear_coeff=0.2,
                              deltaShear_factor=4 / 3, zeta_over_s=0.05, bulk_model="gaussian",
                              bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5)
    return g, m


def ic_fields(g, seed):
    from fivo2d import ic
    T, a, ux, uy, ev = ic.glauber_fields(g, TAU0, seed)
    return T, a, ux, uy


# ----------------------------------------------------------------------------- the learned guess

GUESS_SEEDS = (3001, 3002, 3003)     # training events: never the timed ones (1001 + rank, 1000 + k)
GUESS_TRAIN_STEPS = 220              # per training event (the timed window ends near step 210)


def train_guess(lib, m, g, seeds=GUESS_SEEDS, nsteps=GUESS_TRAIN_STEPS, train_steps=3000):
    """Harvest (features, primitives) pairs from plain runs of seeded training events
    on grid g (every 4th step, every 8th cell), fit the normalisation and train the
    guess network on the GPU. Returns (guess, info)."""
    from fivo2d import _abi as A
    from fivo2d.guess import RecoveryGuess
    from fivo2d.solver import GPUWork2D, set_cells

    t0 = time.perf_counter()
    guess = RecoveryGuess(lib=lib, seed=17)
    guess.reserve(8_000_000)
    harvested_steps = 0
    for s in seeds:
        T, a, ux, uy = ic_fields(g, s)
        U, _ = set_cells(m, TAU0, T, a, ux, uy, lib=lib)
        wt = GPUWork2D(m, g, lib=lib)
        wt.set_state(U)
        wt.finalize_ic(TAU0)
        wt.rhs(TAU0)
        tau = TAU0
        for k in range(nsteps):
            r = wt.advance(tau, 1e9, CFL, CFLTAU, A.FIVO_SSPRK3, max_steps=1)
            if not r["ok"]:
                break
            tau = r["tau"]
            if k % 4 == 0:
                wt.update_primitives(tau)
                guess.harvest(wt, tau, stride=8, phase=(k // 4) % 8)
                harvested_steps += 1
        wt.close()
    t1 = time.perf_counter()
    guess.fit_norm()
    l0, l1 = guess.train(train_steps, ctas_per_step=148, lr=2e-3, seed=5)
    t2 = time.perf_counter()
    return guess, {"samples": guess.nsamples(), "training_events": list(seeds),
                   "harvested_steps": harvested_steps, "train_steps": train_steps,
                   "batch": 148 * 128, "loss_first": l0, "loss_last": l1,
                   "harvest_s": t1 - t0, "train_s": t2 - t1}


def l2_rel(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for line in pathlib.Path(self.f.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- roofline

# Algorithmic bytes per cell of each kernel class: every field read or written
# once per pass (FP64 = 8 B, flags 1 B). nv = 11 state rows here.
def algorithmic_bytes_per_unit(kclass, nv):
    """Compulsory DRAM bytes per unit (cell, or face for "faces") of each kernel class."""
    ndis = nv - 4
    if kclass in ("prim_fast", "prim_slow"):  # U (nv) + warm start (4) in; 9 primitives + ok + warm start out
        return (nv + 4) * 8 + 9 * 8 + 1 + 4 * 8
    if kclass == "faces":       # 4 primitives + mu + dissipatives of the cell in; nv fluxes out
        return (5 + ndis) * 8 + nv * 8
    if kclass == "update":      # U_in, U_old (2 of 3 stages), 2 flux planes sets, P, ux, uy, ok; U_out + bad
        return nv * 8 * (1 + 2 / 3 + 2) + 3 * 8 + 1 + nv * 8 + 1
    if kclass == "adm_slow":    # the cell's conserved state in, bad out
        return nv * 8 + 1
    if kclass == "relax":       # dissipatives in/out, 8 primitives + ok, 3 history planes
        return 2 * ndis * 8 + 8 * 8 + 1 + 3 * 8
    return None


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def from_profiles(kclass, key):
    """A figure of the committed ncu summary of a kernel class (`key: value` line), if present."""
    f = ROOT / "profiles" / f"{kclass}_kernel_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def traffic_from_profiles(kclass):
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    return from_profiles(kclass, "traffic_bytes_per_launch_full_workload")


# ----------------------------------------------------------------------------- our arm

def run_gpu(args):
    import numpy as np
    import torch

    import fivo2d
    from fivo2d import _abi as A
    from fivo2d.solver import GPUWork2D, set_cells

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    lib = A.load_library()
    g, m = model_and_grid()
    guess, ginfo = (train_guess(lib, m, g) if args.guess else (None, None))
    T, a, ux, uy = ic_fields(g, SEED + rank)
    U0, ok = set_cells(m, TAU0, T, a, ux, uy, lib=lib)
    w = GPUWork2D(m, g, lib=lib)
    if guess is not None:
        guess.attach(w)
    if args.fp32_faces:
        w.set_precision(A.FIVO_PRECISION_FP32_FACES)
    stream = torch.cuda.Stream()
    A.check(lib, lib.fivo_ctx_set_stream(w.h, C.c_void_p(stream.cuda_stream)), "set_stream")
    graphs = args.graphs
    w.set_graphs(graphs)       # --graphs: each step's launch sequences replayed as CUDA graphs (same bits)
    w.set_state(U0)
    w.finalize_ic(TAU0)
    nint = g.Nx * g.Ny

    # prime primitives and signal speeds (run_sim_2d!, main2D.jl:418); the first stage
    # also picks the face-pass kernel by timing the candidates (fivo_ctx_set_face_pass)
    w.rhs(TAU0)
    face_pass = [("global" if k == A.FIVO_FACES_GLOBAL else "tile %dx%d" % A.FACE_TILE_SHAPES[k])
                 for k in w.face_pass()]
    tau = TAU0
    res = A.FivoRunResult()
    init = None
    if not args.no_full_run:
        init = GPUWork2D(m, g, lib=lib)          # the state at tau0, for the full-run figure
        A.check(lib, lib.fivo_ctx_set_stream(init.h, C.c_void_p(stream.cuda_stream)), "set_stream")
        init.set_graphs(graphs)
        init.clone_state_from(w)

    def step_on(h, tau_, n):
        A.check(lib, lib.fivo_advance(h, tau_, 1e9, CFL, CFLTAU, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, n,
                                      C.byref(res)), "fivo_advance")
        if not res.ok:
            raise RuntimeError(f"step failed at tau={tau_}")
        return res.tau

    def advance(n):
        nonlocal tau
        tau = step_on(w.h, tau, n)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def l2_flush():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    for _ in range(args.warmup):
        advance(1)

    # A twin context holds the state at the start of the timed window; the same
    # steps are replayed on it afterwards with per-kernel CUDA-event timing, so
    # the timed run itself carries no profiling events.
    twin = GPUWork2D(m, g, lib=lib)
    A.check(lib, lib.fivo_ctx_set_stream(twin.h, C.c_void_p(stream.cuda_stream)), "set_stream")
    twin.clone_state_from(w)
    # the mixed-precision form over the same window, from a device clone (default line only)
    form32 = None
    if guess is None and not args.fp32_faces and not args.no_forms:
        form32 = GPUWork2D(m, g, lib=lib)
        A.check(lib, lib.fivo_ctx_set_stream(form32.h, C.c_void_p(stream.cuda_stream)), "set_stream")
        form32.clone_state_from(w)
        form32.set_graphs(graphs)
        form32.set_precision(A.FIVO_PRECISION_FP32_FACES)
    plain = None
    if guess is not None or args.fp32_faces:
        plain = GPUWork2D(m, g, lib=lib)          # the plain FP64 path over the same steps
        plain.clone_state_from(w)
    if args.fp32_faces:
        twin.set_precision(A.FIVO_PRECISION_FP32_FACES)
    if guess is not None:
        from fivo2d.guess import newton_stats
        guess.attach(twin)
        newton_stats(w, reset=True)

    # ---------------- device-resident timing
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    tau_start = tau
    # the clock samples span the timed steps and their profiled replay (the same work):
    # a window of a few tens of milliseconds alone is shorter than one sampling period
    clk = ClockSampler(local).__enter__()
    kernels0 = w.lockstep_info()["kernels"]
    for k in range(args.steps):
        l2_flush()
        starts[k].record(stream)
        advance(1)
        stops[k].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, stops))
    graph_kernels = w.lockstep_info()["kernels"] - kernels0   # kernels the timed steps' graphs ran

    # ---------------- the same steps again on the twin, kernel by kernel
    A.check(lib, lib.fivo_profile(twin.h, 1), "profile")
    kt = A.FivoKernelTimes()
    lib.fivo_profile_read(twin.h, C.byref(kt), 1)
    tau_r = tau_start
    for k in range(args.steps):
        l2_flush()
        tau_r = step_on(twin.h, tau_r, 1)
    lib.fivo_profile_read(twin.h, C.byref(kt), 1)
    clk.__exit__(None, None, None)
    if plain is None and tau_r != tau:
        raise RuntimeError("the profiled replay left the timed trajectory")
    twin.close()
    forms = None
    if form32 is not None:
        import numpy as np
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        tau_f = tau_start
        torch.cuda.synchronize()
        for k in range(args.steps):
            l2_flush()
            e0[k].record(stream)
            tau_f = step_on(form32.h, tau_f, 1)
            e1[k].record(stream)
        torch.cuda.synchronize()
        ms32 = sum(a_.elapsed_time(b_) for a_, b_ in zip(e0, e1))
        pw, pf = w.primitives(), form32.primitives()
        sx, sy = g.interior()
        okm = ((pw["ok"] == 1) & (pf["ok"] == 1)).reshape(g.Nxtot, g.Nytot)[sx, sy]
        Tw = np.exp(pw["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy][okm]
        Tf = np.exp(pf["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy][okm]
        forms = {"fp32_faces": {"value": args.steps * nint / (ms32 / 1e3), "ms_per_step": ms32 / args.steps,
                                "L2_T_vs_fp64_after_window": l2_rel(Tf, Tw),
                                "note": "the same window replayed from a device clone with the face pass in "
                                        "FP32 (fivo_ctx_set_precision); --fp32-faces makes it the headline"}}
        form32.close()
    learned = None
    vs_plain = None
    if plain is not None:
        import numpy as np
        pw = w.primitives()
        Uw = w.get_state()
        tau_p = tau_start
        for k in range(args.steps):
            tau_p = step_on(plain.h, tau_p, 1)
        pp = plain.primitives()
        Up = plain.get_state()
        sx, sy = g.interior()
        okm = ((pw["ok"] == 1) & (pp["ok"] == 1)).reshape(g.Nxtot, g.Nytot)[sx, sy]

        def inner(p, key):
            return p[key].reshape(g.Nxtot, g.Nytot)[sx, sy][okm]
        iP = m.layout.idx("pixx")
        piw = Uw.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, iP:iP + 3][okm]
        pip = Up.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, iP:iP + 3][okm]
        iN = m.layout.idx("nux")
        vs_plain = {"steps": args.steps, "tau": tau, "tau_plain": tau_p,
                    "L2_T": l2_rel(np.exp(inner(pw, "yT")), np.exp(inner(pp, "yT"))),
                    "Linf_T": float(np.max(np.abs(np.exp(inner(pw, "yT")) - np.exp(inner(pp, "yT"))) /
                                           np.exp(inner(pp, "yT")))),
                    "L2_ux": l2_rel(inner(pw, "ux"), inner(pp, "ux")),
                    "L2_uy": l2_rel(inner(pw, "uy"), inner(pp, "uy")),
                    "L2_pi": l2_rel(piw, pip), "L2_n": l2_rel(inner(pw, "n"), inner(pp, "n"))}
        plain.close()
    if guess is not None:
        st = newton_stats(w)
        learned = dict(ginfo)
        learned.update({
            "accept_rate": st["ok_learn"] / max(1, st["n_learn"]),
            "fallback_rate": 1.0 - st["ok_learn"] / max(1, st["n_learn"]),
            "updates_per_cell": (st["it_learn"] + st["it_fb"]) / max(1, st["n_learn"]),
            "slow_pass_cells_per_step": st["deferred"] / args.steps})
    clocks = clk.summary()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = args.steps * nint * world / (ms_max / 1e3)

    # ---------------- end to end through the C ABI, state in pinned host memory
    Uh = torch.empty((g.Ntot, m.nv), dtype=torch.float64, pin_memory=True)
    Up = C.cast(Uh.data_ptr(), C.POINTER(C.c_double))
    lib.fivo_download_state(w.h, Up, m.nv, g.Ntot)
    e2e_steps = max(1, min(args.steps, 10))
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(e2e_steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(e2e_steps):
        l2_flush()
        ev0[k].record(stream)
        A.check(lib, lib.fivo_upload_state(w.h, Up, m.nv, g.Ntot), "upload")
        advance(1)
        A.check(lib, lib.fivo_download_state(w.h, Up, m.nv, g.Ntot), "download")
        ev1[k].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a_.elapsed_time(b_) for a_, b_ in zip(ev0, ev1))
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    e2e_value = e2e_steps * nint * world / (float(t.item()) / 1e3)
    state_bytes = g.Ntot * m.nv * 8

    # ---------------- the whole configured run, tau0 -> TAU_END, from the initial state
    full_run = None
    if init is not None:
        ev = []
        tau_f = TAU0
        torch.cuda.synchronize()
        while tau_f < TAU_END - 1e-12:
            l2_flush()
            e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0_.record(stream)
            A.check(lib, lib.fivo_advance(init.h, tau_f, TAU_END, CFL, CFLTAU, A.FIVO_SSPRK3, A.FIVO_BC_OUTFLOW, 1,
                                          C.byref(res)), "fivo_advance")
            e1_.record(stream)
            if not res.ok:
                raise RuntimeError(f"the full run failed a step at tau={tau_f}")
            tau_f = res.tau
            ev.append((e0_, e1_))
        torch.cuda.synchronize()
        fms = sum(a_.elapsed_time(b_) for a_, b_ in ev)
        t = torch.tensor([fms], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fms = float(t.item())
        full_run = {"value": len(ev) * nint * world / (fms / 1e3), "unit": UNIT, "steps": len(ev),
                    "tau": [TAU0, tau_f], "ms_per_step": fms / len(ev),
                    "note": "the configured run tau0 -> 10 fm/c from a device copy of the initial state, "
                            "per-step CUDA events, L2 flushed between steps"}
        init.close()

    # ---------------- roofline of the dominant kernel class
    classes = A.KERNEL_CLASSES
    timed = [c for c in classes if c not in ("other", "unused")]
    tot = {c: kt.ms[classes.index(c)] for c in classes if c != "unused"}
    dom = max(timed, key=lambda c: tot[c])
    di = classes.index(dom)
    avg_ms = kt.ms[di] / max(1, kt.launches[di])
    units_launch = kt.units[di] / max(1, kt.launches[di])
    bytes_launch = algorithmic_bytes_per_unit(dom, m.nv) * units_launch
    peak, peak_kind = measured_peaks()
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    traffic = traffic_from_profiles(dom)
    per_class = {}
    for c in timed:
        i = classes.index(c)
        if kt.launches[i] == 0:
            continue
        b = algorithmic_bytes_per_unit(c, m.nv) * kt.units[i]
        per_class[c] = {"launches": int(kt.launches[i]), "ms": kt.ms[i],
                        "share": kt.ms[i] / max(1e-30, sum(tot.values())),
                        "units_per_launch": kt.units[i] / kt.launches[i],
                        "gbs": b / (kt.ms[i] / 1e3) / 1e9 if kt.ms[i] > 0 else None}
    for c in per_class:
        fp = from_profiles(c, "fp64_pipe_active_pct")
        if fp is not None:
            per_class[c]["fp64_pipe_active_pct_ncu"] = fp
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": dom, "peak_source": peak_kind,
            "bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms, "kernels": per_class,
            "fp64_pipe_active_pct_ncu": from_profiles(dom, "fp64_pipe_active_pct"),
            "note": "FP64 Newton/EOS kernels, bound by FP64 latency, not bytes: the bytes-based fraction per "
                    "the contract, and the FP64-pipe activity of the same kernel from the committed ncu "
                    "summary (profiles/<class>_kernel_traffic.txt)"}

    w.close()
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded MC-Glauber event)",
        "config": {"workload": WORKLOAD, "grid": [N_CELLS, N_CELLS], "box_fm": BOX, "tau0": TAU0,
                   "tau_window": [tau_start, tau], "integrator": "ssprk3", "cfl": CFL, "cfltau": CFLTAU,
                   "events_per_gpu": 1, "seed": SEED, "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas{world}",
                   "face_pass_xy": ["global", "global"] if graphs else face_pass,
                   "launch": ("each step's two launch sequences replayed as CUDA graphs on the stream "
                              "(fivo_ctx_set_graphs); the per-kernel roofline times come from the same "
                              "steps replayed kernel by kernel") if graphs else "kernel by kernel"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes, "steps": e2e_steps},
        "full_run": full_run,
        "gpu_launches": int(graph_kernels) if graphs else int(kt.total_launches),
        "roofline": roof,
        "clocks": clocks,
    }
    if vs_plain is not None:
        line["vs_plain_fp64"] = vs_plain
    if forms is not None:
        line["forms"] = forms
    if args.fp32_faces:
        line["config"]["workload"] += "_fp32_faces"
        line["dtype"] = "f64 (faces f32)"
    if learned is not None:
        line["learned_guess"] = learned
        line["config"]["workload"] += "_learned_guess"
        line["config"]["recovery"] = ("learned MLP guess (BF16 tcgen05, FP32 accumulate), fallback to the "
                                      "plain warm start; trained on seeds " + str(list(GUESS_SEEDS)))
    if world == 1 and not args.no_forms and guess is None and not args.fp32_faces and args.batch_events > 0:
        try:
            line["metric_comparison"] = batch_forms(lib, m, args.batch_events, args.batch_steps, value)
            line["metric_summary"] = metric_summary(line["metric_comparison"])
        except Exception as exc:   # the single-event line above stands on its own
            line["metric_comparison"] = {"error": f"{type(exc).__name__}: {exc}"}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_steps)
    return line


# ----------------------------------------------------------------------------- the metric's comparison

def _batch_fields(b, m):
    """T, pibar = pi^eta_eta/(e+P) and the shear rows of every event's interior, and
    the recovered-cell mask, concatenated in event order"""
    import numpy as np
    out = {"T": [], "pibar": [], "pi": [], "ok": []}
    iP, iE = m.layout.idx("pixx"), m.layout.idx("pieta")
    for e, g in zip(b.events, b.grids):
        p = e.primitives()
        U = e.get_state()
        sx, sy = g.interior()
        out["ok"].append((p["ok"] == 1).reshape(g.Nxtot, g.Nytot)[sx, sy].ravel())
        out["T"].append(np.exp(p["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy].ravel())
        wpl = (p["e"] + p["P"]).reshape(g.Nxtot, g.Nytot)[sx, sy].ravel()
        Ur = U.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy]
        out["pibar"].append(Ur[..., iE].ravel() / wpl)
        out["pi"].append(Ur[..., iP:iP + 3].reshape(-1, 3))
    return {k: np.concatenate(v) for k, v in out.items()}


def metric_summary(mc):
    """The metric's own ratio read off the comparison: batched learned+FP32 (the learned
    guess on the deferred cells, FP32, lockstep) against plain FP64, both unbatched (the
    events one at a time) and batched (one stream per event), with its accuracy, and the
    best form beside it"""
    def val(form):
        row = mc.get(form)
        return row.get("value") if isinstance(row, dict) else None

    head = "learned_deferred_fp32_lockstep"
    out = {"form": head, "value": val(head), "plain_unbatched": val("plain_fp64_one_event_at_a_time"),
           "plain_batched": val("plain_fp64"), "best_form": mc.get("best_form"),
           "best_value": val(mc.get("best_form")) if mc.get("best_form") else None}
    if out["value"] and out["plain_unbatched"]:
        out["vs_plain_unbatched"] = out["value"] / out["plain_unbatched"]
    if out["value"] and out["plain_batched"]:
        out["vs_plain_batched"] = out["value"] / out["plain_batched"]
    row = mc.get(head) if isinstance(mc.get(head), dict) else {}
    for k in ("L2_T", "L2_pibar", "meets_L2T_1e-6"):
        if k in row:
            out[k] = row[k]
    return out


def _fields_digest(f):
    """SHA-256 of the bits of T, pibar and the shear rows (bitwise comparison of two batches)"""
    import hashlib
    h = hashlib.sha256()
    for k in ("T", "pibar", "pi"):
        h.update(f[k].tobytes())
    return h.hexdigest()


LOCKSTEP_FORMS = ("plain_fp64_lockstep", "fp32_lockstep", "learned_fp32_lockstep", "learned_deferred_fp32_lockstep",
                  "plain_fp64_lockstep_nograph")


def batch_forms(lib, m, nevents, steps, single_value, warmup=18):
    """The metric's comparison on one GPU: the same nevents seeded events (the
    event-by-event sizes, device IC, seed 1000 + k) advanced in plain FP64, in FP32
    (face pass and relaxation sources), and with the learned guess plus FP32, the
    guess used for every cell or for the cells the warm start defers, each with one
    stream per event; then plain FP64, FP32 and the two learned+FP32 forms in
    lockstep (one launch per kernel over all events, replayed from CUDA graphs, the
    schedule tuned on the first 16 warm-up steps), plain lockstep without graphs,
    and the plain path unbatched (the events one at a time, each alone on the GPU). Zone-updates/s of each (host
    wall clock around the synchronous batch call), each form's L2(T), L2(pibar) and
    L2(pi) against the plain run, and for the lockstep forms whether every event's
    fields equal those of the stream batch of the same precision bit for bit."""
    import numpy as np
    import torch

    from fivo2d import _abi as A
    from fivo2d.events import event_grids
    from fivo2d.guess import newton_stats
    from fivo2d.solver import GPUBatch2D

    grids = event_grids(nevents)
    cells = sum(g.Nx * g.Ny for g in grids)
    g384, _ = model_and_grid()
    guess, ginfo = train_guess(lib, m, g384)
    out = {"events": nevents, "steps": steps, "warmup": warmup, "grids": sorted({g.Nx for g in grids}),
           "zone_updates_per_step": cells, "single_event_plain_fp64": single_value,
           "timing": "host wall clock around the synchronous batch call"}
    ref = None
    stream_fields = {}
    for form in ("plain_fp64", "fp32", "learned_fp32", "learned_deferred_fp32") + LOCKSTEP_FORMS + (
            "plain_fp64_one_event_at_a_time",):
        sequential = form == "plain_fp64_one_event_at_a_time"
        b = GPUBatch2D(m, grids, nworkers=1 if sequential else 0, lib=lib)
        lockstep = form in LOCKSTEP_FORMS
        if lockstep:
            b.set_lockstep(True, graphs=not form.endswith("nograph"), tune=True)
        for k, e in enumerate(b.events):
            e.glauber_ic(TAU0, 1000 + k)
            e.rhs(TAU0)
            if not form.startswith("plain_fp64"):
                e.set_precision(A.FIVO_PRECISION_FP32)
            if form.startswith("learned_fp32"):
                guess.attach(e, A.FIVO_GUESS_EVERY_CELL)
            if form.startswith("learned_deferred_fp32"):
                guess.attach(e, A.FIVO_GUESS_DEFERRED)
        taus = [TAU0] * len(grids)

        def adv(n):
            nonlocal taus
            r = b.advance(taus, 1e9, CFL, CFLTAU, A.FIVO_SSPRK3, max_steps=n)
            if not all(x["ok"] and x["nsteps"] == n for x in r):
                raise RuntimeError(f"a batch event failed a step ({form})")
            taus = [x["tau"] for x in r]

        adv(warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        adv(steps)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        row = {"value": steps * cells / dt, "unit": UNIT, "ms_per_step": 1e3 * dt / steps,
               "schedule": "lockstep" if lockstep else ("one event at a time (the plain path, unbatched)"
                                                         if sequential else "stream per event")}
        f = _batch_fields(b, m)
        if sequential:
            row["bitwise_equal_stream_batch"] = _fields_digest(f) == stream_fields["plain_fp64"]
        elif lockstep:
            info = b.lockstep_info()
            row["lockstep"] = {k: info[k] for k in ("graphs", "chosen", "candidates", "fallbacks")}
            twin = stream_fields[form.replace("_lockstep", "").replace("_nograph", "")]
            row["bitwise_equal_stream_batch"] = _fields_digest(f) == twin
        else:
            stream_fields[form] = _fields_digest(f)
        if ref is None:
            ref = f
        else:
            ok = ref["ok"] & f["ok"]
            row["L2_T"] = l2_rel(f["T"][ok], ref["T"][ok])
            row["Linf_T"] = float(np.max(np.abs(f["T"][ok] - ref["T"][ok]) / ref["T"][ok]))
            row["L2_pibar"] = l2_rel(f["pibar"][ok], ref["pibar"][ok])
            row["L2_pi"] = l2_rel(f["pi"][ok], ref["pi"][ok])
            row["speedup_vs_plain_batch"] = row["value"] / out["plain_fp64"]["value"]
            row["meets_L2T_1e-6"] = bool(row["L2_T"] <= 1e-6)
        if form.startswith("learned"):
            st = {}
            for e in b.events:
                for key, v in newton_stats(e).items():
                    st[key] = st.get(key, 0) + v
            row["guess"] = dict(ginfo if form == "learned_fp32" else {}, mode=form,
                                guesses=st["n_learn"], accept_rate=st["ok_learn"] / max(1, st["n_learn"]),
                                updates_per_guess=(st["it_learn"] + st["it_fb"]) / max(1, st["n_learn"]),
                                full_recoveries=st["deferred"])
        out[form] = row
        b.close()
    guess.close()
    out["plain_batch_vs_single_event"] = out["plain_fp64"]["value"] / single_value
    best = max((f for f in out if isinstance(out[f], dict) and "value" in out[f]), key=lambda f: out[f]["value"])
    out["best_form"] = best
    out["best_form_vs_plain_batch"] = out[best]["value"] / out["plain_fp64"]["value"]
    seq = out["plain_fp64_one_event_at_a_time"]["value"]
    for f in out:
        if isinstance(out[f], dict) and "value" in out[f]:
            out[f]["speedup_vs_plain_one_event_at_a_time"] = out[f]["value"] / seq
    return out


# ----------------------------------------------------------------------------- event batches

def run_batch(args):
    """The event-by-event workload: args.events seeded MC-Glauber events with N drawn
    from {96, 128, 192, 256, 320, 400} (dx = 30/384 fm), split over the ranks by cell
    count; each rank advances its share with the batch API (one stream per event,
    library worker threads). Not the default line: the headline config is the single
    384^2 event."""
    import torch

    from fivo2d import _abi as A
    from fivo2d.events import event_grids, shard_events
    from fivo2d.solver import GPUBatch2D

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    lib = A.load_library()
    _, m = model_and_grid()
    grids = event_grids(args.events)
    mine = shard_events([g.Nx * g.Ny for g in grids], world, rank)
    my_grids = [grids[k] for k in mine]
    guess, ginfo = (None, None)
    if args.guess:
        g384, _ = model_and_grid()
        guess, ginfo = train_guess(lib, m, g384)
    b = GPUBatch2D(m, my_grids, nworkers=args.workers, lib=lib)
    if args.lockstep:
        b.set_lockstep(True, graphs=True, tune=True)
    for e, k in zip(b.events, mine):
        e.glauber_ic(TAU0, 1000 + k)      # the MC-Glauber IC built on the device
        e.rhs(TAU0)
        if guess is not None:
            guess.attach(e)
        if args.fp32_faces:
            e.set_precision(A.FIVO_PRECISION_FP32_FACES)
    taus = [TAU0] * len(mine)

    def adv(n):
        nonlocal taus
        r = b.advance(taus, 1e9, CFL, CFLTAU, A.FIVO_SSPRK3, max_steps=n)
        if not all(x["ok"] and x["nsteps"] == n for x in r):
            raise RuntimeError("a batch event failed a step")
        taus = [x["tau"] for x in r]

    adv(max(args.warmup, 18) if args.lockstep else args.warmup)   # lockstep: the 16 tuning steps are warm-up
    if guess is not None:
        from fivo2d.guess import newton_stats
        for e in b.events:
            newton_stats(e, reset=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    adv(args.steps)          # returns when every event's stream has finished
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    cells = sum(g.Nx * g.Ny for g in my_grids)
    t = torch.tensor([dt, float(cells)], dtype=torch.float64, device="cuda")
    if dist:
        tmax = t[:1].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        csum = t[1:].clone()
        dist.all_reduce(csum, op=dist.ReduceOp.SUM)
        dt, cells_all = float(tmax.item()), float(csum.item())
    else:
        cells_all = float(cells)
    value = args.steps * cells_all / dt
    learned = None
    if guess is not None:
        tot = {}
        for e in b.events:
            for key, v in newton_stats(e).items():
                tot[key] = tot.get(key, 0) + v
        learned = dict(ginfo)
        learned.update({"accept_rate": tot["ok_learn"] / max(1, tot["n_learn"]),
                        "updates_per_cell": (tot["it_learn"] + tot["it_fb"]) / max(1, tot["n_learn"]),
                        "slow_pass_cells_per_step": tot["deferred"] / args.steps})
    # end to end: the host holds every event's state; each step uploads, advances, downloads
    hosts = [e.get_state() for e in b.events]
    e2e_steps = max(1, min(args.steps, 5))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for e, U in zip(b.events, hosts):
            e.set_state(U)
        adv(1)
        hosts = [e.get_state() for e in b.events]
    torch.cuda.synchronize()
    e2e_dt = time.perf_counter() - t0
    t = torch.tensor([e2e_dt], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e = e2e_steps * cells_all / float(t.item())
    state_bytes = sum(g.Ntot for g in my_grids) * m.nv * 8
    b.close()
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return None
    sizes = sorted({g.Nx for g in grids})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded MC-Glauber events)",
        "config": {"workload": f"batch_{args.events}_events_N{sizes[0]}-{sizes[-1]}_dx0.078125_ssprk3_lhrg",
                   "events": args.events, "grids": [g.Nx for g in grids], "tau0": TAU0, "integrator": "ssprk3",
                   "cfl": CFL, "cfltau": CFLTAU, "workers": args.workers, "parallelism": f"events over {world} GPUs",
                   "timing": "host wall clock around the synchronous batch call",
                   "schedule": "lockstep (one launch per kernel over all events, CUDA graphs, tuned)"
                   if args.lockstep else "one stream per event",
                   "l2": "inputs (all events' state) larger than L2"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "steps": e2e_steps},
    }
    if args.fp32_faces:
        line["config"]["workload"] += "_fp32_faces"
        line["dtype"] = "f64 (faces f32)"
    if learned is not None:
        line["learned_guess"] = learned
        line["config"]["workload"] += "_learned_guess"
    if args.lockstep:
        line["config"]["workload"] += "_lockstep"
    return line


# ----------------------------------------------------------------------------- freeze-out

def run_freezeout(args):
    """The axisymmetric control of freezeout2d.jl: the calibrated radial profile on
    200^2 cells over [-18, 18] fm, evolved from tau 0.4 to 16 in chunks of 0.02 with
    the freeze_surface model, the T = 0.156 surface recorded after every chunk, then
    the Cooper-Frye pion yield over it. The 1-D calibration it should reproduce is
    N_pi = 1339.63 (freezeout2d.jl:7-10, 73-75)."""
    import numpy as np
    import torch

    import fivo2d
    from fivo2d import _abi as A
    from fivo2d.freezeout import axisym_fields, cf_params, freeze_model, freeze_surface
    from fivo2d.solver import GPUWork2D, set_cells

    lib = A.load_library()
    g = fivo2d.make_grid2d(200, 200, xmax=18.0, ymax=18.0)
    m = freeze_model()
    T, a, ux, uy = axisym_fields(g, ROOT / "tests" / "golden" / "initial_profiles_physical.csv")
    U, _ = set_cells(m, 0.4, T, a, ux, uy, lib=lib)
    w = GPUWork2D(m, g, lib=lib)
    w.set_state(U)
    w.finalize_ic(0.4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fo, chunks = freeze_surface(w, 0.4, 16.0, dtau=0.02)
    t1 = time.perf_counter()
    s = fo.surface()
    p = cf_params()
    fo.pion_yield(p)                       # warm-up
    reps = 5
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    for _ in range(reps):
        NB, Nb, negf = fo.pion_yield(p)
    t3 = time.perf_counter()
    ncells = int(np.sum(~np.isnan(s["tau_fo"])))
    evals = ncells * p.n_pt * p.n_phi * p.n_eta
    cf_s = (t3 - t2) / reps
    return {
        "metric": "Cooper-Frye integrand evaluations/s (freeze-out surface of the axisymmetric control)",
        "value": evals / cf_s, "unit": "evaluations/s", "n_gpus": 1, "higher_is_better": True,
        "dtype": "f64", "data": "the reference's calibrated radial profile (data/initial_profiles_physical.csv)",
        "config": {"workload": "freezeout_axisym_200x200_box18_tau0.4-16_dtau0.02_Tfo0.156",
                   "grid": [200, 200], "cf_grid": [p.n_pt, p.n_phi, p.n_eta],
                   "timing": "host wall clock around synchronous calls"},
        "freezeout": {"dNdy_boltzmann": NB, "dNdy_bose": Nb, "negative_dsigma_fraction": negf,
                      "calibration_1d": 1339.63, "chunks": chunks, "surface_run_s": t1 - t0,
                      "cooper_frye_ms": 1e3 * cf_s, "cells_hot": s["nhot"], "cells_frozen": s["nfroze"],
                      "reheated_after_freezing": s["refroze"]},
    }


# ----------------------------------------------------------------------------- mixed precision at scale

def _precision_fields(b):
    """T, u^x, u^y, pibar = pi^eta_eta/(e+P) and n of every event's interior, and the
    recovered-cell mask, one array per event"""
    import numpy as np
    m = b.model
    iE = m.layout.idx("pieta")
    out = []
    for e, g in zip(b.events, b.grids):
        p = e.primitives()
        U = e.get_state()
        sx, sy = g.interior()
        r = lambda a: np.asarray(a).reshape(g.Nxtot, g.Nytot)[sx, sy].ravel()  # noqa: E731
        wpl = r(p["e"]) + r(p["P"])
        out.append({"ok": r(p["ok"]) == 1, "T": np.exp(r(p["yT"])), "ux": r(p["ux"]), "uy": r(p["uy"]),
                    "pibar": U.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, iE].ravel() / wpl, "n": r(p["n"])})
    return out


def run_precision(args):
    """The mixed-precision form at scale: the viscous event's physics on 512^2 cells over
    [-15, 15] fm, args.precision_events seeded events (device IC, seed 1000 + k),
    advanced to tau = 4 and on to 10 fm/c in plain FP64 (bitwise the oracle), with the
    FP32 face pass, and with the face pass and the relaxation's sources in FP32. Per
    event and field (T, u^x, u^y, pibar, n) the relative L2 and Linf deviation from the
    FP64 run over the cells recovered in both; the line gives the median and the
    largest over the events, and the time of each form's run."""
    import numpy as np
    import torch

    import fivo2d
    from fivo2d import _abi as A
    from fivo2d.solver import GPUBatch2D

    lib = A.load_library()
    _, m = model_and_grid()
    nev = args.precision_events
    grids = [fivo2d.make_grid2d(512, 512, xmax=15.0, ymax=15.0) for _ in range(nev)]
    fields, runs = {}, {}
    for name, mode in (("fp64", A.FIVO_PRECISION_FP64), ("fp32_faces", A.FIVO_PRECISION_FP32_FACES),
                       ("fp32", A.FIVO_PRECISION_FP32)):
        b = GPUBatch2D(m, grids, lib=lib)
        for k, e in enumerate(b.events):
            e.glauber_ic(TAU0, 1000 + k)
            e.set_precision(mode)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r4 = b.run(TAU0, 4.0, CFL, CFLTAU, A.FIVO_SSPRK3)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if not all(x["ok"] and x["tau"] == 4.0 for x in r4):
            raise RuntimeError(f"an event failed before tau = 4 ({name})")
        f4 = _precision_fields(b)
        r10 = b.advance([x["tau"] for x in r4], 10.0, CFL, CFLTAU, A.FIVO_SSPRK3, max_steps=10 ** 9)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if not all(x["ok"] and x["tau"] == 10.0 for x in r10):
            raise RuntimeError(f"an event failed before tau = 10 ({name})")
        fields[name] = {4.0: f4, 10.0: _precision_fields(b)}
        steps = sum(x["nsteps"] for x in r4) + sum(x["nsteps"] for x in r10)
        runs[name] = {"run_s": t2 - t0, "to_tau4_s": t1 - t0, "steps": steps,
                      "zone_updates_per_s": steps * 512 * 512 / (t2 - t0)}
        b.close()
    errors = {}
    for name in ("fp32_faces", "fp32"):
        errors[name] = {}
        for tau in (4.0, 10.0):
            per = {k: ([], []) for k in ("T", "ux", "uy", "pibar", "n")}
            for a, b_ in zip(fields[name][tau], fields["fp64"][tau]):
                ok = a["ok"] & b_["ok"]
                for k in per:
                    x, y = a[k][ok], b_[k][ok]
                    per[k][0].append(float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300)))
                    per[k][1].append(float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300)))
            errors[name][f"tau_{tau:g}"] = {k: {"L2_median": float(np.median(v[0])), "L2_max": float(np.max(v[0])),
                                                "Linf_median": float(np.median(v[1])),
                                                "Linf_max": float(np.max(v[1]))} for k, v in per.items()}
    return {
        "metric": "relative L2 / Linf deviation of the FP32 forms from FP64 (T, u^x, u^y, pibar, n) at tau = 4, 10",
        "value": errors["fp32"]["tau_4"]["T"]["L2_median"], "unit": "relative L2(T), median over events, tau = 4",
        "n_gpus": 1, "higher_is_better": False, "dtype": "f32/f64", "data": "synthetic (seeded MC-Glauber events)",
        "config": {"workload": f"precision_{nev}x512x512_box15_tau0.6-10_ssprk3", "events": nev, "grid": [512, 512],
                   "reference": "the FP64 run, bitwise the oracle's arithmetic"},
        "errors": errors, "runs": runs,
    }


# ----------------------------------------------------------------------------- CPU legs

def oracle_event():
    sys.path.insert(0, str(ROOT / "tests"))
    import _oracle as O
    g, m = model_and_grid()
    T, a, ux, uy = ic_fields(g, SEED)
    U, ok = O.set_cells(m.params, TAU0, T, a, ux, uy, m.nv)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(TAU0)
    return O, g, m, o


def oracle_steps(o, tau, n):
    """n iterations of run_sim_2d!'s loop on the oracle (oracle_advance)."""
    from fivo2d import _abi as A
    r = o.advance(tau, 1e9, CFL, CFLTAU, A.FIVO_SSPRK3, 0, n)
    if not r["ok"] or r["nsteps"] != n:
        raise RuntimeError("oracle step failed")
    return r["tau"]


def cpu_baseline(nsteps):
    O, g, m, o = oracle_event()
    o.rhs(TAU0)
    t0 = time.perf_counter()
    oracle_steps(o, TAU0, nsteps)
    dt = time.perf_counter() - t0
    return {"value": nsteps * g.Nx * g.Ny / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"{nsteps} run_sim_2d! steps of the {N_CELLS}x{N_CELLS} event from tau0 (oracle/, OpenMP)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return None
    O, g, m, o = oracle_event()
    o.rhs(TAU0)
    tau = TAU0
    tau = oracle_steps(o, tau, args.warmup)
    t0 = time.perf_counter()
    oracle_steps(o, tau, args.steps)
    dt = time.perf_counter() - t0
    value = args.steps * g.Nx * g.Ny / dt
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded MC-Glauber event)",
        "config": {"workload": WORKLOAD, "grid": [N_CELLS, N_CELLS], "box_fm": BOX, "tau0": TAU0,
                   "integrator": "ssprk3", "cfl": CFL, "cfltau": CFLTAU, "seed": SEED},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{args.steps} run_sim_2d! steps after {args.warmup} warm-up steps; "
                                   "reference is Julia (not installed), timed via its C++ restatement"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="event", choices=["event", "batch", "freezeout", "precision"],
                    help="event: the 384^2 viscous event (default); batch: many uneven events")
    ap.add_argument("--events", type=int, default=32, help="batch workload: number of events")
    ap.add_argument("--precision-events", type=int, default=64, help="precision workload: number of 512^2 events")
    ap.add_argument("--workers", type=int, default=0, help="batch workload: host threads (0: library default)")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the FP32-faces replay and the batched forms comparison of the default line")
    ap.add_argument("--no-full-run", action="store_true", help="skip the full tau0 -> 10 fm/c figure")
    ap.add_argument("--batch-events", type=int, default=256, help="events of the metric's batched comparison")
    ap.add_argument("--batch-steps", type=int, default=30, help="timed steps of the batched comparison")
    ap.add_argument("--fp32-faces", action="store_true",
                    help="the mixed-precision form: the face pass in FP32 (fivo_ctx_set_precision)")
    ap.add_argument("--graphs", action="store_true",
                    help="event workload: replay each step's launch sequences as CUDA graphs "
                         "(fivo_ctx_set_graphs) instead of launching kernel by kernel")
    ap.add_argument("--lockstep", action="store_true",
                    help="batch workload: lockstep mode (one launch per kernel over all events, CUDA graphs)")
    ap.add_argument("--guess", action="store_true",
                    help="train the learned recovery guess on other seeded events and time with it attached")
    args = ap.parse_args()
    if args.workload in ("batch", "precision"):
        # more hardware queues for the per-event streams (read when CUDA initialises)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.impl == "reference":
        line = run_reference(args)
    elif args.workload == "batch":
        line = run_batch(args)
    elif args.workload == "freezeout":
        line = run_freezeout(args)
    elif args.workload == "precision":
        line = run_precision(args)
    else:
        line = run_gpu(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
