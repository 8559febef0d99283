#!/usr/bin/env python
"""Benchmark of the split HLLD sweep: FP64 ideal-MHD cell-updates/s at 256^3.

Workload (one "step" = one iteration of PIERNIK's main loop, i.e. time_step +
fluid_update = two time steps of X,Y,Z then Z,Y,X sweeps, each sweep two RK2
stages): decaying ideal-MHD turbulence on one periodic 256^3 block, HLLD
fluxes with GLM divergence cleaning, moncen limiter, CFL 0.5, FP64, seeded
synthetic initial state (density 1 + 1% white noise, velocity from Fourier
modes |k| = 1..4 with amplitude k^-2 at rms Mach 1, B = (0.2,0,0) plus 10%
divergence-free modes, psi = 0).  A cell-update is one cell advanced by one
dt, so one step is 2 * 256^3 cell-updates.

Arms:
  default            the CUDA library through Simulation.run (state resident in HBM)
  --impl reference   the reference's CPU algorithm (the oracle port in oracle/,
                     the Fortran reference cannot be compiled here) on all host
                     threads, on the same 256^3 workload (each step one main-loop
                     iteration of it, a few seconds of CPU work)

Multi-GPU (torchrun): every rank advances its own 256^3 replica (weak scaling);
timing is the max over ranks of CUDA-event time on the library's stream.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 MHD cell-updates/s at 256^3 on 1 B200; adjoint-gradient cost ÷ forward step"
UNIT = "cell-updates/s"
NVAR = 9                         # dn, mx, my, mz, en, Bx, By, Bz, psi
# DRAM bytes per cell of one sweep launch, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the TMA-staged y sweep of a
# 128^3 block (181 MB with guards, above the 126 MB L2) in the tolerance
# arithmetic: 161.11 MB read + 113.07 MB written over 128^3 cells.  Traffic
# grows with the cell count, so the full-size figure is this times n^3.
TRAFFIC_BYTES_PER_CELL = (161.105664e6 + 113.074688e6) / 128 ** 3
# FP64 flops per cell of one sweep (both RK2 stages) without halo
# recomputation: 2 x DFMA + DMUL + DADD thread instructions (ncu
# sm__sass_thread_inst_executed_op_{dfma,dmul,dadd}_pred_on.sum) of the
# TMA-staged whole-pencil x sweep of a 128^3 block over its 128^3 cells, in
# the bit-exact arithmetic (0.8408 G DFMA, 0.9312 G DMUL, 0.9150 G DADD) and in
# the tolerance arithmetic (0.7899 G DFMA, 0.5277 G DMUL, 0.4303 G DADD)
FP64_FLOP_PER_CELL_SWEEP = (2 * 840755524 + 931189733 + 915036464) / 128 ** 3
FP64_FLOP_PER_CELL_SWEEP_FMA = (2 * 789901529 + 527723486 + 430337951) / 128 ** 3
ARITH_NOTE = {
    "fma": "fma: multiply-add contraction and hoisted reciprocals in the fused sweep; agrees with the "
           "reference's arithmetic to <= 1e-12 relative per step and <= 1e-9 after 100 steps (tests/test_gpu_fma.py)",
    "bitexact": "bitexact: the reference's operation order and rounding, equal to the oracle bit for bit",
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--adj-steps", type=int, default=8)
    p.add_argument("--tune-log", default=None)
    p.add_argument("--workload", default="mhd256",
                   choices=["mhd256", "batched", "batched-independent", "adjoint", "ot-gradient",
                            "batched-adjoint", "unsplit"],
                   help="mhd256: the headline 256^3 MHD block; batched: 512 uneven 3-fluid blocks; "
                        "adjoint: gradient of --steps steps of the MHD block at --n; ot-gradient: the "
                        "differentiable Orszag-Tang workload (512^2, K = 100) with its FD check; "
                        "batched-adjoint: gradients of 64 stacked 128^3 turbulence instances (K = 50)")
    p.add_argument("--instances", type=int, default=64)
    p.add_argument("--group", type=int, default=8, help="instances stacked per handle (batched-adjoint)")
    p.add_argument("--k", type=int, default=50, help="time steps differentiated (batched-adjoint)")
    p.add_argument("--nblocks", type=int, default=512)
    p.add_argument("--arith", default="both", choices=["both", "fma", "bitexact"],
                   help="arithmetic of the fused sweep; both: the headline in fma, bitexact beside it")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the bounded C3 / C4 / C5 measurements appended to the headline line")
    p.add_argument("--tiles", default=None,
                   help="fix fused-sweep tiles instead of autotuning, e.g. 'x:1,88,3;y:4,56,2;z:4,56,2' (P,L,variant)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_config(n):
    return {"workload": f"3D ideal-MHD decaying turbulence, one periodic {n}^3 block, HLLD + GLM, moncen, "
                        f"RK2, CFL 0.5, FP64", "n": n, "nvar": NVAR, "riemann": "hlld", "limiter": "moncen",
            "cfl": 0.5, "step": "time_step + fluid_update (2 dt, 6 sweeps)",
            "l2": "state %.2f GB > 126 MB L2, no flush needed" % (NVAR * 8 * (n + 8) ** 3 / 1e9)}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 7 and parts[0].isdigit():
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [int(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample(n, seed):
    """Time the oracle (reference algorithm on the CPU) on one step of the
    workload recipe at n^3; returns (cell-updates/s, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from piernik_b200 import problems
    setup, u, b, psi = problems.mhd_turbulence(n=n, seed=seed)
    ob = oracle.OracleBlock(setup, u, b, psi)
    t0 = time.perf_counter()
    ob.run(1)
    el = time.perf_counter() - t0
    return 2.0 * n ** 3 / el, el, oracle.get_threads()


def reference_arm(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from piernik_b200 import problems
    ns = args.n
    setup, u, b, psi = problems.mhd_turbulence(n=ns, seed=args.seed)
    ob = oracle.OracleBlock(setup, u, b, psi)
    # one warm-up step at most: the CPU path has no caches or kernels to load
    # beyond the first touch of its arrays
    ob.run(min(args.warmup, 1))
    t0 = time.perf_counter()
    ob.run(args.steps)
    el = time.perf_counter() - t0
    value = 2.0 * ns ** 3 * args.steps / el
    threads = oracle.get_threads()
    sample = (f"{args.steps} steps of the workload at {ns}^3 ({2 * ns ** 3 * args.steps} cell-updates, {el:.1f} s; "
              f"oracle/pk_oracle.c, OpenMP over pencils, {threads} threads); the Fortran reference has no "
              f"compiler here")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args.n), "impl": "reference",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def adjoint_cost(sim, stream, args, fwd_ms_per_step, barrier, max_over_ranks):
    """Cost of the gradient of K steps relative to K forward steps.

    backward = pk_grad_backward: recompute each checkpointed segment once
    (fused sweeps) plus one adjoint sweep kernel per forward sweep.  The ratio
    reported is backward / forward; the recorded forward (pk_grad_forward,
    which adds the checkpoint copies) is reported beside it."""
    import numpy as np
    import torch
    K = args.adj_steps
    every = max(1, int(round(np.sqrt(K))))
    st0 = sim.time_state
    # untimed warm-up of the same shape: loads the kernels, allocates the
    # checkpoints and the recomputation pool the timed gradient reuses
    sim.grad_forward(K, every)
    sim.adjoint_set(np.ones(sim.state_shape()))
    sim.grad_backward()
    sim.time_state = st0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    barrier()
    ev[0].record(stream)
    sim.grad_forward(K, every)
    ev[1].record(stream)
    ev[1].synchronize()
    lam = np.ones(sim.state_shape())
    sim.adjoint_set(lam)
    barrier()
    ev[2].record(stream)
    sim.grad_backward()
    ev[3].record(stream)
    ev[3].synchronize()
    # one adjoint sweep kernel per direction, timed alone
    st = sim.time_state
    reps = 3
    ev[4].record(stream)
    for _ in range(reps):
        for d in (1, 2, 3):
            sim.adjoint_sweep(d, st.dt, st.chspeed)
    ev[5].record(stream)
    ev[5].synchronize()
    sim.grad_release()
    sim.time_state = st0
    fwd_rec = max_over_ranks(ev[0].elapsed_time(ev[1]))
    bwd = max_over_ranks(ev[2].elapsed_time(ev[3]))
    adj_sweep = max_over_ranks(ev[4].elapsed_time(ev[5])) / (3 * reps)
    fwd = fwd_ms_per_step * K
    return {"value": bwd / fwd, "definition": "pk_grad_backward time / time of the same K forward steps (pk_run)",
            "steps": K, "checkpoint_every": every, "forward_ms": fwd, "recorded_forward_ms": fwd_rec,
            "backward_ms": bwd, "gradient_total_over_forward": (fwd_rec + bwd) / fwd,
            "adjoint_sweep_ms": adj_sweep, "fused_sweep_ms": fwd_ms_per_step / 6}


def tune_tiles(sim, args, slab, rank):
    """Fused-sweep tiles: --tiles as given, else the autotuner's picks (on a
    multi-rank run rank 0 tunes alone and every rank takes its choice)."""
    import torch
    if args.tiles:
        tiles = {}
        for item in args.tiles.split(";"):
            ax, vals = item.split(":")
            P, Lc, V = (int(x) for x in vals.split(","))
            sim.set_tile("xyz".index(ax), P, Lc, V)
            tiles[ax] = [P, Lc, V]
        return tiles
    if args.no_autotune:
        return None
    from piernik_b200.autotune import autotune
    if slab is not None:
        slab.detach()
    best = autotune(sim, reps=2, verbose=False)
    if slab is not None:
        pick = [best]
        torch.distributed.broadcast_object_list(pick, src=0)
        best = pick[0]
        for d, v in best.items():
            sim.set_tile(d, v["P"], v["L"], v["V"])
        slab.attach()
    return {"xyz"[d]: [v["P"], v["L"], v["V"], round(v["ms"], 4)] for d, v in best.items()}


def our_arm(args):
    import ctypes
    import numpy as np
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from piernik_b200 import _lib, build, problems
    from piernik_b200._lib import PK_LAYOUT_FORTRAN, PkTimeState
    from piernik_b200.sim import Simulation
    build.build()
    n = args.n
    setup, u, b, psi = problems.mhd_turbulence(n=n, seed=args.seed + rank)
    slab = None
    if world > 1:
        # weak scaling: the level is n x n x (n * world), one n^3 slab per rank,
        # z halos moved by NCCL before every z sweep, dt reduced over ranks
        from piernik_b200.slabs import SlabRank, TorchTransport
        gsetup = setup.replace(n=(n, n, n * world),
                               xmax=(setup.xmax[0], setup.xmax[1],
                                     setup.xmin[2] + world * (setup.xmax[2] - setup.xmin[2])))
        slab = SlabRank(gsetup, rank, world, TorchTransport(torch.device("cuda", local)))
        sim = slab.sim
    else:
        sim = Simulation(setup)
    sim.upload(u, b, psi)
    stream = torch.cuda.ExternalStream(sim.stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    hbm, src = peaks()
    peak64 = ctypes.c_double(0.0)
    have64 = _lib.load().pk_fp64_peak(ctypes.byref(peak64)) == 0 and peak64.value > 0
    modes = ["fma", "bitexact"] if args.arith == "both" else [args.arith]
    cell_updates = 2.0 * n ** 3 * args.steps * world
    res = {}
    for mode in modes:
        # every mode starts from the same initial state and time
        sim.upload(u, b, psi)
        sim.time_state = PkTimeState()
        sim.set_arithmetic(mode)
        tiles = tune_tiles(sim, args, slab, rank)
        sim.run(args.warmup)
        barrier()
        clocks = Clocks(local)
        sim.profile(True)
        launches0, _, _ = sim.profile_read()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.run(args.steps)
        e1.record(stream)
        e1.synchronize()
        launches1, nsweep, sweep_ms = sim.profile_read()
        sim.profile(False)
        ck = clocks.stop()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        # roofline of the fused sweep kernel (algorithmic bytes: read + write 9 planes of n^3)
        bytes_per_launch = 2.0 * NVAR * 8 * n ** 3
        launch_ms = sweep_ms / max(nsweep, 1)
        achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "traffic": TRAFFIC_BYTES_PER_CELL * n ** 3,
                    "kernel": f"k_sweep_staged / k_sweep_fused<MHD> as tuned ({mode} arithmetic; one sweep direction, "
                              "both RK2 stages)",
                    "bytes_per_launch": bytes_per_launch, "launch_ms": launch_ms, "peak_source": src}
        # the bound that limits it: FP64 issue, against the device's measured DFMA rate
        roofline_fp64 = None
        fpc = FP64_FLOP_PER_CELL_SWEEP if mode == "bitexact" else FP64_FLOP_PER_CELL_SWEEP_FMA
        if have64 and fpc:
            flops = fpc * n ** 3
            got = flops / (launch_ms / 1e3) / 1e12
            roofline_fp64 = {"bound": "fp64", "achieved": got, "peak": peak64.value, "unit": "TFLOP/s",
                             "frac": got / peak64.value, "flop_per_launch": flops,
                             "flop_count": f"FP64 flops executed per cell by the {mode} whole-pencil sweep (ncu)",
                             "peak_source": "measured (pk_fp64_peak: independent DFMA chains)"}
        res[mode] = {"value": cell_updates / (ms / 1e3), "ms_per_step": ms / args.steps, "roofline": roofline,
                     "roofline_fp64": roofline_fp64, "gpu_launches": launches1 - launches0, "clocks": ck,
                     "tiles_P_L_variant_ms": tiles}
    head = modes[0]
    sim.upload(u, b, psi)
    sim.time_state = PkTimeState()
    sim.set_arithmetic(head)
    if res[head]["tiles_P_L_variant_ms"]:
        for ax, t in res[head]["tiles_P_L_variant_ms"].items():
            sim.set_tile("xyz".index(ax), t[0], t[1], t[2])

    # end to end through the C ABI with host buffers in the reference's layout
    e2e = None
    if not args.no_e2e:
        pu = torch.empty(u.shape, dtype=torch.float64).pin_memory().numpy()
        pb = torch.empty(b.shape, dtype=torch.float64).pin_memory().numpy()
        pp = torch.empty(psi.shape, dtype=torch.float64).pin_memory().numpy()
        pu[...] = u
        pb[...] = b
        pp[...] = psi
        st0 = sim.time_state
        barrier()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            sim.upload(pu, pb, pp, layout=PK_LAYOUT_FORTRAN)
            sim.run(1)
            sim.download(layout=PK_LAYOUT_FORTRAN, out=(pu, pb, pp))
        e3.record(stream)
        e3.synchronize()
        barrier()
        ms2 = max_over_ranks(e2.elapsed_time(e3))
        nbytes = (pu.nbytes + pb.nbytes + pp.nbytes)
        e2e = {"value": cell_updates / (ms2 / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": ms2 / args.steps, "arithmetic": head,
               "path": "pk_upload(Fortran layout, pinned) + pk_run(1) + pk_download per step"}
        sim.time_state = st0

    adjoint = None
    if not args.no_adjoint and world == 1:
        # the adjoint kernels and the recomputation run in the bit-exact
        # arithmetic: compare with forward steps in that arithmetic
        ref = "bitexact" if "bitexact" in res else head
        sim.set_arithmetic(ref)
        adjoint = adjoint_cost(sim, stream, args, res[ref]["ms_per_step"], barrier, max_over_ranks)
        adjoint["forward_arithmetic"] = ref
        sim.set_arithmetic(head)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cn = n
        v, el, thr = cpu_sample(cn, args.seed)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"1 step of the workload at {cn}^3 ({2 * cn ** 3} cell-updates, {el:.1f} s) with "
                         f"oracle/pk_oracle.c on {thr} OpenMP threads"}
    sim.close()

    extras = {}
    if world == 1 and not args.no_extras:
        for name, fn in (("c3_refined", lambda: c3_refined(args, steps=2, warmup=1)),
                         ("c4_ot_gradient", lambda: c4_ot_gradient(args, ndirs=4, n=512, K=100)),
                         ("c5_batched_adjoint", lambda: c5_batched_adjoint(args, K=10, ngroups=1, warmup=1,
                                                                           steps=1))):
            try:
                extras[name] = fn()
            except Exception as e:        # an extra never costs the headline line
                extras[name] = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        r = res[head]
        out = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "arithmetic": ARITH_NOTE[head],
               "config": dict(workload_config(n), parallelism=("one block" if world == 1 else
                                                               f"{world} z-slabs of {n}^3, NCCL halo exchange"),
                              tiles_P_L_variant_ms=r["tiles_P_L_variant_ms"]),
               "roofline": r["roofline"], "roofline_fp64": r["roofline_fp64"], "cpu_baseline": cpu, "e2e": e2e,
               "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
               "adjoint_cost_ratio": adjoint}
        for mode in modes[1:]:
            out[mode] = dict(res[mode], arithmetic=ARITH_NOTE[mode])
        out.update(extras)
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def c3_refined(args, steps=None, warmup=None):
    """The uneven-blocks workload on a three-level refinement
    (problems.refined_blast, seed 4): 515 blocks with edges from
    {16,24,32,48,64} (64 on the base level, 128^3 cells; a level-1 box of
    208^3 and a level-2 box of 240^3 cells around an off-centre blast), ion MHD
    + neutral + dust, vanleer, CFL 0.7.  Each RK stage sweeps every block of a
    level in one launch, finest level first, with the fine->coarse flux
    correction, then copies and prolongs the guard cells; a step's launches
    are replayed from one CUDA graph.  A cell-update is one cell of any block
    (covered ones included: the reference sweeps them too) advanced by one
    dt.  Timed beside one block of the same physics and a similar cell count
    through the single-block fused path, both in the bit-exact arithmetic (the
    stage kernels of refined domains have no other).  Returns the JSON record."""
    steps = steps or args.steps
    warmup = args.warmup if warmup is None else warmup
    import torch
    from piernik_b200 import build, problems
    from piernik_b200.autotune import autotune
    from piernik_b200.sim import Simulation
    build.build()
    torch.cuda.set_device(0)
    dom, blocks = problems.refined_blast()
    cells = sum(int(np.prod(s.n)) for s, *_ in blocks)
    sim = Simulation(blocks[0][0])
    for s, *_ in blocks[1:]:
        sim.add_block(s)
    sim.set_domain(dom, (True, True, True))
    for i, (s, L, off, u, b, psi) in enumerate(blocks):
        sim.place_block(i, off, L)
        sim.upload(u, b, psi, block=i)
    levels = [sum(1 for x in blocks if x[1] == L) for L in range(3)]
    del blocks
    sim.update_boundaries()
    sim.use_graph(True)
    stream = torch.cuda.ExternalStream(sim.stream)
    # launch shape of the batched stage kernel: one captured step each, then the fastest
    tune = {}
    for v in range(4):
        sim.set_stage_variant(v)
        sim.run(1)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        sim.run(1)
        t1.record(stream)
        t1.synchronize()
        tune[v] = t0.elapsed_time(t1)
    best_v = min(tune, key=tune.get)
    sim.set_stage_variant(best_v)
    sim.run(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(0)
    l0, _, _ = sim.profile_read()
    e0.record(stream)
    sim.run(steps)
    e1.record(stream)
    e1.synchronize()
    l1, _, _ = sim.profile_read()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    refined = 2.0 * cells * steps / (ms / 1e3)
    st = sim.time_state
    sim.close()
    # one block of the same physics and a similar number of cells
    side = int(round(cells ** (1.0 / 3.0) / 8.0)) * 8
    one = problems.batched_blocks(nblocks=1, seed=args.seed, sizes=(side,), levels=1)[0]
    s1 = Simulation(one[0])
    s1.upload(*one[1:])
    autotune(s1, reps=1)
    s1.run(warmup)
    st1 = torch.cuda.ExternalStream(s1.stream)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(st1)
    s1.run(steps)
    e3.record(st1)
    e3.synchronize()
    single = 2.0 * side ** 3 * steps / (e2.elapsed_time(e3) / 1e3)
    s1.close()
    out = {"metric": "FP64 3-fluid MHD cell-updates/s, %d blocks on 3 refinement levels" % sum(levels),
           "value": refined, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": {"workload": "refined blast: uneven blocks (edges 16..64) on 3 levels of a periodic 128^3 "
                                  "base domain, ion MHD + neutral + dust, vanleer, CFL 0.7, fine->coarse flux "
                                  "correction, guard prolongation, one launch per level per RK stage, CUDA graph "
                                  "per step", "blocks_per_level": levels, "cells": cells,
                      "stage_variant": best_v, "stage_variant_ms_per_step": tune},
           "single_block": {"n": side, "value": single, "ratio_refined_to_single": refined / single},
           "t_end": st.t, "gpu_launches": l1 - l0, "clocks": ck}
    return out


def batched_arm(args):
    print(json.dumps(c3_refined(args)), flush=True)


def batched_independent_arm(args):
    """512 independent periodic blocks with edges from {16,24,32,48,64}, three
    fluids (ion MHD 5/3, neutral 7/5, dust), one persistent launch per sweep,
    each step's sweeps replayed from a CUDA graph; timed beside one block of
    the same physics and a similar cell count through the single-block path."""
    import torch
    from piernik_b200 import build, problems
    from piernik_b200.autotune import autotune
    from piernik_b200.sim import Simulation
    build.build()
    torch.cuda.set_device(0)
    data = problems.batched_blocks(nblocks=args.nblocks, seed=args.seed)
    cells = sum(int(np.prod(s.n)) for s, *_ in data)
    sim = Simulation(data[0][0])
    for s, *_ in data[1:]:
        sim.add_block(s)
    for i, (s, u, b, psi) in enumerate(data):
        sim.upload(u, b, psi, block=i)
    best = None
    for L, V in ((56, 1), (56, 0), (40, 0), (24, 1), (56, 2)):
        sim.set_batch(True, L, V)
        sim.profile(True)
        sim.profile_read()
        dt, _ = sim.timestep_raw()
        for d in (1, 2, 3):
            sim.sweep(d, 0.25 * dt, 1.0)
        _, nl, ms = sim.profile_read()
        sim.profile(False)
        if best is None or ms < best[0]:
            best = (ms, L, V)
    for i, (s, u, b, psi) in enumerate(data):   # undo the tuning sweeps
        sim.upload(u, b, psi, block=i)
    sim.set_batch(True, best[1], best[2])
    sim.use_graph(True)
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.run(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(0)
    l0, _, _ = sim.profile_read()
    e0.record(stream)
    sim.run(args.steps)
    e1.record(stream)
    e1.synchronize()
    l1, _, _ = sim.profile_read()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    batched = 2.0 * cells * args.steps / (ms / 1e3)
    sim.close()
    # one block of the same physics and a similar number of cells
    side = int(round(cells ** (1.0 / 3.0) / 8.0)) * 8
    one = problems.batched_blocks(nblocks=1, seed=args.seed, sizes=(side,), levels=1)[0]
    s1 = Simulation(one[0])
    s1.upload(*one[1:])
    autotune(s1, reps=1)
    s1.run(args.warmup)
    st1 = torch.cuda.ExternalStream(s1.stream)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(st1)
    s1.run(args.steps)
    e3.record(st1)
    e3.synchronize()
    single = 2.0 * side ** 3 * args.steps / (e2.elapsed_time(e3) / 1e3)
    s1.close()
    out = {"metric": "FP64 3-fluid MHD cell-updates/s, %d uneven blocks, one persistent launch per sweep" % args.nblocks,
           "value": batched, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": {"workload": "batched uneven blocks (edges 16..64, 3 levels, off-centre Sedov), ion MHD + "
                                  "neutral + dust, vanleer, CFL 0.7, CUDA graph per step",
                      "blocks": args.nblocks, "cells": cells, "batch_L_variant": [best[1], best[2]]},
           "single_block": {"n": side, "value": single, "ratio_batched_to_single": batched / single},
           "gpu_launches": l1 - l0, "clocks": ck}
    print(json.dumps(out), flush=True)


def adjoint_arm(args):
    """Gradient of --steps steps of the MHD turbulence block at --n: the
    recorded forward, the backward pass and one adjoint sweep per direction,
    each against the plain forward (also the command the adjoint kernels are
    profiled with)."""
    import torch
    from piernik_b200 import build, problems
    from piernik_b200.sim import Simulation
    build.build()
    setup, u, b, psi = problems.mhd_turbulence(n=args.n, seed=args.seed)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.run(args.warmup)
    st0 = sim.time_state
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(args.steps)
    e1.record(stream)
    e1.synchronize()
    fwd = e0.elapsed_time(e1) / args.steps
    sim.time_state = st0

    class _A:
        adj_steps = args.steps
    res = adjoint_cost(sim, stream, _A, fwd, torch.cuda.synchronize, lambda x: x)
    out = {"workload": f"adjoint of {args.steps} MHD steps at {args.n}^3", "forward_ms_per_step": fwd,
           "adjoint_cost_ratio": res}
    print(json.dumps(out), flush=True)
    sim.close()


def c4_ot_gradient(args, ndirs=16, n=None, K=None):
    """C4: the differentiable Orszag-Tang vortex at 512^2 (--n), loss = magnetic
    energy of the central 128^2 cells after K = --steps steps (default 100
    when --steps is left at 10), gradient with respect to the relative density
    perturbation (1e-3 x a seeded unit-rms Gaussian random field, correlation
    8 cells) through torch.autograd with sqrt(K) checkpointing; checked
    against central differences along 16 seeded directions at eps = 1e-6 and
    1e-7 at the dt sequence of the unperturbed run.  Returns the record."""
    import numpy as np
    import torch
    from piernik_b200 import build, problems
    from piernik_b200.autograd import advance, central_magnetic_energy, last_dts, orszag_tang_state
    from piernik_b200.sim import Simulation
    build.build()
    n = n or (args.n if args.n != 256 else 512)
    K = K or (args.steps if args.steps != 10 else 100)
    s = problems.orszag_tang_fields(n)[0]
    sim = Simulation(s)
    stream = torch.cuda.ExternalStream(sim.stream)
    d0 = torch.tensor(1.0e-3 * problems.orszag_tang_perturbation(n, seed=1), device="cuda", requires_grad=True)
    # plain forward of the same K steps for the cost ratio
    st_init = sim.time_state
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    with torch.no_grad():
        x0 = orszag_tang_state(sim, d0.detach())
    full = torch.zeros(sim.state_shape(), dtype=torch.float64, device="cuda")
    g = s.guards
    full[:, :, g[1]:g[1] + n, g[0]:g[0] + n] = x0
    torch.cuda.synchronize()
    sim.upload_device(full.data_ptr())
    e[0].record(stream)
    sim.run(K)
    e[1].record(stream)
    e[1].synchronize()
    fwd_ms = e[0].elapsed_time(e[1])
    sim.time_state = st_init
    # untimed warm-up gradient (loads the kernels, allocates the checkpoints and pool)
    warm = advance(sim, orszag_tang_state(sim, d0), K)
    central_magnetic_energy(sim, warm).backward()
    d0.grad = None
    sim.time_state = st_init
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t2 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record()
    out = advance(sim, orszag_tang_state(sim, d0), K)
    loss = central_magnetic_energy(sim, out)
    t1.record()
    loss.backward()
    t2.record()
    t2.synchronize()
    dts = last_dts(out)
    grad = d0.grad.detach().cpu().numpy()
    nv, cy = s.nvar, n // 4
    y0 = (n - cy) // 2
    dV = float(np.prod(s.dl))

    def central_b(d):
        with torch.no_grad():
            o = advance(sim, orszag_tang_state(sim, d), K, dts=dts)
            return o[nv:nv + 3, 0, y0:y0 + cy, y0:y0 + cy].cpu().numpy()

    rng = np.random.default_rng(21)
    rows = []
    for k in range(ndirs):
        v = problems.gaussian_random_field((n, n), 8.0, rng)
        vt = torch.tensor(v, device="cuda")
        ad = float(np.sum(grad * v))
        row = {"adjoint": ad}
        for eps in (1.0e-6, 1.0e-7):
            bp, bm = central_b(d0.detach() + eps * vt), central_b(d0.detach() - eps * vt)
            fd = float(0.5 * ((bp - bm) * (bp + bm)).sum() * dV / (2 * eps))
            row[f"fd_{eps:g}"] = fd
            row[f"rel_{eps:g}"] = abs(ad - fd) / max(abs(fd), 1e-300)
        rows.append(row)
    rel6 = [r["rel_1e-06"] for r in rows]
    rel7 = [r["rel_1e-07"] for r in rows]
    res = {"workload": f"differentiable Orszag-Tang {n}^2, K = {K}, loss = central {cy}^2 magnetic energy, "
                       f"{ndirs} FD directions", "arithmetic": "bitexact",
           "forward_ms": fwd_ms, "recorded_forward_plus_loss_ms": t0.elapsed_time(t1),
           "backward_ms": t1.elapsed_time(t2), "gradient_over_forward": t0.elapsed_time(t2) / fwd_ms,
           "fd_rel_error_eps1e-6": {"median": float(np.median(rel6)), "max": float(np.max(rel6))},
           "fd_rel_error_eps1e-7": {"median": float(np.median(rel7)), "max": float(np.max(rel7))},
           "directions": rows}
    sim.close()
    return res


def ot_gradient_arm(args):
    print(json.dumps(c4_ot_gradient(args)), flush=True)


def c5_batched_adjoint(args, K=None, ngroups=None, warmup=None, steps=None):
    """Batched adjoint: --instances independent 128^3 ideal-MHD turbulence
    instances (the 256^3 recipe with rms Mach log-uniform in [0.5, 5] and B0
    uniform in [0.05, 0.5], seeded), loss = sum over instances of the
    kinetic-energy spectrum power in 8 <= |k| <= 16 after K = --k steps,
    gradient with respect to every instance's initial velocity field.

    --group instances are stacked along z in one handle (pk_set_instances):
    each sweep and each adjoint sweep is one launch over the group, every
    instance with its own CFL time step.  The gradient goes through
    torch.autograd (turbulence_state -> advance -> spectrum_power) with
    checkpoints every 2 steps (the memory optimum for 6 stored sweeps per
    step).  A "step" of this workload is the gradient of one group; the
    timed steps cycle over the groups, so --steps = instances / group covers
    the whole ensemble once.  Beside it: K plain forward steps of a group,
    and the gradient of one instance in a handle of its own.  Returns the
    record (K, the number of groups, warm-up and timed steps default to the
    command line's)."""
    import torch
    from piernik_b200 import build, problems
    from piernik_b200._lib import PkTimeState
    from piernik_b200.autograd import advance, spectrum_power, turbulence_state
    from piernik_b200.sim import Simulation
    build.build()
    torch.cuda.set_device(0)
    n = args.n if args.n != 256 else 128
    G, K = args.group, (K or args.k)
    ngroups = ngroups or max(1, args.instances // G)
    steps = steps or (args.steps if args.steps != 10 else ngroups)
    warmup = args.warmup if warmup is None else warmup
    every = 2
    params = problems.turbulence_ensemble(ngroups * G, n, args.seed)
    groups = []
    p0 = None
    for j in range(ngroups):
        f = [problems.mhd_turbulence_fields(n, sd, mach, b0) for sd, mach, b0 in params[j * G:(j + 1) * G]]
        p0 = f[0][3]
        cat = lambda i, ax: torch.tensor(np.concatenate([x[i] for x in f], axis=ax), device="cuda")
        groups.append((cat(0, 0), cat(1, 1), cat(2, 1)))
    setup = problems.turbulence_setup(n, nz=G * n)
    sim = Simulation(setup)
    sim.set_instances(G)
    stream = torch.cuda.ExternalStream(sim.stream)

    def gradient(s, grp, inst):
        rho, v0, b = grp
        v = v0.clone().requires_grad_(True)
        s.time_state = PkTimeState()
        out = advance(s, turbulence_state(s, rho, v, b, p0), K, every=every)
        loss = spectrum_power(s, out, 8.0, 16.0, instances=inst).sum()
        loss.backward()
        return v.grad, loss.detach()

    for w in range(warmup):
        gradient(sim, groups[w % ngroups], G)
    torch.cuda.synchronize()
    clocks = Clocks(0)
    l0, _, _ = sim.profile_read()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = []
    for i in range(steps):
        g, loss = gradient(sim, groups[i % ngroups], G)
        losses.append(loss)
    e1.record()
    e1.synchronize()
    l1, _, _ = sim.profile_read()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    gnorm = float(torch.linalg.vector_norm(g))
    # K plain forward steps of the last group, for the gradient / forward ratio
    rho, v0, b = groups[(steps - 1) % ngroups]
    x0 = turbulence_state(sim, rho, v0, b, p0)
    full = torch.zeros(sim.state_shape(), dtype=torch.float64, device="cuda")
    gd = setup.guards
    full[:, gd[2]:gd[2] + G * n, gd[1]:gd[1] + n, gd[0]:gd[0] + n] = x0
    torch.cuda.synchronize()
    sim.upload_device(full.data_ptr())
    sim.time_state = PkTimeState()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    sim.run(K)
    f1.record(stream)
    f1.synchronize()
    fwd_ms = f0.elapsed_time(f1)
    dts = [sim.instance_state(i).dt for i in range(G)]
    del full
    sim.close()
    # one instance alone, same K and checkpointing
    one = Simulation(problems.turbulence_setup(n))
    single = (groups[0][0][:n], groups[0][1][:, :n], groups[0][2][:, :n])
    gradient(one, single, 1)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    gradient(one, single, 1)
    s1.record()
    s1.synchronize()
    single_ms = s0.elapsed_time(s1)
    one.close()
    cells = G * n ** 3
    value = 2.0 * cells * K * steps / (ms / 1e3)
    out = {"metric": "FP64 MHD cell-updates/s differentiated (forward + adjoint), stacked 128^3 instances",
           "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"batched adjoint: {ngroups * G} independent {n}^3 ideal-MHD turbulence "
                                  f"instances (Mach log-uniform 0.5..5, B0 0.05..0.5), HLLD + GLM, moncen, "
                                  f"CFL 0.5, loss = kinetic-energy shell power 8 <= |k| <= 16 after K = {K} "
                                  f"steps, gradient wrt initial velocity", "instances": ngroups * G,
                      "group": G, "K": K, "checkpoint_every": every,
                      "step": f"gradient of one group of {G} stacked instances",
                      "l2": "group state %.2f GB > 126 MB L2" % (9 * 8 * (n + 8) ** 2 * (G * n + 8) / 1e9)},
           "instance_gradients_per_s": G * steps / (ms / 1e3),
           "gradient_ms_per_instance": ms / (steps * G),
           "forward_ms_per_group": fwd_ms, "gradient_over_forward": (ms / steps) / fwd_ms,
           "single_instance_gradient_ms": single_ms,
           "batched_per_instance_over_single": (ms / (steps * G)) / single_ms,
           "instance_dt_spread": [min(dts), max(dts)],
           "loss_last_group": float(losses[-1]), "grad_norm_last_group": gnorm,
           "gpu_launches": l1 - l0, "clocks": ck}
    return out


def batched_adjoint_arm(args):
    print(json.dumps(c5_batched_adjoint(args)), flush=True)


def unsplit_arm(args):
    """The 256^3 MHD turbulence block through the unsplit scheme
    (solver_str = 'unsplit'): one dt per step, every stage the face fluxes of
    x, y and z from the same state, CFL 0.3 and cfl_glm 0.3 (the values the
    reference recommends for this solver, global.F90:525-533)."""
    import torch
    from piernik_b200 import build, problems
    from piernik_b200.sim import Simulation
    build.build()
    torch.cuda.set_device(0)
    setup, u, b, psi = problems.mhd_turbulence(n=args.n, seed=args.seed, cfl=0.3)
    setup = setup.replace(solver="unsplit", cfl_glm=0.3)
    sim = Simulation(setup)
    sim.upload(u, b, psi)
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.run(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(0)
    l0, _, _ = sim.profile_read()
    e0.record(stream)
    sim.run(args.steps)
    e1.record(stream)
    e1.synchronize()
    l1, _, _ = sim.profile_read()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    n = args.n
    out = {"metric": "FP64 MHD cell-updates/s at %d^3, unsplit scheme" % n, "value": n ** 3 * args.steps / (ms / 1e3),
           "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"3D ideal-MHD decaying turbulence, one periodic {n}^3 block, unsplit HLLD + GLM, "
                                  f"moncen, RK2, CFL 0.3", "step": "time_step + fluid_update_unsplit (1 dt)"},
           "gpu_launches": l1 - l0, "clocks": ck}
    print(json.dumps(out), flush=True)
    sim.close()


def main():
    args = parse()
    if args.workload == "unsplit":
        unsplit_arm(args)
        return
    if args.workload == "batched-adjoint":
        batched_adjoint_arm(args)
        return
    if args.workload == "batched":
        batched_arm(args)
        return
    if args.workload == "batched-independent":
        batched_independent_arm(args)
        return
    if args.workload == "adjoint":
        adjoint_arm(args)
        return
    if args.workload == "ot-gradient":
        ot_gradient_arm(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
