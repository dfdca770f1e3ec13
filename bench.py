#!/usr/bin/env python
"""Benchmark: batched 2-center overlap (+ (zeta, D) gradient step) on B200.

Workload (one GPU / one rank): the ragged mixed-species 2C overlap batch --
4 species with l <= 3 synthetic bases (3-5 s, 2-3 p, 1-2 d, 0-1 f shells,
K in 1..8 primitives per shell, seeded), B = 65,536 pairs per rank with random
species pairs, random directions and |A-B| ~ U[0.5, 8] bohr.  A step is one
forward pass of the FP32-compensated kernel over the whole batch (prep +
species-pair binning + overlap kernel, all on the device).  Weak scaling: each
rank processes its own batch, no collective on the data path.

Also reported: the plain FP64 kernel on the same batch, the FP32C error
against the FP64 oracle, the (zeta, D) gradient step of the overlap loss,
the dominant kernel's roofline, an end-to-end number through the C ABI with
host buffers, and the CPU oracle on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl aok|reference]

With --gpus N > 1 and no torchrun environment (WORLD_SIZE unset), bench.py starts
N ranks itself under torch.distributed.run on 127.0.0.1.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "2c-overlap integrals/s + (ζ,D) grad step, FP32-comp vs FP64, 1 B200, rel err"
UNIT = "integrals/s"
B_PER_RANK = 65536
B_SP = 262144  # the s/p output-bound batch: 14^2 x 4 B x B = 205 MB of FP32 output (> L2)
SEED = 1002


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def workload(rank=0, B=B_PER_RANK):
    import aok_b200 as aok
    W = aok.workloads
    basis = W.config2_basis(seed=SEED)
    pairs = W.ragged_pairs(B, basis.NZ, SEED + 7919 * rank)
    return basis, pairs


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.05)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except Exception:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm),
                "window": "the timed region plus untimed repetitions of the same step right after it "
                          f"({getattr(self, 'extra_s', 0.0):.2f} s) until >= 6 samples"}


def cpu_oracle_rate(basis, pairs, coef, target_s=12.0, nthreads=None):
    """Integrals/s of the oracle (C, OpenMP) on a bounded sample of the workload:
    whole passes over the batch until about `target_s` seconds of CPU work."""
    import oracle
    nthreads = nthreads or os.cpu_count()
    N = basis.nbf_total
    t0 = time.perf_counter()
    passes, done = 0, 0
    while True:
        oracle.overlap2c_orb(basis.ls, coef, basis.zeta, pairs.sidxA, pairs.sidxB, pairs.posA, pairs.posB,
                             nthreads=nthreads)
        passes += 1
        done += pairs.B
        dt = time.perf_counter() - t0
        if dt >= target_s or passes >= 200:
            break
    return N * N * done / dt, nthreads, done, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    basis, pairs = workload(0)
    coef = oracle.compile_coef(basis.zeta, basis.D, basis.ls)
    nth = os.cpu_count()
    N = basis.nbf_total
    bs = 256
    # size the per-step sample so the whole run stays within a few minutes
    t0 = time.perf_counter()
    oracle.overlap2c_orb(basis.ls, coef, basis.zeta, pairs.sidxA[:bs], pairs.sidxB[:bs], pairs.posA[:, :bs],
                         pairs.posB[:, :bs], nthreads=nth)
    dt = time.perf_counter() - t0
    per_step = int(min(pairs.B, max(64, bs * 10.0 / max(dt, 1e-6) / max(1, args.steps + args.warmup) * 3)))
    sl = slice(0, per_step)
    for _ in range(args.warmup):
        oracle.overlap2c_orb(basis.ls, coef, basis.zeta, pairs.sidxA[sl], pairs.sidxB[sl], pairs.posA[:, sl],
                             pairs.posB[:, sl], nthreads=nth)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.overlap2c_orb(basis.ls, coef, basis.zeta, pairs.sidxA[sl], pairs.sidxB[sl], pairs.posA[:, sl],
                             pairs.posB[:, sl], nthreads=nth)
    dt = (time.perf_counter() - t0) / args.steps
    val = N * N * per_step / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "ragged 4-species l<=3 2C overlap, FP64 CPU oracle (C restatement of the "
                               "reference's KernelAbstractions CPU path; Julia is not installed)",
                   "batch_per_step": per_step, "nbf": N},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": nth, "kind": "port",
                         "sample": f"{per_step} pairs of the B=65536 batch per step"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def launch_ranks(args):
    """bench.py --gpus N started without torchrun: start N ranks (one per GPU) on this
    node under torch.distributed.run with the same arguments, and return its status.
    Only rank 0 prints the JSON line."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "1"))
    return subprocess.call(cmd, env=env)


def run_dry(args):
    """The multi-rank structure of a step without a GPU: each rank takes its own batch
    (weak scaling), waits at the barriers of the timed region, reduces its time with a
    max over ranks, and sums a (zeta, D) gradient of the step's shape with the same
    all-reduce the gradient step uses (aok_b200.parallel.allreduce_sum).  Rank r
    contributes r + 1 in every entry, so the sum is known.  Prints one JSON line on
    rank 0 with dry_run: true (no throughput is measured)."""
    import datetime

    import torch
    import torch.distributed as dist

    import aok_b200 as aok
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    basis, pairs = workload(rank, min(args.batch, 4096))
    shape = (basis.nshells, basis.K, basis.NZ)
    ok = True

    def step():
        nonlocal ok
        dz = torch.full(shape, float(rank + 1), dtype=torch.float64)
        dD = torch.full(shape, float(-(rank + 1)), dtype=torch.float64)
        dz, dD = aok.parallel.allreduce_sum([dz, dD])
        want = world * (world + 1) / 2
        ok = ok and bool(torch.all(dz == want)) and bool(torch.all(dD == -want))

    for _ in range(args.warmup):
        step()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    if world > 1:
        dist.barrier()
    ms = (time.perf_counter() - t0) * 1e3 / max(args.steps, 1)
    t = torch.tensor([ms, 0.0 if ok else 1.0], dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": float(t[0]), "higher_is_better": True,
                          "scaling": "weak", "dry_run": True, "allreduce_ok": bool(t[1] == 0.0),
                          "config": {"workload": "rank plumbing only (gloo, CPU)", "batch_per_rank": pairs.B,
                                     "global_batch": pairs.B * world, "gradient_shape": list(shape)}}),
              flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="aok", choices=["aok", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient step")
    ap.add_argument("--profile", action="store_true",
                    help="only the FP32C forward steps (for ncu launch lists / captures); prints no JSON")
    ap.add_argument("--batch", type=int, default=B_PER_RANK, help="pairs per rank")
    ap.add_argument("--workload", default="overlap2c",
                    choices=["overlap2c", "evaluate", "overlap3c", "pullback", "grad", "outputbound", "outputbound_sp"],
                    help="with --profile: which kernel family to run (ncu captures)")
    ap.add_argument("--no-extra", action="store_true", help="skip the config-1/3/4 side measurements")
    ap.add_argument("--fp64", action="store_true", help="with --profile: run the FP64 kernels (overlap2c, overlap3c)")
    ap.add_argument("--timeline", action="store_true",
                    help="with --profile: warm launch list of the steps from CUPTI (torch.profiler): each launch's "
                         "start, end and duration within the last step, and the mean duration per kernel")
    ap.add_argument("--cpu-dry", action="store_true",
                    help="rank plumbing only, on CPU: gloo process group, barriers, max-over-ranks timing and the "
                         "gradient all-reduce of the step, with no kernels (for tests without a GPU)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args)  # one process per GPU under torchrun; rank 0 prints the line
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(args.warmup, 3)
    if args.cpu_dry:
        return run_dry(args)

    import torch
    import torch.distributed as dist

    import aok_b200 as aok
    from aok_b200 import _dev, _lib
    import oracle

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    L = _lib.load()
    basis, pairs = workload(rank, args.batch)
    N, B, ns, K, NZ = basis.nbf_total, pairs.B, basis.nshells, basis.K, basis.NZ
    peaks, peak_kind = _peaks()

    def setup(FT):
        plan = _dev.Plan(basis.ls, K, NZ, _dev.prec_of(FT), B)
        zeta = _dev.to_colmajor(basis.zeta, FT)
        D = _dev.to_colmajor(basis.D, FT)
        coef = _dev.colmajor_empty((ns, K, NZ), FT)
        _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
        pA = _dev.to_colmajor(pairs.posA, FT)
        pB = _dev.to_colmajor(pairs.posB, FT)
        sA = torch.as_tensor(pairs.sidxA).cuda()
        sB = torch.as_tensor(pairs.sidxB).cuda()
        out = _dev.colmajor_empty((N, N, B), FT)
        # compile_basis equivalent: the geometry-free records are fixed once, under the
        # launch shape the autotuner picks for this (basis, B)
        ch = (ctypes.c_int64 * 3)()
        _lib.check(L.aok_plan_autotune(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(pA),
                                       _dev.ptr(pB), ctypes.c_void_p(sA.data_ptr()), ctypes.c_void_p(sB.data_ptr()),
                                       B, 1.0, _dev.stream(), ch))
        _lib.check(L.aok_plan_set_graph(plan.h, 1))  # one captured launch chain per compiled basis
        return dict(plan=plan, zeta=zeta, D=D, coef=coef, pA=pA, pB=pB, sA=sA, sB=sB, out=out, FT=FT,
                    shape={"ctas_per_sm": int(ch[0]), "stage_bytes": int(ch[1])})

    def step(c, with_params=False):
        z = _dev.ptr(c["zeta"]) if with_params else None
        cf = _dev.ptr(c["coef"]) if with_params else None
        _lib.check(L.aok_overlap2c(c["plan"].h, _dev.ptr(c["out"]), z, cf, _dev.ptr(c["pA"]), _dev.ptr(c["pB"]),
                                   ctypes.c_void_p(c["sA"].data_ptr()), ctypes.c_void_p(c["sB"].data_ptr()), B, 1.0,
                                   _dev.stream()))

    def timed(c, steps, warmup, sampler=None):
        for _ in range(warmup):
            step(c)
        barrier()
        torch.cuda.synchronize()
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            st.record()
            for _ in range(steps):
                step(c)  # the plan's CUDA graph (graph mode, timing off)
            en.record()
            torch.cuda.synchronize()
            if sampler is not None:
                # a short timed region ends before nvidia-smi's first 200 ms sample: keep the
                # same step running (untimed) until the clock record holds a few samples
                t0 = time.time()
                while (len(sampler.rows) < 6 and time.time() - t0 < 3.0 and sampler.proc is not None
                       and sampler.proc.poll() is None):
                    for _ in range(50):
                        step(c)
                    torch.cuda.synchronize()
                sampler.extra_s = time.time() - t0
        barrier()
        ms = st.elapsed_time(en) / steps
        # the dominant kernel alone: events around it in a second, shorter loop (direct launches)
        nk = max(3, steps // 5)
        _lib.check(L.aok_plan_timing_enable(c["plan"].h, nk))
        for _ in range(nk):
            step(c)
        torch.cuda.synchronize()
        tot, n = ctypes.c_double(), ctypes.c_int64()
        _lib.check(L.aok_plan_timing_read(c["plan"].h, ctypes.byref(tot), ctypes.byref(n)))
        _lib.check(L.aok_plan_timing_enable(c["plan"].h, 0))
        kms = tot.value / max(n.value, 1)
        return allmax(ms), allmax(kms)

    if args.profile and args.workload not in ("overlap2c", "grad"):
        fn = side_workload(args.workload, L, _dev, _lib, aok, torch, args.batch, torch.float64 if args.fp64 else None)
        if args.timeline:
            return _timeline(fn, args.steps, args.warmup, torch)
        for _ in range(args.warmup + args.steps):
            fn()
        torch.cuda.synchronize()
        return 0

    # ---- FP32C forward (headline) ----
    c32 = setup(torch.float32)
    if args.profile and args.workload == "grad":
        gd = _grad_setup(basis, c32, B, L, _dev, _lib, aok, torch)
        if args.timeline:
            return _timeline(gd["gstep_res"], args.steps, args.warmup, torch)
        for _ in range(args.warmup + args.steps):
            torch.cuda.nvtx.range_push("gradstep")  # ncu --nvtx --nvtx-include "gradstep/" selects the step's launches
            gd["gstep_res"]()
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        return 0
    if args.profile:
        cp = setup(torch.float64) if args.fp64 else c32
        if args.timeline:
            return _timeline(lambda: step(cp), args.steps, args.warmup, torch)
        for _ in range(args.warmup + args.steps):
            step(cp)
        torch.cuda.synchronize()
        return 0
    sampler = ClockSampler(local)
    ms32, kms32 = timed(c32, args.steps, args.warmup, sampler)
    clocks = sampler.summary()
    value = N * N * B * world / (ms32 * 1e-3)
    # the same step when the parameters come with every call (records rebuilt per call)
    ms32p = _time(lambda: step(c32, True), max(20, args.steps // 10), args.warmup, torch, allmax)

    # ---- FP64 forward ----
    c64 = setup(torch.float64)
    ms64, kms64 = timed(c64, max(3, args.steps // 2), args.warmup)
    del c64["plan"]
    value64 = N * N * B * world / (ms64 * 1e-3)

    # ---- (zeta, D) gradient step (config 3): L = sum (S - S_tgt)^2, B = 16384 pairs ----
    grad = None
    if not args.no_grad:
        gd = _grad_setup(basis, c32, B, L, _dev, _lib, aok, torch)
        gstep, fstep = gd["gstep"], gd["fstep"]

        def tloop(fn, n):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            st.record()
            for _ in range(n):
                fn()
            en.record()
            torch.cuda.synchronize()
            return allmax(st.elapsed_time(en) / n)

        ng = max(3, args.steps // 10)
        f_ms = tloop(fstep, ng)
        g_ms = tloop(gstep, ng)
        gr_ms = tloop(gd["gstep_res"], ng)
        Bg = gd["Bg"]
        del gd
        grad = {"workload": "config 3: L = sum (S - S_tgt)^2 over B=16384 pairs, FP32C rrule forward (coef from D, "
                            "pullback records prepared beside the overlap kernel) + the rrule pullback of "
                            "dL/dS = 2 (S - S_tgt), formed inside the pullback kernel "
                            "(aok_overlap_pullback_ps_rrule_residual)",
                "batch": Bg, "forward_ms": f_ms, "step_ms": gr_ms, "step_over_forward": gr_ms / f_ms,
                "launches_per_step": 6 + 3,
                "separate_cotangent": {"note": "dL/dS materialised by torch.sub, the pullback of it, then x2",
                                       "step_ms": g_ms, "step_over_forward": g_ms / f_ms,
                                       "torch_launches_per_step": 2}}

    # ---- error of FP32C and FP64 vs the FP64 oracle on a sample (inputs rounded as the GPU saw them) ----
    nchk = 2048
    S32 = c32["out"][:, :, :nchk].double().cpu().numpy()
    S64 = c64["out"][:, :, :nchk].cpu().numpy()
    z32 = basis.zeta.astype(np.float32).astype(np.float64)
    coef32 = oracle.compile_coef(z32, basis.D.astype(np.float32).astype(np.float64), basis.ls)
    coef32 = coef32.astype(np.float32).astype(np.float64)
    ref32 = oracle.overlap2c_orb(basis.ls, coef32, z32, pairs.sidxA[:nchk], pairs.sidxB[:nchk],
                                 pairs.posA[:, :nchk].astype(np.float32).astype(np.float64),
                                 pairs.posB[:, :nchk].astype(np.float32).astype(np.float64), nthreads=os.cpu_count())
    coef64 = oracle.compile_coef(basis.zeta, basis.D, basis.ls)
    ref64 = oracle.overlap2c_orb(basis.ls, coef64, basis.zeta, pairs.sidxA[:nchk], pairs.sidxB[:nchk],
                                 pairs.posA[:, :nchk], pairs.posB[:, :nchk], nthreads=os.cpu_count())
    err32 = float(np.linalg.norm(S32 - ref32) / np.linalg.norm(ref32))
    err64 = float(np.linalg.norm(S64 - ref64) / np.linalg.norm(ref64))

    def _elem_errs(X, R):
        """max |X - R| and max |X - R| / |R| over elements with |R| > 1e-12 max |R|."""
        d = np.abs(X - R)
        big = np.abs(R) > 1e-12 * np.abs(R).max()
        return {"max_abs": float(d.max()), "max_rel": float((d[big] / np.abs(R[big])).max())}

    err_detail = {"f32c": _elem_errs(S32, ref32), "f64": _elem_errs(S64, ref64)}
    # useful integrals: blocks whose two shells are both present in the pair's species
    present = basis.nprim > 0  # (ns, NZ)
    nbf_sh = (basis.ls + 1) * (basis.ls + 2) // 2
    useful = 0
    sa0, sb0 = np.asarray(pairs.sidxA) - 1, np.asarray(pairs.sidxB) - 1
    for ga in range(NZ):
        for gb in range(NZ):
            cnt = int(np.count_nonzero((sa0 == ga) & (sb0 == gb)))
            if cnt:
                na = int((nbf_sh * present[:, ga]).sum())
                nb = int((nbf_sh * present[:, gb]).sum())
                useful += cnt * na * nb
    useful_frac = useful / float(N * N * B)

    # ---- FMA-pipe peaks of this GPU (denominators for the compute-bound kernels' pipe use) ----
    pipe_peaks = {"method": "aok_measure_fma_peak: independent FMA chains, 8 blocks x 256 threads per SM"}
    for name, prec, paired in (("fp32_tflops", _lib.AOK_PREC_F32C, 0), ("fp32_paired_tflops", _lib.AOK_PREC_F32C, 1),
                               ("fp64_tflops", _lib.AOK_PREC_F64, 0)):
        v = ctypes.c_double()
        _lib.check(L.aok_measure_fma_peak(prec, paired, ctypes.byref(v), _dev.stream()))
        pipe_peaks[name] = allmax(v.value)

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        hA = torch.as_tensor(np.ascontiguousarray(pairs.posA.T.astype(np.float32))).pin_memory()
        hB = torch.as_tensor(np.ascontiguousarray(pairs.posB.T.astype(np.float32))).pin_memory()
        hsA = torch.as_tensor(pairs.sidxA).pin_memory()
        hsB = torch.as_tensor(pairs.sidxB).pin_memory()
        hout = torch.empty((B, N, N), dtype=torch.float32).pin_memory()
        dA = torch.empty((B, 3), dtype=torch.float32, device="cuda")
        dB = torch.empty((B, 3), dtype=torch.float32, device="cuda")
        dsA = torch.empty(B, dtype=torch.int64, device="cuda")
        dsB = torch.empty(B, dtype=torch.int64, device="cuda")
        dout = torch.empty((B, N, N), dtype=torch.float32, device="cuda")

        def e2e_step():
            dA.copy_(hA, non_blocking=True)
            dB.copy_(hB, non_blocking=True)
            dsA.copy_(hsA, non_blocking=True)
            dsB.copy_(hsB, non_blocking=True)
            _lib.check(L.aok_overlap2c(c32["plan"].h, ctypes.c_void_p(dout.data_ptr()), _dev.ptr(c32["zeta"]),
                                       _dev.ptr(c32["coef"]), ctypes.c_void_p(dA.data_ptr()),
                                       ctypes.c_void_p(dB.data_ptr()), ctypes.c_void_p(dsA.data_ptr()),
                                       ctypes.c_void_p(dsB.data_ptr()), B, 1.0, _dev.stream()))
            hout.copy_(dout, non_blocking=True)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ke = max(3, min(200, args.steps // 10))
        st.record()
        for _ in range(ke):
            e2e_step()
        en.record()
        torch.cuda.synchronize()
        barrier()
        ems = allmax(st.elapsed_time(en) / ke)
        e2e = {"value": N * N * B * world / (ems * 1e-3), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": int(hA.numel() * 4 + hB.numel() * 4 + hsA.numel() * 8 + hsB.numel() * 8),
               "d2h_bytes_per_step": int(hout.numel() * 4)}

    # ---- roofline of the dominant kernel (k_overlap2c, FP32C) ----
    alg_bytes = B * (N * N * 4 + 2 * (3 * 4 + 8))
    achieved = alg_bytes / (kms32 * 1e-3) / 1e9
    # DRAM bytes of one ncu capture of this kernel at B = 32768 (read 2.12 MB + write
    # 102.3 MB), scaled to this launch's batch; the output still dirty in L2 when the
    # kernel ends is not counted by dram__bytes_write.
    traffic = (1.786880e6 + 101.915648e6) * B / 32768
    roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "algorithmic_bytes": alg_bytes,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, B=32768 capture scaled by B/32768",
            "kernel": "k_overlap2c<float>",
            "kernel_ms": kms32, "peak_kind": peak_kind,
            "note": "algorithmic bytes = B*(N^2*4 written + 2*(12 B position + 8 B species index) read)"}

    extra = None
    if not args.no_extra:
        extra = side_measurements(args, L, _dev, _lib, aok, torch, oracle, allmax, peaks)

    cpu = None
    if rank == 0 and not args.no_cpu:
        rate, nth, bs, dt = cpu_oracle_rate(basis, pairs, coef64)
        cpu = {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
               "sample": f"{bs} pairs (whole passes over the batch), FP64 oracle, {nth} OpenMP threads, "
                         f"{dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32c", "data": "synthetic",
            "config": {"workload": "ragged 4-species l<=3 2C overlap (config 2), FP32-compensated forward; "
                                   "step = species binning + overlap kernel on a compiled basis "
                                   "(records fixed once, like compile_basis, under the autotuned launch "
                                   "shape; replayed from the plan's CUDA graph)",
                       "batch_per_rank": B, "global_batch": B * world, "nbf": N, "nshells": ns, "K": K,
                       "species": NZ, "l2": "output 321 MB per step > 126 MB L2 (no flush needed)",
                       "launch_shape": c32["shape"]},
            "fp64": {"value": value64, "ms_per_step": ms64, "kernel_ms": kms64, "launch_shape": c64["shape"]},
            "ms_per_step_params_per_call": ms32p,
            "f32c_over_f64": value / value64,
            "rel_err": {"f32c_vs_oracle": err32, "f64_vs_oracle": err64, "sample_pairs": nchk,
                        "elementwise": err_detail},
            "pipe_peaks": pipe_peaks,
            "useful_integrals_per_s": value * useful_frac,
            "useful_integral_fraction": useful_frac,
            "grad_step": grad, "other_configs": extra,
            "roofline": roof, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu,
            "gpu_launches": 3 * args.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _grad_setup(basis, c32, B, L, _dev, _lib, aok, torch):
    import torch.distributed as dist
    """Config 3: L = sum (S - S_tgt)^2 over the first 16384 pairs of the batch, FP32C.
    gstep = rrule forward (coef compiled from D, the pullback's records prepared beside the
    overlap kernel, bins kept) + dL/dS + the rrule's pullback (dzeta, dD); fstep = forward."""
    N, ns, K, NZ = basis.nbf_total, basis.nshells, basis.K, basis.NZ
    Bg = min(16384, B)
    zt, Dt = aok.workloads.config3_target(basis)
    gpl = _dev.Plan(basis.ls, K, NZ, _dev.prec_of(torch.float32), Bg)
    zt_d = _dev.to_colmajor(zt, torch.float32)
    Dt_d = _dev.to_colmajor(Dt, torch.float32)
    ct_d = _dev.colmajor_empty((ns, K, NZ), torch.float32)
    _lib.check(L.aok_compile_coef(gpl.h, _dev.ptr(ct_d), _dev.ptr(zt_d), _dev.ptr(Dt_d), _dev.stream()))
    Sg = _dev.colmajor_empty((N, N, Bg), torch.float32)
    Tg = _dev.colmajor_empty((N, N, Bg), torch.float32)
    dS = _dev.colmajor_empty((N, N, Bg), torch.float32)
    dz = _dev.colmajor_empty((ns, K, NZ), torch.float32)
    dD = _dev.colmajor_empty((ns, K, NZ), torch.float32)
    pA, pB = c32["pA"][:, :Bg], c32["pB"][:, :Bg]
    sA = ctypes.c_void_p(c32["sA"].data_ptr())
    sB = ctypes.c_void_p(c32["sB"].data_ptr())

    def fwd(out, coef):
        _lib.check(L.aok_overlap2c(gpl.h, _dev.ptr(out), _dev.ptr(c32["zeta"]), _dev.ptr(coef), _dev.ptr(pA),
                                   _dev.ptr(pB), sA, sB, Bg, 1.0, _dev.stream()))

    _lib.check(L.aok_overlap2c(gpl.h, _dev.ptr(Tg), _dev.ptr(zt_d), _dev.ptr(ct_d), _dev.ptr(pA), _dev.ptr(pB),
                               sA, sB, Bg, 1.0, _dev.stream()))

    def gstep():
        _lib.check(L.aok_overlap2c_rrule(gpl.h, _dev.ptr(Sg), _dev.ptr(c32["zeta"]), _dev.ptr(c32["D"]),
                                         _dev.ptr(pA), _dev.ptr(pB), sA, sB, Bg, 1.0, _dev.stream()))
        # dL/dS = 2 (S - S_tgt); the pullback is linear in dS, so the factor 2 is applied
        # to the (ns, K, NZ) gradients instead of the (N, N, B) cotangent
        torch.sub(Sg, Tg, out=dS)
        _lib.check(L.aok_overlap_pullback_ps_rrule(gpl.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dS),
                                                   _dev.ptr(c32["zeta"]), _dev.ptr(c32["D"]), _dev.ptr(pA),
                                                   _dev.ptr(pB), sA, sB, Bg, 1.0, _dev.stream()))
        torch._foreach_mul_([dz, dD], 2.0)
        if dist.is_initialized() and dist.get_world_size() > 1:
            aok.parallel.allreduce_sum([dz, dD])  # data-parallel step: sum the ranks' gradients

    def gstep_res():
        # the same step with dL/dS = 2 (S - S_tgt) formed inside the pullback kernel
        _lib.check(L.aok_overlap2c_rrule(gpl.h, _dev.ptr(Sg), _dev.ptr(c32["zeta"]), _dev.ptr(c32["D"]),
                                         _dev.ptr(pA), _dev.ptr(pB), sA, sB, Bg, 1.0, _dev.stream()))
        _lib.check(L.aok_overlap_pullback_ps_rrule_residual(gpl.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(Sg),
                                                            _dev.ptr(Tg), 2.0, _dev.ptr(c32["zeta"]),
                                                            _dev.ptr(c32["D"]), _dev.ptr(pA), _dev.ptr(pB), sA, sB,
                                                            Bg, 1.0, _dev.stream()))
        if dist.is_initialized() and dist.get_world_size() > 1:
            aok.parallel.allreduce_sum([dz, dD])

    def fstep():
        fwd(Sg, c32["coef"])

    return dict(plan=gpl, gstep=gstep, gstep_res=gstep_res, fstep=fstep, Bg=Bg, dz=dz, dD=dD)


def _evaluate_setup(aok, _dev, _lib, torch, L, nX, FT, with_pb=False):
    W = aok.workloads
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    X, sidx = W.config1_points(nX=nX)
    pl = _dev.OrbPlan(b.zeta.shape[0], b.K, b.NZ, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L, orb.Rnl.kind,
                      _dev.prec_of(FT))
    d = dict(plan=pl, X=_dev.to_colmajor(X, FT), sidx=torch.as_tensor(sidx).cuda(), z=_dev.to_colmajor(b.zeta, FT),
             D=_dev.to_colmajor(b.D, FT), P=_dev.colmajor_empty((nX, len(orb)), FT),
             dP=_dev.colmajor_empty((3, nX, len(orb)), FT), nX=nX, nOrb=len(orb), b=b, orb=orb, Xh=X, sh=sidx)
    if with_pb:
        rng = np.random.default_rng(1003)
        d["dPin"] = _dev.to_colmajor(rng.standard_normal((nX, len(orb))), FT)
        d["dX"] = _dev.colmajor_empty((3, nX), FT)
        d["dz"] = _dev.colmajor_empty(b.zeta.shape, FT)
        d["dD"] = _dev.colmajor_empty(b.zeta.shape, FT)
    return d


def _overlap3c_setup(aok, _dev, _lib, torch, L, B, FT):
    W = aok.workloads
    b = W.config0_basis()
    ls, nprim, z, D = W.gb_tables(b)
    # contracted, normalised coefficients from the library's own compile step (FP64)
    coef_full = aok.compile_coef(torch.as_tensor(b.zeta), torch.as_tensor(b.D), b.ls).cpu().numpy()
    coef = np.concatenate([coef_full[s, :nprim[s], 0] for s in range(len(ls))])
    tr = W.config4_triples(B=B)
    N = int(((ls + 1) * (ls + 2) // 2).sum())
    pl = _dev.Plan(ls, int(nprim.max()), 1, _dev.prec_of(FT), B)
    off = np.concatenate([[0], np.cumsum(nprim)])
    d = dict(plan=pl, N=N, B=B, nprim=torch.as_tensor(nprim).cuda(), off=torch.as_tensor(off).cuda(),
             coef=torch.as_tensor(coef).to("cuda", FT), alpha=torch.as_tensor(z).to("cuda", FT),
             pA=_dev.to_colmajor(tr.posA, FT), pB=_dev.to_colmajor(tr.posB, FT), pC=_dev.to_colmajor(tr.posC, FT),
             out=_dev.colmajor_empty((N, N, N, B), FT), ls=ls, nprim_h=nprim, coef_h=coef, z_h=z, tr=tr)
    return d


def _outputbound_setup(aok, _dev, _lib, torch, L, B, FT, basis=None):
    """The output-bound 2C case: config-2 shell structure, one primitive per shell (or
    the given basis, e.g. its s and p shells alone)."""
    ob = basis if basis is not None else aok.workloads.outputbound_basis()
    obp = aok.workloads.ragged_pairs(B, ob.NZ, SEED + 1)
    Nob = ob.nbf_total
    pl = _dev.Plan(ob.ls, ob.K, ob.NZ, _dev.prec_of(FT), obp.B)
    zt, Dt = _dev.to_colmajor(ob.zeta, FT), _dev.to_colmajor(ob.D, FT)
    cf = _dev.colmajor_empty((ob.nshells, ob.K, ob.NZ), FT)
    _lib.check(L.aok_compile_coef(pl.h, _dev.ptr(cf), _dev.ptr(zt), _dev.ptr(Dt), _dev.stream()))
    pa, pb = _dev.to_colmajor(obp.posA, FT), _dev.to_colmajor(obp.posB, FT)
    sa, sb = torch.as_tensor(obp.sidxA).cuda(), torch.as_tensor(obp.sidxB).cuda()
    o = _dev.colmajor_empty((Nob, Nob, obp.B), FT)
    ch = (ctypes.c_int64 * 3)()
    _lib.check(L.aok_plan_autotune(pl.h, _dev.ptr(o), _dev.ptr(zt), _dev.ptr(cf), _dev.ptr(pa), _dev.ptr(pb),
                                   ctypes.c_void_p(sa.data_ptr()), ctypes.c_void_p(sb.data_ptr()), obp.B, 1.0,
                                   _dev.stream(), ch))
    fn = lambda: _lib.check(L.aok_overlap2c(pl.h, _dev.ptr(o), None, None, _dev.ptr(pa), _dev.ptr(pb),
                                            ctypes.c_void_p(sa.data_ptr()), ctypes.c_void_p(sb.data_ptr()),
                                            obp.B, 1.0, _dev.stream()))
    return dict(plan=pl, fn=fn, N=Nob, B=obp.B, keep=(zt, cf, pa, pb, sa, sb, o),
                shape={"ctas_per_sm": int(ch[0]), "stage_bytes": int(ch[1])})


def side_workload(name, L, _dev, _lib, aok, torch, B=None, FT=None):
    """One launch chain of a side workload, for ncu captures (--profile --workload ...)."""
    if name == "outputbound":
        d = _outputbound_setup(aok, _dev, _lib, torch, L, B or B_PER_RANK, FT or torch.float32)
        side_workload.keep = d
        return d["fn"]
    if name == "outputbound_sp":
        d = _outputbound_setup(aok, _dev, _lib, torch, L, B or B_SP, FT or torch.float32,
                               aok.workloads.outputbound_sp_basis())
        side_workload.keep = d
        return d["fn"]
    if name in ("evaluate", "pullback"):
        d = _evaluate_setup(aok, _dev, _lib, torch, L, 1 << 20 if name == "evaluate" else 1 << 18, torch.float32,
                            with_pb=(name == "pullback"))
        if name == "evaluate":
            return lambda: _lib.check(L.aok_evaluate_ed(d["plan"].h, _dev.ptr(d["P"]), _dev.ptr(d["dP"]),
                                                        _dev.ptr(d["X"]), ctypes.c_void_p(d["sidx"].data_ptr()),
                                                        _dev.ptr(d["z"]), _dev.ptr(d["D"]), d["nX"], 1.0,
                                                        _dev.stream()))
        return lambda: _lib.check(L.aok_evaluate_pullback(d["plan"].h, _dev.ptr(d["dX"]), _dev.ptr(d["dz"]),
                                                          _dev.ptr(d["dD"]), _dev.ptr(d["dPin"]), _dev.ptr(d["X"]),
                                                          ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["z"]),
                                                          _dev.ptr(d["D"]), d["nX"], 1.0, _dev.stream()))
    d = _overlap3c_setup(aok, _dev, _lib, torch, L, 4096, FT or torch.float32)
    return lambda: _lib.check(L.aok_overlap3c_gb(d["plan"].h, _dev.ptr(d["out"]), ctypes.c_void_p(d["nprim"].data_ptr()),
                                                 ctypes.c_void_p(d["off"].data_ptr()),
                                                 ctypes.c_void_p(d["coef"].data_ptr()),
                                                 ctypes.c_void_p(d["alpha"].data_ptr()), _dev.ptr(d["pA"]),
                                                 _dev.ptr(d["pB"]), _dev.ptr(d["pC"]), d["B"], _dev.stream()))


def _timeline(fn, steps, warmup, torch):
    """Warm launch list: `warmup` untimed steps, then `steps` steps under torch.profiler (CUPTI
    activity records, device timestamps).  Prints the last step's launches (start and end in us
    from its first launch, duration) and each kernel's mean duration over all profiled steps."""
    from torch.profiler import ProfilerActivity, profile
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(steps):
            fn()
        torch.cuda.synchronize()
    ev = sorted((e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA),
                key=lambda e: e.time_range.start)
    per = max(1, len(ev) // max(steps, 1))
    last = ev[-per:]
    t0 = last[0].time_range.start
    print(f"last step: {per} launches, {last[-1].time_range.end - t0:.1f} us from the first start to the last end")
    print(" start_us   end_us    dur_us  launch")
    for e in last:
        a, b = e.time_range.start - t0, e.time_range.end - t0
        print(f"{a:8.1f} {b:8.1f} {b - a:9.1f}  {e.name[:100]}")
    agg = {}
    for e in ev:
        agg.setdefault(e.name[:100], []).append(e.time_range.end - e.time_range.start)
    print(" mean_us  count  kernel")
    for k, v in sorted(agg.items(), key=lambda kv: -sum(kv[1])):
        print(f"{sum(v) / len(v):8.2f} {len(v):6d}  {k}")
    return 0


def _time(fn, steps, warmup, torch, allmax):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(steps):
        fn()
    en.record()
    torch.cuda.synchronize()
    return allmax(st.elapsed_time(en) / steps)


def side_measurements(args, L, _dev, _lib, aok, torch, oracle, allmax, peaks):
    """Config 1 (evaluate_ed, nX=2^20), the evaluate pullback at nX=2^18 (config 3)
    and config 4 (3C, B=4096): times, throughput and error vs the oracle."""
    out = {}
    n = max(5, min(200, args.steps // 10))
    # output-bound 2C: the config-2 shell structure with one primitive per shell
    # and its low-l classes alone (s and p shells, one primitive each), at a batch whose
    # output is larger than L2
    for key, basis, Bo, note in (
            ("outputbound_2c_K1_B65536", None, B_PER_RANK, "config-2 shell structure, one primitive per shell"),
            ("outputbound_2c_sp_K1_B262144", aok.workloads.outputbound_sp_basis(), B_SP,
             "low-l classes alone: 3-5 s and 2-3 p shells per species, one primitive per shell")):
        res = {}
        for FT, tag in ((torch.float32, "f32c"), (torch.float64, "f64")):
            d = _outputbound_setup(aok, _dev, _lib, torch, L, Bo, FT, basis)
            pl, fn, Nob, obB = d["plan"], d["fn"], d["N"], d["B"]
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            _lib.check(L.aok_plan_timing_enable(pl.h, n))
            ms = _time(fn, n, 0, torch, allmax)
            tot, cnt = ctypes.c_double(), ctypes.c_int64()
            _lib.check(L.aok_plan_timing_read(pl.h, ctypes.byref(tot), ctypes.byref(cnt)))
            kms = tot.value / max(cnt.value, 1)
            fsz = 4 if FT == torch.float32 else 8
            alg = obB * (Nob * Nob * fsz + 2 * (3 * fsz + 8))
            res[tag] = {"ms": ms, "kernel_ms": kms, "integrals_per_s": Nob * Nob * obB / (ms * 1e-3),
                        "shape": d["shape"], "kernel_hbm_gbs": alg / (kms * 1e-3) / 1e9,
                        "kernel_hbm_frac": alg / (kms * 1e-3) / 1e9 / peaks["hbm_gbs"]}
            del pl, d
        out[key] = dict(res, nbf=Nob, batch=Bo, note=note)
    # config 1
    res = {}
    for FT, tag in ((torch.float32, "f32c"), (torch.float64, "f64")):
        d = _evaluate_setup(aok, _dev, _lib, torch, L, 1 << 20, FT)
        fn = lambda: _lib.check(L.aok_evaluate_ed(d["plan"].h, _dev.ptr(d["P"]), _dev.ptr(d["dP"]), _dev.ptr(d["X"]),
                                                  ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["z"]),
                                                  _dev.ptr(d["D"]), d["nX"], 1.0, _dev.stream()))
        ms = _time(fn, n, args.warmup, torch, allmax)
        fsz = 4 if FT == torch.float32 else 8
        alg = d["nX"] * (3 * fsz + 8 + 4 * d["nOrb"] * fsz)
        m = 4096
        zz, DD, XX = d["b"].zeta, d["b"].D, d["Xh"][:, :m]
        if FT == torch.float32:
            zz, DD, XX = [a.astype(np.float32).astype(np.float64) for a in (zz, DD, XX)]
        Pr, dPr = oracle.evaluate_ed(XX, d["sh"][:m], zz, DD, d["orb"].Rnl.powers(), d["orb"].radidx,
                                     d["orb"].ylmidx, d["orb"].L, nthreads=os.cpu_count())
        Pg = d["P"][:m].double().cpu().numpy()
        dPg = d["dP"][:, :m].double().cpu().numpy()
        err = float(np.sqrt(np.sum((Pg - Pr) ** 2) + np.sum((dPg - dPr) ** 2)) / np.sqrt(np.sum(Pr ** 2) + np.sum(dPr ** 2)))
        res[tag] = {"ms": ms, "points_per_s": d["nX"] / (ms * 1e-3), "hbm_gbs": alg / (ms * 1e-3) / 1e9,
                    "hbm_frac": alg / (ms * 1e-3) / 1e9 / peaks["hbm_gbs"], "rel_err_vs_oracle": err}
        del d
    out["config1_evaluate_ed_nX_2^20"] = res
    # config 3, evaluate pullback at nX = 2^18
    d = _evaluate_setup(aok, _dev, _lib, torch, L, 1 << 18, torch.float32, with_pb=True)
    fwd = lambda: _lib.check(L.aok_evaluate_ed(d["plan"].h, _dev.ptr(d["P"]), _dev.ptr(d["dP"]), _dev.ptr(d["X"]),
                                               ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["z"]),
                                               _dev.ptr(d["D"]), d["nX"], 1.0, _dev.stream()))
    pb = lambda: _lib.check(L.aok_evaluate_pullback(d["plan"].h, _dev.ptr(d["dX"]), _dev.ptr(d["dz"]),
                                                    _dev.ptr(d["dD"]), _dev.ptr(d["dPin"]), _dev.ptr(d["X"]),
                                                    ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["z"]),
                                                    _dev.ptr(d["D"]), d["nX"], 1.0, _dev.stream()))
    fms = _time(fwd, n, args.warmup, torch, allmax)
    pms = _time(pb, n, args.warmup, torch, allmax)
    out["config3_evaluate_pullback_nX_2^18_f32c"] = {"evaluate_ed_ms": fms, "pullback_ms": pms,
                                                      "pullback_over_forward": pms / fms}
    del d
    # config 4
    res = {}
    for FT, tag in ((torch.float32, "f32c"), (torch.float64, "f64")):
        d = _overlap3c_setup(aok, _dev, _lib, torch, L, 4096, FT)
        fn = lambda: _lib.check(L.aok_overlap3c_gb(d["plan"].h, _dev.ptr(d["out"]), ctypes.c_void_p(d["nprim"].data_ptr()),
                                                   ctypes.c_void_p(d["off"].data_ptr()),
                                                   ctypes.c_void_p(d["coef"].data_ptr()),
                                                   ctypes.c_void_p(d["alpha"].data_ptr()), _dev.ptr(d["pA"]),
                                                   _dev.ptr(d["pB"]), _dev.ptr(d["pC"]), d["B"], _dev.stream()))
        ms = _time(fn, n, args.warmup, torch, allmax)
        m = 256
        tr = d["tr"]
        cs, zs = d["coef_h"], d["z_h"]
        pa, pb_, pc = tr.posA[:, :m], tr.posB[:, :m], tr.posC[:, :m]
        if FT == torch.float32:
            cs, zs, pa, pb_, pc = [a.astype(np.float32).astype(np.float64) for a in (cs, zs, pa, pb_, pc)]
        ref = oracle.overlap3c_gb(d["ls"], d["nprim_h"], cs, zs, pa, pb_, pc, nthreads=os.cpu_count())
        got = d["out"][:, :, :, :m].double().cpu().numpy()
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        res[tag] = {"ms": ms, "integrals_per_s": d["N"] ** 3 * d["B"] / (ms * 1e-3), "rel_err_vs_oracle": err}
        del d
    res["f32c_over_f64"] = res["f32c"]["integrals_per_s"] / res["f64"]["integrals_per_s"]
    out["config4_overlap3c_B_4096"] = res
    return out


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    sys.exit(main())
