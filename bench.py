#!/usr/bin/env python
"""Throughput of the QMIV metric hot path on B200: IV-PSNR + WS-PSNR + IV-SSIM frame pairs per second
on 4096x2048 10-bit 4:2:0 equirectangular pairs (the reference's workload, synthetic frames).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qmiv|reference]

One step = one pass of the metric pipeline over a batch of 8 frame pairs per GPU. N > 1 runs one
process per GPU (torchrun); pairs are independent, so every rank processes its own 8 pairs (weak
scaling, no collective on the data path) and rank 0 prints one JSON line.

`--impl reference` times the reference's own multithreaded CPU implementation (the QMIV app built
from its sources into oracle/_ref by oracle/Makefile) on the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, BD, CF = 4096, 2048, 10, 420
PAIRS_PER_STEP = 8
METRIC_NAME = "IV-PSNR frame-pairs/s @4096x2048 10b"
# DRAM bytes of one 8-pair k_cps_multi launch: ncu dram__bytes_read.sum + dram__bytes_write.sum of a
# one-pair launch of the same kernel (50.4 MB of frames read, 71.2 MB of IV-SSIM sub-block moments and
# row sums written) times the 8 pairs; every pair is read once and its moments written once
CPS_TRAFFIC_BYTES = 8 * (50.45e6 + 71.17e6)
METRICS = ("IVPSNR", "WSPSNR", "IVSSIM")
# values of the headline pair compared with the reference library's
PARITY_KEYS = ("gcd_r2t", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r", "wspsnr_pic", "ivssim", "ivssim_r2t", "ivssim_t2r")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------
def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, local):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
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
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------------
def make_workload(rank, n=None):
    n = n or PAIRS_PER_STEP
    from qmiv_b200 import synth
    t0 = time.time()
    pairs = [synth.make_pair(W, H, BD, seed=1000 * rank + i) for i in range(n)]
    log(f"[rank {rank}] generated {n} synthetic {W}x{H} {BD}-bit pairs in {time.time() - t0:.1f}s")
    return pairs


def frame_bytes(frame):
    return int(sum(p.nbytes for p in frame))


def cps_candidates(R=2):
    return 2 * W * H * (2 * R + 1) ** 2


def frame_pool(specs):
    """Device-resident synthetic pairs, one per (width, height, bit depth) of the specs."""
    import torch
    from qmiv_b200 import synth
    pool = {}
    for s in specs:
        key = (s["width"], s["height"], s["bitdepth"])
        if key not in pool:
            f0, f1 = synth.make_pair(*key, seed=len(pool))
            pool[key] = (tuple(torch.from_numpy(p).cuda() for p in f0), tuple(torch.from_numpy(p).cuda() for p in f1))
    return pool


def run_serve(ctx, duration_s, rate=200.0, host=True):
    """The serving loop on a seeded Poisson stream of requests (rate per second, each 1..32 pairs of one
    shape and metric set drawn as the mixed set), 40 GB HBM budget. host=True: every request hands
    pinned host frames to the server, which admits it against the budget and uploads its frames (the
    data a request carries crosses the host link inside its latency); the frames come from a pool of 8
    distinct pairs per (resolution, bit depth). host=False: frames already resident on the device."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    reqs = synth.config4_requests(duration_s, rate, seed=4)
    keys = sorted({(s["width"], s["height"], s["bitdepth"]) for r in reqs for s in r.specs})
    npool = 8 if host else 1
    pool = {}
    for k in keys:
        pool[k] = []
        for i in range(npool):
            f0, f1 = synth.make_pair(*k, seed=17 * i + k[0] + k[2])
            if host:
                pool[k].append((tuple(torch.from_numpy(p).pin_memory() for p in f0),
                                tuple(torch.from_numpy(p).pin_memory() for p in f1)))
            else:
                pool[k].append((tuple(torch.from_numpy(p).cuda() for p in f0), tuple(torch.from_numpy(p).cuda() for p in f1)))

    def pairs_of(key, n, off):
        return [pool[key][(off + i) % npool] for i in range(n)]

    sctx = qmiv_b200.Context(ctx.device, hbm_budget=40 << 30)
    srv = qmiv_b200.Server(sctx, max_batch_pairs=64, max_batch_pixels=64 * 4096 * 2048, workers=2)
    # warm-up: every (shape, R) kind once, so kernels are configured and tiles tuned before the stream,
    # then two concurrent requests of the largest size, so that both workers' device scratch has grown
    # to a full batch before the stream (a server reserves its working memory at start-up)
    seen = set()
    for r in reqs:
        s0 = r.specs[0]
        k = (s0["width"], s0["height"], s0["bitdepth"], s0["search_range"], r.metrics)
        if k not in seen:
            seen.add(k)
            srv.wait(srv.submit(pairs_of(k[:3], 1, 0), *k[:3], search_range=k[3], metrics=r.metrics))
    big = max(seen, key=lambda k: k[0] * k[1] * k[2] * (2 * k[3] + 1))
    warm = [srv.submit(pairs_of(big[:3], 32, j), *big[:3], search_range=big[3], metrics=big[4]) for j in range(2)]
    for t in warm:
        srv.wait(t)
    srv.stats(reset=True)
    tickets = []
    t0 = time.perf_counter()
    for j, r in enumerate(reqs):
        delay = t0 + r.arrival_s - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        s0 = r.specs[0]
        key = (s0["width"], s0["height"], s0["bitdepth"])
        tickets.append(srv.submit(pairs_of(key, len(r.specs), j), *key, search_range=s0["search_range"],
                                  metrics=r.metrics))
    queue_ms = []
    for t in tickets:
        _, st = srv.wait(t)
        queue_ms.append(st["admit_ms"] - st["submit_ms"])
    stats = srv.stats()
    srv.close()
    sctx.close()
    queue_ms.sort()
    up = sum(2 * s["width"] * s["height"] * 3 // 2 * (1 if s["bitdepth"] <= 8 else 2) for r in reqs for s in r.specs)
    return {"p50_ms": stats["p50_ms"], "p99_ms": stats["p99_ms"], "pairs_per_s": stats["pairs_per_s"],
            "requests": stats["completed"], "pairs": sum(len(r.specs) for r in reqs),
            "admit_wait_ms_p50": queue_ms[len(queue_ms) // 2], "admit_wait_ms_p99": queue_ms[int(0.99 * (len(queue_ms) - 1))],
            "host_bytes": up if host else 0, "ingest": "host" if host else "device"}


def run_mixed(ctx, steps, int_peak):
    """The mixed-resolution set (64 pairs, resolution / bit depth / R drawn per pair; IV-PSNR + PSNR +
    IV-SSIM): the plain form (one call per pair) against the batched form (one launch per stage,
    graphs, autotuned tiles). Pairs of one (resolution, bit depth) share their synthetic content, each
    from its own device copy."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    specs = synth.config3_specs(64, 3)
    pool = frame_pool(specs)
    # every pair reads its own device copy of its shape's content, so no pair finds another's frames in L2
    own = [tuple(tuple(p.clone() for p in f) for f in pool[(s["width"], s["height"], s["bitdepth"])]) for s in specs]
    mask = qmiv_b200.IVPSNR | qmiv_b200.PSNR | qmiv_b200.IVSSIM
    calcs = {}
    for s in specs:
        k = (s["width"], s["height"], s["bitdepth"], s["search_range"])
        if k not in calcs:
            calcs[k] = qmiv_b200.Calc(ctx, s["width"], s["height"], s["bitdepth"], 420, search_range=s["search_range"])

    def plain():
        return [calcs[(s["width"], s["height"], s["bitdepth"], s["search_range"])].compute(*own[i], mask)
                for i, s in enumerate(specs)]

    descs = [dict(frame0=own[i][0], frame1=own[i][1], width=s["width"], height=s["height"],
                  bitdepth=s["bitdepth"], search_range=s["search_range"], metrics=mask) for i, s in enumerate(specs)]
    batch = qmiv_b200.Batch(ctx, len(specs), sum(s["width"] * s["height"] for s in specs), graph=True, autotune=True)
    out = {}
    for name, fn in (("plain", plain), ("batched", lambda: batch.compute(descs))):
        for _ in range(3):
            r = fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            r = fn()
        torch.cuda.synchronize()
        out[name] = steps * len(specs) / (time.perf_counter() - t0)
        out[name + "_results"] = r
    assert out.pop("plain_results") == out["batched_results"], "plain and batched forms differ on the mixed set"
    # the batched form with two calls in flight (qmiv_batch_submit / qmiv_batch_wait), as the headline runs
    for _ in range(2):
        ta, tb = batch.submit(descs), batch.submit(descs)
        batch.wait(ta)
        batch.wait(tb)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ticket = batch.submit(descs)
    for _ in range(steps - 1):
        nxt = batch.submit(descs)
        assert batch.wait(ticket) == out["batched_results"], "pipelined and synchronous batches differ"
        ticket = nxt
    assert batch.wait(ticket) == out.pop("batched_results"), "pipelined and synchronous batches differ"
    torch.cuda.synchronize()
    out["two_in_flight"] = steps * len(specs) / (time.perf_counter() - t0)
    # CPS search kernel per search range: the batched form on the pairs of one R with the stage timers on
    per_r = {}
    for R in sorted({s["search_range"] for s in specs}):
        sub = [d for d in descs if d["search_range"] == R]
        ctx.stage_times(reset=True)
        ctx.set_profiling(True)
        for _ in range(3):
            batch.compute(sub)
        torch.cuda.synchronize()
        ctx.set_profiling(False)
        ms, n = ctx.stage_times(reset=True)["cps"]
        cand = sum(2 * d["width"] * d["height"] * (2 * R + 1) ** 2 for d in sub)
        per_r[f"R{R}"] = {"pairs": len(sub), "cps_ms": ms / 3, "frac": 8.0 * cand / (ms / 3 * 1e-3) / 1e12 / int_peak}
    batch.close()
    for c in calcs.values():
        c.close()
    return {"plain_pairs_s": out["plain"], "batched_pairs_s": out["batched"], "cps_by_R": per_r,
            "batched_two_in_flight_pairs_s": out["two_in_flight"], "two_in_flight_over_plain": out["two_in_flight"] / out["plain"],
            "batched_over_plain": out["batched"] / out["plain"]}


def run_qmiv(args, world, rank, local):
    import torch
    import qmiv_b200
    from qmiv_b200 import _lib

    torch.cuda.set_device(local)
    pairs = make_workload(rank)
    mask = qmiv_b200.metric_mask(METRICS)
    dev_pairs = [tuple(tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in fr) for fr in pr) for pr in pairs]
    host_pairs = [tuple(tuple(torch.from_numpy(np.ascontiguousarray(p)).pin_memory() for p in fr) for fr in pr)
                  for pr in pairs]
    host_np = [tuple(tuple(t.numpy() for t in fr) for fr in pr) for pr in host_pairs]

    def descs(src):
        return [dict(frame0=a, frame1=b, width=W, height=H, bitdepth=BD, chroma_format=CF, search_range=2,
                     metrics=mask) for a, b in src]

    ctx = qmiv_b200.Context(local)
    batch = qmiv_b200.Batch(ctx, max_pairs=PAIRS_PER_STEP, max_pixels=PAIRS_PER_STEP * W * H, erp=True, graph=True,
                            autotune=not args.no_autotune)
    stream = torch.cuda.ExternalStream(batch.stream(), device=f"cuda:{local}")
    dev_desc, host_desc = descs(dev_pairs), descs(host_np)

    for _ in range(args.warmup):
        batch.compute(dev_desc)
    torch.cuda.synchronize()

    # ---- device-resident inputs (value) ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        results = None
        for _ in range(args.steps):
            results = batch.compute(dev_desc)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms_sync = max_over_ranks(ev0.elapsed_time(ev1), world, local)

    # ---- the same steps with two batches in flight (qmiv_batch_submit / qmiv_batch_wait on two engines
    # and streams): one step's serial pooling chains overlap the next step's search. Every step still
    # computes all of its pairs; the results are checked against the synchronous run. ----
    for _ in range(2):
        ta, tb = batch.submit(dev_desc), batch.submit(dev_desc)
        batch.wait(ta)
        batch.wait(tb)
    torch.cuda.synchronize()
    def pipelined_ms():
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        ticket = batch.submit(dev_desc)
        for _ in range(args.steps - 1):
            nxt = batch.submit(dev_desc)
            assert batch.wait(ticket) == results, "pipelined and synchronous batches differ"
            ticket = nxt
        assert batch.wait(ticket) == results, "pipelined and synchronous batches differ"
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(ev0.elapsed_time(ev1), world, local)

    with ClockSampler(local) as clocks:
        ms_max = pipelined_ms()
    # the same timed region repeated: the spread of the measurement (the headline value is the first)
    rep_ms = [pipelined_ms() for _ in range(5)]

    # ---- per-stage kernel times: the same steps with the library's stage timers (CUDA events on the
    # batch stream around every stage's launch; graphs are not replayed while the timers are on) ----
    ctx.stage_times(reset=True)
    ctx.set_profiling(True)
    prof_steps = max(3, args.steps // 4)
    for _ in range(prof_steps):
        assert batch.compute(dev_desc) == results, "timed and replayed batches differ"
    torch.cuda.synchronize()
    ctx.set_profiling(False)
    stage = ctx.stage_times(reset=True)
    launches_per_step = sum(v[1] for k, v in stage.items() if k not in ("h2d", "d2h")) / prof_steps

    # ---- the plain one-pair-per-call form on the same pairs ----
    calc = qmiv_b200.Calc(ctx, W, H, BD, CF, search_range=2, erp=True)
    for a, b in dev_pairs[:2]:
        calc.compute(a, b, mask)
    torch.cuda.synchronize()
    p0 = time.perf_counter()
    plain_steps = max(1, args.steps // 4)
    for _ in range(plain_steps):
        for i, (a, b) in enumerate(dev_pairs):
            assert calc.compute(a, b, mask) == results[i], "plain and batched forms differ"
    torch.cuda.synchronize()
    plain_value = plain_steps * len(dev_pairs) / (time.perf_counter() - p0)
    calc.close()

    # ---- end to end through the public API, pinned host frames (e2e) ----
    # Two calls in flight (qmiv_batch_submit / qmiv_batch_wait): each step's uploads overlap the
    # previous step's kernels. Every step still copies its frames from pinned host memory and reads
    # its results back inside the timed region.
    for _ in range(max(1, args.warmup // 2)):
        ta, tb = batch.submit(host_desc), batch.submit(host_desc)
        batch.wait(ta)
        batch.wait(tb)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ticket = batch.submit(host_desc)
    for _ in range(args.steps - 1):
        nxt = batch.submit(host_desc)
        host_results = batch.wait(ticket)
        ticket = nxt
    host_results = batch.wait(ticket)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, local)
    assert host_results == results, "host-frame and device-frame results differ"

    cps_tile = batch.tuning(W, H, BD, 2)

    # ---- probes for the search kernel's roofline denominator ----
    lib = qmiv_b200.library()
    int_peak = __import__("ctypes").c_double()
    _lib.check(lib.qmiv_probe_int32_peak(local, 4096, __import__("ctypes").byref(int_peak)), "probe")

    solo = world == 1
    side = max(3, args.steps // 4)

    def leg(name, fn, on):
        if not (solo and on):
            return None
        log(f"[bench] {name}")
        return fn()

    mixed = leg("mixed set", lambda: run_mixed(ctx, side, int_peak.value), not args.no_mixed)
    serve = leg("serving", lambda: {"host": run_serve(ctx, args.serve_seconds, host=True),
                                    "device": run_serve(ctx, args.serve_seconds, host=False)}, args.serve_seconds > 0)
    masked = leg("mask mode", lambda: run_masked(ctx, side), not args.no_masked)
    ssim_modes = leg("ssim options", lambda: run_ssim_modes(ctx, side), not args.no_ssim_modes)
    c0 = leg("1080p 8-bit", lambda: run_config0(ctx, side), not args.no_configs)
    c2 = leg("MS-SSIM workload", lambda: run_config2(ctx, side, hbm_peak()), not args.no_configs)

    batch.close()
    ctx.close()

    units = world * PAIRS_PER_STEP * args.steps
    value = units / (ms_max / 1e3)
    e2e_value = units / (e2e_ms / 1e3)
    cps_ms, cps_n = stage["cps"]
    cps_avg_ms = cps_ms / max(cps_n, 1)
    ops_per_launch = 8.0 * cps_candidates() * PAIRS_PER_STEP  # one work-list launch covers the step's pairs
    achieved = ops_per_launch / (cps_avg_ms * 1e-3) / 1e12
    h2d = sum(frame_bytes(a) + frame_bytes(b) for a, b in pairs)
    d2h = PAIRS_PER_STEP * 632  # sizeof(PairOut), the device result block read back per pair
    value_sync = units / (ms_sync / 1e3)
    rep = sorted(units / (m / 1e3) for m in rep_ms)
    repeats = {"n": len(rep), "steps_each": args.steps, "pairs_s": [round(v, 1) for v in rep],
               "median": rep[len(rep) // 2], "spread": (rep[-1] - rep[0]) / rep[len(rep) // 2]}
    return dict(value=value, value_sync=value_sync, ms=ms_max / args.steps, e2e=e2e_value, stage=stage, cps_avg_ms=cps_avg_ms,
                repeats=repeats,
                achieved=achieved, int_peak=int_peak.value, h2d=h2d, d2h=d2h, clocks=clocks.summary(),
                sample=results[0], launches=int(round(launches_per_step * args.steps)), plain=plain_value,
                cps_tile=cps_tile, mixed=mixed, serve=serve, masked=masked, ssim_modes=ssim_modes, c0=c0, c2=c2)


# ---------------------------------------------------------------------------------------------
# CPU side: the reference app on the host cores
# ---------------------------------------------------------------------------------------------
def reference_app():
    import oracle
    path = os.path.join(oracle.reference_dir(), "QMIV")
    return path if os.path.exists(path) else None


def run_reference_app(n_frames, threads, seed=0, shape=None, metrics=METRICS, erp=True, gen=None):
    """The QMIV app (oracle/_ref) on n_frames synthetic pairs written to /dev/shm: frame-pairs/s from its
    TotalProcessingTime (generation and file writing excluded) and its printed average IV-PSNR.
    shape: (W, H, bit depth), default the headline workload's; gen(i) -> (frame0, frame1)."""
    app = reference_app()
    if app is None:
        return None
    from qmiv_b200 import synth
    w, h, bd = shape or (W, H, BD)
    gen = gen or (lambda i: synth.make_pair(w, h, bd, seed=seed + i))
    tmp = tempfile.mkdtemp(dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    files = [os.path.join(tmp, "in0.yuv"), os.path.join(tmp, "in1.yuv")]
    try:
        with open(files[0], "wb") as f0, open(files[1], "wb") as f1:
            for i in range(n_frames):
                a, b = gen(i)
                for p in a:
                    f0.write(np.ascontiguousarray(p).tobytes())
                for p in b:
                    f1.write(np.ascontiguousarray(p).tobytes())
        cmd = [app, "-i0", files[0], "-i1", files[1], "-ps", f"{w}x{h}", "-bd", str(bd), "-cf", str(CF)]
        cmd += ["-erp"] if erp else []
        cmd += ["-ml", ", ".join(metrics), "-nth", str(threads), "-v", "3"]
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=900).stdout
    finally:
        for f in files:
            if os.path.exists(f):
                os.remove(f)
        os.rmdir(tmp)
    m = re.search(r"TotalProcessingTime\s*=\s*([0-9.]+)\s*s", out)
    if not m:
        raise RuntimeError("could not parse the reference app's output:\n" + out[-2000:])
    secs = float(m.group(1))
    ivpsnr = re.search(r"Average\s+IVPSNR\s+([0-9.]+)", out)
    return dict(value=n_frames / secs, secs=secs, frames=n_frames, threads=threads,
                ivpsnr=float(ivpsnr.group(1)) if ivpsnr else None)


def in_child(fn, *args, timeout=600):
    """fn(*args) in a spawned child process: the reference library runs its own thread pool in native
    code, and a crash there ends only the child (the value is then None and the reason is logged)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        try:
            return pool.apply_async(fn, args).get(timeout)
        except Exception as e:  # the child died or timed out: this field stays empty
            log(f"{fn.__name__} failed in its child process: {e!r}")
            return None


def reference_parity(frame0, frame1, shape, search_range, erp, mask, gpu, keys, threads):
    """The reference library (oracle/_ref, compiled from the reference's sources) on one pair of the
    timed workload: its exact doubles beside the GPU's, and whether every listed value is equal."""
    import oracle
    if not oracle.reference_available():
        return None
    w, h, bd = shape
    ref = oracle.Reference().compute_pair(oracle.make_params(w, h, bd, CF, search_range=search_range, erp=erp,
                                                             num_threads=threads), frame0, frame1, mask)
    return {"bit_exact": all(gpu[k] == ref[k] for k in keys),
            "gpu": {k: gpu[k] for k in keys}, "reference": {k: ref[k] for k in keys}}


C0 = (1920, 1080, 8)      # the reference's CPU-runnable case: one 8-bit 1080p pair, IV-PSNR, R = 2
C2 = (2048, 2048, 10)     # MS-SSIM / IV-MS-SSIM: 16 blurred 2048x2048 10-bit pairs, 5 scales


def run_config0(ctx, steps):
    """1920x1080 8-bit 4:2:0, R = 2, IV-PSNR, one pair per qmiv_frame_pair_compute call (the reference's
    frame-at-a-time method): device frames (value; 24 distinct device copies) and pinned host frames
    with the upload and the result read-back in the timed region (e2e)."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    w, h, bd = C0
    pairs = [synth.make_pair(w, h, bd, seed=500 + i) for i in range(8)]
    # 24 device copies (150 MB, above the 126 MB L2) taken in turn: no call finds its frames in L2
    dev = [tuple(tuple(torch.from_numpy(p).cuda() for p in f) for f in pr) for _ in range(3) for pr in pairs]
    host = [tuple(tuple(torch.from_numpy(p).pin_memory() for p in f) for f in pr) for pr in pairs]
    mask = qmiv_b200.IVPSNR
    out = {}
    with qmiv_b200.Calc(ctx, w, h, bd, CF, search_range=2) as calc:
        for name, src in (("value", dev), ("e2e", host)):
            for a, b in src[:3]:
                r = calc.compute(a, b, mask)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps):
                for a, b in src:
                    r = calc.compute(a, b, mask)
            torch.cuda.synchronize()
            out[name] = steps * len(src) / (time.perf_counter() - t0)
        r0 = calc.compute(dev[0][0], dev[0][1], mask)
    return {"value": out["value"], "e2e": out["e2e"], "result0": r0, "pair0": pairs[0]}


def run_config2(ctx, steps, hbm_peak):
    """MS-SSIM + IV-MS-SSIM of 16 blurred 2048x2048 10-bit 4:2:0 pairs per step through the batched form
    (graphs, autotuned tiles), device frames; the moment kernels (exact sub-block moments with the next
    scale's 2x2 downsampling fused) against the HBM bandwidth."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    w, h, bd = C2
    t0 = time.time()
    pairs = synth.config2(n=16)
    log(f"generated 16 blurred {w}x{h} pairs in {time.time() - t0:.1f}s")
    dev = [tuple(tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f) for f in pr) for pr in pairs]
    mask = qmiv_b200.MSSSIM | qmiv_b200.IVMSSSIM
    descs = [dict(frame0=a, frame1=b, width=w, height=h, bitdepth=bd, search_range=2, metrics=mask) for a, b in dev]
    with qmiv_b200.Batch(ctx, len(descs), len(descs) * w * h, graph=True, autotune=True) as batch:
        for _ in range(3):
            res = batch.compute(descs)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(steps):
            assert batch.compute(descs) == res, "repeated MS-SSIM batches differ"
        torch.cuda.synchronize()
        value = steps * len(descs) / (time.perf_counter() - t1)
        ctx.stage_times(reset=True)
        ctx.set_profiling(True)
        for _ in range(3):
            batch.compute(descs)
        torch.cuda.synchronize()
        ctx.set_profiling(False)
        st = ctx.stage_times(reset=True)
    mom_ms = st["ssim_win"][0] / 3
    # algorithmic bytes of one pair's moment launches: per scale the four pictures (In0, In1 and the two
    # shift-compensated pictures SCP0, SCP1) read once (scale 0: the raw 4:2:0 frames, 3 bytes per pixel,
    # and the 16-bit 4:4:4 SCPs, 6; later scales 16-bit 4:4:4, 6 each), five uint32 moment planes per
    # component per 4x4 block for each of the three pairs of pictures (MS-SSIM (In0, In1), IV-MS-SSIM
    # (In0, SCP1) and (In1, SCP0): 3 x 3.75 bytes per pixel) and, below the last scale, each picture's
    # 2x2 means (16-bit 4:4:4 at a quarter of the pixels) written once
    px = [w * h / 4 ** k for k in range(5)]
    per_pair = px[0] * (3 + 3 + 6 + 6) + sum(px[k] * 4 * 6 for k in range(1, 5))
    per_pair += sum(px[k] * 3 * 3.75 for k in range(5)) + sum(px[k] * 4 * 6 / 4 for k in range(4))
    gbs = per_pair * len(descs) / (mom_ms * 1e-3) / 1e9
    return {"value": value, "stage_ms": {k: v[0] / 3 for k, v in st.items() if v[1]},
            "moments": {"ms_per_step": mom_ms, "bytes_per_pair": per_pair, "achieved_gbs": gbs,
                        "frac": gbs / hbm_peak[0], "peak_gbs": hbm_peak[0], "peak_kind": hbm_peak[1]},
            "result0": res[0], "pair0": pairs[0], "gen": (lambda i: pairs[i])}


def run_masked(ctx, steps):
    """Mask mode on 4096x2048 10-bit 4:2:0 ERP pairs with a block mask (60 % of 16x16 blocks kept,
    8-bit): PSNR-M + WS-PSNR-M + IV-PSNR-M through qmiv_frame_pair_compute_masked, device frames.
    Eight distinct device copies of the pair and mask (470 MB, above the 126 MB L2) are taken in turn,
    so no step finds its inputs in L2; the batched form takes all eight in one call."""
    import torch
    import qmiv_b200
    from qmiv_b200 import synth
    f0, f1 = synth.make_pair(W, H, BD, seed=77)
    m = synth.make_mask(W, H, 8, seed=77)
    nb = 8
    d0 = [tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f0) for _ in range(nb)]
    d1 = [tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f1) for _ in range(nb)]
    dm = [torch.from_numpy(m).cuda() for _ in range(nb)]
    with qmiv_b200.Calc(ctx, W, H, BD, CF, search_range=2, erp=True) as calc:
        for k in range(3):
            r, nnm = calc.compute_masked(d0[k], d1[k], dm[k], 8)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(steps):
            j = (k + 3) % nb
            r, nnm = calc.compute_masked(d0[j], d1[j], dm[j], 8)
        dt = (time.perf_counter() - t0) / steps
    # the batched form: the eight pairs in one call (qmiv_batch_compute_masked)
    pairs = [dict(frame0=d0[k], frame1=d1[k], width=W, height=H, bitdepth=BD, search_range=2,
                  metrics=qmiv_b200.PSNR | qmiv_b200.WSPSNR | qmiv_b200.IVPSNR) for k in range(nb)]
    with qmiv_b200.Batch(ctx, nb, nb * W * H, erp=True) as batch:
        for _ in range(2):
            rb, _ = batch.compute_masked(pairs, dm, [8] * nb)
        assert all(x == r for x in rb), "batched and one-pair mask mode differ"
        t0 = time.perf_counter()
        for _ in range(steps):
            batch.compute_masked(pairs, dm, [8] * nb)
        db = (time.perf_counter() - t0) / steps
    return {"value": 1.0 / dt, "unit": "frame-pairs/s", "ms_per_pair": dt * 1e3, "batched_pairs_s": nb / db,
            "num_non_masked": nnm, "ivpsnr": r["ivpsnr"], "l2": "8 distinct device copies (470 MB) taken in turn"}


def run_reference_masked(threads, seed=77, reps=2):
    """The reference's mask-mode processors (xGlobClrDiff::CalcGlobalColorDiffM, xPSNR::calcPicPSNRM,
    xWSPSNR::calcPicWSPSNRM, xIVPSNRM::calcPicIVPSNRM) in the app's per-frame sequence, through the
    reference library compiled from its sources (oracle/_ref) with a thread pool of `threads`, on the
    masked workload: frame-pairs/s. The app binary itself cannot run its mask mode (its start-frame
    check reads past a two-entry array for the mask input and always fails)."""
    import oracle
    from qmiv_b200 import synth
    if not oracle.reference_available():
        return None
    ref = oracle.Reference()
    a, b = synth.make_pair(W, H, BD, seed=seed)
    m = synth.make_mask(W, H, 8, seed=seed)
    p = oracle.make_params(W, H, BD, CF, search_range=2, erp=True, num_threads=threads)
    r, _ = ref.compute_pair_masked(p, a, b, m, 8)           # warm-up
    t0 = time.perf_counter()
    for _ in range(reps):
        r, _ = ref.compute_pair_masked(p, a, b, m, 8)
    secs = (time.perf_counter() - t0) / reps
    return {"value": 1.0 / secs, "secs": secs, "threads": threads, "ivpsnr": r["ivpsnr"]}


# structural similarity options measured besides the default (BlockAveraged 8/4): (name, mode, border,
# window, stride); the first is the original paper's SSIM (11x11 Gaussian, every pixel)
SSIM_OPTIONS = [("RegularGaussianFlt/None/11/1", 0, 0, 11, 1), ("RegularGaussianInt/None/11/1", 1, 0, 11, 1),
                ("BlockAveraged/None/16/4", 4, 0, 16, 4)]


def ssim_option_windows(mode, window, stride):
    """Windows of one SSIM evaluation of a 4:4:4 picture of W x H (all three components)."""
    if mode <= 2:
        nx, ny = (W - 10 + stride - 1) // stride, (H - 10 + stride - 1) // stride
    else:
        nx, ny = (W - window) // stride + 1, (H - window) // stride + 1
    return 3 * nx * ny


def run_ssim_modes(ctx, steps):
    """SSIM + IV-SSIM (ERP) of one 4096x2048 10-bit 4:2:0 pair per call under other structural similarity
    options, device frames, with the window kernel's FP64 rate against the FP64 multiply/add rate
    measured on this GPU by qmiv_probe_fp64_peak."""
    import ctypes
    import torch
    import qmiv_b200
    from qmiv_b200 import _lib, synth
    f0, f1 = synth.make_pair(W, H, BD, seed=91)
    # three device copies (150 MB, above the 126 MB L2) taken in turn
    cp = [(tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f0),
           tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f1)) for _ in range(3)]
    d0, d1 = cp[0]
    mask = qmiv_b200.SSIM | qmiv_b200.IVSSIM
    peak = ctypes.c_double()
    _lib.check(qmiv_b200.library().qmiv_probe_fp64_peak(ctx.device, 4096, ctypes.byref(peak)), "probe")
    out = {"what": "SSIM + IV-SSIM (ERP) of one 4096x2048 10-bit 4:2:0 pair per synchronous call, device frames "
                   "(three device copies taken in turn)",
           "fp64_peak_tops": peak.value, "options": []}
    for name, mode, border, window, stride in SSIM_OPTIONS:
        with qmiv_b200.Calc(ctx, W, H, BD, CF, search_range=2, erp=True, ssim_mode=mode, ssim_border=border,
                            ssim_window=window, ssim_stride=stride) as calc:
            for _ in range(3):
                r = calc.compute(d0, d1, mask)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in range(steps):
                r = calc.compute(*cp[k % 3], mask)
            dt = (time.perf_counter() - t0) / steps
            ctx.stage_times(reset=True)
            ctx.set_profiling(True)
            for k in range(steps):
                calc.compute(*cp[k % 3], mask)
            ctx.set_profiling(False)
            st = ctx.stage_times(reset=True)
        win_ms, win_n = st["ssim_win"]
        # one window launch evaluates SSIM (In0, In1) and IV-SSIM (In0, SCP1), (In1, SCP0): 3 evaluations
        windows = 3 * ssim_option_windows(mode, window, stride)
        n = 11 if mode <= 2 else window
        ops_per_window = n * n * (10 if mode == 0 else 5)   # float Gaussian: multiply + add per moment and tap
        avg_ms = win_ms / max(win_n, 1)
        achieved = windows * ops_per_window / (avg_ms * 1e-3) / 1e12
        out["options"].append({"option": name, "value": 1.0 / dt, "unit": "frame-pairs/s", "ms_per_pair": dt * 1e3,
                               "ssim_pic": r["ssim_pic"], "ivssim": r["ivssim"],
                               "window_kernel": {"avg_launch_ms": avg_ms, "windows_per_launch": windows,
                                                 "fp64_ops_per_window": ops_per_window, "achieved_tops": achieved,
                                                 "frac": achieved / peak.value if peak.value else None}})
    return out


def run_reference_ssim_option(threads, option, seed=91):
    """The same pair and metrics through the reference library (oracle/_ref, xSSIM / xIVSSIM with
    setStructSimParams) with a thread pool of `threads`: frame-pairs/s of one call."""
    import oracle
    from qmiv_b200 import synth
    if not oracle.reference_available():
        return None
    _, mode, border, window, stride = option
    ref = oracle.Reference()
    a, b = synth.make_pair(W, H, BD, seed=seed)
    p = oracle.make_params(W, H, BD, CF, search_range=2, erp=True, num_threads=threads)
    t0 = time.perf_counter()
    r = ref.compute_pair_ssim(p, a, b, mode, border, window, stride, oracle.SSIM | oracle.IVSSIM)
    secs = time.perf_counter() - t0
    return {"value": 1.0 / secs, "secs": secs, "threads": threads, "ivssim": r["ivssim"], "ssim_pic": r["ssim_pic"]}


def hbm_peak():
    """(GB/s, "measured" | "fallback"): the driver-measured copy bandwidth of this pool's B200s, else
    the earlier measurement on this pool."""
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        with open(pk) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured"
    return 6650.0, "fallback"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def main():
    faulthandler.enable()   # a crash in native code prints the Python stack of every thread to stderr
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["qmiv", "reference"], default="qmiv")
    ap.add_argument("--cpu-frames", type=int, default=4, help="frames of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the plain-vs-batched mixed-resolution comparison")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="length of the serving-loop arrival stream (0: skip)")
    ap.add_argument("--no-masked", action="store_true", help="skip the mask-mode measurement")
    ap.add_argument("--no-ssim-modes", action="store_true", help="skip the structural similarity option measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the 1080p 8-bit and the MS-SSIM workloads")
    ap.add_argument("--size", default=None, help="WxH of a smaller profiling case (not a bench line)")
    ap.add_argument("--pairs", type=int, default=None, help="pairs per step of a smaller profiling case")
    ap.add_argument("--no-autotune", action="store_true",
                    help="profiling case: the default 128x32 CPS tile for the timed workload instead of the autotuner's "
                         "pick (a profiler's replay skews the timings the autotuner compares)")
    args = ap.parse_args()
    global W, H, PAIRS_PER_STEP
    if args.size:
        W, H = (int(x) for x in args.size.lower().split("x"))
    if args.pairs:
        PAIRS_PER_STEP = args.pairs
    if args.warmup < 3:
        log("warm-up raised to 3 steps")
        args.warmup = 3

    world, rank, local = dist_setup(args.gpus)
    cfg = {"workload": "IV-PSNR + WS-PSNR + IV-SSIM, 8 frame pairs per GPU per step, 4096x2048 10-bit 4:2:0 ERP",
           "width": W, "height": H, "bitdepth": BD, "chroma_format": CF, "search_range": 2,
           "pairs_per_step_per_gpu": PAIRS_PER_STEP, "metrics": list(METRICS),
           "l2": "inputs 8 pairs x 50 MB per GPU exceed the 126 MB L2; no flush needed",
           "parallelism": f"replicas{world}"}

    if args.impl == "reference":
        if rank == 0:
            threads = host_threads()
            # each step: one bounded sample of the workload through the reference app
            vals = []
            for s in range(args.warmup + args.steps):
                r = run_reference_app(max(1, args.cpu_frames // 2), threads, seed=s * 100)
                if r is None:
                    print(json.dumps({"impl": "reference", "unavailable": "reference app not built (oracle/_ref missing)"}))
                    return
                if s >= args.warmup:
                    vals.append(r)
            secs = sum(v["secs"] for v in vals)
            frames = sum(v["frames"] for v in vals)
            value = frames / secs
            out = {"metric": METRIC_NAME, "value": value, "unit": "frame-pairs/s", "n_gpus": args.gpus,
                   "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(vals),
                   "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64",
                   "data": "synthetic", "config": cfg, "impl": "reference",
                   "cpu_baseline": {"value": value, "unit": "frame-pairs/s", "cores": threads, "kind": "reference",
                                    "sample": f"{vals[0]['frames']} frame pairs per step through the QMIV app "
                                              f"(oracle/_ref) with -nth {threads}"},
                   "e2e": {"value": value, "unit": "frame-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(out))
        barrier(world)
        return

    r = run_qmiv(args, world, rank, local)
    if rank != 0:
        barrier(world)
        return
    threads = host_threads()
    cpu = parity = None
    c0, c2 = r["c0"], r["c2"]
    if world == 1 and not args.no_cpu_baseline:
        # the CPU-baseline leg: the reference (oracle/_ref, compiled from its sources) on bounded samples
        # of each workload, and its exact values for one pair of each timed workload beside the GPU's
        from qmiv_b200 import synth
        parity = {}
        try:
            c = run_reference_app(args.cpu_frames, threads)
            if c:
                cpu = {"value": c["value"], "unit": "frame-pairs/s", "cores": c["threads"], "kind": "reference",
                       "sample": f"{c['frames']} pairs of the workload, QMIV app -nth {c['threads']}, {c['secs']:.2f} s"}
            parity["headline"] = in_child(reference_parity, *synth.make_pair(W, H, BD, seed=0), (W, H, BD), 2, True,
                                          7 | 32, r["sample"], PARITY_KEYS, threads)
        except Exception as e:  # the GPU number stands without the CPU baseline
            log("cpu baseline failed:", e)
        if c0 is not None:
            try:
                cr = run_reference_app(8, threads, seed=500, shape=C0, metrics=("IVPSNR",), erp=False)
                c0["cpu_reference"] = {"value": cr["value"], "cores": threads, "ivpsnr_avg": cr["ivpsnr"]} if cr else None
                parity["config0"] = in_child(reference_parity, *c0["pair0"], C0, 2, False, 4, c0["result0"],
                                             ("gcd_r2t", "ivpsnr", "ivpsnr_r2t", "ivpsnr_t2r"), threads)
            except Exception as e:
                log("config0 cpu baseline failed:", e)
        if c2 is not None:
            try:
                cr = run_reference_app(2, threads, shape=C2, metrics=("MSSSIM", "IVMSSSIM"), erp=False, gen=c2["gen"])
                c2["cpu_reference"] = {"value": cr["value"], "cores": threads, "sample": "2 pairs"} if cr else None
                parity["config2"] = in_child(reference_parity, *c2["pair0"], C2, 2, False, 16 | 64, c2["result0"],
                                             ("msssim", "msssim_pic", "ivmsssim"), threads)
            except Exception as e:
                log("config2 cpu baseline failed:", e)
        if r["masked"] is not None:
            try:
                cm = in_child(run_reference_masked, threads)
                if cm:
                    r["masked"]["cpu_reference"] = {"value": cm["value"], "cores": cm["threads"], "ivpsnr": cm["ivpsnr"]}
            except Exception as e:
                log("masked cpu baseline failed:", e)
        if r["ssim_modes"] is not None:
            try:
                cs = in_child(run_reference_ssim_option, threads, SSIM_OPTIONS[0])
                if cs:
                    r["ssim_modes"]["options"][0]["cpu_reference"] = {"value": cs["value"], "cores": cs["threads"],
                                                                      "ivssim": cs["ivssim"]}
            except Exception as e:
                log("ssim option cpu baseline failed:", e)
    for c in (c0, c2):
        if c is not None:
            for k in ("result0", "pair0", "gen"):
                c.pop(k, None)
    if r["ssim_modes"] is not None:
        for o in r["ssim_modes"]["options"]:
            o["window_kernel"] = {k: o["window_kernel"][k] for k in ("avg_launch_ms", "achieved_tops", "frac")}
    peak = hbm_peak()
    # key order: the contract's keys, the secondary measurements, then the headline blocks last (the
    # end of the line is what a truncated log keeps)
    out = {"metric": METRIC_NAME, "value": r["value"], "unit": "frame-pairs/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "int32+f64", "data": "synthetic", "config": cfg,
           "e2e": {"value": r["e2e"], "unit": "frame-pairs/s", "h2d_bytes_per_step": r["h2d"],
                   "d2h_bytes_per_step": r["d2h"]},
           "gpu_launches": r["launches"],
           "ssim_modes": r["ssim_modes"],
           "masked_mode": r["masked"],
           "config2_msssim": c2,
           "config0_1080p8": c0,
           "serve": r["serve"],
           "hbm_peak_gbs": peak[0], "hbm_peak_kind": peak[1],
           "clocks": r["clocks"],
           "cpu_baseline": cpu,
           "stage_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in r["stage"].items() if v[1]},
           "repeats": r["repeats"],
           "one_batch_in_flight": r["value_sync"],
           "plain_form": r["plain"],
           "mixed_set": r["mixed"],
           "roofline": {"kernel": "k_cps_multi", "bound": "int32", "achieved": r["achieved"], "peak": r["int_peak"],
                        "unit": "TOP/s", "frac": r["achieved"] / r["int_peak"] if r["int_peak"] else None,
                        "traffic": CPS_TRAFFIC_BYTES, "avg_launch_ms": r["cps_avg_ms"],
                        "tile": f"{r['cps_tile'][0]}x{r['cps_tile'][1]}"},
           "parity": parity}
    print(json.dumps(out))
    barrier(world)


if __name__ == "__main__":
    main()
