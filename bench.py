#!/usr/bin/env python
"""Benchmark of the idx2 encode/decode hot path on B200.

Workload (default, "grf1024"): a 1024^3 float32 k^-5/3 Gaussian random field (seeded,
unit variance) with 20 tanh fronts of width 2 cells, 3 levels, 32^3 bricks, absolute
tolerance 1e-3. One step = encode the field (every level) + decode it back at full
resolution and the encode tolerance. The synthetic field stands in for a simulation
dataset (no dataset is available offline). Inputs are 4.3 GB per direction, far larger
than L2 (126 MB), so no L2 flush is needed between steps.

  value : encode+decode GB/s of raw field bytes (2 x 4.29 GB per step) with the field and
          the compressed dataset resident in HBM (idx2g_encode_device + idx2g_decode into a
          device buffer), timed with CUDA events on the library's stream, max over ranks.
  e2e   : the same metric through the C ABI with host buffers: idx2g_encode of a pinned host
          field (H2D in bands under level 0's launches, kernels, D2H of the streams, packing,
          zstd, files in a tmpfs) + idx2g_dataset_open of the files (read, upload, index) +
          idx2g_decode into a pinned host buffer (D2H in bands under the output level's
          launches). Every copy of the step's data crosses PCIe inside the timed region.

N > 1 (torchrun, or --gpus N, which launches the ranks itself): one dataset of N side^3
blocks (2048x1024x1024 for 2 GPUs, 2048^3 for 8), encoded as N shards: each GPU codes the
subtrees of its run of coarsest bricks from its own block of samples and decodes that block
(weak scaling). The device-resident leg has no collective on its data path; the end-to-end leg
all-gathers the shards' region headers and all-reduces the value range over NCCL before every
rank writes its bytes into the shared files. Timing: barriers, CUDA events on the library's
stream, max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--side 1024]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
LEVELS = 3
TOL = 1e-3
METRIC = "encode+decode GB/s (raw field bytes) at 1e-3 tol"
# DRAM bytes (read + write) of one level-0 k_encode_level launch per brick, from an ncu capture
# of the grf512 workload (the three-CTA build, 444 CTAs, 4,096 bricks: 5.277 GB read + 4.294 GB
# written; the CTAs' FP64 brick slots, 122 MB, no longer fit in L2 beside the streams); the
# traffic of a launch grows with its bricks (every brick makes the same slot sweeps on the same
# grid), so a full launch's traffic is this figure times its bricks.
ENC_L0_TRAFFIC_PER_BRICK = (5.277031e9 + 4.294031e9) / 4096
# FP64 operations of one level-0 k_encode_level launch per brick, from the same kind of ncu
# capture (smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum: 2,872,791,040 adds,
# 1,577,402,368 multiplies, no fused multiply-adds over 4,096 bricks); every brick runs the same
# lifting sweeps, so a launch's count is this figure times its bricks.
ENC_L0_FP64_OPS_PER_BRICK = (2872791040 + 1577402368) / 4096


def fp64_peak(dev):
    """FP64 throughput of this GPU in TFLOP/s: a library DGEMM (torch.matmul in float64,
    4096^3, 2 N^3 flops), best of 5 after two warm-ups, timed with CUDA events. The encode's
    lifting runs separate FP64 adds and multiplies (no fused multiply-add, for bit parity), one
    flop each, against this peak of fused multiply-adds counted as two."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    best = float("inf")
    for i in range(7):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        if i >= 2:
            best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                for n, v in zip(names, s[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_field(side, seed, device):
    from idx2_b200.synthetic import grf_field_torch
    return grf_field_torch(side, side, side, seed=seed, scale="unit", n_fronts=20, device=device)


def reference_sample(side):
    """Bounded CPU sample of the workload: same generator, 512 x 512 x 256 region."""
    import torch
    nx, ny, nz = min(512, side), min(512, side), min(256, side)
    f = make_field(side, 7, "cuda" if torch.cuda.is_available() else "cpu")
    return f[:nz, :ny, :nx].contiguous().cpu().numpy()


def reference_tiles(side):
    """The whole workload field cut into 512 x 512 x 256 tiles (16 distinct tiles at 1024^3), x
    fastest, each a contiguous array: the reference encodes one field per process, single
    threaded, so the host cores share the field tile by tile."""
    import torch
    f = make_field(side, 7, "cuda" if torch.cuda.is_available() else "cpu")
    tx, ty, tz = min(512, side), min(512, side), min(256, side)
    tiles = []
    for z in range(0, side, tz):
        for y in range(0, side, ty):
            for x in range(0, side, tx):
                tiles.append(f[z:z + tz, y:y + ty, x:x + tx].contiguous().cpu().numpy())
    del f
    return tiles


def run_reference_cli(sample, tmp, steps, warmup):
    """Encode + sequential decode of the sample with the reference's own CLI (oracle/_ref)."""
    app = os.path.join(ROOT, "oracle", "_ref", "idx2App")
    nz, ny, nx = sample.shape
    raw = os.path.join(tmp, f"grf-f-[{nx}-{ny}-{nz}]-Float32.raw")
    sample.tofile(raw)
    times = []
    for i in range(warmup + steps):
        out = os.path.join(tmp, "refds")
        shutil.rmtree(out, ignore_errors=True)
        t0 = time.perf_counter()
        r = subprocess.run([app, "--encode", raw, "--num_levels", str(LEVELS), "--tolerance", str(TOL),
                            "--out_dir", out], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-300:] + r.stderr[-300:])
        r = subprocess.run([app, "--decode", os.path.join(out, "grf", "f.idx2"), "--out_dir", tmp,
                            "--out_file", "dec.raw"], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stdout[-300:] + r.stderr[-300:])
        t1 = time.perf_counter()
        if i >= warmup:
            times.append(t1 - t0)
    return times


def cpu_baseline(side, steps=5, warmup=1):
    """The reference CLI on one host core: encode + sequential decode of one 512 x 512 x 256
    tile of the workload field, median of `steps` passes after `warmup` (about 25 s)."""
    app = os.path.join(ROOT, "oracle", "_ref", "idx2App")
    if not os.path.exists(app):
        return {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref was not built on this machine"}
    sample = reference_sample(side)
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as tmp:
        times = run_reference_cli(sample, tmp, steps, warmup)
    t = statistics.median(times)
    nz, ny, nx = sample.shape
    return {"value": 2 * sample.nbytes / t / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
            "sample": f"{nx}x{ny}x{nz} float32 tile of the same field; idx2App --encode (L={LEVELS}, "
                      f"tol {TOL}) + sequential --decode, median of {len(times)} after {warmup} warm-up, "
                      f"{t:.2f} s per pass"}


def run_reference_parallel(tiles, tmp, procs, steps, warmup):
    """The reference CLI on every host core: per step, every tile of the field is encoded and
    decoded (sequential decode) by its own idx2App pipeline, at most `procs` pipelines at once
    (the reference encoder is single-threaded, so one pipeline per core is how it uses the
    host). Returns the wall time of each timed step."""
    app = os.path.join(ROOT, "oracle", "_ref", "idx2App")
    raws = []
    for k, t in enumerate(tiles):
        nz, ny, nx = t.shape
        d = os.path.join(tmp, f"t{k}")
        os.makedirs(d, exist_ok=True)
        raw = os.path.join(d, f"grf-f-[{nx}-{ny}-{nz}]-Float32.raw")
        t.tofile(raw)
        raws.append((d, raw))

    def pipeline(d, raw):
        out = os.path.join(d, "ds")
        shutil.rmtree(out, ignore_errors=True)
        os.makedirs(out)
        enc = [app, "--encode", raw, "--num_levels", str(LEVELS), "--tolerance", str(TOL), "--out_dir", out]
        dec = [app, "--decode", os.path.join(out, "grf", "f.idx2"), "--out_dir", out, "--out_file", "dec.raw"]
        for cmd in (enc, dec):
            r = subprocess.run(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
            if r.returncode:
                raise RuntimeError("reference pipeline failed: " + r.stderr.decode()[-300:])

    from concurrent.futures import ThreadPoolExecutor
    times = []
    with ThreadPoolExecutor(max_workers=procs) as pool:
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            for fut in [pool.submit(pipeline, d, raw) for d, raw in raws]:
                fut.result()
            t1 = time.perf_counter()
            if i >= warmup:
                times.append(t1 - t0)
    return times


def reference_arm(args, rank, world):
    if rank != 0:
        return
    app = os.path.join(ROOT, "oracle", "_ref", "idx2App")
    if not os.path.exists(app):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference built from "
                          "its sources) is not present on this machine"}))
        return
    procs = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    tiles = reference_tiles(args.side)
    raw = sum(t.nbytes for t in tiles)
    nz, ny, nx = tiles[0].shape
    with tempfile.TemporaryDirectory(dir="/dev/shm" if os.path.isdir("/dev/shm") else None) as tmp:
        times = run_reference_parallel(tiles, tmp, procs, args.steps, args.warmup)
    t = sum(times) / len(times)
    v = 2 * raw / t / 1e9
    desc = (f"the whole {args.side}^3 field per step as {len(tiles)} distinct {nx}x{ny}x{nz} float32 tiles, "
            f"each encoded (idx2App --encode, L={LEVELS}, tol {TOL}) and decoded (sequential --decode) by "
            f"its own reference pipeline, {procs} pipelines at once on the {procs} host cores (the "
            f"reference encode is single-threaded); value = 2 x field bytes / wall time")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"grf{args.side}: {args.side}^3 float32 k^-5/3 GRF + 20 fronts, "
                       f"{LEVELS} levels, 32^3 bricks, tol {TOL}; encode + full-res decode",
                       "parallelism": f"dp{world}",
                       "tiling": f"{len(tiles)} tiles of {nx}x{ny}x{nz}, each its own dataset"},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": procs, "kind": "reference", "sample": desc},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def global_dims(side, world):
    """One dataset for `world` GPUs: a side^3 block per GPU, the blocks doubling the dataset
    along x, then y, then z (powers of two; other counts line the blocks up along x)."""
    d = [side, side, side]
    n, k = world, 0
    if n & (n - 1):
        return (side * world, side, side)
    while n > 1:
        d[k % 3] *= 2
        n //= 2
        k += 1
    return tuple(d)


def ours_sharded(args, rank, world, local_rank):
    """N > 1: one dataset of N side^3 blocks (weak scaling), encoded as N shards (each GPU the
    subtrees of its run of coarsest bricks, read from its own block of samples) and decoded
    block by block. value: the device stage of every shard (idx2g_encode_shard, device only)
    + the decode of its block from the resident dataset, max over ranks; e2e: per step the
    block crosses to the device, each shard codes, the ranks all-gather their region headers
    and all-reduce the value range over NCCL, every rank writes its bytes into the shared
    files, opens the dataset and decodes its block into pinned host memory."""
    import ctypes
    import datetime
    import torch
    import torch.distributed as dist
    from idx2_b200 import _lib
    from idx2_b200.sharded import ShardEncode, exchange, shard_region
    from idx2_b200.synthetic import grf_field_torch

    # --dist-backend gloo runs the ranks' logic on fewer GPUs than ranks (a functional check of
    # the multi-process path: the ranks' kernels never wait on one another); measurements use NCCL
    local_rank = local_rank % max(1, torch.cuda.device_count())
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    def note(what):
        if os.environ.get("IDX2G_BENCH_TRACE"):
            print(f"bench rank {rank}: {what}", file=sys.stderr, flush=True)

    note("init")
    dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=120))
    note("process group up")
    stream = torch.cuda.Stream(device=dev)
    note("stream")
    _lib.lib()
    note("library loaded")
    _lib.ctx_on_stream(local_rank, stream)  # the library's work on a stream the events can bracket
    note("context")
    side = args.side
    gd = global_dims(side, world)
    lo, sz = shard_region(gd, "float32", LEVELS, TOL, rank, world)
    note(f"region {lo} {sz} of {gd}")
    field = grf_field_torch(sz[0], sz[1], sz[2], seed=7 + rank, scale="unit", n_fronts=20, device=dev)
    torch.cuda.synchronize()
    note("field")
    raw_bytes = field.numel() * field.element_size()
    tmp = os.path.join("/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir(),
                       f"idx2bench_{os.environ.get('MASTER_PORT', '0')}")
    last = [lo[k] + sz[k] - 1 for k in range(3)]
    L = _lib.lib()
    L.idx2g_ctx_launches.restype = ctypes.c_longlong
    L.idx2g_ctx_launches.argtypes = [ctypes.c_void_p]

    def encode_to(out_dir, src):
        job = ShardEncode(src, lo, gd, out_dir, "grf", "f", LEVELS, TOL, rank, world, local_rank)
        payloads, vmin, vmax = exchange(job.headers, job.vmin, job.vmax)
        info = job.finish(payloads, vmin, vmax)
        dist.barrier()
        return job, info

    def decode_block(ds, out):
        torch.cuda.current_stream(dev).synchronize()
        ds.decode(first=lo, last=last, out=out)

    try:
        if rank == 0:
            shutil.rmtree(tmp, ignore_errors=True)
        dist.barrier()
        note("barrier")
        import idx2_b200 as idx2
        note("setup encode")
        encode_to(os.path.join(tmp, "setup"), field)
        note("setup encoded")
        ds = idx2.Dataset(os.path.join(tmp, "setup", "grf", "f.idx2"))
        out_dev = torch.empty_like(field)
        recs = []

        def device_step():
            job = ShardEncode(field, lo, gd, tmp, "grf", "f", LEVELS, TOL, rank, world, local_rank, device_only=True)
            decode_block(ds, out_dev)
            recs.append(([job.info.level_kernel_ms[i] for i in range(job.info.num_levels)],
                         [job.info.level_out_bytes[i] for i in range(job.info.num_levels)], ds.last_kernel_ms))

        for _ in range(args.warmup):
            device_step()
        note("warmed up")
        recs.clear()
        torch.cuda.synchronize()
        dist.barrier()
        launches0 = L.idx2g_ctx_launches(_lib.ctx(local_rank).h)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as clocks:
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                device_step()
            e1.record(stream)
            torch.cuda.synchronize()
        timed_launches = L.idx2g_ctx_launches(_lib.ctx(local_rank).h) - launches0
        dev_ms = e0.elapsed_time(e1) / args.steps
        max_err = float((out_dev.double() - field.double()).abs().max())
        t = torch.tensor([dev_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t)
        ds.close()
        note("timed")
        # e2e: host block in, files out, the dataset read back and this block decoded to the host
        host = field.cpu().pin_memory()
        out_host = torch.empty(field.shape, dtype=field.dtype).pin_memory()
        staged = torch.empty_like(field)
        e2e = []
        for i in range(args.warmup + args.steps):
            d = os.path.join(tmp, f"e2e{i % 2}")
            if rank == 0:
                shutil.rmtree(d, ignore_errors=True)
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            staged.copy_(host, non_blocking=True)
            torch.cuda.synchronize()
            encode_to(d, staged)
            ds2 = idx2.Dataset(os.path.join(d, "grf", "f.idx2"))
            ds2.decode(first=lo, last=last, out=out_host)
            ds2.close()
            dist.barrier()
            if i >= args.warmup:
                e2e.append(time.perf_counter() - t0)
        tt = torch.tensor([sum(e2e) / len(e2e)], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt)
    finally:
        dist.barrier()
        if rank == 0:
            shutil.rmtree(tmp, ignore_errors=True)
    if rank == 0:
        lvl_ms, lvl_bytes, dec_ms = recs[-1]
        l0_ms = sum(r[0][0] for r in recs) / len(recs)
        l0_bytes = raw_bytes + lvl_bytes[0]
        peak, kind = hbm_peak()
        achieved = l0_bytes / (l0_ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": world * 2 * raw_bytes / (dev_ms * 1e-3) / 1e9, "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded k^-5/3 GRF, 20 tanh fronts, one block per GPU)",
            "config": {"workload": f"grf{side} x {world}: one {gd[0]}x{gd[1]}x{gd[2]} float32 dataset of {world} "
                                   f"{side}^3 blocks, {LEVELS} levels, 32^3 bricks, tol {TOL}; step = sharded encode "
                                   f"(all levels) + decode of each GPU's block",
                       "parallelism": f"{world} shards of one dataset (coarsest-brick runs), no data exchange; "
                                      f"the e2e leg all-gathers region headers over NCCL",
                       "l2": "inputs (4.3 GB per GPU) >> L2; no flush needed"},
            "encode_level_ms": lvl_ms, "decode_ms": dec_ms, "decode_max_abs_err": max_err,
            "roofline": {"bound": "hbm", "kernel": "k_encode_level (level 0, rank 0)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else kind,
                         "algorithmic_bytes": l0_bytes, "traffic": None},
            "cpu_baseline": None,
            "e2e": {"value": world * 2 * raw_bytes / e2e_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(raw_bytes),
                    "d2h_bytes_per_step": int(raw_bytes), "s_per_step": e2e_s},
            "clocks": clocks.summary(), "gpu_launches": int(timed_launches),
        }
        print(json.dumps(line))
    dist.destroy_process_group()


def ours(args, rank, world, local_rank):
    import ctypes
    import torch
    import idx2_b200 as idx2
    from idx2_b200 import _lib

    if world > 1:
        return ours_sharded(args, rank, world, local_rank)
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    side = args.side
    field = make_field(side, 7 + rank, dev)
    raw_bytes = field.numel() * field.element_size()
    stream = torch.cuda.Stream(device=dev)
    h = ctypes.c_void_p()
    rc = _lib.lib().idx2g_ctx_create(local_rank, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h))
    assert rc == 0, rc
    p = _lib.Params(name="grf", field="f", dims=(side, side, side), dtype="float32", num_levels=LEVELS,
                    tolerance=TOL)
    cp = p.to_c()
    tmp = tempfile.mkdtemp(prefix=f"idx2bench{rank}_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        # one encode to files, and the dataset made resident for the device-side decode
        host = field.cpu().pin_memory()
        cpo = _lib.Params(name="grf", field="f", dims=(side, side, side), dtype="float32", num_levels=LEVELS,
                          tolerance=TOL, out_dir=tmp).to_c()
        info = _lib.EncodeInfo()
        rc = _lib.lib().idx2g_encode(h, ctypes.byref(cpo), ctypes.c_void_p(host.data_ptr()), 0, ctypes.byref(info))
        assert rc == 0, rc
        dsp = _lib.Params(input_file=os.path.join(tmp, "grf", "f.idx2"), in_dir=tmp).to_c()
        dsh = ctypes.c_void_p()
        rc = _lib.lib().idx2g_dataset_open(h, ctypes.byref(dsp), ctypes.byref(dsh))
        assert rc == 0, rc
        out_dev = torch.empty_like(field)
        out_host = torch.empty(field.shape, dtype=field.dtype).pin_memory()
        kms = ctypes.c_double(0)

        def device_step(rec):
            einfo = _lib.EncodeInfo()
            rc = _lib.lib().idx2g_encode_device(h, ctypes.byref(cp), ctypes.c_void_p(field.data_ptr()),
                                                ctypes.byref(einfo))
            assert rc == 0, rc
            rc = _lib.lib().idx2g_decode(h, dsh, ctypes.byref(dsp), ctypes.c_void_p(out_dev.data_ptr()),
                                         ctypes.c_size_t(raw_bytes), 1, ctypes.byref(kms))
            assert rc == 0, rc
            if rec is not None:
                rec.append((einfo.num_levels, [einfo.level_kernel_ms[i] for i in range(einfo.num_levels)],
                            [einfo.level_out_bytes[i] for i in range(einfo.num_levels)], kms.value,
                            einfo.kernel_launches))

        for _ in range(args.warmup):
            device_step(None)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        recs = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        L = _lib.lib()
        L.idx2g_ctx_launches.restype = ctypes.c_longlong
        L.idx2g_ctx_launches.argtypes = [ctypes.c_void_p]
        launches0 = L.idx2g_ctx_launches(h)
        with ClockSampler(local_rank) as clocks:
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                device_step(recs)
            e1.record(stream)
            torch.cuda.synchronize()
        timed_launches = L.idx2g_ctx_launches(h) - launches0
        dev_ms = e0.elapsed_time(e1) / args.steps
        # correctness of the timed decode: full-resolution output within the expected error
        max_err = float((out_dev.double() - field.double()).abs().max())
        t = torch.tensor([dev_ms], device=dev, dtype=torch.float64)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t)

        # e2e through the C ABI with host buffers
        e2e_times = []
        e2e_parts = []
        h2d = d2h = 0
        for i in range(0 if args.no_e2e else args.warmup + args.steps):
            shutil.rmtree(os.path.join(tmp, "e2e"), ignore_errors=True)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p2 = _lib.Params(name="grf", field="f", dims=(side, side, side), dtype="float32",
                             num_levels=LEVELS, tolerance=TOL, out_dir=os.path.join(tmp, "e2e")).to_c()
            info2 = _lib.EncodeInfo()
            rc = _lib.lib().idx2g_encode(h, ctypes.byref(p2), ctypes.c_void_p(host.data_ptr()), 0,
                                         ctypes.byref(info2))
            assert rc == 0, rc
            ta = time.perf_counter()
            dp2 = _lib.Params(input_file=os.path.join(tmp, "e2e", "grf", "f.idx2"),
                              in_dir=os.path.join(tmp, "e2e")).to_c()
            dh2 = ctypes.c_void_p()
            rc = _lib.lib().idx2g_dataset_open(h, ctypes.byref(dp2), ctypes.byref(dh2))
            assert rc == 0, rc
            tb = time.perf_counter()
            rc = _lib.lib().idx2g_decode(h, dh2, ctypes.byref(dp2), ctypes.c_void_p(out_host.data_ptr()),
                                         ctypes.c_size_t(raw_bytes), 0, ctypes.byref(kms))
            assert rc == 0, rc
            rsd = ctypes.c_longlong(0)
            _lib.lib().idx2g_dataset_info(dh2, None, None, (ctypes.c_int * 3)(), None, None, None,
                                          ctypes.byref(rsd))
            _lib.lib().idx2g_dataset_close(dh2)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            if i >= args.warmup:
                e2e_times.append(t1 - t0)
                e2e_parts.append({"encode_s": ta - t0, "encode_device_s": info2.device_s,
                                  "encode_pack_s": info2.pack_s, "encode_write_s": info2.write_s,
                                  "open_s": tb - ta, "decode_s": t1 - tb})
                h2d = raw_bytes + rsd.value
                d2h = raw_bytes + info2.stream_bytes + info2.exp_bytes
        tt = torch.tensor([sum(e2e_times) / len(e2e_times) if e2e_times else float("nan")], device=dev,
                          dtype=torch.float64)
        if dist:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt)
        _lib.lib().idx2g_dataset_close(dsh)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        _lib.lib().idx2g_ctx_destroy(h)
        return
    nlev, lvl_ms, lvl_bytes, dec_ms, launches = recs[-1]
    enc_ms = sum(sum(r[1]) for r in recs) / len(recs)
    # dominant kernel: the level-0 encode launch
    l0_ms = sum(r[1][0] for r in recs) / len(recs)
    l0_bytes = raw_bytes + lvl_bytes[0]
    peak, kind = hbm_peak()
    achieved = l0_bytes / (l0_ms * 1e-3) / 1e9
    value = world * 2 * raw_bytes / (dev_ms * 1e-3) / 1e9
    base = cpu_baseline(side) if world == 1 and not args.no_cpu else None
    batch = batched_leg(torch.device("cuda", local_rank), h) if not args.no_batch else None
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded k^-5/3 GRF, 20 tanh fronts)",
        "config": {"workload": f"grf{side}: {side}^3 float32 k^-5/3 GRF + 20 fronts, {LEVELS} levels, 32^3 "
                               f"bricks, tol {TOL}; step = encode (all levels) + full-res decode",
                   "parallelism": f"dp{world} (independent field per GPU)",
                   "l2": "inputs (4.3 GB) >> L2; no flush needed"},
        "encode_gbs": raw_bytes / (enc_ms * 1e-3) / 1e9,
        "decode_gbs": raw_bytes / (dec_ms * 1e-3) / 1e9,
        "encode_level_ms": lvl_ms, "decode_ms": dec_ms,
        "compressed_bytes": int(sum(lvl_bytes)),
        "decode_max_abs_err": max_err,
        "roofline": {"bound": "hbm", "kernel": "k_encode_level (level 0)", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else kind,
                     "algorithmic_bytes": l0_bytes,
                     "traffic": ENC_L0_TRAFFIC_PER_BRICK * (side // 32) ** 3,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the level-0 launch "
                                       "at 512^3 (4,096 bricks), scaled by bricks"},
        "cpu_baseline": base,
        "e2e": {"value": world * 2 * raw_bytes / e2e_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "s_per_step": e2e_s,
                "breakdown_s": ({k: round(sum(d[k] for d in e2e_parts) / len(e2e_parts), 4)
                                 for k in e2e_parts[0]} if e2e_parts else None)},
        "clocks": clocks.summary(),
        "gpu_launches": int(timed_launches),
        "batched_encode": batch,
    }
    # the whole decode (plane and level kernels of every level) against the same roof: the
    # compressed streams and exponents it reads plus the grid it writes
    dec_bytes = int(sum(lvl_bytes)) + raw_bytes
    # the same launch against the FP64 roof (its lifting is FP64 adds and multiplies)
    fp64_tf = fp64_peak(dev)
    fp64_ach = ENC_L0_FP64_OPS_PER_BRICK * (side // 32) ** 3 / (l0_ms * 1e-3) / 1e12
    line["roofline_fp64"] = {"bound": "fp64", "kernel": "k_encode_level (level 0)", "achieved": fp64_ach,
                             "peak": fp64_tf, "unit": "TFLOP/s", "frac": fp64_ach / fp64_tf,
                             "peak_source": "measured here: DGEMM 4096^3 (torch.matmul float64), best of 5",
                             "ops_per_brick": ENC_L0_FP64_OPS_PER_BRICK,
                             "ops_source": "ncu smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum of "
                                           "the level-0 launch at 512^3 (4,096 bricks), scaled by bricks"}
    line["roofline_decode"] = {"bound": "hbm", "kernel": "k_decode_planes + k_decode_level (all levels)",
                               "achieved": dec_bytes / (dec_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                               "frac": dec_bytes / (dec_ms * 1e-3) / 1e9 / peak, "algorithmic_bytes": dec_bytes}
    _lib.lib().idx2g_ctx_destroy(h)
    del field, out_dev, out_host, host
    torch.cuda.empty_cache()
    if world == 1 and not args.no_serve:
        line["serving"] = serve_leg(args, requests=args.bench_serve_requests)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_leg(args)
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def batched_leg(dev, h, nfields=512, seed=7, reps=3):
    """Uneven-field batch (512 seeded k^-5/3 fields, each axis 17-300, 1 in 8 2D, half float32 /
    half float64, levels 1-3, tol 1e-3): the batched device stage (idx2g_encode_batch, level
    launches in one CUDA graph, autotuned launch shape) against the per-field plain device
    stage (idx2g_encode_device in a loop) on the same device-resident fields. Fields the format
    rules reject are drawn but not encoded."""
    import ctypes
    import torch
    from idx2_b200 import _lib
    from idx2_b200.synthetic import grf_field_torch
    rng = np.random.default_rng(seed)
    fields, cps = [], []
    for i in range(nfields):
        dims = [int(rng.integers(17, 301)) for _ in range(3)]
        if rng.integers(0, 8) == 0:
            dims[2] = 1
        dt = "float32" if i % 2 == 0 else "float64"
        lv = int(rng.integers(1, 4))
        bd = (32, 32, 1) if dims[2] == 1 else (32, 32, 32)
        p = _lib.Params(name=f"b{i}", field="f", dims=dims, dtype=dt, brick_dims=bd, num_levels=lv,
                        tolerance=TOL)
        if _lib.check_params(p) != 0:
            continue
        f = grf_field_torch(dims[0], dims[1], dims[2], seed=seed * 1000 + i, scale="range", device=dev)
        fields.append(f.to(torch.float32 if dt == "float32" else torch.float64).contiguous())
        cps.append(p.to_c())
    n = len(fields)
    raw = sum(f.numel() * f.element_size() for f in fields)
    L = _lib.lib()
    L.idx2g_encode_batch.argtypes = [ctypes.c_void_p, ctypes.POINTER(_lib._CParams), ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.POINTER(_lib.EncodeInfo)]
    carr = (_lib._CParams * n)(*cps)
    parr = (ctypes.c_void_p * n)(*[ctypes.c_void_p(f.data_ptr()) for f in fields])
    infos = (_lib.EncodeInfo * n)()
    flags = 1 | 2 | 4  # graph, device stage only, autotuned

    def batched():
        rc = L.idx2g_encode_batch(h, carr, parr, n, 1, flags, infos)
        assert rc == 0, rc

    def plain():
        info = _lib.EncodeInfo()
        for i in range(n):
            rc = L.idx2g_encode_device(h, ctypes.byref(carr[i]), ctypes.c_void_p(fields[i].data_ptr()),
                                       ctypes.byref(info))
            assert rc == 0, rc

    out = {}
    for name, fn in (("plain", plain), ("batched", batched)):
        fn()  # warm-up (and, for the batch, the autotuner's first timing)
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        out[name] = sorted(ts)[len(ts) // 2]
    launches = int(infos[0].kernel_launches)
    del fields
    torch.cuda.empty_cache()
    return {"workload": f"{nfields} drawn uneven fields (axes 17-300, 1/8 2D, f32/f64, levels 1-3, tol {TOL}), "
                        f"{n} accepted by the format rules",
            "fields": n, "raw_bytes": int(raw), "plain_s": out["plain"], "batched_s": out["batched"],
            "plain_gbs": raw / out["plain"] / 1e9, "batched_gbs": raw / out["batched"] / 1e9,
            "speedup": out["plain"] / out["batched"], "batched_launches": launches,
            "timing": "wall clock of the device stage (fields resident on the device), median of 3"}


def serve_leg(args, requests=None):
    """Decode serving: a device-resident compressed k^-5/3 field (3 levels, encoded at 1e-6)
    answering a Poisson stream of ROI requests (sides 32-512, per-axis downsampling 0-3,
    tolerance log-uniform 1e-6..1e-1), batched on arrival under the free-HBM budget, against
    one-request-at-a-time decode of the same schedule. Returns the result as a dict."""
    requests = requests or args.serve_requests
    import torch
    import idx2_b200
    from idx2_b200.synthetic import grf_field_torch
    from idx2_b200.serving import Server, dataset_decoder, free_hbm_budget, poisson_schedule
    dims = tuple(int(x) for x in args.serve_dims.split("x"))
    dev = torch.device("cuda", 0)
    tmp = tempfile.mkdtemp(prefix="idx2serve_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        t0 = time.perf_counter()
        f = grf_field_torch(dims[0], dims[1], dims[2], seed=11, scale="unit", device=dev)
        info = idx2_b200.encode(f, out_dir=tmp, name="serve", field_name="f", num_levels=3, tolerance=1e-6)
        raw = f.numel() * f.element_size()
        del f
        torch.cuda.empty_cache()
        ds = idx2_b200.Dataset(os.path.join(tmp, "serve", "f.idx2"))
        setup_s = time.perf_counter() - t0
        budget = free_hbm_budget()
        dec = dataset_decoder(ds)
        warm = poisson_schedule(32, args.serve_rate, dims, seed=1)
        Server(dec, budget).run(warm, batched=True)
        # warm-up to the largest batch the server admits: device workspaces and the output
        # arena reach their peak before the timed runs, as in a server that has been running
        srv = Server(dec, budget)
        dec(srv.admit(poisson_schedule(srv.max_batch, args.serve_rate, dims, seed=3)))
        res = {}
        for mode in ("batched", "one-at-a-time"):
            sched = poisson_schedule(requests, args.serve_rate, dims, seed=2)
            st = Server(dec, budget).run(sched, batched=(mode == "batched"))
            d = st.as_dict()
            d["decoded_gbs"] = st.decoded_bytes / st.elapsed_s / 1e9
            res[mode] = d
        line = {"metric": "decode serving p50/p99 ms (ROI requests)", "impl": "ours",
                "config": {"workload": f"serving: {dims[0]}x{dims[1]}x{dims[2]} float32 k^-5/3 field, 3 levels, "
                                       f"encoded at 1e-6; Poisson {args.serve_rate:g} req/s, "
                                       f"{requests} requests per mode, ROI sides 32-512, downsampling 0-3, "
                                       f"tolerance log-uniform 1e-6..1e-1",
                           "raw_bytes": int(raw), "compressed_bytes": int(info.file_bytes),
                           "hbm_budget_bytes": int(budget), "setup_s": setup_s},
                "batched": res["batched"], "one_at_a_time": res["one-at-a-time"],
                "p99_speedup": res["one-at-a-time"]["p99_ms"] / max(res["batched"]["p99_ms"], 1e-9)}
        ds.close()
        return line
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        torch.cuda.empty_cache()


def _adjoint_batch(dev, nfields, side, dtype, tmp, seed):
    """Encode nfields seeded k^-5/3 fields of side^3 (2 levels, tolerance 1e-4) and return the
    stacked dequantised coefficients (decoded at tolerance 1e-4), the first field's bit-exact
    decode and the compressed bytes."""
    import torch
    import idx2_b200
    from idx2_b200.diff import Format, coefficients
    from idx2_b200.synthetic import grf_field_torch
    fmt = Format((side, side, side), "float32" if dtype == torch.float32 else "float64", 2)
    cs, first_decode, comp = [], None, 0
    for i in range(nfields):
        f = grf_field_torch(side, side, side, seed=seed + i, scale="unit", device=dev).to(dtype)
        d = os.path.join(tmp, f"a{i}")
        info = idx2_b200.encode(f, out_dir=d, name="adj", field_name="f", num_levels=2, tolerance=1e-4)
        comp += int(info.file_bytes)
        del f
        ds = idx2_b200.Dataset(os.path.join(d, "adj", "f.idx2"))
        cs.append(coefficients(ds, fmt, 1e-4))
        if i == 0:
            first_decode = torch.from_numpy(ds.decode(tolerance=1e-4)).to(dev)
        ds.close()
        shutil.rmtree(d, ignore_errors=True)
    return fmt, torch.stack(cs), first_decode, comp


def _synth_bytes(fmt, nbatch, elem):
    """Algorithmic bytes of one synth (or adjoint) pass over a batch: the coefficient tensor and
    the grid once each, plus the kept bricks of the coarser levels written once and read once."""
    from idx2_b200.diff import coeff_count
    d = fmt.dims
    grid = d[0] * d[1] * d[2]
    coeffs = coeff_count(fmt)
    nb0 = 33 ** 3 * (-(-d[0] // 32)) * (-(-d[1] // 32)) * (-(-d[2] // 32))
    kept = coeffs - nb0  # coarser levels' bricks, one value per coefficient position
    return nbatch * elem * (grid + coeffs + 2 * kept)


def _adjoint_time(fmt, c, target, steps, warmup):
    """Time forward (decode_diff) + MSE + backward over the batch: step ms from CUDA events on
    torch's stream (synchronised on both sides), kernel ms from the library's events."""
    import torch
    from idx2_b200 import diff
    cg = c.detach().clone().requires_grad_(True)

    def step():
        x = diff.decode_diff(cg, fmt)
        loss = torch.mean((x - target) ** 2)
        loss.backward()
        return diff.last_kernel_ms["synth"], diff.last_kernel_ms["adjoint"]

    for _ in range(warmup):
        step()
        cg.grad = None
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fw, bw = [], []
    e0.record()
    for _ in range(steps):
        a, b = step()
        fw.append(a)
        bw.append(b)
        cg.grad = None
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, statistics.median(fw), statistics.median(bw)


def adjoint_leg(args):
    """Differentiable decode: a batch of float32 k^-5/3 fields (2 levels, decoded at downsampling
    0 and tolerance 1e-4) through the torch.autograd.Function, loss = MSE to a second seeded
    field set; a float64 batch at a smaller side. Checks: the float32 gradient against the
    float64 adjoint of the same residual, the dot-product identity, FP64 central differences
    (step 1e-3 on 200 random coefficients), D against the bit-exact decode. Returns the result
    as a dict."""
    import torch
    from idx2_b200 import diff
    from idx2_b200.synthetic import grf_field_torch
    dev = torch.device("cuda", 0)
    nf, side, side64 = args.adjoint_fields, args.adjoint_side, args.adjoint_f64_side
    tmp = tempfile.mkdtemp(prefix="idx2adj_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        t0 = time.perf_counter()
        fmt, c, dec0, comp = _adjoint_batch(dev, nf, side, torch.float32, tmp, seed=300)
        target = torch.stack([grf_field_torch(side, side, side, seed=900 + i, scale="unit", device=dev)
                              for i in range(nf)])
        setup_s = time.perf_counter() - t0
        step_ms, fw_ms, bw_ms = _adjoint_time(fmt, c, target, args.steps, args.warmup)
        nbytes = _synth_bytes(fmt, nf, 4)
        grid_bytes = nf * side ** 3 * 4
        # checks on the float32 batch
        x = diff.synth(c, fmt)
        d_rel = float((x[0] - dec0).abs().max() / dec0.abs().max())
        r = 2.0 * (x - target) / x.numel()
        g32 = diff.synth_adjoint(r, fmt)
        fmt64 = diff.Format(fmt.dims, "float64", 2)
        x64 = diff.synth(c.double(), fmt64)
        g64 = diff.synth_adjoint(2.0 * (x64 - target.double()) / x64.numel(), fmt64)
        g_rel = float((g32.double() - g64).abs().max() / g64.abs().max())
        del x64, g64, r, x
        gen = torch.Generator(device=dev)
        gen.manual_seed(5)
        y = torch.randn(target.shape, generator=gen, device=dev, dtype=torch.float64)
        cd = torch.randn(c.shape, generator=gen, device=dev, dtype=torch.float64)
        lhs = float(torch.sum(diff.synth(cd, fmt64) * y))
        rhs = float(torch.sum(cd * diff.synth_adjoint(y, fmt64)))
        dot64 = abs(lhs - rhs) / abs(lhs)
        lhs = float(torch.sum(diff.synth(cd.float(), fmt).double() * y))
        rhs = float(torch.sum(cd * diff.synth_adjoint(y.float(), fmt).double()))
        dot32 = abs(lhs - rhs) / abs(lhs)
        del y, cd, target, c
        torch.cuda.empty_cache()
        # float64 batch at side64
        fmt_d, c_d, dec0_d, comp_d = _adjoint_batch(dev, nf, side64, torch.float64, tmp, seed=500)
        target_d = torch.stack([grf_field_torch(side64, side64, side64, seed=1900 + i, scale="unit", device=dev)
                                for i in range(nf)]).double()
        step_ms_d, fw_ms_d, bw_ms_d = _adjoint_time(fmt_d, c_d, target_d, args.steps, args.warmup)
        nbytes_d = _synth_bytes(fmt_d, nf, 8)
        x = diff.synth(c_d, fmt_d)
        d_rel64 = float((x[0] - dec0_d).abs().max() / dec0_d.abs().max())
        n_all = x.numel()
        grad = diff.synth_adjoint(2.0 * (x - target_d) / n_all, fmt_d)[0]
        # FP64 central differences on field 0 (only its samples depend on its coefficients)
        c0 = c_d[0].clone()
        t0f = target_d[0]
        rng = np.random.default_rng(8)
        nz = np.nonzero(grad.abs().cpu().numpy() > 0)[0]
        idx = [int(i) for i in rng.permutation(nz)[:200]]
        h = 1e-3
        fd_err = 0.0
        for i in idx:
            old = float(c0[i])
            c0[i] = old + h
            xp = diff.synth(c0, fmt_d)
            c0[i] = old - h
            xm = diff.synth(c0, fmt_d)
            c0[i] = old
            fd = float(torch.sum((xp - t0f) ** 2 - (xm - t0f) ** 2)) / n_all / (2 * h)
            fd_err = max(fd_err, abs(fd - float(grad[i])) / max(abs(fd), 1e-300))
        line = {"metric": "differentiable decode step ms (forward + MSE + backward)", "impl": "ours",
                "unit": "ms", "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
                "data": "synthetic", "dtype": "f32 (f64 variant)",
                "config": {"workload": f"differentiable decode: {nf} float32 k^-5/3 fields of {side}^3, 2 levels, "
                                       f"coefficients decoded at downsampling 0 and tolerance 1e-4, loss = MSE to "
                                       f"{nf} second seeded fields; float64 variant {nf} fields of {side64}^3",
                           "compressed_bytes": comp, "setup_s": setup_s,
                           "l2": "inputs larger than L2 (coefficients and grid)"},
                "float32": {"step_ms": step_ms, "forward_kernel_ms": fw_ms, "backward_kernel_ms": bw_ms,
                            "grid_gbs_per_step": grid_bytes / step_ms / 1e6,
                            "forward_gbs": nbytes / fw_ms / 1e6, "backward_gbs": nbytes / bw_ms / 1e6,
                            "algorithmic_bytes_per_pass": nbytes},
                "float64": {"step_ms": step_ms_d, "forward_kernel_ms": fw_ms_d, "backward_kernel_ms": bw_ms_d,
                            "forward_gbs": nbytes_d / fw_ms_d / 1e6, "backward_gbs": nbytes_d / bw_ms_d / 1e6,
                            "algorithmic_bytes_per_pass": nbytes_d},
                "checks": {"grad_f32_vs_f64_rel": g_rel, "grad_f32_target": 1e-5,
                           "fd_f64_max_rel": fd_err, "fd_points": len(idx), "fd_step": h,
                           "dot_identity_rel_f64": dot64, "dot_identity_rel_f32": dot32,
                           "synth_vs_decode_rel_f32": d_rel, "synth_vs_decode_rel_f64": d_rel64},
                "gpu_launches_per_step": 4}
        return line
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg (profiling runs)")
    ap.add_argument("--no-batch", action="store_true", help="skip the uneven-field batched-encode leg")
    ap.add_argument("--serve", action="store_true", help="run the decode-serving benchmark instead")
    ap.add_argument("--adjoint", action="store_true", help="run the differentiable-decode benchmark instead")
    ap.add_argument("--adjoint-fields", type=int, default=32, help="fields per batch (differentiable decode)")
    ap.add_argument("--adjoint-side", type=int, default=256, help="float32 field side (differentiable decode)")
    ap.add_argument("--adjoint-f64-side", type=int, default=128, help="float64 field side (differentiable decode)")
    ap.add_argument("--serve-dims", default="2048x2048x1024", help="serving field dims (x, y, z)")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="request arrival rate (per second)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="requests per mode")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process group backend for N > 1 (gloo: functional runs with fewer GPUs than ranks)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg of the default run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-decode leg of the default run")
    ap.add_argument("--bench-serve-requests", type=int, default=400,
                    help="requests per mode of the serving leg inside the default run")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: launch the ranks here (the same command under torchrun)
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        env = dict(os.environ)
        if args.dist_backend == "gloo":
            env.setdefault("GLOO_SOCKET_IFNAME", "lo")  # the ranks talk over loopback
        sys.exit(subprocess.call(cmd, env=env))
    if world != args.gpus and rank == 0:
        print(f"bench: --gpus {args.gpus} but WORLD_SIZE={world}; using {world} ranks", file=sys.stderr)
    if args.serve:
        if rank == 0:
            print(json.dumps(serve_leg(args)))
        return
    if args.adjoint:
        if rank == 0:
            print(json.dumps(adjoint_leg(args)))
        return
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
