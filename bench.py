#!/usr/bin/env python
"""Throughput of the AltoPIR answer path on B200: byte-exact QPS of answer batches.  The headline is 128-query
batches on a 1 GiB database (32,768 records x 32 KB), the configuration of the reference's headline batch numbers;
the same JSON line carries the 8 GiB (B = 1, 128, 1024) and 64 GiB (B = 128, 1024) databases under `configs`.

One step = one batch of --batch queries through the whole answer path (validate, limb split, scan, pack, tail).
Every measurement times blocks of exactly --steps steps with CUDA events (a barrier and a synchronisation on both
sides of each block, max over ranks), back to back until the blocks add up to at least one second of device time and
at least five blocks; the figures are over all blocks.
  value : device-resident throughput -- frames already in HBM, batches enqueued back to back (alto_enqueue_device
          rotating through two batch contexts, each replaying its launch sequence as a CUDA graph), timed on the
          engine's stream.  `kernels` and `roofline` come from a second pass of the same batches launched directly on
          one context, each stage bracketed by CUDA events on the engine's stream.
  e2e   : the same metric through the reference-facing C ABI (alto_answer) with pinned HOST frames and output buffers:
          every step uploads its frames and downloads its responses inside the timed region.
Every rank answers its own batches on its own GPU (the answer path needs no exchange between GPUs: replicas, weak
scaling).  `--impl reference` runs the reference's CPU engine (src/amx_kernels.cpp compiled from its own sources by
oracle/Makefile, AMX when the host has it) on the same workload, on rank 0 only, with inputs built by the oracle's
generators so that the engine library is never loaded in that arm.
"""
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
sys.path.insert(0, ROOT)

METRIC = "QPS (byte-exact) at 1/8/64 GB DB, batched vs per-query on 1 B200; p50/p99 ms"
MIN_TIMED_S = 1.0   # device time every measurement accumulates over its blocks of --steps steps
MIN_BLOCKS = 5
# The reference's published QPS for the same record size on 16 cores of a Xeon Silver 4514Y (README: "Benchmark
# without the network", batch 128 at 1 GB, and the Results table at 8 and 64 GB).
PUBLISHED_QPS = {32768: (1986.3, "README bench, 1 GB, batch 128: 64.44 ms median"),
                 262144: (492.0, "README Results table, 8 GB"),
                 2097152: (70.2, "README Results table, 64 GB")}
# The larger configurations measured beside the headline (rows, batch sizes, single queries timed for the plain path).
# the 8 GiB uneven-batch sweep and the 64 GiB batches of the workload list (records, batch sizes, plain queries)
SUB_CONFIGS = ((262144, (1, 7, 33, 128, 200, 512, 1024), 32), (2097152, (128, 1024), 8))


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=32768)
    ap.add_argument("--record-bytes", type=int, default=32768)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--plain-queries", type=int, default=128, help="single-query launches timed for the plain path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the 8 GiB and 64 GiB configurations")
    ap.add_argument("--no-offline", action="store_true",
                    help="skip timing the scheme's offline set-up on the device (alto_engine_offline)")
    ap.add_argument("--serve", type=str, default=None,
                    help="serving mode: comma-separated offered rates in QPS (open-loop Poisson arrivals)")
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--serve-clients", type=int, default=4096, help="seeded clients whose frames are replayed")
    ap.add_argument("--max-batch", type=int, default=1024)
    ap.add_argument("--serve-slots", type=int, default=2, help="device batch contexts of the serving loop")
    ap.add_argument("--serve-queue", type=int, default=2048, help="frames the serving loop's pinned pool holds")
    ap.add_argument("--lanes", type=int, default=2,
                    help="batch contexts the device-resident loop rotates through (1..4; consecutive batches overlap)")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="profiling run for ncu: N batches of the headline configuration through alto_enqueue_device "
                         "(direct launches) and N through alto_answer after the warm-up, no timing loops, no JSON")
    ap.add_argument("--shard", action="store_true",
                    help="column sharding: the ranks split the outputs of one engine state and answer every batch "
                         "together (strong scaling); the default runs one whole engine per rank (replicas)")
    return ap.parse_args(argv)


def l2_note(rows, record_bytes, count=8192):
    db, pm = rows * record_bytes, 4 * record_bytes * count
    return (f"inputs larger than L2 (126 MB): every step streams the {db / 2**30:g} GiB database and the "
            f"{pm / 2**30:g} GiB packing matrix from HBM")


def config_dict(a, rows=None, batch=None):
    """The workload; identical in both arms for the same arguments."""
    rows = a.rows if rows is None else rows
    batch = a.batch if batch is None else batch
    gib = rows * a.record_bytes / 2 ** 30
    return {"workload": f"answer {batch}-query batches over a {gib:g} GiB database ({rows} records x "
                        f"{a.record_bytes} B): synthetic records of the reference generator, seeded keys and queries",
            "rows": rows, "record_bytes": a.record_bytes, "batch": batch, "n": 2048, "tg": 4,
            "l2": l2_note(rows, a.record_bytes)}


# ------------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running; summary() keeps the samples taken inside the
    marked (timed) intervals."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.samples = []
        self.proc = None
        self.marks = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [x.strip() for x in line.split(",")]))

    def mark(self, t0, t1):
        self.marks.append((t0, t1))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, marks=None):
        marks = self.marks if marks is None else marks
        inside = [s for t, s in self.samples if any(a <= t <= b for a, b in marks)]
        use = inside or [s for t, s in self.samples if any(a - 0.25 <= t <= b + 0.25 for a, b in marks)]
        if not use:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"], "samples": 0}
        num = lambda x: x.replace(".", "", 1).isdigit()
        sm = [float(s[1]) for s in use if num(s[1])]
        mx = [float(s[2]) for s in use if num(s[2])]
        pw = [float(s[3]) for s in use if num(s[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in use for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "sm_mhz_min": min(sm) if sm else None, "power_w_median": statistics.median(pw) if pw else None,
                "reasons": reasons, "samples": len(use), "in_timed_region": bool(inside),
                "timed_region_s": sum(b - a for a, b in marks)}


# ------------------------------------------------------------------------------------------------ helpers
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def algorithmic(rows, cols, b, count):
    """Per-batch algorithmic work of the two limb GEMMs: int8 ops (1 multiply-add = 2) and compulsory bytes (the
    database or packing matrix once, the limb operand once, the u32 results once)."""
    return {
        "scan_gemm": {"ops": 2.0 * cols * rows * 4 * b, "bytes": rows * cols + rows * 4 * b + 4 * b * cols},
        "pack_gemm": {"ops": 2.0 * 4 * cols * count * 4 * b, "bytes": 4 * count * cols + 4 * count * b + 4 * b * cols},
    }


def roofline_of(kernel, alg, avg_ms, peaks, peak_src, traffic=None):
    """Roofline of one GEMM: its bound is the slower of its ops at the int8 peak and its compulsory bytes at the HBM
    copy bandwidth; achieved and frac in that unit.  The int8 peak is 2 x the dense bf16 rate of MEASURED_PEAKS.json
    (B200's dense int8 rate is twice its bf16 rate), its sustained figure: the GEMMs are timed inside seconds of
    back-to-back batches at the power cap, the case the sustained figure (bf16 GEMMs back to back for 4 s) measures.
    The fraction of the burst figure is given beside it."""
    burst = 2.0 * peaks["bf16_tflops"]
    sus = peaks.get("bf16_tflops_sustained")
    int8_peak = 2.0 * sus if sus else burst
    t_ops = alg["ops"] / (int8_peak * 1e12)
    t_bytes = alg["bytes"] / (peaks["hbm_gbs"] * 1e9)
    s = avg_ms * 1e-3
    if t_ops >= t_bytes:
        r = {"bound": "tensor", "achieved": alg["ops"] / s / 1e12, "peak": int8_peak, "unit": "TFLOP/s"}
    else:
        r = {"bound": "hbm", "achieved": alg["bytes"] / s / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s"}
    r["frac"] = r["achieved"] / r["peak"]
    which = (f"2 x dense bf16 sustained ({sus} TF/s, GEMMs back to back for 4 s at the power cap; these GEMMs are "
             f"timed inside seconds of back-to-back batches)" if sus else f"2 x dense bf16 burst ({peaks['bf16_tflops']} TF/s)")
    r.update({"kernel": kernel, "traffic": traffic, "avg_ms": avg_ms,
              "peak_source": f"{peak_src}: int8 = {which}; B200's dense int8 rate is twice its bf16 rate; HBM = copy "
                             f"bandwidth ({peaks['hbm_gbs']} GB/s); int8 ops counted as 2 per multiply-add",
              "algorithmic_ops": alg["ops"], "algorithmic_bytes": alg["bytes"],
              "hbm_view": {"achieved_gbs": alg["bytes"] / s / 1e9, "frac": alg["bytes"] / s / 1e9 / peaks["hbm_gbs"]},
              "tensor_view": {"achieved_tops": alg["ops"] / s / 1e12, "frac": alg["ops"] / s / 1e12 / int8_peak}})
    if r["bound"] == "tensor":
        r["frac_of_burst"] = r["achieved"] / burst
        r["burst_peak"] = burst
    return r


def int8_cublas_tops(torch):
    """Dense int8 GEMM throughput of cuBLASLt (torch._int_mm, 8192^3) on this GPU, best of 10: context only."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device="cuda")
        for _ in range(3):
            torch._int_mm(a, b)
        best = 1e9
        for _ in range(10):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e))
        del a, b
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    except Exception:  # noqa: BLE001 -- informational only
        return None


def int8_cublas_pack_shape(torch, count, cols, batch, min_s=1.0):
    """cuBLASLt's int8 GEMM (torch._int_mm) of the pack's shape -- (4 cols) x (tg n) packing-matrix planes times
    (tg n) x (4 batch) key limbs -- back to back for at least min_s, as the GEMMs of the timed region run: the library
    rate under the same power cap (context for the roofline; its int32 output is not reduced mod Q)."""
    try:
        a = torch.randint(-128, 127, (4 * cols, count), dtype=torch.int8, device="cuda")
        b = torch.randint(-128, 127, (count, 4 * batch), dtype=torch.int8, device="cuda")
        for _ in range(3):
            torch._int_mm(a, b)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n, ms = 0, 0.0
        while ms < min_s * 1e3:
            s.record()
            for _ in range(20):
                torch._int_mm(a, b)
            e.record()
            e.synchronize()
            ms += s.elapsed_time(e)
            n += 20
        del a, b
        return {"tops": 2.0 * 4 * cols * count * 4 * batch * n / (ms * 1e-3) / 1e12, "ms": ms / n, "launches": n}
    except Exception as ex:  # noqa: BLE001 -- informational only
        return {"error": str(ex)[:200]}


def traffic_from_profile(kernel, rows, record_bytes, batch):
    """DRAM bytes per batch of `kernel` (dram__bytes_read.sum + dram__bytes_write.sum over its launches in one batch)
    from the committed ncu capture, profiles/ncu_traffic.json; None for a configuration it does not cover."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f).get(kernel, {})
    except OSError:
        return None
    return d.get("per_config", {}).get(f"{rows}x{record_bytes}x{batch}")


# ------------------------------------------------------------------------------------------------ ranks
def max_over_ranks(x, world, device="cuda"):
    """The largest value of x over all ranks (every rank gets it); the timing of a multi-GPU run is the slowest
    rank's."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_qps(world, batch, steps, max_ms):
    """Whole-job throughput: every rank answers `steps` batches of `batch` queries; the job takes the slowest
    rank's time."""
    return world * batch * steps / (max_ms * 1e-3)


def block_count(first_ms, min_s=MIN_TIMED_S, min_blocks=MIN_BLOCKS, max_blocks=5000):
    """Blocks to time, the first included, so that they add up to at least min_s of device time."""
    return int(min(max_blocks, max(min_blocks, math.ceil(min_s * 1e3 / max(first_ms, 1e-3)))))


def timed_blocks(block, world, barrier, min_s=MIN_TIMED_S, min_blocks=MIN_BLOCKS):
    """block() runs one block of steps between synchronisations and returns its device time in ms.  Every rank runs
    the same number of blocks (from the first block's time, max over ranks); returns the per-block times, each the
    max over ranks."""
    barrier()
    times = [max_over_ranks(block(), world)]
    for _ in range(block_count(times[0], min_s, min_blocks) - 1):
        barrier()
        times.append(max_over_ranks(block(), world))
    return times


# ------------------------------------------------------------------------------------------------ reference arm
def run_reference_cpu(st, frames, steps, warmup, sample, min_s=0.0, min_blocks=1):
    """Times the reference engine (or the oracle port when the host cannot run it) on batches of frames (a list of
    uint8 arrays), in blocks of `steps` batches after `warmup` untimed ones, until the blocks add up to min_s.
    Returns (qps, info, first_out)."""
    from oracle import oracle as orc
    methods = orc.ref_methods()
    threads = os.cpu_count() or 1
    if methods:
        ref = orc.RefEngine(st, threads=threads)
        m = methods[0]
        first = None
        for _ in range(warmup):
            r, status, out, _ = ref.answer(frames, m)
            first = out.copy() if first is None else first
        times = []
        while len(times) < steps * min_blocks or sum(times) < min_s:
            for _ in range(steps):
                t0 = time.perf_counter()
                r, status, out, _ = ref.answer(frames, m)
                times.append(time.perf_counter() - t0)
                assert r == len(frames)
        first = out.copy() if first is None else first
        ref.close()
        name = "reference engine src/amx_kernels.cpp (" + ("AMX" if m == 0 else "AVX-512 VNNI") + ")"
        qps = len(frames) * len(times) / sum(times)
        return qps, {"kind": "reference", "cores": threads, "engine": name,
                     "sample": f"{len(times)} timed batches of {len(frames)} queries after {warmup} warm-up, {sample}",
                     "median_batch_ms": 1e3 * statistics.median(times), "timed_s": sum(times)}, first
    # no AVX-512 on this host: the plain-C restatement, on a bounded sample of queries
    o = orc.Oracle()
    sub = frames[:8]
    t0 = time.perf_counter()
    o.answer(st, sub)
    dt = time.perf_counter() - t0
    return len(sub) / dt, {"kind": "port", "cores": threads, "engine": "oracle/alto_oracle.c",
                           "sample": f"one batch of {len(sub)} queries, {sample}"}, None


def main_reference(a):
    """The reference arm: the reference's own CPU engine on this arm's workload.  Its state and frames come from the
    oracle's generators (the same bytes as the engine package's, checked by the CPU tests), so this process never
    loads the engine library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as orc
    o = orc.Oracle()
    p = orc.Params(a.rows, a.record_bytes)
    st = orc.State(p, seed=1, oracle=o)
    frames = o.synthetic_requests(p, a.batch, seed=1000)
    fl = [frames[i] for i in range(a.batch)]
    steps, warmup = max(1, a.steps), max(3, a.warmup)
    qps, info, _ = run_reference_cpu(st, fl, steps, warmup, f"{a.rows * a.record_bytes / 2**30:g} GiB state",
                                     min_s=MIN_TIMED_S)
    line = {"impl": "reference", "metric": METRIC, "value": qps, "unit": "QPS", "n_gpus": a.gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": 1e3 * a.batch / qps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8 x u32 limbs -> int32/u64 (exact integer)", "data": "synthetic",
            "config": config_dict(a), "cpu_baseline": dict(info, value=qps, unit="QPS"),
            "e2e": {"value": qps, "unit": "QPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------ our arm
class Measure:
    """Device-resident, kernel, end-to-end and single-query measurements of one engine at one batch size.  Frames are
    generated on the device (the bytes of service.synthetic_requests) and copied to pinned host memory for the
    end-to-end path."""

    def __init__(self, torch, e, p, B, seed, lanes, barrier, world, sampler):
        from altopir_b200 import service as svc
        self.torch, self.e, self.p, self.B, self.lanes = torch, e, p, B, lanes
        self.barrier, self.world, self.sampler = barrier, world, sampler
        self.rl, self.ql = e.response_len(), e.request_len()
        self.stride = (7 + self.ql + 255) // 256 * 256
        # device-resident frames: frame c at slots[c, 7:7 + ql] (the engine's staged layout)
        self.slots = torch.zeros((B, self.stride), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        svc.synthetic_requests_device(p, B, seed, self.slots.data_ptr(), self.stride)
        self.outs = [torch.zeros((B, self.rl), dtype=torch.uint8, device="cuda") for _ in range(lanes)]
        self.stats = [torch.full((B,), -1, dtype=torch.int32, device="cuda") for _ in range(lanes)]
        # pinned host frames and outputs for the end-to-end path
        self.h_req = torch.empty((B, self.ql), dtype=torch.uint8, pin_memory=True)
        self.h_req.copy_(self.slots[:, 7:7 + self.ql])
        self.h_out = torch.zeros((B, self.rl), dtype=torch.uint8, pin_memory=True)
        self.req_ptrs = (ctypes.c_void_p * B)(*[self.h_req.data_ptr() + c * self.ql for c in range(B)])
        self.lens = (ctypes.c_size_t * B)(*([self.ql] * B))
        self.out_ptrs = (ctypes.c_void_p * B)(*[self.h_out.data_ptr() + c * self.rl for c in range(B)])
        self.h_status = np.full(B, -1, dtype=np.int32)
        self.stream = torch.cuda.ExternalStream(e.stream())
        torch.cuda.synchronize()  # the buffers above were filled on torch's stream, which the engine's does not wait on

    def frames(self):
        return self.h_req.numpy()

    def _enqueue(self, i):
        k = i % self.lanes
        self.e.enqueue_device(self.slots.data_ptr(), self.stride, self.B, self.outs[k].data_ptr(), self.rl,
                              self.stats[k].data_ptr())

    def warm(self, warmup):
        """Untimed: the direct path, alto_answer, then the device path on every lane, each capturing its CUDA graph
        (left on for device()).  Returns the device time of one direct batch, which sizes the blocks of the larger
        configurations."""
        torch, e = self.torch, self.e
        e.set_graphs(False)
        e.set_lanes(1)
        for _ in range(2):
            e.enqueue_device(self.slots.data_ptr(), self.stride, self.B, self.outs[0].data_ptr(), self.rl,
                             self.stats[0].data_ptr())
        e.sync()
        s, t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(self.stream)
        e.enqueue_device(self.slots.data_ptr(), self.stride, self.B, self.outs[0].data_ptr(), self.rl,
                         self.stats[0].data_ptr())
        t.record(self.stream)
        e.sync()
        est = s.elapsed_time(t)
        for _ in range(warmup):
            r = e.answer_raw(self.req_ptrs, self.lens, self.B, self.out_ptrs, self.h_status)
            if r != self.B:
                from altopir_b200 import engine as eng
                raise RuntimeError(f"alto_answer returned {r}: {eng.last_error()}")
        e.set_graphs(True)
        e.set_lanes(self.lanes)
        for i in range(max(warmup, self.lanes)):
            self._enqueue(i)
        e.sync()
        return est

    def _timed(self, body, steps, min_s):
        torch, e = self.torch, self.e
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        marks = []

        def block():
            e.sync()
            torch.cuda.synchronize()
            t0 = time.time()
            ms = body(steps, s_ev, e_ev)
            marks.append((t0, time.time()))
            self.sampler.mark(*marks[-1])
            return ms

        times = timed_blocks(block, self.world, self.barrier, min_s=min_s)
        return times, marks

    def device(self, steps, min_s=MIN_TIMED_S):
        """value: batches back to back on `lanes` batch contexts with CUDA graph replay; the fences put the start
        event before every lane's first batch and the end event after every lane's last."""
        e = self.e
        e.set_graphs(True)
        launches = []

        def body(k, s_ev, e_ev):
            e.set_lanes(self.lanes)  # every block starts at lane 0, so lane j meets the outputs it captured
            e.fence()
            s_ev.record(self.stream)
            e.fence()
            for i in range(k):
                self._enqueue(i)
            e.fence()
            e_ev.record(self.stream)
            launches.append(e.last_launches() * k)
            e.sync()
            return s_ev.elapsed_time(e_ev)

        times, marks = self._timed(body, steps, min_s)
        assert all((s == 0).all().item() for s in self.stats)
        dev_out = self.outs[0].cpu().numpy()
        assert all(np.array_equal(o.cpu().numpy(), dev_out) for o in self.outs[1:])
        e.set_graphs(False)
        e.set_lanes(1)
        return times, marks, sum(launches), dev_out

    def kernels(self, steps, min_s=MIN_TIMED_S / 2):
        """Per-kernel durations: the same batches launched directly on one context, every stage bracketed by CUDA
        events on the engine's stream (graph replays record none)."""
        e = self.e
        e.kernel_times(reset=True)

        def body(k, s_ev, e_ev):
            s_ev.record(self.stream)
            for _ in range(k):
                e.enqueue_device(self.slots.data_ptr(), self.stride, self.B, self.outs[0].data_ptr(), self.rl,
                                 self.stats[0].data_ptr())
            e_ev.record(self.stream)
            e.sync()
            return s_ev.elapsed_time(e_ev)

        self._timed(body, steps, min_s)
        kms, nb = e.kernel_times(reset=True)
        return [x / max(nb, 1) for x in kms], nb

    def end_to_end(self, steps, min_s=MIN_TIMED_S):
        """alto_answer with host buffers: uploads and downloads inside the timed region."""
        e = self.e

        def body(k, s_ev, e_ev):
            s_ev.record(self.stream)
            for _ in range(k):
                r = e.answer_raw(self.req_ptrs, self.lens, self.B, self.out_ptrs, self.h_status)
                if r != self.B:
                    from altopir_b200 import engine as eng
                    raise RuntimeError(f"alto_answer returned {r}: {eng.last_error()}")
            e_ev.record(self.stream)
            self.torch.cuda.synchronize()
            return s_ev.elapsed_time(e_ev)

        times, marks = self._timed(body, steps, min_s)
        return times, marks, self.h_out.numpy().copy()

    def plain(self, queries, warmup):
        """The plain path: one query per batch, each waited for.  As a single-query server does, every frame is
        staged into one fixed slot (a device-to-device copy inside the timed region) and the engine replays the
        launch sequence it captured for that slot as a CUDA graph."""
        torch, e = self.torch, self.e
        one = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stage = torch.zeros((1, self.stride), dtype=torch.uint8, device="cuda")
        stage_out = torch.zeros((1, self.rl), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        e.set_graphs(True)

        def go(c):
            with torch.cuda.stream(self.stream):
                stage.copy_(self.slots[c:c + 1], non_blocking=True)
            e.enqueue_device(stage.data_ptr(), self.stride, 1, stage_out.data_ptr(), self.rl, None)

        for i in range(warmup):  # untimed: kernel loading and the graph's capture
            go(i % self.B)
        e.sync()
        check = bool(torch.equal(stage_out[0], self.outs[0][(warmup - 1) % self.B]))
        self.barrier()
        lat = []
        t0 = time.time()
        for i in range(queries):
            one[0].record(self.stream)
            go(i % self.B)
            one[1].record(self.stream)
            e.sync()
            lat.append(one[0].elapsed_time(one[1]))
        self.sampler.mark(t0, time.time())
        e.set_graphs(False)
        total = max_over_ranks(sum(lat), self.world)
        ls = sorted(lat)
        return {"qps": self.world * queries / (total * 1e-3), "queries": queries, "p50_ms": ls[len(ls) // 2],
                "p99_ms": ls[min(len(ls) - 1, int(len(ls) * 0.99))],
                "api": "alto_enqueue_device, one frame staged into a fixed slot, CUDA graph replay"}, check

    def close(self):
        del self.slots, self.outs, self.stats, self.h_req, self.h_out
        self.torch.cuda.empty_cache()


def summarize(m, p, B, steps, world, dev, kern, e2e, plain, peaks, peak_src, traffic=None):
    """The JSON fields of one configuration from its measurements."""
    (dtimes, dmarks, launches, dev_out), (kms, nb), (etimes, emarks, host_out) = dev, kern, e2e
    nblocks, eblocks = len(dtimes), len(etimes)
    value = job_qps(world, B, steps * nblocks, sum(dtimes))
    e2e_qps = job_qps(world, B, steps * eblocks, sum(etimes))
    alg = algorithmic(p.rows, p.record_bytes, B, p.count)
    avg = {"scan_gemm": kms[2], "pack_gemm": kms[3]}
    dom = max(avg, key=avg.get)
    kernels = {}
    for k, ms in avg.items():
        kernels[k] = {"avg_ms": ms, "tops": alg[k]["ops"] / (ms * 1e-3) / 1e12,
                      "gbs": alg[k]["bytes"] / (ms * 1e-3) / 1e9}
    kernels.update({"validate": {"avg_ms": kms[0]}, "limb_split": {"avg_ms": kms[1]}, "tail": {"avg_ms": kms[4]},
                    "batches_timed": nb})
    bpq = {"value": value, "unit": "QPS", "ms_per_step": sum(dtimes) / (steps * nblocks)}
    return {
        "value": value, "ms_per_step": bpq["ms_per_step"], "steps": steps, "blocks": nblocks,
        "timed_region_s": sum(dtimes) / 1e3,
        "block_ms_per_step": {"min": min(dtimes) / steps, "median": statistics.median(dtimes) / steps,
                              "max": max(dtimes) / steps},
        "e2e": {"value": e2e_qps, "unit": "QPS", "h2d_bytes_per_step": B * m.ql, "d2h_bytes_per_step": B * m.rl + 4 * B,
                "ms_per_step": sum(etimes) / (steps * eblocks), "blocks": eblocks,
                "timed_region_s": sum(etimes) / 1e3, "api": "alto_answer (pinned host frames and outputs)"},
        "gpu_launches": launches,
        "roofline": roofline_of(dom, alg[dom], avg[dom], peaks, peak_src, traffic),
        "kernels": kernels,
        "plain_per_query": dict(plain[0], batched_over_plain=value / plain[0]["qps"]),
        "byte_exact": {"device_vs_host_path": bool(np.array_equal(dev_out, host_out)), "plain_vs_batched": plain[1]},
    }


def lanes_for(lanes, rows, batch):
    """Batch lanes of the device-resident loop: two overlapping batches help while one record chunk of a batch's
    query limbs (4 bytes per record and frame, chunks of 32768 records) is a small part of the 126 MB L2; at 1024
    frames a chunk's limbs are 128 MiB and two batches in flight evict each other's (measured at 8 GiB, B = 1024:
    one lane 32,100-32,600 QPS, two lanes 30,500)."""
    return lanes if 4 * batch * min(rows, 32768) <= (64 << 20) else 1


def engine_for(svc, eng, p, host_db):
    """An engine over the seeded synthetic state; without host_db the database is generated on the device."""
    st = svc.SyntheticState.make(p, seed=1, keep_values=host_db, host_db=host_db)
    e = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
    st.ub = None
    return st, e


def measure_offline(svc, p, e=None, reps=3):
    """The scheme's offline set-up on the device (alto_engine_offline: hint, InspiRING precomputation, packing matrix,
    bold_t_hat, row-0 prefixes, built in HBM for the resident synthetic records), device time of `reps` runs, then
    requests of the client restatement answered by the engine and decrypted.  `e`: an engine over the synthetic
    records whose state may be replaced (a fresh one is made and closed otherwise)."""
    from altopir_b200 import client, offline
    own = e is None
    if own:
        e = offline.blank_engine(p)
    try:
        ms = sorted(offline.prepare(e, p) for _ in range(reps))
        idx = [0, p.rows // 3, p.rows - 1]
        clients = [client.Client(p, seed=900 + k) for k in range(len(idx))]
        frames = [c.request(i) for c, i in zip(clients, idx)]
        out = np.zeros((len(idx), e.response_len()), dtype=np.uint8)
        status = np.full(len(idx), -1, dtype=np.int32)
        e.answer(frames, out, status)
        ok = all(np.array_equal(c.decrypt(out[k]), svc.synthetic_record(i, p.record_bytes))
                 for k, (c, i) in enumerate(zip(clients, idx)))
    finally:
        if own:
            e.close()
    return {"config": f"{p.rows} records x {p.record_bytes} B", "device_ms_min": ms[0],
            "device_ms_median": ms[len(ms) // 2], "runs": reps, "decrypts": bool(ok),
            "requests_decrypted": len(idx)}


OFFLINE_WHAT = ("alto_engine_offline: the scheme's hint, InspiRING precomputation, packing matrix, bold_t_hat and "
                "row-0 prefixes built in HBM for the resident database (Prepared::new); then requests of the client "
                "restatement answered and decrypted")


def main_ours(a):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    import __graft_entry__ as ge
    ge.load()
    from altopir_b200 import engine as eng, service as svc

    def barrier():
        if world > 1:
            dist.barrier()

    eng.init()
    K, W = max(1, a.steps), max(3, a.warmup)
    lanes = max(1, min(4, a.lanes))
    peaks, peak_src = measured_peaks()
    int8_tops = int8_cublas_tops(torch) if rank == 0 and not a.profile else None
    sampler = ClockSampler()
    if rank == 0:
        sampler.start()

    # ---- the headline configuration
    p = svc.params(a.rows, a.record_bytes)
    if a.profile:
        st, e = engine_for(svc, eng, p, host_db=False)
        m = Measure(torch, e, p, a.batch, 1000 + rank, 1, barrier, world, sampler)
        e.set_graphs(False)
        for _ in range(max(1, a.warmup)):
            m._enqueue(0)
        e.sync()
        for _ in range(a.profile):
            m._enqueue(0)
        e.sync()
        for _ in range(a.profile):
            assert e.answer_raw(m.req_ptrs, m.lens, a.batch, m.out_ptrs, m.h_status) == a.batch
        sampler.stop()
        m.close()
        e.close()
        print(f"profile: {a.profile} device batches and {a.profile} alto_answer calls of {a.batch} frames",
              file=sys.stderr)
        return 0
    want_cpu = rank == 0 and world == 1 and not a.no_cpu_baseline
    st, e = engine_for(svc, eng, p, host_db=want_cpu)
    head_lanes = lanes_for(lanes, a.rows, a.batch)
    m = Measure(torch, e, p, a.batch, 1000 + rank, head_lanes, barrier, world, sampler)
    m.warm(W)
    dev = m.device(K)
    kern = m.kernels(K)
    e2e = m.end_to_end(K)
    plain = m.plain(a.plain_queries, W)
    head_clocks = sampler.summary()
    res = summarize(m, p, a.batch, K, world, dev, kern, e2e, plain, peaks, peak_src,
                    traffic_from_profile("scan_gemm" if kern[0][2] >= kern[0][3] else "pack_gemm", a.rows,
                                         a.record_bytes, a.batch))
    frames = m.frames().copy() if want_cpu else None
    m.close()
    e.close()

    cpu_baseline, exact_vs_ref = None, None
    if want_cpu:
        qps_cpu, info, ref_out = run_reference_cpu(st, [frames[i] for i in range(a.batch)], steps=5, warmup=1,
                                                   sample=f"{a.rows * a.record_bytes / 2**30:g} GiB state")
        cpu_baseline = dict(info, value=qps_cpu, unit="QPS")
        if ref_out is not None:
            exact_vs_ref = bool(np.array_equal(ref_out, dev[3]))
    st = None

    cublas_pack = int8_cublas_pack_shape(torch, p.count, p.record_bytes, a.batch) if rank == 0 else None

    # ---- the larger databases (rank 0 of a one-GPU run): blocks of up to K steps, about 0.2 s each
    configs = []
    want_offline, offline_runs = rank == 0 and world == 1 and not a.no_offline, []
    if world == 1 and not a.no_configs:
        for rows, batches, plain_q in SUB_CONFIGS:
            pp = svc.params(rows, a.record_bytes)
            _, e = engine_for(svc, eng, pp, host_db=False)
            for B in batches:
                mark0 = len(sampler.marks)
                m = Measure(torch, e, pp, B, 2000, lanes_for(lanes, rows, B), barrier, world, sampler)
                est = m.warm(W)
                k = int(max(1, min(K, math.ceil(200.0 / max(est, 1e-3)))))
                d = m.device(k)
                kk = m.kernels(k, min_s=0.3)
                ee = m.end_to_end(k)
                pl = m.plain(plain_q, 3)
                r = summarize(m, pp, B, k, world, d, kk, ee, pl, peaks, peak_src)
                pub = PUBLISHED_QPS.get(rows)
                r.update({"config": config_dict(a, rows, B), "clocks": sampler.summary(sampler.marks[mark0:]),
                          "lanes": lanes_for(lanes, rows, B),
                          "vs_baseline": r["value"] / pub[0] if pub else None,
                          "vs_baseline_ref": f"{pub[0]} QPS, {pub[1]}" if pub else None})
                configs.append(r)
                print(f"config {rows} records, B = {B}: {r['value']:.0f} QPS device, {r['e2e']['value']:.0f} e2e, "
                      f"frac {r['roofline']['frac']:.3f}", file=sys.stderr, flush=True)
                m.close()
            if want_offline:
                offline_runs.append(measure_offline(svc, pp, e))
            e.close()
            torch.cuda.empty_cache()
    sampler.stop()
    if want_offline:
        offline_runs.insert(0, measure_offline(svc, p))
    offline_setup = {"what": OFFLINE_WHAT, "runs": offline_runs} if want_offline else None

    if rank == 0:
        pub = PUBLISHED_QPS.get(a.rows) if (a.batch == 128 and a.record_bytes == 32768) else None
        clocks = dict(head_clocks)
        if clocks.get("sm_mhz"):
            clocks["ms_per_step_x_sm_mhz"] = res["ms_per_step"] * clocks["sm_mhz"]
        line = {
            "metric": METRIC, "value": res["value"], "unit": "QPS", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": res["value"] / pub[0] if pub else None,
            "vs_baseline_ref": f"{pub[0]} QPS, {pub[1]}, 16-core Xeon Silver 4514Y (AMX)" if pub else None,
            "dtype": "u8 x u8 limbs -> int32 (tcgen05 kind::i8), exact", "data": "synthetic",
            "config": config_dict(a), "parallelism": f"replicas{world}",
            "blocks": res["blocks"], "timed_region_s": res["timed_region_s"],
            "block_ms_per_step": res["block_ms_per_step"],
            "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
            "api": f"alto_enqueue_device (frames resident in HBM) rotating through {head_lanes} batch context(s) "
                   "(alto_engine_set_lanes; consecutive batches overlap on the device), launch sequence replayed as "
                   "a CUDA graph; kernels and roofline from a second pass of the same batches launched directly on "
                   "one context",
            "roofline": dict(res["roofline"], int8_cublaslt_tops=int8_tops,
                             int8_cublaslt_pack_shape_sustained=cublas_pack),
            "kernels": res["kernels"], "cpu_baseline": cpu_baseline, "clocks": clocks,
            "plain_per_query": res["plain_per_query"],
            "byte_exact": dict(res["byte_exact"], vs_reference_engine=exact_vs_ref),
            "configs": configs,
            "offline_setup": offline_setup,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------ serving mode
def main_serve(a):
    """Open-loop serving: Poisson arrivals at each offered rate into the continuous-batching loop (max_batch
    a.max_batch, --serve-slots device batch contexts, the resident client table at its default size) and into a
    one-query-per-batch loop, answered QPS and latency percentiles from submit to completion, plus the loop's own
    statistics and a summary of its per-batch log.  One JSON line."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import __graft_entry__ as ge
    ge.load()
    from altopir_b200 import engine as eng, service as svc, server as srv
    eng.init()
    p = svc.params(a.rows, a.record_bytes)
    st = svc.SyntheticState.make(p, seed=1, keep_values=False, host_db=False)
    e = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
    st.ub = None
    # the clients' frames, generated on the device in pieces and kept in host memory
    ql = e.request_len()
    stride = (7 + ql + 255) // 256 * 256
    frames = np.empty((a.serve_clients, ql), dtype=np.uint8)
    piece = max(1, min(a.serve_clients, (4 << 30) // stride))
    slots = torch.zeros((piece, stride), dtype=torch.uint8, device="cuda")
    for c0 in range(0, a.serve_clients, piece):
        n = min(piece, a.serve_clients - c0)
        torch.cuda.synchronize()
        svc.synthetic_requests_device(p, n, 2024, slots.data_ptr(), stride, first_client=c0)
        frames[c0:c0 + n] = slots[:n, 7:7 + ql].cpu().numpy()
    del slots
    torch.cuda.empty_cache()
    rates = [float(x) for x in a.serve.split(",")]
    print(f"serve: engine and {a.serve_clients} frames ready", file=sys.stderr, flush=True)
    rows = []
    for label, mb in (("batched", a.max_batch), ("plain", 1)):
        s = srv.Server(e, max_batch=mb, queue_cap=a.serve_queue, slots=a.serve_slots)
        for rate in rates:
            before = s.stats()
            nlog = len(s.log())
            t0 = time.time()
            res, offered, elapsed = srv.poisson_load(s, frames, rate, a.serve_seconds, seed=int(rate), clients=8)
            print(f"serve {label} {rate:g} QPS offered: {offered} requests in {time.time() - t0:.1f} s",
                  file=sys.stderr, flush=True)
            lat = sorted(r[3] * 1e3 for r in res if r[1] == 0)
            ok = len(lat)
            pct = lambda q: lat[min(len(lat) - 1, int(q * len(lat)))] if lat else None
            after = s.stats()
            log = s.log()[nlog:]
            dev = sorted(r["device_ms"] for r in log)
            rows.append({"loop": label, "offered_qps": rate, "requests": offered, "answered": ok,
                         "busy": sum(1 for r in res if r[1] == srv.BUSY),
                         "answered_qps": ok / elapsed, "elapsed_s": elapsed, "p50_ms": pct(0.5), "p99_ms": pct(0.99),
                         "p999_ms": pct(0.999),
                         "batches": len(log), "mean_batch": (sum(r["on_device"] for r in log) / len(log)) if log else 0,
                         "batch_device_ms_p50": dev[len(dev) // 2] if dev else None,
                         "resident_frames": after["resident_hits"] - before["resident_hits"],
                         "packed_frames": sum(r["packed"] for r in log)})
        rows[-1]["loop_stats"] = s.stats()
        s.close()
    line = {"metric": "serving: answered QPS and p50/p99/p99.9 latency (submit to response) under open-loop "
                      "Poisson arrivals", "unit": "QPS", "n_gpus": 1, "data": "synthetic",
            "config": {"workload": f"continuous batching over a {a.rows * a.record_bytes / 2**30:g} GiB database, "
                                   f"{a.serve_clients} seeded clients, {a.serve_seconds} s per rate",
                       "rows": a.rows, "record_bytes": a.record_bytes, "max_batch": a.max_batch,
                       "slots": a.serve_slots, "queue": a.serve_queue},
            "rates": rows}
    print(json.dumps(line))
    e.close()
    return 0


# ------------------------------------------------------------------------------------------------ column shards
class CudaTimer:
    """Device time of a stretch of work on torch's current stream (CUDA events)."""

    def __init__(self, torch):
        self.torch = torch
        self.s, self.e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def sync(self):
        self.torch.cuda.synchronize()

    def start(self):
        self.s.record()

    def stop(self):
        self.e.record()
        self.torch.cuda.synchronize()
        return self.s.elapsed_time(self.e)


class HostTimer:
    """Wall time of a stretch of host work (the CPU ranks of the tests)."""

    def sync(self):
        pass

    def start(self):
        self.t0 = time.perf_counter()

    def stop(self):
        return 1e3 * (time.perf_counter() - self.t0)


def shard_timed(step, timer, steps, warmup, world, device):
    """--shard timing: warm-up steps, a barrier, then exactly `steps` steps timed on this rank; max over ranks."""
    import torch.distributed as dist
    for _ in range(max(3, warmup)):
        step()
    timer.sync()
    dist.barrier()
    timer.start()
    for _ in range(steps):
        step()
    return max_over_ranks(timer.stop(), world, device=device)


def shard_line(a, world, ranges, ms, ms_nccl, exact):
    """Rank 0's JSON line of --shard: the whole job answers --batch queries per step (every rank answers the same
    frames for its parts), so `value` is strong scaling."""
    cfg = config_dict(a)
    return {"metric": METRIC, "value": a.batch * a.steps / (ms * 1e-3), "unit": "QPS", "n_gpus": world,
            "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "u8 x u8 limbs -> int32 (exact)", "data": "synthetic",
            "config": cfg, "parallelism": f"columns{world}", "output_ranges": ranges, "mode": "column shards",
            "exchange": "frames broadcast from rank 0; each rank's tail kernel writes its parts into every rank's "
                        "response buffer (CUDA IPC mappings), then one barrier",
            "nccl_all_gather": {"value": a.batch * a.steps / (ms_nccl * 1e-3), "unit": "QPS",
                                "ms_per_step": ms_nccl / a.steps},
            "byte_exact": exact}


def main_shard(a):
    """Column sharding (altopir_b200.shard): rank r holds the columns of its output range; every step rank 0's batch
    of frames is broadcast and each rank's tail kernel writes its parts into every rank's response buffer (CUDA IPC
    mappings; shard.PeerGather), so that after one barrier every rank holds the full responses.  Timed on the device,
    max over ranks.  Beside it, `nccl_all_gather` times the same answer followed by an NCCL all_gather of the parts.
    Rank 0 checks both against a whole engine (byte-exact)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if "MASTER_ADDR" not in os.environ:  # one process without torchrun: a group of one
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29500 + os.getpid() % 1000))
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=timedelta(seconds=300),
                            device_id=torch.device("cuda", local))
    import __graft_entry__ as ge
    ge.load()
    from altopir_b200 import engine as eng, service as svc, shard
    eng.init()
    p = svc.params(a.rows, a.record_bytes)
    st = svc.SyntheticState.make(p, seed=1, keep_values=False)
    ranges = shard.output_ranges(p.instances, world)
    o0, o1 = ranges[rank]
    e = shard.shard_engine(st, o0, o1, threads=svc.threads())
    B, ql, part_len = a.batch, e.request_len(), st.prefixes[0].size
    stride = (7 + ql + 255) // 256 * 256
    slots = torch.zeros((B, stride), dtype=torch.uint8, device="cuda")
    if rank == 0:
        slots[:, 7:7 + ql] = torch.from_numpy(svc.synthetic_requests(p, B, seed=1000)).cuda()
    # the product path: each rank's tail kernel writes its parts into every rank's response buffer (CUDA IPC
    # mappings, NVLink stores between GPUs); the baseline beside it: answer locally, then NCCL all_gather
    fused = shard.PeerGather(e, ranges, part_len, B)
    gathered = shard.ShardedAnswerer(shard.engine_local(e), ranges, part_len, "cuda")
    timer = CudaTimer(torch)
    ms = shard_timed(lambda: fused.answer(slots, stride, B, src=0), timer, a.steps, a.warmup, world, "cuda")
    status, resp = fused.answer(slots, stride, B, src=0)
    resp = resp.clone()
    ms_nccl = shard_timed(lambda: gathered.answer(slots, stride, B), timer, a.steps, a.warmup, world, "cuda")
    _, resp_nccl = gathered.answer(slots, stride, B)
    fused.close()
    exact = None
    if rank == 0:
        full = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
        want = torch.zeros((B, full.response_len()), dtype=torch.uint8, device="cuda")
        wst = np.full(B, -1, dtype=np.int32)
        torch.cuda.synchronize()
        full.answer_device(slots.data_ptr(), stride, B, want.data_ptr(), full.response_len(), wst)
        exact = {"fused_vs_whole_engine": bool(torch.equal(want, resp)) and list(wst) == list(status),
                 "nccl_vs_whole_engine": bool(torch.equal(want, resp_nccl))}
        full.close()
    dist.barrier()
    if rank == 0:
        print(json.dumps(shard_line(a, world, ranges, ms, ms_nccl, exact)))
    e.close()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    args = parse()
    if args.serve:
        sys.exit(main_serve(args))
    if args.shard and args.impl == "ours":
        sys.exit(main_shard(args))
    sys.exit(main_reference(args) if args.impl == "reference" else main_ours(args))
