"""Autotuner of the GEMM plans: for each database size and batch-size bucket, time every candidate plan (single-CTA
or CTA-pair kernels, wide scan units, limb-column tile cap, scan split target) on the device-resident path, check
that it returns the same bytes as the built-in plan, and write the fastest into tuning.txt next to the library,
which alto_engine_new loads.

    python altopir-public_b200/autotune.py --rows 32768,262144 [--out altopir-public_b200/tuning.txt]
"""
import argparse
import datetime
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

BUCKETS = (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024)


def candidates(b, nchunks):
    limb_cols = 4 * ((b + 3) // 4 * 4)
    out = [(0, -1, 0, 0)]  # single-CTA kernels
    if limb_cols > 16:
        caps = (256, 128) if limb_cols > 128 else (256,)
        for cap in caps:
            wides = (0, 1) if cap == 256 and limb_cols >= 512 else (0,)
            for wide in wides:
                for upp in (6, 12, 24):
                    out.append((1, wide, cap, upp))
    return out


def time_plan(torch, e, slots, stride, b, d_out, rl, iters):
    stream = torch.cuda.ExternalStream(e.stream())
    for _ in range(2):
        e.enqueue_device(slots.data_ptr(), stride, b, d_out.data_ptr(), rl)
    e.sync()
    s, t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(iters):
        e.enqueue_device(slots.data_ptr(), stride, b, d_out.data_ptr(), rl)
    t.record(stream)
    e.sync()
    torch.cuda.synchronize()
    return s.elapsed_time(t) / iters


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", default="32768,262144")
    ap.add_argument("--record-bytes", type=int, default=32768)
    ap.add_argument("--buckets", default=",".join(map(str, BUCKETS)))
    ap.add_argument("--budget-ms", type=float, default=60.0, help="device time per candidate")
    ap.add_argument("--out", default=os.path.join(HERE, "tuning.txt"))
    a = ap.parse_args()
    import torch
    import __graft_entry__ as ge
    ge.load()
    from altopir_b200 import engine as eng, service as svc
    eng.init()
    buckets = [int(x) for x in a.buckets.split(",")]
    lines = []
    for rows in [int(x) for x in a.rows.split(",")]:
        p = svc.params(rows, a.record_bytes)
        st = svc.SyntheticState.make(p, seed=5, keep_values=False)
        e = eng.Engine.from_state(st, threads=svc.threads(), tile=rows * a.record_bytes <= (8 << 30))
        e.set_tuning([])
        nchunks = (rows + 32767) // 32768
        bmax = max(buckets)
        frames = svc.synthetic_requests(p, bmax, seed=6)
        ql, rl = e.request_len(), e.response_len()
        stride = (7 + ql + 255) // 256 * 256
        slots = torch.zeros((bmax, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
        d_out = torch.zeros((bmax, rl), dtype=torch.uint8, device="cuda")
        for b in buckets:
            e.set_tuning([])
            t_ref = time_plan(torch, e, slots, stride, b, d_out, rl, 2)
            want = d_out[:b].clone()
            iters = max(2, int(a.budget_ms / max(t_ref, 1e-3)))
            best = None
            for pair, wide, cap, upp in candidates(b, nchunks):
                e.set_tuning([(b, pair, wide, cap, upp)])
                d_out[:b].zero_()
                ms = time_plan(torch, e, slots, stride, b, d_out, rl, iters)
                if not torch.equal(d_out[:b], want):
                    raise SystemExit(f"plan {(pair, wide, cap, upp)} changed the responses at rows {rows}, b {b}")
                if best is None or ms < best[0]:
                    best = (ms, pair, wide, cap, upp)
                print(f"rows {rows} b {b:5d} plan pair={pair} wide={wide} cap={cap} upp={upp}: {ms:.3f} ms",
                      flush=True)
            ms, pair, wide, cap, upp = best
            lines.append(f"{rows} {b} {pair} {wide} {cap} {upp}   # {ms:.3f} ms per batch, built-in {t_ref:.3f}")
        e.close()
        del slots, d_out
        torch.cuda.empty_cache()
    gpu = torch.cuda.get_device_name(0)
    with open(a.out, "w") as f:
        f.write(f"# GEMM plans chosen by autotune.py on {gpu}, {datetime.date.today()}, record bytes "
                f"{a.record_bytes}\n# rows_max b_max pair wide bn_cap units_per_pair\n")
        f.write("\n".join(lines) + "\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
