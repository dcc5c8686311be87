"""Autotuner of the GEMM plans: for each database size and batch-size bucket, time every candidate plan (single-CTA
or CTA-pair kernels, wide scan units, limb-column tile cap, scan split target) on the device-resident path, check
that it returns the same bytes as the built-in plan, and write the fastest into tuning.txt next to the library,
which alto_engine_new loads.

    python altopir-public_b200/autotune.py --rows 32768,262144 [--out altopir-public_b200/tuning.txt] [--merge]
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
    ap.add_argument("--budget-ms", type=float, default=80.0, help="device time per candidate and round")
    ap.add_argument("--rounds", type=int, default=3)
    ap.add_argument("--margin", type=float, default=0.03, help="required gain over the built-in plan")
    ap.add_argument("--out", default=os.path.join(HERE, "tuning.txt"))
    ap.add_argument("--merge", action="store_true", help="keep the rows of other database sizes already in --out")
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
        st = svc.SyntheticState.make(p, seed=5, keep_values=False, host_db=False)  # database made on the device
        e = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
        e.set_tuning([])
        nchunks = (rows + 32767) // 32768
        bmax = max(buckets)
        ql, rl = e.request_len(), e.response_len()
        stride = (7 + ql + 255) // 256 * 256
        slots = torch.zeros((bmax, stride), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        svc.synthetic_requests_device(p, bmax, 6, slots.data_ptr(), stride)
        d_out = torch.zeros((bmax, rl), dtype=torch.uint8, device="cuda")
        for b in buckets:
            e.set_tuning([])
            time_plan(torch, e, slots, stride, b, d_out, rl, 2)
            want = d_out[:b].clone()
            t_est = time_plan(torch, e, slots, stride, b, d_out, rl, 2)
            iters = max(2, int(a.budget_ms / max(t_est, 1e-3)))
            plans = [None] + candidates(b, nchunks)   # None: the built-in plan
            times = {i: [] for i in range(len(plans))}
            for _ in range(a.rounds):                 # interleaved rounds: clock and power drift hit all plans alike
                for i, plan in enumerate(plans):
                    e.set_tuning([] if plan is None else [(b,) + plan])
                    d_out[:b].zero_()
                    times[i].append(time_plan(torch, e, slots, stride, b, d_out, rl, iters))
                    if not torch.equal(d_out[:b], want):
                        raise SystemExit(f"plan {plan} changed the responses at rows {rows}, b {b}")
            med = {i: sorted(v)[len(v) // 2] for i, v in times.items()}
            for i, plan in enumerate(plans):
                print(f"rows {rows} b {b:5d} plan {plan}: median {med[i]:.3f} ms", flush=True)
            best = min(range(1, len(plans)), key=lambda i: med[i])
            if med[best] <= (1.0 - a.margin) * med[0]:
                pair, wide, cap, upp = plans[best]
                lines.append(f"{rows} {b} {pair} {wide} {cap} {upp}   # {med[best]:.3f} ms per batch, built-in "
                             f"{med[0]:.3f}")
            else:
                lines.append(f"{rows} {b} -1 -1 0 0   # built-in plan kept ({med[0]:.3f} ms; best other "
                             f"{med[best]:.3f})")
        e.close()
        del slots, d_out
        torch.cuda.empty_cache()
    gpu = torch.cuda.get_device_name(0)
    tuned = {int(x) for x in a.rows.split(",")}
    head = [f"# GEMM plans chosen by autotune.py on {gpu}, {datetime.date.today()}, record bytes {a.record_bytes}",
            f"# command: python altopir-public_b200/autotune.py --rows {a.rows} ({a.rounds} interleaved rounds, "
            f"medians, {a.margin:.0%} margin)"]
    kept = []
    if a.merge and os.path.exists(a.out):  # rows of other database sizes stay as they were
        with open(a.out) as f:
            for line in f:
                if line.startswith("#"):
                    if "rows_max" not in line:
                        head.append(line.rstrip("\n"))
                    continue
                if line.split() and int(line.split()[0]) not in tuned:
                    kept.append(line.rstrip("\n"))
    with open(a.out, "w") as f:
        f.write("\n".join(head) + "\n# rows_max b_max pair wide bn_cap units_per_pair\n")
        f.write("\n".join(sorted(kept + lines, key=lambda x: (int(x.split()[0]), int(x.split()[1])))) + "\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
