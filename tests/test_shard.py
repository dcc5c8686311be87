"""Column sharding (altopir_b200.shard) on the CPU: output slices of the state answer the same frames with the parts of
the full answer, checked on the oracle, and two gloo ranks broadcast frames and gather parts into full responses."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_output_ranges_cover_every_output_once(svc):
    from altopir_b200 import shard
    for outputs in (1, 2, 5, 16, 17):
        for world in range(1, min(outputs, 8) + 1):
            r = shard.output_ranges(outputs, world)
            assert r[0][0] == 0 and r[-1][1] == outputs and len(r) == world
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [o1 - o0 for o0, o1 in r]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        shard.output_ranges(2, 3)


def test_slices_reassemble_the_full_answer(oracle, svc):
    # 4 outputs (cols = 4 n): every split over 2..4 ranks gives back the full responses byte for byte
    from altopir_b200 import shard
    p = svc.params(2048, 8192)
    st = svc.SyntheticState.make(p, seed=71, full_prefix=True)
    frames = svc.synthetic_requests(p, 3, seed=72)
    frames[1, 9:13] = 0xFF  # a y word >= Q: status 3 on every shard
    r, status, full = oracle.answer(st, [frames[i] for i in range(3)])
    part_len = st.prefixes[0].size
    for world in (2, 3, 4):
        ranges = shard.output_ranges(p.instances, world)
        parts = []
        for o0, o1 in ranges:
            sl = shard.slice_state(st, o0, o1)
            assert sl.db_col.base is not None  # a view, not a copy
            rr, ss, part = oracle.answer(sl, [frames[i] for i in range(3)])
            assert rr == r and list(ss) == list(status)
            parts.append(part)
        got = shard.assemble(parts, ranges, part_len)
        ok = status == 0
        assert np.array_equal(got[ok], full[ok]), world


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ge.load()
    from altopir_b200 import service as svc, shard
    from oracle.oracle import Oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    p = svc.params(2048, 8192)
    st = svc.SyntheticState.make(p, seed=73)
    ranges = shard.output_ranges(p.instances, world)
    o0, o1 = ranges[rank]
    sl, orc = shard.slice_state(st, o0, o1), Oracle()
    b, ql = 4, svc.request_len(p)
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8)
    if rank == 0:  # only the source rank has the frames before the broadcast
        slots[:, 7:7 + ql] = torch.from_numpy(svc.synthetic_requests(p, b, seed=74))

    def local(slots_, stride_, b_):
        fr = [slots_[c, 7:7 + ql].numpy() for c in range(b_)]
        r, status, part = orc.answer(sl, fr)
        return status, torch.from_numpy(part)

    ans = shard.ShardedAnswerer(local, ranges, st.prefixes[0].size, "cpu")
    status, resp = ans.answer(slots, stride, b)
    # bench.py --shard's rank logic on these ranks: timed steps (max over ranks) and rank 0's JSON line
    import bench
    a = bench.parse(["--shard", "--rows", "2048", "--record-bytes", "8192", "--batch", str(b), "--steps", "2",
                     "--warmup", "1"])
    ms = bench.shard_timed(lambda: ans.answer(slots, stride, b), bench.HostTimer(), a.steps, a.warmup, world, "cpu")
    if rank == 0:
        r, st0, full = orc.answer(st, [slots[c, 7:7 + ql].numpy() for c in range(b)])
        line = bench.shard_line(a, world, ranges, ms, ms, {"nccl_vs_whole_engine": True})
        out[0] = bool(np.array_equal(resp.numpy(), full)) and list(status) == list(st0)
        out[1] = (line["n_gpus"] == world and line["scaling"] == "strong" and line["steps"] == 2 and
                  line["warmup"] == 3 and abs(line["value"] - b * 2 / (ms * 1e-3)) < 1e-6 * line["value"] and
                  line["output_ranges"] == ranges and line["config"] == bench.config_dict(a))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_full_responses(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        assert out[0] is True and out[1] is True
