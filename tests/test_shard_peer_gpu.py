"""Column shards whose tail kernels do the all-gather (shard.PeerGather, alto_answer_device_parts): two processes,
each with the shard engine of half the outputs, map each other's response buffer through CUDA IPC and write their
parts into both; after one barrier both buffers hold the full responses, equal to the oracle's.  Both processes use
GPU 0 here (the path between GPUs is the same IPC mapping, over NVLink); nothing in them waits on the other inside
a kernel -- the ranks meet only at host barriers."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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
    from altopir_b200 import engine as eng, service as svc, shard
    from oracle.oracle import Oracle
    torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    eng.init()
    p = svc.params(2048, 8192)  # 4 outputs, 2 per rank
    st = svc.SyntheticState.make(p, seed=111, full_prefix=True)
    ranges = shard.output_ranges(p.instances, world)
    e = shard.shard_engine(st, *ranges[rank])
    ql, part = svc.request_len(p), st.prefixes[0].size
    stride = (7 + ql + 15) // 16 * 16
    # a small tensor first, so that the gather buffer sits inside the same caching-allocator segment at an offset:
    # the IPC handle names the segment, and the offset must travel with it
    pad = torch.zeros(1024, dtype=torch.uint8, device="cuda")
    gather = shard.PeerGather(e, ranges, part, b_max=8)
    ok = gather.export_offset > 0
    del pad
    for call in range(2):  # two calls in a row over the same buffers
        b = 6 if call == 0 else 8
        frames = svc.synthetic_requests(p, b, seed=112 + call)
        frames[1, 9 + 4 * p.count:13 + 4 * p.count] = 0xFF  # a z word >= Q: status 3, no response
        slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
        status, full = gather.answer(slots, stride, b)
        r, ost, want = Oracle().answer(st, [frames[i] for i in range(b)])
        good = ost == 0
        ok &= list(status) == list(ost) and bool(np.array_equal(full.cpu().numpy()[good], want[good]))
    gather.close()
    e.close()
    out[rank] = ok
    dist.destroy_process_group()


def test_two_shards_gather_their_parts_through_ipc_mappings(gpu):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        assert out[0] is True and out[1] is True
