"""Column shards on the GPU: engines built over output slices of the state (one GPU here, each shard's engine in turn)
return exactly the parts of the full engine's responses, through alto_answer and through the device-resident path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_shard_engines_reassemble_the_full_engine_answer(gpu, svc, eng):
    import torch
    from altopir_b200 import shard
    p = svc.params(4096, 16384)  # 8 outputs
    st = svc.SyntheticState.make(p, seed=81, full_prefix=True)
    b = 10
    frames = svc.synthetic_requests(p, b, seed=82)
    frames[6, 9 + 4 * p.count:13 + 4 * p.count] = 0xFF  # a z word >= Q: status 3
    full = eng.Engine.from_state(st)
    want = np.zeros((b, full.response_len()), dtype=np.uint8)
    want_status = np.full(b, -1, dtype=np.int32)
    full.answer([frames[i] for i in range(b)], want, want_status)
    ql = full.request_len()
    full.close()
    part_len = st.prefixes[0].size
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
    ok = want_status == 0
    for world in (2, 3):
        ranges = shard.output_ranges(p.instances, world)
        host_parts, dev_parts = [], []
        for o0, o1 in ranges:
            e = shard.shard_engine(st, o0, o1)
            assert e.request_len() == ql and e.response_len() == (o1 - o0) * part_len
            out = np.zeros((b, e.response_len()), dtype=np.uint8)
            status = np.full(b, -1, dtype=np.int32)
            e.answer([frames[i] for i in range(b)], out, status)
            assert list(status) == list(want_status)
            host_parts.append(out)
            dstatus, dpart = shard.engine_local(e)(slots, stride, b)
            assert list(dstatus) == list(want_status)
            dev_parts.append(dpart)
            e.close()
        assert np.array_equal(shard.assemble(host_parts, ranges, part_len)[ok], want[ok]), world
        assert np.array_equal(shard.assemble(dev_parts, ranges, part_len).cpu().numpy()[ok], want[ok]), world
