"""Parity at the larger configurations of the benchmark: the uneven-batch sweep over an 8 GiB database against the
reference engine itself (compiled from its own source, when the host CPU can run it), and batches of 128 and 1024
over a 64 GiB database against the oracle on a seeded sample of response parts."""
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _answer(e, frames, b):
    out = np.zeros((b, e.response_len()), dtype=np.uint8)
    status = np.full(b, -1, dtype=np.int32)
    n, _ = e.answer([frames[i] for i in range(b)], out, status)
    return n, status, out


def test_8gib_uneven_batch_sweep_matches_reference(gpu, oracle, svc, eng):
    from oracle.oracle import RefEngine, ref_methods
    p = svc.params(262144, 32768)
    st = svc.SyntheticState.make(p, seed=81)
    e = eng.Engine.from_state(st, threads=svc.threads())
    frames = svc.synthetic_requests(p, 1024, seed=82)
    methods = ref_methods()
    ref = RefEngine(st) if methods else None
    rng = np.random.default_rng(83)
    for b in (1, 7, 33, 128, 200, 512, 1024):
        n, status, out = _answer(e, frames, b)
        assert n == b and (status == 0).all(), b
        if ref is not None:
            rr, rs, rout, _ = ref.answer([frames[i] for i in range(b)], methods[0])
            assert rr == b and np.array_equal(rout, out), f"batch {b} differs from the reference engine"
        else:
            cs = rng.integers(0, b, 4)
            os_ = rng.integers(0, p.instances, 4)
            want = oracle.answer_parts(st, [frames[c] for c in cs], os_)
            part = st.prefixes[0].size
            for k, (c, o) in enumerate(zip(cs, os_)):
                assert np.array_equal(out[c, o * part:(o + 1) * part], want[k]), (b, c, o)
    if ref is not None:
        ref.close()
    e.close()


def _free_bytes():
    import torch
    free, _ = torch.cuda.mem_get_info()
    try:
        import psutil
        host = psutil.virtual_memory().available
    except ImportError:
        host = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    return free, host


def _slice_state(st, o, oracle):
    """The state of output o alone (columns [o n, (o + 1) n)), database columns generated on the host: what the
    oracle and the reference engine need to answer part o of a frame over the full record count."""
    from oracle.oracle import Params
    p = st.p
    sl = type("Slice", (), {})()
    sl.p = Params(p.rows, p.n)
    sl.db_col = oracle.synthetic_db_col(p.rows, o * p.n, p.n)
    sl.U = np.ascontiguousarray(st.U[o * p.n:(o + 1) * p.n])
    sl.that, sl.prefixes, sl.inv_table = [st.that[o]], [st.prefixes[o]], st.inv_table
    return sl


def test_64gib_batches_match_reference_and_oracle(gpu, oracle, svc, eng):
    """A 64 GiB database (2^21 records) generated on the device, batches of 128 and 1024 seeded frames through
    alto_answer.  For two seeded outputs the response parts of the first 64 frames of both batches equal the
    reference engine's (compiled from its own source) over that output's columns of the full database, and 16
    sampled parts per batch equal the oracle's."""
    import torch
    free, host = _free_bytes()
    if free < (100 << 30) or host < (48 << 30):
        pytest.skip(f"needs 100 GB of free device memory and 48 GB of host memory ({free >> 30} / {host >> 30} GB)")
    p = svc.params(1 << 21, 32768)
    st = svc.SyntheticState.make(p, seed=91, host_db=False)
    e = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
    ql, part = e.request_len(), st.prefixes[0].size
    stride = (7 + ql + 255) // 256 * 256
    slots = torch.zeros((1024, stride), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    svc.synthetic_requests_device(p, 1024, 92, slots.data_ptr(), stride)
    frames = slots[:, 7:7 + ql].cpu().numpy()
    del slots
    torch.cuda.empty_cache()
    assert np.array_equal(frames[5], svc.synthetic_requests(p, 1, seed=92, first_client=5)[0])
    rng = np.random.default_rng(93)
    outs = {}
    for b in (128, 1024):
        n, status, out = _answer(e, frames, b)
        assert n == b and (status == 0).all(), b
        outs[b] = out
    e.close()
    from oracle.oracle import RefEngine, ref_methods
    methods = ref_methods()
    for o in sorted(rng.choice(p.instances, 2, replace=False)):
        sl = _slice_state(st, int(o), oracle)
        for b in (128, 1024):
            cs = rng.integers(0, b, 8)
            want = oracle.answer_parts(sl, [frames[c] for c in cs], [0] * len(cs))
            for k, c in enumerate(cs):
                assert np.array_equal(outs[b][c, o * part:(o + 1) * part], want[k]), (b, c, o)
        if methods:
            ref = RefEngine(sl)
            rr, rs, rout, _ = ref.answer([frames[c] for c in range(64)], methods[0])
            ref.close()
            assert rr == 64
            for b in (128, 1024):
                assert np.array_equal(outs[b][:64, o * part:(o + 1) * part], rout), (b, o)
