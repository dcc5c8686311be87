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


@pytest.mark.skipif(os.environ.get("ALTO_BIG") != "1",
                    reason="64 GiB database: set ALTO_BIG=1 (about 80 GB of host and 85 GB of device memory)")
def test_64gib_batches_sampled_parts_match_oracle(gpu, oracle, svc, eng):
    p = svc.params(1 << 21, 32768)
    st = svc.SyntheticState.make(p, seed=91)
    e = eng.Engine.from_state(st, threads=svc.threads(), tile=False)
    frames = svc.synthetic_requests(p, 1024, seed=92)
    rng = np.random.default_rng(93)
    part = st.prefixes[0].size
    first = {}
    for b in (128, 1024):
        n, status, out = _answer(e, frames, b)
        assert n == b and (status == 0).all(), b
        first[b] = out[:64].copy()  # both batches start with the same 64 frames
        cs = rng.integers(0, b, 16)
        os_ = rng.integers(0, p.instances, 16)
        want = oracle.answer_parts(st, [frames[c] for c in cs], os_)
        for k, (c, o) in enumerate(zip(cs, os_)):
            assert np.array_equal(out[c, o * part:(o + 1) * part], want[k]), (b, c, o)
    e.close()
    # the seeded 64-query subset, whole responses, against the reference engine itself when this host can run it
    from oracle.oracle import RefEngine, ref_methods
    methods = ref_methods()
    if methods:
        ref = RefEngine(st)
        rr, rs, rout, _ = ref.answer([frames[c] for c in range(64)], methods[0])
        assert rr == 64
        for b in (128, 1024):
            assert np.array_equal(first[b], rout), b
        ref.close()
