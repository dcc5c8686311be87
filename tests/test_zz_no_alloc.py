"""alto_answer_device_noalloc: answering device-resident frames without allocating device memory.

Some callers cannot call cudaMalloc while they serve: a server that reserves all of its GPU memory at start-up and
must never grow it, code that runs under a memory budget kept by an allocator it does not own, or a latency-critical
thread that cannot afford cudaMalloc's device-wide synchronisation.  This entry point keeps its per-batch scratch in
a fixed 16 MiB array inside the library instead of engine buffers grown on demand.  The test checks, through the C
ABI, that it returns exactly what alto_answer_device returns for the same frames on two calls in a row (for the
CTA-pair GEMM plan, the single-CTA plan of batches of at most four frames, and a database of several 32768-record
chunks), that free device memory does not change across a further call, that the launch count is reported, and
that the batch limit the header documents as a formula is the one the library applies.

This file is collected last so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_answer_device_on_two_calls_in_a_row(gpu, svc, eng):
    import torch
    import altopir_b200 as pkg

    L = pkg.lib()
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=61, full_prefix=True)
    e = eng.Engine.from_state(st)
    b = 6
    frames = svc.synthetic_requests(p, b, seed=62)
    ql, rl = e.request_len(), e.response_len()
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
    slots[3, 7 + 9:7 + 13] = 0xFF  # first y key word of frame 3 >= Q: status 3, its output must stay untouched

    # the existing entry point
    want = torch.full((b, rl), 0x5A, dtype=torch.uint8, device="cuda")
    want_status = np.full(b, -1, dtype=np.int32)
    torch.cuda.synchronize()  # the engine's stream does not wait on torch's
    r = e.answer_device(slots.data_ptr(), stride, b, want.data_ptr(), rl, want_status)
    assert r == b - 1 and list(want_status) == [0, 0, 0, 3, 0, 0]

    d_status = torch.full((b,), -1, dtype=torch.int32, device="cuda")

    def call(out):
        return L.alto_answer_device_noalloc(e.ptr, ctypes.c_void_p(slots.data_ptr()), stride, b,
                                            ctypes.c_void_p(out.data_ptr()), rl, ctypes.c_void_p(d_status.data_ptr()))

    for _ in range(2):
        got = torch.full((b, rl), 0x5A, dtype=torch.uint8, device="cuda")
        d_status.fill_(-1)
        torch.cuda.synchronize()
        rc = call(got)
        assert rc == 0, pkg.last_error()
        assert torch.equal(got, want)
        assert d_status.cpu().numpy().tolist() == want_status.tolist()

    # a further call allocates nothing: free device memory is unchanged
    got = torch.full((b, rl), 0x5A, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    assert call(got) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    assert torch.equal(got, want)

    # a batch whose scratch exceeds the fixed array is refused before any work (buffers sized for it regardless)
    big = 256
    big_slots = torch.zeros((big, stride), dtype=torch.uint8, device="cuda")
    big_out = torch.zeros((big, rl), dtype=torch.uint8, device="cuda")
    big_status = torch.zeros((big,), dtype=torch.int32, device="cuda")
    rc = L.alto_answer_device_noalloc(e.ptr, ctypes.c_void_p(big_slots.data_ptr()), stride, big,
                                      ctypes.c_void_p(big_out.data_ptr()), rl, ctypes.c_void_p(big_status.data_ptr()))
    assert rc == -1 and "scratch" in pkg.last_error()
    e.close()


SCRATCH_BYTES = 16 << 20


def _r256(x):
    return (x + 255) // 256 * 256


def noalloc_bytes(rows, cols, count, b):
    """The scratch a batch of b frames needs, as the header states it."""
    b4 = (b + 3) // 4 * 4
    r = rows if rows <= 32768 else (rows + 32767) // 32768 * 32768
    return _r256(4 * b) + _r256(4 * b4 * r) + _r256(4 * b4 * count) + 2 * _r256(4 * b * cols)


def max_batch(rows, cols, count):
    b = 0
    while noalloc_bytes(rows, cols, count, b + 1) <= SCRATCH_BYTES:
        b += 1
    return b


def _noalloc(L, e, slots, stride, b, out, rl, d_status):
    return L.alto_answer_device_noalloc(e.ptr, ctypes.c_void_p(slots.data_ptr()), stride, b,
                                        ctypes.c_void_p(out.data_ptr()), rl, ctypes.c_void_p(d_status.data_ptr()))


@pytest.mark.parametrize("rows,record_bytes,b", [(2048, 4096, 1), (2048, 4096, 4), (65536, 4096, 6)])
def test_noalloc_other_plans_match_answer_device(gpu, svc, eng, rows, record_bytes, b):
    """b <= 4 runs the single-CTA GEMMs; 65536 records make two record chunks of the query limbs.  Both carve their
    scratch from the array at other offsets than the CTA-pair plan with one chunk."""
    import torch
    import altopir_b200 as pkg
    L = pkg.lib()
    p = svc.Params(rows, record_bytes)
    st = svc.SyntheticState.make(p, seed=71)
    e = eng.Engine.from_state(st)
    ql, rl = e.request_len(), e.response_len()
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    svc.synthetic_requests_device(p, b, 72, slots.data_ptr(), stride)
    want = torch.full((b, rl), 0x5A, dtype=torch.uint8, device="cuda")
    want_status = np.full(b, -1, dtype=np.int32)
    assert e.answer_device(slots.data_ptr(), stride, b, want.data_ptr(), rl, want_status) == b
    d_status = torch.full((b,), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        got = torch.full((b, rl), 0x5A, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(L, e, slots, stride, b, got, rl, d_status) == 0, pkg.last_error()
        assert torch.equal(got, want) and (d_status == 0).all().item()
        assert e.last_launches() == 6
    e.close()


def test_noalloc_batch_limit_follows_the_documented_formula(gpu, svc, eng):
    """The header's formula gives 38 frames at 32768 records of 32 KB; on a small engine the library accepts the
    formula's largest batch and refuses one more frame."""
    import torch
    import altopir_b200 as pkg
    assert max_batch(32768, 32768, 8192) == 38
    L = pkg.lib()
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=73)
    e = eng.Engine.from_state(st)
    bmax = max_batch(p.rows, p.record_bytes, p.count)
    ql, rl = e.request_len(), e.response_len()
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((bmax + 1, stride), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    svc.synthetic_requests_device(p, bmax + 1, 74, slots.data_ptr(), stride)
    out = torch.zeros((bmax + 1, rl), dtype=torch.uint8, device="cuda")
    d_status = torch.full((bmax + 1,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(L, e, slots, stride, bmax, out, rl, d_status) == 0, pkg.last_error()
    assert (d_status[:bmax] == 0).all().item()
    assert _noalloc(L, e, slots, stride, bmax + 1, out, rl, d_status) == -1 and "scratch" in pkg.last_error()
    e.close()
