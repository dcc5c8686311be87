"""alto_answer_device_noalloc: answering device-resident frames without allocating device memory.

Some callers cannot call cudaMalloc while they serve: a server that reserves all of its GPU memory at start-up and
must never grow it, code that runs under a memory budget kept by an allocator it does not own, or a latency-critical
thread that cannot afford cudaMalloc's device-wide synchronisation.  This entry point keeps its per-batch scratch in
a fixed 16 MiB array inside the library instead of engine buffers grown on demand.  The test checks, through the C
ABI, that it returns exactly what alto_answer_device returns for the same frames on two calls in a row, that free
device memory does not change across a further call, and that a batch too large for the array is refused.

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
