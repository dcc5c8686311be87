"""The C-ABI library without a GPU: it loads, exports every symbol include/altopir_gpu.h declares, and rejects the
configurations the reference rejects before touching the device (src/amx_kernels.cpp:551-552)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "altopir_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b([a-z_0-9]+)\s*\(", text)) - {"if", "sizeof"}


def test_library_loads_and_exports_header_symbols():
    import altopir_b200 as pkg
    L = pkg.lib()
    declared = header_symbols()
    assert declared == set(pkg.EXPORTS), declared ^ set(pkg.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared - exported
    assert not missing, missing
    for name in declared:
        assert getattr(L, name) is not None


def test_reference_abi_signatures_match_engine_rs():
    # the extern "C" block of the reference binding (src/engine.rs:4-20), restated: symbol -> parameter count
    expected = {"sw_amx_init": 0, "sw_alloc_zeroed": 1, "sw_alloc": 1, "sw_free": 1, "sw_tile_db": 6,
                "sw_pack_build": 11, "alto_engine_new": 17, "alto_engine_free": 1, "alto_request_len": 1,
                "alto_response_len": 1, "alto_answer": 8}
    text = open(os.path.join(ROOT, "include", "altopir_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    for name, nparams in expected.items():
        m = re.search(r"\b" + name + r"\s*\(([^)]*)\)", text)
        assert m, name
        params = [p for p in m.group(1).split(",") if p.strip() and p.strip() != "void"]
        assert len(params) == nparams, (name, params)


def test_host_allocator_and_tile_db():
    import altopir_b200 as pkg
    L = pkg.lib()
    p = L.sw_alloc_zeroed(3 << 20)
    assert p and p % (2 << 20) == 0
    buf = (ctypes.c_uint8 * (3 << 20)).from_address(p)
    assert max(buf) == 0
    L.sw_free(p)
    L.sw_free(None)
    rows, cols, ld = 128, 64, 192
    db = np.random.default_rng(1).integers(0, 256, (cols, ld), dtype=np.uint8)
    out = np.zeros(rows * cols, dtype=np.uint8)
    L.sw_tile_db(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(db.ctypes.data), ld, rows, cols, 2)
    assert np.array_equal(out.reshape(cols, rows), db[:, :rows])


@pytest.mark.parametrize("bad", ["q", "n0", "n_big", "n16", "cols_n", "rows64", "cols32", "threads", "tgn", "null"])
def test_engine_new_rejects_reference_invalid_configs(bad, svc):
    import altopir_b200 as pkg
    L = pkg.lib()
    rows, cols, n, tg, q, threads = 2048, 4096, 2048, 4, svc.Q, 1
    if bad == "q":
        q = svc.Q + 2
    elif bad == "n0":
        n = 0
    elif bad == "n_big":
        n, cols = 8192, 8192
    elif bad == "n16":
        n = 2056
    elif bad == "cols_n":
        cols = 4096 + 32
    elif bad == "rows64":
        rows = 2048 + 32
    elif bad == "cols32":
        n, cols = 16, 4096 + 16
    elif bad == "threads":
        threads = 0
    elif bad == "tgn":
        n, tg = 16, 1  # (tg * n) % 128 != 0
    dummy = np.zeros(64, dtype=np.uint8)
    ptr = ctypes.c_void_p(dummy.ctypes.data)
    arr = (ctypes.c_void_p * 4)(*([dummy.ctypes.data] * 4))
    null = bad == "null"
    e = L.alto_engine_new(None if null else ptr, ptr, rows, rows, cols, ptr, n, tg, arr, 64, 0, 1024, 10, arr, ptr,
                          q, threads)
    assert not e
    assert pkg.last_error()


def test_service_codec_roundtrip(svc):
    p = svc.params(2048, 4096)
    rng = np.random.default_rng(5)
    y = rng.integers(0, svc.Q, p.count, dtype=np.uint64)
    z = rng.integers(0, svc.Q, p.count, dtype=np.uint64)
    q = rng.integers(0, 1 << 32, p.rows, dtype=np.uint64)
    f = svc.encode_request(p, y, z, q)
    assert f.size == svc.request_len(p) == 9 + 4 * (2 * 4 * 2048 + 2048)
    y2, z2, q2 = svc.decode_request(p, f)
    assert np.array_equal(y2, y) and np.array_equal(z2, z) and np.array_equal(q2, q)
    assert svc.response_len(p) == 2 * 7168 and p.part_len == 7168 and p.row1_off == 36864 and p.q1_bits == 10
    with pytest.raises(ValueError):
        svc.params(3000, 4096)
    with pytest.raises(ValueError):
        svc.params(2048, 4000)
    # synthetic requests are well formed
    fr = svc.synthetic_requests(p, 3, seed=1)
    for i in range(3):
        svc.decode_request(p, fr[i])


def test_ingest_entry_points_reject_bad_arguments_without_a_device(svc):
    # alto_engine_new_empty checks the configuration like alto_engine_new before any CUDA call; the loaders reject a
    # NULL engine
    import altopir_b200 as pkg
    L = pkg.lib()
    dummy = np.zeros(64, dtype=np.uint8)
    ptr = ctypes.c_void_p(dummy.ctypes.data)
    arr = (ctypes.c_void_p * 4)(*([dummy.ctypes.data] * 4))
    for rows, cols, n, q in ((2048, 4096, 2048, svc.Q + 2), (2048 + 32, 4096, 2048, svc.Q), (2048, 4096 + 32, 2048,
                                                                                              svc.Q)):
        assert not L.alto_engine_new_empty(rows, cols, ptr, n, 4, arr, 64, 0, 1024, 10, arr, ptr, q, 1)
        assert pkg.last_error()
    assert L.alto_engine_load_records(None, ptr, 4096, 0, 1) == -1
    assert L.alto_engine_load_file(None, b"/nonexistent", 0) == -1


def test_lane_entry_points_reject_a_null_engine_without_a_device():
    import altopir_b200 as pkg
    L = pkg.lib()
    assert L.alto_engine_set_lanes(None, 2) == -1
    assert L.alto_engine_fence(None) == -1
    assert L.alto_engine_sync(None) == -1
