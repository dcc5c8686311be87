"""Generates tests/golden/golden.json (and resp_small_0.bin) by running the REFERENCE engine -- src/amx_kernels.cpp
compiled unchanged from the reference tree into oracle/_ref/ -- on seeded synthetic state and seeded requests.

The fixtures pin both the oracle restatement (CPU tests) and the CUDA engine (GPU tests) to the reference's own
outputs.  Inputs are regenerated from the seeds recorded here by altopir_b200.service (splitmix64 streams), so only
hashes, statuses and one full response are stored.  Run from the repository root where the reference tree and an
AVX-512 + AMX host CPU are available:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import __graft_entry__ as ge  # noqa: E402

ge.load()
from altopir_b200 import service as svc  # noqa: E402
from oracle import oracle as orc  # noqa: E402
import frames as fr  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run(ref, frames_, method):
    r, status, out, _ = ref.answer(frames_, method)
    return r, status, out


def main():
    orc.build()
    methods = orc.ref_methods()
    assert methods, "the reference engine needs an AVX-512 host and oracle/_ref/libalto_ref.so"
    m0 = methods[0]
    golden = {"generator": "reference src/amx_kernels.cpp via oracle/_ref", "methods_checked": methods, "cases": {}}

    # --- small: 2048 records x 4 KB (the reference tests' size, tests/engine.rs:10-11), random full prefixes
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=3, full_prefix=True)
    ref = orc.RefEngine(st)
    req = svc.synthetic_requests(p, 5, seed=9)
    frames_ = [req[i] for i in range(5)]
    outs = []
    for m in methods:
        r, status, out = run(ref, frames_, m)
        assert r == 5 and (status == 0).all()
        outs.append(out)
    assert all(np.array_equal(outs[0], o) for o in outs)
    golden["cases"]["small"] = {"rows": 2048, "record_bytes": 4096, "state_seed": 3, "full_prefix": True,
                                "request_seed": 9, "b": 5, "status": [0] * 5,
                                "sha256": [sha(outs[0][i]) for i in range(5)]}
    outs[0][0].tofile(os.path.join(HERE, "resp_small_0.bin"))

    # --- malformed frames (tests/engine.rs:128-168)
    r0 = svc.synthetic_requests(p, 1, seed=21, first_client=0)[0]
    r1 = svc.synthetic_requests(p, 1, seed=21, first_client=1)[0]
    mf, want = fr.malformed_table(r0, r1, p.count)
    rl = ref.response_len()
    arena = np.full((len(mf), rl), 0xA5, dtype=np.uint8)
    status = np.full(len(mf), -1, dtype=np.int32)
    r, status, out, _ = ref.answer(mf, m0, out=arena, status=status)
    assert r == 2 and list(status) == want
    assert all((arena[c] == 0xA5).all() for c in range(1, 7))
    golden["cases"]["malformed"] = {"request_seed": 21, "status": [int(s) for s in status],
                                    "sha256_valid": [sha(arena[0]), sha(arena[7])]}

    # --- mutated frames (tests/engine.rs:170-193): statuses from the reference engine
    base = [svc.synthetic_requests(p, 1, seed=33, first_client=i)[0] for i in range(4)]
    statuses = []
    for batch in fr.mutated_batches(base, p.count):
        r, status, out, _ = ref.answer(batch, m0)
        statuses.append([int(s) for s in status])
    golden["cases"]["mutated"] = {"request_seed": 33, "status": statuses}
    ref.close()

    # --- multi-block and chunked batches (tests/engine.rs:196-245): 8192 records x 4 KB
    p8 = svc.params(8192, 4096)
    st8 = svc.SyntheticState.make(p8, seed=5)
    ref8 = orc.RefEngine(st8)
    mb = {}
    for b in (1, 2, 72, 136):
        req = svc.synthetic_requests(p8, b, seed=1000 + b)
        frames_ = [req[i] for i in range(b)]
        res = [run(ref8, frames_, m) for m in methods]
        assert all(r == b for r, _, _ in res) and all(np.array_equal(res[0][2], o) for _, _, o in res)
        mb[str(b)] = {"request_seed": 1000 + b, "sha256": sha(res[0][2])}
    golden["cases"]["multiblock"] = {"rows": 8192, "record_bytes": 4096, "state_seed": 5, "batches": mb}
    ref8.close()

    # --- plain method, small (configs: 2048 records x 32 KB, one query)
    p1 = svc.params(2048, 32768)
    st1 = svc.SyntheticState.make(p1, seed=1)
    ref1 = orc.RefEngine(st1)
    req = svc.synthetic_requests(p1, 1, seed=77)
    res = [run(ref1, [req[0]], m) for m in methods]
    assert all(r == 1 for r, _, _ in res) and all(np.array_equal(res[0][2], o) for _, _, o in res)
    golden["cases"]["plain_2048x32k"] = {"rows": 2048, "record_bytes": 32768, "state_seed": 1, "request_seed": 77,
                                         "sha256": sha(res[0][2])}
    ref1.close()

    # --- packing-matrix build (src/amx_kernels.cpp:311-341) at n = 32, tg = 4, rho = 2, with 64-bit wrap-around
    n, tg, rho = 32, 4, 2
    num_iter = n // 2 - 1
    bold_t = [svc.uniform_u64(num_iter * tg * n, 1 << 32, 500 + o) << np.uint64(30) for o in range(rho)]
    bold_tb = [svc.uniform_u64(num_iter * tg * n, 1 << 32, 600 + o) << np.uint64(31) for o in range(rho)]
    tables = svc.uniform_u32(n * n, n, 700)
    gen_pows = np.array([pow(5, i, 2 * n) for i in range(num_iter)], dtype=np.uint32)
    import ctypes
    L = ctypes.CDLL(orc.REF_SO)
    ub = np.zeros(4 * tg * n * rho * n, dtype=np.int8)
    pp = (ctypes.c_void_p * rho)(*[a.ctypes.data for a in bold_t])
    pb = (ctypes.c_void_p * rho)(*[a.ctypes.data for a in bold_tb])
    L.sw_pack_build.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint64,
                                ctypes.c_int]
    L.sw_pack_build(ub.ctypes.data, pp, pb, tables.ctypes.data, gen_pows.ctypes.data, num_iter, tg, n, rho, svc.Q, 2)
    U = orc.ref_ub_values(ub, rho * n, tg * n)
    golden["cases"]["pack_build"] = {"n": n, "tg": tg, "rho": rho, "num_iter": num_iter,
                                     "bold_t_seeds": [500, 501], "bold_t_shift": 30,
                                     "bold_t_bar_seeds": [600, 601], "bold_t_bar_shift": 31,
                                     "tables_seed": 700, "gen_pows": "5^i mod 2n", "sha256_values": sha(U)}

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
