"""The oracle restatement (oracle/alto_oracle.c) pinned against the reference engine's own outputs: the golden
fixtures of tests/golden/ (produced by src/amx_kernels.cpp compiled unchanged) and, when this host can run it, the
reference engine itself."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, sha
import frames as fr


def test_oracle_matches_golden_small(golden, oracle, svc):
    g = golden["cases"]["small"]
    p = svc.params(g["rows"], g["record_bytes"])
    st = svc.SyntheticState.make(p, seed=g["state_seed"], full_prefix=g["full_prefix"])
    req = svc.synthetic_requests(p, g["b"], seed=g["request_seed"])
    r, status, out = oracle.answer(st, [req[i] for i in range(g["b"])])
    assert r == g["b"] and list(status) == g["status"]
    assert [sha(out[i]) for i in range(g["b"])] == g["sha256"]
    full = np.fromfile(os.path.join(GOLDEN_DIR, "resp_small_0.bin"), dtype=np.uint8)
    assert np.array_equal(out[0], full)


def test_oracle_malformed_and_mutated_statuses(golden, oracle, svc):
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=3, full_prefix=True)
    g = golden["cases"]["malformed"]
    r0 = svc.synthetic_requests(p, 1, seed=g["request_seed"], first_client=0)[0]
    r1 = svc.synthetic_requests(p, 1, seed=g["request_seed"], first_client=1)[0]
    mf, want = fr.malformed_table(r0, r1, p.count)
    assert want == g["status"]
    arena = np.full((len(mf), st.p.instances * st.prefixes[0].size), 0xA5, dtype=np.uint8)
    r, status, out = oracle.answer(st, mf, out=arena)
    assert r == 2 and list(status) == want
    assert all((arena[c] == 0xA5).all() for c in range(1, 7))
    assert [sha(arena[0]), sha(arena[7])] == g["sha256_valid"]
    # the decoder agrees with every status (src/service.rs:200-225)
    for f, s in zip(mf, want):
        try:
            svc.decode_request(p, f)
            ok = True
        except ValueError:
            ok = False
        assert ok == (s == 0)
    gm = golden["cases"]["mutated"]
    base = [svc.synthetic_requests(p, 1, seed=gm["request_seed"], first_client=i)[0] for i in range(4)]
    accepted = 0
    for batch, want_status in zip(fr.mutated_batches(base, p.count), gm["status"]):
        got = [oracle.validate(f, p.count, p.rows) for f in batch]
        assert got == want_status
        accepted += sum(s == 0 for s in got)
    assert 0 < accepted < 512


@pytest.mark.slow
def test_oracle_matches_golden_multiblock(golden, oracle, svc):
    g = golden["cases"]["multiblock"]
    p = svc.params(g["rows"], g["record_bytes"])
    st = svc.SyntheticState.make(p, seed=g["state_seed"])
    for b in ("1", "2", "72"):
        req = svc.synthetic_requests(p, int(b), seed=g["batches"][b]["request_seed"])
        r, status, out = oracle.answer(st, [req[i] for i in range(int(b))])
        assert r == int(b) and sha(out) == g["batches"][b]["sha256"], b


def test_oracle_matches_golden_plain_32k(golden, oracle, svc):
    g = golden["cases"]["plain_2048x32k"]
    p = svc.params(g["rows"], g["record_bytes"])
    st = svc.SyntheticState.make(p, seed=g["state_seed"])
    req = svc.synthetic_requests(p, 1, seed=g["request_seed"])
    r, status, out = oracle.answer(st, [req[0]])
    assert r == 1 and sha(out) == g["sha256"]


def _pack_inputs(g, svc):
    n, tg, rho, it = g["n"], g["tg"], g["rho"], g["num_iter"]
    bt = [svc.uniform_u64(it * tg * n, 1 << 32, s) << np.uint64(g["bold_t_shift"]) for s in g["bold_t_seeds"]]
    btb = [svc.uniform_u64(it * tg * n, 1 << 32, s) << np.uint64(g["bold_t_bar_shift"]) for s in g["bold_t_bar_seeds"]]
    tables = svc.uniform_u32(n * n, n, g["tables_seed"])
    gen_pows = np.array([pow(5, i, 2 * n) for i in range(it)], dtype=np.uint32)
    return bt, btb, tables, gen_pows


def test_pack_build_matches_golden(golden, oracle, svc, eng):
    g = golden["cases"]["pack_build"]
    bt, btb, tables, gen_pows = _pack_inputs(g, svc)
    n, tg, rho, it = g["n"], g["tg"], g["rho"], g["num_iter"]
    U = oracle.pack_build(bt, btb, tables, gen_pows, it, tg, n)
    assert sha(U) == g["sha256_values"]
    # the engine's own sw_pack_build: same values in its (col, plane)-interleaved layout
    ub = np.zeros(4 * tg * n * rho * n, dtype=np.int8)
    eng.build_packing_matrix(ub, bt, btb, tables, gen_pows, it, tg, n, threads=2)
    planes = ub.view(np.uint8).reshape(rho * n, 4, tg * n).astype(np.uint32)
    mine = planes[:, 0] | (planes[:, 1] << 8) | (planes[:, 2] << 16) | (planes[:, 3] << 24)
    assert np.array_equal(mine, U)


def test_oracle_rescale_integer_equals_double_exhaustively(oracle):
    # every v in [0, Q) for the scheme's q1 = 2^10 (src/amx_kernels.cpp:526-529 uses doubles; the oracle and the
    # engine use integer division)
    Q = 4294955009
    assert oracle.rescale_mismatches(0, Q, 1 << 10) == 0
    # other moduli accepted by the engine (q1 < 2^21), on a strided sample
    for q1 in (3, 1000, (1 << 20) + 7, (1 << 21) - 1):
        for v0 in range(0, Q, Q // 16):
            assert oracle.rescale_mismatches(v0, min(v0 + 200000, Q), q1) == 0


def test_engine_rescale_arithmetic_matches_oracle_exhaustively(oracle):
    # the tail kernel's division-free rescale (modq.cuh, compiled for the host here) against the oracle's plain
    # integer division, over every v in [0, Q) for q1 = 2^10 and strided ranges for other q1 < 2^21
    import altopir_b200 as pkg
    L = pkg.lib()
    Q = 4294955009
    assert L.alto_rescale_digest(1 << 10, 0, Q, 0) == oracle.rescale_digest(0, Q, 1 << 10)
    for q1 in (1, 3, 1000, (1 << 20) + 7, (1 << 21) - 1):
        for v0 in (0, Q // 2 - 100000, Q - 200000):
            assert L.alto_rescale_digest(q1, v0, v0 + 200000, 0) == oracle.rescale_digest(v0, v0 + 200000, q1)


def test_synthetic_record_three_ways(oracle, svc):
    for row in (0, 1, 977, 2047, 123456):
        a = svc.synthetic_record(row, 4096)
        b = oracle.synthetic_record(row, 4096)
        assert np.array_equal(a, b)
    db = svc.synthetic_db_col(512, 64, col0=100)
    db2 = oracle.synthetic_db_col(512, 100, 64)
    assert np.array_equal(db, db2)
    rec = oracle.synthetic_record(511, 4096)
    assert np.array_equal(db[:, 511], rec[100:164])


def test_reference_engine_agrees_when_available(oracle, svc):
    from oracle.oracle import RefEngine, ref_methods
    methods = ref_methods()
    if not methods:
        pytest.skip("the reference engine cannot run on this host CPU")
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=41, full_prefix=True)
    req = svc.synthetic_requests(p, 9, seed=42)
    frames_ = [req[i] for i in range(9)]
    r, status, out = oracle.answer(st, frames_)
    ref = RefEngine(st)
    for m in methods:
        rr, rs, rout, _ = ref.answer(frames_, m)
        assert rr == r and np.array_equal(rs, status) and np.array_equal(rout, out)


def test_pack_build_at_the_scheme_shape_matches_oracle(oracle, svc, eng):
    # n = 2048, tg = 4 and the scheme's n/2 - 1 automorphisms, with 64-bit sums that wrap
    n, tg, rho = 2048, 4, 2
    it = n // 2 - 1
    bt = [svc.uniform_u64(it * tg * n, 1 << 32, 900 + o) << np.uint64(31) for o in range(rho)]
    btb = [svc.uniform_u64(it * tg * n, 1 << 32, 950 + o) << np.uint64(30) for o in range(rho)]
    tables = svc.uniform_u32(n * n, n, 990)
    gen_pows = np.array([pow(5, i, 2 * n) for i in range(it)], dtype=np.uint32)
    ub = np.zeros(4 * tg * n * rho * n, dtype=np.int8)
    eng.build_packing_matrix(ub, bt, btb, tables, gen_pows, it, tg, n, threads=4)
    planes = ub.view(np.uint8).reshape(rho * n, 4, tg * n).astype(np.uint32)
    mine = planes[:, 0] | (planes[:, 1] << 8) | (planes[:, 2] << 16) | (planes[:, 3] << 24)
    assert np.array_equal(mine, oracle.pack_build(bt, btb, tables, gen_pows, it, tg, n))


def test_oracle_state_and_frames_equal_the_engine_generators(oracle, svc):
    """The benchmark's reference arm builds its state and frames with the oracle's generators (it must not load the
    engine library); they give the bytes of the engine package's generators that the GPU arm uses."""
    from oracle.oracle import Params, State
    for rows, rb, seed in ((2048, 4096, 1), (4096, 8192, 5)):
        p = svc.params(rows, rb)
        st = svc.SyntheticState.make(p, seed=seed, keep_values=True)
        po = Params(rows, rb)
        assert (po.part_len, po.row1_off, po.count, po.instances) == (p.part_len, p.row1_off, p.count, p.instances)
        so = State(po, seed=seed, oracle=oracle)
        assert np.array_equal(so.db_col, st.db_col)
        assert np.array_equal(so.U, st.U)
        assert all(np.array_equal(a, b) for a, b in zip(so.that, st.that))
        assert all(np.array_equal(a, b) for a, b in zip(so.prefixes, st.prefixes))
        assert np.array_equal(so.inv_table, st.inv_table)
        assert np.array_equal(oracle.synthetic_requests(po, 3, seed=1000, first_client=2),
                              svc.synthetic_requests(p, 3, seed=1000, first_client=2))


def test_oracle_hint_ring_is_the_negacyclic_product_of_the_reference(oracle):
    """orc_hint_ring against a direct restatement of src/server.rs:656-768 at toy sizes: each query polynomial goes
    through util.rs negacyclic_perm (shift 0), is multiplied by the column's polynomial modulo X^n + 1 and Q, and the
    products are summed over the column's polynomials (then negacyclic_perm again when perm_out)."""
    Q = 4294955009
    rng = np.random.default_rng(7)

    def negacyclic_perm(a):  # util.rs:5-21, shift 0
        n = len(a)
        return [a[0] % Q] + [(Q - a[n - i] % Q) % Q for i in range(1, n)]

    def mul(a, b):  # product modulo X^n + 1
        n = len(a)
        out = [0] * n
        for i in range(n):
            for j in range(n):
                if i + j < n:
                    out[i + j] += a[i] * b[j]
                else:
                    out[i + j - n] -= a[i] * b[j]
        return [x % Q for x in out]

    for n, rows, cols, perm_out in ((8, 32, 5, False), (16, 32, 3, True), (4, 4, 2, False)):
        db = rng.integers(0, 256, (cols, rows), dtype=np.uint8)
        query = rng.integers(0, 1 << 63, (rows // n, n), dtype=np.uint64)
        want = np.zeros((n, cols), dtype=np.uint64)
        for c in range(cols):
            acc = [0] * n
            for r in range(rows // n):
                prod = mul(negacyclic_perm([int(x) for x in query[r]]), [int(x) for x in db[c, r * n:(r + 1) * n]])
                acc = [(x + y) % Q for x, y in zip(acc, prod)]
            if perm_out:
                acc = negacyclic_perm(acc)
            want[:, c] = acc
        assert np.array_equal(oracle.hint_ring(db, query, n, 0, cols, perm_out), want), (n, rows, cols)
        assert np.array_equal(oracle.hint_ring(db, query, n, 1, cols, perm_out), want[:, 1:])
