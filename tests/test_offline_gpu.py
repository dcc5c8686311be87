"""The scheme's offline set-up on the device (alto_engine_offline: hint, InspiRING precomputation, packing matrix,
bold_t_hat, prefixes) against the oracle's numpy restatement, and decryption round trips through this engine:
requests of the client restatement, answered on the GPU, decrypt to the records asked for (the check
tests/engine.rs makes of the reference)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clients(client_mod, p, idx, seed0):
    clients = [client_mod.Client(p, seed=seed0 + k) for k in range(len(idx))]
    return clients, [c.request(i) for c, i in zip(clients, idx)]


def _answer(e, frames):
    b = len(frames)
    out = np.zeros((b, e.response_len()), dtype=np.uint8)
    status = np.full(b, -1, dtype=np.int32)
    r, _ = e.answer(frames, out, status)
    assert r == b and list(status) == [0] * b
    return out


def test_engine_over_the_oracle_scheme_state_decrypts(gpu, eng, client_mod, oracle, scheme_state):
    """The engine alone, given the oracle's scheme state (packing matrix from this library's sw_pack_build)."""
    st, p = scheme_state, scheme_state.p
    ub = np.empty(4 * p.record_bytes * p.count, dtype=np.int8)
    eng.build_packing_matrix(ub, st.bold_t, st.bold_t_bar, st.tables, st.gen_pows, p.n // 2 - 1, p.tg, p.n)
    tiled = eng.TiledDb(st.db_col, st.db_col.shape[1], p.rows, p.record_bytes)
    e = eng.Engine(st.db_col, tiled, st.db_col.shape[1], ub, p.n, p.tg, st.prefixes, p.row1_off, 1 << p.q1_bits,
                   p.q1_bits, st.that, st.inv_table)
    try:
        idx = [3, 999, p.rows - 1]
        clients, frames = _clients(client_mod, p, idx, 40)
        out = _answer(e, frames)
        _, _, want = oracle.answer(st, frames)
        assert np.array_equal(out, want)
        for c, resp, i in zip(clients, out, idx):
            assert np.array_equal(c.decrypt(resp), oracle.synthetic_record(i, p.record_bytes))
    finally:
        e.close()


@pytest.mark.parametrize("variant", [{}, {"ALTO_OFFLINE_WALK8": "0"},
                                     {"ALTO_OFFLINE_CLUSTER": "1", "ALTO_OFFLINE_ACT8": "0"}],
                         ids=["register-walk", "cluster-walk", "single-cta-walk"])
def test_device_offline_matches_the_oracle_restatement(gpu, client_mod, oracle, scheme_state, variant, monkeypatch):
    """Every kernel variant of the set-up (the walk with register transforms on a 4-CTA cluster, the walk with
    shared-memory transforms on a cluster, the single-CTA walk with the shared-memory hint transforms) gives the
    oracle's values bit for bit."""
    from altopir_b200 import offline
    for k, v in variant.items():
        monkeypatch.setenv(k, v)
    st, p = scheme_state, scheme_state.p
    e = offline.blank_engine(p, st.db_col)
    try:
        ms, out = offline.prepare(e, p, want=True)
        assert ms > 0
        assert np.array_equal(out["bold_t"][0].astype(np.uint64), st.bold_t[0])
        assert np.array_equal(out["bold_t_bar"][0].astype(np.uint64), st.bold_t_bar[0])
        assert np.array_equal(out["that"][0].astype(np.uint64), st.that[0])
        assert np.array_equal(out["a_hat"][0].astype(np.uint64), st.a_hat[0])
        idx = [0, 1500, 2047]
        clients, frames = _clients(client_mod, p, idx, 50)
        got = _answer(e, frames)
        _, _, want = oracle.answer(st, frames)
        assert np.array_equal(got, want)          # packing matrix, bold_t_hat, prefixes and table as the oracle's
        for c, resp, i in zip(clients, got, idx):
            assert np.array_equal(c.decrypt(resp), oracle.synthetic_record(i, p.record_bytes))
    finally:
        e.close()


@pytest.mark.parametrize("rows,record_bytes", [(32768, 4096), (32768, 32768)])
def test_device_offline_round_trip(gpu, client_mod, svc, rows, record_bytes):
    """A database of synthetic records generated on the device, its scheme state built on the device, answered in
    one batch: every response decrypts to its record (1 GiB at the second size)."""
    from altopir_b200 import offline
    p = svc.params(rows, record_bytes)
    e, ms = offline.scheme_engine(p)
    try:
        idx = [0, 12345, rows // 2 + 7, rows - 1]
        clients, frames = _clients(client_mod, p, idx, 60)
        out = _answer(e, frames)
        for c, resp, i in zip(clients, out, idx):
            assert np.array_equal(c.decrypt(resp), svc.synthetic_record(i, record_bytes))
        print(f"offline set-up of {rows} x {record_bytes} B on the device: {ms:.1f} ms")
    finally:
        e.close()


def test_device_offline_rejects_bad_arguments(gpu, svc):
    import ctypes
    from altopir_b200 import lib, offline
    p = svc.params(2048, 2048)
    e = offline.blank_engine(p, np.zeros((p.record_bytes, p.rows), dtype=np.uint8))
    try:
        q, w, v = offline.public_inputs(p)
        assert lib().alto_engine_offline(e.ptr, None, w.ctypes.data, v.ctypes.data, None, None, None, None,
                                         None) == -1
        assert lib().alto_engine_offline(None, q.ctypes.data, w.ctypes.data, v.ctypes.data, None, None, None, None,
                                         None) == -1
        assert "bad arguments" in lib().alto_last_error().decode()
        ms = ctypes.c_double(-1.0)
        assert lib().alto_engine_offline(e.ptr, q.ctypes.data, w.ctypes.data, v.ctypes.data, None, None, None, None,
                                         ctypes.byref(ms)) == 0 and ms.value > 0
    finally:
        e.close()


def test_serving_loop_answers_the_scheme(gpu, client_mod, svc):
    """The serving loop over an engine with the scheme's state: six clients each send two requests with the same
    packing keys (the second is answered from the resident per-client table, without the pack), and every response
    decrypts to its record."""
    from altopir_b200 import offline, server as srv
    p = svc.params(32768, 4096)
    e, _ = offline.scheme_engine(p)
    s = srv.Server(e, max_batch=8, queue_cap=64, slots=2)
    try:
        clients = [client_mod.Client(p, seed=70 + k) for k in range(6)]
        keys = [c.packing_keys() for c in clients]
        asks = [(k, (977 * k + 13 * r) % p.rows) for r in range(2) for k in range(6)]
        done = []
        for rnd in range(2):   # the second round's keys are resident by then
            tickets = [(k, i, s.submit(clients[k].request(i, keys[k]))) for k, i in asks[6 * rnd:6 * rnd + 6]]
            for k, i, t in tickets:
                assert t >= 0
                st, resp = s.wait(t, timeout_ms=30000)
                assert st == 0
                done.append((k, i, resp))
        for k, i, resp in done:
            assert np.array_equal(clients[k].decrypt(resp), svc.synthetic_record(i, p.record_bytes))
        stats = s.stats()
        assert stats["answered"] == 12 and stats["resident_hits"] >= 6
    finally:
        s.close()
        e.close()


@pytest.mark.parametrize("tg", [2, 8])
def test_device_offline_at_other_key_counts(gpu, client_mod, oracle, svc, tg):
    """tg = 2 and 8 gadget digits (17 and 5 bits; clusters of 2 and 8 CTAs in the walk) against the oracle bit for
    bit; at tg = 8 the responses also decrypt (at tg = 2 the 17-bit digits leave too little noise margin)."""
    from altopir_b200 import offline
    from oracle.scheme import SchemeState
    p = svc.Params(2048, 2048, tg=tg)
    st = SchemeState(p, oracle.synthetic_db_col(p.rows, 0, p.record_bytes), oracle)
    e = offline.blank_engine(p, st.db_col)
    try:
        _, out = offline.prepare(e, p, want=True)
        for k in ("bold_t", "bold_t_bar", "that"):
            assert np.array_equal(out[k][0].astype(np.uint64), getattr(st, k)[0]), k
        assert np.array_equal(out["a_hat"][0].astype(np.uint64), st.a_hat[0])
        idx = [5, 2000]
        clients, frames = _clients(client_mod, p, idx, 80)
        got = _answer(e, frames)
        _, _, want = oracle.answer(st, frames)
        assert np.array_equal(got, want)
        if tg == 8:
            for c, resp, i in zip(clients, got, idx):
                assert np.array_equal(c.decrypt(resp), oracle.synthetic_record(i, p.record_bytes))
    finally:
        e.close()


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["ref_methods"]).ref_methods(),
                    reason="the reference engine needs AVX-512 (and its library in oracle/_ref)")
def test_plain_small_config_against_the_reference_engine(gpu, eng, client_mod, oracle, svc):
    """The plain small configuration: 2,048 synthetic records x 32 KB (64 MiB), the scheme's state built on the device,
    one query of a seeded client; the GPU's response equals the reference engine's (src/amx_kernels.cpp compiled
    unchanged) over the same state byte for byte, and decrypts to the record."""
    from types import SimpleNamespace
    from altopir_b200 import offline
    from oracle.oracle import RefEngine, ref_methods
    from oracle.scheme import prefix_row0, Ring
    p = svc.params(2048, 32768)
    db = oracle.synthetic_db_col(p.rows, 0, p.record_bytes)
    e = offline.blank_engine(p, db)
    try:
        _, out = offline.prepare(e, p, want=True)
        ring = client_mod.Ring(p.n)
        tables = np.stack([Ring(p.n).table(t) for t in range(1, 2 * p.n, 2)]).astype(np.uint32)
        gen_pows = np.array([pow(5, i, 2 * p.n) for i in range(p.n)], dtype=np.uint32)
        bt = [np.ascontiguousarray(out["bold_t"][o], dtype=np.uint64) for o in range(p.instances)]
        btb = [np.ascontiguousarray(out["bold_t_bar"][o], dtype=np.uint64) for o in range(p.instances)]
        st = SimpleNamespace(
            p=p, db_col=db, U=oracle.pack_build(bt, btb, tables, gen_pows, p.n // 2 - 1, p.tg, p.n),
            that=[np.ascontiguousarray(out["that"][o], dtype=np.uint64) for o in range(p.instances)],
            prefixes=[prefix_row0(out["a_hat"][o].astype(np.uint64), p.part_len) for o in range(p.instances)],
            inv_table=client_mod.ntt_inverse_table(ring))
        c = client_mod.Client(p, seed=0x5EED)
        index = 1537
        frame = c.request(index)
        got = _answer(e, [frame])
        ref = RefEngine(st)
        try:
            r, status, want, _ = ref.answer([frame], ref_methods()[0])
        finally:
            ref.close()
        assert r == 1 and list(status) == [0]
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(c.decrypt(got[0]), svc.synthetic_record(index, p.record_bytes))
    finally:
        e.close()


def test_column_shards_build_their_own_scheme_state(gpu, client_mod, svc):
    """Column sharding with the scheme's state: each shard engine (a contiguous range of outputs) runs the device
    set-up over its own columns only; the shards' parts, concatenated in output order, equal the full engine's
    response byte for byte and decrypt to the record."""
    from altopir_b200 import offline
    p = svc.params(32768, 8192)                                   # 4 outputs
    full, _ = offline.scheme_engine(p)
    shards = []
    try:
        for c0, c1 in ((0, 2048), (2048, 8192)):                  # shards of 1 and 3 outputs
            ps = svc.Params(p.rows, c1 - c0)
            e, _ = offline.scheme_engine(ps, np.ascontiguousarray(svc.synthetic_db_col(p.rows, c1 - c0, col0=c0)))
            shards.append(e)
        c = client_mod.Client(p, seed=91)
        frame = c.request(30001)
        want = _answer(full, [frame])[0]
        got = np.concatenate([_answer(e, [frame])[0] for e in shards])
        assert np.array_equal(got, want)
        assert np.array_equal(c.decrypt(got), svc.synthetic_record(30001, p.record_bytes))
    finally:
        full.close()
        for e in shards:
            e.close()


def test_device_path_graphs_and_lanes_see_the_new_state(gpu, client_mod, svc):
    """Graphs captured and lanes made before the set-up replay over the state it writes in place: the engine answers
    device-resident frames of four clients through two lanes with graph replay, then runs alto_engine_offline, and
    the same replayed path now returns responses that decrypt (and equal alto_answer's)."""
    import torch
    from altopir_b200 import offline
    p = svc.params(32768, 4096)
    e = offline.blank_engine(p)
    try:
        idx = [3, 4096, 20000, 32767]
        clients, frames = _clients(client_mod, p, idx, 300)
        ql, rl, b = e.request_len(), e.response_len(), len(frames)
        stride = (7 + ql + 15) // 16 * 16
        slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(np.stack(frames)).cuda()
        e.set_graphs(True)
        e.set_lanes(2)
        stream = torch.cuda.ExternalStream(e.stream())

        def device_answer():
            out = torch.full((b, rl), 0x11, dtype=torch.uint8, device="cuda")
            st = torch.full((b,), -1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            for _ in range(2):   # both lanes capture and replay
                e.enqueue_device(slots.data_ptr(), stride, b, out.data_ptr(), rl, st.data_ptr())
            e.fence()
            with torch.cuda.stream(stream):
                o, s = out.clone(), st.clone()
            stream.synchronize()
            e.sync()
            return o.cpu().numpy(), s.cpu().numpy()

        before, _ = device_answer()
        offline.prepare(e, p)
        after, st = device_answer()
        assert list(st) == [0] * b and not np.array_equal(before, after)
        assert np.array_equal(after, _answer(e, frames))
        for c, resp, i in zip(clients, after, idx):
            assert np.array_equal(c.decrypt(resp), svc.synthetic_record(i, p.record_bytes))
        e.set_lanes(1)
        e.set_graphs(False)
    finally:
        e.close()
