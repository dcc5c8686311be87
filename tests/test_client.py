"""The client restatement (altopir-public_b200/client.py) and the oracle's restatement of the scheme's offline set-up
(oracle/scheme.py): ring arithmetic, automorphism tables, public streams, and decryption round trips through the
reference's own engine (src/amx_kernels.cpp compiled unchanged) and through the oracle's engine."""
import numpy as np
import pytest

from oracle import scheme
from oracle.oracle import RefEngine, ref_methods


@pytest.mark.parametrize("n", [16, 256, 2048])
def test_ring_transforms_invert_and_agree_with_the_oracle(client_mod, n):
    rc, ro = client_mod.Ring(n), scheme.Ring(n)
    assert rc.psi == ro.psi and pow(rc.psi, n, client_mod.Q) == client_mod.Q - 1
    a = np.random.default_rng(n).integers(0, client_mod.Q, (3, n), dtype=np.uint64)
    assert np.array_equal(rc.intt(rc.ntt(a)), a)
    assert np.array_equal(rc.ntt(a), ro.ntt(a)) and np.array_equal(rc.intt(a), ro.intt(a))


def test_ring_product_is_the_negacyclic_schoolbook_product(client_mod):
    n, Q = 16, client_mod.Q
    rng = np.random.default_rng(2)
    a, b = (rng.integers(0, Q, n, dtype=np.uint64) for _ in range(2))
    want = [0] * n
    for i in range(n):
        for j in range(n):
            k, v = i + j, int(a[i]) * int(b[j])
            want[k % n] += -v if k >= n else v
    assert [x % Q for x in want] == [int(x) for x in client_mod.Ring(n).mul(a, b)]


@pytest.mark.parametrize("n", [16, 2048])
def test_automorphism_tables_permute_ntt_slots(client_mod, n):
    """table(t) is the slot permutation of tau_t in NTT form (generate_automorph_tables_brute_force)."""
    r, ro = client_mod.Ring(n), scheme.Ring(n)
    a = np.random.default_rng(3).integers(0, client_mod.Q, n, dtype=np.uint64)
    for t in (5, 25, 2 * n - 1, 2 * n - 5):
        assert np.array_equal(r.ntt(r.automorph(a, t)), r.ntt(a)[r.table(t)])
        assert np.array_equal(r.table(t), ro.table(t))
    assert sorted(r.table(5)) == list(range(n))


def test_engine_inverse_table_makes_halving_butterflies_exact(client_mod):
    """The engine's inverse NTT (src/amx_kernels.cpp:453-498) runs Gentleman-Sande butterflies x' = (x + y) / 2,
    y' = (x - y) w over the table it is given; with psi^-brv / 2 that is this ring's exact inverse transform."""
    n, Q = 256, client_mod.Q
    r = client_mod.Ring(n)
    tw = client_mod.ntt_inverse_table(r)
    half = (Q + 1) // 2
    a = np.random.default_rng(4).integers(0, Q, n, dtype=np.uint64)
    x = [int(v) for v in r.ntt(a)]
    t, h = 1, n // 2
    while h >= 1:
        for i in range(h):
            for j in range(2 * i * t, 2 * i * t + t):
                u, v = x[j], x[j + t]
                x[j], x[j + t] = (u + v) * half % Q, (u - v) * int(tw[h + i]) % Q
        t, h = 2 * t, h // 2
    assert x == [int(v) for v in a]


def test_public_streams_equal_the_oracle_generator(client_mod, oracle):
    for seed in (client_mod.QUERY_MASK_SEED, client_mod.W_MASK_SEED, client_mod.V_MASK_SEED):
        c = client_mod.public_uniform(5000, seed)
        assert np.array_equal(c, scheme.stream_uniform(5000, seed))
        assert np.array_equal(c, oracle.fill_uniform_u64(5000, client_mod.Q, seed))
        assert c.max() < client_mod.Q


def test_request_has_the_reference_frame_layout(client_mod, svc):
    p = svc.params(2048, 2048)
    c = client_mod.Client(p, seed=1)
    frame = c.request(7)
    assert frame.size == svc.request_len(p)
    y, z, q = svc.decode_request(p, frame)
    assert y.size == z.size == p.count and q.size == p.rows
    s = c.s.astype(np.int64)
    s = np.where(s > client_mod.Q // 2, s - client_mod.Q, s)
    assert np.abs(s).max() <= 4 and 0.1 < (s != 0).mean() < 0.35     # D(0.5): 0 with probability 0.787
    # a seeded client is reproducible, and its queries use fresh errors
    c2 = client_mod.Client(p, seed=1)
    assert np.array_equal(c2.request(7), frame)
    assert not np.array_equal(c2.request(7), frame)


def _records(oracle, idx, nbytes):
    return [oracle.synthetic_record(i, nbytes) for i in idx]


def test_round_trip_through_the_oracle_engine(client_mod, oracle, scheme_state):
    p = scheme_state.p
    clients = [client_mod.Client(p, seed=10 + k) for k in range(3)]
    idx = [0, 1234, p.rows - 1]
    frames = [c.request(i) for c, i in zip(clients, idx)]
    r, status, out = oracle.answer(scheme_state, frames)
    assert r == 3 and list(status) == [0, 0, 0]
    for c, resp, want in zip(clients, out, _records(oracle, idx, p.record_bytes)):
        assert np.array_equal(c.decrypt(resp), want)
    # another client's secret decrypts nothing
    assert not np.array_equal(clients[0].decrypt(out[1]), _records(oracle, [idx[1]], p.record_bytes)[0])


@pytest.mark.skipif(not ref_methods(), reason="the reference engine needs AVX-512 (and its library in oracle/_ref)")
def test_round_trip_through_the_reference_engine(client_mod, oracle, scheme_state):
    """Requests of this client, answered by the reference's own engine over the restated offline state, decrypt to
    the records asked for: src/service.rs new_request -> Engine::answer -> decrypt_response, as tests/engine.rs
    checks it."""
    p = scheme_state.p
    clients = [client_mod.Client(p, seed=20 + k) for k in range(4)]
    idx = [5, 77, 1024, 2000]
    frames = [c.request(i) for c, i in zip(clients, idx)]
    ref = RefEngine(scheme_state)
    try:
        outs = []
        for m in ref_methods():
            r, status, out, _ = ref.answer(frames, m)
            assert r == 4 and list(status) == [0] * 4
            outs.append(out.copy())
    finally:
        ref.close()
    assert all(np.array_equal(o, outs[0]) for o in outs)
    for c, resp, want in zip(clients, outs[0], _records(oracle, idx, p.record_bytes)):
        assert np.array_equal(c.decrypt(resp), want)


def test_decrypt_rejects_a_response_of_the_wrong_length(client_mod, svc):
    p = svc.params(2048, 2048)
    with pytest.raises(ValueError, match="expected"):
        client_mod.Client(p, seed=1).decrypt(np.zeros(100, dtype=np.uint8))


def test_query_rejects_an_index_out_of_range(client_mod, svc):
    p = svc.params(2048, 2048)
    with pytest.raises(ValueError):
        client_mod.Client(p, seed=1).query(p.rows)


def test_offline_public_inputs_are_the_client_masks(client_mod, svc):
    from altopir_b200 import offline
    p = svc.params(4096, 2048)
    q, w, v = offline.public_inputs(p)
    a = client_mod.query_masks(p.rows, p.n)
    assert q.shape == (p.rows // p.n, p.n) and np.array_equal((q + a) % client_mod.Q, np.zeros_like(a))
    w2, v2 = client_mod.packing_masks(p.n, p.tg)
    assert np.array_equal(w, w2) and np.array_equal(v, v2) and not np.array_equal(w, v)


def test_gaussian_table_matches_d_half(client_mod):
    """The 64-bit table gives Pr[x] = exp(-2 x^2) / Z to 2^-64; a million samples land within 5 sigma of it."""
    import math
    t = [int(v) for v in client_mod.CDT_THRESHOLDS]
    z = sum(math.exp(-2 * x * x) for x in range(-6, 7))
    for j, x in enumerate(range(-4, 4)):
        want = sum(math.exp(-2 * y * y) for y in range(-6, x + 1)) / z
        assert abs(t[j] / 2 ** 64 - want) < 1e-15
    v = client_mod.gaussian(12345, 1_000_000).astype(np.int64)
    v = np.where(v > client_mod.Q // 2, v - client_mod.Q, v)
    for x, p in ((0, math.exp(0) / z), (1, math.exp(-2) / z), (-1, math.exp(-2) / z)):
        assert abs((v == x).mean() - p) < 5 * math.sqrt(p * (1 - p) / v.size)
