"""Test infrastructure: a numpy restatement of the reference's offline set-up for the scheme itself -- the hint, the
InspiRING precomputation and the row-0 prefixes -- so that an engine can be given state from which its responses
decrypt (the reference's `Prepared::new`, src/service.rs:127-157).  Used only by the tests, as the checker of the
device-side offline set-up and, with the client, for decryption round trips through the reference's own engine.

What the reference computes with spiral-rs (absent here) is restated from the reference's call sites:

* hint: for every database column c, sum_i perm(q_i) * D_{i,c} mod (X^n + 1, Q), q_i the query masks' row 0
  (= -a_i), perm = util.rs negacyclic_perm with shift 0 (src/server.rs:656-768, 711-738);
* prep_pack_lwes: the polynomial of column c's LWE mask is perm(hint column c), in NTT form
  (src/packing.rs:910-974);
* precompute_aggregates_ntt and full_packing_offline_mode: the aggregates r_i, rbar_i and the backward walk that
  yields bold_t, bold_t_bar, bold_t_hat and a_hat (src/packing.rs:2260-2359);
* switch_prefix_row0 (src/modulus_switch.rs:136-147).

The ring is Z_Q[X]/(X^n + 1) with the negacyclic NTT whose slot j is the evaluation at psi^(2 brv(j) + 1), psi
the smallest primitive 2n-th root of unity, and the gadget has t digits of floor(32 / t) + 1 bits.  Public masks
come from the same seeded splitmix64 streams as the client's.  Parity with the reference's own offline values is unpinned (its
masks are ChaCha20 streams of spiral-rs); the restatement is pinned by decryption: responses of the reference's
engine over this state decrypt to the records asked for.
"""
import numpy as np

Q = 4294955009
GEN = 5
QUERY_MASK_SEED = 0x5345454430
W_MASK_SEED = 0x5745454437
V_MASK_SEED = 0x5645454438
_Q = np.uint64(Q)


def stream_uniform(count, seed):
    """Value i: the splitmix64 finaliser of seed + (i + 1) * 0x9e3779b97f4a7c15, times Q by a multiply-high of its
    top 32 bits (the public streams of the client and the server)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(count, dtype=np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(32)) * _Q) >> np.uint64(32)


class Ring:
    def __init__(self, n):
        self.n = n
        logn = n.bit_length() - 1
        self.brv = np.array([int(format(i, f"0{logn}b")[::-1], 2) for i in range(n)], dtype=np.int64)
        for g in range(2, 1000):
            root = pow(g, (Q - 1) // (2 * n), Q)
            if pow(root, n, Q) == Q - 1:
                break
        self.psi = min(pow(root, k, Q) for k in range(1, 2 * n, 2))
        ipsi = pow(self.psi, Q - 2, Q)
        self.w = np.array([pow(self.psi, int(r), Q) for r in self.brv], dtype=np.uint64)
        self.wi = np.array([pow(ipsi, int(r), Q) for r in self.brv], dtype=np.uint64)
        self.ninv = np.uint64(pow(n, Q - 2, Q))

    def ntt(self, a):
        a = np.asarray(a, dtype=np.uint64) % _Q
        shape, n = a.shape, self.n
        a = a.reshape(-1, n)
        m, t = 1, n
        while m < n:
            t //= 2
            v = a.reshape(-1, m, 2, t)
            x, y = v[:, :, 0, :], v[:, :, 1, :] * self.w[m:2 * m, None] % _Q
            a = np.stack(((x + y) % _Q, (x + _Q - y) % _Q), axis=2).reshape(-1, n)
            m *= 2
        return a.reshape(shape)

    def intt(self, a):
        a = np.asarray(a, dtype=np.uint64) % _Q
        shape, n = a.shape, self.n
        a = a.reshape(-1, n)
        t, h = 1, n // 2
        while h >= 1:
            v = a.reshape(-1, h, 2, t)
            x, y = v[:, :, 0, :], v[:, :, 1, :]
            a = np.stack(((x + y) % _Q, (x + _Q - y) % _Q * self.wi[h:2 * h, None] % _Q), axis=2).reshape(-1, n)
            t *= 2
            h //= 2
        return (a * self.ninv % _Q).reshape(shape)

    def table(self, t):
        """generate_automorph_tables_brute_force's table (t - 1) / 2 (src/packing.rs:1082-1110)."""
        k = ((t * (2 * self.brv + 1)) % (2 * self.n) - 1) // 2
        return self.brv[k]


def perm(a):
    """util.rs negacyclic_perm with shift 0: out[0] = a[0], out[i] = -a[n - i] mod Q."""
    a = np.asarray(a, dtype=np.uint64) % _Q
    out = np.empty_like(a)
    out[..., 0] = a[..., 0]
    out[..., 1:] = (_Q - a[..., :0:-1]) % _Q
    return out


def gadget_digits(a, t):
    """gadget_invert_transposed_alloc (src/packing.rs:1468-1493): digits of floor(32 / t) + 1 bits (get_bits_per
    with log2ceil(Q) = 32; one bit when t = 32), (..., n) -> (..., t, n)."""
    a = np.asarray(a, dtype=np.uint64)
    b = 1 if t >= 32 else 32 // t + 1
    return np.stack([(a >> np.uint64(b * k)) & np.uint64((1 << b) - 1) if b * k < 64 else np.zeros_like(a)
                     for k in range(t)], axis=-2)


def hint(ring, db_col, masks):
    """The hint (n, cols): column c = sum_i perm(-a_i) * D_{i,c}, D_{i,c} = records i n .. i n + n - 1 of byte c
    (multiply_with_db_ring over generate_pseudorandom_query, src/server.rs:656-738).  db_col: (cols, rows) bytes;
    masks: (rows / n, n) query masks a_i."""
    n = ring.n
    cols, rows = db_col.shape
    qhat = ring.ntt(perm((_Q - masks % _Q) % _Q))                    # (rows / n, n)
    out = np.zeros((cols, n), dtype=np.uint64)
    for c0 in range(0, cols, 256):
        d = ring.ntt(db_col[c0:c0 + 256].reshape(-1, rows // n, n).astype(np.uint64))
        acc = np.zeros((d.shape[0], n), dtype=np.uint64)
        for i in range(rows // n):
            acc = (acc + d[:, i, :] * qhat[i] % _Q) % _Q
        out[c0:c0 + 256] = ring.intt(acc)
    return out.T.copy()


def prep_lwes(ring, hint_cols):
    """prep_pack_lwes (src/packing.rs:910-942): a_ct_tilde = NTT(perm(mask of column c)), (n_cols, n)."""
    return ring.ntt(perm(hint_cols))


def aggregates(ring, act):
    """precompute_aggregates_ntt (src/packing.rs:2260-2291): evaluations[v] = NTT over j of act[j][v]; r_i gathers
    them through tau_(g^i)'s table, rbar_i through tau_(2n - g^i)'s, both times n^-1; i < n / 2."""
    n = ring.n
    ev = ring.ntt(act.T)                                              # ev[v][slot]
    slots = np.arange(n)
    r = np.empty((n // 2, n), dtype=np.uint64)
    rbar = np.empty((n // 2, n), dtype=np.uint64)
    for i in range(n // 2):
        e = pow(GEN, i, 2 * n)
        r[i] = ev[ring.table(e), slots] * ring.ninv % _Q
        rbar[i] = ev[ring.table(2 * n - e), slots] * ring.ninv % _Q
    return r, rbar


def walk(ring, r, rbar, w, v, tg):
    """full_packing_offline_mode (src/packing.rs:2301-2359): for i = n/2 - 2 .. 0, bold_t[i] = NTT(G^-1(r[i+1])),
    r[i] += sum_k tau_(g^i)(w)[k] bold_t[i][k] (and the same for the bar chain with tau_(2n - g^i)); then
    bold_t_hat = NTT(G^-1(rbar[0])), r[0] += sum_k v[k] bold_t_hat[k], a_hat = r[0] in coefficient form."""
    n = ring.n
    half = n // 2
    r, rbar = r.copy(), rbar.copy()
    bt = np.zeros((half - 1, tg, n), dtype=np.uint64)
    btb = np.zeros((half - 1, tg, n), dtype=np.uint64)
    for i in range(half - 2, -1, -1):
        e = pow(GEN, i, 2 * n)
        wa = w[:, ring.table(e)]
        wb = w[:, ring.table(2 * n - e)]
        dig = ring.ntt(gadget_digits(ring.intt(np.stack([r[i + 1], rbar[i + 1]])), tg))   # (2, tg, n)
        bt[i], btb[i] = dig[0], dig[1]
        r[i] = (r[i] + (wa * dig[0] % _Q).sum(axis=0) % _Q) % _Q
        rbar[i] = (rbar[i] + (wb * dig[1] % _Q).sum(axis=0) % _Q) % _Q
    that = ring.ntt(gadget_digits(ring.intt(rbar[0]), tg))
    a0 = (r[0] + (v * that % _Q).sum(axis=0) % _Q) % _Q
    return bt, btb, that, ring.intt(a0)


def prefix_row0(a_hat, part_len, q2_bits=18):
    """switch_prefix_row0 (src/modulus_switch.rs:136-147): a_hat rescaled to 2^18, 18 bits a value LSB first."""
    a = a_hat.astype(np.int64)
    c = np.where(a >= Q // 2, a - Q, a)
    num = c * (1 << q2_bits) + np.where(c >= 0, Q // 2, -(Q // 2))
    t = (np.where(num >= 0, num // Q, -((-num) // Q)) % (1 << q2_bits)).astype(np.uint64)
    bits = ((t[:, None] >> np.arange(q2_bits, dtype=np.uint64)) & np.uint64(1)).astype(np.uint8).ravel()
    out = np.zeros(part_len, dtype=np.uint8)
    packed = np.packbits(bits, bitorder="little")
    out[:packed.size] = packed
    return out


class SchemeState:
    """Engine state derived from the scheme (what Prepared::new hands to Engine::new), with the attributes the
    oracle's reference-engine wrapper reads: p, db_col, U (packing-matrix values), that, prefixes, inv_table."""

    def __init__(self, p, db_col, oracle, ring=None):
        self.p, self.db_col = p, db_col
        n, tg = p.n, p.tg
        ring = ring or Ring(n)
        self.ring = ring
        masks = stream_uniform(p.rows, QUERY_MASK_SEED).reshape(p.rows // n, n)
        w = stream_uniform(tg * n, W_MASK_SEED).reshape(tg, n)
        v = stream_uniform(tg * n, V_MASK_SEED).reshape(tg, n)
        self.hint = hint(ring, db_col, masks)                              # (n, cols)
        self.bold_t, self.bold_t_bar, self.that, self.a_hat, self.prefixes = [], [], [], [], []
        for o in range(p.instances):
            act = prep_lwes(ring, self.hint[:, o * n:(o + 1) * n].T)
            r, rbar = aggregates(ring, act)
            bt, btb, that, a_hat = walk(ring, r, rbar, w, v, tg)
            self.bold_t.append(np.ascontiguousarray(bt.reshape(-1)))
            self.bold_t_bar.append(np.ascontiguousarray(btb.reshape(-1)))
            self.that.append(np.ascontiguousarray(that.reshape(-1)))
            self.a_hat.append(a_hat)
            self.prefixes.append(prefix_row0(a_hat, p.part_len))
        self.tables = np.stack([ring.table(t) for t in range(1, 2 * n, 2)]).astype(np.uint32)
        self.gen_pows = np.array([pow(GEN, i, 2 * n) for i in range(n)], dtype=np.uint32)
        self.U = oracle.pack_build(self.bold_t, self.bold_t_bar, self.tables, self.gen_pows, n // 2 - 1, tg, n)
        # get_ntt_inverse_table: psi^-brv(i) / 2, the table for which the engine's halving butterflies invert
        self.inv_table = ring.wi * np.uint64((Q + 1) // 2) % _Q
