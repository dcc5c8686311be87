"""The client of the answer path, restated for the CPU with numpy: key generation, the packing keys a request
carries, the query, and decryption of the engine's response (the reference's `service::new_request` and
`service::decrypt_response`, src/service.rs:227-257, over src/client.rs and src/packing.rs).

The reference's client rests on spiral-rs (ring arithmetic, gadget, discrete Gaussian sampling, ChaCha-seeded public
randomness), which is not available here.  This module states the scheme's arithmetic itself:

* the ring Z_Q[X]/(X^n + 1), Q = 4294955009, with the negacyclic NTT whose slot j holds the evaluation at
  psi^(2 brv(j) + 1) -- the slot order the reference's automorphism tables assume
  (`generate_automorph_tables_brute_force`, src/packing.rs:1082-1110) -- computed with the Cooley-Tukey /
  Gentleman-Sande pair of Longa and Naehrig (CANS 2016, Algorithms 1 and 2); psi is the smallest primitive 2n-th
  root of unity mod Q;
* the gadget with t digits of floor(log2ceil(Q) / t) + 1 bits (9 bits for the scheme's t = 4), the decomposition
  `gadget_invert_transposed_alloc` inverts (src/packing.rs:1468-1493);
* secrets and errors from the discrete Gaussian of width 0.5 sqrt(2 pi) (sigma 0.5, `Xs = Xe = D(0.5)`,
  src/scheme.rs:1-4, params.rs:102-104), sampled by an exact 64-bit table from counter-based splitmix64 streams of
  the client's secret seed (the reference draws them from OS entropy; the seed defaults to os.urandom);
* public randomness (the query masks a_i and the packing masks w, v) from seeded splitmix64 streams instead of the
  reference's ChaCha20 streams; the server derives the same masks from the same seeds (`offline.py`).

So a request built here is not the reference's byte for byte (nor can it be: the reference draws its secrets from
OS entropy), but it has the reference's structure and distributions, and the engine's response to it decrypts to
the record asked for.
"""
import math
import os

import numpy as np

from . import service

Q = service.Q
P = 256                                  # plaintext modulus p (src/scheme.rs:3)
DELTA = Q // P                           # scale_k = modulus / pt_modulus (src/client.rs:307)
NOISE_WIDTH = 0.5 * math.sqrt(2 * math.pi)
GEN = 5                                  # generator of the packing automorphisms for gamma = n (src/packing.rs:1697)

# public stream counters (the reference's SEED_0, W_SEED and V_SEED, src/scheme.rs:15-29)
QUERY_MASK_SEED = 0x5345454430           # the query masks a_i
W_MASK_SEED = 0x5745454437               # w: the mask of the rotation key y
V_MASK_SEED = 0x5645454438               # v: the mask of the conjugation key z

_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def public_uniform(count, seed):
    """count values uniform in [0, Q) from the public stream `seed`: value i is the splitmix64 finaliser of
    seed + (i + 1) * gamma, mapped to [0, Q) by a multiply-high of its top 32 bits."""
    return ((splitmix_stream(seed, count) >> np.uint64(32)) * np.uint64(Q)) >> np.uint64(32)


def _brv(n):
    logn = n.bit_length() - 1
    r = np.zeros(n, dtype=np.int64)
    for b in range(logn):
        r |= ((np.arange(n) >> b) & 1) << (logn - 1 - b)
    return r


def smallest_primitive_root(two_n):
    """The smallest primitive two_n-th root of unity mod Q (two_n must divide Q - 1 = 2^12 * 1048573)."""
    if (Q - 1) % two_n:
        raise ValueError("2n must divide Q - 1")
    for g in range(2, 1000):
        psi = pow(g, (Q - 1) // two_n, Q)
        if pow(psi, two_n // 2, Q) == Q - 1:
            break
    return min(pow(psi, k, Q) for k in range(1, two_n, 2))


class Ring:
    """Z_Q[X]/(X^n + 1): coefficient and NTT forms as uint64 arrays whose last axis has length n."""

    def __init__(self, n=service.POLY_LEN):
        self.n, self.logn = n, n.bit_length() - 1
        self.psi = smallest_primitive_root(2 * n)
        inv = pow(self.psi, Q - 2, Q)
        self.brv = _brv(n)
        self.fwd = np.array([pow(self.psi, int(r), Q) for r in self.brv], dtype=np.uint64)
        self.inv = np.array([pow(inv, int(r), Q) for r in self.brv], dtype=np.uint64)
        self.ninv = np.uint64(pow(n, Q - 2, Q))
        self._tables = {}

    def ntt(self, a):
        """Forward negacyclic NTT (Longa-Naehrig Algorithm 1): slot j = a(psi^(2 brv(j) + 1))."""
        a = np.asarray(a, dtype=np.uint64)
        shape, n, q = a.shape, self.n, np.uint64(Q)
        a = (a % q).reshape(-1, n)
        m, t = 1, n
        while m < n:
            t //= 2
            v = a.reshape(-1, m, 2, t)
            u = v[:, :, 0, :]
            w = (v[:, :, 1, :] * self.fwd[m:2 * m].reshape(1, m, 1)) % q
            a = np.stack(((u + w) % q, (u + q - w) % q), axis=2).reshape(-1, n)
            m *= 2
        return a.reshape(shape)

    def intt(self, a):
        """Inverse negacyclic NTT (Longa-Naehrig Algorithm 2, then times n^-1)."""
        a = np.asarray(a, dtype=np.uint64)
        shape, n, q = a.shape, self.n, np.uint64(Q)
        a = (a % q).reshape(-1, n)
        t, m = 1, n
        while m > 1:
            h = m // 2
            v = a.reshape(-1, h, 2, t)
            u, w = v[:, :, 0, :], v[:, :, 1, :]
            d = ((u + q - w) % q * self.inv[h:2 * h].reshape(1, h, 1)) % q
            a = np.stack(((u + w) % q, d), axis=2).reshape(-1, n)
            t *= 2
            m = h
        return (a * self.ninv % q).reshape(shape)

    def mul(self, a, b):
        """Negacyclic product of coefficient-form polynomials."""
        return self.intt(self.ntt(a) * self.ntt(b) % np.uint64(Q))

    def automorph(self, a, t):
        """tau_t(a)(X) = a(X^t) mod X^n + 1 of coefficient-form polynomials (t odd)."""
        a = np.asarray(a, dtype=np.uint64)
        n = self.n
        idx = (np.arange(n) * t) % (2 * n)
        out = np.zeros_like(a)
        pos, neg = idx < n, idx >= n
        out[..., idx[pos]] = a[..., pos]
        out[..., idx[neg] - n] = (np.uint64(Q) - a[..., neg] % np.uint64(Q)) % np.uint64(Q)
        return out

    def table(self, t):
        """The NTT-slot permutation of tau_t: (tau_t a)^[j] = a^[table[j]] (src/packing.rs:1082-1110)."""
        t %= 2 * self.n
        if t not in self._tables:
            s = 2 * self.brv + 1
            k = ((t * s) % (2 * self.n) - 1) // 2
            self._tables[t] = self.brv[k]
        return self._tables[t]


def gadget_bits(t):
    """Bits of a gadget digit for t digits: floor(log2ceil(Q) / t) + 1 = floor(32 / t) + 1, one bit when t = 32
    (spiral-rs get_bits_per); 9 for the scheme's t = 4."""
    return 1 if t >= 32 else 32 // t + 1


def gadget_invert(a, t=service.T_EXP_LEFT):
    """Base-2^gadget_bits(t) digits of coefficient-form values in [0, Q): (..., n) -> (..., t, n), least significant
    first (gadget_invert_transposed_alloc, src/packing.rs:1468-1493)."""
    a = np.asarray(a, dtype=np.uint64)
    b = gadget_bits(t)
    mask = np.uint64((1 << b) - 1)
    return np.stack([(a >> np.uint64(b * k)) & mask if b * k < 64 else np.zeros_like(a) for k in range(t)], axis=-2)


# D(0.5): Pr[x] proportional to exp(-pi x^2 / (0.5 sqrt(2 pi))^2) = exp(-2 x^2).  CDT_THRESHOLDS[j] =
# floor(2^64 Pr[X <= j - 4]) for j = 0..7 (computed at 60 decimal digits); a uniform 64-bit u gives
# x = -4 + #{j : u >= CDT_THRESHOLDS[j]}, so Pr[x] is exact to 2^-64 and the support is [-4, 4] (the mass beyond +-4,
# about 1e-14, goes to +-4).
CDT_THRESHOLDS = np.array([0x2CDC8, 0x33738FE26B, 0x114B1F533EAC34, 0x1B51A6ACA1B1BEEB, 0xE4AE59535E4E4114,
                           0xFFEEB4E0ACC153CB, 0xFFFFFFCC8C701D94, 0xFFFFFFFFFFFD3237], dtype=np.uint64)


def splitmix_stream(seed, count):
    """Value i of the stream `seed`: the splitmix64 finaliser of seed + (i + 1) * 0x9e3779b97f4a7c15."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(count, dtype=np.uint64) + np.uint64(1)) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def gaussian(seed, count):
    """count samples of D(0.5) from the stream `seed`, as values mod Q."""
    u = splitmix_stream(seed, count)
    x = (u[:, None] >= CDT_THRESHOLDS[None, :]).sum(axis=1).astype(np.int64) - 4
    return (x % Q).astype(np.uint64)


def secret_stream(seed, purpose):
    """The stream of a client's secret randomness for one purpose (0: s, 1: y's errors, 2: z's errors, 16 + j: the
    errors of its j-th query)."""
    with np.errstate(over="ignore"):
        return int(np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(purpose) * np.uint64(0xD1B54A32D192ED03))


def rescale_q_to(a, out_mod):
    """spiral-rs `rescale(a, Q, out_mod)` (restated as rescale_i64, src/modulus_switch.rs:116-130): centre a mod Q,
    scale by out_mod / Q rounding half away from zero, reduce mod out_mod; vectorised for out_mod <= 2^18."""
    a = np.asarray(a, dtype=np.int64) % Q
    c = np.where(a >= Q // 2, a - Q, a)
    num = c * out_mod + np.where(c >= 0, Q // 2, -(Q // 2))
    t = np.where(num >= 0, num // Q, -((-num) // Q))
    return (t % out_mod).astype(np.uint64)


def rescale_to_q(v, inp_mod):
    """rescale(v, inp_mod, Q) for a power-of-two inp_mod <= 2^18 (recovering a switched row), vectorised."""
    v = np.asarray(v, dtype=np.int64) % inp_mod
    c = np.where(v >= inp_mod // 2, v - inp_mod, v)
    num = c * Q + np.where(c >= 0, inp_mod // 2, -(inp_mod // 2))
    t = np.where(num >= 0, num // inp_mod, -((-num) // inp_mod))
    return (t % Q).astype(np.uint64)


def read_bits(buf, bit_off, width, count):
    """count values of `width` bits, LSB first, starting at bit bit_off of buf (read_arbitrary_bits)."""
    bits = np.unpackbits(np.frombuffer(bytes(buf), dtype=np.uint8), bitorder="little")
    seg = bits[bit_off:bit_off + width * count].reshape(count, width).astype(np.uint64)
    return (seg << np.arange(width, dtype=np.uint64)).sum(axis=1).astype(np.uint64)


def query_masks(rows, n):
    """The public masks a_i of the query's rows / n RLWE ciphertexts (coefficient form)."""
    return public_uniform(rows, QUERY_MASK_SEED).reshape(rows // n, n)


def packing_masks(n, tg=service.T_EXP_LEFT):
    """The public masks (w, v) of the two key-switching keys, NTT form, (tg, n) each
    (OfflinePackingKeys::init_full, src/packing.rs:1864-1892)."""
    return (public_uniform(tg * n, W_MASK_SEED).reshape(tg, n),
            public_uniform(tg * n, V_MASK_SEED).reshape(tg, n))


def ntt_inverse_table(ring):
    """The inverse-NTT table the engine takes (`get_ntt_inverse_table`): psi^-brv(i) / 2 mod Q, so that the
    engine's halving Gentleman-Sande butterflies (x + y) / 2 and (x - y) w compute this ring's exact inverse NTT."""
    half = np.uint64((Q + 1) // 2)
    return ring.inv * half % np.uint64(Q)


class Client:
    """One client: its secret s, the packing keys (y, z) of its requests, its queries and the decryption of the
    engine's responses (spiral-rs Client + YClient, src/client.rs; service::new_request / decrypt_response)."""

    def __init__(self, p, seed=None, ring=None):
        """seed: the client's secret seed (64 bits; from os.urandom when None -- the reference draws its secrets from
        entropy).  Every secret value comes from counter-based streams of it, so a seeded client is reproducible
        and the C++ client (include/altopir.hpp) with the same seed builds the same frames byte for byte."""
        self.p = p
        self.ring = ring or Ring(p.n)
        self.seed = int.from_bytes(os.urandom(8), "little") if seed is None else int(seed) & ((1 << 64) - 1)
        self.queries = 0
        self.s = gaussian(secret_stream(self.seed, 0), p.n)          # generate_secret_keys: sk_reg ~ D(0.5)
        self.s_hat = self.ring.ntt(self.s)

    def _ksk_body(self, gen, mask, purpose):
        """generate_ksk_body (src/packing.rs:2154-2177): -s * mask + e + tau_gen(s) * g, NTT form, (tg, n)."""
        r, q = self.ring, np.uint64(Q)
        tau_hat = r.ntt(r.automorph(self.s, gen))
        e_hat = r.ntt(gaussian(secret_stream(self.seed, purpose), self.p.tg * self.p.n).reshape(self.p.tg, self.p.n))
        bits = gadget_bits(self.p.tg)
        g = np.array([pow(2, bits * k, Q) for k in range(self.p.tg)], dtype=np.uint64)[:, None]
        minus_s_mask = self.s_hat[None, :] * ((q - mask) % q) % q
        return (minus_s_mask + e_hat + tau_hat[None, :] * g % q) % q

    def packing_keys(self):
        """PackingKeys::init_full (src/packing.rs:1935-1984): y switches tau_5(s) to s under mask w, z switches
        tau_(2n-1)(s) (the conjugation) under mask v.  Returns the condensed (flat, NTT form) y and z."""
        w, v = packing_masks(self.p.n, self.p.tg)
        y = self._ksk_body(GEN, w, 1)
        z = self._ksk_body(2 * self.p.n - 1, v, 2)
        return y.reshape(-1), z.reshape(-1)

    def query(self, index):
        """generate_query (src/client.rs:288-426, InspiRING branch) and new_request's scaling (src/service.rs:
        233-236): rows / n RLWE encryptions (-a_i, s a_i + e_i + mu_i), mu = DELTA at the index's coefficient;
        the query is the bodies' coefficients, switched from Q to 2^32 with rounding."""
        p, r, q = self.p, self.ring, np.uint64(Q)
        if not 0 <= index < p.rows:
            raise ValueError("index out of range")
        a = query_masks(p.rows, p.n)
        err = gaussian(secret_stream(self.seed, 16 + self.queries), p.rows).reshape(a.shape)
        self.queries += 1
        body = (r.intt(self.s_hat[None, :] * r.ntt(a) % q) + err) % q
        body[index // p.n, index % p.n] = (body[index // p.n, index % p.n] + np.uint64(DELTA)) % q
        v = body.reshape(-1)
        return ((v << np.uint64(32)) + np.uint64(Q // 2)) // q & np.uint64(0xFFFFFFFF)

    def request(self, index, keys=None):
        """service::new_request (src/service.rs:227-239): the frame asking for record `index`."""
        y, z = keys if keys is not None else self.packing_keys()
        return service.encode_request(self.p, y, z, self.query(index))

    def decrypt(self, response):
        """service::decrypt_response (src/service.rs:241-257): every part recovered (row 0 from 18 bits, row 1
        from 10 bits), decrypted as s * row0 + row1 and rescaled to p = 256.  Raises ValueError as the reference
        returns Err."""
        p, r, q = self.p, self.ring, np.uint64(Q)
        buf = np.frombuffer(bytes(response), dtype=np.uint8)
        if len(buf) != service.response_len(p):
            raise ValueError(f"response of {len(buf)} bytes, expected {service.response_len(p)}")
        q2_bits, q1_bits = (service.Q2 - 1).bit_length(), (service.Q1 - 1).bit_length()
        part = p.n * (q2_bits + q1_bits) // 8
        out = []
        for k in range(len(buf) // part):
            chunk = buf[k * part:(k + 1) * part]
            row0 = rescale_to_q(read_bits(chunk, 0, q2_bits, p.n), service.Q2)
            row1 = rescale_to_q(read_bits(chunk, q2_bits * p.n, q1_bits, p.n), service.Q1)
            m = (r.mul(self.s, row0) + row1) % q
            v = rescale_q_to(m, P)
            if (v > 255).any():
                raise ValueError("decrypted value out of range")
            out.append(v.astype(np.uint8))
        return np.concatenate(out)
