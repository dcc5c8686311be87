/*
 * alto_oracle.c -- CPU restatement of the AltoPIR answer path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine and the "port" CPU baseline; nothing in
 * the product links it.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it.
 *
 * It restates, in plain C, what the reference engine `src/amx_kernels.cpp` computes (its AMX/VNNI tiling is not
 * followed; only the arithmetic is), plus the reference's synthetic database generator (`src/service.rs`).
 * Every function cites the reference lines whose behaviour it reproduces.  Parity of this restatement with the
 * reference is pinned by tests/golden/ (vectors produced by the reference engine compiled from its own sources,
 * see oracle/Makefile and tests/golden/make_golden.py).
 *
 * Arithmetic facts used throughout (all exact, integer only):
 *   Q = 4294955009 = 2^32 - 12287 (the NTT prime, src/service.rs:25).
 *   scan : acc = sum_k db[col][k] * q[k] mod 2^32, inter = (acc * Q + 2^31) >> 32 (amx_kernels.cpp:287-307).
 *   pack : beta = sum_k y[k] * U[col][k] mod Q, U = folded packing matrix mod Q (amx_kernels.cpp:345-445).
 *   tail : acc = beta + sum_k z[k n + i] * that[k n + i] mod Q, inverse NTT, v = inter + acc mod Q,
 *          centred rescale to q1 with round-half-away-from-zero, bit-packed after the row-0 prefix
 *          (amx_kernels.cpp:447-537, 597-611).
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define ORC_Q 4294955009ull
#define ORC_SEED 0x416c746f504952ull          /* src/service.rs:44 */
#define ORC_GAMMA 0x9e3779b97f4a7c15ull       /* src/service.rs:47 */
#define ORC_ROW_MUL 0xd1b54a32d192ed03ull     /* src/service.rs:56 */

static inline uint32_t ld32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

/* ---------------------------------------------------------------- synthetic database (src/service.rs:43-78) */

/* The finaliser of splitmix64 (src/service.rs:48-51). */
static inline uint64_t orc_finalise(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* synthetic::mix (src/service.rs:46-52): advance the counter by the golden gamma, return its finalised value. */
uint64_t orc_mix(uint64_t *state) {
    *state += ORC_GAMMA;
    return orc_finalise(*state);
}

/* synthetic::record (src/service.rs:54-62), written sequentially exactly as the reference does. */
void orc_synthetic_record(uint8_t *dst, uint64_t row, size_t bytes) {
    uint64_t state = ORC_SEED ^ (ORC_ROW_MUL * (row + 1));
    for (size_t i = 0; i + 1 < bytes; i += 2) {
        uint16_t v = (uint16_t)(orc_mix(&state) % 65535);
        dst[i] = (uint8_t)(v & 0xff);
        dst[i + 1] = (uint8_t)(v >> 8);
    }
}

/* Random access into the same stream: the m-th call of mix on a state s0 returns finalise(s0 + (m+1) * gamma), so
 * byte `col` of record `row` is one finaliser evaluation (equal to orc_synthetic_record(row)[col]). */
uint8_t orc_record_byte(uint64_t row, uint64_t col) {
    uint64_t s0 = ORC_SEED ^ (ORC_ROW_MUL * (row + 1));
    uint16_t v = (uint16_t)(orc_finalise(s0 + (col / 2 + 1) * ORC_GAMMA) % 65535);
    return (col & 1) ? (uint8_t)(v >> 8) : (uint8_t)(v & 0xff);
}

/* The column-order database the reference server builds from synthetic::database (src/service.rs:64-78,
 * src/server.rs:251-366): db[(col - col0) * ld + row] = record(row)[col], for ncols columns starting at col0. */
void orc_synthetic_db_col(uint8_t *db, size_t ld, size_t rows, size_t col0, size_t ncols) {
    #pragma omp parallel for schedule(static)
    for (size_t c = 0; c < ncols; c++)
        for (size_t r = 0; r < rows; r++) db[c * ld + r] = orc_record_byte(r, col0 + c);
}

/* ------------------------------------------------------------------ seeded benchmark inputs
 * The seeded engine state and request frames that the tests and the benchmark give to both engines.  The reference
 * builds its state with spiral-rs and its clients draw secrets from entropy, so these inputs are this project's own
 * definition, not a reference algorithm: value i of a stream with counter `seed` is the splitmix64 finaliser of
 * seed + (i + 1) * gamma, mapped to [0, bound) by a multiply-high of its top 32 bits.  The engine library carries the
 * same generators (alto_fill_*, alto_synthetic_request); this copy lets the benchmark's reference arm build its
 * workload without loading the engine library, and the CPU tests check that the two copies agree byte for byte. */
static inline uint64_t orc_stream_at(uint64_t seed, uint64_t i) { return orc_finalise(seed + (i + 1) * ORC_GAMMA); }
static inline uint64_t orc_bounded(uint64_t x, uint64_t bound) { return ((x >> 32) * bound) >> 32; }

void orc_fill_uniform_u32(uint32_t *dst, size_t count, uint64_t bound, uint64_t seed) {
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < count; i++) dst[i] = (uint32_t)orc_bounded(orc_stream_at(seed, i), bound);
}

void orc_fill_uniform_u64(uint64_t *dst, size_t count, uint64_t bound, uint64_t seed) {
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < count; i++) dst[i] = orc_bounded(orc_stream_at(seed, i), bound);
}

void orc_fill_bytes(uint8_t *dst, size_t count, uint64_t seed) {
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < count; i++) dst[i] = (uint8_t)(orc_stream_at(seed, i) >> 56);
}

/* One well-formed frame of client `client`: [0][u32 tg_n][u32 tg_n][y, z: 2 tg_n words < Q][rows query words], the
 * frame layout of src/service.rs:178-198; stream counter seed ^ ORC_ROW_MUL * (client + 1). */
void orc_synthetic_request(uint8_t *frame, size_t rows, size_t tg_n, uint64_t seed, uint64_t client) {
    const uint64_t s = seed ^ (ORC_ROW_MUL * (client + 1));
    frame[0] = 0;
    for (int b = 0; b < 4; b++) frame[1 + b] = frame[5 + b] = (uint8_t)(tg_n >> (8 * b));
    for (size_t i = 0; i < 2 * tg_n + rows; i++) {
        const uint64_t x = orc_stream_at(s, i);
        const uint32_t v = i < 2 * tg_n ? (uint32_t)orc_bounded(x, ORC_Q) : (uint32_t)(x >> 32);
        for (int b = 0; b < 4; b++) frame[9 + 4 * i + b] = (uint8_t)(v >> (8 * b));
    }
}

/* ------------------------------------------------------------------ request validation (amx_kernels.cpp:572-580) */

/* Status of one request frame, as alto_answer assigns it (amx_kernels.cpp:572-580) and as decode_request rejects it
 * (src/service.rs:200-217): 1 = missing or wrong length, 2 = flag byte or key counts, 3 = a y/z key word >= Q.
 * Query words are not range-checked. */
int orc_validate(const uint8_t *f, size_t len, size_t count, size_t rows) {
    const size_t want = 9 + 4 * (2 * count + rows);
    if (!f || len != want) return 1;
    if (f[0] != 0 || (size_t)ld32(f + 1) != count || (size_t)ld32(f + 5) != count) return 2;
    for (size_t i = 0; i < 2 * count; i++)
        if ((uint64_t)ld32(f + 9 + 4 * i) >= ORC_Q) return 3;
    return 0;
}

/* ------------------------------------------------------------------------------ scan (amx_kernels.cpp:175-309) */

/* acc = sum_k dbcol[k] * q[k] mod 2^32 over one database column (the limb recombination of amx_kernels.cpp:287-300
 * and 86-93 equals this plain wrapping dot product). */
uint32_t orc_scan_acc(const uint8_t *dbcol, const uint8_t *q, size_t rows) {
    uint32_t acc = 0;
    for (size_t k = 0; k < rows; k++) acc += (uint32_t)dbcol[k] * ld32(q + 4 * k);
    return acc;
}

/* Switch from Z_{2^32} to Z_Q with rounding (amx_kernels.cpp:306-307). */
uint32_t orc_mod_switch(uint32_t acc) {
    return (uint32_t)(((uint64_t)acc * ORC_Q + (1ull << 31)) >> 32);
}

/* ------------------------------------------------------------------------------ pack (amx_kernels.cpp:345-445) */

/* beta = sum_k y[k] * urow[k] mod Q; urow holds one row of the packing matrix as values in [0, Q).  The reference's
 * 16-term limb recombination with 2^32 = 12287 folding (amx_kernels.cpp:410-439) computes exactly this residue. */
uint32_t orc_pack_beta(const uint32_t *urow, const uint8_t *y, size_t K) {
    unsigned __int128 s = 0;
    for (size_t k = 0; k < K; k++) s += (unsigned __int128)((uint64_t)urow[k] * ld32(y + 4 * k));
    return (uint32_t)(s % ORC_Q);
}

/* ------------------------------------------------------------------------------ tail (amx_kernels.cpp:447-537) */

/* Inverse NTT over Z_Q (amx_kernels.cpp:461-498).  Stages run with half-length t = 1, 2, 4, ..., n/2; block i of a
 * stage with h = n / (2t) blocks uses the twiddle table[h + i] (only its low 32 bits enter the product, as with the
 * reference's 32x32-bit multiply).  Gentleman-Sande butterfly with halving: x' = (x + y) / 2, y' = (x - y) * w.
 * a[] holds values in [0, Q) on entry and on exit.  Returns -1 when n is not a power of two >= 16. */
int orc_intt(uint64_t *a, const uint64_t *table, size_t n) {
    if (n < 16 || (n & (n - 1))) return -1;
    for (size_t t = 1; t < n; t <<= 1) {
        const size_t h = n / (2 * t);
        for (size_t i = 0; i < h; i++) {
            const uint64_t w = table[h + i] & 0xffffffffull;
            uint64_t *blk = a + 2 * t * i;
            for (size_t j = 0; j < t; j++) {
                const uint64_t x = blk[j], y = blk[t + j];
                uint64_t s = (x + y) % ORC_Q;
                s = (s & 1) ? (s + ORC_Q) >> 1 : s >> 1;
                const uint64_t d = (x + ORC_Q - y) % ORC_Q;
                blk[j] = s;
                blk[t + j] = (uint64_t)(((unsigned __int128)d * w) % ORC_Q);
            }
        }
    }
    return 0;
}

/* Centred rescale of v in [0, Q) from Q to q1, rounding half away from zero, result in [0, q1)
 * (amx_kernels.cpp:522-529).  The reference evaluates (c * q1 +- floor(Q/2)) / Q in double precision and truncates;
 * |c * q1 +- floor(Q/2)| < 2^53 is exact and the quotient's rounding cannot cross an integer (the distance from
 * an integer is at least 1/Q > half an ulp), so C's truncating integer division gives the same value. */
uint32_t orc_rescale(uint64_t v, uint64_t q1) {
    const int64_t half = (int64_t)(ORC_Q / 2);
    const int neg = v >= (uint64_t)half;
    const int64_t c = neg ? (int64_t)v - (int64_t)ORC_Q : (int64_t)v;
    const int64_t x = c * (int64_t)q1 + (neg ? -half : half);
    int64_t t = x / (int64_t)ORC_Q;
    if (t < 0) t += (int64_t)q1;
    if (t >= (int64_t)q1) t -= (int64_t)q1;
    return (uint32_t)t;
}

/* The same rescale evaluated the reference's way, in double precision (amx_kernels.cpp:526-529). */
uint32_t orc_rescale_double(uint64_t v, uint64_t q1) {
    const int64_t half = (int64_t)(ORC_Q / 2);
    const int neg = v >= (uint64_t)half;
    const int64_t c = neg ? (int64_t)v - (int64_t)ORC_Q : (int64_t)v;
    const double x = __builtin_fma((double)c, (double)q1, neg ? -(double)half : (double)half);
    int64_t t = (int64_t)(x / (double)ORC_Q);
    if (t < 0) t += (int64_t)q1;
    if (t >= (int64_t)q1) t -= (int64_t)q1;
    return (uint32_t)t;
}

/* Count of v in [v0, v1) where the integer and double rescales differ (exhaustive check of the claim above). */
uint64_t orc_rescale_mismatches(uint64_t v0, uint64_t v1, uint64_t q1) {
    uint64_t bad = 0;
    #pragma omp parallel for reduction(+ : bad) schedule(static)
    for (int64_t v = (int64_t)v0; v < (int64_t)v1; v++) bad += orc_rescale((uint64_t)v, q1) != orc_rescale_double((uint64_t)v, q1);
    return bad;
}

/* Position-weighted digest of orc_rescale over [v0, v1): sum of rescale(v) * (2v + 1) mod 2^64, to compare a
 * whole range with another implementation in one number. */
uint64_t orc_rescale_digest(uint64_t v0, uint64_t v1, uint64_t q1) {
    uint64_t d = 0;
    #pragma omp parallel for reduction(+ : d) schedule(static)
    for (int64_t v = (int64_t)v0; v < (int64_t)v1; v++) d += (uint64_t)orc_rescale((uint64_t)v, q1) * (2 * (uint64_t)v + 1);
    return d;
}

/* Row 1 of one response part (amx_kernels.cpp:515-537): rescale inter + acc and OR q1_bits-bit values LSB-first into
 * res at bit bit_off + z * q1_bits, never past res_len.  Returns -1 on the reference's parameter check. */
int orc_switch_row1(uint8_t *res, size_t res_len, size_t bit_off, const uint32_t *inter, const uint64_t *acc, size_t n,
                    uint64_t q1, int q1_bits) {
    if (q1 >= (1ull << 21) || n % 8 || (bit_off + n * (size_t)q1_bits + 7) / 8 > res_len || q1_bits > 24) return -1;
    for (size_t z = 0; z < n; z++) {
        const uint64_t v = ((uint64_t)inter[z] + acc[z]) % ORC_Q;
        const uint32_t t = orc_rescale(v, q1);
        const size_t p = bit_off + z * (size_t)q1_bits;
        const uint32_t w = t << (p % 8);
        for (size_t k = 0; k < 4 && p / 8 + k < res_len; k++) res[p / 8 + k] |= (uint8_t)(w >> (8 * k));
    }
    return 0;
}

/* Key-switch accumulate then inverse NTT (amx_kernels.cpp:500-513): acc[i] = beta[i] + sum_{k<tg} z[k n + i] *
 * that[k n + i] mod Q (every operand reduced mod Q first), then orc_intt. */
int orc_tail_ntt(uint64_t *acc, const uint32_t *beta, const uint8_t *z, const uint64_t *that, size_t tg,
                 const uint64_t *table, size_t n) {
    for (size_t i = 0; i < n; i++) {
        uint64_t s = beta[i] % ORC_Q;
        for (size_t k = 0; k < tg; k++) {
            const uint64_t a = ld32(z + 4 * (k * n + i)) % ORC_Q, b = that[k * n + i] % ORC_Q;
            s = (s + (uint64_t)(((unsigned __int128)a * b) % ORC_Q)) % ORC_Q;
        }
        acc[i] = s;
    }
    return orc_intt(acc, table, n);
}

/* ------------------------------------------------------------------- whole answer (amx_kernels.cpp:539-615) */

/* Engine state in plain form: the same borrowed inputs as alto_engine_new (amx_kernels.cpp:546-560) except that the
 * packing matrix is given as values U[col * K + k] in [0, Q) instead of the reference's AMX byte-plane layout. */
typedef struct {
    const uint8_t *db_col; size_t ld, rows, cols;
    const uint32_t *U; size_t n, tg;
    const uint8_t *const *prefix; size_t part_len, row1_off; uint64_t q1; int q1_bits;
    const uint64_t *const *that; const uint64_t *inv_table;
} OrcState;

/* One response part o (n columns) of one valid request frame f: prefix copy, scan, pack, tail
 * (amx_kernels.cpp:597-609 for a single (client, output) work item). */
int orc_answer_part(const OrcState *s, const uint8_t *f, size_t o, uint8_t *res) {
    const size_t n = s->n, count = s->tg * n;
    const uint8_t *y = f + 9, *z = f + 9 + 4 * count, *q = f + 9 + 8 * count;
    uint32_t *inter = (uint32_t *)malloc(sizeof(uint32_t) * n), *beta = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint64_t *acc = (uint64_t *)malloc(sizeof(uint64_t) * n);
    for (size_t i = 0; i < n; i++) {
        const size_t col = o * n + i;
        inter[i] = orc_mod_switch(orc_scan_acc(s->db_col + col * s->ld, q, s->rows));
        beta[i] = orc_pack_beta(s->U + col * count, y, count);
    }
    memcpy(res, s->prefix[o], s->part_len);
    int bad = orc_tail_ntt(acc, beta, z, s->that[o], s->tg, s->inv_table, n) != 0;
    bad |= orc_switch_row1(res, s->part_len, s->row1_off, inter, acc, n, s->q1, s->q1_bits) != 0;
    free(inter); free(beta); free(acc);
    return bad ? -3 : 0;
}

/* alto_answer semantics (amx_kernels.cpp:564-615): statuses for every frame, responses only for valid ones
 * (rejected output buffers are left untouched), returns the number of valid requests or -3 on a tail failure. */
int orc_answer(const OrcState *s, const uint8_t *const *req, const size_t *len, size_t B, uint8_t *const *out,
               int *status) {
    const size_t count = s->tg * s->n, outputs = s->cols / s->n;
    size_t valid = 0;
    for (size_t c = 0; c < B; c++) {
        status[c] = orc_validate(req[c], len[c], count, s->rows);
        valid += status[c] == 0;
    }
    int bad = 0;
    #pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (size_t pi = 0; pi < B * outputs; pi++) {
        const size_t c = pi / outputs, o = pi % outputs;
        if (status[c]) continue;
        bad |= orc_answer_part(s, req[c], o, out[c] + o * s->part_len) != 0;
    }
    return bad ? -3 : (int)valid;
}

/* A list of response parts computed in parallel: part k is output parts[k] of the (valid) frame frames[k], written
 * to out[k] (part_len bytes each).  Returns -3 if any tail failed. */
int orc_answer_parts(const OrcState *s, const uint8_t *const *frames, const size_t *parts, size_t count,
                     uint8_t *const *out) {
    int bad = 0;
    #pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (size_t k = 0; k < count; k++) bad |= orc_answer_part(s, frames[k], parts[k], out[k]) != 0;
    return bad ? -3 : 0;
}

/* ---------------------------------------------------------------- packing matrix (amx_kernels.cpp:311-341) */

/* The dense public packing matrix with the InspiRING automorphisms folded in, as values mod Q:
 * for output column oz = (o, z) and iteration i < num_iter with generator power g = gen_pows[i],
 *   U[oz][k n + tables[(g-1)/2][z]]      += bold_t[o][(i tg + k) n + z]
 *   U[oz][k n + tables[(2n-g-1)/2][z]]   += bold_t_bar[o][(i tg + k) n + z]
 * summed with 64-bit wrap-around and reduced mod Q at the end.  U is (rho n) x (tg n), row-major. */
void orc_pack_build(uint32_t *U, const uint64_t *const *bold_t, const uint64_t *const *bold_t_bar,
                    const uint32_t *tables, const uint32_t *gen_pows, size_t num_iter, size_t tg, size_t n,
                    size_t rho) {
    const size_t K = tg * n;
    #pragma omp parallel
    {
        uint64_t *col = (uint64_t *)malloc(sizeof(uint64_t) * K);
        #pragma omp for schedule(dynamic, 16)
        for (size_t oz = 0; oz < rho * n; oz++) {
            const size_t o = oz / n, z = oz % n;
            memset(col, 0, sizeof(uint64_t) * K);
            for (size_t i = 0; i < num_iter; i++) {
                const size_t g = gen_pows[i];
                const size_t zp = tables[((g - 1) / 2) * n + z], zb = tables[((2 * n - g - 1) / 2) * n + z];
                for (size_t k = 0; k < tg; k++) {
                    const size_t idx = (i * tg + k) * n + z;
                    col[k * n + zp] += bold_t[o][idx];
                    col[k * n + zb] += bold_t_bar[o][idx];
                }
            }
            for (size_t k = 0; k < K; k++) U[oz * K + k] = (uint32_t)(col[k] % ORC_Q);
        }
        free(col);
    }
}

/* ---------------------------------------------------------------- offline hint ring multiply (src/server.rs:656-768) */

/* answer_hint_ring for columns [c0, c1) of a column-order database (db[col * ld + r], rows records, rows % n == 0),
 * schoolbook: hint_col = sum over r < rows / n of perm(q_r) * D_{col,r} mod (X^n + 1, Q), where perm is util.rs
 * negacyclic_perm with shift 0 (perm(a)_0 = a_0, perm(a)_i = -a_{n-i}; the preprocessing of
 * generate_pseudorandom_query, src/server.rs:724-733) and D_{col,r} the polynomial of records [r n, (r + 1) n).  The
 * reference multiplies in the NTT domain and keeps the coefficient-domain sum (src/server.rs:674-697); with
 * perm_out the sum passes through negacyclic_perm once more (src/server.rs:699-705).  out[z * ostride + (col - c0)]. */
void orc_hint_ring(uint64_t *out, size_t ostride, const uint8_t *db, size_t ld, size_t rows, size_t c0, size_t c1,
                   const uint64_t *query, size_t n, int perm_out) {
    const size_t polys = rows / n;
    #pragma omp parallel for schedule(dynamic, 1)
    for (size_t col = c0; col < c1; col++) {
        uint64_t *pos = (uint64_t *)calloc(n, sizeof(uint64_t)), *neg = (uint64_t *)calloc(n, sizeof(uint64_t));
        uint64_t *a = (uint64_t *)malloc(n * sizeof(uint64_t));
        for (size_t p = 0; p < polys; p++) {
            const uint64_t *q = query + p * n;
            a[0] = q[0] % ORC_Q;
            for (size_t i = 1; i < n; i++) a[i] = (ORC_Q - q[n - i] % ORC_Q) % ORC_Q;
            const uint8_t *d = db + col * ld + p * n;
            for (size_t i = 0; i < n; i++) {
                for (size_t j = 0; j < n; j++) {
                    const uint64_t t = a[i] * d[j];           /* < 2^40 */
                    if (i + j < n) pos[i + j] += t; else neg[i + j - n] += t;  /* X^n = -1 */
                }
            }
            for (size_t k = 0; k < n; k++) { pos[k] %= ORC_Q; neg[k] %= ORC_Q; }  /* sums stay below 2^64 */
        }
        for (size_t z = 0; z < n; z++) {
            const size_t src = perm_out && z ? n - z : z;
            uint64_t v = (pos[src] + ORC_Q - neg[src]) % ORC_Q;
            if (perm_out && z) v = (ORC_Q - v) % ORC_Q;
            out[z * ostride + (col - c0)] = v;
        }
        free(pos); free(neg); free(a);
    }
}
