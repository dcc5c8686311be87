// offline.cuh -- the scheme's offline set-up on the device, for an engine whose database is resident: the hint's
// ring multiply kept in NTT form, the InspiRING precomputation of every output, the packing matrix, bold_t_hat and
// the row-0 prefixes (Prepared::new, src/service.rs:127-157; YServer::perform_offline_precomputation_simplepir,
// src/server.rs:947-1021; full_packing_with_preprocessing_offline, src/packing.rs:2260-2359).
//
// Ring Z_Q[X]/(X^n + 1).  NTT form: slot s holds the evaluation at psi^(2 brv(s) + 1) (Longa-Naehrig transforms of
// hint.cuh over the tables psi^brv, psi^-brv), the slot order of the reference's automorphism tables, under which
// tau_t acts as the permutation table_t[s] = brv(((t (2 brv(s) + 1)) mod 2n - 1) / 2).
//
// Per output o (n database columns, n = 2048 in the scheme) the reference computes
//   act[j]  = NTT(perm(hint column o n + j))                       prep_pack_lwes (src/packing.rs:910-942)
//   ev[v]   = NTT over j of act[j][v]                               precompute_aggregates_ntt (:2260-2291)
//   r_i     = n^-1 ev[table_(g^i)[s]][s],  rbar_i the same with 2n - g^i,  g = 5, i < n / 2
//   walk i = n/2 - 2 .. 0:  bold_t[i] = NTT(G^-1(r_(i+1))),  r_i += sum_k tau_(g^i)(w)[k] bold_t[i][k]
//                          (and the bar chain with tau_(2n - g^i) and w)          full_packing_offline_mode (:2301-2359)
//   bold_t_hat = NTT(G^-1(rbar_0)),  a_hat = r_0 + sum_k v[k] bold_t_hat[k] in coefficient form
// with G^-1 the base-2^b digits (b = floor(32 / tg) + 1, gadget_invert_transposed_alloc, :1468-1493).
//
// Two identities let the device skip work the reference does literally:
//   * perm (util.rs negacyclic_perm, shift 0) is the automorphism X -> X^-1, whose slot table is s -> n - 1 - s;
//     NTT(hint column) is the hint's accumulator before its inverse transform, so act[j][s] = acc_j[n - 1 - s];
//   * the packing-matrix fold (sw_pack_build) writes every (column z, slot s, digit k) once: the automorphism that
//     carries z to s is e = (2 brv(s) + 1) (2 brv(z) + 1)^-1 mod 2n, e = g^i or 2n - g^i, so each byte of the
//     matrix is a gather from bold_t or bold_t_bar instead of a scatter-add.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>
#include "hint.cuh"
#include "kernels.cuh"
#include "modq.cuh"

namespace alto {

constexpr int kActCols = 8;  // database columns per CTA of the act kernel: 8 u32 = one 32-byte sector per slot

__device__ __forceinline__ int brv_bits(int x, int logn) { return (int)(__brev((unsigned)x) >> (32 - logn)); }

// table_t[s] of the automorphism tau_t (t odd, < 2n)
__device__ __forceinline__ int auto_slot(int t, int s, int n, int logn) {
  const int e = (t * (2 * brv_bits(s, logn) + 1)) & (2 * n - 1);
  return brv_bits((e - 1) >> 1, logn);
}

// g^i mod 2n, or 2n - g^i for the bar chain (g = 5)
__device__ __forceinline__ int gen_pow(int i, int bar, int n) {
  int r = 1, b = 5;
  for (int k = i; k; k >>= 1) {
    if (k & 1) r = (r * b) & (2 * n - 1);
    b = (b * b) & (2 * n - 1);
  }
  return bar ? 2 * n - r : r;
}

// Forward transforms of `cnt` polynomials stored back to back in shared memory.
__device__ __forceinline__ void ntt_fwd_multi(uint32_t *a, int n, int cnt, const uint32_t *__restrict__ psi) {
  const int half = n >> 1;
  for (int m = 1, t = half; m < n; m <<= 1, t >>= 1) {
    for (int b = threadIdx.x; b < cnt * half; b += blockDim.x) {
      const int p = b / half, bb = b - p * half;
      const int i = bb / t, j = p * n + 2 * i * t + (bb - i * t);
      const uint32_t u = a[j], v = mul_q(a[j + t], __ldg(psi + m + i));
      a[j] = add_q(u, v);
      a[j + t] = sub_q(u, v);
    }
    __syncthreads();
  }
}

// acc = INTT(acc) (times n^-1), then its tg base-2^bits digits into dig[k n + s], all in shared memory.
__device__ __forceinline__ void digits_of(uint32_t *acc, uint32_t *dig, int n, int tg, int bits,
                                         const uint32_t *__restrict__ psi_inv, uint32_t n_inv) {
  hint_ntt_inv(acc, n, psi_inv);
  const uint32_t mask = bits >= 32 ? 0xffffffffu : (1u << bits) - 1u;
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    const uint32_t x = mul_q(acc[s], n_inv);
    for (int k = 0; k < tg; ++k) dig[k * n + s] = bits * k >= 32 ? 0u : (x >> (bits * k)) & mask;
  }
  __syncthreads();
}

// act, one CTA per kActCols consecutive database columns: acc_c = sum_p NTT(D_(p,c)) . qhat_p (qhat = NTT(perm(q_p))),
// stored as actT[o][s][j] = acc_c[n - 1 - s] for column c = o n + j.  Database columns come from the engine's tile
// layout as in hint_ring_kernel.
__global__ void __launch_bounds__(256) offline_act_kernel(const uint8_t *__restrict__ db, size_t kbs, int n,
                                                          int polys, const uint32_t *__restrict__ qhat,
                                                          const uint32_t *__restrict__ psi, uint32_t *__restrict__ act) {
  extern __shared__ uint32_t osm[];
  uint32_t *a = osm, *acc = osm + n;
  const size_t col0 = (size_t)blockIdx.x * kActCols;
  for (int i = threadIdx.x; i < kActCols * n; i += blockDim.x) acc[i] = 0;
  for (int c = 0; c < kActCols; ++c) {
    const size_t col = col0 + c;
    const uint8_t *row = db + (col / 128) * kbs * 16384 + (col % 128) * 128;
    for (int p = 0; p < polys; ++p) {
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const size_t rec = (size_t)p * n + i;
        a[i] = row[(rec >> 7) * 16384 + (rec & 127)];
      }
      __syncthreads();
      hint_ntt_fwd(a, n, psi);
      const uint32_t *qh = qhat + (size_t)p * n;
      for (int i = threadIdx.x; i < n; i += blockDim.x) acc[c * n + i] = add_q(acc[c * n + i], mul_q(a[i], __ldg(qh + i)));
    }
  }
  __syncthreads();
  const size_t o = col0 / n, j0 = col0 % n;  // kActCols divides n: the CTA's columns share their output
  for (int idx = threadIdx.x; idx < n * kActCols; idx += blockDim.x) {
    const int s = idx / kActCols, c = idx - s * kActCols;
    act[(o * n + s) * n + j0 + c] = acc[c * n + (n - 1 - s)];
  }
}

// Positions of a thread's 8 values in a round of s forward stages that starts at half-size t (n / 8 threads; each
// holds 8 / 2^s groups of 2^s values): group grp = g + q n/8 is block blk = grp / d, offset r = grp % d, d = 2t / 2^s,
// and its value b sits at blk 2t + r + b d.
template <int L>
__device__ __forceinline__ int fwd_pos(int g, int q, int b, int s, int t) {
  const int G = 1 << s, d = 2 * t / G, grp = g + q * ((1 << L) / 8);
  return (grp / d) * 2 * t + grp % d + b * d;
}

// One round of s Cooley-Tukey stages (Longa-Naehrig Algorithm 1) on the thread's values: stage k of the round has
// half-size t >> k and m << k blocks; its pairs are b, b + 2^(s-1-k) inside a group, twiddle psi[(m << k) + (blk << k) +
// (b >> (s - k))].
template <int L>
__device__ __forceinline__ void fwd_round(uint32_t (&x)[8], int g, int s, int m, int t,
                                          const uint32_t *__restrict__ psi) {
  const int G = 1 << s, d = 2 * t / G;
#pragma unroll
  for (int q = 0; q < 8 / G; ++q) {
    const int blk = (g + q * ((1 << L) / 8)) / d;
#pragma unroll
    for (int k = 0; k < s; ++k) {
      const int half = G >> (k + 1);
#pragma unroll
      for (int b = 0; b < G; ++b) {
        if (b & half) continue;
        const uint32_t w = __ldg(psi + (m << k) + (blk << k) + (b >> (s - k)));
        const uint32_t u = x[q * G + b], v = mul_q(x[q * G + b + half], w);
        x[q * G + b] = add_q(u, v);
        x[q * G + b + half] = sub_q(u, v);
      }
    }
  }
}

__device__ __forceinline__ int act_swz(int pos) { return pos ^ ((pos >> 5) & 31); }

// The act kernel with the transforms in registers: n / 8 threads, 8 values each, three stages per round and one
// shared-memory exchange between rounds (double-buffered: one barrier an exchange), against a barrier per stage in
// offline_act_kernel; ACOLS columns a CTA.  Same output.
template <int L, int ACOLS>
__global__ void __launch_bounds__((1 << L) / 8) offline_act8_kernel(const uint8_t *__restrict__ db, size_t kbs,
                                                                     int polys, const uint32_t *__restrict__ qhat,
                                                                     const uint32_t *__restrict__ psi,
                                                                     uint32_t *__restrict__ act) {
  constexpr int n = 1 << L, NT = n / 8;
  static_assert(ACOLS >= 1 && n % ACOLS == 0, "columns per CTA");
  extern __shared__ uint32_t osm[];
  uint32_t *accs = osm + 2 * n;  // [column in CTA][position]
  const int g = threadIdx.x;
  const size_t col0 = (size_t)blockIdx.x * ACOLS;
  int ex = 0;  // exchanges so far: buffer ex & 1
  for (int c = 0; c < ACOLS; ++c) {
    const size_t col = col0 + c;
    const uint8_t *row = db + (col / 128) * kbs * 16384 + (col % 128) * 128;
    uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = 0; p < polys; ++p) {
      uint32_t x[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) {  // the first round's positions: g + b n / 8
        const size_t rec = (size_t)p * n + g + b * NT;
        x[b] = row[(rec >> 7) * 16384 + (rec & 127)];
      }
#pragma unroll
      for (int s0 = 0; s0 < L; s0 += 3) {
        const int s = (L - s0) < 3 ? (L - s0) : 3, t = n >> (s0 + 1);
        if (s0 > 0) {
          const int ps = 3, pt = n >> (s0 - 3 + 1);  // every round before the last has three stages
          uint32_t *buf = osm + (ex & 1) * n;
#pragma unroll
          for (int q = 0; q < 8 / (1 << ps); ++q)
#pragma unroll
            for (int b = 0; b < (1 << ps); ++b) buf[act_swz(fwd_pos<L>(g, q, b, ps, pt))] = x[q * (1 << ps) + b];
          __syncthreads();
#pragma unroll
          for (int q = 0; q < 8 / (1 << s); ++q)
#pragma unroll
            for (int b = 0; b < (1 << s); ++b) x[q * (1 << s) + b] = buf[act_swz(fwd_pos<L>(g, q, b, s, t))];
          ++ex;
        }
        fwd_round<L>(x, g, s, 1 << s0, t, psi);
      }
      constexpr int ls = (L % 3) ? (L % 3) : 3, lt = n >> (L - ls + 1);  // the last round
      const uint32_t *qh = qhat + (size_t)p * n;
#pragma unroll
      for (int q = 0; q < 8 / (1 << ls); ++q)
#pragma unroll
        for (int b = 0; b < (1 << ls); ++b) {
          const int i = q * (1 << ls) + b;
          acc[i] = add_q(acc[i], mul_q(x[i], __ldg(qh + fwd_pos<L>(g, q, b, ls, lt))));
        }
    }
#pragma unroll
    for (int q = 0; q < 8 / (1 << ((L % 3) ? (L % 3) : 3)); ++q) {
      constexpr int ls = (L % 3) ? (L % 3) : 3, lt = n >> (L - ls + 1);
#pragma unroll
      for (int b = 0; b < (1 << ls); ++b) accs[c * n + fwd_pos<L>(g, q, b, ls, lt)] = acc[q * (1 << ls) + b];
    }
  }
  __syncthreads();
  const size_t o = col0 / n, j0 = col0 % n;
  for (int idx = threadIdx.x; idx < n * ACOLS; idx += NT) {
    const int s = idx / ACOLS, c = idx - s * ACOLS;
    act[(o * n + s) * n + j0 + c] = accs[c * n + (n - 1 - s)];
  }
}

// ev: forward transform of every row of act in place (one CTA per row of n).
__global__ void __launch_bounds__(256) offline_rows_kernel(uint32_t *__restrict__ rows, int n,
                                                           const uint32_t *__restrict__ psi) {
  extern __shared__ uint32_t osm[];
  uint32_t *r = rows + (size_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) osm[i] = r[i];
  __syncthreads();
  hint_ntt_fwd(osm, n, psi);
  for (int i = threadIdx.x; i < n; i += blockDim.x) r[i] = osm[i];
}

// The backward walk, one CTA per (output o, chain bar): bar 0 walks r with tau_(g^i)(w), bar 1 walks rbar with
// tau_(2n - g^i)(w).  bt[((o 2 + bar) (n/2 - 1) + i) tg + k][s] = bold_t (bar 0) or bold_t_bar (bar 1); the chain's
// final r_0 (rbar_0) goes to last[(o 2 + bar) n + s].
__global__ void __launch_bounds__(1024) offline_walk_kernel(const uint32_t *__restrict__ ev, int n, int logn, int tg,
                                                            int bits, const uint32_t *__restrict__ w,
                                                            const uint32_t *__restrict__ psi,
                                                            const uint32_t *__restrict__ psi_inv, uint32_t n_inv,
                                                            uint32_t *__restrict__ bt, uint32_t *__restrict__ last) {
  extern __shared__ uint32_t osm[];
  uint32_t *cur = osm, *dig = osm + n;
  const int o = blockIdx.x >> 1, bar = blockIdx.x & 1, half = n >> 1;
  const uint32_t *evo = ev + (size_t)o * n * n;
  int e = gen_pow(half - 1, bar, n);
  for (int s = threadIdx.x; s < n; s += blockDim.x) cur[s] = mul_q(evo[(size_t)auto_slot(e, s, n, logn) * n + s], n_inv);
  __syncthreads();
  for (int i = half - 2; i >= 0; --i) {
    digits_of(cur, dig, n, tg, bits, psi_inv, n_inv);
    ntt_fwd_multi(dig, n, tg, psi);
    e = gen_pow(i, bar, n);
    uint32_t *out = bt + (((size_t)(o * 2 + bar) * (half - 1) + i) * tg) * n;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
      const int ts = auto_slot(e, s, n, logn);
      uint32_t acc = mul_q(evo[(size_t)ts * n + s], n_inv);
      for (int k = 0; k < tg; ++k) {
        const uint32_t d = dig[k * n + s];
        out[k * n + s] = d;
        acc = add_q(acc, mul_q(__ldg(w + k * n + ts), d));
      }
      cur[s] = acc;
    }
    __syncthreads();
  }
  for (int s = threadIdx.x; s < n; s += blockDim.x) last[(size_t)(o * 2 + bar) * n + s] = cur[s];
}

// The same walk with one thread-block cluster of C CTAs per (output, chain): every CTA runs the step's inverse
// transform (the same values in each), takes the digits k = c, c + C, ... of its rank c, transforms them and forms
// its part of sum_k tau(w)[k] bold_t[i][k]; the parts are summed through distributed shared memory.  A step costs
// two transforms instead of 1 + tg.  Launched with cluster dimensions (C, 1, 1): CTAs C q .. C q + C - 1 are chain q.
__global__ void __launch_bounds__(1024) offline_walk_cluster_kernel(const uint32_t *__restrict__ ev, int n, int logn,
                                                                    int tg, int bits, const uint32_t *__restrict__ w,
                                                                    const uint32_t *__restrict__ psi,
                                                                    const uint32_t *__restrict__ psi_inv,
                                                                    uint32_t n_inv, uint32_t *__restrict__ bt,
                                                                    uint32_t *__restrict__ last) {
  namespace cg = cooperative_groups;
  extern __shared__ uint32_t osm[];
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), c = (int)cl.block_rank();
  const int chain = blockIdx.x / C, o = chain >> 1, bar = chain & 1, half = n >> 1;
  const int kper = (tg + C - 1) / C;
  uint32_t *cur = osm, *part = osm + n, *dig = osm + 2 * n;
  const uint32_t mask = bits >= 32 ? 0xffffffffu : (1u << bits) - 1u;
  const uint32_t *evo = ev + (size_t)o * n * n;
  int e = gen_pow(half - 1, bar, n);
  for (int s = threadIdx.x; s < n; s += blockDim.x) cur[s] = mul_q(evo[(size_t)auto_slot(e, s, n, logn) * n + s], n_inv);
  __syncthreads();
  constexpr int kAgg = 4;  // slots a thread gathers ahead (n <= kAgg blockDim.x)
  for (int i = half - 2; i >= 0; --i) {
    // this step's aggregate r_i, loaded before the transforms so that its latency hides behind them
    e = gen_pow(i, bar, n);
    uint32_t agg[kAgg];
#pragma unroll
    for (int j = 0; j < kAgg; ++j) {
      const int s = threadIdx.x + j * (int)blockDim.x;
      agg[j] = s < n ? evo[(size_t)auto_slot(e, s, n, logn) * n + s] : 0u;
    }
    hint_ntt_inv(cur, n, psi_inv);
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
      const uint32_t x = mul_q(cur[s], n_inv);
      for (int j = 0; j < kper; ++j) {
        const int k = c + C * j;
        dig[j * n + s] = (k < tg && bits * k < 32) ? (x >> (bits * k)) & mask : 0u;
      }
    }
    __syncthreads();
    ntt_fwd_multi(dig, n, kper, psi);
    uint32_t *out = bt + (((size_t)chain * (half - 1) + i) * tg) * n;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
      const int ts = auto_slot(e, s, n, logn);
      uint32_t p = 0;
      for (int j = 0; j < kper; ++j) {
        const int k = c + C * j;
        if (k < tg) {
          const uint32_t d = dig[j * n + s];
          out[k * n + s] = d;
          p = add_q(p, mul_q(__ldg(w + k * n + ts), d));
        }
      }
      part[s] = p;
    }
    cl.sync();  // every CTA's part is written
#pragma unroll
    for (int j = 0; j < kAgg; ++j) {
      const int s = threadIdx.x + j * (int)blockDim.x;
      if (s >= n) break;
      uint32_t acc = mul_q(agg[j], n_inv);
      for (int r = 0; r < C; ++r) acc = add_q(acc, cl.map_shared_rank(part, r)[s]);
      cur[s] = acc;
    }
    cl.sync();  // every CTA has read the parts (they are rewritten next step) and holds the whole new r_i
  }
  if (c == 0)
    for (int s = threadIdx.x; s < n; s += blockDim.x) last[(size_t)chain * n + s] = cur[s];
}

// The cluster walk with both transforms in registers, for tg CTAs a cluster (one digit each) and n = 2^L: n / 8
// threads hold 8 values each.  The inverse transform runs the tail kernel's Gentleman-Sande rounds (tail_round: the
// thread's 8 consecutive slots first, then three stages per shared-memory exchange); the digit goes back through
// shared memory in natural order and the forward transform runs fwd_round's Cooley-Tukey rounds; the thread then holds
// slots 8 g .. 8 g + 7 of the next r_i in registers.  Every exchange is double-buffered (one barrier each).
template <int L>
__global__ void __launch_bounds__((1 << L) / 8) offline_walk8_kernel(const uint32_t *__restrict__ ev, int tg,
                                                                     int bits, const uint32_t *__restrict__ w,
                                                                     const uint32_t *__restrict__ psi,
                                                                     const uint32_t *__restrict__ psi_inv,
                                                                     uint32_t n_inv, uint32_t *__restrict__ bt,
                                                                     uint32_t *__restrict__ last) {
  namespace cg = cooperative_groups;
  constexpr int n = 1 << L, NT = n / 8;
  constexpr int ls = (L % 3) ? (L % 3) : 3, lt = n >> (L - ls + 1);  // the forward transform's last round
  extern __shared__ uint32_t osm[];
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), k = (int)cl.block_rank();  // this CTA's digit
  const int chain = blockIdx.x / C, o = chain >> 1, bar = chain & 1, half = n >> 1, g = threadIdx.x;
  // parts[buffer][rank][slot]: every CTA pushes its share into every CTA's buffer (remote stores do not stall the
  // thread, where remote loads would), and the buffers alternate by step, so one cluster barrier a step suffices
  uint32_t *parts = osm + 2 * n;
  int pb = 0;
  const uint32_t mask = bits >= 32 ? 0xffffffffu : (1u << bits) - 1u;
  const uint32_t *evo = ev + (size_t)o * n * n;
  int ex = 0;
  uint32_t x[8];
  int e = gen_pow(half - 1, bar, n);
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int sl = 8 * g + m;
    x[m] = mul_q(evo[(size_t)auto_slot(e, sl, n, L) * n + sl], n_inv);
  }
  for (int i = half - 2; i >= 0; --i) {
    // this step's aggregate r_i (gathered from ev), loaded now so that its latency hides behind the transforms
    e = gen_pow(i, bar, n);
    uint32_t agg[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int sl = 8 * g + m;
      agg[m] = evo[(size_t)auto_slot(e, sl, n, L) * n + sl];
    }
    // inverse transform (without n^-1)
    tail_round<L>(x, g, 0, 3, psi_inv);
#pragma unroll
    for (int s0 = 3; s0 < L; s0 += 3) {
      const int r = (L - s0) < 3 ? (L - s0) : 3;
      uint32_t *buf = osm + (ex++ & 1) * n;
#pragma unroll
      for (int m = 0; m < 8; ++m) buf[tail_swz(tail_index<L>(g, m, s0 - 3, 3))] = x[m];
      __syncthreads();
#pragma unroll
      for (int gi = 0; gi < (8 >> r); ++gi) {
        uint32_t *y = x + gi * (1 << r);
#pragma unroll
        for (int m = 0; m < (1 << r); ++m) y[m] = buf[tail_swz(tail_index<L>(gi * NT + g, m, s0, r))];
        tail_round<L>(y, gi * NT + g, s0, r, psi_inv);
      }
    }
    // this CTA's digit, in natural order, to the forward transform's first-round layout
    {
      constexpr int s0l = ((L - 1) / 3) * 3, rl = L - s0l;
      uint32_t *buf = osm + (ex++ & 1) * n;
#pragma unroll
      for (int gi = 0; gi < (8 >> rl); ++gi)
#pragma unroll
        for (int m = 0; m < (1 << rl); ++m) {
          const uint32_t v = mul_q(x[gi * (1 << rl) + m], n_inv);
          buf[act_swz(tail_index<L>(gi * NT + g, m, s0l, rl))] =
              (k < tg && bits * k < 32) ? (v >> (bits * k)) & mask : 0u;
        }
      __syncthreads();
#pragma unroll
      for (int b = 0; b < 8; ++b) x[b] = buf[act_swz(g + b * NT)];
    }
    fwd_round<L>(x, g, 3, 1, n >> 1, psi);
#pragma unroll
    for (int s0 = 3; s0 < L; s0 += 3) {
      const int sr = (L - s0) < 3 ? (L - s0) : 3, t = n >> (s0 + 1), pt = n >> (s0 - 2);
      uint32_t *buf = osm + (ex++ & 1) * n;
#pragma unroll
      for (int b = 0; b < 8; ++b) buf[act_swz(fwd_pos<L>(g, 0, b, 3, pt))] = x[b];
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 8 / (1 << sr); ++q)
#pragma unroll
        for (int b = 0; b < (1 << sr); ++b) x[q * (1 << sr) + b] = buf[act_swz(fwd_pos<L>(g, q, b, sr, t))];
      fwd_round<L>(x, g, sr, 1 << s0, t, psi);
    }
    // bold_t[i][k], this CTA's share of the rotated sum, then the next r_i from every CTA's share
    uint32_t *out = bt + (((size_t)chain * (half - 1) + i) * tg + k) * n;
#pragma unroll
    for (int q = 0; q < 8 / (1 << ls); ++q)
#pragma unroll
      for (int b = 0; b < (1 << ls); ++b) {
        const int pos = fwd_pos<L>(g, q, b, ls, lt);
        const uint32_t d = x[q * (1 << ls) + b];
        if (k < tg) out[pos] = d;
        const uint32_t v = k < tg ? mul_q(__ldg(w + k * n + auto_slot(e, pos, n, L)), d) : 0u;
        for (int r = 0; r < C; ++r) cl.map_shared_rank(parts + ((size_t)pb * C + k) * n, r)[pos] = v;
      }
    cl.sync();  // every share has arrived in every CTA
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int sl = 8 * g + m;
      uint32_t acc = mul_q(agg[m], n_inv);
      for (int r = 0; r < C; ++r) acc = add_q(acc, parts[((size_t)pb * C + r) * n + sl]);
      x[m] = acc;
    }
    pb ^= 1;
  }
  cl.sync();  // no CTA exits while another may still write into its shared memory
  if (k == 0)
#pragma unroll
    for (int m = 0; m < 8; ++m) last[(size_t)chain * n + 8 * g + m] = x[m];
}

// Per output (one CTA each): bold_t_hat = NTT(G^-1(rbar_0)); a_hat = INTT(r_0 + sum_k v[k] bold_t_hat[k]).  Writes
// the engine's bold_t_hat (times the tail's scale 2^-log2 n), the row-0 prefix (a_hat rescaled to 2^q2_bits, packed
// LSB first, the rest of the part zero: switch_prefix_row0, src/modulus_switch.rs:136-147) and, for callers that
// ask, the plain bold_t_hat and a_hat.
__global__ void __launch_bounds__(1024) offline_finish_kernel(const uint32_t *__restrict__ last, int n, int tg,
                                                              int bits, const uint32_t *__restrict__ v,
                                                              const uint32_t *__restrict__ psi,
                                                              const uint32_t *__restrict__ psi_inv, uint32_t n_inv,
                                                              uint32_t tail_scale, uint32_t *__restrict__ that_eng,
                                                              uint8_t *__restrict__ prefix, size_t part_len,
                                                              int q2_bits, uint32_t *__restrict__ that_out,
                                                              uint32_t *__restrict__ a_hat_out) {
  extern __shared__ uint32_t osm[];
  uint32_t *cur = osm, *dig = osm + n;
  const int o = blockIdx.x;
  const size_t count = (size_t)tg * n;
  for (int s = threadIdx.x; s < n; s += blockDim.x) cur[s] = last[(size_t)(o * 2 + 1) * n + s];
  __syncthreads();
  digits_of(cur, dig, n, tg, bits, psi_inv, n_inv);
  ntt_fwd_multi(dig, n, tg, psi);
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    uint32_t acc = last[(size_t)(o * 2) * n + s];
    for (int k = 0; k < tg; ++k) {
      const uint32_t t = dig[k * n + s];
      acc = add_q(acc, mul_q(__ldg(v + k * n + s), t));
      that_eng[o * count + k * n + s] = mul_q(t, tail_scale);
      if (that_out) that_out[o * count + k * n + s] = t;
    }
    cur[s] = acc;
  }
  __syncthreads();
  hint_ntt_inv(cur, n, psi_inv);
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    cur[s] = mul_q(cur[s], n_inv);
    if (a_hat_out) a_hat_out[(size_t)o * n + s] = cur[s];
  }
  __syncthreads();
  // rescale(a, Q, 2^q2_bits): centre, round half away from zero, reduce (src/modulus_switch.rs:116-130)
  const int64_t q = kQ32, half = kQ32 / 2, q2 = int64_t(1) << q2_bits;
  uint8_t *pre = prefix + (size_t)o * part_len;
  const size_t row0_bytes = ((size_t)q2_bits * n + 7) / 8;
  for (size_t b = row0_bytes + threadIdx.x; b < part_len; b += blockDim.x) pre[b] = 0;
  // 8 values of q2_bits bits fill q2_bits whole bytes: thread g packs values 8 g .. 8 g + 7
  for (int g = threadIdx.x; g < n / 8; g += blockDim.x) {
    uint8_t bytes[64] = {};
    for (int u = 0; u < 8; ++u) {
      const int64_t a = cur[8 * g + u];
      const int64_t c = a >= half ? a - q : a;
      int64_t t = (c * q2 + (c >= 0 ? half : -half)) / q;
      t = ((t % q2) + q2) % q2;
      for (int bit = 0; bit < q2_bits; ++bit)
        if ((t >> bit) & 1) bytes[(u * q2_bits + bit) >> 3] |= (uint8_t)(1u << ((u * q2_bits + bit) & 7));
    }
    for (int k = 0; k < q2_bits; ++k) pre[(size_t)g * q2_bits + k] = bytes[k];
  }
}

// The packing matrix in the engine's tile layout, one thread per value (engine column col, key word kk):
// U[col][kk] = bold_t[o][i][k][z] (or bold_t_bar) for the automorphism carrying z to s (see the file comment), zero
// for the two slots no automorphism of the walk reaches; times tail_scale; its 4 bytes go to planes col 4 + j,
// tile (row / 128, kk / 128) at (mt kbs + kb) 16 KB, byte (row % 128) 128 + kk % 128.
__global__ void __launch_bounds__(256) offline_planes_kernel(const uint32_t *__restrict__ bt, int n, int logn, int tg,
                                                             size_t cols, const int16_t *__restrict__ dlog,
                                                             const uint16_t *__restrict__ inv_odd,
                                                             uint32_t tail_scale, uint8_t *__restrict__ ub,
                                                             size_t kbs) {
  const size_t K = (size_t)tg * n;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= cols * K) return;
  const size_t col = idx / K, kk = idx - col * K;
  const int o = (int)(col / n), z = (int)(col % n), k = (int)(kk / n), s = (int)(kk % n), half = n >> 1;
  const int t = ((2 * brv_bits(s, logn) + 1) * (int)__ldg(inv_odd + brv_bits(z, logn))) & (2 * n - 1);
  const int d = __ldg(dlog + ((t - 1) >> 1));
  uint32_t v = 0;
  if (d >= 0 && (d >> 1) <= half - 2)
    v = mul_q(__ldg(bt + (((size_t)(o * 2 + (d & 1)) * (half - 1) + (d >> 1)) * tg + k) * n + z), tail_scale);
  for (int j = 0; j < 4; ++j) {
    const size_t row = col * 4 + j;
    ub[((row >> 7) * kbs + (kk >> 7)) * 16384 + (row & 127) * 128 + (kk & 127)] = (uint8_t)(v >> (8 * j));
  }
}

}  // namespace alto
