// hint.cuh -- the ring multiply of the offline hint on the device: for every database column, the sum over its
// polynomials of a (preprocessed) query polynomial times the column's polynomial, modulo X^n + 1 and Q
// (YServer::answer_hint_ring / multiply_with_db_ring, src/server.rs:656-768).  It runs once per database, at set-up.
//
// The reference multiplies in spiral-rs's NTT domain; the result it keeps is in the coefficient domain, so any
// matched negacyclic transform pair gives the same bytes.  This one is the Cooley-Tukey forward / Gentleman-Sande
// inverse pair with powers of a primitive 2n-th root of unity psi in bit-reversed order (P. Longa and M. Naehrig,
// "Speeding up the Number Theoretic Transform for Faster Ideal Lattice-Based Cryptography", CANS 2016, Algorithms 1
// and 2); n^-1 is folded into the transformed query.  All arithmetic is exact mod Q (modq.cuh).
#pragma once
#include <cstdint>
#include "modq.cuh"

namespace alto {

// Forward negacyclic NTT of a[0..n) in shared memory (standard order in, bit-reversed order out); nt threads.
__device__ __forceinline__ void hint_ntt_fwd(uint32_t *a, int n, const uint32_t *__restrict__ psi) {
  for (int m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1) {
    for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
      const int i = b / t, j = 2 * i * t + (b - i * t);
      const uint32_t u = a[j], v = mul_q(a[j + t], __ldg(psi + m + i));
      a[j] = add_q(u, v);
      a[j + t] = sub_q(u, v);
    }
    __syncthreads();
  }
}

// Inverse (bit-reversed in, standard out), without the final n^-1.
__device__ __forceinline__ void hint_ntt_inv(uint32_t *a, int n, const uint32_t *__restrict__ psi_inv) {
  for (int t = 1, h = n >> 1; t < n; t <<= 1, h >>= 1) {
    for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
      const int i = b / t, j = 2 * i * t + (b - i * t);
      const uint32_t u = a[j], v = a[j + t];
      a[j] = add_q(u, v);
      a[j + t] = mul_q(sub_q(u, v), __ldg(psi_inv + h + i));
    }
    __syncthreads();
  }
}

// The query's preprocessing, one CTA per polynomial: perm(q)[0] = q[0], perm(q)[i] = -q[n - i] (util.rs
// negacyclic_perm with shift 0), then the forward transform, times n^-1.
__global__ void hint_query_kernel(const uint64_t *__restrict__ query, int n, const uint32_t *__restrict__ psi,
                                  uint32_t n_inv, uint32_t *__restrict__ qhat) {
  extern __shared__ uint32_t hsm[];
  const uint64_t *q = query + (size_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t v = red_q64(q[i == 0 ? 0 : n - i]);
    hsm[i] = i == 0 ? v : sub_q(0, v);
  }
  __syncthreads();
  hint_ntt_fwd(hsm, n, psi);
  for (int i = threadIdx.x; i < n; i += blockDim.x) qhat[(size_t)blockIdx.x * n + i] = mul_q(hsm[i], n_inv);
}

// One CTA per database column `col`: acc = sum over its `polys` polynomials r of NTT(D_r) . qhat_r (pointwise), then
// the inverse transform; out[z * cols + col] = acc_z, or perm(acc)_z when perm_out.  D_r is records
// [r n, (r + 1) n) of the column, read from the engine's tile layout (tile (mt, kb) at (mt * kbs + kb) * 16 KB, its
// row col % 128 holding records [128 kb, 128 kb + 128)).
__global__ void hint_ring_kernel(const uint8_t *__restrict__ db, size_t kbs, int n, int polys,
                                 const uint32_t *__restrict__ qhat, const uint32_t *__restrict__ psi,
                                 const uint32_t *__restrict__ psi_inv, uint64_t *__restrict__ out, size_t cols,
                                 int perm_out) {
  extern __shared__ uint32_t hsm[];
  uint32_t *a = hsm, *acc = hsm + n;
  const size_t col = blockIdx.x, mt = col / 128, r = col % 128;
  const uint8_t *row = db + mt * kbs * 16384 + r * 128;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc[i] = 0;
  for (int p = 0; p < polys; ++p) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const size_t rec = (size_t)p * n + i;
      a[i] = row[(rec >> 7) * 16384 + (rec & 127)];
    }
    __syncthreads();
    hint_ntt_fwd(a, n, psi);
    const uint32_t *qh = qhat + (size_t)p * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc[i] = add_q(acc[i], mul_q(a[i], __ldg(qh + i)));
    // the next polynomial's load writes only a[i] of this thread's own i, read above by this thread alone
  }
  __syncthreads();
  hint_ntt_inv(acc, n, psi_inv);
  for (int z = threadIdx.x; z < n; z += blockDim.x) {
    uint32_t v = acc[z];
    if (perm_out && z) v = sub_q(0, acc[n - z]);
    out[(size_t)z * cols + col] = v;
  }
}

// Host: the smallest primitive 2n-th root of unity psi mod Q (2n must divide Q - 1 = 2^12 * 1048573, so n <= 2048)
// and the transform tables psi[k] = psi^brv(k), psi_inv[k] = psi^-brv(k) (brv = bit reversal of log2 n bits).
inline bool hint_tables(int n, std::vector<uint32_t> &psi, std::vector<uint32_t> &psi_inv, uint32_t &n_inv) {
  if (n < 2 || (n & (n - 1)) || (uint64_t)(kQ32 - 1) % (2 * (uint64_t)n)) return false;
  auto pow_q = [](uint32_t b, uint64_t e) {
    uint32_t r = 1;
    while (e) {
      if (e & 1) r = mul_q(r, b);
      b = mul_q(b, b);
      e >>= 1;
    }
    return r;
  };
  uint32_t any = 0;
  for (uint32_t g = 2; g < 1000 && !any; ++g) {
    const uint32_t c = pow_q(g, (kQ32 - 1) / (2 * (uint64_t)n));
    if (pow_q(c, (uint64_t)n) == kQ32 - 1) any = c;  // order exactly 2n
  }
  if (!any) return false;
  // the smallest primitive 2n-th root: the odd powers of any one are all of them
  uint32_t root = any, x = any;
  const uint32_t sq = mul_q(any, any);
  for (int k = 3; k < 2 * n; k += 2) {
    x = mul_q(x, sq);
    root = x < root ? x : root;
  }
  const uint32_t root_inv = pow_q(root, kQ32 - 2);
  int logn = 0;
  while ((1 << logn) < n) ++logn;
  psi.assign(n, 0);
  psi_inv.assign(n, 0);
  for (int k = 0; k < n; ++k) {
    int rev = 0;
    for (int b = 0; b < logn; ++b)
      if (k >> b & 1) rev |= 1 << (logn - 1 - b);
    psi[k] = pow_q(root, rev);
    psi_inv[k] = pow_q(root_inv, rev);
  }
  n_inv = inv_pow2_q(logn);
  return true;
}

}  // namespace alto
