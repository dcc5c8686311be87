// kernels.cuh -- the non-GEMM kernels of the answer path: request validation, byte-limb split of the query and
// key words, and the vector tail (key-switch accumulate, inverse NTT, modulus switch, 10-bit packing).
#pragma once
#include <cstdint>
#include "limb_gemm.cuh"

namespace alto {

// ------------------------------------------------------------------------------------ validate
// One CTA per staged frame; the frame starts `lead` bytes into its slot so that its key words (frame offset 9) are
// 16-byte aligned.  Status 2 for a flag byte != 0 or a key count != tg * n (src/amx_kernels.cpp:575), 3 for any of
// the 2 * count y/z key words >= Q (src/amx_kernels.cpp:576-580), else 0.  Query words are not range-checked, as in
// the reference.  Status 1 (length) is settled by the host before a frame is staged.
__global__ void validate_kernel(const uint8_t *__restrict__ slots, size_t stride, size_t lead, size_t count,
                                size_t rows, int *__restrict__ status) {
  (void)rows;
  const uint8_t *f = slots + (size_t)blockIdx.x * stride + lead;
  const uint32_t c1 = (uint32_t)f[1] | ((uint32_t)f[2] << 8) | ((uint32_t)f[3] << 16) | ((uint32_t)f[4] << 24);
  const uint32_t c2 = (uint32_t)f[5] | ((uint32_t)f[6] << 8) | ((uint32_t)f[7] << 16) | ((uint32_t)f[8] << 24);
  if (f[0] != 0 || (size_t)c1 != count || (size_t)c2 != count) {
    if (threadIdx.x == 0) status[blockIdx.x] = 2;
    return;
  }
  const uint4 *p = reinterpret_cast<const uint4 *>(f + 9);
  int bad = 0;
  for (size_t i = threadIdx.x; i < 2 * count / 4; i += blockDim.x) {
    const uint4 v = p[i];
    bad |= (v.x >= (uint32_t)kQ) | (v.y >= (uint32_t)kQ) | (v.z >= (uint32_t)kQ) | (v.w >= (uint32_t)kQ);
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) status[blockIdx.x] = bad ? 3 : 0;
}

// ------------------------------------------------------------------------------------ limb split
// dst[(c * 4 + j) * words + k] = byte j of word k of slot c, for c < padded (zero rows for c >= slots).  This is
// the K-major B operand of the limb GEMMs.  Each thread moves 16 words (64 bytes in, four 16-byte rows out).
__global__ void limb_split_kernel(const uint8_t *__restrict__ req, size_t stride, size_t word_off, int slots,
                                  int padded, size_t words, uint8_t *__restrict__ dst) {
  const size_t groups = words / 16;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= groups * (size_t)padded) return;
  const int c = (int)(idx / groups);
  const size_t g = idx % groups;
  uint32_t o[4][4];
  if (c < slots) {
    const uint4 *src = reinterpret_cast<const uint4 *>(req + (size_t)c * stride + word_off + g * 64);
    uint32_t w[16];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const uint4 t = src[v];
      w[4 * v] = t.x; w[4 * v + 1] = t.y; w[4 * v + 2] = t.z; w[4 * v + 3] = t.w;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t sel = (uint32_t)j | ((uint32_t)(4 + j) << 4);  // bytes j of the two inputs into bytes 0, 1
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t lo = __byte_perm(w[4 * q], w[4 * q + 1], sel);
        const uint32_t hi = __byte_perm(w[4 * q + 2], w[4 * q + 3], sel);
        o[j][q] = __byte_perm(lo, hi, 0x5410);
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) o[j][q] = 0;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
    *reinterpret_cast<uint4 *>(dst + ((size_t)c * 4 + j) * words + g * 16) = make_uint4(o[j][0], o[j][1], o[j][2], o[j][3]);
}

// ------------------------------------------------------------------------------------ tail
__device__ __forceinline__ uint32_t mulmod_q(uint32_t a, uint32_t b) {
  return (uint32_t)mod_q64((uint64_t)a * b);
}
__device__ __forceinline__ uint32_t addmod_q(uint32_t a, uint32_t b) {
  const uint64_t s = (uint64_t)a + b;
  return (uint32_t)(s >= kQ ? s - kQ : s);
}

// Centred rescale Q -> q1 with round-half-away-from-zero into [0, q1) (src/amx_kernels.cpp:522-529).  The reference
// divides in double precision; |c * q1 +- floor(Q/2)| < 2^53 and the quotient's rounding cannot cross an integer,
// so truncating 64-bit integer division by the constant Q gives the same integer.
__device__ __forceinline__ uint32_t rescale_q1(uint32_t v, int64_t q1) {
  constexpr int64_t half = (int64_t)(kQ / 2);
  const bool neg = v >= (uint32_t)half;
  const int64_t c = neg ? (int64_t)v - (int64_t)kQ : (int64_t)v;
  int64_t t = (c * q1 + (neg ? -half : half)) / (int64_t)kQ;
  if (t < 0) t += q1;
  if (t >= q1) t -= q1;
  return (uint32_t)t;
}

struct TailArgs {
  const uint32_t *acc;      // scan sums mod 2^32, [slot][cols]
  const uint32_t *beta;     // pack results mod Q, [slot][cols]
  const int *status;        // per-slot status; only slots with status 0 are answered
  const uint8_t *req;       // staged request bodies (y, z, q words), [slot][req_stride]
  size_t req_stride;
  size_t z_off;             // byte offset of the z key words within a body
  const uint32_t *that;     // bold_t_hat mod Q, [output][tg * n]
  const uint32_t *twiddle;  // inverse-NTT table, low 32 bits of each entry, [n]
  const uint8_t *prefix;    // row-0 prefixes, [output][part_len]
  uint8_t *resp;            // responses: slot s, part o at resp + s * resp_stride + o * part_len
  size_t resp_stride;
  int n, tg, outputs, cols;
  int part_len, row1_off, q1_bits;
  int64_t q1;
};

// One CTA per (slot, output).  Shared memory: n accumulator words, then the response part as 32-bit words.
// acc[i] = beta + sum_k z[k n + i] * that[k n + i] (mod Q)    (src/amx_kernels.cpp:500-511)
// inverse NTT, stages t = 1..n/2, twiddle table[n/(2t) + block], x' = (x+y)/2, y' = (x-y)w   (:461-498)
// v = rescale(inter + acc) with inter = (acc_scan * Q + 2^31) >> 32 (:306-307, :515-529)
// part = prefix with the q1_bits-bit values ORed in LSB-first from bit row1_off (:530-534, :605-607)
__global__ void __launch_bounds__(256) tail_kernel(TailArgs a) {
  extern __shared__ uint32_t tsm[];
  const int slot = blockIdx.x / a.outputs, o = blockIdx.x % a.outputs;
  if (a.status[slot] != 0) return;  // rejected frames get no response (their output stays untouched)
  const int n = a.n, tid = threadIdx.x, nt = blockDim.x;
  uint32_t *acc = tsm;
  uint32_t *res = tsm + n;
  const int res_words = (a.part_len + 3) / 4 + 1;
  const size_t count = (size_t)a.tg * n;
  const uint32_t *z = reinterpret_cast<const uint32_t *>(a.req + (size_t)slot * a.req_stride + a.z_off);
  const uint32_t *th = a.that + (size_t)o * count;
  const size_t base = (size_t)slot * a.cols + (size_t)o * n;

  for (int i = tid; i < n; i += nt) {
    uint32_t s = a.beta[base + i];
    for (int k = 0; k < a.tg; ++k) s = addmod_q(s, mulmod_q(z[(size_t)k * n + i], th[(size_t)k * n + i]));
    acc[i] = s;
  }
  const uint8_t *pre = a.prefix + (size_t)o * a.part_len;
  for (int w = tid; w < res_words; w += nt) {
    uint32_t v = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int idx = 4 * w + b;
      if (idx < a.part_len) v |= (uint32_t)pre[idx] << (8 * b);
    }
    res[w] = v;
  }
  __syncthreads();

  for (int t = 1; t < n; t <<= 1) {
    const int h = n / (2 * t);
    for (int b = tid; b < n / 2; b += nt) {
      const int blk = b / t, j = b - blk * t;
      const int i0 = 2 * t * blk + j, i1 = i0 + t;
      const uint32_t x = acc[i0], y = acc[i1], w = a.twiddle[h + blk];
      uint64_t s = (uint64_t)x + y;
      if (s >= kQ) s -= kQ;
      s = (s & 1) ? (s + kQ) >> 1 : s >> 1;
      uint64_t d = (uint64_t)x + kQ - y;
      if (d >= kQ) d -= kQ;
      acc[i0] = (uint32_t)s;
      acc[i1] = mulmod_q((uint32_t)d, w);
    }
    __syncthreads();
  }

  for (int i = tid; i < n; i += nt) {
    const uint32_t inter = (uint32_t)(((uint64_t)a.acc[base + i] * kQ + (1ull << 31)) >> 32);
    const uint32_t v = addmod_q(inter, acc[i]);
    const uint32_t t = rescale_q1(v, a.q1);
    const uint32_t p = (uint32_t)a.row1_off + (uint32_t)i * (uint32_t)a.q1_bits;
    const uint32_t sh = p & 31u;
    atomicOr(&res[p >> 5], t << sh);
    if (sh) {
      const uint32_t hi = t >> (32u - sh);
      if (hi) atomicOr(&res[(p >> 5) + 1], hi);
    }
  }
  __syncthreads();

  uint8_t *dst = a.resp + (size_t)slot * a.resp_stride + (size_t)o * a.part_len;
  if ((a.part_len & 3) == 0 && ((reinterpret_cast<uintptr_t>(dst) & 3) == 0)) {
    uint32_t *d32 = reinterpret_cast<uint32_t *>(dst);
    for (int w = tid; w < a.part_len / 4; w += nt) d32[w] = res[w];
  } else {
    for (int b = tid; b < a.part_len; b += nt) dst[b] = (uint8_t)(res[b >> 2] >> (8 * (b & 3)));
  }
}

// ------------------------------------------------------------------------------------ synthetic database
// db[(col - col0) * ld + row] = byte col of synthetic::record(row) (src/service.rs:43-62): the m-th splitmix64
// output of the record's stream is the finaliser of seed_row + (m + 1) * gamma, so every byte is independent.
__device__ __forceinline__ uint64_t splitmix_finalise(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__global__ void synthetic_db_kernel(uint8_t *db, size_t ld, size_t rows, size_t col0, size_t ncols) {
  // each thread writes 4 consecutive rows of one column
  const size_t quads = rows / 4;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= quads * ncols) return;
  const size_t c = idx / quads, r0 = (idx % quads) * 4, col = col0 + c;
  uint32_t word = 0;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const uint64_t row = r0 + b;
    const uint64_t s0 = 0x416c746f504952ull ^ (0xd1b54a32d192ed03ull * (row + 1));
    const uint32_t v = (uint32_t)(splitmix_finalise(s0 + (col / 2 + 1) * 0x9e3779b97f4a7c15ull) % 65535ull);
    word |= ((col & 1) ? (v >> 8) : (v & 0xff)) << (8 * b);
  }
  *reinterpret_cast<uint32_t *>(db + c * ld + r0) = word;
}

}  // namespace alto
