// kernels.cuh -- the non-GEMM kernels of the answer path: request validation, byte-limb split of the query and
// key words, and the vector tail (key-switch accumulate, inverse NTT, modulus switch, 10-bit packing).
#pragma once
#include <cstdint>
#include "limb_gemm.cuh"
#include "modq.cuh"

namespace alto {

// ------------------------------------------------------------------------------------ validate
// One CTA per staged frame; the frame starts `lead` bytes into its slot so that its key words (frame offset 9) are
// 16-byte aligned.  Status 2 for a flag byte != 0 or a key count != tg * n (src/amx_kernels.cpp:575), 3 for any of
// the 2 * count y/z key words >= Q (src/amx_kernels.cpp:576-580), else 0.  Query words are not range-checked, as in
// the reference.  Status 1 (length) is settled by the host before a frame is staged.
// Rearranges a staged slab into the tile-contiguous layout: the stage holds consecutive 128-row tiles (row tile j in
// rows [128 j, 128 j + 128), nr valid rows in all, nk valid bytes of `pitch`), and each becomes `tiles` consecutive
// 128 x 128-byte tiles at dst + (j * kbs + kb0 + t) * 16 KB.  One thread per 16-byte output word; bytes past the
// valid rows or width are zero.
__global__ void tile_slab_kernel(const uint8_t *__restrict__ src, size_t pitch, int nr, int nk, int tiles,
                                 size_t words, uint8_t *__restrict__ dst, size_t kbs, size_t kb0) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= words) return;
  const size_t per = (size_t)tiles * 1024;  // words per row tile
  const size_t j = i / per, rest = i - j * per;
  const int r = (int)((rest >> 3) & 127);
  const size_t row = j * 128 + r, k = (rest >> 10) * 128 + (rest & 7) * 16;
  uint4 v = make_uint4(0, 0, 0, 0);
  if (row < (size_t)nr && k < (size_t)nk) {
    const uint8_t *p = src + row * pitch + k;
    if (k + 16 <= (size_t)nk) {
      v = *reinterpret_cast<const uint4 *>(p);
    } else {
      uint8_t b[16] = {};
      for (size_t q = 0; k + q < (size_t)nk; ++q) b[q] = p[q];
      memcpy(&v, b, 16);
    }
  }
  reinterpret_cast<uint4 *>(dst)[((j * kbs + kb0) << 10) + rest] = v;
}

// Transposes record-major records into the database's tile layout.  The stage holds records [a, a + S) (record i at
// stage + (i - a) * cols); records [lo, hi) are valid.  Block (x, y) fills tile (mt = y, kb = a / 128 + x): tile
// row r is database column 128 mt + r, byte k of it record 128 kb + k.  Records of the tile outside [lo, hi) keep
// their bytes; columns past `cols` are left alone (they stay zero).
__global__ void __launch_bounds__(256) records_to_tiles_kernel(const uint8_t *__restrict__ stage, size_t cols, size_t a,
                                                               size_t lo, size_t hi, uint8_t *__restrict__ db,
                                                               size_t kbs, size_t ncols) {
  __shared__ __align__(16) uint8_t t[128][144];  // [column in tile][record in tile], rows padded to 144 bytes
  const size_t kb = a / 128 + blockIdx.x, mt = blockIdx.y;
  const size_t rec0 = kb * 128, col0 = mt * 128;
  const size_t klo = lo > rec0 ? lo - rec0 : 0, khi = hi < rec0 + 128 ? hi - rec0 : 128;
  // load: 128 records x 8 chunks of 16 bytes, transposed into shared memory byte by byte
  for (int i = threadIdx.x; i < 1024; i += 256) {
    const int k = i >> 3, c16 = i & 7;
    const size_t col = col0 + c16 * 16;
    uint4 v = make_uint4(0, 0, 0, 0);
    if ((size_t)k >= klo && (size_t)k < khi && col < ncols)
      v = *reinterpret_cast<const uint4 *>(stage + (rec0 + k - a) * cols + col);
    const uint8_t *b = reinterpret_cast<const uint8_t *>(&v);
#pragma unroll
    for (int j = 0; j < 16; ++j) t[c16 * 16 + j][k] = b[j];
  }
  __syncthreads();
  uint8_t *tile = db + (mt * kbs + kb) * 16384;
  if (klo == 0 && khi == 128) {
    for (int i = threadIdx.x; i < 1024; i += 256) {  // whole tile: 16-byte stores
      const int r = i >> 3, k16 = i & 7;
      if (col0 + r < ncols)
        *reinterpret_cast<uint4 *>(tile + r * 128 + k16 * 16) = *reinterpret_cast<const uint4 *>(&t[r][k16 * 16]);
    }
  } else {
    for (int i = threadIdx.x; i < 128 * 128; i += 256) {  // part of the records: byte stores of those only
      const int r = i >> 7, k = i & 127;
      if ((size_t)k >= klo && (size_t)k < khi && col0 + r < ncols) tile[r * 128 + k] = t[r][k];
    }
  }
}

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
// Byte j of word k of slot c goes to dst[z][(c * 4 + j)][k - z * chunk] with z = k / chunk, for c < padded (zero
// rows for c >= slots): the K-major B operand of the limb GEMMs, cut into record chunks of `chunk` words (a
// multiple of 16) like the database.  Each thread moves 16 words (64 bytes in, four 16-byte rows out).
__global__ void limb_split_kernel(const uint8_t *__restrict__ req, size_t stride, size_t word_off, int slots,
                                  int padded, size_t words, size_t chunk, uint8_t *__restrict__ dst) {
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
  const size_t k = g * 16, z = k / chunk;
  uint8_t *base = dst + z * (4 * (size_t)padded * chunk) + (k - z * chunk);
#pragma unroll
  for (int j = 0; j < 4; ++j)
    *reinterpret_cast<uint4 *>(base + ((size_t)c * 4 + j) * chunk) = make_uint4(o[j][0], o[j][1], o[j][2], o[j][3]);
}

// ------------------------------------------------------------------------------------ tail
struct TailArgs {
  const uint32_t *acc;      // scan sums mod 2^32, [slot][cols]
  const uint32_t *beta;     // pack results mod Q, [slot][cols]
  const int *status;        // per-slot status; only slots with status 0 are answered
  const uint8_t *req;       // staged request bodies (y, z, q words), [slot][req_stride]
  size_t req_stride;
  size_t z_off;             // byte offset of the z key words within a slot
  const uint32_t *that;     // bold_t_hat mod Q, [output][tg * n]
  const uint32_t *twiddle;  // inverse-NTT table, low 32 bits of each entry, [n]
  const uint8_t *prefix;    // row-0 prefixes, [output][part_len]
  uint8_t *resp;            // responses: slot s, part o at resp + s * resp_stride + o * part_len
  size_t resp_stride;
  int n, tg, outputs, cols;
  int part_len, row1_off, q1_bits;
  int64_t q1;
  int o_begin, o_count;     // this launch answers parts o_begin .. o_begin + o_count of every slot
  // Gather into several response buffers (column shards): when n_resp > 0 the part is written to every
  // resp_list[k] + s * resp_stride + (part_offset + o) * part_len instead of to resp -- buffers of this GPU or of
  // peer GPUs (CUDA IPC mappings over NVLink), so the shards' all-gather happens in this kernel's stores.
  uint8_t *const *resp_list = nullptr;
  int n_resp = 0;
  int part_offset = 0;
};

// The destinations of response part o of slot `slot`: resp, or each gather buffer (see TailArgs).
__device__ __forceinline__ uint8_t *tail_dst(const TailArgs &a, int k, int slot, int o) {
  uint8_t *base = a.n_resp ? a.resp_list[k] : a.resp;
  return base + (size_t)slot * a.resp_stride + (size_t)(a.part_offset + o) * a.part_len;
}

// One response part per CTA (slot, output o), n / 8 threads owning 8 coefficients each.
//   acc[i] = beta[i] + sum_k z[k n + i] * that[k n + i] (mod Q)                    (src/amx_kernels.cpp:500-511)
//   inverse NTT: stages t = 1, 2, ..., n/2; block b of the stage with h = n/(2t) blocks uses table[h + b];
//   x' = (x + y) / 2, y' = (x - y) w (mod Q)                                       (src/amx_kernels.cpp:461-498)
// computed without the halving: a value held after s stages is 2^s times the reference's, so a stage is
// x' = x + y, y' = (x - y) (2 w); the L = log2 n factors of 2 are cancelled in advance, since the transform is linear:
// the engine stores beta's packing matrix and bold_t_hat multiplied by 2^-L and the twiddles doubled (engine set-up),
// so acc enters the transform already scaled by 2^-L and leaves it equal to the reference's, mod Q.
//   v = inter + acc, inter = (scan sum * Q + 2^31) >> 32; rescale to q1; OR the q1_bits-bit values LSB-first into
//   the prefix from bit row1_off                                                   (src/amx_kernels.cpp:306, 515-537)
// The stages run in rounds of three (bits s0..s0+2 of the coefficient index): in a round a thread holds the 8
// coefficients that differ only in those bits, so three stages need one shared-memory exchange.  Coefficient i is
// stored at word i ^ (8 * ((i >> 6) & 3)), which keeps every round's accesses free of bank conflicts.
__device__ __forceinline__ int tail_swz(int i) { return i ^ (((i >> 6) & 3) << 3); }

template <int L>
__device__ __forceinline__ int tail_index(int o, int m, int s0, int r) {
  return ((o >> s0) << (s0 + r)) | (m << s0) | (o & ((1 << s0) - 1));
}

// Three (or fewer) stages on the 2^r coefficients x[0..2^r) of one group, whose index is i(m) = tail_index(o, m).
template <int L>
__device__ __forceinline__ void tail_round(uint32_t *x, int o, int s0, int r, const uint32_t *__restrict__ tw) {
  constexpr int n = 1 << L;
  for (int d = 0; d < r; ++d) {
    const int s = s0 + d, t = 1 << d;
    for (int m = 0; m < (1 << r); ++m) {
      if (m & t) continue;
      const int i = tail_index<L>(o, m, s0, r);
      const uint32_t w = __ldg(tw + (n >> (s + 1)) + (i >> (s + 1)));
      const uint32_t a = x[m], b = x[m + t];
      x[m] = add_q(a, b);
      x[m + t] = mul_q(sub_q(a, b), w);
    }
  }
}

// MINB: CTAs per SM the register budget is sized for (__launch_bounds__): at n = 2048 a batch of 128 clients and 8
// parts is 1024 CTAs, so the register count decides between one wave and one and a fraction.
template <int L, int MINB>
__global__ void __launch_bounds__((1 << L) / 8, MINB) tail_kernel(TailArgs a) {
  constexpr int n = 1 << L, NT = n / 8;
  extern __shared__ uint32_t tsm[];
  const int slot = blockIdx.x / a.o_count, o = a.o_begin + blockIdx.x % a.o_count;
  if (a.status[slot] != 0) return;  // rejected frames get no response (their output stays untouched)
  const int tid = threadIdx.x;
  uint32_t *acc = tsm;
  uint32_t *res = tsm + n;
  const int res_words = (a.part_len + 3) / 4 + 1;
  const size_t count = (size_t)a.tg * n;
  const uint32_t *z = reinterpret_cast<const uint32_t *>(a.req + (size_t)slot * a.req_stride + a.z_off);
  const uint32_t *th = a.that + (size_t)o * count;
  const size_t base = (size_t)slot * a.cols + (size_t)o * n;

  // prefix -> res (32-bit words, little endian)
  const uint8_t *pre = a.prefix + (size_t)o * a.part_len;
  if ((a.part_len & 15) == 0 && (reinterpret_cast<uintptr_t>(pre) & 15) == 0) {
    for (int w = tid; w < a.part_len / 16; w += NT) {
      const uint4 v = *reinterpret_cast<const uint4 *>(pre + 16 * w);
      res[4 * w] = v.x; res[4 * w + 1] = v.y; res[4 * w + 2] = v.z; res[4 * w + 3] = v.w;
    }
    if (tid == 0) res[a.part_len / 4] = 0;
  } else {
    for (int w = tid; w < res_words; w += NT) {
      uint32_t v = 0;
      for (int b = 0; b < 4; ++b)
        if (4 * w + b < a.part_len) v |= (uint32_t)pre[4 * w + b] << (8 * b);
      res[w] = v;
    }
  }

  // key-switch accumulate for coefficients 8 tid .. 8 tid + 7, then stages t = 1, 2, 4 in registers
  uint32_t x[8];
  {
    const int i0 = 8 * tid;
    const uint4 b0 = *reinterpret_cast<const uint4 *>(a.beta + base + i0);
    const uint4 b1 = *reinterpret_cast<const uint4 *>(a.beta + base + i0 + 4);
    // beta + sum_k z_k that_k, each product folded once (< 2^46) and summed in 64 bits: below 2^32 + tg 2^46 <
    // 2^57 for every tg this engine accepts (tg n <= 32768), then reduced once
    uint64_t acc64[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
    for (int k = 0; k < a.tg; ++k) {
      const uint4 z0 = *reinterpret_cast<const uint4 *>(z + (size_t)k * n + i0);
      const uint4 z1 = *reinterpret_cast<const uint4 *>(z + (size_t)k * n + i0 + 4);
      const uint4 t0 = *reinterpret_cast<const uint4 *>(th + (size_t)k * n + i0);
      const uint4 t1 = *reinterpret_cast<const uint4 *>(th + (size_t)k * n + i0 + 4);
      acc64[0] += fold_q64((uint64_t)z0.x * t0.x); acc64[1] += fold_q64((uint64_t)z0.y * t0.y);
      acc64[2] += fold_q64((uint64_t)z0.z * t0.z); acc64[3] += fold_q64((uint64_t)z0.w * t0.w);
      acc64[4] += fold_q64((uint64_t)z1.x * t1.x); acc64[5] += fold_q64((uint64_t)z1.y * t1.y);
      acc64[6] += fold_q64((uint64_t)z1.z * t1.z); acc64[7] += fold_q64((uint64_t)z1.w * t1.w);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) x[m] = red_q64(acc64[m]);
    tail_round<L>(x, tid, 0, 3, a.twiddle);
  }

  // rounds over bits 3..5, 6..8, ...: exchange through shared memory, three stages per round
#pragma unroll
  for (int s0 = 3; s0 < L; s0 += 3) {
    const int r = (L - s0) < 3 ? (L - s0) : 3;
    const int groups = 8 >> r;
    const int ps0 = s0 - 3, pr = 3;  // the previous round's layout (every round but the last has three bits)
    // write the 8 values held from the previous round
    if (s0 == 3) {
      // coefficients 8 tid .. 8 tid + 7 stay contiguous under the swizzle (it only flips bits 3 and 4)
      uint4 *dst4 = reinterpret_cast<uint4 *>(acc + tail_swz(8 * tid));
      dst4[0] = make_uint4(x[0], x[1], x[2], x[3]);
      dst4[1] = make_uint4(x[4], x[5], x[6], x[7]);
    } else {
#pragma unroll
      for (int m = 0; m < 8; ++m) acc[tail_swz(tail_index<L>(tid, m, ps0, pr))] = x[m];
    }
    __syncthreads();
    for (int g = 0; g < groups; ++g) {
      const int oo = g * NT + tid;
      uint32_t y[8];
      for (int m = 0; m < (1 << r); ++m) y[m] = acc[tail_swz(tail_index<L>(oo, m, s0, r))];
      tail_round<L>(y, oo, s0, r, a.twiddle);
      if (s0 + r < L) {
        for (int m = 0; m < 8; ++m) x[m] = y[m];
      } else {
        // last round: back into place (each location is read and written by this thread alone in this round)
        for (int m = 0; m < (1 << r); ++m) acc[tail_swz(tail_index<L>(oo, m, s0, r))] = y[m];
      }
    }
    __syncthreads();
  }

  // modulus switch of coefficients 8 tid .. 8 tid + 7 and their q1_bits-bit values, LSB first, into the response
  // part from bit row1_off: one contiguous run of bits per thread, ORed into the words it covers (the run's first
  // and last words are shared with the neighbouring threads)
  {
    const int i0 = 8 * tid;
    const uint4 v0 = *reinterpret_cast<const uint4 *>(acc + tail_swz(i0));
    const uint4 v1 = *reinterpret_cast<const uint4 *>(acc + tail_swz(i0) + 4);
    const uint4 s0v = *reinterpret_cast<const uint4 *>(a.acc + base + i0);
    const uint4 s1v = *reinterpret_cast<const uint4 *>(a.acc + base + i0 + 4);
    const uint32_t v[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
    const uint32_t sc[8] = {s0v.x, s0v.y, s0v.z, s0v.w, s1v.x, s1v.y, s1v.z, s1v.w};
    const uint32_t qb = (uint32_t)a.q1_bits, p0 = (uint32_t)a.row1_off + (uint32_t)i0 * qb;
    uint32_t word = p0 >> 5, fill = p0 & 31u;
    uint64_t win = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint32_t inter = (uint32_t)(((uint64_t)sc[m] * kQ + (1ull << 31)) >> 32);
      win |= (uint64_t)rescale_q(add_q(inter, v[m]), (uint32_t)a.q1) << fill;
      fill += qb;
      if (fill >= 32) {
        if ((uint32_t)win) atomicOr(&res[word], (uint32_t)win);
        win >>= 32;
        fill -= 32;
        ++word;
      }
    }
    if (fill && (uint32_t)win) atomicOr(&res[word], (uint32_t)win);
  }
  __syncthreads();

  for (int k = 0; k < (a.n_resp ? a.n_resp : 1); ++k) {
    uint8_t *dst = tail_dst(a, k, slot, o);
    if ((a.part_len & 15) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
      for (int w = tid; w < a.part_len / 16; w += NT)
        *reinterpret_cast<uint4 *>(dst + 16 * w) =
            make_uint4(res[4 * w], res[4 * w + 1], res[4 * w + 2], res[4 * w + 3]);
    } else {
      for (int b = tid; b < a.part_len; b += NT) dst[b] = (uint8_t)(res[b >> 2] >> (8 * (b & 3)));
    }
  }
}

// The same computation for small rings (n < 256), one coefficient pair per thread and stage.
__global__ void __launch_bounds__(128) tail_small_kernel(TailArgs a) {
  extern __shared__ uint32_t tsm[];
  const int slot = blockIdx.x / a.o_count, o = a.o_begin + blockIdx.x % a.o_count;
  if (a.status[slot] != 0) return;
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
    for (int k = 0; k < a.tg; ++k) s = add_q(s, mul_q(z[(size_t)k * n + i], th[(size_t)k * n + i]));
    acc[i] = s;
  }
  const uint8_t *pre = a.prefix + (size_t)o * a.part_len;
  for (int w = tid; w < res_words; w += nt) {
    uint32_t v = 0;
    for (int b = 0; b < 4; ++b)
      if (4 * w + b < a.part_len) v |= (uint32_t)pre[4 * w + b] << (8 * b);
    res[w] = v;
  }
  __syncthreads();
  for (int lt = 0; (1 << lt) < n; ++lt) {
    const int t = 1 << lt, h = n >> (lt + 1);
    for (int b = tid; b < n / 2; b += nt) {
      const int blk = b >> lt, j = b & (t - 1);
      const int i0 = 2 * t * blk + j, i1 = i0 + t;
      const uint32_t x = acc[i0], y = acc[i1];
      acc[i0] = add_q(x, y);
      acc[i1] = mul_q(sub_q(x, y), a.twiddle[h + blk]);
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) {
    const uint32_t inter = (uint32_t)(((uint64_t)a.acc[base + i] * kQ + (1ull << 31)) >> 32);
    const uint32_t t = rescale_q(add_q(inter, acc[i]), (uint32_t)a.q1);
    const uint32_t p = (uint32_t)a.row1_off + (uint32_t)i * (uint32_t)a.q1_bits;
    const uint32_t sh = p & 31u;
    atomicOr(&res[p >> 5], t << sh);
    if (sh) {
      const uint32_t hi = t >> (32u - sh);
      if (hi) atomicOr(&res[(p >> 5) + 1], hi);
    }
  }
  __syncthreads();
  for (int k = 0; k < (a.n_resp ? a.n_resp : 1); ++k) {
    uint8_t *dst = tail_dst(a, k, slot, o);
    for (int b = tid; b < a.part_len; b += nt) dst[b] = (uint8_t)(res[b >> 2] >> (8 * (b & 3)));
  }
}

// Multiplies every packing-matrix value by `factor` mod Q in place, in the tile layout (tile t at t * 16 KB holds
// rows (col, plane j) = 4 col + j of 32 columns and 128 key words): value k of column c is byte k of rows 4c..4c+3.
// One thread per (tile, column, 4 consecutive key words): four 32-bit loads, a 4 x 4 byte transpose, four products,
// the transpose back and four stores.
__global__ void scale_planes_kernel(uint8_t *tiles, size_t ntiles, uint32_t factor) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tile = idx >> 10;
  if (tile >= ntiles) return;
  const int c = (int)((idx >> 5) & 31), kq = (int)(idx & 31);
  uint32_t *row = reinterpret_cast<uint32_t *>(tiles + tile * 16384 + (size_t)(4 * c) * 128) + kq;
  const uint32_t b0 = row[0], b1 = row[32], b2 = row[64], b3 = row[96];  // planes 0..3, key words 4kq..4kq+3
  const uint32_t lo01 = __byte_perm(b0, b1, 0x5140), hi01 = __byte_perm(b0, b1, 0x7362);
  const uint32_t lo23 = __byte_perm(b2, b3, 0x5140), hi23 = __byte_perm(b2, b3, 0x7362);
  uint32_t v[4] = {__byte_perm(lo01, lo23, 0x5410), __byte_perm(lo01, lo23, 0x7632), __byte_perm(hi01, hi23, 0x5410),
                   __byte_perm(hi01, hi23, 0x7632)};
#pragma unroll
  for (int t = 0; t < 4; ++t) v[t] = mul_q(v[t], factor);
  const uint32_t p01 = __byte_perm(v[0], v[1], 0x5140), p23 = __byte_perm(v[2], v[3], 0x5140);
  const uint32_t q01 = __byte_perm(v[0], v[1], 0x7362), q23 = __byte_perm(v[2], v[3], 0x7362);
  row[0] = __byte_perm(p01, p23, 0x5410);
  row[32] = __byte_perm(p01, p23, 0x7632);
  row[64] = __byte_perm(q01, q23, 0x5410);
  row[96] = __byte_perm(q01, q23, 0x7632);
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

// The same records written straight into the database's tile layout: tile (mt, kb) at (mt * kbs + kb) * 16 KB, its
// row r = column 128 mt + r, byte k of a row = record 128 kb + k.  Columns 2c and 2c + 1 are the two bytes of one
// splitmix64 output, so a thread takes a pair of tile rows and 16 records: 16 finaliser evaluations fill two 16-byte
// words.  Records >= rows and columns >= cols are zero (cols is even).
__global__ void synthetic_tiles_kernel(uint8_t *db, size_t kbs, size_t tiles, size_t rows, size_t cols) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tile = idx >> 9;  // 64 row pairs x 8 groups of 16 records per tile
  if (tile >= tiles) return;
  const int rp = (int)((idx >> 3) & 63), g = (int)(idx & 7);
  const size_t mt = tile / kbs, kb = tile - mt * kbs;
  const size_t col = mt * 128 + 2 * rp, rec0 = kb * 128 + g * 16;
  uint32_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
  if (col < cols) {
    const uint64_t step = (col / 2 + 1) * 0x9e3779b97f4a7c15ull;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const uint64_t row = rec0 + k;
      if (row < rows) {
        const uint64_t s0 = 0x416c746f504952ull ^ (0xd1b54a32d192ed03ull * (row + 1));
        const uint32_t v = (uint32_t)(splitmix_finalise(s0 + step) % 65535ull);
        lo[k >> 2] |= (v & 0xffu) << (8 * (k & 3));
        hi[k >> 2] |= (v >> 8) << (8 * (k & 3));
      }
    }
  }
  uint8_t *base = db + tile * 16384 + (size_t)(2 * rp) * 128 + g * 16;
  *reinterpret_cast<uint4 *>(base) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  *reinterpret_cast<uint4 *>(base + 128) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
}

// Seeded synthetic request frames (the bytes alto_synthetic_request writes on the host) straight into device slots:
// frame c at slots + c * stride + lead.  Client s = seed ^ 0xd1b54a32d192ed03 (client + 1) draws word i of its keys
// and query from splitmix64 counter s: key words uniform in [0, Q) by a multiply-high of the output's top half,
// query words the output's top half.  The caller puts the key words on a 4-byte boundary ((lead + 9) % 4 == 0 and
// stride % 4 == 0).  Grid: (word blocks, b); thread 0 of block 0 also writes the 9-byte header.
__global__ void synthetic_requests_kernel(uint8_t *slots, size_t stride, size_t lead, size_t rows, size_t tg_n,
                                          uint64_t seed, uint64_t first_client) {
  const uint64_t client = first_client + blockIdx.y;
  const uint64_t s = seed ^ (0xd1b54a32d192ed03ull * (client + 1));
  uint8_t *f = slots + (size_t)blockIdx.y * stride + lead;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x, keys = 2 * tg_n;
  if (i == 0) {
    f[0] = 0;
    for (int b = 0; b < 4; ++b) f[1 + b] = f[5 + b] = (uint8_t)(tg_n >> (8 * b));
  }
  if (i >= keys + rows) return;
  const uint64_t x = splitmix_finalise(s + (i + 1) * 0x9e3779b97f4a7c15ull);
  const uint32_t v = i < keys ? (uint32_t)(((x >> 32) * kQ) >> 32) : (uint32_t)(x >> 32);
  reinterpret_cast<uint32_t *>(f + 9)[i] = v;
}

}  // namespace alto

namespace alto {

constexpr int kTailMinBlocks = 6;  // default register budget of the n = 2048 tail: 40 registers, 6 CTAs per SM

// Launches the tail for `slots` frames on stream st: the radix-8 kernel for n >= 256, the simple one below.
inline cudaError_t launch_tail(const TailArgs &t, size_t slots, cudaStream_t st) {
  const size_t smem = ((size_t)t.n + (t.part_len + 3) / 4 + 1) * sizeof(uint32_t);
  const unsigned grid = (unsigned)(slots * t.o_count);
  cudaError_t err = cudaSuccess;
  auto go = [&](auto kernel, unsigned threads) {
    if (smem > 48 * 1024) err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err == cudaSuccess) {
      kernel<<<grid, threads, smem, st>>>(t);
      err = cudaGetLastError();
    }
  };
  // ALTO_TAIL_MINB = 1, 6 or 8 picks the register budget of the n = 2048 tail (a tuning knob; same results)
  static const int minb = [] {
    const char *v = getenv("ALTO_TAIL_MINB");
    const int m = v ? atoi(v) : kTailMinBlocks;
    return (m == 1 || m == 6 || m == 8) ? m : kTailMinBlocks;
  }();
  switch (t.n) {
    case 256: go(tail_kernel<8, 1>, 32); break;
    case 512: go(tail_kernel<9, 1>, 64); break;
    case 1024: go(tail_kernel<10, 1>, 128); break;
    case 2048:
      if (minb == 8) go(tail_kernel<11, 8>, 256);
      else if (minb == 6) go(tail_kernel<11, 6>, 256);
      else go(tail_kernel<11, 1>, 256);
      break;
    case 4096: go(tail_kernel<12, 1>, 512); break;
    default: go(tail_small_kernel, 128); break;
  }
  return err;
}

}  // namespace alto
