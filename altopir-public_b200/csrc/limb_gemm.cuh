// limb_gemm.cuh -- the two dense contractions of the answer path as tcgen05 kind::i8 GEMMs over byte limbs.
//
//   scan (src/amx_kernels.cpp:175-309): A = database, one row per record byte position (column of the record
//        matrix), K = records, K-major (the server's column-order database) and stored tile by tile: every
//        128-row x 128-byte tile is 16 KB contiguous in HBM (see the engine's set-up); B = the batch's query
//        words split into 4 byte limbs, one row per (client, limb).  D[col][(c, j)] = sum_k db[col][k] * q_c[k]_j.
//        Epilogue: acc = sum_j D << 8j (mod 2^32), added into acc[c][col] with a 32-bit reduction so that split-K
//        chunks (each short enough that no int32 partial sum can overflow) combine modulo 2^32.
//   pack (src/amx_kernels.cpp:345-445): A = the packing matrix as 4 byte planes, rows ordered (col, plane j),
//        K = tg * n, stored tile by tile like the database; B = the packing keys y split into 4 byte limbs, rows
//        (client, limb i).
//        Epilogue: beta[c][col] = sum_{i,j} D[(col, j)][(c, i)] * 2^(8(i+j)) mod Q, the 4 planes of one column
//        sitting in 4 adjacent TMEM lanes of one warp and combined with two shuffles.
//
// One CTA computes one unit (a 128-row tile of A, a BN-column tile of B, one K chunk): warp 0 issues TMA loads of
// 128 x 128-byte A boxes and BN x 128-byte B boxes (128-byte swizzle) into a STAGES-deep ring, warp 1 issues
// 4 MMAs of 128 x BN x 32 per stage into a TMEM accumulator, warps 2-5 drain TMEM with tcgen05.ld.
#pragma once
#include "sm100.cuh"

namespace alto {

constexpr uint64_t kQ = 4294955009ull;  // 2^32 - 12287
constexpr int kBM = 128;                // rows of A per tile = TMEM lanes
constexpr int kBK = 128;                // bytes of K per pipeline stage (one 128-byte swizzle row)
constexpr int kGemmThreads = 192;       // warp 0 TMA, warp 1 MMA + TMEM owner, warps 2..5 epilogue

enum class Epi : int { kScan = 0, kPack = 1 };

struct GemmArgs {
  int num_m;        // tiles of 128 rows along A
  int num_n;        // tiles of BN limb columns along B
  int kb_total;     // 128-byte blocks in the whole reduction
  int kb_per_unit;  // blocks per unit (split-K chunk); scan chunks never exceed 256 blocks (32768 records)
  int rows_a;       // valid rows of A
  int clients;      // valid clients (limb columns beyond 4 * clients are padding)
  int cols;         // record bytes: row stride of the output matrices
  uint32_t *out;    // scan: acc[c * cols + col], pre-zeroed; pack: beta[c * cols + col]
  uint32_t *err;    // device error word
  int b_keep;       // 1: keep the B operand in L2 (evict_last; it is small and read by every unit), 0: normal
  int kb_chunk;     // scan: 128-byte blocks per record chunk of the 3-D query-limb map (units never straddle chunks)
  int m_begin;      // first tile along A (a launch may cover a column group: tiles m_begin .. m_begin + num_m)
  int kb_begin = 0; // first 128-byte block of the reduction (a launch may cover a range of record chunks;
                    // kb_total is then the range's end)
};

// x mod Q for any 64-bit x, using 2^32 = 12287 (mod Q): two folds leave x < 2^32 + 2^28, one subtraction finishes.
__device__ __forceinline__ uint64_t mod_q64(uint64_t x) {
  x = (x >> 32) * 12287ull + (x & 0xffffffffull);
  x = (x >> 32) * 12287ull + (x & 0xffffffffull);
  return x >= kQ ? x - kQ : x;
}

template <int BN>
struct GemmShape {
  static constexpr int kABytes = kBM * kBK;
  static constexpr int kBBytes = BN * kBK;
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kStages = (196608 / kStageBytes) < 8 ? (196608 / kStageBytes) : 8;
  static constexpr int kTmemCols = BN < 32 ? 32 : BN;
  static constexpr int kBarrierBytes = 256;
  static constexpr int kSmemBytes = kStages * kStageBytes + kBarrierBytes + 1024;  // +1024 for manual alignment
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "kind::i8 with M = 128 needs N in [16, 256], N % 16 == 0");
  static_assert(kStageBytes % 1024 == 0, "stages must keep 1024-byte swizzle-atom alignment");
  static_assert(kStages >= 2, "pipeline needs at least two stages");
};

template <int BN, Epi EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    limb_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     GemmArgs args) {
  using S = GemmShape<BN>;
  constexpr int kStages = S::kStages;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base_addr = (raw_addr + 1023u) & ~1023u;
  uint8_t *smem = smem_raw + (base_addr - raw_addr);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * S::kStageBytes);
  // bars[0..S) full, bars[S..2S) empty, bars[2S] accumulator ready
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 1);
  volatile int *bail = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int u = blockIdx.x;
  const int n_tile = u % args.num_n;
  const int m_tile = args.m_begin + (u / args.num_n) % args.num_m;
  const int k_chunk = u / (args.num_n * args.num_m);
  const int kb0 = args.kb_begin + k_chunk * args.kb_per_unit;
  const int kb1 = min(kb0 + args.kb_per_unit, args.kb_total);
  const int nkb = kb1 - kb0;  // >= 1 by construction of the grid

  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages), accum = smem_u32(bars + 2 * kStages);

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(accum, 1);
    *bail = 0;
    fence_barrier_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&map_a);
    tma_prefetch_desc(&map_b);
  }
  if (warp == 1) {
    tmem_alloc(smem_u32(tmem_slot), S::kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  volatile int no_bail = 0;

  if (warp == 0) {
    // ---------------------------------------------------------------- TMA producer
    if (lane == 0) {
      // The A operand (database or packing matrix) streams through once per unit; B (limbs) is shared by all units.
      const uint64_t pol_a = policy_evict_first();
      const uint64_t pol_b = args.b_keep ? policy_evict_last() : policy_evict_normal();
      int issued = 0;
      for (int i = 0; i < nkb; ++i) {
        const int s = i % kStages, round = i / kStages;
        if (round > 0 && !mbar_wait(empty0 + 8 * s, (round - 1) & 1, args.err, ALTO_ERR_WAIT_EMPTY, bail)) break;
        const uint32_t sa = base_addr + s * S::kStageBytes, sb = sa + S::kABytes;
        mbar_arrive_expect_tx(full0 + 8 * s, S::kStageBytes);
        if constexpr (EPI == Epi::kScan) {
          // record chunk z, 128-byte block x inside it
          const int kb = kb0 + i, z = kb / args.kb_chunk, x = (kb - z * args.kb_chunk) * kBK;
          tma_load_tile(sa, &map_a, full0 + 8 * s, kb, m_tile, pol_a);
          tma_load_3d(sb, &map_b, full0 + 8 * s, x, n_tile * BN, z, pol_b);
        } else {
          tma_load_tile(sa, &map_a, full0 + 8 * s, kb0 + i, m_tile, pol_a);
          tma_load_2d(sb, &map_b, full0 + 8 * s, (kb0 + i) * kBK, n_tile * BN, pol_b);
        }
        issued = i + 1;
      }
      if (*bail) {
        // Drain: the last load issued into each stage must land before the CTA may exit.
        for (int i = issued > kStages ? issued - kStages : 0; i < issued; ++i)
          mbar_wait(full0 + 8 * (i % kStages), (i / kStages) & 1, args.err, ALTO_ERR_WAIT_DRAIN, &no_bail);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_u8u8_s32(BN);
      for (int i = 0; i < nkb; ++i) {
        const int s = i % kStages, round = i / kStages;
        if (!mbar_wait(full0 + 8 * s, round & 1, args.err, ALTO_ERR_WAIT_FULL, bail)) break;
        tc_fence_after();
        const uint32_t sa = base_addr + s * S::kStageBytes, sb = sa + S::kABytes;
#pragma unroll
        for (int kk = 0; kk < kBK / 32; ++kk)
          mma_i8(tmem_base, desc_sw128(sa + kk * 32), desc_sw128(sb + kk * 32), idesc, (i | kk) != 0);
        mma_commit(empty0 + 8 * s);
      }
      mma_commit(accum);
      if (*bail) mbar_wait(accum, 0, args.err, ALTO_ERR_WAIT_DRAIN, &no_bail);
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------------- epilogue (warps 2..5)
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const bool ok = mbar_wait(accum, 0, args.err, ALTO_ERR_WAIT_ACCUM, bail);
    tc_fence_after();
    if (ok) {
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16);
      if constexpr (EPI == Epi::kScan) {
        const int col = m_tile * kBM + row;
        const bool row_ok = col < args.rows_a;
#pragma unroll 1
        for (int ch = 0; ch < BN / 16; ++ch) {
          uint32_t r[16];
          tmem_ld16(taddr + ch * 16, r);
          tmem_wait_ld();
#pragma unroll
          for (int cl = 0; cl < 4; ++cl) {
            const uint32_t acc = r[4 * cl] + (r[4 * cl + 1] << 8) + (r[4 * cl + 2] << 16) + (r[4 * cl + 3] << 24);
            const int c = n_tile * (BN / 4) + ch * 4 + cl;
            if (row_ok && c < args.clients) atomicAdd(args.out + (size_t)c * args.cols + col, acc);
          }
        }
      } else {
        const int grow = m_tile * kBM + row;  // = col * 4 + plane
        const int col = grow >> 2, plane = grow & 3;
        const bool row_ok = grow < args.rows_a;
        const uint64_t pw = 1ull << (8 * plane);  // 2^(8j) < Q
#pragma unroll 1
        for (int ch = 0; ch < BN / 16; ++ch) {
          uint32_t r[16];
          tmem_ld16(taddr + ch * 16, r);
          tmem_wait_ld();
#pragma unroll
          for (int cl = 0; cl < 4; ++cl) {
            // partial sums are < 8192 * 255 * 255 < 2^31 (K <= 32768 keeps them below 2^31 as well)
            const uint64_t sum = (uint64_t)r[4 * cl] + ((uint64_t)r[4 * cl + 1] << 8) +
                                 ((uint64_t)r[4 * cl + 2] << 16) + ((uint64_t)r[4 * cl + 3] << 24);
            uint64_t v = mod_q64(mod_q64(sum) * pw);
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v = v >= kQ ? v - kQ : v;
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            v = v >= kQ ? v - kQ : v;
            const int c = n_tile * (BN / 4) + ch * 4 + cl;
            if (plane == 0 && row_ok && c < args.clients) args.out[(size_t)c * args.cols + col] = (uint32_t)v;
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, S::kTmemCols);
  }
}

}  // namespace alto
