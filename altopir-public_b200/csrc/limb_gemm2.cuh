// limb_gemm2.cuh -- the scan and pack limb GEMMs on CTA pairs (tcgen05 cta_group::2), persistent, with two TMEM
// accumulators per CTA so that the epilogue of one unit overlaps the MMAs of the next.
//
// A cluster of two CTAs on two SMs computes a 256-row x BN-column unit: each CTA loads its own 128 rows of A and its
// own BN/2 rows of B (no multicast), the leader CTA (rank 0) issues 256 x BN x 32 MMAs that read both CTAs' shared
// memory, and each CTA's TMEM receives its 128 rows x BN columns.  Per SM this moves (128 + BN/2) x 128 bytes of
// operands per 128 x BN x 128 multiply-adds, half of what a 128-row tile needs for the same work, and the smaller
// stages (32 KB at BN = 256) fit a 6-deep ring.
//
// Barriers (all waits bounded, see sm100.cuh):
//   full[s]      leader only: the leader's producer posts expect_tx for both CTAs' bytes; both CTAs' TMA loads
//                complete on it.
//   empty[s]     both CTAs: released by the leader's MMA commit, multicast to the pair.
//   acc_full[b]  both CTAs: the leader's commit after a unit's last MMA, multicast to the pair.
//   acc_empty[b] leader only: the four epilogue warps of each CTA arrive once the accumulator has been read.
// Units are handed out round-robin: unit u goes to pair u mod P; a unit is (256-row tile m, BN-column tile n, K
// chunk), n varying fastest, so the pairs running at one time share the B tiles of one K chunk through L2.
#pragma once
#include "limb_gemm.cuh"

namespace alto {

// NSUB = 1: a unit is BN limb columns and TMEM holds two accumulators (the epilogue of one unit overlaps the
// MMAs of the next).  NSUB = 2: a unit is 2 x BN limb columns in two sub-accumulators that fill TMEM (one buffer),
// so that every A tile is read once for all of them -- for long scans whose A tiles are too large to be shared
// between pairs through L2.
template <int BN, int NSUB = 1>
struct PairShape {
  static constexpr int kABytes = 128 * kBK;                 // this CTA's 128 rows of A
  static constexpr int kBBytes = NSUB * (BN / 2) * kBK;     // this CTA's BN/2 rows of B for each sub-tile
  static constexpr int kStageBytes = kABytes + kBBytes;
  static constexpr int kStages = (196608 / kStageBytes) < 8 ? (196608 / kStageBytes) : 8;
  static constexpr int kBufs = NSUB == 1 ? 2 : 1;           // accumulator buffers
  static constexpr int kTmemCols = kBufs * NSUB * BN;
  static constexpr int kBarrierBytes = 512;
  static constexpr int kSmemBytes = kStages * kStageBytes + kBarrierBytes + 1024;
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "pair kind::i8 MMA needs N in [32, 256], N % 32 == 0");
  static_assert(kStageBytes % 1024 == 0, "stages must keep 1024-byte swizzle-atom alignment");
  static_assert(kStages >= 3, "pipeline depth");
  static_assert(kTmemCols <= 512, "TMEM has 512 columns");
};

struct PairArgs {
  int num_m;        // tiles of 256 rows along A
  int num_n;        // tiles of BN limb columns along B
  int num_units;    // num_m * num_n * K chunks
  int kb_total;     // 128-byte blocks of the whole reduction
  int kb_per_unit;  // blocks per K chunk (scan chunks never exceed 256 blocks = 32768 records)
  int rows_a;       // valid rows of A
  int clients;      // valid clients
  int cols;         // record bytes: row stride of the outputs
  uint32_t *out;    // scan: acc[c * cols + col] (pre-zeroed, summed mod 2^32); pack: beta[c * cols + col]
  uint32_t *err;    // device error word
  int b_keep;       // 1: keep the B operand in L2 (evict_last; it is small and read by every unit), 0: normal
  int kb_chunk;     // scan: 128-byte blocks per record chunk of the 3-D query-limb map (units never straddle chunks)
  int m_begin;      // first 256-row tile along A (a launch may cover a column group)
  int kb_begin = 0; // first 128-byte block of the reduction (a launch may cover a range of record chunks;
                    // kb_total is then the range's end)
  int nw = 0;       // limb columns a tile computes: a multiple of 32 <= BN (0: BN).  The B boxes are nw/2 rows
                    // (the tensor map's box), loaded from the tile's origin n nw, and the MMAs run N = nw, so a
                    // batch whose limb columns are not a power of two neither loads nor multiplies padding columns
                    // (NSUB = 1 only)
};

// Epilogue of 16 TMEM columns (4 clients x 4 limbs) for one accumulator row of the scan: row = database column.
__device__ __forceinline__ void scan_epilogue16(const uint32_t *r, int col, bool row_ok, int c0, int clients, int cols,
                                                uint32_t *out) {
#pragma unroll
  for (int cl = 0; cl < 4; ++cl) {
    const uint32_t acc = r[4 * cl] + (r[4 * cl + 1] << 8) + (r[4 * cl + 2] << 16) + (r[4 * cl + 3] << 24);
    const int c = c0 + cl;
    if (row_ok && c < clients) atomicAdd(out + (size_t)c * cols + col, acc);
  }
}

// Epilogue of 16 TMEM columns for one accumulator row of the pack: row = (column, plane j); the 4 planes of a column
// are 4 adjacent lanes of one warp.  Each lane reduces its plane's sum S_j = sum_i G_ij 2^(8i) (< 2^57) once,
// shifts it into place (< 2^56), and the four planes are summed in 64 bits by two shuffles (< 2^58) before the one
// final reduction mod Q.
__device__ __forceinline__ void pack_epilogue16(const uint32_t *r, int grow, bool row_ok, int c0, int clients,
                                                int cols, uint32_t *out) {
  const int col = grow >> 2, plane = grow & 3;
#pragma unroll
  for (int cl = 0; cl < 4; ++cl) {
    const uint64_t sum = (uint64_t)r[4 * cl] + ((uint64_t)r[4 * cl + 1] << 8) + ((uint64_t)r[4 * cl + 2] << 16) +
                         ((uint64_t)r[4 * cl + 3] << 24);
    uint64_t u = mod_q64(sum) << (8 * plane);
    u += __shfl_xor_sync(0xffffffffu, u, 1);
    u += __shfl_xor_sync(0xffffffffu, u, 2);
    const int c = c0 + cl;
    if (plane == 0 && row_ok && c < clients) out[(size_t)c * cols + col] = (uint32_t)mod_q64(u);
  }
}

template <int BN, Epi EPI, int NSUB = 1>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kGemmThreads, 1)
    limb_gemm_pair_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                          PairArgs args) {
  using S = PairShape<BN, NSUB>;
  constexpr int kBufs = S::kBufs;
  constexpr int kStages = S::kStages;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base_addr = (raw_addr + 1023u) & ~1023u;
  uint8_t *smem = smem_raw + (base_addr - raw_addr);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kStages * S::kStageBytes);
  // bars: [0, S) full, [S, 2S) empty, 2S + b acc_full[b], 2S + 2 + b acc_empty[b] (b < kBufs)
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 4);
  volatile int *bail = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // the tile width: a multiple of 32 in [32, BN] (the host checks), BN with NSUB = 2
  const int nw = (NSUB == 1 && args.nw >= 32 && args.nw <= BN && args.nw % 32 == 0) ? args.nw : BN;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int pair = blockIdx.x >> 1, pairs = gridDim.x >> 1;
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages);
  const uint32_t accf0 = smem_u32(bars + 2 * kStages), acce0 = smem_u32(bars + 2 * kStages + 2);

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf0 + 8 * b, 1);
      mbar_init(acce0 + 8 * b, 8);  // 4 epilogue warps x 2 CTAs
    }
    *bail = 0;
    fence_barrier_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&map_a);
    tma_prefetch_desc(&map_b);
  }
  if (warp == 1) {
    tmem_alloc_pair(smem_u32(tmem_slot), S::kTmemCols);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // barrier initialisation visible to the peer before any of its loads signal the leader
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  volatile int no_bail = 0;

  auto unit_coords = [&](int u, int &m, int &n, int &kb0, int &nkb) {
    n = u % args.num_n;
    m = args.m_begin + (u / args.num_n) % args.num_m;
    const int kc = u / (args.num_n * args.num_m);
    kb0 = args.kb_begin + kc * args.kb_per_unit;
    nkb = min(kb0 + args.kb_per_unit, args.kb_total) - kb0;
  };

  if (warp == 0) {
    // ------------------------------------------------------------ TMA producer (both CTAs)
    if (lane == 0) {
      // both CTAs' A tiles and B boxes of this stage: the B box is nw/2 rows (the host makes the map with that box)
      const uint32_t stage_tx = 2u * (uint32_t)(S::kABytes + NSUB * (nw / 2) * kBK);
      const uint64_t pol_a = policy_evict_first();
      const uint64_t pol_b = args.b_keep ? policy_evict_last() : policy_evict_normal();
      const uint32_t full_leader0 = map_to_rank(full0, 0);
      int g = 0;
      bool stop = false;
      for (int u = pair; u < args.num_units && !stop; u += pairs) {
        int m, n, kb0, nkb;
        unit_coords(u, m, n, kb0, nkb);
        for (int i = 0; i < nkb; ++i, ++g) {
          const int s = g % kStages, round = g / kStages;
          if (round > 0 && !mbar_wait(empty0 + 8 * s, (round - 1) & 1, args.err, ALTO_ERR_WAIT_EMPTY, bail)) {
            stop = true;
            break;
          }
          const uint32_t sa = base_addr + s * S::kStageBytes, sb = sa + S::kABytes;
          if (leader) mbar_arrive_expect_tx(full0 + 8 * s, stage_tx);
          if constexpr (EPI == Epi::kScan) {
            const int kb = kb0 + i, z = kb / args.kb_chunk, x = (kb - z * args.kb_chunk) * kBK;
            tma_load_tile_pair(sa, &map_a, full_leader0 + 8 * s, kb, 2 * m + (int)rank, pol_a);
#pragma unroll
            for (int t = 0; t < NSUB; ++t)
              tma_load_3d_pair(sb + t * (BN / 2) * kBK, &map_b, full_leader0 + 8 * s, x,
                               (n * NSUB + t) * nw + (int)rank * (nw / 2), z, pol_b);
          } else {
            const int x = (kb0 + i) * kBK;
            tma_load_tile_pair(sa, &map_a, full_leader0 + 8 * s, kb0 + i, 2 * m + (int)rank, pol_a);
#pragma unroll
            for (int t = 0; t < NSUB; ++t)
              tma_load_2d_pair(sb + t * (BN / 2) * kBK, &map_b, full_leader0 + 8 * s, x,
                               (n * NSUB + t) * nw + (int)rank * (nw / 2), pol_b);
          }
        }
      }
      if (stop) {
        // loads already issued land within microseconds; give them a bounded while before the CTA may exit
        const uint64_t t0 = globaltimer();
        while (globaltimer() - t0 < 200000ull) {
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer (leader CTA only)
    if (leader && lane == 0) {
      const uint32_t idesc = idesc_pair_u8u8_s32((uint32_t)nw);
      int g = 0, it = 0;
      bool stop = false;
      for (int u = pair; u < args.num_units && !stop; u += pairs, ++it) {
        int m, n, kb0, nkb;
        unit_coords(u, m, n, kb0, nkb);
        const int ab = it % kBufs, use = it / kBufs;
        if (use > 0 && !mbar_wait(acce0 + 8 * ab, (use - 1) & 1, args.err, ALTO_ERR_WAIT_ACCUM, bail)) break;
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(ab * NSUB * BN);
        for (int i = 0; i < nkb; ++i, ++g) {
          const int s = g % kStages, round = g / kStages;
          if (!mbar_wait(full0 + 8 * s, round & 1, args.err, ALTO_ERR_WAIT_FULL, bail)) {
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t sa = base_addr + s * S::kStageBytes, sb = sa + S::kABytes;
#pragma unroll
          for (int t = 0; t < NSUB; ++t)
#pragma unroll
            for (int kk = 0; kk < kBK / 32; ++kk)
              mma_i8_pair(d_tmem + t * BN, desc_sw128(sa + kk * 32), desc_sw128(sb + t * (BN / 2) * kBK + kk * 32),
                          idesc, (i | kk) != 0);
          mma_commit_pair(empty0 + 8 * s);
        }
        mma_commit_pair(accf0 + 8 * ab);
      }
      if (*bail) {
        // every MMA issued so far completes before this CTA (and its TMEM and shared memory) may go away
        mma_commit_pair(accf0);
        const uint64_t t0 = globaltimer();
        while (globaltimer() - t0 < 200000ull) {
        }
      }
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue (warps 2..5 of both CTAs)
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const uint32_t acce_leader0 = map_to_rank(acce0, 0);
    int it = 0;
    for (int u = pair; u < args.num_units; u += pairs, ++it) {
      int m, n, kb0, nkb;
      unit_coords(u, m, n, kb0, nkb);
      const int ab = it % kBufs, use = it / kBufs;
      if (!mbar_wait(accf0 + 8 * ab, use & 1, args.err, ALTO_ERR_WAIT_ACCUM, bail)) break;
      tc_fence_after();
      const uint32_t taddr = tmem_base + (uint32_t)(ab * NSUB * BN) + ((uint32_t)(q * 32) << 16);
      const int grow = m * 256 + (int)rank * 128 + row;
      const bool row_ok = grow < args.rows_a;
      // 32 columns per TMEM load (one wait per 8 clients instead of per 4)
#pragma unroll 1
      for (int ch = 0; ch < NSUB * nw / 32; ++ch) {
        uint32_t r[32];
        tmem_ld32(taddr + ch * 32, r);
        tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c0 = n * NSUB * (nw / 4) + ch * 8 + h * 4;
          if constexpr (EPI == Epi::kScan)
            scan_epilogue16(r + 16 * h, grow, row_ok, c0, args.clients, args.cols, args.out);
          else
            pack_epilogue16(r + 16 * h, grow, row_ok, c0, args.clients, args.cols, args.out);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(acce_leader0 + 8 * ab);
    }
  }

  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // the peer's last arrivals and TMEM reads are done before either CTA frees anything
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, S::kTmemCols);
  }
  (void)no_bail;
}

}  // namespace alto
