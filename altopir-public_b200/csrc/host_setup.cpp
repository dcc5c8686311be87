// host_setup.cpp -- host-side setup entry points of the C ABI: the 2 MiB-aligned host allocator, the database copy
// that replaces AMX tiling, the packing-matrix build, and the deterministic synthetic inputs used by tests and
// benchmarks.  Nothing here runs per batch.
#include <omp.h>
#include <sys/mman.h>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>

#include "../../include/altopir_gpu.h"
#include "modq.cuh"

namespace {

constexpr uint64_t kQ = 4294955009ull;
constexpr size_t kMapAlign = size_t(2) << 20;

// Header stored in the 64 bytes below every pointer returned by map_aligned.
struct MapHeader {
  void *base;
  size_t len;
};

// An anonymous private mapping whose returned address is 2 MiB aligned with a header in the preceding page.
void *map_aligned(size_t bytes) {
  const size_t body = (bytes + kMapAlign - 1) / kMapAlign * kMapAlign;
  const size_t len = body + 2 * kMapAlign;
  void *base = mmap(nullptr, len, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
  if (base == MAP_FAILED) return nullptr;
  uintptr_t p = (reinterpret_cast<uintptr_t>(base) + kMapAlign) / kMapAlign * kMapAlign;  // >= base + 1 byte room
  if (p - reinterpret_cast<uintptr_t>(base) < sizeof(MapHeader)) p += kMapAlign;
  reinterpret_cast<MapHeader *>(p)[-1] = MapHeader{base, len};
  return reinterpret_cast<void *>(p);
}

inline uint64_t finalise(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
// The i-th output of a splitmix64 stream that starts at counter `seed`.
inline uint64_t stream_at(uint64_t seed, uint64_t i) { return finalise(seed + (i + 1) * 0x9e3779b97f4a7c15ull); }
// Uniform in [0, bound) for bound <= 2^32 by a 32 x 32 multiply-high of the stream's top half.
inline uint64_t bounded(uint64_t x, uint64_t bound) { return ((x >> 32) * bound) >> 32; }

inline uint8_t record_byte(uint64_t row, uint64_t col) {
  const uint64_t s0 = 0x416c746f504952ull ^ (0xd1b54a32d192ed03ull * (row + 1));
  const uint32_t v = static_cast<uint32_t>(finalise(s0 + (col / 2 + 1) * 0x9e3779b97f4a7c15ull) % 65535ull);
  return static_cast<uint8_t>((col & 1) ? (v >> 8) : (v & 0xff));
}

inline int nthreads(int threads) { return threads > 0 ? threads : omp_get_max_threads(); }

}  // namespace

extern "C" {

void *sw_alloc(size_t bytes) { return map_aligned(bytes); }

void *sw_alloc_zeroed(size_t bytes) {
  void *p = map_aligned(bytes);
  if (p) memset(p, 0, (bytes + kMapAlign - 1) / kMapAlign * kMapAlign);
  return p;
}

void sw_free(void *p) {
  if (!p) return;
  const MapHeader h = reinterpret_cast<MapHeader *>(p)[-1];
  munmap(h.base, h.len);
}

void sw_tile_db(uint8_t *dst, const uint8_t *db, size_t ld, size_t k, size_t m, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t col = 0; col < m; ++col) memcpy(dst + col * k, db + col * ld, k);
}

void sw_pack_build(int8_t *ub, const uint64_t *const *bold_t, const uint64_t *const *bold_t_bar,
                   const uint32_t *tables, const uint32_t *gen_pows, size_t num_iter, size_t tg, size_t n, size_t rho,
                   uint64_t q, int threads) {
  const size_t K = tg * n;
  uint8_t *out = reinterpret_cast<uint8_t *>(ub);
#pragma omp parallel num_threads(nthreads(threads))
  {
    std::vector<uint64_t> acc(K);
#pragma omp for schedule(dynamic, 16)
    for (size_t col = 0; col < rho * n; ++col) {
      const size_t o = col / n, z = col % n;
      std::fill(acc.begin(), acc.end(), 0);
      for (size_t i = 0; i < num_iter; ++i) {
        const size_t g = gen_pows[i];
        const size_t zp = tables[((g - 1) / 2) * n + z];          // image of z under x -> x^g
        const size_t zb = tables[((2 * n - g - 1) / 2) * n + z];  // and under x -> x^(2n - g)
        const uint64_t *t = bold_t[o] + i * tg * n + z;
        const uint64_t *tb = bold_t_bar[o] + i * tg * n + z;
        for (size_t k = 0; k < tg; ++k) {
          acc[k * n + zp] += t[k * n];
          acc[k * n + zb] += tb[k * n];
        }
      }
      uint8_t *planes = out + col * 4 * K;
      for (size_t k = 0; k < K; ++k) {
        const uint32_t v = static_cast<uint32_t>(acc[k] % q);
        planes[k] = static_cast<uint8_t>(v);
        planes[K + k] = static_cast<uint8_t>(v >> 8);
        planes[2 * K + k] = static_cast<uint8_t>(v >> 16);
        planes[3 * K + k] = static_cast<uint8_t>(v >> 24);
      }
    }
  }
}

void alto_pack_encode(int8_t *ub, const uint32_t *U, size_t cols, size_t K, int threads) {
  uint8_t *out = reinterpret_cast<uint8_t *>(ub);
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t col = 0; col < cols; ++col) {
    const uint32_t *u = U + col * K;
    uint8_t *planes = out + col * 4 * K;
    for (size_t k = 0; k < K; ++k) {
      planes[k] = static_cast<uint8_t>(u[k]);
      planes[K + k] = static_cast<uint8_t>(u[k] >> 8);
      planes[2 * K + k] = static_cast<uint8_t>(u[k] >> 16);
      planes[3 * K + k] = static_cast<uint8_t>(u[k] >> 24);
    }
  }
}

void alto_synthetic_db_col(uint8_t *db, size_t ld, size_t rows, size_t col0, size_t ncols, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t c = 0; c < ncols; ++c)
    for (size_t r = 0; r < rows; ++r) db[c * ld + r] = record_byte(r, col0 + c);
}

void alto_fill_uniform_u32(uint32_t *dst, size_t count, uint64_t bound, uint64_t seed, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t i = 0; i < count; ++i) dst[i] = static_cast<uint32_t>(bounded(stream_at(seed, i), bound));
}

void alto_fill_uniform_u64(uint64_t *dst, size_t count, uint64_t bound, uint64_t seed, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t i = 0; i < count; ++i) dst[i] = bounded(stream_at(seed, i), bound);
}

void alto_fill_bytes(uint8_t *dst, size_t count, uint64_t seed, int threads) {
#pragma omp parallel for num_threads(nthreads(threads)) schedule(static)
  for (size_t i = 0; i < count; ++i) dst[i] = static_cast<uint8_t>(stream_at(seed, i) >> 56);
}

void alto_synthetic_request(uint8_t *frame, size_t rows, size_t tg_n, uint64_t seed, uint64_t client) {
  const uint64_t s = seed ^ (0xd1b54a32d192ed03ull * (client + 1));
  frame[0] = 0;
  const uint32_t cnt = static_cast<uint32_t>(tg_n);
  memcpy(frame + 1, &cnt, 4);
  memcpy(frame + 5, &cnt, 4);
  uint8_t *w = frame + 9;
  for (size_t i = 0; i < 2 * tg_n; ++i) {
    const uint32_t v = static_cast<uint32_t>(bounded(stream_at(s, i), kQ));
    memcpy(w + 4 * i, &v, 4);
  }
  w += 8 * tg_n;
  for (size_t i = 0; i < rows; ++i) {
    const uint32_t v = static_cast<uint32_t>(stream_at(s, 2 * tg_n + i) >> 32);
    memcpy(w + 4 * i, &v, 4);
  }
}

uint64_t alto_rescale_digest(uint64_t q1, uint64_t v0, uint64_t v1, int threads) {
  uint64_t d = 0;
#pragma omp parallel for num_threads(nthreads(threads)) reduction(+ : d) schedule(static)
  for (int64_t v = (int64_t)v0; v < (int64_t)v1; ++v)
    d += (uint64_t)alto::rescale_q((uint32_t)v, (uint32_t)q1) * (2 * (uint64_t)v + 1);
  return d;
}

}  // extern "C"
