// altopir.hpp -- the C++ host layer over the C ABI of libaltopir_gpu.so (altopir_gpu.h), mirroring the reference's
// Rust host side for the answer path: the engine binding of src/engine.rs (Method, MappedBytes, TiledDb,
// build_packing_matrix, Engine) and the parameter and wire-format helpers of src/service.rs (params, request_len,
// response_len, the synthetic record generator, encode_request / decode_request).  Same names, argument meaning and
// checks; where Rust panics (assert!, unwrap) this layer throws std::invalid_argument or std::runtime_error, and
// decode_request reports its errors with the reference's messages.  Header-only, C++17; link -laltopir_gpu.
#pragma once

#include <array>
#include <cstdint>
#include <cstring>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "altopir_gpu.h"

namespace altopir {

// ============================================================================================ src/engine.rs

// Engine.rs Method (src/engine.rs:22-50): both run the same GPU path.
enum class Method { Amx, Vnni };

inline std::optional<Method> parse_method(const std::string &s) {
  if (s == "amx") return Method::Amx;
  if (s == "vnni") return Method::Vnni;
  return std::nullopt;
}
inline const char *method_name(Method m) { return m == Method::Amx ? "amx" : "vnni"; }
inline int method_code(Method m) { return m == Method::Amx ? 0 : 2; }

// engine::init_amx (src/engine.rs:66-69): here, create the CUDA context on the current device.
inline void init() {
  if (sw_amx_init() != 0) throw std::runtime_error(std::string("no usable CUDA device: ") + alto_last_error());
}

// engine::MappedBytes (src/engine.rs:71-99): a zero-filled host mapping owned by this object.
class MappedBytes {
 public:
  static MappedBytes zeroed(size_t len) {
    if (len == 0) throw std::invalid_argument("MappedBytes of zero bytes");
    void *p = sw_alloc_zeroed(len);
    if (!p) throw std::runtime_error("out of memory");
    return MappedBytes(static_cast<uint8_t *>(p), len);
  }
  MappedBytes(MappedBytes &&o) noexcept : ptr_(std::exchange(o.ptr_, nullptr)), len_(o.len_) {}
  MappedBytes &operator=(MappedBytes &&o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(len_, o.len_);
    return *this;
  }
  MappedBytes(const MappedBytes &) = delete;
  MappedBytes &operator=(const MappedBytes &) = delete;
  ~MappedBytes() { sw_free(ptr_); }
  int8_t *as_i8() { return reinterpret_cast<int8_t *>(ptr_); }
  const int8_t *as_i8() const { return reinterpret_cast<const int8_t *>(ptr_); }
  size_t size() const { return len_; }

 private:
  MappedBytes(uint8_t *p, size_t n) : ptr_(p), len_(n) {}
  uint8_t *ptr_ = nullptr;
  size_t len_ = 0;
};

// engine::TiledDb (src/engine.rs:101-124): sw_tile_db of a column-order database into a buffer of rows * cols.
class TiledDb {
 public:
  TiledDb(const uint8_t *db, size_t db_len, size_t ld, size_t rows, size_t cols, int threads) : rows(rows), cols(cols) {
    if (rows % 64 || cols % 32 || !cols || db_len < (cols - 1) * ld + rows)
      throw std::invalid_argument("TiledDb: rows % 64, cols % 32 or database length");
    ptr_ = static_cast<uint8_t *>(sw_alloc(rows * cols));
    if (!ptr_) throw std::runtime_error("out of memory");
    sw_tile_db(ptr_, db, ld, rows, cols, threads);
  }
  TiledDb(TiledDb &&o) noexcept : rows(o.rows), cols(o.cols), ptr_(std::exchange(o.ptr_, nullptr)) {}
  TiledDb(const TiledDb &) = delete;
  TiledDb &operator=(const TiledDb &) = delete;
  ~TiledDb() { sw_free(ptr_); }
  const uint8_t *data() const { return ptr_; }
  size_t rows, cols;

 private:
  uint8_t *ptr_ = nullptr;
};

// engine::build_packing_matrix (src/engine.rs:126-138): rho = bold_t.size() outputs of n columns.
inline void build_packing_matrix(int8_t *ub, size_t ub_len, const std::vector<const uint64_t *> &bold_t,
                                 const std::vector<const uint64_t *> &bold_t_bar, const uint32_t *tables,
                                 size_t tables_len, const uint32_t *gen_pows, size_t gen_pows_len, size_t num_iter,
                                 size_t tg, size_t n, uint64_t qmod, int threads) {
  const size_t rho = bold_t.size();
  if (ub_len != 4 * tg * n * rho * n || bold_t_bar.size() != rho)
    throw std::invalid_argument("build_packing_matrix: buffer size or output count");
  if (tables_len != n * n || gen_pows_len < num_iter) throw std::invalid_argument("build_packing_matrix: tables");
  sw_pack_build(ub, bold_t.data(), bold_t_bar.data(), tables, gen_pows, num_iter, tg, n, rho, qmod, threads);
}

// engine::Engine (src/engine.rs:140-195).  The device copies every input at construction, so the buffers passed
// here may be released once the constructor returns (the Rust binding borrows them for the engine's lifetime).
class Engine {
 public:
  Engine(const uint8_t *db_col, size_t db_len, const TiledDb &tiled, size_t ld, const int8_t *ub, size_t ub_len,
         size_t n, size_t tg, const std::vector<std::vector<uint8_t>> &prefixes, size_t row1_off, uint64_t q1,
         int q1_bits, const std::vector<const uint64_t *> &that, size_t that_len, const uint64_t *inv_table,
         size_t inv_len, uint64_t q, int threads) {
    const size_t rows = tiled.rows, cols = tiled.cols;
    if (!n || cols % n || db_len < (cols - 1) * ld + rows || ub_len != 4 * tg * n * cols ||
        prefixes.size() != cols / n || that.size() != cols / n || that_len < tg * n || inv_len < n)
      throw std::invalid_argument("Engine: buffer sizes do not match the configuration");
    const size_t part_len = prefixes[0].size();
    std::vector<const uint8_t *> pp;
    for (const auto &p : prefixes) {
      if (p.size() != part_len) throw std::invalid_argument("Engine: prefixes of different lengths");
      pp.push_back(p.data());
    }
    ptr_ = alto_engine_new(db_col, tiled.data(), ld, rows, cols, ub, n, tg, pp.data(), part_len, row1_off, q1, q1_bits,
                           that.data(), inv_table, q, threads);
    if (!ptr_) throw std::runtime_error(std::string("unsupported engine configuration: ") + alto_last_error());
  }
  Engine(Engine &&o) noexcept : ptr_(std::exchange(o.ptr_, nullptr)) {}
  Engine(const Engine &) = delete;
  Engine &operator=(const Engine &) = delete;
  ~Engine() { alto_engine_free(ptr_); }

  size_t request_len() const { return alto_request_len(ptr_); }
  size_t response_len() const { return alto_response_len(ptr_); }

  // Engine::answer: req[c] (request frames, len[c] bytes each, NULL allowed), out[c] (response_len bytes each),
  // status[c]; returns the number of valid requests and stage_ms.  Throws on a negative engine code.
  std::pair<size_t, std::array<double, 4>> answer(const std::vector<const uint8_t *> &req,
                                                  const std::vector<size_t> &len, const std::vector<uint8_t *> &out,
                                                  std::vector<int> &status, Method method) {
    const size_t b = req.size();
    if (len.size() != b || out.size() != b) throw std::invalid_argument("Engine::answer: batch sizes differ");
    status.assign(b, -1);
    std::array<double, 4> stage{};
    const int r = alto_answer(ptr_, req.data(), len.data(), b, out.data(), status.data(), method_code(method),
                              stage.data());
    if (r < 0) throw std::runtime_error("engine error " + std::to_string(r) + ": " + alto_last_error());
    return {static_cast<size_t>(r), stage};
  }

  void *raw() { return ptr_; }

 private:
  void *ptr_ = nullptr;
};

// ============================================================================================ src/service.rs

constexpr size_t MIN_RECORDS = 2048;
constexpr size_t RECORD_UNIT = 2048;
constexpr size_t DEFAULT_RECORD_BYTES = 32768;
constexpr uint64_t Q = 4294955009ull;

// The parameters of service::params (src/service.rs:19-29) that the answer path uses: poly_len n = 2048, t_exp_left
// tg = 4, instances = record_bytes / 2048, q1 = 2^10 (10-bit row 1), row 0 at 18 bits per coefficient.
struct Params {
  size_t rows = 0, record_bytes = 0;
  size_t n = 2048, tg = 4;
  size_t instances() const { return record_bytes / n; }
  size_t count() const { return tg * n; }
  int q1_bits() const { return 10; }
  uint64_t q1() const { return 1ull << q1_bits(); }
  size_t row1_off() const { return 18 * n; }
  size_t part_len() const { return ((18 * n + 10 * n + 63) / 64 * 64 + 7) / 8; }
};

inline Params params(size_t rows, size_t record_bytes) {
  if (rows < MIN_RECORDS || (rows & (rows - 1)))
    throw std::invalid_argument("the number of records must be a power of two and at least " +
                                std::to_string(MIN_RECORDS));
  if (record_bytes == 0 || record_bytes % RECORD_UNIT)
    throw std::invalid_argument("the record size must be a positive multiple of " + std::to_string(RECORD_UNIT) +
                                " bytes");
  Params p;
  p.rows = rows;
  p.record_bytes = record_bytes;
  return p;
}

inline size_t record_bytes(const Params &p) { return p.instances() * p.n; }
inline size_t request_len(const Params &p, size_t rows) { return 9 + 4 * (2 * p.tg * p.n + rows); }
inline size_t response_len(const Params &p) { return p.instances() * p.n * 28 / 8; }

// service::synthetic (src/service.rs:43-78): the reference's benchmark records.
namespace synthetic {
constexpr uint64_t SEED = 0x416c746f504952ull;

inline uint64_t mix(uint64_t &state) {
  state += 0x9e3779b97f4a7c15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

inline std::vector<uint8_t> record(size_t row, size_t bytes) {
  if (bytes % 2) throw std::invalid_argument("record bytes must be even");
  uint64_t state = SEED ^ (0xd1b54a32d192ed03ull * (uint64_t)(row + 1));
  std::vector<uint8_t> out(bytes);
  for (size_t i = 0; i < bytes / 2; ++i) {
    const uint16_t v = (uint16_t)(mix(state) % 65535);
    out[2 * i] = (uint8_t)v;
    out[2 * i + 1] = (uint8_t)(v >> 8);
  }
  return out;
}

// Record-major database of `rows` records (the layout of the reference's flat database).
inline std::vector<uint8_t> database(size_t rows, size_t bytes) {
  std::vector<uint8_t> out(rows * bytes);
  for (size_t r = 0; r < rows; ++r) {
    const auto rec = record(r, bytes);
    std::memcpy(out.data() + r * bytes, rec.data(), bytes);
  }
  return out;
}
}  // namespace synthetic

// service::encode_request (src/service.rs:178-198): [0][u32 count][u32 count][y][z][query], little endian.
inline std::vector<uint8_t> encode_request(const Params &p, const std::vector<uint64_t> &y,
                                           const std::vector<uint64_t> &z, const std::vector<uint64_t> &query,
                                           size_t rows) {
  const size_t count = p.count();
  if (query.size() != rows || y.size() != count || z.size() != count)
    throw std::invalid_argument("encode_request: key or query length");
  std::vector<uint8_t> out;
  out.reserve(request_len(p, rows));
  auto put = [&](uint32_t v) {
    for (int b = 0; b < 4; ++b) out.push_back((uint8_t)(v >> (8 * b)));
  };
  out.push_back(0);
  put((uint32_t)count);
  put((uint32_t)count);
  for (const auto *keys : {&y, &z})
    for (uint64_t v : *keys) {
      if (v >= Q) throw std::invalid_argument("encode_request: packing key coefficient out of range");
      put((uint32_t)v);
    }
  for (uint64_t v : query) {
    if (v > 0xffffffffull) throw std::invalid_argument("encode_request: query word out of range");
    put((uint32_t)v);
  }
  return out;
}

struct Request {
  std::vector<uint32_t> y, z, query;
};

// service::decode_request (src/service.rs:200-225): the keys and query words of a frame, or the reference's error
// message in `error` (the frame checks of the engine's statuses 1, 2 and 3, in that order).
inline std::optional<Request> decode_request(const Params &p, const uint8_t *input, size_t len, size_t rows,
                                             std::string *error) {
  const size_t count = p.count();
  auto fail = [&](const char *msg) -> std::optional<Request> {
    if (error) *error = msg;
    return std::nullopt;
  };
  if (!input || len != request_len(p, rows) || input[0] != 0) return fail("request flag or length");
  auto u32_at = [&](size_t off) {
    uint32_t v;
    std::memcpy(&v, input + off, 4);
    return v;
  };
  if (u32_at(1) != count || u32_at(5) != count) return fail("packing key length");
  Request r;
  r.y.resize(count);
  r.z.resize(count);
  for (size_t i = 0; i < 2 * count; ++i) {
    const uint32_t v = u32_at(9 + 4 * i);
    if (v >= Q) return fail("packing key coefficient out of range");
    (i < count ? r.y[i] : r.z[i - count]) = v;
  }
  r.query.resize(rows);
  const size_t start = 9 + 8 * count;
  for (size_t i = 0; i < rows; ++i) r.query[i] = u32_at(start + 4 * i);
  return r;
}

}  // namespace altopir
