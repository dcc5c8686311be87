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

// ============================================================================================ the client
// service::new_request / decrypt_response (src/service.rs:227-257) over src/client.rs and src/packing.rs, restated
// without spiral-rs, as altopir-public_b200/client.py states it (the two build the same frames from the same seed):
// the ring Z_Q[X]/(X^n + 1) with the negacyclic NTT whose slot j is the evaluation at psi^(2 brv(j) + 1), psi the
// smallest primitive 2n-th root of unity (Longa-Naehrig transforms); gadget digits of floor(32 / tg) + 1 bits (9 at
// tg = 4); secrets and errors from
// D(0.5) (Pr[x] ~ exp(-2 x^2)) by an exact 64-bit table over counter-based splitmix64 streams of the client's seed;
// the public query and key masks from seeded streams that alto_engine_offline's caller uses too.
namespace client {

constexpr uint32_t kQ32 = 4294955009u;
constexpr uint64_t kGamma = 0x9e3779b97f4a7c15ull;
constexpr uint64_t QUERY_MASK_SEED = 0x5345454430ull, W_MASK_SEED = 0x5745454437ull, V_MASK_SEED = 0x5645454438ull;
constexpr int GEN = 5, P = 256;
// bits of a gadget digit for t digits: floor(32 / t) + 1 (get_bits_per with log2ceil(Q) = 32), one bit at t = 32
inline int gadget_bits(size_t t) { return t >= 32 ? 1 : (int)(32 / t) + 1; }
constexpr uint64_t DELTA = Q / P;
// floor(2^64 Pr[X <= j - 4]), j = 0..7, X ~ D(0.5)
constexpr uint64_t kCdt[8] = {0x2CDC8ull,           0x33738FE26Bull,       0x114B1F533EAC34ull, 0x1B51A6ACA1B1BEEBull,
                              0xE4AE59535E4E4114ull, 0xFFEEB4E0ACC153CBull, 0xFFFFFFCC8C701D94ull,
                              0xFFFFFFFFFFFD3237ull};

inline uint64_t stream_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * kGamma;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
inline uint32_t public_uniform_at(uint64_t seed, uint64_t i) {
  return (uint32_t)(((stream_at(seed, i) >> 32) * (uint64_t)kQ32) >> 32);
}
inline uint32_t gaussian_at(uint64_t seed, uint64_t i) {
  const uint64_t u = stream_at(seed, i);
  int x = -4;
  for (uint64_t t : kCdt) x += u >= t;
  return x < 0 ? (uint32_t)(kQ32 + x) : (uint32_t)x;
}
inline uint64_t secret_stream(uint64_t seed, uint64_t purpose) {
  return seed * kGamma + purpose * 0xd1b54a32d192ed03ull;
}
inline uint32_t mulq(uint32_t a, uint32_t b) { return (uint32_t)((uint64_t)a * b % kQ32); }
inline uint32_t addq(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a + b) % kQ32); }
inline uint32_t subq(uint32_t a, uint32_t b) { return a >= b ? a - b : (uint32_t)((uint64_t)a + kQ32 - b); }
inline uint32_t powq(uint32_t b, uint64_t e) {
  uint32_t r = 1;
  for (; e; e >>= 1, b = mulq(b, b))
    if (e & 1) r = mulq(r, b);
  return r;
}

class Ring {
 public:
  explicit Ring(size_t n) : n_(n) {
    if (n < 2 || (n & (n - 1)) || (kQ32 - 1) % (2 * n)) throw std::invalid_argument("Ring: 2n must divide Q - 1");
    while ((size_t(1) << logn_) < n) ++logn_;
    uint32_t any = 0;
    for (uint32_t g = 2; !any; ++g) {
      const uint32_t c = powq(g, (kQ32 - 1) / (2 * n));
      if (powq(c, n) == kQ32 - 1) any = c;
    }
    psi_ = any;
    for (uint32_t x = any, k = 1; k < 2 * n; k += 2, x = mulq(x, mulq(any, any))) psi_ = x < psi_ ? x : psi_;
    const uint32_t ipsi = powq(psi_, kQ32 - 2);
    fwd_.resize(n);
    inv_.resize(n);
    for (size_t k = 0; k < n; ++k) {
      fwd_[k] = powq(psi_, brv(k));
      inv_[k] = powq(ipsi, brv(k));
    }
    ninv_ = powq((uint32_t)n, kQ32 - 2);
  }
  size_t n() const { return n_; }
  uint32_t psi() const { return psi_; }
  size_t brv(size_t x) const {
    size_t r = 0;
    for (int b = 0; b < logn_; ++b) r |= ((x >> b) & 1) << (logn_ - 1 - b);
    return r;
  }
  void ntt(uint32_t *a) const {  // Longa-Naehrig Algorithm 1
    for (size_t m = 1, t = n_ / 2; m < n_; m <<= 1, t >>= 1)
      for (size_t i = 0; i < m; ++i)
        for (size_t j = 2 * i * t; j < 2 * i * t + t; ++j) {
          const uint32_t u = a[j], v = mulq(a[j + t], fwd_[m + i]);
          a[j] = addq(u, v);
          a[j + t] = subq(u, v);
        }
  }
  void intt(uint32_t *a) const {  // Longa-Naehrig Algorithm 2, then times n^-1
    for (size_t t = 1, h = n_ / 2; h >= 1; t <<= 1, h >>= 1)
      for (size_t i = 0; i < h; ++i)
        for (size_t j = 2 * i * t; j < 2 * i * t + t; ++j) {
          const uint32_t u = a[j], v = a[j + t];
          a[j] = addq(u, v);
          a[j + t] = mulq(subq(u, v), inv_[h + i]);
        }
    for (size_t j = 0; j < n_; ++j) a[j] = mulq(a[j], ninv_);
  }
  // tau_t(a)(X) = a(X^t) mod X^n + 1, t odd
  std::vector<uint32_t> automorph(const std::vector<uint32_t> &a, size_t t) const {
    std::vector<uint32_t> out(n_, 0);
    for (size_t i = 0; i < n_; ++i) {
      const size_t k = i * t % (2 * n_);
      if (k < n_) out[k] = a[i];
      else out[k - n_] = subq(0, a[i]);
    }
    return out;
  }
  // the engine's inverse-NTT table (get_ntt_inverse_table): psi^-brv(i) / 2
  std::vector<uint64_t> engine_inverse_table() const {
    std::vector<uint64_t> t(n_);
    for (size_t i = 0; i < n_; ++i) t[i] = mulq(inv_[i], (kQ32 + 1) / 2);
    return t;
  }

 private:
  size_t n_;
  int logn_ = 0;
  uint32_t psi_ = 0, ninv_ = 0;
  std::vector<uint32_t> fwd_, inv_;
};

// The public masks: the query's (rows / n) x n coefficient-form a_i, and the key masks w, v (tg x n, NTT form).
inline std::vector<uint64_t> query_masks(const Params &p) {
  std::vector<uint64_t> a(p.rows);
  for (size_t i = 0; i < p.rows; ++i) a[i] = public_uniform_at(QUERY_MASK_SEED, i);
  return a;
}
inline std::vector<uint64_t> packing_mask(const Params &p, uint64_t seed) {
  std::vector<uint64_t> w(p.count());
  for (size_t i = 0; i < w.size(); ++i) w[i] = public_uniform_at(seed, i);
  return w;
}

class Client {
 public:
  Client(const Params &p, uint64_t seed) : p_(p), ring_(p.n), seed_(seed), s_(p.n), s_hat_(p.n) {
    for (size_t i = 0; i < p.n; ++i) s_[i] = gaussian_at(secret_stream(seed, 0), i);
    s_hat_ = s_;
    ring_.ntt(s_hat_.data());
  }
  const Ring &ring() const { return ring_; }

  // PackingKeys::init_full (src/packing.rs:1935-1984): y switches tau_5(s) to s under w, z switches tau_(2n-1)(s)
  // under v; each -s mask + e + tau(s) g in NTT form, tg x n flattened.
  std::pair<std::vector<uint64_t>, std::vector<uint64_t>> packing_keys() const {
    return {ksk_body(GEN, packing_mask(p_, W_MASK_SEED), 1), ksk_body(2 * p_.n - 1, packing_mask(p_, V_MASK_SEED), 2)};
  }

  // generate_query (src/client.rs:288-426) and new_request's scaling (src/service.rs:233-236): the bodies of rows / n
  // RLWE encryptions (-a_i, s a_i + e_i + mu_i), mu = floor(Q / 256) at the index, switched from Q to 2^32.
  std::vector<uint64_t> query(size_t index) {
    if (index >= p_.rows) throw std::invalid_argument("query: index out of range");
    const size_t n = p_.n;
    const uint64_t es = secret_stream(seed_, 16 + queries_++);
    std::vector<uint64_t> out(p_.rows);
    std::vector<uint32_t> a(n);
    for (size_t i = 0; i < p_.rows / n; ++i) {
      for (size_t z = 0; z < n; ++z) a[z] = public_uniform_at(QUERY_MASK_SEED, i * n + z);
      ring_.ntt(a.data());
      for (size_t z = 0; z < n; ++z) a[z] = mulq(a[z], s_hat_[z]);
      ring_.intt(a.data());
      for (size_t z = 0; z < n; ++z) {
        uint32_t v = addq(a[z], gaussian_at(es, i * n + z));
        if (i * n + z == index) v = addq(v, (uint32_t)DELTA);
        out[i * n + z] = (((uint64_t)v << 32) + Q / 2) / Q & 0xffffffffull;
      }
    }
    return out;
  }

  // service::new_request: the frame asking for record `index`.
  std::vector<uint8_t> request(size_t index) {
    const auto keys = packing_keys();
    return encode_request(p_, keys.first, keys.second, query(index), p_.rows);
  }

  // service::decrypt_response: each part's row 0 (18 bits) and row 1 (10 bits) recovered to Z_Q, s row0 + row1
  // rounded to p = 256.  Throws std::runtime_error with the reference's Err messages.
  std::vector<uint8_t> decrypt(const uint8_t *bytes, size_t len) const {
    if (len != response_len(p_))
      throw std::runtime_error("response of " + std::to_string(len) + " bytes, expected " +
                               std::to_string(response_len(p_)));
    const size_t n = p_.n, part = n * 28 / 8;
    std::vector<uint8_t> out;
    std::vector<uint32_t> r0(n), r1(n);
    for (size_t off = 0; off < len; off += part) {
      for (size_t z = 0; z < n; ++z) {
        r0[z] = recover(bits_at(bytes + off, 18 * z, 18), 18);
        r1[z] = recover(bits_at(bytes + off, 18 * n + 10 * z, 10), 10);
      }
      ring_.ntt(r0.data());
      for (size_t z = 0; z < n; ++z) r0[z] = mulq(r0[z], s_hat_[z]);
      ring_.intt(r0.data());
      for (size_t z = 0; z < n; ++z) {
        const uint32_t m = addq(r0[z], r1[z]);
        const int64_t c = m >= Q / 2 ? (int64_t)m - (int64_t)Q : (int64_t)m;
        const int64_t num = c * P + (c >= 0 ? (int64_t)(Q / 2) : -(int64_t)(Q / 2));
        int64_t v = num / (int64_t)Q;  // truncation, as rescale (src/modulus_switch.rs:116-130)
        v = ((v % P) + P) % P;
        if (v > 255) throw std::runtime_error("decrypted value out of range");
        out.push_back((uint8_t)v);
      }
    }
    return out;
  }

 private:
  std::vector<uint64_t> ksk_body(size_t gen, const std::vector<uint64_t> &mask, uint64_t purpose) const {
    const size_t n = p_.n;
    std::vector<uint32_t> tau = ring_.automorph(s_, gen);
    ring_.ntt(tau.data());
    std::vector<uint64_t> out(p_.count());
    std::vector<uint32_t> e(n);
    for (size_t k = 0; k < p_.tg; ++k) {
      for (size_t z = 0; z < n; ++z) e[z] = gaussian_at(secret_stream(seed_, purpose), k * n + z);
      ring_.ntt(e.data());
      const uint32_t g = powq(2, (uint64_t)gadget_bits(p_.tg) * k);
      for (size_t z = 0; z < n; ++z)
        out[k * n + z] = addq(addq(mulq(s_hat_[z], subq(0, (uint32_t)(mask[k * n + z] % kQ32))), e[z]),
                              mulq(tau[z], g));
    }
    return out;
  }
  static uint64_t bits_at(const uint8_t *buf, size_t off, int width) {
    uint64_t v = 0;
    for (int b = 0; b < width; ++b) v |= (uint64_t)((buf[(off + b) >> 3] >> ((off + b) & 7)) & 1) << b;
    return v;
  }
  // rescale(v, 2^bits, Q)
  static uint32_t recover(uint64_t v, int bits) {
    const int64_t m = int64_t(1) << bits, c = (int64_t)v >= m / 2 ? (int64_t)v - m : (int64_t)v;
    const int64_t num = c * (int64_t)Q + (c >= 0 ? m / 2 : -m / 2);
    int64_t t = num >= 0 ? num / m : -((-num) / m);
    t %= (int64_t)Q;
    return (uint32_t)(t < 0 ? t + (int64_t)Q : t);
  }

  Params p_;
  Ring ring_;
  uint64_t seed_;
  uint64_t queries_ = 0;
  std::vector<uint32_t> s_, s_hat_;
};

// The scheme's offline set-up on the device for an engine whose database is resident (Prepared::new over
// alto_engine_offline): the public masks in, the engine's packing state and inverse table replaced.  Returns the
// device milliseconds.
inline double prepare_offline(void *engine, const Params &p) {
  std::vector<uint64_t> q = query_masks(p);
  for (auto &v : q) v = v ? Q - v : 0;  // row 0 of the query ciphertexts: -a_i
  const auto w = packing_mask(p, W_MASK_SEED), v = packing_mask(p, V_MASK_SEED);
  double ms = 0;
  const int r = alto_engine_offline(engine, q.data(), w.data(), v.data(), nullptr, nullptr, nullptr, nullptr, &ms);
  if (r < 0) throw std::runtime_error("alto_engine_offline " + std::to_string(r) + ": " + alto_last_error());
  return ms;
}

}  // namespace client

}  // namespace altopir
