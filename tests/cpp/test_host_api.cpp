// The C++ host layer (include/altopir.hpp) against the reference's Rust host side it mirrors: run by
// tests/test_host_cpp.py.  "cpu": parameter checks and messages, wire lengths, the request codec and its errors, the
// synthetic records, TiledDb, Method.  "gpu DIR": an engine built through the C++ layer from the state files in
// DIR answers the frames there; the responses and statuses are written back for the test to check.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

#include "altopir.hpp"

using namespace altopir;

static int failures = 0;
#define CHECK(cond)                                                                  \
  do {                                                                               \
    if (!(cond)) {                                                                   \
      std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                                    \
    }                                                                                \
  } while (0)

template <class F>
static std::string thrown(F f) {
  try {
    f();
  } catch (const std::exception &e) {
    return e.what();
  }
  return "";
}

static int cpu() {
  // service::params (src/service.rs:19-29)
  CHECK(thrown([] { params(3000, 4096); }) == "the number of records must be a power of two and at least 2048");
  CHECK(thrown([] { params(1024, 4096); }) == "the number of records must be a power of two and at least 2048");
  CHECK(thrown([] { params(2048, 4000); }) == "the record size must be a positive multiple of 2048 bytes");
  CHECK(thrown([] { params(2048, 0); }) == "the record size must be a positive multiple of 2048 bytes");
  // request and response sizes of the benchmark configurations
  const size_t rows[5] = {2048, 32768, 262144, 2097152, 524288};
  const size_t want[5] = {73737, 196617, 1114121, 8454153, 2162697};
  for (int i = 0; i < 5; ++i) {
    const Params p = params(rows[i], 32768);
    CHECK(request_len(p, rows[i]) == want[i]);
    CHECK(response_len(p) == 114688 && p.part_len() == 7168 && p.row1_off() == 36864 && record_bytes(p) == 32768);
  }
  // codec round trip and the decoder's errors, in the reference's order
  const Params p = params(2048, 4096);
  std::vector<uint64_t> y(p.count()), z(p.count()), q(p.rows);
  uint64_t s = 7;
  for (auto &v : y) v = synthetic::mix(s) % Q;
  for (auto &v : z) v = synthetic::mix(s) % Q;
  for (auto &v : q) v = synthetic::mix(s) & 0xffffffffu;
  std::vector<uint8_t> f = encode_request(p, y, z, q, p.rows);
  CHECK(f.size() == request_len(p, p.rows));
  std::string err;
  auto r = decode_request(p, f.data(), f.size(), p.rows, &err);
  CHECK(r.has_value());
  if (r) {
    bool same = true;
    for (size_t i = 0; i < p.count(); ++i) same &= r->y[i] == y[i] && r->z[i] == z[i];
    for (size_t i = 0; i < p.rows; ++i) same &= r->query[i] == q[i];
    CHECK(same);
  }
  auto bad = f;
  bad[0] = 1;
  CHECK(!decode_request(p, bad.data(), bad.size(), p.rows, &err) && err == "request flag or length");
  CHECK(!decode_request(p, f.data(), f.size() - 1, p.rows, &err) && err == "request flag or length");
  bad = f;
  bad[1] ^= 1;
  CHECK(!decode_request(p, bad.data(), bad.size(), p.rows, &err) && err == "packing key length");
  bad = f;
  bad[9 + 4 * p.count() + 3] = 0xff;
  bad[9 + 4 * p.count() + 2] = 0xff;
  bad[9 + 4 * p.count() + 1] = 0xff;
  bad[9 + 4 * p.count()] = 0xff;  // z[0] = 2^32 - 1 >= q
  CHECK(!decode_request(p, bad.data(), bad.size(), p.rows, &err) && err == "packing key coefficient out of range");
  y[3] = Q;
  CHECK(!thrown([&] { encode_request(p, y, z, q, p.rows); }).empty());
  // synthetic records equal the library's column-order generator
  const size_t nrec = 256, bytes = 4096;
  std::vector<uint8_t> col(bytes * nrec);
  alto_synthetic_db_col(col.data(), nrec, nrec, 0, bytes, 2);
  bool rec_ok = true;
  for (size_t r0 = 0; r0 < nrec; r0 += 37) {
    const auto rec = synthetic::record(r0, bytes);
    for (size_t c = 0; c < bytes; ++c) rec_ok &= rec[c] == col[c * nrec + r0];
  }
  CHECK(rec_ok);
  // TiledDb: the compact column-order copy; its checks
  TiledDb t(col.data(), col.size(), nrec, 128, 64, 2);
  bool tiled_ok = true;
  for (size_t c = 0; c < 64; ++c)
    for (size_t r0 = 0; r0 < 128; ++r0) tiled_ok &= t.data()[c * 128 + r0] == col[c * nrec + r0];
  CHECK(tiled_ok);
  CHECK(!thrown([&] { TiledDb(col.data(), col.size(), nrec, 100, 64, 1); }).empty());
  // Method (src/engine.rs:22-50) and MappedBytes
  CHECK(parse_method("amx") == Method::Amx && parse_method("vnni") == Method::Vnni && !parse_method("avx"));
  CHECK(std::string(method_name(Method::Vnni)) == "vnni" && method_code(Method::Amx) == 0 &&
        method_code(Method::Vnni) == 2);
  MappedBytes m = MappedBytes::zeroed(1 << 20);
  bool zero = true;
  for (size_t i = 0; i < m.size(); ++i) zero &= m.as_i8()[i] == 0;
  CHECK(zero);
  // Engine's own checks come before the device is touched
  CHECK(!thrown([&] {
           std::vector<std::vector<uint8_t>> pre(1, std::vector<uint8_t>(8));
           std::vector<const uint64_t *> that(1, nullptr);
           Engine(col.data(), col.size(), t, nrec, nullptr, 0, 2048, 4, pre, 0, 1024, 10, that, 0, nullptr, 0, Q, 1);
         }).empty());
  return failures;
}

template <class T>
static std::vector<T> read_all(const std::string &path) {
  std::ifstream in(path, std::ios::binary);
  std::vector<char> bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  std::vector<T> out(bytes.size() / sizeof(T));
  std::memcpy(out.data(), bytes.data(), out.size() * sizeof(T));
  return out;
}

static int gpu(const std::string &dir) {
  // meta: rows record_bytes b
  std::ifstream meta(dir + "/meta.txt");
  size_t rows, rb, b;
  meta >> rows >> rb >> b;
  const Params p = params(rows, rb);
  const size_t outputs = p.instances(), count = p.count(), part = p.part_len();
  auto db = read_all<uint8_t>(dir + "/db_col.bin");  // [col][rows]
  auto ub = read_all<int8_t>(dir + "/ub.bin");
  auto that_flat = read_all<uint64_t>(dir + "/that.bin");  // [output][count]
  auto pre_flat = read_all<uint8_t>(dir + "/prefixes.bin");
  auto inv = read_all<uint64_t>(dir + "/inv.bin");
  auto frames = read_all<uint8_t>(dir + "/frames.bin");  // [b][request_len]
  std::vector<std::vector<uint8_t>> prefixes(outputs);
  std::vector<const uint64_t *> that(outputs);
  for (size_t o = 0; o < outputs; ++o) {
    prefixes[o].assign(pre_flat.begin() + o * part, pre_flat.begin() + (o + 1) * part);
    that[o] = that_flat.data() + o * count;
  }
  init();
  TiledDb tiled(db.data(), db.size(), rows, rows, rb, 4);
  Engine e(db.data(), db.size(), tiled, rows, ub.data(), ub.size(), p.n, p.tg, prefixes, p.row1_off(), p.q1(),
           p.q1_bits(), that, count, inv.data(), inv.size(), Q, 4);
  CHECK(e.request_len() == request_len(p, rows) && e.response_len() == response_len(p));
  const size_t ql = e.request_len(), rl = e.response_len();
  std::vector<uint8_t> out(b * rl, 0);
  std::vector<const uint8_t *> req(b);
  std::vector<size_t> len(b, ql);
  std::vector<uint8_t *> outp(b);
  for (size_t c = 0; c < b; ++c) {
    req[c] = frames.data() + c * ql;
    outp[c] = out.data() + c * rl;
  }
  std::vector<int> status;
  auto [n, stage] = e.answer(req, len, outp, status, Method::Amx);
  (void)stage;
  std::ofstream(dir + "/out.bin", std::ios::binary).write(reinterpret_cast<const char *>(out.data()), out.size());
  std::ofstream(dir + "/status.bin", std::ios::binary)
      .write(reinterpret_cast<const char *>(status.data()), status.size() * sizeof(int));
  std::cout << "answered " << n << "\n";
  return failures;
}

// "client DIR": the client of seed / index in DIR/meta.txt ("rows record_bytes seed index") writes its frame to
// DIR/frame.bin; if DIR/response.bin exists, the same client decrypts it into DIR/record.bin.
static int client_files(const std::string &dir) {
  size_t rows = 0, bytes = 0, index = 0;
  uint64_t seed = 0;
  std::ifstream meta(dir + "/meta.txt");
  meta >> rows >> bytes >> seed >> index;
  const Params p = params(rows, bytes);
  client::Client c(p, seed);
  const auto frame = c.request(index);
  std::ofstream(dir + "/frame.bin", std::ios::binary).write((const char *)frame.data(), frame.size());
  std::ifstream resp(dir + "/response.bin", std::ios::binary);
  if (resp) {
    std::vector<uint8_t> r((std::istreambuf_iterator<char>(resp)), std::istreambuf_iterator<char>());
    const auto rec = c.decrypt(r.data(), r.size());
    std::ofstream(dir + "/record.bin", std::ios::binary).write((const char *)rec.data(), rec.size());
  }
  CHECK(thrown([&] { c.decrypt(frame.data(), 10); }).find("expected") != std::string::npos);
  return failures;
}

// "scheme ROWS BYTES": everything in C++ on the GPU -- an engine over the synthetic records generated on the
// device, the scheme's offline set-up on the device, requests of four clients answered in one batch, decrypted.
static int scheme(size_t rows, size_t bytes) {
  init();
  const Params p = params(rows, bytes);
  const size_t outputs = p.instances();
  std::vector<int8_t> ub(4 * bytes * p.count(), 0);
  std::vector<std::vector<uint8_t>> pre(outputs, std::vector<uint8_t>(p.part_len(), 0));
  std::vector<std::vector<uint64_t>> th(outputs, std::vector<uint64_t>(p.count(), 0));
  std::vector<const uint8_t *> pp;
  std::vector<const uint64_t *> tp;
  for (size_t o = 0; o < outputs; ++o) {
    pp.push_back(pre[o].data());
    tp.push_back(th[o].data());
  }
  const auto inv = client::Ring(p.n).engine_inverse_table();
  void *e = alto_engine_new_empty(rows, bytes, ub.data(), p.n, p.tg, pp.data(), p.part_len(), p.row1_off(), p.q1(),
                                  p.q1_bits(), tp.data(), inv.data(), Q, 1);
  CHECK(e != nullptr);
  if (!e) return failures;
  CHECK(alto_engine_fill_synthetic(e) == 0);
  const double ms = client::prepare_offline(e, p);
  CHECK(ms > 0);
  const size_t idx[4] = {0, 7, rows / 2 + 3, rows - 1};
  std::vector<client::Client> clients;
  std::vector<std::vector<uint8_t>> frames, outs(4, std::vector<uint8_t>(response_len(p)));
  std::vector<const uint8_t *> req;
  std::vector<size_t> len;
  std::vector<uint8_t *> outp;
  for (int k = 0; k < 4; ++k) {
    clients.emplace_back(p, 1000 + k);
    frames.push_back(clients.back().request(idx[k]));
  }
  for (int k = 0; k < 4; ++k) {
    req.push_back(frames[k].data());
    len.push_back(frames[k].size());
    outp.push_back(outs[k].data());
  }
  std::vector<int> status(4, -1);
  std::array<double, 4> stage{};
  CHECK(alto_answer(e, req.data(), len.data(), 4, outp.data(), status.data(), 0, stage.data()) == 4);
  for (int k = 0; k < 4; ++k) {
    CHECK(status[k] == 0);
    CHECK(clients[k].decrypt(outs[k].data(), outs[k].size()) == synthetic::record(idx[k], bytes));
  }
  alto_engine_free(e);
  std::cout << "offline set-up " << ms << " ms\n";
  return failures;
}

int main(int argc, char **argv) {
  const std::string mode = argc > 1 ? argv[1] : "cpu";
  int f;
  if (mode == "gpu" && argc > 2) f = gpu(argv[2]);
  else if (mode == "client" && argc > 2) f = client_files(argv[2]);
  else if (mode == "scheme" && argc > 3) f = scheme(std::stoull(argv[2]), std::stoull(argv[3]));
  else f = cpu();
  if (f == 0) std::cout << "OK\n";
  return f == 0 ? 0 : 1;
}
