// serving.cuh -- continuous batching over one engine (the serving loop of src/bin/altopir.rs:245-513, without
// the TCP front end).  Included at the end of alto_engine.cu so that it shares the engine's batch machinery.
//
//   submit  -> a bounded FIFO of request frames; a full queue answers BUSY at once (src/bin/altopir.rs:428-437).
//   batcher -> takes whatever is queued, up to max_batch, as soon as a device batch context is free: it never
//              waits for a batch to fill (src/bin/altopir.rs:460-471).  Statuses 1 and 2 are settled on the host;
//              the other frames are copied into the context's pinned buffer, uploaded with one 2-D copy and answered
//              on the context's own stream.  With several contexts, the next batch uploads and computes while the
//              previous ones are still on the GPU.
//   completer -> waits for contexts in submission order, hands each ticket its status and response, frees the
//              context for the batcher, and records the latency from submit to completion.
// A loopback executor (no engine) answers batches on the host with a deterministic function of the frame; it
// exists to test the queueing and batching logic without a device and is never used by an engine-backed server.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
  std::vector<uint8_t> frame;
  std::vector<uint8_t> resp;
  int status = -1;  // 0..3 as alto_answer, -4 device failure
  bool done = false;
  double t_submit = 0, t_done = 0;
};

struct ServeSlot {
  Batch b;
  uint8_t *h_in = nullptr, *h_out = nullptr;  // pinned frames and responses of the batch
  cudaEvent_t done = nullptr;
  std::vector<long long> ids;   // tickets answered on the device, in slot order
};

struct Server {
  Engine *e = nullptr;               // nullptr: loopback executor
  size_t max_batch = 1, queue_cap = 1, want = 0, resp_len = 0;
  double loop_service_s = 0;         // loopback: simulated device time per batch
  std::vector<ServeSlot> slots;
  std::mutex mu;
  std::condition_variable cv;        // any change of queue, slots, in-flight list or tickets
  std::deque<long long> queue;
  std::unordered_map<long long, Ticket> tickets;
  std::deque<int> free_slots, inflight;
  long long next_id = 0;
  bool stop = false, batcher_done = false;
  std::thread batcher, completer;
  // statistics
  std::vector<double> lat_ms;
  long long answered = 0, rejected = 0, busy = 0, failed = 0, batches = 0, batched_frames = 0;
};

// Deterministic stand-in response of the loopback executor: FNV-1a of the frame, expanded by splitmix64.
void loopback_response(const uint8_t *frame, size_t frame_len, uint8_t *out, size_t len) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < frame_len; ++i) h = (h ^ frame[i]) * 1099511628211ull;
  for (size_t i = 0; i < len; i += 8) {
    h += 0x9e3779b97f4a7c15ull;
    uint64_t z = h;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    for (size_t k = 0; k < 8 && i + k < len; ++k) out[i + k] = (uint8_t)(z >> (8 * k));
  }
}

// Host-side statuses 1 and 2 (length, flag byte, key counts) of a frame for a request of `want` bytes and `count`
// key words (src/amx_kernels.cpp:573-575).
int header_status(const std::vector<uint8_t> &f, size_t want, size_t count) {
  if (f.size() != want) return 1;
  uint32_t c1, c2;
  memcpy(&c1, f.data() + 1, 4);
  memcpy(&c2, f.data() + 5, 4);
  return (f[0] != 0 || c1 != count || c2 != count) ? 2 : 0;
}

void finish_ticket(Server *s, Ticket &t, int status, const uint8_t *resp) {
  t.status = status;
  if (status == 0 && resp) t.resp.assign(resp, resp + s->resp_len);
  t.done = true;
  t.t_done = now_s();
  t.frame.clear();
  t.frame.shrink_to_fit();
  if (status == 0) {
    ++s->answered;
    s->lat_ms.push_back(1e3 * (t.t_done - t.t_submit));
  } else if (status > 0) {
    ++s->rejected;
  } else {
    ++s->failed;
  }
}

void batcher_loop(Server *s) {
  const size_t count = s->e ? s->e->count : 0;
  if (s->e) cudaSetDevice(s->e->dev);
  for (;;) {
    std::vector<long long> ids;
    int si = -1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] { return (s->stop && s->queue.empty()) || (!s->queue.empty() && !s->free_slots.empty()); });
      if (s->queue.empty()) break;  // stopping and drained
      si = s->free_slots.front();
      s->free_slots.pop_front();
      const size_t n = std::min(s->queue.size(), s->max_batch);
      for (size_t i = 0; i < n; ++i) {
        ids.push_back(s->queue.front());
        s->queue.pop_front();
      }
      ++s->batches;
      s->batched_frames += (long long)n;
    }
    ServeSlot &sl = s->slots[si];
    sl.ids.clear();
    std::vector<std::pair<long long, int>> early;  // (ticket, status 1/2) settled on the host
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (long long id : ids) {
        Ticket &t = s->tickets[id];
        const int st = s->e ? header_status(t.frame, s->want, count) : (t.frame.size() == s->want ? 0 : 1);
        if (st) {
          early.push_back({id, st});
          continue;
        }
        memcpy(sl.h_in + sl.ids.size() * s->want, t.frame.data(), s->want);
        sl.ids.push_back(id);
      }
      for (auto &x : early) finish_ticket(s, s->tickets[x.first], x.second, nullptr);
    }
    if (!early.empty()) s->cv.notify_all();
    const size_t nc = sl.ids.size();
    bool ok = true;
    if (nc && s->e) {
      Engine *e = s->e;
      Batch *b = &sl.b;
      ok = cudaSetDevice(e->dev) == cudaSuccess &&
           cudaMemcpy2DAsync(b->d_req + kSlotLead, e->slot_stride, sl.h_in, s->want, s->want, nc,
                             cudaMemcpyHostToDevice, b->st) == cudaSuccess &&
           enqueue_batch(e, b, b->d_req, e->slot_stride, nc, b->d_resp, s->resp_len, true) &&
           cudaMemcpyAsync(sl.h_out, b->d_resp, nc * s->resp_len, cudaMemcpyDeviceToHost, b->st) == cudaSuccess &&
           cudaMemcpyAsync(b->h_err, b->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->st) == cudaSuccess &&
           cudaEventRecord(sl.done, b->st) == cudaSuccess;
    } else if (nc) {
      std::this_thread::sleep_for(std::chrono::duration<double>(s->loop_service_s));
      for (size_t i = 0; i < nc; ++i)
        loopback_response(sl.h_in + i * s->want, s->want, sl.h_out + i * s->resp_len, s->resp_len);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (!ok) {
        for (long long id : sl.ids) finish_ticket(s, s->tickets[id], -4, nullptr);
        sl.ids.clear();
      }
      s->inflight.push_back(si);
    }
    s->cv.notify_all();
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->batcher_done = true;
  s->cv.notify_all();
}

void completer_loop(Server *s) {
  if (s->e) cudaSetDevice(s->e->dev);
  for (;;) {
    int si = -1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [&] { return !s->inflight.empty() || s->batcher_done; });
      if (s->inflight.empty()) break;
      si = s->inflight.front();
    }
    ServeSlot &sl = s->slots[si];
    bool ok = true;
    if (s->e && !sl.ids.empty()) {
      ok = cudaEventSynchronize(sl.done) == cudaSuccess && *sl.b.h_err == 0;
      if (*sl.b.h_err) {  // a kernel wait timed out: clear the word for the next batch of this context
        cudaMemsetAsync(sl.b.d_err, 0, sizeof(uint32_t), sl.b.st);
        cudaStreamSynchronize(sl.b.st);
        *sl.b.h_err = 0;
      }
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (size_t i = 0; i < sl.ids.size(); ++i) {
        Ticket &t = s->tickets[sl.ids[i]];
        const int st = !ok ? -4 : (s->e ? sl.b.h_status[i] : 0);
        finish_ticket(s, t, st, sl.h_out + i * s->resp_len);
      }
      sl.ids.clear();
      s->inflight.pop_front();
      s->free_slots.push_back(si);
    }
    s->cv.notify_all();
  }
}

bool server_start(Server *s, int nslots) {
  s->slots.resize(nslots);
  for (int i = 0; i < nslots; ++i) {
    ServeSlot &sl = s->slots[i];
    if (s->e) {
      if (!init_batch(&sl.b, false) || !ensure_capacity(s->e, &sl.b, s->max_batch)) return false;
      ALTO_CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
      ALTO_CK(cudaHostAlloc(&sl.h_in, s->max_batch * s->want, cudaHostAllocDefault));
      ALTO_CK(cudaHostAlloc(&sl.h_out, s->max_batch * s->resp_len, cudaHostAllocDefault));
    } else {
      sl.h_in = static_cast<uint8_t *>(malloc(s->max_batch * s->want));
      sl.h_out = static_cast<uint8_t *>(malloc(s->max_batch * s->resp_len));
    }
    s->free_slots.push_back(i);
  }
  s->batcher = std::thread(batcher_loop, s);
  s->completer = std::thread(completer_loop, s);
  return true;
}

void server_destroy(Server *s) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->batcher.joinable()) s->batcher.join();
  if (s->completer.joinable()) s->completer.join();
  for (ServeSlot &sl : s->slots) {
    if (s->e) {
      destroy_batch(&sl.b);
      if (sl.done) cudaEventDestroy(sl.done);
      cudaFreeHost(sl.h_in);
      cudaFreeHost(sl.h_out);
    } else {
      free(sl.h_in);
      free(sl.h_out);
    }
  }
  delete s;
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  size_t i = (size_t)(p * (double)v.size());
  return v[std::min(i, v.size() - 1)];
}

}  // namespace

extern "C" {

void *alto_server_new(void *engine, size_t max_batch, size_t queue_cap, int slots) {
  Engine *e = static_cast<Engine *>(engine);
  if (!e || !max_batch || !queue_cap || slots < 1 || slots > 8) {
    set_error("bad serving-loop arguments");
    return nullptr;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess) return nullptr;
  Server *s = new Server;
  s->e = e;
  s->max_batch = max_batch;
  s->queue_cap = queue_cap;
  s->want = e->want;
  s->resp_len = e->resp_len;
  if (!server_start(s, slots)) {
    server_destroy(s);
    return nullptr;
  }
  return s;
}

void *alto_server_new_loopback(size_t request_len, size_t response_len, size_t max_batch, size_t queue_cap, int slots,
                               double service_us) {
  if (!request_len || !response_len || !max_batch || !queue_cap || slots < 1 || slots > 8) return nullptr;
  Server *s = new Server;
  s->max_batch = max_batch;
  s->queue_cap = queue_cap;
  s->want = request_len;
  s->resp_len = response_len;
  s->loop_service_s = service_us * 1e-6;
  server_start(s, slots);
  return s;
}

long long alto_server_submit(void *p, const uint8_t *frame, size_t len) {
  Server *s = static_cast<Server *>(p);
  if (!s || (!frame && len)) return -1;
  long long id;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return -1;
    if (s->queue.size() >= s->queue_cap) {
      ++s->busy;
      return -9;
    }
    id = s->next_id++;
    Ticket &t = s->tickets[id];
    t.frame.assign(frame, frame + len);
    t.t_submit = now_s();
    s->queue.push_back(id);
  }
  s->cv.notify_all();
  return id;
}

int alto_server_wait(void *p, long long id, uint8_t *out, size_t out_len, int timeout_ms, double *latency_ms) {
  Server *s = static_cast<Server *>(p);
  if (!s) return -1;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(id);
  if (it == s->tickets.end()) return -1;
  // submitters insert tickets while this thread waits, and a rehash invalidates iterators but not references
  const Ticket &t = it->second;
  if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return t.done; })) return -5;
  const int st = t.status;
  if (st == 0 && out) memcpy(out, t.resp.data(), std::min(out_len, s->resp_len));
  if (latency_ms) *latency_ms = 1e3 * (t.t_done - t.t_submit);
  s->tickets.erase(id);
  return st;
}

int alto_server_stats(void *p, double *out, size_t n) {
  Server *s = static_cast<Server *>(p);
  if (!s || !out) return -1;
  std::lock_guard<std::mutex> lk(s->mu);
  const double v[11] = {(double)s->answered, (double)s->rejected, (double)s->busy, (double)s->failed,
                        (double)s->batches, s->batches ? (double)s->batched_frames / s->batches : 0.0,
                        percentile(s->lat_ms, 0.5), percentile(s->lat_ms, 0.99), percentile(s->lat_ms, 0.999),
                        s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end()),
                        (double)s->queue.size()};
  for (size_t i = 0; i < n && i < 11; ++i) out[i] = v[i];
  return 0;
}

void alto_server_free(void *p) {
  if (p) server_destroy(static_cast<Server *>(p));
}

}  // extern "C"
