// serving.cuh -- continuous batching over one engine (the engine loop of src/bin/altopir.rs:403-510, without the
// TCP front end).  Included at the end of alto_engine.cu so that it shares the engine's batch machinery.
//
//   submit    -> the frame is copied, by the submitting thread and outside the loop's lock, into a pinned frame pool
//                of queue_cap entries; a full pool answers BUSY at once (src/bin/altopir.rs:428-437).  The hash of the
//                frame's packing keys y is taken here too.
//   batcher   -> takes whatever is queued, up to max_batch, as soon as a device batch context is free: it never
//                waits for a batch to fill (src/bin/altopir.rs:460-471), and frames that arrive while every context is
//                busy join the next batch.  Statuses 1 and 2 are settled on the host.  Each frame is then either
//                resident -- its client's pack product beta = y U is held in HBM from an earlier request with the
//                same y keys (compared byte for byte) -- or new: the batch computes its pack, and when the client is
//                admitted to a row of the resident table (free HBM, or the least recently used idle row) the batch
//                stores its beta there.  New frames go first in the batch and only they run the pack GEMM; resident
//                frames gather their beta rows.  The frames upload straight from the pool (DMA), the batch runs on
//                the context's own stream, and its responses download into the context's pinned buffer.
//   completer -> waits for contexts in submission order, copies each ticket's response out of the context (outside
//                the lock), publishes statuses, records the latency from submit to completion and the batch's log
//                row, and hands the context back to the batcher, which settles the resident table.
// The resident table belongs to the batcher thread alone.  A loopback executor (no engine) answers batches on the
// host with a deterministic function of the frame; it exists to test queueing and batching without a device.
#pragma once
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <thread>
#include <unordered_map>

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// 64-bit hash of a byte run (multiply-xor over 8-byte words); equal hashes are confirmed by comparing the bytes.
uint64_t key_hash(const uint8_t *p, size_t n) {
  uint64_t h = 0x9e3779b97f4a7c15ull ^ n;
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    memcpy(&w, p + i, 8);
    h = (h ^ w) * 0xff51afd7ed558ccdull;
    h ^= h >> 29;
  }
  for (; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h ^ (h >> 32);
}

struct Ticket {
  int pool = -1;  // entry of the frame pool holding the frame, -1 once released
  size_t len = 0;
  uint64_t key = 0;  // key_hash of the y keys
  std::vector<uint8_t> resp;
  int status = -1;  // 0..3 as alto_answer, -4 device failure
  bool done = false;
  double t_submit = 0, t_done = 0;
};

// A resident client: beta = y U (mod Q, scaled as the engine stores it) of its y keys in row `row` of the table.
struct Resident {
  uint64_t key = 0;
  std::vector<uint8_t> y;  // the y key bytes it was admitted with
  int row = -1;
  int in_flight = 0;  // batches in flight that read or write the row
  bool valid = false;  // the row holds beta (the admitting batch completed with status 0)
  std::list<int>::iterator lru;
};

// One row of the per-batch log: [t_dispatch, t_done] on the loop's clock (s), frames taken, frames on the device,
// frames that ran the pack, frames answered from resident rows, then device ms: upload, pack and gather, scan + tails
// + download, total.
constexpr int kLogFields = 10;
constexpr size_t kLogRows = 65536;
constexpr int kBaseSlots = 2;  // contexts that take any batch; the others wait for a deep queue (Server::deep_queue)

struct ServeSlot {
  Batch b;
  uint8_t *h_out = nullptr;  // pinned responses of the batch
  int *h_rows = nullptr, *d_rows = nullptr;  // per frame: table row to gather from (resident) or store into, or -1
  cudaEvent_t done = nullptr, ev0 = nullptr, ev_up = nullptr, ev_pack = nullptr;
  cudaEvent_t ev_valid = nullptr, ev_sgrp[kQueryGroups] = {};  // validation done; each query chunk group split
  std::vector<long long> ids;  // tickets on the device, in batch order
  std::vector<Ticket *> tix;
  std::vector<int> res;  // resident-table entry per frame (-1 none), in batch order
  std::vector<uint8_t> admit;  // 1 when the frame's batch admits its entry
  int n_new = 0, taken = 0;
  bool failed = false;  // the batch did not complete on the device: none of its admissions holds a row
  double t_dispatch = 0;
};

struct Server {
  Engine *e = nullptr;  // nullptr: loopback executor
  size_t max_batch = 1, queue_cap = 1, want = 0, resp_len = 0, pitch = 0;
  double loop_service_s = 0;  // loopback: simulated device time per batch
  std::vector<ServeSlot> slots;
  uint8_t *pool = nullptr;  // frame pool: entry i at pool + i * pitch (pinned for an engine)
  // free pool entries, handed out first in, first out: consecutive tickets get consecutive entries (the entries come
  // back batch by batch in submission order), so a batch's frames upload in a few pitched copies, not one per frame
  std::deque<int> free_pool;
  bool pool_lifo = false;  // ALTO_SERVE_POOL=lifo: last in, first out (the earlier order, for comparison)
  std::mutex mu;
  std::condition_variable cv;  // any change of queue, slots, in-flight or completed lists, or tickets
  std::deque<long long> queue;
  std::unordered_map<long long, Ticket> tickets;
  std::deque<int> free_slots, inflight, completed;
  // contexts beyond the first kBaseSlots take a batch only while the queue holds at least deep_queue frames: a
  // third concurrent full-database scan raises every batch's latency below saturation and pays only at it
  size_t deep_queue = 0;
  long long next_id = 0;
  bool stop = false, batcher_done = false;
  std::thread batcher, completer;
  // resident table (batcher thread only)
  uint32_t *d_table = nullptr;
  size_t table_rows = 0, ybytes = 0;
  std::vector<Resident> res;
  std::vector<int> free_res;
  std::list<int> lru;  // least recently used first
  std::unordered_map<uint64_t, int> by_key;
  // statistics (under mu)
  std::vector<double> lat_ms;
  long long answered = 0, rejected = 0, busy = 0, failed = 0, batches = 0, batched_frames = 0;
  long long hits = 0, admitted = 0, evicted = 0, uncached = 0;
  std::vector<double> log;  // ring of kLogRows rows
  size_t log_rows = 0;
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

// Host-side status 2 (flag byte, key counts) of a frame of the right length (src/amx_kernels.cpp:573-575).
int header_status(const uint8_t *f, size_t count) {
  uint32_t c1, c2;
  memcpy(&c1, f + 1, 4);
  memcpy(&c2, f + 5, 4);
  return (f[0] != 0 || c1 != count || c2 != count) ? 2 : 0;
}

// Under mu.
void finish_ticket(Server *s, Ticket &t, int status) {
  t.status = status;
  t.done = true;
  t.t_done = now_s();
  if (t.pool >= 0) {
    s->free_pool.push_back(t.pool);
    t.pool = -1;
  }
  if (status == 0) {
    ++s->answered;
    s->lat_ms.push_back(1e3 * (t.t_done - t.t_submit));
  } else if (status > 0) {
    ++s->rejected;
  } else {
    ++s->failed;
  }
}

// Beta rows between a batch and the resident table: gather (to_table = 0) copies table row rows[i] into batch row
// first + i; store (to_table = 1) copies batch row first + i into table row rows[i] when the frame is valid.  Rows
// of -1 are skipped.  Grid (16-byte words of a row / 256, frames).
__global__ void beta_rows_kernel(uint32_t *beta, uint32_t *table, const int *rows, const int *status, int first,
                                 size_t cols, int to_table) {
  const int i = blockIdx.y, r = rows[first + i];
  const size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < 0 || w >= cols / 4) return;
  uint4 *b = reinterpret_cast<uint4 *>(beta + (size_t)(first + i) * cols) + w;
  uint4 *t = reinterpret_cast<uint4 *>(table + (size_t)r * cols) + w;
  if (to_table) {
    if (status[first + i] == 0) *t = *b;
  } else {
    *b = *t;
  }
}

// The device part of a serving batch of nc frames already in the context's pool order: frames [0, n_new) run the
// key limb split and the pack GEMM (and, where admitted, store their beta rows), frames [n_new, nc) gather their
// beta rows; validation and the query limb split run on the side stream; then the scan and tails in column groups.
bool enqueue_serving(Server *s, ServeSlot &sl, size_t nc) {
  Engine *e = s->e;
  Batch *bt = &sl.b;
  cudaStream_t st = bt->st, vs = bt->side;
  const size_t n_new = (size_t)sl.n_new;
  int launches = 0;
  ALTO_CK(cudaEventRecord(sl.ev0, st));
  // A database of several record chunks: the headers and keys upload first, then the query words chunk group by
  // chunk group on the side stream, each group split as soon as it is in, and each group's scan starts once its
  // split is done (as alto_answer does), so that the upload of the later chunks overlaps the scan of the earlier
  // ones.  Otherwise the whole frames upload at once.
  const bool piped = e->nchunks > 1 && 4 * nc * e->rows >= e->piped_bytes;
  const size_t qoff = 9 + 8 * e->count;
  auto pool_at = [&](size_t i) { return s->pool + (size_t)sl.tix[i]->pool * s->pitch; };
  if (!copy_runs(
          nc, piped ? qoff : s->want, [&](size_t i) { return (const void *)pool_at(i); },
          [&](size_t i) { return (void *)(bt->d_req + i * e->slot_stride + kSlotLead); }, cudaMemcpyHostToDevice, st))
    return false;
  ALTO_CK(cudaMemcpyAsync(sl.d_rows, sl.h_rows, nc * sizeof(int), cudaMemcpyHostToDevice, st));
  ALTO_CK(cudaEventRecord(sl.ev_up, st));
  // validation, status download and query limb split beside the pack
  ALTO_CK(cudaEventRecord(bt->ev_fork, st));
  ALTO_CK(cudaStreamWaitEvent(vs, bt->ev_fork, 0));
  alto::validate_kernel<<<(unsigned)nc, 256, 0, vs>>>(bt->d_req, e->slot_stride, kSlotLead, e->count, e->rows,
                                                      bt->d_status);
  ALTO_CK(cudaGetLastError());
  ++launches;
  ALTO_CK(cudaMemcpyAsync(bt->h_status, bt->d_status, nc * sizeof(int), cudaMemcpyDeviceToHost, vs));
  ALTO_CK(cudaEventRecord(sl.ev_valid, vs));
  const size_t gsz = (e->nchunks + kQueryGroups - 1) / kQueryGroups;  // chunks per group
  const int qgroups = piped ? (int)((e->nchunks + gsz - 1) / gsz) : 1;
  auto group_rows = [&](int k, size_t *r0, size_t *r1) {
    *r0 = (size_t)k * gsz * e->chunk;
    *r1 = std::min(e->rows, (size_t)(k + 1) * gsz * e->chunk);
  };
  const int bq = (int)round_up(nc, 4);
  if (!piped) {
    if (!enqueue_query_split(e, bt, bt->d_req, e->slot_stride, nc, vs)) return false;
    ++launches;
    ALTO_CK(cudaEventRecord(bt->ev_qready, vs));
  } else {
    ALTO_CK(cudaMemsetAsync(bt->d_acc, 0, nc * e->cols * sizeof(uint32_t), vs));
    for (int k = 0; k < qgroups; ++k) {
      size_t r0, r1;
      group_rows(k, &r0, &r1);
      if (!copy_runs(
              nc, 4 * (r1 - r0), [&](size_t i) { return (const void *)(pool_at(i) + qoff + 4 * r0); },
              [&](size_t i) { return (void *)(bt->d_req + i * e->slot_stride + kSlotLead + qoff + 4 * r0); },
              cudaMemcpyHostToDevice, vs))
        return false;
      const size_t work = ((r1 - r0) / 16) * (size_t)bq;
      alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, vs>>>(
          bt->d_req, e->slot_stride, kSlotLead + qoff + 4 * r0, (int)nc, bq, r1 - r0, e->chunk,
          bt->d_qlimb + (r0 / e->chunk) * (4 * (size_t)bq * e->chunk));
      ALTO_CK(cudaGetLastError());
      ++launches;
      ALTO_CK(cudaEventRecord(sl.ev_sgrp[k], vs));
    }
  }
  const Plan ps = make_plan(e, nc);
  CUtensorMap map_q, map_y, unused;
  if (!make_limb_maps(e, ps, bt->d_qlimb, bt->d_ylimb, round_up(nc, 4), &map_q, &unused)) return false;
  if (n_new) {
    const Plan pp = make_plan(e, n_new);
    const int bp = (int)round_up(n_new, 4);
    if (!make_limb_maps(e, pp, bt->d_qlimb, bt->d_ylimb, bp, &unused, &map_y)) return false;
    const size_t work = (e->count / 16) * (size_t)bp;
    alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(
        bt->d_req, e->slot_stride, kSlotLead + 9, (int)n_new, bp, e->count, e->count, bt->d_ylimb);
    ALTO_CK(cudaGetLastError());
    if (!launch_pack(e, pp, map_y, bt->d_beta, n_new, st, bt->d_err)) return false;
    launches += 2;
  }
  const dim3 rgrid((unsigned)((e->cols / 4 + 255) / 256), 1);
  if (nc > n_new) {
    beta_rows_kernel<<<dim3(rgrid.x, (unsigned)(nc - n_new)), 256, 0, st>>>(bt->d_beta, s->d_table, sl.d_rows,
                                                                          bt->d_status, (int)n_new, e->cols, 0);
    ALTO_CK(cudaGetLastError());
    ++launches;
  }
  ALTO_CK(cudaEventRecord(sl.ev_pack, st));
  ALTO_CK(cudaStreamWaitEvent(st, piped ? sl.ev_valid : bt->ev_qready, 0));
  bool store = false;
  for (size_t i = 0; i < n_new; ++i) store |= sl.admit[i] != 0;
  if (store) {  // after validation (joined above): only valid frames' rows are kept
    beta_rows_kernel<<<dim3(rgrid.x, (unsigned)n_new), 256, 0, st>>>(bt->d_beta, s->d_table, sl.d_rows, bt->d_status,
                                                                    0, e->cols, 1);
    ALTO_CK(cudaGetLastError());
    ++launches;
  }
  // The scan in column groups (with the tails and downloads) covers the last quarter of the chunk groups, which it
  // starts once all query words are in; the chunk groups before it scan all columns as they arrive.  The upload of
  // the query words takes about three quarters of the scan's time (link bytes against int8 work per query word at
  // 32 KB records), so by the time the last words are in, about that share of the scan is done.
  const int qtail = qgroups - std::max(1, qgroups / 4);
  int kb_last = 0;
  if (piped) {
    for (int k = 0; k < qtail; ++k) {
      size_t r0, r1;
      group_rows(k, &r0, &r1);
      ALTO_CK(cudaStreamWaitEvent(st, sl.ev_sgrp[k], 0));
      if (!launch_scan(e, ps, map_q, bt->d_acc, nc, st, bt->d_err, 0, -1, (int)(r0 / alto::kBK),
                       (int)((r1 + alto::kBK - 1) / alto::kBK)))
        return false;
      ++launches;
    }
    size_t r0, r1;
    group_rows(qtail, &r0, &r1);
    ALTO_CK(cudaStreamWaitEvent(st, sl.ev_sgrp[qgroups - 1], 0));
    kb_last = (int)(r0 / alto::kBK);
  }
  const Groups groups = column_groups(e, ps, group_weights(e->overlap ? e->groups : 1, false));
  if (!enqueue_scan_tails(e, bt, ps, map_q, bt->d_req, e->slot_stride, nc, bt->d_resp, s->resp_len, groups, nullptr,
                          &launches, nullptr, nullptr, 8, kb_last))
    return false;
  ALTO_CK(cudaMemcpyAsync(sl.h_out, bt->d_resp, nc * s->resp_len, cudaMemcpyDeviceToHost, st));
  ALTO_CK(cudaMemcpyAsync(bt->h_err, bt->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  ALTO_CK(cudaEventRecord(sl.done, st));
  e->last_launches = launches;
  return true;
}

// Batcher thread: resident-table bookkeeping of a completed batch (its entries' in-flight counts, admissions that
// became valid or failed).
void settle(Server *s, ServeSlot &sl) {
  for (size_t i = 0; i < sl.res.size(); ++i) {
    const int r = sl.res[i];
    if (r < 0) continue;
    Resident &x = s->res[r];
    --x.in_flight;
    if (sl.admit[i]) {
      const bool ok = !sl.failed && sl.b.h_status[i] == 0;
      if (ok) {
        x.valid = true;
      } else {  // an invalid or failed admission frees its row again
        s->by_key.erase(x.key);
        s->lru.erase(x.lru);
        x = Resident{};
        x.lru = s->lru.end();
        s->free_res.push_back(r);
      }
    }
  }
  sl.res.clear();
  sl.admit.clear();
}

// Batcher thread: a row for a new client with key `key` (y bytes y), or -1 when every row is in use by a batch.
int admit(Server *s, uint64_t key, const uint8_t *y) {
  int r = -1;
  if (!s->free_res.empty()) {
    r = s->free_res.back();
    s->free_res.pop_back();
  } else {
    for (auto it = s->lru.begin(); it != s->lru.end(); ++it)
      if (s->res[*it].in_flight == 0) {
        r = *it;
        break;
      }
    if (r < 0) return -1;
    Resident &old = s->res[r];
    s->by_key.erase(old.key);
    s->lru.erase(old.lru);
    ++s->evicted;
  }
  Resident &x = s->res[r];
  x.key = key;
  x.y.assign(y, y + s->ybytes);
  x.row = r;
  x.in_flight = 1;
  x.valid = false;
  x.lru = s->lru.insert(s->lru.end(), r);
  s->by_key[key] = r;
  return r;
}

void batcher_loop(Server *s) {
  const size_t count = s->e ? s->e->count : 0;
  if (s->e) cudaSetDevice(s->e->dev);
  for (;;) {
    std::vector<long long> ids;
    std::vector<Ticket *> tix;
    std::vector<int> done_slots;
    int si = -1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // a free context that may take the queue's frames now: the lowest-numbered one (see deep_queue)
      auto pick = [&]() -> int {
        int best = -1;
        for (int d : s->free_slots)
          if ((d < kBaseSlots || s->queue.size() >= s->deep_queue) && (best < 0 || d < best)) best = d;
        return best;
      };
      s->cv.wait(lk, [&] {
        return (s->stop && s->queue.empty()) || !s->completed.empty() || (!s->queue.empty() && pick() >= 0);
      });
      while (!s->completed.empty()) {
        done_slots.push_back(s->completed.front());
        s->completed.pop_front();
      }
      if (done_slots.empty() && s->queue.empty()) break;  // stopping and drained
      if (!s->queue.empty() && pick() >= 0) {
        si = pick();
        s->free_slots.erase(std::find(s->free_slots.begin(), s->free_slots.end(), si));
        const size_t n = std::min(s->queue.size(), s->max_batch);
        for (size_t i = 0; i < n; ++i) {
          ids.push_back(s->queue.front());
          tix.push_back(&s->tickets[s->queue.front()]);
          s->queue.pop_front();
        }
        ++s->batches;
        s->batched_frames += (long long)n;
      }
    }
    if (!done_slots.empty()) {
      for (int d : done_slots) settle(s, s->slots[d]);
      std::lock_guard<std::mutex> lk(s->mu);
      for (int d : done_slots) s->free_slots.push_back(d);
    }
    if (si < 0) {
      s->cv.notify_all();
      continue;
    }
    ServeSlot &sl = s->slots[si];
    sl.t_dispatch = now_s();
    sl.taken = (int)ids.size();
    sl.failed = false;
    sl.ids.clear();
    sl.tix.clear();
    sl.res.clear();
    sl.admit.clear();
    // classify outside the lock: the tickets' frames and keys do not change once queued
    std::vector<std::pair<Ticket *, int>> early;  // status 2 settled on the host
    std::vector<size_t> fresh, resident;          // indices into ids
    std::vector<int> row_of(ids.size(), -1), entry_of(ids.size(), -1);
    std::vector<uint8_t> admit_of(ids.size(), 0);
    for (size_t i = 0; i < ids.size(); ++i) {
      const uint8_t *f = s->pool + (size_t)tix[i]->pool * s->pitch;
      const int st = s->e ? header_status(f, count) : 0;
      if (st) {
        early.push_back({tix[i], st});
        continue;
      }
      if (!s->e || !s->table_rows) {
        fresh.push_back(i);
        continue;
      }
      auto it = s->by_key.find(tix[i]->key);
      if (it != s->by_key.end()) {
        Resident &x = s->res[it->second];
        if (x.valid && memcmp(x.y.data(), f + 9, s->ybytes) == 0) {
          ++x.in_flight;
          s->lru.splice(s->lru.end(), s->lru, x.lru);
          row_of[i] = entry_of[i] = it->second;
          resident.push_back(i);
        } else {
          fresh.push_back(i);  // admitted by a batch still in flight, or another client with the same hash
        }
        continue;
      }
      const int r = admit(s, tix[i]->key, f + 9);
      row_of[i] = entry_of[i] = r;
      admit_of[i] = r >= 0;
      fresh.push_back(i);
    }
    sl.n_new = (int)fresh.size();
    for (size_t k = 0; k < fresh.size() + resident.size(); ++k) {
      const size_t i = k < fresh.size() ? fresh[k] : resident[k - fresh.size()];
      sl.ids.push_back(ids[i]);
      sl.tix.push_back(tix[i]);
      sl.res.push_back(entry_of[i]);
      sl.admit.push_back(admit_of[i]);
      if (sl.h_rows) sl.h_rows[k] = row_of[i];
    }
    if (!early.empty()) {
      std::lock_guard<std::mutex> lk(s->mu);
      for (auto &x : early) finish_ticket(s, *x.first, x.second);
    }
    if (!early.empty()) s->cv.notify_all();
    const size_t nc = sl.ids.size();
    bool ok = true;
    if (nc && s->e) {
      ok = cudaSetDevice(s->e->dev) == cudaSuccess && enqueue_serving(s, sl, nc);
    } else if (nc) {
      std::this_thread::sleep_for(std::chrono::duration<double>(s->loop_service_s));
      for (size_t i = 0; i < nc; ++i)
        loopback_response(s->pool + (size_t)sl.tix[i]->pool * s->pitch, s->want, sl.h_out + i * s->resp_len,
                          s->resp_len);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->hits += (long long)resident.size();
      for (size_t k = 0; k < fresh.size(); ++k) {
        s->admitted += admit_of[fresh[k]];
        s->uncached += s->table_rows && !admit_of[fresh[k]];
      }
      if (!ok) {
        for (Ticket *t : sl.tix) finish_ticket(s, *t, -4);
        sl.ids.clear();
        sl.tix.clear();
        sl.failed = true;
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
    float ms[4] = {0, 0, 0, 0};
    if (s->e && !sl.ids.empty()) {
      ok = cudaEventSynchronize(sl.done) == cudaSuccess && *sl.b.h_err == 0;
      if (ok) {
        cudaEventElapsedTime(&ms[0], sl.ev0, sl.ev_up);
        cudaEventElapsedTime(&ms[1], sl.ev_up, sl.ev_pack);
        cudaEventElapsedTime(&ms[2], sl.ev_pack, sl.done);
        cudaEventElapsedTime(&ms[3], sl.ev0, sl.done);
      }
      if (*sl.b.h_err) {  // a kernel wait timed out: clear the word for the next batch of this context
        cudaMemsetAsync(sl.b.d_err, 0, sizeof(uint32_t), sl.b.st);
        cudaStreamSynchronize(sl.b.st);
        *sl.b.h_err = 0;
      }
      if (!ok) sl.failed = true;
    }
    // responses out of the context, outside the lock (a ticket's response is read only once it is done)
    std::vector<int> st(sl.ids.size());
    for (size_t i = 0; i < sl.ids.size(); ++i) {
      st[i] = !ok ? -4 : (s->e ? sl.b.h_status[i] : 0);
      if (st[i] == 0) sl.tix[i]->resp.assign(sl.h_out + i * s->resp_len, sl.h_out + (i + 1) * s->resp_len);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (size_t i = 0; i < sl.ids.size(); ++i) finish_ticket(s, *sl.tix[i], st[i]);
      if (s->log.empty()) s->log.assign(kLogRows * kLogFields, 0.0);
      double *row = s->log.data() + (s->log_rows % kLogRows) * kLogFields;
      const double fields[kLogFields] = {sl.t_dispatch, now_s(), (double)sl.taken, (double)sl.ids.size(),
                                         (double)sl.n_new, (double)(sl.ids.size() - sl.n_new),
                                         ms[0], ms[1], ms[2], ms[3]};
      std::copy(fields, fields + kLogFields, row);
      ++s->log_rows;
      sl.ids.clear();
      sl.tix.clear();
      s->inflight.pop_front();
      s->completed.push_back(si);
    }
    s->cv.notify_all();
  }
}

// Device rows of the resident table within key_bytes (each cols * 4 bytes).
size_t table_capacity(const Engine *e, size_t key_bytes) { return key_bytes / (e->cols * sizeof(uint32_t)); }

bool server_start(Server *s, int nslots, size_t key_bytes) {
  s->pitch = round_up(s->want, 64);
  s->slots.resize(nslots);
  // contexts beyond the first two wait for half a maximum batch in the queue (ALTO_SERVE_DEEP: frames, 0 = always)
  s->deep_queue = std::max<size_t>(1, s->max_batch / 2);
  if (const char *v = getenv("ALTO_SERVE_DEEP")) s->deep_queue = (size_t)strtoull(v, nullptr, 10);
  if (s->e) {
    ALTO_CK(cudaHostAlloc(&s->pool, s->queue_cap * s->pitch, cudaHostAllocDefault));
    s->ybytes = 4 * s->e->count;
    s->table_rows = table_capacity(s->e, key_bytes);
    if (s->table_rows) {
      ALTO_CK(cudaMalloc(&s->d_table, s->table_rows * s->e->cols * sizeof(uint32_t)));
      s->res.resize(s->table_rows);
      for (size_t r = 0; r < s->table_rows; ++r) {
        s->res[r].lru = s->lru.end();
        s->free_res.push_back((int)(s->table_rows - 1 - r));
      }
    }
  } else {
    s->pool = static_cast<uint8_t *>(malloc(s->queue_cap * s->pitch));
    if (!s->pool) return false;
  }
  if (const char *v = getenv("ALTO_SERVE_POOL")) s->pool_lifo = strcmp(v, "lifo") == 0;
  for (size_t i = 0; i < s->queue_cap; ++i) s->free_pool.push_back((int)(s->pool_lifo ? s->queue_cap - 1 - i : i));
  for (int i = 0; i < nslots; ++i) {
    ServeSlot &sl = s->slots[i];
    if (s->e) {
      if (!init_batch(&sl.b, false) || !ensure_capacity(s->e, &sl.b, s->max_batch)) return false;
      ALTO_CK(cudaEventCreate(&sl.done));
      ALTO_CK(cudaEventCreate(&sl.ev0));
      ALTO_CK(cudaEventCreate(&sl.ev_up));
      ALTO_CK(cudaEventCreate(&sl.ev_pack));
      ALTO_CK(cudaEventCreateWithFlags(&sl.ev_valid, cudaEventDisableTiming));
      for (cudaEvent_t &ev : sl.ev_sgrp) ALTO_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      ALTO_CK(cudaHostAlloc(&sl.h_out, s->max_batch * s->resp_len, cudaHostAllocDefault));
      ALTO_CK(cudaHostAlloc(&sl.h_rows, s->max_batch * sizeof(int), cudaHostAllocDefault));
      ALTO_CK(cudaMalloc(&sl.d_rows, s->max_batch * sizeof(int)));
    } else {
      sl.h_out = static_cast<uint8_t *>(malloc(s->max_batch * s->resp_len));
      if (!sl.h_out) return false;
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
      for (cudaEvent_t ev : {sl.done, sl.ev0, sl.ev_up, sl.ev_pack, sl.ev_valid})
        if (ev) cudaEventDestroy(ev);
      for (cudaEvent_t ev : sl.ev_sgrp)
        if (ev) cudaEventDestroy(ev);
      cudaFreeHost(sl.h_out);
      cudaFreeHost(sl.h_rows);
      cudaFree(sl.d_rows);
    } else {
      free(sl.h_out);
    }
  }
  if (s->e) {
    cudaFreeHost(s->pool);
    cudaFree(s->d_table);
  } else {
    free(s->pool);
  }
  delete s;
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  size_t i = (size_t)(p * (double)v.size());
  return v[std::min(i, v.size() - 1)];
}

// The resident table's default size: a quarter of the device memory free once the batch contexts exist, at most
// 8 GiB.
size_t default_key_bytes() {
  size_t free_b = 0, total = 0;
  if (cudaMemGetInfo(&free_b, &total) != cudaSuccess) return 0;
  return std::min(free_b / 4, size_t(8) << 30);
}

}  // namespace

extern "C" {

void *alto_server_new_keyed(void *engine, size_t max_batch, size_t queue_cap, int slots, size_t key_bytes) {
  Engine *e = static_cast<Engine *>(engine);
  if (!e || !max_batch || !queue_cap || queue_cap > (size_t(1) << 30) || slots < 1 || slots > 8) {
    set_error("bad serving-loop arguments");
    return nullptr;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess) return nullptr;
  if (key_bytes == SIZE_MAX) key_bytes = default_key_bytes();
  Server *s = new Server;
  s->e = e;
  s->max_batch = max_batch;
  s->queue_cap = queue_cap;
  s->want = e->want;
  s->resp_len = e->resp_len;
  if (!server_start(s, slots, key_bytes)) {
    server_destroy(s);
    return nullptr;
  }
  return s;
}

void *alto_server_new(void *engine, size_t max_batch, size_t queue_cap, int slots) {
  return alto_server_new_keyed(engine, max_batch, queue_cap, slots, SIZE_MAX);
}

void *alto_server_new_loopback(size_t request_len, size_t response_len, size_t max_batch, size_t queue_cap, int slots,
                               double service_us) {
  if (!request_len || !response_len || !max_batch || !queue_cap || queue_cap > (size_t(1) << 30) || slots < 1 ||
      slots > 8)
    return nullptr;
  Server *s = new Server;
  s->max_batch = max_batch;
  s->queue_cap = queue_cap;
  s->want = request_len;
  s->resp_len = response_len;
  s->loop_service_s = service_us * 1e-6;
  if (!server_start(s, slots, 0)) {
    server_destroy(s);
    return nullptr;
  }
  return s;
}

long long alto_server_submit(void *p, const uint8_t *frame, size_t len) {
  Server *s = static_cast<Server *>(p);
  if (!s || (!frame && len)) return -1;
  long long id;
  Ticket *t;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return -1;
    if (len == s->want && (s->free_pool.empty() || s->queue.size() >= s->queue_cap)) {
      ++s->busy;
      return -9;
    }
    id = s->next_id++;
    t = &s->tickets[id];
    t->t_submit = now_s();
    t->len = len;
    if (len != s->want) {  // status 1 at once: the frame never reaches a batch (src/amx_kernels.cpp:573)
      finish_ticket(s, *t, 1);
    } else {
      if (s->pool_lifo) {
        t->pool = s->free_pool.back();
        s->free_pool.pop_back();
      } else {
        t->pool = s->free_pool.front();
        s->free_pool.pop_front();
      }
    }
  }
  if (len != s->want) {
    s->cv.notify_all();
    return id;
  }
  // copy and hash outside the lock: the ticket is not queued yet, so nothing else reads its pool entry
  uint8_t *dst = s->pool + (size_t)t->pool * s->pitch;
  memcpy(dst, frame, len);
  const uint64_t key = s->e && len >= 9 + s->ybytes ? key_hash(dst + 9, s->ybytes) : 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    t->key = key;
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
  const double v[16] = {(double)s->answered, (double)s->rejected, (double)s->busy, (double)s->failed,
                        (double)s->batches, s->batches ? (double)s->batched_frames / s->batches : 0.0,
                        percentile(s->lat_ms, 0.5), percentile(s->lat_ms, 0.99), percentile(s->lat_ms, 0.999),
                        s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end()),
                        (double)s->queue.size(), (double)s->hits, (double)s->admitted, (double)s->evicted,
                        (double)s->uncached, (double)s->table_rows};
  for (size_t i = 0; i < n && i < 16; ++i) out[i] = v[i];
  return 0;
}

int alto_server_log(void *p, double *out, size_t max_rows) {
  Server *s = static_cast<Server *>(p);
  if (!s || (!out && max_rows)) return -1;
  std::lock_guard<std::mutex> lk(s->mu);
  const size_t have = std::min(s->log_rows, kLogRows), n = std::min(have, max_rows);
  for (size_t k = 0; k < n; ++k) {  // the most recent n rows, oldest first
    const size_t row = (s->log_rows - n + k) % kLogRows;
    std::copy(s->log.data() + row * kLogFields, s->log.data() + (row + 1) * kLogFields, out + k * kLogFields);
  }
  return (int)n;
}

void alto_server_free(void *p) {
  if (p) server_destroy(static_cast<Server *>(p));
}

}  // extern "C"
