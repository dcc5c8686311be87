// alto_engine.cu -- the engine object and the per-batch C ABI (alto_engine_new / alto_answer and friends).
//
// Per batch the host settles statuses 1 and 2 from the frame lengths and headers, copies the remaining frames
// into device staging slots, and enqueues on the engine's stream:
//   validate (statuses 0/2/3) -> limb split of query and key words -> scan GEMM -> pack GEMM -> tail.
// The statuses come back early through a pinned buffer while the GEMMs run; the host then queues the copies of the
// valid responses only, so rejected output buffers are never touched.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/altopir_gpu.h"
#include "hint.cuh"
#include "kernels.cuh"
#include "offline.cuh"
#include "limb_gemm2.cuh"

namespace {

thread_local std::string g_last_error;

void set_error(const char *where, cudaError_t e) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
}
void set_error(const std::string &msg) { g_last_error = msg; }

#define ALTO_CK(call)                 \
  do {                                \
    cudaError_t e_ = (call);          \
    if (e_ != cudaSuccess) {          \
      set_error(#call, e_);           \
      return false;                   \
    }                                 \
  } while (0)

constexpr size_t kSlotLead = 7;  // frame offset inside a staging slot: puts the key words on a 16-byte boundary
constexpr int kMarks = 7;          // timing marks per batch (see enqueue_batch)
constexpr int kTimingSets = 128;   // batches that may be in flight with timing marks
constexpr size_t kMaxGather = 64;  // response buffers one alto_answer_device_parts call may write into

// ------------------------------------------------------------------------------------------- tensor maps
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// A row-major u8 matrix of `outer` rows x `inner` bytes (row stride `stride`), read in boxes of 128 bytes x
// box_rows rows with 128-byte swizzling; out-of-range parts of a box read as zero.
bool make_map(CUtensorMap *m, const void *base, uint64_t inner, uint64_t outer, uint64_t stride, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return false;
  }
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {stride};
  const cuuint32_t box[2] = {128, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d) for %llu x %llu, stride %llu, box rows %u", (int)r,
             (unsigned long long)outer, (unsigned long long)inner, (unsigned long long)stride, box_rows);
    set_error(buf);
    return false;
  }
  return true;
}

// The scan operands as 3-D maps: `outer` record chunks of `mid` rows x `inner` bytes (row stride `inner`, chunk
// stride mid * inner), read in boxes of 128 bytes x box_rows rows of one chunk.
bool make_map3(CUtensorMap *m, const void *base, uint64_t inner, uint64_t mid, uint64_t outer, uint32_t box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return false;
  }
  const cuuint64_t dims[3] = {inner, mid, outer};
  const cuuint64_t strides[2] = {inner, inner * mid};
  const cuuint32_t box[3] = {128, box_rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d) for %llu x %llu x %llu, box rows %u", (int)r,
             (unsigned long long)outer, (unsigned long long)mid, (unsigned long long)inner, box_rows);
    set_error(buf);
    return false;
  }
  return true;
}

// A tile-contiguous operand: tile (mt, kb) -- rows [128 mt, 128 mt + 128) x bytes [128 kb, 128 kb + 128) of a
// row-major matrix -- is 16 KB at (mt * kbs + kb) * 16 KB, row r of the tile at + 128 r.  Read one whole tile per box
// (coordinates (0, 0, kb, mt)) with 128-byte swizzling; tiles past `mts` read as zero.
bool make_tile_map(CUtensorMap *m, const void *base, uint64_t kbs, uint64_t mts) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return false;
  }
  const cuuint64_t dims[4] = {128, 128, kbs, mts};
  const cuuint64_t strides[3] = {128, 16384, 16384 * kbs};
  const cuuint32_t box[4] = {128, 128, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d) for %llu x %llu tiles", (int)r,
             (unsigned long long)mts, (unsigned long long)kbs);
    set_error(buf);
    return false;
  }
  return true;
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Uploads a row-major host matrix (nrows rows of k_bytes bytes, row pitch `pitch`) into the tile-contiguous layout
// of kbs x mts tiles at dst (zero where rows or bytes run past the matrix), through a 16 MB device staging buffer: one
// pass per slab of at most 128 KB of every row and as many 128-row tiles as fit.  Runs on the legacy default stream,
// which orders each staging copy after the previous rearrangement.
bool upload_tiled(uint8_t *dst, const uint8_t *src, size_t pitch, size_t nrows, size_t k_bytes, size_t kbs,
                  size_t mts) {
  const size_t stage_bytes = size_t(16) << 20;
  const size_t slab = std::min<size_t>(kbs * 128, 131072);
  const size_t per_pass = std::max<size_t>(1, stage_bytes / (128 * slab));  // row tiles per pass
  uint8_t *stage = nullptr;
  ALTO_CK(cudaMalloc(&stage, per_pass * 128 * slab));
  bool ok = true;
  for (size_t mt = 0; mt < mts && ok; mt += per_pass) {
    const size_t ntr = std::min(per_pass, mts - mt);
    const size_t r0 = mt * 128, nr = r0 < nrows ? std::min(ntr * 128, nrows - r0) : 0;
    for (size_t k0 = 0; k0 < kbs * 128 && ok; k0 += slab) {
      const size_t nk = k0 < k_bytes ? std::min(slab, k_bytes - k0) : 0;
      const size_t tiles = std::min(slab, kbs * 128 - k0) / 128;
      cudaError_t err = cudaSuccess;
      if (nr && nk) err = cudaMemcpy2D(stage, slab, src + r0 * pitch + k0, pitch, nk, nr, cudaMemcpyHostToDevice);
      if (err == cudaSuccess) {
        const size_t words = ntr * tiles * 1024;  // 16-byte words of output
        alto::tile_slab_kernel<<<(unsigned)((words + 255) / 256), 256>>>(
            stage, slab, (int)nr, (int)nk, (int)tiles, words, dst + mt * kbs * 16384, kbs, k0 / 128);
        err = cudaGetLastError();
      }
      if (err != cudaSuccess) {
        set_error("tiled upload", err);
        ok = false;
      }
    }
  }
  const cudaError_t sync = cudaStreamSynchronize(0);
  if (ok && sync != cudaSuccess) {
    set_error("tiled upload", sync);
    ok = false;
  }
  cudaFree(stage);
  return ok;
}

// Records per chunk of the query limbs in HBM (the scan's B operand, [chunk][(client, limb)][record in chunk]).  A
// limb row of R records would otherwise put every row of a TMA box on its own page once R reaches ~2^20 (the TLB
// then misses on every box); chunks of 32768 records keep a box inside a few pages.  32768 is also the longest
// reduction an int32 limb sum can take exactly, so a scan unit never spans more than one chunk.
constexpr size_t kRecordChunk = 32768;
constexpr int kMaxLanes = 4;  // batch contexts alto_enqueue_device can rotate through
constexpr int kQueryGroups = 8;  // alto_answer: at most this many record-chunk groups of query words
// Batches whose query words are fewer bytes upload them at once: the upload is short against one scan launch, and
// each extra scan launch ends on a partial round of its persistent CTA pairs.
constexpr size_t kPipedQueryBytes = size_t(32) << 20;
// alto_answer splits the scan into column groups when a batch's responses are at least this many bytes (16 frames
// of 32 KB records)
constexpr size_t kGroupedRespBytes = size_t(2) << 20;

// ------------------------------------------------------------------------------------------- engine
// The device resources of one batch in flight: its stream, per-batch scratch (grown on demand) and error word.
// An engine answers through its `main` batch; a serving loop keeps several so that batches overlap on the device.
struct Batch {
  cudaStream_t st = nullptr;
  size_t cap = 0;
  uint8_t *d_req = nullptr, *d_qlimb = nullptr, *d_ylimb = nullptr, *d_resp = nullptr;
  int *d_status = nullptr;
  uint32_t *d_acc = nullptr, *d_beta = nullptr;
  int *h_status = nullptr;
  uint32_t *d_err = nullptr, *h_err = nullptr;
  bool timing = false;  // record per-kernel timing marks into the engine's ring (main batch only)
  // Side stream of the overlapped schedule: the query limb split beside the pack, and the tail of each column group
  // but the last beside the scan of the next group.  It forks from and joins back into `st` inside every batch.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_qready = nullptr, ev_join = nullptr, ev_scan[8] = {};
  // alto_answer_device_parts: the response buffers the tails write every part into (device array of pointers,
  // allocated on first use), their count for the batch being enqueued (0 otherwise) and this engine's first part
  uint8_t **d_gather = nullptr;
  int n_gather = 0, gather_offset = 0;
  // CUDA graphs of the device-side launch sequence, one per batch size and buffer set (see enqueue_batch)
  struct GraphEntry {
    size_t slots, stride, resp_stride;
    const uint8_t *d_slots;
    uint8_t *resp;
    bool host_status;
    cudaGraphExec_t exec;
    int launches;  // kernels in the captured sequence (reported by alto_last_launches on every replay)
  };
  std::vector<GraphEntry> graphs;
};

void clear_graphs(Batch *b) {
  for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
  b->graphs.clear();
}

// One row of a tuning table: the plan knobs for batches of at most b_max frames (0 or -1 = the built-in choice).
struct TuneEntry {
  int b_max;
  int pair;            // 1 CTA-pair kernels, 0 single-CTA kernels, -1 pairs when a batch has > 16 limb columns
  int wide;            // 1 wide scan units where possible, 0 never, -1 for databases of several record chunks
  int bn_cap;          // largest limb-column tile of the pair kernels (32..256), 0 = 256
  int units_per_pair;  // scan split target: units per resident CTA pair, 0 = 12
};

struct Engine {
  int dev = -1;
  size_t rows = 0, cols = 0, n = 0, tg = 0, outputs = 0, count = 0, part_len = 0, row1_off = 0, want = 0;
  size_t resp_len = 0, slot_stride = 0;
  size_t chunk = 0, nchunks = 1;  // record chunking of the query limbs
  size_t db_kbs = 0, db_mts = 0, ub_kbs = 0, ub_mts = 0;  // tiles of the database and the packing matrix
  uint64_t q1 = 0;
  int q1_bits = 0, threads = 1;
  bool tail_ok = false;
  // resident state
  uint8_t *d_db = nullptr, *d_ub = nullptr, *d_prefix = nullptr;
  uint32_t *d_that = nullptr, *d_tw = nullptr;
  Batch main;
  // alto_enqueue_device rotates through `lanes` batch contexts -- main, lane[0], lane[1], ... -- so that consecutive
  // asynchronous batches overlap on the device (alto_engine_set_lanes); lanes_made contexts exist, lane_next is the
  // context of the next batch, and ev_lane[k] marks lane k's stream for alto_engine_fence
  Batch lane[kMaxLanes - 1];
  int lanes = 1, lanes_made = 1, lane_next = 0;
  cudaEvent_t ev_lane[kMaxLanes] = {};
  // per call: before the uploads, after the downloads; the query words upload on st_copy
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr, ev_keys = nullptr, ev_queries = nullptr, ev_zkeys = nullptr;
  cudaStream_t st_copy = nullptr;
  // host pipeline of alto_answer: keys uploaded, pack done, statuses ready, each column group's tail done
  cudaEvent_t ev_pack = nullptr, ev_status = nullptr, ev_group[8] = {};
  // alto_answer over several record chunks: each chunk group's query words uploaded, and split
  cudaEvent_t ev_qgrp[kQueryGroups] = {}, ev_sgrp[kQueryGroups] = {};
  // per batch: a ring of kMarks timing marks, accumulated into kernel_ms when the stream is synchronised
  cudaEvent_t marks[kTimingSets][kMarks] = {};
  int mark_next = 0, last_set = 0;
  std::vector<int> pending;
  double kernel_ms[5] = {0, 0, 0, 0, 0};  // validate, limb split + zeroing, scan, pack, tail
  long long kernel_batches = 0;
  CUtensorMap map_db, map_ub;
  std::atomic<int> last_launches{0};  // written by whichever thread enqueued the latest batch (a serving loop's too)
  bool use_graphs = false;  // replay captured launch sequences (alto_engine_set_graphs)
  bool overlap = true;      // the two-stream schedule of a batch (ALTO_OVERLAP=0 runs it on one stream)
  int groups = 2;           // column groups of the scan and tail of a device batch (ALTO_GROUPS: 1, 2, 4 or 8)
  // The column groups of alto_answer, whose downloads overlap the scan, as weights (ALTO_HOST_WEIGHTS, or
  // ALTO_HOST_GROUPS groups with a last one of half the size).  A group's side-stream tail runs once the next group's
  // scan has left the SMs; the tails of the last host_inline groups before the last run on the batch's stream
  // between their scan and the next (ALTO_HOST_INLINE), so that their downloads overlap that scan.  At 1 GiB and
  // B = 128 under the power cap, six groups 3,3,2,2,1,1 with one in-line tail measured 1.104-1.109 ms a call against
  // 1.134-1.136 for four groups 2,2,2,1 with none, 1.115-1.122 for 4,4,3,2,1 and 2,2,2,2 with one (three repetitions,
  // interleaved, same box).
  std::vector<int> host_weights = {3, 3, 2, 2, 1, 1};
  int host_inline = 1;
  // alto_answer and the serving loop upload a batch's query words by record-chunk group from this many bytes of
  // query words on (ALTO_PIPED_BYTES)
  size_t piped_bytes = kPipedQueryBytes;
  std::vector<TuneEntry> tuning;  // sorted by b_max; the first entry with b_max >= batch size applies
};

const TuneEntry *tune_for(const Engine *e, size_t slots) {
  for (const TuneEntry &t : e->tuning)
    if ((size_t)t.b_max >= slots) return &t;
  return nullptr;
}

// The committed tuning table: lines "rows_max b_max pair wide bn_cap units_per_pair" ('#' starts a comment); the
// rows of the smallest rows_max >= the engine's record count apply.  Read from $ALTO_TUNING, else from tuning.txt
// next to this library.
void load_tuning(Engine *e) {
  std::string path;
  if (const char *env = getenv("ALTO_TUNING")) {
    path = env;
  } else {
    Dl_info info;
    if (dladdr(reinterpret_cast<void *>(&load_tuning), &info) && info.dli_fname) {
      path = info.dli_fname;
      const size_t slash = path.find_last_of('/');
      path = (slash == std::string::npos ? std::string() : path.substr(0, slash + 1)) + "tuning.txt";
    }
  }
  FILE *f = path.empty() ? nullptr : fopen(path.c_str(), "r");
  if (!f) return;
  std::vector<std::pair<long long, TuneEntry>> rows;
  char line[256];
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    long long rmax;
    TuneEntry t;
    if (sscanf(line, "%lld %d %d %d %d %d", &rmax, &t.b_max, &t.pair, &t.wide, &t.bn_cap, &t.units_per_pair) == 6)
      rows.push_back({rmax, t});
  }
  fclose(f);
  long long best = -1;
  for (auto &r : rows)
    if (r.first >= (long long)e->rows && (best < 0 || r.first < best)) best = r.first;
  for (auto &r : rows)
    if (r.first == best) e->tuning.push_back(r.second);
  std::sort(e->tuning.begin(), e->tuning.end(), [](const TuneEntry &a, const TuneEntry &b) { return a.b_max < b.b_max; });
}

// Adds the kernel intervals of one recorded timing set to the engine's totals (its last mark must have completed).
bool accumulate(Engine *e, int set) {
  float t[kMarks - 1];
  for (int i = 0; i + 1 < kMarks; ++i) ALTO_CK(cudaEventElapsedTime(&t[i], e->marks[set][i], e->marks[set][i + 1]));
  e->kernel_ms[0] += t[0];          // validate (+ status copy)
  e->kernel_ms[1] += t[1] + t[3];   // key limb split, query limb split + scan-sum zeroing (+ any upload wait)
  e->kernel_ms[2] += t[4];          // scan GEMM
  e->kernel_ms[3] += t[2];          // pack GEMM
  e->kernel_ms[4] += t[5];          // tail
  e->kernel_batches += 1;
  return true;
}

bool accumulate_pending(Engine *e) {
  for (int set : e->pending)
    if (!accumulate(e, set)) return false;
  e->pending.clear();
  return true;
}

// The next timing set; when the ring is full the oldest pending set is waited for and accumulated first.
bool next_set(Engine *e, int *set) {
  *set = e->mark_next;
  e->mark_next = (e->mark_next + 1) % kTimingSets;
  auto it = std::find(e->pending.begin(), e->pending.end(), *set);
  if (it != e->pending.end()) {
    ALTO_CK(cudaEventSynchronize(e->marks[*set][kMarks - 1]));
    if (!accumulate(e, *set)) return false;
    e->pending.erase(it);
  }
  e->pending.push_back(*set);
  e->last_set = *set;
  return true;
}

void free_scratch(Batch *b) {
  clear_graphs(b);  // graphs hold the scratch addresses
  cudaFree(b->d_req);
  cudaFree(b->d_qlimb);
  cudaFree(b->d_ylimb);
  cudaFree(b->d_resp);
  cudaFree(b->d_status);
  cudaFree(b->d_acc);
  cudaFree(b->d_beta);
  cudaFreeHost(b->h_status);
  b->d_req = b->d_qlimb = b->d_ylimb = b->d_resp = nullptr;
  b->d_status = nullptr;
  b->d_acc = b->d_beta = nullptr;
  b->h_status = nullptr;
  b->cap = 0;
}

// Stream, error word and its pinned mirror of a batch (scratch comes later, on demand).
bool init_batch(Batch *b, bool timing) {
  // The batch's stream has the highest priority and the side stream the lowest, so that when a GEMM and a tail are
  // both waiting for SMs the GEMM's persistent CTAs are placed first and the tail's CTAs take the room left beside
  // them, instead of the tail filling the SMs and holding the GEMM back.
  int least = 0, greatest = 0;
  ALTO_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  ALTO_CK(cudaStreamCreateWithPriority(&b->st, cudaStreamNonBlocking, greatest));
  ALTO_CK(cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, least));
  for (cudaEvent_t *ev : {&b->ev_fork, &b->ev_qready, &b->ev_join})
    ALTO_CK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  for (cudaEvent_t &ev : b->ev_scan) ALTO_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  ALTO_CK(cudaMalloc(&b->d_err, sizeof(uint32_t)));
  ALTO_CK(cudaMemset(b->d_err, 0, sizeof(uint32_t)));
  ALTO_CK(cudaHostAlloc(&b->h_err, sizeof(uint32_t), cudaHostAllocDefault));
  b->timing = timing;
  return true;
}

void destroy_batch(Batch *b) {
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->side) cudaStreamSynchronize(b->side);
  free_scratch(b);
  cudaFree(b->d_gather);
  b->d_gather = nullptr;
  cudaFree(b->d_err);
  cudaFreeHost(b->h_err);
  for (cudaEvent_t ev : {b->ev_fork, b->ev_qready, b->ev_join})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : b->ev_scan)
    if (ev) cudaEventDestroy(ev);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->st) cudaStreamDestroy(b->st);
  b->st = b->side = nullptr;
  b->d_err = b->h_err = nullptr;
}

Batch *lane_batch(Engine *e, int k) { return k == 0 ? &e->main : &e->lane[k - 1]; }

void destroy(Engine *e) {
  if (!e) return;
  if (e->dev >= 0) cudaSetDevice(e->dev);
  for (int k = 0; k < e->lanes_made; ++k) {
    Batch *b = lane_batch(e, k);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->side) cudaStreamSynchronize(b->side);
  }
  cudaFree(e->d_db);
  cudaFree(e->d_ub);
  cudaFree(e->d_prefix);
  cudaFree(e->d_that);
  cudaFree(e->d_tw);
  if (e->st_copy) cudaStreamSynchronize(e->st_copy);
  for (cudaEvent_t ev : {e->ev_begin, e->ev_end, e->ev_keys, e->ev_queries, e->ev_zkeys, e->ev_pack, e->ev_status})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : e->ev_group)
    if (ev) cudaEventDestroy(ev);
  for (const cudaEvent_t *set : {e->ev_qgrp, e->ev_sgrp})
    for (int k = 0; k < kQueryGroups; ++k)
      if (set[k]) cudaEventDestroy(set[k]);
  if (e->st_copy) cudaStreamDestroy(e->st_copy);
  for (auto &set : e->marks)
    for (cudaEvent_t &ev : set)
      if (ev) cudaEventDestroy(ev);
  for (int k = e->lanes_made - 1; k >= 1; --k) destroy_batch(&e->lane[k - 1]);
  for (cudaEvent_t ev : e->ev_lane)
    if (ev) cudaEventDestroy(ev);
  destroy_batch(&e->main);
  delete e;
}

bool ensure_capacity(const Engine *e, Batch *b, size_t slots) {
  if (slots <= b->cap) return true;
  ALTO_CK(cudaStreamSynchronize(b->st));
  ALTO_CK(cudaStreamSynchronize(b->side));
  free_scratch(b);
  const size_t cap = round_up(slots, 4);
  ALTO_CK(cudaMalloc(&b->d_req, cap * e->slot_stride));
  ALTO_CK(cudaMalloc(&b->d_qlimb, 4 * cap * e->chunk * e->nchunks));
  ALTO_CK(cudaMalloc(&b->d_ylimb, 4 * cap * e->count));
  ALTO_CK(cudaMalloc(&b->d_resp, cap * e->resp_len));
  ALTO_CK(cudaMalloc(&b->d_status, cap * sizeof(int)));
  ALTO_CK(cudaMalloc(&b->d_acc, cap * e->cols * sizeof(uint32_t)));
  ALTO_CK(cudaMalloc(&b->d_beta, cap * e->cols * sizeof(uint32_t)));
  ALTO_CK(cudaHostAlloc(&b->h_status, cap * sizeof(int), cudaHostAllocDefault));
  b->cap = cap;
  return true;
}

// ------------------------------------------------------------------------------------------- launch helpers
template <int BN, alto::Epi EPI>
bool launch_gemm(const CUtensorMap &a, const CUtensorMap &b, const alto::GemmArgs &g, int units, cudaStream_t st) {
  const int smem = alto::GemmShape<BN>::kSmemBytes;
  ALTO_CK(cudaFuncSetAttribute(alto::limb_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  alto::limb_gemm_kernel<BN, EPI><<<units, alto::kGemmThreads, smem, st>>>(a, b, g);
  ALTO_CK(cudaGetLastError());
  return true;
}

template <alto::Epi EPI>
bool dispatch_gemm(int bn, const CUtensorMap &a, const CUtensorMap &b, const alto::GemmArgs &g, int units,
                   cudaStream_t st) {
  switch (bn) {
    case 16: return launch_gemm<16, EPI>(a, b, g, units, st);
    case 32: return launch_gemm<32, EPI>(a, b, g, units, st);
    case 64: return launch_gemm<64, EPI>(a, b, g, units, st);
    case 128: return launch_gemm<128, EPI>(a, b, g, units, st);
    case 256: return launch_gemm<256, EPI>(a, b, g, units, st);
  }
  set_error("unsupported GEMM tile width");
  return false;
}

template <int BN, alto::Epi EPI, int NSUB = 1>
bool launch_pair(const CUtensorMap &a, const CUtensorMap &b, const alto::PairArgs &g, int pairs, cudaStream_t st) {
  const int smem = alto::PairShape<BN, NSUB>::kSmemBytes;
  ALTO_CK(cudaFuncSetAttribute(alto::limb_gemm_pair_kernel<BN, EPI, NSUB>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  alto::limb_gemm_pair_kernel<BN, EPI, NSUB><<<2 * pairs, alto::kGemmThreads, smem, st>>>(a, b, g);
  ALTO_CK(cudaGetLastError());
  return true;
}

// bn = columns per accumulator; wide = two 256-column accumulators per unit (NSUB = 2, scan only)
template <alto::Epi EPI>
bool dispatch_pair(int bn, const CUtensorMap &a, const CUtensorMap &b, const alto::PairArgs &g, int pairs,
                   cudaStream_t st, bool wide = false) {
  if (wide) {
    if (bn == 256) return launch_pair<256, EPI, 2>(a, b, g, pairs, st);
    set_error("wide pair GEMM needs 256-column accumulators");
    return false;
  }
  switch (bn) {
    case 32: return launch_pair<32, EPI>(a, b, g, pairs, st);
    case 64: return launch_pair<64, EPI>(a, b, g, pairs, st);
    case 128: return launch_pair<128, EPI>(a, b, g, pairs, st);
    case 256: return launch_pair<256, EPI>(a, b, g, pairs, st);
  }
  set_error("unsupported pair GEMM tile width");
  return false;
}

// CTA pairs that can be resident at once (clusters of two CTAs, one CTA per SM); 74 on a 148-SM B200.
int compute_resident_pairs() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sms & ~1);
  cfg.blockDim = dim3(alto::kGemmThreads);
  cfg.dynamicSmemBytes = alto::PairShape<256>::kSmemBytes;
  int clusters = 0;
  cudaFuncSetAttribute(alto::limb_gemm_pair_kernel<256, alto::Epi::kScan>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       alto::PairShape<256>::kSmemBytes);
  if (cudaOccupancyMaxActiveClusters(&clusters, alto::limb_gemm_pair_kernel<256, alto::Epi::kScan>, &cfg) !=
          cudaSuccess ||
      clusters <= 0)
    clusters = sms / 2;
  cudaGetLastError();
  return clusters;
}

// CTA pairs that can be resident at once (clusters of two CTAs, one CTA per SM); 74 on a 148-SM B200.
int resident_pairs() {
  static const int pairs = compute_resident_pairs();  // thread-safe one-time initialisation
  return pairs;
}

int pick_bn(size_t limb_cols) {
  for (int bn : {16, 32, 64, 128})
    if (limb_cols <= (size_t)bn) return bn;
  return 256;
}

struct Plan {
  bool pair = false;  // CTA-pair kernels (limb columns > 16) or the single-CTA kernels
  bool wide = false;  // scan units of 512 limb columns (one read of each database tile for all of them)
  bool pack_wide = false;  // pack units of 512 limb columns (one read of each packing-matrix tile for all of them)
  int scan_n = 1;     // scan tiles along the limb columns (num_n / 2 when wide)
  int kb_chunk = 1;   // scan blocks per record chunk
  int bn = 16, num_n = 1;
  int nw = 16;        // limb columns a pair-kernel tile computes: a multiple of 32 <= bn (bn: the kernel's template
                      // width, a power of two), num_n tiles covering the batch's limb columns with least padding
  int scan_m = 0, scan_split = 1, scan_kb_per = 1, scan_kb = 0;
  int pack_m = 0, pack_kb = 0;
  int pairs_scan = 0, pairs_pack = 0;  // persistent grid of the pair kernels
};

// ALTO_GEMM=single forces the single-CTA kernels (a tuning override; both compute identical results).
bool pair_kernels_enabled() {
  const char *v = getenv("ALTO_GEMM");
  return !(v && strcmp(v, "single") == 0);
}

// The record-axis split is chosen for the whole scan; a scan run in column groups launches each group's share of
// its units (splitting every group for its own tiles measured slower: more units, more partial-sum reductions).
Plan make_plan(const Engine *e, size_t slots) {
  Plan p;
  const size_t limb_cols = 4 * round_up(slots, 4);
  const TuneEntry *tn = tune_for(e, slots);
  p.pair = limb_cols > 16 && pair_kernels_enabled();
  if (tn && tn->pair >= 0) p.pair = tn->pair == 1 && limb_cols > 16 && pair_kernels_enabled();
  p.scan_kb = (int)((e->rows + alto::kBK - 1) / alto::kBK);
  p.pack_kb = (int)(e->count / alto::kBK);
  // with several record chunks a unit must stay inside one: its length divides the 256 blocks of a chunk
  p.kb_chunk = e->nchunks > 1 ? (int)(e->chunk / alto::kBK) : std::max(p.scan_kb, 1);
  auto chunk_aligned = [&](int kb_per) {
    if (e->nchunks == 1) return kb_per;
    int d = p.kb_chunk;
    while (d / 2 >= kb_per && d % 2 == 0) d /= 2;
    return d;  // the smallest divisor of a chunk's blocks (a power of two here) that is >= kb_per
  };
  if (!p.pair) {
    p.bn = p.nw = pick_bn(limb_cols);
    p.num_n = (int)((limb_cols + p.bn - 1) / p.bn);
    p.scan_m = (int)((e->cols + alto::kBM - 1) / alto::kBM);
    p.pack_m = (int)((4 * e->cols + alto::kBM - 1) / alto::kBM);
    // Split the record axis so that (a) no chunk exceeds 256 blocks = 32768 records, which bounds every int32 limb
    // partial sum by 32768 * 255 * 255 < 2^31, and (b) there are about four units per SM, each >= 8 blocks long.
    const long tiles = (long)p.scan_m * p.num_n;
    long split = std::max<long>((p.scan_kb + 255) / 256, (4L * 148 + tiles - 1) / tiles);
    split = std::min<long>(split, std::max<long>(1, p.scan_kb / 8));
    split = std::max<long>(split, (p.scan_kb + 255) / 256);
    p.scan_kb_per = chunk_aligned((int)((p.scan_kb + split - 1) / split));
    p.scan_split = (p.scan_kb + p.scan_kb_per - 1) / p.scan_kb_per;
    return p;
  }
  const int bn_cap = (tn && tn->bn_cap >= 32 && tn->bn_cap <= 256) ? tn->bn_cap : 256;
  // Power-of-two tiles (bn, the kernel's template width), or narrow ones: nw limb columns a tile, nw a multiple of 32
  // (the pair kind::i8 MMA's N), as few tiles as the cap allows, each as narrow as covers the batch.  Narrow tiles are
  // taken when they cut the columns computed by at least 20 %, which leaves out 224-column tiles.  Measured at 8 GiB
  // (scan ms, power-of-two / narrow): 36 clients 1.83 / 1.54 on one 160-column tile (1.60 on 192); 48 clients
  // 1.82 / 1.66 on 192; 136 clients 6.13 / 4.63 on 3 x 192; 70 clients 2.81 / 2.92 on 2 x 160 (the one loss);
  // 224-column tiles (100 or 200 clients) ran 10-11 % slower than 256-column ones.  ALTO_TILE_EXACT=0 never takes
  // narrow tiles, =1 always; ALTO_TILE_ALIGN=64 rounds their width to a multiple of 64.
  {
    int bn2 = 32;
    while (bn2 < bn_cap && (size_t)bn2 < limb_cols) bn2 *= 2;
    const int n2 = (int)((limb_cols + bn2 - 1) / bn2);
    const int nn = (int)((limb_cols + bn_cap - 1) / bn_cap);
    int align = 32;
    if (const char *v = getenv("ALTO_TILE_ALIGN")) align = atoi(v) == 64 ? 64 : 32;
    const int nw = (int)std::min<size_t>(round_up((limb_cols + nn - 1) / nn, align), (size_t)bn_cap);
    bool narrow = (long)nn * nw * 10 <= (long)n2 * bn2 * 8;
    if (const char *v = getenv("ALTO_TILE_EXACT")) narrow = v[0] != '0';
    if (narrow) {
      p.num_n = nn;
      p.nw = nw;
      p.bn = 32;
      while (p.bn < p.nw) p.bn *= 2;
    } else {
      p.bn = p.nw = bn2;
      p.num_n = n2;
    }
  }
  p.scan_m = (int)((e->cols + 255) / 256);
  p.pack_m = (int)((4 * e->cols + 255) / 256);
  const int pairs = resident_pairs();
  // Wide scan units once the database spans several record chunks (its tiles then stream from HBM and cannot be
  // shared between two pairs through L2) and there are at least 512 limb columns; ALTO_SCAN_WIDE=0/1 overrides.
  const bool full = p.bn == 256 && p.nw == 256;  // wide units take two full 256-column sub-accumulators
  p.wide = full && p.num_n >= 2 && e->nchunks > 1;
  if (tn && tn->wide >= 0) p.wide = full && p.num_n >= 2 && tn->wide == 1;
  if (const char *w = getenv("ALTO_SCAN_WIDE")) p.wide = full && p.num_n >= 2 && w[0] == '1';
  p.scan_n = p.wide ? (p.num_n + 1) / 2 : p.num_n;
  // Scan chunks: at most 256 blocks (exactness, as above), at least 8, and about twelve units per resident pair so
  // the persistent pairs finish together.
  const long tiles = (long)p.scan_m * p.scan_n;
  const long upp = (tn && tn->units_per_pair > 0) ? tn->units_per_pair : 12;
  long split = std::max<long>((p.scan_kb + 255) / 256, (upp * pairs + tiles - 1) / tiles);
  split = std::min<long>(split, std::max<long>(1, p.scan_kb / 8));
  split = std::max<long>(split, (p.scan_kb + 255) / 256);
  p.scan_kb_per = chunk_aligned((int)((p.scan_kb + split - 1) / split));
  p.scan_split = (p.scan_kb + p.scan_kb_per - 1) / p.scan_kb_per;
  p.pairs_scan = (int)std::min<long>(pairs, tiles * p.scan_split);
  // Wide pack units (ALTO_PACK_WIDE=1): both 256-column tiles of the limb columns in one unit, so each packing-
  // matrix tile is read once (and the epilogue no longer overlaps the next unit's MMAs)
  if (const char *w = getenv("ALTO_PACK_WIDE")) p.pack_wide = full && p.num_n >= 2 && w[0] == '1';
  const long pack_n = p.pack_wide ? (p.num_n + 1) / 2 : p.num_n;
  p.pairs_pack = (int)std::min<long>(pairs, (long)p.pack_m * pack_n);
  return p;
}

// The scan GEMM (acc sums, pre-zeroed) and the pack GEMM (beta) for `slots` clients under plan p.
bool launch_scan(const Engine *e, const Plan &p, const CUtensorMap &map_q, uint32_t *acc, size_t slots,
                 cudaStream_t st, uint32_t *err, int m0 = 0, int mg = -1, int kb_lo = 0, int kb_hi = -1) {
  // scan tiles [m0, m0 + mg) along the database columns (all of them by default), reduction blocks [kb_lo, kb_hi)
  // (all records by default; a range starts and ends on record-chunk boundaries, so units never straddle one)
  if (mg < 0) mg = p.scan_m;
  if (kb_hi < 0) kb_hi = p.scan_kb;
  const int splits = (kb_hi - kb_lo + p.scan_kb_per - 1) / p.scan_kb_per;
  // The query limbs are re-read by every unit of a K chunk; mark them evict-last only while the whole operand
  // (4 bytes per record and client) is a small part of the 126 MB L2, so stale chunks never crowd it out.
  const int keep_b = 4 * round_up(slots, 4) * e->rows <= (size_t(32) << 20);
  if (p.pair) {
    alto::PairArgs g;
    g.num_m = mg;
    g.m_begin = m0;
    g.num_n = p.scan_n;
    g.num_units = mg * p.scan_n * splits;
    g.kb_total = kb_hi;
    g.kb_begin = kb_lo;
    g.kb_per_unit = p.scan_kb_per;
    g.rows_a = (int)e->cols;
    g.clients = (int)slots;
    g.cols = (int)e->cols;
    g.out = acc;
    g.err = err;
    g.b_keep = keep_b;
    g.kb_chunk = p.kb_chunk;
    g.nw = p.nw;
    return dispatch_pair<alto::Epi::kScan>(p.bn, e->map_db, map_q, g,
                                           std::min(p.pairs_scan, g.num_units), st, p.wide);
  }
  alto::GemmArgs g;
  g.num_m = mg;
  g.m_begin = m0;
  g.num_n = p.num_n;
  g.kb_total = kb_hi;
  g.kb_begin = kb_lo;
  g.kb_per_unit = p.scan_kb_per;
  g.rows_a = (int)e->cols;
  g.clients = (int)slots;
  g.cols = (int)e->cols;
  g.out = acc;
  g.err = err;
  g.b_keep = keep_b;
  g.kb_chunk = p.kb_chunk;
  return dispatch_gemm<alto::Epi::kScan>(p.bn, e->map_db, map_q, g, mg * p.num_n * splits, st);
}

bool launch_pack(const Engine *e, const Plan &p, const CUtensorMap &map_y, uint32_t *beta, size_t slots,
                 cudaStream_t st, uint32_t *err) {
  const int keep_b = 4 * round_up(slots, 4) * e->count <= (size_t(32) << 20);
  if (p.pair) {
    alto::PairArgs g;
    g.num_m = p.pack_m;
    g.m_begin = 0;
    g.num_n = p.pack_wide ? (p.num_n + 1) / 2 : p.num_n;
    g.num_units = p.pack_m * g.num_n;
    g.kb_total = p.pack_kb;
    g.kb_per_unit = p.pack_kb;
    g.rows_a = (int)(4 * e->cols);
    g.clients = (int)slots;
    g.cols = (int)e->cols;
    g.out = beta;
    g.err = err;
    g.b_keep = keep_b;
    g.kb_chunk = 1;
    g.nw = p.nw;
    return dispatch_pair<alto::Epi::kPack>(p.bn, e->map_ub, map_y, g, p.pairs_pack, st, p.pack_wide);
  }
  alto::GemmArgs g;
  g.num_m = p.pack_m;
  g.m_begin = 0;
  g.num_n = p.num_n;
  g.kb_total = p.pack_kb;
  g.kb_per_unit = p.pack_kb;
  g.rows_a = (int)(4 * e->cols);
  g.clients = (int)slots;
  g.cols = (int)e->cols;
  g.out = beta;
  g.err = err;
  g.b_keep = keep_b;
  g.kb_chunk = 1;
  return dispatch_gemm<alto::Epi::kPack>(p.bn, e->map_ub, map_y, g, p.pack_m * p.num_n, st);
}

// Tensor maps of the two limb operands for plan p (B boxes are BN rows for the single-CTA kernels and nw/2 rows,
// one half of a tile per CTA, for the pair kernels).
bool make_limb_maps(const Engine *e, const Plan &p, const uint8_t *qlimb, const uint8_t *ylimb, size_t bp,
                    CUtensorMap *map_q, CUtensorMap *map_y) {
  const uint32_t box = (uint32_t)(p.pair ? p.nw / 2 : p.bn);
  return make_map3(map_q, qlimb, e->chunk, 4 * (uint64_t)bp, e->nchunks, box) &&
         make_map(map_y, ylimb, e->count, 4 * (uint64_t)bp, e->count, box);
}

// Column groups of the scan and tail: group g is the response parts [bounds[g], bounds[g + 1]), whose columns are
// whole scan tiles (a part is n columns; a tile 256 columns for the pair kernels, 128 for the single-CTA ones).
struct Groups {
  int count = 1;
  int bounds[9] = {0};
  int tiles_per_part = 0;
};

// Column groups whose sizes follow `weights` (the first 8 count, each > 0): group i ends at part
// round(outputs * (w_0 + ... + w_i) / total), the last at `outputs`; empty groups are dropped.
Groups column_groups(const Engine *e, const Plan &p, const std::vector<int> &weights) {
  Groups g;
  const int tile_cols = p.pair ? 256 : 128;
  g.bounds[1] = (int)e->outputs;
  const int count = std::min<int>((int)weights.size(), 8);
  if (count <= 1 || e->n % tile_cols) return g;
  g.tiles_per_part = (int)(e->n / tile_cols);
  long total = 0, acc = 0;
  for (int i = 0; i < count; ++i) total += weights[i];
  int k = 0;
  for (int i = 0; i < count; ++i) {
    acc += weights[i];
    const int b = i + 1 == count ? (int)e->outputs : (int)(((long)e->outputs * acc + total / 2) / total);
    if (b > g.bounds[k]) g.bounds[++k] = b;
  }
  g.count = k;
  return g;
}

// Weights of `count` equal groups, or of equal groups but a last one of half the size.
std::vector<int> group_weights(int count, bool small_last) {
  std::vector<int> w(std::max(1, std::min(count, 8)), 2);
  if (small_last && w.size() > 1) w.back() = 1;
  return w;
}

// A comma-separated list of 1 to 8 positive weights; empty when malformed.
std::vector<int> parse_weights(const char *v) {
  std::vector<int> w;
  const char *s = v;
  while (*s) {
    char *end = nullptr;
    const long x = strtol(s, &end, 10);
    if (end == s || x <= 0 || x > 1024 || w.size() == 8 || (*end && *end != ',')) return {};
    w.push_back((int)x);
    s = *end ? end + 1 : end;
  }
  return w;
}

// Tail arguments for the output parts [o_begin, o_begin + o_count) of every frame.
alto::TailArgs tail_args(const Engine *e, const Batch *bt, const uint8_t *d_slots, size_t slot_stride, uint8_t *resp,
                         size_t resp_stride, int o_begin, int o_count) {
  alto::TailArgs t;
  t.acc = bt->d_acc;
  t.beta = bt->d_beta;
  t.status = bt->d_status;
  t.req = d_slots;
  t.req_stride = slot_stride;
  t.z_off = kSlotLead + 9 + 4 * e->count;
  t.that = e->d_that;
  t.twiddle = e->d_tw;
  t.prefix = e->d_prefix;
  t.resp = resp;
  t.resp_stride = resp_stride;
  t.n = (int)e->n;
  t.tg = (int)e->tg;
  t.outputs = (int)e->outputs;
  t.cols = (int)e->cols;
  t.part_len = (int)e->part_len;
  t.row1_off = (int)e->row1_off;
  t.q1_bits = e->q1_bits;
  t.q1 = (int64_t)e->q1;
  t.o_begin = o_begin;
  t.o_count = o_count;
  t.resp_list = bt->n_gather ? bt->d_gather : nullptr;
  t.n_resp = bt->n_gather;
  t.part_offset = bt->gather_offset;
  return t;
}

// Query limb split and zeroing of the scan sums for `slots` staged frames, on stream st.
bool enqueue_query_split(const Engine *e, const Batch *bt, const uint8_t *d_slots, size_t slot_stride, size_t slots,
                         cudaStream_t st) {
  const size_t bp = round_up(slots, 4), work = (e->rows / 16) * bp;
  alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(
      d_slots, slot_stride, kSlotLead + 9 + 8 * e->count, (int)slots, (int)bp, e->rows, e->chunk, bt->d_qlimb);
  ALTO_CK(cudaGetLastError());
  ALTO_CK(cudaMemsetAsync(bt->d_acc, 0, slots * e->cols * sizeof(uint32_t), st));
  return true;
}

// Scan and tail in column groups: the tail of every group but the last runs on the side stream beside the scan of the
// next group (the tail is integer-ALU work, the scan tensor work; the side stream's lower priority lets the scan's
// CTAs be placed first); `done[g]`, when given, is recorded after the tail of group g.
// Groups g >= inline_from run their tail on the batch's stream right after their scan (before the next group's
// scan), so that their responses are complete, and can download, while the next group computes.
bool enqueue_scan_tails(Engine *e, Batch *bt, const Plan &p, const CUtensorMap &map_q, const uint8_t *d_slots,
                        size_t slot_stride, size_t slots, uint8_t *resp, size_t resp_stride, const Groups &gr,
                        const cudaEvent_t *done, int *launches, cudaEvent_t before_last_tail = nullptr,
                        cudaEvent_t last_tail_after = nullptr, int inline_from = 8, int kb_lo = 0) {
  cudaStream_t st = bt->st;
  bool forked = false;
  for (int g = 0; g < gr.count; ++g) {
    const int o0 = gr.bounds[g], parts = gr.bounds[g + 1] - o0;
    const bool ok = gr.count == 1 ? launch_scan(e, p, map_q, bt->d_acc, slots, st, bt->d_err, 0, -1, kb_lo)
                                  : launch_scan(e, p, map_q, bt->d_acc, slots, st, bt->d_err, o0 * gr.tiles_per_part,
                                                parts * gr.tiles_per_part, kb_lo);
    if (!ok) return false;
    const bool last = g + 1 == gr.count;
    cudaStream_t ts = (last || g >= inline_from) ? st : bt->side;
    if (ts != st) {
      ALTO_CK(cudaEventRecord(bt->ev_scan[g], st));
      ALTO_CK(cudaStreamWaitEvent(ts, bt->ev_scan[g], 0));
      forked = true;
    } else if (last && before_last_tail) {
      ALTO_CK(cudaEventRecord(before_last_tail, st));
    }
    if (last_tail_after && ts == st) ALTO_CK(cudaStreamWaitEvent(st, last_tail_after, 0));
    ALTO_CK(alto::launch_tail(tail_args(e, bt, d_slots, slot_stride, resp, resp_stride, o0, parts), slots, ts));
    *launches += 2;
    if (done) ALTO_CK(cudaEventRecord(done[g], ts));
  }
  if (forked) {  // join the side stream's tails
    ALTO_CK(cudaEventRecord(bt->ev_join, bt->side));
    ALTO_CK(cudaStreamWaitEvent(st, bt->ev_join, 0));
  }
  return true;
}

// Enqueues the answer path for `slots` staged frames on the batch's stream: validate, key limb split, pack GEMM,
// query limb split, scan GEMM and tail.  Statuses go to d_status (and to the pinned host copy when host_status);
// responses of valid frames to resp + slot * resp_stride.  With the overlapped schedule validation, the query limb
// split and the zeroing of the scan sums run on the side stream beside the key limb split and the pack, and the
// tails of all column groups but the last beside the scan (enqueue_scan_tails); the side stream forks from and joins
// back into the batch's stream, so the batch is complete when its stream passes it.
bool enqueue_batch_direct(Engine *e, Batch *bt, const uint8_t *d_slots, size_t slot_stride, size_t slots,
                          uint8_t *resp, size_t resp_stride, bool host_status, bool with_marks) {
  cudaStream_t st = bt->st;
  const Plan p = make_plan(e, slots);
  const Groups groups = column_groups(e, p, group_weights(e->overlap ? e->groups : 1, false));
  const int bp = (int)round_up(slots, 4);
  int launches = 0;
  // timing marks (main batch only): 0 begin | validate (one stream only) | 1 | y split | 2 | pack | 3 | (wait for
  // the side stream) | 4 | scan (with all tails but the last beside it) | 5 | last tail | 6.  With two streams the
  // intervals are the exposed times: validation and the query split run beside the key split and the pack.
  cudaEvent_t *mk = nullptr;
  if (bt->timing && with_marks) {
    int set = 0;
    if (!next_set(e, &set)) return false;
    mk = e->marks[set];
  }
  auto mark = [&](int i) { return mk ? cudaEventRecord(mk[i], st) : cudaSuccess; };
  ALTO_CK(mark(0));
  // validation (its statuses are needed by the tails only) and the query limb split: on the side stream when the
  // schedule has two, joined before the scan
  cudaStream_t vs = st;
  if (e->overlap) {
    vs = bt->side;
    ALTO_CK(cudaEventRecord(bt->ev_fork, st));
    ALTO_CK(cudaStreamWaitEvent(vs, bt->ev_fork, 0));
  }
  alto::validate_kernel<<<(unsigned)slots, 256, 0, vs>>>(d_slots, slot_stride, kSlotLead, e->count, e->rows,
                                                         bt->d_status);
  ++launches;
  ALTO_CK(cudaGetLastError());
  if (host_status) ALTO_CK(cudaMemcpyAsync(bt->h_status, bt->d_status, slots * sizeof(int), cudaMemcpyDeviceToHost, vs));
  if (e->overlap) {
    if (!enqueue_query_split(e, bt, d_slots, slot_stride, slots, vs)) return false;
    launches += 1;
    ALTO_CK(cudaEventRecord(bt->ev_qready, vs));
  }
  ALTO_CK(mark(1));

  CUtensorMap map_q, map_y;
  if (!make_limb_maps(e, p, bt->d_qlimb, bt->d_ylimb, bp, &map_q, &map_y)) return false;
  {
    const size_t work = (e->count / 16) * (size_t)bp;
    alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(
        d_slots, slot_stride, kSlotLead + 9, (int)slots, bp, e->count, e->count, bt->d_ylimb);
    ++launches;
    ALTO_CK(cudaGetLastError());
  }
  ALTO_CK(mark(2));
  if (!launch_pack(e, p, map_y, bt->d_beta, slots, st, bt->d_err)) return false;
  ++launches;
  ALTO_CK(mark(3));
  if (e->overlap) {
    ALTO_CK(cudaStreamWaitEvent(st, bt->ev_qready, 0));
  } else {
    if (!enqueue_query_split(e, bt, d_slots, slot_stride, slots, st)) return false;
    launches += 1;
  }
  ALTO_CK(mark(4));
  if (!enqueue_scan_tails(e, bt, p, map_q, d_slots, slot_stride, slots, resp, resp_stride, groups, nullptr,
                          &launches,
                          mk ? mk[5] : nullptr))
    return false;
  ALTO_CK(mark(6));
  e->last_launches = launches;
  return true;
}

// enqueue_batch_direct, or -- when the engine replays graphs -- the same sequence (both streams) as a CUDA graph
// captured on first use for this batch size and these buffers and replayed after.
// Graph replays record no per-kernel timing marks.
bool enqueue_batch(Engine *e, Batch *bt, const uint8_t *d_slots, size_t slot_stride, size_t slots, uint8_t *resp,
                   size_t resp_stride, bool host_status) {
  if (!e->use_graphs)
    return enqueue_batch_direct(e, bt, d_slots, slot_stride, slots, resp, resp_stride, host_status, true);
  for (const Batch::GraphEntry &g : bt->graphs)
    if (g.slots == slots && g.d_slots == d_slots && g.stride == slot_stride && g.resp == resp &&
        g.resp_stride == resp_stride && g.host_status == host_status) {
      ALTO_CK(cudaGraphLaunch(g.exec, bt->st));
      e->last_launches = g.launches;
      return true;
    }
  ALTO_CK(cudaStreamBeginCapture(bt->st, cudaStreamCaptureModeThreadLocal));
  const bool ok =
      enqueue_batch_direct(e, bt, d_slots, slot_stride, slots, resp, resp_stride, host_status, false);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(bt->st, &graph);
  if (!ok || end != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (ok) set_error("graph capture", end);
    return false;
  }
  cudaGraphExec_t exec = nullptr;
  const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  ALTO_CK(inst);
  if (bt->graphs.size() >= 64) {  // bounded cache: drop the oldest graph
    cudaGraphExecDestroy(bt->graphs.front().exec);
    bt->graphs.erase(bt->graphs.begin());
  }
  bt->graphs.push_back({slots, slot_stride, resp_stride, d_slots, resp, host_status, exec, e->last_launches});
  ALTO_CK(cudaGraphLaunch(exec, bt->st));
  return true;
}

// Groups consecutive items whose source and destination addresses advance by constant pitches into one 2-D copy.
template <class SrcAt, class DstAt>
bool copy_runs(size_t items, size_t width, SrcAt src_at, DstAt dst_at, cudaMemcpyKind kind, cudaStream_t st) {
  size_t i = 0;
  while (i < items) {
    size_t j = i + 1;
    long long sp = 0, dp = 0;
    if (j < items) {
      sp = (long long)((const char *)src_at(j) - (const char *)src_at(i));
      dp = (long long)((const char *)dst_at(j) - (const char *)dst_at(i));
      if (sp >= (long long)width && dp >= (long long)width) {
        while (j + 1 < items && (const char *)src_at(j + 1) - (const char *)src_at(j) == sp &&
               (const char *)dst_at(j + 1) - (const char *)dst_at(j) == dp)
          ++j;
        ++j;
      } else {
        j = i + 1;
      }
    }
    if (j - i == 1) {
      ALTO_CK(cudaMemcpyAsync(dst_at(i), src_at(i), width, kind, st));
    } else {
      ALTO_CK(cudaMemcpy2DAsync(dst_at(i), (size_t)dp, src_at(i), (size_t)sp, width, j - i, kind, st));
    }
    i = j;
  }
  return true;
}

// Waits for the engine's stream, folds pending timing marks into the totals and checks (then clears) the device
// error word.
// After a batch's stream has passed a copy of its error word into the pinned mirror: false (and the word reset)
// when a kernel wait timed out.
bool check_batch_error(Batch *b) {
  const uint32_t err = *b->h_err;
  if (err) {
    ALTO_CK(cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), b->st));
    ALTO_CK(cudaStreamSynchronize(b->st));
    *b->h_err = 0;
    char buf[96];
    snprintf(buf, sizeof buf, "a kernel wait timed out (device error word 0x%x)", err);
    set_error(buf);
    return false;
  }
  return true;
}

// The same for the main batch, then the pending timing marks folded into the totals.
bool check_error_word(Engine *e) { return check_batch_error(&e->main) && accumulate_pending(e); }

// Waits for every batch context of the engine and checks (then clears) each one's error word.
bool sync_engine(Engine *e) {
  bool ok = true;
  for (int k = e->lanes_made - 1; k >= 1; --k) {
    Batch *b = &e->lane[k - 1];
    ALTO_CK(cudaMemcpyAsync(b->h_err, b->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->st));
    ALTO_CK(cudaStreamSynchronize(b->st));
    ok = check_batch_error(b) && ok;
  }
  ALTO_CK(cudaMemcpyAsync(e->main.h_err, e->main.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, e->main.st));
  ALTO_CK(cudaStreamSynchronize(e->main.st));
  return check_error_word(e) && ok;
}

bool finish(Engine *e, double *stage_ms) {
  const int set = e->last_set;
  if (!sync_engine(e)) return false;
  if (stage_ms) {
    float a, b, c, d;
    cudaEvent_t *mk = e->marks[set];
    ALTO_CK(cudaEventElapsedTime(&a, e->ev_begin, mk[1]));  // key upload + validate
    ALTO_CK(cudaEventElapsedTime(&b, mk[3], mk[5]));        // query upload wait + query split + scan
    ALTO_CK(cudaEventElapsedTime(&c, mk[1], mk[3]));        // key split + pack
    ALTO_CK(cudaEventElapsedTime(&d, mk[5], e->ev_end));    // tail + download
    stage_ms[0] = a;
    stage_ms[1] = b;
    stage_ms[2] = c;
    stage_ms[3] = d;
  }
  return true;
}

bool host_header_status(const Engine *e, const uint8_t *f, size_t len, int *status) {
  if (!f || len != e->want) {
    *status = 1;
    return false;
  }
  uint32_t c1, c2;
  memcpy(&c1, f + 1, 4);
  memcpy(&c2, f + 5, 4);
  if (f[0] != 0 || c1 != e->count || c2 != e->count) {
    *status = 2;
    return false;
  }
  return true;
}

// alto_answer: header and y keys upload first and the pack starts on them while z keys and query words upload on
// the copy stream; then validation, the query limb split, and the scan and tail in column groups.  The responses of
// a group download (valid frames only, on the copy stream) while the next group computes.  Without the overlapped
// schedule (ALTO_OVERLAP=0) everything but the uploads and downloads runs on the batch's stream, in one group.
int answer_host(Engine *e, const uint8_t *const *req, const size_t *len, size_t b, uint8_t *const *out, int *status,
                double *stage_ms) {
  std::vector<size_t> cand;
  cand.reserve(b);
  for (size_t c = 0; c < b; ++c)
    if (host_header_status(e, req[c], len[c], &status[c])) cand.push_back(c);
  if (stage_ms) std::fill(stage_ms, stage_ms + 4, 0.0);
  e->last_launches = 0;
  if (cand.empty()) return 0;
  if (!e->tail_ok) {
    // The reference computes the statuses, then fails in the tail (src/amx_kernels.cpp:610).
    for (size_t c : cand) {
      int bad = 0;
      for (size_t i = 0; i < 2 * e->count; ++i) {
        uint32_t v;
        memcpy(&v, req[c] + 9 + 4 * i, 4);
        bad |= v >= (uint32_t)alto::kQ;
      }
      status[c] = bad ? 3 : 0;
    }
    return -3;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess || !ensure_capacity(e, &e->main, cand.size())) return -4;
  Batch *bt = &e->main;
  cudaStream_t st = bt->st, sc = e->st_copy;
  const size_t nc = cand.size();
  const Plan p = make_plan(e, nc);
  // Column groups overlap the responses' download with the scan; a batch whose responses are few bytes has little to
  // overlap, and every extra scan launch ends on a partial round of its CTA pairs, so it scans in one launch.
  const bool grouped = e->overlap && nc * e->resp_len >= kGroupedRespBytes;
  const Groups groups = column_groups(e, p, grouped ? e->host_weights : std::vector<int>{1});
  const int bp = (int)round_up(nc, 4);
  const size_t ybytes = 9 + 4 * e->count;  // header and y keys
  int launches = 0;
#define ALTO_H(call)                   \
  do {                                 \
    cudaError_t e_ = (call);           \
    if (e_ != cudaSuccess) {           \
      set_error(#call, e_);            \
      return -4;                       \
    }                                  \
  } while (0)
  ALTO_H(cudaEventRecord(e->ev_begin, st));
  if (!copy_runs(
          nc, ybytes, [&](size_t i) { return (const void *)req[cand[i]]; },
          [&](size_t i) { return (void *)(bt->d_req + i * e->slot_stride + kSlotLead); }, cudaMemcpyHostToDevice, st))
    return -4;
  ALTO_H(cudaEventRecord(e->ev_keys, st));
  ALTO_H(cudaStreamWaitEvent(sc, e->ev_keys, 0));
  // then the query words (the scan's input) and last the z keys, which only validation and the tails read.  A
  // database of several record chunks takes its query words chunk group by chunk group (at most 8 groups), each
  // group's limb split and scan starting as soon as its words are in, so that the upload of the later chunks
  // overlaps the scan of the earlier ones.
  const size_t zbytes = 4 * e->count, qoff = ybytes + zbytes;
  const bool piped = e->overlap && e->nchunks > 1 && 4 * nc * e->rows >= e->piped_bytes;
  const size_t gsz = piped ? (e->nchunks + kQueryGroups - 1) / kQueryGroups : e->nchunks;  // chunks per group
  const int qgroups = (int)((e->nchunks + gsz - 1) / gsz);
  auto group_rows = [&](int k, size_t *r0, size_t *r1) {
    *r0 = (size_t)k * gsz * e->chunk;
    *r1 = std::min(e->rows, (size_t)(k + 1) * gsz * e->chunk);
  };
  for (int k = 0; k < qgroups; ++k) {
    size_t r0, r1;
    group_rows(k, &r0, &r1);
    if (!copy_runs(
            nc, 4 * (r1 - r0), [&](size_t i) { return (const void *)(req[cand[i]] + qoff + 4 * r0); },
            [&](size_t i) { return (void *)(bt->d_req + i * e->slot_stride + kSlotLead + qoff + 4 * r0); },
            cudaMemcpyHostToDevice, sc))
      return -4;
    ALTO_H(cudaEventRecord(piped ? e->ev_qgrp[k] : e->ev_queries, sc));
  }
  if (!copy_runs(
          nc, zbytes, [&](size_t i) { return (const void *)(req[cand[i]] + ybytes); },
          [&](size_t i) { return (void *)(bt->d_req + i * e->slot_stride + kSlotLead + ybytes); },
          cudaMemcpyHostToDevice, sc))
    return -4;
  ALTO_H(cudaEventRecord(e->ev_zkeys, sc));

  CUtensorMap map_q, map_y;
  if (!make_limb_maps(e, p, bt->d_qlimb, bt->d_ylimb, bp, &map_q, &map_y)) return -4;
  {
    const size_t work = (e->count / 16) * (size_t)bp;
    alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(
        bt->d_req, e->slot_stride, kSlotLead + 9, (int)nc, bp, e->count, e->count, bt->d_ylimb);
    ALTO_H(cudaGetLastError());
    ++launches;
  }
  if (!launch_pack(e, p, map_y, bt->d_beta, nc, st, bt->d_err)) return -4;
  ++launches;
  ALTO_H(cudaEventRecord(e->ev_pack, st));
  // the query limb split and the zeroing of the scan sums once the query words are in, then validation and the
  // status download once the z keys are: on the side stream beside the pack (on the batch's stream after the pack
  // without the overlap).  The scans wait for the split only; the last tail also waits for the statuses.
  cudaStream_t vs = e->overlap ? bt->side : st;
  if (!piped) {
    ALTO_H(cudaStreamWaitEvent(vs, e->ev_queries, 0));
    if (!enqueue_query_split(e, bt, bt->d_req, e->slot_stride, nc, vs)) return -4;
    ++launches;
    if (e->overlap) ALTO_H(cudaEventRecord(bt->ev_qready, vs));
  } else {
    ALTO_H(cudaMemsetAsync(bt->d_acc, 0, nc * e->cols * sizeof(uint32_t), vs));
    for (int k = 0; k < qgroups; ++k) {
      size_t r0, r1;
      group_rows(k, &r0, &r1);
      ALTO_H(cudaStreamWaitEvent(vs, e->ev_qgrp[k], 0));
      const size_t work = ((r1 - r0) / 16) * (size_t)bp;
      alto::limb_split_kernel<<<(unsigned)((work + 255) / 256), 256, 0, vs>>>(
          bt->d_req, e->slot_stride, kSlotLead + 9 + 8 * e->count + 4 * r0, (int)nc, bp, r1 - r0, e->chunk,
          bt->d_qlimb + (r0 / e->chunk) * (4 * (size_t)bp * e->chunk));
      ALTO_H(cudaGetLastError());
      ++launches;
      ALTO_H(cudaEventRecord(e->ev_sgrp[k], vs));
    }
  }
  ALTO_H(cudaStreamWaitEvent(vs, e->ev_zkeys, 0));
  alto::validate_kernel<<<(unsigned)nc, 256, 0, vs>>>(bt->d_req, e->slot_stride, kSlotLead, e->count, e->rows,
                                                      bt->d_status);
  ALTO_H(cudaGetLastError());
  ++launches;
  ALTO_H(cudaMemcpyAsync(bt->h_status, bt->d_status, nc * sizeof(int), cudaMemcpyDeviceToHost, vs));
  ALTO_H(cudaEventRecord(e->ev_status, vs));
  // The scan in column groups (with the tails and downloads) covers the last quarter of the chunk groups, which it
  // starts once all query words are in; the chunk groups before it scan all columns as they arrive.  The upload of
  // the query words takes about three quarters of the scan's time (link bytes against int8 work per query word at
  // 32 KB records), so by the time the last words are in, about that share of the scan is done.
  const int qtail = qgroups - std::max(1, qgroups / 4);
  int kb_last = 0;
  if (piped) {
    for (int k = 0; k < qtail; ++k) {  // every earlier chunk group, all columns, as soon as it is split
      size_t r0, r1;
      group_rows(k, &r0, &r1);
      ALTO_H(cudaStreamWaitEvent(st, e->ev_sgrp[k], 0));
      if (!launch_scan(e, p, map_q, bt->d_acc, nc, st, bt->d_err, 0, -1, (int)(r0 / alto::kBK),
                       (int)((r1 + alto::kBK - 1) / alto::kBK)))
        return -4;
      ++launches;
    }
    size_t r0, r1;
    group_rows(qtail, &r0, &r1);
    ALTO_H(cudaStreamWaitEvent(st, e->ev_sgrp[qgroups - 1], 0));
    kb_last = (int)(r0 / alto::kBK);
  } else if (e->overlap) {
    ALTO_H(cudaStreamWaitEvent(st, bt->ev_qready, 0));
  }
  if (!enqueue_scan_tails(e, bt, p, map_q, bt->d_req, e->slot_stride, nc, bt->d_resp, e->resp_len, groups,
                          e->ev_group, &launches, nullptr, e->ev_status, groups.count - e->host_inline - 1, kb_last))
    return -4;
  // the error word comes back behind the last tail, so the final synchronisation covers it
  ALTO_H(cudaMemcpyAsync(bt->h_err, bt->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  e->last_launches = launches;

  // statuses come back as soon as validation is done; then each group's valid responses download on the copy
  // stream behind that group's tail
  ALTO_H(cudaEventSynchronize(e->ev_status));
  std::vector<size_t> ok;  // indices into cand with status 0
  for (size_t i = 0; i < nc; ++i) {
    status[cand[i]] = bt->h_status[i];
    if (bt->h_status[i] == 0) ok.push_back(i);
  }
  for (int g = 0; g < groups.count; ++g) {
    ALTO_H(cudaStreamWaitEvent(sc, e->ev_group[g], 0));
    const size_t off = (size_t)groups.bounds[g] * e->part_len;
    const size_t gbytes = (size_t)(groups.bounds[g + 1] - groups.bounds[g]) * e->part_len;
    if (!copy_runs(
            ok.size(), gbytes, [&](size_t k) { return (const void *)(bt->d_resp + ok[k] * e->resp_len + off); },
            [&](size_t k) { return (void *)(out[cand[ok[k]]] + off); }, cudaMemcpyDeviceToHost, sc))
      return -4;
  }
  ALTO_H(cudaEventRecord(e->ev_end, sc));
  ALTO_H(cudaStreamSynchronize(sc));
  ALTO_H(cudaStreamSynchronize(st));
  if (!check_error_word(e)) return -4;
  if (stage_ms) {
    float t0, t1, t2, t3;
    ALTO_H(cudaEventElapsedTime(&t0, e->ev_begin, e->ev_keys));                // key upload
    ALTO_H(cudaEventElapsedTime(&t1, e->ev_status, e->ev_group[groups.count - 1]));  // query split + scan + tails
    ALTO_H(cudaEventElapsedTime(&t2, e->ev_keys, e->ev_pack));                 // key split + pack
    ALTO_H(cudaEventElapsedTime(&t3, e->ev_group[groups.count - 1], e->ev_end));     // last download
    stage_ms[0] = t0;
    stage_ms[1] = t1;
    stage_ms[2] = t2;
    stage_ms[3] = t3;
  }
#undef ALTO_H
  return (int)ok.size();
}

}  // namespace

// ============================================================================================ C ABI
extern "C" {

const char *alto_last_error(void) { return g_last_error.c_str(); }

int sw_amx_init(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    set_error("no CUDA device");
    return -1;
  }
  if (cudaFree(nullptr) != cudaSuccess) {
    set_error("cannot create a CUDA context");
    return -1;
  }
  return 0;
}

}  // extern "C"

namespace {

// Loads records [first, first + count) from a record-major host buffer (record i at records + (i - first) * pitch,
// cols bytes each) into the database tiles, through a 64 MB device staging buffer: per pass, whole 128-record
// blocks of the tile grid (the first and last may be partly covered, their other records kept).
bool load_records(Engine *e, const uint8_t *records, size_t pitch, size_t first, size_t count) {
  for (int k = 0; k < e->lanes_made; ++k) {  // batches already enqueued read the database
    ALTO_CK(cudaStreamSynchronize(lane_batch(e, k)->st));
    ALTO_CK(cudaStreamSynchronize(lane_batch(e, k)->side));
  }
  const size_t per = std::max<size_t>(128, (size_t(64) << 20) / e->cols / 128 * 128);  // records per pass
  uint8_t *stage = nullptr;
  ALTO_CK(cudaMalloc(&stage, per * e->cols));
  bool ok = true;
  const size_t end = first + count;
  for (size_t a = first / 128 * 128; a < end && ok; a += per) {
    const size_t lo = std::max(a, first), hi = std::min(a + per, end);
    cudaError_t err = cudaMemcpy2D(stage + (lo - a) * e->cols, e->cols, records + (lo - first) * pitch, pitch,
                                   e->cols, hi - lo, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
      const dim3 grid((unsigned)((hi - a + 127) / 128), (unsigned)e->db_mts);
      alto::records_to_tiles_kernel<<<grid, 256>>>(stage, e->cols, a, lo, hi, e->d_db, e->db_kbs, e->cols);
      err = cudaGetLastError();
    }
    if (err != cudaSuccess) {
      set_error("database load", err);
      ok = false;
    }
  }
  const cudaError_t sync = cudaStreamSynchronize(0);
  if (ok && sync != cudaSuccess) {
    set_error("database load", sync);
    ok = false;
  }
  cudaFree(stage);
  return ok;
}

// The engine with the database db_col (column order, row pitch ld), or with a zero database to be loaded later
// (alto_engine_load_records) when db_col is NULL.
void *create_engine(const uint8_t *db_col, size_t ld, size_t rows, size_t cols, const int8_t *ub, size_t n,
                    size_t tg, const uint8_t *const *prefix, size_t part_len, size_t row1_off, uint64_t q1,
                    int q1_bits, const uint64_t *const *that, const uint64_t *inv_table, uint64_t q, int threads) {
  // The reference's checks (src/amx_kernels.cpp:551-552), then this engine's own limits.
  if (!ub || !prefix || !that || !inv_table || q != alto::kQ || !n || n > 4096 || n % 16 ||
      cols % n || rows % 64 || cols % 32 || threads <= 0 || (tg * n) % 128) {
    set_error("unsupported engine configuration");
    return nullptr;
  }
  if (tg < 1 || tg * n > 32768 || ld < rows || !rows || !cols) {
    set_error("configuration outside this engine's limits (1 <= tg, tg * n <= 32768, ld >= rows > 0)");
    return nullptr;
  }
  Engine *e = new Engine;
  e->rows = rows;
  e->cols = cols;
  e->n = n;
  e->tg = tg;
  e->outputs = cols / n;
  e->count = tg * n;
  e->part_len = part_len;
  e->row1_off = row1_off;
  e->q1 = q1;
  e->q1_bits = q1_bits;
  e->threads = threads;
  e->want = 9 + 4 * (2 * e->count + rows);
  e->resp_len = e->outputs * part_len;
  e->slot_stride = round_up(kSlotLead + e->want, 256);
  // The reference's tail checks (src/amx_kernels.cpp:463, 517), evaluated once here and reported per batch.
  e->tail_ok = n >= 16 && (n & (n - 1)) == 0 && q1 < (1ull << 21) && n % 8 == 0 &&
               (row1_off + n * (size_t)q1_bits + 7) / 8 <= part_len && q1_bits <= 24;
  auto fail = [&](const char *where, cudaError_t err) -> void * {
    set_error(where, err);
    destroy(e);
    return nullptr;
  };
  cudaError_t err;
  if ((err = cudaGetDevice(&e->dev)) != cudaSuccess) return fail("cudaGetDevice", err);
  if (!init_batch(&e->main, true)) {
    destroy(e);
    return nullptr;
  }
  if ((err = cudaStreamCreateWithFlags(&e->st_copy, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream", err);
  if (const char *v = getenv("ALTO_OVERLAP")) e->overlap = v[0] != '0';
  if (const char *v = getenv("ALTO_GROUPS")) e->groups = std::max(1, std::min(8, atoi(v)));
  if (const char *v = getenv("ALTO_HOST_GROUPS")) e->host_weights = group_weights(atoi(v), true);
  if (const char *v = getenv("ALTO_HOST_INLINE")) e->host_inline = std::max(0, std::min(7, atoi(v)));
  if (const char *v = getenv("ALTO_PIPED_BYTES")) e->piped_bytes = (size_t)strtoull(v, nullptr, 10);
  if (const char *v = getenv("ALTO_HOST_WEIGHTS")) {
    std::vector<int> w = parse_weights(v);
    if (!w.empty()) e->host_weights = w;
  }
  if ((err = cudaEventCreate(&e->ev_begin)) != cudaSuccess || (err = cudaEventCreate(&e->ev_end)) != cudaSuccess ||
      (err = cudaEventCreate(&e->ev_keys)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&e->ev_queries, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&e->ev_zkeys, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaEventCreate(&e->ev_pack)) != cudaSuccess || (err = cudaEventCreate(&e->ev_status)) != cudaSuccess)
    return fail("event", err);
  for (cudaEvent_t &ev : e->ev_group)
    if ((err = cudaEventCreate(&ev)) != cudaSuccess) return fail("event", err);
  for (cudaEvent_t *set : {e->ev_qgrp, e->ev_sgrp})
    for (int k = 0; k < kQueryGroups; ++k)
      if ((err = cudaEventCreateWithFlags(&set[k], cudaEventDisableTiming)) != cudaSuccess) return fail("event", err);
  for (auto &set : e->marks)
    for (cudaEvent_t &ev : set)
      if ((err = cudaEventCreate(&ev)) != cudaSuccess) return fail("event", err);
  // record chunks of the query limbs (the scan's B operand)
  e->chunk = rows > kRecordChunk ? kRecordChunk : rows;
  e->nchunks = (rows + e->chunk - 1) / e->chunk;
  // The database (rows = record byte positions, K = records) and the packing matrix (rows = (column, plane),
  // K = tg * n) are stored tile by tile, so that every TMA box of the GEMMs is one contiguous 16 KB read: with
  // row-major operands a box is 128 separate 128-byte pieces, one per row, and the GEMMs measured 13 % slower.
  e->db_kbs = (rows + 127) / 128;
  e->db_mts = (cols + 127) / 128;
  e->ub_kbs = e->count / 128;
  e->ub_mts = (4 * cols + 127) / 128;
  if ((err = cudaMalloc(&e->d_db, e->db_mts * e->db_kbs * 16384)) != cudaSuccess) return fail("database", err);
  if (!db_col) {
    if ((err = cudaMemset(e->d_db, 0, e->db_mts * e->db_kbs * 16384)) != cudaSuccess) return fail("database", err);
  } else if (!upload_tiled(e->d_db, db_col, ld, cols, rows, e->db_kbs, e->db_mts)) {
    destroy(e);
    return nullptr;
  }
  if ((err = cudaMalloc(&e->d_ub, e->ub_mts * e->ub_kbs * 16384)) != cudaSuccess) return fail("packing matrix", err);
  if (!upload_tiled(e->d_ub, reinterpret_cast<const uint8_t *>(ub), e->count, 4 * cols, e->count, e->ub_kbs,
                    e->ub_mts)) {
    destroy(e);
    return nullptr;
  }
  // The tail's inverse NTT runs without the reference's halving of every sum (kernels.cuh, tail_kernel): both
  // inputs of the key-switch accumulate -- the packing matrix (through beta) and bold_t_hat -- are stored times
  // 2^-log2(n), and the twiddles doubled, so the transform's output equals the reference's mod Q.
  int logn = 0;
  while ((size_t(1) << logn) < n) ++logn;
  const uint32_t ninv = alto::inv_pow2_q(logn);
  {
    const size_t ntiles = e->ub_mts * e->ub_kbs;
    alto::scale_planes_kernel<<<(unsigned)((ntiles * 1024 + 255) / 256), 256>>>(e->d_ub, ntiles, ninv);
    if ((err = cudaGetLastError()) != cudaSuccess || (err = cudaStreamSynchronize(0)) != cudaSuccess)
      return fail("packing matrix scaling", err);
  }
  {
    std::vector<uint32_t> th(e->outputs * e->count);
    for (size_t o = 0; o < e->outputs; ++o)
      for (size_t k = 0; k < e->count; ++k)
        th[o * e->count + k] = alto::mul_q((uint32_t)(that[o][k] % alto::kQ), ninv);
    if ((err = cudaMalloc(&e->d_that, th.size() * 4)) != cudaSuccess) return fail("bold_t_hat", err);
    if ((err = cudaMemcpy(e->d_that, th.data(), th.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail("bold_t_hat upload", err);
    std::vector<uint32_t> tw(n);
    // the reference multiplies by the low 32 bits of each entry (src/amx_kernels.cpp:459); doubled mod Q here
    for (size_t i = 0; i < n; ++i) tw[i] = alto::red_q64(2 * (inv_table[i] & 0xffffffffull));
    if ((err = cudaMalloc(&e->d_tw, n * 4)) != cudaSuccess) return fail("inverse table", err);
    if ((err = cudaMemcpy(e->d_tw, tw.data(), n * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail("inverse table upload", err);
    std::vector<uint8_t> pre(e->outputs * part_len);
    for (size_t o = 0; o < e->outputs; ++o) memcpy(pre.data() + o * part_len, prefix[o], part_len);
    if ((err = cudaMalloc(&e->d_prefix, pre.size() ? pre.size() : 1)) != cudaSuccess) return fail("prefixes", err);
    if (!pre.empty() && (err = cudaMemcpy(e->d_prefix, pre.data(), pre.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
      return fail("prefix upload", err);
  }
  if (!make_tile_map(&e->map_db, e->d_db, e->db_kbs, e->db_mts) ||
      !make_tile_map(&e->map_ub, e->d_ub, e->ub_kbs, e->ub_mts)) {
    destroy(e);
    return nullptr;
  }
  resident_pairs();  // occupancy query outside any stream capture
  load_tuning(e);
  return e;
}

}  // namespace

extern "C" {

void *alto_engine_new(const uint8_t *db_col, const uint8_t *db_tiled, size_t ld, size_t rows, size_t cols,
                      const int8_t *ub, size_t n, size_t tg, const uint8_t *const *prefix, size_t part_len,
                      size_t row1_off, uint64_t q1, int q1_bits, const uint64_t *const *that,
                      const uint64_t *inv_table, uint64_t q, int threads) {
  if (!db_col || !db_tiled) {  // src/amx_kernels.cpp:551
    set_error("unsupported engine configuration");
    return nullptr;
  }
  return create_engine(db_col, ld, rows, cols, ub, n, tg, prefix, part_len, row1_off, q1, q1_bits, that, inv_table,
                       q, threads);
}

void *alto_engine_new_empty(size_t rows, size_t cols, const int8_t *ub, size_t n, size_t tg,
                            const uint8_t *const *prefix, size_t part_len, size_t row1_off, uint64_t q1, int q1_bits,
                            const uint64_t *const *that, const uint64_t *inv_table, uint64_t q, int threads) {
  return create_engine(nullptr, rows, rows, cols, ub, n, tg, prefix, part_len, row1_off, q1, q1_bits, that, inv_table,
                       q, threads);
}

int alto_engine_load_records(void *p, const uint8_t *records, size_t pitch, size_t first, size_t count) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || (!records && count) || pitch < e->cols || first > e->rows || count > e->rows - first) {
    set_error("alto_engine_load_records: bad arguments");
    return -1;
  }
  if (!count) return 0;
  if (cudaSetDevice(e->dev) != cudaSuccess || !load_records(e, records, pitch, first, count)) return -4;
  return 0;
}

int alto_engine_load_file(void *p, const char *path, size_t num_real_rows) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !path || num_real_rows > e->rows) {
    set_error("alto_engine_load_file: bad arguments");
    return -1;
  }
  FILE *f = fopen(path, "rb");
  if (!f) {
    set_error(std::string("alto_engine_load_file: cannot open ") + path);
    return -2;
  }
  // whole blocks of 128 records per read (about 4 MB per 128 records of 32 KB), at most 64 MB
  const size_t block = std::max<size_t>(128, (size_t(64) << 20) / e->cols / 128 * 128);
  std::vector<uint8_t> buf(block * e->cols);
  int rc = 0;
  if (cudaSetDevice(e->dev) != cudaSuccess) rc = -4;
  for (size_t r0 = 0; r0 < num_real_rows && rc == 0; r0 += block) {
    const size_t nr = std::min(block, num_real_rows - r0);
    if (fread(buf.data(), e->cols, nr, f) != nr) {
      set_error(std::string("alto_engine_load_file: short read in ") + path);
      rc = -2;
    } else if (!load_records(e, buf.data(), e->cols, r0, nr)) {
      rc = -4;
    }
  }
  fclose(f);
  return rc;
}

void alto_engine_free(void *p) { destroy(static_cast<Engine *>(p)); }

size_t alto_request_len(const void *p) {
  const Engine *e = static_cast<const Engine *>(p);
  return 9 + 4 * (2 * e->tg * e->n + e->rows);
}

size_t alto_response_len(const void *p) {
  const Engine *e = static_cast<const Engine *>(p);
  return e->outputs * e->part_len;
}

int alto_answer(void *p, const uint8_t *const *req, const size_t *len, size_t b, uint8_t *const *out, int *status,
                int method, double *stage_ms) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !req || !len || !out || !status || (method != 0 && method != 2)) return -1;
  return answer_host(e, req, len, b, out, status, stage_ms);
}

int alto_answer_device(void *p, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out, size_t out_stride,
                       int *status, double *stage_ms) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !d_req || !d_out || !status || req_stride % 16 || req_stride < round_up(kSlotLead + e->want, 16) ||
      out_stride < e->resp_len)
    return -1;
  if (stage_ms) std::fill(stage_ms, stage_ms + 4, 0.0);
  e->last_launches = 0;
  if (!b) return 0;
  if (!e->tail_ok) return -3;
  if (cudaSetDevice(e->dev) != cudaSuccess || !ensure_capacity(e, &e->main, b)) return -4;
  if (cudaEventRecord(e->ev_begin, e->main.st) != cudaSuccess) return -4;
  if (!enqueue_batch(e, &e->main, d_req, req_stride, b, d_out, out_stride, true)) return -4;
  if (cudaEventRecord(e->ev_end, e->main.st) != cudaSuccess) return -4;
  if (!finish(e, stage_ms)) return -4;
  int valid = 0;
  for (size_t c = 0; c < b; ++c) {
    status[c] = e->main.h_status[c];
    valid += status[c] == 0;
  }
  return valid;
}

int alto_answer_device_parts(void *p, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *const *d_outs,
                             size_t n_outs, size_t out_stride, size_t part_offset, int *status) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !d_req || !d_outs || !status || !n_outs || n_outs > kMaxGather || req_stride % 16 ||
      req_stride < round_up(kSlotLead + e->want, 16) || out_stride < (part_offset + e->outputs) * e->part_len) {
    set_error("alto_answer_device_parts: bad arguments");
    return -1;
  }
  for (size_t k = 0; k < n_outs; ++k)
    if (!d_outs[k]) {
      set_error("alto_answer_device_parts: NULL output buffer");
      return -1;
    }
  e->last_launches = 0;
  if (!b) return 0;
  if (!e->tail_ok) return -3;
  Batch *bt = &e->main;
  if (cudaSetDevice(e->dev) != cudaSuccess || !ensure_capacity(e, bt, b)) return -4;
  if (!bt->d_gather && cudaMalloc(&bt->d_gather, kMaxGather * sizeof(uint8_t *)) != cudaSuccess) {
    set_error("gather list", cudaGetLastError());
    return -4;
  }
  // the previous batch may still read the list; the copy from the caller's array must finish before it returns
  if (cudaStreamSynchronize(bt->st) != cudaSuccess ||
      cudaMemcpy(bt->d_gather, d_outs, n_outs * sizeof(uint8_t *), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("gather list", cudaGetLastError());
    return -4;
  }
  bt->n_gather = (int)n_outs;
  bt->gather_offset = (int)part_offset;
  // launched directly: a captured graph would hold this call's destinations
  const bool ok = enqueue_batch_direct(e, bt, d_req, req_stride, b, nullptr, out_stride, true, true);
  bt->n_gather = 0;
  bt->gather_offset = 0;
  if (!ok || !finish(e, nullptr)) return -4;
  int valid = 0;
  for (size_t c = 0; c < b; ++c) {
    status[c] = bt->h_status[c];
    valid += status[c] == 0;
  }
  return valid;
}

int alto_ipc_export(const void *d_ptr, uint8_t *handle, size_t *offset) {
  if (!d_ptr || !handle || !offset) return -1;
  // An IPC handle names a whole allocation and opens at its base; d_ptr may lie inside a larger one (a caching
  // allocator's segment), so the handle is taken for the base and the offset travels with it.
  using AddressRangeFn = CUresult (*)(CUdeviceptr *, size_t *, CUdeviceptr);
  static AddressRangeFn range_fn = nullptr;
  if (!range_fn) {
    void *fp = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fp, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      range_fn = reinterpret_cast<AddressRangeFn>(fp);
  }
  CUdeviceptr base = 0;
  size_t size = 0;
  if (!range_fn || range_fn(&base, &size, reinterpret_cast<CUdeviceptr>(d_ptr)) != CUDA_SUCCESS) {
    set_error("cuMemGetAddressRange failed: not a device allocation of this process");
    return -4;
  }
  cudaIpcMemHandle_t h;
  const cudaError_t err = cudaIpcGetMemHandle(&h, reinterpret_cast<void *>(base));
  if (err != cudaSuccess) {
    set_error("cudaIpcGetMemHandle", err);
    return -4;
  }
  static_assert(sizeof(h) == 64, "CUDA IPC handles are 64 bytes");
  memcpy(handle, &h, sizeof(h));
  *offset = reinterpret_cast<CUdeviceptr>(d_ptr) - base;
  return 0;
}

void *alto_ipc_import(const uint8_t *handle) {
  if (!handle) return nullptr;
  cudaIpcMemHandle_t h;
  memcpy(&h, handle, sizeof(h));
  void *p = nullptr;
  const cudaError_t err = cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess);
  if (err != cudaSuccess) {
    set_error("cudaIpcOpenMemHandle", err);
    return nullptr;
  }
  return p;
}

int alto_ipc_release(void *d_ptr) {
  if (!d_ptr) return -1;
  const cudaError_t err = cudaIpcCloseMemHandle(d_ptr);
  if (err != cudaSuccess) {
    set_error("cudaIpcCloseMemHandle", err);
    return -4;
  }
  return 0;
}

int alto_enqueue_device(void *p, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out, size_t out_stride,
                        int *d_status) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !d_req || !d_out || req_stride % 16 || req_stride < round_up(kSlotLead + e->want, 16) ||
      out_stride < e->resp_len)
    return -1;
  e->last_launches = 0;
  if (!b) return 0;
  if (!e->tail_ok) return -3;
  Batch *bt = lane_batch(e, e->lane_next);
  e->lane_next = (e->lane_next + 1) % e->lanes;
  if (cudaSetDevice(e->dev) != cudaSuccess || !ensure_capacity(e, bt, b)) return -4;
  if (!enqueue_batch(e, bt, d_req, req_stride, b, d_out, out_stride, false)) return -4;
  if (d_status &&
      cudaMemcpyAsync(d_status, bt->d_status, b * sizeof(int), cudaMemcpyDeviceToDevice, bt->st) != cudaSuccess) {
    set_error("status copy failed");
    return -4;
  }
  return 0;
}

int alto_engine_sync(void *p) {
  Engine *e = static_cast<Engine *>(p);
  if (!e) return -1;
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  return sync_engine(e) ? 0 : -4;
}

void *alto_engine_stream(void *p) { return p ? static_cast<void *>(static_cast<Engine *>(p)->main.st) : nullptr; }

int alto_kernel_times(void *p, double *ms, long long *batches, int reset) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !ms) return -1;
  if (cudaSetDevice(e->dev) != cudaSuccess || !sync_engine(e)) return -4;
  for (int i = 0; i < 5; ++i) ms[i] = e->kernel_ms[i];
  if (batches) *batches = e->kernel_batches;
  if (reset) {
    std::fill(e->kernel_ms, e->kernel_ms + 5, 0.0);
    e->kernel_batches = 0;
  }
  return 0;
}

int alto_last_launches(const void *p) { return p ? static_cast<const Engine *>(p)->last_launches.load() : 0; }

int alto_engine_set_tuning(void *p, const int32_t *entries, size_t n) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || (n && !entries)) return -1;
  if (cudaSetDevice(e->dev) != cudaSuccess || !sync_engine(e)) return -4;
  e->tuning.clear();
  for (size_t i = 0; i < n; ++i)
    e->tuning.push_back({entries[5 * i], entries[5 * i + 1], entries[5 * i + 2], entries[5 * i + 3],
                         entries[5 * i + 4]});
  std::sort(e->tuning.begin(), e->tuning.end(), [](const TuneEntry &a, const TuneEntry &b) { return a.b_max < b.b_max; });
  for (int k = 0; k < e->lanes_made; ++k) clear_graphs(lane_batch(e, k));  // captured sequences follow old plans
  return 0;
}

int alto_engine_set_graphs(void *p, int on) {
  Engine *e = static_cast<Engine *>(p);
  if (!e) return -1;
  if (cudaSetDevice(e->dev) != cudaSuccess || !sync_engine(e)) return -4;
  e->use_graphs = on != 0;
  if (!e->use_graphs)
    for (int k = 0; k < e->lanes_made; ++k) clear_graphs(lane_batch(e, k));
  return 0;
}

int alto_engine_set_lanes(void *p, int lanes) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || lanes < 1 || lanes > kMaxLanes) return -1;
  if (cudaSetDevice(e->dev) != cudaSuccess || !sync_engine(e)) return -4;
  for (int k = 0; k < kMaxLanes; ++k)
    if (!e->ev_lane[k] && cudaEventCreateWithFlags(&e->ev_lane[k], cudaEventDisableTiming) != cudaSuccess) {
      set_error("lane event", cudaGetLastError());
      return -4;
    }
  while (e->lanes_made < lanes) {
    if (!init_batch(&e->lane[e->lanes_made - 1], false)) return -4;
    ++e->lanes_made;
  }
  e->lanes = lanes;
  e->lane_next = 0;
  return 0;
}

int alto_engine_fence(void *p) {
  Engine *e = static_cast<Engine *>(p);
  if (!e) return -1;
  if (e->lanes_made == 1) return 0;
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  for (int k = 0; k < e->lanes_made; ++k)
    if (cudaEventRecord(e->ev_lane[k], lane_batch(e, k)->st) != cudaSuccess) {
      set_error("lane fence", cudaGetLastError());
      return -4;
    }
  for (int j = 0; j < e->lanes_made; ++j)
    for (int k = 0; k < e->lanes_made; ++k)
      if (k != j && cudaStreamWaitEvent(lane_batch(e, j)->st, e->ev_lane[k], 0) != cudaSuccess) {
        set_error("lane fence", cudaGetLastError());
        return -4;
      }
  return 0;
}

int alto_synthetic_db_col_device(uint8_t *d_db, size_t ld, size_t rows, size_t col0, size_t ncols) {
  if (rows % 4 || ld % 4) return -1;
  const size_t work = (rows / 4) * ncols;
  alto::synthetic_db_kernel<<<(unsigned)((work + 255) / 256), 256>>>(d_db, ld, rows, col0, ncols);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error("synthetic database", e);
    return -1;
  }
  return 0;
}

int alto_hint_ring(void *p, const uint64_t *query, uint64_t *out, int perm_out) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !query || !out) {
    set_error("alto_hint_ring: bad arguments");
    return -1;
  }
  std::vector<uint32_t> psi, psi_inv;
  uint32_t n_inv = 0;
  if (e->rows % e->n || !alto::hint_tables((int)e->n, psi, psi_inv, n_inv)) {
    set_error("alto_hint_ring: needs records a multiple of n and n a power of two <= 2048");
    return -1;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  const size_t n = e->n, polys = e->rows / n;
  uint64_t *d_query = nullptr, *d_out = nullptr;
  uint32_t *d_qhat = nullptr, *d_psi = nullptr, *d_psi_inv = nullptr;
  cudaError_t err = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (err == cudaSuccess) err = x;
  };
  step(cudaMalloc(&d_query, e->rows * sizeof(uint64_t)));
  step(cudaMalloc(&d_qhat, e->rows * sizeof(uint32_t)));
  step(cudaMalloc(&d_psi, n * sizeof(uint32_t)));
  step(cudaMalloc(&d_psi_inv, n * sizeof(uint32_t)));
  step(cudaMalloc(&d_out, n * e->cols * sizeof(uint64_t)));
  step(cudaMemcpy(d_query, query, e->rows * sizeof(uint64_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_psi, psi.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_psi_inv, psi_inv.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  const unsigned threads = (unsigned)std::max<size_t>(32, std::min<size_t>(256, n / 2));
  if (err == cudaSuccess) {
    alto::hint_query_kernel<<<(unsigned)polys, threads, n * sizeof(uint32_t)>>>(d_query, (int)n, d_psi, n_inv,
                                                                               d_qhat);
    step(cudaGetLastError());
  }
  if (err == cudaSuccess) {
    alto::hint_ring_kernel<<<(unsigned)e->cols, threads, 2 * n * sizeof(uint32_t)>>>(
        e->d_db, e->db_kbs, (int)n, (int)polys, d_qhat, d_psi, d_psi_inv, d_out, e->cols, perm_out);
    step(cudaGetLastError());
  }
  step(cudaMemcpy(out, d_out, n * e->cols * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  cudaFree(d_query);
  cudaFree(d_qhat);
  cudaFree(d_psi);
  cudaFree(d_psi_inv);
  cudaFree(d_out);
  if (err != cudaSuccess) {
    set_error("alto_hint_ring", err);
    return -4;
  }
  return 0;
}

int alto_engine_offline(void *p, const uint64_t *query, const uint64_t *w_mask, const uint64_t *v_mask,
                        uint32_t *bold_t, uint32_t *bold_t_bar, uint32_t *that, uint32_t *a_hat, double *ms) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !query || !w_mask || !v_mask) {
    set_error("alto_engine_offline: bad arguments");
    return -1;
  }
  const size_t n = e->n, tg = e->tg, cols = e->cols, outputs = e->outputs, half = n / 2;
  std::vector<uint32_t> psi, psi_inv;
  uint32_t n_inv = 0;
  if (n < 8 || e->rows % n || e->row1_off % n || !alto::hint_tables((int)n, psi, psi_inv, n_inv)) {
    set_error("alto_engine_offline: needs n a power of two in [8, 2048], records a multiple of n, row 1 at q2_bits n");
    return -1;
  }
  const int q2_bits = (int)(e->row1_off / n);
  if (q2_bits < 1 || q2_bits > 31 || ((size_t)q2_bits * n + 7) / 8 > e->part_len) {
    set_error("alto_engine_offline: row 0 does not fit the response part");
    return -1;
  }
  int logn = 0;
  while ((size_t(1) << logn) < n) ++logn;
  // gadget digits: floor(32 / t) + 1 bits each (one bit when t = 32), as get_bits_per gives for log2ceil(Q) = 32
  const int bits = tg >= 32 ? 1 : (int)(32 / tg) + 1;
  // dlog[(t - 1) / 2] = 2 i + bar for t = g^i (bar 0) or 2n - g^i (bar 1); inv_odd[x] = (2x + 1)^-1 mod 2n
  std::vector<int16_t> dlog(n, -1);
  std::vector<uint16_t> inv_odd(n);
  for (size_t i = 0, g = 1; i < half; ++i, g = (g * 5) % (2 * n)) {
    dlog[(g - 1) / 2] = (int16_t)(2 * i);
    dlog[(2 * n - g - 1) / 2] = (int16_t)(2 * i + 1);
  }
  for (size_t x = 0; x < n; ++x) {
    const size_t a = 2 * x + 1;
    size_t inv = 1;  // the odd residues mod 2n form a group of order n, so a^(n - 1) = a^-1
    for (size_t k = 0; k + 1 < n; ++k) inv = inv * a % (2 * n);
    inv_odd[x] = (uint16_t)inv;
  }
  for (size_t x = 0; x < n; ++x)
    if (dlog[x] < 0 || (2 * x + 1) * inv_odd[x] % (2 * n) != 1) {
      set_error("alto_engine_offline: automorphism tables");
      return -1;
    }
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  for (int k = 0; k < e->lanes_made; ++k) {  // batches already enqueued read the packing state
    if (cudaStreamSynchronize(lane_batch(e, k)->st) != cudaSuccess ||
        cudaStreamSynchronize(lane_batch(e, k)->side) != cudaSuccess) {
      set_error("alto_engine_offline", cudaGetLastError());
      return -4;
    }
  }
  std::vector<uint32_t> w32(tg * n), v32(tg * n);
  for (size_t i = 0; i < tg * n; ++i) {
    w32[i] = (uint32_t)(w_mask[i] % alto::kQ);
    v32[i] = (uint32_t)(v_mask[i] % alto::kQ);
  }
  const size_t polys = e->rows / n, bt_words = outputs * 2 * (half - 1) * tg * n;
  uint64_t *d_q = nullptr;
  uint32_t *d_qhat = nullptr, *d_psi = nullptr, *d_psi_inv = nullptr, *d_w = nullptr, *d_v = nullptr;
  uint32_t *d_act = nullptr, *d_bt = nullptr, *d_last = nullptr, *d_that = nullptr, *d_ahat = nullptr;
  int16_t *d_dlog = nullptr;
  uint16_t *d_inv_odd = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaError_t err = cudaSuccess;
  auto step = [&](cudaError_t x) {
    if (err == cudaSuccess) err = x;
  };
  step(cudaEventCreate(&t0));
  step(cudaEventCreate(&t1));
  step(cudaMalloc(&d_q, e->rows * sizeof(uint64_t)));
  step(cudaMalloc(&d_qhat, e->rows * sizeof(uint32_t)));
  step(cudaMalloc(&d_psi, n * sizeof(uint32_t)));
  step(cudaMalloc(&d_psi_inv, n * sizeof(uint32_t)));
  step(cudaMalloc(&d_w, tg * n * sizeof(uint32_t)));
  step(cudaMalloc(&d_v, tg * n * sizeof(uint32_t)));
  step(cudaMalloc(&d_act, cols * n * sizeof(uint32_t)));
  step(cudaMalloc(&d_bt, bt_words * sizeof(uint32_t)));
  step(cudaMalloc(&d_last, outputs * 2 * n * sizeof(uint32_t)));
  step(cudaMalloc(&d_dlog, n * sizeof(int16_t)));
  step(cudaMalloc(&d_inv_odd, n * sizeof(uint16_t)));
  if (that) step(cudaMalloc(&d_that, outputs * tg * n * sizeof(uint32_t)));
  if (a_hat) step(cudaMalloc(&d_ahat, outputs * n * sizeof(uint32_t)));
  step(cudaMemcpy(d_q, query, e->rows * sizeof(uint64_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_psi, psi.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_psi_inv, psi_inv.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_w, w32.data(), tg * n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_v, v32.data(), tg * n * sizeof(uint32_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_dlog, dlog.data(), n * sizeof(int16_t), cudaMemcpyHostToDevice));
  step(cudaMemcpy(d_inv_odd, inv_odd.data(), n * sizeof(uint16_t), cudaMemcpyHostToDevice));
  const size_t act_smem = (1 + alto::kActCols) * n * sizeof(uint32_t), walk_smem = (1 + tg) * n * sizeof(uint32_t);
  step(cudaFuncSetAttribute(alto::offline_act_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)act_smem));
  // n = 2048: the act kernel with register transforms (ALTO_OFFLINE_ACT8=0 runs the shared-memory one)
  bool act8 = true;
  if (const char *v = getenv("ALTO_OFFLINE_ACT8")) act8 = v[0] != '0';
  // columns a CTA of the register-transform act kernel accumulates (ALTO_OFFLINE_ACTCOLS: 1, 2, 4 or 8).  Fewer
  // columns keep less shared memory, so more CTAs share an SM: at 64 GiB the set-up took 736 ms with 8, 613 with 4,
  // 586 with 2 and 582 with 1; at 1 GiB 31.4, 29.8, 29.4 and 29.5 ms.
  int act_cols = 2;
  if (const char *v = getenv("ALTO_OFFLINE_ACTCOLS")) {
    const int c = atoi(v);
    act_cols = c == 1 || c == 4 || c == 8 ? c : 2;
  }
  const size_t act8_smem = (2 + (size_t)act_cols) * n * sizeof(uint32_t);
  if (n == 2048) {
    step(cudaFuncSetAttribute(alto::offline_act8_kernel<11, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((2 + 1) * n * sizeof(uint32_t))));
    step(cudaFuncSetAttribute(alto::offline_act8_kernel<11, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((2 + 2) * n * sizeof(uint32_t))));
    step(cudaFuncSetAttribute(alto::offline_act8_kernel<11, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((2 + 4) * n * sizeof(uint32_t))));
    step(cudaFuncSetAttribute(alto::offline_act8_kernel<11, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((2 + 8) * n * sizeof(uint32_t))));
  }
  step(cudaFuncSetAttribute(alto::offline_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)walk_smem));
  step(cudaFuncSetAttribute(alto::offline_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)walk_smem));
  // the walk's cluster: one CTA per gadget digit, at most 8 (the portable cluster size); ALTO_OFFLINE_CLUSTER=1 runs
  // the single-CTA walk
  int cluster = (int)std::min<size_t>(tg, 8);
  if (const char *v = getenv("ALTO_OFFLINE_CLUSTER")) cluster = std::max(1, std::min(8, atoi(v)));
  const size_t cwalk_smem = (2 + (tg + cluster - 1) / cluster) * n * sizeof(uint32_t);
  if (cluster > 1)
    step(cudaFuncSetAttribute(alto::offline_walk_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)cwalk_smem));
  // n = 2048 with one digit a CTA: the walk with register transforms (ALTO_OFFLINE_WALK8=0 runs the other)
  bool walk8 = n == 2048 && cluster == (int)tg;
  if (const char *v = getenv("ALTO_OFFLINE_WALK8")) walk8 = walk8 && v[0] != '0';
  const size_t walk8_smem = (2 + 2 * (size_t)cluster) * n * sizeof(uint32_t);
  if (walk8)
    step(cudaFuncSetAttribute(alto::offline_walk8_kernel<11>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)walk8_smem));
  const unsigned nt = (unsigned)std::max<size_t>(32, std::min<size_t>(256, n / 2));
  // walk and finish threads: at least n / 4 (the cluster walk gathers 4 slots a thread ahead), at most 1024
  const unsigned wt = (unsigned)std::max<size_t>(std::max<size_t>(64, n / 4), std::min<size_t>(1024, tg * n / 2));
  const uint32_t tail_scale = alto::inv_pow2_q(logn);
  const size_t K = tg * n, planes_threads = cols * K;
  if (err == cudaSuccess) {
    step(cudaEventRecord(t0, 0));
    // the hint's query: NTT(perm(q_p)), without the n^-1 the coefficient-domain hint folds in
    alto::hint_query_kernel<<<(unsigned)polys, nt, n * sizeof(uint32_t)>>>(d_q, (int)n, d_psi, 1u, d_qhat);
    step(cudaGetLastError());
    if (n == 2048 && act8 && act_cols == 1) {
      alto::offline_act8_kernel<11, 1><<<(unsigned)cols, 256, act8_smem>>>(e->d_db, e->db_kbs, (int)polys, d_qhat,
                                                                         d_psi, d_act);
    } else if (n == 2048 && act8 && act_cols == 2) {
      alto::offline_act8_kernel<11, 2><<<(unsigned)(cols / 2), 256, act8_smem>>>(e->d_db, e->db_kbs, (int)polys,
                                                                               d_qhat, d_psi, d_act);
    } else if (n == 2048 && act8 && act_cols == 4) {
      alto::offline_act8_kernel<11, 4><<<(unsigned)(cols / 4), 256, act8_smem>>>(e->d_db, e->db_kbs, (int)polys,
                                                                               d_qhat, d_psi, d_act);
    } else if (n == 2048 && act8) {
      alto::offline_act8_kernel<11, 8><<<(unsigned)(cols / 8), 256, act8_smem>>>(e->d_db, e->db_kbs, (int)polys,
                                                                               d_qhat, d_psi, d_act);
    } else {
      alto::offline_act_kernel<<<(unsigned)(cols / alto::kActCols), 256, act_smem>>>(e->d_db, e->db_kbs, (int)n,
                                                                                    (int)polys, d_qhat, d_psi, d_act);
    }
    step(cudaGetLastError());
    alto::offline_rows_kernel<<<(unsigned)cols, nt, n * sizeof(uint32_t)>>>(d_act, (int)n, d_psi);
    step(cudaGetLastError());
    if (cluster > 1) {
      // one cluster of `cluster` CTAs per (output, chain), the digits split between them
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)cluster;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3((unsigned)(outputs * 2 * cluster));
      cfg.blockDim = dim3(wt);
      cfg.dynamicSmemBytes = cwalk_smem;
      cfg.stream = 0;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if (walk8) {  // n = 2048, one digit a CTA: both transforms in registers
        cfg.blockDim = dim3((unsigned)(n / 8));
        cfg.dynamicSmemBytes = walk8_smem;
        step(cudaLaunchKernelEx(&cfg, alto::offline_walk8_kernel<11>, (const uint32_t *)d_act, (int)tg, bits,
                                (const uint32_t *)d_w, (const uint32_t *)d_psi, (const uint32_t *)d_psi_inv, n_inv,
                                d_bt, d_last));
      } else {
        step(cudaLaunchKernelEx(&cfg, alto::offline_walk_cluster_kernel, (const uint32_t *)d_act, (int)n, logn,
                                (int)tg, bits, (const uint32_t *)d_w, (const uint32_t *)d_psi,
                                (const uint32_t *)d_psi_inv, n_inv, d_bt, d_last));
      }
    } else {
      alto::offline_walk_kernel<<<(unsigned)(outputs * 2), wt, walk_smem>>>(d_act, (int)n, logn, (int)tg, bits, d_w,
                                                                            d_psi, d_psi_inv, n_inv, d_bt, d_last);
    }
    step(cudaGetLastError());
    alto::offline_finish_kernel<<<(unsigned)outputs, wt, walk_smem>>>(d_last, (int)n, (int)tg, bits, d_v, d_psi,
                                                                      d_psi_inv, n_inv, tail_scale, e->d_that,
                                                                      e->d_prefix, e->part_len, q2_bits, d_that, d_ahat);
    step(cudaGetLastError());
    alto::offline_planes_kernel<<<(unsigned)((planes_threads + 255) / 256), 256>>>(
        d_bt, (int)n, logn, (int)tg, cols, d_dlog, d_inv_odd, tail_scale, e->d_ub, e->ub_kbs);
    step(cudaGetLastError());
    // the engine's tail twiddles: its inverse table psi^-brv / 2, doubled as create_engine stores it
    step(cudaMemcpyAsync(e->d_tw, d_psi_inv, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, 0));
    step(cudaEventRecord(t1, 0));
    step(cudaEventSynchronize(t1));
  }
  if (err == cudaSuccess && ms) {
    float f = 0.f;
    step(cudaEventElapsedTime(&f, t0, t1));
    *ms = f;
  }
  const size_t per = (half - 1) * tg * n;
  for (size_t o = 0; o < outputs && err == cudaSuccess; ++o) {
    if (bold_t)
      step(cudaMemcpy(bold_t + o * per, d_bt + (o * 2) * per, per * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (bold_t_bar)
      step(cudaMemcpy(bold_t_bar + o * per, d_bt + (o * 2 + 1) * per, per * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  }
  if (that) step(cudaMemcpy(that, d_that, outputs * tg * n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (a_hat) step(cudaMemcpy(a_hat, d_ahat, outputs * n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  for (void *x : {(void *)d_q, (void *)d_qhat, (void *)d_psi, (void *)d_psi_inv, (void *)d_w, (void *)d_v,
                  (void *)d_act, (void *)d_bt, (void *)d_last, (void *)d_dlog, (void *)d_inv_odd, (void *)d_that,
                  (void *)d_ahat})
    cudaFree(x);
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (err != cudaSuccess) {
    set_error("alto_engine_offline", err);
    return -4;
  }
  return 0;
}

int alto_engine_fill_synthetic(void *p) {
  Engine *e = static_cast<Engine *>(p);
  if (!e) {
    set_error("alto_engine_fill_synthetic: NULL engine");
    return -1;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  for (int k = 0; k < e->lanes_made; ++k) {  // batches already enqueued read the database
    if (cudaStreamSynchronize(lane_batch(e, k)->st) != cudaSuccess ||
        cudaStreamSynchronize(lane_batch(e, k)->side) != cudaSuccess) {
      set_error("alto_engine_fill_synthetic", cudaGetLastError());
      return -4;
    }
  }
  const size_t tiles = e->db_mts * e->db_kbs, threads = tiles * 512;
  alto::synthetic_tiles_kernel<<<(unsigned)((threads + 255) / 256), 256>>>(e->d_db, e->db_kbs, tiles, e->rows,
                                                                            e->cols);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaStreamSynchronize(0);
  if (err != cudaSuccess) {
    set_error("alto_engine_fill_synthetic", err);
    return -4;
  }
  return 0;
}

int alto_synthetic_requests_device(uint8_t *d_slots, size_t stride, size_t lead, size_t b, size_t rows, size_t tg_n,
                                   uint64_t seed, uint64_t first_client) {
  if (!d_slots || (lead + 9) % 4 || stride % 4 || stride < lead + 9 + 4 * (2 * tg_n + rows) || b > 65535 ||
      tg_n > 0xffffffffu || (reinterpret_cast<uintptr_t>(d_slots) & 3)) {
    set_error("alto_synthetic_requests_device: bad arguments");
    return -1;
  }
  if (!b) return 0;
  const size_t words = 2 * tg_n + rows;
  const dim3 grid((unsigned)((words + 255) / 256), (unsigned)b);
  alto::synthetic_requests_kernel<<<grid, 256>>>(d_slots, stride, lead, rows, tg_n, seed, first_client);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaStreamSynchronize(0);
  if (err != cudaSuccess) {
    set_error("alto_synthetic_requests_device", err);
    return -4;
  }
  return 0;
}

}  // extern "C"

// ============================================================================================ allocation-free answer
// Some callers cannot allocate device memory at answer time: a server that reserves all of its GPU memory up front
// and must not grow it while serving, code running under a memory budget enforced by a pool that does not belong
// to this library, or a thread that must not take the allocator's locks (cudaMalloc synchronises the device).
// For them alto_answer_device_noalloc answers device-resident frames with its per-batch scratch (statuses, byte
// limbs of queries and keys, scan sums, pack results) in the file-scope array below instead of engine buffers
// grown with cudaMalloc.  The array has a fixed size; every GPU that loads this library holds it until the process
// exits.  All calls share it, so calls whose work overlaps on the GPU (on any engine of the same device) race; the
// array keeps the previous call's contents, and the scan sums, which must start at zero, are cleared by each call.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB per device
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
uint8_t *g_noalloc_addr[kNoAllocMaxDevices] = {};

// The device address of g_noalloc_scratch on device `dev`, which must be current.  In host code the array's name is
// only a host-side stand-in, so the address is looked up with cudaGetSymbolAddress once per device and cached.
bool noalloc_scratch(int dev, uint8_t **addr) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_error("device ordinal outside the allocation-free table");
    return false;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (err != cudaSuccess) {
      set_error("cudaGetSymbolAddress(g_noalloc_scratch)", err);
      return false;
    }
    g_noalloc_addr[dev] = static_cast<uint8_t *>(ptr);
  }
  *addr = g_noalloc_addr[dev];
  return true;
}

struct NoAllocLayout {
  size_t status = 0, qlimb = 0, ylimb = 0, acc = 0, beta = 0, total = 0;
};

NoAllocLayout noalloc_layout(const Engine *e, size_t b) {
  NoAllocLayout l;
  const size_t bp = round_up(b, 4);
  size_t off = 0;
  l.status = off;
  off = round_up(off + b * sizeof(int), 256);
  l.qlimb = off;
  off = round_up(off + 4 * bp * e->chunk * e->nchunks, 256);
  l.ylimb = off;
  off = round_up(off + 4 * bp * e->count, 256);
  l.acc = off;
  off = round_up(off + b * e->cols * sizeof(uint32_t), 256);
  l.beta = off;
  off = round_up(off + b * e->cols * sizeof(uint32_t), 256);
  l.total = off;
  return l;
}

// The launch sequence of the answer path (validate, limb splits, scan, pack, tail) on scratch carved from the
// static array; statuses are copied to the caller's device array.
bool enqueue_noalloc(Engine *e, uint8_t *scratch, const NoAllocLayout &l, const uint8_t *d_slots, size_t stride,
                     size_t b, uint8_t *resp, size_t resp_stride, int *d_status) {
  cudaStream_t st = e->main.st;
  const Plan p = make_plan(e, b);
  const int bp = (int)round_up(b, 4);
  int *status = reinterpret_cast<int *>(scratch + l.status);
  uint8_t *qlimb = scratch + l.qlimb, *ylimb = scratch + l.ylimb;
  uint32_t *acc = reinterpret_cast<uint32_t *>(scratch + l.acc), *beta = reinterpret_cast<uint32_t *>(scratch + l.beta);
  const unsigned split_threads = 256;

  alto::validate_kernel<<<(unsigned)b, 256, 0, st>>>(d_slots, stride, kSlotLead, e->count, e->rows, status);
  ALTO_CK(cudaGetLastError());
  const size_t qwork = (e->rows / 16) * (size_t)bp;
  alto::limb_split_kernel<<<(unsigned)((qwork + split_threads - 1) / split_threads), split_threads, 0, st>>>(
      d_slots, stride, kSlotLead + 9 + 8 * e->count, (int)b, bp, e->rows, e->chunk, qlimb);
  ALTO_CK(cudaGetLastError());
  ALTO_CK(cudaMemsetAsync(acc, 0, b * e->cols * sizeof(uint32_t), st));  // the scan adds into these sums
  const size_t ywork = (e->count / 16) * (size_t)bp;
  alto::limb_split_kernel<<<(unsigned)((ywork + split_threads - 1) / split_threads), split_threads, 0, st>>>(
      d_slots, stride, kSlotLead + 9, (int)b, bp, e->count, e->count, ylimb);
  ALTO_CK(cudaGetLastError());
  CUtensorMap map_q, map_y;
  if (!make_limb_maps(e, p, qlimb, ylimb, bp, &map_q, &map_y)) return false;
  if (!launch_scan(e, p, map_q, acc, b, st, e->main.d_err)) return false;
  if (!launch_pack(e, p, map_y, beta, b, st, e->main.d_err)) return false;
  alto::TailArgs t;
  t.acc = acc;
  t.beta = beta;
  t.status = status;
  t.req = d_slots;
  t.req_stride = stride;
  t.z_off = kSlotLead + 9 + 4 * e->count;
  t.that = e->d_that;
  t.twiddle = e->d_tw;
  t.prefix = e->d_prefix;
  t.resp = resp;
  t.resp_stride = resp_stride;
  t.n = (int)e->n;
  t.tg = (int)e->tg;
  t.outputs = (int)e->outputs;
  t.cols = (int)e->cols;
  t.part_len = (int)e->part_len;
  t.row1_off = (int)e->row1_off;
  t.q1_bits = e->q1_bits;
  t.q1 = (int64_t)e->q1;
  t.o_begin = 0;
  t.o_count = (int)e->outputs;
  ALTO_CK(alto::launch_tail(t, b, st));
  ALTO_CK(cudaMemcpyAsync(d_status, status, b * sizeof(int), cudaMemcpyDeviceToDevice, st));
  e->last_launches = 6;  // validate, two limb splits, scan, pack, tail
  return true;
}

}  // namespace

extern "C" int alto_answer_device_noalloc(void *p, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out,
                                          size_t out_stride, int *d_status) {
  Engine *e = static_cast<Engine *>(p);
  if (!e || !d_req || !d_out || !d_status || req_stride % 16 || req_stride < round_up(kSlotLead + e->want, 16) ||
      out_stride < e->resp_len) {
    set_error("bad arguments");
    return -1;
  }
  e->last_launches = 0;
  if (!b) return 0;
  if (!e->tail_ok) return -3;
  const NoAllocLayout l = noalloc_layout(e, b);
  if (l.total > kNoAllocScratchBytes) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "batch of %zu needs %zu bytes of scratch; the allocation-free entry point has %zu bytes per device",
             b, l.total, kNoAllocScratchBytes);
    set_error(buf);
    return -1;
  }
  if (cudaSetDevice(e->dev) != cudaSuccess) return -4;
  uint8_t *scratch = nullptr;
  if (!noalloc_scratch(e->dev, &scratch)) return -4;
  if (!enqueue_noalloc(e, scratch, l, d_req, req_stride, b, d_out, out_stride, d_status)) return -4;
  // wait and check the engine's device error word (its pinned host mirror already exists)
  if (cudaMemcpyAsync(e->main.h_err, e->main.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, e->main.st) != cudaSuccess ||
      cudaStreamSynchronize(e->main.st) != cudaSuccess) {
    set_error("allocation-free batch failed", cudaGetLastError());
    return -4;
  }
  if (*e->main.h_err) {
    char buf[96];
    snprintf(buf, sizeof buf, "a kernel wait timed out (device error word 0x%x)", *e->main.h_err);
    set_error(buf);
    cudaMemsetAsync(e->main.d_err, 0, sizeof(uint32_t), e->main.st);
    cudaStreamSynchronize(e->main.st);
    return -4;
  }
  return 0;
}

#include "serving.cuh"
