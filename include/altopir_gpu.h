/*
 * altopir_gpu.h -- C ABI of the B200 AltoPIR answer engine (libaltopir_gpu.so).
 *
 * The first block is a drop-in for the reference engine's C ABI: the same symbols, signatures, argument meaning,
 * return codes and ownership rules that the reference's Rust wrapper binds (src/engine.rs:4-20), so a build that
 * links this library instead of compiling src/amx_kernels.cpp needs no change to the Rust side.  The answer path
 * runs on the current CUDA device (one engine per device); there is no CPU fallback: without a usable GPU,
 * sw_amx_init() and alto_engine_new() fail.
 *
 * The second block holds extensions with no counterpart in the reference.
 */
#ifndef ALTOPIR_GPU_H
#define ALTOPIR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ================================================================ reference C ABI (src/engine.rs:4-20) */

/* Replaces sw_amx_init (src/amx_kernels.cpp:151), which asks the kernel for AMX tile state.  Here it creates the
 * CUDA context on the current device.  Returns 0 on success, -1 when no usable CUDA device is present. */
int sw_amx_init(void);

/* Replace sw_alloc_zeroed / sw_alloc / sw_free (src/amx_kernels.cpp:97-113): anonymous host mappings aligned to
 * 2 MiB (zero-filled for sw_alloc_zeroed); sw_free(NULL) is a no-op.  Used by the caller for the tiled database and
 * the packing matrix, which alto_engine_new copies into device memory. */
void *sw_alloc_zeroed(size_t bytes);
void *sw_alloc(size_t bytes);
void sw_free(void *p);

/* Replaces sw_tile_db (src/amx_kernels.cpp:138-149).  Copies the k x m column-order database db[col * ld + r]
 * into dst as a compact column-order matrix dst[col * k + r] (k records per column, no padding).  The engine does
 * not read this copy: alto_engine_new builds its own tiles of 128 columns x 128 records in device memory from
 * db_col.  Kept so that callers written for the reference link unchanged.  Uses `threads` host threads. */
void sw_tile_db(uint8_t *dst, const uint8_t *db, size_t ld, size_t k, size_t m, int threads);

/* Replaces sw_pack_build (src/amx_kernels.cpp:311-341).  Folds the InspiRING automorphisms into the dense packing
 * matrix U ((rho * n) columns x (tg * n) key words, values mod q) exactly as the reference does and stores it in
 * this engine's layout: ub[(col * 4 + j) * (tg * n) + k] = byte j of U[col][k] (4 * tg * n * rho * n bytes, the
 * same size as the reference's buffer).  q must be 4294955009. */
void sw_pack_build(int8_t *ub, const uint64_t *const *bold_t, const uint64_t *const *bold_t_bar,
                   const uint32_t *tables, const uint32_t *gen_pows, size_t num_iter, size_t tg, size_t n, size_t rho,
                   uint64_t q, int threads);

/* Replaces alto_engine_new (src/amx_kernels.cpp:546-560).  Same configuration checks as the reference (NULL for
 * q != 4294955009, n == 0, n > 4096, n % 16, cols % n, rows % 64, cols % 32, threads <= 0, (tg * n) % 128, or a
 * NULL pointer), plus two limits of this engine: 1 <= tg and tg * n <= 32768 (keeps every int32 limb partial sum
 * of the packing product exact).  The database is read from db_col (db_col[col * ld + r], r < rows, col < cols);
 * db_tiled must be non-NULL but is not read.  The database, the packing matrix `ub` (layout of sw_pack_build),
 * the row-0 prefixes (cols / n buffers of part_len bytes), bold_t_hat (`that`, cols / n arrays of tg * n words,
 * reduced mod q) and the low 32 bits of inv_table[0..n) are copied into device memory, so the caller may free all
 * of them once this returns.  `ub` must have been written by this library's sw_pack_build (or alto_pack_encode):
 * a buffer in the reference's AMX layout (sw_ubt, -128-biased tile order), for example one cached from a build of
 * src/amx_kernels.cpp, has the same size but other bytes, and the engine would answer with wrong responses.
 * Returns NULL when the configuration is unsupported or the device lacks memory (alto_last_error() says which). */
void *alto_engine_new(const uint8_t *db_col, const uint8_t *db_tiled, size_t ld, size_t rows, size_t cols,
                      const int8_t *ub, size_t n, size_t tg, const uint8_t *const *prefix, size_t part_len,
                      size_t row1_off, uint64_t q1, int q1_bits, const uint64_t *const *that,
                      const uint64_t *inv_table, uint64_t q, int threads);

/* Replaces alto_engine_free (src/amx_kernels.cpp:561).  NULL is a no-op. */
void alto_engine_free(void *engine);

/* Replace alto_request_len / alto_response_len (src/amx_kernels.cpp:562-563):
 * 9 + 4 * (2 * tg * n + rows) and (cols / n) * part_len. */
size_t alto_request_len(const void *engine);
size_t alto_response_len(const void *engine);

/* Replaces alto_answer (src/amx_kernels.cpp:564-615).  Answers a batch of b request frames in host memory:
 *   status[c] = 1 for a NULL frame or a length other than alto_request_len, 2 for a flag byte != 0 or a key count
 *   != tg * n, 3 for a y or z key word >= q, else 0 (query words are not range-checked);
 *   out[c] (alto_response_len bytes) is written for status 0 only, other output buffers stay untouched.
 * method must be 0 (the reference's AMX code) or 2 (VNNI); both run the same GPU path.  The header and y keys upload
 * first and the pack runs while the z keys and query words upload; the scan and tail then run in column groups
 * whose responses download while the next group computes.  When stage_ms is not NULL it receives device times in
 * ms: [0] header and y-key upload, [1] validation, query split, scans and tails, [2] key split and pack, [3] the
 * last group's download.
 * Returns the number of valid requests, -1 for bad arguments, -3 when the tail parameters are invalid (n not a
 * power of two >= 16, q1 >= 2^21, q1_bits > 24, n % 8, or row 1 not fitting in part_len), -4 when the device
 * failed (CUDA error or a kernel wait that timed out; alto_last_error() has the reason).  Calls on one engine must
 * not overlap; different engines may be used from different threads.  Pinned host buffers make the copies
 * asynchronous DMA; pageable buffers work but copy through a staging buffer. */
int alto_answer(void *engine, const uint8_t *const *req, const size_t *len, size_t b, uint8_t *const *out,
                int *status, int method, double *stage_ms);

/* ================================================================ extensions (no counterpart in the reference) */

/* Text of the last error recorded by this library on the calling thread ("" if none). */
const char *alto_last_error(void);

/* alto_answer for frames that are already resident in device memory: frame c (the full frame, header included)
 * starts at d_req + c * req_stride + 7, which puts its key words on a 16-byte boundary; req_stride is a multiple of
 * 16 and at least 7 + alto_request_len rounded up to 16.  The header is checked on the device.  Responses go to
 * d_out + c * out_stride (device memory, out_stride >= alto_response_len), statuses to the host array status[b].
 * Returns what alto_answer returns. */
int alto_answer_device(void *engine, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out,
                       size_t out_stride, int *status, double *stage_ms);

/* Column shards (a database split by output ranges over several GPUs, one engine per GPU over its columns):
 * alto_answer_device for an engine that holds outputs [part_offset, part_offset + its outputs) of the full response,
 * writing every valid frame's parts into each buffer d_outs[k], at d_outs[k] + c * out_stride +
 * (part_offset + o) * part_len.  The buffers may be this GPU's or other GPUs' (mapped with alto_ipc_import): once
 * every shard has answered the same frames, each buffer holds the full responses -- the shards' all-gather is done
 * by the tail kernel's own stores, over NVLink between GPUs, with no separate collective.  1 <= n_outs <= 64,
 * out_stride >= (part_offset + outputs) * part_len; statuses to the host array status[b].  Returns the number of
 * valid frames, or -1/-3/-4 as alto_answer_device.  The caller orders the shards' calls with the readers of the
 * buffers (a barrier between ranks after every call).
 * alto_ipc_export writes the 64-byte CUDA IPC handle of the device allocation that contains d_ptr into handle[64]
 * and d_ptr's offset inside it into *offset (0, -1, -4); alto_ipc_import maps another process's handle into this
 * one and returns the base of the mapping (NULL on failure) -- the exporter's pointer is that base plus the offset;
 * alto_ipc_release unmaps a base returned by alto_ipc_import. */
int alto_answer_device_parts(void *engine, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *const *d_outs,
                             size_t n_outs, size_t out_stride, size_t part_offset, int *status);
int alto_ipc_export(const void *d_ptr, uint8_t *handle, size_t *offset);
void *alto_ipc_import(const uint8_t *handle);
int alto_ipc_release(void *d_ptr);

/* Count of kernel launches issued by the most recent batch of this engine. */
int alto_last_launches(const void *engine);

/* Asynchronous form of alto_answer_device: enqueues the whole batch on the engine's stream and returns at once
 * (0, or -1/-3/-4 as alto_answer).  Statuses are written to the device array d_status[b] when it is not NULL.
 * Completion and kernel wait failures are reported by alto_engine_sync. */
int alto_enqueue_device(void *engine, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out,
                        size_t out_stride, int *d_status);

/* Waits for every batch enqueued on this engine; returns 0, or -4 when a kernel wait timed out since the last
 * check (the device error word is cleared). */
int alto_engine_sync(void *engine);

/* Batch lanes of alto_enqueue_device (default 1).  With 2..4 lanes consecutive calls rotate through that many batch
 * contexts -- the engine's own, then contexts with streams and scratch of their own, made on first use -- so that
 * a batch overlaps the previous one on the device (its tail, and its GEMMs' last partial round of units).  Batches
 * in flight at once must not write the same outputs or statuses.  alto_engine_set_lanes waits for the engine first
 * and returns 0, -1 (lanes outside 1..4) or -4.  alto_engine_sync waits for every lane.  alto_engine_fence makes
 * every lane's stream wait for the work enqueued so far on every other lane, without a host wait, so that work
 * ordered on alto_engine_stream after a fence follows every lane's batches (and batches enqueued after a fence
 * follow work put on that stream before it); 0, -1 or -4. */
int alto_engine_set_lanes(void *engine, int lanes);
int alto_engine_fence(void *engine);

/* The cudaStream_t the engine launches its kernels on (for events and stream ordering in the caller). */
void *alto_engine_stream(void *engine);

/* Tuning table of this engine: n entries of 5 ints {b_max, pair, wide, bn_cap, units_per_pair}; the first entry
 * (in b_max order) with b_max >= the batch size chooses the GEMM plan: pair = 1 CTA-pair kernels, 0 single-CTA
 * kernels; wide = 1 scan units of 512 limb columns, 0 never; bn_cap = largest limb-column tile (32..256);
 * units_per_pair = scan split target; -1 or 0 keeps the built-in choice.  Every plan computes identical results.
 * alto_engine_new loads the committed table from $ALTO_TUNING or tuning.txt next to this library (lines
 * "rows_max b_max pair wide bn_cap units_per_pair", the rows of the smallest rows_max >= the engine's records).
 * n = 0 clears the table.  Returns 0, -1 for bad arguments, -4 on a device failure. */
int alto_engine_set_tuning(void *engine, const int32_t *entries, size_t n);

/* Replay the device-side launch sequence of a batch (validate .. tail) as a CUDA graph, captured on the first batch
 * of each size and buffer set (on = 1), or launch kernels directly (on = 0, the default).  Applies to
 * alto_answer_device, alto_enqueue_device and serving loops created afterwards; alto_answer keeps direct launches
 * because its pack overlaps the query upload on another stream.  Graph replays record no timing marks for
 * alto_kernel_times.  Returns 0, or -4 on a device failure. */
int alto_engine_set_graphs(void *engine, int on);

/* Device time in ms summed over the batches since the last reset, measured with CUDA events on the engine's
 * stream: ms[0] validate, ms[1] limb split + accumulator zeroing, ms[2] scan GEMM, ms[3] pack GEMM, ms[4] tail;
 * *batches receives the number of batches.  Synchronises the engine.  Returns 0, or -4 on a device failure. */
int alto_kernel_times(void *engine, double *ms, long long *batches, int reset);

/* No counterpart in the reference.  alto_answer_device without any device allocation, for callers that cannot
 * call cudaMalloc while they serve: a server that reserves its GPU memory once at start-up and must not grow it,
 * code that runs under a memory budget kept by an allocator it does not own, or a thread that must not stall on
 * cudaMalloc's device-wide synchronisation.  Frames and outputs are laid out as for alto_answer_device; statuses go
 * to the device array d_status[b].  The per-batch scratch (statuses, byte limbs, scan sums, pack results) lives in
 * a fixed 16 MiB array inside this library, which every GPU that loads the library holds until the process exits;
 * a batch whose scratch would exceed it is rejected with -1 and a message in alto_last_error().  A batch of b frames
 * needs, with every term rounded up to 256 bytes and b4 = b rounded up to 4, R = rows (rows rounded up to 32768 above
 * 32768 records), cols = record bytes, K = tg * n:  4 b + 4 b4 R + 4 b4 K + 2 * 4 b cols <= 16 MiB.  At 32768 records
 * of 32 KB (K = 8192) that allows 38 frames.  The first call on a device looks up the array's device address (set-up done
 * once per device), so that first call should come before any stream capture.  All calls share the array: calls
 * whose work overlaps on the GPU race, even on different engines of the same device.  Returns 0 once the batch has
 * completed, -1, -3 or -4 as alto_answer. */
int alto_answer_device_noalloc(void *engine, const uint8_t *d_req, size_t req_stride, size_t b, uint8_t *d_out,
                               size_t out_stride, int *d_status);

/* Serving loop with continuous batching over one engine (the engine loop of src/bin/altopir.rs:403-510 without the
 * TCP front end).  alto_server_submit copies a frame into a pinned pool of queue_cap frames (outside the loop's lock);
 * a batcher thread takes whatever is queued, up to max_batch, as soon as one of `slots` device batch contexts (1..8)
 * is free -- it never holds a request back to fill a batch, and frames that arrive while every context is busy join
 * the next batch -- and answers it on that context's stream, so up to `slots` batches upload and compute at once.
 * Contexts beyond the first two take a batch only while at least max_batch / 2 frames are queued (environment
 * ALTO_SERVE_DEEP: frames, 0 = always): a third concurrent full-database scan pays only at saturation.
 * Per-client state in HBM: the pack product beta = y U of a client's packing keys y depends on nothing else, so the
 * loop keeps it in a resident table of key_bytes / (cols * 4) rows.  A frame whose y keys equal, byte for byte, those
 * of a resident client skips the pack GEMM and gathers its row; a new client is admitted to a free row, or to the
 * least recently used row that no batch in flight uses, and its batch stores its beta there (valid frames only).
 * When no row can be had the frame is answered all the same, with its pack computed and not kept.  Responses are
 * the same bytes either way.
 *   alto_server_new_keyed  returns NULL for bad arguments (1 <= slots <= 8, queue_cap <= 2^30) or when the device
 *                          or pinned host memory is short; key_bytes = 0 disables the table, SIZE_MAX picks the
 *                          default (a quarter of the free device memory, at most 8 GiB).
 *   alto_server_new        alto_server_new_keyed with the default table.
 *   alto_server_submit     copies the frame and returns a ticket >= 0, -9 when the pool is full (the reference
 *                          server's BUSY status 9), -1 for bad arguments.  A frame of the wrong length gets a ticket
 *                          that completes at once with status 1.
 *   alto_server_wait       waits up to timeout_ms for a ticket; returns its status (0..3 as alto_answer, with the
 *                          response copied to out for 0), -4 on a device failure, -5 on timeout (the ticket stays
 *                          valid), -1 for an unknown ticket; *latency_ms (if not NULL) receives the time from
 *                          submit to completion measured by the loop.  A completed ticket is released by this call.
 *   alto_server_stats      out[0..15] = answered, rejected (status 1..3), busy, failed, batches, mean batch size,
 *                          latency p50, p99, p99.9 and max in ms (submit to completion), frames still queued,
 *                          frames answered from resident rows, clients admitted, rows evicted, frames answered
 *                          without a row (table full of rows in use), table rows.
 *   alto_server_log        the per-batch log (src/bin/altopir.rs:472-510, --log): up to max_rows of the most recent
 *                          batches, oldest first, 10 doubles each: dispatch and completion time (s, the loop's
 *                          clock), frames taken, frames on the device, frames that ran the pack, frames answered from
 *                          resident rows, device ms of the upload, of the pack and row gather, of the scan, tails
 *                          and download, and in total.  Returns the number of rows written, -1 for bad arguments.
 *   alto_server_free       answers everything queued, then stops the threads and frees the contexts and the table.
 * alto_server_new_loopback builds the same loop without an engine: batches are answered on the host after
 * service_us microseconds by a deterministic function of the frame, to test queueing and batching without a
 * device.  None of these has a counterpart in the reference's C ABI.
 * The loop answers in batch contexts of its own, so while it runs, one other thread may still call alto_answer,
 * alto_answer_device or alto_enqueue_device on the same engine; alto_engine_set_tuning, alto_engine_set_graphs,
 * the ingest calls and alto_engine_free must wait until alto_server_free has returned. */
void *alto_server_new(void *engine, size_t max_batch, size_t queue_cap, int slots);
void *alto_server_new_keyed(void *engine, size_t max_batch, size_t queue_cap, int slots, size_t key_bytes);
void *alto_server_new_loopback(size_t request_len, size_t response_len, size_t max_batch, size_t queue_cap, int slots,
                               double service_us);
long long alto_server_submit(void *server, const uint8_t *frame, size_t len);
int alto_server_wait(void *server, long long ticket, uint8_t *out, size_t out_len, int timeout_ms,
                     double *latency_ms);
int alto_server_stats(void *server, double *out, size_t n);
int alto_server_log(void *server, double *out, size_t max_rows);
void alto_server_free(void *server);

/* A database too large to hold in host memory in column order, or stored on disk record by record, is loaded
 * straight into the engine's device tiles instead of through alto_engine_new's db_col (the counterpart of the
 * reference server's streaming reader, src/server.rs:380-500, which transposes a record-major file into the
 * column-order buffer).
 * alto_engine_new_empty: alto_engine_new without the database (same checks, same copies of the other state); the
 *   database starts as zeros, as the reference's padding records are.
 * alto_engine_load_records: copies records [first, first + count) -- record i at records + (i - first) * pitch,
 *   cols bytes each, pitch >= cols -- into the engine's database, transposing them on the device.  Any run of
 *   records, in any order; records not loaded keep their bytes.  Waits for the engine's enqueued batches first;
 *   must not overlap another call on the same engine.  0, -1 for bad arguments (first + count > rows, ...), -4 for
 *   a device failure.
 * alto_engine_load_file: loads the first num_real_rows records of a flat record-major file (num_real_rows records
 *   of cols bytes each, the reference's on-disk database) in 64 MB reads; the rest stay zero.  0, -1 for bad
 *   arguments, -2 when the file cannot be opened or is short, -4 for a device failure. */
void *alto_engine_new_empty(size_t rows, size_t cols, const int8_t *ub, size_t n, size_t tg,
                            const uint8_t *const *prefix, size_t part_len, size_t row1_off, uint64_t q1, int q1_bits,
                            const uint64_t *const *that, const uint64_t *inv_table, uint64_t q, int threads);
int alto_engine_load_records(void *engine, const uint8_t *records, size_t pitch, size_t first, size_t count);
int alto_engine_load_file(void *engine, const char *path, size_t num_real_rows);

/* Deterministic synthetic inputs (test and benchmark data; not part of the answer path).
 * alto_synthetic_db_col: db[(col - col0) * ld + r] = byte col of the reference's synthetic record r
 *   (src/service.rs:43-62, splitmix64 seed 0x416c746f504952), for r < rows and ncols columns from col0.
 * alto_synthetic_db_col_device: the same into device memory (rows % 4 == 0, ld % 4 == 0); 0 on success.
 * alto_fill_uniform_u32: dst[i] = a uniform value in [0, bound) drawn from splitmix64 counter `seed` + i.
 * alto_fill_uniform_u64: the same with 64-bit outputs (bound <= 2^32).
 * alto_fill_bytes: dst[i] = uniform bytes from the same counter construction.
 * alto_synthetic_request: a well-formed frame of alto_request_len bytes for a seeded client: y, z uniform in
 *   [0, 4294955009), query words uniform over u32 (the distribution of rounded RLWE query words).
 * alto_pack_encode: packing-matrix values U[col * K + k] (< 2^32) into the layout of sw_pack_build.
 * alto_engine_fill_synthetic: fills the whole database of an engine with the synthetic records on the device (the
 *   bytes alto_synthetic_db_col gives), so large databases need no host copy; waits for the engine's batches first.
 *   0, -1 (NULL engine) or -4.
 * alto_synthetic_requests_device: b frames of alto_synthetic_request (clients first_client ..), frame c written to
 *   d_slots + c * stride + lead in device memory; needs (lead + 9) % 4 == 0, stride % 4 == 0, d_slots 4-byte aligned,
 *   stride >= lead + 9 + 4 * (2 * tg_n + rows), b <= 65535.  0, -1 (bad arguments) or -4. */
void alto_synthetic_db_col(uint8_t *db, size_t ld, size_t rows, size_t col0, size_t ncols, int threads);
int alto_synthetic_db_col_device(uint8_t *d_db, size_t ld, size_t rows, size_t col0, size_t ncols);
int alto_engine_fill_synthetic(void *engine);
int alto_synthetic_requests_device(uint8_t *d_slots, size_t stride, size_t lead, size_t b, size_t rows, size_t tg_n,
                                   uint64_t seed, uint64_t first_client);
void alto_fill_uniform_u32(uint32_t *dst, size_t count, uint64_t bound, uint64_t seed, int threads);
void alto_fill_uniform_u64(uint64_t *dst, size_t count, uint64_t bound, uint64_t seed, int threads);
void alto_fill_bytes(uint8_t *dst, size_t count, uint64_t seed, int threads);
void alto_synthetic_request(uint8_t *frame, size_t rows, size_t tg_n, uint64_t seed, uint64_t client);
void alto_pack_encode(int8_t *ub, const uint32_t *U, size_t cols, size_t K, int threads);

/* Offline hint on the device (row (f)1 of the offline set-up): the ring multiply of YServer::answer_hint_ring /
 * multiply_with_db_ring (src/server.rs:656-768) over this engine's resident database, once per database.  query
 * holds rows / n raw query polynomials of n coefficients (u64, reduced mod q here) -- the pseudorandom query of
 * generate_pseudorandom_query (src/server.rs:714-738) before its preprocessing, which this call applies: polynomial
 * r is negated and reversed as util.rs negacyclic_perm does (shift 0) and multiplied, modulo X^n + 1 and q, by the
 * polynomial of records [r n, (r + 1) n) of each column.  out[z * cols + col] (n * cols u64 values < q, the layout
 * answer_hint_ring returns) = coefficient z of the sum over r, passed once more through negacyclic_perm when
 * perm_out != 0 (the reference does so for seed 0 outside SimplePIR mode, src/server.rs:699-705).  Needs rows a
 * multiple of n and n a power of two <= 2048 (2n must divide q - 1).  Allocates its device scratch (about
 * 8 n cols bytes) for the call.  0, -1 for bad arguments or an unsupported n, -4 for a device failure. */
int alto_hint_ring(void *engine, const uint64_t *query, uint64_t *out, int perm_out);

/* The scheme's offline set-up on the device, for an engine whose database is resident (Prepared::new,
 * src/service.rs:127-157, over YServer::perform_offline_precomputation_simplepir, src/server.rs:947-1021): the
 * hint's ring multiply (as alto_hint_ring, kept in NTT form), the InspiRING precomputation of every output
 * (full_packing_with_preprocessing_offline, src/packing.rs:2260-2359), the packing matrix (sw_pack_build), bold_t_hat
 * and the row-0 prefixes (switch_prefix_row0), written into the engine in place of the state it was created with,
 * and the engine's inverse-NTT table set to the ring's.  After it the engine answers requests whose responses
 * decrypt under the client's secret.
 *   query: (records / n) x n raw polynomials, row 0 of the query's RLWE ciphertexts (-a_i mod q), as alto_hint_ring;
 *   w_mask, v_mask: tg x n NTT-form masks of the rotation and conjugation keys (OfflinePackingKeys::init_full).
 * Ring: Z_q[X]/(X^n + 1), NTT slot s = evaluation at psi^(2 brv(s) + 1), psi the smallest primitive 2n-th root of
 * unity; gadget digits of floor(32 / tg) + 1 bits.  Optional host outputs (NULL to skip), all u32 in [0, q):
 * bold_t and bold_t_bar, outputs x (n/2 - 1) x tg x n each; that (bold_t_hat), outputs x tg x n; a_hat, outputs x n.
 * ms (optional) receives the device time of the set-up.  Waits for the engine's batches in flight (a serving loop
 * must not run on the engine meanwhile); allocates about 4 n cols + 4 tg n cols + 12 records bytes of device scratch
 * for the call (1.3 GB at 32 KB records, n = 2048, tg = 4).  0, -1 for bad arguments or an unsupported
 * configuration (the engine is untouched), -4 for a device failure (the engine's packing state is then undefined:
 * call again or free it). */
int alto_engine_offline(void *engine, const uint64_t *query, const uint64_t *w_mask, const uint64_t *v_mask,
                        uint32_t *bold_t, uint32_t *bold_t_bar, uint32_t *that, uint32_t *a_hat, double *ms);

/* Self-check of the engine's modulus-switch arithmetic on the host: sum over v in [v0, v1) of rescale(v) * (2v + 1)
 * modulo 2^64, where rescale is the exact integer centred rescale Q -> q1 that the tail kernel runs. */
uint64_t alto_rescale_digest(uint64_t q1, uint64_t v0, uint64_t v1, int threads);

#ifdef __cplusplus
}
#endif

#endif /* ALTOPIR_GPU_H */
