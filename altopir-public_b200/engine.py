"""Engine wrapper mirroring the reference's Rust binding (src/engine.rs): Method, MappedBytes-style host buffers,
TiledDb, build_packing_matrix and Engine, all calling the C ABI of libaltopir_gpu.so."""
import ctypes
import enum
import os

import numpy as np

from . import lib, last_error
from .service import Q


class Method(enum.IntEnum):
    """Engine.rs Method codes (src/engine.rs:22-50).  The GPU engine accepts both and runs the same path."""
    AMX = 0
    VNNI = 2


def init():
    """engine::init_amx (src/engine.rs:66-69): here, create the CUDA context; raises without a usable device."""
    r = lib().sw_amx_init()
    if r != 0:
        raise RuntimeError(f"no usable CUDA device: {last_error()}")


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _ptrs(arrays):
    return (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


class TiledDb:
    """TiledDb::new (src/engine.rs:111-118): sw_tile_db into a buffer of rows * cols bytes."""

    def __init__(self, db_col, ld, rows, cols, threads=1):
        assert rows % 64 == 0 and cols % 32 == 0 and db_col.size >= (cols - 1) * ld + rows
        self.rows, self.cols = rows, cols
        self.buf = np.empty(rows * cols, dtype=np.uint8)
        lib().sw_tile_db(_p(self.buf), _p(db_col), ld, rows, cols, threads)


def build_packing_matrix(ub, bold_t, bold_t_bar, tables, gen_pows, num_iter, tg, n, qmod=Q, threads=1):
    """build_packing_matrix (src/engine.rs:127-138) over sw_pack_build."""
    rho = len(bold_t)
    assert ub.size == 4 * tg * n * rho * n and len(bold_t_bar) == rho
    assert tables.size == n * n and gen_pows.size >= num_iter
    for s in list(bold_t) + list(bold_t_bar):
        assert s.size >= num_iter * tg * n and s.dtype == np.uint64
    tables = np.ascontiguousarray(tables, dtype=np.uint32)     # held here: ctypes keeps only the address
    gen_pows = np.ascontiguousarray(gen_pows, dtype=np.uint32)
    lib().sw_pack_build(_p(ub), _ptrs(bold_t), _ptrs(bold_t_bar), _p(tables), _p(gen_pows), num_iter, tg, n, rho,
                        qmod, threads)


class EngineError(RuntimeError):
    pass


class Engine:
    """Engine<'a> (src/engine.rs:140-195).  The device copies every input at construction, so the arrays passed
    here may be dropped afterwards."""

    def __init__(self, db_col, tiled, ld, ub, n, tg, prefixes, row1_off, q1, q1_bits, that, inv_table, q=Q,
                 threads=1):
        rows, cols = tiled.rows, tiled.cols
        assert db_col.size >= (cols - 1) * ld + rows and ub.size == 4 * tg * n * cols and len(prefixes) == cols // n
        assert len(that) == cols // n and all(t.size >= tg * n for t in that) and inv_table.size >= n
        part_len = prefixes[0].size
        assert all(p.size == part_len for p in prefixes)
        # arrays converted here are held in locals until the call returns: ctypes keeps only their addresses
        pre = [np.ascontiguousarray(p, dtype=np.uint8) for p in prefixes]
        that64 = [np.ascontiguousarray(t, dtype=np.uint64) for t in that]
        inv = np.ascontiguousarray(inv_table, dtype=np.uint64)
        db_col = np.ascontiguousarray(db_col)
        ub = np.ascontiguousarray(ub)
        self.rows, self.cols = rows, cols
        self.ptr = lib().alto_engine_new(_p(db_col), _p(tiled.buf), ld, rows, cols, _p(ub), n, tg, _ptrs(pre),
                                         part_len, row1_off, q1, q1_bits, _ptrs(that64), _p(inv), q, threads)
        if not self.ptr:
            raise EngineError(f"unsupported engine configuration: {last_error()}")

    @classmethod
    def empty(cls, rows, cols, ub, n, tg, prefixes, row1_off, q1, q1_bits, that, inv_table, q=Q, threads=1):
        """alto_engine_new_empty: the engine without its database, which starts as zeros and is filled with
        load_records or load_file (the reference server's streaming reader, src/server.rs:380-500)."""
        assert ub.size == 4 * tg * n * cols and len(prefixes) == cols // n and len(that) == cols // n
        self = cls.__new__(cls)
        self.rows, self.cols = rows, cols
        pre = [np.ascontiguousarray(p, dtype=np.uint8) for p in prefixes]
        that64 = [np.ascontiguousarray(t, dtype=np.uint64) for t in that]
        inv = np.ascontiguousarray(inv_table, dtype=np.uint64)
        ub = np.ascontiguousarray(ub)
        self.ptr = lib().alto_engine_new_empty(rows, cols, _p(ub), n, tg, _ptrs(pre), pre[0].size, row1_off, q1,
                                               q1_bits, _ptrs(that64), _p(inv), q, threads)
        if not self.ptr:
            raise EngineError(f"unsupported engine configuration: {last_error()}")
        return self

    def load_records(self, records, first):
        """alto_engine_load_records: records is a (count, cols) uint8 array of consecutive records from `first`."""
        records = np.ascontiguousarray(records, dtype=np.uint8)
        r = lib().alto_engine_load_records(self.ptr, _p(records), records.shape[1], first, records.shape[0])
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")

    def load_file(self, path, num_real_rows):
        """alto_engine_load_file: the first num_real_rows records of a flat record-major database file."""
        r = lib().alto_engine_load_file(self.ptr, os.fsencode(path), num_real_rows)
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")

    def hint_ring(self, query, perm_out=False):
        """alto_hint_ring: the offline hint's ring multiply over the resident database (YServer::answer_hint_ring,
        src/server.rs:656-768).  query: (rows / n, n) raw query polynomials; returns the (n, cols) uint64 hint."""
        q = np.ascontiguousarray(query, dtype=np.uint64)
        n = q.shape[1]
        assert q.shape[0] * n == self.rows, "one raw polynomial per n records"
        out = np.empty((n, self.cols), dtype=np.uint64)
        r = lib().alto_hint_ring(self.ptr, _p(q), _p(out), int(perm_out))
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")
        return out

    def offline(self, query, w_mask, v_mask, want=False):
        """alto_engine_offline: the scheme's offline set-up on the device (Prepared::new, src/service.rs:127-157) --
        hint, InspiRING precomputation, packing matrix, bold_t_hat, row-0 prefixes -- written into this engine.
        query: (rows / n, n) row-0 query polynomials (-a_i mod Q); w_mask, v_mask: (tg, n) NTT-form masks.
        Returns the device time in ms, and with want=True also a dict of the per-output bold_t, bold_t_bar, that
        (bold_t_hat) and a_hat as uint32 arrays."""
        q = np.ascontiguousarray(query, dtype=np.uint64)
        w = np.ascontiguousarray(w_mask, dtype=np.uint64)
        v = np.ascontiguousarray(v_mask, dtype=np.uint64)
        n = q.shape[1]
        assert q.size == self.rows and w.size == v.size and w.size % n == 0
        tg, outputs = w.size // n, self.cols // n
        out = {}
        if want:
            per = (n // 2 - 1) * tg * n
            out = {"bold_t": np.empty((outputs, per), dtype=np.uint32),
                   "bold_t_bar": np.empty((outputs, per), dtype=np.uint32),
                   "that": np.empty((outputs, tg * n), dtype=np.uint32),
                   "a_hat": np.empty((outputs, n), dtype=np.uint32)}
        ms = ctypes.c_double(0.0)
        ptr = (lambda k: _p(out[k]) if want else None)
        r = lib().alto_engine_offline(self.ptr, _p(q), _p(w), _p(v), ptr("bold_t"), ptr("bold_t_bar"), ptr("that"),
                                      ptr("a_hat"), ctypes.byref(ms))
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")
        return (ms.value, out) if want else ms.value

    def fill_synthetic(self):
        """alto_engine_fill_synthetic: the whole database becomes the synthetic records, generated on the device."""
        r = lib().alto_engine_fill_synthetic(self.ptr)
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")

    @staticmethod
    def from_state(st, threads=1, tile=True):
        """Prepared::engine (src/service.rs:159-170) for a service.SyntheticState.  With tile=False no tiled copy
        is made (this engine reads the column-order database and never the tiled one), which halves the host
        memory of very large databases."""
        p = st.p
        if st.db_col is None:  # a state without a host database: the synthetic records are generated on the device
            e = Engine.empty(p.rows, p.record_bytes, st.ub, p.n, p.tg, st.prefixes, p.row1_off, 1 << p.q1_bits,
                             p.q1_bits, st.that, st.inv_table, Q, threads)
            e.fill_synthetic()
            return e
        if tile:
            tiled = TiledDb(st.db_col, st.db_col.shape[1], p.rows, p.record_bytes, threads)
        else:
            tiled = TiledDb.__new__(TiledDb)
            tiled.rows, tiled.cols, tiled.buf = p.rows, p.record_bytes, np.zeros(64, dtype=np.uint8)
        return Engine(st.db_col, tiled, st.db_col.shape[1], st.ub, p.n, p.tg, st.prefixes, p.row1_off, 1 << p.q1_bits,
                      p.q1_bits, st.that, st.inv_table, Q, threads)

    def request_len(self):
        return lib().alto_request_len(self.ptr)

    def response_len(self):
        return lib().alto_response_len(self.ptr)

    def answer(self, reqs, out, status, method=Method.AMX):
        """Engine::answer (src/engine.rs:174-188).  reqs: a sequence of uint8 arrays (or a 2-D array, one frame per
        row); out: a (b, response_len) uint8 array or a sequence of uint8 arrays; status: int32 array of b.
        Returns (answered, stage_ms[4]); raises EngineError on a negative return."""
        b = len(reqs)
        frames = [reqs[i] for i in range(b)]
        outs = [out[i] for i in range(b)]
        assert len(outs) == b and status.size == b and status.dtype == np.int32
        rl = self.response_len()
        assert all(o.size == rl and o.dtype == np.uint8 and o.flags.c_contiguous for o in outs)
        req_p = (ctypes.c_void_p * b)(*[f.ctypes.data if f is not None else None for f in frames])
        lens = (ctypes.c_size_t * b)(*[f.size if f is not None else 0 for f in frames])
        out_p = (ctypes.c_void_p * b)(*[o.ctypes.data for o in outs])
        stage = (ctypes.c_double * 4)()
        r = lib().alto_answer(self.ptr, req_p, lens, b, out_p,
                              status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(method), stage)
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")
        return r, list(stage)

    def answer_raw(self, req_ptrs, lens, b, out_ptrs, status, method=Method.AMX, stage=None):
        """alto_answer on prepared ctypes arrays (no per-call Python list building); returns the raw code."""
        return lib().alto_answer(self.ptr, req_ptrs, lens, b, out_ptrs,
                                 status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(method), stage)

    def answer_device(self, d_req, req_stride, b, d_out, out_stride, status, stage=None):
        """alto_answer_device: frames already in device memory (frame c at d_req + c * req_stride + 7)."""
        return lib().alto_answer_device(self.ptr, ctypes.c_void_p(d_req), req_stride, b, ctypes.c_void_p(d_out),
                                        out_stride, status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), stage)

    def answer_device_parts(self, d_req, req_stride, b, d_outs, out_stride, part_offset, status):
        """alto_answer_device_parts: this shard's response parts written into every buffer of d_outs (device
        pointers, local or mapped from other GPUs) at column offset part_offset * part_len."""
        outs = (ctypes.c_void_p * len(d_outs))(*d_outs)
        return lib().alto_answer_device_parts(self.ptr, ctypes.c_void_p(d_req), req_stride, b, outs, len(d_outs),
                                              out_stride, part_offset,
                                              status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    def enqueue_device(self, d_req, req_stride, b, d_out, out_stride, d_status=None):
        """alto_enqueue_device: enqueue without waiting; check completion with sync()."""
        r = lib().alto_enqueue_device(self.ptr, ctypes.c_void_p(d_req), req_stride, b, ctypes.c_void_p(d_out),
                                      out_stride, ctypes.c_void_p(d_status) if d_status else None)
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")

    def sync(self):
        r = lib().alto_engine_sync(self.ptr)
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")

    def stream(self):
        """The engine's cudaStream_t as an integer handle (torch.cuda.ExternalStream accepts it)."""
        return lib().alto_engine_stream(self.ptr)

    def kernel_times(self, reset=True):
        """(ms summed per kernel [validate, split, scan, pack, tail], batches) since the last reset."""
        ms = (ctypes.c_double * 5)()
        nb = ctypes.c_longlong(0)
        r = lib().alto_kernel_times(self.ptr, ms, ctypes.byref(nb), int(reset))
        if r < 0:
            raise EngineError(f"engine error {r}: {last_error()}")
        return list(ms), nb.value

    def set_tuning(self, entries):
        """alto_engine_set_tuning: entries = [(b_max, pair, wide, bn_cap, units_per_pair), ...]; [] clears."""
        arr = np.ascontiguousarray(np.array(entries, dtype=np.int32).reshape(-1))
        if lib().alto_engine_set_tuning(self.ptr, ctypes.c_void_p(arr.ctypes.data) if arr.size else None,
                                        len(entries)) < 0:
            raise EngineError(last_error())

    def set_graphs(self, on=True):
        """alto_engine_set_graphs: replay captured CUDA graphs for device-resident batches."""
        if lib().alto_engine_set_graphs(self.ptr, int(on)) < 0:
            raise EngineError(last_error())

    def set_lanes(self, lanes):
        """alto_engine_set_lanes: enqueue_device rotates through `lanes` batch contexts (1..4)."""
        if lib().alto_engine_set_lanes(self.ptr, int(lanes)) < 0:
            raise EngineError(last_error())

    def fence(self):
        """alto_engine_fence: every lane's stream waits for the others' work enqueued so far (no host wait)."""
        if lib().alto_engine_fence(self.ptr) < 0:
            raise EngineError(last_error())

    def last_launches(self):
        return lib().alto_last_launches(self.ptr)

    def close(self):
        if getattr(self, "ptr", None):
            lib().alto_engine_free(self.ptr)
            self.ptr = None

    def __del__(self):
        # at interpreter exit the module's globals (the library handle among them) may already be gone; an
        # explicit close() is the supported way to free device memory
        if lib is not None:
            self.close()
