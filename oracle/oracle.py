"""ctypes access to the test oracle.  TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the engine.

  Oracle     -- the plain-C restatement in alto_oracle.c (liboracle.so), portable, OpenMP.
  RefEngine  -- the reference engine src/amx_kernels.cpp compiled unchanged from its own source (_ref/), driven
                through its own C ABI (src/engine.rs:4-20).  Needs AVX-512 (+ AMX for method 0) on the host CPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libalto_ref.so")
Q = 4294955009


# Where the reference tree is mounted when this repository is built (override with ALTO_REFERENCE_DIR); the GPU
# machines have no reference tree and use the _ref/ library built here.
REFERENCE_DIR = os.environ.get("ALTO_REFERENCE_DIR", "/root/reference")


def build():
    """Compiles liboracle.so (and _ref/ from the reference's own source when the reference tree is present) with
    oracle/Makefile."""
    import subprocess
    args = ["make", "-s", "-C", HERE]
    if os.path.isdir(REFERENCE_DIR):
        args.append(f"REFERENCE_DIR={REFERENCE_DIR}")
    r = subprocess.run(args, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def cpu_flags():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


REF_NEEDS = {"avx512f", "avx512bw", "avx512dq", "avx512vl", "avx512_vnni", "avx2", "fma", "bmi2"}


def ref_methods():
    """Methods of the reference engine this host can run: [] when the library is absent or the CPU lacks AVX-512."""
    if not os.path.exists(REF_SO):
        return []
    fl = cpu_flags()
    if not REF_NEEDS <= fl:
        return []
    return ([0] if {"amx_int8", "amx_tile"} <= fl else []) + [2]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _ptrs(arrays):
    return (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


class _OrcState(ctypes.Structure):
    _fields_ = [
        ("db_col", ctypes.c_void_p), ("ld", ctypes.c_size_t), ("rows", ctypes.c_size_t), ("cols", ctypes.c_size_t),
        ("U", ctypes.c_void_p), ("n", ctypes.c_size_t), ("tg", ctypes.c_size_t),
        ("prefix", ctypes.c_void_p), ("part_len", ctypes.c_size_t), ("row1_off", ctypes.c_size_t),
        ("q1", ctypes.c_uint64), ("q1_bits", ctypes.c_int),
        ("that", ctypes.c_void_p), ("inv_table", ctypes.c_void_p),
    ]


class Oracle:
    """The restatement (alto_oracle.c) over a service.SyntheticState-like object."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        c = ctypes
        P, S, U32, U64, I = c.c_void_p, c.c_size_t, c.c_uint32, c.c_uint64, c.c_int
        for name, res, args in [
            ("orc_mix", U64, [c.POINTER(U64)]),
            ("orc_synthetic_record", None, [P, U64, S]),
            ("orc_record_byte", c.c_uint8, [U64, U64]),
            ("orc_synthetic_db_col", None, [P, S, S, S, S]),
            ("orc_validate", I, [P, S, S, S]),
            ("orc_scan_acc", U32, [P, P, S]),
            ("orc_mod_switch", U32, [U32]),
            ("orc_pack_beta", U32, [P, P, S]),
            ("orc_intt", I, [P, P, S]),
            ("orc_rescale", U32, [U64, U64]),
            ("orc_rescale_double", U32, [U64, U64]),
            ("orc_rescale_mismatches", U64, [U64, U64, U64]),
            ("orc_rescale_digest", U64, [U64, U64, U64]),
            ("orc_switch_row1", I, [P, S, S, P, P, S, U64, I]),
            ("orc_tail_ntt", I, [P, P, P, P, S, P, S]),
            ("orc_answer_part", I, [c.POINTER(_OrcState), P, S, P]),
            ("orc_answer", I, [c.POINTER(_OrcState), c.POINTER(P), c.POINTER(S), S, c.POINTER(P), c.POINTER(I)]),
            ("orc_pack_build", None, [P, c.POINTER(P), c.POINTER(P), P, P, S, S, S, S]),
            ("orc_answer_parts", I, [c.POINTER(_OrcState), c.POINTER(P), c.POINTER(S), S, c.POINTER(P)]),
            ("orc_fill_uniform_u32", None, [P, S, U64, U64]),
            ("orc_fill_uniform_u64", None, [P, S, U64, U64]),
            ("orc_fill_bytes", None, [P, S, U64]),
            ("orc_synthetic_request", None, [P, S, S, U64, U64]),
            ("orc_hint_ring", None, [P, S, P, S, S, S, S, P, S, I]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.L = L

    # the engine-level functions --------------------------------------------------------------------
    def _state(self, st):
        p = st.p
        keep = {
            "pre": [np.ascontiguousarray(x, dtype=np.uint8) for x in st.prefixes],
            "that": [np.ascontiguousarray(t, dtype=np.uint64) for t in st.that],
            "U": np.ascontiguousarray(st.U, dtype=np.uint32),
            "inv": np.ascontiguousarray(st.inv_table, dtype=np.uint64),
        }
        keep["pre_p"] = _ptrs(keep["pre"])
        keep["that_p"] = _ptrs(keep["that"])
        s = _OrcState(st.db_col.ctypes.data, st.db_col.shape[1], p.rows, p.record_bytes, keep["U"].ctypes.data, p.n,
                      p.tg, ctypes.cast(keep["pre_p"], ctypes.c_void_p), keep["pre"][0].size, p.row1_off,
                      1 << p.q1_bits, p.q1_bits, ctypes.cast(keep["that_p"], ctypes.c_void_p),
                      keep["inv"].ctypes.data)
        return s, keep

    def answer(self, st, frames, out=None, status=None):
        """alto_answer semantics; frames: list of uint8 arrays (None = missing frame).  Returns (ret, status, out)."""
        b = len(frames)
        rl = st.p.instances * st.prefixes[0].size
        if out is None:
            out = np.zeros((b, rl), dtype=np.uint8)
        if status is None:
            status = np.full(b, -1, dtype=np.int32)
        s, keep = self._state(st)
        req = (ctypes.c_void_p * b)(*[f.ctypes.data if f is not None else None for f in frames])
        lens = (ctypes.c_size_t * b)(*[f.size if f is not None else 0 for f in frames])
        outp = (ctypes.c_void_p * b)(*[out[i].ctypes.data for i in range(b)])
        r = self.L.orc_answer(ctypes.byref(s), req, lens, b, outp, status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return r, status, out

    def answer_part(self, st, frame, o):
        """One response part (n columns) of one valid frame."""
        s, keep = self._state(st)
        res = np.zeros(st.prefixes[0].size, dtype=np.uint8)
        r = self.L.orc_answer_part(ctypes.byref(s), _p(frame), o, _p(res))
        if r:
            raise RuntimeError(f"oracle tail failure {r}")
        return res

    def answer_parts(self, st, frames, parts):
        """Output part parts[k] of frame frames[k] for every k, computed in parallel; returns a (k, part_len) array."""
        s, keep = self._state(st)
        k = len(frames)
        out = np.zeros((k, st.prefixes[0].size), dtype=np.uint8)
        fp = (ctypes.c_void_p * k)(*[f.ctypes.data for f in frames])
        pp = (ctypes.c_size_t * k)(*[int(x) for x in parts])
        op = (ctypes.c_void_p * k)(*[out[i].ctypes.data for i in range(k)])
        r = self.L.orc_answer_parts(ctypes.byref(s), fp, pp, k, op)
        if r:
            raise RuntimeError(f"oracle tail failure {r}")
        return out

    def validate(self, frame, count, rows):
        if frame is None:
            return self.L.orc_validate(None, 0, count, rows)
        return self.L.orc_validate(_p(frame), frame.size, count, rows)

    def rescale_mismatches(self, v0, v1, q1):
        return self.L.orc_rescale_mismatches(v0, v1, q1)

    def rescale_digest(self, v0, v1, q1):
        return self.L.orc_rescale_digest(v0, v1, q1)

    def rescale(self, v, q1):
        return self.L.orc_rescale(v, q1)

    def synthetic_record(self, row, nbytes):
        out = np.empty(nbytes, dtype=np.uint8)
        self.L.orc_synthetic_record(_p(out), row, nbytes)
        return out

    def synthetic_db_col(self, rows, col0, ncols):
        db = np.empty((ncols, rows), dtype=np.uint8)
        self.L.orc_synthetic_db_col(_p(db), rows, rows, col0, ncols)
        return db

    def pack_build(self, bold_t, bold_t_bar, tables, gen_pows, num_iter, tg, n):
        rho = len(bold_t)
        U = np.empty((rho * n, tg * n), dtype=np.uint32)
        tables = np.ascontiguousarray(tables, dtype=np.uint32)
        gen_pows = np.ascontiguousarray(gen_pows, dtype=np.uint32)
        self.L.orc_pack_build(_p(U), _ptrs(bold_t), _ptrs(bold_t_bar), _p(tables), _p(gen_pows), num_iter, tg, n, rho)
        return U

    def mod_switch(self, acc):
        return self.L.orc_mod_switch(acc)

    def scan_acc(self, dbcol, qwords_u8):
        return self.L.orc_scan_acc(_p(dbcol), _p(qwords_u8), dbcol.size)


    def fill_uniform_u32(self, count, bound, seed):
        out = np.empty(count, dtype=np.uint32)
        self.L.orc_fill_uniform_u32(_p(out), count, bound, seed)
        return out

    def fill_uniform_u64(self, count, bound, seed):
        out = np.empty(count, dtype=np.uint64)
        self.L.orc_fill_uniform_u64(_p(out), count, bound, seed)
        return out

    def fill_bytes(self, count, seed):
        out = np.empty(count, dtype=np.uint8)
        self.L.orc_fill_bytes(_p(out), count, seed)
        return out

    def hint_ring(self, db_col, query, n, c0, c1, perm_out=False):
        """The offline hint's ring multiply (orc_hint_ring) for columns [c0, c1) of a column-order database:
        an (n, c1 - c0) uint64 array."""
        q = np.ascontiguousarray(query, dtype=np.uint64)
        out = np.empty((n, c1 - c0), dtype=np.uint64)
        self.L.orc_hint_ring(_p(out), c1 - c0, _p(db_col), db_col.shape[1], db_col.shape[1], c0, c1, _p(q), n,
                             int(perm_out))
        return out

    def synthetic_requests(self, p, b, seed, first_client=0):
        """b frames of the seeded synthetic clients first_client .. as a (b, request_len) uint8 array."""
        out = np.empty((b, 9 + 4 * (2 * p.count + p.rows)), dtype=np.uint8)
        for c in range(b):
            self.L.orc_synthetic_request(_p(out[c]), p.rows, p.count, seed, first_client + c)
        return out


# --------------------------------------------------------------------------------------------- seeded state
class Params:
    """The scheme parameters of the answer path (src/service.rs:19-41, params.rs:97-125): n = 2048, tg = 4, row 0
    switched to 18 bits and row 1 to 10 bits, so a response part is 7168 bytes."""

    def __init__(self, rows, record_bytes, n=2048, tg=4, q1_bits=10, q2_bits=18):
        self.rows, self.record_bytes, self.n, self.tg = rows, record_bytes, n, tg
        self.q1_bits, self.row1_off = q1_bits, q2_bits * n
        self.instances, self.count = record_bytes // n, tg * n
        self.row0_bytes = (q2_bits * n + 7) // 8
        self.part_len = ((q2_bits * n + q1_bits * n + 63) // 64 * 64 + 7) // 8


def inverse_ntt_table(n):
    """Inverse powers of a primitive 2n-th root of unity mod Q in bit-reversed order, the table shape the engines
    index as [h + i] for block i of the stage with h blocks."""
    logn = n.bit_length() - 1
    for g in range(2, 1000):
        psi = pow(g, (Q - 1) // (2 * n), Q)
        if pow(psi, n, Q) == Q - 1:
            break
    inv = pow(psi, Q - 2, Q)
    rev = [int(format(i, f"0{logn}b")[::-1], 2) if logn else 0 for i in range(n)]
    return np.array([pow(inv, r, Q) for r in rev], dtype=np.uint64)


class State:
    """Seeded engine state with the shapes of the reference's (src/service.rs:127-170): the synthetic column-order
    database, packing-matrix values U uniform in [0, Q), bold_t_hat uniform in [0, Q), row-0 prefixes (random bytes
    in the row-0 bits, zero after them) and an inverse-NTT table.  Built with this oracle's generators only; for the
    same (rows, record_bytes, seed) it holds the bytes that the engine package's SyntheticState.make produces."""

    def __init__(self, p, seed=1, oracle=None):
        o = oracle or Oracle()
        self.p, self.seed = p, seed
        self.db_col = o.synthetic_db_col(p.rows, 0, p.record_bytes)
        base = seed * 0x1000193
        self.U = o.fill_uniform_u32(p.record_bytes * p.count, Q, base + 1).reshape(p.record_bytes, p.count)
        self.that = [o.fill_uniform_u64(p.count, Q, base + 2 + k) for k in range(p.instances)]
        self.prefixes = []
        for k in range(p.instances):
            pre = o.fill_bytes(p.part_len, base + 100 + k)
            pre[p.row0_bytes:] = 0
            self.prefixes.append(pre)
        self.inv_table = inverse_ntt_table(p.n)


# --------------------------------------------------------------------------------------------- reference engine
def ref_ub_layout(U):
    """The reference's AMX byte-plane layout of the packing matrix (sw_ubt, src/amx_kernels.cpp:39-41, written by
    sw_pack_build at :331-337): plane j of column col = 16 ct + nn and key word k = 64 kc + 4 r + t is stored, as
    byte - 128, at ((j (CT/2) + ct/2) KC + kc) 2048 + (ct % 2) 1024 + 64 r + 4 nn + t."""
    cols, K = U.shape
    CT, KC = cols // 16, K // 64
    out = np.empty((4, CT // 2, KC, 2, 16, 16, 4), dtype=np.int8)
    for j in range(4):
        plane = (((U >> np.uint32(8 * j)) & np.uint32(0xFF)).astype(np.int16) - 128).astype(np.int8)
        v = plane.reshape(CT // 2, 2, 16, KC, 16, 4)          # ct2, ctp, nn, kc, r, t
        out[j] = v.transpose(0, 3, 1, 4, 2, 5)                # ct2, kc, ctp, r, nn, t
    return out.reshape(-1)


def ref_ub_values(ub, cols, K):
    """Inverse of ref_ub_layout: packing-matrix values from the reference's layout."""
    CT, KC = cols // 16, K // 64
    v = ub.view(np.int8).reshape(4, CT // 2, KC, 2, 16, 16, 4).astype(np.int16) + 128
    U = np.zeros((cols, K), dtype=np.uint32)
    for j in range(4):
        U |= v[j].transpose(0, 2, 4, 1, 3, 5).reshape(cols, K).astype(np.uint32) << np.uint32(8 * j)
    return U


class RefEngine:
    """The reference engine (amx_kernels.cpp compiled from its own source) over a SyntheticState."""

    def __init__(self, st, threads=None):
        L = ctypes.CDLL(REF_SO)
        c = ctypes
        P, S, I, U64 = c.c_void_p, c.c_size_t, c.c_int, c.c_uint64
        PP = c.POINTER(P)
        for name, res, args in [
            ("sw_amx_init", I, []), ("sw_tile_db", None, [P, P, S, S, S, I]),
            ("sw_pack_build", None, [P, PP, PP, P, P, S, S, S, S, U64, I]),
            ("alto_engine_new", P, [P, P, S, S, S, P, S, S, PP, S, S, U64, I, PP, P, U64, I]),
            ("alto_engine_free", None, [P]), ("alto_request_len", S, [P]), ("alto_response_len", S, [P]),
            ("alto_answer", I, [P, PP, c.POINTER(S), S, PP, c.POINTER(I), I, c.POINTER(c.c_double)]),
        ]:
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.L = L
        self.threads = threads or os.cpu_count() or 1
        if 0 in ref_methods():
            L.sw_amx_init()
        p = st.p
        self.p = p
        cols, rows = p.record_bytes, p.rows
        self.db = st.db_col
        self.tiled = np.empty(rows * cols, dtype=np.uint8)
        L.sw_tile_db(_p(self.tiled), _p(self.db), self.db.shape[1], rows, cols, self.threads)
        self.ub = ref_ub_layout(st.U)
        self.pre = [np.ascontiguousarray(x, dtype=np.uint8) for x in st.prefixes]
        self.that = [np.ascontiguousarray(t, dtype=np.uint64) for t in st.that]
        self.inv = np.ascontiguousarray(st.inv_table, dtype=np.uint64)
        self.e = L.alto_engine_new(_p(self.db), _p(self.tiled), self.db.shape[1], rows, cols, _p(self.ub), p.n, p.tg,
                                   _ptrs(self.pre), self.pre[0].size, p.row1_off, 1 << p.q1_bits, p.q1_bits,
                                   _ptrs(self.that), _p(self.inv), Q, self.threads)
        if not self.e:
            raise RuntimeError("reference engine rejected the configuration")

    def response_len(self):
        return self.L.alto_response_len(self.e)

    def answer(self, frames, method, out=None, status=None):
        b = len(frames)
        rl = self.response_len()
        if out is None:
            out = np.zeros((b, rl), dtype=np.uint8)
        if status is None:
            status = np.full(b, -1, dtype=np.int32)
        req = (ctypes.c_void_p * b)(*[f.ctypes.data if f is not None else None for f in frames])
        lens = (ctypes.c_size_t * b)(*[f.size if f is not None else 0 for f in frames])
        outp = (ctypes.c_void_p * b)(*[out[i].ctypes.data for i in range(b)])
        stage = (ctypes.c_double * 4)()
        r = self.L.alto_answer(self.e, req, lens, b, outp, status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               method, stage)
        return r, status, out, list(stage)

    def close(self):
        if self.e:
            self.L.alto_engine_free(self.e)
            self.e = None

    def __del__(self):
        self.close()
