"""Service glue of the answer path, mirroring the reference's src/service.rs: scheme parameters, request and response
sizes, the request codec, the synthetic database, plus seeded synthetic engine state and requests for tests and
benchmarks (the reference builds its state with spiral-rs, which is not available here)."""
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

from . import lib

Q = 4294955009                      # src/service.rs:25, params.rs:97-125
MIN_RECORDS = 2048                  # src/service.rs:15
RECORD_UNIT = 2048                  # src/service.rs:16
DEFAULT_RECORD_BYTES = 32768        # src/service.rs:17
POLY_LEN = 2048                     # ring dimension n (src/service.rs:26-27)
T_EXP_LEFT = 4                      # tg
Q1, Q2 = 1 << 10, 1 << 18           # the two switching moduli (params.rs:97-98)
SEED = 0x416C746F504952             # synthetic::SEED (src/service.rs:44)


def threads():
    return os.cpu_count() or 1


@dataclass(frozen=True)
class Params:
    rows: int
    record_bytes: int
    n: int = POLY_LEN
    tg: int = T_EXP_LEFT

    @property
    def instances(self):
        return self.record_bytes // self.n

    @property
    def count(self):
        return self.tg * self.n

    @property
    def q1_bits(self):
        return (Q1 - 1).bit_length()

    @property
    def row1_off(self):
        return (Q2 - 1).bit_length() * self.n

    @property
    def part_len(self):
        # switch_prefix_row0 (src/modulus_switch.rs:136-147): row 0 at 18 bits, row 1 at 10 bits, rounded to 64 bits
        bits = ((Q2 - 1).bit_length() * self.n + self.q1_bits * self.n + 63) // 64 * 64
        return (bits + 7) // 8


def params(rows, record_bytes=DEFAULT_RECORD_BYTES):
    """service::params (src/service.rs:19-29)."""
    if rows < MIN_RECORDS or rows & (rows - 1):
        raise ValueError(f"the number of records must be a power of two and at least {MIN_RECORDS}")
    if record_bytes <= 0 or record_bytes % RECORD_UNIT:
        raise ValueError(f"the record size must be a positive multiple of {RECORD_UNIT} bytes")
    return Params(rows, record_bytes)


def request_len(p: Params, rows=None):
    """service::request_len (src/service.rs:35-37)."""
    return 9 + 4 * (2 * p.tg * p.n + (p.rows if rows is None else rows))


def response_len(p: Params):
    """service::response_len (src/service.rs:39-41): instances * poly_len * 28 / 8."""
    return p.instances * p.n * 28 // 8


def encode_request(p: Params, y, z, query):
    """service::encode_request (src/service.rs:178-198): [0][u32 count][u32 count][y][z][query], little endian."""
    count = p.count
    y, z, query = (np.asarray(a, dtype=np.uint64) for a in (y, z, query))
    if len(y) != count or len(z) != count or len(query) != p.rows:
        raise ValueError("key or query length")
    if (y >= Q).any() or (z >= Q).any() or (query > 0xFFFFFFFF).any():
        raise ValueError("value out of range")
    head = np.zeros(9, dtype=np.uint8)
    head[1:5] = np.frombuffer(np.uint32(count).tobytes(), dtype=np.uint8)
    head[5:9] = head[1:5]
    body = np.concatenate([y, z, query]).astype("<u4").view(np.uint8)
    return np.concatenate([head, body])


def decode_request(p: Params, frame):
    """service::decode_request (src/service.rs:200-225) without the spiral-rs key objects: returns (y, z, query) as
    uint32 arrays, or raises ValueError with the reference's reason."""
    f = np.frombuffer(bytes(frame), dtype=np.uint8) if not isinstance(frame, np.ndarray) else frame
    count = p.count
    if len(f) != request_len(p) or f[0] != 0:
        raise ValueError("request flag or length")
    words = f[1:9].view("<u4")
    if words[0] != count or words[1] != count:
        raise ValueError("packing key length")
    keys = f[9:9 + 8 * count].view("<u4")
    if (keys >= Q).any():
        raise ValueError("packing key coefficient out of range")
    query = f[9 + 8 * count:].view("<u4")
    return keys[:count], keys[count:], query


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


# ------------------------------------------------------------------------------------------ synthetic inputs
def synthetic_record(row, nbytes):
    """synthetic::record (src/service.rs:54-62): splitmix64 from SEED ^ 0xd1b54a32d192ed03 * (row + 1), each output
    % 65535 as a little-endian u16.  The m-th output is finalise(s0 + (m + 1) * gamma), evaluated here for all m."""
    m = np.arange(nbytes // 2, dtype=np.uint64)
    s0 = np.uint64(SEED ^ ((0xD1B54A32D192ED03 * (row + 1)) & 0xFFFFFFFFFFFFFFFF))
    with np.errstate(over="ignore"):
        z = s0 + (m + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z % np.uint64(65535)).astype("<u2").view(np.uint8)


def write_record_file(path, db_col, num_real_rows, block=4096):
    """Writes the first num_real_rows records of a column-order database (db_col[col][r]) as the reference's on-disk
    database: records one after another, each the record's bytes in column order (the input of its streaming reader,
    src/server.rs:380-500)."""
    with open(path, "wb") as f:
        for r0 in range(0, num_real_rows, block):
            f.write(np.ascontiguousarray(db_col[:, r0:min(r0 + block, num_real_rows)].T).tobytes())


def synthetic_db_col(rows, cols, col0=0, ld=None):
    """The server's column-order database of the synthetic records: db[col][row] = record(row)[col0 + col]
    (src/service.rs:64-78 followed by the column-major transpose of src/server.rs:251-366)."""
    ld = rows if ld is None else ld
    db = np.empty((cols, ld), dtype=np.uint8)
    lib().alto_synthetic_db_col(_ptr(db), ld, rows, col0, cols, threads())
    return db


def uniform_u32(count, bound, seed):
    out = np.empty(count, dtype=np.uint32)
    lib().alto_fill_uniform_u32(_ptr(out), count, bound, seed, threads())
    return out


def uniform_u64(count, bound, seed):
    out = np.empty(count, dtype=np.uint64)
    lib().alto_fill_uniform_u64(_ptr(out), count, bound, seed, threads())
    return out


def random_bytes(count, seed):
    out = np.empty(count, dtype=np.uint8)
    lib().alto_fill_bytes(_ptr(out), count, seed, threads())
    return out


def synthetic_requests(p: Params, b, seed, first_client=0):
    """b well-formed request frames from seeded synthetic clients, as a (b, request_len) uint8 array: y and z
    uniform in [0, Q), query words uniform over u32 (rounded RLWE query words are near-uniform)."""
    rl = request_len(p)
    out = np.empty((b, rl), dtype=np.uint8)
    for c in range(b):
        lib().alto_synthetic_request(_ptr(out[c]), p.rows, p.count, seed, first_client + c)
    return out


def synthetic_requests_device(p: Params, b, seed, d_slots, stride, lead=7, first_client=0):
    """The frames of synthetic_requests written straight into device memory: frame c at d_slots + c * stride +
    lead (alto_synthetic_requests_device)."""
    r = lib().alto_synthetic_requests_device(ctypes.c_void_p(d_slots), stride, lead, b, p.rows, p.count, seed,
                                             first_client)
    if r < 0:
        raise RuntimeError(f"alto_synthetic_requests_device: {lib().alto_last_error().decode()}")


def _pow(a, e):
    return pow(int(a), int(e), Q)


def inverse_ntt_table(n):
    """An inverse-NTT twiddle table of the shape the engine reads (entry h + i for block i of the stage with h
    blocks): inverse powers of a primitive 2n-th root of unity psi in bit-reversed order.  The engine is exact for
    any table; this one makes the inverse NTT a genuine negacyclic transform."""
    logn = n.bit_length() - 1
    for g in range(2, 1000):
        psi = _pow(g, (Q - 1) // (2 * n))
        if _pow(psi, n) == Q - 1:
            break
    inv = _pow(psi, Q - 2)
    rev = [int(format(i, f"0{logn}b")[::-1], 2) if logn else 0 for i in range(n)]
    return np.array([_pow(inv, r) for r in rev], dtype=np.uint64)


@dataclass
class SyntheticState:
    """Seeded engine state of the shapes the reference builds (src/service.rs:127-170): the synthetic column-order
    database, a packing matrix with values uniform in [0, Q), bold_t_hat uniform in [0, Q), row-0 prefixes (random
    bytes in the row-0 bits, zero after them as switch_prefix_row0 leaves them, or random throughout when
    full_prefix) and an inverse-NTT table."""
    p: Params
    seed: int
    db_col: np.ndarray
    U: np.ndarray = field(repr=False)          # (cols, count) uint32 values, or None when not materialised
    ub: np.ndarray = field(repr=False)         # engine layout of sw_pack_build
    that: list = field(repr=False)
    prefixes: list = field(repr=False)
    inv_table: np.ndarray = field(repr=False)

    @staticmethod
    def make(p: Params, seed=1, full_prefix=False, keep_values=True, host_db=True):
        """host_db=False leaves db_col None: Engine.from_state then generates the same records on the device."""
        cols, count, outputs = p.record_bytes, p.count, p.instances
        db = synthetic_db_col(p.rows, cols) if host_db else None
        U = uniform_u32(cols * count, Q, seed * 0x1000193 + 1).reshape(cols, count)
        ub = np.empty(4 * cols * count, dtype=np.int8)
        lib().alto_pack_encode(_ptr(ub), _ptr(U), cols, count, threads())
        that = [uniform_u64(count, Q, seed * 0x1000193 + 2 + o) for o in range(outputs)]
        row0_bytes = ((Q2 - 1).bit_length() * p.n + 7) // 8
        prefixes = []
        for o in range(outputs):
            pre = random_bytes(p.part_len, seed * 0x1000193 + 100 + o)
            if not full_prefix:
                pre[row0_bytes:] = 0
            prefixes.append(pre)
        return SyntheticState(p, seed, db, U if keep_values else None, ub, that, prefixes, inverse_ntt_table(p.n))
