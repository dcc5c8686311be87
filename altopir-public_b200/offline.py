"""The scheme's offline set-up on the device (the reference's `Prepared::new`, src/service.rs:127-157): an engine
whose database is resident gets the hint, the InspiRING precomputation, the packing matrix, bold_t_hat and the row-0
prefixes of the scheme from `alto_engine_offline`, with the public masks of `client.py`, so that its responses
decrypt under the client's secret."""
import numpy as np

from . import client, service
from .engine import Engine, TiledDb

Q = service.Q


def public_inputs(p):
    """The offline set-up's public inputs: the query's row-0 polynomials -a_i (rows / n, n) and the masks (w, v)."""
    masks = client.query_masks(p.rows, p.n)
    w, v = client.packing_masks(p.n, p.tg)
    return (np.uint64(Q) - masks) % np.uint64(Q), w, v


def prepare(engine, p, want=False):
    """Runs the offline set-up on `engine` (its database already resident).  Returns the device time in ms, and with
    want=True also the per-output bold_t, bold_t_bar, that and a_hat (Engine.offline)."""
    q, w, v = public_inputs(p)
    return engine.offline(q, w, v, want=want)


def _blank(p):
    n, cols, outputs = p.n, p.record_bytes, p.instances
    ub = np.zeros(4 * cols * p.count, dtype=np.int8)
    prefixes = [np.zeros(p.part_len, dtype=np.uint8) for _ in range(outputs)]
    that = [np.zeros(p.count, dtype=np.uint64) for _ in range(outputs)]
    inv = client.ntt_inverse_table(client.Ring(n))
    return ub, prefixes, that, inv


def blank_engine(p, db_col=None, threads=1):
    """An engine over `db_col` ((record_bytes, rows) column-order bytes), or over the synthetic records generated on
    the device when db_col is None, created with zero packing state (to be replaced by prepare)."""
    ub, prefixes, that, inv = _blank(p)
    if db_col is None:
        e = Engine.empty(p.rows, p.record_bytes, ub, p.n, p.tg, prefixes, p.row1_off, 1 << p.q1_bits, p.q1_bits,
                         that, inv, Q, threads)
        e.fill_synthetic()
        return e
    tiled = TiledDb.__new__(TiledDb)   # the engine reads the column-order database; no tiled host copy
    tiled.rows, tiled.cols, tiled.buf = p.rows, p.record_bytes, np.zeros(64, dtype=np.uint8)
    return Engine(db_col, tiled, db_col.shape[1], ub, p.n, p.tg, prefixes, p.row1_off, 1 << p.q1_bits, p.q1_bits,
                  that, inv, Q, threads)


def scheme_engine(p, db_col=None, threads=1):
    """blank_engine with the scheme's state built on the device.  Returns (engine, set-up ms)."""
    e = blank_engine(p, db_col, threads)
    return e, prepare(e, p)
