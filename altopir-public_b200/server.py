"""Serving loop with continuous batching (alto_server_*): the engine loop of the reference's server
(src/bin/altopir.rs:245-513) without its TCP front end, plus an open-loop Poisson load generator."""
import ctypes
import threading
import time

import numpy as np

from . import lib, last_error

BUSY = -9       # alto_server_submit: the queue is full (the reference server's status 9)
TIMEOUT = -5    # alto_server_wait: not done within the timeout
FAILED = -4     # device failure


class Server:
    """A serving loop on an engine (engine.Engine), or on the host loopback executor when engine is None."""

    DEFAULT_KEYS = (1 << 64) - 1  # alto_server_new_keyed: SIZE_MAX picks the default resident table

    def __init__(self, engine=None, max_batch=128, queue_cap=512, slots=2, request_len=None, response_len=None,
                 service_us=0.0, key_bytes=DEFAULT_KEYS):
        """key_bytes: HBM for the resident per-client table (0 = none; the default is a quarter of the free device
        memory, at most 8 GiB)."""
        if engine is not None:
            self.ptr = lib().alto_server_new_keyed(engine.ptr, max_batch, queue_cap, slots, key_bytes)
            self.response_len = engine.response_len()
            self.request_len = engine.request_len()
        else:
            self.ptr = lib().alto_server_new_loopback(request_len, response_len, max_batch, queue_cap, slots,
                                                      float(service_us))
            self.response_len, self.request_len = response_len, request_len
        if not self.ptr:
            raise RuntimeError(f"serving loop not created: {last_error()}")
        self._engine = engine  # the engine must outlive the loop

    def submit(self, frame):
        """Queue one frame (uint8 array); returns a ticket >= 0 or BUSY."""
        f = np.ascontiguousarray(frame, dtype=np.uint8)
        return lib().alto_server_submit(self.ptr, ctypes.c_void_p(f.ctypes.data), f.size)

    def wait(self, ticket, timeout_ms=60000, with_latency=False):
        """(status, response or None) of a ticket; status as alto_server_wait.  with_latency adds the loop's own
        submit-to-completion time in ms as a third element."""
        out = np.empty(self.response_len, dtype=np.uint8)
        lat = ctypes.c_double(0.0)
        st = lib().alto_server_wait(self.ptr, ticket, ctypes.c_void_p(out.ctypes.data), out.size, timeout_ms,
                                    ctypes.byref(lat))
        if with_latency:
            return st, (out if st == 0 else None), lat.value
        return st, (out if st == 0 else None)

    STATS = ("answered", "rejected", "busy", "failed", "batches", "mean_batch", "p50_ms", "p99_ms", "p999_ms",
             "max_ms", "queued", "resident_hits", "admitted", "evicted", "uncached", "table_rows")
    LOG = ("t_dispatch", "t_done", "taken", "on_device", "packed", "resident", "upload_ms", "pack_ms", "rest_ms",
           "device_ms")

    def stats(self):
        v = (ctypes.c_double * len(self.STATS))()
        lib().alto_server_stats(self.ptr, v, len(self.STATS))
        return dict(zip(self.STATS, list(v)))

    def log(self, max_rows=65536):
        """The per-batch log, oldest first: a list of dicts with the LOG fields."""
        buf = (ctypes.c_double * (max_rows * len(self.LOG)))()
        n = lib().alto_server_log(self.ptr, buf, max_rows)
        w = len(self.LOG)
        return [dict(zip(self.LOG, buf[k * w:(k + 1) * w])) for k in range(max(n, 0))]

    def close(self):
        if getattr(self, "ptr", None):
            lib().alto_server_free(self.ptr)
            self.ptr = None

    def __del__(self):
        # at interpreter exit the module's globals (the library handle among them) may already be gone; an
        # explicit close() is the supported way to free device memory
        if lib is not None:
            self.close()


def poisson_load(server, frames, rate_qps, seconds, seed=1, clients=4, grace_s=120.0):
    """Open-loop load: arrival times drawn from a Poisson process of rate_qps over `seconds`, frames taken round
    robin from `frames`, submitted by `clients` threads at their due times; each thread then collects its tickets.
    Returns (results, offered, elapsed_s) with results[i] = (frame index, status, response, latency_s), where the
    latency is the loop's own time from submit to completion and elapsed_s runs from the first arrival to the last
    completion.  The whole run is bounded: tickets not complete `grace_s` after the last arrival are reported as
    TIMEOUT instead of being waited for one by one."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_qps, size=int(rate_qps * seconds * 1.5) + 8))
    t = t[t < seconds]
    results = [None] * len(t)
    start = time.perf_counter() + 0.05
    t_first = start
    done_at = [0.0] * clients

    def worker(k):
        mine = []
        for i in range(k, len(t), clients):
            due = start + t[i]
            while True:
                d = due - time.perf_counter()
                if d <= 0:
                    break
                time.sleep(min(d, 0.002))
            mine.append((i, server.submit(frames[i % len(frames)])))
        deadline = start + seconds + grace_s
        for i, ticket in mine:
            if ticket < 0:
                results[i] = (i % len(frames), ticket, None, 0.0)
                continue
            left_ms = int(max(0.0, deadline - time.perf_counter()) * 1e3)
            st, resp, lat_ms = server.wait(ticket, timeout_ms=left_ms, with_latency=True)
            results[i] = (i % len(frames), st, resp, lat_ms * 1e-3)
            done_at[k] = max(done_at[k], t_first + t[i] + lat_ms * 1e-3)

    th = [threading.Thread(target=worker, args=(k,)) for k in range(clients)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    elapsed = max(max(done_at) - start, seconds) if len(t) else seconds
    return results, len(t), elapsed
