"""The serving loop's queueing and batching logic on the host loopback executor (no device): every ticket gets the
answer to its own frame, a full queue answers BUSY, batches form under load without holding a lone request back,
and the statistics add up."""
import threading
import time

import numpy as np
import pytest


def loopback_expected(frame, length):
    h = 1469598103934665603
    for c in bytes(frame):
        h = ((h ^ c) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    out = bytearray()
    while len(out) < length:
        h = (h + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = h
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        out += z.to_bytes(8, "little")
    return np.frombuffer(bytes(out[:length]), dtype=np.uint8)


@pytest.fixture()
def server_mod():
    from altopir_b200 import server
    return server


def test_every_ticket_gets_the_answer_to_its_own_frame(server_mod):
    s = server_mod.Server(None, max_batch=16, queue_cap=1000, slots=2, request_len=64, response_len=40,
                          service_us=300)
    rng = np.random.default_rng(3)
    frames = [rng.integers(0, 256, 64, dtype=np.uint8) for _ in range(300)]
    results = {}

    def client(k):
        for i in range(k, 300, 4):
            t = s.submit(frames[i])
            assert t >= 0
            results[i] = t
            time.sleep(rng.uniform(0, 0.0005))

    th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    [x.start() for x in th]
    [x.join() for x in th]
    for i, t in results.items():
        st, resp = s.wait(t)
        assert st == 0 and np.array_equal(resp, loopback_expected(frames[i], 40)), i
    bad = s.submit(np.zeros(10, dtype=np.uint8))  # wrong length: status 1, no response
    assert s.wait(bad) == (1, None)
    stats = s.stats()
    assert stats["answered"] == 300 and stats["rejected"] == 1 and stats["failed"] == 0
    assert stats["batches"] >= 300 / 16 and stats["mean_batch"] > 1.0
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] <= stats["max_ms"]
    s.close()


def test_full_queue_answers_busy_and_lone_requests_are_not_held(server_mod):
    s = server_mod.Server(None, max_batch=4, queue_cap=8, slots=1, request_len=16, response_len=8,
                          service_us=20000)
    f = np.arange(16, dtype=np.uint8)
    tickets = [s.submit(f) for _ in range(40)]
    busy = [t for t in tickets if t == server_mod.BUSY]
    assert busy, "a burst beyond the queue capacity must see BUSY"
    for t in tickets:
        if t >= 0:
            assert s.wait(t)[0] == 0
    assert s.stats()["busy"] == len(busy)
    # an idle loop answers a lone request after about one service time, not after a batch fills
    t0 = time.perf_counter()
    assert s.wait(s.submit(f))[0] == 0
    assert time.perf_counter() - t0 < 0.5
    s.close()


def test_wait_timeout_and_unknown_ticket(server_mod):
    s = server_mod.Server(None, max_batch=1, queue_cap=4, slots=1, request_len=8, response_len=8, service_us=200000)
    t = s.submit(np.zeros(8, dtype=np.uint8))
    assert s.wait(t, timeout_ms=1)[0] == server_mod.TIMEOUT
    assert s.wait(t, timeout_ms=5000)[0] == 0
    assert s.wait(t)[0] == -1  # released by the successful wait
    s.close()
