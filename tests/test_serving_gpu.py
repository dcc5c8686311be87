"""Continuous batching on the device: requests arriving while others are on the GPU join the next batch, batches
overlap on the device, and each response is the same as the engine's answer to the request alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# the loop's host waits are bounded (60 s a ticket); the whole test is bounded too, so that a stalled loop fails
# the run instead of holding it
@pytest.mark.timeout(300, method="thread")
def test_each_result_is_the_same_alone_and_in_the_mix(gpu, svc, eng):
    from altopir_b200 import server as srv
    import frames as fr
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=71, full_prefix=True)
    e = eng.Engine.from_state(st)
    frames = svc.synthetic_requests(p, 48, seed=72)
    # a few malformed frames mixed in (statuses 1, 2, 3)
    mf, want = fr.malformed_table(frames[0], frames[1], p.count)
    mixed = [frames[i] for i in range(48)] + mf[1:7]
    alone = []
    for i in range(48):
        out = np.zeros((1, e.response_len()), dtype=np.uint8)
        status = np.full(1, -1, dtype=np.int32)
        assert e.answer([frames[i]], out, status)[0] == 1
        alone.append(out[0].copy())
    s = srv.Server(e, max_batch=16, queue_cap=256, slots=3)
    results, offered, elapsed = srv.poisson_load(s, mixed, rate_qps=4000, seconds=0.25, seed=73, clients=3)
    assert offered > 40
    for idx, status, resp, lat in results:
        if idx < 48:
            assert status == 0 and np.array_equal(resp, alone[idx]), idx
        else:
            assert status == want[idx - 48 + 1] and resp is None
    stats = s.stats()
    assert stats["failed"] == 0 and stats["busy"] == 0 and stats["answered"] > 0 and stats["batches"] > 1
    assert stats["p50_ms"] > 0 and stats["p99_ms"] >= stats["p50_ms"]
    s.close()
    e.close()


@pytest.mark.timeout(300, method="thread")
def test_direct_answers_beside_a_running_loop(gpu, svc, eng):
    # the loop answers in batch contexts of its own, so alto_answer on the same engine may run beside it
    from altopir_b200 import server as srv
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=81, full_prefix=True)
    e = eng.Engine.from_state(st)
    frames = svc.synthetic_requests(p, 40, seed=82)
    rl = e.response_len()
    alone = np.zeros((40, rl), dtype=np.uint8)
    status = np.full(40, -1, dtype=np.int32)
    assert e.answer([frames[i] for i in range(40)], alone, status)[0] == 40
    s = srv.Server(e, max_batch=8, queue_cap=64, slots=2)
    for rep in range(3):
        tickets = [s.submit(frames[i]) for i in range(24)]
        assert all(t >= 0 for t in tickets)
        direct = np.zeros((16, rl), dtype=np.uint8)
        dst = np.full(16, -1, dtype=np.int32)
        assert e.answer([frames[24 + i] for i in range(16)], direct, dst)[0] == 16
        assert np.array_equal(direct, alone[24:]), rep
        for i, t in enumerate(tickets):
            code, resp = s.wait(t)
            assert code == 0 and np.array_equal(resp, alone[i]), (rep, i)
    assert s.stats()["failed"] == 0
    s.close()
    e.close()


@pytest.mark.timeout(300, method="thread")
def test_resident_clients_skip_the_pack_and_answer_the_same(gpu, svc, eng):
    """Clients whose packing keys y are resident skip the pack GEMM: with a table of four rows, ten clients sending
    new queries with their own keys again and again are answered exactly as the engine answers each frame alone,
    rows are admitted, reused and evicted, a frame with a y key >= Q (status 3) is never kept, and the per-batch log
    accounts for every frame."""
    from altopir_b200 import server as srv
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=91, full_prefix=True)
    e = eng.Engine.from_state(st)
    base = svc.synthetic_requests(p, 10, seed=92)
    queries = svc.synthetic_requests(p, 60, seed=93)
    q0 = 9 + 8 * p.count
    frames = []
    for k in range(60):  # client k % 10 with the query words of frame k
        f = base[k % 10].copy()
        f[q0:] = queries[k][q0:]
        frames.append(f)
    bad = base[3].copy()
    bad[9:13] = 0xFF  # first y key word >= Q
    frames.append(bad)
    rl = e.response_len()
    alone = []
    for f in frames:
        out = np.zeros((1, rl), dtype=np.uint8)
        status = np.full(1, -1, dtype=np.int32)
        e.answer([f], out, status)
        alone.append((int(status[0]), out[0].copy()))
    assert alone[-1][0] == 3
    row_bytes = p.record_bytes * 4
    for key_bytes, expect_hits in ((4 * row_bytes, True), (0, False)):
        s = srv.Server(e, max_batch=8, queue_cap=128, slots=2, key_bytes=key_bytes)
        for rnd in range(3):
            order = list(range(len(frames)))
            np.random.default_rng(rnd).shuffle(order)
            tickets = [(i, s.submit(frames[i])) for i in order]
            for i, t in tickets:
                code, resp = s.wait(t)
                assert code == alone[i][0], (key_bytes, rnd, i)
                if code == 0:
                    assert np.array_equal(resp, alone[i][1]), (key_bytes, rnd, i)
        stats = s.stats()
        log = s.log()
        assert stats["failed"] == 0 and stats["answered"] == 3 * 60 and stats["rejected"] == 3
        assert len(log) == stats["batches"]
        assert all(r["packed"] + r["resident"] == r["on_device"] <= r["taken"] <= 8 for r in log)
        assert sum(r["on_device"] for r in log) == 3 * 61
        assert sum(r["resident"] for r in log) == stats["resident_hits"]
        if expect_hits:
            assert stats["table_rows"] == 4 and stats["resident_hits"] > 0 and stats["evicted"] > 0
            assert stats["admitted"] >= 10
        else:
            assert stats["table_rows"] == 0 and stats["resident_hits"] == 0 and stats["admitted"] == 0
        s.close()
    e.close()


@pytest.mark.timeout(300, method="thread")
def test_serving_over_several_record_chunks(gpu, svc, eng, monkeypatch):
    """A database of three record chunks (the last one partial), every batch pipelined (ALTO_PIPED_BYTES=0): the loop
    uploads each batch's query words chunk group by chunk group and starts each group's scan once it is split; every
    response equals the engine's answer to the frame alone, with resident clients and a status-3 frame in the mix."""
    from altopir_b200 import server as srv
    monkeypatch.setenv("ALTO_PIPED_BYTES", "0")
    p = svc.Params(2 * 32768 + 8192, 4096)
    st = svc.SyntheticState.make(p, seed=151, full_prefix=True)
    e = eng.Engine.from_state(st)
    frames = [f for f in svc.synthetic_requests(p, 12, seed=152)]
    frames[5] = frames[5].copy()
    frames[5][9:13] = 0xFF  # y[0] >= Q: status 3
    rl = e.response_len()
    alone = []
    for f in frames:
        out = np.zeros((1, rl), dtype=np.uint8)
        status = np.full(1, -1, dtype=np.int32)
        e.answer([f], out, status)
        alone.append((int(status[0]), out[0].copy()))
    s = srv.Server(e, max_batch=8, queue_cap=64, slots=2)
    for rnd in range(3):  # the second and third rounds find the valid clients resident
        tickets = [(i, s.submit(frames[i])) for i in range(len(frames))]
        for i, t in tickets:
            code, resp = s.wait(t)
            assert code == alone[i][0], (rnd, i)
            if code == 0:
                assert np.array_equal(resp, alone[i][1]), (rnd, i)
    stats = s.stats()
    assert stats["failed"] == 0 and stats["resident_hits"] > 0
    s.close()
    e.close()
