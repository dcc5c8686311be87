"""Parity of the CUDA engine with the reference, through the C ABI (alto_answer): byte-for-byte against the golden
vectors the reference engine produced (tests/golden/) and against the oracle restatement on the same seeded
inputs.  Mirrors the reference's tests/engine.rs (responses, malformed and mutated frames, multi-block and chunked
batches) and adds the larger configurations of the benchmark."""
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, sha
import frames as fr

pytestmark = pytest.mark.gpu


def _engine(svc, eng, rows, rb, seed, full_prefix=False, keep_values=True):
    p = svc.params(rows, rb)
    st = svc.SyntheticState.make(p, seed=seed, full_prefix=full_prefix, keep_values=keep_values)
    return p, st, eng.Engine.from_state(st, threads=svc.threads())


def _answer(e, frames, fill=0):
    b = len(frames)
    out = np.full((b, e.response_len()), fill, dtype=np.uint8)
    status = np.full(b, -1, dtype=np.int32)
    n, stage = e.answer(frames, out, status)
    return n, status, out


def test_small_matches_golden_and_oracle(gpu, golden, oracle, svc, eng):
    g = golden["cases"]["small"]
    p, st, e = _engine(svc, eng, g["rows"], g["record_bytes"], g["state_seed"], g["full_prefix"])
    assert e.request_len() == svc.request_len(p) and e.response_len() == svc.response_len(p)
    req = svc.synthetic_requests(p, g["b"], seed=g["request_seed"])
    n, status, out = _answer(e, [req[i] for i in range(g["b"])])
    assert n == g["b"] and list(status) == g["status"]
    assert [sha(out[i]) for i in range(g["b"])] == g["sha256"]
    assert np.array_equal(out[0], np.fromfile(os.path.join(GOLDEN_DIR, "resp_small_0.bin"), dtype=np.uint8))
    r, ost, oout = oracle.answer(st, [req[i] for i in range(g["b"])])
    assert np.array_equal(out, oout)
    for method in (eng.Method.AMX, eng.Method.VNNI):
        out2 = np.zeros_like(out)
        status2 = np.full(g["b"], -1, dtype=np.int32)
        e.answer([req[i] for i in range(g["b"])], out2, status2, method)
        assert np.array_equal(out2, out)
    e.close()


def test_malformed_requests_are_rejected_like_the_decoder(gpu, golden, svc, eng):
    p, st, e = _engine(svc, eng, 2048, 4096, 3, True)
    g = golden["cases"]["malformed"]
    r0 = svc.synthetic_requests(p, 1, seed=g["request_seed"], first_client=0)[0]
    r1 = svc.synthetic_requests(p, 1, seed=g["request_seed"], first_client=1)[0]
    mf, want = fr.malformed_table(r0, r1, p.count)
    n, status, arena = _answer(e, mf, fill=0xA5)
    assert n == 2 and list(status) == want
    for c in range(1, 7):
        assert (arena[c] == 0xA5).all(), "a rejected buffer was written"
    assert [sha(arena[0]), sha(arena[7])] == g["sha256_valid"]
    # a NULL frame is status 1 as well
    frames_ = [None, r0]
    n, status, out = _answer(e, frames_, fill=0x5A)
    assert n == 1 and list(status) == [1, 0] and (out[0] == 0x5A).all()
    e.close()


def test_mutated_frames_agree_with_reference_statuses(gpu, golden, oracle, svc, eng):
    p, st, e = _engine(svc, eng, 2048, 4096, 3, True)
    gm = golden["cases"]["mutated"]
    base = [svc.synthetic_requests(p, 1, seed=gm["request_seed"], first_client=i)[0] for i in range(4)]
    for batch, want in zip(fr.mutated_batches(base, p.count), gm["status"]):
        n, status, out = _answer(e, batch, fill=0x33)
        assert list(status) == want
        assert n == sum(s == 0 for s in want)
        for i, s in enumerate(want):
            if s != 0:
                assert (out[i] == 0x33).all()
        ok = [i for i, s in enumerate(want) if s == 0]
        if ok:
            r, ost, oout = oracle.answer(st, [batch[i] for i in ok[:4]])
            assert np.array_equal(out[ok[:4]], oout)
    e.close()


def test_multi_block_and_chunked_batches_match_golden(gpu, golden, svc, eng):
    g = golden["cases"]["multiblock"]
    p, st, e = _engine(svc, eng, g["rows"], g["record_bytes"], g["state_seed"])
    for b, case in g["batches"].items():
        b = int(b)
        req = svc.synthetic_requests(p, b, seed=case["request_seed"])
        n, status, out = _answer(e, [req[i] for i in range(b)])
        assert n == b and (status == 0).all()
        assert sha(out) == case["sha256"], f"batch {b}"
    e.close()


def test_plain_small_config_matches_golden(gpu, golden, svc, eng):
    g = golden["cases"]["plain_2048x32k"]
    p, st, e = _engine(svc, eng, g["rows"], g["record_bytes"], g["state_seed"])
    req = svc.synthetic_requests(p, 1, seed=g["request_seed"])
    n, status, out = _answer(e, [req[0]])
    assert n == 1 and sha(out) == g["sha256"]
    e.close()


def test_each_response_is_the_same_alone_and_in_the_mix(gpu, oracle, svc, eng):
    p, st, e = _engine(svc, eng, 4096, 8192, 17, True)
    req = svc.synthetic_requests(p, 37, seed=18)
    frames_ = [req[i] for i in range(37)]
    n, status, mixed = _answer(e, frames_)
    assert n == 37
    for i in (0, 5, 36):
        n1, s1, alone = _answer(e, [frames_[i]])
        assert n1 == 1 and np.array_equal(alone[0], mixed[i])
    r, ost, oout = oracle.answer(st, frames_)
    assert np.array_equal(mixed, oout)
    # capacity shrinking and growing between calls
    for b in (3, 37, 1):
        n, status, out = _answer(e, frames_[:b])
        assert np.array_equal(out, mixed[:b])
    e.close()


def test_device_resident_path_matches_host_path(gpu, svc, eng):
    import torch
    p, st, e = _engine(svc, eng, 2048, 4096, 23)
    b = 9
    req = svc.synthetic_requests(p, b, seed=24)
    n, status, want = _answer(e, [req[i] for i in range(b)])
    stride = (7 + e.request_len() + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    slots[:, 7:7 + e.request_len()] = torch.from_numpy(req).cuda()
    slots[4, 7 + 9] = 0xFF  # key word out of range in frame 4: y[0] >= Q
    slots[4, 7 + 10:7 + 13] = 0xFF
    d_out = torch.zeros((b, e.response_len()), dtype=torch.uint8, device="cuda")
    st_dev = np.full(b, -1, dtype=np.int32)
    torch.cuda.synchronize()  # the engine's stream does not wait on torch's
    r = e.answer_device(slots.data_ptr(), stride, b, d_out.data_ptr(), e.response_len(), st_dev)
    torch.cuda.synchronize()
    assert r == b - 1 and list(st_dev) == [0, 0, 0, 0, 3, 0, 0, 0, 0]
    got = d_out.cpu().numpy()
    assert np.array_equal(np.delete(got, 4, 0), np.delete(want, 4, 0))
    assert (got[4] == 0).all()
    e.close()


@pytest.mark.slow
def test_1gb_batch_128_sampled_parts_match_oracle(gpu, oracle, svc, eng):
    # 32768 records x 32 KB (1 GiB), one batch of 128: every response against the reference engine when this host
    # can run it, and a seeded sample of response parts against the oracle restatement.
    from oracle.oracle import RefEngine, ref_methods
    p, st, e = _engine(svc, eng, 32768, 32768, 31)
    b = 128
    req = svc.synthetic_requests(p, b, seed=32)
    frames_ = [req[i] for i in range(b)]
    n, status, out = _answer(e, frames_)
    assert n == b and (status == 0).all()
    rng = np.random.default_rng(33)
    part = st.prefixes[0].size
    for c, o in zip(rng.integers(0, b, 10), rng.integers(0, p.instances, 10)):
        want = oracle.answer_part(st, frames_[c], int(o))
        assert np.array_equal(out[c, o * part:(o + 1) * part], want), (c, o)
    methods = ref_methods()
    if methods:
        ref = RefEngine(st)
        rr, rs, rout, _ = ref.answer(frames_, methods[0])
        assert rr == b and np.array_equal(rout, out)
        ref.close()
    e.close()


def test_every_plan_and_the_graph_path_return_identical_bytes(gpu, svc, eng):
    import torch
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=27)
    e = eng.Engine.from_state(st)
    b = 136
    frames = svc.synthetic_requests(p, b, seed=28)
    ql, rl = e.request_len(), e.response_len()
    stride = (7 + ql + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
    status = np.full(b, -1, dtype=np.int32)

    def run():
        out = torch.zeros((b, rl), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()  # the engine's stream does not wait on torch's
        assert e.answer_device(slots.data_ptr(), stride, b, out.data_ptr(), rl, status) == b
        return out.cpu().numpy()

    want = run()
    plans = [(b, 0, -1, 0, 0), (b, 1, 0, 64, 4), (b, 1, 0, 128, 24), (b, 1, 1, 256, 12), (b, 1, 0, 32, 6)]
    for plan in plans:
        e.set_tuning([plan])
        assert np.array_equal(run(), want), plan
    e.set_tuning([])
    e.set_graphs(True)
    for _ in range(3):  # capture on the first call, replay after
        assert np.array_equal(run(), want)
        assert e.last_launches() > 0  # a replay reports the kernels of its captured sequence
    for bb in (1, 5, 136):
        out = torch.zeros((bb, rl), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        e.enqueue_device(slots.data_ptr(), stride, bb, out.data_ptr(), rl)
        e.sync()
        assert np.array_equal(out.cpu().numpy(), want[:bb]), bb
    e.set_graphs(False)
    e.close()


def test_every_schedule_returns_identical_bytes(gpu, svc, eng, monkeypatch):
    # one stream or two (ALTO_OVERLAP), and 1..8 column groups for the device path (ALTO_GROUPS) and alto_answer
    # (ALTO_HOST_GROUPS, or group sizes as weights in ALTO_HOST_WEIGHTS, which wins; a malformed list is ignored);
    # the knobs are read when an engine is created
    import torch
    p = svc.params(4096, 32768)  # 16 response parts, so every group count divides
    st = svc.SyntheticState.make(p, seed=41)
    b = 24
    frames = svc.synthetic_requests(p, b, seed=42)
    frames[3, 9:13] = 0xFF  # y[0] >= Q: status 3
    want = None
    for overlap, groups, host_groups, weights in ((0, 1, 1, None), (1, 1, 1, None), (1, 2, 2, None), (1, 4, 4, None),
                                                  (1, 8, 8, None), (1, 2, 4, None), (1, 2, 4, "8,4,2,1,1"),
                                                  (1, 2, 4, "6,5,3,2"), (1, 2, 4, "1,1,1,1,1,1,1,1"),
                                                  (1, 2, 3, "3,x")):
        monkeypatch.setenv("ALTO_OVERLAP", str(overlap))
        monkeypatch.setenv("ALTO_GROUPS", str(groups))
        monkeypatch.setenv("ALTO_HOST_GROUPS", str(host_groups))
        if weights is None:
            monkeypatch.delenv("ALTO_HOST_WEIGHTS", raising=False)
        else:
            monkeypatch.setenv("ALTO_HOST_WEIGHTS", weights)
        e = eng.Engine.from_state(st)
        ql, rl = e.request_len(), e.response_len()
        n, status, host = _answer(e, [frames[i] for i in range(b)], fill=0x11)
        stride = (7 + ql + 15) // 16 * 16
        slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
        out = torch.full((b, rl), 0x11, dtype=torch.uint8, device="cuda")
        dstat = np.full(b, -1, dtype=np.int32)
        torch.cuda.synchronize()  # the engine's stream does not wait on torch's
        assert e.answer_device(slots.data_ptr(), stride, b, out.data_ptr(), rl, dstat) == b - 1
        assert n == b - 1 and status[3] == 3 and list(dstat) == list(status)
        dev = out.cpu().numpy()
        assert np.array_equal(dev, host) and (host[3] == 0x11).all()
        if want is None:
            want = host
        assert np.array_equal(host, want), (overlap, groups, host_groups, weights)
        e.close()


def test_narrow_tiles_return_the_oracles_bytes(gpu, oracle, svc, eng, monkeypatch):
    """The pair GEMMs' run-time tile width (multiples of 32 limb columns, ALTO_TILE_EXACT) against power-of-two
    tiles and the oracle, for batches whose limb columns fall just above a power of two and for several tiles."""
    p = svc.params(2048, 4096)
    st = svc.SyntheticState.make(p, seed=51)
    for b in (9, 33, 65, 72, 100, 200):
        frames = svc.synthetic_requests(p, b, seed=52 + b)
        outs = []
        for exact in ("1", "0"):
            monkeypatch.setenv("ALTO_TILE_EXACT", exact)
            e = eng.Engine.from_state(st)
            n, status, out = _answer(e, [frames[i] for i in range(b)])
            assert n == b and (status == 0).all()
            outs.append(out)
            e.close()
        assert np.array_equal(outs[0], outs[1]), b
        r, ost, oout = oracle.answer(st, [frames[i] for i in (0, b // 2, b - 1)])
        assert np.array_equal(outs[0][[0, b // 2, b - 1]], oout), b


def test_record_count_off_the_tile_grid_matches_oracle(gpu, oracle, svc, eng):
    # 2112 records: the last 128-record block of the tiled database is half padding, which must read as zero.  The
    # service layer only takes powers of two (as the reference's does); the engine's C ABI takes any multiple of 64.
    p = svc.Params(2112, 4096)
    st = svc.SyntheticState.make(p, seed=51, full_prefix=True)
    e = eng.Engine.from_state(st, threads=svc.threads())
    req = svc.synthetic_requests(p, 9, seed=52)
    frames_ = [req[i] for i in range(9)]
    n, status, out = _answer(e, frames_)
    assert n == 9 and (status == 0).all()
    r, ost, oout = oracle.answer(st, frames_)
    assert np.array_equal(out, oout)
    e.close()


@pytest.mark.parametrize("n,record_bytes", [(64, 4096), (256, 4096), (1024, 4096), (4096, 8192)])
def test_other_ring_dimensions_match_oracle(gpu, oracle, svc, eng, n, record_bytes):
    # the engine takes any power-of-two n in [16, 4096] (src/amx_kernels.cpp:551): the small-n tail, the
    # register-blocked tail at 2^8 .. 2^12 and the GEMM tilings other than the scheme's n = 2048.  Q - 1 = 2^12 (2^20 -
    # 3), so n = 4096 has no genuine negacyclic table; the engine and the oracle are exact for any table.
    p = svc.Params(2048, record_bytes, n=n, tg=4)
    st = svc.SyntheticState.make(p, seed=100 + n, full_prefix=True)
    e = eng.Engine.from_state(st)
    frames = svc.synthetic_requests(p, 9, seed=200 + n)
    frames[4, 9:13] = 0xFF  # y[0] >= Q: status 3
    n_ok, status, out = _answer(e, [frames[i] for i in range(9)], fill=0x77)
    r, ost, oout = oracle.answer(st, [frames[i] for i in range(9)])
    assert n_ok == r == 8 and list(status) == list(ost)
    ok = status == 0
    assert np.array_equal(out[ok], oout[ok]) and (out[4] == 0x77).all()
    e.close()


@pytest.mark.parametrize("tg,q1_bits", [(1, 10), (2, 12), (8, 10), (4, 20)])
def test_other_key_counts_and_row1_moduli_match_oracle(gpu, oracle, svc, eng, tg, q1_bits):
    # tg (key blocks: the pack's K = tg n and the tail's key switch) and the row-1 modulus q1 = 2^q1_bits (the
    # rescale and the bit packing of row 1; the engine takes q1 < 2^21), which the scheme fixes at 4 and 2^10
    class P(svc.Params):
        @property
        def q1_bits(self):
            return q1_bits

    p = P(2048, 4096, tg=tg)
    st = svc.SyntheticState.make(p, seed=300 + tg + q1_bits, full_prefix=True)
    e = eng.Engine.from_state(st)
    assert e.request_len() == 9 + 4 * (2 * tg * 2048 + 2048) and e.response_len() == 2 * p.part_len
    frames = svc.synthetic_requests(p, 6, seed=400 + tg)
    n_ok, status, out = _answer(e, [frames[i] for i in range(6)])
    r, ost, oout = oracle.answer(st, [frames[i] for i in range(6)])
    assert n_ok == r == 6 and np.array_equal(out, oout)
    e.close()


def test_batch_lanes_return_the_same_bytes(gpu, svc, eng):
    # alto_engine_set_lanes: consecutive enqueue_device batches rotate through 1..4 batch contexts and overlap on the
    # device; every batch's responses and statuses equal alto_answer's, with and without graph replay, and work put
    # on the engine's stream after alto_engine_fence (no host wait in between) sees every lane's results
    import torch
    p = svc.params(4096, 32768)
    st = svc.SyntheticState.make(p, seed=51)
    e = eng.Engine.from_state(st)
    ql, rl = e.request_len(), e.response_len()
    stride = (7 + ql + 15) // 16 * 16
    batches = []
    for j, b in enumerate((24, 17, 32)):
        frames = svc.synthetic_requests(p, b, seed=60 + j)
        if j == 1:
            frames[2, 9:13] = 0xFF  # y[0] >= Q: status 3
        want = np.full((b, rl), 0x11, dtype=np.uint8)
        wst = np.full(b, -1, dtype=np.int32)
        e.answer([frames[i] for i in range(b)], want, wst)
        slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
        batches.append((b, slots, want, wst))
    assert batches[1][3][2] == 3
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(e.stream())
    for graphs in (False, True):
        e.set_graphs(graphs)
        for lanes in (1, 2, 3, 4):
            e.set_lanes(lanes)
            for rep in range(2):
                outs = [torch.full((b, rl), 0x11, dtype=torch.uint8, device="cuda") for b, *_ in batches]
                stats = [torch.full((b,), -1, dtype=torch.int32, device="cuda") for b, *_ in batches]
                torch.cuda.synchronize()
                for (b, slots, _, _), out, s in zip(batches, outs, stats):
                    e.enqueue_device(slots.data_ptr(), stride, b, out.data_ptr(), rl, s.data_ptr())
                e.fence()
                with torch.cuda.stream(stream):
                    copies = [o.clone() for o in outs]
                    stat_copies = [s.clone() for s in stats]
                stream.synchronize()
                for (b, _, want, wst), c, sc in zip(batches, copies, stat_copies):
                    assert np.array_equal(c.cpu().numpy(), want), (graphs, lanes, rep, b)
                    assert list(sc.cpu().numpy()) == list(wst), (graphs, lanes, rep, b)
                e.sync()
    e.set_lanes(1)
    e.set_graphs(False)
    e.close()


@pytest.mark.parametrize("piped_bytes", ["0", str(1 << 40)])
def test_answer_over_several_record_chunks_pipelines_the_upload(gpu, oracle, svc, eng, monkeypatch, piped_bytes):
    """alto_answer over a database of six record chunks (the last one partial): with ALTO_PIPED_BYTES=0 the query
    words upload chunk group by chunk group and each group's scan starts as soon as its words are split (large
    batches do so by default), with a threshold above the batch they upload at once; the responses equal the device
    path's (one scan over all records) and the oracle's."""
    import torch
    monkeypatch.setenv("ALTO_PIPED_BYTES", piped_bytes)
    p = svc.Params(5 * 32768 + 8192, 4096)
    st = svc.SyntheticState.make(p, seed=131, full_prefix=True)
    e = eng.Engine.from_state(st)
    b = 6
    req = svc.synthetic_requests(p, b, seed=132)
    req[2, 9:13] = 0xFF  # y[0] >= Q: status 3, no response
    n, status, out = _answer(e, [req[i] for i in range(b)])
    assert n == b - 1 and list(status) == [0, 0, 3, 0, 0, 0]
    stride = (7 + e.request_len() + 15) // 16 * 16
    slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
    slots[:, 7:7 + e.request_len()] = torch.from_numpy(req).cuda()
    d_out = torch.zeros((b, e.response_len()), dtype=torch.uint8, device="cuda")
    dst = np.full(b, -1, dtype=np.int32)
    torch.cuda.synchronize()
    assert e.answer_device(slots.data_ptr(), stride, b, d_out.data_ptr(), e.response_len(), dst) == b - 1
    dev = d_out.cpu().numpy()
    ok = [c for c in range(b) if c != 2]
    assert np.array_equal(dev[ok], out[ok])
    part = st.prefixes[0].size
    want = oracle.answer_parts(st, [req[c] for c in ok], [c % p.instances for c in ok])
    for k, c in enumerate(ok):
        o = c % p.instances
        assert np.array_equal(out[c, o * part:(o + 1) * part], want[k]), c
    e.close()


def test_wide_pack_units_return_identical_bytes(gpu, svc, eng, monkeypatch):
    """ALTO_PACK_WIDE=1: pack units of 512 limb columns (two 256-column sub-accumulators over one read of each
    packing-matrix tile), for an even and an odd count of 256-column tiles, on the host and device paths."""
    import torch
    p = svc.params(2048, 8192)
    st = svc.SyntheticState.make(p, seed=141)
    e = eng.Engine.from_state(st)
    ql, rl = e.request_len(), e.response_len()
    for b in (128, 136):
        frames = svc.synthetic_requests(p, b, seed=142)
        monkeypatch.delenv("ALTO_PACK_WIDE", raising=False)
        n, status, want = _answer(e, [frames[i] for i in range(b)])
        assert n == b
        monkeypatch.setenv("ALTO_PACK_WIDE", "1")
        n, status, got = _answer(e, [frames[i] for i in range(b)])
        assert n == b and np.array_equal(got, want), b
        stride = (7 + ql + 15) // 16 * 16
        slots = torch.zeros((b, stride), dtype=torch.uint8, device="cuda")
        slots[:, 7:7 + ql] = torch.from_numpy(frames).cuda()
        out = torch.zeros((b, rl), dtype=torch.uint8, device="cuda")
        dst = np.full(b, -1, dtype=np.int32)
        torch.cuda.synchronize()
        assert e.answer_device(slots.data_ptr(), stride, b, out.data_ptr(), rl, dst) == b
        assert np.array_equal(out.cpu().numpy(), want), b
    monkeypatch.delenv("ALTO_PACK_WIDE", raising=False)
    e.close()


def test_tail_register_budgets_return_identical_bytes(gpu, oracle, svc, eng):
    """ALTO_TAIL_MINB (read once per process): the n = 2048 tail built for 1, 6 and 8 CTAs per SM answers the same
    frames with the oracle's bytes; each budget runs in a process of its own."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "import __graft_entry__ as ge; ge.load()\n"
        "from altopir_b200 import engine as eng, service as svc\n"
        "from oracle.oracle import Oracle\n"
        "eng.init(); p = svc.params(2048, 4096); st = svc.SyntheticState.make(p, seed=161, full_prefix=True)\n"
        "e = eng.Engine.from_state(st); f = svc.synthetic_requests(p, 9, seed=162)\n"
        "out = np.zeros((9, e.response_len()), dtype=np.uint8); s = np.full(9, -1, dtype=np.int32)\n"
        "assert e.answer([f[i] for i in range(9)], out, s)[0] == 9\n"
        "r, _, want = Oracle().answer(st, [f[i] for i in range(9)])\n"
        "assert np.array_equal(out, want); e.close(); print('OK')\n" % (ROOT, os.path.join(ROOT, "tests")))
    for minb in ("1", "6", "8"):
        env = dict(os.environ, ALTO_TAIL_MINB=minb)
        res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, env=env,
                             cwd=ROOT)
        assert res.returncode == 0 and "OK" in res.stdout, (minb, res.stderr[-2000:])
