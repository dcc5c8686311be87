"""Loading the database straight into the engine's device tiles (alto_engine_new_empty, alto_engine_load_records,
alto_engine_load_file): the engine answers exactly as one built from the column-order database, for records loaded
in uneven pieces that straddle the 128-record tile grid, and for a record-major file shorter than the database (the
reference's streaming reader pads the remaining records with zeros, src/server.rs:380-500)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _empty_like(eng, st):
    p = st.p
    return eng.Engine.empty(p.rows, p.record_bytes, st.ub, p.n, p.tg, st.prefixes, p.row1_off, 1 << p.q1_bits,
                            p.q1_bits, st.that, st.inv_table)


def _answer(e, frames):
    b = len(frames)
    out = np.zeros((b, e.response_len()), dtype=np.uint8)
    status = np.full(b, -1, dtype=np.int32)
    r, _ = e.answer([frames[i] for i in range(b)], out, status)
    assert r == b
    return out


def test_records_loaded_in_pieces_answer_like_the_column_order_database(gpu, svc, eng):
    p = svc.params(4096, 8192)
    st = svc.SyntheticState.make(p, seed=91, full_prefix=True)
    frames = svc.synthetic_requests(p, 6, seed=92)
    full = eng.Engine.from_state(st)
    want = _answer(full, frames)
    full.close()
    e = _empty_like(eng, st)
    assert e.request_len() == svc.request_len(p)
    for a, b in ((3000, 4096), (0, 1000), (1000, 1100), (1100, 3000)):  # uneven, out of order, off the tile grid
        e.load_records(st.db_col[:, a:b].T, a)
    assert np.array_equal(_answer(e, frames), want)
    # reloading a run with other bytes changes the answer; loading the originals back restores it
    e.load_records(np.zeros((300, p.record_bytes), dtype=np.uint8), 2000)
    assert not np.array_equal(_answer(e, frames), want)
    e.load_records(st.db_col[:, 2000:2300].T, 2000)
    assert np.array_equal(_answer(e, frames), want)
    with pytest.raises(eng.EngineError):
        e.load_records(st.db_col[:, :200].T, 4000)  # runs past the database
    e.close()


def test_record_file_shorter_than_the_database_reads_as_zero_padded(gpu, oracle, svc, eng, tmp_path):
    p = svc.params(4096, 8192)
    st = svc.SyntheticState.make(p, seed=93, full_prefix=True)
    real = 2500
    path = tmp_path / "db.bin"
    svc.write_record_file(path, st.db_col, real)
    assert path.stat().st_size == real * p.record_bytes
    e = _empty_like(eng, st)
    e.load_file(path, real)
    frames = svc.synthetic_requests(p, 5, seed=94)
    got = _answer(e, frames)
    st.db_col[:, real:] = 0  # what the reference's reader leaves past the real records
    full = eng.Engine.from_state(st)
    assert np.array_equal(got, _answer(full, frames))
    full.close()
    r, status, oout = oracle.answer(st, [frames[i] for i in range(5)])
    assert np.array_equal(got, oout)
    with pytest.raises(eng.EngineError):
        e.load_file(tmp_path / "missing.bin", real)
    with pytest.raises(eng.EngineError):
        e.load_file(path, real + 128)  # the file is short
    e.close()


def test_database_and_frames_generated_on_the_device_equal_the_host_generators(gpu, svc, eng, oracle):
    """alto_engine_fill_synthetic writes the synthetic records into the tiles (including a record count off the
    128-record grid, whose padding records stay zero) and alto_synthetic_requests_device writes the frames of
    alto_synthetic_request: the engine answers as one built from the host's column-order database."""
    import torch
    for rows, rb in ((4096, 8192), (8256, 4096)):
        p = svc.Params(rows, rb)
        st = svc.SyntheticState.make(p, seed=95)
        dev = svc.SyntheticState.make(p, seed=95, host_db=False)
        assert dev.db_col is None
        ql = svc.request_len(p)
        stride = (7 + ql + 255) // 256 * 256
        slots = torch.zeros((5, stride), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        svc.synthetic_requests_device(p, 5, 96, slots.data_ptr(), stride, first_client=3)
        frames = slots[:, 7:7 + ql].cpu().numpy()
        assert np.array_equal(frames, svc.synthetic_requests(p, 5, seed=96, first_client=3))
        full = eng.Engine.from_state(st)
        want = _answer(full, frames)
        full.close()
        e = eng.Engine.from_state(dev)
        assert np.array_equal(_answer(e, frames), want)
        e.close()
        r, _, ref = oracle.answer(st, [frames[i] for i in range(5)])
        assert r == 5 and np.array_equal(ref, want)
