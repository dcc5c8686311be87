"""The C++ host layer (include/altopir.hpp), the C++ counterpart of the reference's Rust host side for the answer
path: tests/cpp/test_host_api.cpp compiled here against the library.  On the CPU: parameter checks with the
reference's messages, wire lengths, the request codec and its errors, synthetic records, TiledDb, Method.  On the GPU:
an engine built through the C++ layer answers the golden case byte for byte.  The C++ client builds the Python
client's frames and decrypts; on the GPU the whole scheme (device offline set-up, requests, decryption) runs
through the C++ layer."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, sha

PKG = os.path.join(ROOT, "altopir-public_b200")


@pytest.fixture(scope="session")
def host_api_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "test_host_api")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "test_host_api.cpp"), "-L", PKG, "-laltopir_gpu",
           f"-Wl,-rpath,{PKG}", "-o", out]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return out


def test_cpp_host_layer_on_the_cpu(host_api_bin):
    res = subprocess.run([host_api_bin, "cpu"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0 and "OK" in res.stdout, res.stderr


@pytest.mark.gpu
def test_cpp_engine_answers_the_golden_case(gpu, golden, oracle, svc, host_api_bin, tmp_path):
    g = golden["cases"]["small"]
    p = svc.params(g["rows"], g["record_bytes"])
    st = svc.SyntheticState.make(p, seed=g["state_seed"], full_prefix=g["full_prefix"])
    frames = svc.synthetic_requests(p, g["b"], seed=g["request_seed"])
    np.ascontiguousarray(st.db_col[:, :p.rows]).tofile(tmp_path / "db_col.bin")
    st.ub.tofile(tmp_path / "ub.bin")
    np.stack([np.asarray(t, dtype=np.uint64) for t in st.that]).tofile(tmp_path / "that.bin")
    np.concatenate([np.asarray(x, dtype=np.uint8) for x in st.prefixes]).tofile(tmp_path / "prefixes.bin")
    np.asarray(st.inv_table, dtype=np.uint64).tofile(tmp_path / "inv.bin")
    frames.tofile(tmp_path / "frames.bin")
    (tmp_path / "meta.txt").write_text(f"{p.rows} {p.record_bytes} {g['b']}\n")
    res = subprocess.run([host_api_bin, "gpu", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and "OK" in res.stdout, res.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.uint8).reshape(g["b"], -1)
    status = np.fromfile(tmp_path / "status.bin", dtype=np.int32)
    assert list(status) == g["status"]
    assert [sha(out[i]) for i in range(g["b"])] == g["sha256"]
    r, ost, oout = oracle.answer(st, [frames[i] for i in range(g["b"])])
    assert np.array_equal(out, oout)


def test_modular_arithmetic_of_the_kernels(tmp_path):
    """modq.cuh, the mod-Q helpers the tail kernels and the host share, against 128-bit arithmetic (edge values and
    20 million seeded random cases per operation)."""
    out = str(tmp_path / "test_modq")
    res = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", os.path.join(ROOT, "tests", "cpp",
                                                                                       "test_modq.cpp"), "-o", out],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    res = subprocess.run([out], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and "OK" in res.stdout, res.stdout + res.stderr


def test_cpp_client_builds_the_python_clients_frames_and_decrypts(host_api_bin, client_mod, oracle, scheme_state,
                                                                  tmp_path):
    """The C++ client (include/altopir.hpp, client::Client) and the Python client with the same seed build the same
    frame byte for byte; the C++ client decrypts the response the oracle's engine gives over the scheme's state."""
    p = scheme_state.p
    seed, index = 0xC0FFEE, 1234
    (tmp_path / "meta.txt").write_text(f"{p.rows} {p.record_bytes} {seed} {index}\n")
    res = subprocess.run([host_api_bin, "client", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and "OK" in res.stdout, res.stderr
    frame = np.fromfile(tmp_path / "frame.bin", dtype=np.uint8)
    assert np.array_equal(frame, client_mod.Client(p, seed=seed).request(index))
    _, status, out = oracle.answer(scheme_state, [frame])
    assert list(status) == [0]
    out[0].tofile(tmp_path / "response.bin")
    res = subprocess.run([host_api_bin, "client", str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    rec = np.fromfile(tmp_path / "record.bin", dtype=np.uint8)
    assert np.array_equal(rec, oracle.synthetic_record(index, p.record_bytes))


@pytest.mark.gpu
def test_cpp_scheme_round_trip_on_the_gpu(gpu, host_api_bin):
    """Everything through the C++ layer: engine, device offline set-up, four clients' requests, decryption."""
    res = subprocess.run([host_api_bin, "scheme", "32768", "4096"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and "OK" in res.stdout, res.stdout + res.stderr
