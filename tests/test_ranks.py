"""The multi-GPU path of bench.py on CPU: two gloo ranks aggregate their timings the way `bench.py --gpus N` does
under torchrun (max over ranks, whole-job throughput), and non-zero ranks of the reference arm exit without work."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, times, out):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    m = bench.max_over_ranks(times[rank], world, device="cpu")
    dist.barrier()
    out[rank] = (m, bench.job_qps(world, 128, 10, m))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        times = [12.5, 17.25]
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, times, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert out[0] == out[1] == (17.25, 2 * 128 * 10 / 17.25e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"gpus": 2, "steps": 1, "warmup": 1, "rows": 2048, "record_bytes": 4096, "batch": 1})()
    assert bench.main_reference(args) == 0  # returns before touching any state or device


def test_reference_arm_never_loads_the_engine_library():
    """The reference arm builds its state and frames with the oracle's generators: the process maps only oracle/
    libraries, and its JSON line carries the same config as the GPU arm for the same arguments."""
    import json
    import subprocess
    code = (
        "import sys, json; sys.path.insert(0, %r); import bench\n"
        "a = bench.parse(['--impl', 'reference', '--rows', '2048', '--record-bytes', '4096', '--batch', '4',\n"
        "                 '--steps', '2', '--warmup', '3'])\n"
        "bench.MIN_TIMED_S = 0.05\n"
        "bench.main_reference(a)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'maps_engine': 'libaltopir_gpu' in maps, 'maps_ref': 'libalto_ref' in maps or\n"
        "                  'liboracle' in maps, 'config': bench.config_dict(a)}))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, check = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2 and line["warmup"] == 3
    assert line["config"] == check["config"]
    assert not check["maps_engine"] and check["maps_ref"]
