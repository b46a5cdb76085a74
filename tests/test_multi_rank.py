"""bench.py --gpus N runs independent replicas (one lattice per rank, no data-path collective): the
rank plumbing it uses -- process-group set-up, barrier, max-over-ranks timing, the weak-scaling
aggregate and the reference arm's rank-0-only rule -- exercised as two gloo ranks on the CPU, each
advancing its own seeded lattice with the CPU restatement."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    r, w, _ = bench.dist_setup(world, backend="gloo")
    orc = bench.load_oracle()
    orc.set_threads(1)
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, 100 + r)  # each replica its own seed
    orc.hb_sweep(U, L, 6.0, 1, 100 + r, 0)
    ms = 10.0 * (r + 1)  # per-rank "duration": the job time is the slowest rank's
    bench.barrier(w)
    mx = bench.max_over_ranks(ms, w)
    out.put((r, w, mx, orc.plaquette(U, L), bench.replica_rate(1000.0, mx, w)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert all(x[2] == 20.0 for x in res)  # max over ranks on every rank
    assert res[0][3] != res[1][3]  # independent replicas
    assert all(x[4] == pytest.approx(2 * 1000.0 / 0.020) for x in res)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, gpus = 1, 0, 2

    assert bench.run_reference(Args, rank=1, world=2) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_json_line():
    """The reference arm prints one JSON line with the bench contract's keys, timing the reference's
    own heatbath (oracle/_ref) on the host cores for the same workload, step, metric and unit as the
    CUDA arm."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "link-upd/s" and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "hb_fp64_32^4" and d["dtype"] == "f64" and d["vs_baseline"] is None
    assert d["config"]["step"].startswith("one full checkerboard sweep") and "parallelism" in d["config"]
    cb = d["cpu_baseline"]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref

    assert cb["kind"] == ("reference" if ref.available() else "port")
    assert cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "link-upd/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_clock_summary_parses_nvidia_smi_lines():
    """The clock sampler's reading of nvidia-smi's csv,noheader,nounits lines: median SM clock,
    max clock, the reasons seen active at any sample; malformed samples are skipped."""
    import tempfile

    sys.path.insert(0, ROOT)
    import bench

    c = bench.Clocks.__new__(bench.Clocks)
    c.proc = object()
    c.f = tempfile.TemporaryFile(mode="w+")
    c.f.write("0, 1950, 1965, 980.12, 0x0000000000000004, Not Active, Not Active, Not Active, Active\n"
              "0, [N/A], 1965, 990.00, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active\n"
              "0, 1890, 1965, 1001.50, 0x0000000000000008, Active, Not Active, Not Active, Not Active\n"
              "garbage\n")
    s = c.summary()
    assert s == {"sm_mhz": 1920.0, "sm_max_mhz": 1965.0, "reasons": ["hw_slowdown", "sw_power_cap"],
                 "samples": 2}
    c.proc = None
    assert c.summary()["reasons"] == ["nvidia-smi unavailable"]
