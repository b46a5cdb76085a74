"""The GPU heatbath run driver (reference driver behaviour): input file, schedule, text outputs,
ILDG saves, and resume that continues the chain bit for bit."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "ecmc-qcb_b200", "qcb_hb_cb")

INPUT = """#Lattice params
L_core=4
n_core_dims=2
cold_start=false
seed=12345
N_shift_therm = 2
N_shift={n_shift}
N_switch_eo=2
beta = 6.0
N_sweeps = 1
N_hits = 1
N_shift_plaquette = 1
topo = true
N_shift_topo = 2
N_steps_gf = 3
N_rk_steps = 1
run_name = r
run_dir = {run_dir}
save_each_shifts = {save_each}
"""


def drive(tmp, n_shift, save_each, name):
    inp = tmp / f"{name}.txt"
    inp.write_text(INPUT.format(n_shift=n_shift, run_dir=str(tmp / name), save_each=save_each))
    r = subprocess.run([DRIVER, str(inp)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout[-2000:]
    return r.stdout


def test_run_outputs(gpu, tmp_path):
    out = drive(tmp_path, 4, 2, "a")
    d = tmp_path / "a" / "r"
    plaq = (d / "r_plaquette.txt").read_text().splitlines()
    assert len(plaq) == 4 and all(len(x.split(".")[1]) == 10 for x in plaq)
    assert all(0.4 < float(x) < 0.7 for x in plaq)
    topo = [l.split() for l in (d / "r_topo.txt").read_text().splitlines()]
    assert len(topo) == 2 * 3 and all(len(t) == 3 for t in topo)
    assert [float(t[0]) for t in topo[:3]] == [0.0, 0.02, 0.04]
    params = (d / "r_params.txt").read_text()
    assert "Saved shift 2" in params and "Saved shift 4" in params and "Saved final state !" in params
    assert gpu.ildg_probe(str(d / "r")) == ((8, 8, 8, 8), 64)
    assert "Shift (" in out and "Elapsed time" in out
    f = gpu.GaugeField((8, 8, 8, 8))
    f.read_ildg(str(d / "r"))
    assert abs(f.plaquette() - float(plaq[-1])) < 1e-9


def test_resume_continues_the_chain(gpu, tmp_path):
    drive(tmp_path, 4, 100, "whole")
    drive(tmp_path, 2, 100, "split")
    out = drive(tmp_path, 2, 100, "split")
    assert "Resuming" in out
    a = open(tmp_path / "whole" / "r" / "r", "rb").read()
    b = open(tmp_path / "split" / "r" / "r", "rb").read()
    assert a == b


CONFIG1 = """L_core=4
n_core_dims=2
cold_start=true
seed=12345
N_shift_therm = 100
N_shift=50
N_switch_eo=2
beta = 6.0
N_sweeps = 1
N_hits = 1
N_shift_plaquette = 1
topo = true
N_shift_topo = 10
N_steps_gf = 51
N_rk_steps = 1
run_name = c1
run_dir = {run_dir}
save_each_shifts = 1000
"""


def test_config1_run_matches_oracle_replay(gpu, orc, tmp_path):
    """The small reference configuration end to end: 8^4 cold start, beta 6.0, N_hits 1, N_switch_eo 2,
    100 thermalisation + 50 measured shifts, plaquette every shift, flow to t = 1.0 (51 points) every
    10th shift.  The oracle replays the same schedule -- the shifts the driver printed, its Philox key
    (from the saved heatbath state) and one sweep index per parity call -- and the driver's plaquette
    series and t Q E files must agree with it to 1e-10 (the files hold 10 decimals)."""
    inp = tmp_path / "c1.txt"
    inp.write_text(CONFIG1.format(run_dir=str(tmp_path / "run")))
    r = subprocess.run([DRIVER, str(inp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout[-2000:]
    d = tmp_path / "run" / "c1"
    shifts = [tuple(int(v) for v in m) for m in re.findall(r"Shift \((\d+), (\d+), (\d+), (\d+)\)", r.stdout)]
    assert len(shifts) == 150
    state = dict(line.split() for line in open(next(d.rglob("c1_hb_state.txt"))).read().splitlines())
    key = int(state["philox_key"])
    assert int(state["next_sweep"]) == 150 * 2 * 2

    L = (8, 8, 8, 8)
    U = orc.cold_start(L)
    k = 0
    plaq, tqe = [], []
    for i, s in enumerate(shifts):
        orc.shift(U, L, s)
        for _ in range(2):  # N_switch_eo x samples(even): N_sweeps x (sweep EV; sweep OD)
            for p in (0, 1):
                for mu in range(4):
                    orc.hb_subsweep(U, L, 6.0, 1, key, k, p, mu)
                k += 1
        if i >= 100:
            plaq.append(orc.plaquette(U, L))
            if (i - 100) % 10 == 0:
                tqe.append(orc.flow_measure(U, L, 0.02, 51, 1))
    got_p = np.array([float(x) for x in (d / "c1_plaquette.txt").read_text().split()])
    got_t = np.array([[float(v) for v in line.split()] for line in (d / "c1_topo.txt").read_text().splitlines()])
    want_t = np.concatenate(tqe)
    assert got_p.shape == (50,) and got_t.shape == (5 * 51, 3)
    dp = float(np.max(np.abs(got_p - np.array(plaq))))
    dt = float(np.max(np.abs(got_t - want_t)))
    assert dp < 1e-10 and dt < 1e-10, (dp, dt)
