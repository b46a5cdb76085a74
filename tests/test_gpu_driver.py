"""The GPU heatbath run driver (reference driver behaviour): input file, schedule, text outputs,
ILDG saves, and resume that continues the chain bit for bit."""
import os
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
