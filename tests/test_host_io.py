"""The driver's input-file front end and text formats (host C++, no GPU): the reference's keys,
defaults and quirks (src/io/io.cpp:434-481)."""
import os
import subprocess

import pytest

from conftest import ROOT

HOST = os.path.join(ROOT, "ecmc-qcb_b200", "host", "src")


@pytest.fixture(scope="module")
def dump(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("io") / "params_dump")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + HOST, os.path.join(ROOT, "tests", "cpp", "params_dump.cpp"),
                    os.path.join(HOST, "io", "io.cpp"), "-o", exe], check=True)
    return exe


def parse(exe, path):
    r = subprocess.run([exe, path], capture_output=True, text=True)
    return r.returncode, dict(line.split(" ", 1) for line in r.stdout.strip().splitlines())


def test_reference_keys_and_quirks(dump):
    rc, p = parse(dump, os.path.join(ROOT, "tests", "golden", "hb_input.txt"))
    assert rc == 0
    assert p["L_core"] == "4" and p["n_core_dims"] == "2"
    assert p["cold_start"] == "0"          # only the literal "true" is true: "hot" means a hot start
    assert p["N_therm"] == "3"             # key N_shift_therm
    assert p["N_samples"] == "1"           # forced to 1 whatever the file says
    assert p["N_hits"] == "2" and p["beta"] == "6"
    assert p["topo"] == "1" and p["N_steps_gf"] == "4"
    assert p["run_name"] == "hb8" and p["run_dir"] == "data"
    assert p["save_each_shifts"] == "3"
    assert p["format"] == "3.14"


def test_defaults_and_missing_file(dump, tmp_path):
    f = tmp_path / "empty.txt"
    f.write_text("# nothing\n")
    rc, p = parse(dump, str(f))
    assert rc == 0
    assert (p["L_core"], p["n_core_dims"], p["cold_start"], p["seed"]) == ("6", "2", "1", "123")
    assert (p["N_switch_eo"], p["N_shift"], p["N_therm"], p["N_rk_steps"]) == ("3", "2", "100", "40")
    rc, _ = parse(dump, str(tmp_path / "missing.txt"))
    assert rc == 3


def test_reference_signature_program_compiles_and_links(tmp_path):
    """A C++ program written against the reference's declarations (GaugeField, GeometryCB,
    mpi::heatbathcb::samples, GradientFlow, mpi::observables, ILDG, shift) compiles against
    host/src/ and links against libqcb_compat.a and libqcb.so: the drop-in boundary holds at build
    time, with no GPU.  Running it is the GPU test tests/test_gpu_compat.py."""
    pkg = os.path.join(ROOT, "ecmc-qcb_b200")
    exe = str(tmp_path / "compat_check")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I" + os.path.join(pkg, "host", "src"),
                        os.path.join(ROOT, "tests", "cpp", "compat_check.cpp"), os.path.join(pkg, "libqcb_compat.a"),
                        "-L" + pkg, "-lqcb", "-Wl,-rpath," + pkg, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert os.path.exists(exe)
