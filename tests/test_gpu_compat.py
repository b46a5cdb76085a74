"""The C++ layer with the reference's signatures (GaugeField, GeometryCB, heatbathcb::hit and
samples, GradientFlow, observables, ILDG, shift) against the oracle, through a compiled C++ program."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu

PKG = os.path.join(ROOT, "ecmc-qcb_b200")
HOST = os.path.join(PKG, "host", "src")


@pytest.fixture(scope="module")
def run(tmp_path_factory, gpu):
    d = tmp_path_factory.mktemp("compat")
    exe = str(d / "compat_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + HOST, os.path.join(ROOT, "tests", "cpp", "compat_check.cpp"),
                    os.path.join(PKG, "libqcb_compat.a"), "-L" + PKG, "-lqcb", "-Wl,-rpath," + PKG, "-o", exe],
                   check=True)
    r = subprocess.run([exe, str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        parts = line.split()
        if parts and parts[0] in ("hot_key", "plaq_hot", "halo_diff", "staple00", "hb_key", "hb_sweep", "plaq_hb",
                                  "tqe", "ildg_diff", "plaq_edit", "hit_key", "hit_staple",
                                  "members_vs_rk3", "clover_site", "local_qe", "levi"):
            out[parts[0]] = parts[1:]
    return d, out


def load(d, name):
    return np.fromfile(str(d / name), dtype=np.complex128).reshape(-1, 4, 3, 3)


def test_hot_start_and_host_views(run, orc):
    d, out = run
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, int(out["hot_key"][0]))
    assert rel_err(load(d, "hot.bin"), U) < 1e-12
    assert abs(float(out["plaq_hot"][0]) - orc.plaquette(U, L)) < 1e-12
    assert float(out["halo_diff"][0]) == 0.0
    A = orc.staple_field(U, L, 1)[0]
    assert abs(complex(float(out["staple00"][0]), float(out["staple00"][1])) - A[0, 0]) < 1e-12


def test_samples_and_flow(run, orc):
    d, out = run
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, int(out["hot_key"][0]))
    key = int(out["hb_key"][0])
    # samples(even) on the single even-parity rank: 2 x (sweep EV; sweep OD), sweep indices 0..3
    for k in range(4):
        for mu in range(4):
            orc.hb_subsweep(U, L, 6.0, 1, key, k, k % 2, mu)
    assert out["hb_sweep"][0] == "4"
    assert rel_err(load(d, "hb.bin"), U) < 1e-11
    assert abs(float(out["plaq_hb"][0]) - orc.plaquette(U, L)) < 1e-12
    tqe = np.array([float(x) for x in out["tqe"]]).reshape(-1, 3)
    ref = orc.flow_measure(load(d, "hb.bin"), L, 0.02, 3, 2)
    assert np.max(np.abs(tqe - ref)) < 1e-10


def test_ildg_edit_shift(run, orc):
    d, out = run
    L = (4, 4, 4, 4)
    assert float(out["ildg_diff"][0]) == 0.0
    E = load(d, "edit.bin")
    assert np.array_equal(E[0, 0], np.eye(3))  # halo'd site (1,1,1,1) is site 0 of the periodic lattice
    assert abs(float(out["plaq_edit"][0]) - orc.plaquette(E, L)) < 1e-12
    S = E.copy()
    orc.shift(S, L, [1, 2, 0, 3])
    assert np.array_equal(load(d, "shift.bin"), S)


def test_hit_with_reference_signature(run, orc):
    """mpi::heatbathcb::hit on one link: the staple left in A and the updated link against the oracle's
    update of that link (one hit, Philox key = the hit's draw of its std::mt19937_64, sweep 0); every
    other link unchanged."""
    d, out = run
    L = (4, 4, 4, 4)
    S = load(d, "shift.bin")
    A = np.array([float(x) for x in out["hit_staple"]]).view(np.complex128).reshape(3, 3)
    assert rel_err(A, orc.staple_field(S, L, 1)[1]) < 1e-12
    W = S.copy()
    orc.hb_subsweep(W, L, 6.0, 1, int(out["hit_key"][0]), 0, 1, 1)  # site 1 has parity 1
    H = load(d, "hit.bin")
    assert rel_err(H[1, 1], W[1, 1]) < 1e-12
    H[1, 1] = S[1, 1]
    assert np.array_equal(H, S)


def test_flow_members_and_site_observables(run, orc):
    """GradientFlow::compute_force / compute_w1-3 / replace_force_0 in rk3_step's order equal rk3_step;
    clover_site and local_q_e_clover at one site against the oracle; levi_civita."""
    d, out = run
    L = (4, 4, 4, 4)
    assert float(out["members_vs_rk3"][0]) < 1e-13
    H = load(d, "hit.bin")  # the field the C++ program measured
    F = np.array([float(x) for x in out["clover_site"]]).view(np.complex128).reshape(3, 3)
    assert np.max(np.abs(F.conj().T + F)) < 1e-14  # anti-Hermitian
    q, e = orc.clover_qe_density(H, L)
    assert abs(float(out["local_qe"][0]) - q[1]) < 1e-12 and abs(float(out["local_qe"][1]) - e[1]) < 1e-12 * e[1]
    assert out["levi"] == ["1", "-1", "0"]
