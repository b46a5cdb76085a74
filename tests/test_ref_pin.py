"""The restated CPU oracle against the reference's own hot-path code (no GPU).

Two pins:
  * tests/golden/ref_4444.npz, written by tests/golden/make_ref_golden.py from the reference's
    unchanged sources (always runs);
  * the reference library oracle/_ref/libqcb_ref.so itself, on 4^4, 6^4 and 8^4 lattices (runs
    where that library is built).

Tolerance: 1e-12 relative for links, staples, plaquette and E; Q, a signed sum near zero, within
1e-12 * max(1, sum_x |q(x)|).  The heatbath uses the CUDA path's Philox link streams on both sides
(the reference's std::mt19937_64 replaced by their replay), so its updates are compared link by
link, after single (parity, mu) sets and after chained sweeps.
"""
import os

import numpy as np
import pytest

from conftest import rel_err

TOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_4444.npz")


@pytest.fixture(scope="module")
def rg():
    g = np.load(GOLDEN)
    return {k: g[k] for k in g.files}


def q_tol(orc, U, L):
    q, _ = orc.clover_qe_density(U, L)
    return TOL * max(1.0, float(np.abs(q).sum()))


# ---------------------------------------------------------------- fixtures from the reference
def test_fixture_observables_and_staples(orc, rg):
    L = tuple(int(v) for v in rg["L"])
    U = np.ascontiguousarray(rg["U"])
    for mu in range(4):
        assert rel_err(orc.staple_field(U, L, mu), rg["staple"][mu]) < TOL
    assert abs(orc.plaquette(U, L) - rg["plaq"]) < TOL * abs(rg["plaq"])
    Q, E = orc.clover_qe(U, L)
    assert abs(Q - rg["Q"]) < q_tol(orc, U, L)
    assert abs(E - rg["E"]) < TOL * rg["E"]
    q, e = orc.clover_qe_density(U, L)
    assert np.max(np.abs(q - rg["q_site"])) < TOL * max(1.0, np.abs(rg["q_site"]).max())
    assert rel_err(e, rg["e_site"]) < TOL


def test_fixture_flow(orc, rg):
    L = tuple(int(v) for v in rg["L"])
    U = np.ascontiguousarray(rg["U"])
    assert rel_err(orc.flow_rk3(U, L, 0.02, 1), rg["U_rk3"]) < TOL
    tqe = orc.flow_measure(U, L, 0.02, 5, 2)
    assert np.array_equal(tqe[:, 0], rg["tQE"][:, 0])
    assert np.max(np.abs(tqe[:, 1] - rg["tQE"][:, 1])) < q_tol(orc, U, L)
    assert rel_err(tqe[:, 2], rg["tQE"][:, 2]) < TOL


def test_fixture_heatbath(orc, rg):
    L = tuple(int(v) for v in rg["L"])
    W = np.array(rg["U"], copy=True)
    orc.hb_subsweep(W, L, 6.0, 2, 12345, 3, 0, 1)
    assert rel_err(W, rg["U_hb_sub"]) < TOL
    W = np.array(rg["U"], copy=True)
    orc.hb_sweep(W, L, 6.0, 2, 12345, 3)
    assert rel_err(W, rg["U_hb_sweep"]) < TOL


def test_fixture_su3_pieces(orc, rg):
    for m, want in zip(rg["lie_in"], rg["lie_out"]):
        assert np.max(np.abs(orc.proj_lie_su3(m) - want)) < 1e-15
    for k, c in enumerate(rg["exp_coeff"]):
        for z, want in zip(rg["exp_in"], rg["exp_out"][k]):
            assert np.max(np.abs(orc.exp_su3(z, c) - want)) < 1e-15


# ---------------------------------------------------------------- the reference library, live
def _config(orc, L, seed):
    LL = (L,) * 4
    U = orc.hot_start(LL, seed)
    orc.hb_sweep(U, LL, 6.0, 2, seed + 1, 0)
    return LL, U


@pytest.mark.parametrize("L", [4, 6, 8])
def test_reference_stencils_and_observables(orc, refc, L):
    LL, U = _config(orc, L, 11)
    r = refc.RefLattice(L, U)
    assert np.array_equal(r.get(), U)
    for mu in range(4):
        assert rel_err(orc.staple_field(U, LL, mu), r.staple_field(mu)) < TOL
    assert abs(orc.plaquette(U, LL) - r.plaquette()) < TOL * abs(r.plaquette())
    Q, E = r.clover_qe()
    Qo, Eo = orc.clover_qe(U, LL)
    assert abs(Qo - Q) < q_tol(orc, U, LL)
    assert abs(Eo - E) < TOL * E
    q, e = r.clover_density()
    qo, eo = orc.clover_qe_density(U, LL)
    assert np.max(np.abs(qo - q)) < TOL * max(1.0, np.abs(q).max())
    assert rel_err(eo, e) < TOL


@pytest.mark.parametrize("L", [4, 6])
def test_reference_flow(orc, refc, L):
    LL, U = _config(orc, L, 21)
    r = refc.RefLattice(L, U)
    r.flow_rk3(0.02, 3)
    assert rel_err(orc.flow_rk3(U, LL, 0.02, 3), r.get()) < TOL
    r = refc.RefLattice(L, U)
    want = r.flow_measure(0.02, 6, 2)
    got = orc.flow_measure(U, LL, 0.02, 6, 2)
    assert np.array_equal(got[:, 0], want[:, 0])
    assert np.max(np.abs(got[:, 1] - want[:, 1])) < q_tol(orc, U, LL)
    assert rel_err(got[:, 2], want[:, 2]) < TOL


@pytest.mark.parametrize("L,nh", [(4, 1), (6, 2), (8, 2)])
def test_reference_heatbath_sets_link_by_link(orc, refc, L, nh):
    """Each (parity, mu) set of the reference's hit() against the oracle, from the same input."""
    LL, U = _config(orc, L, 31)
    r = refc.RefLattice(L)
    for p in range(2):
        for mu in range(4):
            r.set(U)
            r.hb_subsweep(6.0, nh, 777, 5, p, mu)
            W = U.copy()
            orc.hb_subsweep(W, LL, 6.0, nh, 777, 5, p, mu)
            assert rel_err(W, r.get()) < TOL, (p, mu)


@pytest.mark.parametrize("L", [4, 8])
def test_reference_heatbath_chained_sweeps(orc, refc, L):
    """Three chained sweeps: the oracle restates the reference's arithmetic, so no rounding
    difference compounds and the 1e-12 bound holds after every sweep."""
    LL, U = _config(orc, L, 41)
    r = refc.RefLattice(L, U)
    for s in range(3):
        r.hb_sweep(6.0, 2, 4242, s)
        orc.hb_sweep(U, LL, 6.0, 2, 4242, s)
        assert rel_err(U, r.get()) < TOL, s
    assert abs(orc.plaquette(U, LL) - r.plaquette()) < TOL


def test_reference_hit_returns_staple(orc, refc):
    """mpi::heatbathcb::hit leaves the link's staple in its SU3& argument."""
    LL, U = _config(orc, 4, 51)
    r = refc.RefLattice(4, U)
    lex, mu = 37, 2
    A = r.hb_link(lex, mu, 6.0, 2, 9, 1)
    assert rel_err(A, orc.staple_field(U, LL, mu)[lex]) < TOL


@pytest.mark.parametrize("s", [(1, 2, 3, 1), (0, 0, 4, 3), (5, 0, 1, 6)])
def test_reference_shift_and_projection(orc, refc, s):
    LL, U = _config(orc, 6, 61)
    r = refc.RefLattice(6, U)
    r.shift(s)
    W = U.copy()
    orc.shift(W, LL, s)
    assert np.array_equal(W, r.get())
    rng = np.random.default_rng(3)
    P = U + 1e-3 * (rng.normal(size=U.shape) + 1j * rng.normal(size=U.shape))
    r.set(P)
    r.projection()
    orc.reunitarize(P, LL)
    assert rel_err(P, r.get()) < TOL


def test_reference_su3_pieces(orc, refc):
    rng = np.random.default_rng(8)
    for _ in range(16):
        M = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        assert np.max(np.abs(orc.proj_lie_su3(M) - refc.proj_lie_su3(M))) < 1e-15
        Z = 0.5 * refc.proj_lie_su3(M)
        for c in (0.005, 0.25, 1.0):
            assert np.max(np.abs(orc.exp_su3(Z, c) - refc.exp_su3_luscher(Z, c))) < 1e-15


def test_reference_flow_member_passes(orc, refc):
    """GradientFlow's member passes in rk3_step's order (with its halo exchanges) are one RK3 step."""
    LL, U = _config(orc, 6, 71)
    r = refc.RefLattice(6, U)
    r.flow_passes(0.02, [0, 2, 1, 3, 4, 1, 5])
    assert rel_err(r.get(), orc.flow_rk3(U, LL, 0.02, 1)) < TOL


def test_reference_ildg_round_trip(orc, refc, tmp_path):
    """The reference's own save_ildg_clime / read_ildg_clime (LIME framing by the project's
    stand-in for c-lime): a written configuration reads back exactly; the file has the reference's
    two records (ildg-format MB=1 ME=1, ildg-binary-data MB=0 ME=1) and big-endian payload."""
    import struct

    LL, U = _config(orc, 4, 81)
    r = refc.RefLattice(4, U)
    path = r.ildg_write(str(tmp_path), "cfg")
    b = open(path, "rb").read()
    magic, ver, flags, n = struct.unpack(">IHHQ", b[:16])
    assert (magic, ver, flags >> 14) == (0x456789AB, 1, 3) and b[16:27] == b"ildg-format"
    off = 144 + ((n + 7) & ~7)
    magic, ver, flags, n2 = struct.unpack(">IHHQ", b[off:off + 16])
    assert flags >> 14 == 1 and b[off + 16:off + 32] == b"ildg-binary-data" and n2 == 256 * 72 * 8
    payload = np.frombuffer(b[off + 144:off + 144 + n2], dtype=">f8").astype(np.float64)
    assert np.array_equal(payload.view(np.complex128).reshape(U.shape), U)
    s = refc.RefLattice(4)
    s.ildg_read(str(tmp_path), "cfg")
    assert np.array_equal(s.get(), U)
