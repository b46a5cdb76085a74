"""The CPU oracle against the golden fixtures and analytic known answers (no GPU).

These tests pin the oracle to an independent numpy restatement (tests/golden/make_golden.py)
and to closed-form results.  Its pin to the reference's own compiled hot-path code is in
tests/test_ref_pin.py.
"""
import math
import os

import numpy as np
import pytest
import scipy.linalg as sla

from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_4444.npz")
TOL = 1e-12  # FP64 parity tolerance (relative)


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN)
    return {k: g[k] for k in g.files}


def test_philox_known_answers(orc):
    # Random123 known-answer vectors for philox4x32-10
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_golden_staples_plaquette_clover(orc, golden):
    L = tuple(int(v) for v in golden["L"])
    U = np.ascontiguousarray(golden["U"])
    for mu in range(4):
        assert rel_err(orc.staple_field(U, L, mu), golden["staple"][mu]) < TOL
    assert abs(orc.plaquette(U, L) - golden["plaq"]) < TOL * abs(golden["plaq"]) + 1e-15
    Q, E = orc.clover_qe(U, L)
    assert abs(Q - golden["Q"]) < TOL * max(1.0, abs(golden["Q"]))
    assert abs(E - golden["E"]) < TOL * golden["E"]


def test_golden_flow(orc, golden):
    L = tuple(int(v) for v in golden["L"])
    U = np.ascontiguousarray(golden["U"])
    assert rel_err(orc.flow_rk3(U, L, 0.02, 1), golden["U_rk3"]) < TOL
    tqe = orc.flow_measure(U, L, 0.02, 4, 2)
    assert np.allclose(tqe[:, 0], golden["tQE"][:, 0], rtol=0, atol=1e-15)
    assert np.max(np.abs(tqe[:, 1] - golden["tQE"][:, 1])) < TOL
    assert rel_err(tqe[:, 2], golden["tQE"][:, 2]) < TOL


def test_golden_heatbath(orc, golden):
    L = tuple(int(v) for v in golden["L"])
    U = np.array(golden["U"])
    orc.hb_subsweep(U, L, 6.0, 2, 12345, 3, 0, 1)
    assert rel_err(U, golden["U_hb"]) < TOL


def test_refcost_sweep_is_identical(orc):
    """Recomputing the staple per hit (the reference's cost structure) changes no bit."""
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, 5)
    a, b = U.copy(), U.copy()
    orc.hb_sweep(a, L, 6.0, 2, 77, 0)
    orc.hb_sweep(b, L, 6.0, 2, 77, 0, refcost=True)
    assert np.array_equal(a, b)


def test_thread_count_independence(orc):
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, 9)
    res = []
    for n in (1, 3):
        orc.set_threads(n)
        W = U.copy()
        orc.hb_sweep(W, L, 5.8, 1, 1, 2)
        res.append((W, orc.plaquette(W, L), orc.clover_qe(W, L)))
    orc.set_threads(0)
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1] and res[0][2] == res[1][2]


def test_cold_start_known_answers(orc):
    L = (4, 4, 4, 4)
    U = orc.cold_start(L)
    assert orc.plaquette(U, L) == 1.0
    assert orc.clover_qe(U, L) == (0.0, 0.0)
    W = orc.flow_rk3(U, L, 0.02, 3)
    assert np.array_equal(W, U)  # a flat field is a fixed point of the flow


def test_abelian_plaquette(orc):
    """U_mu(x) = diag(e^{i th_mu x_nu...}): constant field strength, closed-form plaquette."""
    L = (4, 4, 4, 4)
    V = 256
    U = np.zeros((V, 4, 3, 3), complex)
    th = 2 * math.pi / 4  # flux quantum: one unit of flux through each (0,1) plane
    for s in range(V):
        x = s % 4
        y = (s // 4) % 4
        for mu in range(4):
            U[s, mu] = np.eye(3)
        # U_1(x) = exp(i th x lambda), lambda = diag(1,-1,0); U_0 = 1 except at x = L-1 to close the flux
        ph = th * x
        U[s, 1] = np.diag([np.exp(1j * ph), np.exp(-1j * ph), 1.0])
        if x == 3:
            U[s, 0] = np.diag([np.exp(-1j * th * 4 * y), np.exp(1j * th * 4 * y), 1.0])
    # every (0,1) plaquette carries phase e^{i th} on (1,1) and e^{-i th} on (2,2)
    p01 = (2 * math.cos(th) + 1) / 3
    expected = (p01 + 5 * 1.0) / 6
    assert abs(orc.plaquette(U, L) - expected) < 1e-14


def test_exp_su3_against_pade(orc):
    rng = np.random.default_rng(3)
    for c in (0.01, 0.25, 1.0):
        for _ in range(5):
            A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
            Z = orc.proj_lie_su3(A) * 0.3
            assert np.max(np.abs(orc.exp_su3(Z, c) - sla.expm(c * Z))) < 1e-13


def test_exp_su3_diagonal_closed_form(orc):
    a, b = 0.3, -0.7
    Z = np.diag([1j * a, 1j * b, -1j * (a + b)])
    assert np.max(np.abs(orc.exp_su3(Z, 1.0) - np.diag(np.exp(np.diag(Z))))) < 1e-15


def test_proj_lie_properties(orc):
    rng = np.random.default_rng(4)
    A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    Z = orc.proj_lie_su3(A)
    assert np.max(np.abs(Z + Z.conj().T)) == 0.0
    assert abs(np.trace(Z)) < 1e-15


def test_hot_start_unitary_and_haar_moments(orc):
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, 7)
    mx, mean = orc.unitarity(U, L)
    assert mx < 1e-14
    det = np.linalg.det(U.reshape(-1, 3, 3))
    assert np.max(np.abs(det - 1)) < 1e-14
    tr = np.trace(U.reshape(-1, 3, 3), axis1=1, axis2=2)
    # Haar SU(3): E[tr U] = 0, E[|tr U|^2] = 1
    assert abs(tr.mean()) < 5 / math.sqrt(tr.size)
    assert abs((np.abs(tr) ** 2).mean() - 1) < 0.1


def random_gauge(rng, V):
    z = rng.normal(size=(V, 3, 3)) + 1j * rng.normal(size=(V, 3, 3))
    q, r = np.linalg.qr(z)
    q = q * (np.diagonal(r, axis1=1, axis2=2) / np.abs(np.diagonal(r, axis1=1, axis2=2)))[:, None, :]
    q[:, :, 2] /= np.linalg.det(q)[:, None]
    return q


def neighbour(L, s, mu):
    c = [s % L[0], (s // L[0]) % L[1], (s // (L[0] * L[1])) % L[2], s // (L[0] * L[1] * L[2])]
    c[mu] = (c[mu] + 1) % L[mu]
    return ((c[3] * L[2] + c[2]) * L[1] + c[1]) * L[0] + c[0]


def test_gauge_invariance(orc):
    """P, Q, E are invariant under U_mu(x) -> g(x) U_mu(x) g(x+mu)^dag (a correct transformation,
    unlike the reference's GaugeField::gauge_transform, GaugeField.cpp:100-114)."""
    L = (4, 4, 4, 4)
    V = 256
    U = orc.hot_start(L, 11)
    orc.hb_sweep(U, L, 6.0, 1, 1, 0)
    g = random_gauge(np.random.default_rng(5), V)
    W = np.empty_like(U)
    for s in range(V):
        for mu in range(4):
            W[s, mu] = g[s] @ U[s, mu] @ g[neighbour(L, s, mu)].conj().T
    assert abs(orc.plaquette(W, L) - orc.plaquette(U, L)) < 1e-13
    q0, e0 = orc.clover_qe(U, L)
    q1, e1 = orc.clover_qe(W, L)
    assert abs(q0 - q1) < 1e-12 and abs(e0 - e1) < 1e-12 * e0


def test_shift_translation_invariance(orc):
    L = (4, 6, 4, 2)
    U = orc.hot_start(L, 13)
    W = U.copy()
    orc.shift(W, L, [1, 2, 3, 1])
    assert abs(orc.plaquette(W, L) - orc.plaquette(U, L)) < 1e-14
    # U'(x) = U(x - s): site 0 of W holds what site (-1,-2,-3,-1) held
    src = ((1 * L[2] + 1) * L[1] + 4) * L[0] + 3
    assert np.array_equal(W[0], U[src])
    s = orc.random_shift_draw(12345, 7, L)
    assert all(0 <= s[d] < L[d] for d in range(4))
    s4 = orc.random_shift_draw(12345, 7, L, max_shift=4)
    assert all(0 <= v < 4 for v in s4)


def test_heatbath_unitarity_and_acceptance(orc):
    L = (4, 4, 4, 4)
    U = orc.cold_start(L)
    for sweep in range(20):
        orc.hb_sweep(U, L, 6.0, 1, 12345, sweep)
    mx, _ = orc.unitarity(U, L)
    assert mx < 1e-12  # ||U^dag U - 1|| < 1e-12 without reprojection
    assert 0.55 < orc.plaquette(U, L) < 0.65


def test_projection_su3(orc):
    rng = np.random.default_rng(6)
    M = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    P = orc.projection_su3(M)
    assert np.max(np.abs(P @ P.conj().T - np.eye(3))) < 1e-14
    assert abs(np.linalg.det(P) - 1) < 1e-14


def test_clover_halves_from_staple_differences(orc):
    """The measured flow's clover (k_flow_stage1_meas + k_clover_halves) rests on this identity: with
    D(y) the forward minus the backward staple of link (y, mu) in plane nu (the oracle's staple
    terms), acc(sum of the four leaves of x) = acc(U_mu(x) D(x)) + acc(D(x - mu) U_mu(x - mu)), where
    acc(M) = (M_ij - conj(M_ji) for i < j, Im M_ii).  From the nu links the same plane comes with the
    orientation reversed and the sign of acc flipped."""
    L = (4, 6, 2, 4)
    U = orc.hot_start(L, 17)
    V = int(np.prod(L))

    def co(i):
        c = []
        for d in range(4):
            c.append(i % L[d])
            i //= L[d]
        return c

    def mv(i, d, s):
        c = co(i)
        c[d] = (c[d] + s) % L[d]
        return c[0] + L[0] * (c[1] + L[1] * (c[2] + L[2] * c[3]))

    def dag(m):
        return m.conj().T

    def acc(m):
        return np.array([m[0, 1] - np.conj(m[1, 0]), m[0, 2] - np.conj(m[2, 0]), m[1, 2] - np.conj(m[2, 1]),
                         m[0, 0].imag, m[1, 1].imag, m[2, 2].imag])

    def leaves(x, mu, nu):  # observables_mpi.cpp:66-90, the four leaves in the reference's order
        xm, xn, xmm, xmn = mv(x, mu, 1), mv(x, nu, 1), mv(x, mu, -1), mv(x, nu, -1)
        return (U[x, mu] @ U[xm, nu] @ dag(U[xn, mu]) @ dag(U[x, nu])
                + U[x, nu] @ dag(U[mv(xmm, nu, 1), mu]) @ dag(U[xmm, nu]) @ U[xmm, mu]
                + dag(U[xmm, mu]) @ dag(U[mv(xmm, nu, -1), nu]) @ U[mv(xmm, nu, -1), mu] @ U[xmn, nu]
                + dag(U[xmn, nu]) @ U[xmn, mu] @ U[mv(xm, nu, -1), nu] @ dag(U[x, mu]))

    def D(y, mu, nu):  # compute_staple's two terms of plane nu (GaugeField.cpp:74-97)
        sf = U[mv(y, mu, 1), nu] @ dag(U[mv(y, nu, 1), mu]) @ dag(U[y, nu])
        sb = dag(U[mv(mv(y, mu, 1), nu, -1), nu]) @ dag(U[mv(y, nu, -1), mu]) @ U[mv(y, nu, -1), nu]
        return sf - sb

    err = 0.0
    for x in range(V):
        for mu in range(4):
            for nu in range(mu + 1, 4):
                a = acc(leaves(x, mu, nu))
                y, z = mv(x, mu, -1), mv(x, nu, -1)
                b = acc(U[x, mu] @ D(x, mu, nu)) + acc(D(y, mu, nu) @ U[y, mu])
                c = -(acc(U[x, nu] @ D(x, nu, mu)) + acc(D(z, nu, mu) @ U[z, nu]))
                err = max(err, np.abs(a - b).max(), np.abs(a - c).max())
    assert err < 1e-13
