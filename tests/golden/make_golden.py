"""Generates tests/golden/golden_4444.npz with an independent numpy / pure-Python restatement.

    python tests/golden/make_golden.py

The reference (yacobozdalkiran/ECMC-QCB) ships no test vectors and cannot be compiled in this
image (Eigen, MPI and c-lime are absent), so these fixtures come from a second restatement of
its algorithms, written with numpy array shifts instead of the C++ oracle's per-site loops and
with scipy's Pade matrix exponential instead of the Cayley-Hamilton series.  The C++ oracle and
the CUDA library are both checked against them.

Contents (lattice L = (4,4,4,4), AoS order: site lexicographic with x fastest, mu, row-major 3x3):
  U        Haar-random SU(3) configuration (numpy PCG64 seed 2024, QR with phase fix, det = 1)
  staple   staples A_mu(x) for mu = 0..3, shape (4, V, 3, 3)       GaugeField.cpp:74-97
  plaq     mean plaquette                                            observables_mpi.cpp:11-48
  Q, E     clover charge and energy density                          observables_mpi.cpp:66-156
  U_rk3    U after one RK3 Wilson-flow step of eps = 0.02            gradient_flow.cpp:17-135
  tQE      topo_charge_flowed(N_steps_gf = 4, N_rk_steps = 2)        observables_mpi.cpp:159-186
  U_hb     U after one heatbath update of the (parity 0, mu 1) links, beta = 6.0, N_hits = 2,
           Philox4x32-10 link streams keyed on seed 12345, sweep 3    heatbath.cpp:8-44, heatbath_mpi.cpp:10-33
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.linalg as sla

L = (4, 4, 4, 4)
V = L[0] * L[1] * L[2] * L[3]
AX = {0: 3, 1: 2, 2: 1, 3: 0}  # direction mu -> array axis of the (t, z, y, x) grid


def grid(U):
    return U.reshape(L[3], L[2], L[1], L[0], 4, 3, 3)


def flat(G):
    return np.ascontiguousarray(G.reshape(V, 4, 3, 3))


def sh(A, mu, d):
    """A(x + d*mu) on the periodic grid."""
    return np.roll(A, -d, axis=AX[mu])


def dag(A):
    return np.conj(np.swapaxes(A, -1, -2))


def haar_su3(rng, n):
    z = (rng.normal(size=(n, 3, 3)) + 1j * rng.normal(size=(n, 3, 3))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    ph = np.diagonal(r, axis1=1, axis2=2)
    q = q * (ph / np.abs(ph))[:, None, :]
    det = np.linalg.det(q)
    q[:, :, 2] /= det[:, None]
    return q


def staples(G):
    out = []
    for mu in range(4):
        A = np.zeros(G.shape[:4] + (3, 3), dtype=complex)
        for nu in range(4):
            if nu == mu:
                continue
            Unu, Umu = G[..., nu, :, :], G[..., mu, :, :]
            A += sh(Unu, mu, 1) @ dag(sh(Umu, nu, 1)) @ dag(Unu)
            A += dag(sh(sh(Unu, mu, 1), nu, -1)) @ dag(sh(Umu, nu, -1)) @ sh(Unu, nu, -1)
        out.append(A)
    return out


def plaquette(G):
    s = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            Umu, Unu = G[..., mu, :, :], G[..., nu, :, :]
            P = Umu @ sh(Unu, mu, 1) @ dag(sh(Umu, nu, 1)) @ dag(Unu)
            s += np.trace(P, axis1=-2, axis2=-1).real.sum() / 3.0
    return s / (6.0 * V)


def clover(G, mu, nu):
    Umu, Unu = G[..., mu, :, :], G[..., nu, :, :]
    m = lambda A, d: sh(A, mu, d)  # noqa: E731
    n = lambda A, d: sh(A, nu, d)  # noqa: E731
    C = Umu @ m(Unu, 1) @ dag(n(Umu, 1)) @ dag(Unu)
    C = C + Unu @ dag(n(m(Umu, -1), 1)) @ dag(m(Unu, -1)) @ m(Umu, -1)
    C = C + dag(m(Umu, -1)) @ dag(n(m(Unu, -1), -1)) @ n(m(Umu, -1), -1) @ n(Unu, -1)
    C = C + dag(n(Unu, -1)) @ n(Umu, -1) @ n(m(Unu, 1), -1) @ dag(Umu)
    return (C - dag(C)) * 0.125


def clover_qe(G):
    F = {(a, b): clover(G, a, b) for a in range(4) for b in range(a + 1, 4)}
    tr = lambda A, B: np.trace(A @ B, axis1=-2, axis2=-1).real  # noqa: E731
    q = tr(F[0, 1], F[2, 3]) - tr(F[0, 2], F[1, 3]) + tr(F[0, 3], F[1, 2])
    e = 0.5 * sum((np.abs(f) ** 2).sum(axis=(-2, -1)) for f in F.values())
    return q.sum() / (4 * math.pi ** 2), e.sum() / V


def proj_lie(A):
    B = 0.5 * (A - dag(A))
    tr = np.trace(B, axis1=-2, axis2=-1) / 3.0
    return B - tr[..., None, None] * np.eye(3)


def expm_all(X):
    flatX = X.reshape(-1, 3, 3)
    return np.stack([sla.expm(x) for x in flatX]).reshape(X.shape)


def force(G):
    A = np.stack(staples(G), axis=4)
    return proj_lie(-(G @ A))


def rk3(G, eps):
    Z0 = force(G)
    W1 = expm_all(0.25 * eps * Z0) @ G
    Z1 = force(W1)
    W2 = expm_all((8.0 / 9.0) * eps * Z1 - (17.0 / 36.0) * eps * Z0) @ W1
    Z0b = (8.0 / 9.0) * Z1 - (17.0 / 36.0) * Z0
    Z2 = force(W2)
    return expm_all(0.75 * eps * Z2 - eps * Z0b) @ W2


# ---------------------------------------------------------------- heatbath (pure Python)
M32 = 0xFFFFFFFF


def philox(ctr, key):
    c = list(ctr)
    k0, k1 = key
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & M32
            k1 = (k1 + 0xBB67AE85) & M32
        p0 = 0xD2511F53 * c[0]
        p1 = 0xCD9E8D57 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & M32, p1 & M32, ((p0 >> 32) ^ c[3] ^ k1) & M32, p0 & M32]
    return c


class Stream:
    def __init__(self, seed, link, sweep, tag=0x48420001):
        self.key = (seed & M32, seed >> 32)
        self.ctr = [0, link, sweep, tag]
        self.buf = []

    def next(self):
        if not self.buf:
            o = philox(self.ctr, self.key)
            self.ctr[0] += 1
            u = lambda hi, lo: (((hi << 32) | lo) >> 11) * 2.0 ** -53  # noqa: E731
            self.buf = [u(o[0], o[1]), u(o[2], o[3])]
        return self.buf.pop(0)


def kp(beta, k, rng):
    alpha = beta * k * 2.0 / 3.0
    while True:
        delta, r1, r2, r3 = rng.next(), rng.next(), rng.next(), rng.next()
        c = math.cos(2 * math.pi * r2)
        lsq = -0.5 / alpha * (math.log(r1) + (c * c) * math.log(r3))
        if delta * delta <= 1.0 - lsq:
            a0 = 1.0 - 2.0 * lsq
            break
    rs = math.sqrt(1.0 - a0 * a0)
    phi = 2.0 * math.pi * rng.next()
    ct = 2.0 * rng.next() - 1.0
    st = math.sqrt(1.0 - ct * ct)
    return np.array([a0, rs * st * math.cos(phi), rs * st * math.sin(phi), rs * ct])


def qmult(q, p):
    return np.array([q[0] * p[0] - q[1] * p[1] - q[2] * p[2] - q[3] * p[3],
                     q[0] * p[1] + q[1] * p[0] + q[2] * p[3] - q[3] * p[2],
                     q[0] * p[2] - q[1] * p[3] + q[2] * p[0] + q[3] * p[1],
                     q[0] * p[3] + q[1] * p[2] - q[2] * p[1] + q[3] * p[0]])


def heatbath_links(U, parity, mu, beta, n_hits, seed, sweep):
    G = grid(U)
    A = staples(G)[mu].reshape(V, 3, 3)
    out = U.copy()
    for s in range(V):
        x = s % L[0]
        y = (s // L[0]) % L[1]
        z = (s // (L[0] * L[1])) % L[2]
        t = s // (L[0] * L[1] * L[2])
        if (x + y + z + t) % 2 != parity:
            continue
        rng = Stream(seed, s * 4 + mu, sweep)
        u = out[s, mu].copy()
        for _ in range(n_hits):
            for (i, j) in ((0, 1), (1, 2), (0, 2)):
                W = u @ A[s]
                w = np.array([(W[i, i] + W[j, j]).real / 2, (W[i, j] + W[j, i]).imag / 2,
                              (W[i, j] - W[j, i]).real / 2, (W[i, i] - W[j, j]).imag / 2])
                k = math.sqrt(float(w @ w))
                v = w / k
                r = qmult(kp(beta, k, rng), np.array([v[0], -v[1], -v[2], -v[3]]))
                R = np.eye(3, dtype=complex)
                R[i, i] = complex(r[0], r[3])
                R[j, j] = complex(r[0], -r[3])
                R[i, j] = complex(r[2], r[1])
                R[j, i] = complex(-r[2], r[1])
                u = R @ u
        out[s, mu] = u
    return out


def main():
    rng = np.random.default_rng(2024)
    U = haar_su3(rng, V * 4).reshape(V, 4, 3, 3)
    G = grid(U)
    st = np.stack([a.reshape(V, 3, 3) for a in staples(G)])
    plaq = plaquette(G)
    Q, E = clover_qe(G)
    U1 = flat(rk3(G, 0.02))
    tqe = []
    W, t = G, 0.0
    for step in range(4):
        q, e = clover_qe(W)
        tqe.append((t, q, e))
        if step != 3:
            for _ in range(2):
                W = rk3(W, 0.02)
                t += 0.02
    Uhb = heatbath_links(U, 0, 1, 6.0, 2, 12345, 3)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_4444.npz")
    np.savez_compressed(out, L=np.array(L), U=U, staple=st, plaq=plaq, Q=Q, E=E, U_rk3=U1, tQE=np.array(tqe),
                        U_hb=Uhb)
    print(out, plaq, Q, E)


if __name__ == "__main__":
    main()
