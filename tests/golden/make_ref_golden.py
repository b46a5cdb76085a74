"""Writes tests/golden/ref_4444.npz: outputs of the reference's own hot-path code on a 4^4 lattice.

    make -C oracle ref            # compiles the reference's sources into oracle/_ref/libqcb_ref.so
    python tests/golden/make_ref_golden.py

Every output below is computed by the reference's unchanged sources (GaugeField::compute_staple,
mean_plaquette_global, topo_q_e_clover_global, local_q_e_clover, GradientFlow::rk3_step,
topo_charge_flowed, mpi::heatbathcb::hit, exp_su3_luscher, proj_lie_su3), compiled into
oracle/_ref/libqcb_ref.so against the project's one-rank MPI and Eigen-API stand-ins.  The
heatbath draws come from the Philox link stream the CUDA path uses (seed 12345, sweep 3), replayed
through the reference's own uniform_real_distribution.  The input configuration is the oracle's
Haar hot start (seed 7; the reference's random_su3 needs a QR decomposition the stand-in does not
provide) followed by two sweeps of the reference's hit() at beta 6.0, N_hits 2, seed 99.

These fixtures let the GPU tests pin the CUDA path to the reference even where the reference
library is not built.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as orc  # noqa: E402
import ref  # noqa: E402

L = 4
EPS = 0.02


def main() -> None:
    if not ref.available() and not ref.build():
        raise SystemExit("oracle/_ref/libqcb_ref.so is not built and the reference tree is absent")
    LL = (L,) * 4
    U0 = orc.hot_start(LL, 7)
    r = ref.RefLattice(L, U0)
    for s in range(2):
        r.hb_sweep(6.0, 2, 99, s)
    U = r.get()

    out = {"L": np.array(LL, dtype=np.int32), "U": U}
    out["staple"] = np.stack([r.staple_field(mu) for mu in range(4)])
    out["plaq"] = np.float64(r.plaquette())
    Q, E = r.clover_qe()
    out["Q"], out["E"] = np.float64(Q), np.float64(E)
    out["q_site"], out["e_site"] = r.clover_density()
    out["tQE"] = r.flow_measure(EPS, 5, 2)

    f = ref.RefLattice(L, U)
    f.flow_rk3(EPS, 1)
    out["U_rk3"] = f.get()

    h = ref.RefLattice(L, U)
    h.hb_subsweep(6.0, 2, 12345, 3, 0, 1)
    out["U_hb_sub"] = h.get()
    h = ref.RefLattice(L, U)
    h.hb_sweep(6.0, 2, 12345, 3)
    out["U_hb_sweep"] = h.get()

    rng = np.random.default_rng(5)
    M = rng.normal(size=(8, 3, 3)) + 1j * rng.normal(size=(8, 3, 3))
    out["lie_in"] = M
    out["lie_out"] = np.stack([ref.proj_lie_su3(m) for m in M])
    Z = 0.4 * out["lie_out"]
    out["exp_in"] = Z
    out["exp_coeff"] = np.array([0.005, 0.25, 1.0])
    out["exp_out"] = np.stack([[ref.exp_su3_luscher(z, c) for z in Z] for c in out["exp_coeff"]])

    path = os.path.join(HERE, "ref_4444.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: plaquette {out['plaq']:.15f} Q {Q:.6e} E {E:.12f}")


if __name__ == "__main__":
    main()
