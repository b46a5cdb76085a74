"""Drives every kernel family of libqcb_checked.so -- libqcb.so built with QCB_CHECKED, whose
kernels validate every (mu, parity, h) of a field access on the device -- and prints the
out-of-bounds record as one JSON line.

Run in a process of its own (the binding binds one library per process):

    python tests/checked_workload.py

The workload covers the single-lattice kernels of all four link formats on small and ragged
lattices (Lt = 2, a 2^4 lattice whose neighbours wrap onto themselves), the flow, the
observables, shifts, ILDG, the batched and tuned sweeps, the server's shared and single-lattice
paths, and the allocation-free plaquette.  Then it runs the positive control: two probes of
links outside the field, which the device check must count and record.  tests/test_gpu_checked.py
asserts on the output.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from conftest import load_package  # noqa: E402
from test_zz_no_alloc import soa_fp64  # noqa: E402

FORMATS = [(64, 0), (64, 1), (32, 0), (32, 1)]
SHAPES = [(4, 6, 2, 8), (6, 4, 4, 2), (2, 2, 2, 2)]


def fields(qcb, tmp):
    for prec, store in FORMATS:
        for L in SHAPES:
            f = qcb.GaugeField(L, prec, store)
            f.cold_start()
            f.hot_start(3)
            for s in range(2):
                f.hb_sweep(6.0, 2, 1, s)
            for p in range(2):
                for mu in range(4):
                    f.hb_subsweep(6.0, 1, 2, 0, p, mu)
            f.plaquette()
            f.clover_qe()
            f.unitarity()
            f.reunitarize()
            f.shift((1, 0, 1, 1))
            f.random_shift(4, 0)
            for mu in range(4):
                f.staple(mu)
            f.upload(f.download())
            g = qcb.GaugeField(L, prec, store)
            g.copy_from(f)
            fl = qcb.GradientFlow(f, 0.02)
            fl.measure(f, 3, 1, plaquette=True)
            fl.rk3_step(2)
            if prec == 64:
                path = os.path.join(tmp, f"cfg_{store}_{L[3]}")
                f.save_ildg(path, scidac_checksum=True)
                g.read_ildg(path)
            fl.close()
            g.close()
            f.close()


def batches(qcb):
    for prec, store in FORMATS:
        b = qcb.Batch([(4, 6, 2, 8), (8, 8, 8, 8), (6, 4, 4, 2), (2, 2, 2, 2)], [5.9, 6.0, 6.1, 6.2], [1, 2, 3, 4],
                      prec, store)
        b.hot_start()
        b.sweep(2, 2)
        b.plaquette()
        b.tune(1, 1, allow_store_change=(prec == 64 and store == 0))
        b.sweep(1, 1)
        b.download(1)
        b.close()


def serving(qcb):
    rng = np.random.default_rng(0)
    for prec in (32, 64):
        srv = qcb.Server(8 << 30, prec, 0)
        reqs = [((4, 4, 4, 4), 4), ((8, 8, 8, 8), 3), ((6, 4, 4, 2), 5), ((24, 24, 24, 24), 2)]
        for rid, (L, n) in enumerate(reqs):
            f = qcb.GaugeField(L, 64, 0)
            f.hot_start(int(rng.integers(1 << 30)))
            srv.submit(rid, L, f.download(), 0.02, n)
            f.close()
        srv.wait(120.0)
        while srv.poll() is not None:
            pass
        srv.close()


def noalloc(qcb):
    import torch

    L = (4, 6, 2, 8)
    f = qcb.GaugeField(L, 64, 0)
    f.hot_start(9)
    links = torch.from_numpy(soa_fp64(f.download(), L)).to("cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    qcb.plaquette_noalloc(L, links.data_ptr(), out.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    f.close()


def main():
    qcb = load_package()
    qcb.load_library(qcb.CHECKED_LIB_PATH)
    checked, _, _ = qcb.debug_oob()
    with tempfile.TemporaryDirectory() as tmp:
        fields(qcb, tmp)
    batches(qcb)
    serving(qcb)
    noalloc(qcb)
    _, count, first = qcb.debug_oob()
    # positive control: links outside the field, caught and redirected by the device check
    L = (4, 4, 4, 4)
    f = qcb.GaugeField(L, 64, 0)
    f.hot_start(1)
    plaq_before = f.plaquette()
    probes = []
    for mu, par, h in [(0, 1, 128 + 3), (5, 0, 7)]:
        f.debug_probe_link(mu, par, h)
        _, n, fst = qcb.debug_oob()
        probes.append({"mu": mu, "par": par, "h": h, "count": n, "kind": fst >> 62, "mu_rec": (fst >> 56) & 63,
                       "par_rec": (fst >> 48) & 255, "h_rec": fst & ((1 << 48) - 1)})
    plaq_after = f.plaquette()
    f.close()
    print(json.dumps({"checked": checked, "count": count, "first": first, "probes": probes,
                      "plaquette_before_probes": plaq_before, "plaquette_after_probes": plaq_after}))


if __name__ == "__main__":
    main()
