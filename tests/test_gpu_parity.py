"""CUDA path vs the CPU oracle and the golden fixtures, FP64 builds, through the C ABI.

Tolerance: 1e-12 relative (links, plaquette, E and the heatbath updates); Q, being a signed sum
near zero, is compared with an absolute bound of 1e-12 * max(1, sum_x |q(x)|).
"""
import os
import struct

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_4444.npz")
TOL = 1e-12
STORES = [0, 1]  # 18-real and 12-real link storage


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN)
    return {k: g[k] for k in g.files}


def q_tol(orc, U, L):
    q, _ = orc.clover_qe_density(U, L)
    return TOL * max(1.0, float(np.abs(q).sum()))


def test_philox_matches_oracle(gpu, orc):
    rng = np.random.default_rng(1)
    for _ in range(4):
        ctr = [int(v) for v in rng.integers(0, 2**32, 4)]
        key = [int(v) for v in rng.integers(0, 2**32, 2)]
        dev = gpu.philox(ctr, key, 64)
        for i in (0, 1, 63):
            c = list(ctr)
            c[0] = (c[0] + i) & 0xFFFFFFFF
            assert list(dev[i]) == orc.philox(c, key)


def test_exp_su3_matches_oracle(gpu, orc):
    rng = np.random.default_rng(2)
    Z = np.stack([orc.proj_lie_su3(rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))) * 0.4 for _ in range(64)])
    for c in (0.005, 0.25, 1.0):
        dev = gpu.exp_su3(Z, c)
        ref = np.stack([orc.exp_su3(z, c) for z in Z])
        assert np.max(np.abs(dev - ref)) < 1e-14


@pytest.mark.parametrize("store", STORES)
def test_cold_start(gpu, store):
    f = gpu.GaugeField((4, 4, 4, 4), 64, store)
    assert f.plaquette() == 1.0
    assert f.clover_qe() == (0.0, 0.0)
    U = f.download()
    assert np.array_equal(U, np.broadcast_to(np.eye(3), U.shape))


@pytest.mark.parametrize("store", STORES)
def test_golden_observables_and_staples(gpu, orc, golden, store):
    L = tuple(int(v) for v in golden["L"])
    U = np.ascontiguousarray(golden["U"])
    f = gpu.GaugeField(L, 64, store)
    f.upload(U)
    assert rel_err(f.download(), U) < (0 if store == 0 else 1e-14) + 1e-300
    assert abs(f.plaquette() - golden["plaq"]) < TOL * abs(golden["plaq"]) + 1e-16
    Q, E = f.clover_qe()
    assert abs(Q - golden["Q"]) < q_tol(orc, U, L)
    assert abs(E - golden["E"]) < TOL * golden["E"]
    for mu in range(4):
        assert rel_err(f.staple(mu), golden["staple"][mu]) < TOL


@pytest.mark.parametrize("store", STORES)
def test_golden_flow_step_and_measure(gpu, orc, golden, store):
    L = tuple(int(v) for v in golden["L"])
    U = np.ascontiguousarray(golden["U"])
    f = gpu.GaugeField(L, 64, store)
    f.upload(U)
    fl = gpu.GradientFlow(f, 0.02)
    fl.rk3_step(1)
    assert rel_err(fl.field.download(), golden["U_rk3"]) < TOL
    tqe = fl.measure(f, 4, 2)
    assert np.array_equal(tqe[:, 0], golden["tQE"][:, 0])
    assert np.max(np.abs(tqe[:, 1] - golden["tQE"][:, 1])) < q_tol(orc, U, L)
    assert rel_err(tqe[:, 2], golden["tQE"][:, 2]) < TOL


def test_golden_heatbath_link_by_link(gpu, golden):
    L = tuple(int(v) for v in golden["L"])
    f = gpu.GaugeField(L, 64, 0)
    f.upload(np.ascontiguousarray(golden["U"]))
    f.hb_subsweep(6.0, 2, 12345, 3, 0, 1)
    assert rel_err(f.download(), golden["U_hb"]) < TOL


@pytest.mark.parametrize("L", [(8, 8, 8, 8), (4, 6, 2, 8)])
def test_hot_start_matches_oracle(gpu, orc, L):
    f = gpu.GaugeField(L, 64, 0)
    f.hot_start(7)
    assert rel_err(f.download(), orc.hot_start(L, 7)) < TOL


@pytest.mark.parametrize("L,nh", [((8, 8, 8, 8), 2), ((4, 6, 2, 8), 1)])
def test_heatbath_harness_link_by_link(gpu, orc, L, nh):
    """Every (parity, mu) update, fed the same input and the same Philox draws as
    the oracle's restatement of the reference's update routine, matches link by link to 1e-12."""
    U = orc.hot_start(L, 99)
    f = gpu.GaugeField(L, 64, 0)
    for sweep in range(2):
        for p in range(2):
            for mu in range(4):
                f.upload(U)
                f.hb_subsweep(6.0, nh, 2024, sweep, p, mu)
                orc.hb_subsweep(U, L, 6.0, nh, 2024, sweep, p, mu)
                assert rel_err(f.download(), U) < TOL, (sweep, p, mu)


@pytest.mark.parametrize("L,nh", [((8, 8, 8, 8), 2), ((4, 6, 2, 8), 1)])
def test_heatbath_sweeps_chained(gpu, orc, L, nh):
    """One full sweep from the same start matches to 1e-12.  Chained sweeps compound the FMA /
    libm rounding differences through ill-conditioned links of a random start (1/|w| in su2_step),
    so three chained sweeps are held to 1e-10 and must show no accept/reject flip (which would
    produce O(1) differences)."""
    U = orc.hot_start(L, 99)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    for sweep in range(3):
        f.hb_sweep(6.0, nh, 2024, sweep)
        orc.hb_sweep(U, L, 6.0, nh, 2024, sweep)
        assert rel_err(f.download(), U) < (TOL if sweep == 0 else 1e-10), sweep
    assert abs(f.plaquette() - orc.plaquette(U, L)) < 1e-12
    mx, _ = f.unitarity()
    assert mx < 1e-12


def test_flow_measure_thermalised(gpu, orc):
    L = (8, 8, 8, 8)
    U = orc.hot_start(L, 3)
    for s in range(5):
        orc.hb_sweep(U, L, 6.0, 1, 5, s)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    fl = gpu.GradientFlow(f, 0.02)
    tqe, pl = fl.measure(f, 6, 2, plaquette=True)
    ref = orc.flow_measure(U, L, 0.02, 6, 2)
    assert np.max(np.abs(tqe[:, 1] - ref[:, 1])) < q_tol(orc, U, L)
    assert rel_err(tqe[:, 2], ref[:, 2]) < TOL
    W = orc.flow_rk3(U, L, 0.02, 10)
    assert abs(pl[-1] - orc.plaquette(W, L)) < TOL


def test_shift_and_random_shift(gpu, orc):
    L = (4, 6, 2, 8)
    U = orc.hot_start(L, 21)
    f = gpu.GaugeField(L, 64, 1)
    f.upload(U)
    f.shift([1, 5, 1, 3])
    orc.shift(U, L, [1, 5, 1, 3])
    assert rel_err(f.download(), U) < 1e-14
    s = f.random_shift(12345, 4)
    assert s == orc.random_shift_draw(12345, 4, L)
    orc.shift(U, L, s)
    assert rel_err(f.download(), U) < 1e-14


def test_reunitarize(gpu, orc):
    L = (4, 4, 4, 4)
    U = orc.hot_start(L, 1) * (1 + 1e-6)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    mx0, _ = f.unitarity()
    f.reunitarize()
    mx1, _ = f.unitarity()
    orc.reunitarize(U, L)
    assert mx0 > 1e-6 and mx1 < 1e-14
    assert rel_err(f.download(), U) < TOL


def test_determinism(gpu):
    res = []
    for _ in range(2):
        f = gpu.GaugeField((8, 8, 8, 8), 64, 0)
        f.hot_start(5)
        for s in range(2):
            f.hb_sweep(6.0, 2, 1, s)
        fl = gpu.GradientFlow(f, 0.02)
        res.append((f.download(), f.plaquette(), tuple(fl.measure(f, 3, 1).ravel())))
    assert np.array_equal(res[0][0], res[1][0]) and res[0][1:] == res[1][1:]


def test_ildg_round_trip_and_bytes(gpu, orc, tmp_path):
    L = (4, 6, 2, 8)
    U = orc.hot_start(L, 8)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    p = str(tmp_path / "cfg")
    f.save_ildg(p)
    raw = open(p, "rb").read()
    # record 1: ildg-format (MB=1, ME=1); record 2: ildg-binary-data (MB=0, ME=1)
    magic, ver, flags, _, n1 = struct.unpack(">IHBBQ", raw[:16])
    assert magic == 0x456789AB and ver == 1 and flags == 0xC0
    assert raw[16:27] == b"ildg-format"
    off = 144 + ((n1 + 7) // 8) * 8
    magic, ver, flags, _, n2 = struct.unpack(">IHBBQ", raw[off:off + 16])
    assert flags == 0x40 and raw[off + 16:off + 32] == b"ildg-binary-data"
    V = U.shape[0]
    assert n2 == V * 72 * 8
    payload = np.frombuffer(raw[off + 144:off + 144 + n2], dtype=">f8").astype(np.float64)
    assert np.array_equal(payload.view(np.complex128).reshape(U.shape), U)
    assert gpu.ildg_probe(p) == (L, 64)
    g = gpu.GaugeField(L, 64, 0)
    g.read_ildg(p)
    assert np.array_equal(g.download(), U)
    wrong = gpu.GaugeField((4, 4, 4, 4), 64, 0)
    with pytest.raises(gpu.QcbError) as e:
        wrong.read_ildg(p)
    assert e.value.code == -4


def test_ildg_32bit_payload(gpu, orc, tmp_path):
    from test_abi import ildg_xml, lime_record

    L = (4, 4, 4, 2)
    U = orc.hot_start(L, 4)
    V = U.shape[0]
    body = U.view(np.float64).astype(">f4").tobytes()
    p = tmp_path / "c32"
    p.write_bytes(lime_record(b"ildg-format", ildg_xml(L, 32), True, True) +
                  lime_record(b"ildg-binary-data", body, False, True))
    f = gpu.GaugeField(L, 64, 0)
    f.read_ildg(str(p))
    assert np.max(np.abs(f.download() - U)) < 1e-7
    assert V * 72 * 4 == len(body)


def test_ildg_scidac_checksum_write_and_verify(gpu, orc, tmp_path):
    """The checksum record a write adds matches zlib's restatement over the payload; the file
    reads back exactly; one flipped payload byte, or a wrong sum, makes the read fail."""
    from test_abi import scidac_sums_zlib

    L = (4, 6, 2, 8)
    U = orc.hot_start(L, 12)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    p = tmp_path / "cfg"
    f.save_ildg(str(p), scidac_checksum=True)
    raw = p.read_bytes()
    recs, off = [], 0
    while off < len(raw):
        _, _, flags, _, n = struct.unpack(">IHBBQ", raw[off:off + 16])
        recs.append((raw[off + 16:off + 144].rstrip(b"\0"), flags, raw[off + 144:off + 144 + n]))
        off += 144 + ((n + 7) // 8) * 8
    assert [(t, fl) for t, fl, _ in recs] == [(b"ildg-format", 0xC0), (b"ildg-binary-data", 0x00),
                                               (b"scidac-checksum", 0x40)]
    a, b = scidac_sums_zlib(recs[1][2], 576)
    assert f"<suma>{a:x}</suma><sumb>{b:x}</sumb>".encode() in recs[2][2]
    g = gpu.GaugeField(L, 64, 0)
    g.read_ildg(str(p))
    assert np.array_equal(g.download(), U)
    # the default write is the reference's two records: the same bytes up to the end of the
    # binary payload, with that record ending the message (ME set) and no checksum record
    off_bin = 144 + ((len(recs[0][2]) + 7) // 8) * 8
    plain = bytearray(raw[:off_bin + 144 + len(recs[1][2])])
    plain[off_bin + 6] = 0x40
    q = tmp_path / "plain"
    f.save_ildg(str(q))
    assert q.read_bytes() == bytes(plain)
    bad = bytearray(raw)
    bad[off_bin + 144 + 1000] ^= 0x01  # inside the binary payload
    (tmp_path / "bad").write_bytes(bytes(bad))
    with pytest.raises(gpu.QcbError) as e:
        g.read_ildg(str(tmp_path / "bad"))
    assert e.value.code == -4


def test_ildg_scidac_checksum_32bit_interop(gpu, orc, tmp_path):
    """A 32-bit file written outside the library with a zlib-computed checksum is accepted, and
    rejected once its sum is wrong."""
    from test_abi import ildg_xml, lime_record, scidac_record, scidac_sums_zlib

    L = (4, 4, 2, 4)
    U = orc.hot_start(L, 6)
    body = U.view(np.float64).astype(">f4").tobytes()
    a, b = scidac_sums_zlib(body, 288)
    for sums, ok in [((a, b), True), ((a ^ 1, b), False)]:
        p = tmp_path / f"c32_{ok}"
        p.write_bytes(lime_record(b"ildg-format", ildg_xml(L, 32), True, True) +
                      lime_record(b"ildg-binary-data", body, False, False) +
                      lime_record(b"scidac-checksum", scidac_record(*sums), False, True))
        f = gpu.GaugeField(L, 64, 0)
        if ok:
            f.read_ildg(str(p))
            assert np.max(np.abs(f.download() - U)) < 1e-7
        else:
            with pytest.raises(gpu.QcbError) as e:
                f.read_ildg(str(p))
            assert e.value.code == -4


def test_invalid_arguments(gpu):
    with pytest.raises(gpu.QcbError) as e:
        gpu.GaugeField((5, 4, 4, 4))
    assert e.value.code == -1
    f = gpu.GaugeField((4, 4, 4, 4))
    with pytest.raises(gpu.QcbError):
        f.hb_subsweep(6.0, 1, 1, 0, 2, 0)
    with pytest.raises(gpu.QcbError):
        f.hb_subsweep(-1.0, 1, 1, 0, 0, 0)


@pytest.mark.parametrize("prec,store", [(64, 0), (64, 1), (32, 0), (32, 1)])
def test_flow_graphs_match_plain_launches(gpu, orc, prec, store):
    """qcb_flow_rk3 and qcb_flow_measure replay captured CUDA graphs (pairs of RK3 steps; measurement
    blocks) unless per-launch timing is on, in which case every stage is a plain launch.  Both ways
    run the same kernels with the same arguments: the flowed links and every (t, Q, E, P) agree bit for
    bit, for odd and even step counts and for n_rk = 1, 2, 3 (graph replays from either buffer)."""
    L = (8, 8, 8, 8)
    U = orc.hot_start(L, 3)
    orc.hb_sweep(U, L, 6.0, 1, 3, 0)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    a = gpu.GradientFlow(f, 0.02, prec=prec, store=store)
    b = gpu.GradientFlow(f, 0.02, prec=prec, store=store)
    b.field.timing(True)
    n0 = gpu.launch_count()
    for n in (5, 4, 1, 2):
        a.rk3_step(n)
        b.rk3_step(n)
        assert np.array_equal(a.field.download(), b.field.download()), n
    assert gpu.launch_count() - n0 >= 2 * 3 * 12  # every stage counted, replayed or not
    for n_rk in (1, 2, 3, 1):
        ta, pa = a.measure(f, 6, n_rk, plaquette=True)
        tb, pb = b.measure(f, 6, n_rk, plaquette=True)
        assert np.array_equal(ta, tb) and np.array_equal(pa, pb), n_rk
        assert np.array_equal(a.field.download(), b.field.download()), n_rk


@pytest.mark.parametrize("prec,store", [(64, 0), (64, 1), (32, 0), (32, 1)])
def test_measured_flow_from_stage1_matches_clover_pass(gpu, orc, prec, store):
    """qcb_flow_measure takes each measurement (Q, E, plaquette) of a configuration that an RK3 step
    follows from that step's stage 1 (clover halves of the force's staples) instead of a clover
    pass.  Every row equals the clover pass on the same configuration: to 1e-12 in FP64 (Q to
    1e-12 * sum |q|), to FP32 rounding in FP32; the flowed links are those of plain RK3 steps."""
    L = (8, 6, 4, 10)
    U = orc.hot_start(L, 31)
    orc.hb_sweep(U, L, 6.0, 2, 32, 0)
    f = gpu.GaugeField(L, 64, 0)
    f.upload(U)
    tol = TOL if prec == 64 else 2e-6
    qscale = max(1.0, float(np.abs(orc.clover_qe_density(U, L)[0]).sum()))
    for n_rk in (1, 2):
        a = gpu.GradientFlow(f, 0.02, prec=prec, store=store)
        t, p = a.measure(f, 5, n_rk, plaquette=True)
        b = gpu.GradientFlow(f, 0.02, prec=prec, store=store)
        for s in range(5):
            Q, E = b.field.clover_qe()
            assert abs(t[s, 1] - Q) < tol * qscale, (n_rk, s)
            assert abs(t[s, 2] - E) < tol * abs(E), (n_rk, s)
            assert abs(p[s] - b.field.plaquette()) < tol, (n_rk, s)
            if s < 4:
                b.rk3_step(n_rk)
        assert np.array_equal(a.field.download(), b.field.download()), n_rk
        a.close()
        b.close()
