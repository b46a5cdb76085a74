"""Precision and physics forms: FP32 (18- and 12-real) links, staples and RK3 stages with FP64
reprojection, Cayley-Hamilton coefficients and sums, against the FP64 path; and independent GPU
chains against an oracle chain at beta = 6.0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DQ_MAX = 1e-4  # bound on |Q_fp32 - Q_fp64|
DE_REL_MAX = 1e-6  # |E_fp32 - E_fp64| / E_fp64
DP_MAX = 1e-6  # |P_fp32 - P_fp64|


@pytest.fixture(scope="module")
def thermalised(gpu):
    f = gpu.GaugeField((12, 12, 12, 12), 64, 0)
    f.hot_start(99)
    for k in range(40):
        f.hb_sweep(6.2, 1, 99, k)
    return f


@pytest.mark.parametrize("store", [0, 1])
def test_fp32_flow_against_fp64(gpu, thermalised, store):
    n = 101  # t = 0 .. 2.0
    ref = gpu.GradientFlow(thermalised, 0.02, prec=64, store=0)
    t64, p64 = ref.measure(thermalised, n, 1, plaquette=True)
    fl = gpu.GradientFlow(thermalised, 0.02, prec=32, store=store)
    t32, p32 = fl.measure(thermalised, n, 1, plaquette=True)
    assert np.max(np.abs(t32[:, 1] - t64[:, 1])) < DQ_MAX
    assert np.max(np.abs(t32[:, 2] - t64[:, 2]) / t64[:, 2]) < DE_REL_MAX
    assert np.max(np.abs(p32 - p64)) < DP_MAX
    mx, _ = fl.field.unitarity()
    assert mx < 1e-6  # reprojected in FP64 after every RK3 step, stored in FP32


@pytest.mark.parametrize("store", [0, 1])
def test_fp32_member_passes_equal_fused_step(gpu, thermalised, store):
    """GradientFlow's separate passes (compute_force, compute_w1/2/3, replace_force_0) on FP32 links,
    reprojected once after compute_w3 as the fused step is after its third stage, give the fused
    RK3 step's links to FP32 rounding."""
    fused = gpu.GradientFlow(thermalised, 0.02, prec=32, store=store)
    fused.rk3_step(1)
    fl = gpu.GradientFlow(thermalised, 0.02, prec=32, store=store)
    for p in (fl.FORCE0, fl.W1, fl.FORCE1, fl.W2, fl.REPLACE_F0, fl.FORCE1, fl.W3):
        fl.run_pass(p)
    assert np.max(np.abs(fl.field.download() - fused.field.download())) < 1e-5
    mx, _ = fl.field.unitarity()
    assert mx < 1e-6
    fl.close()
    fused.close()


def test_fp32_heatbath_stays_on_su3(gpu):
    f = gpu.GaugeField((8, 8, 8, 8), 32, 0)
    f.hot_start(3)
    for k in range(30):
        f.hb_sweep(6.0, 2, 3, k)
    mx, _ = f.unitarity()
    assert mx < 1e-6
    assert 0.55 < f.plaquette() < 0.65


def binned_mean(x, nbin=10):
    b = np.array([c.mean() for c in np.array_split(np.asarray(x), nbin)])
    return b.mean(), b.std(ddof=1) / np.sqrt(nbin)


def test_independent_chains_reproduce_oracle_plaquette(gpu, orc):
    """<P> of independent GPU chains at beta = 6.0 agrees with independent oracle
    chains within 2 sigma, and the links stay unitary to 1e-12 without reprojection.  Both sides
    start cold, thermalise 100 sweeps and measure 500; errors come from bins of 50 sweeps (many
    autocorrelation times of the plaquette) combined over 4 oracle and 32 GPU chains."""
    L = (8, 8, 8, 8)
    n_therm, n_meas, bin_len = 100, 500, 50

    def chain_stats(series):
        per = [binned_mean(x, n_meas // bin_len) for x in series]
        return np.mean([m for m, _ in per]), np.sqrt(np.sum([e * e for _, e in per])) / len(per)

    po = []
    for c in range(4):
        U = orc.cold_start(L)
        x = []
        for k in range(n_therm + n_meas):
            orc.hb_sweep(U, L, 6.0, 1, 1000 + c, k)
            if k >= n_therm:
                x.append(orc.plaquette(U, L))
        po.append(x)
    mo, eo = chain_stats(po)
    n_ch = 32
    b = gpu.Batch([L] * n_ch, [6.0] * n_ch, list(range(1, n_ch + 1)))
    b.sweep(1, n_therm)
    pg = []
    for k in range(n_meas):
        b.sweep(1, 1)
        pg.append(b.plaquette())
    pg = np.array(pg)
    mg, eg = chain_stats([pg[:, c] for c in range(n_ch)])
    sigma = np.hypot(eo, eg)
    assert abs(mg - mo) < 2 * sigma, (mg, mo, sigma)
    assert 0.58 < mg < 0.61
    for i in range(n_ch):
        V = b.download(i).reshape(-1, 3, 3)
        assert np.abs(V @ np.conj(np.swapaxes(V, 1, 2)) - np.eye(3)).max() < 1e-12


@pytest.mark.parametrize("L,beta,p_lit", [((16, 16, 16, 16), 6.0, 0.5937), ((24, 24, 24, 24), 6.2, 0.6136)])
def test_plaquette_matches_published_value(gpu, L, beta, p_lit):
    """An external pin of the whole heatbath chain, independent of the oracle: the mean plaquette
    of the Wilson action at large volume is 0.5937 at beta = 6.0 and 0.6136 at beta = 6.2 (the
    lattice literature's values, to four digits).  A cold start, 300 thermalisation sweeps and 200
    measured ones (N_hits = 2); the statistical error of the mean and the finite-volume shift at
    these sizes are both well below the 3e-4 bound."""
    f = gpu.GaugeField(L, 64, 0)
    f.cold_start()
    for s in range(300):
        f.hb_sweep(beta, 2, 4242, s)
    ps = []
    for s in range(300, 500):
        f.hb_sweep(beta, 2, 4242, s)
        ps.append(f.plaquette())
    p = float(np.mean(ps))
    assert abs(p - p_lit) < 3e-4, (p, p_lit)
