"""Continuous-batching flow server: each request's result is the same alone and in the mix, equals
the plain flow path (topo_charge_flowed) and the oracle, and admission respects the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 0.02


def config(gpu, L, seed, sweeps=3):
    f = gpu.GaugeField(L, 64, 0)
    f.hot_start(seed)
    for k in range(sweeps):
        f.hb_sweep(6.0, 1, seed, k)
    return f, f.download()


def run(server, reqs, timeout=300.0):
    for rid, L, U, n in reqs:
        server.submit(rid, L, U, EPS, n)
    server.wait(timeout)
    out = {}
    while True:
        r = server.poll()
        if r is None:
            break
        out[r[0]] = r
    return out


@pytest.mark.parametrize("prec,store", [(32, 0), (32, 1), (64, 0)])
def test_alone_equals_plain_flow(gpu, prec, store):
    """A small request's rows equal the plain measured flow's: both take each measurement from the
    measuring stage 1 (clover halves; the per-site values are the same), summed in different orders,
    so Q agrees to 1e-10 and E to 1e-12 in every precision."""
    f, U = config(gpu, (8, 8, 8, 8), 11)
    s = gpu.Server(1 << 30, prec=prec, store=store)
    res = run(s, [(7, f.L, U, 6)])
    assert set(res) == {7}
    tqe = res[7][1]
    fl = gpu.GradientFlow(f, EPS, prec=prec, store=store)
    ref = fl.measure(f, 6, 1)
    assert np.array_equal(tqe[:, 0], ref[:, 0])
    assert np.max(np.abs(tqe[:, 1] - ref[:, 1])) < 1e-10
    assert np.max(np.abs(tqe[:, 2] - ref[:, 2]) / ref[:, 2]) < 1e-12
    t_sub, t_adm, t_done = res[7][2]
    assert t_sub <= t_adm <= t_done


def test_fp64_server_matches_oracle(gpu, orc):
    L = (4, 6, 2, 8)
    f, U = config(gpu, L, 5)
    s = gpu.Server(1 << 28, prec=64)
    tqe = run(s, [(1, L, U, 5)])[1][1]
    ref = orc.flow_measure(U, L, EPS, 5, 1)
    q, _ = orc.clover_qe_density(U, L)
    assert np.max(np.abs(tqe[:, 1] - ref[:, 1])) < 1e-12 * max(1.0, np.abs(q).sum())
    assert np.max(np.abs(tqe[:, 2] - ref[:, 2]) / ref[:, 2]) < 1e-12


def test_result_same_alone_and_in_mix(gpu):
    """A request's result does not depend on which other requests share its launches."""
    cfgs = {i: config(gpu, L, 20 + i)[1] for i, L in enumerate([(8,) * 4, (12,) * 4, (4, 4, 4, 4), (8, 8, 4, 6)])}
    Ls = {0: (8,) * 4, 1: (12,) * 4, 2: (4, 4, 4, 4), 3: (8, 8, 4, 6)}
    steps = {0: 9, 1: 5, 2: 12, 3: 7}
    alone = {}
    for i in cfgs:
        s = gpu.Server(1 << 30, prec=32)
        alone[i] = run(s, [(i, Ls[i], cfgs[i], steps[i])])[i][1]
        s.close()
    s = gpu.Server(1 << 30, prec=32)
    mix = run(s, [(i, Ls[i], cfgs[i], steps[i]) for i in cfgs])
    for i in cfgs:
        assert np.array_equal(mix[i][1], alone[i]), i
    st = s.stats()
    assert st["completed"] == 4 and st["peak_resident"] >= 2  # the requests overlapped on the GPU


def test_budget_admission_queues_requests(gpu):
    f, U = config(gpu, (8,) * 4, 3)
    one = 8 ** 4 * (4 * (2 * 72 + 32) + 114 * 4) + 4096  # ~ one FP32 8^4 request (links, Z, clover halves)
    s = gpu.Server(int(one * 1.5), prec=32)
    res = run(s, [(k, f.L, U, 4) for k in range(4)])
    assert sorted(res) == [0, 1, 2, 3]
    st = s.stats()
    assert st["peak_resident"] == 1 and st["bytes_in_use"] == 0
    first = res[0][1]
    for k in range(1, 4):
        assert np.array_equal(res[k][1], first)


def test_server_errors(gpu):
    s = gpu.Server(1 << 20, prec=32)
    f, U = config(gpu, (8,) * 4, 3, sweeps=0)
    with pytest.raises(gpu.QcbError) as e:
        s.submit(1, (8,) * 4, U, EPS, 10)  # needs more than the 1 MiB budget
    assert e.value.code == -2
    with pytest.raises(gpu.QcbError) as e:
        s.submit(1, (5, 8, 8, 8), U, EPS, 10)
    assert e.value.code == -1
    s2 = gpu.Server(1 << 30, prec=32)
    big, Ub = config(gpu, (16,) * 4, 1, sweeps=0)
    s2.submit(9, big.L, Ub, EPS, 400)
    with pytest.raises(gpu.QcbError) as e:
        s2.wait(1e-4)  # bounded host wait runs out while the request is still flowing
    assert e.value.code == -6
    s2.wait(300.0)
    assert s2.poll()[0] == 9


def test_big_request_single_lattice_path(gpu):
    """A request of 2^17 half-sites or more (here 24^4) runs the single-lattice kernels: its result is
    bit-identical to the plain measured flow and the same alone and next to small requests."""
    f, U = config(gpu, (24,) * 4, 31, sweeps=1)
    s = gpu.Server(8 << 30, prec=32)
    alone = run(s, [(1, f.L, U, 4)])[1][1]
    s.close()
    fl = gpu.GradientFlow(f, EPS, prec=32, store=0)
    ref = fl.measure(f, 4, 1)
    assert np.array_equal(alone, ref)
    g, Ug = config(gpu, (8,) * 4, 32)
    s = gpu.Server(8 << 30, prec=32)
    mix = run(s, [(1, f.L, U, 4), (2, g.L, Ug, 6), (3, g.L, Ug, 3)])
    assert np.array_equal(mix[1][1], alone)
    assert s.stats()["peak_resident"] >= 2


@pytest.mark.parametrize("n_rk", [1, 2])
def test_tick_graphs_match_plain_launches(gpu, n_rk):
    """While the resident set of small requests is unchanged, their shared launches of a tick are
    replayed from CUDA graphs; every result equals the one-by-one launches' bit for bit (requests
    leaving at different ticks change the set, so both paths and the recaptures are exercised)."""
    reqs = []
    for i, (L, n) in enumerate([((8, 8, 8, 8), 9), ((12, 12, 12, 12), 5), ((8, 8, 8, 8), 14), ((4, 6, 2, 8), 7)]):
        _, U = config(gpu, L, 40 + i)
        reqs.append((i, L, U, n))
    out = {}
    for on in (True, False):
        s = gpu.Server(1 << 30, prec=32, store=0, n_rk=n_rk)
        s.set_graphs(on)
        out[on] = run(s, reqs)
        s.close()
    assert set(out[True]) == set(out[False]) == {0, 1, 2, 3}
    for rid in range(4):
        assert np.array_equal(out[True][rid][1], out[False][rid][1]), rid
