"""Pipelined upload (qcb_field_prefetch_aos / qcb_field_commit_prefetch) against the synchronous
qcb_field_upload_aos: the same configurations, sweeps and observables, bit for bit, with the next
configuration's copy overlapping the current sweep; and the staging buffer's ownership rules.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)


def configs(gpu, n):
    f = gpu.GaugeField(L, 64, 0)
    out = []
    for k in range(n):
        f.hot_start(100 + k)
        out.append(f.download())
    f.close()
    return out


@pytest.mark.parametrize("pinned", [False, True])
def test_pipelined_upload_matches_synchronous(gpu, pinned):
    Us = configs(gpu, 4)
    a = gpu.GaugeField(L, 64, 0)
    ref = []
    for k, U in enumerate(Us):
        a.upload(U)
        a.hb_sweep(6.0, 2, 9, k)
        ref.append((a.plaquette(), a.download()))
    b = gpu.GaugeField(L, 64, 0)
    if pinned:
        import torch

        bufs = [torch.from_numpy(U.view(np.float64).ravel().copy()).pin_memory() for U in Us]
        start = lambda k: b.prefetch_ptr(bufs[k].data_ptr())  # noqa: E731
    else:
        start = lambda k: b.prefetch(Us[k])  # noqa: E731
    start(0)
    for k in range(len(Us)):
        b.commit_prefetch()
        b.hb_sweep(6.0, 2, 9, k)
        if k + 1 < len(Us):
            start(k + 1)  # the next configuration's copy overlaps this sweep
        p = b.plaquette()
        assert p == ref[k][0], k
        if k + 1 == len(Us):
            assert np.array_equal(b.download(), ref[k][1])


def test_staging_ownership(gpu):
    U0, U1 = configs(gpu, 2)
    f = gpu.GaugeField(L, 64, 0)
    with pytest.raises(gpu.QcbError) as e:
        f.commit_prefetch()
    assert e.value.code == -1
    f.upload(U0)
    f.prefetch(U1)
    for call in (lambda: f.prefetch(U0), lambda: f.upload(U0), lambda: f.download(), lambda: f.staple(0)):
        with pytest.raises(gpu.QcbError) as e:
            call()
        assert e.value.code == -1
    f.hb_sweep(6.0, 1, 1, 0)  # the links are not the staging buffer: work goes on meanwhile
    f.commit_prefetch()
    assert np.array_equal(f.download(), U1)
    g = gpu.GaugeField(L, 64, 0)
    g.prefetch(U0)
    g.close()  # a pending prefetch is dropped with its field
