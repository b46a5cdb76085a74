"""The allocation-free plaquette entry point against the regular one, through the C ABI.

qcb_plaquette_noalloc serves callers that cannot let the library allocate device memory (they
own every byte through their own pool, or may not allocate after start-up): the links and the
output live in memory the caller allocated -- here with torch -- and the reduction scratch is a
static device array inside libqcb.so.  Two calls in a row must both agree with qcb_plaquette on
the same configuration, which also shows that the shared scratch left by one call does not leak
into the next.  This file is named to be collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same tolerance as the FP64 parity tests


def soa_fp64(U: np.ndarray, L) -> np.ndarray:
    """AoS (V,4,3,3) complex -> parity-split FP64 layout [mu][parity][9][V/2] of (re, im) pairs."""
    V = U.shape[0]
    lex = np.arange(V)
    x0 = lex % L[0]
    x1 = (lex // L[0]) % L[1]
    x2 = (lex // (L[0] * L[1])) % L[2]
    x3 = lex // (L[0] * L[1] * L[2])
    par = (x0 + x1 + x2 + x3) % 2
    out = np.zeros((4, 2, 9, V // 2), dtype=np.complex128)
    for mu in range(4):
        out[mu, par, :, lex // 2] = U[:, mu].reshape(V, 9)
    return np.ascontiguousarray(out).view(np.float64)


@pytest.mark.parametrize("L", [(8, 8, 8, 8), (4, 6, 2, 8)])
def test_noalloc_plaquette_matches_regular_entry(gpu, orc, L):
    import torch

    U = orc.hot_start(L, 31)
    orc.hb_sweep(U, L, 6.0, 1, 7, 0)
    f = gpu.GaugeField(L, gpu.PREC_F64, gpu.STORE_18)
    f.upload(U)
    ref = f.plaquette()
    links = torch.from_numpy(soa_fp64(U, L)).to("cuda")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for k in range(2):
        out.fill_(float("nan"))
        stream.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        gpu.plaquette_noalloc(L, links.data_ptr(), out.data_ptr(), stream.cuda_stream)
        stream.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert abs(out.item() - ref) < TOL * abs(ref)
        if k == 1:  # the defining property: a call after the first allocates no device memory
            assert free_after == free_before, (free_before, free_after)


def test_noalloc_rejects_bad_sizes(gpu):
    import torch

    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    links = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.QcbError) as e:
        gpu.plaquette_noalloc((5, 4, 4, 4), links.data_ptr(), out.data_ptr())
    assert e.value.code == -1
    with pytest.raises(gpu.QcbError) as e:
        gpu.plaquette_noalloc((2048, 2048, 2048, 2), links.data_ptr(), out.data_ptr())
    assert e.value.code == -1
    # a view offset by one double is only 8-byte aligned: refused, never sent to the device
    with pytest.raises(gpu.QcbError) as e:
        gpu.plaquette_noalloc((4, 4, 4, 4), links[1:].data_ptr(), out.data_ptr())
    assert e.value.code == -1
