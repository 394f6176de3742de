"""Batched FFT row convolution (DftTools::convolve, aux/src/DftTools.cxx:145-168,
over many rows; the long-range response step of ImpactTransform::waveform,
gen/src/ImpactTransform.cxx:327-343) against NumPy in FP64."""

import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2


def _ref(x, resp, nfft, n_out):
    X = np.fft.rfft(x.astype(np.float64), nfft, axis=1)
    R = np.fft.rfft(resp.astype(np.float64), nfft)
    return np.fft.irfft(X * R[None, :], nfft, axis=1)[:, :n_out]


def test_argument_checks_need_no_gpu(wct):
    L = wct.lib()
    p = C.c_void_p(16)  # never dereferenced: the checks fail first
    assert L.wct_convolve_rows_device(None, 8, 1, 8, p, 4, 0, p, 8, 8, None) == wct.WCT_ERR_ARG
    assert L.wct_convolve_rows_device(p, 8, 1, 8, p, 4, 1331, p, 8, 8, None) == wct.WCT_ERR_SIZE
    assert L.wct_convolve_rows_device(p, 8, 1, 8, p, 4, 6, p, 8, 8, None) == wct.WCT_ERR_SIZE
    assert L.wct_convolve_rows_device(p, 8, 1, 8, p, 4, 16, p, 32, 20, None) == wct.WCT_ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("nrows,n_in,n_resp,nfft", [(7, 300, 200, 0), (96, 3000, 200, 3200), (3, 1000, 1500, 0),
                                                     (40, 6000, 200, 8192), (5, 2000, 2000, 2048)])
def test_convolve_rows_matches_numpy(wct, nrows, n_in, n_resp, nfft):
    import torch
    rng = np.random.default_rng(nrows + n_in)
    x = rng.normal(size=(nrows, n_in)).astype(np.float32)
    resp = rng.normal(size=n_resp).astype(np.float32)
    N = nfft or None
    dx = torch.from_numpy(x).cuda()
    dr = torch.from_numpy(resp).cuda()
    if N is None:
        # the library picks the smallest supported length >= n_in + n_resp - 1: a linear convolution
        n_out = n_in + n_resp - 1
        want = np.stack([np.convolve(r.astype(np.float64), resp.astype(np.float64)) for r in x])
    else:
        n_out = min(N, n_in)
        want = _ref(x, resp, N, n_out)
    do = torch.zeros((nrows, n_out + 3), dtype=torch.float32, device="cuda")
    wct.convolve_rows(dx.data_ptr(), n_in, nrows, n_in, dr.data_ptr(), n_resp, do.data_ptr(), n_out + 3, n_out,
                      nfft=nfft)
    torch.cuda.synchronize()
    got = do.cpu().numpy()
    assert rel_l2(got[:, :n_out], want) < 2e-6
    assert not got[:, n_out:].any()


@pytest.mark.gpu
@pytest.mark.parametrize("nrows,n_in,n_resp,nfft", [
    (1500, 3000, 200, 3200),  # M = 1600: persistent forward (one first-stage butterfly per thread) and inverse
    (1500, 6000, 200, 6400),  # M = 3200: persistent forward with two butterflies per thread, per-row inverse
    (1500, 1700, 100, 2048),  # M = 1024: persistent forward and inverse (four values per thread)
    (1300, 900, 100, 1000),   # M = 500, not a multiple of 16: the per-row kernels
])
def test_convolve_many_rows_matches_numpy(wct, nrows, n_in, n_resp, nfft):
    """Enough rows (at least two per resident block) for the persistent row
    transforms; each shape against numpy in float64."""
    import torch
    rng = np.random.default_rng(nrows + nfft)
    x = rng.normal(size=(nrows, n_in)).astype(np.float32)
    resp = rng.normal(size=n_resp).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    dr = torch.from_numpy(resp).cuda()
    n_out = min(nfft, n_in)
    want = _ref(x, resp, nfft, n_out)
    do = torch.zeros((nrows, n_out), dtype=torch.float32, device="cuda")
    wct.convolve_rows(dx.data_ptr(), n_in, nrows, n_in, dr.data_ptr(), n_resp, do.data_ptr(), n_out, n_out,
                      nfft=nfft)
    torch.cuda.synchronize()
    assert rel_l2(do.cpu().numpy(), want) < 2e-6
