"""The allocation-free row convolution (wct_convolve_rows_device_noalloc).

It exists for callers that may not allocate device memory once running (an
online trigger or DAQ process with a device-memory budget fixed at start-up,
or a host framework that owns all device memory through its own pool).  Its
scratch is a fixed 32 MiB device array shared by every call, so these tests
check that it gives the same rows as the allocating entry point on two calls
in a row -- the second call finds the first call's data in the scratch -- and
that sizes beyond the fixed array are refused before any device work.

This file is collected at the end (test_zz_*) so a run that stops at the
first failure has already run the other tests."""

import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

TOL = 2e-6  # the same tolerance as the allocating entry point's own tests


def test_oversize_request_is_refused_without_device_work(wct):
    L = wct.lib()
    p = C.c_void_p(16)  # never dereferenced: the size check fails first
    # (nrows + 3) * nfft / 2 must stay within 4194304 complex values
    rc = L.wct_convolve_rows_device_noalloc(p, 8192, 1100, 8192, p, 200, 8192, p, 8192, 8192, None)
    assert rc == wct.WCT_ERR_SIZE
    assert b"32 MiB" in L.wct_last_error()
    rc = L.wct_convolve_rows_device_noalloc(None, 8, 1, 8, p, 4, 0, p, 8, 8, None)
    assert rc == wct.WCT_ERR_ARG


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_on_two_calls(wct):
    import torch
    torch.cuda.set_device(0)
    rng = np.random.default_rng(2024)
    cases = [
        # (nrows, n_in, n_resp, nfft): a larger call first, then a smaller one that
        # reuses the scratch the first call left behind
        (200, 6000, 200, 8192),
        (37, 3000, 1200, 0),
    ]
    for nrows, n_in, n_resp, nfft in cases:
        x = rng.normal(size=(nrows, n_in)).astype(np.float32)
        resp = rng.normal(size=n_resp).astype(np.float32)
        n_out = n_in
        dx = torch.from_numpy(x).cuda()
        dr = torch.from_numpy(resp).cuda()
        want = torch.zeros((nrows, n_out), dtype=torch.float32, device="cuda")
        got = torch.full((nrows, n_out), 7.0, dtype=torch.float32, device="cuda")
        wct.convolve_rows(dx.data_ptr(), n_in, nrows, n_in, dr.data_ptr(), n_resp, want.data_ptr(), n_out, n_out,
                          nfft=nfft)
        wct.convolve_rows_noalloc(dx.data_ptr(), n_in, nrows, n_in, dr.data_ptr(), n_resp, got.data_ptr(), n_out,
                                  n_out, nfft=nfft)
        torch.cuda.synchronize()
        w = want.cpu().numpy()
        g = got.cpu().numpy()
        assert np.abs(w).max() > 0
        assert rel_l2(g, w) < TOL, (nrows, n_in, rel_l2(g, w))


@pytest.mark.gpu
def test_noalloc_strided_on_a_stream_and_at_the_limit(wct):
    """Strided rows in and out, fewer output samples than input samples, a
    caller's stream (the twiddle tables are built on it), and a call whose
    (nrows + 3) * nfft / 2 is exactly the 4194304 complex values the fixed
    array holds; each against the allocating entry point on the same stream."""
    import torch
    torch.cuda.set_device(0)
    rng = np.random.default_rng(77)
    st = torch.cuda.Stream()
    cases = [
        # (nrows, n_in, ld_in, n_resp, nfft, n_out, ld_out)
        (64, 3000, 3072, 300, 0, 2500, 2600),
        (1021, 6000, 6000, 200, 8192, 6000, 6000),  # (1021 + 3) * 4096 = 4194304
    ]
    for nrows, n_in, ld_in, n_resp, nfft, n_out, ld_out in cases:
        if nfft:
            assert (nrows + 3) * nfft // 2 == 4194304
        x = rng.normal(size=(nrows, ld_in)).astype(np.float32)
        resp = rng.normal(size=n_resp).astype(np.float32)
        with torch.cuda.stream(st):
            dx = torch.from_numpy(x).cuda()
            dr = torch.from_numpy(resp).cuda()
            want = torch.full((nrows, ld_out), -3.0, dtype=torch.float32, device="cuda")
            got = torch.full((nrows, ld_out), 7.0, dtype=torch.float32, device="cuda")
        st.synchronize()
        wct.convolve_rows(dx.data_ptr(), ld_in, nrows, n_in, dr.data_ptr(), n_resp, want.data_ptr(), ld_out, n_out,
                          nfft=nfft, stream=st.cuda_stream)
        wct.convolve_rows_noalloc(dx.data_ptr(), ld_in, nrows, n_in, dr.data_ptr(), n_resp, got.data_ptr(), ld_out,
                                  n_out, nfft=nfft, stream=st.cuda_stream)
        st.synchronize()
        w = want.cpu().numpy()
        g = got.cpu().numpy()
        assert np.abs(w[:, :n_out]).max() > 0
        assert rel_l2(g[:, :n_out], w[:, :n_out]) < TOL, (nrows, n_in, rel_l2(g[:, :n_out], w[:, :n_out]))
        # the row padding beyond n_out is not written
        assert (g[:, n_out:] == 7.0).all() and (w[:, n_out:] == -3.0).all()
