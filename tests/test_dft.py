"""GPU IDFT (iface/inc/WireCellIface/IDFT.h) against numpy.fft in float64.

The reference's own IDFT checks (aux/test/test_idft.cxx: zero arrays,
impulses with flat spectra, 1b impulses along either axis in and out of
place, 2d impulses, forward/inverse round trips) plus comparisons with
numpy.fft at 7-smooth lengths (shared-memory FFT) and at lengths with
larger prime factors (Bluestein's chirp-z transform)."""

import numpy as np
import pytest

from conftest import rel_l2

SMOOTH = [1, 2, 7, 64, 1000, 1024, 3200, 6000, 14336, 16384, 100000]   # above 14336: four steps
OTHER = [11, 13, 97, 1009, 4097, 7001, 7177, 9317, 20011]              # above 7168: Bluestein in global memory


def _rand(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.fixture(scope="module")
def dft(wct):
    return wct.IDFT()


@pytest.mark.gpu
@pytest.mark.parametrize("n", SMOOTH + OTHER)
def test_1d_against_numpy(dft, n):
    rng = np.random.default_rng(n)
    x = _rand(rng, n)
    X = dft.fwd1d(x)
    ref = np.fft.fft(x.astype(np.complex128))
    tol = (2e-6 if n <= 14336 else 5e-6) if n in SMOOTH else 2e-5
    assert rel_l2(X, ref) < tol
    back = dft.inv1d(X)
    assert rel_l2(back, x) < 2 * tol
    assert rel_l2(dft.inv1d(x), np.fft.ifft(x.astype(np.complex128))) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1024, 1013])
def test_1d_zero_and_impulse(dft, n):
    z = np.zeros(n, np.complex64)
    assert np.all(dft.fwd1d(z) == 0) and np.all(dft.inv1d(z) == 0)
    x = np.zeros(n, np.complex64)
    x[0] = 1.0
    X = dft.fwd1d(x)
    assert np.allclose(X, 1.0, atol=1e-5)
    back = dft.inv1d(X)
    assert abs(back[0] - 1.0) < 1e-5 and np.max(np.abs(back[1:])) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(128, 128), (37, 200), (100, 13), (3, 1)])
@pytest.mark.parametrize("axis", [0, 1])
def test_1b_against_numpy(dft, shape, axis):
    rng = np.random.default_rng(sum(shape) + axis)
    x = _rand(rng, *shape)
    X = dft.fwd1b(x, axis)
    ref = np.fft.fft(x.astype(np.complex128), axis=axis)
    assert rel_l2(X, ref) < 1e-5
    assert rel_l2(dft.inv1b(X, axis), x) < 2e-5


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [0, 1])
def test_1b_impulse_in_place(wct, axis):
    """aux/test/test_idft.cxx test_1b_impulse: a unit impulse at [0, 0] gives
    |X| = 1 along the transformed axis' first row/column, zero elsewhere; the
    in-place device call gives the same."""
    import torch
    nrows = ncols = 128
    x = torch.zeros((nrows, ncols), dtype=torch.complex64, device="cuda")
    x[0, 0] = 1.0
    wct.dft_1b_device(x.data_ptr(), x.data_ptr(), nrows, ncols, axis)
    torch.cuda.synchronize()
    a = x.abs().cpu().numpy()
    if axis:  # rows transformed: row 0 is flat
        assert np.allclose(a[0], 1.0, atol=1e-6) and np.max(a[1:]) < 1e-6
    else:
        assert np.allclose(a[:, 0], 1.0, atol=1e-6) and np.max(a[:, 1:]) < 1e-6
    wct.dft_1b_device(x.data_ptr(), x.data_ptr(), nrows, ncols, axis, inverse=True)
    torch.cuda.synchronize()
    b = x.cpu().numpy()
    assert abs(b[0, 0] - 1.0) < 1e-6 and np.max(np.abs(b.reshape(-1)[1:])) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(128, 128), (64, 3200), (37, 64), (1, 97), (1024, 1024)])
def test_2d_against_numpy(dft, shape):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    x = _rand(rng, *shape)
    X = dft.fwd2d(x)
    ref = np.fft.fft2(x.astype(np.complex128))
    assert rel_l2(X, ref) < 1e-5
    assert rel_l2(dft.inv2d(X), x) < 2e-5
    assert rel_l2(dft.inv2d(x), np.fft.ifft2(x.astype(np.complex128))) < 1e-5


@pytest.mark.gpu
def test_2d_impulse_and_round_trip(dft):
    x = np.zeros((128, 128), np.complex64)
    x[0, 0] = 1.0
    X = dft.fwd2d(x)
    assert np.allclose(X, 1.0, atol=1e-5)
    back = dft.inv2d(X)
    assert abs(back[0, 0] - 1.0) < 1e-5 and np.max(np.abs(back.reshape(-1)[1:])) < 1e-5
    z = np.zeros((256, 256), np.complex64)
    for _ in range(3):  # aux/test/test_idft.cxx fwdrev: zeros stay exactly zero
        z = dft.inv2d(dft.fwd2d(z))
    assert np.all(z == 0)


@pytest.mark.gpu
def test_transpose(wct, dft):
    import torch
    rng = np.random.default_rng(3)
    r = rng.standard_normal((37, 129)).astype(np.float32)
    assert np.array_equal(dft.transpose(r), r.T)
    c = _rand(rng, 300, 41)
    assert np.array_equal(dft.transpose(c), c.T)
    d = torch.from_numpy(c.copy()).cuda()
    wct.lib().wct_dft_transpose_device(d.data_ptr(), d.data_ptr(), 300, 41, 1, None)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().reshape(41, 300), c.T)


@pytest.mark.gpu
def test_device_2d_matches_host(wct, dft):
    import torch
    rng = np.random.default_rng(9)
    x = _rand(rng, 96, 250)
    d = torch.from_numpy(x).cuda()
    out = torch.empty_like(d)
    s = torch.cuda.Stream()
    wct.dft_2d_device(d.data_ptr(), out.data_ptr(), 96, 250, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), dft.fwd2d(x))


@pytest.mark.gpu
def test_errors(wct, dft):
    with pytest.raises(wct.WctError) as e:
        dft.fwd1b(np.zeros((4, 4), np.complex64), 2)
    assert e.value.code == 1
    assert dft.fwd1d(np.zeros(0, np.complex64)).size == 0
