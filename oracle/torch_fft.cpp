// TEST INFRASTRUCTURE ONLY -- NOT PART OF THE PRODUCT.
//
// libtorch-CPU (Intel MKL) transforms for the oracle's timed CPU baseline:
// the reference's own alternative IDFT backend is TorchDFT
// (pytorch/src/DFT.cxx:80-123), which hands every 1-D / 1-b / 2-D transform
// to torch::fft on the configured device.  Its FFTW default (FftwDFT,
// aux/src/FftwDFT.cxx) is not installed here.  The oracle calls
// orc_torch_fft through orc_set_fft_backend (wct_oracle.cpp) in place of its
// own scalar Stockham transforms, so the baseline's FFT stage runs at an
// optimised library's speed.  Parity runs do not use it.
//
// orc_torch_fft(a, nrows, ncols, axis, sign, fp64): a is a row-major
// [nrows][ncols] array of complex float (fp64 = 0) or complex double values,
// transformed in place along axis (1: each row, 0: each column), sign -1
// forward / +1 backward, both unnormalised (IDFT.h conventions, the caller
// divides).  The intra-op thread count is libtorch's (torch.set_num_threads).

#include <ATen/ATen.h>

extern "C" void orc_torch_fft(void* a, int nrows, int ncols, int axis, int sign, int fp64)
{
    const auto dt = fp64 ? at::kComplexDouble : at::kComplexFloat;
    at::Tensor t = at::from_blob(a, {nrows, ncols}, at::TensorOptions().dtype(dt));
    const int64_t dim = axis == 1 ? 1 : 0;
    // "backward" scales only the inverse and "forward" only the forward: an
    // unnormalised transform either way
    at::Tensor r = sign < 0 ? at::fft_fft(t, c10::nullopt, dim, "backward")
                            : at::fft_ifft(t, c10::nullopt, dim, "forward");
    t.copy_(r);
}
