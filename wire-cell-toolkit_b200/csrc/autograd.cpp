// libtorch autograd wrapper of the DepoTransform forward and its adjoint.
//
// DepoTransformFn::apply(depos, drift_params, handle) runs wct_dt_forward_device
// on the current CUDA stream and returns the dense frame [nrows][nticks]
// (float32); its backward runs wct_dt_adjoint_device, which recomputes the
// patches from the saved depos (nothing but the inputs is kept between the
// two passes).  Inputs:
//   depos        [n][7] float64 CUDA tensor: t, q, x, y, z, extent_long, extent_tran
//   drift_params [3] float64 CPU tensor (DL, DT, lifetime) or an empty tensor
//                when the component drifts nothing / the values stay as configured
//   handle       the wct_depotransform* of a configured component
// Gradients: d/d depos [n][7] float64 (CUDA), d/d drift_params [3] float64 (CPU).

#include <torch/extension.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include "../../include/wctb200.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

void check(int rc)
{
    TORCH_CHECK(rc == WCT_OK, "wctb200: ", wct_last_error(), " (status ", rc, ")");
}

wct_depotransform* as_handle(int64_t h)
{
    TORCH_CHECK(h != 0, "wctb200: null component handle");
    return reinterpret_cast<wct_depotransform*>(static_cast<intptr_t>(h));
}

void set_params(wct_depotransform* h, const torch::Tensor& dp)
{
    if (!dp.defined() || dp.numel() == 0) return;
    TORCH_CHECK(dp.numel() == 3, "drift_params must hold DL, DT, lifetime");
    auto p = dp.detach().to(torch::kCPU, torch::kFloat64).contiguous();
    const double* v = p.data_ptr<double>();
    check(wct_dt_set_drift_params(h, v[0], v[1], v[2]));
}

// The launch stream: torch's current stream.  Torch's default stream has the
// handle 0, which the C ABI reads as "the component's own stream", so it is
// passed as the explicit legacy default-stream handle instead.
cudaStream_t launch_stream(const torch::Tensor& t)
{
    cudaStream_t s = c10::cuda::getCurrentCUDAStream(t.device().index()).stream();
    return s ? s : cudaStreamLegacy;
}

void check_depos(const torch::Tensor& d)
{
    TORCH_CHECK(d.is_cuda(), "depos must be a CUDA tensor");
    TORCH_CHECK(d.scalar_type() == torch::kFloat64, "depos must be float64");
    TORCH_CHECK(d.dim() == 2 && d.size(1) == 7, "depos must be [n][7]");
}

struct DepoTransformFn : public torch::autograd::Function<DepoTransformFn> {
    static torch::Tensor forward(AutogradContext* ctx, torch::Tensor depos, torch::Tensor drift_params,
                                 int64_t handle)
    {
        check_depos(depos);
        auto* h = as_handle(handle);
        const c10::cuda::CUDAGuard guard(depos.device());
        auto d = depos.contiguous();
        set_params(h, drift_params);
        int nrows = 0, nticks = 0;
        check(wct_dt_frame_shape(h, &nrows, &nticks));
        auto frame = torch::empty({nrows, nticks}, d.options().dtype(torch::kFloat32));
        check(wct_dt_forward_device(h, d.data_ptr<double>(), (size_t)d.size(0), frame.data_ptr<float>(), nullptr,
                                    nullptr, launch_stream(d)));
        ctx->save_for_backward({d, drift_params});
        ctx->saved_data["handle"] = handle;
        return frame;
    }

    static variable_list backward(AutogradContext* ctx, variable_list grads)
    {
        auto saved = ctx->get_saved_variables();
        auto d = saved[0];
        auto dp = saved[1];
        auto* h = as_handle(ctx->saved_data["handle"].toInt());
        const c10::cuda::CUDAGuard guard(d.device());
        set_params(h, dp);
        auto g = grads[0].to(torch::kFloat32).contiguous();
        TORCH_CHECK(g.is_cuda() && g.device() == d.device(), "frame gradient on another device");
        auto gd = torch::empty_like(d);
        auto gg = torch::zeros({3}, d.options());
        check(wct_dt_adjoint_device(h, d.data_ptr<double>(), (size_t)d.size(0), g.data_ptr<float>(),
                                    d.size(0) ? gd.data_ptr<double>() : nullptr, gg.data_ptr<double>(),
                                    launch_stream(d)));
        torch::Tensor gdp;
        if (dp.defined() && dp.numel() == 3) gdp = gg.to(dp.device()).reshape(dp.sizes());
        return {gd, gdp, torch::Tensor()};
    }
};

torch::Tensor depo_transform(torch::Tensor depos, torch::Tensor drift_params, int64_t handle)
{
    return DepoTransformFn::apply(depos, drift_params, handle);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.doc() = "torch.autograd wrapper of the DepoTransform forward and adjoint (libwctb200)";
    m.def("depo_transform", &depo_transform, "frame = DepoTransform(depos; DL, DT, lifetime), differentiable",
          pybind11::arg("depos"), pybind11::arg("drift_params"), pybind11::arg("handle"));
}
