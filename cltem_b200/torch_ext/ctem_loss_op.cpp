// ctem_loss_op.cpp — the differentiable CTEM image loss as a libtorch autograd Function.
//
// forward(xyz [n,3] float64, lens [2] float64 = (C10, C30) in Å) -> loss (0-d float64): sets the atoms and the
// lens of an mslice simulation and runs the adjoint's forward half, mslice_ctem_loss_forward (include/mslice.h),
// which keeps the checkpoints the backward half needs. backward runs mslice_ctem_loss_backward and returns
// grad_output * dL/dxyz and grad_output * dL/d(C10, C30); a forward with no backward costs only the forward.
// The simulation handle, the atomic numbers and the target image are fixed per op instance.
#include <torch/extension.h>

#include "../../include/mslice.h"

#include <stdexcept>
#include <vector>

using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

namespace {

void check(int rc) {
    if (rc != MSLICE_OK) throw std::runtime_error(std::string("mslice: ") + mslice_last_error());
}

struct CtemImageLoss : public torch::autograd::Function<CtemImageLoss> {
    static torch::Tensor forward(AutogradContext *ctx, torch::Tensor xyz, torch::Tensor lens, int64_t sim_handle,
                                 torch::Tensor Z, torch::Tensor target, int64_t checkpoint_every) {
        auto sim = reinterpret_cast<mslice_sim *>(sim_handle);
        auto p = xyz.detach().to(torch::kCPU, torch::kFloat64).contiguous();
        auto z = Z.to(torch::kCPU, torch::kInt32).contiguous();
        auto t = target.detach().to(torch::kCPU, torch::kFloat64).contiguous();
        auto l = lens.detach().to(torch::kCPU, torch::kFloat64).contiguous();
        const int64_t n = p.size(0);
        std::vector<double> x(n), y(n), w(n);
        const double *pp = p.data_ptr<double>();
        for (int64_t i = 0; i < n; i++) { x[i] = pp[3 * i]; y[i] = pp[3 * i + 1]; w[i] = pp[3 * i + 2]; }
        check(mslice_set_c10_c30(sim, l.data_ptr<double>()[0], l.data_ptr<double>()[1]));
        check(mslice_set_atoms(sim, z.data_ptr<int>(), x.data(), y.data(), w.data(), (size_t)n));
        double loss = 0;
        unsigned long long token = 0;
        check(mslice_ctem_loss_forward(sim, t.data_ptr<double>(), &loss, (int)checkpoint_every, &token));
        ctx->saved_data["sim"] = sim_handle;
        ctx->saved_data["token"] = (int64_t)token;
        ctx->saved_data["n"] = n;
        return torch::tensor(loss, torch::kFloat64).to(xyz.device());
    }

    static tensor_list backward(AutogradContext *ctx, tensor_list grad_outputs) {
        auto sim = reinterpret_cast<mslice_sim *>(ctx->saved_data["sim"].toInt());
        const auto token = (unsigned long long)ctx->saved_data["token"].toInt();
        const int64_t n = ctx->saved_data["n"].toInt();
        double g10 = 0, g30 = 0;
        auto gxyz = torch::zeros({n, 3}, torch::kFloat64);
        check(mslice_ctem_loss_backward(sim, token, gxyz.data_ptr<double>(), &g10, &g30));
        auto glens = torch::tensor({g10, g30}, torch::kFloat64);
        auto go = grad_outputs[0].to(torch::kCPU);
        return {gxyz * go, glens * go, torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor()};
    }
};

torch::Tensor ctem_image_loss(torch::Tensor xyz, torch::Tensor lens, int64_t sim_handle, torch::Tensor Z,
                              torch::Tensor target, int64_t checkpoint_every) {
    return CtemImageLoss::apply(xyz, lens, sim_handle, Z, target, checkpoint_every);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.def("ctem_image_loss", &ctem_image_loss, "differentiable CTEM image loss (adjoint multislice)");
}
