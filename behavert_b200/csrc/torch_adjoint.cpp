// torch_adjoint.cpp -- libtorch autograd binding of the differentiable rollout
// (no reference counterpart).
//
// FlockLoss is a torch::autograd::Function whose forward runs the taped
// rollout of a brt_engine (brt_adjoint_forward) and returns the FP64 loss of
// every flock, and whose backward runs the hand-written CUDA adjoint
// (brt_adjoint_backward).  Inputs:
//   weights  [nflocks, 3] float32 CUDA  separation / alignment / cohesion
//   pos0     [N, 3]       float32 CUDA  initial positions (agent-id order)
//   vel0     [N, 3]       float32 CUDA  initial velocities (forward * speed)
//   target   [N, 3]       float32 CUDA  target final positions
// Gradients flow to weights, pos0 and vel0 (the initial smoothed
// acceleration is zero).  Everything goes through the C-ABI; the engine runs
// on its own stream, synchronised with torch's current stream on entry and
// exit.
#include <torch/extension.h>
#include <c10/cuda/CUDAStream.h>

#include <string>
#include <vector>

#include "../../include/behavert_b200.h"

namespace {

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::tensor_list;

brt_engine* engineOf(int64_t h) { return reinterpret_cast<brt_engine*>(static_cast<intptr_t>(h)); }

void check(int status, const char* what) {
  if (status != BRT_OK) {
    const char* msg = brt_last_error();
    TORCH_CHECK(false, what, " failed: status ", status, " (", msg ? msg : "", ")");
  }
}

Tensor asFloat4(const Tensor& x, float w) {
  auto out = torch::full({x.size(0), 4}, w, x.options().dtype(torch::kFloat32));
  out.narrow(1, 0, 3).copy_(x.narrow(1, 0, 3));
  return out.contiguous();
}

void checkInput(const Tensor& t, const char* name, int64_t rows, int64_t cols) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.scalar_type() == torch::kFloat32, name, " must be float32");
  TORCH_CHECK(t.dim() == 2 && t.size(0) == rows && t.size(1) == cols, name, " has the wrong shape");
}

class FlockLoss : public torch::autograd::Function<FlockLoss> {
 public:
  static Tensor forward(AutogradContext* ctx, int64_t engine, Tensor weights, Tensor pos0, Tensor vel0, Tensor target,
                        double dt, int64_t nsteps, int64_t checkpoint_every) {
    brt_engine* e = engineOf(engine);
    uint32_t n = 0;
    check(brt_engine_num_agents(e, &n), "brt_engine_num_agents");
    const int64_t nflocks = weights.size(0);
    checkInput(weights, "weights", nflocks, 3);
    checkInput(pos0, "pos0", n, 3);
    checkInput(vel0, "vel0", n, 3);
    checkInput(target, "target", n, 3);
    torch::NoGradGuard noGrad;
    Tensor w = weights.contiguous();
    Tensor pos4 = asFloat4(pos0, 1.0f);
    Tensor v = vel0.narrow(1, 0, 3);
    Tensor speed = v.norm(2, 1, true);
    Tensor fwd4 = torch::cat({v / speed, speed}, 1).contiguous();
    Tensor acc4 = torch::zeros_like(pos4);
    Tensor tgt4 = asFloat4(target, 1.0f);
    Tensor loss = torch::empty({nflocks}, weights.options().dtype(torch::kFloat64));
    c10::cuda::getCurrentCUDAStream().synchronize();
    check(brt_set_steering_weights(e, w.data_ptr<float>(), BRT_MEM_DEVICE), "brt_set_steering_weights");
    check(brt_set_state(e, pos4.data_ptr<float>(), fwd4.data_ptr<float>(), acc4.data_ptr<float>(), nullptr, BRT_MEM_DEVICE),
          "brt_set_state");
    check(brt_adjoint_forward(e, (float)dt, (uint32_t)nsteps, (uint32_t)checkpoint_every, tgt4.data_ptr<float>(),
                              BRT_MEM_DEVICE, loss.data_ptr<double>()),
          "brt_adjoint_forward");
    check(brt_sync(e), "brt_sync");
    ctx->saved_data["engine"] = engine;
    ctx->saved_data["nflocks"] = nflocks;
    ctx->saved_data["n"] = (int64_t)n;
    return loss;
  }

  static tensor_list backward(AutogradContext* ctx, tensor_list grads) {
    brt_engine* e = engineOf(ctx->saved_data["engine"].toInt());
    const int64_t nflocks = ctx->saved_data["nflocks"].toInt();
    const int64_t n = ctx->saved_data["n"].toInt();
    Tensor g = grads[0];
    std::vector<double> scale(nflocks, 0.0);
    if (g.defined()) {
      Tensor gc = g.to(torch::kCPU, torch::kFloat64).contiguous();
      for (int64_t f = 0; f < nflocks; ++f) scale[f] = gc.data_ptr<double>()[f];
    }
    auto opts = torch::TensorOptions().device(torch::kCUDA, c10::cuda::current_device());
    Tensor gpos = torch::empty({n, 4}, opts.dtype(torch::kFloat32));
    Tensor gvel = torch::empty({n, 4}, opts.dtype(torch::kFloat32));
    Tensor gw = torch::empty({nflocks, 3}, opts.dtype(torch::kFloat64));
    c10::cuda::getCurrentCUDAStream().synchronize();
    check(brt_adjoint_backward(e, scale.data(), nullptr, nullptr, nullptr, BRT_MEM_DEVICE, gpos.data_ptr<float>(), nullptr,
                               gvel.data_ptr<float>(), nullptr, gw.data_ptr<double>(), BRT_MEM_DEVICE),
          "brt_adjoint_backward");
    check(brt_sync(e), "brt_sync");
    return {Tensor(), gw.to(torch::kFloat32), gpos.narrow(1, 0, 3), gvel.narrow(1, 0, 3), Tensor(), Tensor(), Tensor(),
            Tensor()};
  }
};

Tensor flockLoss(int64_t engine, Tensor weights, Tensor pos0, Tensor vel0, Tensor target, double dt, int64_t nsteps,
                 int64_t checkpoint_every) {
  return FlockLoss::apply(engine, weights, pos0, vel0, target, dt, nsteps, checkpoint_every);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "libtorch autograd binding of the behavert_b200 differentiable rollout";
  m.def("flock_loss", &flockLoss,
        "Per-flock FP64 loss of a taped rollout; differentiable in weights, pos0 and vel0",
        py::arg("engine"), py::arg("weights"), py::arg("pos0"), py::arg("vel0"), py::arg("target"), py::arg("dt"),
        py::arg("nsteps"), py::arg("checkpoint_every"));
}
