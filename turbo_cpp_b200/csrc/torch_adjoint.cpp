// torch_adjoint.cpp -- a thin libtorch torch::autograd::Function over the C ABI's differentiable
// decoder (tc_adjoint_forward / tc_adjoint_backward), used by the scale-training harness only.
//
// decode(llr, scales, adjoint_handle, code_blocks, post_len, window, guard, convention)
//   -> posterior
//   llr:         float32 CUDA tensor, [d0|d1|d2] per block at the descriptors' offsets
//   scales:      float32 tensor of 2 * iterations extrinsic scales (any device; read on the host)
//   adjoint_handle: the tc_adjoint* (as an integer) created through the C ABI
//   code_blocks: int64 CPU tensor [n, 4]: K, filler, llr offset, posterior offset
//   convention:  TC_CONVENTION_REFERENCE or TC_CONVENTION_3GPP (the code of the LLRs)
// The backward pass returns d loss / d llr and d loss / d scales; the LLR tensor is saved and
// must not be modified in place before the backward pass.
#include <torch/extension.h>

#include <c10/cuda/CUDAStream.h>

#include <string>
#include <vector>

#include "turbo_b200.h"

namespace {

void check(int rc, const char* what) {
  TORCH_CHECK(rc == TC_OK, what, ": ", tc_status_name(rc), ": ", tc_last_error());
}

class TurboDecode : public torch::autograd::Function<TurboDecode> {
 public:
  static torch::Tensor forward(torch::autograd::AutogradContext* ctx, torch::Tensor llr,
                               torch::Tensor scales, int64_t handle, torch::Tensor code_blocks,
                               int64_t post_len, int64_t window, int64_t guard,
                               int64_t convention) {
    TORCH_CHECK(llr.is_cuda() && llr.scalar_type() == torch::kFloat && llr.is_contiguous(),
                "llr must be a contiguous float32 CUDA tensor");
    TORCH_CHECK(code_blocks.device().is_cpu() && code_blocks.scalar_type() == torch::kLong &&
                    code_blocks.dim() == 2 && code_blocks.size(1) == 4,
                "code_blocks must be an int64 CPU tensor [n, 4]");
    const auto sc = scales.detach().to(torch::kCPU, torch::kFloat).contiguous();
    TORCH_CHECK(sc.numel() >= 2 && sc.numel() % 2 == 0, "scales: two per iteration");
    const auto cb = code_blocks.contiguous();
    const int64_t n = cb.size(0);
    std::vector<tc_code_block> d(static_cast<size_t>(n));
    const int64_t* c = cb.data_ptr<int64_t>();
    for (int64_t i = 0; i < n; ++i) {
      d[i].k = static_cast<int32_t>(c[4 * i]);
      d[i].filler = static_cast<int32_t>(c[4 * i + 1]);
      d[i].llr_offset = c[4 * i + 2];
      d[i].out_offset = c[4 * i + 3];
    }
    auto post = torch::zeros({post_len}, llr.options());
    const c10::cuda::CUDAStream stream = c10::cuda::getCurrentCUDAStream(llr.get_device());
    uint64_t tape = 0;
    auto* adj = reinterpret_cast<tc_adjoint*>(handle);
    check(tc_adjoint_forward_conv(static_cast<int>(convention), adj, static_cast<size_t>(n),
                                  d.data(), static_cast<size_t>(llr.numel()),
                                  llr.data_ptr<float>(), static_cast<size_t>(post_len),
                                  post.data_ptr<float>(), static_cast<uint32_t>(sc.numel() / 2),
                                  sc.data_ptr<float>(), static_cast<int32_t>(window),
                                  static_cast<int32_t>(guard), stream.stream(), &tape),
          "tc_adjoint_forward_conv");
    ctx->save_for_backward({llr, scales});
    ctx->saved_data["handle"] = handle;
    ctx->saved_data["tape"] = static_cast<int64_t>(tape);
    return post;
  }

  static torch::autograd::tensor_list backward(torch::autograd::AutogradContext* ctx,
                                               torch::autograd::tensor_list grads) {
    const auto saved = ctx->get_saved_variables();
    const torch::Tensor& llr = saved[0];
    const torch::Tensor& scales = saved[1];
    auto* adj = reinterpret_cast<tc_adjoint*>(ctx->saved_data["handle"].toInt());
    const auto tape = static_cast<uint64_t>(ctx->saved_data["tape"].toInt());
    const auto gp = grads[0].to(torch::kFloat).contiguous();
    auto g_llr = torch::empty_like(llr);
    auto g_s = torch::empty({scales.numel()}, llr.options());
    const c10::cuda::CUDAStream stream = c10::cuda::getCurrentCUDAStream(llr.get_device());
    check(tc_adjoint_backward(adj, tape, gp.data_ptr<float>(), g_llr.data_ptr<float>(),
                              g_s.data_ptr<float>(), stream.stream()),
          "tc_adjoint_backward");
    return {g_llr, g_s.to(scales.options()).view(scales.sizes()), torch::Tensor(),
            torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor(), torch::Tensor()};
  }
};

torch::Tensor decode(torch::Tensor llr, torch::Tensor scales, int64_t handle,
                     torch::Tensor code_blocks, int64_t post_len, int64_t window, int64_t guard,
                     int64_t convention) {
  return TurboDecode::apply(llr, scales, handle, code_blocks, post_len, window, guard, convention);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("decode", &decode,
        "differentiable turbo decode (posterior LLRs) through the hand-written adjoint");
}
