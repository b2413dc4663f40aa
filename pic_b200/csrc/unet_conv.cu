// unet_conv.cu -- 3x3 convolutions of the learned preconditioner on the
// 5th-generation tensor cores.
//
// Implicit-GEMM convolutions built from the CUTLASS SM100 collectives:
// TMA im2col/tiled loads into shared memory, tcgen05.mma (kind::f16, BF16
// operands for both A and B, FP32 accumulation in TMEM), TMA-store epilogue.
// Two kernels (the weight gradient is unet_wgrad in unet_ops.cu):
//   fprop  y = ReLU(conv(x, W) + b)      BF16 out, bias + ReLU fused
//   dgrad  dx = conv^T(dy, W)            BF16 out
// Activations are NHWC, filters KRSC.  Channel counts must be multiples of
// 8 (16-byte TMA rows).  Cluster shape 1x1x1: no TMA multicast.
#include "cutlass/cutlass.h"
#include "cutlass/kernel_hardware_info.hpp"
#include "cute/tensor.hpp"
#include "cutlass/conv/convnd_problem_shape.hpp"
#include "cutlass/conv/dispatch_policy.hpp"
#include "cutlass/conv/collective/collective_builder.hpp"
#include "cutlass/conv/kernel/conv_universal.hpp"
#include "cutlass/conv/device/conv_universal_adapter.hpp"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/epilogue/thread/activation.h"
#include "cutlass/epilogue/fusion/operations.hpp"

#include "../../include/picunet.h"

using namespace cute;

namespace {

using BF16 = cutlass::bfloat16_t;
using TileShape = Shape<_128, _64, Shape<_64>>;
using ClusterShape = Shape<_1, _1, _1>;

template <cutlass::conv::Operator Op, class ElementOut, class FusionOp>
struct ConvT {
  using CollectiveEpilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, TileShape, ClusterShape,
      cutlass::epilogue::collective::EpilogueTileAuto, float, float, ElementOut, cutlass::layout::TensorNHWC,
      128 / cutlass::sizeof_bits<ElementOut>::value, ElementOut, cutlass::layout::TensorNHWC,
      128 / cutlass::sizeof_bits<ElementOut>::value, cutlass::epilogue::collective::EpilogueScheduleAuto,
      FusionOp>::CollectiveOp;
  using CollectiveMainloop = typename cutlass::conv::collective::CollectiveBuilder<
      cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, Op, BF16, cutlass::layout::TensorNHWC, 8, BF16,
      cutlass::layout::TensorNHWC, 8, float, TileShape, ClusterShape,
      cutlass::conv::collective::StageCountAutoCarveout<static_cast<int>(
          sizeof(typename CollectiveEpilogue::SharedStorage))>,
      cutlass::conv::collective::KernelScheduleAuto>::CollectiveOp;
  using ProblemShape =
      cutlass::conv::ConvProblemShape<Op, CollectiveMainloop::DispatchPolicy::NumSpatialDimensions>;
  using Kernel = cutlass::conv::kernel::ConvUniversal<ProblemShape, CollectiveMainloop, CollectiveEpilogue>;
  using Device = cutlass::conv::device::ConvUniversalAdapter<Kernel>;
};

using FpropFusion = cutlass::epilogue::fusion::LinCombPerColBiasEltAct<cutlass::epilogue::thread::ReLu, BF16,
                                                                        float, BF16, BF16>;
using Fprop = ConvT<cutlass::conv::Operator::kFprop, BF16, FpropFusion>;
using Dgrad = ConvT<cutlass::conv::Operator::kDgrad, BF16,
                    cutlass::epilogue::fusion::LinearCombination<BF16, float, BF16, float>>;

template <class T>
typename T::ProblemShape problem(int n, int h, int w, int c, int k) {
  return typename T::ProblemShape(cutlass::conv::Mode::kCrossCorrelation, {n, h, w, c}, {k, 3, 3, c}, {1, 1},
                                  {1, 1}, {1, 1}, {1, 1}, 1);
}

// NHWC strides of the epilogue's C/D tensors, ((W, H, N), _1, _0), from the
// problem's own C tensor (whose strides are listed N, H, W, C).
template <class T>
typename T::Kernel::StrideC out_stride(const typename T::ProblemShape &ps) {
  typename T::Kernel::StrideC s{};
  cute::get<0, 0>(s) = ps.stride_C[2];
  cute::get<0, 1>(s) = ps.stride_C[1];
  cute::get<0, 2>(s) = ps.stride_C[0];
  return s;
}

template <class T>
int run_conv(typename T::Device::Arguments &args, void *ws, size_t ws_bytes, size_t *ws_need, void *stream) {
  typename T::Device op;
  if (op.can_implement(args) != cutlass::Status::kSuccess) return UNET_ERR_SHAPE;
  size_t need = T::Device::get_workspace_size(args);
  if (ws_need) *ws_need = need;
  if (!stream && ws_need && !ws) return UNET_OK;  // size query only
  if (need > ws_bytes) return UNET_ERR_WORKSPACE;
  if (op.initialize(args, ws, (cudaStream_t)stream) != cutlass::Status::kSuccess) return UNET_ERR_CUDA;
  if (op.run((cudaStream_t)stream) != cutlass::Status::kSuccess) return UNET_ERR_CUDA;
  return UNET_OK;
}

}  // namespace

extern "C" int unet_conv(int32_t op, int32_t n, int32_t h, int32_t w, int32_t c, int32_t k, const void *a,
                         const void *b, void *d, const void *bias, void *workspace, size_t ws_bytes,
                         size_t *ws_need, void *stream) {
  if (n < 1 || h < 1 || w < 1 || c < 8 || k < 8 || (c % 8) || (k % 8)) return UNET_ERR_SHAPE;
  const bool query = (ws_need && !workspace && !stream);
  if (!query && (!a || !b || !d)) return UNET_ERR_SHAPE;
  if (op == UNET_FPROP_RELU) {
    if (!query && !bias) return UNET_ERR_SHAPE;
    auto ps = problem<Fprop>(n, h, w, c, k);
    auto sd = out_stride<Fprop>(ps);
    typename Fprop::Device::Arguments args{ps, {(const BF16 *)a, (const BF16 *)b},
                                           {{}, (const BF16 *)d, sd, (BF16 *)d, sd}};
    args.epilogue.thread.alpha = 1.0f;
    args.epilogue.thread.beta = 0.0f;
    args.epilogue.thread.bias_ptr = (const BF16 *)bias;
    return run_conv<Fprop>(args, workspace, ws_bytes, ws_need, stream);
  }
  if (op == UNET_DGRAD) {
    auto ps = problem<Dgrad>(n, h, w, c, k);
    auto sd = out_stride<Dgrad>(ps);
    typename Dgrad::Device::Arguments args{ps, {(const BF16 *)a, (const BF16 *)b},
                                           {{}, (const BF16 *)d, sd, (BF16 *)d, sd}};
    args.epilogue.thread.alpha = 1.0f;
    args.epilogue.thread.beta = 0.0f;
    return run_conv<Dgrad>(args, workspace, ws_bytes, ws_need, stream);
  }
  return UNET_ERR_SHAPE;
}
