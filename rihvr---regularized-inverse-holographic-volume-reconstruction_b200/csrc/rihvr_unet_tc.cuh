// tcgen05 (5th-generation tensor core) 3x3x3 convolution of the warm-start
// U-Net: layers whose width is a multiple of 128 (rihvr_unet_tc.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace rihvr {
namespace unet {

// width a multiple of 128, Cin a multiple of 16, Cn 16, 32, 48 or 64
bool conv3_tc_supported(int W, int Cin, int Cn);

// Y[v][co0 + j] = act(bias[co0 + j] + sum over taps and ci of X[v + off][ci] Wt[co0 + j][tap][ci]),
// j < Cn; taps mirrored when `mirror`.  X: D x H x W x Cin FP32 channels-last,
// Wt: Cout x 27 x Cin BF16, Y: D x H x W x Cout FP32.  *err is set to 1 when a
// bounded wait for the tensor cores ran out (the output is then incomplete).
cudaError_t conv3_tc(const float* X, int Cin, const __nv_bfloat16* Wt, int Cout, int co0, int Cn, const float* bias,
                     float* Y, int D, int H, int W, int relu, int mirror, int* err, cudaStream_t st);

}  // namespace unet
}  // namespace rihvr
