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

// Inference form with BF16 activations (channels-last, C a multiple of 16):
// the input arrives by TMA through a tensor map made by tc_map_encode, the
// weights by a bulk copy from the layout tc_weights writes, the output is
// BF16 with bias and ReLU, or (head != NULL, Cout 16) the head's
// x0 = sigmoid(w . relu(y) + b) alpha scale xbp.
struct TcMap {
  alignas(64) unsigned char bytes[128];  // a CUtensorMap
};
struct TcHead {
  const float* w = nullptr;      // 16 weights, bias, alpha
  const float2* xbp = nullptr;
  float scale = 1.f;
  float2* x0 = nullptr;
};
bool tc_map_encode(TcMap* m, const __nv_bfloat16* X, int C, int D, int H, int W);
bool conv3_tc_bf16_supported(int D, int H, int W, int Cin, int Cout);
size_t tc_weights_elems(int Cout, int Cin);
cudaError_t tc_weights(const float* w, int Cout, int Cin, __nv_bfloat16* wp, cudaStream_t st);
cudaError_t conv3_tc_bf16(const TcMap& xmap, int Cin, const __nv_bfloat16* Wp, const float* bias, int Cout,
                          __nv_bfloat16* Y, int D, int H, int W, const TcHead* head, int* err, cudaStream_t st);

// The z-walking form of the same convolution (16 input channels, 16 or 32
// output channels; the head with 16): a block walks z over one (x, y) tile
// with a ring of three input planes, each loaded once, through a tensor map
// made by tc_zmap_encode with `rows` = tcz_rows(Cin) + 2.
bool tcz_supported(int W, int Cin, int Cout);
int tcz_rows(int Cin);
bool tc_zmap_encode(TcMap* m, const __nv_bfloat16* X, int C, int D, int H, int W, int rows);
cudaError_t conv3_tcz(const TcMap& zmap, int Cin, const __nv_bfloat16* Wp, const float* bias, int Cout,
                      __nv_bfloat16* Y, int D, int H, int W, const TcHead* head, int* err, cudaStream_t st);

}  // namespace unet
}  // namespace rihvr
