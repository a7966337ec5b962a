// Learned warm start: a 3-D U-Net that maps the back-propagated volume
// t A^H b to an initial FISTA iterate.  No counterpart in the reference (its
// reconstruction always starts from x = 0, sparse_compressive_holo.cu:273);
// plain FISTA from zero stays the fallback and the reference for the result.
//
// Network (3 levels, 16/32/64 channels), activations FP32 channels-last
// [z][y][x][c], weights FP32 masters with BF16 copies:
//   input  |xbp| / rms(|xbp|)                        1 channel (padded to 16)
//   enc1   conv3 16 -> 16, ReLU, conv3 16 -> 16, ReLU           = s1
//   pool   2x2x2 average
//   enc2   conv3 16 -> 32, ReLU, conv3 32 -> 32, ReLU           = s2
//   pool
//   bottom conv3 32 -> 64, ReLU, conv3 64 -> 64, ReLU
//   up     nearest x2, concat s2 (96): conv3 96 -> 32, ReLU, conv3 32 -> 32, ReLU
//   up     nearest x2, concat s1 (48): conv3 48 -> 16, ReLU, conv3 16 -> 16, ReLU
//   head   1x1x1 16 -> 1, sigmoid = gain g
//   output x0 = g * alpha * xbp (alpha a learned scalar)
// Loss: sum |x0 - x*|^2 / sum |x*|^2 against the plain-FISTA solution x*.
//
// The 3x3x3 convolutions are implicit GEMMs on the tensor cores.  Layers
// whose width is a multiple of 128 run on the 5th-generation tensor cores
// (tcgen05.mma with accumulators in tensor memory, rihvr_unet_tc.cu); the
// others on the warp-level instruction (mma.sync m16n8k16, BF16 operands,
// FP32 accumulation): a block computes 64
// output voxels x all output channels; the K loop runs over the 27 taps and
// 16-channel slices, staging a 64 x 16 activation tile (zero outside the
// volume, converted to BF16) and a 16 x Cout weight tile in shared memory.
// The data gradient is the same kernel with the taps mirrored and the weight
// matrix transposed; the weight gradient is a split-K GEMM (K = voxels) on the
// same instruction with FP32 atomics into the gradient.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/rihvr.h"
#include "rihvr_kernels.cuh"
#include "rihvr_unet_tc.cuh"

namespace rihvr {
namespace unet {

struct Vol {
  int D, H, W;
  __host__ __device__ long long n() const { return (long long)D * H * W; }
};

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (low half) = lo
  return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// tap k = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1); mirrored tap = 26 - k
__device__ __forceinline__ void tap_offsets(int k, int* dz, int* dy, int* dx) {
  *dz = k / 9 - 1;
  *dy = (k / 3) % 3 - 1;
  *dx = k % 3 - 1;
}

// Y[v][co] = act(bias[co] + sum_k sum_ci X[v + off_k][ci] Wt[co][k][ci]) for
// the output channels co0 .. co0 + Cn - 1 of Cout (Cn a multiple of 8, at most
// 64); Cin a multiple of 16.  Taps are mirrored when `mirror` (the data
// gradient).
//
// A block makes a brick of 2 (z) x 2 MT (y) x 16 (x) output voxels; each of
// its 4 warps MT rows of 16 voxels (MT m-tiles) and NT tiles of 8 output
// channels.  Per 16-channel slice of the input it stages the brick's halo
// (4 x (2 MT + 2) x 18 voxels, zero outside the volume, BF16) and the slice's
// weights for all 27 taps in shared memory, then runs the 27 taps from there:
// the A fragment of a tap is the halo shifted by the tap's offset, so nothing
// is restaged between taps.  A shared row holds 16 BF16 (two 16-byte chunks)
// with no padding; chunk c of row r sits at position c ^ ((r >> 2) & 1), so the
// 8 consecutive rows of a fragment load cover the 32 banks once whatever the
// first row (rows r and r + 4 land 16 bytes apart).  Narrow layers (16 or 32
// channels) take MT = 4: taller bricks, fewer halo voxels per output and
// smaller weight tiles, so more blocks fit per SM.
constexpr int kConvThreads = 128;
constexpr int kBZ = 2, kBX = 16, kHX = kBX + 2;
constexpr int kRow = 16;  // BF16 per shared row

// element offset of 16-byte chunk c (0 or 1) of shared row r
__device__ __forceinline__ int swz(int r, int c) { return r * kRow + ((c ^ (r >> 2)) & 1) * 8; }

template <int MT>
struct Brick {
  static constexpr int BY = 2 * MT, HZ = kBZ + 2, HY = BY + 2, HALO = HZ * HY * kHX;
};
template <int MT>
constexpr size_t conv_smem(int Cn) {
  return sizeof(__nv_bfloat16) * kRow * (Brick<MT>::HALO + 27 * (size_t)Cn);
}

template <int NT, int MT>
__global__ void __launch_bounds__(kConvThreads) k_conv3(const float* __restrict__ X, int Cin,
                                                        const __nv_bfloat16* __restrict__ Wt, int Cout, int co0,
                                                        const float* __restrict__ bias, float* __restrict__ Y,
                                                        Vol v, int relu, int mirror) {
  using Bk = Brick<MT>;
  constexpr int Cn = NT * 8;
  extern __shared__ __align__(16) __nv_bfloat16 csm[];
  __nv_bfloat16* Hs = csm;                    // [HALO][kRow]
  __nv_bfloat16* Ws = csm + Bk::HALO * kRow;  // [27 * Cn][kRow]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nbx = (v.W + kBX - 1) / kBX, nby = (v.H + Bk::BY - 1) / Bk::BY;
  const int bx = blockIdx.x % nbx, by = (blockIdx.x / nbx) % nby, bz = blockIdx.x / (nbx * nby);
  const int x0 = bx * kBX, y0 = by * Bk::BY, z0 = bz * kBZ;
  float acc[MT][NT][4];
#pragma unroll
  for (int r = 0; r < MT; ++r)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[r][j][0] = acc[r][j][1] = acc[r][j][2] = acc[r][j][3] = 0.f;
  const int nslice = Cin / 16;
  for (int s = 0; s < nslice; ++s) {
    // halo of the brick, 16 channels: two threads a voxel row of 8 channels
    for (int e = tid; e < Bk::HALO * 2; e += kConvThreads) {
      const int h = e >> 1, half = e & 1;
      const int hx = h % kHX, hy = (h / kHX) % Bk::HY, hz = h / (kHX * Bk::HY);
      const int xx = x0 + hx - 1, yy = y0 + hy - 1, zz = z0 + hz - 1;
      float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), hi = lo;
      if (xx >= 0 && xx < v.W && yy >= 0 && yy < v.H && zz >= 0 && zz < v.D) {
        const float* src = X + (((long long)zz * v.H + yy) * v.W + xx) * Cin + s * 16 + half * 8;
        lo = *reinterpret_cast<const float4*>(src);
        hi = *reinterpret_cast<const float4*>(src + 4);
      }
      uint4 pk;
      pk.x = pack_bf16(lo.x, lo.y);
      pk.y = pack_bf16(lo.z, lo.w);
      pk.z = pack_bf16(hi.x, hi.y);
      pk.w = pack_bf16(hi.z, hi.w);
      *reinterpret_cast<uint4*>(Hs + swz(h, half)) = pk;
    }
    // weights of the slice for every tap: row k * Cn + co
    for (int e = tid; e < 27 * Cn * 2; e += kConvThreads) {
      const int row = e >> 1, half = e & 1;
      const int k = row / Cn, co = row - k * Cn;
      *reinterpret_cast<uint4*>(Ws + swz(row, half)) =
          *reinterpret_cast<const uint4*>(Wt + ((long long)(co0 + co) * 27 + k) * Cin + s * 16 + half * 8);
    }
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < 27; ++k) {
      int dz, dy, dx;
      tap_offsets(mirror ? 26 - k : k, &dz, &dy, &dx);
      unsigned b[NT][2];
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int br = k * Cn + j * 8 + g;
        b[j][0] = *reinterpret_cast<const unsigned*>(Ws + swz(br, 0) + 2 * t);
        b[j][1] = *reinterpret_cast<const unsigned*>(Ws + swz(br, 1) + 2 * t);
      }
#pragma unroll
      for (int r = 0; r < MT; ++r) {
        // m-tile r of this warp: the x-row (z, y) of the brick, voxels x = 0..15
        const int row = warp * MT + r;
        const int mz = row / Bk::BY, my = row % Bk::BY;
        const int hb = ((mz + dz + 1) * Bk::HY + (my + dy + 1)) * kHX + dx + 1;
        const int rl = hb + g, rh = hb + g + 8;
        const unsigned a0 = *reinterpret_cast<const unsigned*>(Hs + swz(rl, 0) + 2 * t);
        const unsigned a1 = *reinterpret_cast<const unsigned*>(Hs + swz(rh, 0) + 2 * t);
        const unsigned a2 = *reinterpret_cast<const unsigned*>(Hs + swz(rl, 1) + 2 * t);
        const unsigned a3 = *reinterpret_cast<const unsigned*>(Hs + swz(rh, 1) + 2 * t);
#pragma unroll
        for (int j = 0; j < NT; ++j) mma_bf16(acc[r][j], a0, a1, a2, a3, b[j][0], b[j][1]);
      }
    }
    __syncthreads();
  }
  // epilogue: rows g and g + 8 of each m-tile, columns 2t, 2t + 1 of each n-tile
#pragma unroll
  for (int r = 0; r < MT; ++r) {
    const int row = warp * MT + r;
    const int zz = z0 + row / Bk::BY, yy = y0 + row % Bk::BY;
    if (zz >= v.D || yy >= v.H) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int co = co0 + j * 8 + 2 * t;
      const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int xx = x0 + g + h * 8;
        if (xx >= v.W) continue;
        float y0v = acc[r][j][2 * h] + b0, y1v = acc[r][j][2 * h + 1] + b1;
        if (relu) {
          y0v = fmaxf(y0v, 0.f);
          y1v = fmaxf(y1v, 0.f);
        }
        *reinterpret_cast<float2*>(Y + (((long long)zz * v.H + yy) * v.W + xx) * Cout + co) =
            make_float2(y0v, y1v);
      }
    }
  }
}

template <int NT, int MT>
cudaError_t conv3_launch(const float* X, int Cin, const __nv_bfloat16* Wt, int Cout, int co0, const float* bias,
                         float* Y, Vol v, int relu, int mirror, cudaStream_t st) {
  const size_t smem = conv_smem<MT>(NT * 8);
  static bool opted = false;  // shared-memory opt-in, once per instantiation
  if (!opted) {
    const cudaError_t e = cudaFuncSetAttribute(k_conv3<NT, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  const unsigned blocks = (unsigned)(((v.W + kBX - 1) / kBX) * ((v.H + Brick<MT>::BY - 1) / Brick<MT>::BY) *
                                     ((v.D + kBZ - 1) / kBZ));
  k_conv3<NT, MT><<<blocks, kConvThreads, smem, st>>>(X, Cin, Wt, Cout, co0, bias, Y, v, relu, mirror);
  return cudaGetLastError();
}

// the z-walking form of the BF16 convolutions, where a layer qualifies,
// unless RIHVR_UNET_ZWALK=0
bool use_zwalk() {
  static const bool on = [] {
    const char* e = std::getenv("RIHVR_UNET_ZWALK");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

// the tcgen05 path is used where it applies unless RIHVR_UNET_MMA=sync
bool use_tcgen05() {
  static const bool on = [] {
    const char* e = std::getenv("RIHVR_UNET_MMA");
    return !(e && std::strcmp(e, "sync") == 0);
  }();
  return on;
}

// output channels co0 .. co0 + Cn - 1 (Cn 16, 32, 48 or 64); `err` receives 1
// if a tcgen05 launch's bounded wait ran out
cudaError_t conv3(const float* X, int Cin, const __nv_bfloat16* Wt, int Cout, int co0, int Cn, const float* bias,
                  float* Y, Vol v, int relu, int mirror, int* err, cudaStream_t st) {
  if (use_tcgen05() && conv3_tc_supported(v.W, Cin, Cn))
    return conv3_tc(X, Cin, Wt, Cout, co0, Cn, bias, Y, v.D, v.H, v.W, relu, mirror, err, st);
  switch (Cn) {
    case 16: return conv3_launch<2, 4>(X, Cin, Wt, Cout, co0, bias, Y, v, relu, mirror, st);
    case 32: return conv3_launch<4, 4>(X, Cin, Wt, Cout, co0, bias, Y, v, relu, mirror, st);
    case 48: return conv3_launch<6, 2>(X, Cin, Wt, Cout, co0, bias, Y, v, relu, mirror, st);
    case 64: return conv3_launch<8, 2>(X, Cin, Wt, Cout, co0, bias, Y, v, relu, mirror, st);
    default: return cudaErrorInvalidValue;
  }
}

// dW[co][k][ci] += sum_v dY[v][co] X[v + off_k][ci] over a chunk of voxels:
// M = Cout (up to 4 tiles of 16), N = 16 input channels, K = voxels.  Each
// warp takes its own 16-voxel steps and adds its partial tile with atomics.
// Grid: (voxel chunks, 27 taps, Cin / 16 slices).
constexpr int kWgVox = 1024;  // voxels a block
__global__ void __launch_bounds__(128) k_conv3_wgrad(const float* __restrict__ X, int Cin,
                                                      const float* __restrict__ dY, int Cout,
                                                      float* __restrict__ dW, Vol v) {
  __shared__ __align__(16) __nv_bfloat16 At[4][64][16];  // [warp][co][voxel]
  __shared__ __align__(16) __nv_bfloat16 Bt[4][16][16];  // [warp][ci][voxel]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int k = blockIdx.y, s = blockIdx.z;
  int dz, dy, dx;
  tap_offsets(k, &dz, &dy, &dx);
  const long long n = v.n();
  const int mt = Cout / 16;
  float acc[4][2][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = acc[i][j][2] = acc[i][j][3] = 0.f;
  const long long base = (long long)blockIdx.x * kWgVox;
  for (int step = warp; step < kWgVox / 16; step += 4) {
    const long long v0 = base + step * 16;
    if (v0 >= n) break;
    // dY tile, transposed: At[co][i] = dY[v0 + i][co]
    for (int e = lane; e < 16 * Cout; e += 32) {
      const int i = e / Cout, co = e - i * Cout;
      const long long vv = v0 + i;
      At[warp][co][i] = __float2bfloat16_rn(vv < n ? dY[vv * Cout + co] : 0.f);
    }
    // X tile at the tap, transposed: Bt[ci][i] = X[v0 + i + off][16 s + ci]
    for (int e = lane; e < 256; e += 32) {
      const int i = e >> 4, ci = e & 15;
      const long long vv = v0 + i;
      float x = 0.f;
      if (vv < n) {
        const int xx = (int)(vv % v.W) + dx, yy = (int)((vv / v.W) % v.H) + dy,
                  zz = (int)(vv / ((long long)v.W * v.H)) + dz;
        if (zz >= 0 && zz < v.D && yy >= 0 && yy < v.H && xx >= 0 && xx < v.W)
          x = X[(((long long)zz * v.H + yy) * v.W + xx) * Cin + s * 16 + ci];
      }
      Bt[warp][ci][i] = __float2bfloat16_rn(x);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i >= mt) continue;
      const unsigned a0 = *reinterpret_cast<const unsigned*>(&At[warp][i * 16 + g][2 * t]);
      const unsigned a1 = *reinterpret_cast<const unsigned*>(&At[warp][i * 16 + g + 8][2 * t]);
      const unsigned a2 = *reinterpret_cast<const unsigned*>(&At[warp][i * 16 + g][2 * t + 8]);
      const unsigned a3 = *reinterpret_cast<const unsigned*>(&At[warp][i * 16 + g + 8][2 * t + 8]);
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const unsigned b0 = *reinterpret_cast<const unsigned*>(&Bt[warp][j * 8 + g][2 * t]);
        const unsigned b1 = *reinterpret_cast<const unsigned*>(&Bt[warp][j * 8 + g][2 * t + 8]);
        mma_bf16(acc[i][j], a0, a1, a2, a3, b0, b1);
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= mt) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int co = i * 16 + g + h * 8, ci = s * 16 + j * 8 + 2 * t;
        float* d = dW + ((long long)co * 27 + k) * Cin + ci;
        atomicAdd(d, acc[i][j][2 * h]);
        atomicAdd(d + 1, acc[i][j][2 * h + 1]);
      }
  }
}

// db[co] += sum_v dY[v][co]
__global__ void k_bias_grad(const float* __restrict__ dY, int C, long long n, float* __restrict__ db) {
  __shared__ float part[64];
  if (threadIdx.x < 64) part[threadIdx.x] = 0.f;
  __syncthreads();
  const int c = threadIdx.x % C;
  const int lanes = blockDim.x / C;
  float s = 0.f;
  for (long long vv = (long long)blockIdx.x * lanes + threadIdx.x / C; vv < n; vv += (long long)gridDim.x * lanes)
    if (threadIdx.x < lanes * C) s += dY[vv * C + c];
  if (threadIdx.x < lanes * C) atomicAdd(&part[c], s);
  __syncthreads();
  if (threadIdx.x < C) atomicAdd(&db[threadIdx.x], part[threadIdx.x]);
}

// dY *= (Y > 0): through the ReLU whose output is Y
__global__ void k_relu_back(float* __restrict__ dY, const float* __restrict__ Y, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(Y[i] > 0.f)) dY[i] = 0.f;
}

// 2x2x2 average pool (fine volume f, coarse c) and its gradient
__global__ void k_pool(const float* __restrict__ X, float* __restrict__ Y, Vol c, int C) {
  const long long n = c.n() * C;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % C);
    const long long vv = e / C;
    const int x = (int)(vv % c.W), y = (int)((vv / c.W) % c.H), z = (int)(vv / ((long long)c.W * c.H));
    const int W2 = 2 * c.W, H2 = 2 * c.H;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      s += X[((((long long)(2 * z + (q >> 2)) * H2 + 2 * y + ((q >> 1) & 1)) * W2) + 2 * x + (q & 1)) * C + ch];
    Y[e] = s * 0.125f;
  }
}
// dX = (gradient through the pool) + S, S the skip gradient of the same tensor
__global__ void k_pool_back(const float* __restrict__ dY, const float* __restrict__ S, float* __restrict__ dX,
                            Vol f, int C) {
  const long long n = f.n() * C;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % C);
    const long long vv = e / C;
    const int x = (int)(vv % f.W), y = (int)((vv / f.W) % f.H), z = (int)(vv / ((long long)f.W * f.H));
    dX[e] = 0.125f * dY[((((long long)(z >> 1) * (f.H >> 1)) + (y >> 1)) * (f.W >> 1) + (x >> 1)) * C + ch] + S[e];
  }
}

// nearest x2 upsampling of Cu channels into channels [0, Cu) of a (Cu + Cs)-
// channel tensor whose channels [Cu, Cu + Cs) are the skip tensor S
__global__ void k_up_concat(const float* __restrict__ U, int Cu, const float* __restrict__ S, int Cs,
                            float* __restrict__ Y, Vol f) {
  const int C = Cu + Cs;
  const long long n = f.n() * C;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % C);
    const long long vv = e / C;
    if (ch >= Cu) {
      Y[e] = S[vv * Cs + ch - Cu];
    } else {
      const int x = (int)(vv % f.W), y = (int)((vv / f.W) % f.H), z = (int)(vv / ((long long)f.W * f.H));
      Y[e] = U[((((long long)(z >> 1) * (f.H >> 1)) + (y >> 1)) * (f.W >> 1) + (x >> 1)) * Cu + ch];
    }
  }
}
// its gradient: dU (coarse) = sum of the 8 children of channels [0, Cu);
// dS = channels [Cu, Cu + Cs)
__global__ void k_up_concat_back(const float* __restrict__ dY, int Cu, int Cs, float* __restrict__ dU,
                                 float* __restrict__ dS, Vol c) {
  const int C = Cu + Cs;
  const int W2 = 2 * c.W, H2 = 2 * c.H;
  const long long nu = c.n() * Cu;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nu; e += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % Cu);
    const long long vv = e / Cu;
    const int x = (int)(vv % c.W), y = (int)((vv / c.W) % c.H), z = (int)(vv / ((long long)c.W * c.H));
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q)
      s += dY[((((long long)(2 * z + (q >> 2)) * H2 + 2 * y + ((q >> 1) & 1)) * W2) + 2 * x + (q & 1)) * C + ch];
    dU[e] = s;
  }
  const long long ns = c.n() * 8 * Cs;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ns; e += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(e % Cs);
    const long long vv = e / Cs;
    dS[e] = dY[vv * C + Cu + ch];
  }
}

// input channel 0 = |xbp| / rms, channels 1..15 = 0
__global__ void k_input(const float2* __restrict__ xbp, long long n, const float* __restrict__ rms,
                        float* __restrict__ X) {
  const float inv = 1.f / fmaxf(rms[0], 1e-30f);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = xbp[i];
    float4* d = reinterpret_cast<float4*>(X + i * 16);
    d[0] = make_float4(sqrtf(a.x * a.x + a.y * a.y) * inv, 0.f, 0.f, 0.f);
    d[1] = d[2] = d[3] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// sum |xbp|^2 (FP64 partials into out[0]) and sum |x*|^2 (out[1])
__global__ void k_sumsq(const float2* __restrict__ a, const float2* __restrict__ b, long long n,
                        double* __restrict__ out) {
  double sa = 0, sb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 p = a[i];
    sa += (double)p.x * p.x + (double)p.y * p.y;
    if (b) {
      const float2 q = b[i];
      sb += (double)q.x * q.x + (double)q.y * q.y;
    }
  }
  for (int o = 16; o; o >>= 1) {
    sa += __shfl_xor_sync(0xffffffffu, sa, o);
    sb += __shfl_xor_sync(0xffffffffu, sb, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, sa);
    if (b) atomicAdd(out + 1, sb);
  }
}
__global__ void k_rms(const double* __restrict__ s, long long n, float* __restrict__ rms) {
  rms[0] = (float)sqrt(s[0] / (double)n);
}

// head: z = b + sum_c w[c] h[v][c]; g = sigmoid(z); x0 = g alpha scale xbp
__global__ void k_head(const float* __restrict__ Hh, const float* __restrict__ w, const float2* __restrict__ xbp,
                       long long n, float scale, float* __restrict__ gout, float2* __restrict__ x0) {
  const float b = w[16], alpha = w[17] * scale;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float z = b;
#pragma unroll
    for (int c = 0; c < 16; ++c) z += w[c] * Hh[i * 16 + c];
    const float g = 1.f / (1.f + expf(-z));
    if (gout) gout[i] = g;
    const float2 a = xbp[i];
    x0[i] = make_float2(g * alpha * a.x, g * alpha * a.y);
  }
}

// loss = sum |x0 - x*|^2 / S* and the gradients: dz[v] (through the sigmoid),
// head weights/bias and alpha (FP32 atomics into dw[0..17]), loss (FP64)
__global__ void k_head_back(const float* __restrict__ Hh, const float* __restrict__ w,
                            const float2* __restrict__ xbp, const float2* __restrict__ xs,
                            const float* __restrict__ gbuf, long long n, const double* __restrict__ sums,
                            float* __restrict__ dH, float* __restrict__ dw, double* __restrict__ loss) {
  const float alpha = w[17];
  const double Sstar = fmax(sums[1], 1e-300);
  const float inv = (float)(1.0 / Sstar);
  float dwl[18];
#pragma unroll
  for (int c = 0; c < 18; ++c) dwl[c] = 0.f;
  double l = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float g = gbuf[i];
    const float2 a = xbp[i], s = xs[i];
    const float er = g * alpha * a.x - s.x, ei = g * alpha * a.y - s.y;
    l += (double)er * er + (double)ei * ei;
    const float proj = er * a.x + ei * a.y;           // Re(conj(e) xbp)
    const float dg = 2.f * inv * alpha * proj;        // dL/dg
    const float dz = dg * g * (1.f - g);              // through the sigmoid
    dwl[17] += 2.f * inv * g * proj;                  // dL/dalpha
    dwl[16] += dz;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      dwl[c] += dz * Hh[i * 16 + c];
      dH[i * 16 + c] = dz * w[c];
    }
  }
  for (int o = 16; o; o >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o);
#pragma unroll
    for (int c = 0; c < 18; ++c) dwl[c] += __shfl_xor_sync(0xffffffffu, dwl[c], o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(loss, l / Sstar);
#pragma unroll
    for (int c = 0; c < 18; ++c) atomicAdd(&dw[c], dwl[c]);
  }
}

// Adam (FP32 masters) and the BF16 copies the convolutions read; the
// transposed copy Wt[ci][k][co] = W[co][k][ci] feeds the data gradient (the
// convolution kernel mirrors the taps' offsets there)
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ s,
                       const float* __restrict__ gr, long long n, float lr, float b1, float b2, float c1, float c2,
                       float eps) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, si = b2 * s[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    s[i] = si;
    w[i] -= lr * (mi * c1) / (sqrtf(si * c2) + eps);
  }
}
__global__ void k_weights_bf16(const float* __restrict__ w, int Cout, int Cin, __nv_bfloat16* __restrict__ wb,
                               __nv_bfloat16* __restrict__ wt) {
  const long long n = (long long)Cout * 27 * Cin;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin), k = (int)((i / Cin) % 27), co = (int)(i / (27LL * Cin));
    const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
    wb[i] = b;
    wt[((long long)ci * 27 + k) * Cout + co] = b;
  }
}

// ---- inference with BF16 activations (channels-last, 8 channels = 16 bytes)

__device__ __forceinline__ unsigned short bf16_bits(float v) {
  const __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<const unsigned short*>(&b);
}

// input channel 0 = |xbp| / rms (the FP32 value k_input writes, rounded as
// the convolutions round their operands), channels 1..15 = 0
__global__ void k_input_bf16(const float2* __restrict__ xbp, long long n, const float* __restrict__ rms,
                             __nv_bfloat16* __restrict__ X) {
  const float inv = 1.f / fmaxf(rms[0], 1e-30f);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = xbp[i];
    uint4* d = reinterpret_cast<uint4*>(X + i * 16);
    d[0] = make_uint4((unsigned)bf16_bits(sqrtf(a.x * a.x + a.y * a.y) * inv), 0u, 0u, 0u);
    d[1] = make_uint4(0u, 0u, 0u, 0u);
  }
}

__device__ __forceinline__ void bf16x8_add(float (&acc)[8], uint4 q) {
  const unsigned u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    acc[2 * j] += __uint_as_float(u[j] << 16);
    acc[2 * j + 1] += __uint_as_float(u[j] & 0xFFFF0000u);
  }
}

// 2x2x2 average pool, 8 channels a thread: FP32 sum of the 8 children in the
// order of k_pool, times 1/8, rounded to BF16
__global__ void k_pool_bf16(const __nv_bfloat16* __restrict__ X, __nv_bfloat16* __restrict__ Y, Vol c, int C) {
  const int G = C / 8;
  const long long n = c.n() * G;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(e % G);
    const long long vv = e / G;
    const int x = (int)(vv % c.W), y = (int)((vv / c.W) % c.H), z = (int)(vv / ((long long)c.W * c.H));
    const int W2 = 2 * c.W, H2 = 2 * c.H;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long src = (((long long)(2 * z + (q >> 2)) * H2 + 2 * y + ((q >> 1) & 1)) * W2) + 2 * x + (q & 1);
      bf16x8_add(acc, *reinterpret_cast<const uint4*>(X + src * C + g * 8));
    }
    uint4 o;
    o.x = (unsigned)bf16_bits(acc[0] * 0.125f) | ((unsigned)bf16_bits(acc[1] * 0.125f) << 16);
    o.y = (unsigned)bf16_bits(acc[2] * 0.125f) | ((unsigned)bf16_bits(acc[3] * 0.125f) << 16);
    o.z = (unsigned)bf16_bits(acc[4] * 0.125f) | ((unsigned)bf16_bits(acc[5] * 0.125f) << 16);
    o.w = (unsigned)bf16_bits(acc[6] * 0.125f) | ((unsigned)bf16_bits(acc[7] * 0.125f) << 16);
    *reinterpret_cast<uint4*>(Y + vv * C + g * 8) = o;
  }
}

// nearest x2 upsampling of U (Cu channels) and concatenation with S (Cs), 8
// channels a thread
__global__ void k_up_concat_bf16(const __nv_bfloat16* __restrict__ U, int Cu, const __nv_bfloat16* __restrict__ S,
                                 int Cs, __nv_bfloat16* __restrict__ Y, Vol f) {
  const int C = Cu + Cs, G = C / 8;
  const long long n = f.n() * G;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(e % G);
    const long long vv = e / G;
    uint4 v;
    if (g * 8 >= Cu) {
      v = *reinterpret_cast<const uint4*>(S + vv * Cs + g * 8 - Cu);
    } else {
      const int x = (int)(vv % f.W), y = (int)((vv / f.W) % f.H), z = (int)(vv / ((long long)f.W * f.H));
      const long long src = (((long long)(z >> 1) * (f.H >> 1)) + (y >> 1)) * (f.W >> 1) + (x >> 1);
      v = *reinterpret_cast<const uint4*>(U + src * Cu + g * 8);
    }
    *reinterpret_cast<uint4*>(Y + vv * C + g * 8) = v;
  }
}

}  // namespace unet
}  // namespace rihvr

using namespace rihvr;
using namespace rihvr::unet;

namespace {

int unet_fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

#define UCK(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return unet_fail(e_ == cudaErrorMemoryAllocation ? RIHVR_ERR_OUT_OF_MEMORY : RIHVR_ERR_CUDA, \
                       std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

int blocks_for(long long n, int threads = 256) {
  const long long b = (n + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

// one 3x3x3 convolution layer
struct Conv {
  int cin, cout, level;
  size_t w_off, b_off;  // offsets in the parameter vector
};

// layers in order; the head (16 weights, bias) and alpha follow them
const Conv kLayers[] = {
    {16, 16, 0, 0, 0}, {16, 16, 0, 0, 0},  // enc1
    {16, 32, 1, 0, 0}, {32, 32, 1, 0, 0},  // enc2
    {32, 64, 2, 0, 0}, {64, 64, 2, 0, 0},  // bottom
    {96, 32, 1, 0, 0}, {32, 32, 1, 0, 0},  // dec2
    {48, 16, 0, 0, 0}, {16, 16, 0, 0, 0},  // dec1
};
constexpr int kNumConv = 10;

}  // namespace

struct rihvr_unet {
  Vol lv[3];
  Conv layers[kNumConv];
  size_t nparam = 0, head_off = 0;
  // parameters, gradients, Adam moments (FP32); BF16 copies per layer (the
  // weights and their mirrored transpose for the data gradient)
  float *w = nullptr, *gw = nullptr, *m = nullptr, *s = nullptr;
  __nv_bfloat16 *wb = nullptr, *wt = nullptr;
  size_t wb_off[kNumConv] = {};
  int step = 0;
  // forward: act[i] = output of conv i (after its ReLU); in0 the input;
  // p1, p2 the pooled tensors; c2, c1 the concatenations; gbuf the gain
  float* act[kNumConv] = {};
  float *in0 = nullptr, *p1 = nullptr, *p2 = nullptr, *c2 = nullptr, *c1 = nullptr, *gbuf = nullptr;
  // backward scratch: level 0 (16 ch: A0a, A0b, S0; 48 ch: C0), level 1
  // (32 ch: B1a, B1b, S1; 96 ch: C1; 16 ch: P1), level 2 (64 ch: D2a, D2b; 32 ch: P2)
  float *A0a = nullptr, *A0b = nullptr, *S0 = nullptr, *C0 = nullptr;
  float *B1a = nullptr, *B1b = nullptr, *S1 = nullptr, *C1 = nullptr, *P1 = nullptr;
  float *D2a = nullptr, *D2b = nullptr, *P2 = nullptr;
  // inference with BF16 activations (predict on widths that are multiples of
  // 512, where every level runs on tcgen05): weights in the bulk-copy layout,
  // activations allocated on first use, one TMA tensor map per layer input
  __nv_bfloat16* wtc = nullptr;
  size_t wtc_off[kNumConv] = {};
  bool bf_ready = false;
  bool bf_failed = false;  // the tensor maps could not be made: predict keeps the FP32 path
  __nv_bfloat16 *b_in0 = nullptr, *b_a0 = nullptr, *b_a1 = nullptr, *b_c1 = nullptr;  // level 0
  __nv_bfloat16 *b_p1 = nullptr, *b_a2 = nullptr, *b_a3 = nullptr, *b_c2 = nullptr, *b_a7 = nullptr;  // level 1
  __nv_bfloat16 *b_p2 = nullptr, *b_a4 = nullptr, *b_a5 = nullptr;  // level 2
  TcMap maps[kNumConv];
  TcMap zmaps[kNumConv];  // the z-walking form's maps, where a layer takes it
  bool zwalk[kNumConv] = {};
  double* sums = nullptr;   // [0] sum |xbp|^2, [1] sum |x*|^2, [2] loss
  int* tc_err = nullptr;    // set by a tcgen05 convolution whose bounded wait ran out
  float* rms = nullptr;
  float2* x0tmp = nullptr;  // prediction during training
  cudaStream_t st = nullptr;
  std::vector<void*> allocs;
  long long launches = 0;
  ~rihvr_unet() {
    for (void* p : allocs) cudaFree(p);
  }
};

namespace {

template <typename T>
int ualloc(rihvr_unet* u, T** p, size_t count) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess)
    return unet_fail(RIHVR_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  u->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return RIHVR_OK;
}

int conv_fwd(rihvr_unet* u, int li, const float* X, float* Y) {
  const Conv& L = u->layers[li];
  const Vol v = u->lv[L.level];
  UCK(conv3(X, L.cin, u->wb + u->wb_off[li], L.cout, 0, L.cout, u->w + L.b_off, Y, v, 1, 0, u->tc_err, u->st));
  ++u->launches;
  return RIHVR_OK;
}

// dY: gradient at the layer's output, taken through its ReLU in place; adds
// the weight and bias gradients; dX (may be null) = gradient at its input
int conv_back(rihvr_unet* u, int li, const float* X, float* dY, float* dX) {
  const Conv& L = u->layers[li];
  const Vol v = u->lv[L.level];
  const long long n = v.n();
  k_relu_back<<<blocks_for(n * L.cout), 256, 0, u->st>>>(dY, u->act[li], n * L.cout);
  dim3 grid((unsigned)((n + kWgVox - 1) / kWgVox), 27, L.cin / 16);
  k_conv3_wgrad<<<grid, 128, 0, u->st>>>(X, L.cin, dY, L.cout, u->gw + L.w_off, v);
  k_bias_grad<<<(unsigned)std::min<long long>(1024, (n + 7) / 8), 256, 0, u->st>>>(dY, L.cout, n, u->gw + L.b_off);
  u->launches += 3;
  // the data gradient: output channels of the transposed weights in windows of 64
  for (int co0 = 0; dX && co0 < L.cin; co0 += 64) {
    UCK(conv3(dY, L.cout, u->wt + u->wb_off[li], L.cin, co0, std::min(64, L.cin - co0), nullptr, dX, v, 0, 1,
              u->tc_err, u->st));
    ++u->launches;
  }
  UCK(cudaGetLastError());
  return RIHVR_OK;
}

int refresh_bf16(rihvr_unet* u) {
  for (int i = 0; i < kNumConv; ++i) {
    const Conv& L = u->layers[i];
    k_weights_bf16<<<blocks_for((long long)L.cout * 27 * L.cin), 256, 0, u->st>>>(
        u->w + L.w_off, L.cout, L.cin, u->wb + u->wb_off[i], u->wt + u->wb_off[i]);
    UCK(tc_weights(u->w + L.w_off, L.cout, L.cin, u->wtc + u->wtc_off[i], u->st));
    u->launches += 2;
  }
  UCK(cudaGetLastError());
  return RIHVR_OK;
}

// forward pass to the gain and x0 = g alpha scale xbp; with xs the sums for
// the loss are formed too
int forward(rihvr_unet* u, const float2* xbp, const float2* xs, float2* x0, float scale = 1.f) {
  const long long n0 = u->lv[0].n();
  UCK(cudaMemsetAsync(u->sums, 0, 3 * sizeof(double), u->st));
  k_sumsq<<<blocks_for(n0), 256, 0, u->st>>>(xbp, xs, n0, u->sums);
  k_rms<<<1, 1, 0, u->st>>>(u->sums, n0, u->rms);
  k_input<<<blocks_for(n0), 256, 0, u->st>>>(xbp, n0, u->rms, u->in0);
  u->launches += 3;
  int rc;
  if ((rc = conv_fwd(u, 0, u->in0, u->act[0])) || (rc = conv_fwd(u, 1, u->act[0], u->act[1]))) return rc;
  k_pool<<<blocks_for(u->lv[1].n() * 16), 256, 0, u->st>>>(u->act[1], u->p1, u->lv[1], 16);
  if ((rc = conv_fwd(u, 2, u->p1, u->act[2])) || (rc = conv_fwd(u, 3, u->act[2], u->act[3]))) return rc;
  k_pool<<<blocks_for(u->lv[2].n() * 32), 256, 0, u->st>>>(u->act[3], u->p2, u->lv[2], 32);
  if ((rc = conv_fwd(u, 4, u->p2, u->act[4])) || (rc = conv_fwd(u, 5, u->act[4], u->act[5]))) return rc;
  k_up_concat<<<blocks_for(u->lv[1].n() * 96), 256, 0, u->st>>>(u->act[5], 64, u->act[3], 32, u->c2, u->lv[1]);
  if ((rc = conv_fwd(u, 6, u->c2, u->act[6])) || (rc = conv_fwd(u, 7, u->act[6], u->act[7]))) return rc;
  k_up_concat<<<blocks_for(n0 * 48), 256, 0, u->st>>>(u->act[7], 32, u->act[1], 16, u->c1, u->lv[0]);
  if ((rc = conv_fwd(u, 8, u->c1, u->act[8])) || (rc = conv_fwd(u, 9, u->act[8], u->act[9]))) return rc;
  k_head<<<blocks_for(n0), 256, 0, u->st>>>(u->act[9], u->w + u->head_off, xbp, n0, scale, u->gbuf, x0);
  u->launches += 5;
  UCK(cudaGetLastError());
  return RIHVR_OK;
}

// gradients of the loss into gw (zeroed here), loss into sums[2]
int backward(rihvr_unet* u, const float2* xbp, const float2* xs) {
  const long long n0 = u->lv[0].n(), n1 = u->lv[1].n();
  UCK(cudaMemsetAsync(u->gw, 0, sizeof(float) * u->nparam, u->st));
  k_head_back<<<blocks_for(n0), 256, 0, u->st>>>(u->act[9], u->w + u->head_off, xbp, xs, u->gbuf, n0, u->sums,
                                                u->A0a, u->gw + u->head_off, u->sums + 2);
  ++u->launches;
  int rc;
  if ((rc = conv_back(u, 9, u->act[8], u->A0a, u->A0b))) return rc;  // dec1b
  if ((rc = conv_back(u, 8, u->c1, u->A0b, u->C0))) return rc;        // dec1a: 48 ch
  k_up_concat_back<<<blocks_for(n0 * 16), 256, 0, u->st>>>(u->C0, 32, 16, u->B1a, u->S0, u->lv[1]);
  if ((rc = conv_back(u, 7, u->act[6], u->B1a, u->B1b))) return rc;  // dec2b
  if ((rc = conv_back(u, 6, u->c2, u->B1b, u->C1))) return rc;        // dec2a: 96 ch
  k_up_concat_back<<<blocks_for(n1 * 32), 256, 0, u->st>>>(u->C1, 64, 32, u->D2a, u->S1, u->lv[2]);
  if ((rc = conv_back(u, 5, u->act[4], u->D2a, u->D2b))) return rc;  // bottom b
  if ((rc = conv_back(u, 4, u->p2, u->D2b, u->P2))) return rc;        // bottom a
  k_pool_back<<<blocks_for(n1 * 32), 256, 0, u->st>>>(u->P2, u->S1, u->B1a, u->lv[1], 32);
  if ((rc = conv_back(u, 3, u->act[2], u->B1a, u->B1b))) return rc;  // enc2b
  if ((rc = conv_back(u, 2, u->p1, u->B1b, u->P1))) return rc;        // enc2a
  k_pool_back<<<blocks_for(n0 * 16), 256, 0, u->st>>>(u->P1, u->S0, u->A0a, u->lv[0], 16);
  if ((rc = conv_back(u, 1, u->act[0], u->A0a, u->A0b))) return rc;  // enc1b
  if ((rc = conv_back(u, 0, u->in0, u->A0b, nullptr))) return rc;     // enc1a
  u->launches += 4;
  UCK(cudaGetLastError());
  return RIHVR_OK;
}

// The BF16-activation path applies where every level's width is a multiple
// of 128 (tcgen05) and the tensor-map encoder is there; RIHVR_UNET_MMA=sync
// keeps the FP32 path everywhere.
bool bf16_path(const rihvr_unet* u) {
  if (!use_tcgen05() || u->bf_failed) return false;
  for (int i = 0; i < kNumConv; ++i) {
    const Conv& L = u->layers[i];
    const Vol v = u->lv[L.level];
    if (!conv3_tc_bf16_supported(v.D, v.H, v.W, L.cin, L.cout)) return false;
  }
  return true;
}

// activations and tensor maps of the BF16 path, on first use
int bf16_prepare(rihvr_unet* u) {
  if (u->bf_ready) return RIHVR_OK;
  const long long n0 = u->lv[0].n(), n1 = u->lv[1].n(), n2 = u->lv[2].n();
  int rc = RIHVR_OK;
  auto A = [&](__nv_bfloat16** p, size_t n) {
    if (rc == RIHVR_OK) rc = ualloc(u, p, n);
  };
  A(&u->b_in0, n0 * 16);
  A(&u->b_a0, n0 * 16);
  A(&u->b_a1, n0 * 16);
  A(&u->b_c1, n0 * 48);
  A(&u->b_p1, n1 * 16);
  A(&u->b_a2, n1 * 32);
  A(&u->b_a3, n1 * 32);
  A(&u->b_c2, n1 * 96);
  A(&u->b_a7, n1 * 32);
  A(&u->b_p2, n2 * 32);
  A(&u->b_a4, n2 * 64);
  A(&u->b_a5, n2 * 64);
  if (rc != RIHVR_OK) return rc;
  // layer inputs: enc1 in0, a0; enc2 p1, a2; bottom p2, a4; dec2 c2, a6 (= a2);
  // dec1 c1, a8 (= a0)
  const __nv_bfloat16* in[kNumConv] = {u->b_in0, u->b_a0, u->b_p1, u->b_a2, u->b_p2,
                                       u->b_a4, u->b_c2, u->b_a2, u->b_c1, u->b_a0};
  for (int i = 0; i < kNumConv; ++i) {
    const Conv& L = u->layers[i];
    const Vol v = u->lv[L.level];
    if (!tc_map_encode(&u->maps[i], in[i], L.cin, v.D, v.H, v.W)) {
      u->bf_failed = true;
      return RIHVR_OK;
    }
    u->zwalk[i] = use_zwalk() && tcz_supported(v.W, L.cin, L.cout) &&
                  tc_zmap_encode(&u->zmaps[i], in[i], L.cin, v.D, v.H, v.W, tcz_rows(L.cin) + 2);
  }
  u->bf_ready = true;
  return RIHVR_OK;
}

int conv_bf16(rihvr_unet* u, int li, __nv_bfloat16* Y, const TcHead* head = nullptr) {
  const Conv& L = u->layers[li];
  const Vol v = u->lv[L.level];
  if (u->zwalk[li])
    UCK(conv3_tcz(u->zmaps[li], L.cin, u->wtc + u->wtc_off[li], u->w + L.b_off, L.cout, Y, v.D, v.H, v.W, head,
                  u->tc_err, u->st));
  else
    UCK(conv3_tc_bf16(u->maps[li], L.cin, u->wtc + u->wtc_off[li], u->w + L.b_off, L.cout, Y, v.D, v.H, v.W, head,
                      u->tc_err, u->st));
  ++u->launches;
  return RIHVR_OK;
}

// x0 = g alpha scale xbp with BF16 activations between the layers: the
// convolution operands are the BF16 values the FP32 path rounds them to, so
// the two paths differ only where the 2x2x2 pools average (BF16 inputs here,
// FP32 there); the head works on the last layer's FP32 values
int forward_bf16(rihvr_unet* u, const float2* xbp, float2* x0, float scale) {
  int rc = bf16_prepare(u);
  if (rc != RIHVR_OK) return rc;
  const long long n0 = u->lv[0].n(), n1 = u->lv[1].n(), n2 = u->lv[2].n();
  UCK(cudaMemsetAsync(u->sums, 0, 3 * sizeof(double), u->st));
  k_sumsq<<<blocks_for(n0), 256, 0, u->st>>>(xbp, nullptr, n0, u->sums);
  k_rms<<<1, 1, 0, u->st>>>(u->sums, n0, u->rms);
  k_input_bf16<<<blocks_for(n0), 256, 0, u->st>>>(xbp, n0, u->rms, u->b_in0);
  u->launches += 3;
  if ((rc = conv_bf16(u, 0, u->b_a0)) || (rc = conv_bf16(u, 1, u->b_a1))) return rc;
  k_pool_bf16<<<blocks_for(n1 * 2), 256, 0, u->st>>>(u->b_a1, u->b_p1, u->lv[1], 16);
  if ((rc = conv_bf16(u, 2, u->b_a2)) || (rc = conv_bf16(u, 3, u->b_a3))) return rc;
  k_pool_bf16<<<blocks_for(n2 * 4), 256, 0, u->st>>>(u->b_a3, u->b_p2, u->lv[2], 32);
  if ((rc = conv_bf16(u, 4, u->b_a4)) || (rc = conv_bf16(u, 5, u->b_a5))) return rc;
  k_up_concat_bf16<<<blocks_for(n1 * 12), 256, 0, u->st>>>(u->b_a5, 64, u->b_a3, 32, u->b_c2, u->lv[1]);
  if ((rc = conv_bf16(u, 6, u->b_a2)) || (rc = conv_bf16(u, 7, u->b_a7))) return rc;
  k_up_concat_bf16<<<blocks_for(n0 * 6), 256, 0, u->st>>>(u->b_a7, 32, u->b_a1, 16, u->b_c1, u->lv[0]);
  if ((rc = conv_bf16(u, 8, u->b_a0))) return rc;
  TcHead hd;
  hd.w = u->w + u->head_off;
  hd.xbp = xbp;
  hd.scale = scale;
  hd.x0 = x0;
  if ((rc = conv_bf16(u, 9, nullptr, &hd))) return rc;
  u->launches += 4;
  UCK(cudaGetLastError());
  return RIHVR_OK;
}

// prediction: the BF16 path where it applies, else the FP32 forward pass
int predict(rihvr_unet* u, const float2* xbp, float2* x0, float scale) {
  if (bf16_path(u)) {
    const int rc = bf16_prepare(u);
    if (rc != RIHVR_OK) return rc;
    if (!u->bf_failed) return forward_bf16(u, xbp, x0, scale);
  }
  return forward(u, xbp, nullptr, x0, scale);
}

int check_net(const rihvr_unet* u) {
  if (!u) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL network");
  return RIHVR_OK;
}

// after a synchronisation: did a tcgen05 convolution give up waiting?  (the
// flag is cleared for the next call)
int check_tc(rihvr_unet* u) {
  int e = 0;
  UCK(cudaMemcpy(&e, u->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    UCK(cudaMemset(u->tc_err, 0, sizeof(int)));
    return unet_fail(RIHVR_ERR_CUDA, "a tensor-core convolution timed out waiting for its MMAs");
  }
  return RIHVR_OK;
}

}  // namespace

namespace rihvr {
// x0 = net(xbp) with the output scaled by `scale` (the input is normalised, so
// the gain does not depend on it), on stream st
int unet_predict_on(rihvr_unet* u, const float2* xbp, float scale, float2* x0, cudaStream_t st) {
  if (!u || !xbp || !x0) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  u->st = st;
  const int rc = predict(u, xbp, x0, scale);
  if (rc != RIHVR_OK) return rc;
  UCK(cudaStreamSynchronize(st));
  return check_tc(u);
}
void unet_dims(const rihvr_unet* u, int* D, int* H, int* W) {
  *D = u->lv[0].D;
  *H = u->lv[0].H;
  *W = u->lv[0].W;
}
}  // namespace rihvr

extern "C" {

int rihvr_unet_create(int depth, int height, int width, unsigned long long seed, rihvr_unet** out) {
  if (!out) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL output");
  *out = nullptr;
  if (depth < 4 || height < 4 || width < 4 || depth % 4 || height % 4 || width % 4)
    return unet_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "depth, height and width must be multiples of 4 (two poolings)");
  rihvr_unet* u = new (std::nothrow) rihvr_unet();
  if (!u) return unet_fail(RIHVR_ERR_OUT_OF_MEMORY, "host allocation failed");
  auto bail = [&](int rc) {
    delete u;
    return rc;
  };
  u->lv[0] = Vol{depth, height, width};
  u->lv[1] = Vol{depth / 2, height / 2, width / 2};
  u->lv[2] = Vol{depth / 4, height / 4, width / 4};
  size_t off = 0, boff = 0;
  for (int i = 0; i < kNumConv; ++i) {
    u->layers[i] = kLayers[i];
    u->layers[i].w_off = off;
    off += (size_t)kLayers[i].cout * 27 * kLayers[i].cin;
    u->layers[i].b_off = off;
    off += (size_t)kLayers[i].cout;
    u->wb_off[i] = boff;
    u->wtc_off[i] = boff;  // same sizes: Cout x 27 x Cin
    boff += (size_t)kLayers[i].cout * 27 * kLayers[i].cin;
  }
  u->head_off = off;
  u->nparam = off + 18;
  const long long n0 = u->lv[0].n(), n1 = u->lv[1].n(), n2 = u->lv[2].n();
  int rc = RIHVR_OK;
  auto A = [&](float** p, size_t n) {
    if (rc == RIHVR_OK) rc = ualloc(u, p, n);
  };
  A(&u->w, u->nparam);
  A(&u->gw, u->nparam);
  A(&u->m, u->nparam);
  A(&u->s, u->nparam);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->wb, boff);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->wt, boff);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->wtc, boff);
  for (int i = 0; i < kNumConv; ++i) A(&u->act[i], (size_t)u->lv[kLayers[i].level].n() * kLayers[i].cout);
  A(&u->in0, n0 * 16);
  A(&u->p1, n1 * 16);
  A(&u->p2, n2 * 32);
  A(&u->c2, n1 * 96);
  A(&u->c1, n0 * 48);
  A(&u->gbuf, n0);
  A(&u->A0a, n0 * 16);
  A(&u->A0b, n0 * 16);
  A(&u->S0, n0 * 16);
  A(&u->C0, n0 * 48);
  A(&u->B1a, n1 * 32);
  A(&u->B1b, n1 * 32);
  A(&u->S1, n1 * 32);
  A(&u->C1, n1 * 96);
  A(&u->P1, n1 * 16);
  A(&u->D2a, n2 * 64);
  A(&u->D2b, n2 * 64);
  A(&u->P2, n2 * 32);
  A(&u->rms, 1);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->sums, 3);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->tc_err, 1);
  if (rc == RIHVR_OK) rc = ualloc(u, &u->x0tmp, (size_t)n0);
  if (rc != RIHVR_OK) return bail(rc);
  // He-normal weights (fan-in 27 x real input channels; only channel 0 of the
  // first layer's padded input is used), zero biases, head small, alpha 1
  std::vector<float> h(u->nparam, 0.f);
  std::mt19937_64 rng(seed);
  for (int i = 0; i < kNumConv; ++i) {
    const Conv& L = u->layers[i];
    const int cin_real = i == 0 ? 1 : L.cin;
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (27.f * cin_real)));
    for (int co = 0; co < L.cout; ++co)
      for (int k = 0; k < 27; ++k)
        for (int ci = 0; ci < cin_real; ++ci) h[L.w_off + ((size_t)co * 27 + k) * L.cin + ci] = nd(rng);
  }
  std::normal_distribution<float> nh(0.f, 0.1f);
  for (int c = 0; c < 16; ++c) h[u->head_off + c] = nh(rng);
  h[u->head_off + 16] = 0.f;
  h[u->head_off + 17] = 1.f;
  if (cudaMemcpy(u->w, h.data(), sizeof(float) * u->nparam, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(u->m, 0, sizeof(float) * u->nparam) != cudaSuccess ||
      cudaMemset(u->s, 0, sizeof(float) * u->nparam) != cudaSuccess ||
      cudaMemset(u->tc_err, 0, sizeof(int)) != cudaSuccess)
    return bail(unet_fail(RIHVR_ERR_CUDA, "initial copies failed"));
  u->st = nullptr;
  if ((rc = refresh_bf16(u)) != RIHVR_OK) return bail(rc);
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) return bail(unet_fail(RIHVR_ERR_CUDA, "initialisation failed"));
  *out = u;
  return RIHVR_OK;
}

void rihvr_unet_destroy(rihvr_unet* u) {
  if (!u) return;
  cudaDeviceSynchronize();
  delete u;
}

long long rihvr_unet_param_count(const rihvr_unet* u) { return u ? (long long)u->nparam : 0; }

int rihvr_unet_get_params(rihvr_unet* u, float* out) {
  if (check_net(u) || !out) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  UCK(cudaMemcpy(out, u->w, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost));
  return RIHVR_OK;
}

int rihvr_unet_set_params(rihvr_unet* u, const float* in) {
  if (check_net(u) || !in) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  UCK(cudaMemcpy(u->w, in, sizeof(float) * u->nparam, cudaMemcpyHostToDevice));
  UCK(cudaMemset(u->m, 0, sizeof(float) * u->nparam));
  UCK(cudaMemset(u->s, 0, sizeof(float) * u->nparam));
  u->step = 0;
  u->st = nullptr;
  const int rc = refresh_bf16(u);
  if (rc != RIHVR_OK) return rc;
  UCK(cudaStreamSynchronize(nullptr));
  return RIHVR_OK;
}

int rihvr_unet_predict(rihvr_unet* u, const float* xbp, float* x0) {
  if (check_net(u) || !xbp || !x0) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  u->st = nullptr;
  const int rc = predict(u, reinterpret_cast<const float2*>(xbp), reinterpret_cast<float2*>(x0), 1.f);
  if (rc != RIHVR_OK) return rc;
  UCK(cudaStreamSynchronize(nullptr));
  return check_tc(u);
}

int rihvr_unet_gradients(rihvr_unet* u, const float* xbp, const float* xstar, float* grad_out, double* loss) {
  if (check_net(u) || !xbp || !xstar) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  u->st = nullptr;
  const float2* a = reinterpret_cast<const float2*>(xbp);
  const float2* b = reinterpret_cast<const float2*>(xstar);
  int rc = forward(u, a, b, u->x0tmp);
  if (rc == RIHVR_OK) rc = backward(u, a, b);
  if (rc != RIHVR_OK) return rc;
  if (grad_out) UCK(cudaMemcpy(grad_out, u->gw, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost));
  double h[3];
  UCK(cudaMemcpy(h, u->sums, sizeof(h), cudaMemcpyDeviceToHost));
  if (loss) *loss = h[2];
  return check_tc(u);
}

int rihvr_unet_train_step(rihvr_unet* u, const float* xbp, const float* xstar, float lr, double* loss) {
  if (!(lr > 0)) return unet_fail(RIHVR_ERR_INVALID_ARGUMENT, "learning rate must be positive");
  int rc = rihvr_unet_gradients(u, xbp, xstar, nullptr, loss);
  if (rc != RIHVR_OK) return rc;
  const float b1 = 0.9f, b2 = 0.999f;
  u->step += 1;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)u->step)), c2 = 1.f / (1.f - std::pow(b2, (float)u->step));
  k_adam<<<blocks_for((long long)u->nparam), 256, 0, u->st>>>(u->w, u->m, u->s, u->gw, (long long)u->nparam, lr, b1,
                                                              b2, c1, c2, 1e-8f);
  ++u->launches;
  if ((rc = refresh_bf16(u)) != RIHVR_OK) return rc;
  UCK(cudaStreamSynchronize(nullptr));
  return RIHVR_OK;
}

long long rihvr_unet_launch_count(const rihvr_unet* u) { return u ? u->launches : 0; }

int rihvr_unet_activation_bits(rihvr_unet* u) {
  if (check_net(u)) return 0;
  if (bf16_path(u) && bf16_prepare(u) == RIHVR_OK && !u->bf_failed) return 16;
  return 32;
}

}  // extern "C"
