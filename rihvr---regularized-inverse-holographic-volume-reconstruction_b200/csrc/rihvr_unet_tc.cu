// 3x3x3 convolution of the warm-start U-Net on the 5th-generation tensor
// cores (tcgen05.mma, kind::f16: BF16 operands from shared memory, FP32
// accumulators in tensor memory), for layers whose width is a multiple of 128.
//
// Implicit GEMM: D[voxel][co] = sum over 27 taps and the input channels of
// A[voxel + offset(tap)][ci] B[tap][co][ci].  One MMA multiplies a 128-voxel
// x-row (M = 128) by Cn output channels (N = Cn) over 16 input channels
// (K = 16).  A block owns kTcYT consecutive x-rows of one z-plane (kTcYT
// accumulators of Cn FP32 columns in tensor memory).  Per 16-channel slice it
// stages, in BF16:
//   A: the halo of its rows, 3 (z) x (kTcYT + 2) (y) x 130 (x) voxels, as two
//      planes (channels 0-7 and 8-15) of 16 bytes a voxel;
//   B: every tap's Cn x 16 weight tile, as two planes of 16 bytes a row.
// In this K-major, unswizzled layout a "core matrix" (8 rows x 16 bytes) is 8
// consecutive voxels (or output channels) of one plane, so a tap's shifted
// window of an x-row is directly an operand: start at the shifted voxel, core
// matrices 128 bytes apart along M (SBO), the second channel plane LBO bytes
// away.  No im2col copy is made.  One thread issues the 27 x kTcYT MMAs of a
// slice and commits them to an mbarrier; every wait on it is bounded.  The
// epilogue reads the accumulators with tcgen05.ld (warp w holds voxels
// 32w..32w+31 of each row), adds the bias, applies the ReLU and stores FP32
// channels-last.  Output values match the mma.sync kernel up to the order of
// the FP32 accumulation.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "rihvr_unet_tc.cuh"

namespace rihvr {
namespace unet {

namespace {

constexpr int kTcX = 128;                           // voxels of an x-row: the MMA's M
constexpr int kTcYT = 4;                            // x-rows a block
constexpr int kTcThreads = 128;                     // 4 warps: one per 32 TMEM lanes
constexpr int kTcHX = kTcX + 2, kTcHY = kTcYT + 2, kTcHZ = 3;
constexpr int kTcHalo = kTcHZ * kTcHY * kTcHX;      // staged voxels
constexpr unsigned kTcMaxSpins = 1u << 26;          // bounded mbarrier wait

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

// shared-memory matrix descriptor: K-major, no swizzle, Blackwell version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((start >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcX >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for phase `parity` of the barrier with a bound; false when it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned i = 0; i < kTcMaxSpins; ++i)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tap_off(int k, int* dz, int* dy, int* dx) {
  *dz = k / 9 - 1;
  *dy = (k / 3) % 3 - 1;
  *dx = k % 3 - 1;
}

template <int CN>
constexpr uint32_t tmem_cols() {
  constexpr int need = kTcYT * CN;
  return need <= 32 ? 32u : need <= 64 ? 64u : need <= 128 ? 128u : need <= 256 ? 256u : 512u;
}

template <int CN>
constexpr size_t tc_smem() {
  return (size_t)2 * kTcHalo * 16 + (size_t)2 * 27 * CN * 16 + 16;
}

template <int CN>
__global__ void __launch_bounds__(kTcThreads) k_conv3_tc(const float* __restrict__ X, int Cin,
                                                         const __nv_bfloat16* __restrict__ Wt, int Cout, int co0,
                                                         const float* __restrict__ bias, float* __restrict__ Y,
                                                         int D, int H, int W, int relu, int mirror,
                                                         int* __restrict__ err) {
  static_assert(CN % 16 == 0 && CN >= 16 && CN <= 64, "N of the MMA");
  constexpr uint32_t NCOLS = tmem_cols<CN>();
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* A0 = tsm;                             // [kTcHalo] x 16 B, channels 0-7
  unsigned char* A1 = A0 + kTcHalo * 16;               // channels 8-15
  unsigned char* B0 = A1 + kTcHalo * 16;               // [27 * CN] x 16 B
  unsigned char* B1 = B0 + 27 * CN * 16;
  uint64_t* bar = reinterpret_cast<uint64_t*>(B1 + 27 * CN * 16);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nbx = W / kTcX, nby = (H + kTcYT - 1) / kTcYT;
  const int bx = blockIdx.x % nbx, by = (blockIdx.x / nbx) % nby, z0 = blockIdx.x / (nbx * nby);
  const int x0 = bx * kTcX, y0 = by * kTcYT;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = *tslot;
  const uint32_t bar_a = saddr(bar);
  const uint32_t idesc = instr_desc(CN);
  const uint32_t a_lbo = kTcHalo * 16, b_lbo = 27 * CN * 16;
  uint32_t parity = 0;
  bool ok = true;

  const int nslice = Cin / 16;
  for (int s = 0; s < nslice && ok; ++s) {
    if (s > 0) {  // the previous slice's MMAs have read the staged tiles
      ok = mbar_wait(bar_a, parity);
      parity ^= 1u;
      if (!ok) break;
    }
    // A: halo voxels of slice s, zero outside the volume
    for (int h = tid; h < kTcHalo; h += kTcThreads) {
      const int hx = h % kTcHX, hy = (h / kTcHX) % kTcHY, hz = h / (kTcHX * kTcHY);
      const int xx = x0 + hx - 1, yy = y0 + hy - 1, zz = z0 + hz - 1;
      uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
      if (xx >= 0 && xx < W && yy >= 0 && yy < H && zz >= 0 && zz < D) {
        const float4* src = reinterpret_cast<const float4*>(X + (((long long)zz * H + yy) * W + xx) * Cin + s * 16);
        const float4 f0 = src[0], f1 = src[1], f2 = src[2], f3 = src[3];
        lo = make_uint4(pack2(f0.x, f0.y), pack2(f0.z, f0.w), pack2(f1.x, f1.y), pack2(f1.z, f1.w));
        hi = make_uint4(pack2(f2.x, f2.y), pack2(f2.z, f2.w), pack2(f3.x, f3.y), pack2(f3.z, f3.w));
      }
      *reinterpret_cast<uint4*>(A0 + h * 16) = lo;
      *reinterpret_cast<uint4*>(A1 + h * 16) = hi;
    }
    // B: row k * CN + co holds Wt[co0 + co][k][16 s .. 16 s + 15]
    for (int e = tid; e < 27 * CN * 2; e += kTcThreads) {
      const int row = e >> 1, half = e & 1;
      const int k = row / CN, co = row - k * CN;
      const uint4 w = *reinterpret_cast<const uint4*>(Wt + ((long long)(co0 + co) * 27 + k) * Cin + s * 16 + half * 8);
      *reinterpret_cast<uint4*>((half ? B1 : B0) + row * 16) = w;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor-core reads
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = saddr(A0), b0 = saddr(B0);
      for (int k = 0; k < 27; ++k) {
        int dz, dy, dx;
        tap_off(mirror ? 26 - k : k, &dz, &dy, &dx);
        const uint64_t bd = smem_desc(b0 + (uint32_t)(k * CN * 16), b_lbo, 128);
#pragma unroll
        for (int m = 0; m < kTcYT; ++m) {
          const int h = ((1 + dz) * kTcHY + (m + 1 + dy)) * kTcHX + (1 + dx);
          const uint64_t ad = smem_desc(a0 + (uint32_t)(h * 16), a_lbo, 128);
          mma_bf16_ss(tbase + (uint32_t)(m * CN), ad, bd, idesc, (s > 0 || k > 0) ? 1u : 0u);
        }
      }
      mma_commit(bar_a);
    }
  }
  if (ok) {
    ok = mbar_wait(bar_a, parity);
    parity ^= 1u;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int xx = x0 + warp * 32 + lane;
#pragma unroll 1
    for (int m = 0; m < kTcYT; ++m) {
      const int yy = y0 + m;
#pragma unroll
      for (int c16 = 0; c16 < CN / 16; ++c16) {
        float v[16];
        // every lane of the warp takes part in the load, also for rows past H
        tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * CN + c16 * 16), v);
        if (yy < H) {
          float* dst = Y + (((long long)z0 * H + yy) * W + xx) * Cout + co0 + c16 * 16;
#pragma unroll
          for (int j = 0; j < 16; j += 4) {
            float4 o;
            o.x = v[j] + (bias ? bias[co0 + c16 * 16 + j] : 0.f);
            o.y = v[j + 1] + (bias ? bias[co0 + c16 * 16 + j + 1] : 0.f);
            o.z = v[j + 2] + (bias ? bias[co0 + c16 * 16 + j + 2] : 0.f);
            o.w = v[j + 3] + (bias ? bias[co0 + c16 * 16 + j + 3] : 0.f);
            if (relu) {
              o.x = fmaxf(o.x, 0.f);
              o.y = fmaxf(o.y, 0.f);
              o.z = fmaxf(o.z, 0.f);
              o.w = fmaxf(o.w, 0.f);
            }
            *reinterpret_cast<float4*>(dst + j) = o;
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
    // give the committed MMAs a last bounded chance to finish before the
    // tensor memory they write is released
    mbar_wait(bar_a, parity);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(NCOLS) : "memory");
  }
}

template <int CN>
cudaError_t tc_launch(const float* X, int Cin, const __nv_bfloat16* Wt, int Cout, int co0, const float* bias,
                      float* Y, int D, int H, int W, int relu, int mirror, int* err, cudaStream_t st) {
  constexpr size_t smem = tc_smem<CN>();
  static bool opted = false;  // shared-memory opt-in, once per instantiation
  if (!opted) {
    const cudaError_t e = cudaFuncSetAttribute(k_conv3_tc<CN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  const unsigned blocks = (unsigned)((W / kTcX) * ((H + kTcYT - 1) / kTcYT) * D);
  k_conv3_tc<CN><<<blocks, kTcThreads, smem, st>>>(X, Cin, Wt, Cout, co0, bias, Y, D, H, W, relu, mirror, err);
  return cudaGetLastError();
}

}  // namespace

bool conv3_tc_supported(int W, int Cin, int Cn) {
  return W % kTcX == 0 && Cin % 16 == 0 && (Cn == 16 || Cn == 32 || Cn == 48 || Cn == 64);
}

cudaError_t conv3_tc(const float* X, int Cin, const __nv_bfloat16* Wt, int Cout, int co0, int Cn, const float* bias,
                     float* Y, int D, int H, int W, int relu, int mirror, int* err, cudaStream_t st) {
  if (!conv3_tc_supported(W, Cin, Cn)) return cudaErrorInvalidValue;
  switch (Cn) {
    case 16: return tc_launch<16>(X, Cin, Wt, Cout, co0, bias, Y, D, H, W, relu, mirror, err, st);
    case 32: return tc_launch<32>(X, Cin, Wt, Cout, co0, bias, Y, D, H, W, relu, mirror, err, st);
    case 48: return tc_launch<48>(X, Cin, Wt, Cout, co0, bias, Y, D, H, W, relu, mirror, err, st);
    default: return tc_launch<64>(X, Cin, Wt, Cout, co0, bias, Y, D, H, W, relu, mirror, err, st);
  }
}

}  // namespace unet
}  // namespace rihvr
