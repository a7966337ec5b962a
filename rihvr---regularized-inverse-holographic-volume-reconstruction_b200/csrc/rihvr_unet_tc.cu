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
#include <cuda.h>  // CUtensorMap and its enums; the encoder is resolved at run time
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

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


// The 27 x YT MMAs of one 16-channel slice, fully unrolled: ad[dz + 1] is the
// A descriptor of the slab (or halo plane) a tap reads at z offset dz, bd the
// descriptor of the slice's first tap; a tap's shifted window and weights
// are fixed offsets into those (descriptor start addresses count 16-byte units
// in their low 14 bits, and every offset stays inside the 228 KB of shared
// memory, so adding to the descriptor adds to the address).
template <int CN, int YT, int HY, bool MIRROR>
__device__ __forceinline__ void issue_slice(uint32_t tbase, const uint64_t (&ad)[3], uint64_t bd, uint32_t idesc,
                                            bool accumulate) {
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const int kk = MIRROR ? 26 - k : k;
    const int dz = kk / 9 - 1, dy = (kk / 3) % 3 - 1, dx = kk % 3 - 1;
    const uint64_t b = bd + (uint64_t)(k * CN);  // k * CN * 16 bytes
#pragma unroll
    for (int m = 0; m < YT; ++m) {
      const uint64_t a = ad[dz + 1] + (uint64_t)((m + 1 + dy) * kTcHX + (1 + dx));
      mma_bf16_ss(tbase + (uint32_t)(m * CN), a, b, idesc, (accumulate || k > 0) ? 1u : 0u);
    }
  }
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
      const uint64_t bd = smem_desc(b0, b_lbo, 128);
      const uint64_t a_lo = smem_desc(a0, a_lbo, 128);
      const uint64_t ad[3] = {a_lo, a_lo + (uint64_t)(kTcHY * kTcHX), a_lo + (uint64_t)(2 * kTcHY * kTcHX)};
      if (mirror) issue_slice<CN, kTcYT, kTcHY, true>(tbase, ad, bd, idesc, s > 0);
      else issue_slice<CN, kTcYT, kTcHY, false>(tbase, ad, bd, idesc, s > 0);
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

// ---------------------------------------------------------------------------
// Inference form with BF16 activations.  The block, tile and MMA sequence are
// those above; what changes is how the operands arrive and leave:
//   A: two TMA tensor loads per 16-channel slice (channels 0-7 and 8-15, box
//      8 channels x 130 x (kTcYT + 2) x 3 of the channels-last BF16 input),
//      which land in exactly the two-plane layout the descriptors read; the
//      halo outside the volume is the TMA's zero fill;
//   B: one bulk copy of the slice's weights, kept in global memory already in
//      the [plane][tap][co][8 channels] order;
//   both complete on one mbarrier (transaction bytes), issued and awaited by
//   the thread that issues the MMAs, so no other thread touches them;
//   output: bias and ReLU in FP32, rounded to BF16 and stored channels-last,
//   or, for the last layer (HEAD), the 1x1x1 head, sigmoid and
//   x0 = g alpha scale xbp computed from the FP32 values in the epilogue.
// Every wait is bounded; a wait that runs out sets *err.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
               "r"(bytes)
               : "memory");
}

// TMA load of a 4-D box (coordinates innermost first; the first, a channel
// index, is a multiple of 8, i.e. 16 bytes) into shared memory, completing
// on the mbarrier.  No multicast.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

constexpr uint32_t kTcBoxBytes = 8u * 2u * kTcHalo;  // one channel plane of the halo (the TMA box)
// planes start 1024 bytes apart, so that every TMA destination is aligned
constexpr uint32_t kTcPlaneBytes = (kTcBoxBytes + 1023u) / 1024u * 1024u;

template <int CN>
constexpr size_t tcb_smem() {
  return (size_t)2 * kTcPlaneBytes + (size_t)2 * 27 * CN * 16 + 32;
}

template <int CN, bool HEAD>
__global__ void __launch_bounds__(kTcThreads) k_conv3_tc_bf16(const __grid_constant__ CUtensorMap xmap, int Cin,
                                                              const __nv_bfloat16* __restrict__ Wp,
                                                              const float* __restrict__ bias,
                                                              __nv_bfloat16* __restrict__ Y, int D, int H, int W,
                                                              TcHead hd, int* __restrict__ err) {
  static_assert(CN % 16 == 0 && CN >= 16 && CN <= 64, "N of the MMA");
  static_assert(!HEAD || CN == 16, "the head takes 16 channels");
  constexpr uint32_t NCOLS = tmem_cols<CN>();
  constexpr uint32_t BBYTES = 2u * 27u * CN * 16u;
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* A0 = tsm;                   // channels 0-7 of the halo, 16 B a voxel
  unsigned char* A1 = A0 + kTcPlaneBytes;    // channels 8-15
  unsigned char* B0 = A1 + kTcPlaneBytes;    // [2][27 * CN] x 16 B
  uint64_t* bars = reinterpret_cast<uint64_t*>(B0 + BBYTES);  // [0] operands landed, [1] MMAs done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  int* s_state = reinterpret_cast<int*>(tslot + 1);  // [0] ok, [1] parity of the last commit
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
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bars)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bars + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = *tslot;
  const uint32_t bar_full = saddr(bars), bar_mma = saddr(bars + 1);

  if (tid == 0) {
    const uint32_t idesc = instr_desc(CN);
    const uint32_t a0 = saddr(A0), b0 = saddr(B0);
    const int nslice = Cin / 16;
    uint32_t pf = 0, pm = 0;
    bool ok = true;
    int committed = 0;  // commits not yet awaited
    for (int s = 0; s < nslice; ++s) {
      if (s > 0) {  // the previous slice's MMAs have read the operands
        ok = mbar_wait(bar_mma, pm);
        pm ^= 1u;
        committed = 0;
        if (!ok) break;
      }
      mbar_expect_tx(bar_full, 2u * kTcBoxBytes + BBYTES);
      tma_load_4d(a0, &xmap, 16 * s, x0 - 1, y0 - 1, z0 - 1, bar_full);
      tma_load_4d(a0 + kTcPlaneBytes, &xmap, 16 * s + 8, x0 - 1, y0 - 1, z0 - 1, bar_full);
      bulk_load(b0, Wp + (size_t)s * (BBYTES / 2), BBYTES, bar_full);
      ok = mbar_wait(bar_full, pf);
      pf ^= 1u;
      if (!ok) {
        mbar_wait(bar_full, pf ^ 1u);  // a last bounded chance for the copies in flight
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint64_t bd = smem_desc(b0, 27 * CN * 16, 128);
      const uint64_t a_lo = smem_desc(a0, kTcPlaneBytes, 128);
      const uint64_t ad[3] = {a_lo, a_lo + (uint64_t)(kTcHY * kTcHX), a_lo + (uint64_t)(2 * kTcHY * kTcHX)};
      issue_slice<CN, kTcYT, kTcHY, false>(tbase, ad, bd, idesc, s > 0);
      mma_commit(bar_mma);
      committed = 1;
    }
    if (!ok) {
      atomicExch(err, 1);
      if (committed) mbar_wait(bar_mma, pm);  // let committed MMAs finish before the memory is released
    }
    s_state[0] = ok ? 1 : 0;
    s_state[1] = (int)pm;
  }
  __syncthreads();
  bool ok = s_state[0] != 0;
  if (ok) {
    ok = mbar_wait(bar_mma, (uint32_t)s_state[1]);
    if (!ok) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int xx = x0 + warp * 32 + lane;
#pragma unroll 1
    for (int m = 0; m < kTcYT; ++m) {
      const int yy = y0 + m;
      const long long vox = ((long long)z0 * H + yy) * W + xx;
      float zsum = 0.f;
      if constexpr (HEAD) zsum = hd.w[16];
#pragma unroll
      for (int c16 = 0; c16 < CN / 16; ++c16) {
        float v[16];
        // every lane of the warp takes part in the load, also for rows past H
        tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * CN + c16 * 16), v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + bias[c16 * 16 + j], 0.f);
        if constexpr (HEAD) {
#pragma unroll
          for (int j = 0; j < 16; ++j) zsum += hd.w[j] * v[j];
        } else if (yy < H) {
          uint4 o0, o1;
          o0.x = pack2(v[0], v[1]);
          o0.y = pack2(v[2], v[3]);
          o0.z = pack2(v[4], v[5]);
          o0.w = pack2(v[6], v[7]);
          o1.x = pack2(v[8], v[9]);
          o1.y = pack2(v[10], v[11]);
          o1.z = pack2(v[12], v[13]);
          o1.w = pack2(v[14], v[15]);
          uint4* dst = reinterpret_cast<uint4*>(Y + vox * CN + c16 * 16);
          dst[0] = o0;
          dst[1] = o1;
        }
      }
      if constexpr (HEAD) {
        if (yy < H) {
          const float g = 1.f / (1.f + expf(-zsum));
          const float alpha = hd.w[17] * hd.scale;
          const float2 a = hd.xbp[vox];
          hd.x0[vox] = make_float2(g * alpha * a.x, g * alpha * a.y);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(NCOLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// z-walking form of the inference convolution, for layers with 16 input
// channels (the template also takes more slices, NS).  A block keeps one
// (x-tile of 128 voxels, y-tile of YT rows) column and walks a range of z.
// Shared memory holds a ring of 3 input slabs (one z-plane each: YT + 2 rows x
// 130 voxels, every slice in two 8-channel planes, the layout the descriptors
// read), so each input plane is loaded once per block instead of three times,
// and the weights of all slices, loaded once per block.  Per output plane z:
//   thread 0 waits for slab z+1, issues the 27 x YT x slices MMAs into the
//   tensor-memory accumulator and commits them; once they are done it reuses
//   slab z-1's slot for slab z+2 (one TMA box per slice and half, completing on
//   that slot's mbarrier) while all threads drain the accumulator (bias, ReLU,
//   BF16 store, or the head).  The TMA copy overlaps the epilogue, and a
//   second block on the SM (16 channels: 89 KB a block) fills the tensor pipe
//   while this one drains.
// Every wait is bounded; a wait that runs out sets *err, the block lets its
// copies and MMAs in flight finish (bounded) and leaves.
// ---------------------------------------------------------------------------
template <int YT, int NS>  // x-rows a block, 16-channel slices
struct TczShape {
  static constexpr int HY = YT + 2;
  static constexpr uint32_t BOX = 16u * kTcHX * HY;                 // one 8-channel plane of a slab
  static constexpr uint32_t PLANE = (BOX + 127u) / 128u * 128u;     // planes 128 bytes apart
  static constexpr uint32_t SLAB = 2u * NS * PLANE;
  static constexpr int R = 3;                                        // slabs in the ring
};

template <int CN, int YT, int NS>
constexpr size_t tcz_smem() {
  using S = TczShape<YT, NS>;
  return 1024 + (size_t)S::R * S::SLAB + (size_t)NS * 2 * 27 * CN * 16 + 64;
}

template <int CN, bool HEAD, int YT, int NS>
__global__ void __launch_bounds__(kTcThreads) k_conv3_tcz(const __grid_constant__ CUtensorMap zmap,
                                                          const __nv_bfloat16* __restrict__ Wp,
                                                          const float* __restrict__ bias,
                                                          __nv_bfloat16* __restrict__ Y, int D, int H, int W,
                                                          int zper, TcHead hd, int* __restrict__ err) {
  static_assert(CN % 16 == 0 && CN >= 16 && CN <= 64, "N of the MMA");
  static_assert(!HEAD || CN == 16, "the head takes 16 channels");
  using S = TczShape<YT, NS>;
  constexpr uint32_t NCOLS = YT * CN <= 32 ? 32u : YT * CN <= 64 ? 64u : YT * CN <= 128 ? 128u : 256u;
  constexpr uint32_t BBYTES = 2u * 27u * CN * 16u;  // one slice's weights
  extern __shared__ unsigned char tzraw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tzraw) + 1023) & ~uintptr_t(1023));
  unsigned char* slabs = base;                          // [R][NS][2 planes] of PLANE bytes
  unsigned char* B0 = slabs + S::R * S::SLAB;           // [NS][2][27 * CN] x 16 B
  uint64_t* bars = reinterpret_cast<uint64_t*>(B0 + NS * BBYTES);  // [0..2] slabs, [3] weights, [4] MMAs
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
  int* s_ok = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nbx = W / kTcX, nby = (H + YT - 1) / YT;
  const int bx = blockIdx.x % nbx, by = (blockIdx.x / nbx) % nby, zp = blockIdx.x / (nbx * nby);
  const int x0 = bx * kTcX, y0 = by * YT;
  const int zb = zp * zper, ze = min(D, zb + zper);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < 5; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tbase = *tslot;
  const uint32_t idesc = instr_desc(CN);
  const uint32_t s0 = saddr(slabs), b0 = saddr(B0);
  uint32_t phase[S::R] = {0u, 0u, 0u};  // thread 0: parity of each slot's next completion
  bool busy[S::R] = {false, false, false};  // a copy into the slot not yet awaited
  uint32_t pm = 0;                      // parity of the MMA barrier
  bool mma_busy = false, w_busy = false;
  bool ok = true;
  // slot of the slab of plane z: the ring starts with plane zb - 1 in slot 0
  auto slot_of = [&](int z) { return (uint32_t)((z - zb + 1) % S::R); };
  auto load_slab = [&](int z) {  // thread 0
    const uint32_t sl = slot_of(z);
    const uint32_t bar = saddr(bars + sl);
    busy[sl] = true;
    mbar_expect_tx(bar, 2u * NS * S::BOX);
#pragma unroll
    for (int sc = 0; sc < NS; ++sc)
#pragma unroll
      for (int p = 0; p < 2; ++p)
        tma_load_4d(s0 + sl * S::SLAB + (uint32_t)(sc * 2 + p) * S::PLANE, &zmap, 16 * sc + 8 * p, x0 - 1, y0 - 1,
                    z, bar);
  };
  if (tid == 0 && zb < ze) {
    mbar_expect_tx(saddr(bars + 3), NS * BBYTES);
    bulk_load(b0, Wp, NS * BBYTES, saddr(bars + 3));
    w_busy = true;
    for (int z = zb - 1; z <= zb + 1; ++z) load_slab(z);  // planes outside the volume read as zeros
    ok = mbar_wait(saddr(bars + 3), 0);
    w_busy = !ok;
    for (int z = zb - 1; z <= zb && ok; ++z) {
      ok = mbar_wait(saddr(bars + slot_of(z)), phase[slot_of(z)]);
      if (ok) {
        phase[slot_of(z)] ^= 1u;
        busy[slot_of(z)] = false;
      }
    }
  }
  for (int z = zb; z < ze; ++z) {
    if (tid == 0) {
      if (ok) {  // slab z+1, the last one this plane reads
        ok = mbar_wait(saddr(bars + slot_of(z + 1)), phase[slot_of(z + 1)]);
        if (ok) {
          phase[slot_of(z + 1)] ^= 1u;
          busy[slot_of(z + 1)] = false;
        }
      }
      if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int sc = 0; sc < NS; ++sc) {
          uint64_t ad[3];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            ad[d] = smem_desc(s0 + slot_of(z + d - 1) * S::SLAB + (uint32_t)(sc * 2) * S::PLANE, S::PLANE, 128);
          const uint64_t bd = smem_desc(b0 + (uint32_t)sc * BBYTES, 27 * CN * 16, 128);
          issue_slice<CN, YT, S::HY, false>(tbase, ad, bd, idesc, sc > 0);
        }
        mma_commit(saddr(bars + 4));
        mma_busy = true;
        ok = mbar_wait(saddr(bars + 4), pm);
        if (ok) {
          pm ^= 1u;
          mma_busy = false;
        }
        // slab z-1 is no longer read: its slot takes slab z+2 for the next plane
        if (ok && z + 1 < ze) load_slab(z + 2);
      }
      if (!ok) *s_ok = 0;
    }
    __syncthreads();
    if (!*s_ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int xx = x0 + warp * 32 + lane;
#pragma unroll 1
    for (int m = 0; m < YT; ++m) {
      const int yy = y0 + m;
      const long long vox = ((long long)z * H + yy) * W + xx;
      float zsum = 0.f;
      if constexpr (HEAD) zsum = hd.w[16];
#pragma unroll
      for (int c16 = 0; c16 < CN / 16; ++c16) {
        float v[16];
        tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * CN + c16 * 16), v);
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j] + bias[c16 * 16 + j], 0.f);
        if constexpr (HEAD) {
#pragma unroll
          for (int j = 0; j < 16; ++j) zsum += hd.w[j] * v[j];
        } else if (yy < H) {
          uint4 o0, o1;
          o0.x = pack2(v[0], v[1]);
          o0.y = pack2(v[2], v[3]);
          o0.z = pack2(v[4], v[5]);
          o0.w = pack2(v[6], v[7]);
          o1.x = pack2(v[8], v[9]);
          o1.y = pack2(v[10], v[11]);
          o1.z = pack2(v[12], v[13]);
          o1.w = pack2(v[14], v[15]);
          uint4* dst = reinterpret_cast<uint4*>(Y + vox * CN + c16 * 16);
          dst[0] = o0;
          dst[1] = o1;
        }
      }
      if constexpr (HEAD) {
        if (yy < H) {
          const float g = 1.f / (1.f + expf(-zsum));
          const float alpha = hd.w[17] * hd.scale;
          const float2 a = hd.xbp[vox];
          hd.x0[vox] = make_float2(g * alpha * a.x, g * alpha * a.y);
        }
      }
    }
    // every thread's accumulator reads come before the next plane's MMAs
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  if (tid == 0 && !ok) {
    atomicExch(err, 1);
    // a last bounded wait for the copies and MMAs still in flight before the
    // shared and tensor memory are released
    if (mma_busy) mbar_wait(saddr(bars + 4), pm);
    for (int i = 0; i < S::R; ++i)
      if (busy[i]) mbar_wait(saddr(bars + i), phase[i]);
    if (w_busy) mbar_wait(saddr(bars + 3), 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(NCOLS) : "memory");
  }
}

// cuTensorMapEncodeTiled, resolved once through the runtime
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

template <int CN, bool HEAD>
cudaError_t tcb_launch(const TcMap& m, int Cin, const __nv_bfloat16* Wp, const float* bias, __nv_bfloat16* Y, int D,
                       int H, int W, const TcHead& hd, int* err, cudaStream_t st) {
  constexpr size_t smem = tcb_smem<CN>();
  static bool opted = false;
  if (!opted) {
    const cudaError_t e = cudaFuncSetAttribute(k_conv3_tc_bf16<CN, HEAD>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  CUtensorMap map;
  static_assert(sizeof(map) == sizeof(m.bytes), "tensor map size");
  std::memcpy(&map, m.bytes, sizeof(map));
  const unsigned blocks = (unsigned)((W / kTcX) * ((H + kTcYT - 1) / kTcYT) * D);
  k_conv3_tc_bf16<CN, HEAD><<<blocks, kTcThreads, smem, st>>>(map, Cin, Wp, bias, Y, D, H, W, hd, err);
  return cudaGetLastError();
}

// Wp[s][p][k][co][8] = bf16(w[co][k][16 s + 8 p + j]) for one layer
__global__ void k_weights_tc(const float* __restrict__ w, int Cout, int Cin, __nv_bfloat16* __restrict__ wp) {
  const long long n = (long long)Cout * 27 * Cin;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin), k = (int)((i / Cin) % 27), co = (int)(i / (27LL * Cin));
    const int s = ci >> 4, p = (ci >> 3) & 1, j = ci & 7;
    wp[((((long long)s * 2 + p) * 27 + k) * Cout + co) * 8 + j] = __float2bfloat16_rn(w[i]);
  }
}

}  // namespace

bool tc_map_encode(TcMap* m, const __nv_bfloat16* X, int C, int D, int H, int W) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || !X || (reinterpret_cast<uintptr_t>(X) & 15) != 0 || C % 16 != 0) return false;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D};
  const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)kTcHX, (cuuint32_t)kTcHY, (cuuint32_t)kTcHZ};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(X), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  static_assert(sizeof(map) == sizeof(m->bytes), "tensor map size");
  std::memcpy(m->bytes, &map, sizeof(map));
  return true;
}

// x-rows a block of the z-walking form takes
int tcz_rows(int) { return 4; }

bool tc_zmap_encode(TcMap* m, const __nv_bfloat16* X, int C, int D, int H, int W, int rows) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || !X || (reinterpret_cast<uintptr_t>(X) & 15) != 0 || C % 16 != 0 || rows < 1 || rows > 256) return false;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D};
  const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)kTcHX, (cuuint32_t)rows, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(X), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  std::memcpy(m->bytes, &map, sizeof(map));
  return true;
}

// 16 input channels only: with three slices (48 channels) the ring and the
// weights fill the shared memory of one block an SM, and that layer measured
// slower walking z (a block's loads, MMAs and epilogue then have nothing to
// overlap with) than in the per-tile kernel.
bool tcz_supported(int W, int Cin, int Cout) {
  return W % kTcX == 0 && Cin == 16 && (Cout == 16 || Cout == 32) && encode_tiled() != nullptr;
}

namespace {
template <int CN, bool HEAD, int YT, int NS>
cudaError_t tcz_launch(const TcMap& m, const __nv_bfloat16* Wp, const float* bias, __nv_bfloat16* Y, int D, int H,
                       int W, const TcHead& hd, int* err, cudaStream_t st) {
  constexpr size_t smem = tcz_smem<CN, YT, NS>();
  static bool opted = false;
  if (!opted) {
    const cudaError_t e = cudaFuncSetAttribute(k_conv3_tcz<CN, HEAD, YT, NS>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    opted = true;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3_tcz<CN, HEAD, YT, NS>, kTcThreads, smem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  // z-ranges per (x, y) column: about four waves of blocks in all
  const long long xy = (long long)(W / kTcX) * ((H + YT - 1) / YT);
  const long long target = 4LL * sms * per_sm;
  const int zsplit = (int)std::max(1LL, std::min<long long>(D, (target + xy - 1) / xy));
  const int zper = (D + zsplit - 1) / zsplit;
  const long long blocks = xy * ((D + zper - 1) / zper);
  if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
  CUtensorMap map;
  std::memcpy(&map, m.bytes, sizeof(map));
  k_conv3_tcz<CN, HEAD, YT, NS><<<(unsigned)blocks, kTcThreads, smem, st>>>(map, Wp, bias, Y, D, H, W, zper, hd, err);
  return cudaGetLastError();
}
}  // namespace

cudaError_t conv3_tcz(const TcMap& zmap, int Cin, const __nv_bfloat16* Wp, const float* bias, int Cout,
                      __nv_bfloat16* Y, int D, int H, int W, const TcHead* head, int* err, cudaStream_t st) {
  if (!tcz_supported(W, Cin, Cout) || (head && Cout != 16)) return cudaErrorInvalidValue;
  const TcHead hd = head ? *head : TcHead{};
  if (head) return tcz_launch<16, true, 4, 1>(zmap, Wp, bias, Y, D, H, W, hd, err, st);
  return Cout == 16 ? tcz_launch<16, false, 4, 1>(zmap, Wp, bias, Y, D, H, W, hd, err, st)
                    : tcz_launch<32, false, 4, 1>(zmap, Wp, bias, Y, D, H, W, hd, err, st);
}

bool conv3_tc_bf16_supported(int D, int H, int W, int Cin, int Cout) {
  return W % kTcX == 0 && Cin % 16 == 0 && (Cout == 16 || Cout == 32 || Cout == 48 || Cout == 64) && D >= 1 &&
         H >= 1 && encode_tiled() != nullptr;
}

size_t tc_weights_elems(int Cout, int Cin) { return (size_t)Cout * 27 * Cin; }

cudaError_t tc_weights(const float* w, int Cout, int Cin, __nv_bfloat16* wp, cudaStream_t st) {
  const long long n = (long long)Cout * 27 * Cin;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 1184);
  k_weights_tc<<<blocks, 256, 0, st>>>(w, Cout, Cin, wp);
  return cudaGetLastError();
}

cudaError_t conv3_tc_bf16(const TcMap& xmap, int Cin, const __nv_bfloat16* Wp, const float* bias, int Cout,
                          __nv_bfloat16* Y, int D, int H, int W, const TcHead* head, int* err, cudaStream_t st) {
  if (!conv3_tc_bf16_supported(D, H, W, Cin, Cout)) return cudaErrorInvalidValue;
  const TcHead hd = head ? *head : TcHead{};
  if (head) {
    if (Cout != 16) return cudaErrorInvalidValue;
    return tcb_launch<16, true>(xmap, Cin, Wp, bias, Y, D, H, W, hd, err, st);
  }
  switch (Cout) {
    case 16: return tcb_launch<16, false>(xmap, Cin, Wp, bias, Y, D, H, W, hd, err, st);
    case 32: return tcb_launch<32, false>(xmap, Cin, Wp, bias, Y, D, H, W, hd, err, st);
    case 48: return tcb_launch<48, false>(xmap, Cin, Wp, bias, Y, D, H, W, hd, err, st);
    default: return tcb_launch<64, false>(xmap, Cin, Wp, bias, Y, D, H, W, hd, err, st);
  }
}

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
