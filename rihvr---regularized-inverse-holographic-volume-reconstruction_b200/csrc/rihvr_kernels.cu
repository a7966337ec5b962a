// sm_100a kernels of the reconstruction hot path.
//
// Operator structure (RIHVR src/core/sparse_compressive_holo.cu:1935-2077 forward,
// src/core/sparse_gradient.cu:47-165 adjoint), restated by linearity:
//   forward  d   = Re( F^-1 sum_z H'_z F(x_z) ),  H'_z = exp(i z c(f))
//   adjoint  g_z = F^-1( conj(H'_z) F(r) )
// with c(f) = 2 pi / lambda (sqrt(1 - (lambda f)^2) - 1).  The per-plane carrier
// factor exp(-+ i 2 pi z / lambda) that the reference applies separately is folded
// into H'_z.  The 2-D DFT of a plane is a row pass plus a column pass; the column
// passes carry the transfer-function multiply (regenerated from an FP64 table of
// c/(2 pi) per frequency, phase reduced mod 1 turn in FP64) and, for the forward
// operator, the sum over z, so the Nz transformed planes never go back to memory.
#include <cuda.h>  // CUtensorMap and its enums; the encoder is resolved at run time

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "rihvr_device.cuh"
#include "rihvr_kernels.cuh"

namespace rihvr {

// ---------------------------------------------------------------------------
// line configurations: N = N1 * N2, N1 threads per line, N2 elements each.
// After the exchange a thread holds M stage-B rows of N1 elements (VS values).
// Where N1 divides N2 every thread holds N2 / N1 rows; otherwise (side 640 =
// 20 x 32) the N2 rows are dealt round-robin and a thread's last row exists
// only when t + N1 (M - 1) < N2 (EXACT false): the missing rows are computed
// on zeros and never stored.
// ---------------------------------------------------------------------------
template <int N>
struct LineCfg;
#define RIHVR_LINE(NN, NN1)                                                              \
  template <>                                                                            \
  struct LineCfg<NN> {                                                                   \
    static constexpr int N = NN, N1 = NN1, N2 = NN / NN1, M = (NN / NN1) / NN1;          \
    static constexpr int LD = NN1 + 1, VS = N2;                                          \
    static constexpr bool EXACT = true;                                                  \
    static_assert((NN / NN1) % NN1 == 0, "N1 must divide N2");                           \
  };
RIHVR_LINE(32, 4)
RIHVR_LINE(48, 4)
RIHVR_LINE(64, 8)
RIHVR_LINE(128, 8)
RIHVR_LINE(256, 16)
RIHVR_LINE(384, 8)
RIHVR_LINE(512, 16)
RIHVR_LINE(768, 16)
RIHVR_LINE(1024, 32)
RIHVR_LINE(2304, 48)  // the 2048 x 2048 hologram padded by 128 on each side
#undef RIHVR_LINE
template <>
struct LineCfg<640> {  // 20 threads a line, 32 elements each; 12 of them take a second stage-B row
  static constexpr int N = 640, N1 = 20, N2 = 32, M = 2;
  static constexpr int LD = N1 + 1, VS = M * N1;
  static constexpr bool EXACT = false;
};

// the first K values of a register array, as an array of K
template <int K, int L>
__device__ __forceinline__ float2 (&head(float2 (&a)[L]))[K] {
  static_assert(K <= L, "prefix longer than the array");
  return *reinterpret_cast<float2(*)[K]>(&a[0]);
}

// does stage-B row j of thread t exist (always, for the exact splits)
template <int N>
__device__ __forceinline__ bool row_ok(int t, int j) {
  using C = LineCfg<N>;
  if constexpr (C::EXACT) return true;
  else return t + C::N1 * j < C::N2;
}

#define RIHVR_FOR_EACH_SIZE(X) X(32) X(48) X(64) X(128) X(256) X(384) X(512) X(640) X(768) X(1024) X(2304)

bool line_size_supported(int n) {
  switch (n) {
#define RIHVR_CASE(NN) case NN:
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    return true;
    default:
      return false;
  }
}

// SM count of the current device, cached per device ordinal.  Worker threads of
// a frame batch and callers on other host threads read it concurrently, so the
// cache entries are atomics (a racing first fill writes the same value twice).
constexpr int kSmCacheDevices = 64;
static std::atomic<int> g_num_sms[kSmCacheDevices];
static int num_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  std::atomic<int>* slot = (dev >= 0 && dev < kSmCacheDevices) ? &g_num_sms[dev] : nullptr;
  int n = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (n <= 0) {
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if (slot) slot->store(n, std::memory_order_relaxed);
  }
  return n;
}

template <typename K>
static cudaError_t allow_smem(K kernel, size_t bytes) {
  // dynamic plus static shared memory above 48 KB needs the opt-in
  if (bytes + 4096 <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N1, int VS, bool INV>
__device__ __forceinline__ void stage_b_dft(float2 (&w)[VS]) {
  constexpr int M = VS / N1;
#pragma unroll
  for (int j = 0; j < M; ++j) {
    float2 s[N1];
#pragma unroll
    for (int k = 0; k < N1; ++k) s[k] = w[j * N1 + k];
    reg_fft<N1, INV>(s);
#pragma unroll
    for (int k = 0; k < N1; ++k) w[j * N1 + k] = s[k];
  }
}

// ---------------------------------------------------------------------------
// Row pass: one line per N1-thread group, lines contiguous in memory.
// ---------------------------------------------------------------------------
constexpr int kRowThreads = 256;

template <int N>
struct RowLayout {
  using C = LineCfg<N>;
  static constexpr int LPB = kRowThreads / C::N1;
  // lines of 48 threads straddle warps: the block then holds whole lines only
  // and exchanges through a block barrier instead of a warp one
  static constexpr bool WARP_LINES = (32 % C::N1) == 0;
  static constexpr int THREADS = LPB * C::N1;
  static constexpr int base_ls = C::N2 * C::LD;
  // pad the per-line stride so that lines sharing a half-warp hit different banks
  static constexpr int LS = (C::N1 >= 16) ? base_ls : base_ls + (((C::N1 % 16) - (base_ls % 16) + 16) % 16);
  static constexpr int SMEM = LPB * LS;  // float2 elements
  static constexpr size_t SMEM_BYTES = sizeof(float2) * SMEM;
};

// element of kind IN (compile time) as a complex value
template <int IN>
__device__ __forceinline__ float2 load_as(const void* p, size_t i) {
  if constexpr (IN == ELEM_R32) return make_float2(static_cast<const float*>(p)[i], 0.f);
  else if constexpr (IN == ELEM_STORE_BF16) return Store<__nv_bfloat162>::ld(static_cast<const __nv_bfloat162*>(p) + i);
  else if constexpr (IN == ELEM_STORE_F16) return Store<__half2>::ld(static_cast<const __half2*>(p) + i);
  else return static_cast<const float2*>(p)[i];
}

// The input element kind is a template parameter: with it known at compile
// time the N2 loads of a thread issue back to back (a run-time kind switch
// around each load serialises them).  Output is complex FP32.
template <int N, bool INV, int IN>
__global__ void __launch_bounds__(kRowThreads) k_rows(const void* __restrict__ in, float2* __restrict__ out,
                                                     long long nlines, float scale) {
  using C = LineCfg<N>;
  using Lay = RowLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, LD = C::LD;
  static_assert(Lay::WARP_LINES || Lay::THREADS <= kRowThreads, "whole lines per block");
  extern __shared__ __align__(128) float2 sm[];
  const int li = threadIdx.x / N1, t = threadIdx.x % N1;
  long long L = (long long)blockIdx.x * Lay::LPB + li;
  const bool active = L < nlines;
  if (!active) L = nlines - 1;
  const size_t base = (size_t)L * N;
  float2 v[C::VS];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) v[n2] = load_as<IN>(in, base + t + N1 * n2);
  reg_fft<N2, INV>(head<N2>(v));
  line_twiddle<N, N2, INV>(head<N2>(v), t);
  float2* sl = sm + li * Lay::LS;
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) sl[k2 * LD + t] = v[k2];
  if constexpr (Lay::WARP_LINES) {
    __syncwarp();
  } else {
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const bool ok = row_ok<N>(t, j);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[j * N1 + n1] = ok ? sl[(t + N1 * j) * LD + n1] : make_float2(0.f, 0.f);
  }
  stage_b_dft<N1, C::VS, INV>(v);
  if (active) {
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (row_ok<N>(t, j))
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) out[base + t + N1 * j + N2 * k1] = cscale(v[j * N1 + k1], scale);
  }
}

template <int N, bool INV, int IN>
static cudaError_t rows_launch(const void* in, float2* out, long long nlines, float scale, cudaStream_t st) {
  using Lay = RowLayout<N>;
  const long long blocks = (nlines + Lay::LPB - 1) / Lay::LPB;
  if (blocks <= 0) return cudaSuccess;
  cudaError_t e = allow_smem(k_rows<N, INV, IN>, Lay::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  k_rows<N, INV, IN><<<(unsigned)blocks, Lay::THREADS, Lay::SMEM_BYTES, st>>>(in, out, nlines, scale);
  return cudaGetLastError();
}

template <int N>
static cudaError_t rows_n(int inverse, int in_kind, const void* in, int out_kind, void* out, long long nlines,
                          float scale, cudaStream_t st) {
  if (out_kind != ELEM_C32) return cudaErrorInvalidValue;
  float2* o = static_cast<float2*>(out);
  if (inverse) {
    if (in_kind != ELEM_C32 && in_kind != ELEM_STORE_F32) return cudaErrorInvalidValue;
    return rows_launch<N, true, ELEM_C32>(in, o, nlines, scale, st);
  }
  switch (in_kind) {
    case ELEM_C32:
    case ELEM_STORE_F32: return rows_launch<N, false, ELEM_C32>(in, o, nlines, scale, st);
    case ELEM_R32: return rows_launch<N, false, ELEM_R32>(in, o, nlines, scale, st);
    case ELEM_STORE_BF16: return rows_launch<N, false, ELEM_STORE_BF16>(in, o, nlines, scale, st);
    case ELEM_STORE_F16: return rows_launch<N, false, ELEM_STORE_F16>(in, o, nlines, scale, st);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t launch_rows_fast(int inverse, int in_kind, const void* in, int out_kind, void* out, int W,
                                    long long nlines, float scale, cudaStream_t st) {
  switch (W) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return rows_n<NN>(inverse, in_kind, in, out_kind, out, nlines, scale, st);
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// Column passes: CC columns per block, N1 threads per column (lanes: column
// fastest so each warp-wide access covers CC*8 contiguous bytes of a row).
// Shared layout [k2][n1][c] with n1 padded to LD.
// ---------------------------------------------------------------------------
template <int N>
struct ColLayout {
  using C = LineCfg<N>;
  // columns per block.  Sides 256, 512 and 1024 take 128-thread blocks: two
  // or more blocks share an SM, so one block's barriers no longer idle the
  // whole SM (measured 10-17 % faster column passes than 256-thread blocks).
  // Sides 384 and 768 measured no gain or a loss and keep 256 threads.
  // Side 2304 (48 threads a column, 48 elements a thread) takes 4 columns:
  // 192 threads, so that the forward pass's 255 registers a thread fit.
  // Side 640 (20 threads a column) takes 8 columns: 160 threads.
  static constexpr int CC = (N == 256 || N == 512 || N == 1024) ? 128 / C::N1
                            : N == 2304                        ? 4
                            : N == 640                         ? 8
                                                               : (C::N1 >= 32 ? 8 : (C::N1 >= 16 ? 16 : 32));
  static constexpr int THREADS = CC * C::N1;
  static constexpr int SMEM_ELEMS = C::N2 * C::LD * CC;
  static constexpr size_t SMEM_BYTES = sizeof(float2) * SMEM_ELEMS;
  // one plane's column strip (N rows x CC columns) of complex values
  static constexpr size_t STRIP_ELEMS = (size_t)N * CC;
  // staging strips in shared memory next to the exchange buffer: two for the
  // forward pass (double-buffered prefetch), one complex + one FP64 strip for
  // the adjoint (spectrum and phase table, constant over z)
  // (only where two blocks still fit on an SM: side 2304 would take 222 KB)
  static constexpr bool STAGE = (N % CC == 0) && (SMEM_BYTES + 2 * sizeof(float2) * STRIP_ELEMS <= 113 * 1024);
  static constexpr size_t STAGE_BYTES = SMEM_BYTES + (STAGE ? 2 * sizeof(float2) * STRIP_ELEMS : 0);
};

// 16-byte asynchronous global -> shared copies (Ampere+ cp.async, L2 only)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory");
}

// Copy the CC-column strip starting at column x0 of an N x N plane into a
// dense [row][CC] shared buffer (16-byte pieces spread over the block).
template <int N, typename T>
__device__ __forceinline__ void strip_async(T* dst, const T* plane, int x0) {
  using Lay = ColLayout<N>;
  constexpr int CC = Lay::CC;
  constexpr int PER_ROW = CC * (int)sizeof(T) / 16;  // 16-byte pieces per strip row
  constexpr int PIECES = N * PER_ROW;
  const char* src = reinterpret_cast<const char*>(plane + x0);
  char* d = reinterpret_cast<char*>(dst);
  for (int k = threadIdx.x; k < PIECES; k += Lay::THREADS) {
    const int row = k / PER_ROW, piece = k - row * PER_ROW;
    cp_async16(d + ((size_t)row * CC * sizeof(T) + piece * 16), src + ((size_t)row * N * sizeof(T) + piece * 16));
  }
}

// Phase-table reads are issued in groups separated by a compiler scheduling
// fence so that the FP64 table values of a whole line are not all live at once.
constexpr int kPhaseGroup = 8;
__device__ __forceinline__ void sched_fence() { asm volatile("" ::: "memory"); }
// Hide a pointer's loop invariance from the compiler: the z loops re-read the
// phase table (and the residual spectrum) from L1/L2 every plane instead of
// pinning a whole line of them in registers.
template <typename T>
__device__ __forceinline__ const T* launder(const T* p) {
  asm volatile("mov.b64 %0, %0;" : "+l"(p));
  return p;
}
// Same for the twiddle index: recomputing a line's inter-stage twiddles every
// plane costs two sincospi and ~N2 complex products, far less than keeping
// N2 complex twiddles live across the z loop.
__device__ __forceinline__ int launder_i(int v) {
  asm volatile("mov.b32 %0, %0;" : "+r"(v));
  return v;
}

// Tensor-memory-accelerator (TMA) store of a dense shared-memory tile
// [rows][CC] of 8-byte elements to a 3-D (x, row, plane) tensor.  Stores only,
// no multicast.  The coordinates are non-negative and x * 8 bytes is a
// multiple of 16.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* smem, int x, int y, int z) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<unsigned long long>(map)),
               "r"(s), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the source tiles of every committed store have been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// order this thread's shared-memory writes before later async-proxy reads
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// rows per TMA box: the largest divisor of N not above 256 (the box limit)
template <int N>
constexpr int tma_rows() {
  int r = 1;
  for (int d = 1; d <= 256 && d <= N; ++d)
    if (N % d == 0) r = d;
  return r;
}

// Exchange + stage B shared by all column kernels.  On entry v holds the
// twiddled stage-A output of this thread; on exit the stage-B output.
template <int N, bool INV>
__device__ __forceinline__ void col_exchange(float2 (&v)[LineCfg<N>::VS], float2* sm, int c, int t) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, LD = C::LD, CC = Lay::CC;
  __syncthreads();  // previous users of sm are done
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) sm[(k2 * LD + t) * CC + c] = v[k2];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < M; ++j) {
    const bool ok = row_ok<N>(t, j);
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      v[j * N1 + n1] = ok ? sm[((t + N1 * j) * LD + n1) * CC + c] : make_float2(0.f, 0.f);
  }
  stage_b_dft<N1, C::VS, INV>(v);
}

// The column passes walk many planes with the same thread-to-row assignment,
// so a thread's inter-stage twiddles are the same for every plane.  For lines
// of up to 32 elements a thread they are computed once and kept in registers
// (one complex product an element per plane instead of two plus the anchor
// products); shared memory limits the column passes to 8 warps per SM, which
// leaves the registers free.  Longer lines regenerate them every plane.
template <int N>
constexpr bool kHoistTw = LineCfg<N>::N2 <= 32 && LineCfg<N>::EXACT;

template <int N, int N2, bool INV>
__device__ __forceinline__ void apply_twiddles(float2 (&v)[N2], const float2 (&tw)[kHoistTw<N> ? N2 : 1], int t) {
  if constexpr (kHoistTw<N>) {
#pragma unroll
    for (int k = 1; k < N2; ++k) v[k] = cmul(v[k], tw[k]);
  } else {
    line_twiddle<N, N2, INV>(v, launder_i(t));
  }
}

// acc += v h: four fused multiply-adds where the twiddles are hoisted (lines
// of up to 32 elements a thread); the longer lines keep the product-then-add
// form, whose shorter live ranges keep them within the register file
template <int N>
__device__ __forceinline__ void cmac(float2& acc, float2 v, float2 h) {
  if constexpr (kHoistTw<N>) {
    acc.x = fmaf(v.x, h.x, fmaf(-v.y, h.y, acc.x));
    acc.y = fmaf(v.x, h.y, fmaf(v.y, h.x, acc.y));
  } else {
    acc = cadd(acc, cmul(v, h));
  }
}

// Adjoint column pass: U_z(:, x) = IDFT_y( conj(H'_z(:, x)) * Rs(:, x) ), z in [zb, ze).
// Square planes: the row pitch equals the line length N, so every element
// offset below is a compile-time multiple of N.  Rs already carries 1/(W H).
// The spectrum and phase-table strips are the same for every plane: they are
// staged in shared memory once per block when they fit.
template <int N, bool TMA>
__global__ void __launch_bounds__(ColLayout<N>::THREADS) k_adj_col(const float2* __restrict__ Rs,
                                                                   const double* __restrict__ cturn,
                                                                   const double* __restrict__ zlist,
                                                                   float2* __restrict__ U, int z0, int z1,
                                                                   int zpb, const __grid_constant__ CUtensorMap umap) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, CC = Lay::CC;
  constexpr int W = N;
  extern __shared__ __align__(128) float2 sm[];  // TMA sources need 128-byte alignment
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  constexpr size_t HW = (size_t)N * W;
  float2* s_rs = sm + Lay::SMEM_ELEMS;
  double* s_ct = reinterpret_cast<double*>(s_rs + Lay::STRIP_ELEMS);
  if constexpr (Lay::STAGE) {
    strip_async<N>(s_rs, Rs, blockIdx.x * CC);
    strip_async<N>(s_ct, cturn, blockIdx.x * CC);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
  }
  const float2* rs = Rs + (size_t)t * W + x;
  const double* ct = cturn + (size_t)t * W + x;
  float2 tw[kHoistTw<N> ? N2 : 1];
  if constexpr (kHoistTw<N>) line_twiddles<N, N2, true>(tw, t);
  double znext = zb < ze ? zlist[zb] : 0.0;
#pragma unroll 1
  for (int z = zb; z < ze; ++z) {
    const double zz = znext;
    if (z + 1 < ze) znext = zlist[z + 1];  // in flight during this plane
    float2 v[C::VS];
    if constexpr (Lay::STAGE) {
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) {
        const int i = (t + N1 * n2) * CC + c;
        v[n2] = cmul(s_rs[i], transfer(zz, s_ct[i], true));
      }
    } else {
      const float2* rsz = launder(rs);
      const double* ctz = launder(ct);
#pragma unroll
      for (int g = 0; g < N2; g += kPhaseGroup) {
#pragma unroll
        for (int q = 0; q < kPhaseGroup; ++q) {
          const int n2 = g + q;
          v[n2] = cmul(__ldg(rsz + (size_t)n2 * N1 * W), transfer(zz, __ldg(ctz + (size_t)n2 * N1 * W), true));
        }
        sched_fence();
      }
    }
    reg_fft<N2, true>(head<N2>(v));
    apply_twiddles<N, N2, true>(head<N2>(v), tw, t);
    // the exchange buffer also holds the previous plane's output tile: its
    // store must have read it (the exchange starts with a barrier)
    if (TMA && threadIdx.x == 0) bulk_wait_read_all();
    col_exchange<N, true>(v, sm, c, t);
    if constexpr (TMA) {
      // plane z's [N][CC] column strip goes out through the TMA from the
      // exchange buffer, as a few bulk stores instead of N2 8-byte stores a thread
      __syncthreads();  // every thread is done reading the exchange
#pragma unroll
      for (int j = 0; j < M; ++j)
        if (row_ok<N>(t, j))
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) sm[(N1 * j + N2 * k1 + t) * CC + c] = v[j * N1 + k1];
      fence_smem_async();
      __syncthreads();
      if (threadIdx.x == 0) {
        constexpr int R = tma_rows<N>();
#pragma unroll 1
        for (int b = 0; b < N; b += R) tma_store_3d(&umap, sm + b * CC, blockIdx.x * CC, b, z);
        bulk_commit();
      }
    } else if (col_ok) {
      float2* Uz = U + (size_t)z * HW + (size_t)t * W + x;
#pragma unroll
      for (int j = 0; j < M; ++j)
        if (row_ok<N>(t, j))
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) Uz[(size_t)(N1 * j + N2 * k1) * W] = v[j * N1 + k1];
    }
  }
  if (TMA && threadIdx.x == 0) bulk_wait_all();
}

// Inter-stage twiddles as a per-block table in shared memory, for column
// kernels that run three blocks an SM: w^(t k) for the N1 thread rows t and
// the N2 elements k of a line, the same values (same FP32 expression) that
// line_twiddles keeps in registers, so results are bit-identical to the
// register-resident form while 2 N2 registers a thread are freed.  Rows are
// padded to an even length (16-byte aligned pairs) that spreads the 8 rows a
// warp reads over all 32 banks.
template <int N>
struct TwTable {
  using C = LineCfg<N>;
  static constexpr int LDT = C::N2 + 2;  // float2 per row
  static constexpr int ELEMS = C::N1 * LDT;
  static constexpr size_t BYTES = sizeof(float2) * ELEMS;
};

// Blocks an SM the table-twiddle column kernels are compiled for: three for
// lines of up to 32 elements a thread; one for 48 (sides 384, 768 and 2304),
// whose lines alone take most of the register file.
template <int N>
constexpr int col3_minb() {
  return LineCfg<N>::N2 <= 32 ? 3 : 1;
}

template <int N, bool INV>
__device__ __forceinline__ void tw_table_build(float2* tab) {
  using C = LineCfg<N>;
  constexpr int N2 = C::N2, LDT = TwTable<N>::LDT;
  const float sgn = INV ? 2.0f : -2.0f;
  for (int i = threadIdx.x; i < C::N1 * N2; i += ColLayout<N>::THREADS) {
    const int t = i / N2, k = i - t * N2;
    float s, c;
    sincospif(sgn * (float)((t * k) % N) / (float)N, &s, &c);
    tab[t * LDT + k] = make_float2(c, s);
  }
}

// v[k] *= w^(t k), k >= 1, from the table (pairs of twiddles per 16-byte load)
template <int N>
__device__ __forceinline__ void tw_table_apply(float2 (&v)[LineCfg<N>::N2], const float2* tab, int t) {
  constexpr int N2 = LineCfg<N>::N2;
  static_assert(N2 % 2 == 0, "twiddle pairs");
  const float4* row = reinterpret_cast<const float4*>(tab + t * TwTable<N>::LDT);
#pragma unroll
  for (int k = 0; k < N2; k += 2) {
    const float4 q = row[k / 2];
    if (k > 0) v[k] = cmul(v[k], make_float2(q.x, q.y));
    v[k + 1] = cmul(v[k + 1], make_float2(q.z, q.w));
  }
}

// Transfer function H'_z = exp(i 2 pi u), u = frac(z * cturn), with the
// accurate sincospi: used where a value seeds many planes (the recurrence
// below), so its error is not multiplied by the plane count.
__device__ __forceinline__ float2 transfer_accurate(double z, double cturn, bool conj_) {
  double u = z * cturn;
  u -= rint(u);
  float s, c;
  sincospif(2.0f * (float)u, &s, &c);
  return make_float2(c, conj_ ? -s : s);
}

// Planes between exact re-anchorings of the adjoint recurrence.  FP32
// rotations drift by about one rounding a step; 16 steps keep that near 1e-6.
constexpr int kAdjAnchor = 16;

// Adjoint column pass for evenly spaced planes (z_{k+1} - z_k = dz for all k):
// Y_z = conj(H'_z) Rs advances from plane to plane by the rotation
// D = conj(H'_dz), one complex product an element, instead of an FP64 phase
// reduction and a sincos.  Y lives in registers and D in shared memory, which
// replaces both staged strips of k_adj_col (spectrum and phase table): 66 KB
// a block at side 1024 instead of 98 KB, so three blocks share an SM.  Every
// kAdjAnchor planes Y is recomputed exactly from Rs and the FP64 phase table.
// Lines of up to 32 elements a thread only (the inter-stage twiddles are
// regenerated each plane to leave registers for Y).
//
// TWM selects the inter-stage twiddles: 1 keeps them in registers as k_adj_col
// does (fewest instructions a plane, two blocks an SM); 0 regenerates them
// each plane (three blocks fit, twice the instructions); 2 reads them from a
// per-block shared table (one 16-byte load per two elements, three blocks an
// SM).  The autotuner picks one of these or the direct evaluation.
template <int N, bool TMA, int TWM>
__global__ void __launch_bounds__(ColLayout<N>::THREADS, TWM == 1 ? 2 : col3_minb<N>())
    k_adj_col_rec(const float2* __restrict__ Rs, const double* __restrict__ cturn, const double* __restrict__ zlist,
                  double dz, float2* __restrict__ U, int z0, int z1, int zpb,
                  const __grid_constant__ CUtensorMap umap) {
  constexpr bool HOIST = TWM == 1;
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, CC = Lay::CC;
  static_assert(N2 <= (TWM == 2 ? 48 : 32), "the recurrence keeps a line's elements in registers");
  constexpr int W = N;
  extern __shared__ __align__(128) float2 sm[];
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  if (zb >= ze) return;
  float2* s_d = sm + Lay::SMEM_ELEMS;  // this thread's rotations, [row][CC] (thread-private slots)
  float2* s_tw = s_d + Lay::STRIP_ELEMS;  // twiddle table (TWM 2)
  const float2* rs = Rs + (size_t)t * W + x;
  const double* ct = cturn + (size_t)t * W + x;
  float2 tw[HOIST ? N2 : 1];
  if constexpr (HOIST) line_twiddles<N, N2, true>(tw, t);
  if constexpr (TWM == 2) {
    tw_table_build<N, true>(s_tw);
    __syncthreads();
  }
  float2 y[N2];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) {
    const double cn = __ldg(ct + (size_t)n2 * N1 * W);
    s_d[(t + N1 * n2) * CC + c] = transfer_accurate(dz, cn, true);
    y[n2] = cmul(__ldg(rs + (size_t)n2 * N1 * W), transfer_accurate(zlist[zb], cn, true));
  }
#pragma unroll 1
  for (int z = zb; z < ze; ++z) {
    if (z > zb) {
      if ((z - zb) % kAdjAnchor == 0) {
        const double zz = zlist[z];
        const float2* rsz = launder(rs);
        const double* ctz = launder(ct);
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2)
          y[n2] = cmul(__ldg(rsz + (size_t)n2 * N1 * W), transfer_accurate(zz, __ldg(ctz + (size_t)n2 * N1 * W), true));
      } else {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) y[n2] = cmul(y[n2], s_d[(t + N1 * n2) * CC + c]);
      }
    }
    float2 v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) v[n2] = y[n2];
    reg_fft<N2, true>(v);
    if constexpr (HOIST) {
#pragma unroll
      for (int k = 1; k < N2; ++k) v[k] = cmul(v[k], tw[k]);
    } else if constexpr (TWM == 2) {
      tw_table_apply<N>(v, s_tw, t);
    } else {
      line_twiddle<N, N2, true>(v, launder_i(t));
    }
    if (TMA && threadIdx.x == 0) bulk_wait_read_all();
    col_exchange<N, true>(v, sm, c, t);
    if constexpr (TMA) {
      __syncthreads();
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) sm[(N1 * j + N2 * k1 + t) * CC + c] = v[j * N1 + k1];
      fence_smem_async();
      __syncthreads();
      if (threadIdx.x == 0) {
        constexpr int R = tma_rows<N>();
#pragma unroll 1
        for (int b = 0; b < N; b += R) tma_store_3d(&umap, sm + b * CC, blockIdx.x * CC, b, z);
        bulk_commit();
      }
    } else if (col_ok) {
      float2* Uz = U + (size_t)z * ((size_t)N * W) + (size_t)t * W + x;
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) Uz[(size_t)(N1 * j + N2 * k1) * W] = v[j * N1 + k1];
    }
  }
  if (TMA && threadIdx.x == 0) bulk_wait_all();
}

// Forward column pass with the z-sum: Spart[chunk](:, x) = sum_z H'_z(:, x) DFT_y(T_z(:, x)).
// When they fit next to the exchange buffer, the block's strip of the phase
// table (constant over z) and one strip of T are staged in shared memory:
// plane z+1's strip is fetched asynchronously once the exchange of plane z has
// consumed the buffer, and overlaps the transfer-function multiply and sum.
template <int N>
__global__ void __launch_bounds__(ColLayout<N>::THREADS) k_fwd_col(const float2* __restrict__ T,
                                                                   const double* __restrict__ cturn,
                                                                   const double* __restrict__ zlist,
                                                                   float2* __restrict__ Spart, int z0, int z1,
                                                                   int zpb) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, CC = Lay::CC;
  constexpr int W = N;
  extern __shared__ __align__(128) float2 sm[];
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  constexpr size_t HW = (size_t)N * W;
  const double* ct = cturn + (size_t)t * W + x;
  float2* const s_t = sm + Lay::SMEM_ELEMS;                                  // one strip of T
  const double* const s_ct = reinterpret_cast<const double*>(s_t + Lay::STRIP_ELEMS);  // phase-table strip
  if constexpr (Lay::STAGE) {
    strip_async<N>(const_cast<double*>(s_ct), cturn, blockIdx.x * CC);
    if (zb < ze) strip_async<N>(s_t, T + (size_t)zb * HW, blockIdx.x * CC);
    cp_async_commit();
  }
  float2 acc[C::VS];
#pragma unroll
  for (int i = 0; i < C::VS; ++i) acc[i] = make_float2(0.f, 0.f);
  float2 tw[kHoistTw<N> ? N2 : 1];
  if constexpr (kHoistTw<N>) line_twiddles<N, N2, false>(tw, t);
  double znext = zb < ze ? zlist[zb] : 0.0;
#pragma unroll 1
  for (int z = zb; z < ze; ++z) {
    const double zz = znext;
    if (z + 1 < ze) znext = zlist[z + 1];  // in flight during this plane
    float2 v[C::VS];
    if constexpr (Lay::STAGE) {
      cp_async_wait<0>();
      __syncthreads();
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = s_t[(t + N1 * n2) * CC + c];
    } else {
      const float2* Tz = T + (size_t)z * HW + (size_t)t * W + x;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = Tz[(size_t)n2 * N1 * W];
    }
    reg_fft<N2, false>(head<N2>(v));
    apply_twiddles<N, N2, false>(head<N2>(v), tw, t);
    // the exchange's first barrier also orders every thread's reads of s_t
    // before the refill below
    col_exchange<N, false>(v, sm, c, t);
    if constexpr (Lay::STAGE) {
      if (z + 1 < ze) strip_async<N>(s_t, T + (size_t)(z + 1) * HW, blockIdx.x * CC);
      cp_async_commit();
#pragma unroll
      for (int j = 0; j < M; ++j)
        if (row_ok<N>(t, j))
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) {
            const float2 h = transfer(zz, s_ct[(N1 * j + N2 * k1 + t) * CC + c], false);
            cmac<N>(acc[j * N1 + k1], v[j * N1 + k1], h);
          }
    } else {
      const double* ctz = launder(ct);
#pragma unroll
      for (int g = 0; g < C::VS; g += kPhaseGroup) {
#pragma unroll
        for (int q = 0; q < kPhaseGroup; ++q) {
          const int j = (g + q) / N1, k1 = (g + q) % N1;
          if (row_ok<N>(t, j)) {
            const float2 h = transfer(zz, __ldg(ctz + (size_t)(N1 * j + N2 * k1) * W), false);
            cmac<N>(acc[j * N1 + k1], v[j * N1 + k1], h);
          }
        }
        sched_fence();
      }
    }
  }
  if constexpr (Lay::STAGE) cp_async_wait<0>();
  if (col_ok) {
    float2* Sp = Spart + (size_t)blockIdx.y * HW + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (row_ok<N>(t, j))
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) Sp[(size_t)(N1 * j + N2 * k1) * W] = acc[j * N1 + k1];
  }
}

// Forward column pass for evenly spaced planes, by Horner's scheme: with
// H'_z = H'_{zb} D^(z - zb) and D = H'_dz,
//   sum_{z in [zb, ze)} H'_z V_z = H'_{zb} (((V_{ze-1} D + V_{ze-2}) D + ...) D + V_{zb}),
// so each plane costs one complex multiply-add by D (held in shared memory in
// place of the FP64 phase-table strip) instead of an FP64 phase reduction, a
// sincos and a multiply-add; H'_{zb} is applied once, exactly, at the end.  The
// planes go in descending order.  D^k carries the rounding of D k times (about
// k x 6e-8 in phase), which stays near 1e-5 for the longest z-chunks used.
template <int N>
__global__ void __launch_bounds__(ColLayout<N>::THREADS) k_fwd_col_horner(const float2* __restrict__ T,
                                                                          const double* __restrict__ cturn,
                                                                          const double* __restrict__ zlist, double dz,
                                                                          float2* __restrict__ Spart, int z0, int z1,
                                                                          int zpb) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, CC = Lay::CC;
  static_assert(Lay::STAGE && C::EXACT, "staged square sizes only");
  constexpr int W = N;
  extern __shared__ __align__(128) float2 sm[];
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  constexpr size_t HW = (size_t)N * W;
  const double* ct = cturn + (size_t)t * W + x;
  float2* const s_t = sm + Lay::SMEM_ELEMS;       // one strip of T
  float2* const s_d = s_t + Lay::STRIP_ELEMS;     // this thread's rotations D, stage-B layout
  if (zb < ze) strip_async<N>(s_t, T + (size_t)(ze - 1) * HW, blockIdx.x * CC);
  cp_async_commit();
#pragma unroll
  for (int j = 0; j < M; ++j)
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1)
      s_d[(N1 * j + N2 * k1 + t) * CC + c] = transfer_accurate(dz, __ldg(ct + (size_t)(N1 * j + N2 * k1) * W), false);
  float2 acc[N2];
#pragma unroll
  for (int i = 0; i < N2; ++i) acc[i] = make_float2(0.f, 0.f);
  float2 tw[kHoistTw<N> ? N2 : 1];
  if constexpr (kHoistTw<N>) line_twiddles<N, N2, false>(tw, t);
#pragma unroll 1
  for (int z = ze - 1; z >= zb; --z) {
    cp_async_wait<0>();
    __syncthreads();
    float2 v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) v[n2] = s_t[(t + N1 * n2) * CC + c];
    reg_fft<N2, false>(v);
    apply_twiddles<N, N2, false>(v, tw, t);
    // the exchange's first barrier orders every thread's reads of s_t before the refill
    col_exchange<N, false>(v, sm, c, t);
    if (z - 1 >= zb) strip_async<N>(s_t, T + (size_t)(z - 1) * HW, blockIdx.x * CC);
    cp_async_commit();
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 d = s_d[(N1 * j + N2 * k1 + t) * CC + c];
        float2& a = acc[j * N1 + k1];
        const float2 u = v[j * N1 + k1];
        const float ax = a.x;
        a.x = fmaf(ax, d.x, fmaf(-a.y, d.y, u.x));
        a.y = fmaf(ax, d.y, fmaf(a.y, d.x, u.y));
      }
  }
  cp_async_wait<0>();
  if (col_ok && zb < ze) {
    const double zz = zlist[zb];
    float2* Sp = Spart + (size_t)blockIdx.y * HW + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 h = transfer_accurate(zz, __ldg(ct + (size_t)(N1 * j + N2 * k1) * W), false);
        Sp[(size_t)(N1 * j + N2 * k1) * W] = cmul(acc[j * N1 + k1], h);
      }
  } else if (col_ok) {
    float2* Sp = Spart + (size_t)blockIdx.y * HW + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) Sp[(size_t)(N1 * j + N2 * k1) * W] = make_float2(0.f, 0.f);
  }
}

// The same Horner sum with three blocks an SM instead of two.  Shared memory
// per block drops from three column strips to two plus the twiddle table: T
// lands in the exchange buffer itself, and plane z-1's strip is requested as
// soon as every thread has read plane z's exchange, so its load overlaps the
// second DFT stage and the multiply-add (and the other blocks' work).  The
// inter-stage twiddles come from the per-block table, which frees the
// registers the third block needs.  Same arithmetic, same bits as
// k_fwd_col_horner.
template <int N>
constexpr size_t horner1_smem() {
  using Lay = ColLayout<N>;
  constexpr size_t buf = Lay::SMEM_ELEMS > Lay::STRIP_ELEMS ? (size_t)Lay::SMEM_ELEMS : Lay::STRIP_ELEMS;
  return sizeof(float2) * (buf + Lay::STRIP_ELEMS) + TwTable<N>::BYTES + 16;  // + the mbarrier
}

// Square sizes that have the table-twiddle forms (k_fwd_col_horner1, and
// k_adj_col_rec with TWM 2): whole lines a thread (N1 | N2), column blocks
// that tile the row, up to 48 elements a thread, and the exchange buffer,
// the rotation strip and the table within the 227 KB a block may take.
template <int N>
constexpr bool kTableCols = LineCfg<N>::EXACT && (N % ColLayout<N>::CC == 0) && LineCfg<N>::N2 <= 48 &&
                            LineCfg<N>::N2 % 2 == 0 && horner1_smem<N>() <= 227 * 1024;

// Bounded waits of the TMA-fed column passes that ran out since the last read
// (col_wait_timeouts).  None is expected: a wait covers one strip copy.
__device__ unsigned g_col_wait_timeouts;
constexpr unsigned kColMaxSpins = 1u << 26;

__device__ __forceinline__ void col_mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(bar),
               "r"(bytes)
               : "memory");
}

// wait for phase `parity` of the mbarrier, at most kColMaxSpins tries; false when the bound ran out
__device__ __forceinline__ bool col_mbar_wait(unsigned bar, unsigned parity) {
  for (unsigned i = 0; i < kColMaxSpins; ++i) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// TMA load of a [rows][CC] box of 8-byte elements (x, row, plane) into shared
// memory, completing on the mbarrier.  No multicast; x * 8 bytes is a multiple
// of 16 and every coordinate lies inside the tensor.
__device__ __forceinline__ void tma_load_3d(void* smem, const CUtensorMap* map, int x, int y, int z, unsigned bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(d),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// With TMA, one thread loads each plane's strip as tma_rows<N>-row boxes that
// complete on an mbarrier, instead of every thread issuing 16-byte cp.async
// pieces.  Every wait on the mbarrier is bounded: when one runs out, the block
// counts it in g_col_wait_timeouts (read back by col_wait_timeouts), gives the
// copy in flight one more bounded wait and leaves without writing its sums.
template <int N, bool TMA>
__global__ void __launch_bounds__(ColLayout<N>::THREADS, col3_minb<N>())
    k_fwd_col_horner1(const float2* __restrict__ T, const double* __restrict__ cturn,
                      const double* __restrict__ zlist, double dz, float2* __restrict__ Spart, int z0, int z1,
                      int zpb, const __grid_constant__ CUtensorMap tmap) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, LD = C::LD, CC = Lay::CC;
  static_assert(C::EXACT && N % CC == 0 && N2 <= 48, "square sizes of up to 48 elements a thread");
  constexpr int W = N;
  constexpr size_t BUF = Lay::SMEM_ELEMS > Lay::STRIP_ELEMS ? (size_t)Lay::SMEM_ELEMS : Lay::STRIP_ELEMS;
  extern __shared__ __align__(128) float2 sm[];
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  constexpr size_t HW = (size_t)N * W;
  const double* ct = cturn + (size_t)t * W + x;
  float2* const s_d = sm + BUF;                  // this thread's rotations D, stage-B layout
  float2* const s_tw = s_d + Lay::STRIP_ELEMS;   // twiddle table
  uint64_t* const bar = reinterpret_cast<uint64_t*>(s_tw + TwTable<N>::ELEMS);
  const unsigned sbar = (unsigned)__cvta_generic_to_shared(bar);
  unsigned phase = 0;
  constexpr int R = tma_rows<N>();
  constexpr unsigned kStripBytes = (unsigned)(sizeof(float2) * Lay::STRIP_ELEMS);
  // plane z's strip into the buffer: by TMA (thread 0) or cp.async (all threads)
  auto request = [&](int z) {
    if constexpr (TMA) {
      if (threadIdx.x == 0) {
        fence_smem_async();  // the block's reads of the buffer come before the copy's writes
        col_mbar_expect_tx(sbar, kStripBytes);
#pragma unroll 1
        for (int b = 0; b < N; b += R) tma_load_3d(sm + b * CC, &tmap, blockIdx.x * CC, b, z, sbar);
      }
    } else {
      strip_async<N>(sm, T + (size_t)z * HW, blockIdx.x * CC);
      cp_async_commit();
    }
  };
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  if (zb < ze) request(ze - 1);
  tw_table_build<N, false>(s_tw);
#pragma unroll
  for (int j = 0; j < M; ++j)
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1)
      s_d[(N1 * j + N2 * k1 + t) * CC + c] = transfer_accurate(dz, __ldg(ct + (size_t)(N1 * j + N2 * k1) * W), false);
  float2 acc[N2];
#pragma unroll
  for (int i = 0; i < N2; ++i) acc[i] = make_float2(0.f, 0.f);
#pragma unroll 1
  for (int z = ze - 1; z >= zb; --z) {
    if constexpr (TMA) {
      const bool ok = col_mbar_wait(sbar, phase);
      if (__syncthreads_or(!ok)) {  // a wait ran out: count it, let the copy land, leave
        if (threadIdx.x == 0) {
          atomicAdd(&g_col_wait_timeouts, 1u);
          col_mbar_wait(sbar, phase);
        }
        return;
      }
      phase ^= 1u;
    } else {
      cp_async_wait<0>();
      __syncthreads();  // plane z's strip (and, the first time, the table) is visible
    }
    float2 v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) v[n2] = sm[(t + N1 * n2) * CC + c];
    reg_fft<N2, false>(v);
    tw_table_apply<N>(v, s_tw, t);
    __syncthreads();  // every thread has read the strip: the buffer becomes the exchange
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) sm[(k2 * LD + t) * CC + c] = v[k2];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[j * N1 + n1] = sm[((t + N1 * j) * LD + n1) * CC + c];
    __syncthreads();  // every thread has read the exchange: refill with plane z-1
    if (z - 1 >= zb) request(z - 1);
    stage_b_dft<N1, C::VS, false>(v);
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 d = s_d[(N1 * j + N2 * k1 + t) * CC + c];
        float2& a = acc[j * N1 + k1];
        const float2 u = v[j * N1 + k1];
        const float ax = a.x;
        a.x = fmaf(ax, d.x, fmaf(-a.y, d.y, u.x));
        a.y = fmaf(ax, d.y, fmaf(a.y, d.x, u.y));
      }
  }
  if constexpr (!TMA) cp_async_wait<0>();
  if (col_ok && zb < ze) {
    const double zz = zlist[zb];
    float2* Sp = Spart + (size_t)blockIdx.y * HW + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 h = transfer_accurate(zz, __ldg(ct + (size_t)(N1 * j + N2 * k1) * W), false);
        Sp[(size_t)(N1 * j + N2 * k1) * W] = cmul(acc[j * N1 + k1], h);
      }
  } else if (col_ok) {
    float2* Sp = Spart + (size_t)blockIdx.y * HW + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) Sp[(size_t)(N1 * j + N2 * k1) * W] = make_float2(0.f, 0.f);
  }
}

// Plain column DFT of one (square) plane.
template <int N, bool INV>
__global__ void __launch_bounds__(ColLayout<N>::THREADS) k_plane_col(const float2* __restrict__ in,
                                                                     float2* __restrict__ out, float scale) {
  using C = LineCfg<N>;
  using Lay = ColLayout<N>;
  constexpr int N1 = C::N1, N2 = C::N2, M = C::M, CC = Lay::CC;
  constexpr int W = N;
  extern __shared__ __align__(128) float2 sm[];
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const int xr = blockIdx.x * CC + c;
  const bool col_ok = xr < W;
  const int x = col_ok ? xr : W - 1;
  const float2* src = in + (size_t)t * W + x;
  float2 v[C::VS];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) v[n2] = src[(size_t)n2 * N1 * W];
  reg_fft<N2, INV>(head<N2>(v));
  line_twiddle<N, N2, INV>(head<N2>(v), t);
  col_exchange<N, INV>(v, sm, c, t);
  if (col_ok) {
    float2* dst = out + (size_t)t * W + x;
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (row_ok<N>(t, j))
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) dst[(size_t)(N1 * j + N2 * k1) * W] = cscale(v[j * N1 + k1], scale);
  }
}

template <int N>
static int col_strips(int W) {
  return (W + ColLayout<N>::CC - 1) / ColLayout<N>::CC;
}

// cuTensorMapEncodeTiled, resolved once through the runtime (no link-time
// dependence on the driver library); null when unavailable
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
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

// 3-D map (column, row, plane) of nz square N x N planes of 8-byte elements
// with a box of CC columns x rows rows x 1 plane
static bool plane_stack_map(CUtensorMap* m, void* base, int n, int nz, int cc, int rows) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)n * 8, (cuuint64_t)n * n * 8};
  const cuuint32_t box[3] = {(cuuint32_t)cc, (cuuint32_t)rows, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int N>
static cudaError_t adj_col_n(const float2* Rs, const double* cturn, const double* zlist, float2* U, int W,
                             int z0, int z1, cudaStream_t st, int chunks_hint, double dz_uniform, int rec_mode) {
  using Lay = ColLayout<N>;
  const int nz = z1 - z0;
  if (nz <= 0) return cudaSuccess;
  const int strips = col_strips<N>(W);
  // the recurrence variants: evenly spaced planes, lines of <= 32 elements a
  // thread; `rec_mode` 1 regenerates the twiddles each plane, 2 keeps them;
  // 3 reads them from a shared table (lines of up to 48 elements)
  constexpr bool kRecOk = kHoistTw<N> && (N % Lay::CC == 0);
  const bool rec = dz_uniform != 0.0 && ((kRecOk && rec_mode != 0) || (kTableCols<N> && rec_mode == 3));
  const int target = (rec && rec_mode != 2 ? 12 : 8) * num_sms();
  int chunks = chunks_hint > 0 ? chunks_hint : (target + strips - 1) / strips;
  if (chunks > nz) chunks = nz;
  if (chunks < 1) chunks = 1;
  const int zpb = (nz + chunks - 1) / chunks;
  chunks = (nz + zpb - 1) / zpb;
  CUtensorMap umap;
  std::memset(&umap, 0, sizeof(umap));
  const bool tma = (W == N) && (N % Lay::CC == 0) && plane_stack_map(&umap, U, N, z1, Lay::CC, tma_rows<N>());
  cudaError_t e;
  if constexpr (kRecOk || kTableCols<N>) {
    if (rec) {
      // the twiddle table follows the rotation strip (rec_mode 3)
      const size_t smem =
          Lay::SMEM_BYTES + sizeof(float2) * Lay::STRIP_ELEMS + (rec_mode == 3 ? TwTable<N>::BYTES : 0);
      auto go = [&](auto kern) -> cudaError_t {
        cudaError_t e2 = allow_smem(kern, smem);
        if (e2 != cudaSuccess) return e2;
        kern<<<dim3(strips, chunks), Lay::THREADS, smem, st>>>(Rs, cturn, zlist, dz_uniform, U, z0, z1, zpb, umap);
        return cudaGetLastError();
      };
      if constexpr (kTableCols<N>) {
        if (rec_mode == 3) return tma ? go(k_adj_col_rec<N, true, 2>) : go(k_adj_col_rec<N, false, 2>);
      }
      if constexpr (kRecOk) {
        if (rec_mode == 2) return tma ? go(k_adj_col_rec<N, true, 1>) : go(k_adj_col_rec<N, false, 1>);
        return tma ? go(k_adj_col_rec<N, true, 0>) : go(k_adj_col_rec<N, false, 0>);
      }
    }
  }
  if (tma) {
    e = allow_smem(k_adj_col<N, true>, Lay::STAGE_BYTES);
    if (e != cudaSuccess) return e;
    k_adj_col<N, true><<<dim3(strips, chunks), Lay::THREADS, Lay::STAGE_BYTES, st>>>(Rs, cturn, zlist, U, z0, z1,
                                                                                        zpb, umap);
  } else {
    e = allow_smem(k_adj_col<N, false>, Lay::STAGE_BYTES);
    if (e != cudaSuccess) return e;
    k_adj_col<N, false><<<dim3(strips, chunks), Lay::THREADS, Lay::STAGE_BYTES, st>>>(Rs, cturn, zlist, U, z0, z1,
                                                                                         zpb, umap);
  }
  return cudaGetLastError();
}

bool adj_recurrence_supported(int W, int H, int rec_mode) {
  if (W != H) return false;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return rec_mode == 3 ? kTableCols<NN> : (kHoistTw<NN> && (NN % ColLayout<NN>::CC == 0));
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return false;
  }
}

static cudaError_t launch_adj_col_fast(const float2* Rs, const double* cturn, const double* zlist, float2* U, int W,
                                      int H, int z0, int z1, cudaStream_t st, int chunks_hint, double dz_uniform,
                                      int rec_mode) {
  if (W != H) return cudaErrorInvalidValue;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return adj_col_n<NN>(Rs, cturn, zlist, U, W, z0, z1, st, chunks_hint, dz_uniform, rec_mode);
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

static int fwd_col_chunks_fast(int W, int H, int Nz) {
  int cc = 8;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    cc = ColLayout<NN>::CC; break;
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      break;
  }
  const int strips = (W + cc - 1) / cc;
  const int target = 4 * num_sms();
  int chunks = (target + strips - 1) / strips;
  // partial spectra cost one plane of traffic each: keep them few
  if (chunks > 16) chunks = 16;
  if (chunks > Nz) chunks = Nz;
  if (chunks < 1) chunks = 1;
  return chunks;
}

template <int N>
static cudaError_t fwd_col_n(const float2* T, const double* cturn, const double* zlist, float2* Spart, int W,
                             int z0, int z1, int nchunks, cudaStream_t st, double dz_uniform, int horner_mode) {
  using Lay = ColLayout<N>;
  const int nz = z1 - z0;
  if (nz <= 0) return cudaSuccess;
  const int strips = col_strips<N>(W);
  const int zpb = (nz + nchunks - 1) / nchunks;
  const int chunks = (nz + zpb - 1) / zpb;
  cudaError_t e;
  if (chunks < nchunks) {  // unused chunk slots must read as zero
    e = cudaMemsetAsync(Spart + (size_t)chunks * N * W, 0, sizeof(float2) * (size_t)(nchunks - chunks) * N * W, st);
    if (e != cudaSuccess) return e;
  }
  if constexpr (kTableCols<N>) {
    if (dz_uniform != 0.0 && (horner_mode == 2 || horner_mode == 3)) {
      constexpr size_t smem = horner1_smem<N>();
      CUtensorMap tmap;
      std::memset(&tmap, 0, sizeof(tmap));
      // mode 3: TMA strip loads where the map can be made (square planes, column blocks that tile the row)
      const bool tma = horner_mode == 3 && W == N && (N % Lay::CC == 0) &&
                       plane_stack_map(&tmap, const_cast<float2*>(T), N, z1, Lay::CC, tma_rows<N>());
      auto go = [&](auto kern) -> cudaError_t {
        cudaError_t e2 = allow_smem(kern, smem);
        if (e2 != cudaSuccess) return e2;
        kern<<<dim3(strips, chunks), Lay::THREADS, smem, st>>>(T, cturn, zlist, dz_uniform, Spart, z0, z1, zpb, tmap);
        return cudaGetLastError();
      };
      return tma ? go(k_fwd_col_horner1<N, true>) : go(k_fwd_col_horner1<N, false>);
    }
  }
  if constexpr (Lay::STAGE && LineCfg<N>::EXACT) {
    if (dz_uniform != 0.0) {
      e = allow_smem(k_fwd_col_horner<N>, Lay::STAGE_BYTES);
      if (e != cudaSuccess) return e;
      k_fwd_col_horner<N><<<dim3(strips, chunks), Lay::THREADS, Lay::STAGE_BYTES, st>>>(T, cturn, zlist, dz_uniform,
                                                                                         Spart, z0, z1, zpb);
      return cudaGetLastError();
    }
  }
  e = allow_smem(k_fwd_col<N>, Lay::STAGE_BYTES);
  if (e != cudaSuccess) return e;
  k_fwd_col<N><<<dim3(strips, chunks), Lay::THREADS, Lay::STAGE_BYTES, st>>>(T, cturn, zlist, Spart, z0, z1, zpb);
  return cudaGetLastError();
}

bool fwd_horner_supported(int W, int H, int horner_mode) {
  if (W != H) return false;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return horner_mode >= 2 ? kTableCols<NN> : (ColLayout<NN>::STAGE && LineCfg<NN>::EXACT);
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return false;
  }
}

static cudaError_t launch_fwd_col_fast(const float2* T, const double* cturn, const double* zlist, float2* Spart,
                                      int W, int H, int z0, int z1, int nchunks, cudaStream_t st, double dz_uniform,
                                      int horner_mode) {
  if (W != H) return cudaErrorInvalidValue;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return fwd_col_n<NN>(T, cturn, zlist, Spart, W, z0, z1, nchunks, st, dz_uniform, horner_mode);
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <int N>
static cudaError_t plane_col_n(int inverse, const float2* in, float2* out, int W, float scale, cudaStream_t st) {
  using Lay = ColLayout<N>;
  const int strips = col_strips<N>(W);
  cudaError_t e;
  if (inverse) {
    e = allow_smem(k_plane_col<N, true>, Lay::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    k_plane_col<N, true><<<strips, Lay::THREADS, Lay::SMEM_BYTES, st>>>(in, out, scale);
  } else {
    e = allow_smem(k_plane_col<N, false>, Lay::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    k_plane_col<N, false><<<strips, Lay::THREADS, Lay::SMEM_BYTES, st>>>(in, out, scale);
  }
  return cudaGetLastError();
}

static cudaError_t launch_plane_col_fast(int inverse, const float2* in, float2* out, int W, int H, float scale,
                                        cudaStream_t st) {
  if (W != H) return cudaErrorInvalidValue;
  switch (H) {
#define RIHVR_CASE(NN) \
  case NN:             \
    return plane_col_n<NN>(inverse, in, out, W, scale, st);
    RIHVR_FOR_EACH_SIZE(RIHVR_CASE)
#undef RIHVR_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------------------
// sum of partial spectra (fixed order: deterministic)
// ---------------------------------------------------------------------------
__global__ void k_sum_chunks(const float2* __restrict__ Spart, int nchunks, float2* __restrict__ S, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float2 a = Spart[i];
    for (int k = 1; k < nchunks; ++k) a = cadd(a, Spart[(size_t)k * n + i]);
    S[i] = a;
  }
}

cudaError_t launch_sum_chunks(const float2* Spart, int nchunks, float2* S, long long n, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 4 * num_sms()) blocks = 4 * num_sms();
  k_sum_chunks<<<blocks, 256, 0, st>>>(Spart, nchunks, S, n);
  return cudaGetLastError();
}

struct SlabSources {
  const float2* p[kMaxSlabs];
};

__global__ void k_sum_slabs(SlabSources s, int n, float2* __restrict__ dst, long long count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    float2 a = s.p[0][i];
    for (int k = 1; k < n; ++k) a = cadd(a, s.p[k][i]);
    dst[i] = a;
  }
}

cudaError_t launch_sum_slabs(const float2* const* src, int n, float2* dst, long long count, cudaStream_t st) {
  if (n < 1 || n > kMaxSlabs) return cudaErrorInvalidValue;
  SlabSources s{};
  for (int k = 0; k < n; ++k) s.p[k] = src[k];
  int blocks = (int)((count + 255) / 256);
  if (blocks > 4 * num_sms()) blocks = 4 * num_sms();
  k_sum_slabs<<<blocks, 256, 0, st>>>(s, n, dst, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// block reduction of kNumSums doubles into partials[block]
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void block_write_sums(double (&acc)[kNumSums], double* partials, int block) {
  __shared__ double red[NT / 32][kNumSums];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) {
    double v = warp_sum(acc[k]);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNumSums) {
    double s = 0;
    for (int w = 0; w < NT / 32; ++w) s += red[w][threadIdx.x];
    partials[(size_t)block * kNumSums + threadIdx.x] = s;
  }
}

// Restart statistic weights: sparse_fistaRestart_kernel<512> (RIHVR
// sparse_compressive_holo.cu:4393-4432) overwrites the second element's real
// product with its imaginary one and re-adds the first element's imaginary
// product (:4411-4413): within each 1024-element chunk of a plane, elements
// 0..511 count Re + 2 Im and elements 512..1023 count Im only.
__device__ __forceinline__ void restart_w(size_t e, int faithful, float* wr, float* wi) {
  if (!faithful) {
    *wr = 1.f;
    *wi = 1.f;
  } else if ((e & 1023u) < 512u) {
    *wr = 1.f;
    *wi = 2.f;
  } else {
    *wr = 0.f;
    *wi = 1.f;
  }
}

// Soft thresholds: block_soft_threshold_kernel (sparse_compressive_holo.cu:
// 3065-3110) shrinks Re and Im separately; the non-faithful variant shrinks
// the complex modulus.
__device__ __forceinline__ float2 shrink(float2 v, float T, int faithful) {
  if (T <= 0.f) return v;
  if (faithful) {
    const float mr = fabsf(v.x) - T, mi = fabsf(v.y) - T;
    return make_float2(mr > 0.f ? copysignf(mr, v.x) : 0.f, mi > 0.f ? copysignf(mi, v.y) : 0.f);
  }
  const float a = sqrtf(v.x * v.x + v.y * v.y);
  if (a <= T) return make_float2(0.f, 0.f);
  const float f = (a - T) / a;
  return make_float2(v.x * f, v.y * f);
}

__device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// The prox arguments with the step and momentum scalars taken from their
// device copy when one is given (captured launches, see ProxArgs::dscal).
__device__ __forceinline__ ProxArgs resolve_scalars(const ProxArgs& a0) {
  ProxArgs a = a0;
  if (a0.dscal) {
    a.beta = __ldg(a0.dscal + 0);
    a.t = __ldg(a0.dscal + 1);
    a.mu = __ldg(a0.dscal + 2);
    a.s = __ldg(a0.dscal + 3);
    a.thr = __ldg(a0.dscal + 4);
  }
  return a;
}

// Square roots of the objective's norm terms (L1 and TV sums) use the
// hardware approximation (PTX sqrt.approx.f32, one instruction): they only
// feed the reported objective, summed over millions of voxels in FP64.
__device__ __forceinline__ float norm_sqrt(float q) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(q));
  return r;
}

// ---------------------------------------------------------------------------
// Fused 2-D TV prox (mode 7): proximalFusedLasso2d, sparse_compressive_holo.cu:
// 3652-3732 with kernels :3478-3597.  Per plane tile, with the momentum point
// formed on the fly:
//   x = P + beta (P - Pprev);  xh = x - t g
//   gx = gy = 0; n_tv times: y = xh - mu div(g);  g = (g + s grad y)/max(1, |.|)
//   y = xh - mu div(g);  p = shrink(y, thr)
// div uses forward periodic differences, grad backward periodic differences and
// the projection norm is taken over the four real components (Jacobi updates,
// as the reference's two kernels per iteration).
//
// Layout: a block holds a 64 x 64 tile (columns x rows) with a recomputed halo
// of n_tv + 1 pixels on every side, which makes the interior exact.  Warp w owns
// rows [8w, 8w+8); lane l owns columns 2l and 2l+1.  The Chambolle state (xh, gx,
// gy) stays in registers; each TV iteration sweeps a thread's 8 rows top to
// bottom so that y is only ever live for one row, right neighbours of gx and
// left neighbours of y move by warp shuffles, and only the first/last row of
// each warp's run crosses warps, through double-buffered shared memory (one
// barrier per iteration).  The row above a run is recomputed from the published
// last row of the warp above instead of being waited for.
// The final sweep also accumulates the line-search sums, the restart statistic
// and (optionally) the L1/TV norms of p and x.
// ---------------------------------------------------------------------------
constexpr int TV_CPL = 2;                  // columns per lane
constexpr int TV_EW = 32 * TV_CPL;         // tile width incl. halo
constexpr int TV_R = 8;                    // rows per thread
constexpr int TV_NW = 8;                   // warps, stacked vertically
constexpr int TV_EH = TV_NW * TV_R;        // tile height incl. halo
constexpr int TV_THREADS = 32 * TV_NW;
constexpr int TV_BND = TV_NW * TV_EW;      // one boundary row per warp
constexpr size_t TV_SMEM = sizeof(float2) * (2 * TV_EH * TV_EW + 3 * 2 * TV_BND + TV_BND);

__device__ __forceinline__ float2 shfl_down2(float2 v) {
  return make_float2(__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1));
}
__device__ __forceinline__ float2 shfl_up2(float2 v) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}

// y = xh - mu ((gxr - gx) + (gyd - gy)), packed: nmu = (-mu, -mu)
__device__ __forceinline__ float2 tv_estimate(float2 xh, float2 gx, float2 gxr, float2 gy, float2 gyd, float2 nmu) {
  return f2fma(nmu, f2add(f2sub(gxr, gx), f2sub(gyd, gy)), xh);
}

// hardware reciprocal square root (PTX rsqrt.approx.f32), one instruction
// wherever it is inlined
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// g = P(g + s grad y) for one pixel: px = gx + s (yl - y), py = gy + s (yu - y),
// divided by max(1, |(px, py)|) over the four real components.
__device__ __forceinline__ void tv_dual(float2& gx, float2& gy, float2 y, float2 yl, float2 yu, float2 s2) {
  const float2 px = f2fma(s2, f2sub(yl, y), gx);
  const float2 py = f2fma(s2, f2sub(yu, y), gy);
  const float2 q = f2fma(py, py, f2mul(px, px));
  const float n2 = q.x + q.y;
  // 1 / max(1, sqrt(n2)) as min(1, rsqrt(n2)): one instruction instead of a
  // compare and a select (n2 = 0 gives rsqrt = inf, hence 1)
  const float sc = fminf(1.f, rsqrt_approx(n2));
  const float2 sc2 = make_float2(sc, sc);
  gx = f2mul(px, sc2);
  gy = f2mul(py, sc2);
}

// wrap an index that lies within one period of [0, n)
__device__ __forceinline__ int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

template <typename ST>
struct Pair;  // two adjacent complex values in storage layout
template <>
struct Pair<float2> {
  using T = float4;
  static __device__ __forceinline__ void ld(const float2* p, float2& a, float2& b) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  }
};
template <>
struct Pair<__nv_bfloat162> {
  static __device__ __forceinline__ void ld(const __nv_bfloat162* p, float2& a, float2& b) {
    const uint2 v = *reinterpret_cast<const uint2*>(p);
    a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
    b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
  }
};
template <>
struct Pair<__half2> {
  static __device__ __forceinline__ void ld(const __half2* p, float2& a, float2& b) {
    const uint2 v = *reinterpret_cast<const uint2*>(p);
    a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
  }
};

template <typename ST>
__global__ void __launch_bounds__(TV_THREADS, 2) k_prox_tv2d(ProxArgs a0) {
  const ProxArgs a = resolve_scalars(a0);
  static_assert(TV_CPL == 2, "paired loads assume two columns per lane");
  extern __shared__ float2 smem[];
  float2* s_g = smem;                      // [EH][EW] gradient at load
  float2* s_P = s_g + TV_EH * TV_EW;       // [EH][EW] P at load
  float2* s_gyf = s_P + TV_EH * TV_EW;     // [2][NW][EW] first-row gy of each run
  float2* s_gxl = s_gyf + 2 * TV_BND;      // [2][NW][EW] last-row gx
  float2* s_gyl = s_gxl + 2 * TV_BND;      // [2][NW][EW] last-row gy
  float2* s_xhl = s_gyl + 2 * TV_BND;      // [NW][EW]   last-row xh
  const int W = a.W, H = a.H;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int h = a.n_tv + 1, VW = TV_EW - 2 * h, VH = TV_EH - 2 * h;
  const int ox = blockIdx.x * VW - h, oy = blockIdx.y * VH - h;
  const size_t plane = (size_t)blockIdx.z * W * H;
  const ST* P = static_cast<const ST*>(a.P) + plane;
  const ST* Pp = static_cast<const ST*>(a.Pprev) + plane;
  const float2* G = a.G + plane;
  const float t = a.t, beta = a.beta;
  const float2 nmu = make_float2(-a.mu, -a.mu), s2 = make_float2(a.s, a.s);
  const int col0 = lane * TV_CPL;
  // tiles are at most one period outside the plane when it is at least as
  // large as a tile; smaller planes wrap several times
  const bool small = (W < TV_EW) || (H < TV_EH);
  // adjacent column pairs are contiguous and 16-byte aligned when the tile
  // origin is even (the plane side is even)
  const bool paired = !small && ((ox & 1) == 0);

  float2 xh[TV_R][TV_CPL], gx[TV_R][TV_CPL], gy[TV_R][TV_CPL];
  int gc[TV_CPL];
#pragma unroll
  for (int c = 0; c < TV_CPL; ++c) gc[c] = small ? ((ox + col0 + c) % W + W) % W : wrap1(ox + col0 + c, W);
#pragma unroll
  for (int i = 0; i < TV_R; ++i) {
    const int row = w * TV_R + i;
    const int gr = small ? ((oy + row) % H + H) % H : wrap1(oy + row, H);
    const size_t rbase = (size_t)gr * W;
    float2 p[TV_CPL], pp[TV_CPL], g[TV_CPL];
    if (paired) {
      Pair<ST>::ld(P + rbase + gc[0], p[0], p[1]);
      Pair<ST>::ld(Pp + rbase + gc[0], pp[0], pp[1]);
      Pair<float2>::ld(G + rbase + gc[0], g[0], g[1]);
    } else {
#pragma unroll
      for (int c = 0; c < TV_CPL; ++c) {
        p[c] = Store<ST>::ld(P + rbase + gc[c]);
        pp[c] = Store<ST>::ld(Pp + rbase + gc[c]);
        g[c] = G[rbase + gc[c]];
      }
    }
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) {
      const float2 x = f2fma(make_float2(beta, beta), f2sub(p[c], pp[c]), p[c]);
      xh[i][c] = f2fma(make_float2(-t, -t), g[c], x);
      gx[i][c] = make_float2(0.f, 0.f);
      gy[i][c] = make_float2(0.f, 0.f);
    }
    *reinterpret_cast<float4*>(s_g + row * TV_EW + col0) = make_float4(g[0].x, g[0].y, g[1].x, g[1].y);
    *reinterpret_cast<float4*>(s_P + row * TV_EW + col0) = make_float4(p[0].x, p[0].y, p[1].x, p[1].y);
  }
#pragma unroll
  for (int c = 0; c < TV_CPL; ++c) s_xhl[w * TV_EW + col0 + c] = xh[TV_R - 1][c];

  for (int k = 0; k < a.n_tv; ++k) {
    float2* gyf = s_gyf + (k & 1) * TV_BND;
    float2* gxl = s_gxl + (k & 1) * TV_BND;
    float2* gyl = s_gyl + (k & 1) * TV_BND;
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) {
      gyf[w * TV_EW + col0 + c] = gy[0][c];
      gxl[w * TV_EW + col0 + c] = gx[TV_R - 1][c];
      gyl[w * TV_EW + col0 + c] = gy[TV_R - 1][c];
    }
    __syncthreads();
    // y of the row above this run, recomputed from the published last row of warp w-1
    float2 yu[TV_CPL];
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) {
      yu[c] = make_float2(0.f, 0.f);  // top halo rows: value irrelevant
      if (w > 0) {
        const int col = col0 + c, b = (w - 1) * TV_EW;
        const float2 gxu = gxl[b + col], gyu = gyl[b + col];
        const float2 gxru = (col + 1 < TV_EW) ? gxl[b + col + 1] : gxu;
        yu[c] = tv_estimate(s_xhl[b + col], gxu, gxru, gyu, gy[0][c], nmu);
      }
    }
#pragma unroll
    for (int i = 0; i < TV_R; ++i) {
      float2 gxr[TV_CPL], gyd[TV_CPL], y[TV_CPL], yl[TV_CPL];
#pragma unroll
      for (int c = 0; c < TV_CPL - 1; ++c) gxr[c] = gx[i][c + 1];
      gxr[TV_CPL - 1] = shfl_down2(gx[i][0]);  // lane 31 gets its own (halo column)
#pragma unroll
      for (int c = 0; c < TV_CPL; ++c) {
        if (i < TV_R - 1) gyd[c] = gy[i + 1][c];
        else gyd[c] = (w < TV_NW - 1) ? gyf[(w + 1) * TV_EW + col0 + c] : gy[i][c];
        y[c] = tv_estimate(xh[i][c], gx[i][c], gxr[c], gy[i][c], gyd[c], nmu);
      }
      yl[0] = shfl_up2(y[TV_CPL - 1]);  // lane 0 gets its own (halo column)
#pragma unroll
      for (int c = 1; c < TV_CPL; ++c) yl[c] = y[c - 1];
#pragma unroll
      for (int c = 0; c < TV_CPL; ++c) {
        tv_dual(gx[i][c], gy[i][c], y[c], yl[c], yu[c], s2);
        yu[c] = y[c];
      }
    }
  }

  // final estimate and shrink: p replaces gx in registers
  {
    float2* gyf = s_gyf + (a.n_tv & 1) * TV_BND;
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) gyf[w * TV_EW + col0 + c] = gy[0][c];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < TV_R; ++i) {
      float2 gxr[TV_CPL];
#pragma unroll
      for (int c = 0; c < TV_CPL - 1; ++c) gxr[c] = gx[i][c + 1];
      gxr[TV_CPL - 1] = shfl_down2(gx[i][0]);
#pragma unroll
      for (int c = 0; c < TV_CPL; ++c) {
        float2 gyd;
        if (i < TV_R - 1) gyd = gy[i + 1][c];
        else gyd = (w < TV_NW - 1) ? gyf[(w + 1) * TV_EW + col0 + c] : gy[i][c];
        const float2 y = tv_estimate(xh[i][c], gx[i][c], gxr[c], gy[i][c], gyd, nmu);
        gx[i][c] = shrink(y, a.thr, a.faithful);
      }
    }
  }
  // last-row p and x of each run for the TV norms of the run below
  float2* pl_last = s_gxl;  // reused: no TV reads remain
  float2* xl_last = s_gyl;
  const float2 t2 = make_float2(t, t);
  if (a.want_norms) {
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) {
      const int col = col0 + c;
      const float2 g = s_g[(w * TV_R + TV_R - 1) * TV_EW + col];
      pl_last[w * TV_EW + col] = gx[TV_R - 1][c];
      xl_last[w * TV_EW + col] = f2fma(t2, g, xh[TV_R - 1][c]);
    }
  }
  __syncthreads();

  // per-thread FP32 partials over at most 16 pixels, FP64 from there on
  float acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.f;
  ST* Pn = static_cast<ST*>(a.Pnew) + plane;
  float2 pu[TV_CPL], xu[TV_CPL];
#pragma unroll
  for (int c = 0; c < TV_CPL; ++c) {
    pu[c] = make_float2(0.f, 0.f);
    xu[c] = make_float2(0.f, 0.f);
    if (w > 0 && a.want_norms) {
      pu[c] = pl_last[(w - 1) * TV_EW + col0 + c];
      xu[c] = xl_last[(w - 1) * TV_EW + col0 + c];
    }
  }
#pragma unroll
  for (int i = 0; i < TV_R; ++i) {
    const int row = w * TV_R + i;
    const int grow = oy + row;
    const bool row_ok = row >= h && row < h + VH && grow < H;
    float2 x[TV_CPL], pl[TV_CPL], xl[TV_CPL], g[TV_CPL], y0[TV_CPL];
    {
      const float4 gv = *reinterpret_cast<const float4*>(s_g + row * TV_EW + col0);
      const float4 pv = *reinterpret_cast<const float4*>(s_P + row * TV_EW + col0);
      g[0] = make_float2(gv.x, gv.y);
      g[1] = make_float2(gv.z, gv.w);
      y0[0] = make_float2(pv.x, pv.y);
      y0[1] = make_float2(pv.z, pv.w);
    }
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) x[c] = f2fma(t2, g[c], xh[i][c]);
    pl[0] = shfl_up2(gx[i][TV_CPL - 1]);
    xl[0] = shfl_up2(x[TV_CPL - 1]);
#pragma unroll
    for (int c = 1; c < TV_CPL; ++c) {
      pl[c] = gx[i][c - 1];
      xl[c] = x[c - 1];
    }
#pragma unroll
    for (int c = 0; c < TV_CPL; ++c) {
      const int col = col0 + c, gcl = ox + col;
      const float2 p = gx[i][c];
      if (row_ok && col >= h && col < h + VW && gcl < W) {
        const size_t e = (size_t)grow * W + gcl;
        Store<ST>::st(Pn + e, p);
        const float2 d = f2sub(p, x[c]);
        const float2 dg = f2mul(d, g[c]);
        acc[SUM_LIM1] += dg.x + dg.y;
        acc[SUM_LIM2] += cabs2(d);
        float wr, wi;
        restart_w(e, a.faithful, &wr, &wi);
        const float2 uv = f2mul(f2sub(x[c], p), f2sub(p, y0[c]));
        acc[SUM_RS] += fmaf(wr, uv.x, wi * uv.y);
        if (a.want_norms) {
          acc[SUM_L1P] += norm_sqrt(cabs2(p));
          acc[SUM_TVP] += norm_sqrt(cabs2(f2sub(pl[c], p)) + cabs2(f2sub(pu[c], p)));
          acc[SUM_L1X] += norm_sqrt(cabs2(x[c]));
          acc[SUM_TVX] += norm_sqrt(cabs2(f2sub(xl[c], x[c])) + cabs2(f2sub(xu[c], x[c])));
        }
      }
      pu[c] = p;
      xu[c] = x[c];
    }
  }
  double dacc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) dacc[k] = (double)acc[k];
  const int blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  block_write_sums<TV_THREADS>(dacc, a.partials, blk);
}

template <typename ST>
struct Raw2;  // two adjacent complex values as loaded from storage
template <>
struct Raw2<float2> {
  using T = float4;
  static __device__ __forceinline__ T ld(const float2* p) { return *reinterpret_cast<const float4*>(p); }
  static __device__ __forceinline__ void cvt(T v, float2& a, float2& b) {
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  }
  static __device__ __forceinline__ void st(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
  }
};
template <>
struct Raw2<__nv_bfloat162> {
  using T = uint2;
  static __device__ __forceinline__ T ld(const __nv_bfloat162* p) { return *reinterpret_cast<const uint2*>(p); }
  static __device__ __forceinline__ void cvt(T v, float2& a, float2& b) {
    a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.x));
    b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v.y));
  }
  static __device__ __forceinline__ void st(__nv_bfloat162* p, float2 a, float2 b) {
    const __nv_bfloat162 u = __float22bfloat162_rn(a), v = __float22bfloat162_rn(b);
    *reinterpret_cast<uint2*>(p) =
        make_uint2(*reinterpret_cast<const unsigned*>(&u), *reinterpret_cast<const unsigned*>(&v));
  }
};
template <>
struct Raw2<__half2> {
  using T = uint2;
  static __device__ __forceinline__ T ld(const __half2* p) { return *reinterpret_cast<const uint2*>(p); }
  static __device__ __forceinline__ void cvt(T v, float2& a, float2& b) {
    a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
  }
  static __device__ __forceinline__ void st(__half2* p, float2 a, float2 b) {
    const __half2 u = __float22half2_rn(a), v = __float22half2_rn(b);
    *reinterpret_cast<uint2*>(p) =
        make_uint2(*reinterpret_cast<const unsigned*>(&u), *reinterpret_cast<const unsigned*>(&v));
  }
};

struct TvsGrid {
  int nstrips, nseg, seg_len;
};

// ---------------------------------------------------------------------------
// Streaming form of the same prox (1 <= n_tv <= 10), the default.  The tiled
// kernel above recomputes a halo of n_tv + 1 rows and columns around every
// 64 x 64 tile, so a third of its work is thrown away, and it needs a block
// barrier per TV iteration.  Here a lane owns CPL adjacent columns and a warp a
// strip of 32 CPL columns with an x halo of HX (n_tv + 1 rounded up to a
// multiple of CPL) on each side; the warp walks a run of rows with the n_tv
// Chambolle iterations pipelined one row apart: at the step that loads row j,
// iteration k updates row j - k from iteration k-1's rows j-k (kept from the
// previous step) and j-k+1 (produced this step), and the final estimate and
// shrink produce row j - n_tv - 1.  A run starts 2 (n_tv + 1) rows early
// (periodic wrap) so that its first output row is exact, which removes the y
// halo.  Warps are independent and exchange x neighbours by shuffles only.
//
// Per lane, the state is one row of (gx, gy) and one row of y per iteration in
// registers.  Rows arrive one step ahead by cp.async into a per-lane ring of D
// rows in shared memory holding (raw Pprev, overwritten by xh), G and raw P;
// each lane reads back only what it copied, so no barrier is involved.
// Iteration 1 starts from g = 0, where the estimate is xh itself.  The
// arithmetic is the tiled kernel's operation for operation, so P_new has the
// same bits; the sums differ only in summation order.
//
// The step loop is unrolled by four (by two it needs 10% more instructions; by
// eight the loop body outgrows the instruction cache).  With a step count that
// is not a multiple of the unroll factor, unrolled builds gave the last row of a
// run 1 ulp away from the tiled kernel, so runs start up to three rows earlier
// and every run has a multiple of four steps.
// ---------------------------------------------------------------------------
template <int NTV, int CPL>
struct TvwShape {
  static constexpr int h = NTV + 1;
  static constexpr int AL = CPL < 2 ? 2 : CPL;
  static constexpr int HX = (h + AL - 1) / AL * AL;   // keeps each lane's columns aligned
  static constexpr int SW = 32 * CPL;                 // strip width
  static constexpr int VW = SW - 2 * HX;              // valid columns per strip
  static constexpr int D = (h + 2 <= 8) ? 8 : 16;     // rows in use: h + 1, plus one landing
  static constexpr int F4 = CPL / 2;                  // float4 per array per lane row (FP32)
  static constexpr int SLOT = 3 * F4 * 32;            // float4 per ring slot, whole warp
  // Two warps per block.  Without the objective's norm terms and with the
  // 8-row ring (n_tv <= 5), the kernel fits 128 registers with at most a few
  // bytes of spill, and 8 blocks (16 warps) share an SM; the norm terms need
  // about 160 registers, which caps them at 6 blocks (12 warps).  At
  // 1024 x 1024 x 1000 (n_tv = 5, no norm terms) a launch took 10.42 ms with
  // 4-warp blocks at 12 warps per SM, 9.5 ms with 2-warp blocks at 16.
  static constexpr int NW = 2;
  static constexpr size_t SMEM = sizeof(float4) * (size_t)SLOT * D * NW;
  static_assert(CPL == 2 || CPL == 4, "columns per lane");
  static_assert(VW > 0, "halo wider than the strip");
};

// Blocks per SM the register allocation targets (__launch_bounds__).  At 7
// two-warp blocks ptxas caps the kernel at 128 registers (8 blocks then fit,
// as registers are split per scheduler); asking for 8 gives the same cap with
// ten times the spill.
template <int NTV, bool NORMS>
constexpr int tvw_minb() {
  return TvwShape<NTV, 2>::D == 8 ? (NORMS ? 6 : 7) : 4;
}

// copy CPL complex values in storage type (16-byte aligned source for
// CPL * sizeof(ST) >= 16, else 8-byte aligned) to shared memory
template <typename ST, int CPL>
__device__ __forceinline__ void cp_async_run(float4* smem, const ST* gmem) {
  constexpr int BYTES = CPL * (int)sizeof(ST);
  if constexpr (BYTES >= 16) {
#pragma unroll
    for (int k = 0; k < BYTES / 16; ++k) {
      const unsigned d = (unsigned)__cvta_generic_to_shared(smem + k * 32);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d),
                   "l"(reinterpret_cast<const char*>(gmem) + 16 * k)
                   : "memory");
    }
  } else {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gmem) : "memory");
  }
}

// CPL complex values of storage type ST from their ring copy (16-byte pieces
// 32 float4 apart)
template <typename ST, int CPL>
__device__ __forceinline__ void ring_vals(const float4* e, float2 (&v)[CPL]) {
  if constexpr (sizeof(ST) == 8) {
#pragma unroll
    for (int k = 0; k < CPL / 2; ++k) {
      const float4 f = e[k * 32];
      v[2 * k] = make_float2(f.x, f.y);
      v[2 * k + 1] = make_float2(f.z, f.w);
    }
  } else {
#pragma unroll
    for (int k = 0; k < (CPL + 3) / 4; ++k) {
      const float4 f = e[k * 32];
      const unsigned u[4] = {__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z), __float_as_uint(f.w)};
#pragma unroll
      for (int j = 0; j < 4 && 4 * k + j < CPL; ++j) {
        float2 a, b;
        Raw2<ST>::cvt(make_uint2(u[j], 0u), a, b);
        v[4 * k + j] = a;
      }
    }
  }
}

template <typename ST, int CPL>
__device__ __forceinline__ void store_run(ST* p, const float2 (&v)[CPL]) {
#pragma unroll
  for (int c = 0; c < CPL; c += 2) Raw2<ST>::st(p + c, v[c], v[c + 1]);
}

template <typename ST, int NTV, bool NORMS, int CPL = 2, int NW = TvwShape<NTV, CPL>::NW,
          int MINB = tvw_minb<NTV, NORMS>(), int UNR = 4, int PADTO = 4, int PART = 0>
__global__ void __launch_bounds__(32 * NW, MINB) k_prox_tv2d_strip(ProxArgs a0, TvsGrid gr) {
  const ProxArgs a = resolve_scalars(a0);
  using Sh = TvwShape<NTV, CPL>;
  constexpr int h = Sh::h, HX = Sh::HX, VW = Sh::VW, D = Sh::D, RM = D - 1, F4 = Sh::F4;
  constexpr int QS = F4 * 32;     // float4 between the arrays of a slot
  constexpr int SL = 3 * QS;      // float4 per slot
  static_assert(PART == 0 || CPL == 2, "the two-part forms move a lane's two columns as one float4");
  extern __shared__ float4 tvw_ring[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float4* ring = tvw_ring + (size_t)w * SL * D + lane;
  // second part: 2 rows of the stored duals (gx pair, gy pair) after the warps' rings
  float4* gring = tvw_ring + (size_t)NW * SL * D + (size_t)w * 2 * 32 * 2 + lane;
  const int W = a.W, H = a.H;
  const long long work = (long long)blockIdx.x * NW + w;
  const long long nwork = (long long)gr.nstrips * gr.nseg * a.Nz;

  double dacc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) dacc[k] = 0.0;

  if (work < nwork) {
    const int strip = (int)(work % gr.nstrips);
    const long long rest = work / gr.nstrips;
    const int seg = (int)(rest % gr.nseg);
    const size_t plane = (size_t)(rest / gr.nseg) * W * H;
    const ST* P = static_cast<const ST*>(a.P) + plane;
    const ST* Pp = static_cast<const ST*>(a.Pprev) + plane;
    const float2* G = a.G + plane;
    ST* Pn = static_cast<ST*>(a.Pnew) + plane;
    const float t = a.t, beta = a.beta;
    const float2 nmu = make_float2(-a.mu, -a.mu), s2 = make_float2(a.s, a.s);
    const float2 bb = make_float2(beta, beta), nt2 = make_float2(-t, -t), t2 = make_float2(t, t);
    const float2 z2 = make_float2(0.f, 0.f);
    const float thr = a.thr;
    const int faithful = a.faithful;
    constexpr int NS = NORMS ? kNumSums : SUM_RS + 1;  // sums this kernel accumulates

    const int cu = strip * VW - HX + CPL * lane;   // first column of this lane, unwrapped
    const int gc = ((cu % W) + W) % W;             // a multiple of CPL; W is one too
    const bool lane_ok = (CPL * lane >= HX) && (CPL * lane < HX + VW) && (cu < W);
    const int r0 = seg * gr.seg_len;
    const int r1 = min(H, r0 + gr.seg_len);
    // runs start up to PADTO - 1 rows earlier so that the step count is a
    // multiple of PADTO (the unroll factor)
    const int pad = (PADTO - ((r1 - r0 + 2 * h) % PADTO)) % PADTO;
    const int nsteps = (r1 - r0) + 2 * h + pad;
    // the warm-up may reach back more than one plane height on short planes
    int lrow = ((r0 - h - pad) % H + H) % H;
    int orow = ((r0 - 2 * h - pad) % H + H) % H;

    // Ring slots are read as rows above r0 - h before any copy lands there;
    // those rows only feed rows above r0, which are not written.
    // the first part's duals on row `off` (second part): a 2-row ring, so
    // the copy for the next step is issued once this step has read its rows
    auto request_g = [&](size_t off, int step) {
      if constexpr (PART == 2) {
        float4* gslot = gring + (step & 1) * 2 * 32;
        cp_async_run<float2, CPL>(gslot, a.gdx + plane + off);
        cp_async_run<float2, CPL>(gslot + 32, a.gdy + plane + off);
        cp_async_commit();
      }
    };
    size_t goff = 0;  // row offset of the last main-ring request
    auto request = [&](int slot) {
      const size_t off = (size_t)lrow * W + gc;
      float4* e = ring + slot * SL;
      cp_async_run<ST, CPL>(e, Pp + off);
      cp_async_run<float2, CPL>(e + QS, G + off);
      cp_async_run<ST, CPL>(e + 2 * QS, P + off);
      cp_async_commit();
      goff = off;
      lrow = (lrow + 1 == H) ? 0 : lrow + 1;
    };
    request(0);
    request_g(goff, 0);

    float2 gX[NTV][CPL], gY[NTV][CPL], yU[NTV][CPL];
#pragma unroll
    for (int k = 0; k < NTV; ++k)
#pragma unroll
      for (int c = 0; c < CPL; ++c) gX[k][c] = gY[k][c] = yU[k][c] = z2;
    float2 pu[CPL], xu[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) pu[c] = xu[c] = z2;
    float acc[kNumSums];
#pragma unroll
    for (int k = 0; k < kNumSums; ++k) acc[k] = 0.f;

#pragma unroll UNR
    for (int i = 0; i < nsteps; ++i) {
      cp_async_wait<0>();
      // stage 0: xh = P + beta (P - Pprev) - t G replaces Pprev in the slot
      {
        float4* e = ring + (i & RM) * SL;
        float2 p[CPL], q[CPL], g[CPL];
        ring_vals<ST, CPL>(e + 2 * QS, p);
        ring_vals<ST, CPL>(e, q);
        ring_vals<float2, CPL>(e + QS, g);
#pragma unroll
        for (int k = 0; k < F4; ++k) {
          const float2 xa = f2fma(nt2, g[2 * k], f2fma(bb, f2sub(p[2 * k], q[2 * k]), p[2 * k]));
          const float2 xb = f2fma(nt2, g[2 * k + 1], f2fma(bb, f2sub(p[2 * k + 1], q[2 * k + 1]), p[2 * k + 1]));
          e[k * 32] = make_float4(xa.x, xa.y, xb.x, xb.y);
        }
      }
      if (i + 1 < nsteps) request((i + 1) & RM);

      float2 ny[CPL];   // gy of the iteration before, on the row below
      // iteration 1 on row j-1: g^0 = 0, so the estimate is xh itself; in the
      // second part g^0 is the first part's dual, loaded with the rows
      {
        float2 y[CPL], yl[CPL], g0x[CPL], g0y[CPL];
        ring_vals<float2, CPL>(ring + ((i - 1) & RM) * SL, y);
        if constexpr (PART == 2) {
          float2 g1y[CPL], gxr[CPL];
          const float4* gp = gring + ((i - 1) & 1) * 2 * 32;  // row j-1
          const float4* gq = gring + (i & 1) * 2 * 32;        // row j
          ring_vals<float2, CPL>(gp, g0x);
          ring_vals<float2, CPL>(gp + 32, g0y);
          ring_vals<float2, CPL>(gq + 32, g1y);
#pragma unroll
          for (int c = 0; c < CPL - 1; ++c) gxr[c] = g0x[c + 1];
          gxr[CPL - 1] = shfl_down2(g0x[0]);
#pragma unroll
          for (int c = 0; c < CPL; ++c) y[c] = tv_estimate(y[c], g0x[c], gxr[c], g0y[c], g1y[c], nmu);
          // row j-1's values have been used, so its slot is free: the next
          // step's row goes there
          if (i + 1 < nsteps) request_g(goff, i + 1);
        } else {
#pragma unroll
          for (int c = 0; c < CPL; ++c) g0x[c] = g0y[c] = z2;
        }
        yl[0] = shfl_up2(y[CPL - 1]);
#pragma unroll
        for (int c = 1; c < CPL; ++c) yl[c] = y[c - 1];
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          float2 gx = g0x[c], gy = g0y[c];
          tv_dual(gx, gy, y[c], yl[c], yU[0][c], s2);
          yU[0][c] = y[c];
          ny[c] = gy;
          // the new row replaces the one above it, which moves to (y, yl)
          const float2 ogx = gX[0][c], ogy = gY[0][c];
          gX[0][c] = gx;
          gY[0][c] = gy;
          y[c] = ogx;
          yl[c] = ogy;
        }
        // from here (y, yl) carry the previous iteration's (gx, gy) on the
        // row the next stage works on
#pragma unroll
        for (int L = 1; L <= NTV; ++L) {
          // stage L+1 (iteration L+1, or the final stage when L == NTV) on row j-1-L
          const float4* e = ring + ((i - 1 - L) & RM) * SL;
          float2 xh[CPL];
          ring_vals<float2, CPL>(e, xh);
          float2 gxr[CPL], yy[CPL];
#pragma unroll
          for (int c = 0; c < CPL - 1; ++c) gxr[c] = y[c + 1];
          gxr[CPL - 1] = shfl_down2(y[0]);
#pragma unroll
          for (int c = 0; c < CPL; ++c) yy[c] = tv_estimate(xh[c], y[c], gxr[c], yl[c], ny[c], nmu);
          if (L < NTV) {
            float2 yls[CPL];
            yls[0] = shfl_up2(yy[CPL - 1]);
#pragma unroll
            for (int c = 1; c < CPL; ++c) yls[c] = yy[c - 1];
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
              float2 gx = y[c], gy = yl[c];
              tv_dual(gx, gy, yy[c], yls[c], yU[L][c], s2);
              yU[L][c] = yy[c];
              ny[c] = gy;
              const float2 ogx = gX[L][c], ogy = gY[L][c];
              gX[L][c] = gx;
              gY[L][c] = gy;
              y[c] = ogx;
              yl[c] = ogy;
            }
          } else if constexpr (PART == 1) {
            // first part: (y, yl) hold this kernel's last dual on row j - h; it
            // goes to memory for the second part instead of the estimate
            if (i >= 2 * h + pad && lane_ok) {
              const size_t eo = plane + (size_t)orow * W + gc;
              *reinterpret_cast<float4*>(a.gdx + eo) = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
              *reinterpret_cast<float4*>(a.gdy + eo) = make_float4(yl[0].x, yl[0].y, yl[1].x, yl[1].y);
            }
          } else {
            // final stage: p = shrink(estimate) on row j - h, then the sums
            float2 p[CPL], x[CPL], g[CPL], y0[CPL];
            ring_vals<float2, CPL>(e + QS, g);
            ring_vals<ST, CPL>(e + 2 * QS, y0);
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
              p[c] = shrink(yy[c], thr, faithful);
              x[c] = f2fma(t2, g[c], xh[c]);
            }
            if (i >= 2 * h + pad) {  // row orow is exact
              float2 pl0 = z2, xl0 = z2;
              if (NORMS) {
                pl0 = shfl_up2(p[CPL - 1]);
                xl0 = shfl_up2(x[CPL - 1]);
              }
              if (lane_ok) {
                const size_t eo = (size_t)orow * W + gc;
                store_run<ST, CPL>(Pn + eo, p);
                float wr, wi;
                restart_w(eo, faithful, &wr, &wi);
#pragma unroll
                for (int c = 0; c < CPL; ++c) {
                  const float2 d = f2sub(p[c], x[c]);
                  const float2 dg = f2mul(d, g[c]);
                  acc[SUM_LIM1] += dg.x + dg.y;
                  acc[SUM_LIM2] += cabs2(d);
                  const float2 uv = f2mul(f2sub(x[c], p[c]), f2sub(p[c], y0[c]));
                  acc[SUM_RS] += fmaf(wr, uv.x, wi * uv.y);
                  if (NORMS) {
                    const float2 pl = c ? p[c - 1] : pl0, xl = c ? x[c - 1] : xl0;
                    acc[SUM_L1P] += norm_sqrt(cabs2(p[c]));
                    acc[SUM_TVP] += norm_sqrt(cabs2(f2sub(pl, p[c])) + cabs2(f2sub(pu[c], p[c])));
                    acc[SUM_L1X] += norm_sqrt(cabs2(x[c]));
                    acc[SUM_TVX] += norm_sqrt(cabs2(f2sub(xl, x[c])) + cabs2(f2sub(xu[c], x[c])));
                  }
                }
              }
              if (((i - 2 * h - pad) & 7) == 7) {  // FP32 partials over at most 8 rows
#pragma unroll
                for (int k = 0; k < NS; ++k) {
                  dacc[k] += (double)acc[k];
                  acc[k] = 0.f;
                }
              }
            }
            if (NORMS) {
#pragma unroll
              for (int c = 0; c < CPL; ++c) {
                pu[c] = p[c];
                xu[c] = x[c];
              }
            }
          }
        }
      }
      orow = (orow + 1 == H) ? 0 : orow + 1;
    }
    cp_async_wait<0>();
#pragma unroll
    for (int k = 0; k < NS; ++k) dacc[k] += (double)acc[k];
  }
  if constexpr (PART != 1) block_write_sums<32 * NW>(dacc, a.partials, blockIdx.x);
}

// Runs per plane: enough warps for several full waves, while keeping the
// warm-up rows of each run small against the run length.
static TvsGrid tvs_grid(int W, int H, int Nz, int VW, int warps_per_sm, int warm) {
  TvsGrid g;
  g.nstrips = (W + VW - 1) / VW;
  const double slots = (double)num_sms() * warps_per_sm;  // resident warps
  double best = 1e300;
  g.nseg = 1;
  for (int ns = 1; ns <= 64 && ns <= H; ++ns) {
    const int len = (H + ns - 1) / ns;
    if (ns > 1 && len < 2 * warm) break;
    const double runs = (double)g.nstrips * ns * Nz;
    const double waves = std::ceil(runs / slots);
    const double cost = waves * (len + warm);  // steps on the critical path
    if (cost < best * 0.999) {
      best = cost;
      g.nseg = ns;
    }
  }
  g.seg_len = (H + g.nseg - 1) / g.nseg;
  g.nseg = (H + g.seg_len - 1) / g.seg_len;
  return g;
}

// Warps a block of the streaming prox: 2 (built in), or 4 when the tuning
// asks for it (tv_kernel 3) and the 8-row ring applies (n_tv <= 5), where
// three 4-warp blocks (12 warps) share an SM at up to 168 registers.
template <int NTV, bool NORMS, int NW>
constexpr int tvw_minb_nw() {
  return NW == 2 ? tvw_minb<NTV, NORMS>() : 3;
}

template <typename ST, int NTV, bool NORMS, int NW, int PART = 0>
static cudaError_t strip_launch_nw(const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  using Sh = TvwShape<NTV, 2>;
  constexpr int MINB = tvw_minb_nw<NTV, NORMS, NW>();
  // one ring a warp, and for the second part a 4-row ring of the stored duals
  constexpr size_t SMEM = Sh::SMEM / Sh::NW * NW + (PART == 2 ? (size_t)NW * 2 * 32 * 2 * sizeof(float4) : 0);
  auto kern = k_prox_tv2d_strip<ST, NTV, NORMS, 2, NW, MINB, 4, 4, PART>;
  cudaError_t e = allow_smem(kern, SMEM);
  if (e != cudaSuccess) return e;
  // resident blocks per SM, for the choice of runs per plane
  static const int resident = [kern] {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, 32 * NW, SMEM) != cudaSuccess || b <= 0) {
      cudaGetLastError();
      b = MINB;
    }
    return b;
  }();
  TvsGrid g = tvs_grid(a.W, a.H, a.Nz, Sh::VW, NW * resident, 2 * Sh::h + 3);
  if (a.tv_nseg > 0) {  // tuned number of runs per plane
    g.seg_len = (a.H + min(a.tv_nseg, a.H) - 1) / min(a.tv_nseg, a.H);
    g.nseg = (a.H + g.seg_len - 1) / g.seg_len;
  }
  const long long runs = (long long)g.nstrips * g.nseg * a.Nz;
  const long long blocks = (runs + NW - 1) / NW;
  if (blocks > 0x7fffffffLL || blocks > a.partial_cap) return cudaErrorInvalidConfiguration;
  *nblocks_out = (int)blocks;
  kern<<<(unsigned)blocks, 32 * NW, SMEM, st>>>(a, g);
  return cudaGetLastError();
}

template <typename ST, int NTV, bool NORMS>
static cudaError_t strip_launch_n(const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  if constexpr (TvwShape<NTV, 2>::D == 8) {
    if (a.tv_kernel == 3) return strip_launch_nw<ST, NTV, NORMS, 4>(a, nblocks_out, st);
  }
  return strip_launch_nw<ST, NTV, NORMS, 2>(a, nblocks_out, st);
}

template <typename ST, int NTV>
static cudaError_t strip_launch(const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  return a.want_norms ? strip_launch_n<ST, NTV, true>(a, nblocks_out, st)
                      : strip_launch_n<ST, NTV, false>(a, nblocks_out, st);
}

// n_tv = K1 + K2 Chambolle iterations as two streaming launches: the first
// runs iterations 1..K1 and stores the dual (gx, gy) of every voxel (gx in
// a.gdx, gy in a.gdy, FP32 complex); the second starts from that dual, runs
// iterations K1+1..n_tv, the estimate, the shrink and the sums.  Each launch
// needs an x halo of K + 1 columns instead of n_tv + 1 and the 8-row ring, so
// at n_tv = 10 a 64-column strip keeps 52 valid columns instead of 40 and 16
// warps share an SM instead of 8.  The arithmetic is the single pass's, in the
// same order, and the dual goes through memory unrounded, so P_new has the
// same bits; only the second launch writes block partials.
template <typename ST, int K1, int K2>
static cudaError_t strip_launch_split(const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  int nb1 = 0;
  cudaError_t e = strip_launch_nw<ST, K1, false, 2, 1>(a, &nb1, st);
  if (e != cudaSuccess) return e;
  return a.want_norms ? strip_launch_nw<ST, K2, true, 2, 2>(a, nblocks_out, st)
                      : strip_launch_nw<ST, K2, false, 2, 2>(a, nblocks_out, st);
}

template <typename ST>
static cudaError_t strip_dispatch(const ProxArgs& a, int* nb, cudaStream_t st) {
  if (a.gdx && a.gdy && a.tv_kernel != 4) {  // two launches for more than 5 iterations
    switch (a.n_tv) {
      case 6: return strip_launch_split<ST, 3, 3>(a, nb, st);
      case 7: return strip_launch_split<ST, 3, 4>(a, nb, st);
      case 8: return strip_launch_split<ST, 4, 4>(a, nb, st);
      case 9: return strip_launch_split<ST, 4, 5>(a, nb, st);
      case 10: return strip_launch_split<ST, 5, 5>(a, nb, st);
      default: break;
    }
  }
  switch (a.n_tv) {
    case 1: return strip_launch<ST, 1>(a, nb, st);
    case 2: return strip_launch<ST, 2>(a, nb, st);
    case 3: return strip_launch<ST, 3>(a, nb, st);
    case 4: return strip_launch<ST, 4>(a, nb, st);
    case 5: return strip_launch<ST, 5>(a, nb, st);
    case 6: return strip_launch<ST, 6>(a, nb, st);
    case 7: return strip_launch<ST, 7>(a, nb, st);
    case 8: return strip_launch<ST, 8>(a, nb, st);
    case 9: return strip_launch<ST, 9>(a, nb, st);
    case 10: return strip_launch<ST, 10>(a, nb, st);
    default: return cudaErrorInvalidValue;
  }
}
constexpr int kStripNtvMax = 10;

// RIHVR_TV_KERNEL=tiles forces the tiled kernel (comparison and fallback);
// read once per process.
static bool tv_stream_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("RIHVR_TV_KERNEL");
    return !(v && std::strcmp(v, "tiles") == 0);
  }();
  return on;
}
// RIHVR_TV_KERNEL=strip4 (4-warp blocks) or strip1 (one launch for 6-10
// iterations) as tv_kernel 3 or 4; 0 when unset
static int tv_kernel_forced() {
  static const int k = [] {
    const char* v = std::getenv("RIHVR_TV_KERNEL");
    if (v && std::strcmp(v, "strip4") == 0) return 3;
    if (v && std::strcmp(v, "strip1") == 0) return 4;
    return 0;
  }();
  return k;
}

static void tv_grid(const ProxArgs& a, dim3* g) {
  const int h = a.n_tv + 1;
  const int VW = TV_EW - 2 * h, VH = TV_EH - 2 * h;
  *g = dim3((a.W + VW - 1) / VW, (a.H + VH - 1) / VH, a.Nz);
}

size_t max_partial_blocks(int W, int H, int Nz) {
  // the tiled TV prox with the largest halo it accepts (n_tv <= 20)
  const int h = 21, VW = TV_EW - 2 * h, VH = TV_EH - 2 * h;
  const size_t tv = (size_t)((W + VW - 1) / VW) * ((H + VH - 1) / VH) * Nz;
  // the streaming TV prox with its narrowest strips (n_tv = 10) and the most
  // runs per plane (64), one block per run
  using Sh = TvwShape<kStripNtvMax, 2>;
  const size_t strip = (size_t)((W + Sh::VW - 1) / Sh::VW) * (size_t)std::min(64, H) * Nz;
  const size_t flat = 4096;
  return std::max(std::max(tv, strip), flat);
}

cudaError_t launch_prox_tv2d(int storage, const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  if (a.n_tv < 0 || a.n_tv > 20) return cudaErrorInvalidValue;
  if (a.n_tv >= 1 && a.n_tv <= kStripNtvMax && a.tv_kernel != 1 && tv_stream_enabled()) {
    ProxArgs b = a;
    if (tv_kernel_forced()) b.tv_kernel = tv_kernel_forced();
    switch (storage) {
      case STORE_BF16: return strip_dispatch<__nv_bfloat162>(b, nblocks_out, st);
      case STORE_F16: return strip_dispatch<__half2>(b, nblocks_out, st);
      default: return strip_dispatch<float2>(b, nblocks_out, st);
    }
  }
  dim3 g;
  tv_grid(a, &g);
  *nblocks_out = (int)(g.x * g.y * g.z);
  cudaError_t e;
  switch (storage) {
    case STORE_BF16:
      e = allow_smem(k_prox_tv2d<__nv_bfloat162>, TV_SMEM);
      if (e != cudaSuccess) return e;
      k_prox_tv2d<__nv_bfloat162><<<g, TV_THREADS, TV_SMEM, st>>>(a);
      break;
    case STORE_F16:
      e = allow_smem(k_prox_tv2d<__half2>, TV_SMEM);
      if (e != cudaSuccess) return e;
      k_prox_tv2d<__half2><<<g, TV_THREADS, TV_SMEM, st>>>(a);
      break;
    default:
      e = allow_smem(k_prox_tv2d<float2>, TV_SMEM);
      if (e != cudaSuccess) return e;
      k_prox_tv2d<float2><<<g, TV_THREADS, TV_SMEM, st>>>(a);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Elementwise prox (mode 5): proximalL1, sparse_compressive_holo.cu:3274-3392,
// p = shrink(x - t g, t l1), plus the same sums (TV terms absent).
// ---------------------------------------------------------------------------
constexpr int FLAT_THREADS = 256;

template <typename ST>
__global__ void __launch_bounds__(FLAT_THREADS) k_prox_l1(ProxArgs a0) {
  const ProxArgs a = resolve_scalars(a0);
  const size_t HW = (size_t)a.W * a.H, n = HW * a.Nz;
  const ST* P = static_cast<const ST*>(a.P);
  const ST* Pp = static_cast<const ST*>(a.Pprev);
  ST* Pn = static_cast<ST*>(a.Pnew);
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 y0 = Store<ST>::ld(P + i), pp = Store<ST>::ld(Pp + i), g = a.G[i];
    const float2 x = make_float2(fmaf(a.beta, y0.x - pp.x, y0.x), fmaf(a.beta, y0.y - pp.y, y0.y));
    const float2 xh = make_float2(fmaf(-a.t, g.x, x.x), fmaf(-a.t, g.y, x.y));
    const float2 p = shrink(xh, a.thr, a.faithful);
    Store<ST>::st(Pn + i, p);
    const float2 d = csub(p, x);
    acc[SUM_LIM1] += (double)(d.x * g.x) + (double)(d.y * g.y);
    acc[SUM_LIM2] += (double)cabs2(d);
    float wr, wi;
    restart_w(i % HW, a.faithful, &wr, &wi);
    const float2 u = csub(x, p), v = csub(p, y0);
    acc[SUM_RS] += (double)(wr * u.x * v.x) + (double)(wi * u.y * v.y);
    if (a.want_norms) {
      acc[SUM_L1P] += (double)norm_sqrt(cabs2(p));
      acc[SUM_L1X] += (double)norm_sqrt(cabs2(x));
    }
  }
  block_write_sums<FLAT_THREADS>(acc, a.partials, blockIdx.x);
}

static int flat_blocks(size_t n) {
  size_t b = (n + FLAT_THREADS - 1) / FLAT_THREADS;
  size_t cap = (size_t)8 * num_sms();
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

cudaError_t launch_prox_l1(int storage, const ProxArgs& a, int* nblocks_out, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)a.W * a.H * a.Nz);
  *nblocks_out = blocks;
  switch (storage) {
    case STORE_BF16:
      k_prox_l1<__nv_bfloat162><<<blocks, FLAT_THREADS, 0, st>>>(a);
      break;
    case STORE_F16:
      k_prox_l1<__half2><<<blocks, FLAT_THREADS, 0, st>>>(a);
      break;
    default:
      k_prox_l1<float2><<<blocks, FLAT_THREADS, 0, st>>>(a);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// reduction of block partials in two fixed-shape stages (deterministic):
// stage 1 sums contiguous slices of the partials, stage 2 sums the slices.
// ---------------------------------------------------------------------------
constexpr int RED_THREADS = 256;
constexpr int RED_SLICES = 512;

__global__ void __launch_bounds__(RED_THREADS) k_reduce_stage(const double* __restrict__ in, int n, int per_block,
                                                              double* __restrict__ out) {
  __shared__ double red[RED_THREADS / 32][kNumSums];
  const int b0 = blockIdx.x * per_block, b1 = min(n, b0 + per_block);
  // thread j handles slot j % kNumSums of rows b0 + j / kNumSums, strided
  const int slot = threadIdx.x % kNumSums, lane_row = threadIdx.x / kNumSums;
  constexpr int ROWS_PER_PASS = RED_THREADS / kNumSums;
  double v = 0.0;
  for (int b = b0 + lane_row; b < b1; b += ROWS_PER_PASS) v += in[(size_t)b * kNumSums + slot];
  // gather per-slot sums: rows of the same slot are kNumSums lanes apart
#pragma unroll
  for (int o = 16; o >= kNumSums; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane < kNumSums) red[wid][lane] = v;
  __syncthreads();
  if (threadIdx.x < kNumSums) {
    double s = 0.0;
    for (int w = 0; w < RED_THREADS / 32; ++w) s += red[w][threadIdx.x];
    out[(size_t)blockIdx.x * kNumSums + threadIdx.x] = s;
  }
}

cudaError_t launch_reduce_partials(const double* partials, int nblocks, double* scratch, double* out,
                                   cudaStream_t st) {
  if (nblocks <= RED_THREADS) {
    k_reduce_stage<<<1, RED_THREADS, 0, st>>>(partials, nblocks, nblocks, out);
    return cudaGetLastError();
  }
  const int per = (nblocks + RED_SLICES - 1) / RED_SLICES;
  const int slices = (nblocks + per - 1) / per;
  k_reduce_stage<<<slices, RED_THREADS, 0, st>>>(partials, nblocks, per, scratch);
  k_reduce_stage<<<1, RED_THREADS, 0, st>>>(scratch, slices, slices, out);
  return cudaGetLastError();
}

size_t reduce_scratch_doubles() { return (size_t)RED_SLICES * kNumSums; }

// ---------------------------------------------------------------------------
// plane-level kernels
// ---------------------------------------------------------------------------
// d = Re(c); sum (d - b)^2.  back_propagate_finish_kernel (:1918-1933) keeps
// only the real part; calcResidual (:2676-2723) forms r = estimate - measured.
__global__ void __launch_bounds__(FLAT_THREADS) k_finish_forward(const float2* __restrict__ c,
                                                                 const float* __restrict__ b,
                                                                 float* __restrict__ dnew, long long n,
                                                                 double* partials) {
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = c[i].x;
    dnew[i] = d;
    const float r = d - b[i];
    acc[SUM_RR] += (double)r * (double)r;
  }
  block_write_sums<FLAT_THREADS>(acc, partials, blockIdx.x);
}

cudaError_t launch_finish_forward(const float2* c, const float* b, float* dnew, long long n, double* partials,
                                  int* nblocks_out, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)n);
  *nblocks_out = blocks;
  k_finish_forward<<<blocks, FLAT_THREADS, 0, st>>>(c, b, dnew, n, partials);
  return cudaGetLastError();
}

// Counter-based uniform fill in [-1, 1) for both parts of a complex volume
// (splitmix64 of the seed and the element index), so that a host model can
// regenerate exactly the same start vector.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ float unit_from_bits(unsigned long long r) {
  // top 24 bits -> [0, 1), then [-1, 1): exact in float
  return (float)(r >> 40) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}
__global__ void __launch_bounds__(FLAT_THREADS) k_fill_uniform_c(float2* __restrict__ x, long long n,
                                                                 unsigned long long seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = seed * 0x100000001B3ull + 2ull * (unsigned long long)i;
    x[i] = make_float2(unit_from_bits(splitmix64(k)), unit_from_bits(splitmix64(k + 1)));
  }
}

cudaError_t launch_fill_uniform_c(float2* x, long long n, unsigned long long seed, cudaStream_t st) {
  k_fill_uniform_c<<<flat_blocks((size_t)n), FLAT_THREADS, 0, st>>>(x, n, seed);
  return cudaGetLastError();
}

// sum x^2 over n floats in FP64 (the SUM_RR entry of the block partials)
__global__ void __launch_bounds__(FLAT_THREADS) k_sumsq(const float* __restrict__ x, long long n, double* partials) {
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i];
    acc[SUM_RR] += v * v;
  }
  block_write_sums<FLAT_THREADS>(acc, partials, blockIdx.x);
}

cudaError_t launch_sumsq(const float* x, long long n, double* partials, int* nblocks_out, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)n);
  *nblocks_out = blocks;
  k_sumsq<<<blocks, FLAT_THREADS, 0, st>>>(x, n, partials);
  return cudaGetLastError();
}

// Momentum in hologram space (:480-498, fistaUpdate on holograms :4599-4642):
// dX = d + beta (d - dY0); dY0 = d; r = dX - b.
__global__ void __launch_bounds__(FLAT_THREADS) k_holo_momentum(const float* __restrict__ dnew, float* dY0,
                                                                float* __restrict__ dX, const float* __restrict__ b,
                                                                float* __restrict__ r, float beta0, long long n,
                                                                double* partials, const float* __restrict__ dbeta) {
  const float beta = dbeta ? __ldg(dbeta) : beta0;  // device copy for captured launches
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = dnew[i], d0 = dY0[i];
    const float x = fmaf(beta, d - d0, d);
    dX[i] = x;
    dY0[i] = d;
    const float rr = x - b[i];
    r[i] = rr;
    acc[SUM_RR] += (double)rr * (double)rr;
  }
  block_write_sums<FLAT_THREADS>(acc, partials, blockIdx.x);
}

cudaError_t launch_holo_momentum(const float* dnew, float* dY0, float* dX, const float* b, float* r, float beta,
                                 long long n, double* partials, int* nblocks_out, cudaStream_t st,
                                 const float* dbeta) {
  const int blocks = flat_blocks((size_t)n);
  *nblocks_out = blocks;
  k_holo_momentum<<<blocks, FLAT_THREADS, 0, st>>>(dnew, dY0, dX, b, r, beta, n, partials, dbeta);
  return cudaGetLastError();
}

// L1 and TV norms of the momentum point x = P + beta (P - Pprev):
// calcL1NormComplex (sparse_volume.cu:194-235), calcTVNorm2d (:365-446),
// calcTVNorm (:240-363, periodic in z).

template <typename ST>
__global__ void __launch_bounds__(FLAT_THREADS) k_momentum_norms(const ST* __restrict__ P, const ST* __restrict__ Pp,
                                                                 float beta, int W, int H, int Nz, int mode,
                                                                 double* partials) {
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  const size_t HW = (size_t)W * H, n = HW * Nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i / HW);
    const size_t e = i - (size_t)z * HW;
    const int yy = (int)(e / W), xx = (int)(e - (size_t)yy * W);
    const float2 x = xval(P, Pp, beta, i);
    acc[SUM_L1X] += (double)norm_sqrt(cabs2(x));
    acc[SUM_LIM1] += (x.x != 0.f || x.y != 0.f) ? 1.0 : 0.0;  // non-zero voxels
    if (mode == 7 || mode == 6) {
      const int xm = xx > 0 ? xx - 1 : W - 1, ym = yy > 0 ? yy - 1 : H - 1;
      const float2 xl = xval(P, Pp, beta, (size_t)z * HW + (size_t)yy * W + xm);
      const float2 xu = xval(P, Pp, beta, (size_t)z * HW + (size_t)ym * W + xx);
      float q = cabs2(csub(xl, x)) + cabs2(csub(xu, x));
      if (mode == 6) {
        const int zm = z > 0 ? z - 1 : Nz - 1;
        q += cabs2(csub(xval(P, Pp, beta, (size_t)zm * HW + e), x));
      }
      acc[SUM_TVX] += (double)norm_sqrt(q);
    }
  }
  block_write_sums<FLAT_THREADS>(acc, partials, blockIdx.x);
}

cudaError_t launch_momentum_norms(int storage, const void* P, const void* Pprev, float beta, int W, int H, int Nz,
                                  int mode, double* partials, int* nblocks_out, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)W * H * Nz);
  *nblocks_out = blocks;
  switch (storage) {
    case STORE_BF16:
      k_momentum_norms<__nv_bfloat162><<<blocks, FLAT_THREADS, 0, st>>>(
          (const __nv_bfloat162*)P, (const __nv_bfloat162*)Pprev, beta, W, H, Nz, mode, partials);
      break;
    case STORE_F16:
      k_momentum_norms<__half2><<<blocks, FLAT_THREADS, 0, st>>>((const __half2*)P, (const __half2*)Pprev, beta, W,
                                                                  H, Nz, mode, partials);
      break;
    default:
      k_momentum_norms<float2><<<blocks, FLAT_THREADS, 0, st>>>((const float2*)P, (const float2*)Pprev, beta, W, H,
                                                                 Nz, mode, partials);
  }
  return cudaGetLastError();
}

template <typename ST>
__global__ void k_materialize_x(const ST* __restrict__ P, const ST* __restrict__ Pp, float beta, float2* out,
                                long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = xval(P, Pp, beta, (size_t)i);
}

cudaError_t launch_materialize_x(int storage, const void* P, const void* Pprev, float beta, float2* out, long long n,
                                 cudaStream_t st) {
  const int blocks = flat_blocks((size_t)n);
  switch (storage) {
    case STORE_BF16:
      k_materialize_x<<<blocks, FLAT_THREADS, 0, st>>>((const __nv_bfloat162*)P, (const __nv_bfloat162*)Pprev, beta,
                                                       out, n);
      break;
    case STORE_F16:
      k_materialize_x<<<blocks, FLAT_THREADS, 0, st>>>((const __half2*)P, (const __half2*)Pprev, beta, out, n);
      break;
    default:
      k_materialize_x<<<blocks, FLAT_THREADS, 0, st>>>((const float2*)P, (const float2*)Pprev, beta, out, n);
  }
  return cudaGetLastError();
}

template <typename ST>
__global__ void k_store_volume(const float2* __restrict__ in, ST* __restrict__ out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    Store<ST>::st(out + i, in[i]);
}

cudaError_t launch_store_volume(int storage, const float2* in, void* out, long long n, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)n);
  switch (storage) {
    case STORE_BF16:
      k_store_volume<<<blocks, FLAT_THREADS, 0, st>>>(in, (__nv_bfloat162*)out, n);
      break;
    case STORE_F16:
      k_store_volume<<<blocks, FLAT_THREADS, 0, st>>>(in, (__half2*)out, n);
      break;
    default:
      k_store_volume<<<blocks, FLAT_THREADS, 0, st>>>(in, (float2*)out, n);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// 3-D fused lasso (mode 6): proximalFusedLasso (:3422-3475) with
// totalVariationProjection (:3832-4018): half threshold, n_tv unnormalised dual
// steps over the whole volume (periodic in x, y, z; the projection is disabled
// at :3964), final estimate, half threshold.
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void k_prox6_init(ProxArgs a, float2* __restrict__ X1) {
  const size_t n = (size_t)a.W * a.H * a.Nz;
  const ST* P = static_cast<const ST*>(a.P);
  const ST* Pp = static_cast<const ST*>(a.Pprev);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float2 x = xval(P, Pp, a.beta, i), g = a.G[i];
    const float2 xh = make_float2(fmaf(-a.t, g.x, x.x), fmaf(-a.t, g.y, x.y));
    X1[i] = shrink(xh, 0.5f * a.thr, a.faithful);
  }
}

cudaError_t launch_prox6_init(int storage, const ProxArgs& a, float2* X1, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)a.W * a.H * a.Nz);
  switch (storage) {
    case STORE_BF16:
      k_prox6_init<__nv_bfloat162><<<blocks, FLAT_THREADS, 0, st>>>(a, X1);
      break;
    case STORE_F16:
      k_prox6_init<__half2><<<blocks, FLAT_THREADS, 0, st>>>(a, X1);
      break;
    default:
      k_prox6_init<float2><<<blocks, FLAT_THREADS, 0, st>>>(a, X1);
  }
  return cudaGetLastError();
}

__global__ void k_tv3_estimate(const float2* __restrict__ X1, const float2* __restrict__ gx,
                               const float2* __restrict__ gy, const float2* __restrict__ gz, float2* __restrict__ Y,
                               int W, int H, int Nz, float mu) {
  const size_t HW = (size_t)W * H, n = HW * Nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i / HW);
    const size_t e = i - (size_t)z * HW;
    const int yy = (int)(e / W), xx = (int)(e - (size_t)yy * W);
    const int xp = xx < W - 1 ? xx + 1 : 0, yp = yy < H - 1 ? yy + 1 : 0, zp = z < Nz - 1 ? z + 1 : 0;
    const float2 d1 = csub(gx[(size_t)z * HW + (size_t)yy * W + xp], gx[i]);
    const float2 d2 = csub(gy[(size_t)z * HW + (size_t)yp * W + xx], gy[i]);
    const float2 d3 = csub(gz[(size_t)zp * HW + e], gz[i]);
    const float2 dv = cadd(cadd(d1, d2), d3);
    Y[i] = make_float2(fmaf(-mu, dv.x, X1[i].x), fmaf(-mu, dv.y, X1[i].y));
  }
}

cudaError_t launch_tv3_estimate(const float2* X1, const float2* gx, const float2* gy, const float2* gz, float2* Y,
                                int W, int H, int Nz, float mu, cudaStream_t st) {
  k_tv3_estimate<<<flat_blocks((size_t)W * H * Nz), FLAT_THREADS, 0, st>>>(X1, gx, gy, gz, Y, W, H, Nz, mu);
  return cudaGetLastError();
}

__global__ void k_tv3_dual(const float2* __restrict__ Y, float2* gx, float2* gy, float2* gz, int W, int H, int Nz,
                           float s) {
  const size_t HW = (size_t)W * H, n = HW * Nz;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i / HW);
    const size_t e = i - (size_t)z * HW;
    const int yy = (int)(e / W), xx = (int)(e - (size_t)yy * W);
    const int xm = xx > 0 ? xx - 1 : W - 1, ym = yy > 0 ? yy - 1 : H - 1, zm = z > 0 ? z - 1 : Nz - 1;
    const float2 yv = Y[i];
    const float2 a1 = csub(Y[(size_t)z * HW + (size_t)yy * W + xm], yv);
    const float2 a2 = csub(Y[(size_t)z * HW + (size_t)ym * W + xx], yv);
    const float2 a3 = csub(Y[(size_t)zm * HW + e], yv);
    gx[i] = make_float2(fmaf(s, a1.x, gx[i].x), fmaf(s, a1.y, gx[i].y));
    gy[i] = make_float2(fmaf(s, a2.x, gy[i].x), fmaf(s, a2.y, gy[i].y));
    gz[i] = make_float2(fmaf(s, a3.x, gz[i].x), fmaf(s, a3.y, gz[i].y));
  }
}

cudaError_t launch_tv3_dual(const float2* Y, float2* gx, float2* gy, float2* gz, int W, int H, int Nz, float s,
                            cudaStream_t st) {
  k_tv3_dual<<<flat_blocks((size_t)W * H * Nz), FLAT_THREADS, 0, st>>>(Y, gx, gy, gz, W, H, Nz, s);
  return cudaGetLastError();
}

template <typename ST>
__global__ void __launch_bounds__(FLAT_THREADS) k_prox6_finish(ProxArgs a, const float2* __restrict__ Y) {
  const int W = a.W, H = a.H, Nz = a.Nz;
  const size_t HW = (size_t)W * H, n = HW * Nz;
  const ST* P = static_cast<const ST*>(a.P);
  const ST* Pp = static_cast<const ST*>(a.Pprev);
  ST* Pn = static_cast<ST*>(a.Pnew);
  const float T = 0.5f * a.thr;
  double acc[kNumSums];
#pragma unroll
  for (int k = 0; k < kNumSums; ++k) acc[k] = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(i / HW);
    const size_t e = i - (size_t)z * HW;
    const int yy = (int)(e / W), xx = (int)(e - (size_t)yy * W);
    const float2 p = shrink(Y[i], T, a.faithful);
    Store<ST>::st(Pn + i, p);
    const float2 y0 = Store<ST>::ld(P + i);
    const float2 x = xval(P, Pp, a.beta, i), g = a.G[i];
    const float2 d = csub(p, x);
    acc[SUM_LIM1] += (double)(d.x * g.x) + (double)(d.y * g.y);
    acc[SUM_LIM2] += (double)cabs2(d);
    float wr, wi;
    restart_w(e, a.faithful, &wr, &wi);
    const float2 u = csub(x, p), v = csub(p, y0);
    acc[SUM_RS] += (double)(wr * u.x * v.x) + (double)(wi * u.y * v.y);
    if (a.want_norms) {
      const int xm = xx > 0 ? xx - 1 : W - 1, ym = yy > 0 ? yy - 1 : H - 1, zm = z > 0 ? z - 1 : Nz - 1;
      const size_t il = (size_t)z * HW + (size_t)yy * W + xm, iu = (size_t)z * HW + (size_t)ym * W + xx,
                   ib = (size_t)zm * HW + e;
      const float2 pl = shrink(Y[il], T, a.faithful), pu = shrink(Y[iu], T, a.faithful),
                   pb = shrink(Y[ib], T, a.faithful);
      acc[SUM_L1P] += (double)norm_sqrt(cabs2(p));
      acc[SUM_TVP] += (double)norm_sqrt(cabs2(csub(pl, p)) + cabs2(csub(pu, p)) + cabs2(csub(pb, p)));
      const float2 xl = xval(P, Pp, a.beta, il), xu = xval(P, Pp, a.beta, iu), xb = xval(P, Pp, a.beta, ib);
      acc[SUM_L1X] += (double)norm_sqrt(cabs2(x));
      acc[SUM_TVX] += (double)norm_sqrt(cabs2(csub(xl, x)) + cabs2(csub(xu, x)) + cabs2(csub(xb, x)));
    }
  }
  block_write_sums<FLAT_THREADS>(acc, a.partials, blockIdx.x);
}

cudaError_t launch_prox6_finish(int storage, const ProxArgs& a, const float2* Y, int* nblocks_out, cudaStream_t st) {
  const int blocks = flat_blocks((size_t)a.W * a.H * a.Nz);
  *nblocks_out = blocks;
  switch (storage) {
    case STORE_BF16:
      k_prox6_finish<__nv_bfloat162><<<blocks, FLAT_THREADS, 0, st>>>(a, Y);
      break;
    case STORE_F16:
      k_prox6_finish<__half2><<<blocks, FLAT_THREADS, 0, st>>>(a, Y);
      break;
    default:
      k_prox6_finish<float2><<<blocks, FLAT_THREADS, 0, st>>>(a, Y);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Generic line FFT: plane sides without a register-resident four-step
// configuration above (any length up to 8192 whose prime factors are 2, 3, 5
// and 7, such as 640, 1536, 2048 or 2304) and rectangular planes.  The
// reference takes such sizes through cuFFT (sparse_compressive_holo.cu:98);
// W and H are multiples of 16 there (:126, 1948).
//
// A block transforms C lines of length n held in shared memory as [n][C]
// (C a power of two, n C <= kGElems) by a self-sorting Stockham sequence of
// radix-4, 2, 3, 5 and 7 stages between two shared-memory buffers: each
// butterfly reads its R inputs, multiplies by the twiddles of the previous
// stages' size, transforms in registers and writes its outputs in sorted
// position.  Twiddles come from a per-length FP64-built table of
// exp(-2 pi i k / n).  Rows load C contiguous lines, columns C adjacent
// columns of a plane of any row pitch; the column passes keep the same fusion
// as the fast ones (transfer function on the fly, z-sum in registers).
// ---------------------------------------------------------------------------
constexpr int kGThreads = 256;
constexpr int kGElems = 4096;          // complex values per row block (two 32 KB buffers)
constexpr int kGColElems = 9216;       // per column block: 4 columns of 2304 (two 72 KB buffers)
constexpr int kGMaxStages = 16;

struct GPlan {
  int n, ns;
  int r[kGMaxStages];
};

static bool gplan_make(int n, GPlan* p) {
  if (n < 2 || n > kGElems) return false;
  p->n = n;
  p->ns = 0;
  int m = n;
  const int order[5] = {4, 2, 3, 5, 7};
  for (int k = 0; k < 5; ++k) {
    while (m % order[k] == 0) {
      if (p->ns == kGMaxStages) return false;
      p->r[p->ns++] = order[k];
      m /= order[k];
    }
  }
  return m == 1;
}

bool generic_size_supported(int n) {
  GPlan p;
  return gplan_make(n, &p);
}

static int ilog2(int c) {
  int l = 0;
  while ((1 << l) < c) ++l;
  return l;
}

// lines per block: the largest power of two with n C <= budget, capped
static int gplan_lines(int n, int cap, int budget = kGElems) {
  int c = 1;
  while (2 * c * n <= budget && 2 * c <= cap) c *= 2;
  return c;
}

__global__ void k_gtwiddles(int n, float2* __restrict__ tw) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

// exp(-2 pi i k / n), k < n: one table per (device, n), built once and kept
// for the life of the process (at most 64 KB each)
static const float2* gtwiddles(int n, cudaStream_t st, cudaError_t* err) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, float2*> tables;
  int dev = 0;
  *err = cudaGetDevice(&dev);
  if (*err != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  auto it = tables.find({dev, n});
  if (it != tables.end()) return it->second;
  float2* t = nullptr;
  *err = cudaMalloc(&t, sizeof(float2) * (size_t)n);
  if (*err != cudaSuccess) return nullptr;
  k_gtwiddles<<<(n + 255) / 256, 256, 0, st>>>(n, t);
  *err = cudaStreamSynchronize(st);
  if (*err != cudaSuccess) {
    cudaFree(t);
    return nullptr;
  }
  tables[{dev, n}] = t;
  return t;
}

template <int R, bool INV>
__device__ __forceinline__ void gstage(const float2* src, float2* dst, int n, int logc, int ns,
                                       const float2* __restrict__ tw) {
  const int C = 1 << logc;
  const int m = n / R;
  const int total = m << logc;
  const int tstep = n / (ns * R);
  for (int b = threadIdx.x; b < total; b += kGThreads) {
    const int c = b & (C - 1), j = b >> logc;
    const int k = j % ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 x = src[((j + r * m) << logc) + c];
      if (r > 0 && k > 0) {
        float2 w = __ldg(tw + k * r * tstep);
        if (INV) w.y = -w.y;
        x = cmul(x, w);
      }
      v[r] = x;
    }
    small_dft<R, INV>(v);
    const int d = (((j - k) * R + k) << logc) + c;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[d + ((r * ns) << logc)] = v[r];
  }
  __syncthreads();
}

// DFT of the C lines in buf[0] ([n][C]), using buf[1] as the other half of the
// ping-pong; returns the buffer holding the result.  Every thread of the block
// calls it, after a barrier that makes buf[0] complete.
template <bool INV>
__device__ float2* gfft(float2* b0, float2* b1, int logc, const GPlan& p, const float2* __restrict__ tw) {
  int ns = 1;
  float2* src = b0;
  float2* dst = b1;
  for (int s = 0; s < p.ns; ++s) {
    switch (p.r[s]) {
      case 4: gstage<4, INV>(src, dst, p.n, logc, ns, tw); break;
      case 2: gstage<2, INV>(src, dst, p.n, logc, ns, tw); break;
      case 3: gstage<3, INV>(src, dst, p.n, logc, ns, tw); break;
      case 5: gstage<5, INV>(src, dst, p.n, logc, ns, tw); break;
      default: gstage<7, INV>(src, dst, p.n, logc, ns, tw); break;
    }
    ns *= p.r[s];
    float2* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

template <bool INV, int IN>
__global__ void __launch_bounds__(kGThreads) k_grows(GPlan p, const float2* __restrict__ tw,
                                                     const void* __restrict__ in, float2* __restrict__ out,
                                                     long long nlines, float scale, int logc) {
  extern __shared__ __align__(128) float2 gbuf[];
  const int n = p.n, C = 1 << logc;
  float2* const gb1 = gbuf + n * C;
  const long long l0 = (long long)blockIdx.x << logc;
  const int nl = (int)min((long long)C, nlines - l0);
  for (int e = threadIdx.x; e < n * C; e += kGThreads) {
    const int c = e / n, k = e - c * n;  // consecutive threads, consecutive elements of a line
    gbuf[(k << logc) + c] = c < nl ? load_as<IN>(in, (size_t)(l0 + c) * n + k) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = gfft<INV>(gbuf, gb1, logc, p, tw);
  for (int e = threadIdx.x; e < n * C; e += kGThreads) {
    const int c = e / n, k = e - c * n;
    if (c < nl) out[(size_t)(l0 + c) * n + k] = cscale(res[(k << logc) + c], scale);
  }
}

template <bool INV, int IN>
static cudaError_t grows_launch(const GPlan& p, const float2* tw, const void* in, float2* out, long long nlines,
                                float scale, int C, cudaStream_t st) {
  const size_t smem = 2 * sizeof(float2) * (size_t)p.n * C;
  const long long blocks = (nlines + C - 1) / C;
  if (blocks <= 0) return cudaSuccess;
  cudaError_t e = allow_smem(k_grows<INV, IN>, smem);
  if (e != cudaSuccess) return e;
  k_grows<INV, IN><<<(unsigned)blocks, kGThreads, smem, st>>>(p, tw, in, out, nlines, scale, ilog2(C));
  return cudaGetLastError();
}

// adjoint column pass: U_z(:, x) = IDFT_y(conj(H'_z(:, x)) Rs(:, x)) for the
// C columns x0.. of the block, planes [zb, ze)
__global__ void __launch_bounds__(kGThreads) k_gadj_col(GPlan p, const float2* __restrict__ tw,
                                                        const float2* __restrict__ Rs,
                                                        const double* __restrict__ cturn,
                                                        const double* __restrict__ zlist, float2* __restrict__ U,
                                                        int W, int z0, int z1, int zpb, int logc) {
  extern __shared__ __align__(128) float2 gbuf[];
  const int H = p.n, C = 1 << logc;
  float2* const gb1 = gbuf + H * C;
  const int x0 = blockIdx.x << logc;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  const size_t HW = (size_t)H * W;
  for (int z = zb; z < ze; ++z) {
    const double zz = zlist[z];
    for (int e = threadIdx.x; e < H * C; e += kGThreads) {
      const int c = e & (C - 1), y = e >> logc, x = x0 + c;
      float2 v = make_float2(0.f, 0.f);
      if (x < W) {
        const size_t i = (size_t)y * W + x;
        v = cmul(Rs[i], transfer(zz, cturn[i], true));
      }
      gbuf[e] = v;
    }
    __syncthreads();
    const float2* res = gfft<true>(gbuf, gb1, logc, p, tw);
    float2* Uz = U + (size_t)z * HW;
    for (int e = threadIdx.x; e < H * C; e += kGThreads) {
      const int c = e & (C - 1), y = e >> logc, x = x0 + c;
      if (x < W) Uz[(size_t)y * W + x] = res[e];
    }
    __syncthreads();
  }
}

constexpr int kGAcc = kGColElems / kGThreads;  // elements a thread accumulates

// forward column pass with the z-sum: Spart[chunk](:, x) = sum_z H'_z(:, x) DFT_y(T_z(:, x))
__global__ void __launch_bounds__(kGThreads) k_gfwd_col(GPlan p, const float2* __restrict__ tw,
                                                        const float2* __restrict__ T,
                                                        const double* __restrict__ cturn,
                                                        const double* __restrict__ zlist, float2* __restrict__ Spart,
                                                        int W, int z0, int z1, int zpb, int logc) {
  extern __shared__ __align__(128) float2 gbuf[];
  const int H = p.n, C = 1 << logc;
  float2* const gb1 = gbuf + H * C;
  const int x0 = blockIdx.x << logc;
  const int zb = z0 + blockIdx.y * zpb, ze = min(zb + zpb, z1);
  const size_t HW = (size_t)H * W;
  float2 acc[kGAcc];
#pragma unroll
  for (int i = 0; i < kGAcc; ++i) acc[i] = make_float2(0.f, 0.f);
  for (int z = zb; z < ze; ++z) {
    const double zz = zlist[z];
    const float2* Tz = T + (size_t)z * HW;
    for (int e = threadIdx.x; e < H * C; e += kGThreads) {
      const int c = e & (C - 1), y = e >> logc, x = x0 + c;
      gbuf[e] = x < W ? Tz[(size_t)y * W + x] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* res = gfft<false>(gbuf, gb1, logc, p, tw);
#pragma unroll
    for (int i = 0; i < kGAcc; ++i) {
      const int e = threadIdx.x + i * kGThreads;
      if (e < H * C) {
        const int c = e & (C - 1), y = e >> logc, x = x0 + c;
        if (x < W) acc[i] = cadd(acc[i], cmul(res[e], transfer(zz, cturn[(size_t)y * W + x], false)));
      }
    }
    __syncthreads();
  }
  float2* Sp = Spart + (size_t)blockIdx.y * HW;
#pragma unroll
  for (int i = 0; i < kGAcc; ++i) {
    const int e = threadIdx.x + i * kGThreads;
    if (e < H * C) {
      const int c = e & (C - 1), y = e >> logc, x = x0 + c;
      if (x < W) Sp[(size_t)y * W + x] = acc[i];
    }
  }
}

template <bool INV>
__global__ void __launch_bounds__(kGThreads) k_gplane_col(GPlan p, const float2* __restrict__ tw,
                                                          const float2* __restrict__ in, float2* __restrict__ out, int W,
                                                          float scale, int logc) {
  extern __shared__ __align__(128) float2 gbuf[];
  const int H = p.n, C = 1 << logc;
  float2* const gb1 = gbuf + H * C;
  const int x0 = blockIdx.x << logc;
  for (int e = threadIdx.x; e < H * C; e += kGThreads) {
    const int c = e & (C - 1), y = e >> logc, x = x0 + c;
    gbuf[e] = x < W ? in[(size_t)y * W + x] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = gfft<INV>(gbuf, gb1, logc, p, tw);
  for (int e = threadIdx.x; e < H * C; e += kGThreads) {
    const int c = e & (C - 1), y = e >> logc, x = x0 + c;
    if (x < W) out[(size_t)y * W + x] = cscale(res[e], scale);
  }
}

// columns per block of the generic column passes: 8-byte elements, 16 columns
// make 128-byte row segments
constexpr int kGColsMax = 16;

static bool fast_square(int W, int H) { return W == H && line_size_supported(W); }

static int fwd_col_chunks_generic(int W, int H, int Nz) {
  const int C = gplan_lines(H, kGColsMax, kGColElems);
  const int strips = (W + C - 1) / C;
  int chunks = (4 * num_sms() + strips - 1) / strips;
  if (chunks > 16) chunks = 16;
  if (chunks > Nz) chunks = Nz;
  if (chunks < 1) chunks = 1;
  return chunks;
}

int fwd_col_chunks(int W, int H, int Nz) {
  return fast_square(W, H) ? fwd_col_chunks_fast(W, H, Nz) : fwd_col_chunks_generic(W, H, Nz);
}

cudaError_t launch_rows(int inverse, int in_kind, const void* in, int out_kind, void* out, int W, long long nlines,
                        float scale, cudaStream_t st) {
  if (line_size_supported(W)) return launch_rows_fast(inverse, in_kind, in, out_kind, out, W, nlines, scale, st);
  if (out_kind != ELEM_C32) return cudaErrorInvalidValue;
  GPlan p;
  if (!gplan_make(W, &p)) return cudaErrorInvalidValue;
  cudaError_t e;
  const float2* tw = gtwiddles(W, st, &e);
  if (!tw) return e;
  const int C = gplan_lines(W, 64);
  float2* o = static_cast<float2*>(out);
  if (inverse) {
    if (in_kind != ELEM_C32 && in_kind != ELEM_STORE_F32) return cudaErrorInvalidValue;
    return grows_launch<true, ELEM_C32>(p, tw, in, o, nlines, scale, C, st);
  }
  switch (in_kind) {
    case ELEM_C32:
    case ELEM_STORE_F32: return grows_launch<false, ELEM_C32>(p, tw, in, o, nlines, scale, C, st);
    case ELEM_R32: return grows_launch<false, ELEM_R32>(p, tw, in, o, nlines, scale, C, st);
    case ELEM_STORE_BF16: return grows_launch<false, ELEM_STORE_BF16>(p, tw, in, o, nlines, scale, C, st);
    case ELEM_STORE_F16: return grows_launch<false, ELEM_STORE_F16>(p, tw, in, o, nlines, scale, C, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_adj_col(const float2* Rs, const double* cturn, const double* zlist, float2* U, int W, int H,
                           int z0, int z1, cudaStream_t st, int chunks_hint, double dz_uniform, int rec_mode) {
  if (fast_square(W, H))
    return launch_adj_col_fast(Rs, cturn, zlist, U, W, H, z0, z1, st, chunks_hint, dz_uniform, rec_mode);
  const int nz = z1 - z0;
  if (nz <= 0) return cudaSuccess;
  GPlan p;
  if (!gplan_make(H, &p)) return cudaErrorInvalidValue;
  cudaError_t e;
  const float2* tw = gtwiddles(H, st, &e);
  if (!tw) return e;
  const int C = gplan_lines(H, kGColsMax, kGColElems), logc = ilog2(C);
  const int strips = (W + C - 1) / C;
  int chunks = chunks_hint > 0 ? chunks_hint : (8 * num_sms() + strips - 1) / strips;
  if (chunks > nz) chunks = nz;
  if (chunks < 1) chunks = 1;
  const int zpb = (nz + chunks - 1) / chunks;
  chunks = (nz + zpb - 1) / zpb;
  const size_t smem = 2 * sizeof(float2) * (size_t)H * C;
  e = allow_smem(k_gadj_col, smem);
  if (e != cudaSuccess) return e;
  k_gadj_col<<<dim3(strips, chunks), kGThreads, smem, st>>>(p, tw, Rs, cturn, zlist, U, W, z0, z1, zpb, logc);
  return cudaGetLastError();
}

cudaError_t col_wait_timeouts(cudaStream_t st, unsigned* count) {
  unsigned zero = 0;
  cudaError_t e = cudaMemcpyFromSymbolAsync(count, g_col_wait_timeouts, sizeof(unsigned), 0, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && *count) e = cudaMemcpyToSymbolAsync(g_col_wait_timeouts, &zero, sizeof(unsigned), 0,
                                                              cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && *count) e = cudaStreamSynchronize(st);
  return e;
}

cudaError_t launch_fwd_col(const float2* T, const double* cturn, const double* zlist, float2* Spart, int W, int H,
                           int z0, int z1, int nchunks, cudaStream_t st, double dz_uniform, int horner_mode) {
  if (fast_square(W, H))
    return launch_fwd_col_fast(T, cturn, zlist, Spart, W, H, z0, z1, nchunks, st, dz_uniform, horner_mode);
  const int nz = z1 - z0;
  if (nz <= 0) return cudaSuccess;
  GPlan p;
  if (!gplan_make(H, &p)) return cudaErrorInvalidValue;
  cudaError_t e;
  const float2* tw = gtwiddles(H, st, &e);
  if (!tw) return e;
  const int C = gplan_lines(H, kGColsMax, kGColElems), logc = ilog2(C);
  const int strips = (W + C - 1) / C;
  const int zpb = (nz + nchunks - 1) / nchunks;
  const int chunks = (nz + zpb - 1) / zpb;
  if (chunks < nchunks) {  // unused chunk slots must read as zero
    e = cudaMemsetAsync(Spart + (size_t)chunks * H * W, 0, sizeof(float2) * (size_t)(nchunks - chunks) * H * W, st);
    if (e != cudaSuccess) return e;
  }
  const size_t smem = 2 * sizeof(float2) * (size_t)H * C;
  e = allow_smem(k_gfwd_col, smem);
  if (e != cudaSuccess) return e;
  k_gfwd_col<<<dim3(strips, chunks), kGThreads, smem, st>>>(p, tw, T, cturn, zlist, Spart, W, z0, z1, zpb, logc);
  return cudaGetLastError();
}

cudaError_t launch_plane_col(int inverse, const float2* in, float2* out, int W, int H, float scale,
                             cudaStream_t st) {
  if (fast_square(W, H)) return launch_plane_col_fast(inverse, in, out, W, H, scale, st);
  GPlan p;
  if (!gplan_make(H, &p)) return cudaErrorInvalidValue;
  cudaError_t e;
  const float2* tw = gtwiddles(H, st, &e);
  if (!tw) return e;
  const int C = gplan_lines(H, kGColsMax, kGColElems), logc = ilog2(C);
  const int strips = (W + C - 1) / C;
  const size_t smem = 2 * sizeof(float2) * (size_t)H * C;
  if (inverse) {
    e = allow_smem(k_gplane_col<true>, smem);
    if (e != cudaSuccess) return e;
    k_gplane_col<true><<<strips, kGThreads, smem, st>>>(p, tw, in, out, W, scale, logc);
  } else {
    e = allow_smem(k_gplane_col<false>, smem);
    if (e != cudaSuccess) return e;
    k_gplane_col<false><<<strips, kGThreads, smem, st>>>(p, tw, in, out, W, scale, logc);
  }
  return cudaGetLastError();
}

}  // namespace rihvr
