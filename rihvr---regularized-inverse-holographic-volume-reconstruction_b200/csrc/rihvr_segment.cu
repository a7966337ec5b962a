// Particle segmentation of a reconstructed volume: threshold, morphological
// closing, 26-connected labelling and per-object centroids.
//
// The reference runs this as a separate program on the voxel list that the
// reconstruction wrote (src/core/main_segmentation.cu:37-138): it loads
// x, y, z, |v|^2 from inverse_voxels_XXXX.csv as the complex value
// (sqrt(|v|^2), 0) (sparse_volume.cu:562-665), binarizes against a fraction of
// the largest intensity (sparse_segmentation.cu:61-112), closes with a ball of
// radius segment_close_size (dilate then erode, :186-372), labels the
// 26-connected components with the smallest linear index of each
// (:467-555), and makes one object per label in order of first appearance
// (object_cloud.cu:127-265) with its intensity-weighted centroid
// (object_cloud.cu:269-289, blob3d.cu getCentroid/getWeightedCentroid), drops
// objects under segment_min_area voxels by swapping in the last one
// (object_cloud.cu:313-328) and writes three centroid CSV files
// (object_cloud.cu:408-470).
//
// Here the same steps run on the dense volume in device memory:
//  * the voxel values are reduced to q = fl(fl(sqrt(I))^2) with I the
//    intensity the CSV would hold, which is what every step of the reference
//    computes from a loaded voxel; only the CSV's printing of I to seven
//    significant digits is skipped (rihvr_segment_intensity takes I as given,
//    so a CSV's values reproduce the reference's input exactly);
//  * the binary volumes are bit-packed, 32 voxels of a row per word, rows
//    padded to whole words; binarization packs with a warp ballot;
//  * dilation and erosion by the ball are word-parallel: for every (dz, dy)
//    of the ball, the row's bits shifted by -rx..rx (funnel shifts across the
//    neighbouring words) are OR-ed (dilation) or AND-ed (erosion).  This is
//    the reference's count test: a dilated voxel has a non-zero count, an
//    eroded one a count equal to the ball's size, where ball positions outside
//    the volume count nothing;
//  * labelling is a lock-free union-find in which every link points to a
//    smaller linear index, so each root is its component's smallest index,
//    the reference's label;
//  * object ids follow the order of the roots (an exclusive scan of per-word
//    root counts), which is the reference's order of first appearance; each
//    object's voxels are sorted by index and reduced by one thread in that
//    order, so the FP32 weighted sums round exactly as the reference's
//    sequential loops do.  The final divisions and the size filter run on the
//    host, in the reference's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rihvr.h"
#include "rihvr_kernels.cuh"

namespace rihvr {
namespace seg {

constexpr int kMaxClose = 15;                              // ball radius limit (shifts stay within one word)
constexpr int kMaxRows = (2 * kMaxClose + 1) * (2 * kMaxClose + 1);
__constant__ int c_rows[kMaxRows];                         // (dz + 64) << 16 | (dy + 64) << 8 | rx
constexpr int kMaxFind = 1 << 26;                          // pointer-chasing bound (error flag beyond)

struct Dims {
  int W, H, Nz, WW;       // WW: 32-bit words per row
  long long nwords;       // WW * H * Nz
  unsigned long long nvox;
};

// intensity as the reference's voxel file holds it, |v|^2 in FP32 without
// contraction (sparse_volume.cu:550), then the loaded value's square
// (sqrt(I) stored as the real part, :645-650)
__device__ __forceinline__ float q_from_intensity(float I) {
  const float s = sqrtf(I);
  return __fmul_rn(s, s);
}
__device__ __forceinline__ float q_at(const float2* v, size_t i) {
  const float2 a = v[i];
  return q_from_intensity(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)));
}
__device__ __forceinline__ float q_at(const float* v, size_t i) { return q_from_intensity(v[i]); }

// largest q (non-negative floats order like their bit patterns)
template <typename SRC>
__global__ void k_max_q(const SRC* __restrict__ src, unsigned long long n, unsigned* __restrict__ out_bits) {
  unsigned m = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(q_at(src, i)));
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, m);
}

// one warp per word: lane b holds voxel 32 w + b of the row; q > thr compared
// in FP64 as binarize_kernel does (sparse_segmentation.cu:39-49)
template <typename SRC>
__global__ void k_binarize(const SRC* __restrict__ src, Dims d, double thr, unsigned* __restrict__ bits) {
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = warp; w < d.nwords; w += nwarps) {
    const long long row = w / d.WW;
    const int x = (int)(w - row * d.WW) * 32 + lane;
    bool on = false;
    if (x < d.W) on = (double)q_at(src, (size_t)row * d.W + x) > thr;
    const unsigned b = __ballot_sync(0xffffffffu, on);
    if (lane == 0) bits[w] = b;
  }
}

__device__ __forceinline__ unsigned shifted(unsigned wm1, unsigned w0, unsigned wp1, int s) {
  // bit b of the result is bit b + s of the row (s may be negative)
  return s >= 0 ? __funnelshift_r(w0, wp1, s) : __funnelshift_l(wm1, w0, -s);
}

// One output word a thread.  DILATE: OR over the ball of the in-bounds input
// bits; otherwise (erosion) AND over the ball with out-of-bounds positions
// as 0.  Bits past the row's end stay 0.
template <bool DILATE>
__global__ void k_morph(const unsigned* __restrict__ in, unsigned* __restrict__ out, Dims d, int nrows) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < d.nwords;
       w += (long long)gridDim.x * blockDim.x) {
    const long long row = w / d.WW;
    const int wx = (int)(w - row * d.WW);
    const int y = (int)(row % d.H), z = (int)(row / d.H);
    unsigned acc = DILATE ? 0u : ~0u;
    for (int r = 0; r < nrows; ++r) {
      const int e = c_rows[r];
      const int dz = (e >> 16) - 64, dy = ((e >> 8) & 0xff) - 64, rx = e & 0xff;
      const int zz = z + dz, yy = y + dy;
      if (zz < 0 || zz >= d.Nz || yy < 0 || yy >= d.H) {
        if (DILATE) continue;
        acc = 0u;
        break;
      }
      const unsigned* rp = in + ((long long)zz * d.H + yy) * d.WW;
      const unsigned w0 = __ldg(rp + wx);
      const unsigned wm1 = wx > 0 ? __ldg(rp + wx - 1) : 0u;
      const unsigned wp1 = wx + 1 < d.WW ? __ldg(rp + wx + 1) : 0u;
      unsigned a = w0;
      for (int s = 1; s <= rx; ++s) {
        const unsigned l = shifted(wm1, w0, wp1, -s), h = shifted(wm1, w0, wp1, s);
        a = DILATE ? (a | l | h) : (a & l & h);
      }
      acc = DILATE ? (acc | a) : (acc & a);
      if (!DILATE && acc == 0u) break;
    }
    const int valid = d.W - wx * 32;
    if (valid < 32) acc &= (1u << valid) - 1u;
    out[w] = acc;
  }
}

__device__ __forceinline__ unsigned lab_ld(const unsigned* L, unsigned i) { return __ldcg(L + i); }

__device__ __forceinline__ unsigned find_root(const unsigned* L, unsigned x, int* err) {
  unsigned p = lab_ld(L, x);
  int n = 0;
  while (p != x) {
    x = p;
    p = lab_ld(L, x);
    if (++n > kMaxFind) {
      atomicExch(err, 1);
      break;
    }
  }
  return x;
}

// link the two trees; every link points to the smaller index
__device__ void unite(unsigned* L, unsigned a, unsigned b, int* err) {
  for (int n = 0; n < kMaxFind; ++n) {
    a = find_root(L, a, err);
    b = find_root(L, b, err);
    if (a == b) return;
    if (a < b) {
      const unsigned t = a;
      a = b;
      b = t;
    }
    const unsigned old = atomicMin(L + a, b);
    if (old == a) return;
    a = old;
  }
  atomicExch(err, 1);
}

__device__ __forceinline__ bool bit_at(const unsigned* bits, const Dims& d, int x, int y, int z) {
  const long long w = ((long long)z * d.H + y) * d.WW + (x >> 5);
  return (__ldg(bits + w) >> (x & 31)) & 1u;
}

// in-plane neighbour (x + dx, y + dy).  Reference neighbourhood (faithful):
// the linear offset dy W + dx inside the plane, so a step past a row's end
// continues on the next row (sparse_segmentation.cu:493-511); otherwise the
// geometric 3x3 neighbourhood.
__device__ __forceinline__ bool neighbour_xy(const Dims& d, int faithful, int x, int y, int dx, int dy, int* nx,
                                             int* ny) {
  if (faithful) {
    const long long l = (long long)(y + dy) * d.W + x + dx;
    if (l < 0 || l >= (long long)d.W * d.H) return false;
    *ny = (int)(l / d.W);
    *nx = (int)(l - (long long)*ny * d.W);
    return true;
  }
  *nx = x + dx;
  *ny = y + dy;
  return *nx >= 0 && *nx < d.W && *ny >= 0 && *ny < d.H;
}

template <int PHASE>  // 0: labels[i] = i; 1: unite with the 13 earlier neighbours; 2: labels[i] = root
__global__ void k_ccl(const unsigned* __restrict__ bits, unsigned* L, Dims d, int faithful, int* err) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < d.nwords;
       w += (long long)gridDim.x * blockDim.x) {
    unsigned m = bits[w];
    if (!m) continue;
    const long long row = w / d.WW;
    const int x0 = (int)(w - row * d.WW) * 32;
    const int y = (int)(row % d.H), z = (int)(row / d.H);
    const unsigned base = (unsigned)(row * d.W);
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      const int x = x0 + b;
      const unsigned i = base + (unsigned)x;
      if (PHASE == 0) {
        L[i] = i;
      } else if (PHASE == 2) {
        L[i] = find_root(L, i, err);
      } else {
#pragma unroll 1
        for (int dz = -1; dz <= 0; ++dz) {
          const int zz = z + dz;
          if (zz < 0) continue;
#pragma unroll 1
          for (int dy = -1; dy <= 1; ++dy)
#pragma unroll 1
            for (int dx = -1; dx <= 1; ++dx) {
              // earlier neighbours only: the plane below, or a negative in-plane offset
              if (dz == 0 && dy * d.W + dx >= 0) continue;
              int nx, ny;
              if (!neighbour_xy(d, faithful, x, y, dx, dy, &nx, &ny)) continue;
              if (!bit_at(bits, d, nx, ny, zz)) continue;
              unite(L, i, (unsigned)(((long long)zz * d.H + ny) * d.W + nx), err);
            }
        }
      }
    }
  }
}

// roots (labels[i] == i) as a bit volume, and their count a word
__global__ void k_roots(const unsigned* __restrict__ bits, const unsigned* __restrict__ L, Dims d,
                        unsigned* __restrict__ rbits, unsigned* __restrict__ rcount) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < d.nwords;
       w += (long long)gridDim.x * blockDim.x) {
    unsigned m = bits[w], r = 0;
    const long long row = w / d.WW;
    const unsigned base = (unsigned)(row * d.W) + (unsigned)(w - row * d.WW) * 32u;
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      if (L[base + b] == base + b) r |= 1u << b;
    }
    rbits[w] = r;
    rcount[w] = __popc(r);
  }
}

// object id of root r: roots before it in index order
__device__ __forceinline__ unsigned object_of(unsigned r, const Dims& d, const unsigned* rbits,
                                              const unsigned* roff) {
  const unsigned row = r / (unsigned)d.W;
  const unsigned x = r - row * (unsigned)d.W;
  const long long w = (long long)row * d.WW + (x >> 5);
  return roff[w] + __popc(rbits[w] & ((1u << (x & 31)) - 1u));
}

template <int PHASE>  // 0: count voxels per object; 1: scatter voxel indices
__global__ void k_objects(const unsigned* __restrict__ bits, const unsigned* __restrict__ L, Dims d,
                          const unsigned* __restrict__ rbits, const unsigned* __restrict__ roff,
                          unsigned* __restrict__ cnt, const unsigned* __restrict__ off,
                          unsigned* __restrict__ vox) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < d.nwords;
       w += (long long)gridDim.x * blockDim.x) {
    unsigned m = bits[w];
    const long long row = w / d.WW;
    const unsigned base = (unsigned)(row * d.W) + (unsigned)(w - row * d.WW) * 32u;
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      const unsigned i = base + b;
      const unsigned o = object_of(L[i], d, rbits, roff);
      const unsigned k = atomicAdd(cnt + o, 1u);
      if (PHASE == 1) vox[off[o] + k] = i;
    }
  }
}

struct ObjSums {
  long long sx, sy, sz;      // integer coordinate sums
  float wsx, wsy, wsz, wsum; // FP32 intensity-weighted sums, in index order
  float vmax;
  double vsum;               // FP64 sum of the intensities (std::accumulate with 0.0)
  int n, xmin, xmax, ymin, ymax, zmin, zmax;
};

// in-place heapsort of one object's voxel indices (distinct keys)
__device__ void heap_sort(unsigned* a, unsigned n) {
  auto sift = [&](unsigned i, unsigned end) {
    for (;;) {
      unsigned c = 2 * i + 1;
      if (c >= end) return;
      if (c + 1 < end && a[c + 1] > a[c]) ++c;
      if (a[i] >= a[c]) return;
      const unsigned t = a[i];
      a[i] = a[c];
      a[c] = t;
      i = c;
    }
  };
  if (n < 2) return;
  for (unsigned i = n / 2; i-- > 0;) sift(i, n);
  for (unsigned end = n - 1; end > 0; --end) {
    const unsigned t = a[0];
    a[0] = a[end];
    a[end] = t;
    sift(0, end);
  }
}

// One object a thread: sort its voxels, then the reference's sequential sums.
// The weight of a voxel is its q where the thresholded volume had it (the
// masked complex volume, sparse_segmentation.cu:51-59, 95-96), else 0
// (object_cloud.cu:269-289).
template <typename SRC>
__global__ void k_finish(const SRC* __restrict__ src, const unsigned* __restrict__ bits0, Dims d,
                         const unsigned* __restrict__ off, unsigned nobj, unsigned* __restrict__ vox,
                         ObjSums* __restrict__ out) {
  const unsigned o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nobj) return;
  unsigned* v = vox + off[o];
  const unsigned n = off[o + 1] - off[o];
  heap_sort(v, n);
  ObjSums s;
  s.sx = s.sy = s.sz = 0;
  s.wsx = s.wsy = s.wsz = s.wsum = 0.f;
  s.vsum = 0.0;
  s.n = (int)n;
  float vmax = 0.f;
  const unsigned HW = (unsigned)d.W * (unsigned)d.H;
  for (unsigned k = 0; k < n; ++k) {
    const unsigned i = v[k];
    const int z = (int)(i / HW);
    const unsigned p = i - (unsigned)z * HW;
    const int y = (int)(p / (unsigned)d.W), x = (int)(p - (unsigned)y * d.W);
    const long long w = ((long long)z * d.H + y) * d.WW + (x >> 5);
    const bool on = (bits0[w] >> (x & 31)) & 1u;
    const float q = on ? q_at(src, i) : 0.f;
    s.sx += x;
    s.sy += y;
    s.sz += z;
    s.wsx = __fadd_rn(s.wsx, __fmul_rn(q, (float)x));
    s.wsy = __fadd_rn(s.wsy, __fmul_rn(q, (float)y));
    s.wsz = __fadd_rn(s.wsz, __fmul_rn(q, (float)z));
    s.wsum = __fadd_rn(s.wsum, q);
    s.vsum = __dadd_rn(s.vsum, (double)q);
    vmax = (k == 0 || q > vmax) ? q : vmax;
    if (k == 0) {
      s.xmin = s.xmax = x;
      s.ymin = s.ymax = y;
      s.zmin = s.zmax = z;
    } else {
      s.xmin = min(s.xmin, x);
      s.xmax = max(s.xmax, x);
      s.ymin = min(s.ymin, y);
      s.ymax = max(s.ymax, y);
      s.zmin = min(s.zmin, z);
      s.zmax = max(s.zmax, z);
    }
  }
  s.vmax = vmax;
  out[o] = s;
}

// ---------------------------------------------------------------------------
// exclusive scan of unsigned counts (totals fit in 32 bits): blocks of
// kScanItems, block totals scanned recursively, then added back
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 512, kScanPer = 8, kScanItems = kScanThreads * kScanPer;

__global__ void k_scan_block(const unsigned* __restrict__ in, unsigned* __restrict__ out, long long n,
                             unsigned* __restrict__ block_sums) {
  __shared__ unsigned warp_tot[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kScanItems + (long long)threadIdx.x * kScanPer;
  unsigned v[kScanPer], t = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = base + k < n ? in[base + k] : 0u;
    t += v[k];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned incl = t;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    unsigned wt = lane < kScanThreads / 32 ? warp_tot[lane] : 0u, wi = wt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += u;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = wi - wt;
    if (lane == kScanThreads / 32 - 1 && block_sums) block_sums[blockIdx.x] = wi;
  }
  __syncthreads();
  unsigned run = warp_tot[wid] + incl - t;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
}

__global__ void k_scan_add(unsigned* __restrict__ out, long long n, const unsigned* __restrict__ block_offs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_offs[i / kScanItems];
}

}  // namespace seg
}  // namespace rihvr

using namespace rihvr;
using namespace rihvr::seg;

namespace {

int seg_fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

#define SCK(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return seg_fail(e_ == cudaErrorMemoryAllocation ? RIHVR_ERR_OUT_OF_MEMORY : RIHVR_ERR_CUDA,   \
                      std::string(#call) + ": " + cudaGetErrorString(e_));                         \
  } while (0)

// device buffers of one call, released on every return path
struct Buffers {
  std::vector<void*> ptrs;
  ~Buffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t count) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) ptrs.push_back(q);
    *p = static_cast<T*>(q);
    return e;
  }
};

int grid_for(long long items, int threads) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const long long want = (items + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(want, (long long)sms * 16));
}

// exclusive scan of n counts, out[n] = total (out has n + 1 entries)
int scan_exclusive(const unsigned* in, unsigned* out, long long n, Buffers& buf, cudaStream_t st,
                   long long* launches) {
  const long long nb = (n + kScanItems - 1) / kScanItems;
  unsigned* sums = nullptr;
  SCK(buf.alloc(&sums, (size_t)nb + 1));
  k_scan_block<<<(unsigned)std::max<long long>(nb, 1), kScanThreads, 0, st>>>(in, out, n, sums);
  SCK(cudaGetLastError());
  ++*launches;
  if (nb > 1) {
    unsigned* offs = nullptr;
    SCK(buf.alloc(&offs, (size_t)nb + 1));
    int rc = scan_exclusive(sums, offs, nb, buf, st, launches);
    if (rc != RIHVR_OK) return rc;
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, offs);
    SCK(cudaGetLastError());
    ++*launches;
    SCK(cudaMemcpyAsync(out + n, offs + nb, sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
  } else {
    SCK(cudaMemcpyAsync(out + n, sums, sizeof(unsigned), cudaMemcpyDeviceToDevice, st));
  }
  return RIHVR_OK;
}

// the ball's rows (dz, dy) with their half-width rx, and the ball's size
int ball_rows(int cs, std::vector<int>& rows, int* nstrel) {
  rows.clear();
  *nstrel = 0;
  for (int dz = -cs; dz <= cs; ++dz)
    for (int dy = -cs; dy <= cs; ++dy) {
      int rx = -1;
      for (int dx = 0; dx <= cs; ++dx)
        if (dx * dx + dy * dy + dz * dz <= cs * cs) rx = dx;
      if (rx < 0) continue;
      rows.push_back(((dz + 64) << 16) | ((dy + 64) << 8) | rx);
      *nstrel += 2 * rx + 1;
    }
  return (int)rows.size();
}

template <typename SRC>
int segment_impl(const SRC* src, int W, int H, int Nz, const rihvr_segment_params* sp, rihvr_object* objects,
                 int max_objects, int* num_objects, rihvr_segment_info* info, cudaStream_t st) {
  if (!sp || !num_objects || (max_objects > 0 && !objects) || max_objects < 0)
    return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL or negative argument");
  if (W <= 0 || H <= 0 || Nz <= 0) return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "volume dimensions must be positive");
  const unsigned long long nvox = (unsigned long long)W * H * Nz;
  if (nvox >= 0xffffffffull)
    return seg_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "volumes of 2^32 - 1 voxels or more are not supported (32-bit labels)");
  if (sp->close_size > kMaxClose)
    return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "close_size above " + std::to_string(kMaxClose));
  Dims d;
  d.W = W;
  d.H = H;
  d.Nz = Nz;
  d.WW = (W + 31) / 32;
  d.nwords = (long long)d.WW * H * Nz;
  d.nvox = nvox;
  long long launches = 0;
  Buffers buf;
  unsigned *maxbits, *bits0, *bits1, *bits2, *labels, *rbits, *rcount, *roff;
  int* err;
  SCK(buf.alloc(&maxbits, 1));
  SCK(buf.alloc(&err, 1));
  SCK(buf.alloc(&bits0, (size_t)d.nwords));
  SCK(buf.alloc(&bits1, (size_t)d.nwords));
  SCK(buf.alloc(&bits2, (size_t)d.nwords));
  SCK(buf.alloc(&labels, (size_t)nvox));
  SCK(buf.alloc(&rbits, (size_t)d.nwords));
  SCK(buf.alloc(&rcount, (size_t)d.nwords));
  SCK(buf.alloc(&roff, (size_t)d.nwords + 1));
  SCK(cudaMemsetAsync(maxbits, 0, sizeof(unsigned), st));
  SCK(cudaMemsetAsync(err, 0, sizeof(int), st));

  // binarize (sparse_segmentation.cu:61-112): thr = min_intensity * max / 256
  k_max_q<<<grid_for((long long)nvox, 256), 256, 0, st>>>(src, nvox, maxbits);
  SCK(cudaGetLastError());
  ++launches;
  unsigned mb = 0;
  SCK(cudaMemcpyAsync(&mb, maxbits, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  float maxq;
  std::memcpy(&maxq, &mb, sizeof(float));
  const double thr = sp->min_intensity * (double)maxq / 256.0;
  k_binarize<<<grid_for(d.nwords * 32, 256), 256, 0, st>>>(src, d, thr, bits0);
  SCK(cudaGetLastError());
  ++launches;

  // closing (:186-372): dilate then erode with the ball of radius close_size
  const unsigned* closed = bits0;
  int nstrel = 0;
  if (sp->close_size > 0) {
    std::vector<int> rows;
    const int nrows = ball_rows(sp->close_size, rows, &nstrel);
    SCK(cudaMemcpyToSymbolAsync(c_rows, rows.data(), sizeof(int) * nrows, 0, cudaMemcpyHostToDevice, st));
    k_morph<true><<<grid_for(d.nwords, 256), 256, 0, st>>>(bits0, bits1, d, nrows);
    SCK(cudaGetLastError());
    k_morph<false><<<grid_for(d.nwords, 256), 256, 0, st>>>(bits1, bits2, d, nrows);
    SCK(cudaGetLastError());
    launches += 2;
    closed = bits2;
  }

  // 26-connected labels, smallest linear index of each component (:467-555)
  const int gw = grid_for(d.nwords, 256);
  k_ccl<0><<<gw, 256, 0, st>>>(closed, labels, d, sp->faithful, err);
  SCK(cudaGetLastError());
  k_ccl<1><<<gw, 256, 0, st>>>(closed, labels, d, sp->faithful, err);
  SCK(cudaGetLastError());
  k_ccl<2><<<gw, 256, 0, st>>>(closed, labels, d, sp->faithful, err);
  SCK(cudaGetLastError());
  k_roots<<<gw, 256, 0, st>>>(closed, labels, d, rbits, rcount);
  SCK(cudaGetLastError());
  launches += 4;
  int rc = scan_exclusive(rcount, roff, d.nwords, buf, st, &launches);
  if (rc != RIHVR_OK) return rc;
  unsigned nobj = 0;
  int herr = 0;
  SCK(cudaMemcpyAsync(&nobj, roff + d.nwords, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SCK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  if (herr) return seg_fail(RIHVR_ERR_INFINITE_LOOP, "connected-component labelling exceeded its iteration bound");

  // objects in root order, each reduced over its voxels in index order
  std::vector<ObjSums> sums(nobj);
  unsigned nclosed = 0;
  if (nobj > 0) {
    unsigned *cnt, *off, *vox;
    ObjSums* osum;
    SCK(buf.alloc(&cnt, nobj));
    SCK(buf.alloc(&off, (size_t)nobj + 1));
    SCK(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * nobj, st));
    k_objects<0><<<gw, 256, 0, st>>>(closed, labels, d, rbits, roff, cnt, nullptr, nullptr);
    SCK(cudaGetLastError());
    ++launches;
    rc = scan_exclusive(cnt, off, nobj, buf, st, &launches);
    if (rc != RIHVR_OK) return rc;
    SCK(cudaMemcpyAsync(&nclosed, off + nobj, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    SCK(buf.alloc(&vox, nclosed));
    SCK(buf.alloc(&osum, nobj));
    SCK(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * nobj, st));
    k_objects<1><<<gw, 256, 0, st>>>(closed, labels, d, rbits, roff, cnt, off, vox);
    SCK(cudaGetLastError());
    k_finish<<<(nobj + 127) / 128, 128, 0, st>>>(src, bits0, d, off, nobj, vox, osum);
    SCK(cudaGetLastError());
    launches += 2;
    SCK(cudaMemcpyAsync(sums.data(), osum, sizeof(ObjSums) * nobj, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
  }

  // Blob3d::getCentroid / getWeightedCentroid / getMaxValue / getMeanValue /
  // getBounds (blob3d.cu), then ObjectCloud::blobSizeFilter (object_cloud.cu:313-328)
  std::vector<rihvr_object> objs(nobj);
  for (unsigned o = 0; o < nobj; ++o) {
    const ObjSums& s = sums[o];
    rihvr_object& r = objs[o];
    const float n = (float)s.n;
    r.x = (float)s.sx / n;
    r.y = (float)s.sy / n;
    r.z = (float)s.sz / n;
    r.wx = s.wsx / s.wsum;
    r.wy = s.wsy / s.wsum;
    r.wz = s.wsz / s.wsum;
    r.num_voxels = s.n;
    r.max_value = s.vmax;
    r.mean_value = (float)s.vsum / n;
    r.xmin = s.xmin;
    r.xmax = s.xmax;
    r.ymin = s.ymin;
    r.ymax = s.ymax;
    r.zmin = s.zmin;
    r.zmax = s.zmax;
  }
  long long kept = nobj;
  for (long long n = 0; n < kept; ++n)
    if (objs[n].num_voxels < sp->min_area) {
      objs[n] = objs[kept - 1];
      --n;
      --kept;
    }
  if (info) {
    info->max_intensity = (double)maxq;
    info->threshold = thr;
    info->closed_voxels = nclosed;
    info->labelled_objects = nobj;
    info->strel_size = nstrel;
    info->kernel_launches = launches;
  }
  *num_objects = (int)kept;
  if (kept > max_objects)
    return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, std::to_string(kept) + " objects do not fit in " +
                                                    std::to_string(max_objects) + " entries");
  std::copy(objs.begin(), objs.begin() + kept, objects);
  return RIHVR_OK;
}

}  // namespace

namespace rihvr {
int segment_complex(const float2* vol, int W, int H, int Nz, const rihvr_segment_params* sp, rihvr_object* objects,
                    int max_objects, int* num_objects, rihvr_segment_info* info, cudaStream_t st) {
  return segment_impl(vol, W, H, Nz, sp, objects, max_objects, num_objects, info, st);
}
}  // namespace rihvr

extern "C" {

int rihvr_segment_params_default(rihvr_segment_params* sp) {
  if (!sp) return RIHVR_ERR_INVALID_ARGUMENT;
  // HoloUi::HoloUi (holo_ui.cpp:44-46)
  sp->min_intensity = 1.0;
  sp->close_size = 3;
  sp->min_area = 2;
  sp->faithful = 1;
  return RIHVR_OK;
}

int rihvr_segment_intensity(const float* intensity, int width, int height, int num_planes, int is_device,
                            const rihvr_segment_params* sp, rihvr_object* objects, int max_objects,
                            int* num_objects, rihvr_segment_info* info) {
  if (!intensity) return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL intensity");
  if (width <= 0 || height <= 0 || num_planes <= 0)
    return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "volume dimensions must be positive");
  // the legacy default stream: ordered after work the caller queued on other
  // blocking streams (such as the one that produced a device-resident input)
  cudaStream_t st = nullptr;
  const float* src = intensity;
  float* staged = nullptr;
  const size_t bytes = sizeof(float) * (size_t)width * height * num_planes;
  int rc = RIHVR_OK;
  if (!is_device) {
    cudaError_t e = cudaMalloc(&staged, bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(staged, intensity, bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) rc = seg_fail(RIHVR_ERR_CUDA, std::string("staging the intensities: ") + cudaGetErrorString(e));
    src = staged;
  }
  if (rc == RIHVR_OK)
    rc = segment_impl(src, width, height, num_planes, sp, objects, max_objects, num_objects, info, st);
  cudaStreamSynchronize(st);
  if (staged) cudaFree(staged);
  return rc;
}

int rihvr_write_centroids(const char* filename, const rihvr_object* objects, int n, int weighted, int verbose) {
  if (!filename || (n > 0 && !objects) || n < 0) return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "bad argument");
  // ObjectCloud::writeCentroids (object_cloud.cu:408-470)
  FILE* f = std::fopen(filename, "w");
  if (!f) return seg_fail(RIHVR_ERR_BAD_FILENAME, std::string("Unable to open file: ") + filename);
  if (!verbose) {
    std::fprintf(f, "x (pixels), y (pixels), z (planes), # of voxels\n");
  } else {
    std::fprintf(f, "x (pixels), y (pixels), z (planes), weighted x, weighted y, weighted z, # of voxels, "
                    "max value, mean value, xmin, xmax, ymin, ymax, zmin, zmax\n");
  }
  for (int i = 0; i < n; ++i) {
    const rihvr_object& o = objects[i];
    if (!verbose) {
      if (weighted)
        std::fprintf(f, "%f, %f, %f, %d\n", o.wx, o.wy, o.wz, o.num_voxels);
      else
        std::fprintf(f, "%f, %f, %f, %d\n", o.x, o.y, o.z, o.num_voxels);
    } else {
      std::fprintf(f, "%f, %f, %f, %f, %f, %f, %d, %e, %e, %d, %d, %d, %d, %d, %d\n", o.x, o.y, o.z, o.wx, o.wy,
                   o.wz, o.num_voxels, o.max_value, o.mean_value, o.xmin, o.xmax, o.ymin, o.ymax, o.zmin, o.zmax);
    }
  }
  std::fclose(f);
  return RIHVR_OK;
}

}  // extern "C"
