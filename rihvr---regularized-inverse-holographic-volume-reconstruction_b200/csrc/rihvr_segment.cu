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
//    so a CSV's values reproduce the reference's input exactly).  The
//    solver's volume is read in place, x = P + beta (P - Pprev) formed per
//    voxel as the solver forms it;
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
//  * labels live in rank space (one entry per voxel that is on after the
//    closing, numbered in index order), so memory follows the particles, not
//    the volume;
//  * object ids follow the order of the roots (an exclusive scan of root
//    flags), which is the reference's order of first appearance; a stable
//    radix sort (CUB) on the object id puts each object's voxels together in
//    index order, and one thread per object reduces them in that order, so
//    the FP32 weighted sums round exactly as the reference's sequential loops
//    do.  The final divisions and the size filter run on the host, in the
//    reference's order.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/rihvr.h"
#include "rihvr_device.cuh"
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
__device__ __forceinline__ float q_from_value(float2 a) {
  return q_from_intensity(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)));
}

// Voxel sources.  IntensitySrc: the intensities of a voxel file.  VolumeSrc:
// the solver's volume x = P + beta (P - Pprev), formed on the fly as the
// solver forms it, in the storage type of P.
struct IntensitySrc {
  const float* I;
  __device__ __forceinline__ float q(size_t i) const { return q_from_intensity(__ldg(I + i)); }
};
// q values already formed (stored by the max pass)
struct QSrc {
  const float* q_;
  __device__ __forceinline__ float q(size_t i) const { return __ldg(q_ + i); }
};
template <typename ST>
struct VolumeSrc {
  const ST* P;
  const ST* Pp;
  float beta;
  __device__ __forceinline__ float q(size_t i) const { return q_from_value(xval(P, Pp, beta, i)); }
};

// largest q (non-negative floats order like their bit patterns); four
// independent loads a thread in flight
// (qout, when given, receives every q for the threshold pass)
template <typename SRC>
__global__ void k_max_q(SRC src, unsigned long long n, unsigned* __restrict__ out_bits, float* __restrict__ qout) {
  unsigned m = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    const float a = src.q(i), b = src.q(i + stride), c = src.q(i + 2 * stride), e = src.q(i + 3 * stride);
    if (qout) {
      qout[i] = a;
      qout[i + stride] = b;
      qout[i + 2 * stride] = c;
      qout[i + 3 * stride] = e;
    }
    m = max(m, max(max(__float_as_uint(a), __float_as_uint(b)), max(__float_as_uint(c), __float_as_uint(e))));
  }
  for (; i < n; i += stride) {
    const float a = src.q(i);
    if (qout) qout[i] = a;
    m = max(m, __float_as_uint(a));
  }
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, m);
}

// A warp makes eight words at a time (eight loads a lane in flight): lane b
// holds voxel 32 w + b of its row; q > thr compared in FP64 as binarize_kernel
// does (sparse_segmentation.cu:39-49).  Rows with a voxel on are flagged for
// the morphology.
template <typename SRC>
__global__ void k_binarize(SRC src, Dims d, double thr, unsigned* __restrict__ bits,
                           unsigned char* __restrict__ row_on) {
  constexpr int U = 8;
  const int lane = threadIdx.x & 31;
  const unsigned nw = (unsigned)d.nwords, WW = (unsigned)d.WW;  // indices fit in 32 bits
  const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  for (unsigned w0 = warp * U; w0 < nw; w0 += nwarps * U) {
    float q[U];
    unsigned row[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const unsigned w = w0 + k;
      row[k] = w / WW;
      const int x = (int)(w - row[k] * WW) * 32 + lane;
      q[k] = (w < nw && x < d.W) ? src.q((size_t)row[k] * d.W + x) : -1.f;
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const unsigned b = __ballot_sync(0xffffffffu, q[k] >= 0.f && (double)q[k] > thr);
      const unsigned w = w0 + k;
      if (lane == 0 && w < nw) {
        bits[w] = b;
        if (b) row_on[row[k]] = 1;
      }
    }
  }
}

__device__ __forceinline__ unsigned shifted(unsigned wm1, unsigned w0, unsigned wp1, int s) {
  // bit b of the result is bit b + s of the row (s may be negative)
  return s >= 0 ? __funnelshift_r(w0, wp1, s) : __funnelshift_l(wm1, w0, -s);
}

// One warp per 32 consecutive words of a row; lane l makes word 32 c + l.
// DILATE: OR over the ball of the in-bounds input bits; otherwise (erosion)
// AND over the ball with out-of-bounds positions as 0.  Bits past the row's
// end stay 0.  The ball's rows are taken 32 at a time: each lane looks up
// one row's flag (row_in: the row has a voxel on), a ballot gives the warp the
// rows to visit; the dilation visits only those, the erosion ends at 0 when
// any is missing.  Rows of the output with a voxel on are flagged in row_out.
template <bool DILATE>
__global__ void k_morph(const unsigned* __restrict__ in, unsigned* __restrict__ out, Dims d, int nrows,
                        const unsigned char* __restrict__ row_in, unsigned char* __restrict__ row_out) {
  const int lane = threadIdx.x & 31;
  const unsigned WW = (unsigned)d.WW, Hu = (unsigned)d.H;  // 32-bit indices
  const unsigned chunks = (WW + 31) / 32;
  const unsigned ntask = (unsigned)d.H * (unsigned)d.Nz * chunks;
  const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
  for (unsigned task = warp; task < ntask; task += nwarps) {
    const unsigned row = task / chunks;
    const int wx = (int)(task - row * chunks) * 32 + lane;
    const unsigned zu = row / Hu;
    const int y = (int)(row - zu * Hu), z = (int)zu;
    unsigned acc = DILATE ? 0u : ~0u;
    bool zero = false;
    for (int r0 = 0; r0 < nrows && !zero; r0 += 32) {
      const int r = r0 + lane;
      bool live = false;
      if (r < nrows) {
        const int e = c_rows[r];
        const int zz = z + (e >> 16) - 64, yy = y + ((e >> 8) & 0xff) - 64;
        live = zz >= 0 && zz < d.Nz && yy >= 0 && yy < d.H && __ldg(row_in + (unsigned)zz * Hu + yy);
      }
      unsigned mask = __ballot_sync(0xffffffffu, live);
      const int nin = min(32, nrows - r0);
      if (!DILATE && mask != (nin == 32 ? 0xffffffffu : (1u << nin) - 1u)) {
        zero = true;
        break;
      }
      for (; mask; mask &= mask - 1) {
        const int e = c_rows[r0 + __ffs(mask) - 1];
        const int zz = z + (e >> 16) - 64, yy = y + ((e >> 8) & 0xff) - 64, rx = e & 0xff;
        if (wx >= d.WW) continue;
        const unsigned* rp = in + ((unsigned)zz * Hu + yy) * WW;
        const unsigned w0 = __ldg(rp + wx);
        const unsigned wm1 = wx > 0 ? __ldg(rp + wx - 1) : 0u;
        const unsigned wp1 = wx + 1 < d.WW ? __ldg(rp + wx + 1) : 0u;
        unsigned a = w0;
        for (int s = 1; s <= rx; ++s) {
          const unsigned l = shifted(wm1, w0, wp1, -s), h = shifted(wm1, w0, wp1, s);
          a = DILATE ? (a | l | h) : (a & l & h);
        }
        acc = DILATE ? (acc | a) : (acc & a);
      }
    }
    if (zero) acc = 0u;
    if (wx < d.WW) {
      const int valid = d.W - wx * 32;
      if (valid < 32) acc &= (1u << valid) - 1u;
      out[row * WW + wx] = acc;
    }
    if (__any_sync(0xffffffffu, wx < d.WW && acc != 0u) && lane == 0) row_out[row] = 1;
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

// rank of an on voxel among all on voxels in index order: the on-voxel count
// of the words before it plus the bits below it in its word
__device__ __forceinline__ unsigned rank_at(const unsigned* bits, const unsigned* onoff, const Dims& d, int x,
                                            int y, int z, bool* on) {
  const unsigned w = ((unsigned)z * (unsigned)d.H + (unsigned)y) * (unsigned)d.WW + (unsigned)(x >> 5);
  const unsigned m = __ldg(bits + w);
  *on = (m >> (x & 31)) & 1u;
  return __ldg(onoff + w) + __popc(m & ((1u << (x & 31)) - 1u));
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

// Labels live in rank space (one entry per on voxel, in index order), so a
// smaller rank is a smaller linear index and each root is its component's
// smallest index.
__global__ void k_label_init(unsigned* __restrict__ L, unsigned m) {
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) L[r] = r;
}

// linear index of every on voxel, by rank
__global__ void k_rank_index(const unsigned* __restrict__ bits, const unsigned* __restrict__ onoff, Dims d,
                             unsigned* __restrict__ idx) {
  const unsigned nw = (unsigned)d.nwords, WW = (unsigned)d.WW;
  for (unsigned w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += gridDim.x * blockDim.x) {
    unsigned m = bits[w];
    if (!m) continue;
    const unsigned row = w / WW;
    const unsigned base = row * (unsigned)d.W + (w - row * WW) * 32u;
    for (unsigned r = onoff[w]; m; m &= m - 1, ++r) idx[r] = base + (unsigned)(__ffs(m) - 1);
  }
}

// union of every on voxel (one thread each) with its 13 earlier neighbours
// (the plane below, or a negative in-plane offset).  When the voxel before it
// in the row (offset -1) is on, the neighbours the two share are already
// joined to that voxel by its own thread, and only the 4 on the far side
// (dx = +1: one in the plane, three below) remain.
__global__ void k_label_merge(const unsigned* __restrict__ bits, const unsigned* __restrict__ onoff,
                              const unsigned* __restrict__ idx, unsigned* L, unsigned m, Dims d, int faithful,
                              int* err) {
  const unsigned HW = (unsigned)d.W * (unsigned)d.H;
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const unsigned i = idx[r];
    const int z = (int)(i / HW);
    const unsigned pl = i - (unsigned)z * HW;
    const int y = (int)(pl / (unsigned)d.W), x = (int)(pl - (unsigned)y * d.W);
    int nx, ny;
    bool left = false;
    if (neighbour_xy(d, faithful, x, y, -1, 0, &nx, &ny)) {
      const unsigned rl = rank_at(bits, onoff, d, nx, ny, z, &left);
      if (left) unite(L, r, rl, err);
    }
#pragma unroll 1
    for (int dz = -1; dz <= 0; ++dz) {
      const int zz = z + dz;
      if (zz < 0) continue;
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          if (dz == 0 && (dy * d.W + dx >= 0 || (dy == 0 && dx == -1))) continue;  // later, or the left one
          if (left && dx != 1) continue;
          if (!neighbour_xy(d, faithful, x, y, dx, dy, &nx, &ny)) continue;
          bool on;
          const unsigned rj = rank_at(bits, onoff, d, nx, ny, zz, &on);
          if (on) unite(L, r, rj, err);
        }
    }
  }
}

// labels to roots; root flags for the object numbering
__global__ void k_label_flatten(unsigned* L, unsigned m, unsigned* __restrict__ is_root, int* err) {
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const unsigned root = find_root(L, r, err);
    L[r] = root;
    is_root[r] = root == r;
  }
}

// object of every on voxel (the number of roots before its root), its rank
// as the sort value, and the voxel counts per object
__global__ void k_object_keys(const unsigned* __restrict__ L, const unsigned* __restrict__ root_rank, unsigned m,
                              unsigned* __restrict__ key, unsigned* __restrict__ val, unsigned* __restrict__ cnt) {
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const unsigned o = root_rank[L[r]];
    key[r] = o;
    val[r] = r;
    atomicAdd(cnt + o, 1u);
  }
}

__global__ void k_popc(const unsigned* __restrict__ bits, unsigned* __restrict__ cnt, long long n) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x)
    cnt[w] = __popc(bits[w]);
}

struct ObjSums {
  long long sx, sy, sz;      // integer coordinate sums
  float wsx, wsy, wsz, wsum; // FP32 intensity-weighted sums, in index order
  float vmax;
  double vsum;               // FP64 sum of the intensities (std::accumulate with 0.0)
  int n, xmin, xmax, ymin, ymax, zmin, zmax;
};

// Voxels sorted by (object, index): their coordinates and weights, in that
// order.  The weight of a voxel is its q where the thresholded volume had it
// (the masked complex volume, sparse_segmentation.cu:51-59, 95-96), else 0
// (object_cloud.cu:269-289).
template <typename SRC>
__global__ void k_gather(SRC src, const unsigned* __restrict__ bits0, Dims d,
                         const unsigned* __restrict__ idx, const unsigned* __restrict__ sorted_rank, unsigned m,
                         int4* __restrict__ rec) {
  const unsigned HW = (unsigned)d.W * (unsigned)d.H;
  for (unsigned j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const unsigned i = idx[sorted_rank[j]];
    const int z = (int)(i / HW);
    const unsigned pl = i - (unsigned)z * HW;
    const int y = (int)(pl / (unsigned)d.W), x = (int)(pl - (unsigned)y * d.W);
    const long long w = ((long long)z * d.H + y) * d.WW + (x >> 5);
    const bool on = (bits0[w] >> (x & 31)) & 1u;
    rec[j] = make_int4(x, y, z, __float_as_int(on ? src.q(i) : 0.f));
  }
}

// One object a thread, over its voxels in index order: the reference's
// sequential sums (Blob3d::getCentroid, getWeightedCentroid, getMaxValue,
// getMeanValue, findBounds).
__global__ void k_finish(const int4* __restrict__ rec, const unsigned* __restrict__ off, unsigned nobj,
                         ObjSums* __restrict__ out) {
  const unsigned o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nobj) return;
  const unsigned j0 = off[o], j1 = off[o + 1];
  ObjSums s;
  s.sx = s.sy = s.sz = 0;
  s.wsx = s.wsy = s.wsz = s.wsum = 0.f;
  s.vsum = 0.0;
  s.n = (int)(j1 - j0);
  const int4 f = rec[j0];
  s.xmin = s.xmax = f.x;
  s.ymin = s.ymax = f.y;
  s.zmin = s.zmax = f.z;
  float vmax = __int_as_float(f.w);
  for (unsigned j = j0; j < j1; ++j) {
    const int4 e = rec[j];
    const int x = e.x, y = e.y, z = e.z;
    const float q = __int_as_float(e.w);
    s.sx += x;
    s.sy += y;
    s.sz += z;
    s.wsx = __fadd_rn(s.wsx, __fmul_rn(q, (float)x));
    s.wsy = __fadd_rn(s.wsy, __fmul_rn(q, (float)y));
    s.wsz = __fadd_rn(s.wsz, __fmul_rn(q, (float)z));
    s.wsum = __fadd_rn(s.wsum, q);
    s.vsum = __dadd_rn(s.vsum, (double)q);
    vmax = q > vmax ? q : vmax;
    s.xmin = min(s.xmin, x);
    s.xmax = max(s.xmax, x);
    s.ymin = min(s.ymin, y);
    s.ymax = max(s.ymax, y);
    s.zmin = min(s.zmin, z);
    s.zmax = max(s.zmax, z);
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

}  // namespace

namespace rihvr {
// Device buffers of the segmentation, kept between calls and grown on demand:
// a context owns one, so repeated segmentations allocate nothing after the
// first; a standalone call uses a temporary one.
struct SegWorkspace {
  static constexpr int kSlots = 32;
  void* p[kSlots] = {};
  size_t cap[kSlots] = {};
  int device = -1;
  ~SegWorkspace() {
    for (void* q : p)
      if (q) cudaFree(q);
  }
  template <typename T>
  cudaError_t get(int slot, T** out, size_t count) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (cap[slot] < bytes) {
      if (p[slot]) cudaFree(p[slot]);
      p[slot] = nullptr;
      cap[slot] = 0;
      const cudaError_t e = cudaMalloc(&p[slot], bytes);
      if (e != cudaSuccess) return e;
      cap[slot] = bytes;
    }
    *out = static_cast<T*>(p[slot]);
    return cudaSuccess;
  }
};
SegWorkspace* seg_workspace_create() { return new SegWorkspace(); }
void seg_workspace_destroy(SegWorkspace* ws) { delete ws; }
}  // namespace rihvr

namespace {

enum Slot { S_MAX, S_ERR, S_Q, S_BITS0, S_BITS1, S_BITS2, S_ROW0, S_ROW1, S_ROW2, S_ONCNT, S_ONOFF, S_IDX, S_LAB, S_ROOT, S_RRANK, S_CNT,
            S_OFF, S_KEY, S_VAL, S_KEY_S, S_VAL_S, S_REC, S_SUMS, S_SORT_TMP,
            S_SCAN0 };  // S_SCAN0.. : block sums of the scan levels

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
int scan_exclusive(const unsigned* in, unsigned* out, long long n, SegWorkspace& ws, int level, cudaStream_t st,
                   long long* launches) {
  if (S_SCAN0 + 2 * level + 1 >= SegWorkspace::kSlots) return seg_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "scan too deep");
  const long long nb = (n + kScanItems - 1) / kScanItems;
  unsigned* sums = nullptr;
  SCK(ws.get(S_SCAN0 + 2 * level, &sums, (size_t)nb + 1));
  k_scan_block<<<(unsigned)std::max<long long>(nb, 1), kScanThreads, 0, st>>>(in, out, n, sums);
  SCK(cudaGetLastError());
  ++*launches;
  if (nb > 1) {
    unsigned* offs = nullptr;
    SCK(ws.get(S_SCAN0 + 2 * level + 1, &offs, (size_t)nb + 1));
    const int rc = scan_exclusive(sums, offs, nb, ws, level + 1, st, launches);
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
int segment_impl(SRC src, int W, int H, int Nz, const rihvr_segment_params* sp, rihvr_object* objects,
                 int max_objects, int* num_objects, rihvr_segment_info* info, SegWorkspace& ws, cudaStream_t st) {
  if (!sp || !num_objects || (max_objects > 0 && !objects) || max_objects < 0)
    return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL or negative argument");
  if (W <= 0 || H <= 0 || Nz <= 0) return seg_fail(RIHVR_ERR_INVALID_ARGUMENT, "volume dimensions must be positive");
  const unsigned long long nvox = (unsigned long long)W * H * Nz;
  if (nvox >= 0xffffffffull)
    return seg_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "volumes of 2^32 - 1 voxels or more are not supported (32-bit indices)");
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
  unsigned *maxbits, *bits0, *bits1, *bits2, *oncnt, *onoff;
  int* err;
  SCK(ws.get(S_MAX, &maxbits, 1));
  SCK(ws.get(S_ERR, &err, 1));
  SCK(ws.get(S_BITS0, &bits0, (size_t)d.nwords));
  SCK(ws.get(S_BITS1, &bits1, (size_t)d.nwords));
  SCK(ws.get(S_BITS2, &bits2, (size_t)d.nwords));
  SCK(ws.get(S_ONCNT, &oncnt, (size_t)d.nwords));
  SCK(ws.get(S_ONOFF, &onoff, (size_t)d.nwords + 1));
  unsigned char *row0, *row1, *row2;
  const size_t nrows_vol = (size_t)H * Nz;
  SCK(ws.get(S_ROW0, &row0, nrows_vol));
  SCK(ws.get(S_ROW1, &row1, nrows_vol));
  SCK(ws.get(S_ROW2, &row2, nrows_vol));
  SCK(cudaMemsetAsync(row0, 0, nrows_vol, st));
  SCK(cudaMemsetAsync(row1, 0, nrows_vol, st));
  SCK(cudaMemsetAsync(row2, 0, nrows_vol, st));
  SCK(cudaMemsetAsync(maxbits, 0, sizeof(unsigned), st));
  SCK(cudaMemsetAsync(err, 0, sizeof(int), st));

  // binarize (sparse_segmentation.cu:61-112): thr = min_intensity * max / 256.
  // A volume source's q values are kept from the max pass (4 bytes a voxel
  // instead of reading P and Pprev again); intensities are read directly.
  constexpr bool kStoreQ = !std::is_same<SRC, IntensitySrc>::value;
  float* qbuf = nullptr;
  if (kStoreQ) SCK(ws.get(S_Q, &qbuf, (size_t)nvox));
  k_max_q<<<grid_for((long long)nvox, 256), 256, 0, st>>>(src, nvox, maxbits, qbuf);
  SCK(cudaGetLastError());
  ++launches;
  unsigned mb = 0;
  SCK(cudaMemcpyAsync(&mb, maxbits, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  float maxq;
  std::memcpy(&maxq, &mb, sizeof(float));
  const double thr = sp->min_intensity * (double)maxq / 256.0;
  if (kStoreQ)
    k_binarize<<<grid_for(d.nwords * 4, 256), 256, 0, st>>>(QSrc{qbuf}, d, thr, bits0, row0);
  else
    k_binarize<<<grid_for(d.nwords * 4, 256), 256, 0, st>>>(src, d, thr, bits0, row0);
  SCK(cudaGetLastError());
  ++launches;

  // closing (:186-372): dilate then erode with the ball of radius close_size
  const unsigned* closed = bits0;
  int nstrel = 0;
  const int gw = grid_for(d.nwords, 256);
  if (sp->close_size > 0) {
    std::vector<int> rows;
    const int nrows = ball_rows(sp->close_size, rows, &nstrel);
    SCK(cudaMemcpyToSymbolAsync(c_rows, rows.data(), sizeof(int) * nrows, 0, cudaMemcpyHostToDevice, st));
    const long long mtasks = (long long)H * Nz * ((d.WW + 31) / 32);
    k_morph<true><<<grid_for(mtasks * 32, 256), 256, 0, st>>>(bits0, bits1, d, nrows, row0, row1);
    SCK(cudaGetLastError());
    k_morph<false><<<grid_for(mtasks * 32, 256), 256, 0, st>>>(bits1, bits2, d, nrows, row1, row2);
    SCK(cudaGetLastError());
    launches += 2;
    closed = bits2;
  }

  // on voxels in index order (their ranks), then 26-connected labels in rank
  // space: each root is its component's smallest index (:467-555)
  k_popc<<<gw, 256, 0, st>>>(closed, oncnt, d.nwords);
  SCK(cudaGetLastError());
  ++launches;
  int rc = scan_exclusive(oncnt, onoff, d.nwords, ws, 0, st, &launches);
  if (rc != RIHVR_OK) return rc;
  unsigned non = 0;
  SCK(cudaMemcpyAsync(&non, onoff + d.nwords, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SCK(cudaStreamSynchronize(st));
  unsigned nobj = 0;
  std::vector<ObjSums> sums;
  if (non > 0) {
    unsigned *idx, *lab, *is_root, *root_rank, *cnt, *off, *key, *val, *key_s, *val_s;
    int4* rec;
    ObjSums* osum;
    SCK(ws.get(S_IDX, &idx, non));
    SCK(ws.get(S_LAB, &lab, non));
    SCK(ws.get(S_ROOT, &is_root, non));
    SCK(ws.get(S_RRANK, &root_rank, (size_t)non + 1));
    const int gm = grid_for(non, 256);
    k_rank_index<<<gw, 256, 0, st>>>(closed, onoff, d, idx);
    SCK(cudaGetLastError());
    k_label_init<<<gm, 256, 0, st>>>(lab, non);
    SCK(cudaGetLastError());
    k_label_merge<<<gm, 256, 0, st>>>(closed, onoff, idx, lab, non, d, sp->faithful, err);
    SCK(cudaGetLastError());
    k_label_flatten<<<gm, 256, 0, st>>>(lab, non, is_root, err);
    SCK(cudaGetLastError());
    launches += 4;
    rc = scan_exclusive(is_root, root_rank, non, ws, 0, st, &launches);
    if (rc != RIHVR_OK) return rc;
    int herr = 0;
    SCK(cudaMemcpyAsync(&nobj, root_rank + non, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SCK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    if (herr) return seg_fail(RIHVR_ERR_INFINITE_LOOP, "connected-component labelling exceeded its iteration bound");

    // voxels ordered by (object, index): a stable radix sort on the object id
    // of voxels listed in index order; then each object is reduced in order
    SCK(ws.get(S_CNT, &cnt, nobj));
    SCK(ws.get(S_OFF, &off, (size_t)nobj + 1));
    SCK(ws.get(S_KEY, &key, non));
    SCK(ws.get(S_VAL, &val, non));
    SCK(ws.get(S_KEY_S, &key_s, non));
    SCK(ws.get(S_VAL_S, &val_s, non));
    SCK(ws.get(S_REC, &rec, non));
    SCK(ws.get(S_SUMS, &osum, nobj));
    SCK(cudaMemsetAsync(cnt, 0, sizeof(unsigned) * nobj, st));
    k_object_keys<<<gm, 256, 0, st>>>(lab, root_rank, non, key, val, cnt);
    SCK(cudaGetLastError());
    ++launches;
    rc = scan_exclusive(cnt, off, nobj, ws, 0, st, &launches);
    if (rc != RIHVR_OK) return rc;
    int end_bit = 1;
    while (end_bit < 32 && (nobj >> end_bit) != 0) ++end_bit;
    size_t tmp_bytes = 0;
    SCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key_s, val, val_s, (int)non, 0, end_bit, st));
    unsigned char* tmp = nullptr;
    SCK(ws.get(S_SORT_TMP, &tmp, tmp_bytes));
    SCK(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key_s, val, val_s, (int)non, 0, end_bit, st));
    k_gather<<<gm, 256, 0, st>>>(src, bits0, d, idx, val_s, non, rec);
    SCK(cudaGetLastError());
    k_finish<<<(nobj + 127) / 128, 128, 0, st>>>(rec, off, nobj, osum);
    SCK(cudaGetLastError());
    launches += 2;
    sums.resize(nobj);
    SCK(cudaMemcpyAsync(sums.data(), osum, sizeof(ObjSums) * nobj, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
  }
  const unsigned nclosed = non;

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
int segment_volume(int storage, const void* P, const void* Pprev, float beta, int W, int H, int Nz,
                   const rihvr_segment_params* sp, rihvr_object* objects, int max_objects, int* num_objects,
                   rihvr_segment_info* info, SegWorkspace* ws, cudaStream_t st) {
  switch (storage) {
    case STORE_BF16:
      return segment_impl(VolumeSrc<__nv_bfloat162>{(const __nv_bfloat162*)P, (const __nv_bfloat162*)Pprev, beta},
                          W, H, Nz, sp, objects, max_objects, num_objects, info, *ws, st);
    case STORE_F16:
      return segment_impl(VolumeSrc<__half2>{(const __half2*)P, (const __half2*)Pprev, beta}, W, H, Nz, sp,
                          objects, max_objects, num_objects, info, *ws, st);
    default:
      return segment_impl(VolumeSrc<float2>{(const float2*)P, (const float2*)Pprev, beta}, W, H, Nz, sp, objects,
                          max_objects, num_objects, info, *ws, st);
  }
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
  if (rc == RIHVR_OK) {
    SegWorkspace ws;
    rc = segment_impl(IntensitySrc{src}, width, height, num_planes, sp, objects, max_objects, num_objects, info,
                      ws, st);
    cudaStreamSynchronize(st);
  }
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
