// Camera frames on the device.
//
// 1. Preprocessing (rihvr_set_hologram_frame): the raw frame travels to the
//    GPU as stored (1 or 2 bytes a sample instead of 4) and one pass makes the
//    hologram: fl(v / 255), then I/mean - 1 (hologram.cu:332-358) or
//    (I - B) / max(sqrt(B), 0.1) (:1365-1432), crop (:768-887) and zero
//    padding (:889-945).  Every float operation is the IEEE-rounded one the
//    host path (rihvr_image.cpp) performs, and the mean comes from the same
//    exact integer sum, so the two agree bit for bit.
// 2. Background generation (main_create_background.cu):
//    - mean (HoloSequence::useBackgroundSubtraction, holo_sequence.cu:309-447):
//      the frames summed in order in FP32 (cv::add), scaled by the FP32
//      factor fl(1/n) (Mat /= n is convertTo with alpha 1/n, an FP32
//      multiply), and the statistics alpha, beta, minimum, average from
//      per-frame FP64 mean and standard deviation of frame - background
//      (cv::meanStdDev);
//    - running median of five (median_background_calc, :103-193), with the
//      reference's order of replacing frames in its five-frame stack.
// All kernels are HBM-bound streams over the frames.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/rihvr.h"
#include "rihvr_frame.cuh"
#include "rihvr_image.h"
#include "rihvr_kernels.cuh"

namespace rihvr {

namespace {

int ffail(int code, const std::string& msg) {
  set_last_error(msg.c_str());
  return code;
}

#define FCK(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return ffail(e_ == cudaErrorMemoryAllocation ? RIHVR_ERR_OUT_OF_MEMORY : RIHVR_ERR_CUDA,     \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                           \
  } while (0)

#define FRC(call)                   \
  do {                              \
    int r_ = (call);                \
    if (r_ != RIHVR_OK) return r_;  \
  } while (0)

size_t sample_bytes(int bits) { return bits == 8 ? 1 : bits == 16 ? 2 : 4; }

__device__ __forceinline__ float as_float(uint8_t v) { return (float)v; }
__device__ __forceinline__ float as_float(uint16_t v) { return (float)v; }
__device__ __forceinline__ float as_float(float v) { return v; }

// a value an 8- or 16-bit image can hold (floats only need the check)
template <typename T>
__device__ __forceinline__ bool is_sample(float v) {
  if constexpr (std::is_same<T, float>::value) return v >= 0.f && v <= 65535.f && v == floorf(v);
  return true;
}

int grid_for(size_t n, int threads) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t want = (n + threads - 1) / threads;
  return (int)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8));
}

// Exact sum of fl(v / 255) in units of 2^-31 (128 bits: acc[0] low word,
// acc[1] carries) and the count of values that are not samples (acc[2]).
// Integer sums do not depend on the order, so the result is deterministic
// and equal to the host's.
template <typename T>
__global__ void k_frame_unit_sum(const T* __restrict__ f, size_t n, unsigned long long* __restrict__ acc) {
  unsigned long long s = 0, bad = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = as_float(f[i]);
    if (!is_sample<T>(v)) {
      ++bad;
      continue;
    }
    // fl(v/255) * 2^31 is an integer below 2^40; a thread adds at most
    // n / (grid threads) of them and a warp 32 times that, far below 2^64
    s += (unsigned long long)__float2ull_rn(__fdiv_rn(v, 255.0f) * 2147483648.0f);
  }
  for (int o = 16; o; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s) {
      const unsigned long long old = atomicAdd(&acc[0], s);
      if (old + s < old) atomicAdd(&acc[1], 1ull);
    }
    if (bad) atomicAdd(&acc[2], bad);
  }
}

// One output sample per thread (grid-stride over the padded W x H hologram).
template <typename T, bool BG>
__global__ void k_frame_prep(const T* __restrict__ f, const T* __restrict__ bg, int W0, int H0, int rx, int ry,
                             int rw, int rh, int pad, int W, int H, float mf, float* __restrict__ out) {
  const size_t n = (size_t)W * H;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i - (size_t)y * W);
    const int cx = x - pad, cy = y - pad;
    float o = 0.f;
    if (cx >= 0 && cy >= 0 && cx < rw && cy < rh) {
      const int sx = rx + cx, sy = ry + cy;
      if (sx >= 0 && sy >= 0 && sx < W0 && sy < H0) {
        const size_t s = (size_t)sy * W0 + sx;
        const float v = __fdiv_rn(as_float(f[s]), 255.0f);
        if constexpr (BG) {
          const float B = __fdiv_rn(as_float(bg[s]), 255.0f);
          float sb = __fsqrt_rn(B);
          if (sb < 0.1f) sb = 0.1f;
          o = __fdiv_rn(__fsub_rn(v, B), sb);
        } else {
          o = __fsub_rn(__fdiv_rn(v, mf), 1.0f);
        }
      }
    }
    out[i] = o;
  }
}

// acc = acc + frame_k for k = 0 .. nf-1 in order (start from 0 when first)
template <typename T>
__global__ void k_bg_accumulate(float* __restrict__ acc, const T* __restrict__ frames, int nf, size_t npx,
                                int first) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += (size_t)gridDim.x * blockDim.x) {
    float a = first ? 0.f : acc[i];
    for (int k = 0; k < nf; ++k) a = __fadd_rn(a, as_float(frames[(size_t)k * npx + i]));
    acc[i] = a;
  }
}

// per-block FP64 partial sums, reduced in a fixed order
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0)
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) t += sh[j];
  return t;
}

// bg = fl(acc * s) and the partial sums of bg (for its mean)
__global__ void k_bg_scale(const float* __restrict__ acc, float s, size_t npx, float* __restrict__ bg,
                           double* __restrict__ partial) {
  __shared__ double sh[32];
  double t = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += (size_t)gridDim.x * blockDim.x) {
    const float b = __fmul_rn(acc[i], s);
    bg[i] = b;
    t += (double)b;
  }
  t = block_sum(t, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// per frame (blockIdx.y): partial sums of d and d^2 in FP64, d = fl(frame - bg)
template <typename T>
__global__ void k_bg_moments(const T* __restrict__ frames, const float* __restrict__ bg, size_t npx,
                             double* __restrict__ partial) {
  __shared__ double sh[32];
  const T* f = frames + (size_t)blockIdx.y * npx;
  double s1 = 0, s2 = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += (size_t)gridDim.x * blockDim.x) {
    const double d = (double)__fsub_rn(as_float(f[i]), bg[i]);
    s1 += d;
    s2 += d * d;
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    double* p = partial + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 2;
    p[0] = s1;
    p[1] = s2;
  }
}

// median of five values: order two pairs, drop the smallest of the four,
// bring in the fifth, and once more; the median is the smaller of what is
// left at the top of the two pairs
__device__ __forceinline__ float median5(float a, float b, float c, float d, float e) {
  if (a > b) { const float t = a; a = b; b = t; }
  if (c > d) { const float t = c; c = d; d = t; }
  if (a > c) { float t = a; a = c; c = t; t = b; b = d; d = t; }
  a = e;  // a was the smallest of a, b, c, d
  if (a > b) { const float t = a; a = b; b = t; }
  if (a > c) { float t = a; a = c; c = t; t = b; b = d; d = t; }
  return b < c ? b : c;  // a is the smallest of the four left
}

// output j (blockIdx.y) = per-pixel median of the five frames sel[5 j .. 5 j + 4]
template <typename T>
__global__ void k_median5(const T* __restrict__ frames, const int* __restrict__ sel, size_t npx,
                          float* __restrict__ out) {
  const int* s = sel + 5 * blockIdx.y;
  const T* f0 = frames + (size_t)s[0] * npx;
  const T* f1 = frames + (size_t)s[1] * npx;
  const T* f2 = frames + (size_t)s[2] * npx;
  const T* f3 = frames + (size_t)s[3] * npx;
  const T* f4 = frames + (size_t)s[4] * npx;
  float* o = out + (size_t)blockIdx.y * npx;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += (size_t)gridDim.x * blockDim.x)
    o[i] = median5(as_float(f0[i]), as_float(f1[i]), as_float(f2[i]), as_float(f3[i]), as_float(f4[i]));
}

template <typename F>
int dispatch_bits(int bits, F&& f) {
  switch (bits) {
    case 8: return f(uint8_t{});
    case 16: return f(uint16_t{});
    case 32: return f(float{});
    default: return ffail(RIHVR_ERR_INVALID_ARGUMENT, "bits must be 8, 16 or 32");
  }
}

// a device buffer that grows
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int reserve(size_t bytes) {
    if (bytes <= cap) return RIHVR_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    FCK(cudaMalloc(&p, bytes));
    cap = bytes;
    return RIHVR_OK;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

// owned stream for the context-free entry points
struct Stream {
  cudaStream_t s = nullptr;
  ~Stream() {
    if (s) cudaStreamDestroy(s);
  }
};

}  // namespace

struct FrameWorkspace {
  DevBuf raw, bg, out, acc;
  unsigned long long* acc_h = nullptr;  // pinned [6]
  ~FrameWorkspace() {
    if (acc_h) cudaFreeHost(acc_h);
  }
};

void frame_workspace_free(FrameWorkspace* ws) { delete ws; }

int frame_to_hologram(FrameWorkspace** wsp, const void* frame, int bits, int W0, int H0, const void* background,
                      const rihvr_file_params* files, int pad, int W, int H, int is_device, cudaStream_t st,
                      const float** out, long long* launches) {
  if (!frame || W0 <= 0 || H0 <= 0 || !out) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "NULL frame or empty size");
  if (bits != 8 && bits != 16 && bits != 32) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "bits must be 8, 16 or 32");
  rihvr_io::Preprocess pp;
  if (files) {
    pp.remove_background = files->remove_background != 0;
    pp.roi_x = files->roi_x;
    pp.roi_y = files->roi_y;
    pp.roi_size = files->roi_size;
    pp.roi_rect_x = files->roi_rect_x;
    pp.roi_rect_y = files->roi_rect_y;
    pp.roi_rect_w = files->roi_rect_w;
    pp.roi_rect_h = files->roi_rect_h;
  }
  if (pp.remove_background && !background)
    return ffail(RIHVR_ERR_MISSING_DATA, "background division is set but no background was given");
  const rihvr_io::CropRect cr = rihvr_io::crop_rect(pp, W0, H0);
  if (cr.w <= 0 || cr.h <= 0 || cr.w + 2 * pad != W || cr.h + 2 * pad != H)
    return ffail(RIHVR_ERR_INVALID_ARGUMENT, "the cropped and padded frame is " + std::to_string(cr.w + 2 * pad) +
                                                 " x " + std::to_string(cr.h + 2 * pad) + ", the context " +
                                                 std::to_string(W) + " x " + std::to_string(H));
  if (!*wsp) {
    *wsp = new FrameWorkspace();
    FCK(cudaMallocHost(&(*wsp)->acc_h, 6 * sizeof(unsigned long long)));
  }
  FrameWorkspace* ws = *wsp;
  const size_t n0 = (size_t)W0 * H0, sb = sample_bytes(bits);
  FRC(ws->out.reserve(sizeof(float) * (size_t)W * H));
  FRC(ws->acc.reserve(6 * sizeof(unsigned long long)));
  const void* f = frame;
  const void* b = background;
  if (!is_device) {
    FRC(ws->raw.reserve(n0 * sb));
    FCK(cudaMemcpyAsync(ws->raw.p, frame, n0 * sb, cudaMemcpyHostToDevice, st));
    f = ws->raw.p;
    if (pp.remove_background) {
      FRC(ws->bg.reserve(n0 * sb));
      FCK(cudaMemcpyAsync(ws->bg.p, background, n0 * sb, cudaMemcpyHostToDevice, st));
      b = ws->bg.p;
    }
  }
  auto* acc = static_cast<unsigned long long*>(ws->acc.p);
  float mf = 0.f;
  const bool need_sum = !pp.remove_background;
  const bool need_check = bits == 32;  // float samples must hold 8/16-bit values
  if (need_sum || need_check) {
    FCK(cudaMemsetAsync(acc, 0, 6 * sizeof(unsigned long long), st));
    const int grid = grid_for(n0, 256);
    FRC(dispatch_bits(bits, [&](auto tag) -> int {
      using T = decltype(tag);
      k_frame_unit_sum<T><<<grid, 256, 0, st>>>(static_cast<const T*>(f), n0, acc);
      FCK(cudaGetLastError());
      ++*launches;
      if (pp.remove_background && bits == 32) {
        k_frame_unit_sum<T><<<grid, 256, 0, st>>>(static_cast<const T*>(b), n0, acc + 3);
        FCK(cudaGetLastError());
        ++*launches;
      }
      return RIHVR_OK;
    }));
    FCK(cudaMemcpyAsync(ws->acc_h, acc, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    const unsigned long long bad = ws->acc_h[2] + ws->acc_h[5];
    if (bad)
      return ffail(RIHVR_ERR_INVALID_DATA,
                   std::to_string(bad) + " samples are not integers in [0, 65535] (8- or 16-bit image values)");
    if (need_sum) {
      const double m = rihvr_io::unit_mean_from_sum(ws->acc_h[0], ws->acc_h[1], n0);
      if (!(m != 0)) return ffail(RIHVR_ERR_INVALID_DATA, "hologram mean is zero");
      mf = (float)m;
    }
  }
  const int grid = grid_for((size_t)W * H, 256);
  FRC(dispatch_bits(bits, [&](auto tag) -> int {
    using T = decltype(tag);
    float* o = static_cast<float*>(ws->out.p);
    if (pp.remove_background)
      k_frame_prep<T, true><<<grid, 256, 0, st>>>(static_cast<const T*>(f), static_cast<const T*>(b), W0, H0, cr.x,
                                                  cr.y, cr.w, cr.h, pad, W, H, 0.f, o);
    else
      k_frame_prep<T, false><<<grid, 256, 0, st>>>(static_cast<const T*>(f), nullptr, W0, H0, cr.x, cr.y, cr.w,
                                                   cr.h, pad, W, H, mf, o);
    FCK(cudaGetLastError());
    ++*launches;
    return RIHVR_OK;
  }));
  *out = static_cast<const float*>(ws->out.p);
  return RIHVR_OK;
}

namespace {

// frames [k0, k0 + nk) resident on the device: the caller's pointer, or a
// copy made into buf
int frames_on_device(const void* frames, int is_device, size_t frame_bytes, int k0, int nk, DevBuf& buf,
                     cudaStream_t st, const void** dev) {
  const char* src = static_cast<const char*>(frames) + (size_t)k0 * frame_bytes;
  if (is_device) {
    *dev = src;
    return RIHVR_OK;
  }
  FRC(buf.reserve((size_t)nk * frame_bytes));
  FCK(cudaMemcpyAsync(buf.p, src, (size_t)nk * frame_bytes, cudaMemcpyHostToDevice, st));
  *dev = buf.p;
  return RIHVR_OK;
}

// frames a batch holds: all when they fit in a quarter of the free memory
// (and in one grid's y dimension)
int batch_frames(size_t frame_bytes, int count) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)1 << 30;
  const size_t fit = std::max<size_t>(1, (free_b / 4) / std::max<size_t>(frame_bytes, 1));
  return (int)std::min<size_t>(std::min<size_t>((size_t)count, fit), 65535);
}

int check_frames(const void* frames, int bits, int width, int height, int count, int min_count) {
  if (!frames || width <= 0 || height <= 0) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "NULL frames or empty size");
  if (bits != 8 && bits != 16 && bits != 32) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "bits must be 8, 16 or 32");
  if (count < min_count)
    return ffail(RIHVR_ERR_INVALID_ARGUMENT, "needs at least " + std::to_string(min_count) + " frames, got " +
                                                 std::to_string(count));
  return RIHVR_OK;
}

}  // namespace

}  // namespace rihvr

using namespace rihvr;

extern "C" {

int rihvr_background_mean(const void* frames, int bits, int width, int height, int count, int is_device,
                          float* background, double* stats) {
  FRC(check_frames(frames, bits, width, height, count, 1));
  if (!background) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "NULL background");
  const size_t npx = (size_t)width * height, fb = npx * sample_bytes(bits);
  Stream s;
  FCK(cudaStreamCreateWithFlags(&s.s, cudaStreamNonBlocking));
  DevBuf fbuf, acc, bg, part;
  FRC(acc.reserve(npx * sizeof(float)));
  FRC(bg.reserve(npx * sizeof(float)));
  const int grid = grid_for(npx, 256);
  const int batch = batch_frames(fb, count);
  const bool resident = batch == count;
  FRC(part.reserve(sizeof(double) * std::max<size_t>((size_t)grid, (size_t)grid * 2 * batch)));
  std::vector<double> ph((size_t)grid * 2 * batch);
  return dispatch_bits(bits, [&](auto tag) -> int {
    using T = decltype(tag);
    // pass 1: the frames summed in order, then scaled (holo_sequence.cu:359-383)
    const void* dev = nullptr;
    for (int k0 = 0; k0 < count; k0 += batch) {
      const int nk = std::min(batch, count - k0);
      FRC(frames_on_device(frames, is_device, fb, k0, nk, fbuf, s.s, &dev));
      k_bg_accumulate<T><<<grid, 256, 0, s.s>>>(static_cast<float*>(acc.p), static_cast<const T*>(dev), nk, npx,
                                                k0 == 0);
      FCK(cudaGetLastError());
    }
    const float scale = (float)(1.0 / (double)count);
    k_bg_scale<<<grid, 256, 0, s.s>>>(static_cast<const float*>(acc.p), scale, npx, static_cast<float*>(bg.p),
                                      static_cast<double*>(part.p));
    FCK(cudaGetLastError());
    FCK(cudaMemcpyAsync(ph.data(), part.p, sizeof(double) * grid, cudaMemcpyDeviceToHost, s.s));
    FCK(cudaStreamSynchronize(s.s));
    double bsum = 0;
    for (int j = 0; j < grid; ++j) bsum += ph[j];
    const double average = bsum / (double)npx;  // cv::mean of the background (:385)
    // pass 2: mean and standard deviation of each frame - background (:389-412)
    double mean_sum = 0, std_sum = 0;
    for (int k0 = 0; k0 < count; k0 += batch) {
      const int nk = std::min(batch, count - k0);
      if (!resident || k0 > 0 || !dev) FRC(frames_on_device(frames, is_device, fb, k0, nk, fbuf, s.s, &dev));
      k_bg_moments<T><<<dim3(grid, nk), 256, 0, s.s>>>(static_cast<const T*>(dev), static_cast<const float*>(bg.p),
                                                       npx, static_cast<double*>(part.p));
      FCK(cudaGetLastError());
      FCK(cudaMemcpyAsync(ph.data(), part.p, sizeof(double) * grid * 2 * nk, cudaMemcpyDeviceToHost, s.s));
      FCK(cudaStreamSynchronize(s.s));
      for (int k = 0; k < nk; ++k) {
        double s1 = 0, s2 = 0;
        for (int j = 0; j < grid; ++j) {
          s1 += ph[((size_t)k * grid + j) * 2];
          s2 += ph[((size_t)k * grid + j) * 2 + 1];
        }
        const double m = s1 / (double)npx;
        mean_sum += m;
        std_sum += std::sqrt(std::max(s2 / (double)npx - m * m, 0.0));
      }
    }
    const double mean_mean = mean_sum / count, mean_std = std_sum / count;
    constexpr double kScale1 = 5;  // bg_scale1 (holo_sequence.cu:22)
    if (stats) {
      stats[0] = mean_mean - kScale1 * mean_std;  // alpha (:418)
      stats[1] = 255 / (2 * mean_std * kScale1);  // beta (:419)
      stats[2] = 0;                               // minimum grey, bg_min_grey (:23)
      stats[3] = average;
    }
    FCK(cudaMemcpyAsync(background, bg.p, npx * sizeof(float),
                        is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s.s));
    FCK(cudaStreamSynchronize(s.s));
    return RIHVR_OK;
  });
}

int rihvr_background_median5_frames(int count, int* sel) {
  if (count < 5) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "the median background needs at least 5 frames");
  // the five-frame stack of median_background_calc (main_create_background.cu:126-187):
  // frames 0-4 give backgrounds 0, 1 and 2; background i (3 <= i < count - 2)
  // comes after frame i replaces stack slot (i - 3) mod 5
  int stack[5] = {0, 1, 2, 3, 4};
  int j = 0;
  for (int r = 0; r < 3; ++r, ++j)
    for (int m = 0; m < 5; ++m) sel[5 * j + m] = stack[m];
  for (int i = 3; i < count - 2; ++i, ++j) {
    stack[(i - 3) % 5] = i;
    for (int m = 0; m < 5; ++m) sel[5 * j + m] = stack[m];
  }
  return RIHVR_OK;
}

int rihvr_background_median5(const void* frames, int bits, int width, int height, int count, int is_device,
                             float* backgrounds) {
  FRC(check_frames(frames, bits, width, height, count, 5));
  if (!backgrounds) return ffail(RIHVR_ERR_INVALID_ARGUMENT, "NULL backgrounds");
  const int nout = count - 2;
  std::vector<int> sel((size_t)5 * nout);
  FRC(rihvr_background_median5_frames(count, sel.data()));
  const size_t npx = (size_t)width * height, fb = npx * sample_bytes(bits);
  Stream s;
  FCK(cudaStreamCreateWithFlags(&s.s, cudaStreamNonBlocking));
  DevBuf fbuf, obuf, sbuf;
  // outputs in chunks whose frames (at most chunk + 4 consecutive ones) and
  // results fit in a quarter of the free memory
  int chunk = std::max(1, batch_frames(fb + npx * sizeof(float), nout) - 5);
  chunk = std::min(chunk, nout);
  FRC(sbuf.reserve(sizeof(int) * 5 * (size_t)chunk));
  if (!is_device) FRC(obuf.reserve(sizeof(float) * npx * chunk));
  const int grid = std::max(1, grid_for(npx, 256) / std::max(1, std::min(chunk, 8)));
  return dispatch_bits(bits, [&](auto tag) -> int {
    using T = decltype(tag);
    std::vector<int> local((size_t)5 * chunk);
    for (int j0 = 0; j0 < nout; j0 += chunk) {
      const int nj = std::min(chunk, nout - j0);
      int lo = count, hi = -1;
      for (size_t q = (size_t)5 * j0; q < (size_t)5 * (j0 + nj); ++q) {
        lo = std::min(lo, sel[q]);
        hi = std::max(hi, sel[q]);
      }
      for (size_t q = 0; q < (size_t)5 * nj; ++q) local[q] = sel[(size_t)5 * j0 + q] - lo;
      const void* dev = nullptr;
      FRC(frames_on_device(frames, is_device, fb, lo, hi - lo + 1, fbuf, s.s, &dev));
      FCK(cudaMemcpyAsync(sbuf.p, local.data(), sizeof(int) * 5 * nj, cudaMemcpyHostToDevice, s.s));
      float* o = is_device ? backgrounds + (size_t)j0 * npx : static_cast<float*>(obuf.p);
      k_median5<T><<<dim3(grid, nj), 256, 0, s.s>>>(static_cast<const T*>(dev), static_cast<const int*>(sbuf.p), npx,
                                                    o);
      FCK(cudaGetLastError());
      if (!is_device)
        FCK(cudaMemcpyAsync(backgrounds + (size_t)j0 * npx, o, sizeof(float) * npx * nj, cudaMemcpyDeviceToHost,
                            s.s));
      FCK(cudaStreamSynchronize(s.s));  // the host table and buffers are reused by the next chunk
    }
    return RIHVR_OK;
  });
}

}  // extern "C"
