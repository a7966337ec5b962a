// Allocation-free variant of the adjoint operator (rihvr_adjoint_noalloc).
//
// Some callers cannot allocate device memory: plugin hosts that hand out every
// byte of device memory from their own pool and forbid other allocations, and
// real-time pipelines that must not take the latency (and the implicit device
// synchronisation) of cudaMalloc inside their loop.  This entry point needs no
// context and no allocation: the caller passes the input residual and the
// output volume (device memory), and the scratch the adjoint needs lives in one
// file-scope __device__ array of fixed size.
//
// Limits: square planes of a supported side up to 1024 and at most 4096
// planes.  The array takes 24 MiB + 32 KiB on every GPU that loads the library
// and is held until the process exits.  All calls share it and it keeps the
// last call's contents (every region is fully rewritten before it is read, so
// nothing needs clearing); calls that overlap on the GPU (different streams or
// host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/rihvr.h"
#include "rihvr_kernels.cuh"

using namespace rihvr;

namespace {

constexpr int kMaxSide = 1024;
constexpr int kMaxPlanes = 4096;
constexpr size_t kMaxPlaneElems = (size_t)kMaxSide * kMaxSide;
// layout: residual spectrum (float2) | column-pass intermediate, one plane or
// more (float2) | phase turns c(f)/2pi (double) | plane positions (double)
constexpr size_t kSpecOff = 0;
constexpr size_t kInterOff = kSpecOff + kMaxPlaneElems * sizeof(float2);
constexpr size_t kTurnsOff = kInterOff + kMaxPlaneElems * sizeof(float2);
constexpr size_t kZOff = kTurnsOff + kMaxPlaneElems * sizeof(double);
constexpr size_t kScratchBytes = kZOff + (size_t)kMaxPlanes * sizeof(double);

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// c(f)/2pi per frequency and the float plane list, as the context path builds
// them on the host (rihvr_solver.cu:phase_turns, rihvr_params.cpp:rihvr_plane_list).
__global__ void k_noalloc_tables(double* __restrict__ turns, double* __restrict__ zlist, int W, int H, int Nz,
                                 double dx, double lambda, float z0, float dz) {
  const double q = (lambda / dx) * (lambda / dx);
  const size_t n = (size_t)W * H;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i - (size_t)y * W);
    const double fy = (double)(((y + H / 2) % H) - (H / 2)) / (double)H;
    const double fx = (double)(((x + W / 2) % W) - (W / 2)) / (double)W;
    const double a = q * (fx * fx + fy * fy);
    const double sm1 = (a >= 1.0) ? -1.0 : -a / (sqrt(1.0 - a) + 1.0);
    turns[i] = sm1 / lambda;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Nz; i += gridDim.x * blockDim.x)
    zlist[i] = (double)__fadd_rn(z0, __fmul_rn((float)i, dz));
}

namespace {

int noalloc_fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());  // reported by rihvr_last_error
  return code;
}

// Device address of the scratch array in the current device's context.  In
// host code the array's name is only a host-side stand-in, never a device
// address, so every call asks the runtime with the target device current.  The
// lookup is a cheap host query; it is repeated on each call instead of cached
// because the address belongs to a context: after cudaDeviceReset, or when a
// host makes its own driver-API context current, the array lives elsewhere.
// The first call in a context may also load the library's module there.
int scratch_address(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return noalloc_fail(RIHVR_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  *out = static_cast<unsigned char*>(p);
  return RIHVR_OK;
}

#define NA_CK(call)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess) return noalloc_fail(RIHVR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

extern "C" int rihvr_adjoint_noalloc(const rihvr_params* p, int width, int height, const float* residual,
                                     float* volume_out, void* stream) {
  if (!p || !residual || !volume_out) return noalloc_fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (width > kMaxSide || height > kMaxSide)
    return noalloc_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "plane side " + std::to_string(width > height ? width : height) +
                                                        " exceeds the allocation-free maximum of 1024");
  if (width != height || !line_size_supported(width))
    return noalloc_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "planes must be square with a supported side");
  if (p->num_planes < 1 || p->num_planes > kMaxPlanes)
    return noalloc_fail(RIHVR_ERR_UNSUPPORTED_SIZE, "num_planes " + std::to_string(p->num_planes) +
                                                        " outside the allocation-free range 1..4096");
  if (!(p->wavelength > 0.f) || !(p->resolution > 0.f))
    return noalloc_fail(RIHVR_ERR_INVALID_ARGUMENT, "wavelength and resolution must be positive");
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != RIHVR_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int W = width, H = height, Nz = p->num_planes;
  const size_t HW = (size_t)W * H;
  float2* spec = reinterpret_cast<float2*>(base + kSpecOff);
  float2* inter = reinterpret_cast<float2*>(base + kInterOff);
  double* turns = reinterpret_cast<double*>(base + kTurnsOff);
  double* zlist = reinterpret_cast<double*>(base + kZOff);

  k_noalloc_tables<<<256, 256, 0, st>>>(turns, zlist, W, H, Nz, (double)p->resolution, (double)p->wavelength,
                                        p->start_plane, p->plane_stepsize);
  NA_CK(cudaGetLastError());
  // R / (W H) = FFT2(r) / (W H); the intermediate region holds the row pass
  NA_CK(launch_rows(0, ELEM_R32, residual, ELEM_C32, inter, W, H, 1.0f, st));
  NA_CK(launch_plane_col(0, inter, spec, W, H, 1.0f / (float)HW, st));
  // planes in chunks that fit the intermediate region
  const int per = (int)(kMaxPlaneElems / HW);
  float2* out = reinterpret_cast<float2*>(volume_out);
  for (int z0 = 0; z0 < Nz; z0 += per) {
    const int z1 = (z0 + per < Nz) ? z0 + per : Nz;
    NA_CK(launch_adj_col(spec, turns, zlist + z0, inter, W, H, 0, z1 - z0, st));
    NA_CK(launch_rows(1, ELEM_C32, inter, ELEM_C32, out + (size_t)z0 * HW, W, (long long)(z1 - z0) * H, 1.0f, st));
  }
  return RIHVR_OK;
}
