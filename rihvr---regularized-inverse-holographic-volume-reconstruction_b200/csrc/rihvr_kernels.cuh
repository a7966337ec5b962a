// Kernel launchers shared by the solver (all asynchronous on the given stream).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rihvr.h"

namespace rihvr {

// Slots of the per-block FP64 partial sums written by reduction kernels.
constexpr int kNumSums = 8;
enum SumIndex {
  SUM_LIM1 = 0,  // sum over real components of (p - x) * g          (line-search term 1)
  SUM_LIM2 = 1,  // sum |p - x|^2                                     (line-search term 2)
  SUM_RS = 2,    // restart statistic sum (x - p) * (p - y0)
  SUM_L1P = 3,   // sum |p|      (complex modulus)
  SUM_TVP = 4,   // TV(p)
  SUM_L1X = 5,   // sum |x|
  SUM_TVX = 6,   // TV(x)
  SUM_RR = 7,    // sum r^2 of a residual plane
};

enum StorageKind { STORE_F32 = 0, STORE_BF16 = 1, STORE_F16 = 2 };
enum ElemKind { ELEM_C32 = 0, ELEM_R32 = 1, ELEM_STORE_F32 = 2, ELEM_STORE_BF16 = 3, ELEM_STORE_F16 = 4 };

struct ProxArgs {
  const void* P;      // previous prox output y0 (storage type)
  const void* Pprev;  // the prox output before it (storage type)
  const float2* G;    // gradient volume A^H r(x)
  void* Pnew;         // new prox output (storage type)
  int W, H, Nz;
  float beta;         // momentum point x = P + beta (P - Pprev)
  float t;            // step size
  float mu;           // t * tv
  float s;            // dual step 1 / (12 t tv)
  float thr;          // shrink threshold (0 = no shrink)
  int n_tv;           // Chambolle iterations
  int faithful;       // reference quirks (separable shrink, restart weights)
  int want_norms;     // accumulate L1/TV of p and x
  double* partials;   // [blocks][kNumSums]
  long long partial_cap = 0;  // blocks partials holds; a launch needing more is refused
  // tuning knobs (0 = built-in choice): runs per plane of the streaming 2-D TV
  // prox, and the 2-D TV kernel (1 tiled, 2 streaming in 2-warp blocks,
  // 3 streaming in 4-warp blocks where the 8-row ring applies, n_tv <= 5,
  // 4 streaming in one launch where two would be taken, 6 <= n_tv <= 10)
  int tv_nseg = 0;
  int tv_kernel = 0;
  // dual of the first of two streaming launches (6 <= n_tv <= 10): gx and gy
  // of every voxel, FP32 complex; null = one launch
  float2* gdx = nullptr;
  float2* gdy = nullptr;
  // device copy of (beta, t, mu, s, thr); when set, the 2-D TV and L1 prox
  // kernels read these instead of the values above, so that a captured
  // launch picks up each attempt's step and momentum
  const float* dscal = nullptr;
};

bool line_size_supported(int n);
// sides the generic line FFT handles (prime factors 2, 3, 5, 7; up to 8192)
bool generic_size_supported(int n);
// message returned by rihvr_last_error on this thread
void set_last_error(const char* msg);

// particle segmentation of the volume x = P + beta (P - Pprev) on stream st,
// with device buffers kept in a workspace between calls (rihvr_segment.cu)
struct SegWorkspace;
SegWorkspace* seg_workspace_create();
void seg_workspace_destroy(SegWorkspace* ws);
// learned warm start (rihvr_unet.cu)
int unet_predict_on(rihvr_unet* u, const float2* xbp, float scale, float2* x0, cudaStream_t st);
void unet_dims(const rihvr_unet* u, int* D, int* H, int* W);

int segment_volume(int storage, const void* P, const void* Pprev, float beta, int W, int H, int Nz,
                   const rihvr_segment_params* sp, rihvr_object* objects, int max_objects, int* num_objects,
                   rihvr_segment_info* info, SegWorkspace* ws, cudaStream_t st);
size_t max_partial_blocks(int W, int H, int Nz);

// square sizes whose adjoint column pass has the recurrence variant
bool adj_recurrence_supported(int W, int H, int rec_mode = 2);
// dz_uniform != 0: the planes are evenly spaced by dz_uniform (z_{k+1} - z_k,
// exact in FP64), which lets the square fast sizes advance the transfer
// function by a recurrence (rec_mode 1: twiddles regenerated each plane, three
// blocks an SM; 2: twiddles kept in registers, two blocks an SM; 3: twiddles
// from a per-block shared table, three blocks an SM); rec_mode 0 or
// dz_uniform 0 takes the direct evaluation at every plane.
cudaError_t launch_adj_col(const float2* Rs, const double* cturn, const double* zlist, float2* U, int W,
                           int H, int z0, int z1, cudaStream_t st, int chunks_hint = 0, double dz_uniform = 0.0,
                           int rec_mode = 0);
cudaError_t launch_rows(int inverse, int in_kind, const void* in, int out_kind, void* out, int W,
                        long long nlines, float scale, cudaStream_t st);
// dz_uniform != 0 (evenly spaced planes): square staged sizes sum over z by
// Horner's scheme with the rotation H'_dz (fwd_horner_supported); horner_mode
// 1 stages T in its own double buffer (two blocks an SM), 2 in the exchange
// buffer with the twiddles in a shared table (three blocks an SM), 3 the same
// with each strip loaded by TMA (bounded mbarrier waits, col_wait_timeouts).
cudaError_t launch_fwd_col(const float2* T, const double* cturn, const double* zlist, float2* Spart, int W,
                           int H, int z0, int z1, int nchunks, cudaStream_t st, double dz_uniform = 0.0,
                           int horner_mode = 1);
bool fwd_horner_supported(int W, int H, int horner_mode = 1);
// Bounded waits of the TMA-fed column passes that ran out since the last call
// (synchronises the stream; clears the count).  Nonzero means a forward sum
// was left incomplete.
cudaError_t col_wait_timeouts(cudaStream_t st, unsigned* count);
int fwd_col_chunks(int W, int H, int Nz);
cudaError_t launch_plane_col(int inverse, const float2* in, float2* out, int W, int H, float scale,
                             cudaStream_t st);
cudaError_t launch_sum_chunks(const float2* Spart, int nchunks, float2* S, long long n, cudaStream_t st);
// Partial spectra of the z-slabs of one hologram summed in slab order,
// dst = ((src[0] + src[1]) + src[2]) + ...; sources on other devices are read
// through peer mappings with plain loads.
constexpr int kMaxSlabs = 16;
cudaError_t launch_sum_slabs(const float2* const* src, int n, float2* dst, long long count, cudaStream_t st);
cudaError_t launch_prox_tv2d(int storage, const ProxArgs& a, int* nblocks_out, cudaStream_t st);
cudaError_t launch_prox_l1(int storage, const ProxArgs& a, int* nblocks_out, cudaStream_t st);
cudaError_t launch_reduce_partials(const double* partials, int nblocks, double* scratch, double* out,
                                   cudaStream_t st);
size_t reduce_scratch_doubles();
cudaError_t launch_fill_uniform_c(float2* x, long long n, unsigned long long seed, cudaStream_t st);
cudaError_t launch_sumsq(const float* x, long long n, double* partials, int* nblocks_out, cudaStream_t st);
cudaError_t launch_finish_forward(const float2* c, const float* b, float* dnew, long long n, double* partials,
                                  int* nblocks_out, cudaStream_t st);
cudaError_t launch_holo_momentum(const float* dnew, float* dY0, float* dX, const float* b, float* r,
                                 float beta, long long n, double* partials, int* nblocks_out, cudaStream_t st,
                                 const float* dbeta = nullptr);
cudaError_t launch_momentum_norms(int storage, const void* P, const void* Pprev, float beta, int W, int H,
                                  int Nz, int mode, double* partials, int* nblocks_out, cudaStream_t st);
cudaError_t launch_materialize_x(int storage, const void* P, const void* Pprev, float beta, float2* out,
                                 long long n, cudaStream_t st);
cudaError_t launch_store_volume(int storage, const float2* in, void* out, long long n, cudaStream_t st);
cudaError_t launch_prox6_init(int storage, const ProxArgs& a, float2* X1, cudaStream_t st);
cudaError_t launch_tv3_estimate(const float2* X1, const float2* gx, const float2* gy, const float2* gz, float2* Y,
                                int W, int H, int Nz, float mu, cudaStream_t st);
cudaError_t launch_tv3_dual(const float2* Y, float2* gx, float2* gy, float2* gz, int W, int H, int Nz, float s,
                            cudaStream_t st);
cudaError_t launch_prox6_finish(int storage, const ProxArgs& a, const float2* Y, int* nblocks_out,
                                cudaStream_t st);

}  // namespace rihvr
