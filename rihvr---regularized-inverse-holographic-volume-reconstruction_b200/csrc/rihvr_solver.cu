// Host side of the C ABI: context, device buffers and the FISTA/FASTA loop of
// SparseCompressiveHolo::inverseReconstruct (RIHVR src/core/
// sparse_compressive_holo.cu:173-633), arranged around three volume buffers.
//
// Volume buffers rotate through the roles P_{k-1}, P_k, P_{k+1} (prox outputs).
// The momentum point x_k = P_k + beta_k (P_k - P_{k-1}) (fistaUpdate, :4496-4576)
// is never stored: the prox kernel forms it on the fly, and the forward operator
// at x_k follows by linearity from the two stored hologram estimates
// (:480-498).  The gradient volume A^H r(x_k) is computed once per iteration and
// reused by every backtracking attempt (the reference recomputes it per plane
// access, sparse_gradient.cu:125-165).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <new>
#include <string>
#include <atomic>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>  // header-only; ranges cost nothing without a profiler

#include "../../include/rihvr.h"
#include "rihvr_frame.cuh"
#include "rihvr_kernels.cuh"

using namespace rihvr;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

}  // namespace

void rihvr::set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

namespace {

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      return fail(e_ == cudaErrorMemoryAllocation ? RIHVR_ERR_OUT_OF_MEMORY : RIHVR_ERR_CUDA,      \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                            \
    }                                                                                              \
  } while (0)

// kernel launch: check and count (one of our kernels per launcher call)
#define KL(call)        \
  do {                  \
    CK(call);           \
    ++c->launches;      \
  } while (0)

#define RC(call)                     \
  do {                               \
    int r_ = (call);                 \
    if (r_ != RIHVR_OK) return r_;   \
  } while (0)

// NVTX range over a scope: the solver's phases (iterations, attempts,
// momentum step, autotuning, hologram set-up, batches) show in a timeline
// profiler; in graph-captured iterations they mark the host-side launches.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

enum KernelClass { K_ADJ_COL = 0, K_ADJ_ROW, K_PROX, K_FWD_ROW, K_FWD_COL, K_PLANE, K_NUM };
const char* kClassNames[K_NUM] = {"adj_col", "adj_row", "prox", "fwd_row", "fwd_col", "plane"};

enum Slot { SLOT_PROX = 0, SLOT_FWD = 1, SLOT_MOM = 2, SLOT_NORM = 3, NUM_SLOTS = 4 };

constexpr int kMaxFwdChunks = 16;  // partial spectra the forward column pass may use

}  // namespace

namespace {

// FISTA control state kept on the device, so that whole iterations (attempt,
// backtracks, momentum) replay as one graph without a host round trip.
struct IterCtl {
  double t, alpha1, beta, prev_f_resid;  // the host fields of the same names
  double f_resid, lim, ratio;            // of the last attempt
  int bt, it, it_base, pad;
};
// One iteration's record as the device writes it, plus the x-norm sums of its
// first prox sweep, which settle the previous record (objective recording).
struct DevRec {
  rihvr_iter_record rec;
  double prev_l1x, prev_tvx;
};
constexpr int kDevLogCap = 256;  // iterations between two host reads of the log

// The attempt's prox scalars from t and beta, as prox_args computes them.
__global__ void k_ctl_prep(IterCtl* s, float* scal, double tv, double l1, int zero_thr, int first) {
  if (first) s->bt = 0;
  const double t = s->t;
  scal[0] = (float)s->beta;
  scal[1] = (float)t;
  scal[2] = (float)__dmul_rn(t, tv);
  scal[3] = tv > 0 ? (float)__ddiv_rn(1.0, __dmul_rn(__dmul_rn(12.0, t), tv)) : 0.f;
  scal[4] = zero_thr ? 0.f : (float)__dmul_rn(t, l1);
}

// Backtracking test of one_iteration: ratio = f_resid / (prev + lim); halve t
// and go again while the ratio is outside [0, 1] and backtracks remain.
__global__ void k_ctl_decide(IterCtl* s, const double* sums, int max_bt, cudaGraphConditionalHandle h, DevRec* log,
                             int first) {
  const double* sp = sums + SLOT_PROX * kNumSums;
  if (first) {
    DevRec& r = log[s->it - s->it_base];
    r.prev_l1x = sp[SUM_L1X];
    r.prev_tvx = sp[SUM_TVX];
  }
  const double t = s->t;
  const double f_resid = 0.5 * sums[SLOT_FWD * kNumSums + SUM_RR];
  const double lim = __dadd_rn(sp[SUM_LIM1], __ddiv_rn(sp[SUM_LIM2], __dmul_rn(2.0, t)));
  const double ratio = __ddiv_rn(f_resid, __dadd_rn(s->prev_f_resid, lim));
  s->f_resid = f_resid;
  s->lim = lim;
  s->ratio = ratio;
  unsigned again = 0;
  if (((ratio > 1.0) || (ratio < 0.0)) && s->bt < max_bt) {
    s->t = t * 0.5;
    s->bt += 1;
    again = 1;
  }
  cudaGraphSetConditional(h, again);
}

// Record of the accepted attempt, fistaRestart (:471-475) and the alpha/beta
// update (:476-481); beta goes to the hologram momentum.
__global__ void k_ctl_finish(IterCtl* s, const double* sums, float* scal, DevRec* log, double l1, double tvw) {
  const double* sp = sums + SLOT_PROX * kNumSums;
  rihvr_iter_record& rec = log[s->it - s->it_base].rec;
  rec.f_resid_prox = s->f_resid;
  rec.lim = s->lim;
  rec.ratio = s->ratio;
  rec.t = s->t;
  rec.backtracks = s->bt;
  rec.restart_sum = sp[SUM_RS];
  rec.f_prox = __dadd_rn(__dadd_rn(s->f_resid, __dmul_rn(l1, sp[SUM_L1P])), __dmul_rn(tvw, sp[SUM_TVP]));
  rec.l1_x = rec.tv_x = 0.0;
  const bool restarted = sp[SUM_RS] > 0.0;
  const double alpha0 = restarted ? 1.0 : s->alpha1;
  const double alpha1 = __ddiv_rn(__dadd_rn(1.0, sqrt(__dadd_rn(1.0, __dmul_rn(__dmul_rn(4.0, alpha0), alpha0)))), 2.0);
  const double beta = __ddiv_rn(alpha0 - 1.0, alpha1);
  rec.beta = beta;
  rec.restarted = restarted ? 1 : 0;
  s->alpha1 = alpha1;
  s->beta = beta;
  scal[8] = (float)beta;
}

// Residual at the new momentum point closes the record.
__global__ void k_ctl_post(IterCtl* s, const double* sums, DevRec* log) {
  rihvr_iter_record& rec = log[s->it - s->it_base].rec;
  s->prev_f_resid = 0.5 * sums[SLOT_MOM * kNumSums + SUM_RR];
  rec.f_resid_x = s->prev_f_resid;
  rec.f_x = rec.f_resid_x;
  s->it += 1;
}

}  // namespace

struct rihvr_ctx {
  rihvr_params p{};
  int W = 0, H = 0, Nz = 0;
  int z_first = 0;  // first plane held, of p.num_planes (z-slab contexts hold Nz < p.num_planes)
  size_t HW = 0, V = 0;
  int mode = 7;
  int storage = 0;
  size_t esize = 8;
  int device = 0;
  cudaStream_t st = nullptr;

  void* vol[3] = {nullptr, nullptr, nullptr};
  int iPrev = 0, iCur = 1, iNew = 2;
  float2* G = nullptr;    // gradient volume
  float2* U = nullptr;    // column/row intermediate volume
  float2* gdy = nullptr;  // gy of the two-launch TV prox (6-10 iterations; gx goes to U)
  float2* Spart = nullptr;
  float2* S = nullptr;
  float2* pc1 = nullptr;
  float2* pc2 = nullptr;
  float2* Rs = nullptr;   // residual spectrum / (W H)
  float* b = nullptr;
  float* dnew = nullptr;
  float* dY0 = nullptr;
  float* dX = nullptr;
  float* r = nullptr;
  double* cturn = nullptr;
  double* zlist = nullptr;
  double dz_uniform = 0;  // plane spacing when every z_{k+1} - z_k is the same (FP64), else 0
  // column-pass variants for evenly spaced planes (need dz_uniform): the
  // adjoint's transfer function by recurrence (1: twiddles regenerated each
  // plane, 2: twiddles kept, 3: twiddles from a shared table) or direct (0);
  // the forward's z-sum by Horner's scheme (1: two blocks an SM; 2, 3: three
  // blocks an SM, the strip copied by cp.async or TMA) or direct (0).
  // Autotuned; RIHVR_ADJ_COL and RIHVR_FWD_COL select one by name.
  int tune_adj_rec = 0;
  int tune_fwd_horner = 3;  // TMA-fed Horner pass; sizes without it take the two-block form (1)
  double* partials = nullptr;
  unsigned* nonfinite_d = nullptr;  // count of non-finite hologram samples (rihvr_set_hologram)
  size_t partial_cap = 0;
  double* sums_d = nullptr;
  double* red_scratch = nullptr;
  double* sums_h = nullptr;  // pinned
  int nchunks = 1;        // z-chunks of the forward column pass (Spart holds kMaxFwdChunks)
  // Step and momentum scalars of the current attempt: pinned host copy and the
  // device copy the prox and momentum kernels read ([0..4] beta, t, mu, s, thr;
  // [8] hologram momentum beta), so that captured graphs replay every attempt.
  float* scal_d = nullptr;
  float* scal_h = nullptr;
  cudaGraphExec_t g_att[2][3] = {};  // [backtrack attempt][index of P_k among the 3 volumes]
  int g_att_n[2][3] = {};            // kernels in each graph
  cudaGraphExec_t g_mom = nullptr;
  int g_mom_n = 0;
  bool graphs = true;                // cleared when a capture fails
  // whole iterations with the backtracking decided on the device: one graph
  // per index of P_k, kernels in [first attempt + finish/momentum, backtrack]
  cudaGraphExec_t g_iter[3] = {};
  int g_iter_n[3][2] = {};
  bool dev_loop = true;              // cleared when building such a graph fails
  IterCtl* ctl_d = nullptr;
  IterCtl* ctl_h = nullptr;          // pinned
  DevRec* dlog_d = nullptr;
  DevRec* dlog_h = nullptr;          // pinned
  bool warm = false;                 // one iteration ran eagerly (attributes, tables)
  SegWorkspace* seg_ws = nullptr;    // segmentation buffers, grown on first use
  FrameWorkspace* frame_ws = nullptr;  // raw-frame uploads (rihvr_set_hologram_frame), grown on first use
  // launch shapes chosen by the autotuner (0 = built-in choice)
  int tune_adj_chunks = 0, tune_tv_nseg = 0, tune_tv_kernel = 0;
  bool tuned = false;
  float2 *X1 = nullptr, *gx = nullptr, *gy = nullptr, *gz = nullptr, *Y = nullptr;  // mode 6

  double t = 0, alpha1 = 1, beta = 0, prev_f_resid = 0;
  int it = 0;
  bool have_holo = false;
  std::vector<rihvr_iter_record> log;
  int pending_x = -1;  // record whose x-terms arrive with the next prox sweep

  bool profiling = false;
  struct Ev {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Ev> evs;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  size_t bytes = 0;
  long long launches = 0;  // kernels launched by this context
  unsigned long long uid = 0;  // unique for the process (a reused address gets a new one)
  unsigned graph_gen = 0;      // advanced whenever the context's captured graphs are dropped
  cudaEvent_t slab_ev = nullptr;  // end of the slab's partial spectrum (rihvr_slab_iterate)
  float2* slab_stage_h = nullptr; // pinned copy of the spectrum for host-staged reducers
  std::vector<void*> allocs;
};

namespace {

// Allocation-failure injection for the cleanup tests (rihvr_debug_fail_allocations_after):
// when >= 0, the number of device or pinned host allocations that still
// succeed; the one after them fails as if the device were out of memory.
std::atomic<int> g_alloc_budget{-1};

bool injected_alloc_failure() {
  int b = g_alloc_budget.load();
  while (b >= 0) {
    if (g_alloc_budget.compare_exchange_weak(b, b - 1)) return b == 0;
  }
  return false;
}

int dalloc(rihvr_ctx* c, void** p, size_t n) {
  if (injected_alloc_failure()) {
    *p = nullptr;
    return fail(RIHVR_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(n) + " bytes failed (injected)");
  }
  cudaError_t e = cudaMalloc(p, n);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(RIHVR_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(n) + " bytes failed: " +
                                             cudaGetErrorString(e));
  }
  c->allocs.push_back(*p);
  c->bytes += n;
  return RIHVR_OK;
}

template <typename T>
int dalloc_t(rihvr_ctx* c, T** p, size_t count) {
  return dalloc(c, reinterpret_cast<void**>(p), sizeof(T) * count);
}

// pinned host memory; rihvr_destroy frees what is not NULL
template <typename T>
int halloc(T** p, size_t bytes) {
  *p = nullptr;
  if (injected_alloc_failure() || cudaMallocHost(reinterpret_cast<void**>(p), bytes) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(RIHVR_ERR_OUT_OF_MEMORY, "cudaMallocHost of " + std::to_string(bytes) + " bytes failed");
  }
  return RIHVR_OK;
}

// Non-finite samples of a device hologram: one atomic per warp that holds any.
__global__ void k_count_nonfinite(const float* __restrict__ b, size_t n, unsigned* __restrict__ count) {
  unsigned bad = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    bad += isfinite(b[i]) ? 0u : 1u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(count, bad);
}

int elem_kind(int storage) {
  return storage == STORE_BF16 ? ELEM_STORE_BF16 : storage == STORE_F16 ? ELEM_STORE_F16 : ELEM_STORE_F32;
}

cudaEvent_t take_event(rihvr_ctx* c) {
  if (c->ev_used < c->ev_pool.size()) return c->ev_pool[c->ev_used++];
  cudaEvent_t e;
  cudaEventCreate(&e);
  c->ev_pool.push_back(e);
  c->ev_used++;
  return e;
}

struct ProfScope {
  rihvr_ctx* c;
  int cls;
  cudaEvent_t a = nullptr;
  ProfScope(rihvr_ctx* c_, int cls_) : c(c_), cls(cls_) {
    if (c->profiling) {
      a = take_event(c);
      cudaEventRecord(a, c->st);
    }
  }
  ~ProfScope() {
    if (c->profiling) {
      cudaEvent_t b = take_event(c);
      cudaEventRecord(b, c->st);
      c->evs.push_back({cls, a, b});
    }
  }
};

// --- plane-level helpers ----------------------------------------------------

// Rs = FFT2(r) / (W H)  (SparseGradient::reconstruct, sparse_gradient.cu:47-75)
// A variant chosen by name in the environment variable `var` (its index in
// `names`), else `tuned`.
int env_variant(const char* var, std::initializer_list<const char*> names, int tuned) {
  const char* v = std::getenv(var);
  if (!v) return tuned;
  int i = 0;
  for (const char* n : names) {
    if (std::strcmp(v, n) == 0) return i;
    ++i;
  }
  return tuned;
}

int residual_spectrum(rihvr_ctx* c) {
  ProfScope ps(c, K_PLANE);
  KL(launch_rows(0, ELEM_R32, c->r, ELEM_C32, c->pc1, c->W, c->H, 1.0f, c->st));
  KL(launch_plane_col(0, c->pc1, c->Rs, c->W, c->H, 1.0f / (float)c->HW, c->st));
  return RIHVR_OK;
}

int reduce_into(rihvr_ctx* c, int nblocks, int slot) {
  KL(launch_reduce_partials(c->partials, nblocks, c->red_scratch, c->sums_d + slot * kNumSums, c->st));
  if (nblocks > 256) ++c->launches;  // two-stage reduction
  return RIHVR_OK;
}

// G = A^H r: column pass from the spectrum, then the inverse row pass.
int adjoint_volume(rihvr_ctx* c) {
  NvtxRange nvtx_("rihvr: adjoint");
  {
    ProfScope ps(c, K_ADJ_COL);
    const int rec = env_variant("RIHVR_ADJ_COL", {"direct", "recurrence", "recurrence_hoisted", "recurrence_table"},
                                c->tune_adj_rec);
    KL(launch_adj_col(c->Rs, c->cturn, c->zlist, c->U, c->W, c->H, 0, c->Nz, c->st, c->tune_adj_chunks,
                      rec ? c->dz_uniform : 0.0, rec));
  }
  {
    ProfScope ps(c, K_ADJ_ROW);
    KL(launch_rows(1, ELEM_C32, c->U, ELEM_C32, c->G, c->W, (long long)c->Nz * c->H, 1.0f, c->st));
  }
  return RIHVR_OK;
}

// S = sum over the context's planes of H'_z FFT2(vol_z) (the volume in `kind`
// layout): the row and column passes and the sum of the z-chunks.
int forward_partial(rihvr_ctx* c, int kind, const void* vol) {
  {
    ProfScope ps(c, K_FWD_ROW);
    KL(launch_rows(0, kind, vol, ELEM_C32, c->U, c->W, (long long)c->Nz * c->H, 1.0f, c->st));
  }
  {
    ProfScope ps(c, K_FWD_COL);
    const int hor = env_variant("RIHVR_FWD_COL", {"direct", "horner", "horner_onebuf", "horner_tma"},
                                c->tune_fwd_horner);
    KL(launch_fwd_col(c->U, c->cturn, c->zlist, c->Spart, c->W, c->H, 0, c->Nz, c->nchunks, c->st,
                      hor ? c->dz_uniform : 0.0, hor));
  }
  ProfScope ps(c, K_PLANE);
  KL(launch_sum_chunks(c->Spart, c->nchunks, c->S, (long long)c->HW, c->st));
  return RIHVR_OK;
}

// dnew = Re(IFFT2(S_all)) / (W H) from a summed spectrum; sum (dnew - b)^2 into SLOT_FWD.
int forward_from_spectrum(rihvr_ctx* c, const float2* S_all) {
  ProfScope ps(c, K_PLANE);
  KL(launch_plane_col(1, S_all, c->pc1, c->W, c->H, 1.0f, c->st));
  KL(launch_rows(1, ELEM_C32, c->pc1, ELEM_C32, c->pc2, c->W, c->H, 1.0f / (float)c->HW, c->st));
  int nb = 0;
  KL(launch_finish_forward(c->pc2, c->b, c->dnew, (long long)c->HW, c->partials, &nb, c->st));
  return reduce_into(c, nb, SLOT_FWD);
}

// dnew = A vol (the volume in `kind` layout), sum (dnew - b)^2 into SLOT_FWD.
int forward_volume(rihvr_ctx* c, int kind, const void* vol) {
  NvtxRange nvtx_("rihvr: forward");
  RC(forward_partial(c, kind, vol));
  return forward_from_spectrum(c, c->S);
}

ProxArgs prox_args(rihvr_ctx* c, double t, bool device_scalars = false) {
  ProxArgs a;
  a.P = c->vol[c->iCur];
  a.Pprev = c->vol[c->iPrev];
  a.G = c->G;
  a.Pnew = c->vol[c->iNew];
  a.W = c->W;
  a.H = c->H;
  a.Nz = c->Nz;
  a.beta = (float)c->beta;
  a.t = (float)t;
  const double tv = (double)c->p.regularization_TV_param;
  a.mu = (float)(t * tv);
  a.s = tv > 0 ? (float)(1.0 / (4.0 * 3.0 * t * tv)) : 0.f;
  a.thr = (float)(t * (double)c->p.regularization_param);
  a.n_tv = c->p.num_tv_iterations;
  a.faithful = c->p.faithful;
  a.want_norms = c->p.record_objective;
  a.partials = c->partials;
  a.partial_cap = (long long)c->partial_cap;
  a.tv_nseg = c->tune_tv_nseg;
  a.tv_kernel = c->tune_tv_kernel;
  if (c->gdy) {
    a.gdx = c->U;
    a.gdy = c->gdy;
  }
  // proximalFusedLasso2d shrinks only if l1 > 0 (:3715)
  if (c->mode == 7 && !(c->p.regularization_param > 0.f)) a.thr = 0.f;
  if (device_scalars && c->mode != 6) a.dscal = c->scal_d;
  return a;
}

// P_{k+1} = prox(x_k - t G) for the active mode; sums into SLOT_PROX.
int prox_volume(rihvr_ctx* c, double t, bool device_scalars = false) {
  NvtxRange nvtx_("rihvr: prox");
  ProxArgs a = prox_args(c, t, device_scalars);
  int nb = 0;
  ProfScope ps(c, K_PROX);
  if (c->mode == 7) {
    // proximalFusedLasso2d (:3652-3732)
    KL(launch_prox_tv2d(c->storage, a, &nb, c->st));
  } else if (c->mode == 5) {
    KL(launch_prox_l1(c->storage, a, &nb, c->st));
  } else {
    KL(launch_prox6_init(c->storage, a, c->X1, c->st));
    CK(cudaMemsetAsync(c->gx, 0, sizeof(float2) * c->V, c->st));
    CK(cudaMemsetAsync(c->gy, 0, sizeof(float2) * c->V, c->st));
    CK(cudaMemsetAsync(c->gz, 0, sizeof(float2) * c->V, c->st));
    for (int i = 0; i < a.n_tv; ++i) {
      KL(launch_tv3_estimate(c->X1, c->gx, c->gy, c->gz, c->Y, c->W, c->H, c->Nz, a.mu, c->st));
      KL(launch_tv3_dual(c->Y, c->gx, c->gy, c->gz, c->W, c->H, c->Nz, a.s, c->st));
    }
    KL(launch_tv3_estimate(c->X1, c->gx, c->gy, c->gz, c->Y, c->W, c->H, c->Nz, a.mu, c->st));
    KL(launch_prox6_finish(c->storage, a, c->Y, &nb, c->st));
  }
  return reduce_into(c, nb, SLOT_PROX);
}

int fetch_sums(rihvr_ctx* c) {
  CK(cudaMemcpyAsync(c->sums_h, c->sums_d, sizeof(double) * kNumSums * NUM_SLOTS, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RIHVR_OK;
}

double tv_weight(const rihvr_ctx* c) { return c->mode == 5 ? 0.0 : (double)c->p.regularization_TV_param; }

int state_reset(rihvr_ctx* c) {
  for (int i = 0; i < 3; ++i) CK(cudaMemsetAsync(c->vol[i], 0, c->esize * c->V, c->st));
  CK(cudaMemsetAsync(c->dnew, 0, sizeof(float) * c->HW, c->st));
  CK(cudaMemsetAsync(c->dY0, 0, sizeof(float) * c->HW, c->st));
  c->iPrev = 0;
  c->iCur = 1;
  c->iNew = 2;
  c->beta = 0;
  c->alpha1 = 1;
  c->t = c->p.initial_step > 0 ? c->p.initial_step : 1.0 / (double)c->p.num_planes;
  c->it = 0;
  c->log.clear();
  c->pending_x = -1;
  // x = 0: d = 0, r = -b (:273)
  int nb = 0;
  KL(launch_holo_momentum(c->dnew, c->dY0, c->dX, c->b, c->r, 0.f, (long long)c->HW, c->partials, &nb, c->st));
  RC(reduce_into(c, nb, SLOT_MOM));
  RC(residual_spectrum(c));
  RC(fetch_sums(c));
  c->prev_f_resid = 0.5 * c->sums_h[SLOT_MOM * kNumSums + SUM_RR];
  return RIHVR_OK;
}

// Fill the momentum-point terms of the last record from the x-norm sums.
void settle_x_terms(rihvr_ctx* c, const double* s) {
  if (c->pending_x < 0) return;
  rihvr_iter_record& rec = c->log[c->pending_x];
  rec.l1_x = s[SUM_L1X];
  rec.tv_x = s[SUM_TVX];
  rec.f_x = rec.f_resid_x + (double)c->p.regularization_param * rec.l1_x + tv_weight(c) * rec.tv_x;
  c->pending_x = -1;
}

int norms_at_x(rihvr_ctx* c, double* l1x, double* tvx, double* nnz = nullptr) {
  int nb = 0;
  KL(launch_momentum_norms(c->storage, c->vol[c->iCur], c->vol[c->iPrev], (float)c->beta, c->W, c->H, c->Nz,
                           c->mode, c->partials, &nb, c->st));
  RC(reduce_into(c, nb, SLOT_NORM));
  RC(fetch_sums(c));
  *l1x = c->sums_h[SLOT_NORM * kNumSums + SUM_L1X];
  *tvx = c->sums_h[SLOT_NORM * kNumSums + SUM_TVX];
  if (nnz) *nnz = c->sums_h[SLOT_NORM * kNumSums + SUM_LIM1];
  return RIHVR_OK;
}

// GPU work of one attempt: the attempt's scalars to the device, the gradient
// (first attempt of an iteration), the prox, the forward operator and the sums
// back to pinned host memory.  No host synchronisation inside: the same
// sequence is launched eagerly or captured into a graph.
int enqueue_attempt(rihvr_ctx* c, bool with_adjoint) {
  CK(cudaMemcpyAsync(c->scal_d, c->scal_h, 5 * sizeof(float), cudaMemcpyHostToDevice, c->st));
  if (with_adjoint) RC(adjoint_volume(c));
  RC(prox_volume(c, c->t, true));
  RC(forward_volume(c, elem_kind(c->storage), c->vol[c->iNew]));
  CK(cudaMemcpyAsync(c->sums_h, c->sums_d, sizeof(double) * kNumSums * NUM_SLOTS, cudaMemcpyDeviceToHost, c->st));
  return RIHVR_OK;
}

// Hologram momentum, residual at the new momentum point and its spectrum.
int enqueue_momentum(rihvr_ctx* c) {
  CK(cudaMemcpyAsync(c->scal_d + 8, c->scal_h + 8, sizeof(float), cudaMemcpyHostToDevice, c->st));
  int nb = 0;
  KL(launch_holo_momentum(c->dnew, c->dY0, c->dX, c->b, c->r, c->scal_h[8], (long long)c->HW, c->partials, &nb,
                          c->st, c->scal_d + 8));
  RC(reduce_into(c, nb, SLOT_MOM));
  RC(residual_spectrum(c));
  CK(cudaMemcpyAsync(c->sums_h, c->sums_d, sizeof(double) * kNumSums * NUM_SLOTS, cudaMemcpyDeviceToHost, c->st));
  return RIHVR_OK;
}

void drop_graphs(rihvr_ctx* c) {
  ++c->graph_gen;
  for (auto& row : c->g_att)
    for (auto& g : row)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  if (c->g_mom) cudaGraphExecDestroy(c->g_mom);
  c->g_mom = nullptr;
  for (auto& g : c->g_iter)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

bool use_graphs(const rihvr_ctx* c) { return c->graphs && c->warm && !c->profiling && c->mode != 6; }

// Run `enqueue` as a CUDA graph (captured on first use) or eagerly.  A failed
// capture turns graphs off for the context and runs the work eagerly.
template <typename F>
int run_captured(rihvr_ctx* c, cudaGraphExec_t* g, int* nkernels, F enqueue) {
  if (!use_graphs(c)) return enqueue();
  if (!*g) {
    const long long l0 = c->launches;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue();
    cudaError_t e = cudaStreamEndCapture(c->st, &graph);
    if (rc == RIHVR_OK && e == cudaSuccess) e = cudaGraphInstantiate(g, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    const int n = (int)(c->launches - l0);
    c->launches = l0;
    if (rc != RIHVR_OK || e != cudaSuccess) {
      *g = nullptr;
      cudaGetLastError();
      c->graphs = false;
      return enqueue();
    }
    *nkernels = n;
  }
  CK(cudaGraphLaunch(*g, c->st));
  c->launches += *nkernels;
  return RIHVR_OK;
}

// Device-decided iterations.  An attempt: scalars from the device state, the
// gradient (first attempt only), the prox, the forward operator and the
// backtracking test, which sets the graph condition for another attempt.
int enqueue_attempt_dev(rihvr_ctx* c, bool first, cudaGraphConditionalHandle h) {
  const double tv = (double)c->p.regularization_TV_param, l1 = (double)c->p.regularization_param;
  const int zero_thr = (c->mode == 7 && !(c->p.regularization_param > 0.f)) ? 1 : 0;
  KL((k_ctl_prep<<<1, 1, 0, c->st>>>(c->ctl_d, c->scal_d, tv, l1, zero_thr, first ? 1 : 0), cudaGetLastError()));
  if (first) RC(adjoint_volume(c));
  RC(prox_volume(c, c->t, true));
  RC(forward_volume(c, elem_kind(c->storage), c->vol[c->iNew]));
  KL((k_ctl_decide<<<1, 1, 0, c->st>>>(c->ctl_d, c->sums_d, c->p.max_backtracks, h, c->dlog_d, first ? 1 : 0),
      cudaGetLastError()));
  return RIHVR_OK;
}

// Record, restart and momentum factor, then the hologram momentum, the residual
// at the new momentum point and its spectrum.
int enqueue_momentum_dev(rihvr_ctx* c) {
  KL((k_ctl_finish<<<1, 1, 0, c->st>>>(c->ctl_d, c->sums_d, c->scal_d, c->dlog_d,
                                       (double)c->p.regularization_param, tv_weight(c)),
      cudaGetLastError()));
  int nb = 0;
  KL(launch_holo_momentum(c->dnew, c->dY0, c->dX, c->b, c->r, 0.f, (long long)c->HW, c->partials, &nb, c->st,
                          c->scal_d + 8));
  RC(reduce_into(c, nb, SLOT_MOM));
  RC(residual_spectrum(c));
  KL((k_ctl_post<<<1, 1, 0, c->st>>>(c->ctl_d, c->sums_d, c->dlog_d), cudaGetLastError()));
  return RIHVR_OK;
}

// One iteration captured into graph g as a branch of its own (root nodes, no
// dependencies): first attempt, a WHILE node whose body is a backtracking
// attempt (run while the test asks for one), then the momentum step.  The
// condition handle belongs to g, so several contexts' iterations can share
// one graph.  n_main / n_body: kernels outside / inside the WHILE body.
int capture_iteration(rihvr_ctx* c, cudaGraph_t g, int* n_main, int* n_body) {
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  const long long l0 = c->launches;
  struct LaunchGuard {
    rihvr_ctx* c;
    long long l0;
    ~LaunchGuard() { c->launches = l0; }
  } lguard{c, l0};
  CK(cudaStreamBeginCaptureToGraph(c->st, g, nullptr, nullptr, 0, mode));
  int rc = enqueue_attempt_dev(c, true, h);
  cudaStreamCaptureStatus status;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(c->st, &status, nullptr, nullptr, &deps, &ndeps);
  std::vector<cudaGraphNode_t> tail(deps, deps + (e == cudaSuccess ? ndeps : 0));
  cudaGraph_t cap = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(c->st, &cap);
  if (rc != RIHVR_OK) return rc;
  CK(e);
  CK(e2);
  const long long l1 = c->launches;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond;
  CK(cudaGraphAddNode(&cond, g, tail.data(), tail.size(), &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, mode));
  rc = enqueue_attempt_dev(c, false, h);
  e = cudaStreamEndCapture(c->st, &cap);
  if (rc != RIHVR_OK) return rc;
  CK(e);
  const long long l2 = c->launches;
  CK(cudaStreamBeginCaptureToGraph(c->st, g, &cond, nullptr, 1, mode));
  rc = enqueue_momentum_dev(c);
  e = cudaStreamEndCapture(c->st, &cap);
  if (rc != RIHVR_OK) return rc;
  CK(e);
  *n_main = (int)((l1 - l0) + (c->launches - l2));
  *n_body = (int)(l2 - l1);
  return RIHVR_OK;
}

struct GraphGuard {
  cudaGraph_t g = nullptr;
  ~GraphGuard() {
    if (g) cudaGraphDestroy(g);
  }
};

// One iteration of one context as an executable graph.
int build_iter_graph(rihvr_ctx* c, cudaGraphExec_t* out, int* n_main, int* n_body) {
  GraphGuard guard;
  CK(cudaGraphCreate(&guard.g, 0));
  RC(capture_iteration(c, guard.g, n_main, n_body));
  CK(cudaGraphInstantiate(out, guard.g, 0));
  return RIHVR_OK;
}

// Append the device log of n iterations to the host log, settling the
// momentum-point terms of each record from the next iteration's first sweep
// (what settle_x_terms does on the host path).
void pull_dev_log(rihvr_ctx* c, int n) {
  for (int k = 0; k < n; ++k) {
    const DevRec& d = c->dlog_h[k];
    if (c->p.record_objective) {
      double sx[kNumSums] = {0};
      sx[SUM_L1X] = d.prev_l1x;
      sx[SUM_TVX] = d.prev_tvx;
      settle_x_terms(c, sx);
    }
    c->log.push_back(d.rec);
    c->pending_x = (int)c->log.size() - 1;
  }
}

// n iterations without host synchronisation between them: the graphs are
// launched back to back and the log is read every kDevLogCap iterations.
// The host's loop state into the pinned control block, before a run of
// device-decided iterations.
void stage_ctl(rihvr_ctx* c) {
  IterCtl& h = *c->ctl_h;
  h.t = c->t;
  h.alpha1 = c->alpha1;
  h.beta = c->beta;
  h.prev_f_resid = c->prev_f_resid;
  h.f_resid = h.lim = h.ratio = 0.0;
  h.bt = 0;
  h.it = c->it;
  h.it_base = c->it;
  h.pad = 0;
}

// After m device-decided iterations (control block and log read back): the
// loop state, the launch count of the backtracking attempts (n_body kernels
// each) and the iteration log.
void take_ctl(rihvr_ctx* c, int m, int n_body) {
  const IterCtl& h = *c->ctl_h;
  c->t = h.t;
  c->alpha1 = h.alpha1;
  c->beta = h.beta;
  c->prev_f_resid = h.prev_f_resid;
  c->it = h.it;
  for (int k = 0; k < m; ++k) c->launches += (long long)c->dlog_h[k].rec.backtracks * n_body;
  pull_dev_log(c, m);
}

void rotate(rihvr_ctx* c) {
  const int old_prev = c->iPrev;
  c->iPrev = c->iCur;
  c->iCur = c->iNew;
  c->iNew = old_prev;
}

int run_iterations_dev(rihvr_ctx* c, int n) {
  NvtxRange nvtx_("rihvr: device-decided iterations");
  for (int done = 0; done < n;) {
    const int m = std::min(n - done, kDevLogCap);
    stage_ctl(c);
    CK(cudaMemcpyAsync(c->ctl_d, c->ctl_h, sizeof(IterCtl), cudaMemcpyHostToDevice, c->st));
    for (int k = 0; k < m; ++k) {
      const int slot = c->iCur;
      CK(cudaGraphLaunch(c->g_iter[slot], c->st));
      c->launches += c->g_iter_n[slot][0];
      rotate(c);
    }
    CK(cudaMemcpyAsync(c->ctl_h, c->ctl_d, sizeof(IterCtl), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(c->dlog_h, c->dlog_d, sizeof(DevRec) * m, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    take_ctl(c, m, c->g_iter_n[0][1]);
    done += m;
  }
  return RIHVR_OK;
}

// Several contexts' iterations as one graph launch per iteration: each
// context's iteration is a branch of the same graph with its own WHILE node
// and condition, so the frames' kernels run concurrently and the host launches
// once per iteration for all of them.  Every branch is the sequence
// build_iter_graph captures for its context alone, so each frame's iterates
// are those of run_iterations_dev, bit for bit.
struct BatchGraphs {
  cudaGraphExec_t g[3] = {};
  std::vector<int> n_main[3];
  std::vector<int> n_body;
  BatchGraphs() = default;
  BatchGraphs(const BatchGraphs&) = delete;
  BatchGraphs& operator=(const BatchGraphs&) = delete;
  ~BatchGraphs() {
    for (auto& x : g)
      if (x) cudaGraphExecDestroy(x);
  }
};

// One graph per position of P_k in the rotation, as ensure_iter_graphs.
int build_batch_graphs(rihvr_ctx* const* cs, int n, BatchGraphs& B) {
  B.n_body.assign(n, 0);
  for (int slot = 0; slot < 3; ++slot) {
    B.n_main[slot].assign(n, 0);
    GraphGuard guard;
    CK(cudaGraphCreate(&guard.g, 0));
    for (int i = 0; i < n; ++i) {
      rihvr_ctx* c = cs[i];
      const int p0 = c->iPrev, c0 = c->iCur, n0 = c->iNew;
      c->iCur = slot;
      c->iPrev = (slot + 2) % 3;
      c->iNew = (slot + 1) % 3;
      const int rc = capture_iteration(c, guard.g, &B.n_main[slot][i], &B.n_body[i]);
      c->iPrev = p0;
      c->iCur = c0;
      c->iNew = n0;
      if (rc != RIHVR_OK) return rc;
    }
    CK(cudaGraphInstantiate(&B.g[slot], guard.g, 0));
  }
  return RIHVR_OK;
}

struct EventGuard {
  cudaEvent_t e = nullptr;
  ~EventGuard() {
    if (e) cudaEventDestroy(e);
  }
};

// n iterations of every context through the batch graphs, launched on the
// first context's stream; the other streams are ordered before and after it.
// The contexts share a device and a rotation position.
int run_iterations_batch(rihvr_ctx* const* cs, int nc, int n, const BatchGraphs& B) {
  cudaStream_t st = cs[0]->st;
  EventGuard ev;
  CK(cudaEventCreateWithFlags(&ev.e, cudaEventDisableTiming));
  for (int i = 1; i < nc; ++i) {
    CK(cudaEventRecord(ev.e, cs[i]->st));
    CK(cudaStreamWaitEvent(st, ev.e, 0));
  }
  for (int done = 0; done < n;) {
    const int m = std::min(n - done, kDevLogCap);
    for (int i = 0; i < nc; ++i) {
      stage_ctl(cs[i]);
      CK(cudaMemcpyAsync(cs[i]->ctl_d, cs[i]->ctl_h, sizeof(IterCtl), cudaMemcpyHostToDevice, st));
    }
    for (int k = 0; k < m; ++k) {
      const int slot = cs[0]->iCur;
      CK(cudaGraphLaunch(B.g[slot], st));
      for (int i = 0; i < nc; ++i) {
        cs[i]->launches += B.n_main[slot][i];
        rotate(cs[i]);
      }
    }
    for (int i = 0; i < nc; ++i) {
      CK(cudaMemcpyAsync(cs[i]->ctl_h, cs[i]->ctl_d, sizeof(IterCtl), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(cs[i]->dlog_h, cs[i]->dlog_d, sizeof(DevRec) * m, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    for (int i = 0; i < nc; ++i) take_ctl(cs[i], m, B.n_body[i]);
    done += m;
  }
  CK(cudaEventRecord(ev.e, st));
  for (int i = 1; i < nc; ++i) CK(cudaStreamWaitEvent(cs[i]->st, ev.e, 0));
  return RIHVR_OK;
}

// Whole solves as one graph launch (batch mode 2).  Every frame is a branch of
// one graph: a kernel that sets the frame's loop condition from its device
// loop state, then a WHILE node whose body selects the iteration capture for
// the frame's current rotation position with a SWITCH node (three bodies,
// each the sequence capture_iteration records, with its own WHILE node of
// backtracking attempts) and advances the loop state.  Each frame loops on the
// device at its own pace, with its own iteration count; the host launches the
// graph once for up to kDevLogCap iterations of every frame.  Every body is
// the sequence build_iter_graph captures, so the iterates are those of
// run_iterations_dev, bit for bit.
struct LoopCtl {
  int remaining;  // iterations still to run in this launch
  int slot;       // position of P_k in the rotation
};

__global__ void k_loop_init(const LoopCtl* L, cudaGraphConditionalHandle hw) {
  cudaGraphSetConditional(hw, L->remaining > 0 ? 1u : 0u);
}
__global__ void k_loop_select(const LoopCtl* L, cudaGraphConditionalHandle hs) {
  cudaGraphSetConditional(hs, (unsigned)L->slot);
}
__global__ void k_loop_step(LoopCtl* L, cudaGraphConditionalHandle hw) {
  L->remaining -= 1;
  L->slot = L->slot == 2 ? 0 : L->slot + 1;  // rotate(): the new P_k is the old P_{k+1}
  cudaGraphSetConditional(hw, L->remaining > 0 ? 1u : 0u);
}

struct SolveGraph {
  cudaGraphExec_t g = nullptr;
  LoopCtl* L_d = nullptr;  // one per frame
  LoopCtl* L_h = nullptr;  // pinned staging
  std::vector<int> n_main, n_body;
  SolveGraph() = default;
  SolveGraph(const SolveGraph&) = delete;
  SolveGraph& operator=(const SolveGraph&) = delete;
  ~SolveGraph() {
    if (g) cudaGraphExecDestroy(g);
    if (L_d) cudaFree(L_d);
    if (L_h) cudaFreeHost(L_h);
  }
};

// capture `enqueue` (kernel launches on c->st) into graph g after `deps`;
// `tail` receives the capture's last nodes
template <typename F>
int capture_into(rihvr_ctx* c, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
                 std::vector<cudaGraphNode_t>* tail, F enqueue) {
  CK(cudaStreamBeginCaptureToGraph(c->st, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                   cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue();
  cudaStreamCaptureStatus status;
  const cudaGraphNode_t* d = nullptr;
  size_t nd = 0;
  const cudaError_t e = cudaStreamGetCaptureInfo(c->st, &status, nullptr, nullptr, &d, &nd);
  if (tail) tail->assign(d, d + (e == cudaSuccess ? nd : 0));
  cudaGraph_t cap = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(c->st, &cap);
  if (rc != RIHVR_OK) return rc;
  CK(e);
  CK(e2);
  return RIHVR_OK;
}

int build_solve_graph(rihvr_ctx* const* cs, int n, SolveGraph& S) {
  S.n_main.assign(n, 0);
  S.n_body.assign(n, 0);
  CK(cudaMalloc(&S.L_d, sizeof(LoopCtl) * n));
  CK(cudaMallocHost(&S.L_h, sizeof(LoopCtl) * n));
  GraphGuard guard;
  CK(cudaGraphCreate(&guard.g, 0));
  for (int i = 0; i < n; ++i) {
    rihvr_ctx* c = cs[i];
    LoopCtl* L = S.L_d + i;
    cudaGraphConditionalHandle hw, hs;
    CK(cudaGraphConditionalHandleCreate(&hw, guard.g, 0, 0));
    std::vector<cudaGraphNode_t> tail;
    RC(capture_into(c, guard.g, {}, &tail, [&]() -> int {
      CK((k_loop_init<<<1, 1, 0, c->st>>>(L, hw), cudaGetLastError()));
      return RIHVR_OK;
    }));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    CK(cudaGraphAddNode(&wnode, guard.g, tail.data(), tail.size(), &wp));
    cudaGraph_t body = wp.conditional.phGraph_out[0];
    CK(cudaGraphConditionalHandleCreate(&hs, body, 0, 0));
    RC(capture_into(c, body, {}, &tail, [&]() -> int {
      CK((k_loop_select<<<1, 1, 0, c->st>>>(L, hs), cudaGetLastError()));
      return RIHVR_OK;
    }));
    cudaGraphNodeParams sp = {};
    sp.type = cudaGraphNodeTypeConditional;
    sp.conditional.handle = hs;
    sp.conditional.type = cudaGraphCondTypeSwitch;
    sp.conditional.size = 3;
    cudaGraphNode_t snode;
    CK(cudaGraphAddNode(&snode, body, tail.data(), tail.size(), &sp));
    const int p0 = c->iPrev, c0 = c->iCur, n0 = c->iNew;
    for (int slot = 0; slot < 3; ++slot) {
      c->iCur = slot;
      c->iPrev = (slot + 2) % 3;
      c->iNew = (slot + 1) % 3;
      const int rc = capture_iteration(c, sp.conditional.phGraph_out[slot], &S.n_main[i], &S.n_body[i]);
      c->iPrev = p0;
      c->iCur = c0;
      c->iNew = n0;
      if (rc != RIHVR_OK) return rc;
    }
    RC(capture_into(c, body, {snode}, nullptr, [&]() -> int {
      CK((k_loop_step<<<1, 1, 0, c->st>>>(L, hw), cudaGetLastError()));
      return RIHVR_OK;
    }));
  }
  CK(cudaGraphInstantiate(&S.g, guard.g, 0));
  return RIHVR_OK;
}

// The last solve graph built, kept for the next batch call on the same
// contexts: its key is every context's uid and graph generation, in order, so
// a context that was re-tuned (its graphs dropped) or destroyed never reuses
// it; rihvr_destroy releases it when one of its contexts goes.
struct SolveCache {
  std::mutex mu;
  std::vector<std::pair<unsigned long long, unsigned>> key;
  std::unique_ptr<SolveGraph> S;
};
SolveCache& solve_cache() {
  static SolveCache* cache = new SolveCache;  // never destroyed: no CUDA calls at process exit
  return *cache;
}

std::vector<std::pair<unsigned long long, unsigned>> solve_key(rihvr_ctx* const* cs, int n) {
  std::vector<std::pair<unsigned long long, unsigned>> k(n);
  for (int i = 0; i < n; ++i) k[i] = {cs[i]->uid, cs[i]->graph_gen};
  return k;
}

// the cached solve graph for these contexts (removed from the cache while in
// use), or a newly built one; null on failure
std::unique_ptr<SolveGraph> take_solve_graph(rihvr_ctx* const* cs, int n) {
  const auto key = solve_key(cs, n);
  {
    SolveCache& sc = solve_cache();
    std::lock_guard<std::mutex> lk(sc.mu);
    if (sc.S && sc.key == key) {
      sc.key.clear();
      return std::move(sc.S);
    }
  }
  std::unique_ptr<SolveGraph> S(new (std::nothrow) SolveGraph);
  if (!S || build_solve_graph(cs, n, *S) != RIHVR_OK) return nullptr;
  return S;
}

void keep_solve_graph(rihvr_ctx* const* cs, int n, std::unique_ptr<SolveGraph> S) {
  SolveCache& sc = solve_cache();
  std::lock_guard<std::mutex> lk(sc.mu);
  sc.key = solve_key(cs, n);
  sc.S = std::move(S);  // the previous one, if any, is released here
}

// a context is going away: drop a cached solve graph that runs it
void forget_solve_graph(const rihvr_ctx* c) {
  SolveCache& sc = solve_cache();
  std::lock_guard<std::mutex> lk(sc.mu);
  for (const auto& k : sc.key)
    if (k.first == c->uid) {
      sc.S.reset();
      sc.key.clear();
      return;
    }
}

// iters[i] iterations of every context through the solve graph, at most
// kDevLogCap a launch, on the first context's stream (the other streams are
// ordered before and after it).  The contexts share a device.
int run_solves_graph(rihvr_ctx* const* cs, int nc, const std::vector<int>& iters, const SolveGraph& S) {
  cudaStream_t st = cs[0]->st;
  EventGuard ev;
  CK(cudaEventCreateWithFlags(&ev.e, cudaEventDisableTiming));
  for (int i = 1; i < nc; ++i) {
    CK(cudaEventRecord(ev.e, cs[i]->st));
    CK(cudaStreamWaitEvent(st, ev.e, 0));
  }
  std::vector<int> done(nc, 0);
  for (;;) {
    bool any = false;
    std::vector<int> m(nc, 0);
    for (int i = 0; i < nc; ++i) {
      m[i] = std::min(iters[i] - done[i], kDevLogCap);
      any = any || m[i] > 0;
    }
    if (!any) break;
    for (int i = 0; i < nc; ++i) {
      S.L_h[i].remaining = m[i];
      S.L_h[i].slot = cs[i]->iCur;
      stage_ctl(cs[i]);
      CK(cudaMemcpyAsync(cs[i]->ctl_d, cs[i]->ctl_h, sizeof(IterCtl), cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(S.L_d, S.L_h, sizeof(LoopCtl) * nc, cudaMemcpyHostToDevice, st));
    CK(cudaGraphLaunch(S.g, st));
    for (int i = 0; i < nc; ++i) {
      CK(cudaMemcpyAsync(cs[i]->ctl_h, cs[i]->ctl_d, sizeof(IterCtl), cudaMemcpyDeviceToHost, st));
      if (m[i] > 0)
        CK(cudaMemcpyAsync(cs[i]->dlog_h, cs[i]->dlog_d, sizeof(DevRec) * m[i], cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    for (int i = 0; i < nc; ++i) {
      if (m[i] == 0) continue;
      cs[i]->launches += 1 + (long long)m[i] * (S.n_main[i] + 2);  // + the loop kernels
      take_ctl(cs[i], m[i], S.n_body[i]);
      for (int k = 0; k < m[i]; ++k) rotate(cs[i]);
      done[i] += m[i];
    }
  }
  CK(cudaEventRecord(ev.e, st));
  for (int i = 1; i < nc; ++i) CK(cudaStreamWaitEvent(cs[i]->st, ev.e, 0));
  return RIHVR_OK;
}

// RIHVR_ITER_LOOP=host selects the host-synchronised loop (one_iteration)
// instead, for comparison; both give the same iterates bit for bit.
bool dev_loop_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("RIHVR_ITER_LOOP");
    return !(v && std::strcmp(v, "host") == 0);
  }();
  return on;
}

// How rihvr_reconstruct_batch runs the iterations after the first
// (rihvr_set_batch_mode): 0 = each frame's own device loop on its own host
// thread and stream, 1 = one graph launch per iteration for all frames,
// 2 = one graph launch for the whole solves of all frames.
std::atomic<int> g_batch_mode{0};

// whether the last rihvr_reconstruct_batch call on this host thread ran its
// frames as one graph launch per iteration
thread_local int g_batch_combined = 0;

bool use_dev_loop(const rihvr_ctx* c) { return c->dev_loop && dev_loop_enabled() && use_graphs(c) && c->mode != 6; }

// The three iteration graphs, one per position of P_k in the rotation
// (iPrev, iCur, iNew) = (iCur + 2, iCur, iCur + 1) mod 3, built before any is
// launched; on failure none is kept.
int ensure_iter_graphs(rihvr_ctx* c) {
  const int p0 = c->iPrev, c0 = c->iCur, n0 = c->iNew;
  int rc = RIHVR_OK;
  for (int slot = 0; slot < 3 && rc == RIHVR_OK; ++slot) {
    if (c->g_iter[slot]) continue;
    c->iCur = slot;
    c->iPrev = (slot + 2) % 3;
    c->iNew = (slot + 1) % 3;
    rc = build_iter_graph(c, &c->g_iter[slot], &c->g_iter_n[slot][0], &c->g_iter_n[slot][1]);
    if (rc != RIHVR_OK) c->g_iter[slot] = nullptr;
  }
  c->iPrev = p0;
  c->iCur = c0;
  c->iNew = n0;
  if (rc != RIHVR_OK) {
    for (auto& g : c->g_iter)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    cudaGetLastError();
  }
  return rc;
}

// One FISTA iteration (:299-611): one host synchronisation per attempt and one
// after the momentum step.
int one_iteration(rihvr_ctx* c) {
  NvtxRange nvtx_("rihvr: iteration (host-decided)");
  double alpha0 = c->alpha1;
  int bt = 0;
  double f_resid = 0, lim = 0, ratio = 0;
  const double* sp = c->sums_h + SLOT_PROX * kNumSums;
  for (;;) {
    {
      const ProxArgs a = prox_args(c, c->t);
      c->scal_h[0] = a.beta;
      c->scal_h[1] = a.t;
      c->scal_h[2] = a.mu;
      c->scal_h[3] = a.s;
      c->scal_h[4] = a.thr;
    }
    const int first = bt == 0 ? 0 : 1;
    RC(run_captured(c, &c->g_att[first][c->iCur], &c->g_att_n[first][c->iCur],
                    [&]() { return enqueue_attempt(c, bt == 0); }));
    CK(cudaStreamSynchronize(c->st));
    if (bt == 0 && c->p.record_objective) settle_x_terms(c, sp);
    f_resid = 0.5 * c->sums_h[SLOT_FWD * kNumSums + SUM_RR];
    lim = sp[SUM_LIM1] + sp[SUM_LIM2] / (2.0 * c->t);
    ratio = f_resid / (c->prev_f_resid + lim);
    if (((ratio > 1.0) || (ratio < 0.0)) && bt < c->p.max_backtracks) {
      c->t *= 0.5;  // stepsize_shrinkage (:63)
      ++bt;
      continue;
    }
    break;
  }
  rihvr_iter_record rec{};
  rec.f_resid_prox = f_resid;
  rec.lim = lim;
  rec.ratio = ratio;
  rec.t = c->t;
  rec.backtracks = bt;
  rec.restart_sum = sp[SUM_RS];
  rec.f_prox = f_resid + (double)c->p.regularization_param * sp[SUM_L1P] + tv_weight(c) * sp[SUM_TVP];
  // fistaRestart (:471-475) and the alpha/beta update (:476-481)
  const bool restarted = sp[SUM_RS] > 0.0;
  if (restarted) alpha0 = 1.0;
  c->alpha1 = (1.0 + std::sqrt(1.0 + 4.0 * alpha0 * alpha0)) / 2.0;
  const double beta = (alpha0 - 1.0) / c->alpha1;
  rec.beta = beta;
  rec.restarted = restarted ? 1 : 0;
  // hologram momentum, residual at the new momentum point and its spectrum
  c->scal_h[8] = (float)beta;
  RC(run_captured(c, &c->g_mom, &c->g_mom_n, [&]() { return enqueue_momentum(c); }));
  CK(cudaStreamSynchronize(c->st));
  // rotate: P_{k-1} <- P_k, P_k <- P_{k+1}
  const int old_prev = c->iPrev;
  c->iPrev = c->iCur;
  c->iCur = c->iNew;
  c->iNew = old_prev;
  c->beta = beta;
  c->prev_f_resid = 0.5 * c->sums_h[SLOT_MOM * kNumSums + SUM_RR];
  rec.f_resid_x = c->prev_f_resid;
  rec.f_x = rec.f_resid_x;
  c->log.push_back(rec);
  c->pending_x = (int)c->log.size() - 1;
  c->it++;
  c->warm = true;
  return RIHVR_OK;
}

// The momentum-point terms of the last record, when the objective is recorded.
int settle_pending(rihvr_ctx* c) {
  if (c->p.record_objective && c->pending_x >= 0) {
    double l1x, tvx;
    RC(norms_at_x(c, &l1x, &tvx));
    double s[kNumSums] = {0};
    s[SUM_L1X] = l1x;
    s[SUM_TVX] = tvx;
    settle_x_terms(c, s);
  }
  return RIHVR_OK;
}

// Iterations i .. n-1 of a run, after the eager first one (when it ran).
int run_iterations_from(rihvr_ctx* c, int i, int n) {
  if (i < n && use_dev_loop(c)) {
    if (ensure_iter_graphs(c) == RIHVR_OK) {
      RC(run_iterations_dev(c, n - i));
      i = n;
    } else {
      c->dev_loop = false;  // the attempt and momentum graphs of one_iteration instead
    }
  }
  for (; i < n; ++i) RC(one_iteration(c));
  return settle_pending(c);
}

// The first iteration of a context runs eagerly (it sets kernel attributes
// and builds tables that graph capture must not see); returns how many ran.
int eager_start(rihvr_ctx* c, int n, int* ran) {
  *ran = 0;
  if (n > 0 && !c->warm) {
    RC(one_iteration(c));
    *ran = 1;
  }
  return RIHVR_OK;
}

// The TMA-fed forward column pass bounds its waits; a wait that ran out left a
// forward sum incomplete, which is reported here instead of a wrong result.
int check_col_waits(rihvr_ctx* c) {
  unsigned n = 0;
  CK(col_wait_timeouts(c->st, &n));
  if (n)
    return fail(RIHVR_ERR_CUDA, std::to_string(n) + " bounded wait(s) of the forward column pass ran out");
  return RIHVR_OK;
}

// Whole-volume operations refuse a context that holds only some planes.
int whole_volume(const rihvr_ctx* c, const char* what) {
  if (c->Nz < c->p.num_planes)
    return fail(RIHVR_ERR_INVALID_STATE, std::string(what) + " needs every plane; this z-slab context holds " +
                                             std::to_string(c->Nz) + " of " + std::to_string(c->p.num_planes) +
                                             " (whole solves of slabs go through rihvr_slab_iterate)");
  return RIHVR_OK;
}

int run_iterations(rihvr_ctx* c, int n) {
  RC(whole_volume(c, "iterating"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  int i = 0;
  RC(eager_start(c, n, &i));
  RC(run_iterations_from(c, i, n));
  return check_col_waits(c);
}

int copy_out(rihvr_ctx* c, void* dst, const void* src, size_t bytes, int is_device) {
  CK(cudaMemcpyAsync(dst, src, bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return RIHVR_OK;
}

int copy_in(rihvr_ctx* c, void* dst, const void* src, size_t bytes, int is_device) {
  CK(cudaMemcpyAsync(dst, src, bytes, is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st));
  return RIHVR_OK;
}

int validate(const rihvr_params* p, int W, int H) {
  if (!p) return fail(RIHVR_ERR_INVALID_ARGUMENT, "params is NULL");
  if (W <= 0 || H <= 0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "width and height must be positive");
  // Square planes of side 32, 48, 64, 128, 256, 384, 512, 640, 768, 1024 or 2304 take the
  // register-resident FFT passes; any other even width and height from 16 to
  // 4096 whose prime factors are 2, 3, 5 and 7 takes the generic passes (the
  // reference needs multiples of 16, :126, 1948).
  for (int n : {W, H}) {
    if (n < 16 || (n & 1) || !(line_size_supported(n) || generic_size_supported(n)))
      return fail(RIHVR_ERR_UNSUPPORTED_SIZE,
                  "unsupported plane size " + std::to_string(W) + " x " + std::to_string(H) +
                      " (each side even, 16..4096, prime factors 2, 3, 5, 7 only)");
  }
  if (p->num_planes < 1) return fail(RIHVR_ERR_INVALID_ARGUMENT, "num_planes must be >= 1");
  if (p->mode != 5 && p->mode != 6 && p->mode != 7)
    return fail(RIHVR_ERR_UNKNOWN_MODE, "mode must be 5, 6 or 7 (unsupported mode)");
  if (p->storage < 0 || p->storage > 2) return fail(RIHVR_ERR_INVALID_ARGUMENT, "storage must be 0, 1 or 2");
  // BF16 storage rounds every stored iterate to 8 significant bits; at the
  // 1024 x 1024 x 1000 workload the objective then ends 2.3e-2 from the FP64
  // solution, outside the 1e-2 tolerance of reduced-precision storage.  FP16
  // (11 bits, 2.6e-4 there) meets it, so reference-faithful solves refuse BF16.
  if (p->storage == STORE_BF16 && p->faithful)
    return fail(RIHVR_ERR_INVALID_ARGUMENT,
                "BF16 volume storage misses the 1e-2 objective tolerance of faithful solves; use FP16 (storage 2) "
                "or faithful = 0");
  if (p->num_tv_iterations < 0 || p->num_tv_iterations > 20)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "num_tv_iterations must be in 0..20");
  if (!(p->wavelength > 0.f) || !(p->resolution > 0.f))
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "wavelength and resolution must be positive");
  if (p->regularization_param < 0.f || p->regularization_TV_param < 0.f)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "regularization weights must be non-negative");
  if (p->max_backtracks < 0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "max_backtracks must be >= 0");
  return RIHVR_OK;
}

// c(f)/(2 pi) per frequency, in turns per unit z (sparse_rs_exponent_kernel,
// :38-56, combined with the carrier phase of sparse_phase_scale_kernel).
void phase_turns(int H, int W, double dx, double lambda, std::vector<double>& out) {
  out.resize((size_t)H * W);
  const double q = (lambda / dx) * (lambda / dx);
  for (int y = 0; y < H; ++y) {
    const double fy = (double)(((y + H / 2) % H) - (H / 2)) / (double)H;
    for (int x = 0; x < W; ++x) {
      const double fx = (double)(((x + W / 2) % W) - (W / 2)) / (double)W;
      const double a = q * (fx * fx + fy * fy);
      const double sm1 = (a >= 1.0) ? -1.0 : -a / (std::sqrt(1.0 - a) + 1.0);
      out[(size_t)y * W + x] = sm1 / lambda;  // (2 pi / lambda)(s - 1) / (2 pi)
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* rihvr_last_error(void) { return g_last_error.c_str(); }

const char* rihvr_status_string(int s) {
  switch (s) {
    case RIHVR_OK: return "ok";
    case RIHVR_ERR_UNKNOWN_TYPE: return "unknown type";
    case RIHVR_ERR_BAD_FILENAME: return "bad filename";
    case RIHVR_ERR_MISSING_DATA: return "missing data";
    case RIHVR_ERR_INVALID_STATE: return "invalid state";
    case RIHVR_ERR_OUT_OF_MEMORY: return "out of memory";
    case RIHVR_ERR_UNKNOWN_MODE: return "unknown mode";
    case RIHVR_ERR_INVALID_ARGUMENT: return "invalid argument";
    case RIHVR_ERR_UNKNOWN_ERROR: return "unknown error";
    case RIHVR_ERR_INVALID_FILE: return "invalid file";
    case RIHVR_ERR_INVALID_DATA: return "invalid data";
    case RIHVR_ERR_CRITICAL_ASSUMPTION: return "critical assumption";
    case RIHVR_ERR_INFINITE_LOOP: return "infinite loop";
    case RIHVR_ERR_CUDA: return "CUDA error";
    case RIHVR_ERR_NO_DEVICE: return "no CUDA device";
    case RIHVR_ERR_UNSUPPORTED_SIZE: return "unsupported size";
    default: return "unrecognised status";
  }
}

int rihvr_debug_fail_allocations_after(int n) { return g_alloc_budget.exchange(n < 0 ? -1 : n); }

}  // extern "C"

namespace {

// A context for planes [z_first, z_first + z_count) of the plane list
// (all of them for rihvr_create); params and sizes already validated.
int create_ctx(const rihvr_params* params, int width, int height, int z_first, int z_count, rihvr_ctx** out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(RIHVR_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  rihvr_ctx* c = new (std::nothrow) rihvr_ctx();
  if (!c) return fail(RIHVR_ERR_OUT_OF_MEMORY, "host allocation failed");
  static std::atomic<unsigned long long> next_uid{1};
  c->uid = next_uid.fetch_add(1);
  c->p = *params;
  c->W = width;
  c->H = height;
  c->Nz = z_count;
  c->z_first = z_first;
  c->HW = (size_t)width * height;
  c->V = c->HW * c->Nz;
  // No TV regularisation means the L1 prox (:187-195)
  c->mode = params->regularization_TV_param == 0.f ? 5 : params->mode;
  c->storage = params->storage;
  c->esize = params->storage == STORE_F32 ? 8 : 4;
  cudaGetDevice(&c->device);
  auto cleanup = [&](int rc) {
    rihvr_destroy(c);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(RIHVR_ERR_CUDA, "cudaStreamCreate failed"));
  int rc = RIHVR_OK;
  for (int i = 0; i < 3 && rc == RIHVR_OK; ++i) rc = dalloc(c, &c->vol[i], c->esize * c->V);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->G, c->V);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->U, c->V);
  c->nchunks = fwd_col_chunks(width, height, c->Nz);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->Spart, c->HW * kMaxFwdChunks);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->S, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->pc1, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->pc2, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->Rs, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->b, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->dnew, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->dY0, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->dX, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->r, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->cturn, c->HW);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->zlist, (size_t)c->Nz);
  // 6-10 TV iterations run as two streaming launches whose dual goes through
  // memory: gx in U (free during the prox) and gy in one more volume
  if (c->mode == 7 && c->p.num_tv_iterations >= 6 && c->p.num_tv_iterations <= 10 && rc == RIHVR_OK)
    rc = dalloc_t(c, &c->gdy, c->V);
  if (c->mode == 6) {
    if (rc == RIHVR_OK) rc = dalloc_t(c, &c->X1, c->V);
    if (rc == RIHVR_OK) rc = dalloc_t(c, &c->gx, c->V);
    if (rc == RIHVR_OK) rc = dalloc_t(c, &c->gy, c->V);
    if (rc == RIHVR_OK) rc = dalloc_t(c, &c->gz, c->V);
    if (rc == RIHVR_OK) rc = dalloc_t(c, &c->Y, c->V);
  }
  c->partial_cap = max_partial_blocks(width, height, c->Nz);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->partials, c->partial_cap * kNumSums);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->sums_d, (size_t)kNumSums * NUM_SLOTS);
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->red_scratch, reduce_scratch_doubles());
  if (rc == RIHVR_OK) rc = dalloc_t(c, &c->nonfinite_d, 1);
  if (rc != RIHVR_OK) return cleanup(rc);
  if (halloc(&c->sums_h, sizeof(double) * kNumSums * NUM_SLOTS) != RIHVR_OK) return cleanup(RIHVR_ERR_OUT_OF_MEMORY);
  if (halloc(&c->scal_h, 16 * sizeof(float)) != RIHVR_OK) return cleanup(RIHVR_ERR_OUT_OF_MEMORY);
  std::memset(c->scal_h, 0, 16 * sizeof(float));
  if (dalloc_t(c, &c->scal_d, 16) != RIHVR_OK) return cleanup(RIHVR_ERR_OUT_OF_MEMORY);
  if (halloc(&c->ctl_h, sizeof(IterCtl)) != RIHVR_OK || halloc(&c->dlog_h, sizeof(DevRec) * kDevLogCap) != RIHVR_OK)
    return cleanup(RIHVR_ERR_OUT_OF_MEMORY);
  if (dalloc_t(c, &c->ctl_d, 1) != RIHVR_OK || dalloc_t(c, &c->dlog_d, kDevLogCap) != RIHVR_OK)
    return cleanup(RIHVR_ERR_OUT_OF_MEMORY);
  std::vector<double> ct;
  phase_turns(height, width, (double)params->resolution, (double)params->wavelength, ct);
  std::vector<double> zall((size_t)params->num_planes);
  rihvr_plane_list(params, zall.data());
  const std::vector<double> zl(zall.begin() + z_first, zall.begin() + z_first + z_count);
  // evenly spaced planes (exactly, in FP64) let the adjoint advance H'_z by a recurrence
  c->dz_uniform = c->Nz > 1 ? zl[1] - zl[0] : 1.0;
  for (int k = 1; k + 1 < c->Nz && c->dz_uniform != 0; ++k)
    if (zl[(size_t)k + 1] - zl[(size_t)k] != c->dz_uniform) c->dz_uniform = 0;
  if (cudaMemcpy(c->cturn, ct.data(), sizeof(double) * ct.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->zlist, zl.data(), sizeof(double) * zl.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemsetAsync(c->b, 0, sizeof(float) * c->HW, c->st) != cudaSuccess)
    return cleanup(fail(RIHVR_ERR_CUDA, "initial copies failed"));
  *out = c;
  return RIHVR_OK;
}

}  // namespace

extern "C" {

int rihvr_create(const rihvr_params* params, int width, int height, rihvr_ctx** out) {
  if (!out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  RC(validate(params, width, height));
  return create_ctx(params, width, height, 0, params->num_planes, out);
}

int rihvr_create_slab(const rihvr_params* params, int width, int height, int z_first, int z_count,
                      rihvr_ctx** out) {
  if (!out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  RC(validate(params, width, height));
  if (z_first < 0 || z_count < 1 || z_count > params->num_planes - z_first)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "planes [" + std::to_string(z_first) + ", " +
                                                std::to_string((long long)z_first + z_count) + ") are not within 0.." +
                                                std::to_string(params->num_planes));
  // 3-D TV (mode 6) couples each plane to its neighbours across slab boundaries
  if (params->regularization_TV_param != 0.f && params->mode == 6)
    return fail(RIHVR_ERR_UNKNOWN_MODE, "z-slabs need a plane-separable prox (mode 5 or 7), not 3-D TV (mode 6)");
  return create_ctx(params, width, height, z_first, z_count, out);
}

void rihvr_destroy(rihvr_ctx* c) {
  if (!c) return;
  if (c->st) cudaStreamSynchronize(c->st);
  forget_solve_graph(c);
  drop_graphs(c);
  if (c->seg_ws) seg_workspace_destroy(c->seg_ws);
  frame_workspace_free(c->frame_ws);
  for (void* p : c->allocs) cudaFree(p);
  if (c->sums_h) cudaFreeHost(c->sums_h);
  if (c->scal_h) cudaFreeHost(c->scal_h);
  if (c->ctl_h) cudaFreeHost(c->ctl_h);
  if (c->dlog_h) cudaFreeHost(c->dlog_h);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  if (c->slab_ev) cudaEventDestroy(c->slab_ev);
  if (c->slab_stage_h) cudaFreeHost(c->slab_stage_h);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

int rihvr_set_hologram(rihvr_ctx* c, const float* b, int is_device) {
  NvtxRange nvtx_("rihvr: set hologram");
  if (!c || !b) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  // A NaN or infinite sample would poison every later iterate.  The reference
  // only prints a warning per bad sample and carries on (check_isnan_mdata,
  // sparse_compressive_holo.cu:9-35); here the hologram is refused with the
  // reference's HOLO_ERROR_INVALID_DATA code and the context keeps its state.
  size_t bad = 0;
  if (!is_device) {
    for (size_t i = 0; i < c->HW; ++i) bad += std::isfinite(b[i]) ? 0 : 1;
  } else {
    CK(cudaMemsetAsync(c->nonfinite_d, 0, sizeof(unsigned), c->st));
    const int blocks = (int)std::min<size_t>((c->HW + 255) / 256, 1184);
    KL((k_count_nonfinite<<<blocks, 256, 0, c->st>>>(b, c->HW, c->nonfinite_d), cudaGetLastError()));
    unsigned n = 0;
    CK(cudaMemcpyAsync(&n, c->nonfinite_d, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    bad = n;
  }
  if (bad)
    return fail(RIHVR_ERR_INVALID_DATA, "hologram has " + std::to_string(bad) + " non-finite samples");
  RC(copy_in(c, c->b, b, sizeof(float) * c->HW, is_device));
  c->have_holo = true;
  RC(state_reset(c));
  if (c->p.autotune && !c->tuned) RC(rihvr_autotune(c, nullptr));
  return RIHVR_OK;
}

int rihvr_set_hologram_frame(rihvr_ctx* c, const void* frame, int bits, int width, int height,
                             const void* background, const rihvr_file_params* files, int is_device) {
  if (!c || !frame) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  const float* staged = nullptr;
  // the frame is preprocessed into the workspace; the context's hologram and
  // state change only when that succeeded
  RC(frame_to_hologram(&c->frame_ws, frame, bits, width, height, background, files, c->p.zero_padding, c->W, c->H,
                       is_device, c->st, &staged, &c->launches));
  RC(copy_in(c, c->b, staged, sizeof(float) * c->HW, 1));
  c->have_holo = true;
  RC(state_reset(c));
  if (c->p.autotune && !c->tuned) RC(rihvr_autotune(c, nullptr));
  return RIHVR_OK;
}

int rihvr_get_hologram(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  return copy_out(c, out, c->b, sizeof(float) * c->HW, is_device);
}

}  // extern "C"

namespace {

// Launch shapes tuned per (device, W, H, Nz, n_tv, mode, storage, norms).
struct TuneKey {
  int dev, W, H, Nz, ntv, mode, storage, norms;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, W, H, Nz, ntv, mode, storage, norms) <
           std::tie(o.dev, o.W, o.H, o.Nz, o.ntv, o.mode, o.storage, o.norms);
  }
};
struct TuneVal {
  int adj_chunks, fwd_chunks, tv_nseg, tv_kernel, adj_rec, fwd_horner;
  double ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

// fastest of three timed launches after one warm-up, in ms
template <typename F>
int time_min(rihvr_ctx* c, cudaEvent_t e0, cudaEvent_t e1, F launch, float* best) {
  RC(launch());
  *best = 1e30f;
  for (int r = 0; r < 3; ++r) {
    CK(cudaEventRecord(e0, c->st));
    RC(launch());
    CK(cudaEventRecord(e1, c->st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *best = std::min(*best, ms);
  }
  return RIHVR_OK;
}

int autotune_run(rihvr_ctx* c, cudaEvent_t e0, cudaEvent_t e1, TuneVal* out) {
  drop_graphs(c);  // captured launches carry the old shapes
  const int prev_profiling = c->profiling;
  c->profiling = false;
  float best;
  // 1. the adjoint column pass: transfer function by recurrence over evenly
  //    spaced planes or evaluated at every plane, and its z-chunks
  int best_adj = 0, best_rec = 0;
  float t_adj = 1e30f;
  for (int rec : {0, 2, 1, 3}) {
    if (rec && (c->dz_uniform == 0 || !adj_recurrence_supported(c->W, c->H, rec))) continue;
    for (int ch : {0, 2, 4, 8, 16, 32}) {
      if (ch > c->Nz) continue;
      RC(time_min(c, e0, e1, [&]() -> int {
        KL(launch_adj_col(c->Rs, c->cturn, c->zlist, c->U, c->W, c->H, 0, c->Nz, c->st, ch,
                          rec ? c->dz_uniform : 0.0, rec));
        return RIHVR_OK;
      }, &best));
      if (best < t_adj * 0.98f) {
        t_adj = best;
        best_adj = ch;
        best_rec = rec;
      }
    }
  }
  c->tune_adj_chunks = best_adj;
  c->tune_adj_rec = best_rec;
  // a valid gradient volume for the prox candidates
  KL(launch_rows(1, ELEM_C32, c->U, ELEM_C32, c->G, c->W, (long long)c->Nz * c->H, 1.0f, c->st));
  // 2. 2-D TV prox: streaming in 2- or 4-warp blocks with 1..8 runs per
  //    plane or the built-in count, in one launch or two (6-10 iterations),
  //    or tiled
  float t_tv = 0.f;
  if (c->mode == 7 && c->p.num_tv_iterations >= 1 && c->p.regularization_TV_param > 0.f) {
    const int cand[11][2] = {{0, 0}, {2, 1}, {2, 2}, {2, 4}, {2, 8}, {3, 0}, {3, 2}, {3, 4}, {4, 0}, {4, 2}, {1, 0}};
    t_tv = 1e30f;
    int bk = 0, bn = 0;
    for (const auto& cd : cand) {
      c->tune_tv_kernel = cd[0];
      c->tune_tv_nseg = cd[1];
      ProxArgs a = prox_args(c, c->t);
      RC(time_min(c, e0, e1, [&]() -> int {
        int nb = 0;
        KL(launch_prox_tv2d(c->storage, a, &nb, c->st));
        return RIHVR_OK;
      }, &best));
      if (best < t_tv * 0.98f) {
        t_tv = best;
        bk = cd[0];
        bn = cd[1];
      }
    }
    c->tune_tv_kernel = bk;
    c->tune_tv_nseg = bn;
  }
  // 3. the forward column pass: z-sum by Horner's scheme over evenly spaced
  //    planes or with the transfer function at every plane, and its z-chunks
  //    (with the sum of the partial spectra)
  int best_fwd = c->nchunks, best_horner = 0;
  float t_fwd = 1e30f;
  for (int hor : {1, 2, 3, 0}) {
    if (hor && (c->dz_uniform == 0 || !fwd_horner_supported(c->W, c->H, hor))) continue;
    for (int ch : {c->nchunks, 1, 2, 4, 8, 16}) {
      if (ch > c->Nz || ch > kMaxFwdChunks) continue;
      RC(time_min(c, e0, e1, [&]() -> int {
        KL(launch_fwd_col(c->U, c->cturn, c->zlist, c->Spart, c->W, c->H, 0, c->Nz, ch, c->st,
                          hor ? c->dz_uniform : 0.0, hor));
        KL(launch_sum_chunks(c->Spart, ch, c->S, (long long)c->HW, c->st));
        return RIHVR_OK;
      }, &best));
      if (best < t_fwd * 0.98f) {
        t_fwd = best;
        best_fwd = ch;
        best_horner = hor;
      }
    }
  }
  c->nchunks = best_fwd;
  c->tune_fwd_horner = best_horner;
  c->profiling = prev_profiling;
  *out = TuneVal{c->tune_adj_chunks, c->nchunks, c->tune_tv_nseg, c->tune_tv_kernel, c->tune_adj_rec,
                 c->tune_fwd_horner, (double)t_adj + (double)t_tv + (double)t_fwd};
  return RIHVR_OK;
}

}  // namespace

extern "C" {

int rihvr_tuning(const rihvr_ctx* c, int* adj_chunks, int* fwd_chunks, int* tv_runs, int* tv_kernel,
                 int* adj_recurrence, int* fwd_horner) {
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  if (adj_chunks) *adj_chunks = c->tune_adj_chunks;
  if (adj_recurrence)
    *adj_recurrence =
        (c->tune_adj_rec && c->dz_uniform != 0 && adj_recurrence_supported(c->W, c->H, c->tune_adj_rec))
            ? c->tune_adj_rec
            : 0;
  if (fwd_horner) {
    // the variant that runs: a table-twiddle form (2, 3) falls back to the
    // two-block form (1), and that to the direct pass (0), at sizes without it
    const int hm = c->dz_uniform == 0 ? 0 : c->tune_fwd_horner;
    *fwd_horner = (hm >= 2 && fwd_horner_supported(c->W, c->H, hm)) ? hm
                  : (hm >= 1 && fwd_horner_supported(c->W, c->H, 1)) ? 1
                                                                     : 0;
  }
  if (fwd_chunks) *fwd_chunks = c->nchunks;
  if (tv_runs) *tv_runs = c->tune_tv_nseg;
  if (tv_kernel) *tv_kernel = c->tune_tv_kernel;
  return RIHVR_OK;
}

int rihvr_autotune(rihvr_ctx* c, double* best_ms) {
  NvtxRange nvtx_("rihvr: autotune");
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  const TuneKey key{c->device, c->W, c->H, c->Nz, c->p.num_tv_iterations, c->mode, c->storage,
                    c->p.record_objective ? 1 : 0};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      drop_graphs(c);
      c->tune_adj_chunks = it->second.adj_chunks;
      c->nchunks = it->second.fwd_chunks;
      c->tune_tv_nseg = it->second.tv_nseg;
      c->tune_tv_kernel = it->second.tv_kernel;
      c->tune_adj_rec = it->second.adj_rec;
      c->tune_fwd_horner = it->second.fwd_horner;
      c->tuned = true;
      if (best_ms) *best_ms = it->second.ms;
      return RIHVR_OK;
    }
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  TuneVal v{};
  const int rc = autotune_run(c, e0, e1, &v);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != RIHVR_OK) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = v;
  }
  c->tuned = true;
  if (best_ms) *best_ms = v.ms;
  return RIHVR_OK;
}

int rihvr_reset(rihvr_ctx* c) {
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  return state_reset(c);
}

}  // extern "C"

namespace {

// Checkpoint file: a fixed header, the iteration log, the hologram-space
// buffers that carry from one iteration to the next, and the two volumes
// P_k and P_{k-1} in the context's storage type.
constexpr char kStateMagic[8] = {'R', 'I', 'H', 'V', 'R', 'S', 'T', '1'};
struct StateHeader {
  char magic[8];
  int32_t version, W, H, Nz, storage, mode, faithful, n_tv, max_backtracks, record_objective;
  float z0, dz, lambda, dx, l1, tv;
  double t, alpha1, beta, prev_f_resid;
  int32_t it, pending_x, nlog, esize;
  int32_t z_first, num_planes;  // the planes held, of the whole volume's (z-slabs)
};

void state_header_of(const rihvr_ctx* c, StateHeader* h) {
  std::memset(h, 0, sizeof(*h));
  std::memcpy(h->magic, kStateMagic, 8);
  h->version = 2;
  h->W = c->W;
  h->H = c->H;
  h->Nz = c->Nz;
  h->storage = c->storage;
  h->mode = c->mode;
  h->faithful = c->p.faithful;
  h->n_tv = c->p.num_tv_iterations;
  h->max_backtracks = c->p.max_backtracks;
  h->record_objective = c->p.record_objective;
  h->z0 = c->p.start_plane;
  h->dz = c->p.plane_stepsize;
  h->lambda = c->p.wavelength;
  h->dx = c->p.resolution;
  h->l1 = c->p.regularization_param;
  h->tv = c->p.regularization_TV_param;
  h->esize = (int32_t)c->esize;
  h->z_first = c->z_first;
  h->num_planes = c->p.num_planes;
}

struct FileGuard {
  FILE* f = nullptr;
  ~FileGuard() {
    if (f) std::fclose(f);
  }
};

struct PinnedGuard {
  void* p = nullptr;
  ~PinnedGuard() {
    if (p) cudaFreeHost(p);
  }
};

constexpr size_t kStateChunk = 64u << 20;  // bytes staged through pinned memory at a time

// device buffer <-> file through a pinned staging buffer
int state_write_dev(rihvr_ctx* c, FILE* f, const void* dev, size_t bytes, void* stage) {
  for (size_t o = 0; o < bytes; o += kStateChunk) {
    const size_t n = std::min(kStateChunk, bytes - o);
    CK(cudaMemcpyAsync(stage, static_cast<const char*>(dev) + o, n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (std::fwrite(stage, 1, n, f) != n) return fail(RIHVR_ERR_BAD_FILENAME, "writing the state file failed");
  }
  return RIHVR_OK;
}

int state_read_dev(rihvr_ctx* c, FILE* f, void* dev, size_t bytes, void* stage) {
  for (size_t o = 0; o < bytes; o += kStateChunk) {
    const size_t n = std::min(kStateChunk, bytes - o);
    if (std::fread(stage, 1, n, f) != n) return fail(RIHVR_ERR_INVALID_FILE, "the state file is truncated");
    CK(cudaMemcpyAsync(static_cast<char*>(dev) + o, stage, n, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  return RIHVR_OK;
}

// the buffers a checkpoint carries, in file order
template <typename F>
int each_state_buffer(rihvr_ctx* c, F fn) {
  const size_t HW = c->HW;
  RC(fn(c->b, sizeof(float) * HW));
  RC(fn(c->dnew, sizeof(float) * HW));
  RC(fn(c->dY0, sizeof(float) * HW));
  RC(fn(c->dX, sizeof(float) * HW));
  RC(fn(c->r, sizeof(float) * HW));
  RC(fn(c->Rs, sizeof(float2) * HW));
  RC(fn(c->vol[c->iCur], c->esize * c->V));
  return fn(c->vol[c->iPrev], c->esize * c->V);
}

}  // namespace

extern "C" {

int rihvr_save_state(rihvr_ctx* c, const char* path) {
  if (!c || !path) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  StateHeader h;
  state_header_of(c, &h);
  h.t = c->t;
  h.alpha1 = c->alpha1;
  h.beta = c->beta;
  h.prev_f_resid = c->prev_f_resid;
  h.it = c->it;
  h.pending_x = c->pending_x;
  h.nlog = (int32_t)c->log.size();
  FileGuard fg;
  fg.f = std::fopen(path, "wb");
  if (!fg.f) return fail(RIHVR_ERR_BAD_FILENAME, std::string("cannot open ") + path + " for writing");
  if (std::fwrite(&h, sizeof(h), 1, fg.f) != 1 ||
      (h.nlog > 0 && std::fwrite(c->log.data(), sizeof(rihvr_iter_record), (size_t)h.nlog, fg.f) != (size_t)h.nlog))
    return fail(RIHVR_ERR_BAD_FILENAME, "writing the state file failed");
  PinnedGuard stage;
  CK(cudaMallocHost(&stage.p, kStateChunk));
  CK(cudaStreamSynchronize(c->st));
  RC(each_state_buffer(c, [&](const void* dev, size_t bytes) { return state_write_dev(c, fg.f, dev, bytes, stage.p); }));
  if (std::fflush(fg.f) != 0) return fail(RIHVR_ERR_BAD_FILENAME, "writing the state file failed");
  return RIHVR_OK;
}

int rihvr_load_state(rihvr_ctx* c, const char* path) {
  if (!c || !path) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  FileGuard fg;
  fg.f = std::fopen(path, "rb");
  if (!fg.f) return fail(RIHVR_ERR_BAD_FILENAME, std::string("cannot open ") + path);
  StateHeader h, mine;
  if (std::fread(&h, sizeof(h), 1, fg.f) != 1 || std::memcmp(h.magic, kStateMagic, 8) != 0 || h.version != 2)
    return fail(RIHVR_ERR_INVALID_FILE, "not a reconstruction state file");
  state_header_of(c, &mine);
  // the solve it resumes must be this context's: sizes, storage, mode and the
  // parameters every iteration reads
  if (h.W != mine.W || h.H != mine.H || h.Nz != mine.Nz || h.storage != mine.storage || h.mode != mine.mode ||
      h.faithful != mine.faithful || h.n_tv != mine.n_tv || h.max_backtracks != mine.max_backtracks ||
      h.record_objective != mine.record_objective || h.esize != mine.esize || h.z0 != mine.z0 || h.dz != mine.dz ||
      h.lambda != mine.lambda || h.dx != mine.dx || h.l1 != mine.l1 || h.tv != mine.tv ||
      h.z_first != mine.z_first || h.num_planes != mine.num_planes)
    return fail(RIHVR_ERR_INVALID_FILE, "the state file belongs to a solve with other sizes or parameters");
  if (h.nlog < 0 || h.nlog > (1 << 24) || h.it < 0 || h.pending_x < -1 || h.pending_x >= h.nlog)
    return fail(RIHVR_ERR_INVALID_FILE, "the state file's iteration log is inconsistent");
  std::vector<rihvr_iter_record> log((size_t)h.nlog);
  if (h.nlog > 0 && std::fread(log.data(), sizeof(rihvr_iter_record), (size_t)h.nlog, fg.f) != (size_t)h.nlog)
    return fail(RIHVR_ERR_INVALID_FILE, "the state file is truncated");
  PinnedGuard stage;
  CK(cudaMallocHost(&stage.p, kStateChunk));
  CK(cudaStreamSynchronize(c->st));
  c->iPrev = 0;
  c->iCur = 1;
  c->iNew = 2;
  const int rc =
      each_state_buffer(c, [&](void* dev, size_t bytes) { return state_read_dev(c, fg.f, dev, bytes, stage.p); });
  if (rc != RIHVR_OK) {
    c->have_holo = false;  // partly overwritten: the context needs a hologram again
    return rc;
  }
  c->t = h.t;
  c->alpha1 = h.alpha1;
  c->beta = h.beta;
  c->prev_f_resid = h.prev_f_resid;
  c->it = h.it;
  c->pending_x = h.pending_x;
  c->log.swap(log);
  c->have_holo = true;
  return RIHVR_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Z-slab sharding of one hologram.  A slab context holds planes
// [z_first, z_first + Nz) of the volume and its own copy of every
// hologram-space buffer.  The gradient, the prox and the forward pass up to
// the partial spectrum S_s = sum over the slab's planes of H'_z FFT2(P_z) are
// the slab's own; one attempt exchanges S_s (summed over the slabs in slab
// order, so that every slab holds the same total) and the slabs' FP64 prox
// sums.  After the sum every slab runs the same arithmetic on the same values
// (the plane pass, d, r, the residual spectrum, the decisions), so no other
// exchange is needed.  The decisions are those of one_iteration.
// ---------------------------------------------------------------------------

namespace {

struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int d) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != d) cudaSetDevice(d);
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

struct SlabGroup {
  rihvr_ctx* const* cs;
  int n;
  const rihvr_slab_reducer* red;  // other processes' slabs, or NULL

  int sum_over_processes(void* data, long long count, int dtype, int on_device) const {
    if (!red) return RIHVR_OK;
    const int rc = red->sum(red->user, data, count, dtype, on_device);
    if (rc != 0) return fail(RIHVR_ERR_UNKNOWN_ERROR, "the slab reducer failed with " + std::to_string(rc));
    return RIHVR_OK;
  }
};

// The group must tile the plane list in order (in-process slabs), share
// sizes and parameters, hold a hologram and stand at the same iteration.
int check_slab_group(const SlabGroup& g) {
  if (!g.cs || g.n < 1 || g.n > kMaxSlabs)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "1.." + std::to_string(kMaxSlabs) + " slab contexts expected");
  if (g.red && (g.n != 1 || !g.red->sum))
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "a reducer takes exactly one local slab and a sum function");
  const rihvr_ctx* c0 = g.cs[0];
  int next = 0;
  for (int i = 0; i < g.n; ++i) {
    const rihvr_ctx* c = g.cs[i];
    if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL slab context");
    if (c->W != c0->W || c->H != c0->H || std::memcmp(&c->p, &c0->p, sizeof(rihvr_params)) != 0)
      return fail(RIHVR_ERR_INVALID_ARGUMENT, "slab contexts differ in size or parameters");
    if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set on slab " + std::to_string(i));
    if (c->it != c0->it || c->iCur != c0->iCur || c->prev_f_resid != c0->prev_f_resid)
      return fail(RIHVR_ERR_INVALID_STATE, "slab " + std::to_string(i) +
                                               " holds another hologram or stands at another iteration");
    if (!g.red && c->z_first != next)
      return fail(RIHVR_ERR_INVALID_ARGUMENT, "slab " + std::to_string(i) + " starts at plane " +
                                                  std::to_string(c->z_first) + ", expected " + std::to_string(next));
    next = c->z_first + c->Nz;
  }
  if (!g.red && next != c0->p.num_planes)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "the slabs end at plane " + std::to_string(next) + " of " +
                                                std::to_string(c0->p.num_planes));
  return RIHVR_OK;
}

// Peer mappings between the devices of an in-process group.
int enable_slab_peers(const SlabGroup& g) {
  for (int i = 0; i < g.n; ++i)
    for (int j = 0; j < g.n; ++j) {
      const int a = g.cs[i]->device, b = g.cs[j]->device;
      if (a == b) continue;
      int ok = 0;
      CK(cudaDeviceCanAccessPeer(&ok, a, b));
      if (!ok)
        return fail(RIHVR_ERR_CUDA, "device " + std::to_string(a) + " cannot read device " + std::to_string(b));
      DeviceScope ds(a);
      const cudaError_t e = cudaDeviceEnablePeerAccess(b, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled)
        cudaGetLastError();
      else if (e != cudaSuccess)
        return fail(RIHVR_ERR_CUDA, std::string("cudaDeviceEnablePeerAccess: ") + cudaGetErrorString(e));
    }
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    if (!c->slab_ev) CK(cudaEventCreateWithFlags(&c->slab_ev, cudaEventDisableTiming));
    if (g.red && g.red->host_staged && !c->slab_stage_h && halloc(&c->slab_stage_h, sizeof(float2) * c->HW) != RIHVR_OK)
      return fail(RIHVR_ERR_OUT_OF_MEMORY, "pinned staging buffer");
  }
  return RIHVR_OK;
}

// One attempt over the group: per slab the gradient (first attempt), the prox
// and the partial spectrum; the spectra summed; per slab the rest of the
// forward pass.  sp receives the prox sums over all slabs, *f_resid the
// residual term of the new prox output.
int slab_attempt(const SlabGroup& g, bool first, double* sp, double* f_resid) {
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    CK(cudaMemcpyAsync(c->scal_d, c->scal_h, 5 * sizeof(float), cudaMemcpyHostToDevice, c->st));
    if (first) RC(adjoint_volume(c));
    RC(prox_volume(c, c->t, true));
    {
      NvtxRange nvtx_("rihvr: forward (slab part)");
      RC(forward_partial(c, elem_kind(c->storage), c->vol[c->iNew]));
    }
    CK(cudaEventRecord(c->slab_ev, c->st));
  }
  std::vector<const float2*> total((size_t)g.n);
  if (!g.red) {
    std::vector<const float2*> src((size_t)g.n);
    for (int i = 0; i < g.n; ++i) src[(size_t)i] = g.cs[i]->S;
    for (int i = 0; i < g.n; ++i) {
      rihvr_ctx* c = g.cs[i];
      DeviceScope ds(c->device);
      for (int j = 0; j < g.n; ++j)
        if (j != i) CK(cudaStreamWaitEvent(c->st, g.cs[j]->slab_ev, 0));
      KL(launch_sum_slabs(src.data(), g.n, c->Spart, (long long)c->HW, c->st));
      total[(size_t)i] = c->Spart;
    }
  } else {
    rihvr_ctx* c = g.cs[0];
    DeviceScope ds(c->device);
    NvtxRange nvtx_("rihvr: slab spectrum exchange");
    if (g.red->host_staged) {
      CK(cudaMemcpyAsync(c->slab_stage_h, c->S, sizeof(float2) * c->HW, cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      RC(g.sum_over_processes(c->slab_stage_h, 2 * (long long)c->HW, RIHVR_DTYPE_F32, 0));
      CK(cudaMemcpyAsync(c->S, c->slab_stage_h, sizeof(float2) * c->HW, cudaMemcpyHostToDevice, c->st));
    } else {
      CK(cudaStreamSynchronize(c->st));
      RC(g.sum_over_processes(c->S, 2 * (long long)c->HW, RIHVR_DTYPE_F32, 1));
    }
    total[0] = c->S;
  }
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    RC(forward_from_spectrum(c, total[(size_t)i]));
    CK(cudaMemcpyAsync(c->sums_h, c->sums_d, sizeof(double) * kNumSums * NUM_SLOTS, cudaMemcpyDeviceToHost, c->st));
  }
  for (int i = 0; i < g.n; ++i) {
    DeviceScope ds(g.cs[i]->device);
    CK(cudaStreamSynchronize(g.cs[i]->st));
  }
  for (int k = 0; k < kNumSums; ++k) {
    double v = 0;
    for (int i = 0; i < g.n; ++i) v += g.cs[i]->sums_h[SLOT_PROX * kNumSums + k];
    sp[k] = v;
  }
  RC(g.sum_over_processes(sp, kNumSums, RIHVR_DTYPE_F64, 0));
  *f_resid = 0.5 * g.cs[0]->sums_h[SLOT_FWD * kNumSums + SUM_RR];
  return RIHVR_OK;
}

// One FISTA iteration of the group (one_iteration's decisions on the summed
// values; every slab takes the same step, momentum and record).
int slab_iteration(const SlabGroup& g) {
  NvtxRange nvtx_("rihvr: iteration (z-slabs)");
  rihvr_ctx* c0 = g.cs[0];
  double alpha0 = c0->alpha1;
  int bt = 0;
  double f_resid = 0, lim = 0, ratio = 0;
  double sp[kNumSums];
  for (;;) {
    for (int i = 0; i < g.n; ++i) {
      rihvr_ctx* c = g.cs[i];
      const ProxArgs a = prox_args(c, c->t);
      c->scal_h[0] = a.beta;
      c->scal_h[1] = a.t;
      c->scal_h[2] = a.mu;
      c->scal_h[3] = a.s;
      c->scal_h[4] = a.thr;
    }
    RC(slab_attempt(g, bt == 0, sp, &f_resid));
    if (bt == 0 && c0->p.record_objective)
      for (int i = 0; i < g.n; ++i) settle_x_terms(g.cs[i], sp);
    lim = sp[SUM_LIM1] + sp[SUM_LIM2] / (2.0 * c0->t);
    ratio = f_resid / (c0->prev_f_resid + lim);
    if (((ratio > 1.0) || (ratio < 0.0)) && bt < c0->p.max_backtracks) {
      for (int i = 0; i < g.n; ++i) g.cs[i]->t *= 0.5;  // stepsize_shrinkage (:63)
      ++bt;
      continue;
    }
    break;
  }
  rihvr_iter_record rec{};
  rec.f_resid_prox = f_resid;
  rec.lim = lim;
  rec.ratio = ratio;
  rec.t = c0->t;
  rec.backtracks = bt;
  rec.restart_sum = sp[SUM_RS];
  rec.f_prox = f_resid + (double)c0->p.regularization_param * sp[SUM_L1P] + tv_weight(c0) * sp[SUM_TVP];
  const bool restarted = sp[SUM_RS] > 0.0;  // fistaRestart (:471-475)
  if (restarted) alpha0 = 1.0;
  const double alpha1 = (1.0 + std::sqrt(1.0 + 4.0 * alpha0 * alpha0)) / 2.0;
  const double beta = (alpha0 - 1.0) / alpha1;
  rec.beta = beta;
  rec.restarted = restarted ? 1 : 0;
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    c->scal_h[8] = (float)beta;
    RC(enqueue_momentum(c));
  }
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    CK(cudaStreamSynchronize(c->st));
    const int old_prev = c->iPrev;
    c->iPrev = c->iCur;
    c->iCur = c->iNew;
    c->iNew = old_prev;
    c->alpha1 = alpha1;
    c->beta = beta;
    c->prev_f_resid = 0.5 * c->sums_h[SLOT_MOM * kNumSums + SUM_RR];
    rihvr_iter_record r = rec;
    r.f_resid_x = c->prev_f_resid;
    r.f_x = r.f_resid_x;
    c->log.push_back(r);
    c->pending_x = (int)c->log.size() - 1;
    c->it++;
    c->warm = true;
  }
  return RIHVR_OK;
}

// The momentum-point terms of the last record from the norms over all slabs.
int slab_settle_pending(const SlabGroup& g) {
  rihvr_ctx* c0 = g.cs[0];
  if (!c0->p.record_objective || c0->pending_x < 0) return RIHVR_OK;
  double s[kNumSums] = {0};
  for (int i = 0; i < g.n; ++i) {
    rihvr_ctx* c = g.cs[i];
    DeviceScope ds(c->device);
    double l1x, tvx;
    RC(norms_at_x(c, &l1x, &tvx));
    s[SUM_L1X] += l1x;
    s[SUM_TVX] += tvx;
  }
  RC(g.sum_over_processes(s, kNumSums, RIHVR_DTYPE_F64, 0));
  for (int i = 0; i < g.n; ++i) settle_x_terms(g.cs[i], s);
  return RIHVR_OK;
}

}  // namespace

extern "C" {

int rihvr_slab_iterate(rihvr_ctx* const* ctxs, int n, int iterations, const rihvr_slab_reducer* reducer) {
  NvtxRange nvtx_("rihvr: slab iterate");
  if (iterations < 0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "iterations must be >= 0");
  const SlabGroup g{ctxs, n, reducer};
  RC(check_slab_group(g));
  RC(enable_slab_peers(g));
  for (int k = 0; k < iterations; ++k) RC(slab_iteration(g));
  RC(slab_settle_pending(g));
  for (int i = 0; i < n; ++i) {
    DeviceScope ds(ctxs[i]->device);
    RC(check_col_waits(ctxs[i]));
  }
  return RIHVR_OK;
}

int rihvr_slab_range(const rihvr_ctx* c, int* z_first, int* z_count) {
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  if (z_first) *z_first = c->z_first;
  if (z_count) *z_count = c->Nz;
  return RIHVR_OK;
}

int rihvr_iterate(rihvr_ctx* c, int n) {
  NvtxRange nvtx_("rihvr: iterate");
  if (!c || n < 0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "bad argument");
  return run_iterations(c, n);
}

int rihvr_iterate_timed(rihvr_ctx* c, int n, float* ms) {
  if (!c || n < 0 || !ms) return fail(RIHVR_ERR_INVALID_ARGUMENT, "bad argument");
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, c->st));
  int rc = run_iterations(c, n);
  cudaEventRecord(b, c->st);
  cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int rihvr_reconstruct(rihvr_ctx* c, double* final_objective) {
  NvtxRange nvtx_("rihvr: reconstruct");
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  RC(whole_volume(c, "rihvr_reconstruct"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  RC(state_reset(c));
  RC(run_iterations(c, c->p.num_inverse_iterations));
  if (final_objective) RC(rihvr_objective(c, final_objective, nullptr));
  return RIHVR_OK;
}

int rihvr_reconstruct_batch(rihvr_ctx* const* ctxs, int n, const float* const* holograms, int is_device,
                            double* final_objectives, int* statuses) {
  NvtxRange nvtx_("rihvr: reconstruct batch");
  g_batch_combined = 0;
  if (!ctxs || !holograms || n <= 0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "empty or NULL batch");
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || !holograms[i]) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context or hologram in batch");
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return fail(RIHVR_ERR_INVALID_ARGUMENT, "a context appears twice in the batch");
  }
  for (int i = 0; i < n; ++i) RC(whole_volume(ctxs[i], "rihvr_reconstruct_batch"));
  std::vector<int> st(n, RIHVR_OK), ran(n, 0);
  std::vector<std::string> msg(n);
  // run fn on every frame still without error, one host thread per frame
  auto each_frame = [&](auto fn) {
    auto one = [&](int i) -> void {
      if (st[i] != RIHVR_OK) return;
      rihvr_ctx* c = ctxs[i];
      int rc = cudaSetDevice(c->device) == cudaSuccess ? RIHVR_OK : RIHVR_ERR_CUDA;
      if (rc == RIHVR_OK) rc = fn(i, c);
      st[i] = rc;
      if (rc != RIHVR_OK) msg[i] = g_last_error;  // thread-local: carried back to the caller's thread
    };
    std::vector<std::thread> workers;
    workers.reserve(n - 1);
    for (int i = 1; i < n; ++i) workers.emplace_back(one, i);
    one(0);
    for (auto& w : workers) w.join();
  };
  // hologram in, state reset and the eager first iteration, frames overlapping
  each_frame([&](int i, rihvr_ctx* c) -> int {
    RC(rihvr_set_hologram(c, holograms[i], is_device));
    RC(state_reset(c));
    return eager_start(c, c->p.num_inverse_iterations, &ran[i]);
  });
  // the remaining iterations: in batch mode 1, one graph launch per iteration
  // for all frames when they share a device, run the device-decided loop and
  // are at the same point; in batch mode 2, one graph launch for the whole
  // solves of all frames that share a device and run the device-decided loop
  // (any iteration counts); else each frame's own loop on its own thread
  const int bmode = g_batch_mode.load();
  bool combined = n > 1 && bmode != 0;
  const int rest = ctxs[0]->p.num_inverse_iterations - ran[0];
  std::vector<int> rests(n, 0);
  bool any_rest = false;
  for (int i = 0; i < n && combined; ++i) {
    const rihvr_ctx* c = ctxs[i];
    rests[i] = c->p.num_inverse_iterations - ran[i];
    any_rest = any_rest || rests[i] > 0;
    combined = st[i] == RIHVR_OK && use_dev_loop(c) && c->device == ctxs[0]->device;
    if (bmode == 1) combined = combined && rests[i] == rest && c->iCur == ctxs[0]->iCur;
  }
  combined = combined && (bmode == 2 ? any_rest : rest > 0);
  if (combined && bmode == 2) {
    std::unique_ptr<SolveGraph> S;
    if (cudaSetDevice(ctxs[0]->device) == cudaSuccess) S = take_solve_graph(ctxs, n);
    if (S) {
      const int rc = run_solves_graph(ctxs, n, rests, *S);
      for (int i = 0; i < n; ++i) {
        st[i] = rc;
        if (rc != RIHVR_OK) msg[i] = g_last_error;
      }
      if (rc == RIHVR_OK) keep_solve_graph(ctxs, n, std::move(S));
      g_batch_combined = 2;
    } else {
      cudaGetLastError();
      combined = false;
    }
  } else if (combined) {
    BatchGraphs B;
    if (cudaSetDevice(ctxs[0]->device) == cudaSuccess && build_batch_graphs(ctxs, n, B) == RIHVR_OK) {
      const int rc = run_iterations_batch(ctxs, n, rest, B);
      for (int i = 0; i < n; ++i) {
        st[i] = rc;
        if (rc != RIHVR_OK) msg[i] = g_last_error;
      }
      g_batch_combined = 1;
    } else {
      cudaGetLastError();
      combined = false;
    }
  }
  each_frame([&](int i, rihvr_ctx* c) -> int {
    if (combined) RC(settle_pending(c));
    else RC(run_iterations_from(c, ran[i], c->p.num_inverse_iterations));
    double f = 0.0;
    RC(rihvr_objective(c, &f, nullptr));
    if (final_objectives) final_objectives[i] = f;
    return RIHVR_OK;
  });
  int first = RIHVR_OK;
  for (int i = 0; i < n; ++i) {
    if (final_objectives && st[i] != RIHVR_OK) final_objectives[i] = 0.0;
    if (statuses) statuses[i] = st[i];
    if (first == RIHVR_OK && st[i] != RIHVR_OK) {
      first = st[i];
      g_last_error = "frame " + std::to_string(i) + ": " + msg[i];
    }
  }
  return first;
}

int rihvr_set_batch_mode(int mode) {
  if (mode < 0 || mode > 2) return fail(RIHVR_ERR_INVALID_ARGUMENT, "batch mode must be 0, 1 or 2");
  g_batch_mode.store(mode);
  return RIHVR_OK;
}

int rihvr_batch_last_combined(void) { return g_batch_combined; }

int rihvr_iteration_count(const rihvr_ctx* c) { return c ? c->it : -1; }

int rihvr_objective(rihvr_ctx* c, double* f, double* terms3) {
  if (!c || !f) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(whole_volume(c, "rihvr_objective"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  double l1x, tvx;
  RC(norms_at_x(c, &l1x, &tvx));
  const double fr = c->prev_f_resid;
  *f = fr + (double)c->p.regularization_param * l1x + tv_weight(c) * tvx;
  if (terms3) {
    terms3[0] = fr;
    terms3[1] = l1x;
    terms3[2] = c->mode == 5 ? 0.0 : tvx;
  }
  return RIHVR_OK;
}

int rihvr_sparsity(rihvr_ctx* c, double* fraction) {
  if (!c || !fraction) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  double l1x, tvx, nnz;
  RC(norms_at_x(c, &l1x, &tvx, &nnz));
  *fraction = nnz / (double)c->V;
  return RIHVR_OK;
}

int rihvr_initial_estimate(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(whole_volume(c, "rihvr_initial_estimate"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  // gradient.reconstruct(measured) then backPropagateInitial: A (t A^H b), t = 1/Nz
  CK(cudaMemcpyAsync(c->r, c->b, sizeof(float) * c->HW, cudaMemcpyDeviceToDevice, c->st));
  RC(residual_spectrum(c));
  RC(adjoint_volume(c));
  RC(forward_volume(c, ELEM_C32, c->G));
  std::vector<float> d(c->HW);
  CK(cudaMemcpyAsync(d.data(), c->dnew, sizeof(float) * c->HW, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const float t = (float)(1.0 / (double)c->p.num_planes);
  for (float& v : d) v *= t;
  CK(cudaMemcpy(out, d.data(), sizeof(float) * c->HW, is_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost));
  return state_reset(c);
}

}  // extern "C"

namespace {

// Start from the volume in U (complex FP32): P_{k-1} = P_k = x0 in the
// storage type, beta = 0, the estimated hologram and residual of x0.
int start_from_U(rihvr_ctx* c) {
  KL(launch_store_volume(c->storage, c->U, c->vol[c->iCur], (long long)c->V, c->st));
  CK(cudaMemcpyAsync(c->vol[c->iPrev], c->vol[c->iCur], c->esize * c->V, cudaMemcpyDeviceToDevice, c->st));
  // the estimated hologram of the stored x0, then the momentum step with beta = 0:
  // d(x) = d(P_k) = A x0, r = d - b and its spectrum
  RC(forward_volume(c, elem_kind(c->storage), c->vol[c->iCur]));
  int nb = 0;
  KL(launch_holo_momentum(c->dnew, c->dY0, c->dX, c->b, c->r, 0.f, (long long)c->HW, c->partials, &nb, c->st));
  RC(reduce_into(c, nb, SLOT_MOM));
  RC(residual_spectrum(c));
  RC(fetch_sums(c));
  c->prev_f_resid = 0.5 * c->sums_h[SLOT_MOM * kNumSums + SUM_RR];
  return RIHVR_OK;
}

int flat_blocks_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

__global__ void k_scale_c(float2* __restrict__ v, long long n, float s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = make_float2(v[i].x * s, v[i].y * s);
}

// G = A^H b (the residual of x = 0 with the sign flipped)
int backproject_into_G(rihvr_ctx* c) {
  CK(cudaMemcpyAsync(c->r, c->b, sizeof(float) * c->HW, cudaMemcpyDeviceToDevice, c->st));
  RC(residual_spectrum(c));
  return adjoint_volume(c);
}

}  // namespace

extern "C" {

int rihvr_set_initial_volume(rihvr_ctx* c, const float* x0, int is_device) {
  if (!c || !x0) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(whole_volume(c, "rihvr_set_initial_volume"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  RC(state_reset(c));
  RC(copy_in(c, c->U, x0, sizeof(float2) * c->V, is_device));
  return start_from_U(c);
}

int rihvr_backpropagate(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  RC(state_reset(c));
  RC(backproject_into_G(c));
  KL((k_scale_c<<<flat_blocks_for(c->V), 256, 0, c->st>>>(c->G, (long long)c->V, (float)c->t), cudaGetLastError()));
  RC(copy_out(c, out, c->G, sizeof(float2) * c->V, is_device));
  return state_reset(c);
}

int rihvr_warm_start(rihvr_ctx* c, rihvr_unet* net) {
  if (!c || !net) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(whole_volume(c, "rihvr_warm_start"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  int D, H, W;
  unet_dims(net, &D, &H, &W);
  if (D != c->Nz || H != c->H || W != c->W)
    return fail(RIHVR_ERR_INVALID_ARGUMENT, "network volume " + std::to_string(D) + "x" + std::to_string(H) + "x" +
                                                std::to_string(W) + " differs from the context's");
  RC(state_reset(c));
  RC(backproject_into_G(c));
  // x0 = g alpha t A^H b into U
  const int rc = unet_predict_on(net, c->G, (float)c->t, c->U, c->st);
  if (rc != RIHVR_OK) return rc;
  return start_from_U(c);
}

int rihvr_get_iterations(const rihvr_ctx* c, rihvr_iter_record* out, int max_records, int* n_out) {
  if (!c || !n_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  const int n = (int)c->log.size();
  *n_out = n;
  if (out)
    for (int i = 0; i < n && i < max_records; ++i) out[i] = c->log[i];
  return RIHVR_OK;
}

int rihvr_get_volume(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  // materialise x = P + beta (P - Pprev) into the intermediate buffer
  KL(launch_materialize_x(c->storage, c->vol[c->iCur], c->vol[c->iPrev], (float)c->beta, c->U, (long long)c->V,
                          c->st));
  return copy_out(c, out, c->U, sizeof(float2) * c->V, is_device);
}

int rihvr_get_volume_ptr(rihvr_ctx* c, const void** dev_ptr, int* dtype) {
  if (!c || !dev_ptr) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  KL(launch_materialize_x(c->storage, c->vol[c->iCur], c->vol[c->iPrev], (float)c->beta, c->U, (long long)c->V,
                          c->st));
  CK(cudaStreamSynchronize(c->st));
  *dev_ptr = c->U;
  if (dtype) *dtype = 0;
  return RIHVR_OK;
}

int rihvr_segment(rihvr_ctx* c, const rihvr_segment_params* sp, rihvr_object* objects, int max_objects,
                  int* num_objects, rihvr_segment_info* info) {
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  RC(whole_volume(c, "rihvr_segment"));
  // the volume rihvr_get_volume returns, read in place
  if (!c->seg_ws) c->seg_ws = seg_workspace_create();
  rihvr_segment_info local{};
  const int rc = segment_volume(c->storage, c->vol[c->iCur], c->vol[c->iPrev], (float)c->beta, c->W, c->H, c->Nz,
                                sp, objects, max_objects, num_objects, &local, c->seg_ws, c->st);
  c->launches += local.kernel_launches;
  if (info) *info = local;
  return rc;
}

int rihvr_get_plane(rihvr_ctx* c, int z, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (z < 0 || z >= c->Nz) return fail(RIHVR_ERR_INVALID_ARGUMENT, "plane out of bounds");  // :950-954
  const size_t off = (size_t)z * c->HW;
  const char* P = static_cast<const char*>(c->vol[c->iCur]) + off * c->esize;
  const char* Pp = static_cast<const char*>(c->vol[c->iPrev]) + off * c->esize;
  KL(launch_materialize_x(c->storage, P, Pp, (float)c->beta, c->pc1, (long long)c->HW, c->st));
  return copy_out(c, out, c->pc1, sizeof(float2) * c->HW, is_device);
}

int rihvr_get_estimate(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  return copy_out(c, out, c->dX, sizeof(float) * c->HW, is_device);
}

int rihvr_get_residual(rihvr_ctx* c, float* out, int is_device) {
  if (!c || !out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  return copy_out(c, out, c->r, sizeof(float) * c->HW, is_device);
}

int rihvr_lipschitz(rihvr_ctx* c, int iterations, unsigned long long seed, double* L_out, double* history) {
  if (!c || !L_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (iterations < 1 || iterations > 100000) return fail(RIHVR_ERR_INVALID_ARGUMENT, "iterations must be 1..100000");
  RC(whole_volume(c, "rihvr_lipschitz"));
  if (!c->have_holo) return fail(RIHVR_ERR_MISSING_DATA, "no hologram set");
  // FP64 sum of squares of n floats on the device, read back
  auto sumsq = [&](const float* x, long long n, double* out) -> int {
    int nb = 0;
    KL(launch_sumsq(x, n, c->partials, &nb, c->st));
    RC(reduce_into(c, nb, SLOT_NORM));
    RC(fetch_sums(c));
    *out = c->sums_h[SLOT_NORM * kNumSums + SUM_RR];
    return RIHVR_OK;
  };
  // x_0: seeded uniform entries in [-1, 1) for both parts, held in G
  KL(launch_fill_uniform_c(c->G, (long long)c->V, seed, c->st));
  double nx2 = 0;
  RC(sumsq(reinterpret_cast<const float*>(c->G), 2LL * (long long)c->V, &nx2));
  double L = 0;
  for (int k = 0; k < iterations; ++k) {
    // A x_k (dnew), its squared norm, and the Rayleigh quotient ||A x||^2 / ||x||^2
    RC(forward_volume(c, ELEM_C32, c->G));
    double ax2 = 0;
    RC(sumsq(c->dnew, (long long)c->HW, &ax2));
    L = ax2 / nx2;
    if (history) history[k] = L;
    // x_{k+1} = A^H A x_k / ||A^H A x_k||
    CK(cudaMemcpyAsync(c->r, c->dnew, sizeof(float) * c->HW, cudaMemcpyDeviceToDevice, c->st));
    RC(residual_spectrum(c));
    RC(adjoint_volume(c));
    double ny2 = 0;
    RC(sumsq(reinterpret_cast<const float*>(c->G), 2LL * (long long)c->V, &ny2));
    if (!(ny2 > 0)) break;
    const float scale = (float)(1.0 / std::sqrt(ny2));
    KL((k_scale_c<<<1184, 256, 0, c->st>>>(c->G, (long long)c->V, scale), cudaGetLastError()));
    nx2 = ny2 * (double)scale * (double)scale;
  }
  *L_out = L;
  // the operator passes overwrote the hologram-side buffers: restart from x = 0
  return state_reset(c);
}

int rihvr_forward(rihvr_ctx* c, const float* volume, float* holo_out, int is_device) {
  if (!c || !volume || !holo_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(copy_in(c, c->G, volume, sizeof(float2) * c->V, is_device));
  RC(forward_volume(c, ELEM_C32, c->G));
  RC(check_col_waits(c));
  return copy_out(c, holo_out, c->dnew, sizeof(float) * c->HW, is_device);
}

int rihvr_adjoint(rihvr_ctx* c, const float* residual, float* volume_out, int is_device) {
  if (!c || !residual || !volume_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  RC(copy_in(c, c->r, residual, sizeof(float) * c->HW, is_device));
  RC(residual_spectrum(c));
  RC(adjoint_volume(c));
  return copy_out(c, volume_out, c->G, sizeof(float2) * c->V, is_device);
}

int rihvr_prox_step(rihvr_ctx* c, const float* x, const float* residual, double t, float* p_out, double* sums3,
                    int is_device) {
  if (!c || !x || !residual || !p_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!(t > 0)) return fail(RIHVR_ERR_INVALID_ARGUMENT, "t must be positive");
  // x into the P_k slot (storage type) and P_{k-1} = P_k with beta = 0
  RC(copy_in(c, c->U, x, sizeof(float2) * c->V, is_device));
  KL(launch_store_volume(c->storage, c->U, c->vol[c->iCur], (long long)c->V, c->st));
  CK(cudaMemcpyAsync(c->vol[c->iPrev], c->vol[c->iCur], c->esize * c->V, cudaMemcpyDeviceToDevice, c->st));
  const double saved_beta = c->beta;
  c->beta = 0;
  RC(copy_in(c, c->r, residual, sizeof(float) * c->HW, is_device));
  RC(residual_spectrum(c));
  RC(adjoint_volume(c));
  int rc = prox_volume(c, t);
  c->beta = saved_beta;
  if (rc != RIHVR_OK) return rc;
  RC(fetch_sums(c));
  if (sums3) {
    sums3[0] = c->sums_h[SLOT_PROX * kNumSums + SUM_LIM1];
    sums3[1] = c->sums_h[SLOT_PROX * kNumSums + SUM_LIM2];
    sums3[2] = c->sums_h[SLOT_PROX * kNumSums + SUM_RS];
  }
  KL(launch_materialize_x(c->storage, c->vol[c->iNew], c->vol[c->iNew], 0.f, c->U, (long long)c->V, c->st));
  // the context's solve state is no longer meaningful after this call
  c->have_holo = false;
  return copy_out(c, p_out, c->U, sizeof(float2) * c->V, is_device);
}

int rihvr_set_profiling(rihvr_ctx* c, int enable) {
  if (!c) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL context");
  CK(cudaStreamSynchronize(c->st));
  c->profiling = enable != 0;
  c->evs.clear();
  c->ev_used = 0;
  return RIHVR_OK;
}

int rihvr_kernel_times(rihvr_ctx* c, const char** names, double* total_ms, int* launches, int max, int* n_out) {
  if (!c || !n_out) return fail(RIHVR_ERR_INVALID_ARGUMENT, "NULL argument");
  CK(cudaStreamSynchronize(c->st));
  double tot[K_NUM] = {0};
  int cnt[K_NUM] = {0};
  for (const auto& e : c->evs) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
      tot[e.cls] += ms;
      cnt[e.cls]++;
    }
  }
  *n_out = K_NUM;
  for (int k = 0; k < K_NUM && k < max; ++k) {
    if (names) names[k] = kClassNames[k];
    if (total_ms) total_ms[k] = tot[k];
    if (launches) launches[k] = cnt[k];
  }
  return RIHVR_OK;
}

size_t rihvr_device_bytes(const rihvr_ctx* c) { return c ? c->bytes : 0; }

long long rihvr_launch_count(const rihvr_ctx* c) { return c ? c->launches : -1; }

void* rihvr_get_stream(rihvr_ctx* c) { return c ? (void*)c->st : nullptr; }

}  // extern "C"
