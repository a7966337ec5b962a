// Harness around the reference's own hot-path kernels (TEST INFRASTRUCTURE
// ONLY; built by oracle/build_ref.py into oracle/_ref/libref_kernels.so).
//
// The kernels come verbatim from the reference sources (ref_kernels.cuh is
// generated at build time and never committed).  This file restates the
// reference's HOST code around them - launch shapes, call order, cuFFT calls,
// FP32 partial sums finished on the host - from these reference functions:
//   SparseCompressiveHolo ctor     sparse_compressive_holo.cu:58-135  (cuFFT plan :98, exponent table :117-123)
//   backPropagate                  :1935-2077 (dense planes; the reference skips empty planes, which add zero)
//   calcResidual / calcResidualFrom :2676-2723, :4644-4742 (mode RM_EST_TRUE: r = estimate - measured)
//   calcResidualObjective          :2773-2790 with OpticalField::calcSumMagnitude (optical_field.cu:448-483)
//   calcObjectiveFunction          :2838-2899 with SparseVolume::calcL1NormComplex (sparse_volume.cu:194-235)
//                                  and calcTVNorm2d (sparse_volume.cu:392-446)
//   proximalL1                     :3274-3392
//   proximalFusedLasso2d           :3652-3732
//   calcLineSearchLimit            :4307-4390
//   fistaRestart                   :4434-4482
//   fistaUpdate (volume, hologram) :4496-4580, :4597-4642
//   inverseReconstruct             :173-633
//   SparseGradient::reconstruct / getPlane  sparse_gradient.cu:47-75, :125-165
// Volumes are dense (the reference's COO SparseVolume stores the same values
// without the zeros).  Every function takes and returns host arrays and
// allocates its own device memory; complex arrays are interleaved floats.
//
// Preconditions of the reference kernels, checked before any launch: width
// and height multiples of 16 (grids of W/16 x H/16 blocks, no bounds check in
// several kernels) and width*height a multiple of 1024 (the reductions read
// element i + 512 of each 1024-element chunk unguarded).
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ref_kernels.cuh"

namespace {

thread_local std::string g_err;

struct Fail {};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    throw Fail{};
  }
}
void ckf(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) {
    g_err = std::string(what) + ": cufft error " + std::to_string((int)r);
    throw Fail{};
  }
}
void require(bool ok, const char* what) {
  if (!ok) {
    g_err = what;
    throw Fail{};
  }
}

template <typename T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  explicit Dev(size_t count) : n(count) { ck(cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc"); }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  ~Dev() { cudaFree(p); }
  void from(const void* h) { ck(cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice), "H2D"); }
  void to(void* h) const { ck(cudaMemcpy(h, p, n * sizeof(T), cudaMemcpyDeviceToHost), "D2H"); }
  void zero() { ck(cudaMemset(p, 0, n * sizeof(T)), "cudaMemset"); }
};

void check_shape(int W, int H, int Nz) {
  require(W > 0 && H > 0 && Nz > 0, "sizes must be positive");
  require(W % 16 == 0 && H % 16 == 0, "width and height must be multiples of 16 (reference grids)");
  require(((size_t)W * H) % 1024 == 0, "width*height must be a multiple of 1024 (reference reductions)");
}

// The state the reference keeps in SparseCompressiveHolo and SparseGradient.
struct Ctx {
  int W, H, Nz;
  float lambda, dx;       // Parameters::wavelength, resolution (float, holo_ui.h:97-121)
  std::vector<float> z;   // Parameters::plane_list (float)
  size_t HW;
  dim3 b2{16, 16}, g2;
  cufftHandle plan = 0;
  Dev<double> exp_fwd, exp_adj;   // exponent_data of the two classes
  Dev<float2> buffer_plane, holo_fft;  // buffer_plane_d (:121), SparseGradient::holo_fft_d

  Ctx(int W_, int H_, int Nz_, const float* zlist, float lam, float dx_)
      : W(W_), H(H_), Nz(Nz_), lambda(lam), dx(dx_), z(zlist, zlist + Nz_), HW((size_t)W_ * H_),
        g2(W_ / 16, H_ / 16), exp_fwd(HW), exp_adj(HW), buffer_plane(HW), holo_fft(HW) {
    ckf(cufftPlan2d(&plan, H, W, CUFFT_C2C), "cufftPlan2d");  // :98
    sparse_rs_exponent_kernel<<<g2, b2>>>(exp_fwd.p, W, H, lambda, dx);  // :120-121
    ck(cudaGetLastError(), "sparse_rs_exponent_kernel");
  }
  ~Ctx() {
    if (plan) cufftDestroy(plan);
  }

  // backPropagate (:1935-2077): holo = finish(IFFT(sum_z rs(-z) FFT(phase(-z) x_z))) ; planes dense
  void forward(const float2* vol_d, float2* holo_d) {
    ck(cudaMemset(holo_d, 0, HW * sizeof(float2)), "memset holo");
    const double scale = 2 / std::sqrt(2 * Nz);
    for (int zid = 0; zid < Nz; ++zid) {
      const double zz = z[zid];
      float2* plane_d = const_cast<float2*>(vol_d) + (size_t)zid * HW;
      sparse_phase_scale_kernel<<<g2, b2>>>(buffer_plane.p, plane_d, W, H, lambda, -zz);
      ckf(cufftExecC2C(plan, buffer_plane.p, buffer_plane.p, CUFFT_FORWARD), "fft fwd");
      sparse_rs_phase_mult_kernel<<<g2, b2>>>(buffer_plane.p, buffer_plane.p, W, H, exp_fwd.p, -zz, scale);
      sparse_add_plane_kernel<<<g2, b2>>>(holo_d, buffer_plane.p, W, H);
    }
    ckf(cufftExecC2C(plan, holo_d, holo_d, CUFFT_INVERSE), "fft inv");
    back_propagate_finish_kernel<<<g2, b2>>>(holo_d, W, H);
    ck(cudaGetLastError(), "forward kernels");
    // mult(holo, depth / planes_used) with every plane used: a factor of 1
  }

  // SparseGradient::reconstruct (sparse_gradient.cu:47-75)
  void gradient_reconstruct(const float2* resid_d) {
    ck(cudaMemcpy(holo_fft.p, resid_d, HW * sizeof(float2), cudaMemcpyDeviceToDevice), "copy r");
    ckf(cufftExecC2C(plan, holo_fft.p, holo_fft.p, CUFFT_FORWARD), "fft r");
    sparse_rs_exponent_kernel2<<<g2, b2>>>(exp_adj.p, W, H, lambda, dx);
    ck(cudaGetLastError(), "sparse_rs_exponent_kernel2");
  }

  // SparseGradient::getPlane (sparse_gradient.cu:125-165)
  void gradient_plane(int zid, float2* plane_d) {
    const float zf = z[zid];
    sparse_rs_phase_mult_kernel2<<<g2, b2>>>(plane_d, holo_fft.p, W, H, exp_adj.p, zf);
    ckf(cufftExecC2C(plan, plane_d, plane_d, CUFFT_INVERSE), "fft grad plane");
    const double scale = 2 / std::sqrt(2 * Nz);
    sparse_phase_scale_kernel2<<<g2, b2>>>(plane_d, plane_d, W, H, lambda, zf, scale);
    ck(cudaGetLastError(), "gradient plane kernels");
  }
};

// FP32 block partials finished on the host in float, as the reference does
// after each reduction launch (:4338-4375, :4461-4469, optical_field.cu:474-481).
struct Reducer {
  int grid;
  Dev<float> buf;
  std::vector<float> host;
  explicit Reducer(size_t size) : grid((int)std::ceil(size / (512.0 * 2.0))), buf(grid), host(grid) {}
  float sum() {
    buf.to(host.data());
    float s = 0;
    for (int i = 0; i < grid; ++i) s += host[i];
    return s;
  }
};

// f_x, f_resid_x, f_prox, lim, ratio, stepsize, beta, backtracks, restarted, restart_sum
constexpr int kRecordFields = 10;

struct Solver {
  Ctx& c;
  int mode;
  double reg, reg_tv;  // regularization, regularization_TV (double members from float params)
  int n_tv;
  double stepsize = 1.0;
  Dev<float2> x1, x0, y0, y1, grad_plane, gx, gy, temp;
  Dev<float2> measured, residual, estimated, previous_est, current_est;
  Dev<float> tv_plane;
  Reducer red;
  int grid1;  // 1-D grids of 256 threads over a plane (:3652-3660 and friends)

  Solver(Ctx& ctx, int mode_, double reg_, double reg_tv_, int n_tv_)
      : c(ctx), mode(mode_), reg(reg_), reg_tv(reg_tv_), n_tv(n_tv_),
        x1(ctx.HW * ctx.Nz), x0(ctx.HW * ctx.Nz), y0(ctx.HW * ctx.Nz), y1(ctx.HW * ctx.Nz),
        grad_plane(ctx.HW), gx(ctx.HW), gy(ctx.HW), temp(ctx.HW), measured(ctx.HW), residual(ctx.HW),
        estimated(ctx.HW), previous_est(ctx.HW), current_est(ctx.HW), tv_plane(ctx.HW * 2), red(ctx.HW),
        grid1((int)std::ceil(ctx.HW / 256.0)) {
    if (reg_tv_ == 0.0) mode = 5;  // :192-195
  }

  float2* plane(Dev<float2>& v, int zid) { return v.p + (size_t)zid * c.HW; }

  // proximalL1 (:3274-3392) / proximalFusedLasso2d (:3652-3732): x1 = prox(x0 - t grad)
  void denoise() {
    for (int zid = 0; zid < c.Nz; ++zid) {
      c.gradient_plane(zid, grad_plane.p);
      float2* x_d = plane(x1, zid);
      float2* xm1_d = plane(x0, zid);
      if (mode == 5) {
        block_soft_threshold_FASTA_kernel<<<grid1, 256>>>(x_d, xm1_d, grad_plane.p, stepsize, reg, c.HW);
      } else {
        const double scale = 1 / (4 * 3 * stepsize * reg_tv);
        sparse_get_xhat_kernel<<<grid1, 256>>>(x_d, xm1_d, grad_plane.p, stepsize, c.HW);
        gx.zero();
        gy.zero();
        for (int i = 0; i < n_tv; ++i) {
          tv_denoised_estimate_2d_kernel<<<c.g2, c.b2>>>(temp.p, x_d, gx.p, gy.p, stepsize * reg_tv, c.W, c.H);
          tv_gradient_projection_2d_kernel<<<c.g2, c.b2>>>(gx.p, gy.p, temp.p, scale, c.W, c.H);
        }
        tv_denoised_estimate_2d_kernel<<<c.g2, c.b2>>>(temp.p, x_d, gx.p, gy.p, stepsize * reg_tv, c.W, c.H);
        ck(cudaMemcpy(x_d, temp.p, c.HW * sizeof(float2), cudaMemcpyDeviceToDevice), "copy xhat");
        if (reg > 0.0) block_soft_threshold_kernel<<<grid1, 256>>>(x_d, stepsize, reg, c.HW);
      }
      ck(cudaGetLastError(), "prox kernels");
    }
  }

  // calcResidual (:2676-2723): estimate = A x1, residual = estimate - measured
  void calc_residual() {
    c.forward(x1.p, estimated.p);
    calc_residual_from();
  }
  // calcResidualFrom (:4644-4742)
  void calc_residual_from() {
    const size_t dim_grid = (size_t)std::ceil((float)c.HW / (float)256);
    sparse_calc_residual_inverse_kernel<<<dim_grid, 256>>>(residual.p, measured.p, estimated.p, c.HW);
    ck(cudaGetLastError(), "residual kernel");
  }
  // calcSumMagnitude (optical_field.cu:448-483), as a float
  float sum_magnitude(const float2* d) {
    my_summag_kernel<512><<<red.grid, 512, 512 * sizeof(float)>>>(const_cast<float2*>(d), red.buf.p, (int)c.HW);
    ck(cudaGetLastError(), "my_summag_kernel");
    return red.sum();
  }
  double residual_objective() { return 0.5 * sum_magnitude(residual.p); }  // :2773-2790

  // calcL1NormComplex (sparse_volume.cu:194-235): host loop in double over the nonzero voxels
  double l1_norm() {
    std::vector<float2> h(c.HW);
    double norm = 0;
    for (int zid = 0; zid < c.Nz; ++zid) {
      ck(cudaMemcpy(h.data(), plane(x1, zid), c.HW * sizeof(float2), cudaMemcpyDeviceToHost), "D2H plane");
      for (size_t i = 0; i < c.HW; ++i) {
        const float2 v = h[i];
        if (v.x != 0.f || v.y != 0.f) norm += std::sqrt(v.x * v.x + v.y * v.y);
      }
    }
    return norm;
  }
  // calcTVNorm2d (sparse_volume.cu:392-446)
  double tv_norm_2d() {
    double norm = 0;
    for (int zid = 0; zid < c.Nz; ++zid) {
      tv_norm_2d_kernel<<<c.g2, c.b2>>>(tv_plane.p, plane(x1, zid), c.W, c.H);
      tv_summation_kernel<512><<<red.grid, 512, 512 * sizeof(float)>>>(tv_plane.p, red.buf.p, (int)c.HW);
      ck(cudaGetLastError(), "tv norm kernels");
      red.buf.to(red.host.data());
      for (int i = 0; i < red.grid; ++i) norm += red.host[i];
    }
    return norm;
  }
  // calcObjectiveFunction (:2838-2899); terms: 0.5 resid_norm, l1, tv
  double objective(double* terms) {
    const float resid_norm = sum_magnitude(residual.p);
    const double l1 = l1_norm();
    double f = 0.5 * resid_norm + reg * l1;
    double tv = 0;
    if (mode == 7) {
      tv = tv_norm_2d();
      f = f + reg_tv * tv;
    }
    if (terms) {
      terms[0] = 0.5 * resid_norm;
      terms[1] = l1;
      terms[2] = tv;
    }
    return f;
  }

  // calcLineSearchLimit (:4307-4390)
  double line_search_limit(float* s1, float* s2) {
    float sum1 = 0, sum2 = 0;
    for (int zid = 0; zid < c.Nz; ++zid) {
      c.gradient_plane(zid, grad_plane.p);
      sparse_linesearch_1_kernel<512><<<red.grid, 512, 512 * sizeof(float)>>>(plane(x1, zid), plane(x0, zid),
                                                                               grad_plane.p, red.buf.p, (int)c.HW);
      ck(cudaGetLastError(), "linesearch_1");
      red.buf.to(red.host.data());
      for (int i = 0; i < red.grid; ++i) sum1 += red.host[i];
      sparse_linesearch_2_kernel<512><<<red.grid, 512, 512 * sizeof(float)>>>(plane(x1, zid), plane(x0, zid),
                                                                               red.buf.p, (int)c.HW);
      ck(cudaGetLastError(), "linesearch_2");
      red.buf.to(red.host.data());
      for (int i = 0; i < red.grid; ++i) sum2 += red.host[i];
    }
    if (s1) *s1 = sum1;
    if (s2) *s2 = sum2;
    return sum1 + sum2 / (2 * stepsize);
  }

  // fistaRestart (:4434-4482)
  float restart_sum(Dev<float2>& a0, Dev<float2>& a1, Dev<float2>& accel) {
    float sum1 = 0;
    for (int zid = 0; zid < c.Nz; ++zid) {
      sparse_fistaRestart_kernel<512><<<red.grid, 512, 512 * sizeof(float)>>>(plane(a0, zid), plane(a1, zid),
                                                                              plane(accel, zid), red.buf.p,
                                                                              (int)c.HW);
      ck(cudaGetLastError(), "fistaRestart");
      red.buf.to(red.host.data());
      for (int i = 0; i < red.grid; ++i) sum1 += red.host[i];
    }
    return sum1;
  }

  // fistaUpdate (:4496-4580 per plane, :4597-4642 hologram): out = cur + step (cur - prev)
  void fista_update(float2* out, float2* prev, float2* cur, size_t n, double step) {
    const int grid = (int)std::ceil(n / (double)256);
    sparse_fistaUpdate_kernel<<<grid, 256>>>(out, prev, cur, step, n);
    ck(cudaGetLastError(), "fistaUpdate");
  }
  void copy(Dev<float2>& dst, const Dev<float2>& src) {
    ck(cudaMemcpy(dst.p, src.p, dst.n * sizeof(float2), cudaMemcpyDeviceToDevice), "copy");
  }

  // inverseReconstruct (:173-633), from x = 0, `n_iter` iterations
  void solve(int n_iter, double* rec) {
    stepsize = 1.0 / (double)c.Nz;  // :247
    x1.zero();
    copy(x0, x1);  // :258-259 (x0 = x1; y0 = x1)
    copy(y0, x1);
    double alpha1 = 1.0;
    previous_est.zero();
    current_est.zero();
    calc_residual();                             // :273
    double prev_f_resid = residual_objective();  // :276-277
    c.gradient_reconstruct(residual.p);          // :286
    for (int it = 0; it < n_iter; ++it) {
      copy(x0, x1);  // :368
      double alpha0 = alpha1;
      denoise();      // :372
      int backtrack_count = 0;
      calc_residual();  // :388
      double lim = line_search_limit(nullptr, nullptr);
      double f_resid = residual_objective();
      double ratio = f_resid / (prev_f_resid + lim);  // :403
      while (((ratio > 1.0) || (ratio < 0)) && (backtrack_count < 2)) {  // :423
        stepsize *= 0.5;  // stepsize_shrinkage (:67)
        denoise();
        calc_residual();
        lim = line_search_limit(nullptr, nullptr);
        f_resid = residual_objective();
        ratio = f_resid / (prev_f_resid + lim);
        backtrack_count++;
      }
      const double f_prox = objective(nullptr);  // f at the accepted prox output (:389, :438)
      const float rsum = restart_sum(x0, x1, y0);  // :471
      const bool restarted = rsum > 0;
      if (restarted) alpha0 = 1;
      alpha1 = (1.0 + std::sqrt(1.0 + 4.0 * alpha0 * alpha0)) / 2.0;
      copy(y1, x1);  // :480
      const double step = (alpha0 - 1) / alpha1;
      fista_update(x1.p, y0.p, y1.p, c.HW * c.Nz, step);  // :483
      copy(y0, y1);
      copy(previous_est, current_est);  // :494-498
      copy(current_est, estimated);
      fista_update(estimated.p, previous_est.p, current_est.p, c.HW, step);
      copy(previous_est, current_est);
      calc_residual_from();                // :545
      c.gradient_reconstruct(residual.p);  // :547
      double t3[3];
      const double f = objective(t3);      // :548
      prev_f_resid = residual_objective();  // :549
      double* r = rec + (size_t)it * kRecordFields;
      r[0] = f;
      r[1] = prev_f_resid;
      r[2] = f_prox;
      r[3] = lim;
      r[4] = ratio;
      r[5] = stepsize;
      r[6] = step;
      r[7] = backtrack_count;
      r[8] = restarted ? 1.0 : 0.0;
      r[9] = rsum;
    }
  }
};

template <typename F>
int guarded(F&& f) {
  try {
    f();
    ck(cudaDeviceSynchronize(), "sync");
    return 0;
  } catch (const Fail&) {
    return 1;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }
int ref_record_fields(void) { return kRecordFields; }

// backPropagate: holo_out (H x W complex) = A vol (Nz x H x W complex)
int ref_forward(const float* vol, int W, int H, int Nz, const float* zlist, float lambda, float dx, float* holo_out) {
  return guarded([&] {
    check_shape(W, H, Nz);
    Ctx c(W, H, Nz, zlist, lambda, dx);
    Dev<float2> v(c.HW * Nz), h(c.HW);
    v.from(vol);
    c.forward(v.p, h.p);
    h.to(holo_out);
  });
}

// SparseGradient::reconstruct + getPlane of every plane: vol_out = A^H resid
int ref_adjoint(const float* resid, int W, int H, int Nz, const float* zlist, float lambda, float dx, float* vol_out) {
  return guarded([&] {
    check_shape(W, H, Nz);
    Ctx c(W, H, Nz, zlist, lambda, dx);
    Dev<float2> r(c.HW), v(c.HW * Nz);
    r.from(resid);
    c.gradient_reconstruct(r.p);
    for (int zid = 0; zid < Nz; ++zid) c.gradient_plane(zid, v.p + (size_t)zid * c.HW);
    v.to(vol_out);
  });
}

// One denoise(mode) call: x1_out = prox(x0 - stepsize * A^H resid) for mode 5
// (proximalL1) or 7 (proximalFusedLasso2d).  sums_out (may be NULL) receives
// the line-search sums of calcLineSearchLimit (sum1, sum2, lim) and the
// restart sum of fistaRestart(x0, x1, y0) for these x1, x0 (y0 may be NULL:
// y0 = x0).
int ref_prox(const float* x0, const float* y0, const float* resid, int W, int H, int Nz, const float* zlist,
             float lambda, float dx, int mode, double stepsize, double reg, double reg_tv, int n_tv, float* x1_out,
             double* sums_out) {
  return guarded([&] {
    check_shape(W, H, Nz);
    require(mode == 5 || mode == 7, "mode must be 5 or 7");
    Ctx c(W, H, Nz, zlist, lambda, dx);
    Solver s(c, mode, reg, reg_tv, n_tv);
    s.stepsize = stepsize;
    Dev<float2> r(c.HW);
    r.from(resid);
    c.gradient_reconstruct(r.p);
    s.x0.from(x0);
    s.denoise();
    s.x1.to(x1_out);
    if (sums_out) {
      float s1 = 0, s2 = 0;
      sums_out[2] = s.line_search_limit(&s1, &s2);
      sums_out[0] = s1;
      sums_out[1] = s2;
      if (y0) s.y0.from(y0); else s.copy(s.y0, s.x0);
      sums_out[3] = s.restart_sum(s.x0, s.x1, s.y0);
    }
  });
}

// fistaRestart's sum over three volumes (x0, x1, y0), with the reference's summation.
int ref_restart_sum(const float* x0, const float* x1, const float* y0, int W, int H, int Nz, double* sum_out) {
  return guarded([&] {
    check_shape(W, H, Nz);
    std::vector<float> z(Nz, 0.f);
    Ctx c(W, H, Nz, z.data(), 0.5f, 1.0f);
    Solver s(c, 7, 0, 1, 0);
    s.x0.from(x0);
    s.x1.from(x1);
    s.y0.from(y0);
    *sum_out = s.restart_sum(s.x0, s.x1, s.y0);
  });
}

// calcObjectiveFunction for residual `resid` (H x W complex) and volume `vol`;
// terms3 = (0.5 |r|^2, L1, TV2d), f_out = the objective for `mode`.
int ref_objective(const float* resid, const float* vol, int W, int H, int Nz, int mode, double reg, double reg_tv,
                  double* f_out, double* terms3) {
  return guarded([&] {
    check_shape(W, H, Nz);
    std::vector<float> z(Nz, 0.f);
    Ctx c(W, H, Nz, z.data(), 0.5f, 1.0f);
    Solver s(c, mode, reg, reg_tv, 0);
    s.residual.from(resid);
    s.x1.from(vol);
    *f_out = s.objective(terms3);
  });
}

// inverseReconstruct from x = 0 for `n_iter` iterations on the real hologram
// `holo` (H x W floats, imaginary part 0 as Hologram stores it).  records
// receives ref_record_fields() doubles per iteration: f (objective at the
// momentum point, :548), 0.5|r|^2 there (:549), f at the accepted prox output,
// lim, ratio, stepsize, beta, backtracks, restarted, restart sum.  vol_out (may be NULL) receives the final momentum
// point x1 (Nz x H x W complex).
int ref_solve(const float* holo, int W, int H, int Nz, const float* zlist, float lambda, float dx, float reg,
              float reg_tv, int n_tv, int mode, int n_iter, double* records, float* vol_out) {
  return guarded([&] {
    check_shape(W, H, Nz);
    require(mode == 5 || mode == 7, "mode must be 5 or 7");
    require(n_iter >= 0, "n_iter must be non-negative");
    Ctx c(W, H, Nz, zlist, lambda, dx);
    Solver s(c, mode, reg, reg_tv, n_tv);
    std::vector<float2> m(c.HW);
    for (size_t i = 0; i < c.HW; ++i) m[i] = make_float2(holo[i], 0.f);
    s.measured.from(m.data());
    s.solve(n_iter, records);
    if (vol_out) s.x1.to(vol_out);
  });
}

}  // extern "C"
