/*
 * FP64 CPU oracle of RIHVR's sparse inverse reconstruction (FASTA/FISTA with
 * L1 + TV regularisation over a Rayleigh-Sommerfeld forward model).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * path is compared against; nothing in the product links or calls it.  It is
 * also the timed CPU baseline ("port": the reference has no CPU path and its
 * CUDA build needs OpenCV C++, which is absent).
 *
 * Parity status: pinned to the reference's own kernels.  The reference ships
 * no golden vectors, fixtures or test bodies for this path, and cannot be
 * built whole here (OpenCV C++ is absent), but its hot-path CUDA kernels
 * compile alone: oracle/build_ref.py builds them, unchanged, behind the
 * harness oracle/ref_harness.cu, and tests/test_gpu_ref_pin.py checks every
 * operation of this file and its whole FISTA loop against them on a GPU.  It
 * is also checked against numpy.fft and mathematical known answers (adjoint
 * identity, unit-modulus transfer function, TV fixed points, shrink on
 * scalars).
 *
 * Everything is double precision complex.  Every function below cites the
 * reference function it restates (paths relative to the RIHVR source tree).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cd;

#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Mixed-radix Stockham FFT (radices 4, 2, 3, 5 and any odd prime), FP64.   */
/* cuFFT's cufftExecC2C is what the reference calls                          */
/* (src/core/sparse_compressive_holo.cu:98 plan, :1994 and :2054 exec;       */
/* src/core/sparse_gradient.cu:62, :151): unnormalised in both directions.   */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n;
    int nf;
    int fac[64];
    cd *tw; /* tw[m] = exp(-2*pi*i*m/n) */
} orc_fft_plan;

static void plan_init(orc_fft_plan *p, int n)
{
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->fac[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->fac[p->nf++] = 5; m /= 5; }
    for (int q = 7; m > 1; q += 2)
        while (m % q == 0) { p->fac[p->nf++] = q; m /= q; }
    p->tw = (cd *)malloc(sizeof(cd) * (size_t)n);
    for (int k = 0; k < n; ++k) {
        double a = -2.0 * ORC_PI * (double)k / (double)n;
        p->tw[k] = cos(a) + I * sin(a);
    }
}

static void plan_free(orc_fft_plan *p) { free(p->tw); p->tw = NULL; }

/* In-place R-point DFT of v[0..R) with sign -1 (forward) or +1 (inverse). */
static void small_dft(cd *v, int R, int inverse, const orc_fft_plan *p)
{
    const double s = inverse ? 1.0 : -1.0;
    if (R == 2) {
        cd a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    } else if (R == 4) {
        cd a = v[0] + v[2], b = v[0] - v[2];
        cd c = v[1] + v[3], d = (v[1] - v[3]) * (s * I);
        v[0] = a + c;
        v[2] = a - c;
        v[1] = b + d;
        v[3] = b - d;
    } else {
        cd out[64];
        cd *tmp = (R <= 64) ? out : (cd *)malloc(sizeof(cd) * (size_t)R);
        const int step = p->n / R;
        for (int q = 0; q < R; ++q) {
            cd acc = 0;
            for (int r = 0; r < R; ++r) {
                cd w = p->tw[(size_t)((r * q) % R) * step];
                acc += v[r] * (inverse ? conj(w) : w);
            }
            tmp[q] = acc;
        }
        memcpy(v, tmp, sizeof(cd) * (size_t)R);
        if (tmp != out) free(tmp);
    }
    (void)s;
}

/* Stockham autosort (Govindaraju et al. 2008 formulation): stage with radix
 * R reads x[j + r*n/R], applies twiddles exp(-+2 pi i k r/(Ns R)) with
 * k = j mod Ns, does an R-point DFT and writes x[(j/Ns)*Ns*R + k + r*Ns]. */
static void fft1d(const orc_fft_plan *p, cd *x, cd *work, int inverse)
{
    const int n = p->n;
    cd *in = x, *out = work;
    int Ns = 1;
    cd v[64];
    for (int s = 0; s < p->nf; ++s) {
        const int R = p->fac[s];
        const int m = n / R;
        const int tws = n / (Ns * R);
        cd *vv = (R <= 64) ? v : (cd *)malloc(sizeof(cd) * (size_t)R);
        for (int j = 0; j < m; ++j) {
            const int k = j % Ns;
            for (int r = 0; r < R; ++r) {
                cd a = in[j + r * m];
                if (r && k) {
                    cd w = p->tw[(size_t)k * r * tws];
                    a *= inverse ? conj(w) : w;
                }
                vv[r] = a;
            }
            small_dft(vv, R, inverse, p);
            const int base = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) out[base + r * Ns] = vv[r];
        }
        if (vv != v) free(vv);
        cd *t = in; in = out; out = t;
        Ns *= R;
    }
    if (in != x) memcpy(x, in, sizeof(cd) * (size_t)n);
}

/* Unnormalised 2D DFT of an H x W row-major plane (rows, then columns). */
static void fft2d_plans(const orc_fft_plan *pw, const orc_fft_plan *ph, int H, int W,
                        cd *a, int inverse, cd *work)
{
    /* work must hold max(W, H) * 9 elements */
    for (int y = 0; y < H; ++y) fft1d(pw, a + (size_t)y * W, work, inverse);
    enum { CB = 8 };
    cd *col = work + (H > W ? H : W);
    for (int x0 = 0; x0 < W; x0 += CB) {
        const int cb = (W - x0) < CB ? (W - x0) : CB;
        for (int y = 0; y < H; ++y)
            for (int c = 0; c < cb; ++c) col[(size_t)c * H + y] = a[(size_t)y * W + x0 + c];
        for (int c = 0; c < cb; ++c) fft1d(ph, col + (size_t)c * H, work, inverse);
        for (int y = 0; y < H; ++y)
            for (int c = 0; c < cb; ++c) a[(size_t)y * W + x0 + c] = col[(size_t)c * H + y];
    }
}

void orc_fft2(int H, int W, cd *a, int inverse)
{
    orc_fft_plan pw, ph;
    plan_init(&pw, W);
    plan_init(&ph, H);
    cd *work = (cd *)malloc(sizeof(cd) * (size_t)(H > W ? H : W) * 9);
    fft2d_plans(&pw, &ph, H, W, a, inverse, work);
    free(work);
    plan_free(&pw);
    plan_free(&ph);
}

void orc_fft1(int n, cd *a, int inverse)
{
    orc_fft_plan p;
    plan_init(&p, n);
    cd *work = (cd *)malloc(sizeof(cd) * (size_t)n);
    fft1d(&p, a, work, inverse);
    free(work);
    plan_free(&p);
}

/* ------------------------------------------------------------------------ */
/* Parameters                                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    int W, H, Nz;
    double dx;         /* pixel pitch (params.resolution) */
    double lambda;     /* wavelength (params.wavelength) */
    const double *z;   /* Nz plane positions (params.plane_list) */
    double l1;         /* regularization_param */
    double tv;         /* regularization_TV_param */
    int n_tv;          /* num_tv_iterations */
    int mode;          /* 5 = FASTA_L1, 6 = FUSED_LASSO (3-D TV), 7 = FUSED_LASSO_2D */
    int faithful;      /* 1 = reference arithmetic quirks, 0 = textbook variants */
    int max_backtracks;/* 2 in the reference (sparse_compressive_holo.cu:423) */
    int n_threads;     /* 0 = OpenMP default */
    double t0;         /* initial step; <= 0 means 1/Nz as in the reference (:247) */
} orc_params;

typedef struct {
    double f_prox;       /* objective at the accepted prox output */
    double f_resid_prox; /* 0.5*||A p - b||^2 */
    double lim;          /* line-search limit */
    double ratio;        /* backtracking ratio of the accepted step */
    double t;            /* step size used */
    double beta;         /* momentum factor (alpha0-1)/alpha1 */
    double f_x;          /* objective at the momentum point ("new f") */
    double f_resid_x;    /* 0.5*||A x - b||^2 at the momentum point */
    double l1_x, tv_x;   /* regulariser norms at the momentum point */
    double restart_sum;  /* restart test statistic */
    int backtracks;
    int restarted;
} orc_iter;

/* ------------------------------------------------------------------------ */
/* Transfer function                                                        */
/* ------------------------------------------------------------------------ */

/* Phase coefficient per frequency: c = (2 pi / lambda) (sqrt(1 - a) - 1),
 * a = (lambda/dx)^2 (fx^2 + fy^2), fx in FFT order, sqrt clamped at 0.
 * This folds the two phase factors the reference applies per plane:
 *   exp(-i 2 pi z / lambda)          (sparse_phase_scale_kernel, :1842-1861)
 *   exp(+i z 2 pi sqrt(...)/lambda)  (sparse_rs_exponent_kernel :38-56 and
 *                                     sparse_rs_phase_mult_kernel :1863-1888)
 * into H'_z = exp(i z c).  sqrt(1-a)-1 is written as -a/(sqrt(1-a)+1) to avoid
 * cancellation; for a >= 1 (evanescent, clamped) it is -1. */
void orc_phase_table(int H, int W, double dx, double lambda, double *c)
{
    const double k = 2.0 * ORC_PI / lambda;
    const double q = (lambda / dx) * (lambda / dx);
    for (int y = 0; y < H; ++y) {
        const double fy = (double)(((y + H / 2) % H) - (H / 2)) / (double)H;
        for (int x = 0; x < W; ++x) {
            const double fx = (double)(((x + W / 2) % W) - (W / 2)) / (double)W;
            const double a = q * (fx * fx + fy * fy);
            double sm1;
            if (a >= 1.0) sm1 = -1.0;
            else sm1 = -a / (sqrt(1.0 - a) + 1.0);
            c[(size_t)y * W + x] = k * sm1;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Workspace                                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
    orc_fft_plan pw, ph;
    double *c;     /* phase coefficients, H*W */
    int nthreads;
} orc_ws;

static void ws_init(orc_ws *ws, const orc_params *p)
{
    plan_init(&ws->pw, p->W);
    plan_init(&ws->ph, p->H);
    ws->c = (double *)malloc(sizeof(double) * (size_t)p->W * p->H);
    orc_phase_table(p->H, p->W, p->dx, p->lambda, ws->c);
#ifdef _OPENMP
    ws->nthreads = p->n_threads > 0 ? p->n_threads : omp_get_max_threads();
#else
    ws->nthreads = 1;
#endif
}

static void ws_free(orc_ws *ws)
{
    plan_free(&ws->pw);
    plan_free(&ws->ph);
    free(ws->c);
}

static inline cd cexpi(double ph) { return cos(ph) + I * sin(ph); }

/* ------------------------------------------------------------------------ */
/* Forward operator: SparseCompressiveHolo::backPropagate                    */
/* (src/core/sparse_compressive_holo.cu:1935-2077).                          */
/* d = Re( IFFT2( sum_z H'_z . FFT2(x_z) ) / (W H) )                         */
/* Planes are summed in fixed z-chunks so the result does not depend on the  */
/* thread count.                                                             */
/* ------------------------------------------------------------------------ */

#define ORC_ZCHUNKS 32

static void forward_ws(const orc_params *p, orc_ws *ws, const cd *vol, double *d_out, cd *spec_out)
{
    const size_t N = (size_t)p->W * p->H;
    const int nz = p->Nz;
    const int nch = nz < ORC_ZCHUNKS ? nz : ORC_ZCHUNKS;
    cd *part = (cd *)calloc((size_t)nch * N, sizeof(cd));
#pragma omp parallel for schedule(dynamic, 1) num_threads(ws->nthreads)
    for (int ch = 0; ch < nch; ++ch) {
        const int z0 = (int)((long)nz * ch / nch), z1 = (int)((long)nz * (ch + 1) / nch);
        cd *plane = (cd *)malloc(sizeof(cd) * N);
        cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
        cd *acc = part + (size_t)ch * N;
        for (int z = z0; z < z1; ++z) {
            memcpy(plane, vol + (size_t)z * N, sizeof(cd) * N);
            fft2d_plans(&ws->pw, &ws->ph, p->H, p->W, plane, 0, work);
            const double zz = p->z[z];
            for (size_t i = 0; i < N; ++i) acc[i] += plane[i] * cexpi(zz * ws->c[i]);
        }
        free(plane);
        free(work);
    }
    cd *S = (cd *)calloc(N, sizeof(cd));
    for (int ch = 0; ch < nch; ++ch)
        for (size_t i = 0; i < N; ++i) S[i] += part[(size_t)ch * N + i];
    free(part);
    if (spec_out) memcpy(spec_out, S, sizeof(cd) * N);
    cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
    fft2d_plans(&ws->pw, &ws->ph, p->H, p->W, S, 1, work);
    free(work);
    for (size_t i = 0; i < N; ++i) d_out[i] = creal(S[i]) / (double)N;
    free(S);
}

int orc_forward(const orc_params *p, const cd *vol, double *d_out)
{
    orc_ws ws;
    ws_init(&ws, p);
    forward_ws(p, &ws, vol, d_out, NULL);
    ws_free(&ws);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Adjoint operator: SparseGradient::reconstruct + getPlane                  */
/* (src/core/sparse_gradient.cu:47-75, :125-165).                            */
/* R = FFT2(r); g_z = IFFT2( conj(H'_z) . R ) / (W H)                        */
/* ------------------------------------------------------------------------ */

static void residual_spectrum(const orc_params *p, orc_ws *ws, const double *r, cd *R)
{
    const size_t N = (size_t)p->W * p->H;
    for (size_t i = 0; i < N; ++i) R[i] = r[i];
    cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
    fft2d_plans(&ws->pw, &ws->ph, p->H, p->W, R, 0, work);
    free(work);
}

static void adjoint_plane(const orc_params *p, orc_ws *ws, const cd *R, int z, cd *g, cd *work)
{
    const size_t N = (size_t)p->W * p->H;
    const double zz = p->z[z];
    for (size_t i = 0; i < N; ++i) g[i] = R[i] * cexpi(-zz * ws->c[i]) / (double)N;
    fft2d_plans(&ws->pw, &ws->ph, p->H, p->W, g, 1, work);
}

int orc_adjoint(const orc_params *p, const double *r, cd *vol_out)
{
    orc_ws ws;
    ws_init(&ws, p);
    const size_t N = (size_t)p->W * p->H;
    cd *R = (cd *)malloc(sizeof(cd) * N);
    residual_spectrum(p, &ws, r, R);
#pragma omp parallel for schedule(dynamic, 1) num_threads(ws.nthreads)
    for (int z = 0; z < p->Nz; ++z) {
        cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
        adjoint_plane(p, &ws, R, z, vol_out + (size_t)z * N, work);
        free(work);
    }
    free(R);
    ws_free(&ws);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Soft thresholds                                                          */
/* ------------------------------------------------------------------------ */

/* Separable shrink of each real component: block_soft_threshold_kernel and
 * block_soft_threshold_FASTA_kernel (sparse_compressive_holo.cu:3065-3157):
 * c <- c * m / (m + T), m = max(|c| - T, 0), i.e. sign(c) max(|c| - T, 0).
 * The reference produces 0/0 at c = 0 when T = 0; T = 0 is the identity here.
 * Non-faithful mode uses the complex-modulus shrink z max(|z|-T,0)/|z|. */
static inline cd shrink(cd v, double T, int faithful)
{
    if (T <= 0.0) return v;
    if (faithful) {
        double re = creal(v), im = cimag(v);
        double mr = fabs(re) - T, mi = fabs(im) - T;
        re = mr > 0 ? (re > 0 ? mr : -mr) : 0.0;
        im = mi > 0 ? (im > 0 ? mi : -mi) : 0.0;
        return re + I * im;
    }
    double a = cabs(v);
    if (a <= T) return 0.0;
    return v * ((a - T) / a);
}

/* ------------------------------------------------------------------------ */
/* 2-D TV prox for one plane: proximalFusedLasso2d                           */
/* (sparse_compressive_holo.cu:3652-3732, kernels :3478-3597).               */
/*  xh = x0 - t g;  gx = gy = 0;                                             */
/*  T times: y = xh - mu div(g);  g = P(g + s grad(y))                       */
/*  y = xh - mu div(g); optional separable shrink with t*l1                  */
/*  mu = t*tv, s = 1/(12 t tv), div forward-periodic, grad backward-periodic, */
/*  P divides by max(1, ||(gx,gy)|| over the 4 real components).            */
/* ------------------------------------------------------------------------ */

static void tv2d_prox_plane(int H, int W, const cd *xh, double mu, double s, int n_tv,
                            cd *y, cd *gx, cd *gy)
{
    const size_t N = (size_t)H * W;
    memset(gx, 0, sizeof(cd) * N);
    memset(gy, 0, sizeof(cd) * N);
    for (int it = 0; it <= n_tv; ++it) {
        for (int yy = 0; yy < H; ++yy) {
            const int yp = (yy < H - 1) ? yy + 1 : 0;
            for (int xx = 0; xx < W; ++xx) {
                const int xp = (xx < W - 1) ? xx + 1 : 0;
                const size_t i = (size_t)yy * W + xx;
                cd div = gx[(size_t)yy * W + xp] - gx[i] + gy[(size_t)yp * W + xx] - gy[i];
                y[i] = xh[i] - mu * div;
            }
        }
        if (it == n_tv) break;
        for (int yy = 0; yy < H; ++yy) {
            const int ym = (yy > 0) ? yy - 1 : H - 1;
            for (int xx = 0; xx < W; ++xx) {
                const int xm = (xx > 0) ? xx - 1 : W - 1;
                const size_t i = (size_t)yy * W + xx;
                cd px = gx[i] + s * (y[(size_t)yy * W + xm] - y[i]);
                cd py = gy[i] + s * (y[(size_t)ym * W + xx] - y[i]);
                double nrm = creal(px) * creal(px) + cimag(px) * cimag(px) +
                             creal(py) * creal(py) + cimag(py) * cimag(py);
                nrm = sqrt(nrm);
                if (nrm < 1.0) nrm = 1.0;
                gx[i] = px / nrm;
                gy[i] = py / nrm;
            }
        }
    }
}

/* One plane of the mode-5 or mode-7 prox.  x0 is the point the step starts
 * from, g the gradient plane, out receives the prox output. */
static void prox_plane_57(const orc_params *p, const cd *x0, const cd *g, double t, cd *out,
                          cd *xh, cd *gx, cd *gy)
{
    const size_t N = (size_t)p->W * p->H;
    const int mode = (p->tv == 0.0) ? 5 : p->mode;
    if (mode == 5) {
        /* proximalL1 (sparse_compressive_holo.cu:3274-3392) */
        for (size_t i = 0; i < N; ++i) out[i] = shrink(x0[i] - t * g[i], t * p->l1, p->faithful);
        return;
    }
    for (size_t i = 0; i < N; ++i) xh[i] = x0[i] - t * g[i];
    const double mu = t * p->tv;
    const double s = 1.0 / (4.0 * 3.0 * t * p->tv);
    tv2d_prox_plane(p->H, p->W, xh, mu, s, p->n_tv, out, gx, gy);
    if (p->l1 > 0.0)
        for (size_t i = 0; i < N; ++i) out[i] = shrink(out[i], t * p->l1, p->faithful);
}

int orc_prox_plane(const orc_params *p, const cd *x0, const cd *g, double t, cd *out)
{
    const size_t N = (size_t)p->W * p->H;
    cd *xh = (cd *)malloc(sizeof(cd) * N), *gx = (cd *)malloc(sizeof(cd) * N),
       *gy = (cd *)malloc(sizeof(cd) * N);
    prox_plane_57(p, x0, g, t, out, xh, gx, gy);
    free(xh); free(gx); free(gy);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* 3-D fused lasso prox: proximalFusedLasso (sparse_compressive_holo.cu:      */
/* 3422-3475) with totalVariationProjection (:3832-4018).  Half threshold,   */
/* n_tv unnormalised dual steps (the projection is disabled at :3964),       */
/* final estimate, half threshold.  Periodic in x, y and z.                  */
/* ------------------------------------------------------------------------ */

static void prox_volume_6(const orc_params *p, const cd *x0, const cd *g, double t, cd *out)
{
    const int W = p->W, H = p->H, Z = p->Nz;
    const size_t N = (size_t)W * H, V = N * Z;
    cd *gx = (cd *)calloc(V, sizeof(cd)), *gy = (cd *)calloc(V, sizeof(cd)),
       *gz = (cd *)calloc(V, sizeof(cd)), *y = (cd *)malloc(sizeof(cd) * V);
    const double Th = t * p->l1 / 2.0;
    for (size_t i = 0; i < V; ++i) out[i] = shrink(x0[i] - t * g[i], Th, p->faithful);
    const double mu = t * p->tv;
    const double s = 1.0 / (4.0 * 3.0 * t * p->tv);
    for (int it = 0; it <= p->n_tv; ++it) {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < Z; ++z) {
            const int zp = (z < Z - 1) ? z + 1 : 0;
            for (int yy = 0; yy < H; ++yy) {
                const int yp = (yy < H - 1) ? yy + 1 : 0;
                for (int xx = 0; xx < W; ++xx) {
                    const int xp = (xx < W - 1) ? xx + 1 : 0;
                    const size_t i = (size_t)z * N + (size_t)yy * W + xx;
                    cd div = gx[(size_t)z * N + (size_t)yy * W + xp] - gx[i] +
                             gy[(size_t)z * N + (size_t)yp * W + xx] - gy[i] +
                             gz[(size_t)zp * N + (size_t)yy * W + xx] - gz[i];
                    y[i] = out[i] - mu * div;
                }
            }
        }
        if (it == p->n_tv) break;
#pragma omp parallel for schedule(static)
        for (int z = 0; z < Z; ++z) {
            const int zm = (z > 0) ? z - 1 : Z - 1;
            for (int yy = 0; yy < H; ++yy) {
                const int ym = (yy > 0) ? yy - 1 : H - 1;
                for (int xx = 0; xx < W; ++xx) {
                    const int xm = (xx > 0) ? xx - 1 : W - 1;
                    const size_t i = (size_t)z * N + (size_t)yy * W + xx;
                    gx[i] += s * (y[(size_t)z * N + (size_t)yy * W + xm] - y[i]);
                    gy[i] += s * (y[(size_t)z * N + (size_t)ym * W + xx] - y[i]);
                    gz[i] += s * (y[(size_t)zm * N + (size_t)yy * W + xx] - y[i]);
                }
            }
        }
    }
    for (size_t i = 0; i < V; ++i) out[i] = shrink(y[i], Th, p->faithful);
    free(gx); free(gy); free(gz); free(y);
}

/* ------------------------------------------------------------------------ */
/* Norms: SparseVolume::calcL1NormComplex (sparse_volume.cu:194-235),        */
/* calcTVNorm2d (:365-446), calcTVNorm (:240-363), OpticalField::            */
/* calcSumMagnitude (optical_field.cu:411-483).                              */
/* ------------------------------------------------------------------------ */

static double l1_plane(size_t N, const cd *x)
{
    double s = 0;
    for (size_t i = 0; i < N; ++i) s += cabs(x[i]);
    return s;
}

static double tv2d_plane(int H, int W, const cd *x)
{
    double s = 0;
    for (int yy = 0; yy < H; ++yy) {
        const int ym = (yy > 0) ? yy - 1 : H - 1;
        for (int xx = 0; xx < W; ++xx) {
            const int xm = (xx > 0) ? xx - 1 : W - 1;
            const size_t i = (size_t)yy * W + xx;
            cd a = x[(size_t)yy * W + xm] - x[i], b = x[(size_t)ym * W + xx] - x[i];
            s += sqrt(creal(a) * creal(a) + cimag(a) * cimag(a) + creal(b) * creal(b) + cimag(b) * cimag(b));
        }
    }
    return s;
}

static double tv3d_plane(int H, int W, const cd *x, const cd *xprev)
{
    double s = 0;
    for (int yy = 0; yy < H; ++yy) {
        const int ym = (yy > 0) ? yy - 1 : H - 1;
        for (int xx = 0; xx < W; ++xx) {
            const int xm = (xx > 0) ? xx - 1 : W - 1;
            const size_t i = (size_t)yy * W + xx;
            cd a = x[(size_t)yy * W + xm] - x[i], b = x[(size_t)ym * W + xx] - x[i], c = xprev[i] - x[i];
            s += sqrt(creal(a) * creal(a) + cimag(a) * cimag(a) + creal(b) * creal(b) + cimag(b) * cimag(b) +
                      creal(c) * creal(c) + cimag(c) * cimag(c));
        }
    }
    return s;
}

/* Regulariser norms of a volume for the objective of the given mode. */
static void reg_norms(const orc_params *p, const cd *vol, double *l1, double *tv, int nthreads)
{
    const size_t N = (size_t)p->W * p->H;
    const int mode = (p->tv == 0.0) ? 5 : p->mode;
    double sl1 = 0, stv = 0;
#pragma omp parallel for reduction(+ : sl1, stv) schedule(static) num_threads(nthreads)
    for (int z = 0; z < p->Nz; ++z) {
        const cd *x = vol + (size_t)z * N;
        sl1 += l1_plane(N, x);
        if (mode == 7) stv += tv2d_plane(p->H, p->W, x);
        else if (mode == 6) {
            const int zm = (z > 0) ? z - 1 : p->Nz - 1;
            stv += tv3d_plane(p->H, p->W, x, vol + (size_t)zm * N);
        }
    }
    *l1 = sl1;
    *tv = stv;
}

/* calcObjectiveFunction (sparse_compressive_holo.cu:2838-2899) */
double orc_objective(const orc_params *p, const double *r, const cd *vol, double *terms3)
{
    const size_t N = (size_t)p->W * p->H;
    double rr = 0;
    for (size_t i = 0; i < N; ++i) rr += r[i] * r[i];
    double l1, tv;
    reg_norms(p, vol, &l1, &tv, p->n_threads > 0 ? p->n_threads : 1);
    if (terms3) { terms3[0] = 0.5 * rr; terms3[1] = l1; terms3[2] = tv; }
    return 0.5 * rr + p->l1 * l1 + p->tv * tv;
}

/* Restart statistic weights.  sparse_fistaRestart_kernel<512>
 * (sparse_compressive_holo.cu:4393-4432) overwrites the real product of the
 * second element of each pair with its imaginary product and reuses the
 * first element's imaginary product (:4411-4413).  Within each 1024-element
 * chunk of a plane, elements 0..511 therefore count Re + 2*Im and elements
 * 512..1023 count Im only. */
static inline void restart_weights(size_t i, int faithful, double *wr, double *wi)
{
    if (!faithful) { *wr = 1; *wi = 1; return; }
    if ((i & 1023u) < 512u) { *wr = 1; *wi = 2; }
    else { *wr = 0; *wi = 1; }
}

/* ------------------------------------------------------------------------ */
/* Prox + forward for a whole volume with the line-search and restart sums   */
/* (calcLineSearchLimit :4307-4390, fistaRestart :4434-4482).                */
/* ------------------------------------------------------------------------ */

typedef struct {
    double lim1, lim2, rs;
} step_sums;

static void prox_step(const orc_params *p, orc_ws *ws, const cd *X, const cd *Y0, const cd *R,
                      double t, cd *P, step_sums *sums)
{
    const size_t N = (size_t)p->W * p->H;
    const int nz = p->Nz;
    const int mode = (p->tv == 0.0) ? 5 : p->mode;
    double lim1 = 0, lim2 = 0, rs = 0;
    if (mode == 6) {
        cd *G = (cd *)malloc(sizeof(cd) * N * nz);
#pragma omp parallel for schedule(dynamic, 1) num_threads(ws->nthreads)
        for (int z = 0; z < nz; ++z) {
            cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
            adjoint_plane(p, ws, R, z, G + (size_t)z * N, work);
            free(work);
        }
        prox_volume_6(p, X, G, t, P);
#pragma omp parallel for reduction(+ : lim1, lim2, rs) schedule(static) num_threads(ws->nthreads)
        for (int z = 0; z < nz; ++z) {
            for (size_t i = 0; i < N; ++i) {
                const size_t k = (size_t)z * N + i;
                cd dpx = P[k] - X[k];
                lim1 += creal(dpx) * creal(G[k]) + cimag(dpx) * cimag(G[k]);
                lim2 += creal(dpx) * creal(dpx) + cimag(dpx) * cimag(dpx);
                double wr, wi;
                restart_weights(i, p->faithful, &wr, &wi);
                cd a = X[k] - P[k], b = P[k] - Y0[k];
                rs += wr * creal(a) * creal(b) + wi * cimag(a) * cimag(b);
            }
        }
        free(G);
    } else {
#pragma omp parallel for reduction(+ : lim1, lim2, rs) schedule(dynamic, 1) num_threads(ws->nthreads)
        for (int z = 0; z < nz; ++z) {
            cd *work = (cd *)malloc(sizeof(cd) * (size_t)(p->H > p->W ? p->H : p->W) * 9);
            cd *g = (cd *)malloc(sizeof(cd) * N), *xh = (cd *)malloc(sizeof(cd) * N),
               *gx = (cd *)malloc(sizeof(cd) * N), *gy = (cd *)malloc(sizeof(cd) * N);
            adjoint_plane(p, ws, R, z, g, work);
            const cd *x = X + (size_t)z * N;
            cd *pz = P + (size_t)z * N;
            prox_plane_57(p, x, g, t, pz, xh, gx, gy);
            const cd *y0 = Y0 + (size_t)z * N;
            double a1 = 0, a2 = 0, a3 = 0;
            for (size_t i = 0; i < N; ++i) {
                cd dpx = pz[i] - x[i];
                a1 += creal(dpx) * creal(g[i]) + cimag(dpx) * cimag(g[i]);
                a2 += creal(dpx) * creal(dpx) + cimag(dpx) * cimag(dpx);
                double wr, wi;
                restart_weights(i, p->faithful, &wr, &wi);
                cd a = x[i] - pz[i], b = pz[i] - y0[i];
                a3 += wr * creal(a) * creal(b) + wi * cimag(a) * cimag(b);
            }
            lim1 += a1; lim2 += a2; rs += a3;
            free(work); free(g); free(xh); free(gx); free(gy);
        }
    }
    sums->lim1 = lim1;
    sums->lim2 = lim2;
    sums->rs = rs;
}

/* ------------------------------------------------------------------------ */
/* Outer loop: SparseCompressiveHolo::inverseReconstruct                     */
/* (sparse_compressive_holo.cu:173-633).                                     */
/*  - x = 0 start, step t = 1/Nz (:247), alpha1 = 1                          */
/*  - ratio = f_resid(p) / (f_resid(x) + lim) (:402-403); while ratio        */
/*    outside [0, 1] and fewer than max_backtracks: t *= 0.5 and redo (:423)  */
/*  - restart if the restart statistic is > 0 (:471-475)                     */
/*  - alpha1 = (1 + sqrt(1 + 4 alpha0^2))/2, beta = (alpha0 - 1)/alpha1      */
/*  - x = p + beta (p - y0), y0 = p; d(x) by the same combination of d(p)    */
/*    and d(y0) (:480-498); r = d(x) - b; new gradient and objective.        */
/*  forced_bt / forced_rs (may be NULL) replay a given decision sequence:    */
/*  forced_bt[it] >= 0 fixes the backtrack count, forced_rs[it] >= 0 the      */
/*  restart decision.                                                        */
/* ------------------------------------------------------------------------ */

int orc_solve(const orc_params *p, const double *b, int n_iter, const int *forced_bt,
              const int *forced_rs, orc_iter *log, cd *x_out, cd *p_out, double *est_out,
              double *f0_out)
{
    orc_ws ws;
    ws_init(&ws, p);
    const size_t N = (size_t)p->W * p->H;
    const size_t V = N * (size_t)p->Nz;
    cd *X = (cd *)calloc(V, sizeof(cd));
    cd *Y0 = (cd *)calloc(V, sizeof(cd));
    cd *P = (cd *)calloc(V, sizeof(cd));
    if (!X || !Y0 || !P) { free(X); free(Y0); free(P); ws_free(&ws); return -1; }
    double *dX = (double *)calloc(N, sizeof(double));   /* d at the momentum point */
    double *dY0 = (double *)calloc(N, sizeof(double));  /* d at the previous prox output */
    double *dP = (double *)calloc(N, sizeof(double));   /* d at the new prox output */
    double *r = (double *)malloc(sizeof(double) * N);
    cd *R = (cd *)malloc(sizeof(cd) * N);

    double t = (p->t0 > 0.0) ? p->t0 : 1.0 / (double)p->Nz;
    double alpha1 = 1.0;
    /* x = 0: d = 0, r = -b */
    for (size_t i = 0; i < N; ++i) r[i] = dX[i] - b[i];
    double rr = 0;
    for (size_t i = 0; i < N; ++i) rr += r[i] * r[i];
    double prev_f_resid = 0.5 * rr;
    if (f0_out) *f0_out = prev_f_resid; /* l1 and tv of x = 0 vanish */
    residual_spectrum(p, &ws, r, R);

    for (int it = 0; it < n_iter; ++it) {
        double alpha0 = alpha1;
        int bt = 0;
        step_sums ss;
        double f_resid, lim, ratio;
        const int want_bt = forced_bt ? forced_bt[it] : -1;
        for (;;) {
            prox_step(p, &ws, X, Y0, R, t, P, &ss);
            forward_ws(p, &ws, P, dP, NULL);
            rr = 0;
            for (size_t i = 0; i < N; ++i) { double e = dP[i] - b[i]; rr += e * e; }
            f_resid = 0.5 * rr;
            lim = ss.lim1 + ss.lim2 / (2.0 * t);
            ratio = f_resid / (prev_f_resid + lim);
            int again;
            if (want_bt >= 0) again = bt < want_bt;
            else again = ((ratio > 1.0) || (ratio < 0.0)) && (bt < p->max_backtracks);
            if (!again) break;
            t *= 0.5;
            bt++;
        }
        double l1p, tvp;
        reg_norms(p, P, &l1p, &tvp, ws.nthreads);
        int restarted = (ss.rs > 0.0);
        if (forced_rs && forced_rs[it] >= 0) restarted = forced_rs[it];
        if (restarted) alpha0 = 1.0;
        alpha1 = (1.0 + sqrt(1.0 + 4.0 * alpha0 * alpha0)) / 2.0;
        const double beta = (alpha0 - 1.0) / alpha1;
#pragma omp parallel for schedule(static) num_threads(ws.nthreads)
        for (long long k = 0; k < (long long)V; ++k) {
            X[k] = P[k] + beta * (P[k] - Y0[k]);
            Y0[k] = P[k];
        }
        for (size_t i = 0; i < N; ++i) {
            dX[i] = dP[i] + beta * (dP[i] - dY0[i]);
            dY0[i] = dP[i];
            r[i] = dX[i] - b[i];
        }
        rr = 0;
        for (size_t i = 0; i < N; ++i) rr += r[i] * r[i];
        prev_f_resid = 0.5 * rr;
        residual_spectrum(p, &ws, r, R);
        double l1x, tvx;
        reg_norms(p, X, &l1x, &tvx, ws.nthreads);
        if (log) {
            orc_iter *L = &log[it];
            L->f_resid_prox = f_resid;
            L->f_prox = f_resid + p->l1 * l1p + p->tv * tvp;
            L->lim = lim;
            L->ratio = ratio;
            L->t = t;
            L->beta = beta;
            L->f_resid_x = prev_f_resid;
            L->l1_x = l1x;
            L->tv_x = tvx;
            L->f_x = prev_f_resid + p->l1 * l1x + p->tv * tvx;
            L->restart_sum = ss.rs;
            L->backtracks = bt;
            L->restarted = restarted;
        }
    }
    if (x_out) memcpy(x_out, X, sizeof(cd) * V);
    if (p_out) memcpy(p_out, Y0, sizeof(cd) * V);
    if (est_out) memcpy(est_out, dX, sizeof(double) * N);
    free(X); free(Y0); free(P); free(dX); free(dY0); free(dP); free(r); free(R);
    ws_free(&ws);
    return 0;
}

/* One prox step from a given point with a given residual (the reference's
 * test_denoised hook, sparse_compressive_holo.cu:1207-1252, generalised):
 * P = prox(X - t A^H r).  Also returns the line-search sums. */
int orc_prox_from(const orc_params *p, const cd *X, const cd *Y0, const double *r, double t,
                  cd *P, double *sums3)
{
    orc_ws ws;
    ws_init(&ws, p);
    const size_t N = (size_t)p->W * p->H;
    cd *R = (cd *)malloc(sizeof(cd) * N);
    residual_spectrum(p, &ws, r, R);
    step_sums ss;
    prox_step(p, &ws, X, Y0, R, t, P, &ss);
    if (sums3) { sums3[0] = ss.lim1; sums3[1] = ss.lim2; sums3[2] = ss.rs; }
    free(R);
    ws_free(&ws);
    return 0;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Particle segmentation: the reference's separate segmentation program     */
/* (src/core/main_segmentation.cu:37-138) on a dense stack of voxel          */
/* intensities, the values its voxel file holds (zero = no voxel).  FP32    */
/* where the reference computes in FP32, in the reference's loop order.      */
/* ------------------------------------------------------------------------ */

typedef struct {
    float x, y, z, wx, wy, wz;
    int num_voxels;
    float max_value, mean_value;
    int xmin, xmax, ymin, ymax, zmin, zmax;
} orc_object;

typedef struct {
    long long sx, sy, sz;
    float wsx, wsy, wsz, wsum, vmax;
    double vsum;
    int n, xmin, xmax, ymin, ymax, zmin, zmax;
} orc_blob;

/* SparseSegmentation::simpleMorph (sparse_segmentation.cu:265-372): for every
 * on voxel, +1 at each in-bounds position of the ball around it; dilation
 * keeps non-zero counts, erosion counts above (ball size - 0.1). */
static void seg_morph(const unsigned char *in, unsigned char *out, int W, int H, int Nz, int cs, int erode)
{
    const size_t HW = (size_t)W * H, N = HW * Nz;
    int *cnt = (int *)calloc(N, sizeof(int));
    int nstrel = 0;
    for (int sz = -cs; sz <= cs; ++sz)
        for (int sx = -cs; sx <= cs; ++sx)
            for (int sy = -cs; sy <= cs; ++sy)
                if (sx * sx + sy * sy + sz * sz <= cs * cs) nstrel++;
    for (int z = 0; z < Nz; ++z)
        for (size_t p = 0; p < HW; ++p) {
            if (!in[(size_t)z * HW + p]) continue;
            const int x = (int)(p % W), y = (int)(p / W);
            for (int sz = -cs; sz <= cs; ++sz) {
                const int tz = z + sz;
                if (tz < 0 || tz >= Nz) continue;
                for (int sx = -cs; sx <= cs; ++sx)
                    for (int sy = -cs; sy <= cs; ++sy) {
                        const int tx = x + sx, ty = y + sy;
                        if (sx * sx + sy * sy + sz * sz <= cs * cs && tx >= 0 && tx < W && ty >= 0 && ty < H)
                            cnt[(size_t)tz * HW + (size_t)ty * W + tx] += 1;
                    }
            }
        }
    const double thr = nstrel - 0.1;
    for (size_t i = 0; i < N; ++i) out[i] = erode ? ((double)cnt[i] > thr) : (cnt[i] != 0);
    free(cnt);
}

/* In-plane neighbour of plane position p at offset (dx, dy): the reference's
 * linear offset dy*W + dx, any position inside the plane (faithful,
 * sparse_segmentation.cu:493-511), or the geometric neighbour. */
static long long seg_neighbour(int W, int H, int faithful, size_t p, int dx, int dy)
{
    const int x = (int)(p % W), y = (int)(p / W);
    if (faithful) {
        const long long l = (long long)p + (long long)dy * W + dx;
        return (l >= 0 && l < (long long)W * H) ? l : -1;
    }
    if (x + dx < 0 || x + dx >= W || y + dy < 0 || y + dy >= H) return -1;
    return (long long)(y + dy) * W + (x + dx);
}

/* SparseSegmentation::labelConnectedComponents (:467-555): every on voxel
 * starts with its linear index; sweeps in index order replace it with the
 * smallest label among its 27-neighbourhood until nothing changes.  Planes
 * outside the volume have no voxels. */
static void seg_label(const unsigned char *on, unsigned long long *lab, int W, int H, int Nz, int faithful)
{
    const size_t HW = (size_t)W * H, N = HW * Nz;
    for (size_t i = 0; i < N; ++i) lab[i] = on[i] ? (unsigned long long)i : ~0ull;
    int changed = 1;
    while (changed) {
        changed = 0;
        for (int z = 0; z < Nz; ++z)
            for (size_t p = 0; p < HW; ++p) {
                const size_t i = (size_t)z * HW + p;
                if (!on[i]) continue;
                unsigned long long v = lab[i];
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy) {
                        const long long q = seg_neighbour(W, H, faithful, p, dx, dy);
                        if (q < 0) continue;
                        for (int dz = -1; dz <= 1; ++dz) {
                            const int zz = z + dz;
                            if (zz < 0 || zz >= Nz) continue;
                            const size_t j = (size_t)zz * HW + (size_t)q;
                            if (on[j] && lab[j] < v) {
                                v = lab[j];
                                changed = 1;
                            }
                        }
                    }
                lab[i] = v;
            }
    }
}

/* Whole pipeline: binarize (:61-112; max from SparseVolume::calcMaxIntensity,
 * sparse_volume.cu:482-516), close (:186-263), label, objects in order of
 * first appearance (object_cloud.cu:127-265) with their intensities
 * (:269-289) and Blob3d's centroid, weighted centroid, max, mean and bounds
 * (blob3d.cu), blobSizeFilter (object_cloud.cu:313-328).  Returns the number
 * of objects kept (or -1 if more than max_out); info2 = {max, threshold}. */
int orc_segment(const float *inten, int W, int H, int Nz, double min_intensity, int close_size, int min_area,
                int faithful, orc_object *out, int max_out, double *info2)
{
    const size_t HW = (size_t)W * H, N = HW * Nz;
    float *q = (float *)malloc(sizeof(float) * N);
    unsigned char *on0 = (unsigned char *)malloc(N), *on1 = (unsigned char *)malloc(N);
    double maxq = 0.0;
    for (size_t i = 0; i < N; ++i) {
        /* the loaded voxel is (sqrt(I), 0); its intensity is re*re + im*im */
        const float s = sqrtf(inten[i]);
        q[i] = s * s;
        const double d = q[i];
        if (d > maxq) maxq = d;
    }
    const double thr = min_intensity * maxq / 256.0;
    for (size_t i = 0; i < N; ++i) on0[i] = (double)q[i] > thr;
    const unsigned char *closed = on0;
    if (close_size > 0) {
        unsigned char *dil = (unsigned char *)malloc(N);
        seg_morph(on0, dil, W, H, Nz, close_size, 0);
        seg_morph(dil, on1, W, H, Nz, close_size, 1);
        free(dil);
        closed = on1;
    }
    unsigned long long *lab = (unsigned long long *)malloc(sizeof(unsigned long long) * N);
    seg_label(closed, lab, W, H, Nz, faithful);
    /* object of each label: first appearance while scanning by index */
    long long *obj_of = (long long *)malloc(sizeof(long long) * N);
    for (size_t i = 0; i < N; ++i) obj_of[i] = -1;
    size_t nobj = 0, cap = 1024;
    orc_blob *b = (orc_blob *)malloc(sizeof(orc_blob) * cap);
    for (size_t i = 0; i < N; ++i) {
        if (!closed[i]) continue;
        long long o = obj_of[lab[i]];
        if (o < 0) {
            if (nobj == cap) {
                cap *= 2;
                b = (orc_blob *)realloc(b, sizeof(orc_blob) * cap);
            }
            o = (long long)nobj++;
            obj_of[lab[i]] = o;
            memset(&b[o], 0, sizeof(orc_blob));
        }
        orc_blob *s = &b[o];
        const int z = (int)(i / HW), y = (int)((i % HW) / W), x = (int)(i % W);
        const float w = on0[i] ? q[i] : 0.0f; /* masked complex volume, :51-59 */
        s->sx += x;
        s->sy += y;
        s->sz += z;
        s->wsx += w * (float)x;
        s->wsy += w * (float)y;
        s->wsz += w * (float)z;
        s->wsum += w;
        s->vsum += (double)w;
        if (s->n == 0 || w > s->vmax) s->vmax = w;
        if (s->n == 0) {
            s->xmin = s->xmax = x;
            s->ymin = s->ymax = y;
            s->zmin = s->zmax = z;
        } else {
            if (x < s->xmin) s->xmin = x;
            if (x > s->xmax) s->xmax = x;
            if (y < s->ymin) s->ymin = y;
            if (y > s->ymax) s->ymax = y;
            if (z < s->zmin) s->zmin = z;
            if (z > s->zmax) s->zmax = z;
        }
        s->n += 1;
    }
    orc_object *o = (orc_object *)malloc(sizeof(orc_object) * (nobj ? nobj : 1));
    for (size_t k = 0; k < nobj; ++k) {
        const orc_blob *s = &b[k];
        const float n = (float)s->n;
        o[k].x = (float)s->sx / n;
        o[k].y = (float)s->sy / n;
        o[k].z = (float)s->sz / n;
        o[k].wx = s->wsx / s->wsum;
        o[k].wy = s->wsy / s->wsum;
        o[k].wz = s->wsz / s->wsum;
        o[k].num_voxels = s->n;
        o[k].max_value = s->vmax;
        o[k].mean_value = (float)s->vsum / n;
        o[k].xmin = s->xmin;
        o[k].xmax = s->xmax;
        o[k].ymin = s->ymin;
        o[k].ymax = s->ymax;
        o[k].zmin = s->zmin;
        o[k].zmax = s->zmax;
    }
    long long kept = (long long)nobj;
    for (long long n = 0; n < kept; ++n)
        if (o[n].num_voxels < min_area) {
            o[n] = o[kept - 1];
            --n;
            --kept;
        }
    int rc = (int)kept;
    if (kept > max_out) rc = -1;
    else if (kept > 0) memcpy(out, o, sizeof(orc_object) * (size_t)kept);
    if (info2) {
        info2[0] = maxq;
        info2[1] = thr;
    }
    free(o);
    free(b);
    free(obj_of);
    free(lab);
    free(q);
    free(on0);
    free(on1);
    return rc;
}
