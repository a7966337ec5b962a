// Device building blocks for the sm_100a reconstruction kernels:
//  - complex helpers,
//  - compile-time unrolled in-register mixed-radix DFTs (Stockham autosort,
//    twiddles folded to immediates),
//  - the four-step split used by every line FFT (N = N1 * N2, N1 | N2):
//    thread n1 of a line owns x[n1 + N1*n2]; an N2-point DFT in registers,
//    an inter-stage twiddle, one shared-memory transpose, m = N2/N1
//    N1-point DFTs in registers.  Output element w[j*N1 + k1] of thread t is
//    X[(t + N1*j) + N2*k1].
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <type_traits>
#include <utility>

namespace rihvr {

// ---------------------------------------------------------------------------
// compile-time loops and trigonometry
// ---------------------------------------------------------------------------
template <typename F, int... Is>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

constexpr double kPi = 3.141592653589793238462643383279502884;

// Taylor series after reduction to [-pi, pi]; evaluated by the compiler only.
constexpr double cx_reduce(double x) {
  double t = x / (2.0 * kPi);
  long long k = (long long)(t >= 0 ? t + 0.5 : t - 0.5);
  return x - (double)k * 2.0 * kPi;
}
constexpr double cx_sin(double x) {
  x = cx_reduce(x);
  double term = x, sum = x;
  for (int n = 1; n < 40; ++n) {
    term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double cx_cos(double x) {
  x = cx_reduce(x);
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 40; ++n) {
    term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}

// exp(-+ 2 pi i K / N): forward transforms use the minus sign.
template <int K, int N, bool INV>
struct Tw {
  static constexpr double ang = (INV ? 2.0 : -2.0) * kPi * (double)K / (double)N;
  static constexpr float re = (float)cx_cos(ang);
  static constexpr float im = (float)cx_sin(ang);
};

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// Packed FP32x2 arithmetic (sm_100a): one instruction for both components of a
// complex value, bit-identical to two scalar round-to-nearest operations.
__device__ __forceinline__ unsigned long long f2_bits(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 f2_from(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from(r);
}
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from(r);
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from(r);
}
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) {  // a * b + c
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return f2_from(r);
}

// multiply by -i (fwd) or +i (inv)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// multiply by the compile-time twiddle exp(-+2 pi i K/N), exact for multiples of 1/8 turn
template <int K, int N, bool INV>
__device__ __forceinline__ float2 cmul_tw(float2 a) {
  constexpr int Kr = ((K % N) + N) % N;
  if constexpr (Kr == 0) {
    return a;
  } else if constexpr (4 * Kr == N) {
    return mul_mi<INV>(a);
  } else if constexpr (2 * Kr == N) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (4 * Kr == 3 * N) {
    return mul_mi<!INV>(a);
  } else if constexpr (8 * Kr == N || 8 * Kr == 3 * N || 8 * Kr == 5 * N || 8 * Kr == 7 * N) {
    constexpr float r = 0.70710678118654752440f;
    constexpr float cr = Tw<K, N, INV>::re > 0 ? r : -r;
    constexpr float ci = Tw<K, N, INV>::im > 0 ? r : -r;
    // (a.x + i a.y)(cr + i ci)
    return make_float2(cr * a.x - ci * a.y, cr * a.y + ci * a.x);
  } else {
    constexpr float wr = Tw<K, N, INV>::re, wi = Tw<K, N, INV>::im;
    return make_float2(fmaf(a.x, wr, -a.y * wi), fmaf(a.x, wi, a.y * wr));
  }
}

// ---------------------------------------------------------------------------
// in-register DFTs
// ---------------------------------------------------------------------------
template <int R, bool INV>
__device__ __forceinline__ void small_dft(float2 (&a)[R]) {
  // Radix 2 and 4 use packed FP32x2 adds (one instruction per complex add,
  // same bits as two scalar adds).  The radix-4 outputs t1 -+ i d mix the
  // halves of d, so they stay scalar; the swap and sign fold into the adds.
  if constexpr (R == 2) {
    const float2 t = a[0];
    a[0] = f2add(t, a[1]);
    a[1] = f2sub(t, a[1]);
  } else if constexpr (R == 4) {
    const float2 t0 = f2add(a[0], a[2]), t1 = f2sub(a[0], a[2]);
    const float2 t2 = f2add(a[1], a[3]), d = f2sub(a[1], a[3]);
    a[0] = f2add(t0, t2);
    a[2] = f2sub(t0, t2);
    if (INV) {  // t3 = +i d = (-d.y, d.x)
      a[1] = make_float2(t1.x - d.y, t1.y + d.x);
      a[3] = make_float2(t1.x + d.y, t1.y - d.x);
    } else {    // t3 = -i d = (d.y, -d.x)
      a[1] = make_float2(t1.x + d.y, t1.y - d.x);
      a[3] = make_float2(t1.x - d.y, t1.y + d.x);
    }
  } else if constexpr (R == 3) {
    constexpr float h = 0.86602540378443864676f;  // sqrt(3)/2
    float2 t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
    float2 m = make_float2(a[0].x - 0.5f * t1.x, a[0].y - 0.5f * t1.y);
    // s = -+ i h t2
    float2 s = INV ? make_float2(-h * t2.y, h * t2.x) : make_float2(h * t2.y, -h * t2.x);
    a[0] = cadd(a[0], t1);
    a[1] = cadd(m, s);
    a[2] = csub(m, s);
  } else {
    float2 o[R];
    static_for<R>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      float2 acc = a[0];
      static_for<R - 1>([&](auto rc) {
        constexpr int r = decltype(rc)::value + 1;
        acc = cadd(acc, cmul_tw<(r * q) % R, R, INV>(a[r]));
      });
      o[q] = acc;
    });
    static_for<R>([&](auto qc) { a[decltype(qc)::value] = o[decltype(qc)::value]; });
  }
}

template <int N>
constexpr int first_radix() {
  return (N % 4 == 0) ? 4 : (N % 2 == 0) ? 2 : (N % 3 == 0) ? 3 : (N % 5 == 0) ? 5 : N;
}

// One Stockham stage (published formulation of Govindaraju et al. 2008),
// with all indices and twiddles resolved at compile time.
template <int N, int R, int Ns, bool INV>
__device__ __forceinline__ void reg_stage(const float2 (&in)[N], float2 (&out)[N]) {
  constexpr int m = N / R;
  static_for<m>([&](auto jc) {
    constexpr int j = decltype(jc)::value;
    constexpr int k = j % Ns;
    float2 a[R];
    static_for<R>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      a[r] = cmul_tw<k * r, Ns * R, INV>(in[j + r * m]);
    });
    small_dft<R, INV>(a);
    constexpr int base = (j / Ns) * Ns * R + k;
    static_for<R>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      out[base + r * Ns] = a[r];
    });
  });
}

template <int N, int Ns, bool INV>
__device__ __forceinline__ void reg_fft_rec(float2 (&a)[N]) {
  if constexpr (Ns < N) {
    constexpr int R = first_radix<N / Ns>();
    float2 b[N];
    reg_stage<N, R, Ns, INV>(a, b);
#pragma unroll
    for (int i = 0; i < N; ++i) a[i] = b[i];
    reg_fft_rec<N, Ns * R, INV>(a);
  }
}

// Unnormalised N-point DFT of a register array, natural order in and out.
template <int N, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&a)[N]) {
  reg_fft_rec<N, 1, INV>(a);
}

// ---------------------------------------------------------------------------
// runtime twiddles exp(-+2 pi i n1 k / N), k = 0..N2-1, from two accurate
// anchors (sincospi) and short product chains (<= 15 complex products).
// ---------------------------------------------------------------------------
template <int N, int N2, bool INV>
__device__ __forceinline__ void line_twiddle(float2 (&v)[N2], int n1) {
  if (n1 == 0) return;
  // chain length: the largest of 8, 4, 2, 1 that divides N2 (every element is twiddled)
  constexpr int B = (N2 % 8 == 0) ? 8 : (N2 % 4 == 0) ? 4 : (N2 % 2 == 0) ? 2 : 1;
  static_assert(N2 % B == 0, "anchor blocks must tile the line");
  const float sgn = INV ? 2.0f : -2.0f;
  float s1, c1, s8, c8;
  sincospif(sgn * (float)n1 / (float)N, &s1, &c1);
  sincospif(sgn * (float)(n1 * B) / (float)N, &s8, &c8);
  const float2 w1 = make_float2(c1, s1), wB = make_float2(c8, s8);
  float2 pw[B];
  pw[0] = make_float2(1.f, 0.f);
#pragma unroll
  for (int b = 1; b < B; ++b) pw[b] = cmul(pw[b - 1], w1);
  float2 anchor = make_float2(1.f, 0.f);
#pragma unroll
  for (int a = 0; a < N2 / B; ++a) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      if (a == 0 && b == 0) continue;
      v[a * B + b] = cmul(v[a * B + b], cmul(anchor, pw[b]));
    }
    anchor = cmul(anchor, wB);
  }
}

// The same twiddles w^(n1 k), k = 0..N2-1, each from its own sincospi, for
// kernels that keep them in registers across many lines of the same n1.
template <int N, int N2, bool INV>
__device__ __forceinline__ void line_twiddles(float2 (&tw)[N2], int n1) {
  const float sgn = INV ? 2.0f : -2.0f;
#pragma unroll
  for (int k = 0; k < N2; ++k) {
    float s, c;
    sincospif(sgn * (float)((n1 * k) % N) / (float)N, &s, &c);
    tw[k] = make_float2(c, s);
  }
}

// ---------------------------------------------------------------------------
// storage types for the volumes (complex, interleaved)
// ---------------------------------------------------------------------------
template <typename ST>
struct Store;
template <>
struct Store<float2> {
  static __device__ __forceinline__ float2 ld(const float2* p) { return *p; }
  static __device__ __forceinline__ void st(float2* p, float2 v) { *p = v; }
};
template <>
struct Store<__nv_bfloat162> {
  static __device__ __forceinline__ float2 ld(const __nv_bfloat162* p) { return __bfloat1622float2(*p); }
  static __device__ __forceinline__ void st(__nv_bfloat162* p, float2 v) { *p = __float22bfloat162_rn(v); }
};
template <>
struct Store<__half2> {
  static __device__ __forceinline__ float2 ld(const __half2* p) { return __half22float2(*p); }
  static __device__ __forceinline__ void st(__half2* p, float2 v) { *p = __float22half2_rn(v); }
};

// ---------------------------------------------------------------------------
// propagation phase: H'_z(fy, fx) = exp(i 2 pi u), u = frac(z * cturns[fy, fx])
// computed in FP64 (product and reduction), then FP32 sincos on |2 pi u| <= pi.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 transfer(double z, double cturn, bool conj_) {
  double u = z * cturn;
  u -= rint(u);
  float s, c;
  __sincosf(6.28318530717958647692f * (float)u, &s, &c);
  return make_float2(c, conj_ ? -s : s);
}

// warp-level FP64 sum
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// the FISTA point x = P + beta (P - Pprev) of voxel i, as every kernel that
// reads the volume forms it
template <typename ST>
__device__ __forceinline__ float2 xval(const ST* P, const ST* Pp, float beta, size_t i) {
  const float2 p = Store<ST>::ld(P + i), pp = Store<ST>::ld(Pp + i);
  return make_float2(fmaf(beta, p.x - pp.x, p.x), fmaf(beta, p.y - pp.y, p.y));
}

}  // namespace rihvr
