// Paired FP32 complex arithmetic on sm_100's packed f32x2 pipe.
//
// A P2 holds one complex value of each of TWO pencils that undergo the same
// transform (two rows of a field), stored planar: re = (re_a, re_b),
// im = (im_a, im_b).  Every operation of a radix-R DFT then runs once for both
// pencils as one packed instruction (FADD2 / FMUL2 / FFMA2 from __fadd2_rn,
// __fmul2_rn, __ffma2_rn), which halves the FP32 instruction count of the
// butterflies; multiplying by +-i costs nothing because it only swaps which
// register pair is used, and real constants live in register pairs (c, c).
// Each lane rounds exactly as the scalar fmaf / fadd / fmul would.
#pragma once
#include <cuda_runtime.h>

#include "sc_twiddles.h"

namespace sc {

struct P2 {
  float2 re, im;
};

__device__ __forceinline__ float2 c2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as one packed FMA: b * (-1) is exact, so the result is the rounded difference
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ P2 padd(P2 a, P2 b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__device__ __forceinline__ P2 psub(P2 a, P2 b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }
__device__ __forceinline__ P2 pzero() { return {make_float2(0.f, 0.f), make_float2(0.f, 0.f)}; }

// Twiddle w = c + i s as register pairs C = (c, c), S = (s, s), NS = (-s, -s).
struct TwP {
  float2 C, S, NS;
};
// v * w (4 packed instructions)
__device__ __forceinline__ P2 pmul(P2 v, const TwP& w) {
  return {fma2(v.im, w.NS, mul2(v.re, w.C)), fma2(v.re, w.S, mul2(v.im, w.C))};
}
// v * conj(w)
__device__ __forceinline__ P2 pmulc(P2 v, const TwP& w) {
  return {fma2(v.im, w.S, mul2(v.re, w.C)), fma2(v.re, w.NS, mul2(v.im, w.C))};
}
// v * (c + i s) for compile-time constants
__device__ __forceinline__ P2 pmulk(P2 v, float c, float s) {
  return {fma2(v.im, c2(-s), mul2(v.re, c2(c))), fma2(v.re, c2(s), mul2(v.im, c2(c)))};
}

// ---------------------------------------------------------------------------
// radix-R DFTs.  Forward: X_k = sum_m x_m exp(-2 pi i m k / R); INV: exp(+...).
// ---------------------------------------------------------------------------
template <int R, bool INV> struct PDFT;

template <bool INV> struct PDFT<2, INV> {
  static __device__ __forceinline__ void run(P2* v) {
    const P2 a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
  }
};

// X1 = a - (b + c)/2 -+ i s3 (b - c), X2 = a - (b + c)/2 +- i s3 (b - c)
// (upper signs forward); -i d = (d.im, -d.re).
template <bool INV> struct PDFT<3, INV> {
  static __device__ __forceinline__ void run(P2* v) {
    const float s3 = INV ? -0.8660254037844386f : 0.8660254037844386f;
    const P2 a = v[0], b = v[1], c = v[2];
    const P2 t1 = padd(b, c), d = psub(b, c);
    const P2 t2 = {fma2(t1.re, c2(-0.5f), a.re), fma2(t1.im, c2(-0.5f), a.im)};
    v[0] = padd(a, t1);
    v[1] = {fma2(d.im, c2(s3), t2.re), fma2(d.re, c2(-s3), t2.im)};
    v[2] = {fma2(d.im, c2(-s3), t2.re), fma2(d.re, c2(s3), t2.im)};
  }
};

// Five-point DFT with the symmetric / antisymmetric split of the scalar
// engine: r_j = a + c_j (v1 + v4) + c_2j (v2 + v3),
// q_j = s_j (v1 - v4) + s_2j (v2 - v3); X_j = r_j -+ i q_j, X_{5-j} = r_j +- i q_j.
template <bool INV> struct PDFT<5, INV> {
  static __device__ __forceinline__ void run(P2* v) {
    const float c1 = 0.30901699437494745f, cc2 = -0.8090169943749475f;
    const float s1 = 0.9510565162951535f, s2 = 0.5877852522924731f;
    const P2 a = v[0];
    const P2 be = padd(v[1], v[4]), bm = psub(v[1], v[4]);
    const P2 cd = padd(v[2], v[3]), cm = psub(v[2], v[3]);
    const P2 r1 = {fma2(cd.re, c2(cc2), fma2(be.re, c2(c1), a.re)), fma2(cd.im, c2(cc2), fma2(be.im, c2(c1), a.im))};
    const P2 r2 = {fma2(cd.re, c2(c1), fma2(be.re, c2(cc2), a.re)), fma2(cd.im, c2(c1), fma2(be.im, c2(cc2), a.im))};
    const P2 q1 = {fma2(cm.re, c2(s2), mul2(bm.re, c2(s1))), fma2(cm.im, c2(s2), mul2(bm.im, c2(s1)))};
    const P2 q2 = {fma2(cm.re, c2(-s1), mul2(bm.re, c2(s2))), fma2(cm.im, c2(-s1), mul2(bm.im, c2(s2)))};
    v[0] = padd(a, padd(be, cd));
    if (!INV) {  // X_j = r_j - i q_j = (r.re + q.im, r.im - q.re)
      v[1] = {add2(r1.re, q1.im), sub2(r1.im, q1.re)};
      v[4] = {sub2(r1.re, q1.im), add2(r1.im, q1.re)};
      v[2] = {add2(r2.re, q2.im), sub2(r2.im, q2.re)};
      v[3] = {sub2(r2.re, q2.im), add2(r2.im, q2.re)};
    } else {
      v[1] = {sub2(r1.re, q1.im), add2(r1.im, q1.re)};
      v[4] = {add2(r1.re, q1.im), sub2(r1.im, q1.re)};
      v[2] = {sub2(r2.re, q2.im), add2(r2.im, q2.re)};
      v[3] = {add2(r2.re, q2.im), sub2(r2.im, q2.re)};
    }
  }
};

// 9 = 3 x 3 (Cooley-Tukey): input index 3 m1 + m2, output k1 + 3 k2,
// inner twiddles exp(-+2 pi i m2 k1 / 9).
template <bool INV> struct PDFT<9, INV> {
  static __device__ __forceinline__ void run(P2* v) {
    P2 y[9];
#pragma unroll
    for (int m2 = 0; m2 < 3; ++m2) {
      P2 t[3] = {v[m2], v[3 + m2], v[6 + m2]};
      PDFT<3, INV>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) {
        const int j = m2 * k1;
        if (j == 0) {
          y[m2 * 3 + k1] = t[k1];
        } else {
          const float wc = float(tw_cos(9, j));
          const float ws = INV ? float(tw_sin(9, j)) : float(-tw_sin(9, j));
          y[m2 * 3 + k1] = pmulk(t[k1], wc, ws);
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
      P2 t[3] = {y[k1], y[3 + k1], y[6 + k1]};
      PDFT<3, INV>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) v[k1 + 3 * k2] = t[k2];
    }
  }
};

// 10 = 2 x 5 (prime factor, no twiddles): input (5 n1 + 2 n2) mod 10,
// output (5 k1 + 6 k2) mod 10.
template <bool INV> struct PDFT<10, INV> {
  static __device__ __forceinline__ void run(P2* v) {
    P2 y[10];
#pragma unroll
    for (int n1 = 0; n1 < 2; ++n1) {
      P2 t[5];
#pragma unroll
      for (int n2 = 0; n2 < 5; ++n2) t[n2] = v[(5 * n1 + 2 * n2) % 10];
      PDFT<5, INV>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < 5; ++k2) y[n1 * 5 + k2] = t[k2];
    }
#pragma unroll
    for (int k2 = 0; k2 < 5; ++k2) {
      P2 s[2] = {y[k2], y[5 + k2]};
      PDFT<2, INV>::run(s);
#pragma unroll
      for (int k1 = 0; k1 < 2; ++k1) v[(5 * k1 + 6 * k2) % 10] = s[k1];
    }
  }
};

}  // namespace sc
