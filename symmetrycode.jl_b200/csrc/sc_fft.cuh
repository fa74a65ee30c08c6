// Mixed-radix (2, 3, 5) FFT engine for a tile of pencils held in shared memory.
//
// Every spectral transform of the solver (the cuFFT/FFTW `plan_rfft` calls of
// src/solver.jl:210-215,432-453 in the reference) is built from this engine: a
// CTA loads a tile of NPEN pencils of length N into shared memory, runs the
// passes of a Stockham autosort FFT with radices from {2..16} drawn from
// N = 2^a 3^b 5^c, and writes the tile back.  Each pass reads the R inputs of
// its butterflies into registers, applies the twiddles, computes the radix-R DFT
// in registers (composite radices by an in-register P x Q split), waits at a
// barrier and writes the R outputs in place, so one shared buffer suffices.
//
// Layout flags:
//   COL  -- element e of pencil p at s[e * NPEN + p]: pencils are the fastest
//           index; used by the strided y/z sweeps where NPEN consecutive kx
//           are loaded as one coalesced row.
//   !COL -- element e of pencil p at s[p * N + e]: used by the x sweep where a
//           pencil is one contiguous row.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sc {

// ---------------------------------------------------------------------------
// compact (2/3-rule) layout of a transform axis: kpos modes e < kpos kept in
// place, kneg modes e >= N - kneg moved down by N - kpos - kneg
// ---------------------------------------------------------------------------
// compact position of transform index f, -1 when f is not retained
__device__ __forceinline__ int cpos(int f, int N, int kpos, int kneg) {
  return f < kpos ? f : (f >= N - kneg ? f - N + kpos + kneg : -1);
}

// Where a block of B consecutive transform indices e0 .. e0 + B - 1 falls in
// the compact layout (kpos modes e < kpos kept in place, kneg modes
// e >= N - kneg moved down by N - kpos - kneg): 0 every index kept in place,
// 1 every index moved, 2 none kept, 3 the block straddles a boundary.
constexpr int crange(int e0, int B, int N, int kpos, int kneg) {
  return e0 + B - 1 < kpos ? 0 : (e0 >= N - kneg ? 1 : (e0 >= kpos && e0 + B - 1 < N - kneg ? 2 : 3));
}

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
template <typename R> struct V2;
template <> struct V2<float> { using T = float2; };
template <> struct V2<double> { using T = double2; };

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C c; c.x = a; c.y = b; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return mk<C>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_mi(C a) {
  return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}

// exact twiddle constants exp(2 pi i j / R) for the composite radices
// (correctly rounded doubles of cos/sin at these angles)
}  // namespace sc
#include "sc_twiddles.h"
namespace sc {

// ---------------------------------------------------------------------------
// radix-R DFTs in registers.  Forward: X_k = sum_m x_m exp(-2 pi i m k / R).
// ---------------------------------------------------------------------------
template <int R, bool INV, typename C> struct DFT;

template <bool INV, typename C> struct DFT<1, INV, C> {
  static __device__ __forceinline__ void run(C*) {}
};

template <bool INV, typename C> struct DFT<2, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV, typename C> struct DFT<3, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R s3 = R(0.8660254037844386);
    C a = v[0], b = v[1], c = v[2];
    C t1 = cadd(b, c);
    C t2 = mk<C>(a.x - R(0.5) * t1.x, a.y - R(0.5) * t1.y);
    C d = csub(b, c);
    C t3 = mul_mi<INV>(cscale(d, s3));  // -i s3 (b - c) forward
    v[0] = cadd(a, t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

template <bool INV, typename C> struct DFT<4, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1], c = v[2], d = v[3];
    C s0 = cadd(a, c), d0 = csub(a, c);
    C s1 = cadd(b, d), d1 = mul_mi<INV>(csub(b, d));
    v[0] = cadd(s0, s1);
    v[2] = csub(s0, s1);
    v[1] = cadd(d0, d1);
    v[3] = csub(d0, d1);
  }
};

template <bool INV, typename C> struct DFT<5, INV, C> {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R c1 = R(0.30901699437494745), c2 = R(-0.8090169943749475);
    const R s1 = R(0.9510565162951535), s2 = R(0.5877852522924731);
    C a = v[0];
    C be = cadd(v[1], v[4]), bm = csub(v[1], v[4]);
    C cd = cadd(v[2], v[3]), cm = csub(v[2], v[3]);
    C r1 = mk<C>(a.x + c1 * be.x + c2 * cd.x, a.y + c1 * be.y + c2 * cd.y);
    C r2 = mk<C>(a.x + c2 * be.x + c1 * cd.x, a.y + c2 * be.y + c1 * cd.y);
    C i1 = mul_mi<INV>(mk<C>(s1 * bm.x + s2 * cm.x, s1 * bm.y + s2 * cm.y));
    C i2 = mul_mi<INV>(mk<C>(s2 * bm.x - s1 * cm.x, s2 * bm.y - s1 * cm.y));
    v[0] = mk<C>(a.x + be.x + cd.x, a.y + be.y + cd.y);
    v[1] = cadd(r1, i1);
    v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2);
    v[3] = csub(r2, i2);
  }
};

// Composite radix R = P * Q: input index Q*m1 + m2, output index k1 + P*k2.
template <int P, int Q, bool INV, typename C> struct DFTPQ {
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    constexpr int RR = P * Q;
    C y[RR];
#pragma unroll
    for (int m2 = 0; m2 < Q; ++m2) {
      C t[P];
#pragma unroll
      for (int m1 = 0; m1 < P; ++m1) t[m1] = v[Q * m1 + m2];
      DFT<P, INV, C>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) {
        const int j = (m2 * k1) % RR;
        if (j == 0) {
          y[m2 * P + k1] = t[k1];
        } else {
          const R wc = R(tw_cos(RR, j));
          const R ws = INV ? R(tw_sin(RR, j)) : R(-tw_sin(RR, j));
          y[m2 * P + k1] = cmul(t[k1], mk<C>(wc, ws));
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      C t[Q];
#pragma unroll
      for (int m2 = 0; m2 < Q; ++m2) t[m2] = y[m2 * P + k1];
      DFT<Q, INV, C>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = t[k2];
    }
  }
};

// Prime-factor (Good-Thomas) composite for coprime P, Q: input index
// n = (Q n1 + P n2) mod N, output index k with k = k1 (mod P), k = k2 (mod Q);
// then X = DFT_P over n1 of DFT_Q over n2, with no twiddle factors.  Both index
// maps are compile-time, so in registers they cost nothing.
constexpr int sc_modinv(int a, int m) {
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return 1;
}
template <int P, int Q, bool INV, typename C> struct DFTPFA {
  static __device__ __forceinline__ void run(C* v) {
    constexpr int N = P * Q;
    constexpr int EP = Q * sc_modinv(Q % P, P);  // = 1 (mod P), 0 (mod Q)
    constexpr int EQ = P * sc_modinv(P % Q, Q);  // = 0 (mod P), 1 (mod Q)
    C y[N];
#pragma unroll
    for (int n1 = 0; n1 < P; ++n1) {
      C t[Q];
#pragma unroll
      for (int n2 = 0; n2 < Q; ++n2) t[n2] = v[(Q * n1 + P * n2) % N];
      DFT<Q, INV, C>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < Q; ++k2) y[n1 * Q + k2] = t[k2];
    }
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) {
      C s[P];
#pragma unroll
      for (int n1 = 0; n1 < P; ++n1) s[n1] = y[n1 * Q + k2];
      DFT<P, INV, C>::run(s);
#pragma unroll
      for (int k1 = 0; k1 < P; ++k1) v[(k1 * EP + k2 * EQ) % N] = s[k1];
    }
  }
};

template <bool INV, typename C> struct DFT<6, INV, C> : DFTPFA<2, 3, INV, C> {};
template <bool INV, typename C> struct DFT<8, INV, C> : DFTPQ<2, 4, INV, C> {};
template <bool INV, typename C> struct DFT<9, INV, C> : DFTPQ<3, 3, INV, C> {};
template <bool INV, typename C> struct DFT<10, INV, C> : DFTPFA<2, 5, INV, C> {};
template <bool INV, typename C> struct DFT<12, INV, C> : DFTPFA<4, 3, INV, C> {};
template <bool INV, typename C> struct DFT<15, INV, C> : DFTPFA<3, 5, INV, C> {};
template <bool INV, typename C> struct DFT<16, INV, C> : DFTPQ<4, 4, INV, C> {};
template <bool INV, typename C> struct DFT<18, INV, C> : DFTPFA<2, 9, INV, C> {};
template <bool INV, typename C> struct DFT<20, INV, C> : DFTPFA<4, 5, INV, C> {};
template <bool INV, typename C> struct DFT<24, INV, C> : DFTPFA<8, 3, INV, C> {};
template <bool INV, typename C> struct DFT<25, INV, C> : DFTPQ<5, 5, INV, C> {};
template <bool INV, typename C> struct DFT<27, INV, C> : DFTPQ<3, 9, INV, C> {};
template <bool INV, typename C> struct DFT<30, INV, C> : DFTPFA<3, 10, INV, C> {};
template <bool INV, typename C> struct DFT<32, INV, C> : DFTPQ<4, 8, INV, C> {};
template <bool INV, typename C> struct DFT<36, INV, C> : DFTPFA<4, 9, INV, C> {};
template <bool INV, typename C> struct DFT<40, INV, C> : DFTPFA<8, 5, INV, C> {};
template <bool INV, typename C> struct DFT<45, INV, C> : DFTPFA<5, 9, INV, C> {};

// ---------------------------------------------------------------------------
// radix schedule for N = 2^a 3^b 5^c (compile time)
// ---------------------------------------------------------------------------
struct RadixPlan {
  int np;
  int r[10];
};

__host__ __device__ constexpr RadixPlan make_radix_plan(int N) {
  RadixPlan p{0, {1, 1, 1, 1, 1, 1, 1, 1, 1, 1}};
  int a = 0, b = 0, c = 0, m = N;
  while (m % 2 == 0) { ++a; m /= 2; }
  while (m % 3 == 0) { ++b; m /= 3; }
  while (m % 5 == 0) { ++c; m /= 5; }
  if (m != 1) { p.np = -1; return p; }
  while (c > 0) {
    if (a > 0) { p.r[p.np++] = 10; --a; --c; }
    else if (b > 0) { p.r[p.np++] = 15; --b; --c; }
    else { p.r[p.np++] = 5; --c; }
  }
  while (b >= 2) { p.r[p.np++] = 9; b -= 2; }
  while (a >= 4) { p.r[p.np++] = 16; a -= 4; }
  if (b == 1) {
    if (a >= 2) { p.r[p.np++] = 12; a -= 2; }
    else if (a == 1) { p.r[p.np++] = 6; a -= 1; }
    else { p.r[p.np++] = 3; }
  }
  if (a == 3) p.r[p.np++] = 8;
  else if (a == 2) p.r[p.np++] = 4;
  else if (a == 1) p.r[p.np++] = 2;
  return p;
}

__host__ __device__ constexpr int radix_at(int N, int pass) { return make_radix_plan(N).r[pass]; }
__host__ __device__ constexpr int num_passes(int N) { return make_radix_plan(N).np; }
__host__ __device__ constexpr int stride_before(int N, int pass) {
  int s = 1;
  for (int i = 0; i < pass; ++i) s *= make_radix_plan(N).r[i];
  return s;
}
__host__ __device__ constexpr int min_radix(int N) {
  int m = 1 << 30;
  for (int i = 0; i < make_radix_plan(N).np; ++i)
    m = make_radix_plan(N).r[i] < m ? make_radix_plan(N).r[i] : m;
  return m;
}

// ---------------------------------------------------------------------------
// shared-memory tile FFT
// ---------------------------------------------------------------------------
template <bool COL, int NPEN, int N>
__device__ __forceinline__ int tidx(int p, int e) {
  return COL ? e * NPEN + p : p * N + e;
}

// One Stockham pass of radix radix_at(N, PASS) over NPEN pencils with NT threads.
// `tw` holds exp(-2 pi i m / N), m = 0..N-1.
template <typename C, int N, int NPEN, int NT, bool INV, bool COL, int PASS>
__device__ __forceinline__ void fft_pass(C* __restrict__ s, const C* __restrict__ tw) {
  constexpr int RR = radix_at(N, PASS);
  constexpr int NS = stride_before(N, PASS);
  constexpr int NB = N / RR;
  constexpr int TOT = NPEN * NB;
  constexpr int M = (TOT + NT - 1) / NT;
  constexpr int TWS = N / (NS * RR);
  C v[M][RR];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int q = threadIdx.x + m * NT;
    if ((TOT % NT == 0) || q < TOT) {
      const int p = COL ? q % NPEN : q / NB;
      const int b = COL ? q / NPEN : q % NB;
#pragma unroll
      for (int r = 0; r < RR; ++r) v[m][r] = s[tidx<COL, NPEN, N>(p, b + r * NB)];
      if (NS > 1) {
        const int k = b % NS;
#pragma unroll
        for (int r = 1; r < RR; ++r) {
          C w = __ldg(&tw[k * r * TWS]);
          if (INV) w.y = -w.y;
          v[m][r] = cmul(v[m][r], w);
        }
      }
      DFT<RR, INV, C>::run(v[m]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int q = threadIdx.x + m * NT;
    if ((TOT % NT == 0) || q < TOT) {
      const int p = COL ? q % NPEN : q / NB;
      const int b = COL ? q / NPEN : q % NB;
      const int k = b % NS;
      const int base = (b / NS) * NS * RR + k;
#pragma unroll
      for (int r = 0; r < RR; ++r) s[tidx<COL, NPEN, N>(p, base + r * NS)] = v[m][r];
    }
  }
  __syncthreads();
}

template <typename C, int N, int NPEN, int NT, bool INV, bool COL, int PASS>
struct FFTPasses {
  static __device__ __forceinline__ void run(C* s, const C* tw) {
    fft_pass<C, N, NPEN, NT, INV, COL, PASS>(s, tw);
    FFTPasses<C, N, NPEN, NT, INV, COL, PASS + 1>::run(s, tw);
  }
};
template <typename C, int N, int NPEN, int NT, bool INV, bool COL>
struct FFTPasses<C, N, NPEN, NT, INV, COL, 10> {
  static __device__ __forceinline__ void run(C*, const C*) {}
};

// Full transform of the tile; the caller must __syncthreads() after filling s.
template <typename C, int N, int NPEN, int NT, bool INV, bool COL>
__device__ __forceinline__ void tile_fft(C* s, const C* tw) {
  static_assert(num_passes(N) > 0, "N must be 2^a 3^b 5^c");
  if constexpr (num_passes(N) >= 1) fft_pass<C, N, NPEN, NT, INV, COL, 0>(s, tw);
  if constexpr (num_passes(N) >= 2) fft_pass<C, N, NPEN, NT, INV, COL, 1>(s, tw);
  if constexpr (num_passes(N) >= 3) fft_pass<C, N, NPEN, NT, INV, COL, 2>(s, tw);
  if constexpr (num_passes(N) >= 4) fft_pass<C, N, NPEN, NT, INV, COL, 3>(s, tw);
  if constexpr (num_passes(N) >= 5) fft_pass<C, N, NPEN, NT, INV, COL, 4>(s, tw);
  if constexpr (num_passes(N) >= 6) fft_pass<C, N, NPEN, NT, INV, COL, 5>(s, tw);
}

}  // namespace sc
