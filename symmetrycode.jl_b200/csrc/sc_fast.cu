// Two-level register FFT sweeps for the FP32 solver sizes (sm_100a).
//
// A length-N transform is split N = N1 * N2 (810 = 27 * 30, 256 = 16 * 16,
// 128 = 16 * 8, 64 = 8 * 8):
//   step 1  thread (pencil, n2) gathers x[N2 n1 + n2], n1 = 0..N1-1, straight
//           from global memory into registers, runs a radix-N1 DFT in
//           registers, multiplies by exp(-+2 pi i n2 k1 / N) and writes one
//           row of the shared exchange buffer;
//   step 2  thread (pencil, k1) reads the N2 values of its column, runs a
//           radix-N2 DFT in registers and stores X[k1 + N1 k2] straight to
//           global memory (pruned to the retained modes on the forward side).
// Each element crosses shared memory once (one store, one load) instead of
// once per radix pass, and every thread keeps N1 independent global loads in
// flight.  These kernels replace the Stockham-engine sweeps of sc_kernels.cu
// for FP32 at the sizes of the DNS and LES configurations; the results are the
// same transforms (tests compare both against the FP64 oracle).
#include "sc_fft.cuh"
#include "sc_internal.h"

namespace sc {

// N = N1 * N2 of the two-level column sweeps; S = 1 is the transposed split,
// one of the autotuner's candidates (the x sweeps use S = 0).
template <int N, int S = 0> struct Split;
template <> struct Split<810, 0> { static constexpr int N1 = 27, N2 = 30; };
template <> struct Split<810, 1> { static constexpr int N1 = 30, N2 = 27; };
template <> struct Split<256, 0> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Split<256, 1> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Split<128, 0> { static constexpr int N1 = 16, N2 = 8; };
template <> struct Split<128, 1> { static constexpr int N1 = 8, N2 = 16; };
template <> struct Split<64, 0> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<64, 1> { static constexpr int N1 = 8, N2 = 8; };

// ---------------------------------------------------------------------------
// column sweeps: tile of T consecutive kx, one column c, all N elements
// ---------------------------------------------------------------------------
template <int N, int T, int S = 0> struct Col2Cfg {
  static constexpr int N1 = Split<N, S>::N1, N2 = Split<N, S>::N2;
  static constexpr int NJ = N1 > N2 ? N1 : N2;
  static constexpr int NT = T * NJ;
  static constexpr int SR = N2 * T + 8;  // exchange row stride (+8: half-bank shift between rows)
  static constexpr size_t SMEM = size_t(N1) * SR * sizeof(float2);
  // at 810 the tile of 8 columns keeps 80 registers and three CTAs per SM
  static constexpr int MINB = N == 810 ? (T == 4 ? 6 : (T == 8 ? 3 : 1)) : 1;
};

// DRV: the launch carries derivative outputs (ColArgs::ndrv > 0).  Without it
// the wavenumber scaling is compiled out; otherwise the compiler hoists the
// int -> double -> float conversions of every element out of the `drv` branch
// and pays for them on the XU pipe even for plain components.
// FULL: the transform axis has the 2/3-rule compact layout of the solver
// (kpos = N/3 + 1, kneg = N/3), so which of each thread's N1 gathers (inverse)
// or N2 stores (forward) touch a retained mode is known at compile time except
// in the one block that straddles a boundary; the unused forward outputs are
// then never formed.
template <int N, int T, bool INV, bool DRV, bool FULL, int S = 0>
__global__ void __launch_bounds__(Col2Cfg<N, T, S>::NT, Col2Cfg<N, T, S>::MINB)
k_col2(const ColArgs a, const float2* __restrict__ tw) {
  using C = float2;
  using Cfg = Col2Cfg<N, T, S>;
  constexpr int N1 = Cfg::N1, N2 = Cfg::N2, SR = Cfg::SR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* ys = reinterpret_cast<C*>(smem_raw);
  const int t = threadIdx.x % T, j = threadIdx.x / T;
  const int kx = blockIdx.x * T + t;
  const int c = blockIdx.y;
  const int q = blockIdx.z;
  const bool drv = DRV && q >= a.ncomp;
  const C* __restrict__ in = static_cast<const C*>(a.in[drv ? a.drv_src[q - a.ncomp] : q]);
  C* __restrict__ out = static_cast<C*>(a.out[q]);
  const bool live = kx < a.K1;
  constexpr int KP = N / 3 + 1, KN = N / 3;
  const int kpos = FULL ? KP : a.kpos, kneg = FULL ? KN : a.kneg;
  const int Kc = kpos + kneg;
  // element offsets fit in 32 bits for every sweep (at most ~3.5e8 elements
  // per component), so the per-element address arithmetic stays 32-bit
  const int ies = int(a.in_es), oes = int(a.out_es);
  if (j < N2) {
    C v[N1];
    const C* base = in + kx + (long long)c * a.in_cs;
    if (INV) {
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const int e = N2 * n1 + j;
        v[n1] = mk<C>(0.f, 0.f);
        const int rg = FULL ? crange(N2 * n1, N2, N, KP, KN) : 3;
        if (rg == 2) continue;
        const int p = rg == 0 ? e : (rg == 1 ? e - N + Kc : cpos(e, N, kpos, kneg));
        if (live && p >= 0 && !(a.zero_origin && kx == 0 && c == 0 && p == 0)) {
          v[n1] = __ldg(base + p * ies);
          if (drv) {
            const float kk = float(a.kfac * double(p < kpos ? p : p - Kc));
            v[n1] = mk<C>(-kk * v[n1].y, kk * v[n1].x);
          }
        }
      }
    } else {
      const C* bj = base + j * ies;
      const int st = N2 * ies;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[n1] = live ? __ldg(bj + n1 * st) : mk<C>(0.f, 0.f);
    }
    DFT<N1, INV, C>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
      C w = __ldg(&tw[j * k1]);
      if (INV) w.y = -w.y;
      v[k1] = cmul(v[k1], w);
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) ys[k1 * SR + j * T + t] = v[k1];
  }
  __syncthreads();
  if (j < N1 && live) {
    C w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = ys[j * SR + n2 * T + t];
    DFT<N2, INV, C>::run(w);
    C* obase = out + kx + (long long)c * a.out_cs;
    if (INV) {
      C* oj = obase + j * oes;
      const int st = N1 * oes;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) oj[k2 * st] = w[k2];
    } else {
      // retained e = j + N1 k2: e < kpos keeps its index, e >= N - kneg moves down by N - Kc
      const int shift = N - Kc;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int e = j + N1 * k2;
        const int rg = FULL ? crange(N1 * k2, N1, N, KP, KN) : 3;
        if (rg == 0) obase[e * oes] = w[k2];
        else if (rg == 1) obase[(e - shift) * oes] = w[k2];
        else if (rg == 3) {
          if (e < kpos) obase[e * oes] = w[k2];
          else if (e >= N - kneg) obase[(e - shift) * oes] = w[k2];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16_cg(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// x sweep with the Navier-Stokes products (rows are contiguous)
// ---------------------------------------------------------------------------
template <int N> struct X2Rows;
template <> struct X2Rows<810> { static constexpr int TR = 2; };
template <> struct X2Rows<256> { static constexpr int TR = 4; };
template <> struct X2Rows<128> { static constexpr int TR = 8; };
template <> struct X2Rows<64> { static constexpr int TR = 16; };

template <int N, int D> struct X2Cfg {
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, N2P = N2 + 1;
  static constexpr int TR = X2Rows<N>::TR;
  static constexpr int K1M = N / 3 + 1;           // widest input row (2/3-truncated spectrum)
  static constexpr int NPI = D == 3 ? 2 * TR : TR;   // inverse pencils
  static constexpr int NPF = D == 3 ? 3 * TR : 2 * TR;  // forward pencils
  static constexpr int NT = 192;
  static constexpr size_t RIN = size_t(D) * TR * K1M * sizeof(float2);
  static constexpr size_t UPH = size_t(D) * TR * N * sizeof(float);
  static constexpr size_t ZB = size_t(NPF) * (2 * K1M - 1) * sizeof(float2);
  static constexpr size_t A0 = (RIN + UPH) > ZB ? (RIN + UPH) : ZB;  // Rin+U, later aliased by Z
  static constexpr size_t YB = size_t(NPF) * N1 * N2P * sizeof(float2);
  static constexpr size_t SMEM = A0 + YB;
};

template <int N> __device__ __forceinline__ float2 hext2(const float2* row, int K1, int f) {
  const int kmax = K1 - 1;
  if (f == 0) return make_float2(row[0].x, 0.f);
  if (f <= kmax) return row[f];
  if (f >= N - kmax) { const float2 v = row[N - f]; return make_float2(v.x, -v.y); }
  return make_float2(0.f, 0.f);
}

template <int N, int D>
__global__ void __launch_bounds__(X2Cfg<N, D>::NT)
k_xsweep2(const XArgs a, const float2* __restrict__ tw) {
  using C = float2;
  using Cfg = X2Cfg<N, D>;
  constexpr int N1 = Cfg::N1, N2 = Cfg::N2, N2P = Cfg::N2P, TR = Cfg::TR, K1M = Cfg::K1M;
  constexpr int NPI = Cfg::NPI, NPF = Cfg::NPF, NT = Cfg::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* rin = reinterpret_cast<C*>(smem_raw);                        // [D][TR][K1M]
  float* uph = reinterpret_cast<float*>(smem_raw + Cfg::RIN);     // [D][TR][N]
  C* zb = reinterpret_cast<C*>(smem_raw);                         // [NPF][2*K1M-1] (after F1)
  C* yb = reinterpret_cast<C*>(smem_raw + Cfg::A0);               // [NPF][N1][N2P]
  const long long row0 = (long long)blockIdx.x * TR;
  const int K1 = a.K1in;
  const int ko = a.K1out - 1;
  constexpr int ZS = 2 * K1M - 1;

  // L: stage the TR spectral rows of each component (contiguous in global memory)
  {
    constexpr int TOT = D * TR * K1M;
    constexpr int LPT = (TOT + NT - 1) / NT;
    // select the component pointer instead of indexing the parameter array at run time
    const C* in0 = static_cast<const C*>(a.in[0]);
    const C* in1 = static_cast<const C*>(a.in[1]);
    const C* in2 = static_cast<const C*>(a.in[D == 3 ? 2 : 1]);
    C v[LPT];
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      v[i] = make_float2(0.f, 0.f);
      const int cmp = idx / (TR * K1M), r = (idx / K1M) % TR, kx = idx % K1M;
      if (idx < TOT && kx < K1 && row0 + r < a.nrows)
        v[i] = __ldg((cmp == 0 ? in0 : cmp == 1 ? in1 : in2) + (row0 + r) * K1 + kx);
    }
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      if (idx < TOT) rin[idx] = v[i];
    }
  }
  __syncthreads();

  // I1: inverse step 1 (pencil p: row p % TR; kind 0: u1 + i u2, kind 1: u3)
  for (int it = threadIdx.x; it < NPI * N2; it += NT) {
    const int p = it / N2, j = it % N2;
    const int r = p % TR, kind = p / TR;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int f = N2 * n1 + j;
      if (kind == 0) {
        const C x1 = hext2<N>(rin + (0 * TR + r) * K1M, K1, f);
        const C x2 = hext2<N>(rin + (1 * TR + r) * K1M, K1, f);
        v[n1] = make_float2(x1.x - x2.y, x1.y + x2.x);
      } else {
        v[n1] = hext2<N>(rin + (2 * TR + r) * K1M, K1, f);
      }
    }
    DFT<N1, true, C>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
      const C w = __ldg(&tw[j * k1]);
      v[k1] = cmul(v[k1], make_float2(w.x, -w.y));
    }
    C* yp = yb + p * N1 * N2P;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
  }
  __syncthreads();

  // I2: inverse step 2 -> physical velocities at x = i + N1 k2
  for (int it = threadIdx.x; it < NPI * N1; it += NT) {
    const int p = it / N1, i = it % N1;
    const int r = p % TR, kind = p / TR;
    C w[N2];
    const C* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
    DFT<N2, true, C>::run(w);
    if (kind == 0) {
      float* u1 = uph + (0 * TR + r) * N;
      float* u2 = uph + (1 * TR + r) * N;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) { u1[i + N1 * k2] = w[k2].x; u2[i + N1 * k2] = w[k2].y; }
    } else {
      float* u3 = uph + (2 * TR + r) * N;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) u3[i + N1 * k2] = w[k2].x;
    }
  }
  __syncthreads();

  // F1: products (scaled) and forward step 1
  const float sc = float(a.scale);
  for (int it = threadIdx.x; it < NPF * N2; it += NT) {
    const int p = it / N2, j = it % N2;
    const int r = p % TR, kind = p / TR;
    const float* u1 = uph + (0 * TR + r) * N;
    const float* u2 = uph + (1 * TR + r) * N;
    const float* u3 = uph + ((D == 3 ? 2 : 0) * TR + r) * N;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int x = N2 * n1 + j;
      const float a1 = u1[x], a2 = u2[x];
      if (D == 3) {
        const float a3 = u3[x];
        v[n1] = kind == 0 ? make_float2(a1 * a1 * sc, a2 * a2 * sc)
              : kind == 1 ? make_float2(a3 * a3 * sc, a1 * a2 * sc)
                          : make_float2(a2 * a3 * sc, a3 * a1 * sc);
      } else {
        v[n1] = kind == 0 ? make_float2(a1 * a1 * sc, a2 * a2 * sc) : make_float2(a1 * a2 * sc, 0.f);
      }
    }
    DFT<N1, false, C>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], __ldg(&tw[j * k1]));
    C* yp = yb + p * N1 * N2P;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
  }
  __syncthreads();

  // F2: forward step 2, keep X[k] for k <= ko and k >= N - ko
  for (int it = threadIdx.x; it < NPF * N1; it += NT) {
    const int p = it / N1, i = it % N1;
    C w[N2];
    const C* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
    DFT<N2, false, C>::run(w);
    C* zp = zb + p * ZS;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int k = i + N1 * k2;
      if (k <= ko) zp[k] = w[k2];
      else if (k >= N - ko) zp[ko + (N - k)] = w[k2];
    }
  }
  __syncthreads();

  // S: split the paired spectra and store the product rows
  constexpr int NBF = NPF / TR;
  const int K1o = a.K1out;
  const long long ldo = a.ldo > 0 ? a.ldo : K1o;
  for (int it = threadIdx.x; it < TR * K1o; it += NT) {
    const int r = it / K1o, kx = it % K1o;
    const long long row = row0 + r;
    if (row >= a.nrows) continue;
#pragma unroll
    for (int b = 0; b < NBF; ++b) {
      const C* zp = zb + (b * TR + r) * ZS;
      const C z = zp[kx], zc = zp[kx == 0 ? 0 : ko + kx];
      const C xa = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
      const C xbv = make_float2(0.5f * (z.y + zc.y), 0.5f * (zc.x - z.x));
      static_cast<C*>(a.out[2 * b])[row * ldo + kx] = xa;
      if (2 * b + 1 < (D == 3 ? 6 : 3)) static_cast<C*>(a.out[2 * b + 1])[row * ldo + kx] = xbv;
    }
  }
}

// ---------------------------------------------------------------------------
// 3D x sweep, rows paired: u3 of rows 2q and 2q+1 share one inverse transform
// (1.5 inverse transforms per row instead of 2) and the forward side runs in
// two halves of TR/2 rows so that every phase keeps ~90 % of the threads busy.
// ---------------------------------------------------------------------------
template <int N> struct X3Rows;
template <> struct X3Rows<810> { static constexpr int TR = 4; };
template <> struct X3Rows<256> { static constexpr int TR = 8; };
template <> struct X3Rows<128> { static constexpr int TR = 16; };
template <> struct X3Rows<64> { static constexpr int TR = 32; };

template <int N> struct X3Cfg {
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, N2P = N2 + 1;
  static constexpr int TR = X3Rows<N>::TR, TH = TR / 2;
  static constexpr int K1M = N / 3 + 1;
  static constexpr int NPI = TR + TH;   // inverse pencils: u1 + i u2 per row, u3 pairs
  static constexpr int NPF = 3 * TH;    // forward pencils of one half
  static constexpr int NT = 192;
  static constexpr size_t RIN = size_t(3) * TR * K1M * sizeof(float2);
  static constexpr size_t ZB = size_t(NPF) * (2 * K1M - 1) * sizeof(float2);
  static constexpr size_t A0 = RIN > ZB ? RIN : ZB;  // Rin, later Z of each half
  static constexpr size_t UPH = size_t(3) * TR * N * sizeof(float);
  static constexpr int NPY = NPI > NPF ? NPI : NPF;
  static constexpr size_t YB = size_t(NPY) * N1 * N2P * sizeof(float2);
  static constexpr size_t SMEM = A0 + UPH + YB;
};

template <int N>
__global__ void __launch_bounds__(X3Cfg<N>::NT)
k_xsweep3(const XArgs a, const float2* __restrict__ tw) {
  using C = float2;
  using Cfg = X3Cfg<N>;
  constexpr int N1 = Cfg::N1, N2 = Cfg::N2, N2P = Cfg::N2P, TR = Cfg::TR, TH = Cfg::TH, K1M = Cfg::K1M;
  constexpr int NPI = Cfg::NPI, NPF = Cfg::NPF, NT = Cfg::NT;
  constexpr int ZS = 2 * K1M - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* rin = reinterpret_cast<C*>(smem_raw);                         // [3][TR][K1M]
  C* zb = reinterpret_cast<C*>(smem_raw);                          // [NPF][ZS] after I1
  float* uph = reinterpret_cast<float*>(smem_raw + Cfg::A0);       // [3][TR][N]
  C* yb = reinterpret_cast<C*>(smem_raw + Cfg::A0 + Cfg::UPH);     // [NPY][N1][N2P]
  const long long row0 = (long long)blockIdx.x * TR;
  const int K1 = a.K1in;
  const int ko = a.K1out - 1;
  {
    constexpr int TOT = 3 * TR * K1M;
    constexpr int LPT = (TOT + NT - 1) / NT;
    // select the component pointer instead of indexing the parameter array at run time
    const C* in0 = static_cast<const C*>(a.in[0]);
    const C* in1 = static_cast<const C*>(a.in[1]);
    const C* in2 = static_cast<const C*>(a.in[2]);
    C v[LPT];
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      v[i] = make_float2(0.f, 0.f);
      const int cmp = idx / (TR * K1M), r = (idx / K1M) % TR, kx = idx % K1M;
      if (idx < TOT && kx < K1 && row0 + r < a.nrows)
        v[i] = __ldg((cmp == 0 ? in0 : cmp == 1 ? in1 : in2) + (row0 + r) * K1 + kx);
    }
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      if (idx < TOT) rin[idx] = v[i];
    }
  }
  __syncthreads();
  // I1: pencils p < TR: u1 + i u2 of row p; p >= TR: u3(row 2q) + i u3(row 2q+1), q = p - TR
  for (int it = threadIdx.x; it < NPI * N2; it += NT) {
    const int p = it / N2, j = it % N2;
    const C* ra;
    const C* rb;
    if (p < TR) { ra = rin + (0 * TR + p) * K1M; rb = rin + (1 * TR + p) * K1M; }
    else { const int q = p - TR; ra = rin + (2 * TR + 2 * q) * K1M; rb = rin + (2 * TR + 2 * q + 1) * K1M; }
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int f = N2 * n1 + j;
      const C x1 = hext2<N>(ra, K1, f), x2 = hext2<N>(rb, K1, f);
      v[n1] = make_float2(x1.x - x2.y, x1.y + x2.x);
    }
    DFT<N1, true, C>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
      const C w = __ldg(&tw[j * k1]);
      v[k1] = cmul(v[k1], make_float2(w.x, -w.y));
    }
    C* yp = yb + p * N1 * N2P;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
  }
  __syncthreads();
  // I2: physical velocities
  for (int it = threadIdx.x; it < NPI * N1; it += NT) {
    const int p = it / N1, i = it % N1;
    C w[N2];
    const C* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
    DFT<N2, true, C>::run(w);
    float* oa;
    float* ob;
    if (p < TR) { oa = uph + (0 * TR + p) * N; ob = uph + (1 * TR + p) * N; }
    else { const int q = p - TR; oa = uph + (2 * TR + 2 * q) * N; ob = uph + (2 * TR + 2 * q + 1) * N; }
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) { oa[i + N1 * k2] = w[k2].x; ob[i + N1 * k2] = w[k2].y; }
  }
  __syncthreads();
  const float sc = float(a.scale);
  const int K1o = a.K1out;
  const long long ldo = a.ldo > 0 ? a.ldo : K1o;
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    // F1: products of the half's rows, forward step 1 (pencil p: row half*TH + p % TH, kind p / TH)
    for (int it = threadIdx.x; it < NPF * N2; it += NT) {
      const int p = it / N2, j = it % N2;
      const int r = half * TH + p % TH, kind = p / TH;
      const float* u1 = uph + (0 * TR + r) * N;
      const float* u2 = uph + (1 * TR + r) * N;
      const float* u3 = uph + (2 * TR + r) * N;
      C v[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const int x = N2 * n1 + j;
        const float a1 = u1[x], a2 = u2[x], a3 = u3[x];
        v[n1] = kind == 0 ? make_float2(a1 * a1 * sc, a2 * a2 * sc)
              : kind == 1 ? make_float2(a3 * a3 * sc, a1 * a2 * sc)
                          : make_float2(a2 * a3 * sc, a3 * a1 * sc);
      }
      DFT<N1, false, C>::run(v);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], __ldg(&tw[j * k1]));
      C* yp = yb + p * N1 * N2P;
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
    }
    __syncthreads();
    // F2: forward step 2 into Z (the staged input rows are no longer needed)
    for (int it = threadIdx.x; it < NPF * N1; it += NT) {
      const int p = it / N1, i = it % N1;
      C w[N2];
      const C* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
      DFT<N2, false, C>::run(w);
      C* zp = zb + p * ZS;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int k = i + N1 * k2;
        if (k <= ko) zp[k] = w[k2];
        else if (k >= N - ko) zp[ko + (N - k)] = w[k2];
      }
    }
    __syncthreads();
    // S: split and store the half's product rows
    for (int it = threadIdx.x; it < TH * K1o; it += NT) {
      const int rr = it / K1o, kx = it % K1o;
      const long long row = row0 + half * TH + rr;
      if (row >= a.nrows) continue;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const C* zp = zb + (b * TH + rr) * ZS;
        const C z = zp[kx], zc = zp[kx == 0 ? 0 : ko + kx];
        static_cast<C*>(a.out[2 * b])[row * ldo + kx] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
        static_cast<C*>(a.out[2 * b + 1])[row * ldo + kx] = make_float2(0.5f * (z.y + zc.y), 0.5f * (zc.x - z.x));
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// 3D x sweep for N = 810 = 9 * 9 * 10, one row pair per 96-thread block.
//
// Inverse (c2r of the Hermitian-extended rows, k = 9 m1 + m2):
//   Ia  thread t = 9 q + m2 (81): radix-10 over p of Z[81 p + t] (straight
//       from global memory), twiddle exp(+2 pi i q s_a / 90)         -> X
//   Ib  thread 9 s_a + m2 (90): radix-9 over q, twiddle exp(+2 pi i m2 s1 / 810),
//       s1 = s_a + 10 s_b                                            -> Y
//   Ic  thread s1 (90): radix-9 over m2 -> physical x = s1 + 90 s2 in registers.
// Forward (x = 90 m1 + m2, k = s1' + 9 s_a + 81 s_b):
//   F1  the same thread (m2 = s1) forms the products at its 9 points and runs
//       the first radix-9 over m1 in registers, twiddle exp(-2 pi i m2 s1' / 810)
//                                                                     -> W
//   F2  thread 10 s1' + q (90): radix-9 over p (m2 = 10 p + q), twiddle
//       exp(-2 pi i q s_a / 90)                                       -> V
//   F3  thread 9 s1' + s_a (81): radix-10 over q, retained k only      -> Z
//   S   split the paired spectra and store the six product rows.
// Because the last inverse pass leaves every thread holding exactly the points
// its first forward pass needs, the products never go through shared memory.
// Pencils: A = u1 + i u2 (row r), A' = u1 + i u2 (row r'), B = u3(r) + i u3(r');
// forward pencils per row: (u1 u1, u2 u2), (u3 u3, u1 u2), (u2 u3, u3 u1).
// Shared memory: two regions of three pencil slots; the layouts below keep
// every exchange free of bank conflicts except the F3 loads, which meet two
// addresses on one or two bank pairs per half-warp (no linear placement of the
// F2 -> F3 exchange does better without making the F2 stores conflict).
// ---------------------------------------------------------------------------
struct X4Cfg {
  static constexpr int N = 810, NT = 96;
  static constexpr int PS = 882;  // pencil slot (X uses 89 s_a + 9 q + m2 < 882)
  static constexpr size_t SMEM = size_t(6) * PS * sizeof(float2);
};

// Z[k] = Ua[k] + i Ub[k], k = 81 p + t, of two real rows given by their staged
// half spectra (ra, rb: kmax + 1 modes).  FULL: kmax = 270, so the range of k
// for each p is known and 324 <= k <= 485 (p = 4, 5) never holds a mode.
template <bool FULL>
__device__ __forceinline__ float2 x4_gather(const float2* ra, const float2* rb, int p, int t, int kmax) {
  constexpr int N = 810;
  const int k = 81 * p + t;
  bool direct, mirror;
  if (FULL) {
    direct = p <= 2 || (p == 3 && t <= 27);
    mirror = p >= 7 || (p == 6 && t >= 54);
  } else {
    direct = k <= kmax;
    mirror = k >= N - kmax;
  }
  if (direct) {
    float2 x = ra[k], y = rb[k];
    if (k == 0) { x.y = 0.f; y.y = 0.f; }  // a real row's mean: imaginary part dropped
    return make_float2(x.x - y.y, x.y + y.x);
  }
  if (mirror) {
    const float2 x = ra[N - k], y = rb[N - k];
    return make_float2(x.x + y.y, y.x - x.y);
  }
  return make_float2(0.f, 0.f);
}

// products of one row at this thread's 9 points, first forward radix-9, twiddle.
// KIND selects the pencil at compile time (0: u1 u1 + i u2 u2, 1: u3 u3 + i u1 u2,
// 2: u2 u3 + i u3 u1), so each point costs two multiplies and no selects.
template <int KIND>
__device__ __forceinline__ void x4_f1_kind(const float* u1, const float* u2, const float* u3,
                                           const float2* wf, float2* region, int t) {
  using C = float2;
  C v[9];
#pragma unroll
  for (int m1 = 0; m1 < 9; ++m1) {
    const float a1 = u1[m1], a2 = u2[m1], a3 = u3[m1];
    const float pa = KIND == 0 ? a1 * a1 : KIND == 1 ? a3 * a3 : a2 * a3;
    const float pb = KIND == 0 ? a2 * a2 : KIND == 1 ? a1 * a2 : a3 * a1;
    v[m1] = make_float2(pa, pb);
  }
  DFT<9, false, C>::run(v);
  C* ws = region + KIND * X4Cfg::PS + t;
  ws[0] = v[0];
#pragma unroll
  for (int s = 1; s < 9; ++s) ws[90 * s] = cmul(v[s], wf[s]);
}
__device__ __forceinline__ void x4_f1_row(const float* u1, const float* u2, const float* u3,
                                          const float2* wf, float2* region, int t) {
  x4_f1_kind<0>(u1, u2, u3, wf, region, t);
  x4_f1_kind<1>(u1, u2, u3, wf, region, t);
  x4_f1_kind<2>(u1, u2, u3, wf, region, t);
}

template <bool FULL>
__global__ void __launch_bounds__(X4Cfg::NT, 5)
k_xsweep4(const XArgs a, const float2* __restrict__ tw) {
  using C = float2;
  constexpr int N = 810, PS = X4Cfg::PS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  C* reg0 = sm;           // slots 0..2
  C* reg1 = sm + 3 * PS;  // slots 3..5
  const int t = threadIdx.x;
  const long long r0 = (long long)blockIdx.x * 2;
  const bool has1 = r0 + 1 < a.nrows;
  const int K1 = FULL ? 271 : a.K1in, kmax = K1 - 1;
  const int K1o = FULL ? 271 : a.K1out, ko = K1o - 1;
  const int ldo = a.ldo > 0 ? a.ldo : K1o;

  // L: stage the six input rows (u1, u2, u3 of rows r, r') in region 1 with one
  // round of asynchronous copies; region 1 is not written before Ib.
  C* rin = reg1;  // [3][2][K1]
  {
    const C* in0 = static_cast<const C*>(a.in[0]);
    const C* in1 = static_cast<const C*>(a.in[1]);
    const C* in2 = static_cast<const C*>(a.in[2]);
    // FULL with both rows present: rows r0 (even) and r0 + 1 of a component are
    // 2 x 271 contiguous elements starting 4336 r0/2 bytes into the component,
    // so with 16-byte aligned components each row pair is 271 16-byte copies
    const bool pair16 =
        FULL && has1 &&
        ((reinterpret_cast<unsigned long long>(in0) | reinterpret_cast<unsigned long long>(in1) |
          reinterpret_cast<unsigned long long>(in2)) & 15) == 0;
    if (pair16) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const C* src = (c == 0 ? in0 : c == 1 ? in1 : in2) + r0 * K1;
        C* dst = rin + 2 * c * K1;
        for (int j = t; j < K1; j += X4Cfg::NT) cp_async16_cg(dst + 2 * j, src + 2 * j);
      }
    } else {
      for (int i = t; i < 6 * K1; i += X4Cfg::NT) {
        const int cr = i / K1, kx = i - cr * K1;
        const C* src = cr < 2 ? in0 : cr < 4 ? in1 : in2;  // no dynamic index into the parameter array
        C* dst = rin + i;
        if ((cr & 1) == 0 || has1) cp_async8(dst, src + (r0 + (cr & 1)) * K1 + kx);
        else *dst = make_float2(0.f, 0.f);
      }
    }
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  // Ia
  if (t < 81) {
    const int q = t / 9;
    C w[10];
#pragma unroll
    for (int sa = 1; sa < 10; ++sa) { const C v = __ldg(&tw[9 * q * sa]); w[sa] = make_float2(v.x, -v.y); }
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      // A: u1, u2 of row r; A': u1, u2 of row r'; B: u3 of rows r and r'
      const C* ra = rin + (j < 2 ? j : 4) * K1;
      const C* rb = rin + (j < 2 ? 2 + j : 5) * K1;
      C v[10];
#pragma unroll
      for (int p = 0; p < 10; ++p) {
        if (p == 4 || p == 5) v[p] = make_float2(0.f, 0.f);  // 324 <= k <= 485 is never retained
        else v[p] = x4_gather<FULL>(ra, rb, p, t, kmax);
      }
      DFT<10, true, C>::run(v);
      C* xs = reg0 + j * PS;
      xs[t] = v[0];
#pragma unroll
      for (int sa = 1; sa < 10; ++sa) xs[89 * sa + t] = cmul(v[sa], w[sa]);
    }
  }
  __syncthreads();
  // Ib
  if (t < 90) {
    const int sa = t / 9, m2 = t - 9 * sa;
    C w[9];
#pragma unroll
    for (int sb = 0; sb < 9; ++sb) { const C v = __ldg(&tw[m2 * (sa + 10 * sb)]); w[sb] = make_float2(v.x, -v.y); }
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      const C* xs = reg0 + j * PS + 89 * sa + m2;
      C v[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) v[q] = xs[9 * q];
      DFT<9, true, C>::run(v);
      C* ys = reg1 + j * PS + t;
#pragma unroll
      for (int sb = 0; sb < 9; ++sb) ys[90 * sb] = cmul(v[sb], w[sb]);
    }
  }
  __syncthreads();
  // Ic + F1
  // the products enter the forward transform unscaled; the 1/n^D scale is
  // applied with the 1/2 of the final split (the transform is linear)
  float u1[9], u2[9], u3[9], u3b[9];
  C wf[9];
  if (t < 90) {
#pragma unroll
    for (int s = 1; s < 9; ++s) wf[s] = __ldg(&tw[t * s]);
    C v[9];
    const C* ya = reg1 + 9 * t;
#pragma unroll
    for (int m2 = 0; m2 < 9; ++m2) v[m2] = ya[m2];
    DFT<9, true, C>::run(v);
#pragma unroll
    for (int s = 0; s < 9; ++s) { u1[s] = v[s].x; u2[s] = v[s].y; }
    const C* yb = reg1 + 2 * PS + 9 * t;
#pragma unroll
    for (int m2 = 0; m2 < 9; ++m2) v[m2] = yb[m2];
    DFT<9, true, C>::run(v);
#pragma unroll
    for (int s = 0; s < 9; ++s) { u3[s] = v[s].x; u3b[s] = v[s].y; }
    x4_f1_row(u1, u2, u3, wf, reg0, t);
    const C* yc = reg1 + PS + 9 * t;
#pragma unroll
    for (int m2 = 0; m2 < 9; ++m2) v[m2] = yc[m2];
    DFT<9, true, C>::run(v);
#pragma unroll
    for (int s = 0; s < 9; ++s) { u1[s] = v[s].x; u2[s] = v[s].y; }
  }
  __syncthreads();
  if (t < 90) x4_f1_row(u1, u2, u3b, wf, reg1, t);
  __syncthreads();
  // F2, in place per region: read all three pencils, barrier, write
  {
    const int s1 = t / 10, q = t - 10 * s1;
    C w2[9];
    if (t < 90) {
#pragma unroll
      for (int s = 1; s < 9; ++s) w2[s] = __ldg(&tw[9 * q * s]);
    }
#pragma unroll 1
    for (int g = 0; g < 2; ++g) {
      C* rg = g ? reg1 : reg0;
      C v[3][9];
      if (t < 90) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const C* ws = rg + j * PS + 90 * s1 + q;
#pragma unroll
          for (int p = 0; p < 9; ++p) v[j][p] = ws[10 * p];
          DFT<9, false, C>::run(v[j]);
#pragma unroll
          for (int s = 1; s < 9; ++s) v[j][s] = cmul(v[j][s], w2[s]);
        }
      }
      __syncthreads();
      if (t < 90) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          C* vs = rg + j * PS + 90 * s1 + 9 * q;
#pragma unroll
          for (int s = 0; s < 9; ++s) vs[s] = v[j][s];
        }
      }
    }
  }
  __syncthreads();
  // F3, in place per region, pruned to the retained modes (outputs s_b = 4, 5,
  // k in [324, 485], are never retained and are not formed)
  {
    const int s1 = t / 9, sa = t - 9 * s1;
    const int kb = s1 + 9 * sa;
#pragma unroll 1
    for (int g = 0; g < 2; ++g) {
      C* rg = g ? reg1 : reg0;
      C v[3][10];
      if (t < 81) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const C* vs = rg + j * PS + 90 * s1 + sa;
#pragma unroll
          for (int q = 0; q < 10; ++q) v[j][q] = vs[9 * q];
          DFT<10, false, C>::run(v[j]);
        }
      }
      __syncthreads();
      if (t < 81) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          C* zs = rg + j * PS;
#pragma unroll
          for (int sb = 0; sb < 10; ++sb) {
            if (sb == 4 || sb == 5) continue;
            const int k = kb + 81 * sb;
            if (FULL) {
              if (sb <= 2 || (sb == 3 && k <= 270)) zs[k] = v[j][sb];
              else if (sb >= 7 || (sb == 6 && k >= 540)) zs[270 + (N - k)] = v[j][sb];
            } else {
              if (k <= ko) zs[k] = v[j][sb];
              else if (k >= N - ko) zs[ko + (N - k)] = v[j][sb];
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // S
  const float hsc = 0.5f * float(a.scale);
  C* o0 = static_cast<C*>(a.out[0]);
  C* o1 = static_cast<C*>(a.out[1]);
  C* o2 = static_cast<C*>(a.out[2]);
  C* o3 = static_cast<C*>(a.out[3]);
  C* o4 = static_cast<C*>(a.out[4]);
  C* o5 = static_cast<C*>(a.out[5]);
  for (int it = t; it < 2 * K1o; it += X4Cfg::NT) {
    const int rr = it >= K1o, kx = it - rr * K1o;
    if (rr == 1 && !has1) continue;
    const int o = int(r0 + rr) * ldo + kx;  // < 810^2 rows x 407: 32-bit
    const C* zs = rr ? reg1 : reg0;
    const int kc = kx == 0 ? 0 : ko + kx;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const C z = zs[b * PS + kx], zc = zs[b * PS + kc];
      C* oa = b == 0 ? o0 : b == 1 ? o2 : o4;
      C* ob = b == 0 ? o1 : b == 1 ? o3 : o5;
      oa[o] = make_float2(hsc * (z.x + zc.x), hsc * (z.y - zc.y));
      ob[o] = make_float2(hsc * (z.y + zc.y), hsc * (zc.x - z.x));
    }
  }
}

// ---------------------------------------------------------------------------
// plain x transforms (to_phys! / to_spec! along x, the closures' and les!'s
// batches of fields): two-level register FFT per pencil, a pencil being one
// row of two components packed as a + i b
// ---------------------------------------------------------------------------
template <int N> struct XPF;
template <> struct XPF<810> { static constexpr int TP = 8; };
template <> struct XPF<256> { static constexpr int TP = 16; };
template <> struct XPF<128> { static constexpr int TP = 32; };
template <> struct XPF<64> { static constexpr int TP = 32; };

template <int N> struct XPFCfg {
  static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, N2P = N2 + 1;
  static constexpr int TP = XPF<N>::TP, NT = 256;
  static constexpr int KMAX = N / 2 + 1;  // widest spectral row (full RFFT layout)
  static constexpr size_t RIN = size_t(TP) * 2 * KMAX * sizeof(float2);    // c2r: staged rows; r2c: Z rows
  static constexpr size_t YB = size_t(TP) * N1 * N2P * sizeof(float2);
  static constexpr size_t SMEM = RIN + YB;
};

// Hermitian extension of one real row's half spectrum (K1 modes), the imaginary
// parts of the mean and of the Nyquist mode dropped (a real row's c2r ignores them)
template <int N> __device__ __forceinline__ float2 hext3(const float2* row, int K1, int f) {
  const int kmax = K1 - 1;
  if (f == 0) return make_float2(row[0].x, 0.f);
  if (f <= kmax) {
    float2 v = row[f];
    if (2 * f == N) v.y = 0.f;
    return v;
  }
  if (f >= N - kmax) { const float2 v = row[N - f]; return make_float2(v.x, -v.y); }
  return make_float2(0.f, 0.f);
}

template <int N>
__global__ void __launch_bounds__(XPFCfg<N>::NT) k_xc2r_fast(const XPlainArgs a, const float2* __restrict__ tw) {
  using Cfg = XPFCfg<N>;
  constexpr int N1 = Cfg::N1, N2 = Cfg::N2, N2P = Cfg::N2P, TP = Cfg::TP, NT = Cfg::NT, KMAX = Cfg::KMAX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* rin = reinterpret_cast<float2*>(smem_raw);              // [TP][2][KMAX]
  float2* yb = reinterpret_cast<float2*>(smem_raw + Cfg::RIN);    // [TP][N1][N2P]
  // pencil, row and element indices stay 32-bit (at most 810^2 rows x 406
  // modes per component); one warp stages one row, so no per-element division
  const int npair = (a.ncomp + 1) / 2, K1 = a.K1;
  const int npen = int(a.nrows) * npair, pen0 = blockIdx.x * TP;
  // both loops have compile-time trip counts and are unrolled, so each thread
  // issues all of its loads before the first store (a rolled loop waited out
  // one global-load latency per element)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  static_assert((2 * TP) % (NT / 32) == 0, "whole rows per warp");
#pragma unroll
  for (int i = 0; i < 2 * TP / (NT / 32); ++i) {
    const int s = warp + i * (NT / 32);
    const int pen = pen0 + (s >> 1);
    const float2* src = nullptr;
    if (pen < npen) {
      const int row = pen / npair, q = 2 * (pen - row * npair) + (s & 1);
      if (q < a.ncomp) src = static_cast<const float2*>(a.in[q]) + row * K1;
    }
    float2* dst = rin + s * KMAX;
#pragma unroll
    for (int u = 0; u < (KMAX + 31) / 32; ++u) {
      const int kx = lane + 32 * u;
      if (kx < K1) dst[kx] = src ? __ldg(src + kx) : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < TP * N2; it += NT) {
    const int p = it / N2, j = it - p * N2;
    const float2* ra = rin + (p * 2) * KMAX;
    const float2* rb = ra + KMAX;
    float2 v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int f = N2 * n1 + j;
      const float2 x = hext3<N>(ra, K1, f), y = hext3<N>(rb, K1, f);
      v[n1] = make_float2(x.x - y.y, x.y + y.x);
    }
    DFT<N1, true, float2>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) {
      const float2 w = __ldg(&tw[j * k1]);
      v[k1] = cmul(v[k1], make_float2(w.x, -w.y));
    }
    float2* yp = yb + p * N1 * N2P;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
  }
  __syncthreads();
  const float sc = float(a.scale);
  for (int it = threadIdx.x; it < TP * N1; it += NT) {
    const int p = it / N1, i = it - p * N1;
    const int pen = pen0 + p;
    if (pen >= npen) continue;
    float2 w[N2];
    const float2* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
    DFT<N2, true, float2>::run(w);
    const int row = pen / npair;
    const int pr = pen - row * npair;
    float* oa = static_cast<float*>(a.out[2 * pr]) + row * N + i;
    float* ob = 2 * pr + 1 < a.ncomp ? static_cast<float*>(a.out[2 * pr + 1]) + row * N + i : nullptr;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      oa[N1 * k2] = w[k2].x * sc;
      if (ob) ob[N1 * k2] = w[k2].y * sc;
    }
  }
}

template <int N>
__global__ void __launch_bounds__(XPFCfg<N>::NT) k_xr2c_fast(const XPlainArgs a, const float2* __restrict__ tw) {
  using Cfg = XPFCfg<N>;
  constexpr int N1 = Cfg::N1, N2 = Cfg::N2, N2P = Cfg::N2P, TP = Cfg::TP, NT = Cfg::NT, KMAX = Cfg::KMAX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* zb = reinterpret_cast<float2*>(smem_raw);               // [TP][2 KMAX]: kept outputs
  float2* yb = reinterpret_cast<float2*>(smem_raw + Cfg::RIN);    // [TP][N1][N2P]
  const int npair = (a.ncomp + 1) / 2, K1 = a.K1, ko = K1 - 1;
  const int npen = int(a.nrows) * npair, pen0 = blockIdx.x * TP;  // 32-bit, as in k_xc2r_fast
  const float sc = float(a.scale);
  for (int it = threadIdx.x; it < TP * N2; it += NT) {
    const int p = it / N2, j = it - p * N2;
    const int pen = pen0 + p;
    float2 v[N1];
    const float* ia = nullptr;
    const float* ib = nullptr;
    if (pen < npen) {
      const int row = pen / npair;
      const int pr = pen - row * npair;
      ia = static_cast<const float*>(a.in[2 * pr]) + row * N;
      if (2 * pr + 1 < a.ncomp) ib = static_cast<const float*>(a.in[2 * pr + 1]) + row * N;
    }
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int x = N2 * n1 + j;
      v[n1] = make_float2(ia ? __ldg(ia + x) * sc : 0.f, ib ? __ldg(ib + x) * sc : 0.f);
    }
    DFT<N1, false, float2>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], __ldg(&tw[j * k1]));
    float2* yp = yb + p * N1 * N2P;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yp[k1 * N2P + j] = v[k1];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < TP * N1; it += NT) {
    const int p = it / N1, i = it - p * N1;
    float2 w[N2];
    const float2* yp = yb + p * N1 * N2P + i * N2P;
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = yp[n2];
    DFT<N2, false, float2>::run(w);
    float2* zp = zb + p * 2 * KMAX;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int k = i + N1 * k2;
      if (k <= ko) zp[k] = w[k2];
      else if (k >= N - ko) zp[ko + (N - k)] = w[k2];
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int p = warp; p < TP; p += NT / 32) {
    const int pen = pen0 + p;
    if (pen >= npen) continue;
    const int row = pen / npair;
    const int pr = pen - row * npair;
    const float2* zp = zb + p * 2 * KMAX;
    float2* oa = static_cast<float2*>(a.out[2 * pr]) + row * K1;
    float2* ob = 2 * pr + 1 < a.ncomp ? static_cast<float2*>(a.out[2 * pr + 1]) + row * K1 : nullptr;
    for (int kx = lane; kx < K1; kx += 32) {
      // X[k] = (Z[k] + conj Z[-k]) / 2, Y[k] = (Z[k] - conj Z[-k]) / 2i; Z[-0] = Z[0],
      // and Z[-N/2] = Z[N/2] at the Nyquist mode of a full-layout row
      const int kc = kx == 0 ? 0 : (2 * kx == N ? kx : ko + kx);
      const float2 z = zp[kx], zc = zp[kc];
      oa[kx] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
      if (ob) ob[kx] = make_float2(0.5f * (z.y + zc.y), 0.5f * (zc.x - z.x));
    }
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
template <typename F> static void set_smem2(F* f, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

// Column-sweep variants the autotuner chooses from, per N: (tile width T,
// split S).  Variant 0 is the default; launches with derivative outputs always
// use variant 0.
template <int N> struct ColVariants;
template <> struct ColVariants<810> {
  static constexpr int count = 4;
  static constexpr int T[4] = {8, 8, 4, 16}, S[4] = {0, 1, 0, 0};
};
static_assert(ColVariants<810>::count == kColTmaVariant, "the TMA-fed sweep follows the k_col2 variants");
template <> struct ColVariants<256> {
  static constexpr int count = 2;
  static constexpr int T[2] = {16, 8}, S[2] = {0, 0};
};
template <> struct ColVariants<128> {
  static constexpr int count = 3;
  static constexpr int T[3] = {16, 8, 16}, S[3] = {0, 0, 1};
};
template <> struct ColVariants<64> {
  static constexpr int count = 2;
  static constexpr int T[2] = {16, 8}, S[2] = {0, 0};
};

template <int N, int T, int S> static void init_col2_variant() {
  using Cfg = Col2Cfg<N, T, S>;
  set_smem2(k_col2<N, T, true, false, false, S>, Cfg::SMEM);
  set_smem2(k_col2<N, T, true, false, true, S>, Cfg::SMEM);
  set_smem2(k_col2<N, T, false, false, false, S>, Cfg::SMEM);
  set_smem2(k_col2<N, T, false, false, true, S>, Cfg::SMEM);
}

template <int N, int V = 0> static void init_col2_variants() {
  if constexpr (V < ColVariants<N>::count) {
    init_col2_variant<N, ColVariants<N>::T[V], ColVariants<N>::S[V]>();
    init_col2_variants<N, V + 1>();
  }
}

template <int N> static void init_xplain();

template <int N> static void init_fast_n() {
  constexpr int T = ColVariants<N>::T[0];
  set_smem2(k_col2<N, T, true, true, false>, Col2Cfg<N, T>::SMEM);
  set_smem2(k_col2<N, T, true, true, true>, Col2Cfg<N, T>::SMEM);
  init_col2_variants<N>();
  set_smem2(k_xsweep2<N, 2>, X2Cfg<N, 2>::SMEM);
  set_smem2(k_xsweep2<N, 3>, X2Cfg<N, 3>::SMEM);
  set_smem2(k_xsweep3<N>, X3Cfg<N>::SMEM);
  if (N == 810) set_smem2(k_xsweep4<true>, X4Cfg::SMEM), set_smem2(k_xsweep4<false>, X4Cfg::SMEM);
  init_xplain<N>();
}

bool fast_supported(int N) { return N == 810 || N == 256 || N == 128 || N == 64; }

template <int N> static void init_xplain() {
  set_smem2(k_xc2r_fast<N>, XPFCfg<N>::SMEM);
  set_smem2(k_xr2c_fast<N>, XPFCfg<N>::SMEM);
}

// ---------------------------------------------------------------------------
// x c2r for N = 64 and 128 with one warp per packed row pair, in registers
// ---------------------------------------------------------------------------
// Z[f] = X_a[f] + i X_b[f] (the Hermitian extensions of two real rows' half
// spectra); lane l holds Z[l + 32 q], q < Q = N / 32.  A radix-Q inverse DFT
// over q and the twiddles exp(+2 pi i l k1 / N) in registers, then for each
// k1 a 32-point inverse DFT across the lanes (five radix-2 decimation-in-
// frequency stages on warp shuffles), which leaves X[k1 + Q k2] with k2 the
// 5-bit reversal of the lane: x_a = Re, x_b = Im.  No shared memory and no
// CTA barrier; each warp's loads of a row are one or two 128-byte lines.
template <int N>
__global__ void __launch_bounds__(256) k_xc2r_warp(const XPlainArgs a, const float2* __restrict__ tw) {
  constexpr int Q = N / 32;
  const int lane = threadIdx.x & 31;
  const int pen = int(blockIdx.x) * 8 + (threadIdx.x >> 5);
  const int npair = (a.ncomp + 1) / 2, K1 = a.K1, kmax = K1 - 1;
  if (pen >= int(a.nrows) * npair) return;  // whole warps leave together
  const int row = pen / npair, pr = pen - row * npair;
  const float2* ra = static_cast<const float2*>(a.in[2 * pr]) + row * K1;
  const float2* rb = 2 * pr + 1 < a.ncomp ? static_cast<const float2*>(a.in[2 * pr + 1]) + row * K1 : nullptr;
  auto hext = [&](const float2* r, int f) -> float2 {
    if (!r) return make_float2(0.f, 0.f);
    if (f == 0) return make_float2(__ldg(&r[0].x), 0.f);
    if (f <= kmax) {
      float2 v = __ldg(&r[f]);
      if (2 * f == N) v.y = 0.f;
      return v;
    }
    if (f >= N - kmax) { const float2 v = __ldg(&r[N - f]); return make_float2(v.x, -v.y); }
    return make_float2(0.f, 0.f);
  };
  float2 v[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int f = lane + 32 * q;
    const float2 x = hext(ra, f), y = hext(rb, f);
    v[q] = make_float2(x.x - y.y, x.y + y.x);
  }
  DFT<Q, true, float2>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < Q; ++k1) {
    const float2 w = __ldg(&tw[lane * k1]);  // exp(-2 pi i lane k1 / N), conjugated below
    v[k1] = cmul(v[k1], make_float2(w.x, -w.y));
  }
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    const bool hi = (lane & h) != 0;
    // exp(+2 pi i (lane mod h) (16 / h) / 32) = conj(tw[(lane mod h) (16 / h) Q])
    const float2 w = __ldg(&tw[(lane & (h - 1)) * (16 / h) * Q]);
#pragma unroll
    for (int k1 = 0; k1 < Q; ++k1) {
      const float ux = __shfl_xor_sync(0xffffffffu, v[k1].x, h);
      const float uy = __shfl_xor_sync(0xffffffffu, v[k1].y, h);
      if (!hi) {
        v[k1] = make_float2(v[k1].x + ux, v[k1].y + uy);
      } else {
        v[k1] = cmul(make_float2(ux - v[k1].x, uy - v[k1].y), make_float2(w.x, -w.y));
      }
    }
  }
  const int k2 = __brev(unsigned(lane)) >> 27;
  const float sc = float(a.scale);
  float* oa = static_cast<float*>(a.out[2 * pr]) + row * N;
  float* ob = 2 * pr + 1 < a.ncomp ? static_cast<float*>(a.out[2 * pr + 1]) + row * N : nullptr;
#pragma unroll
  for (int k1 = 0; k1 < Q; ++k1) {
    oa[k1 + Q * k2] = v[k1].x * sc;
    if (ob) ob[k1 + Q * k2] = v[k1].y * sc;
  }
}

template <int N> static void xplain_n(bool inv, const XPlainArgs& a, const void* tw, cudaStream_t st) {
  using Cfg = XPFCfg<N>;
  const long long npen = a.nrows * ((a.ncomp + 1) / 2);
  const unsigned nb = unsigned((npen + Cfg::TP - 1) / Cfg::TP);
  const float2* t2 = static_cast<const float2*>(tw);
  if (inv && (N == 64 || N == 128)) {
    k_xc2r_warp<N == 64 ? 64 : 128><<<unsigned((npen + 7) / 8), 256, 0, st>>>(a, t2);
    return;
  }
  if (inv) k_xc2r_fast<N><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
  else k_xr2c_fast<N><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
}

bool launch_xplain_fast(int N, bool inv, const XPlainArgs& a, const void* tw, cudaStream_t st) {
  if (a.K1 > N / 2 + 1 || a.K1 < 1) return false;
  if (a.nrows * N >= (1ll << 31)) return false;  // the kernels index rows and elements in 32 bits
  switch (N) {
    case 810: xplain_n<810>(inv, a, tw, st); return true;
    case 256: xplain_n<256>(inv, a, tw, st); return true;
    case 128: xplain_n<128>(inv, a, tw, st); return true;
    case 64: xplain_n<64>(inv, a, tw, st); return true;
    default: return false;
  }
}

bool init_fast(int N) {
  switch (N) {
    case 810: init_fast_n<810>(); init_xpair810(); colt_init(); break;
    case 256: init_fast_n<256>(); break;
    case 128: init_fast_n<128>(); break;
    case 64: init_fast_n<64>(); break;
    default: return false;
  }
  return cudaGetLastError() == cudaSuccess;
}

// Every column sweep runs one two-level tile per CTA (k_col2), which keeps
// shared-memory traffic at one exchange per element; at three CTAs per SM it
// beat persistent cp.async-staged variants (one or two CTAs per SM, double-
// buffered tiles) in both directions (810^3 inverse y sweep, 81 planes:
// 0.166 ms against 0.283 ms for a persistent three-level kernel).
template <int N, int T, int S, bool INV> static void col2_launch(const ColArgs& a, const float2* t2, cudaStream_t st) {
  using Cfg = Col2Cfg<N, T, S>;
  dim3 grid((a.K1 + T - 1) / T, a.ncols, a.ncomp);
  const bool full = a.kpos == N / 3 + 1 && a.kneg == N / 3;
  if (full) k_col2<N, T, INV, false, true, S><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
  else k_col2<N, T, INV, false, false, S><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
}

template <int N, bool INV, int V = 0> static void col2_variant(int v, const ColArgs& a, const float2* t2,
                                                              cudaStream_t st) {
  if constexpr (V < ColVariants<N>::count) {
    if (v == V) col2_launch<N, ColVariants<N>::T[V], ColVariants<N>::S[V], INV>(a, t2, st);
    else col2_variant<N, INV, V + 1>(v, a, t2, st);
  }
}

template <int N, bool INV> static void col2_n(const ColArgs& a, const void* tw, cudaStream_t st) {
  const float2* t2 = static_cast<const float2*>(tw);
  if constexpr (INV) {
    if (a.ndrv > 0) {
      constexpr int T = ColVariants<N>::T[0];
      using Cfg = Col2Cfg<N, T>;
      dim3 grid((a.K1 + T - 1) / T, a.ncols, a.ncomp + a.ndrv);
      const bool full = a.kpos == N / 3 + 1 && a.kneg == N / 3;
      if (full) k_col2<N, T, true, true, true><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
      else k_col2<N, T, true, true, false><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, t2);
      return;
    }
  }
  if (N == 810 && a.variant >= kColTmaVariant && a.variant < kColTmaVariant + kColTmaConfigs &&
      launch_colt(N, INV, a, tw, a.variant - kColTmaVariant, st))
    return;
  const int v = a.variant >= 0 && a.variant < ColVariants<N>::count ? a.variant : 0;
  col2_variant<N, INV>(v, a, t2, st);
}

bool launch_col2(int N, bool inv, const ColArgs& a, const void* tw, cudaStream_t st) {
  switch (N) {
#define SC_C2(NN) \
  case NN: if (inv) col2_n<NN, true>(a, tw, st); else col2_n<NN, false>(a, tw, st); return true;
    SC_C2(810) SC_C2(256) SC_C2(128) SC_C2(64)
#undef SC_C2
    default: return false;
  }
}

int col2_variants(int N) {
  switch (N) {
    case 810: return ColVariants<810>::count + kColTmaConfigs;  // + the TMA-fed sweeps
    case 256: return ColVariants<256>::count;
    case 128: return ColVariants<128>::count;
    case 64: return ColVariants<64>::count;
    default: return 1;
  }
}

// x-sweep variants (3D): at 810, 0 = the scalar three-level sweep (default:
// the fastest measured), 1 = the paired-row f32x2 sweep at five CTAs per SM,
// 2 = the same at four CTAs per SM (registers for its twiddles), 3 = the
// two-level sweep of four rows per CTA; elsewhere 0 = the two-level four-row-
// group sweep, 1 = the plain two-level sweep.
template <int N> static void x2_n(const XArgs& a, const void* tw, cudaStream_t st) {
  const float2* t2 = static_cast<const float2*>(tw);
  const unsigned nb = unsigned((a.nrows + X2Rows<N>::TR - 1) / X2Rows<N>::TR);
  const unsigned nb3 = unsigned((a.nrows + X3Rows<N>::TR - 1) / X3Rows<N>::TR);
  if (a.D == 2) {
    k_xsweep2<N, 2><<<nb, X2Cfg<N, 2>::NT, X2Cfg<N, 2>::SMEM, st>>>(a, t2);
  } else if (N == 810) {
    if (a.variant == 1 || a.variant == 2) {
      launch_xpair810(a, t2 + 810, a.variant == 2 ? 4 : 5, st);
    } else if (a.variant == 3) {
      k_xsweep3<N><<<nb3, X3Cfg<N>::NT, X3Cfg<N>::SMEM, st>>>(a, t2);
    } else {
      const unsigned nb4 = unsigned((a.nrows + 1) / 2);
      if (a.K1in == 271 && a.K1out == 271) k_xsweep4<true><<<nb4, X4Cfg::NT, X4Cfg::SMEM, st>>>(a, t2);
      else k_xsweep4<false><<<nb4, X4Cfg::NT, X4Cfg::SMEM, st>>>(a, t2);
    }
  } else if (a.variant == 1) {
    k_xsweep2<N, 3><<<nb, X2Cfg<N, 3>::NT, X2Cfg<N, 3>::SMEM, st>>>(a, t2);
  } else {
    k_xsweep3<N><<<nb3, X3Cfg<N>::NT, X3Cfg<N>::SMEM, st>>>(a, t2);
  }
}

int xsweep_variants(int N, int D) {
  if (D != 3 || !fast_supported(N)) return 1;
  return N == 810 ? 4 : 2;
}

bool launch_xsweep2(int N, const XArgs& a, const void* tw, cudaStream_t st) {
  if (a.K1in > N / 3 + 1 || a.K1out > a.K1in) return false;
  switch (N) {
    case 810: x2_n<810>(a, tw, st); return true;
    case 256: x2_n<256>(a, tw, st); return true;
    case 128: x2_n<128>(a, tw, st); return true;
    case 64: x2_n<64>(a, tw, st); return true;
    default: return false;
  }
}

}  // namespace sc
