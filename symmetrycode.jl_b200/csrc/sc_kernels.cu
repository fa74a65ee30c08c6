// Sweep kernels of the pseudo-spectral Navier-Stokes pipeline (sm_100a).
//
// One right-hand side (reference: `convectiondiffusion!`, src/solver.jl:949,
// which runs `nonlinearity!` src/solver.jl:434-456, `viscosity!` :458-476 and
// `tensordivergence!` :509-521 around 9 cuFFT calls) is five sweeps over HBM:
//
//   k_col_inv   z: compact 2/3 cube (kx, ky, kz)  -> (kx, ky, z)     3 comps
//   k_col_inv   y: (kx, ky, z)                    -> (kx, y, z)      3 comps
//   k_xsweep_ns x: c2r, u_i u_j / n^D, r2c        -> (kx, y, z)      6 comps
//   k_col_fwd   y: (kx, y, z)                     -> (kx, ky, z)     6 comps
//   k_col_fwd   z: (kx, ky, z)                    -> (kx, ky, kz)    6 comps
//   k_epilogue     viscous term, divergence, projection, forcing, RK update
//
// Only the modes kept by the 2/3 rule (|k_i| <= n/3) are ever stored, so the
// zero modes `twothirds!` (src/solver.jl:371-389) would mask are never read.
#include "sc_fft.cuh"
#include "sc_internal.h"

#include <cstdlib>
#include <cstring>

namespace sc {

// ---------------------------------------------------------------------------
// tile configuration
// ---------------------------------------------------------------------------
template <typename R, int N> struct ColCfg {
  static constexpr int T = sizeof(R) == 4 ? 16 : 8;  // kx per tile: 128-byte rows
  static constexpr int NT = T * N >= 4096 ? 512 : 256;
  static constexpr size_t SMEM = size_t(T) * N * sizeof(typename V2<R>::T);
};

template <typename R, int N> struct XCfg {
  static constexpr int CB = int(sizeof(typename V2<R>::T));
  static constexpr int TR0 = (100 * 1024) / (3 * N * CB);
  static constexpr int TR = TR0 < 1 ? 1 : (TR0 > 32 ? 32 : TR0);  // rows per CTA
  static constexpr int NT = TR * N >= 2048 ? 512 : 256;
  static constexpr size_t SMEM = size_t(3) * TR * N * CB;
};

template <typename R, int N> struct XPCfg {  // plain c2r / r2c: one buffer per row pair
  static constexpr int CB = int(sizeof(typename V2<R>::T));
  static constexpr int TR0 = (64 * 1024) / (N * CB);
  static constexpr int TR = TR0 < 1 ? 1 : (TR0 > 32 ? 32 : TR0);  // row pairs per CTA
  static constexpr int NT = TR * N >= 2048 ? 512 : 256;
  static constexpr size_t SMEM = size_t(TR) * N * CB;
};

template <typename F> static void set_smem(F* f, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

__device__ __forceinline__ int compact_pos(int f, int N, int kpos, int kneg) {
  return f < kpos ? f : (f >= N - kneg ? f - N + kpos + kneg : -1);
}

// ---------------------------------------------------------------------------
// column sweeps
// ---------------------------------------------------------------------------
template <typename R, int N>
__global__ void __launch_bounds__(ColCfg<R, N>::NT)
k_col_inv(const ColArgs a, const typename V2<R>::T* __restrict__ tw) {
  using C = typename V2<R>::T;
  constexpr int T = ColCfg<R, N>::T, NT = ColCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int kx0 = blockIdx.x * T;
  const int c = blockIdx.y;
  const int q = blockIdx.z;
  const bool drv = q >= a.ncomp;
  const int src = drv ? a.drv_src[q - a.ncomp] : q;
  const C* __restrict__ in = static_cast<const C*>(a.in[src]);
  C* __restrict__ out = static_cast<C*>(a.out[q]);
  const int Kc = a.kpos + a.kneg;
  // all loads of the tile are issued before the first shared-memory store so
  // that each thread keeps LPT requests in flight
  constexpr int LPT = (T * N + NT - 1) / NT;
  C v[LPT];
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    const int t = idx % T, e = idx / T;
    const int kx = kx0 + t;
    v[i] = mk<C>(R(0), R(0));
    const int p = compact_pos(e, N, a.kpos, a.kneg);
    if ((T * N % NT == 0 || idx < T * N) && kx < a.K1 && p >= 0 && !(a.zero_origin && kx == 0 && c == 0 && p == 0))
      v[i] = in[kx + (long long)c * a.in_cs + (long long)p * a.in_es];
  }
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    if (T * N % NT == 0 || idx < T * N) {
      const int t = idx % T, e = idx / T;
      C w = v[i];
      if (drv) {  // multiply by i k_e
        const int p = compact_pos(e, N, a.kpos, a.kneg);
        const R kk = R(a.kfac * double(p < a.kpos ? p : p - Kc));
        w = mk<C>(-kk * w.y, kk * w.x);
      }
      s[e * T + t] = w;
    }
  }
  __syncthreads();
  tile_fft<C, N, T, NT, true, true>(s, tw);
#pragma unroll 4
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    const int t = idx % T, e = idx / T;
    const int kx = kx0 + t;
    if ((T * N % NT == 0 || idx < T * N) && kx < a.K1)
      out[kx + (long long)c * a.out_cs + (long long)e * a.out_es] = s[e * T + t];
  }
}

template <typename R, int N>
__global__ void __launch_bounds__(ColCfg<R, N>::NT)
k_col_fwd(const ColArgs a, const typename V2<R>::T* __restrict__ tw) {
  using C = typename V2<R>::T;
  constexpr int T = ColCfg<R, N>::T, NT = ColCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int kx0 = blockIdx.x * T;
  const int c = blockIdx.y;
  const C* __restrict__ in = static_cast<const C*>(a.in[blockIdx.z]);
  C* __restrict__ out = static_cast<C*>(a.out[blockIdx.z]);
  constexpr int LPT = (T * N + NT - 1) / NT;
  C v[LPT];
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    const int t = idx % T, e = idx / T;
    const int kx = kx0 + t;
    v[i] = mk<C>(R(0), R(0));
    if ((T * N % NT == 0 || idx < T * N) && kx < a.K1) v[i] = in[kx + (long long)c * a.in_cs + (long long)e * a.in_es];
  }
#pragma unroll
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    if (T * N % NT == 0 || idx < T * N) s[(idx / T) * T + idx % T] = v[i];
  }
  __syncthreads();
  tile_fft<C, N, T, NT, false, true>(s, tw);
#pragma unroll 4
  for (int i = 0; i < LPT; ++i) {
    const int idx = threadIdx.x + i * NT;
    const int t = idx % T, e = idx / T;
    const int kx = kx0 + t;
    const int p = compact_pos(e, N, a.kpos, a.kneg);
    if ((T * N % NT == 0 || idx < T * N) && kx < a.K1 && p >= 0)
      out[kx + (long long)c * a.out_cs + (long long)p * a.out_es] = s[e * T + t];
  }
}

// ---------------------------------------------------------------------------
// x sweep helpers
// ---------------------------------------------------------------------------
// Hermitian extension of a half-spectrum row U[0..K1-1] to FFT index f of a
// length-N complex spectrum.  DC (and Nyquist, when stored) keep only their
// real part, as the c2r transform does.
template <typename C, int N>
__device__ __forceinline__ C hext(const C* __restrict__ row, int K1, int f) {
  using R = decltype(C::x);
  const int kmax = K1 - 1;
  if (f == 0) return mk<C>(row[0].x, R(0));
  if (f <= kmax) {
    C v = row[f];
    if (2 * f == N) v.y = R(0);
    return v;
  }
  if (f >= N - kmax) return cconj(row[N - f]);
  return mk<C>(R(0), R(0));
}

// z = a + i b for complex a, b
template <typename C> __device__ __forceinline__ C pack_pair(C a, C b) { return mk<C>(a.x - b.y, a.y + b.x); }

// ---------------------------------------------------------------------------
// x sweep with the Navier-Stokes products
// ---------------------------------------------------------------------------
template <typename R, int N, int D>
__global__ void __launch_bounds__(XCfg<R, N>::NT)
k_xsweep_ns(const XArgs a, const typename V2<R>::T* __restrict__ tw) {
  using C = typename V2<R>::T;
  constexpr int TR = XCfg<R, N>::TR, NT = XCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);  // [3][TR][N]
  C* s0 = s;
  C* s1 = s + TR * N;
  C* s2 = s + 2 * TR * N;
  const long long row0 = (long long)blockIdx.x * TR;
  const C* in0 = static_cast<const C*>(a.in[0]);
  const C* in1 = static_cast<const C*>(a.in[1]);
  const C* in2 = D == 3 ? static_cast<const C*>(a.in[2]) : nullptr;
  {
    constexpr int LPT = (TR * N + NT - 1) / NT;
    C z1[LPT], z2[LPT];
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      const int t = idx / N, f = idx % N;
      const long long row = row0 + t;
      z1[i] = mk<C>(R(0), R(0));
      z2[i] = mk<C>(R(0), R(0));
      if ((TR * N % NT == 0 || idx < TR * N) && row < a.nrows) {
        const long long off = row * a.K1in;
        z1[i] = pack_pair(hext<C, N>(in0 + off, a.K1in, f), hext<C, N>(in1 + off, a.K1in, f));
        if (D == 3) z2[i] = hext<C, N>(in2 + off, a.K1in, f);
      }
    }
#pragma unroll
    for (int i = 0; i < LPT; ++i) {
      const int idx = threadIdx.x + i * NT;
      if (TR * N % NT == 0 || idx < TR * N) {
        s0[idx] = z1[i];
        if (D == 3) s1[idx] = z2[i];
      }
    }
  }
  __syncthreads();
  // inverse transforms: TR pencils (2D) or 2*TR pencils (3D, buffers 0 and 1)
  tile_fft<C, N, (D == 3 ? 2 * TR : TR), NT, true, false>(s, tw);
  const R sc = R(a.scale);
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const C z1 = s0[idx];
    const R u1 = z1.x, u2 = z1.y;
    if (D == 3) {
      const R u3 = s1[idx].x;
      s0[idx] = mk<C>(u1 * u1 * sc, u2 * u2 * sc);
      s1[idx] = mk<C>(u3 * u3 * sc, u1 * u2 * sc);
      s2[idx] = mk<C>(u2 * u3 * sc, u3 * u1 * sc);
    } else {
      s0[idx] = mk<C>(u1 * u1 * sc, u2 * u2 * sc);
      s1[idx] = mk<C>(u1 * u2 * sc, R(0));
    }
  }
  __syncthreads();
  tile_fft<C, N, (D == 3 ? 3 * TR : 2 * TR), NT, false, false>(s, tw);
  // split the paired spectra: X_a = (Z_k + conj Z_{N-k})/2, X_b = -i/2 (Z_k - conj Z_{N-k})
  constexpr int NB = D == 3 ? 3 : 2;
  const int nout = D == 3 ? 6 : 3;
  const long long ldo = a.ldo > 0 ? a.ldo : a.K1out;
  for (int idx = threadIdx.x; idx < TR * a.K1out; idx += NT) {
    const int t = idx / a.K1out, kx = idx % a.K1out;
    const long long row = row0 + t;
    if (row >= a.nrows) continue;
    const int kn = kx == 0 ? 0 : N - kx;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const C* sb = s + (b * TR + t) * N;
      const C z = sb[kx], zc = sb[kn];
      const C xa = mk<C>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y - zc.y));
      const C xb = mk<C>(R(0.5) * (z.y + zc.y), R(0.5) * (zc.x - z.x));
      static_cast<C*>(a.out[2 * b])[row * ldo + kx] = xa;
      if (2 * b + 1 < nout) static_cast<C*>(a.out[2 * b + 1])[row * ldo + kx] = xb;
    }
  }
}

// ---------------------------------------------------------------------------
// plain x-direction c2r / r2c (pairs of fields per complex transform)
// ---------------------------------------------------------------------------
// c2r: rows of spectral component q (extent K1) -> physical rows of N reals.
// CTA handles TR "row pairs": a pair is two fields (q0, q1) of the same row.
template <typename R, int N>
__global__ void __launch_bounds__(XPCfg<R, N>::NT)
k_x_c2r(const XPlainArgs a, const typename V2<R>::T* __restrict__ tw) {
  using C = typename V2<R>::T;
  constexpr int TR = XPCfg<R, N>::TR, NT = XPCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int npair = (a.ncomp + 1) / 2;
  const long long npen = a.nrows * npair;  // pencil = (row, pair)
  const long long pen0 = (long long)blockIdx.x * TR;
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const int t = idx / N, f = idx % N;
    const long long pen = pen0 + t;
    C z = mk<C>(R(0), R(0));
    if (pen < npen) {
      const long long row = pen / npair;
      const int pr = int(pen % npair);
      const int q0 = 2 * pr, q1 = 2 * pr + 1;
      const C za = hext<C, N>(static_cast<const C*>(a.in[q0]) + row * a.K1, a.K1, f);
      C zb = mk<C>(R(0), R(0));
      if (q1 < a.ncomp) zb = hext<C, N>(static_cast<const C*>(a.in[q1]) + row * a.K1, a.K1, f);
      z = pack_pair(za, zb);
    }
    s[t * N + f] = z;
  }
  __syncthreads();
  tile_fft<C, N, TR, NT, true, false>(s, tw);
  const R sc = R(a.scale);
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const int t = idx / N, e = idx % N;
    const long long pen = pen0 + t;
    if (pen >= npen) continue;
    const long long row = pen / npair;
    const int pr = int(pen % npair);
    const C z = s[idx];
    static_cast<R*>(a.out[2 * pr])[row * N + e] = z.x * sc;
    if (2 * pr + 1 < a.ncomp) static_cast<R*>(a.out[2 * pr + 1])[row * N + e] = z.y * sc;
  }
}

// r2c: physical rows of N reals -> spectral rows (extent K1), times scale.
template <typename R, int N>
__global__ void __launch_bounds__(XPCfg<R, N>::NT)
k_x_r2c(const XPlainArgs a, const typename V2<R>::T* __restrict__ tw) {
  using C = typename V2<R>::T;
  constexpr int TR = XPCfg<R, N>::TR, NT = XPCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int npair = (a.ncomp + 1) / 2;
  const long long npen = a.nrows * npair;
  const long long pen0 = (long long)blockIdx.x * TR;
  const R sc = R(a.scale);
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const int t = idx / N, e = idx % N;
    const long long pen = pen0 + t;
    C z = mk<C>(R(0), R(0));
    if (pen < npen) {
      const long long row = pen / npair;
      const int pr = int(pen % npair);
      z.x = static_cast<const R*>(a.in[2 * pr])[row * N + e] * sc;
      if (2 * pr + 1 < a.ncomp) z.y = static_cast<const R*>(a.in[2 * pr + 1])[row * N + e] * sc;
    }
    s[t * N + e] = z;
  }
  __syncthreads();
  tile_fft<C, N, TR, NT, false, false>(s, tw);
  for (int idx = threadIdx.x; idx < TR * a.K1; idx += NT) {
    const int t = idx / a.K1, kx = idx % a.K1;
    const long long pen = pen0 + t;
    if (pen >= npen) continue;
    const long long row = pen / npair;
    const int pr = int(pen % npair);
    const C* sb = s + t * N;
    const C z = sb[kx], zc = sb[kx == 0 ? 0 : N - kx];
    const C xa = mk<C>(R(0.5) * (z.x + zc.x), R(0.5) * (z.y - zc.y));
    const C xb = mk<C>(R(0.5) * (z.y + zc.y), R(0.5) * (zc.x - z.x));
    static_cast<C*>(a.out[2 * pr])[row * a.K1 + kx] = xa;
    if (2 * pr + 1 < a.ncomp) static_cast<C*>(a.out[2 * pr + 1])[row * a.K1 + kx] = xb;
  }
}

// ---------------------------------------------------------------------------
// spectral epilogue on the compact cube
// ---------------------------------------------------------------------------
// sigma_ij = F[u_i u_j]/n^D - nu i (k_j u_i + k_i u_j)      (viscosity!, src/solver.jl:458-476)
// du_i     = -i k_j sigma_ij                                (tensordivergence!, :509-521)
// k        = du, or P(du) + A u on the forced band (RK4)    (project!, :350-368)
// out_a    = base_a + ca k   (projected when proj_a: wray3!, :992-1001)
// out_b    = base_b + cb k
template <typename R, int D>
__global__ void __launch_bounds__(256) k_epilogue(const EpiArgs a) {
  using C = typename V2<R>::T;
  const long long nm = (long long)a.K1 * a.K2 * (D == 3 ? a.K2 : 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const int ix = int(i % a.K1);
  const long long r = i / a.K1;
  const int py = int(r % a.K2);
  const int pz = D == 3 ? int(r / a.K2) : 0;
  const int iky = py <= a.kc ? py : py - a.K2;
  const int ikz = pz <= a.kc ? pz : pz - a.K2;
  const R kf = R(a.kfac);
  const R k[3] = {kf * R(ix), kf * R(iky), kf * R(ikz)};
  const R nu = R(a.visc);
  C u[3], s[6];
#pragma unroll
  for (int c = 0; c < D; ++c) u[c] = static_cast<const C*>(a.us[c])[i];
  constexpr int NP = D == 3 ? 6 : 3;
#pragma unroll
  for (int c = 0; c < NP; ++c) s[c] = static_cast<const C*>(a.sig[c])[i];
  if (a.has_sig2) {
#pragma unroll
    for (int c = 0; c < NP; ++c) s[c] = cadd(s[c], static_cast<const C*>(a.sig2[c])[i]);
  }
  // pair order: 3D xx yy zz xy yz zx ; 2D xx yy xy
  constexpr int P3[3][3] = {{0, 3, 5}, {3, 1, 4}, {5, 4, 2}};
  constexpr int P2[2][2] = {{0, 2}, {2, 1}};
  // viscous stress: sigma_ij -= nu i (k_j u_i + k_i u_j)
  C du[3];
#pragma unroll
  for (int ii = 0; ii < D; ++ii) {
    C acc = mk<C>(R(0), R(0));
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const int pc = D == 3 ? P3[ii][j] : P2[ii][j];
      C sg = s[pc];
      // - nu i (k_j u_i + k_i u_j)
      const C t = mk<C>(k[j] * u[ii].x + k[ii] * u[j].x, k[j] * u[ii].y + k[ii] * u[j].y);
      sg = mk<C>(sg.x + nu * t.y, sg.y - nu * t.x);
      // du_i += -i k_j sigma_ij
      acc = mk<C>(acc.x + k[j] * sg.y, acc.y - k[j] * sg.x);
    }
    du[ii] = acc;
  }
  R k2 = R(0);
#pragma unroll
  for (int c = 0; c < D; ++c) k2 += k[c] * k[c];
  const bool origin = (ix == 0 && iky == 0 && ikz == 0);
  if (a.proj_k && !origin) {
    C kd = mk<C>(R(0), R(0));
#pragma unroll
    for (int c = 0; c < D; ++c) kd = mk<C>(kd.x + k[c] * du[c].x, kd.y + k[c] * du[c].y);
    const C p = mk<C>(kd.x / k2, kd.y / k2);
#pragma unroll
    for (int c = 0; c < D; ++c) du[c] = mk<C>(du[c].x - k[c] * p.x, du[c].y - k[c] * p.y);
  }
  if (a.forcing != nullptr) {
    const int k2i = ix * ix + iky * iky + ikz * ikz;
    if (k2i >= 1 && k2i < 9) {
      const R A = R(*a.forcing);
#pragma unroll
      for (int c = 0; c < D; ++c) du[c] = mk<C>(du[c].x + A * u[c].x, du[c].y + A * u[c].y);
    }
  }
  const R ca = R(a.ca), cb = R(a.cb), mix = R(a.mix);
  C va[3], vb[3];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    C bb = mk<C>(R(0), R(0));
    if (a.has_b || a.mix_a) bb = static_cast<const C*>(a.base_b[c])[i];
    C b = mk<C>(R(0), R(0));
    if (a.mix_a) b = mk<C>(bb.x + mix * (u[c].x - bb.x), bb.y + mix * (u[c].y - bb.y));
    else if (a.base_a[c] != nullptr) b = static_cast<const C*>(a.base_a[c])[i];
    va[c] = mk<C>(b.x + ca * du[c].x, b.y + ca * du[c].y);
    if (a.has_b) vb[c] = mk<C>(bb.x + cb * du[c].x, bb.y + cb * du[c].y);
  }
  if (a.proj_a && !origin) {
    C kd = mk<C>(R(0), R(0));
#pragma unroll
    for (int c = 0; c < D; ++c) kd = mk<C>(kd.x + k[c] * va[c].x, kd.y + k[c] * va[c].y);
    const C p = mk<C>(kd.x / k2, kd.y / k2);
#pragma unroll
    for (int c = 0; c < D; ++c) va[c] = mk<C>(va[c].x - k[c] * p.x, va[c].y - k[c] * p.y);
  }
#pragma unroll
  for (int c = 0; c < D; ++c) {
    if (a.out_a[c] != nullptr) static_cast<C*>(a.out_a[c])[i] = va[c];
    if (a.has_b) static_cast<C*>(a.out_b[c])[i] = vb[c];
  }
}

// ---------------------------------------------------------------------------
// DNS -> LES filter (sfs!, src/data.jl:625-642)
// ---------------------------------------------------------------------------
// pass 0: ubar = twothirds(G_delta cutoff(u))                 (cutoff!, gaussianfilter!, twothirds!)
// pass 1: tau  = tracefree(twothirds(G_delta cutoff(sigma_dns) - sigma_les(ubar)))
// cutoff! (src/filtering.jl:9-34) copies the DNS mode with the same wavenumber;
// gaussianfilter! (src/filtering.jl:44-67) spares |k|^2 < (3 * 2 pi / l)^2.
template <typename R, int D>
__global__ void k_filter(const FilterArgs a) {
  using C = typename V2<R>::T;
  const int K1 = a.kcl + 1, K2 = 2 * a.kcl + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const int ix = int(i % K1);
  const long long r = i / K1;
  const int py = int(r % K2);
  const int pz = D == 3 ? int(r / K2) : 0;
  const int iy = py <= a.kcl ? py : py - K2;
  const int iz = pz <= a.kcl ? pz : pz - K2;
  const bool origin = ix == 0 && iy == 0 && iz == 0;
  const double k2 = a.kfac * a.kfac * double(ix * ix + iy * iy + iz * iz);
  double w = 1.0;
  if (a.delta > 0 && !(k2 < 9.0 * a.kfac * a.kfac)) w = exp(-a.delta * a.delta * k2 / 24.0);
  const R wr = R(w);
  if (a.pass == 0) {
    const int K1d = a.kcd + 1, K2d = 2 * a.kcd + 1;
    const int qy = iy >= 0 ? iy : iy + K2d;
    const int qz = iz >= 0 ? iz : iz + K2d;
    const long long j = ix + (long long)K1d * (qy + (long long)K2d * (D == 3 ? qz : 0));
    for (int c = 0; c < D; ++c) {
      C v = mk<C>(R(0), R(0));
      if (!origin) {
        const C u = static_cast<const C*>(a.udns[c])[j];
        v = mk<C>(wr * u.x, wr * u.y);
      }
      static_cast<C*>(a.ubar[c])[i] = v;
    }
  } else {
    constexpr int NP = D == 3 ? 6 : 3;
    C t[NP];
    for (int c = 0; c < NP; ++c) {
      const C s1 = static_cast<const C*>(a.sig1[c])[i];
      const C s2 = static_cast<const C*>(a.tau[c])[i];
      t[c] = origin ? mk<C>(R(0), R(0)) : mk<C>(wr * s1.x - s2.x, wr * s1.y - s2.y);
    }
    C tr = mk<C>(R(0), R(0));
    for (int c = 0; c < D; ++c) tr = cadd(tr, t[c]);
    tr = mk<C>(tr.x / R(D), tr.y / R(D));
    for (int c = 0; c < D; ++c) t[c] = csub(t[c], tr);
    for (int c = 0; c < NP; ++c) static_cast<C*>(a.tau[c])[i] = t[c];
  }
}

// ---------------------------------------------------------------------------
// pack / unpack between the full RFFT layout and the compact 2/3 cube
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_pack(const PackArgs a) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1, Kf = a.n / 2 + 1;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const int ix = int(i % K1);
  const long long r = i / K1;
  const int py = int(r % K2);
  const int pz = a.D == 3 ? int(r / K2) : 0;
  const int fy = py <= a.kc ? py : py + a.n - K2;
  const int fz = pz <= a.kc ? pz : pz + a.n - K2;
  const long long j = ix + (long long)Kf * (fy + (long long)a.n * fz);
  const C* src = static_cast<const C*>(a.src[blockIdx.y]);
  static_cast<C*>(a.dst[blockIdx.y])[i] = src[j];
}

template <typename R>
__global__ void k_unpack(const PackArgs a) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1, Kf = a.n / 2 + 1;
  const long long nm = (long long)Kf * a.n * (a.D == 3 ? a.n : 1);
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nm) return;
  const int ix = int(j % Kf);
  const long long r = j / Kf;
  const int fy = int(r % a.n);
  const int fz = a.D == 3 ? int(r / a.n) : 0;
  const int py = compact_pos(fy, a.n, a.kc + 1, a.kc);
  const int pz = a.D == 3 ? compact_pos(fz, a.n, a.kc + 1, a.kc) : 0;
  C v = mk<C>(R(0), R(0));
  if (ix < K1 && py >= 0 && pz >= 0) {
    const long long i = ix + (long long)K1 * (py + (long long)K2 * pz);
    v = static_cast<const C*>(a.src[blockIdx.y])[i];
  }
  static_cast<C*>(a.dst[blockIdx.y])[j] = v;
}

// ---------------------------------------------------------------------------
// FP64 reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) red[w] = v;
  __syncthreads();
  v = 0;
  if (w == 0) {
    v = l < int(blockDim.x / 32) ? red[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// band |k|^2 in [1, 9): kx in 0..2, ky, kz in -2..2 on the compact cube
template <typename R>
__global__ void k_band_forcing(const PackArgs a, double eps, double* A) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  double e = 0;
  const int t = threadIdx.x;  // 3 * 5 * 5 = 75 candidates per component
  if (t < 75) {
    const int ix = t % 3, iy = (t / 3) % 5 - 2, iz = t / 15 - 2;
    const int k2 = ix * ix + iy * iy + (a.D == 3 ? iz * iz : 0);
    const bool ok = ix <= a.kc && iy <= a.kc && -iy <= a.kc && (a.D == 2 ? iz == 0 : (iz <= a.kc && -iz <= a.kc));
    if (ok && k2 >= 1 && k2 < 9) {
      const int py = iy >= 0 ? iy : iy + K2;
      const int pz = iz >= 0 ? iz : iz + K2;
      const long long i = ix + (long long)K1 * (py + (long long)K2 * (a.D == 3 ? pz : 0));
      const double w = ix > 0 ? 2.0 : 1.0;
      for (int c = 0; c < a.D; ++c) {
        const C v = static_cast<const C*>(a.src[c])[i];
        e += w * (double(v.x) * double(v.x) + double(v.y) * double(v.y));
      }
    }
  }
  e = block_sum(e);
  if (threadIdx.x == 0) {
    const double ef = 0.5 * e;
    *A = ef > 0 ? eps / (2.0 * ef) : 0.0;
  }
}

template <typename R>
__global__ void k_spectral_energy(const PackArgs a, int K1, int K2, int compact, double kfac, int weight_k2,
                                  double* out, int mask23) {
  using C = typename V2<R>::T;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  double e = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const int ix = int(i % K1);
    double w = (ix == 0 || (!compact && 2 * ix == a.n)) ? 1.0 : 2.0;
    if (weight_k2 || mask23) {
      const long long r = i / K1;
      const int py = int(r % K2);
      const int pz = a.D == 3 ? int(r / K2) : 0;
      int iky, ikz;
      if (compact) {
        iky = py <= a.kc ? py : py - K2;
        ikz = pz <= a.kc ? pz : pz - K2;
      } else {
        iky = py < a.n / 2 ? py : py - a.n;
        ikz = pz < a.n / 2 ? pz : pz - a.n;
      }
      if (weight_k2) w *= kfac * kfac * double(ix * ix + iky * iky + ikz * ikz);
      if (mask23 && (ix > a.kc || iky > a.kc || -iky > a.kc || ikz > a.kc || -ikz > a.kc)) w = 0.0;
    }
    double s = 0;
    for (int c = 0; c < a.ncomp; ++c) {
      const C v = static_cast<const C*>(a.src[c])[i];
      s += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    e += w * s;
  }
  e = block_sum(e);
  if (threadIdx.x == 0) atomicAdd(out, e);
}

// ---------------------------------------------------------------------------
// CFL velocity maximum, shell clamp, spectrum
// ---------------------------------------------------------------------------
// max over physical points of |u| from D spectral x-rows (propose_timestep,
// src/solver.jl:931-947); the rows hold the y/z-inverse transforms of P u.
// Result as float bits (non-negative floats order like their bit patterns).
template <typename R, int N>
__global__ void __launch_bounds__(XPCfg<R, N>::NT)
k_x_vmax(const XPlainArgs a, const typename V2<R>::T* __restrict__ tw, unsigned long long* out) {
  using C = typename V2<R>::T;
  constexpr int TR = XPCfg<R, N>::TR / 2 > 0 ? XPCfg<R, N>::TR / 2 : 1, NT = XPCfg<R, N>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);  // [2][TR][N]: (u1 + i u2) and (u3 + 0 i) per row
  const long long row0 = (long long)blockIdx.x * TR;
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const int t = idx / N, f = idx % N;
    const long long row = row0 + t;
    C z1 = mk<C>(R(0), R(0)), z2 = mk<C>(R(0), R(0));
    if (row < a.nrows) {
      z1 = pack_pair(hext<C, N>(static_cast<const C*>(a.in[0]) + row * a.K1, a.K1, f),
                     hext<C, N>(static_cast<const C*>(a.in[1]) + row * a.K1, a.K1, f));
      if (a.ncomp == 3) z2 = hext<C, N>(static_cast<const C*>(a.in[2]) + row * a.K1, a.K1, f);
    }
    s[t * N + f] = z1;
    s[(TR + t) * N + f] = z2;
  }
  __syncthreads();
  tile_fft<C, N, 2 * TR, NT, true, false>(s, tw);
  double m = 0;
  for (int idx = threadIdx.x; idx < TR * N; idx += NT) {
    const int t = idx / N;
    if (row0 + t >= a.nrows) continue;
    const C z1 = s[idx], z2 = s[TR * N + idx];
    const double v = sqrt(double(z1.x) * z1.x + double(z1.y) * z1.y + double(z2.x) * z2.x);
    m = v > m ? v : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double q = __shfl_down_sync(0xffffffffu, m, o);
    m = q > m ? q : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// maintain_shell_energy! (src/solver.jl:1135-1152) for shells 1..2 on the
// compact state in one block: energies of 1 <= |k|^2 < 4 and 4 <= |k|^2 < 9
// (RFFT double count), then u *= sqrt(eref / e) on each shell.  mode 0 only
// measures (eref output), mode 1 rescales to eref.
template <typename R>
__global__ void k_shell_clamp(const PackArgs a, double* eref, int mode) {
  using C = typename V2<R>::T;
  __shared__ double e1s[32], e2s[32];
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  double e1 = 0, e2 = 0;
  const int t = threadIdx.x;  // 3 * 5 * 5 candidates
  long long idx = -1;
  int shell = 0;
  if (t < 75) {
    const int ix = t % 3, iy = (t / 3) % 5 - 2, iz = t / 15 - 2;
    const int k2 = ix * ix + iy * iy + (a.D == 3 ? iz * iz : 0);
    const bool ok = ix <= a.kc && iy <= a.kc && -iy <= a.kc && (a.D == 2 ? iz == 0 : (iz <= a.kc && -iz <= a.kc));
    if (ok && k2 >= 1 && k2 < 9) {
      const int py = iy >= 0 ? iy : iy + K2, pz = iz >= 0 ? iz : iz + K2;
      idx = ix + (long long)K1 * (py + (long long)K2 * (a.D == 3 ? pz : 0));
      shell = k2 < 4 ? 1 : 2;
      const double w = ix > 0 ? 2.0 : 1.0;
      double e = 0;
      for (int c = 0; c < a.D; ++c) {
        const C v = static_cast<const C*>(a.dst[c])[idx];
        e += w * (double(v.x) * v.x + double(v.y) * v.y);
      }
      if (shell == 1) e1 = 0.5 * e; else e2 = 0.5 * e;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    e1 += __shfl_down_sync(0xffffffffu, e1, o);
    e2 += __shfl_down_sync(0xffffffffu, e2, o);
  }
  if ((t & 31) == 0) { e1s[t / 32] = e1; e2s[t / 32] = e2; }
  __syncthreads();
  double E1 = 0, E2 = 0;
  for (int w = 0; w < int(blockDim.x / 32); ++w) { E1 += e1s[w]; E2 += e2s[w]; }
  if (mode == 0) {
    if (t == 0) { eref[0] = E1; eref[1] = E2; }
    return;
  }
  if (idx >= 0) {
    const double es = shell == 1 ? E1 : E2, er = shell == 1 ? eref[0] : eref[1];
    const R f = R(sqrt(er / es));
    for (int c = 0; c < a.D; ++c) {
      C* p = static_cast<C*>(a.dst[c]) + idx;
      *p = mk<C>(p->x * f, p->y * f);
    }
  }
}

// spectrum (src/solver.jl:693-699): s[i-1] += 1/2 sum over modes with i <= |k| < i+1 (RFFT double count)
template <typename R>
__global__ void k_spectrum(const PackArgs a, int nshell, double* s) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const int ix = int(i % K1);
    const long long r = i / K1;
    const int py = int(r % K2), pz = a.D == 3 ? int(r / K2) : 0;
    const int iy = py <= a.kc ? py : py - K2, iz = pz <= a.kc ? pz : pz - K2;
    const long long k2 = (long long)ix * ix + (long long)iy * iy + (long long)iz * iz;
    int sh = int(sqrt(double(k2)));
    while ((long long)(sh + 1) * (sh + 1) <= k2) ++sh;
    while ((long long)sh * sh > k2) --sh;
    if (sh < 1 || sh > nshell) continue;
    double e = 0;
    for (int c = 0; c < a.D; ++c) {
      const C v = static_cast<const C*>(a.src[c])[i];
      e += double(v.x) * v.x + double(v.y) * v.y;
    }
    atomicAdd(&s[sh - 1], 0.5 * (ix > 0 ? 2.0 : 1.0) * e);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
#define SC_SIZES(X) \
  X(4) X(6) X(8) X(10) X(12) X(16) X(18) X(20) X(24) X(30) X(32) X(36) X(40) X(48) X(60) X(64) X(72) X(80) \
  X(90) X(96) X(120) X(128) X(160) X(180) X(192) X(240) X(256) X(270) X(320) X(360) X(384) X(512) X(540) \
  X(640) X(720) X(768) X(810) X(1024)

bool fft_size_supported(int n) {
  switch (n) {
#define SC_CASE(N) case N: return true;
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}

template <typename R, int N>
static bool col_inv_n(const ColArgs& a, const void* tw, cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = ColCfg<R, N>;
  dim3 grid((a.K1 + Cfg::T - 1) / Cfg::T, a.ncols, a.ncomp + a.ndrv);
  k_col_inv<R, N><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  return true;
}
template <typename R, int N>
static bool col_fwd_n(const ColArgs& a, const void* tw, cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = ColCfg<R, N>;
  dim3 grid((a.K1 + Cfg::T - 1) / Cfg::T, a.ncols, a.ncomp);
  k_col_fwd<R, N><<<grid, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  return true;
}
template <typename R, int N>
static bool xsweep_n(const XArgs& a, const void* tw, cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = XCfg<R, N>;
  const unsigned nb = unsigned((a.nrows + Cfg::TR - 1) / Cfg::TR);
  if (a.D == 3) k_xsweep_ns<R, N, 3><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  else k_xsweep_ns<R, N, 2><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  return true;
}
template <typename R, int N>
static bool xc2r_n(const XPlainArgs& a, const void* tw, cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = XPCfg<R, N>;
  const long long npen = a.nrows * ((a.ncomp + 1) / 2);
  const unsigned nb = unsigned((npen + Cfg::TR - 1) / Cfg::TR);
  k_x_c2r<R, N><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  return true;
}
template <typename R, int N>
static bool xr2c_n(const XPlainArgs& a, const void* tw, cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = XPCfg<R, N>;
  const long long npen = a.nrows * ((a.ncomp + 1) / 2);
  const unsigned nb = unsigned((npen + Cfg::TR - 1) / Cfg::TR);
  k_x_r2c<R, N><<<nb, Cfg::NT, Cfg::SMEM, st>>>(a, static_cast<const C*>(tw));
  return true;
}

template <typename R, int N> static bool init_n() {
  set_smem(k_col_inv<R, N>, ColCfg<R, N>::SMEM);
  set_smem(k_col_fwd<R, N>, ColCfg<R, N>::SMEM);
  set_smem(k_xsweep_ns<R, N, 2>, XCfg<R, N>::SMEM);
  set_smem(k_xsweep_ns<R, N, 3>, XCfg<R, N>::SMEM);
  set_smem(k_x_c2r<R, N>, XPCfg<R, N>::SMEM);
  set_smem(k_x_r2c<R, N>, XPCfg<R, N>::SMEM);
  return cudaGetLastError() == cudaSuccess;
}

// Raise the dynamic shared-memory limits of every kernel of size N (once per
// process and device, before any launch or stream capture).
template <typename R> bool init_kernels(int N) {
  if (sizeof(R) == 4 && fast_supported(N) && !init_fast(N)) return false;
  switch (N) {
#define SC_CASE(NN) case NN: return init_n<R, NN>();
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}

template <typename R> static bool use_fast(int N) {
  return sizeof(R) == 4 && fast_supported(N);
}

template <typename R> bool launch_col_inv(int N, const ColArgs& a, const void* tw, cudaStream_t st) {
  if (use_fast<R>(N)) return launch_col2(N, true, a, tw, st);
  switch (N) {
#define SC_CASE(NN) case NN: return col_inv_n<R, NN>(a, tw, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}
template <typename R> bool launch_col_fwd(int N, const ColArgs& a, const void* tw, cudaStream_t st) {
  if (use_fast<R>(N)) return launch_col2(N, false, a, tw, st);
  switch (N) {
#define SC_CASE(NN) case NN: return col_fwd_n<R, NN>(a, tw, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}
template <typename R> bool launch_xsweep_ns(int N, const XArgs& a, const void* tw, cudaStream_t st) {
  if (use_fast<R>(N) && launch_xsweep2(N, a, tw, st)) return true;
  switch (N) {
#define SC_CASE(NN) case NN: return xsweep_n<R, NN>(a, tw, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}
template <typename R> bool launch_x_c2r(int N, const XPlainArgs& a, const void* tw, cudaStream_t st) {
  if (use_fast<R>(N) && launch_xplain_fast(N, true, a, tw, st)) return true;
  switch (N) {
#define SC_CASE(NN) case NN: return xc2r_n<R, NN>(a, tw, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}
template <typename R> bool launch_x_r2c(int N, const XPlainArgs& a, const void* tw, cudaStream_t st) {
  if (use_fast<R>(N) && launch_xplain_fast(N, false, a, tw, st)) return true;
  switch (N) {
#define SC_CASE(NN) case NN: return xr2c_n<R, NN>(a, tw, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}

template <typename R, int N> static bool xvmax_n(const XPlainArgs& a, const void* tw, unsigned long long* out,
                                                 cudaStream_t st) {
  using C = typename V2<R>::T;
  using Cfg = XPCfg<R, N>;
  constexpr int TR = Cfg::TR / 2 > 0 ? Cfg::TR / 2 : 1;
  const size_t smem = size_t(2) * TR * N * sizeof(C);
  static bool init = false;
  if (!init) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_x_vmax<R, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    init = true;
  }
  const unsigned nb = unsigned((a.nrows + TR - 1) / TR);
  k_x_vmax<R, N><<<nb, Cfg::NT, smem, st>>>(a, static_cast<const C*>(tw), out);
  return true;
}

template <typename R> bool launch_x_vmax(int N, const XPlainArgs& a, const void* tw, unsigned long long* out,
                                         cudaStream_t st) {
  switch (N) {
#define SC_CASE(NN) case NN: return xvmax_n<R, NN>(a, tw, out, st);
    SC_SIZES(SC_CASE)
#undef SC_CASE
    default: return false;
  }
}

template <typename R> void launch_shell_clamp(const PackArgs& a, double* eref, int mode, cudaStream_t st) {
  k_shell_clamp<R><<<1, 96, 0, st>>>(a, eref, mode);
}

template <typename R> void launch_spectrum(const PackArgs& a, int nshell, double* s, cudaStream_t st) {
  const long long nm = (long long)(a.kc + 1) * (2 * a.kc + 1) * (a.D == 3 ? (2 * a.kc + 1) : 1);
  long long nb = (nm + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  k_spectrum<R><<<unsigned(nb), 256, 0, st>>>(a, nshell, s);
}

template <typename R> void launch_epilogue(const EpiArgs& a, cudaStream_t st) {
  const long long nm = (long long)a.K1 * a.K2 * (a.D == 3 ? a.K2 : 1);
  const unsigned nb = unsigned((nm + 255) / 256);
  if (a.D == 3) k_epilogue<R, 3><<<nb, 256, 0, st>>>(a);
  else k_epilogue<R, 2><<<nb, 256, 0, st>>>(a);
}

template <typename R> void launch_pack(const PackArgs& a, cudaStream_t st) {
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  dim3 grid(unsigned((nm + 255) / 256), a.ncomp);
  k_pack<R><<<grid, 256, 0, st>>>(a);
}
template <typename R> void launch_unpack(const PackArgs& a, cudaStream_t st) {
  const long long nm = (long long)(a.n / 2 + 1) * a.n * (a.D == 3 ? a.n : 1);
  dim3 grid(unsigned((nm + 255) / 256), a.ncomp);
  k_unpack<R><<<grid, 256, 0, st>>>(a);
}
template <typename R> void launch_band_forcing(const void* const* u, int D, int K1, int K2, int kc,
                                               double eps, double* A, cudaStream_t st) {
  PackArgs a{};
  for (int c = 0; c < D; ++c) a.src[c] = u[c];
  a.ncomp = D; a.D = D; a.kc = kc; a.n = 0;
  (void)K1; (void)K2;
  k_band_forcing<R><<<1, 128, 0, st>>>(a, eps, A);
}
template <typename R> void launch_filter(const FilterArgs& a, cudaStream_t st) {
  const int K1 = a.kcl + 1, K2 = 2 * a.kcl + 1;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  const unsigned nb = unsigned((nm + 255) / 256);
  if (a.D == 3) k_filter<R, 3><<<nb, 256, 0, st>>>(a);
  else k_filter<R, 2><<<nb, 256, 0, st>>>(a);
}

template <typename R> void launch_spectral_energy(const void* const* u, int ncomp, int D, int n, int K1,
                                                  int K2, int compact, int kc, double kfac, int weight_k2,
                                                  double* out, cudaStream_t st, int mask23) {
  PackArgs a{};
  for (int c = 0; c < ncomp; ++c) a.src[c] = u[c];
  a.ncomp = ncomp; a.D = D; a.n = n; a.kc = kc;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  long long nb = (nm + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  if (nb < 1) nb = 1;
  k_spectral_energy<R><<<unsigned(nb), 256, 0, st>>>(a, K1, K2, compact, kfac, weight_k2, out, mask23);
}

// ---------------------------------------------------------------------------
// full-layout point kernels: twothirds! and project!
// ---------------------------------------------------------------------------
// twothirds! (src/solver.jl:371-389): keep |k_i| <= n/3 on every axis, zero k = 0
template <typename R>
__global__ void k_twothirds_full(const PackArgs a) {
  using C = typename V2<R>::T;
  const int Kf = a.n / 2 + 1;
  const long long nm = (long long)Kf * a.n * (a.D == 3 ? a.n : 1);
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nm) return;
  const int ix = int(j % Kf);
  const long long r = j / Kf;
  const int fy = int(r % a.n);
  const int fz = a.D == 3 ? int(r / a.n) : 0;
  const int ky = fy < a.n / 2 ? fy : fy - a.n;
  const int kz = fz < a.n / 2 ? fz : fz - a.n;
  const bool keep = ix <= a.kc && ky <= a.kc && -ky <= a.kc && kz <= a.kc && -kz <= a.kc &&
                    !(ix == 0 && ky == 0 && kz == 0);
  if (!keep) static_cast<C*>(a.dst[blockIdx.y])[j] = mk<C>(R(0), R(0));
}

// project! (src/solver.jl:350-368): u -= k (k.u)/k^2, k = 0 left intact
template <typename R>
__global__ void k_project_full(const PackArgs a, double kfac) {
  using C = typename V2<R>::T;
  const int Kf = a.n / 2 + 1;
  const long long nm = (long long)Kf * a.n * (a.D == 3 ? a.n : 1);
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nm) return;
  const int ix = int(j % Kf);
  const long long r = j / Kf;
  const int fy = int(r % a.n);
  const int fz = a.D == 3 ? int(r / a.n) : 0;
  const R k[3] = {R(kfac * ix), R(kfac * (fy < a.n / 2 ? fy : fy - a.n)),
                  R(kfac * (fz < a.n / 2 ? fz : fz - a.n))};
  if (ix == 0 && fy == 0 && fz == 0) return;
  C u[3];
  C kd = mk<C>(R(0), R(0));
  R k2 = R(0);
  for (int c = 0; c < a.D; ++c) {
    u[c] = static_cast<C*>(a.dst[c])[j];
    kd = mk<C>(kd.x + k[c] * u[c].x, kd.y + k[c] * u[c].y);
    k2 += k[c] * k[c];
  }
  const C p = mk<C>(kd.x / k2, kd.y / k2);
  for (int c = 0; c < a.D; ++c) static_cast<C*>(a.dst[c])[j] = mk<C>(u[c].x - k[c] * p.x, u[c].y - k[c] * p.y);
}

template <typename R> void launch_twothirds_full(const PackArgs& a, cudaStream_t st) {
  const long long nm = (long long)(a.n / 2 + 1) * a.n * (a.D == 3 ? a.n : 1);
  dim3 grid(unsigned((nm + 255) / 256), a.ncomp);
  k_twothirds_full<R><<<grid, 256, 0, st>>>(a);
}
template <typename R> void launch_project_full(const PackArgs& a, double kfac, cudaStream_t st) {
  const long long nm = (long long)(a.n / 2 + 1) * a.n * (a.D == 3 ? a.n : 1);
  k_project_full<R><<<unsigned((nm + 255) / 256), 256, 0, st>>>(a, kfac);
}

#define SC_INST(R)                                                                                      \
  template bool init_kernels<R>(int);                                                                   \
  template void launch_twothirds_full<R>(const PackArgs&, cudaStream_t);                                \
  template void launch_project_full<R>(const PackArgs&, double, cudaStream_t);                          \
  template bool launch_col_inv<R>(int, const ColArgs&, const void*, cudaStream_t);                      \
  template bool launch_col_fwd<R>(int, const ColArgs&, const void*, cudaStream_t);                      \
  template bool launch_xsweep_ns<R>(int, const XArgs&, const void*, cudaStream_t);                      \
  template bool launch_x_c2r<R>(int, const XPlainArgs&, const void*, cudaStream_t);                     \
  template bool launch_x_r2c<R>(int, const XPlainArgs&, const void*, cudaStream_t);                     \
  template void launch_epilogue<R>(const EpiArgs&, cudaStream_t);                                       \
  template void launch_pack<R>(const PackArgs&, cudaStream_t);                                          \
  template void launch_unpack<R>(const PackArgs&, cudaStream_t);                                        \
  template void launch_band_forcing<R>(const void* const*, int, int, int, int, double, double*,         \
                                       cudaStream_t);                                                   \
  template void launch_spectral_energy<R>(const void* const*, int, int, int, int, int, int, int, double, \
                                          int, double*, cudaStream_t, int);                               \
  template void launch_filter<R>(const FilterArgs&, cudaStream_t);                                   \
  template bool launch_x_vmax<R>(int, const XPlainArgs&, const void*, unsigned long long*, cudaStream_t); \
  template void launch_shell_clamp<R>(const PackArgs&, double*, int, cudaStream_t);                   \
  template void launch_spectrum<R>(const PackArgs&, int, double*, cudaStream_t);
SC_INST(float)
SC_INST(double)

}  // namespace sc
