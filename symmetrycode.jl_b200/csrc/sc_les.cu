// LES closure kernels (reference: src/closures.jl, les! in src/les.jl:4-33).
//
// Spectral kernels act on the compact 2/3 cube (x extent K1 = kc+1, y/z extent
// K2 = 2 kc + 1, same layout as the solver state); physical kernels act
// pointwise on (n, n[, n]) real fields.  Symmetric tensors use the reference's
// pair order xx, yy[, zz], xy[, yz, zx]; velocity gradients the order
// G[a + D b] = d u_a / d x_b (tensorfield_nonsym, src/solver.jl:264-277).
#include <math.h>

#include "sc_fft.cuh"
#include "sc_les.h"

namespace sc {

struct Modes {
  int ix, iy, iz;
  bool origin;
};

__device__ __forceinline__ Modes decode(long long i, int kc, int D) {
  const int K1 = kc + 1, K2 = 2 * kc + 1;
  Modes m;
  m.ix = int(i % K1);
  const long long r = i / K1;
  const int py = int(r % K2);
  const int pz = D == 3 ? int(r / K2) : 0;
  m.iy = py <= kc ? py : py - K2;
  m.iz = pz <= kc ? pz : pz - K2;
  m.origin = m.ix == 0 && m.iy == 0 && m.iz == 0;
  return m;
}

// vectorgradient! (src/solver.jl:711-733): G[a + D b] = i k_b u_a
template <typename R, int D>
__global__ void k_grad(const LesSpecArgs a) {
  using C = typename V2<R>::T;
  const long long nm = a.nmodes;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const Modes m = decode(i, a.kc, D);
  const R k[3] = {R(a.kfac * m.ix), R(a.kfac * m.iy), R(a.kfac * m.iz)};
  for (int c = 0; c < D; ++c) {
    const C u = static_cast<const C*>(a.in[c])[i];
    for (int b = 0; b < D; ++b) static_cast<C*>(a.out[c + D * b])[i] = mk<C>(-k[b] * u.y, k[b] * u.x);
  }
}

// strainrate! (src/solver.jl:776-794)
template <typename R, int D>
__global__ void k_strain(const LesSpecArgs a) {
  using C = typename V2<R>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nmodes) return;
  const Modes m = decode(i, a.kc, D);
  const R k[3] = {R(a.kfac * m.ix), R(a.kfac * m.iy), R(a.kfac * m.iz)};
  C u[3];
  for (int c = 0; c < D; ++c) u[c] = static_cast<const C*>(a.in[c])[i];
  constexpr int NP = D == 3 ? 6 : 3;
  constexpr int PI[6] = {0, 1, 2, 0, 1, 2};
  constexpr int PJ3[6] = {0, 1, 2, 1, 2, 0};
  constexpr int PJ2[3] = {0, 1, 1};
  for (int q = 0; q < NP; ++q) {
    const int ii = D == 3 ? PI[q] : (q < 2 ? q : 0);
    const int jj = D == 3 ? PJ3[q] : PJ2[q];
    C v;
    if (ii == jj) {
      v = mk<C>(-k[ii] * u[ii].y, k[ii] * u[ii].x);
    } else {
      const R re = k[jj] * u[ii].x + k[ii] * u[jj].x, im = k[jj] * u[ii].y + k[ii] * u[jj].y;
      v = mk<C>(-im / R(2), re / R(2));
    }
    static_cast<C*>(a.out[q])[i] = v;
  }
}

// out = twothirds(gaussianfilter(in, delta)) (delta <= 0: no Gaussian), times `scale`
// (and times the device scalar *dscale when given); k = 0 is zeroed.
template <typename R, int D>
__global__ void k_spec_filter(const LesSpecArgs a) {
  using C = typename V2<R>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nmodes) return;
  const Modes m = decode(i, a.kc, D);
  const double k2 = a.kfac * a.kfac * double(m.ix * m.ix + m.iy * m.iy + m.iz * m.iz);
  double w = a.scale;
  if (a.dscale) w *= *a.dscale;
  if (a.delta > 0 && !(k2 < 9.0 * a.kfac * a.kfac)) w *= exp(-a.delta * a.delta * k2 / 24.0);
  if (m.origin) w = 0.0;
  const R wr = R(w);
  for (int c = 0; c < a.ncomp; ++c) {
    const C v = static_cast<const C*>(a.in[c])[i];
    static_cast<C*>(a.out[c])[i] = mk<C>(wr * v.x, wr * v.y);
  }
}

// ---------------------------------------------------------------------------
// physical pointwise kernels
// ---------------------------------------------------------------------------
template <typename R, int D>
__device__ __forceinline__ void load_grad(const LesPhysArgs& a, long long i, R G[3][3]) {
  for (int aa = 0; aa < D; ++aa)
    for (int b = 0; b < D; ++b) G[aa][b] = static_cast<const R*>(a.in[aa + D * b])[i];
}

template <typename R, int D>
__device__ __forceinline__ void store_sym(const LesPhysArgs& a, long long i, const R t[3][3]) {
  // store_symtensor! (src/closures.jl:14-28)
  R* o[6];
  for (int q = 0; q < (D == 3 ? 6 : 3); ++q) o[q] = static_cast<R*>(a.out[q]);
  if (D == 3) {
    o[0][i] = t[0][0]; o[1][i] = t[1][1]; o[2][i] = t[2][2];
    o[3][i] = t[0][1]; o[4][i] = t[1][2]; o[5][i] = t[2][0];
  } else {
    o[0][i] = t[0][0]; o[1][i] = t[1][1]; o[2][i] = t[0][1];
  }
}

// clark_kernel! / smagorinsky_kernel! / verstappen_kernel! (src/closures.jl:37-62)
template <typename R, int D>
__global__ void k_closure_pt(const LesPhysArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  R G[3][3] = {};
  load_grad<R, D>(a, i, G);
  R t[3][3] = {};
  const R d2 = R(a.delta * a.delta);
  if (a.kind == kClark) {
    for (int p = 0; p < D; ++p)
      for (int q = 0; q < D; ++q) {
        R s = 0;
        for (int k = 0; k < D; ++k) s += G[p][k] * G[q][k];
        t[p][q] = d2 / R(12) * s;
      }
  } else {
    R S[3][3];
    R ss = 0;
    for (int p = 0; p < D; ++p)
      for (int q = 0; q < D; ++q) {
        S[p][q] = (G[p][q] + G[q][p]) / R(2);
        ss += S[p][q] * S[p][q];
      }
    R nu;
    if (a.kind == kSmagorinsky) {
      const R cs = R(a.p0);
      nu = cs * cs * d2 * sqrt(R(2) * ss);
    } else {  // Verstappen: q = tr(S S)/2, r = tr(S S S)/3, nu = C^2 Delta^2 |r| / q
      R SS[3][3];
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) {
          R s = 0;
          for (int k = 0; k < 3; ++k) s += S[p][k] * S[k][q];
          SS[p][q] = s;
        }
      R trss = 0, trsss = 0;
      for (int p = 0; p < 3; ++p) {
        trss += SS[p][p];
        for (int k = 0; k < 3; ++k) trsss += SS[p][k] * S[k][p];
      }
      const R qq = trss / R(2), rr = trsss / R(3);
      const R c = R(a.p0);
      nu = c * c * d2 * fabs(rr) / qq;
    }
    for (int p = 0; p < D; ++p)
      for (int q = 0; q < D; ++q) t[p][q] = -R(2) * nu * S[p][q];
  }
  store_sym<R, D>(a, i, t);
}

// smagorinsky_tensor! (src/closures.jl:117-150) with C_s = 1, in place allowed
template <typename R, int D>
__global__ void k_smag_tensor(const LesPhysArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  constexpr int NP = D == 3 ? 6 : 3;
  R s[6];
  for (int q = 0; q < NP; ++q) s[q] = static_cast<const R*>(a.in[q])[i];
  R s2 = 0;
  for (int q = 0; q < D; ++q) s2 += s[q] * s[q];
  for (int q = D; q < NP; ++q) s2 += R(2) * s[q] * s[q];
  const R nu = R(a.delta * a.delta) * sqrt(R(2) * s2);
  for (int q = 0; q < NP; ++q) static_cast<R*>(a.out[q])[i] = -R(2) * nu * s[q];
}

// out_ij = in_ij - u_i u_j (in place allowed), optionally made trace-free
// (Bardina, src/closures.jl:81-115; Germano L, src/closures.jl:222-228)
template <typename R, int D>
__global__ void k_sub_products(const LesPhysArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  constexpr int NP = D == 3 ? 6 : 3;
  constexpr int PI3[6] = {0, 1, 2, 0, 1, 2}, PJ3[6] = {0, 1, 2, 1, 2, 0};
  constexpr int PI2[3] = {0, 1, 0}, PJ2[3] = {0, 1, 1};
  R u[3];
  for (int c = 0; c < D; ++c) u[c] = static_cast<const R*>(a.in2[c])[i];
  R t[6];
  for (int q = 0; q < NP; ++q) {
    const int ii = D == 3 ? PI3[q] : PI2[q], jj = D == 3 ? PJ3[q] : PJ2[q];
    t[q] = static_cast<const R*>(a.in[q])[i] - u[ii] * u[jj];
  }
  if (a.kind) {
    R tr = 0;
    for (int q = 0; q < D; ++q) tr += t[q];
    tr /= R(D);
    for (int q = 0; q < D; ++q) t[q] -= tr;
  }
  for (int q = 0; q < NP; ++q) static_cast<R*>(a.out[q])[i] = t[q];
}

__device__ __forceinline__ double block_sum_d(double v) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  v = 0;
  if (w == 0) {
    v = l < int(blockDim.x / 32) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// smagorinsky_ml_mm! (src/closures.jl:152-179) on L = L1 - u~_i u~_j, M = M1 - m2,
// summed in FP64: sums[0] += sum(M:L), sums[1] += sum(M:M)
template <typename R, int D>
__global__ void k_dynsmag_mlmm(const LesPhysArgs a, double* sums) {
  constexpr int NP = D == 3 ? 6 : 3;
  constexpr int PI3[6] = {0, 1, 2, 0, 1, 2}, PJ3[6] = {0, 1, 2, 1, 2, 0};
  constexpr int PI2[3] = {0, 1, 0}, PJ2[3] = {0, 1, 1};
  double ml = 0, mm = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.npts;
       i += (long long)gridDim.x * blockDim.x) {
    R u[3];
    for (int c = 0; c < D; ++c) u[c] = static_cast<const R*>(a.in2[c])[i];
    R L[6], M[6];
    for (int q = 0; q < NP; ++q) {
      const int ii = D == 3 ? PI3[q] : PI2[q], jj = D == 3 ? PJ3[q] : PJ2[q];
      L[q] = static_cast<const R*>(a.in[q])[i] - u[ii] * u[jj];
      M[q] = static_cast<const R*>(a.in3[q])[i] - static_cast<const R*>(a.in4[q])[i];
    }
    R tr = 0;
    for (int q = 0; q < D; ++q) tr += L[q];
    tr /= R(D);
    for (int q = 0; q < D; ++q) L[q] -= tr;
    R pml = 0, pmm = 0;
    for (int q = 0; q < D; ++q) { pml += M[q] * L[q]; pmm += M[q] * M[q]; }
    for (int q = D; q < NP; ++q) { pml += R(2) * M[q] * L[q]; pmm += R(2) * M[q] * M[q]; }
    ml += double(pml);
    mm += double(pmm);
  }
  ml = block_sum_d(ml);
  mm = block_sum_d(mm);
  if (threadIdx.x == 0) {
    atomicAdd(&sums[0], ml);
    atomicAdd(&sums[1], mm);
  }
}

// c = max(-<ML>/<MM>, 0), 0 when <MM> = 0 (src/closures.jl:258-262)
__global__ void k_dynsmag_coeff(double* sums) {
  const double ml = sums[0], mm = sums[1];
  sums[2] = (mm == 0.0) ? 0.0 : fmax(-ml / mm, 0.0);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static unsigned nb(long long n) { return unsigned((n + 255) / 256); }

template <typename R> void launch_grad(const LesSpecArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_grad<R, 3><<<nb(a.nmodes), 256, 0, st>>>(a);
  else k_grad<R, 2><<<nb(a.nmodes), 256, 0, st>>>(a);
}
template <typename R> void launch_strain(const LesSpecArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_strain<R, 3><<<nb(a.nmodes), 256, 0, st>>>(a);
  else k_strain<R, 2><<<nb(a.nmodes), 256, 0, st>>>(a);
}
template <typename R> void launch_spec_filter(const LesSpecArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_spec_filter<R, 3><<<nb(a.nmodes), 256, 0, st>>>(a);
  else k_spec_filter<R, 2><<<nb(a.nmodes), 256, 0, st>>>(a);
}
template <typename R> void launch_closure_pt(const LesPhysArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_closure_pt<R, 3><<<nb(a.npts), 256, 0, st>>>(a);
  else k_closure_pt<R, 2><<<nb(a.npts), 256, 0, st>>>(a);
}
template <typename R> void launch_smag_tensor(const LesPhysArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_smag_tensor<R, 3><<<nb(a.npts), 256, 0, st>>>(a);
  else k_smag_tensor<R, 2><<<nb(a.npts), 256, 0, st>>>(a);
}
template <typename R> void launch_sub_products(const LesPhysArgs& a, int D, cudaStream_t st) {
  if (D == 3) k_sub_products<R, 3><<<nb(a.npts), 256, 0, st>>>(a);
  else k_sub_products<R, 2><<<nb(a.npts), 256, 0, st>>>(a);
}
template <typename R> void launch_dynsmag_mlmm(const LesPhysArgs& a, int D, double* sums, cudaStream_t st) {
  long long b = (a.npts + 255) / 256;
  if (b > 148 * 4) b = 148 * 4;
  if (D == 3) k_dynsmag_mlmm<R, 3><<<unsigned(b), 256, 0, st>>>(a, sums);
  else k_dynsmag_mlmm<R, 2><<<unsigned(b), 256, 0, st>>>(a, sums);
  k_dynsmag_coeff<<<1, 1, 0, st>>>(sums);
}

#define SC_LES_INST(R)                                                              \
  template void launch_grad<R>(const LesSpecArgs&, int, cudaStream_t);              \
  template void launch_strain<R>(const LesSpecArgs&, int, cudaStream_t);            \
  template void launch_spec_filter<R>(const LesSpecArgs&, int, cudaStream_t);       \
  template void launch_closure_pt<R>(const LesPhysArgs&, int, cudaStream_t);        \
  template void launch_smag_tensor<R>(const LesPhysArgs&, int, cudaStream_t);       \
  template void launch_sub_products<R>(const LesPhysArgs&, int, cudaStream_t);      \
  template void launch_dynsmag_mlmm<R>(const LesPhysArgs&, int, double*, cudaStream_t);
SC_LES_INST(float)
SC_LES_INST(double)

}  // namespace sc
