// Adjoint (transpose) of the LES right-hand side with a CNN closure, for the
// a-posteriori training of the closure through the solver (new; the reference
// trains a-priori only, src/training.jl:3-109).
//
// Inner product: <a, b> = sum over the compact half-spectrum of w(k) Re(conj a b),
// w = 1 at kx = 0 and 2 otherwise -- the physical-space inner product divided
// by N = n^D (Parseval).  Under it the diagonal spectral multipliers m(k) have
// adjoint conj(m(k)), the projection is self-adjoint, to_spec (r2c / N) has
// adjoint to_phys / N and to_phys has adjoint N to_spec.
//
// Forward, per stage: F(u) = P[-i k_j Sigma_ij],
//   Sigma_ij = S[v_i v_j] + S[tau_ij(v, z)] - nu i (k_j u_i + k_i u_j),  v = T(u).
#include "sc_fft.cuh"
#include "sc_cnn_cc.h"

namespace sc {

namespace {
struct Mode {
  int ix, iy, iz;
  bool origin;
};
__device__ __forceinline__ Mode dmode(long long i, int kc, int D) {
  const int K1 = kc + 1, K2 = 2 * kc + 1;
  Mode m;
  m.ix = int(i % K1);
  const long long r = i / K1;
  const int py = int(r % K2), pz = D == 3 ? int(r / K2) : 0;
  m.iy = py <= kc ? py : py - K2;
  m.iz = pz <= kc ? pz : pz - K2;
  m.origin = m.ix == 0 && m.iy == 0 && m.iz == 0;
  return m;
}
}  // namespace

// Lambda = P lam;  lsig_p = D^T Lambda;  mu = viscous adjoint.
template <typename R, int D>
__global__ void k_adj_spec(const AdjSpecArgs a) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const Mode md = dmode(i, a.kc, D);
  const R k[3] = {R(a.kfac * md.ix), R(a.kfac * md.iy), R(a.kfac * md.iz)};
  C L[3];
  for (int c = 0; c < D; ++c) L[c] = static_cast<const C*>(a.lam[c])[i];
  if (!md.origin) {  // projection (k = 0 left intact, as project!)
    R k2 = 0;
    C kd = mk<C>(R(0), R(0));
    for (int c = 0; c < D; ++c) {
      k2 += k[c] * k[c];
      kd = mk<C>(kd.x + k[c] * L[c].x, kd.y + k[c] * L[c].y);
    }
    for (int c = 0; c < D; ++c) L[c] = mk<C>(L[c].x - k[c] * kd.x / k2, L[c].y - k[c] * kd.y / k2);
  }
  // pairs: 3D xx yy zz xy yz zx, 2D xx yy xy
  constexpr int NP = D == 3 ? 6 : 3;
  constexpr int PI3[6] = {0, 1, 2, 0, 1, 2}, PJ3[6] = {0, 1, 2, 1, 2, 0};
  constexpr int PI2[3] = {0, 1, 0}, PJ2[3] = {0, 1, 1};
  C ls[6];
  for (int p = 0; p < NP; ++p) {
    const int ii = D == 3 ? PI3[p] : PI2[p], jj = D == 3 ? PJ3[p] : PJ2[p];
    // du_i = -i k_j Sigma_ij  ->  lsig_p = i k_j L_i (+ i k_i L_j when i != j)
    C s = mk<C>(-k[jj] * L[ii].y, k[jj] * L[ii].x);
    if (ii != jj) s = mk<C>(s.x - k[ii] * L[jj].y, s.y + k[ii] * L[jj].x);
    ls[p] = s;
    static_cast<C*>(a.lsig[p])[i] = s;
  }
  // Sigma_ij -= nu i (k_j u_i + k_i u_j): mu_i = sum over pairs of conj(-nu i k) lsig
  const R nu = R(a.visc);
  C mu[3] = {mk<C>(R(0), R(0)), mk<C>(R(0), R(0)), mk<C>(R(0), R(0))};
  for (int p = 0; p < NP; ++p) {
    const int ii = D == 3 ? PI3[p] : PI2[p], jj = D == 3 ? PJ3[p] : PJ2[p];
    if (ii == jj) {
      const R f = R(2) * nu * k[ii];  // coefficient of u_i: -2 nu i k_i
      mu[ii] = mk<C>(mu[ii].x - f * ls[p].y, mu[ii].y + f * ls[p].x);
    } else {
      const R fi = nu * k[jj], fj = nu * k[ii];
      mu[ii] = mk<C>(mu[ii].x - fi * ls[p].y, mu[ii].y + fi * ls[p].x);
      mu[jj] = mk<C>(mu[jj].x - fj * ls[p].y, mu[jj].y + fj * ls[p].x);
    }
  }
  for (int c = 0; c < D; ++c) static_cast<C*>(a.mu[c])[i] = mu[c];
}

// lv_i = sum_j c_ij v_j m_ij / N (+ add_i): adjoint of the products v_i v_j
template <typename R, int D>
__global__ void k_adj_products(const AdjPhysArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npts) return;
  R v[3], m[6], lv[3] = {0, 0, 0};
  for (int c = 0; c < D; ++c) v[c] = static_cast<const R*>(a.v[c])[i];
  const R s = R(a.inv_npts);
  constexpr int NP = D == 3 ? 6 : 3;
  constexpr int PI3[6] = {0, 1, 2, 0, 1, 2}, PJ3[6] = {0, 1, 2, 1, 2, 0};
  constexpr int PI2[3] = {0, 1, 0}, PJ2[3] = {0, 1, 1};
  for (int p = 0; p < NP; ++p) m[p] = static_cast<const R*>(a.m[p])[i] * s;
  for (int p = 0; p < NP; ++p) {
    const int ii = D == 3 ? PI3[p] : PI2[p], jj = D == 3 ? PJ3[p] : PJ2[p];
    if (ii == jj) lv[ii] += R(2) * v[ii] * m[p];
    else { lv[ii] += v[jj] * m[p]; lv[jj] += v[ii] * m[p]; }
  }
  for (int c = 0; c < D; ++c) {
    R x = lv[c];
    if (a.add[c]) x += static_cast<const R*>(a.add[c])[i];
    static_cast<R*>(a.lv[c])[i] = x;
  }
}

template <typename R, int D>
__global__ void k_adj_acc(const AdjAccArgs a) {
  using C = typename V2<R>::T;
  const int K1 = a.kc + 1, K2 = 2 * a.kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  const Mode md = dmode(i, a.kc, D);
  double zc = 0;
  if (a.lamz) zc = *a.lamz / (a.sigma * *a.a2);
  const R k2 = R(a.kfac * a.kfac * double(md.ix * md.ix + md.iy * md.iy + md.iz * md.iz));
  for (int c = 0; c < D; ++c) {
    C m = static_cast<C*>(a.mu[c])[i];
    if (!md.origin) {
      const C x = static_cast<const C*>(a.x[c])[i];
      m = mk<C>(m.x + R(a.scale) * x.x, m.y + R(a.scale) * x.y);
    }
    if (a.lamz) {
      const C u = static_cast<const C*>(a.u[c])[i];
      m = mk<C>(m.x + R(zc) * k2 * u.x, m.y + R(zc) * k2 * u.y);
    }
    static_cast<C*>(a.mu[c])[i] = m;
  }
}

struct Ptr3 {
  void* p[3];
};
struct CPtr3 {
  const void* p[3];
};

template <typename R>
__global__ void k_axpby(Ptr3 y, CPtr3 x, double ax, double ay, int D, long long nm) {
  using C = typename V2<R>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nm) return;
  for (int c = 0; c < D; ++c) {
    C v = static_cast<C*>(y.p[c])[i];
    v = mk<C>(R(ay) * v.x, R(ay) * v.y);
    if (x.p[c]) {
      const C w = static_cast<const C*>(x.p[c])[i];
      v = mk<C>(v.x + R(ax) * w.x, v.y + R(ax) * w.y);
    }
    static_cast<C*>(y.p[c])[i] = v;
  }
}

template <typename R>
__global__ void k_mse(CPtr3 u, CPtr3 t, Ptr3 g, double coef, int D, int kc, double* loss) {
  using C = typename V2<R>::T;
  const int K1 = kc + 1, K2 = 2 * kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const double w = (i % K1) == 0 ? 1.0 : 2.0;
    for (int c = 0; c < D; ++c) {
      const C a = static_cast<const C*>(u.p[c])[i], b = static_cast<const C*>(t.p[c])[i];
      const double dx = double(a.x) - double(b.x), dy = double(a.y) - double(b.y);
      acc += w * (dx * dx + dy * dy);
      if (g.p[c]) static_cast<C*>(g.p[c])[i] = mk<C>(R(coef * dx), R(coef * dy));
    }
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w_ = 0; w_ < int(blockDim.x / 32); ++w_) s += red[w_];
    atomicAdd(loss, s);
  }
}

static unsigned nb(long long n) { return unsigned((n + 255) / 256); }

template <typename R> void launch_adj_spec(const AdjSpecArgs& a, cudaStream_t st) {
  const long long nm = (long long)(a.kc + 1) * (2 * a.kc + 1) * (a.D == 3 ? (2 * a.kc + 1) : 1);
  if (a.D == 3) k_adj_spec<R, 3><<<nb(nm), 256, 0, st>>>(a);
  else k_adj_spec<R, 2><<<nb(nm), 256, 0, st>>>(a);
}
template <typename R> void launch_adj_products(const AdjPhysArgs& a, cudaStream_t st) {
  if (a.D == 3) k_adj_products<R, 3><<<nb(a.npts), 256, 0, st>>>(a);
  else k_adj_products<R, 2><<<nb(a.npts), 256, 0, st>>>(a);
}
template <typename R> void launch_adj_acc(const AdjAccArgs& a, cudaStream_t st) {
  const long long nm = (long long)(a.kc + 1) * (2 * a.kc + 1) * (a.D == 3 ? (2 * a.kc + 1) : 1);
  if (a.D == 3) k_adj_acc<R, 3><<<nb(nm), 256, 0, st>>>(a);
  else k_adj_acc<R, 2><<<nb(nm), 256, 0, st>>>(a);
}
template <typename R> void launch_axpby(void* const* y, const void* const* x, double ax, double ay, int D,
                                        long long nm, cudaStream_t st) {
  Ptr3 yy{};
  CPtr3 xx{};
  for (int c = 0; c < D; ++c) { yy.p[c] = y[c]; xx.p[c] = x ? x[c] : nullptr; }
  k_axpby<R><<<nb(nm), 256, 0, st>>>(yy, xx, ax, ay, D, nm);
}
template <typename R> void launch_mse(const void* const* u, const void* const* t, void* const* g, double coef, int D,
                                      int kc, double* loss, cudaStream_t st) {
  CPtr3 uu{}, tt{};
  Ptr3 gg{};
  for (int c = 0; c < D; ++c) { uu.p[c] = u[c]; tt.p[c] = t[c]; gg.p[c] = g ? g[c] : nullptr; }
  const long long nm = (long long)(kc + 1) * (2 * kc + 1) * (D == 3 ? (2 * kc + 1) : 1);
  long long b = (nm + 255) / 256;
  if (b > 1024) b = 1024;
  k_mse<R><<<unsigned(b), 256, 0, st>>>(uu, tt, gg, coef, D, kc, loss);
}

#define SC_ADJ_INST(R)                                                                                         \
  template void launch_adj_spec<R>(const AdjSpecArgs&, cudaStream_t);                                          \
  template void launch_adj_products<R>(const AdjPhysArgs&, cudaStream_t);                                      \
  template void launch_adj_acc<R>(const AdjAccArgs&, cudaStream_t);                                            \
  template void launch_axpby<R>(void* const*, const void* const*, double, double, int, long long, cudaStream_t); \
  template void launch_mse<R>(const void* const*, const void* const*, void* const*, double, int, int, double*,  \
                              cudaStream_t);
SC_ADJ_INST(float)
SC_ADJ_INST(double)

}  // namespace sc
