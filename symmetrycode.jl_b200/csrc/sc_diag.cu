// Device reductions for the a-posteriori diagnostics of an LES state
// (reduce! in solve_les!, src/les.jl:94-148), all accumulated in FP64:
//  - k_epost: ||u - twothirds(u_ref)||^2 and ||twothirds(u_ref)||^2 over the
//    stored RFFT arrays (no conjugate weights: the reference's `norm`);
//  - k_sfs_diag: on the retained (compact) modes, with tau_dev the trace-free
//    closure stress spectrum and S = i/2 (k_j u_i + k_i u_j):
//      eps = sum w Re(tau_dev : conj S)       (Parseval for mean(tau_dev : S))
//      T[shell] += w Re(conj(u_i) (-i k_j tau_dev_ij)),
//    w = 2 for interior kx (the conjugate half of the RFFT), shells
//    i <= |k| < i+1 as in spectrum (src/solver.jl:664-699, 1080-1129).
#include "sc_fft.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < int(blockDim.x / 32); ++w) s += red[w];
  __syncthreads();
  return s;
}

template <typename R>
__global__ void k_epost(const DiagArgs a, double* sums) {
  using C = typename V2<R>::T;
  __shared__ double red[32];
  const int nx = a.n / 2 + 1;
  const long long nm = (long long)nx * a.n * (a.D == 3 ? a.n : 1);
  double dd = 0, rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const int ix = int(i % nx);
    const long long r = i / nx;
    const int iy = int(r % a.n), iz = a.D == 3 ? int(r / a.n) : 0;
    const int ky = iy <= a.n / 2 ? iy : iy - a.n, kz = iz <= a.n / 2 ? iz : iz - a.n;
    const bool keep = ix <= a.kc && abs(ky) <= a.kc && abs(kz) <= a.kc && (ix | ky | kz) != 0;
    for (int c = 0; c < a.D; ++c) {
      const C u = static_cast<const C*>(a.u[c])[i];
      C v = static_cast<const C*>(a.uref[c])[i];
      if (!keep) v = mk<C>(R(0), R(0));
      const double dx = double(u.x) - double(v.x), dy = double(u.y) - double(v.y);
      dd += dx * dx + dy * dy;
      rr += double(v.x) * v.x + double(v.y) * v.y;
    }
  }
  dd = block_sum(dd, red);
  rr = block_sum(rr, red);
  if (threadIdx.x == 0) { atomicAdd(&sums[0], dd); atomicAdd(&sums[1], rr); }
}

template <typename R>
__global__ void k_sfs_diag(const DiagArgs a, int nshell, double* eps, double* T) {
  using C = typename V2<R>::T;
  extern __shared__ double sh[];  // [nshell]
  __shared__ double red[32];
  for (int i = threadIdx.x; i < nshell; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int D = a.D, kc = a.kc, K1 = kc + 1, K2 = 2 * kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  double e = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const int ix = int(i % K1);
    const long long r = i / K1;
    const int py = int(r % K2), pz = D == 3 ? int(r / K2) : 0;
    const int ky = py <= kc ? py : py - K2, kz = pz <= kc ? pz : pz - K2;
    const double k[3] = {a.kfac * ix, a.kfac * ky, a.kfac * kz};
    double ur[3], ui[3];
    for (int c = 0; c < D; ++c) {
      const C v = static_cast<const C*>(a.u[c])[i];
      ur[c] = v.x; ui[c] = v.y;
    }
    // trace-free stress, full symmetric matrix
    double tr[3][3], ti[3][3];
    const int NP = D == 3 ? 6 : 3;
    const int pi[6] = {0, 1, 2, 0, 1, 2}, pj3[6] = {0, 1, 2, 1, 2, 0};
    const int pi2[3] = {0, 1, 0}, pj2[3] = {0, 1, 1};
    for (int m = 0; m < NP; ++m) {
      const C v = static_cast<const C*>(a.th[m])[i];
      const int ii = D == 3 ? pi[m] : pi2[m], jj = D == 3 ? pj3[m] : pj2[m];
      tr[ii][jj] = tr[jj][ii] = v.x;
      ti[ii][jj] = ti[jj][ii] = v.y;
    }
    double trr = 0, tri = 0;
    for (int c = 0; c < D; ++c) { trr += tr[c][c]; tri += ti[c][c]; }
    for (int c = 0; c < D; ++c) { tr[c][c] -= trr / D; ti[c][c] -= tri / D; }
    const double w = ix > 0 ? 2.0 : 1.0;
    // tau_dev : conj(S), S_ij = i/2 (k_j u_i + k_i u_j); Re(tau conj(i s)) = tau_r (-s_i)... use S = i q, q real-linear
    double c_ = 0;
    for (int ii = 0; ii < D; ++ii)
      for (int jj = 0; jj < D; ++jj) {
        const double qr = 0.5 * (k[jj] * ur[ii] + k[ii] * ur[jj]), qi = 0.5 * (k[jj] * ui[ii] + k[ii] * ui[jj]);
        // S = i q = (-qi, qr); Re(conj(tau) S) = tau_r (-qi) + tau_i qr
        c_ += tr[ii][jj] * (-qi) + ti[ii][jj] * qr;
      }
    e += w * c_;
    // transfer: clo_i = -i sum_j k_j tau_ij = (sum k_j tau_i_ij, -sum k_j tau_r_ij)
    double t = 0;
    for (int ii = 0; ii < D; ++ii) {
      double sr = 0, si = 0;
      for (int jj = 0; jj < D; ++jj) { sr += k[jj] * tr[ii][jj]; si += k[jj] * ti[ii][jj]; }
      const double cr = si, ci = -sr;
      t += ur[ii] * cr + ui[ii] * ci;
    }
    const long long k2 = (long long)ix * ix + (long long)ky * ky + (long long)kz * kz;
    int s = int(sqrt(double(k2)));
    while ((long long)(s + 1) * (s + 1) <= k2) ++s;
    while ((long long)s * s > k2) --s;
    if (s >= 1 && s <= nshell) atomicAdd(&sh[s - 1], w * t);
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) atomicAdd(eps, e);
  __syncthreads();
  for (int i = threadIdx.x; i < nshell; i += blockDim.x)
    if (sh[i] != 0.0) atomicAdd(&T[i], sh[i]);
}

}  // namespace

template <typename R> void launch_epost(const DiagArgs& a, double* sums, cudaStream_t st) {
  const long long nm = (long long)(a.n / 2 + 1) * a.n * (a.D == 3 ? a.n : 1);
  long long nb = (nm + 255) / 256;
  if (nb > 148 * 8) nb = 148 * 8;
  k_epost<R><<<unsigned(nb), 256, 0, st>>>(a, sums);
}

template <typename R> void launch_sfs_diag(const DiagArgs& a, int nshell, double* eps, double* T, cudaStream_t st) {
  const long long K2 = 2 * a.kc + 1;
  const long long nm = (long long)(a.kc + 1) * K2 * (a.D == 3 ? K2 : 1);
  long long nb = (nm + 255) / 256;
  if (nb > 148 * 4) nb = 148 * 4;
  k_sfs_diag<R><<<unsigned(nb), 256, size_t(nshell > 0 ? nshell : 1) * sizeof(double), st>>>(a, nshell, eps, T);
}

template void launch_epost<float>(const DiagArgs&, double*, cudaStream_t);
template void launch_epost<double>(const DiagArgs&, double*, cudaStream_t);
template void launch_sfs_diag<float>(const DiagArgs&, int, double*, double*, cudaStream_t);
template void launch_sfs_diag<double>(const DiagArgs&, int, double*, double*, cudaStream_t);

}  // namespace sc
