// Seeded random initial field on the device: randomfield (src/solver.jl:576-641)
// with peak_profile (src/solver.jl:523), on the compact 2/3 cube.
//
// The steps of the reference, in FP64: complex normal coefficients (each part
// N(0, 1/2), Julia's complex randn), symmetrize! of the kx = 0 plane
// (src/solver.jl:398-430), project! (:350-368), twothirds! (:371-389, which
// also zeroes k = 0), and a per-shell rescale of floor|k| = s to
// totalenergy * profile(s) / sum profile (:610-640); modes outside the cube
// are zero before the rescale, so only the cube is drawn.  The coefficients
// come either from the caller (device arrays, e.g. drawn on the host with the
// same generator as symcode.fields) or from a counter-based generator here
// (splitmix64 of (seed, component, mode, part), Box-Muller), so that an 810^3
// field needs no host round trip.  Julia's Xoshiro stream is not reproduced.
#include <math.h>
#include <stdint.h>

#include "sc_fft.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

// splitmix64 (Steele, Lea and Flood; the seeding generator of the xoshiro family)
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// uniform in (0, 1] from the top 53 bits
__device__ __forceinline__ double unit53(uint64_t x) { return (double((x >> 11) + 1)) * (1.0 / 9007199254740992.0); }

// signed wavenumber of compact index p (0..k, then -k..-1)
__device__ __forceinline__ int kwave(int p, int kc) { return p <= kc ? p : p - (2 * kc + 1); }

__global__ void k_rf_draws(double2* u0, double2* u1, double2* u2, int D, long long nm, uint64_t seed) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  double2* u[3] = {u0, u1, u2};
  for (int c = 0; c < D; ++c) {
    const uint64_t key = splitmix64(seed ^ splitmix64(uint64_t(c) * 0x100000000000ull + uint64_t(m)));
    const double r = sqrt(-2.0 * log(unit53(splitmix64(key))));
    double sn, cs;
    sincospi(2.0 * unit53(splitmix64(key + 1)), &sn, &cs);
    // Box-Muller pair of N(0, 1), scaled to N(0, 1/2) per part
    u[c][m] = make_double2(0.7071067811865476 * r * cs, 0.7071067811865476 * r * sn);
  }
}

// symmetrize! on the kx = 0 plane: a mode whose partner (-ky, -kz) comes first
// in (kz, ky) FFT order takes the partner's conjugate; the partner itself is
// never written, so the update is in place.
__global__ void k_rf_hermitian(double2* u0, double2* u1, double2* u2, int D, int n, int K1, int kc) {
  const int K2 = 2 * kc + 1;
  const long long np = D == 3 ? (long long)K2 * K2 : K2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int py = int(i % K2), pz = D == 3 ? int(i / K2) : 0;
  const int ky = kwave(py, kc), kz = kwave(pz, kc);
  const int fy = (ky + n) % n, fz = (kz + n) % n;       // FFT indices
  const int gy = (n - fy) % n, gz = (n - fz) % n;       // partner's FFT indices
  const bool take = D == 3 ? (fy > gy || (fy == gy && fz > gz)) : fy > gy;
  double2* u[3] = {u0, u1, u2};
  if (take) {
    const int qy = -ky < 0 ? -ky + K2 : -ky, qz = -kz < 0 ? -kz + K2 : -kz;  // partner's compact indices
    const long long src = (long long)K1 * (qy + (long long)K2 * qz);
    const long long dst = (long long)K1 * (py + (long long)K2 * pz);
    for (int c = 0; c < D; ++c) u[c][dst] = make_double2(u[c][src].x, -u[c][src].y);
  }
}

// project! (k = 0 untouched) then twothirds!'s k = 0, and the shell energies
// with the RFFT double count of kx > 0: each block sums its shells in shared
// memory, then one FP64 atomic per shell and block
__device__ void rf_project_mode(double2* u0, double2* u1, double2* u2, int D, int K1, int kc, long long m,
                                double* ssh);

__global__ void k_rf_project(double2* u0, double2* u1, double2* u2, int D, int K1, int kc, int nshell,
                             double* eshell) {
  extern __shared__ double ssh[];
  for (int i = threadIdx.x; i < nshell; i += blockDim.x) ssh[i] = 0.0;
  __syncthreads();
  const int K2 = 2 * kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += (long long)gridDim.x * blockDim.x)
    rf_project_mode(u0, u1, u2, D, K1, kc, m, ssh);
  __syncthreads();
  for (int i = threadIdx.x; i < nshell; i += blockDim.x)
    if (ssh[i] != 0.0) atomicAdd(&eshell[i], ssh[i]);
}

__device__ void rf_project_mode(double2* u0, double2* u1, double2* u2, int D, int K1, int kc, long long m,
                                double* ssh) {
  const int K2 = 2 * kc + 1;
  const int ix = int(m % K1);
  const long long r = m / K1;
  const int iy = kwave(int(r % K2), kc), iz = D == 3 ? kwave(int(r / K2), kc) : 0;
  double2* u[3] = {u0, u1, u2};
  const double k[3] = {double(ix), double(iy), double(iz)};
  const long long k2 = (long long)ix * ix + (long long)iy * iy + (long long)iz * iz;
  if (k2 == 0) {
    for (int c = 0; c < D; ++c) u[c][m] = make_double2(0.0, 0.0);
    return;
  }
  double pr = 0, pi = 0;
  for (int c = 0; c < D; ++c) { pr += k[c] * u[c][m].x; pi += k[c] * u[c][m].y; }
  pr /= double(k2);
  pi /= double(k2);
  double e = 0;
  for (int c = 0; c < D; ++c) {
    const double2 v = make_double2(u[c][m].x - k[c] * pr, u[c][m].y - k[c] * pi);
    u[c][m] = v;
    e += v.x * v.x + v.y * v.y;
  }
  int s = int(sqrt(double(k2)));
  while ((long long)(s + 1) * (s + 1) <= k2) ++s;
  while ((long long)s * s > k2) --s;
  atomicAdd(&ssh[s], (ix > 0 ? 2.0 : 1.0) * 0.5 * e);
}

// rescale shell s by sqrt(target_s / E_s) and write the plan's precision
template <typename R>
__global__ void k_rf_scale(const double2* u0, const double2* u1, const double2* u2, R* o0, R* o1, R* o2, int D,
                           int K1, int kc, const double* eshell, const double* target) {
  using C = typename V2<R>::T;
  const int K2 = 2 * kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  const int ix = int(m % K1);
  const long long r = m / K1;
  const int iy = kwave(int(r % K2), kc), iz = D == 3 ? kwave(int(r / K2), kc) : 0;
  const long long k2 = (long long)ix * ix + (long long)iy * iy + (long long)iz * iz;
  int s = int(sqrt(double(k2)));
  while ((long long)(s + 1) * (s + 1) <= k2) ++s;
  while ((long long)s * s > k2) --s;
  const double f = eshell[s] > 0 ? sqrt(target[s] / eshell[s]) : 0.0;
  const double2* u[3] = {u0, u1, u2};
  C* o[3] = {reinterpret_cast<C*>(o0), reinterpret_cast<C*>(o1), reinterpret_cast<C*>(o2)};
  for (int c = 0; c < D; ++c) {
    C v;
    v.x = R(u[c][m].x * f);
    v.y = R(u[c][m].y * f);
    o[c][m] = v;
  }
}

unsigned nb(long long n) { return unsigned((n + 255) / 256); }

}  // namespace

void launch_random_draws(void* const* w, int D, int K1, int kc, unsigned long long seed, cudaStream_t st) {
  const long long nm = (long long)K1 * (2 * kc + 1) * (D == 3 ? 2 * kc + 1 : 1);
  double2* u[3] = {static_cast<double2*>(w[0]), static_cast<double2*>(w[1]),
                   static_cast<double2*>(D == 3 ? w[2] : w[1])};
  k_rf_draws<<<nb(nm), 256, 0, st>>>(u[0], u[1], u[2], D, nm, seed);
}

template <typename R>
void launch_random_finish(void* const* w, void* const* out, int D, int n, int K1, int kc, double* eshell,
                          const double* target, cudaStream_t st) {
  const int K2 = 2 * kc + 1;
  const long long nm = (long long)K1 * K2 * (D == 3 ? K2 : 1);
  double2* u[3] = {static_cast<double2*>(w[0]), static_cast<double2*>(w[1]),
                   static_cast<double2*>(D == 3 ? w[2] : w[1])};
  R* o[3] = {static_cast<R*>(out[0]), static_cast<R*>(out[1]), static_cast<R*>(D == 3 ? out[2] : out[1])};
  k_rf_hermitian<<<nb(D == 3 ? (long long)K2 * K2 : K2), 256, 0, st>>>(u[0], u[1], u[2], D, n, K1, kc);
  // shells 0 .. floor(sqrt(D) kc) hold the cube's modes
  const int smax = int(floor(sqrt(double(D)) * (n / 2)));  // the caller's eshell has smax + 1 entries
  int nshell = int(sqrt(double(D)) * kc) + 2;
  if (nshell > smax + 1) nshell = smax + 1;
  long long nbp = nb(nm);
  if (nbp > 148 * 8) nbp = 148 * 8;
  k_rf_project<<<unsigned(nbp), 256, nshell * sizeof(double), st>>>(u[0], u[1], u[2], D, K1, kc, nshell, eshell);
  k_rf_scale<R><<<nb(nm), 256, 0, st>>>(u[0], u[1], u[2], o[0], o[1], o[2], D, K1, kc, eshell, target);
}

template void launch_random_finish<float>(void* const*, void* const*, int, int, int, int, double*, const double*,
                                          cudaStream_t);
template void launch_random_finish<double>(void* const*, void* const*, int, int, int, int, double*, const double*,
                                           cudaStream_t);

}  // namespace sc
