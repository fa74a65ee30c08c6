// Internal launch interface between the C ABI (sc_api.cu) and the kernels (sc_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace sc {

constexpr int kMaxComp = 12;

// A batched 1D transform along a strided axis ("column sweep").  Element
// (kx, c, e) of component q lives at in[q][kx + c*in_cs + e*in_es]; NPEN
// consecutive kx form one tile.  Along the transform axis only the compact
// index set {0..kpos-1} U {N-kneg..N-1} of FFT indices is stored (at compact
// positions 0..kpos+kneg-1): it is zero-padded on input (inverse) or pruned on
// output (forward).
struct ColArgs {
  const void* in[kMaxComp];
  void* out[kMaxComp];
  int ncomp;
  int K1;     // number of kx (tile axis extent)
  int ncols;  // number of columns c
  long long in_cs, in_es, out_cs, out_es;
  int kpos, kneg;     // compact mapping of the transform axis
  int zero_origin;    // inverse only: treat (kx, c, e) = (0, 0, 0) as zero (k = 0 mode)
  // optional derivative outputs (inverse only): out[ncomp + j] = transform of
  // (i * kfac * k_e) * in[deriv_src[j]] where k_e is the signed wavenumber of
  // compact position e; ndrv = 0 disables
  int ndrv;
  int drv_src[kMaxComp];
  double kfac;
  int variant;  // FP32 fast sizes: kernel variant chosen by the autotuner (0 = default)
  // bounded device waits of the TMA-fed sweeps: polls before a wait gives up
  // and the plan's device error word it then sets (nullptr: no TMA sweep)
  long long wait_limit;
  int* err;
};

// The x sweep of the Navier-Stokes right-hand side: per row (y[, z]) read the
// D velocity components' kx row (kx = 0..K1in-1), c2r to physical space,
// form the symmetric products u_i u_j scaled by `scale`, r2c and store the
// first K1out kx of each product row.
struct XArgs {
  const void* in[3];
  void* out[6];
  int D;
  int K1in, K1out;
  long long nrows;
  double scale;
  int variant;  // FP32 fast sizes: kernel variant chosen by the autotuner (0 = default)
  int ldo;      // row stride of the outputs (elements; 0: K1out)
};

// Plain batched c2r / r2c along x for `ncomp` rows-of-fields (FFT API).
struct XPlainArgs {
  const void* in[kMaxComp];
  void* out[kMaxComp];
  int ncomp;
  int K1;          // spectral row extent (kx = 0..K1-1)
  long long nrows;
  double scale;    // applied to the output
};

// Pointwise spectral epilogue over the compact 2/3 cube (see k_epilogue).
struct EpiArgs {
  const void* sig[6];   // compact product spectra F[u_i u_j]/n^D, pair order of `pairs`
  const void* us[3];    // stage input (viscous term, forcing)
  const void* base_a[3];
  void* out_a[3];
  const void* base_b[3];
  void* out_b[3];
  int D;
  int K1, K2, kc;       // compact extents, kc = n/3
  double kfac;          // 2 pi / l
  double visc;
  double ca, cb;        // out_a = P?(base_a + ca*k), out_b = base_b + cb*k
  int proj_k;           // project the derivative k (RK4)
  int proj_a;           // project out_a (Wray3)
  int has_b;
  const double* forcing;  // device scalar A (nullptr: no forcing)
  const void* sig2[6];    // optional second stress spectrum added to sig (closure stress)
  int has_sig2;
  // mix_a: the base of out_a is base_b + mix (us - base_b) instead of base_a
  // (RK4 stage 2 rebuilds the accumulator from the stage input it reads
  // anyway); out_a[c] == nullptr: out_a is not written
  int mix_a;
  double mix;
};

struct PackArgs {
  const void* src[kMaxComp];
  void* dst[kMaxComp];
  int ncomp;
  int D, n;
  int kc;  // compact half-width
};

// DNS -> LES filter on the LES compact cube (sfs!, src/data.jl:625-642).
struct FilterArgs {
  const void* udns[3];  // DNS compact state (half-width kcd)
  const void* sig1[6];  // DNS product spectra on the LES compact cube
  void* ubar[3];        // LES compact filtered velocity
  void* tau[6];         // in: LES product spectra of ubar; out: tau (in place)
  int D;
  int kcd, kcl;         // DNS / LES compact half-widths
  double kfac, delta;   // delta <= 0: no Gaussian
  int pass;             // 0: ubar, 1: tau
};

template <typename R> bool launch_col_inv(int N, const ColArgs& a, const void* tw, cudaStream_t st);
template <typename R> bool launch_col_fwd(int N, const ColArgs& a, const void* tw, cudaStream_t st);
template <typename R> bool launch_xsweep_ns(int N, const XArgs& a, const void* tw, cudaStream_t st);
template <typename R> bool launch_x_c2r(int N, const XPlainArgs& a, const void* tw, cudaStream_t st);
template <typename R> bool launch_x_r2c(int N, const XPlainArgs& a, const void* tw, cudaStream_t st);
template <typename R> void launch_epilogue(const EpiArgs& a, cudaStream_t st);
template <typename R> void launch_filter(const FilterArgs& a, cudaStream_t st);
// max |u| over the physical points of D rows-of-spectra (x inverse fused with the reduction)
template <typename R> bool launch_x_vmax(int N, const XPlainArgs& a, const void* tw, unsigned long long* out,
                                         cudaStream_t st);
// shells 1..2 on the compact state held in a.dst: mode 0 measures into eref[0..1], mode 1 rescales
template <typename R> void launch_shell_clamp(const PackArgs& a, double* eref, int mode, cudaStream_t st);
template <typename R> void launch_spectrum(const PackArgs& a, int nshell, double* s, cudaStream_t st);
template <typename R> void launch_pack(const PackArgs& a, cudaStream_t st);
template <typename R> void launch_unpack(const PackArgs& a, cudaStream_t st);
// forcing coefficient A = eps / (2 E_band) of the compact state u into *A
template <typename R> void launch_band_forcing(const void* const* u, int D, int K1, int K2, int kc,
                                               double eps, double* A, cudaStream_t st);
// FP64 sum over a spectral array of w(kx) * |u|^2 (w = 1 at kx = 0 and kx = n/2, else 2),
// optionally times nu*k^2; accumulated (atomically) into *out.
template <typename R> void launch_spectral_energy(const void* const* u, int ncomp, int D, int n,
                                                  int K1, int K2, int compact, int kc,
                                                  double kfac, int weight_k2, double* out,
                                                  cudaStream_t st, int mask23 = 0);
bool fft_size_supported(int n);
// two-level FP32 engine (sc_fast.cu) for N in {64, 128, 256, 810}
bool fast_supported(int N);
bool init_fast(int N);
bool launch_col2(int N, bool inv, const ColArgs& a, const void* tw, cudaStream_t st);
bool launch_xsweep2(int N, const XArgs& a, const void* tw, cudaStream_t st);
// randomfield on the device (sc_random.cu): counter-based N(0, 1/2) draws into
// the FP64 compact work arrays w, then symmetrize!, project!, twothirds! and
// the per-shell rescale to target[s] (eshell: smax + 1 zeroed doubles) into
// the compact arrays out of the plan's precision
void launch_random_draws(void* const* w, int D, int K1, int kc, unsigned long long seed, cudaStream_t st);
template <typename R>
void launch_random_finish(void* const* w, void* const* out, int D, int n, int K1, int kc, double* eshell,
                          const double* target, cudaStream_t st);
// FP32 plain c2r (inv) / r2c along x for the fast sizes (sc_fast.cu); false when not applicable
bool launch_xplain_fast(int N, bool inv, const XPlainArgs& a, const void* tw, cudaStream_t st);
// number of autotuner variants of the FP32 column sweeps / 3D x sweep of size N
int col2_variants(int N);
// TMA-fed persistent column sweeps for N = 810 (sc_coltma.cu): column-sweep
// variants kColTmaVariant + which, which < kColTmaConfigs; false when the
// geometry does not allow them (the caller then launches k_col2)
constexpr int kColTmaVariant = 4, kColTmaConfigs = 3;
bool colt_init();
bool launch_colt(int N, bool inv, const ColArgs& a, const void* tw, int which, cudaStream_t st);
int xsweep_variants(int N, int D);
// FP32 n = 810 x sweep on paired rows (sc_xpair.cu).  Its twiddles are the
// plain table's exp(-2 pi i j / 810) as register-pair entries
// (c, c, s, s, -s, -s, 0, 0), stored in the same device buffer right after the
// plain table (byte offset 810 * 8).
size_t xpair810_twiddle_bytes();
void xpair810_twiddles(const float2* tw, float* out8);
bool init_xpair810();
void launch_xpair810(const XArgs& a, const void* twp_table, int minb, cudaStream_t st);
// bytes of a plan's twiddle buffer: the plain table plus, for FP32 n = 810, the pair table
inline size_t twiddle_buffer_bytes(int n, size_t esz) {
  return (size_t)n * esz + (esz == 8 && n == 810 ? xpair810_twiddle_bytes() : 0);
}
template <typename R> bool init_kernels(int N);
template <typename R> void launch_twothirds_full(const PackArgs& a, cudaStream_t st);  // in place on a.dst
template <typename R> void launch_project_full(const PackArgs& a, double kfac, cudaStream_t st);

// Records "what: detail" (or "what") as the thread's last error string and returns code.
int api_fail(int code, const char* what, const char* detail);

// a-posteriori diagnostics of an LES state (sc_diag.cu)
struct DiagArgs {
  const void* u[3];     // compact state (sfs) or full layout (epost)
  const void* uref[3];  // full layout (epost)
  const void* th[6];    // compact closure stress spectrum (sfs)
  int D, n, kc;
  double kfac;
};
// sums[0] += ||u - twothirds(uref)||^2, sums[1] += ||twothirds(uref)||^2 (zero them first)
template <typename R> void launch_epost(const DiagArgs& a, double* sums, cudaStream_t st);
// *eps += sum w Re(tau_dev : conj S); T[0..nshell-1] += shell transfer (zero them first)
template <typename R> void launch_sfs_diag(const DiagArgs& a, int nshell, double* eps, double* T, cudaStream_t st);

}  // namespace sc
