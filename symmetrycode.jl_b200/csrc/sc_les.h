// Internal interface of the LES closure kernels (sc_les.cu).
#pragma once
#include <cuda_runtime.h>

namespace sc {

// closure kinds (values match include/symcode.h SC_CLOSURE_*)
enum { kNoClosure = 0, kClark = 1, kSmagorinsky = 2, kVerstappen = 3, kDynSmagorinsky = 4, kBardina = 5, kCnn = 6,
       kCnnFp = 7, kMlp = 8, kTbnn = 9 };

struct LesSpecArgs {
  const void* in[9];
  void* out[9];
  int ncomp;
  int kc;             // compact half-width
  long long nmodes;   // (kc+1) (2kc+1)^(D-1)
  double kfac;        // 2 pi / l
  double delta;       // Gaussian width (spec_filter), <= 0: none
  double scale;       // spec_filter: constant factor
  const double* dscale;  // spec_filter: optional device factor
};

struct LesPhysArgs {
  const void* in[9];
  const void* in2[3];
  const void* in3[6];
  const void* in4[6];
  void* out[6];
  long long npts;
  int kind;       // closure kind (k_closure_pt) / trace-free flag (k_sub_products)
  double delta;
  double p0;      // C_s (Smagorinsky) or C (Verstappen)
};

template <typename R> void launch_grad(const LesSpecArgs& a, int D, cudaStream_t st);
template <typename R> void launch_strain(const LesSpecArgs& a, int D, cudaStream_t st);
template <typename R> void launch_spec_filter(const LesSpecArgs& a, int D, cudaStream_t st);
template <typename R> void launch_closure_pt(const LesPhysArgs& a, int D, cudaStream_t st);
template <typename R> void launch_smag_tensor(const LesPhysArgs& a, int D, cudaStream_t st);
template <typename R> void launch_sub_products(const LesPhysArgs& a, int D, cudaStream_t st);
// accumulates sum(M:L), sum(M:M) into sums[0..1] (zero them first) and sets sums[2] = c
template <typename R> void launch_dynsmag_mlmm(const LesPhysArgs& a, int D, double* sums, cudaStream_t st);

// pointwise MLP closure (sc_mlp.cu): fullchain(mlp) of src/nets.jl:311-331
constexpr int kMlpMaxWidth = 128;
constexpr int kMlpMaxLayers = 8;
struct MlpArgs {
  const void* G[9];   // physical VGT, channel a + D b = d_b u_a
  void* tau[6];       // physical tau, pair order
  long long npts;
  int D, nl;
  int w[kMlpMaxLayers + 1];  // widths: w[0] = D^2 (+1 with the Re_Delta channel) ... w[nl] = 3 | 6
  const void* theta;  // per layer W[c_out][c_in], then b[c_out] (all layers but the last)
  double delta;
  const double* z;    // set by launch_mlp
  int mode;           // 0: fullchain(mlp); 1: tbnn (invariants in, basis coefficients out)
};
// zbuf: two device doubles when the Re_Delta channel is used, else null
template <typename R>
void launch_mlp(const MlpArgs& a, double* zbuf, double nu, double mu, double sigma, cudaStream_t st);

}  // namespace sc
