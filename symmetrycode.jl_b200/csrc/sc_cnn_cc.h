// Internal interface of the CUDA-core CNN (sc_cnn_cc.cu) and the adjoint kernels (sc_adjoint.cu).
#pragma once
#include <cuda_runtime.h>

namespace sc {

struct ConvArgs {
  const void* in;   // [cin][npts] layer input (forward) / layer input for the weight gradient
  const void* w;    // [cout][cin][27]
  const void* b;    // [cout] or nullptr
  void* out;        // [cout][npts] forward output / gradient w.r.t. the output (backward)
  void* in_grad;    // [cin][npts] gradient w.r.t. the input (backward; nullptr: skip)
  int n, cin, cout;
};

template <typename R> void launch_conv_fwd(const ConvArgs& a, cudaStream_t st);
// accumulates (atomically, FP64) into gw [cout][cin][27] and gb [cout] when non-null
template <typename R> void launch_conv_bwd(const ConvArgs& a, double* gw, double* gb, cudaStream_t st);
template <typename R> void launch_gelu(const R* pre, R* post, long long n, cudaStream_t st);
template <typename R> void launch_gelu_bwd(const R* pre, R* g, long long n, cudaStream_t st);
template <typename R> void launch_cc_input(const R* vx, const R* vy, const R* vz, const double* z, R* a0,
                                           long long npts, cudaStream_t st);
template <typename R> void launch_sum(const R* x, long long n, double* s, cudaStream_t st);

// ---- adjoint of the LES right-hand side (sc_adjoint.cu) ----------------------
struct AdjSpecArgs {
  const void* lam[3];   // adjoint of the stage derivative (compact)
  const void* u[3];     // stage input (compact)
  void* lsig[6];        // out: adjoint of the stress spectra (compact)
  void* mu[3];          // out: viscous part of the adjoint (compact)
  int D, kc;
  double kfac, visc;
};
template <typename R> void launch_adj_spec(const AdjSpecArgs& a, cudaStream_t st);

struct AdjPhysArgs {
  const void* v[3];     // physical velocity of the stage
  const void* m[6];     // physical adjoint of sigma (T(lsig), unnormalised)
  const void* add[3];   // optional extra physical adjoint of v (CNN input gradient) or nullptr
  void* lv[3];          // out: physical adjoint of v
  int D;
  long long npts;
  double inv_npts;      // 1/N applied to m
};
template <typename R> void launch_adj_products(const AdjPhysArgs& a, cudaStream_t st);

// mu += scale * (x with k = 0 zeroed) + zc * k^2 u, zc = *lamz / (sigma * *a2) (when lamz != nullptr)
struct AdjAccArgs {
  void* mu[3];
  const void* x[3];
  const void* u[3];
  const double* lamz;
  const double* a2;
  double sigma, scale, kfac;
  int D, kc;
};
template <typename R> void launch_adj_acc(const AdjAccArgs& a, cudaStream_t st);

// y = ax * x + ay * y on D compact components (x may be nullptr: y = ay * y)
template <typename R> void launch_axpby(void* const* y, const void* const* x, double ax, double ay, int D,
                                        long long nm, cudaStream_t st);
// loss += sum_k w |u - t|^2; g = coef * (u - t) (g may be nullptr)
template <typename R> void launch_mse(const void* const* u, const void* const* t, void* const* g, double coef, int D,
                                      int kc, double* loss, cudaStream_t st);

}  // namespace sc
