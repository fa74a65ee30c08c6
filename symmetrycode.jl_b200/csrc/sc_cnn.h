// Internal interface of the tensor-core CNN closure (sc_cnn.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace sc {

struct TauPtrs {
  float* p[6];
};

struct CnnArgs {
  const void* u[3];            // physical velocity (FP32, 128^3)
  const __nv_bfloat16* w[4];   // packed weights per layer
  const float* b[4];           // biases per layer (padded)
  __nv_bfloat16* act0;         // [n^3][16]
  __nv_bfloat16* act1;         // [n^3][32]
  __nv_bfloat16* act2;         // [n^3][32]
  TauPtrs tau;                 // 6 physical FP32 outputs
  const double* a2;            // <|grad u|^2> (device, FP64)
  double* z;                   // device scalar for the Re_Delta channel
  double delta, nu, mu, sigma;
  int* err;                    // set to 1 when a bounded wait times out
  int nsm;
};

bool cnn_supported(int n, int D);
void cnn_init();
void launch_cnn_forward(const CnnArgs& a, cudaStream_t st);
// *z = (log(delta^2 sqrt(*a2) / nu) - mu) / sigma
void launch_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma, cudaStream_t st);

}  // namespace sc
