// Internal interface of the tensor-core CNN closure (sc_cnn.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace sc {

struct TauPtrs {
  float* p[6];
};

struct GinPtrs {
  float* p[4];
};

struct CnnArgs {
  int n;                       // 64 or 128
  const void* u[3];            // physical velocity (FP32, n^3)
  const __nv_bfloat16* w[4];   // packed weights per layer
  const float* b[4];           // biases per layer (padded)
  __nv_bfloat16* act0;         // [n^3][16]
  __nv_bfloat16* act1;         // [n^3][32]
  __nv_bfloat16* act2;         // [n^3][32]
  __nv_bfloat16* act3;         // [n^3][32] input of layer 4; null: act1 is reused
  float* pre[3];               // FP32 [n^3][32] pre-activations of layers 1-3 (kept for the adjoint), or null
  TauPtrs tau;                 // 6 physical FP32 outputs
  const double* a2;            // <|grad u|^2> (device, FP64)
  double* z;                   // device scalar for the Re_Delta channel
  double delta, nu, mu, sigma;
  int* err;                    // set to 1 when a bounded wait times out
  int nsm;
  long long wait_limit;        // polls of each mbarrier wait before it gives up (kDefaultWaitLimit)
  // split precision (split = true): every layer is three MMA passes over FP16
  // hi/lo operands, A_hi W_hi + A_lo W_hi + A_hi W_lo, accumulated in FP32
  bool split;
  const __half* wh[4];         // FP16 high parts of the forward weights (x kSplitScale), same layout as w
  const __half* wl[4];         // FP16 low parts
  __half* acth[4];             // FP16 high parts of the layer inputs act0..act3 ([n^3][16], [n^3][32] x 3)
  __half* actl[4];             // FP16 low parts
  float* acc;                  // FP32 [n^3][32] accumulator of the layers whose pre[l] is null (and of layer 4)
};

// The FP16 forward weights of the split precision are stored x kSplitScale (a
// power of two, so exactly) so that their low parts stay normal FP16 numbers;
// the accumulator is scaled back in the last pass's epilogue.
constexpr float kSplitScale = 64.f;

// Default bound of the CNN kernels' mbarrier waits (polls of try_wait).
constexpr long long kDefaultWaitLimit = 1ll << 26;

// Backward pass of the network after a forward pass that kept act0..act3 and
// the pre-activations: from dL/dtau to dL/d(input channels) and the weight and
// bias gradients (accumulated in FP64 into gw at the flat offsets woff[l]:
// [Cout][Cin][27] weights, then [Cout] biases, PyTorch order).
struct CnnBwdArgs {
  int n;
  TauPtrs gtau;                       // dL/dtau, 6 planar FP32
  const __nv_bfloat16* wt[4];         // packed transposed, flipped weights per layer
  const __nv_bfloat16* act[4];        // layer inputs (BF16 channels-last)
  const float* pre[3];                // pre-activations h1..h3
  __nv_bfloat16* gbf;                 // scratch BF16 [n^3][32]
  float* gf;                          // scratch FP32 [n^3][32]
  GinPtrs gin_planar;                 // out: dL/d(u_x, u_y, u_z, z channel), planar FP32
  double* gw;
  long long woff[4];
  int* err;
  int nsm;
  long long wait_limit;
  // split precision: BF16 hi/lo gradients and transposed weights, FP16 hi/lo layer inputs
  bool split;
  const __nv_bfloat16* wtl[4];        // BF16 low parts of wt
  const __half* acth[4];              // FP16 layer inputs (high parts)
  const __half* actl[4];              // FP16 layer inputs (low parts)
  __nv_bfloat16* gbf_lo;              // scratch BF16 [n^3][32], low parts of gbf
};

// An encoded tensor map (CUtensorMap, 128 bytes) for the bulk tensor copies
// that stage the convolutions' input rows; one per 8-channel chunk.
struct alignas(64) TmaMap {
  unsigned char b[128];
};
struct ConvMaps {
  TmaMap m[4];
};
// Encodes a 4D BF16 tiled tensor map (dims innermost first, strides of dims
// 1..3 in bytes); false when the driver entry point or the encoding fails.
// Implemented beside the column sweeps' maps (sc_coltma.cu).
bool tma_encode_bf16_4d(TmaMap* map, const void* base, const unsigned long long dims[4],
                        const unsigned long long strides[3], const unsigned box[4]);

bool cnn_supported(int n, int D);
void cnn_init();
void launch_cnn_forward(const CnnArgs& a, cudaStream_t st);
void launch_cnn_backward(const CnnBwdArgs& a, cudaStream_t st);
// *z = (log(delta^2 sqrt(*a2) / nu) - mu) / sigma
void launch_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma, cudaStream_t st);

}  // namespace sc
