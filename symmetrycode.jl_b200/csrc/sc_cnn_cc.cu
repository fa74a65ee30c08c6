// CUDA-core CNN closure in FP32 or FP64 (any grid size): forward with stored
// pre-activations, and the backward pass (input gradient, weight and bias
// gradients) used by the hand-written adjoint of the LES rollout.  The same
// network as the tensor-core closure (sc_cnn.cu) without BF16 rounding, so
// that its derivatives are the derivatives of the computed function.
//
// Activations are planar, act[c * npts + v], v = x + n (y + n z); weights are
// in the PyTorch conv3d layout w[co][ci][kz][ky][kx] (tap t = kz 9 + ky 3 + kx,
// a cross-correlation with periodic wrap).
#include <math.h>

#include "sc_cnn_cc.h"

namespace sc {

template <typename R> struct Acc;
template <> struct Acc<float> { using T = float; };
template <> struct Acc<double> { using T = double; };

__device__ __forceinline__ long long nbr(long long v, int n, int t, int sign) {
  const int x = int(v % n), y = int((v / n) % n), z = int(v / ((long long)n * n));
  const int dz = (t / 9 - 1) * sign, dy = ((t / 3) % 3 - 1) * sign, dx = (t % 3 - 1) * sign;
  const int xx = (x + dx + n) % n, yy = (y + dy + n) % n, zz = (z + dz + n) % n;
  return xx + (long long)n * (yy + (long long)n * zz);
}

// out[co][v] = b[co] + sum_{ci, t} w[co][ci][t] in[ci][v + off(t)]
template <typename R>
__global__ void k_conv_fwd(const ConvArgs a) {
  const long long npts = (long long)a.n * a.n * a.n;
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= npts) return;
  const R* in = static_cast<const R*>(a.in);
  const R* w = static_cast<const R*>(a.w);
  R acc[32];
#pragma unroll
  for (int co = 0; co < 32; ++co) acc[co] = (co < a.cout && a.b) ? static_cast<const R*>(a.b)[co] : R(0);
  for (int t = 0; t < 27; ++t) {
    const long long q = nbr(v, a.n, t, 1);
    for (int ci = 0; ci < a.cin; ++ci) {
      const R x = in[ci * npts + q];
#pragma unroll
      for (int co = 0; co < 32; ++co)
        if (co < a.cout) acc[co] += __ldg(&w[(co * a.cin + ci) * 27 + t]) * x;
    }
  }
  R* out = static_cast<R*>(a.out);
#pragma unroll
  for (int co = 0; co < 32; ++co)
    if (co < a.cout) out[co * npts + v] = acc[co];
}

// gin[ci][v] = sum_{co, t} w[co][ci][t] gout[co][v - off(t)]   (the transposed correlation)
template <typename R>
__global__ void k_conv_bwd_in(const ConvArgs a) {
  const long long npts = (long long)a.n * a.n * a.n;
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= npts) return;
  const R* g = static_cast<const R*>(a.out);
  const R* w = static_cast<const R*>(a.w);
  R acc[32];
#pragma unroll
  for (int ci = 0; ci < 32; ++ci) acc[ci] = R(0);
  for (int t = 0; t < 27; ++t) {
    const long long q = nbr(v, a.n, t, -1);
    for (int co = 0; co < a.cout; ++co) {
      const R y = g[co * npts + q];
#pragma unroll
      for (int ci = 0; ci < 32; ++ci)
        if (ci < a.cin) acc[ci] += __ldg(&w[(co * a.cin + ci) * 27 + t]) * y;
    }
  }
  R* gin = static_cast<R*>(a.in_grad);
#pragma unroll
  for (int ci = 0; ci < 32; ++ci)
    if (ci < a.cin) gin[ci * npts + v] = acc[ci];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// gw[co][ci][t] += sum_v gout[co][v] in[ci][v + off(t)];  block (ci * 27 + t, chunk)
template <typename R>
__global__ void k_conv_bwd_w(const ConvArgs a, double* gw) {
  const long long npts = (long long)a.n * a.n * a.n;
  const int ci = blockIdx.x / 27, t = blockIdx.x % 27;
  const R* g = static_cast<const R*>(a.out);
  const R* in = static_cast<const R*>(a.in);
  double acc[32];
#pragma unroll
  for (int co = 0; co < 32; ++co) acc[co] = 0;
  for (long long v = (long long)blockIdx.y * blockDim.x + threadIdx.x; v < npts; v += (long long)gridDim.y * blockDim.x) {
    const double x = double(in[ci * npts + nbr(v, a.n, t, 1)]);
#pragma unroll
    for (int co = 0; co < 32; ++co)
      if (co < a.cout) acc[co] += double(g[co * npts + v]) * x;
  }
  __shared__ double red[32][33];
  const int lane = threadIdx.x % 32, wid = threadIdx.x / 32;
#pragma unroll
  for (int co = 0; co < 32; ++co) {
    const double s = warp_sum(acc[co]);
    if (lane == 0) red[co][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < 32 && threadIdx.x < a.cout) {
    double s = 0;
    for (int w_ = 0; w_ < int(blockDim.x / 32); ++w_) s += red[threadIdx.x][w_];
    atomicAdd(&gw[(threadIdx.x * a.cin + ci) * 27 + t], s);
  }
}

// gb[co] += sum_v gout[co][v]
template <typename R>
__global__ void k_bias_grad(const ConvArgs a, double* gb) {
  const long long npts = (long long)a.n * a.n * a.n;
  const int co = blockIdx.x;
  const R* g = static_cast<const R*>(a.out);
  double s = 0;
  for (long long v = (long long)blockIdx.y * blockDim.x + threadIdx.x; v < npts; v += (long long)gridDim.y * blockDim.x)
    s += double(g[co * npts + v]);
  __shared__ double red[32];
  s = warp_sum(s);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0;
    for (int w_ = 0; w_ < int(blockDim.x / 32); ++w_) tot += red[w_];
    atomicAdd(&gb[co], tot);
  }
}

// GELU in the tanh form of NNlib's gelu (the activation of the reference's nets)
// and its derivative: u = c (x + a x^3), gelu = x (1 + tanh u) / 2,
// gelu' = (1 + tanh u) / 2 + x (1 - tanh^2 u) c (1 + 3 a x^2) / 2
template <typename R>
__global__ void k_gelu(const R* pre, R* post, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const R x = pre[i];
  const R u = R(0.79788456080286535588) * (x + R(0.044715) * x * x * x);
  post[i] = R(0.5) * x * (R(1) + tanh(u));
}

template <typename R>
__global__ void k_gelu_bwd(const R* pre, R* g, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const R x = pre[i];
  const R c = R(0.79788456080286535588), a = R(0.044715);
  const R t = tanh(c * (x + a * x * x * x));
  g[i] *= R(0.5) * (R(1) + t) + R(0.5) * x * (R(1) - t * t) * c * (R(1) + R(3) * a * x * x);
}

// a0 = [v_x, v_y, v_z, z] (planar, 4 channels)
template <typename R>
__global__ void k_cc_input(const R* vx, const R* vy, const R* vz, const double* z, R* a0, long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  a0[i] = vx[i];
  a0[npts + i] = vy[i];
  a0[2 * npts + i] = vz[i];
  a0[3 * npts + i] = R(*z);
}

// *s += sum_i x[i]
template <typename R>
__global__ void k_sum(const R* x, long long n, double* s) {
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += double(x[i]);
  __shared__ double red[32];
  acc = warp_sum(acc);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0;
    for (int w_ = 0; w_ < int(blockDim.x / 32); ++w_) tot += red[w_];
    atomicAdd(s, tot);
  }
}

static unsigned nblk(long long n) { return unsigned((n + 255) / 256); }

template <typename R> void launch_conv_fwd(const ConvArgs& a, cudaStream_t st) {
  const long long npts = (long long)a.n * a.n * a.n;
  k_conv_fwd<R><<<nblk(npts), 256, 0, st>>>(a);
}
template <typename R> void launch_conv_bwd(const ConvArgs& a, double* gw, double* gb, cudaStream_t st) {
  const long long npts = (long long)a.n * a.n * a.n;
  if (a.in_grad) k_conv_bwd_in<R><<<nblk(npts), 256, 0, st>>>(a);
  if (gw) {
    int chunks = int((npts + 256 * 64 - 1) / (256 * 64));
    if (chunks < 1) chunks = 1;
    k_conv_bwd_w<R><<<dim3(a.cin * 27, chunks), 256, 0, st>>>(a, gw);
  }
  if (gb) k_bias_grad<R><<<dim3(a.cout, 32), 256, 0, st>>>(a, gb);
}
template <typename R> void launch_gelu(const R* pre, R* post, long long n, cudaStream_t st) {
  k_gelu<R><<<nblk(n), 256, 0, st>>>(pre, post, n);
}
template <typename R> void launch_gelu_bwd(const R* pre, R* g, long long n, cudaStream_t st) {
  k_gelu_bwd<R><<<nblk(n), 256, 0, st>>>(pre, g, n);
}
template <typename R> void launch_cc_input(const R* vx, const R* vy, const R* vz, const double* z, R* a0, long long npts,
                                           cudaStream_t st) {
  k_cc_input<R><<<nblk(npts), 256, 0, st>>>(vx, vy, vz, z, a0, npts);
}
template <typename R> void launch_sum(const R* x, long long n, double* s, cudaStream_t st) {
  long long b = (n + 255) / 256;
  if (b > 1024) b = 1024;
  k_sum<R><<<unsigned(b), 256, 0, st>>>(x, n, s);
}

#define SC_CC_INST(R)                                                                                        \
  template void launch_conv_fwd<R>(const ConvArgs&, cudaStream_t);                                           \
  template void launch_conv_bwd<R>(const ConvArgs&, double*, double*, cudaStream_t);                         \
  template void launch_gelu<R>(const R*, R*, long long, cudaStream_t);                                       \
  template void launch_gelu_bwd<R>(const R*, R*, long long, cudaStream_t);                                   \
  template void launch_cc_input<R>(const R*, const R*, const R*, const double*, R*, long long, cudaStream_t); \
  template void launch_sum<R>(const R*, long long, double*, cudaStream_t);
SC_CC_INST(float)
SC_CC_INST(double)

}  // namespace sc
