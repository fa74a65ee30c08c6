// Pointwise learned closures on CUDA cores in the plan's precision:
// fullchain(setup, mlp(...)) (src/nets.jl:311-331, 248-296) and tbnn
// (src/nets.jl:560-588).  One thread per grid point;
// the point's activations live in shared memory as [channel][thread] (64
// threads per CTA), weights are read with warp-uniform loads (broadcast).
#include <math.h>

#include "sc_les.h"

namespace sc {

namespace {

constexpr int kMlpThreads = 64;

template <typename R> __device__ __forceinline__ R gelu_t(R x) {
  const R u = R(0.79788456080286535588) * (x + R(0.044715) * x * x * x);
  return R(0.5) * x * (R(1) + tanh(u));
}

template <typename R> struct Eps;
template <> struct Eps<float> { static constexpr float v = 1.1920929e-07f; };
template <> struct Eps<double> { static constexpr double v = 2.220446049250313e-16; };

// 3 x 3 helpers (a 2D tensor sits in the upper-left 2 x 2 block)
template <typename R> struct M3 { R m[3][3]; };
template <typename R> __device__ __forceinline__ M3<R> mul(const M3<R>& x, const M3<R>& y) {
  M3<R> z;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) z.m[i][j] = x.m[i][0] * y.m[0][j] + x.m[i][1] * y.m[1][j] + x.m[i][2] * y.m[2][j];
  return z;
}
template <typename R> __device__ __forceinline__ M3<R> sub(const M3<R>& x, const M3<R>& y) {
  M3<R> z;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) z.m[i][j] = x.m[i][j] - y.m[i][j];
  return z;
}
template <typename R> __device__ __forceinline__ R trace(const M3<R>& x) { return x.m[0][0] + x.m[1][1] + x.m[2][2]; }
// M - tr(M) / D on the first D diagonal entries
template <typename R> __device__ __forceinline__ M3<R> dev(M3<R> x, int D) {
  const R t = trace(x) / R(D);
  for (int i = 0; i < D; ++i) x.m[i][i] -= t;
  return x;
}

// MODE 0: fullchain(mlp) (src/nets.jl:311-331); MODE 1: tbnn (src/nets.jl:560-588,
// invariants and basis of tb_kernel!, src/nets.jl:393-505)
template <typename R, int MODE>
__global__ void __launch_bounds__(kMlpThreads) k_mlp(const MlpArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  R* act = reinterpret_cast<R*>(smraw);  // [2][kMlpMaxWidth][kMlpThreads]
  const int t = threadIdx.x;
  const long long p = (long long)blockIdx.x * kMlpThreads + t;
  const bool live = p < a.npts;
  const int D = a.D, DD = D * D;
  R* in = act;
  R* out = act + kMlpMaxWidth * kMlpThreads;
  R a2 = 0;
  M3<R> S{}, Rm{};
  if (MODE == 0) {
    for (int c = 0; c < DD; ++c) {
      const R g = live ? static_cast<const R*>(a.G[c])[p] : R(0);
      in[c * kMlpThreads + t] = g;
      a2 += g * g;
    }
    const R inv = R(1) / (sqrt(a2) + Eps<R>::v);
    for (int c = 0; c < DD; ++c) in[c * kMlpThreads + t] *= inv;
    if (a.z) in[DD * kMlpThreads + t] = R(*a.z);
  } else {
    M3<R> A{};
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {  // A_ij = d_j u_i = channel i + D j
        const R g = live ? static_cast<const R*>(a.G[i + D * j])[p] : R(0);
        A.m[i][j] = g;
        a2 += g * g;
      }
    const R inv = R(1) / (sqrt(a2) + Eps<R>::v);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) A.m[i][j] *= inv;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        S.m[i][j] = (A.m[i][j] + A.m[j][i]) / R(2);
        Rm.m[i][j] = (A.m[i][j] - A.m[j][i]) / R(2);
      }
    const M3<R> SS = mul(S, S), RR = mul(Rm, Rm);
    int ni = 2;
    in[0 * kMlpThreads + t] = trace(SS);
    in[1 * kMlpThreads + t] = trace(RR);
    if (D == 3) {
      in[2 * kMlpThreads + t] = trace(mul(SS, S));
      in[3 * kMlpThreads + t] = trace(mul(S, RR));
      in[4 * kMlpThreads + t] = trace(mul(SS, RR));
      ni = 5;
    }
    if (a.z) in[ni * kMlpThreads + t] = R(*a.z);
  }
  const R* th = static_cast<const R*>(a.theta);
  for (int l = 0; l < a.nl; ++l) {
    const int cin = a.w[l], cout = a.w[l + 1];
    const bool last = l == a.nl - 1;
    const R* W = th;
    const R* b = last ? nullptr : th + (size_t)cin * cout;
    for (int co = 0; co < cout; ++co) {
      R s = b ? __ldg(b + co) : R(0);
      const R* wr = W + (size_t)co * cin;
      for (int ci = 0; ci < cin; ++ci) s += __ldg(wr + ci) * in[ci * kMlpThreads + t];
      out[co * kMlpThreads + t] = last ? s : gelu_t(s);
    }
    th += (size_t)cin * cout + (last ? 0 : cout);
    R* tmp = in; in = out; out = tmp;
  }
  if (!live) return;
  const R sc = R(a.delta * a.delta) * a2;
  if (MODE == 1) {
    // basis contraction: M = sum_k w_k B_k (deviatoric basis tensors)
    const R* w = in;
    M3<R> M{};
    auto add = [&](const M3<R>& B, R wk) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M.m[i][j] += wk * B.m[i][j];
    };
    const M3<R> SR = mul(S, Rm), RS = mul(Rm, S);
    add(dev(S, D), w[0 * kMlpThreads + t]);
    if (D == 2) {
      add(dev(sub(SR, RS), D), w[1 * kMlpThreads + t]);
      static_cast<R*>(a.tau[0])[p] = M.m[0][0] * sc;
      static_cast<R*>(a.tau[1])[p] = M.m[1][1] * sc;
      static_cast<R*>(a.tau[2])[p] = M.m[0][1] * sc;
      return;
    }
    const M3<R> SS = mul(S, S), RR = mul(Rm, Rm);
    add(dev(SS, D), w[1 * kMlpThreads + t]);
    add(dev(RR, D), w[2 * kMlpThreads + t]);
    add(dev(sub(SR, RS), D), w[3 * kMlpThreads + t]);
    add(dev(mul(RS, Rm), D), w[4 * kMlpThreads + t]);
    add(dev(sub(mul(RS, S), mul(SS, Rm)), D), w[5 * kMlpThreads + t]);
    add(dev(sub(mul(mul(RS, Rm), Rm), mul(RR, SR)), D), w[6 * kMlpThreads + t]);
    static_cast<R*>(a.tau[0])[p] = M.m[0][0] * sc;
    static_cast<R*>(a.tau[1])[p] = M.m[1][1] * sc;
    static_cast<R*>(a.tau[2])[p] = M.m[2][2] * sc;
    static_cast<R*>(a.tau[3])[p] = M.m[0][1] * sc;
    static_cast<R*>(a.tau[4])[p] = M.m[1][2] * sc;
    static_cast<R*>(a.tau[5])[p] = M.m[2][0] * sc;
    return;
  }
  if (D == 3) {
    const R tr = (in[0 * kMlpThreads + t] + in[1 * kMlpThreads + t] + in[2 * kMlpThreads + t]) / R(3);
    for (int m = 0; m < 6; ++m) {
      const R y = in[m * kMlpThreads + t] - (m < 3 ? tr : R(0));
      static_cast<R*>(a.tau[m])[p] = y * sc;
    }
  } else {
    const R tr = (in[0 * kMlpThreads + t] + in[1 * kMlpThreads + t]) / R(2);
    for (int m = 0; m < 3; ++m) {
      const R y = in[m * kMlpThreads + t] - (m < 2 ? tr : R(0));
      static_cast<R*>(a.tau[m])[p] = y * sc;
    }
  }
}

// sum over points of |G|^2 -> *s (FP64)
template <typename R>
__global__ void k_gsq_sum(const MlpArgs a, double* s) {
  __shared__ double red[32];
  double acc = 0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < a.npts; p += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < a.D * a.D; ++c) {
      const double g = double(static_cast<const R*>(a.G[c])[p]);
      acc += g * g;
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0;
    for (int w = 0; w < int(blockDim.x / 32); ++w) tot += red[w];
    atomicAdd(s, tot);
  }
}

// z = (log(Delta^2 sqrt(sum / npts) / nu) - mu) / sigma
__global__ void k_mlp_redelta(const double* s, long long npts, double delta, double nu, double mu, double sigma,
                              double* z) {
  const double re = delta * delta * sqrt(*s / double(npts)) / nu;
  *z = (log(re) - mu) / sigma;
}

}  // namespace

template <typename R>
void launch_mlp(const MlpArgs& a, double* zbuf, double nu, double mu, double sigma, cudaStream_t st) {
  MlpArgs b = a;
  b.z = nullptr;
  if (zbuf) {  // zbuf[0]: sum of |G|^2, zbuf[1]: z
    cudaMemsetAsync(zbuf, 0, sizeof(double), st);
    long long nb = (a.npts + 255) / 256;
    if (nb > 148 * 8) nb = 148 * 8;
    k_gsq_sum<R><<<unsigned(nb), 256, 0, st>>>(a, zbuf);
    k_mlp_redelta<<<1, 1, 0, st>>>(zbuf, a.npts, a.delta, nu, mu, sigma, zbuf + 1);
    b.z = zbuf + 1;
  }
  const size_t sm = size_t(2) * kMlpMaxWidth * kMlpThreads * sizeof(R);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_mlp<float, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(2 * kMlpMaxWidth * kMlpThreads * 4));
    cudaFuncSetAttribute(k_mlp<double, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(2 * kMlpMaxWidth * kMlpThreads * 8));
    cudaFuncSetAttribute(k_mlp<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(2 * kMlpMaxWidth * kMlpThreads * 4));
    cudaFuncSetAttribute(k_mlp<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(2 * kMlpMaxWidth * kMlpThreads * 8));
    attr = true;
  }
  const unsigned nb = unsigned((a.npts + kMlpThreads - 1) / kMlpThreads);
  if (a.mode == 1) k_mlp<R, 1><<<nb, kMlpThreads, sm, st>>>(b);
  else k_mlp<R, 0><<<nb, kMlpThreads, sm, st>>>(b);
}

template void launch_mlp<float>(const MlpArgs&, double*, double, double, double, cudaStream_t);
template void launch_mlp<double>(const MlpArgs&, double*, double, double, double, cudaStream_t);

}  // namespace sc
