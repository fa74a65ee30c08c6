// TMA-fed column sweeps of the 810^3 FP32 transforms (sm_100a).
//
// The same two-level 27 x 30 register FFT as k_col2 (tile of T = 8
// consecutive kx, one column, all rows of the transform axis), but the input
// tile reaches shared memory by tensor-memory-access bulk copies instead of
// per-thread loads, and each CTA is persistent with two tile stages:
//
//   stage s holds item i (TMA, completed on mbarrier full[s]) while stage s^1
//   receives item i + G; step 1 reads the tile from stage s, the exchange
//   between the two radix passes is written over the same stage, step 2
//   stores to global memory, and only then does thread 0 re-arm full[s] and
//   issue the copies of item i + 2G into it.
//
// So the next tile's HBM reads always overlap this tile's arithmetic, and no
// thread spends issue slots or registers on the loads.  Configurations: 8 kx
// per tile with two stages and two CTAs of 240 threads per SM (2 x 2 x 53.6 KB
// of stages), 16 kx (128-byte box rows) with two stages and one CTA of 480
// threads, 8 kx with three stages and one CTA.  The tensor maps cover the
// padded intermediates of the product pipeline (row length K1 + 1 = 272
// complex, so every row starts on a 16-byte boundary); each box is T complex
// (8 T bytes) wide, starts at kx = T b (a multiple of 16 bytes) and at most 256
// rows high, so a tile is 3 (compact inverse input, 541 rows) or 4 (810 rows)
// boxes.  Rows past the end of the axis and the kx past K1 are filled with
// zeros by the copy engine.  Only plain per-CTA loads of this GPU's own
// memory are issued, each into the issuing CTA's shared memory.
//
// Every mbarrier wait is bounded (SC_OPT_WAIT_LIMIT polls): when thread 0's
// wait runs out, the CTA sets the plan's error word, waits with the default
// bound for its copies still in flight and returns; sc_plan_status reports
// SC_ERR_TIMEOUT.
#include <cuda.h>
#include <stdint.h>

#include "sc_cnn.h"
#include "sc_fft.cuh"
#include "sc_internal.h"

namespace sc {

namespace {

constexpr int kN = 810, kN1 = 27, kN2 = 30;
constexpr int kKP = kN / 3 + 1, kKN = kN / 3, kKc = kKP + kKN;  // compact transform axis: 271 + 270

// T: kx per tile (box rows of 8 T bytes); NS: tile stages per CTA
template <int T, int NS> struct ColTCfg {
  static constexpr int NT = T * kN2;                    // threads
  static constexpr int SR = kN2 * T + 8;                // exchange row stride (complex)
  static constexpr int EXCH = kN1 * SR * 8;
  static constexpr int TILE = 4 * 204 * T * 8;          // 810 rows in 4 boxes of 204
  static constexpr int STAGE = ((EXCH > TILE ? EXCH : TILE) + 127) / 128 * 128;
  static constexpr int SMEM = NS * STAGE + 128;         // + NS mbarriers and the wait flag
  static constexpr int MINB = 2 * (SMEM + 1024) <= 232448 ? 2 : 1;
};

struct ColTParams {
  CUtensorMap map[kMaxComp];  // one per component, over a.in[q]
  ColArgs a;
  int nitems, ntile;
  int nbox, box_rows;
  int rows_dim1;       // 1: the transform axis is tensor dimension 1, else dimension 2
  unsigned tx_bytes;   // bytes of one tile (nbox boxes)
  long long wait_limit;
  int* err;
};

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t a = su32(bar);
  for (long long it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// thread 0: arm the stage's mbarrier with the tile's byte count and issue its boxes
template <int T>
__device__ __forceinline__ void issue_tile(const ColTParams& P, int it, unsigned char* stage, uint64_t* bar) {
  const int b = it % P.ntile, rest = it / P.ntile;
  const int c = rest % P.a.ncols, q = rest / P.a.ncols;
  const CUtensorMap* map = &P.map[q];
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(P.tx_bytes)
               : "memory");
  const int x = b * 2 * T;  // float coordinate of kx = T b: a multiple of 16 floats (64 bytes)
  for (int k = 0; k < P.nbox; ++k) {
    const int r0 = k * P.box_rows;
    const int y = P.rows_dim1 ? r0 : c, z = P.rows_dim1 ? c : r0;
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(su32(stage + k * P.box_rows * T * 8)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(su32(bar))
        : "memory");
  }
}

template <int T, int NS, bool INV>
__global__ void __launch_bounds__(ColTCfg<T, NS>::NT, ColTCfg<T, NS>::MINB)
k_colt(const __grid_constant__ ColTParams P, const float2* __restrict__ tw) {
  using C = float2;
  using Cfg = ColTCfg<T, NS>;
  constexpr int SR = Cfg::SR, STAGE = Cfg::STAGE;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * STAGE);
  int& s_ok = *reinterpret_cast<int*>(smem_raw + NS * STAGE + 8 * NS);  // thread 0's wait outcome
  const int tid = threadIdx.x, t = tid % T, j = tid / T;
  const int G = gridDim.x;
  const ColArgs& a = P.a;
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(&full[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < NS; ++s) {
      const int it = blockIdx.x + s * G;
      if (it < P.nitems) issue_tile<T>(P, it, smem_raw + s * STAGE, &full[s]);
    }
  }
  __syncthreads();
  const int oes = int(a.out_es);
  int k = 0;
  for (int it = blockIdx.x; it < P.nitems; it += G, ++k) {
    const int s = k % NS;
    const uint32_t par = uint32_t(k / NS) & 1u;
    C* tile = reinterpret_cast<C*>(smem_raw + s * STAGE);
    if (tid == 0) s_ok = bar_wait(&full[s], par, P.wait_limit) ? 1 : 0;
    __syncthreads();
    if (!s_ok) {
      if (tid == 0) {
        atomicExch(P.err, 1);
        // copies still in flight into this CTA's shared memory (this item's
        // and the next NS - 1 items'), each waited for with the default bound
        // before the CTA exits
        for (int m = 0; m < NS; ++m)
          if (it + m * G < P.nitems) bar_wait(&full[(k + m) % NS], uint32_t((k + m) / NS) & 1u, kDefaultWaitLimit);
      }
      return;
    }
    if (tid != 0) bar_wait(&full[s], par, P.wait_limit);  // completed: acquires the copied tile
    const int b = it % P.ntile, rest = it / P.ntile;
    const int c = rest % a.ncols, q = rest / a.ncols;
    const int kx = b * T + t;
    const bool live = kx < a.K1;
    // step 1: thread (j, t) takes rows 30 n1 + j of column t of the tile
    C v[kN1];
    if (INV) {
#pragma unroll
      for (int n1 = 0; n1 < kN1; ++n1) {
        const int e = kN2 * n1 + j;
        const int rg = crange(kN2 * n1, kN2, kN, kKP, kKN);
        v[n1] = mk<C>(0.f, 0.f);
        if (rg == 2) continue;
        const int p = rg == 0 ? e : (rg == 1 ? e - kN + kKc : cpos(e, kN, kKP, kKN));
        if (p >= 0) v[n1] = tile[p * T + t];
      }
    } else {
#pragma unroll
      for (int n1 = 0; n1 < kN1; ++n1) v[n1] = tile[(kN2 * n1 + j) * T + t];
    }
    DFT<kN1, INV, C>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < kN1; ++k1) {
      C w = __ldg(&tw[j * k1]);
      if (INV) w.y = -w.y;
      v[k1] = cmul(v[k1], w);
    }
    __syncthreads();  // every thread has read its rows: the exchange overwrites the tile
    C* ys = tile;
#pragma unroll
    for (int k1 = 0; k1 < kN1; ++k1) ys[k1 * SR + j * T + t] = v[k1];
    __syncthreads();
    if (j < kN1 && live) {
      C w[kN2];
#pragma unroll
      for (int n2 = 0; n2 < kN2; ++n2) w[n2] = ys[j * SR + n2 * T + t];
      DFT<kN2, INV, C>::run(w);
      C* obase = static_cast<C*>(a.out[q]) + kx + (long long)c * a.out_cs;
      if (INV) {
        C* oj = obase + j * oes;
        const int st = kN1 * oes;
#pragma unroll
        for (int k2 = 0; k2 < kN2; ++k2) oj[k2 * st] = w[k2];
      } else {
        const int shift = kN - kKc;
#pragma unroll
        for (int k2 = 0; k2 < kN2; ++k2) {
          const int e = j + kN1 * k2;
          const int rg = crange(kN1 * k2, kN1, kN, kKP, kKN);
          if (rg == 0) obase[e * oes] = w[k2];
          else if (rg == 1) obase[(e - shift) * oes] = w[k2];
          else if (rg == 3) {
            if (e < kKP) obase[e * oes] = w[k2];
            else if (e >= kN - kKN) obase[(e - shift) * oes] = w[k2];
          }
        }
      }
    }
    // the stage's generic-proxy reads and writes are ordered before the copy
    // engine overwrites it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0 && it + NS * G < P.nitems) issue_tile<T>(P, it + NS * G, smem_raw + s * STAGE, &full[s]);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return EncodeTiled(nullptr);
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

template <int T, int NS> bool set_attr() {
  using Cfg = ColTCfg<T, NS>;
  return cudaFuncSetAttribute(k_colt<T, NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM) ==
             cudaSuccess &&
         cudaFuncSetAttribute(k_colt<T, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM) ==
             cudaSuccess;
}

template <int T, int NS>
bool launch_cfg(bool inv, const ColArgs& a, const float2* tw, cudaStream_t st) {
  using Cfg = ColTCfg<T, NS>;
  const EncodeTiled enc = encode_fn();
  if (!enc) return false;
  const long long R = inv ? kKc : kN;  // stored rows of the transform axis
  const bool rows_dim1 = a.in_es < a.in_cs;
  const long long e1 = rows_dim1 ? R : a.ncols, s1 = rows_dim1 ? a.in_es : a.in_cs;
  const long long e2 = rows_dim1 ? a.ncols : R, s2 = rows_dim1 ? a.in_cs : a.in_es;
  if (s2 < e1 * s1 || s1 < a.K1) return false;
  ColTParams P{};  // copied into the launch's parameters
  P.a = a;
  P.ntile = (a.K1 + T - 1) / T;
  P.nitems = P.ntile * a.ncols * a.ncomp;
  P.nbox = int((R + 255) / 256);
  P.box_rows = int((R + P.nbox - 1) / P.nbox);
  P.box_rows += P.box_rows & 1;  // even: every box starts 128-byte aligned in shared memory
  P.rows_dim1 = rows_dim1 ? 1 : 0;
  P.tx_bytes = unsigned(P.nbox * P.box_rows * T * 8);
  P.wait_limit = a.wait_limit;
  P.err = a.err;
  if (P.box_rows > 256 || int(P.tx_bytes) > Cfg::STAGE) return false;
  const cuuint64_t gdim[3] = {cuuint64_t(2 * a.K1), cuuint64_t(e1), cuuint64_t(e2)};
  const cuuint64_t gstr[2] = {cuuint64_t(s1 * 8), cuuint64_t(s2 * 8)};
  const cuuint32_t box[3] = {cuuint32_t(2 * T), cuuint32_t(rows_dim1 ? P.box_rows : 1),
                             cuuint32_t(rows_dim1 ? 1 : P.box_rows)};
  const cuuint32_t estr[3] = {1, 1, 1};
  for (int q = 0; q < a.ncomp; ++q) {
    if (enc(&P.map[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(a.in[q]), gdim, gstr, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  static const int nsm = sm_count();
  const int slots = Cfg::MINB * nsm;
  const int grid = P.nitems < slots ? P.nitems : slots;
  if (inv) k_colt<T, NS, true><<<grid, Cfg::NT, Cfg::SMEM, st>>>(P, tw);
  else k_colt<T, NS, false><<<grid, Cfg::NT, Cfg::SMEM, st>>>(P, tw);
  return true;
}

}  // namespace

bool tma_encode_bf16_4d(TmaMap* map, const void* base, const unsigned long long dims[4],
                        const unsigned long long strides[3], const unsigned box[4]) {
  static_assert(sizeof(CUtensorMap) == sizeof(TmaMap), "tensor map size");
  const EncodeTiled enc = encode_fn();
  if (!enc || (reinterpret_cast<uintptr_t>(base) & 15)) return false;
  const cuuint64_t gdim[4] = {dims[0], dims[1], dims[2], dims[3]};
  const cuuint64_t gstr[3] = {strides[0], strides[1], strides[2]};
  const cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), gdim,
             gstr, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool colt_init() { return set_attr<8, 2>() && set_attr<16, 2>() && set_attr<8, 3>(); }

// Launches TMA-fed sweep configuration `which` (0: T = 8 with two stages and two
// CTAs per SM; 1: T = 16, 128-byte box rows, two stages, one CTA per SM;
// 2: T = 8 with three stages, one CTA per SM) when the geometry allows it:
// N = 810, the solver's compact transform axis (kpos = 271, kneg = 270), no
// derivative outputs, no k = 0 mask, 16-byte aligned inputs with 16-byte row
// and column strides, and the two strides nested (the larger at least the
// smaller times its extent).  Returns false otherwise (the caller launches
// k_col2).
bool launch_colt(int N, bool inv, const ColArgs& a, const void* tw, int which, cudaStream_t st) {
  if (N != kN || a.ndrv > 0 || a.zero_origin || a.kpos != kKP || a.kneg != kKN) return false;
  if (a.ncomp < 1 || a.ncomp > kMaxComp || a.K1 < 1 || a.ncols < 1 || !a.err) return false;
  if ((a.in_es & 1) || (a.in_cs & 1)) return false;
  for (int q = 0; q < a.ncomp; ++q)
    if (reinterpret_cast<uintptr_t>(a.in[q]) & 15) return false;
  const float2* t2 = static_cast<const float2*>(tw);
  switch (which) {
    case 0: return launch_cfg<8, 2>(inv, a, t2, st);
    case 1: return launch_cfg<16, 2>(inv, a, t2, st);
    case 2: return launch_cfg<8, 3>(inv, a, t2, st);
    default: return false;
  }
}

}  // namespace sc
