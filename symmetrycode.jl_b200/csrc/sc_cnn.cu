// CNN closure (new; no reference counterpart): 3x3x3 periodic convolutions on
// the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32
// accumulators in tensor memory).
//
// Network (per LES instance, 128^3): input u (3 physical channels) and the
// standardised log Re_Delta as a constant 4th channel, conv 4->32, GELU,
// conv 32->32, GELU, conv 32->32, GELU, conv 32->6 -> tau (pair order).
//
// One CTA computes one output x-row (128 voxels = the MMA's M) at a time.  The
// nine input rows (y-1..y+1, z-1..z+1) are staged once in shared memory in the
// UMMA K-major no-swizzle layout [row][k-chunk][x+1][8 channels] with a one-voxel
// periodic halo in x, so the 27 taps are 27 descriptors into the same slab:
// the x shift of a tap is a 16-byte offset of the descriptor's start address.
// All weights of the layer stay in shared memory for the CTA's lifetime.
// One elected thread issues the MMAs; tcgen05.commit signals an mbarrier; the
// accumulator (128 lanes x C_out columns) is read back with tcgen05.ld for the
// bias + GELU + BF16 epilogue.  Every mbarrier wait is bounded: on timeout the
// kernel raises an error flag, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "sc_cnn.h"

namespace sc {

namespace {

constexpr int kN = 128;        // grid size handled (one x-row = one MMA tile)
constexpr int kRowPlane = (kN + 2) * 16;  // bytes of one k-chunk plane of one staged row
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // UMMA shared-memory descriptor, K-major, no swizzle (layout type 0), version 1
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFF);
  d |= uint64_t((lbo >> 4) & 0x3FFF) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFF) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

template <int NOUT>
__host__ __device__ constexpr uint32_t make_idesc() {
  // kind::f16: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16 (10-12 = 1),
  // both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128)
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(NOUT >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  uint32_t mask[4] = {0, 0, 0, 0};
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(mask[0]), "r"(mask[1]), "r"(mask[2]), "r"(mask[3]));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long it = 0; it < kSpinLimit; ++it) {
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

template <int NCOL>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float* v);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// GELU in the tanh form of NNlib's gelu (the activation of the reference's nets):
// 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))).  The hardware tanh.approx
// (relative error about 2^-11) is below the BF16 rounding of the activations.
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * x * (1.f + 0.044715f * x * x);
  return 0.5f * x * (1.f + tanh_hw(u));
}

}  // namespace

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// One convolution layer.  act_in: BF16 channels-last [n^3][CP]; weights:
// BF16 [27][CP/8][COP][8] (UMMA K-major planes per tap); out: BF16 channels-last
// [n^3][COP] with GELU (LAST = false) or FP32 planar tau (LAST = true).
// Each CTA walks a contiguous run of x-rows (y fastest), software-pipelined
// with one CTA barrier per row and three warp roles:
//  - warp 0, one thread: issues the 27 x CP/16 MMAs of row y into one of two
//    tensor-memory accumulators;
//  - warps 1-3: once the MMAs of row y-1 are done, fetch row y+3 with cp.async
//    into the ring slot that row y-2 left (kSlots y-slots per z-offset; row
//    y+2 is already resident, so each fetch has two rows of time to land);
//  - warps 4-11 (two per tensor-memory lane quadrant): the bias + GELU
//    epilogue of row y-1 from the other accumulator, while row y computes.
// A change of z-plane drains the pipeline and restages the new plane.
constexpr int kSlots = 5;
constexpr int kConvThreads = 384;

template <int CP, int COP, bool LAST>
__global__ void __launch_bounds__(kConvThreads, 1)
k_conv3(const __nv_bfloat16* __restrict__ act_in, const __nv_bfloat16* __restrict__ wgt,
        const float* __restrict__ bias, __nv_bfloat16* __restrict__ act_out, const TauPtrs tau_out,
        int* __restrict__ err) {
  constexpr int CPC = CP / 8;              // 16-byte channel chunks
  constexpr int PLANE_ROW = CPC * kRowPlane;
  constexpr int SIN = 3 * kSlots * PLANE_ROW;  // [zr][slot] staged rows
  constexpr int SW = 27 * CPC * COP * 16;
  constexpr uint32_t IDESC = make_idesc<COP>();
  constexpr uint32_t kTmemCols = 64;       // two accumulators of COP <= 32 columns
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* s_in = sm;
  unsigned char* s_w = sm + SIN;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + SIN + SW);       // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + SIN + SW + 16);
  const int tid = threadIdx.x, warp = tid / 32;
  const bool is_stage = warp >= 1 && warp < 4;
  // epilogue warps: lane quadrant warp % 4, columns ecol0 .. ecol0 + 15
  const int lane_base = 32 * (warp % 4);
  const int ecol0 = warp >= 8 ? COP / 2 : 0;
  const bool is_epi = warp >= 4 && (COP / 2 == 16 || warp < 8);

  for (int i = tid; i < SW / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(s_w)[i] = __ldg(reinterpret_cast<const uint4*>(wgt) + i);
  float bia[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) bia[c] = (is_epi && (!LAST || c < 6)) ? __ldg(bias + ecol0 + c) : 0.f;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + 1)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tslot;
  uint32_t phase = 0;     // bit b: parity of the next wait on buffer b (same in every thread)
  uint32_t inflight = 0;  // bit b: a committed MMA group of buffer b not yet waited for
  bool ok = true;

  // copy x-rows ylo..yhi of the three z-offsets of plane z into their ring slots
  auto stage = [&](int z, int ylo, int yhi, int t0, int tstride) {
    const int nyr = yhi - ylo + 1;
    const int chunks = 3 * nyr * (kN + 2) * CPC;
    for (int i = t0; i < chunks; i += tstride) {
      const int kc = i % CPC;
      const int xi = (i / CPC) % (kN + 2);
      const int q = i / (CPC * (kN + 2));
      const int zr = q / nyr, yv = ylo + q % nyr;
      const int zz = (z + zr - 1 + kN) % kN, yy = (yv + kN) % kN;
      const int x = (xi - 1 + kN) % kN;
      const long long vox = ((long long)zz * kN + yy) * kN + x;
      unsigned char* dst = s_in + (zr * kSlots + (yv + kN) % kSlots) * PLANE_ROW + kc * kRowPlane + xi * 16;
      cp_async16(dst, reinterpret_cast<const uint4*>(act_in + vox * CP) + kc);
    }
  };
  auto commit = [] { asm volatile("cp.async.commit_group;" ::: "memory"); };
  // bounded wait of this thread for the MMAs of buffer b
  auto wait_buf = [&](int b) -> bool {
    const bool r = mbar_wait(bar + b, (phase >> b) & 1u);
    asm volatile("tcgen05.fence::after_thread_sync;");
    return r;
  };
  // bias + activation of row prow from accumulator buffer b (epilogue warps)
  auto epilogue = [&](int prow, int b) {
    if (!is_epi) return;
    float v[16];
    tmem_ld<16>(tmem + (uint32_t(lane_base) << 16) + uint32_t(b * 32 + ecol0), v);
    const long long vox = (long long)prow * kN + lane_base + tid % 32;
    if (!LAST) {
      __align__(16) __nv_bfloat16 o[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) o[c] = __float2bfloat16_rn(gelu(v[c] + bia[c]));
      uint4* dst = reinterpret_cast<uint4*>(act_out + vox * COP + ecol0);
      dst[0] = reinterpret_cast<uint4*>(o)[0];
      dst[1] = reinterpret_cast<uint4*>(o)[1];
    } else {
#pragma unroll
      for (int c = 0; c < 6; ++c) tau_out.p[c][vox] = v[c] + bia[c];
    }
  };
  // wait for buffer b everywhere, run its epilogue, barrier; false on a timeout
  auto drain = [&](int prow) -> bool {
    const int b = prow & 1;
    const bool mine = wait_buf(b);
    if (mine) epilogue(prow, b);
    asm volatile("tcgen05.fence::before_thread_sync;");
    const bool all = __syncthreads_and(mine) != 0;
    if (all) { phase ^= 1u << b; inflight &= ~(1u << b); }
    return all;
  };

  const int nrows = kN * kN;
  const int per = (nrows + gridDim.x - 1) / gridDim.x;
  const int rbeg = blockIdx.x * per;
  const int rend = min(rbeg + per, nrows);
  int cur_z = -1;
  int pending = -1;  // row whose accumulator still needs its epilogue
  for (int row = rbeg; row < rend; ++row) {
    const int y = row % kN, z = row / kN;
    if (z != cur_z) {
      // new plane: drain, then stage rows y-1 .. y+2 as one group (all threads)
      if (pending >= 0) {
        ok = drain(pending);
        pending = -1;
        if (!ok) break;
      }
      stage(z, y - 1, min(y + 2, kN), tid, kConvThreads);
      commit();
      cur_z = z;
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 1;" ::: "memory");  // row y+1 has landed; row y+2 may be in flight
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const int b = row & 1;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      // descriptors are a base plus a compile-time offset (start-address field
      // in 16-byte units); only the three ring slots of this row are run-time
      const uint64_t DA0 = make_desc(smem_u32(s_in), kRowPlane, 128);
      const uint64_t DB0 = make_desc(smem_u32(s_w), COP * 16, 128);
      const uint32_t dcol = tmem + uint32_t(b * 32);
      uint32_t sl[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) sl[d] = uint32_t((y + d - 1 + kN) % kSlots) * (PLANE_ROW >> 4);
#pragma unroll
      for (int t = 0; t < 27; ++t) {
        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
        const uint64_t arow = DA0 + sl[dy] + uint32_t(dz * kSlots * (PLANE_ROW >> 4) + dx);
#pragma unroll
        for (int h = 0; h < CPC / 2; ++h) {
          const uint64_t da = arow + uint32_t(2 * h * (kRowPlane >> 4));
          const uint64_t db = DB0 + uint32_t((t * CPC + 2 * h) * COP);
          mma_bf16(dcol, da, db, IDESC, (t | h) ? 1u : 0u);
        }
      }
      mma_commit(bar + b);
    }
    inflight |= 1u << b;
    bool mine = true;
    if (pending >= 0 && warp != 0) mine = wait_buf(pending & 1);  // the last readers of row y-2's slot
    // prefetch row y+3 (read first by the MMAs of row y+2, when this CTA runs
    // that row in this plane); every thread commits a group, empty or not
    if (is_stage && mine && y + 2 < kN && row + 2 < rend) stage(z, y + 3, y + 3, tid - 32, 96);
    commit();
    if (pending >= 0 && mine) epilogue(pending, pending & 1);
    asm volatile("tcgen05.fence::before_thread_sync;");
    ok = __syncthreads_and(mine) != 0;
    if (!ok) break;
    if (pending >= 0) { phase ^= 1u << (pending & 1); inflight &= ~(1u << (pending & 1)); }
    pending = row;
  }
  if (ok && pending >= 0) ok = drain(pending);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // a wait ran out: give the MMAs still in flight one more bounded wait before
    // the tensor memory they write is released
    for (int bb = 0; bb < 2; ++bb)
      if ((inflight >> bb) & 1u) mbar_wait(bar + bb, (phase >> bb) & 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// input channels: u (3 physical FP32 fields) and the constant channel *z -> BF16 [n^3][16]
__global__ void k_cnn_input(const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
                            const double* __restrict__ z, __nv_bfloat16* __restrict__ out, long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  __align__(16) __nv_bfloat16 o[16];
  o[0] = __float2bfloat16_rn(ux[i]);
  o[1] = __float2bfloat16_rn(uy[i]);
  o[2] = __float2bfloat16_rn(uz[i]);
  o[3] = __float2bfloat16_rn(float(*z));
#pragma unroll
  for (int c = 4; c < 16; ++c) o[c] = __float2bfloat16_rn(0.f);
  uint4* dst = reinterpret_cast<uint4*>(out + i * 16);
  dst[0] = reinterpret_cast<uint4*>(o)[0];
  dst[1] = reinterpret_cast<uint4*>(o)[1];
}

// z = (log(Delta^2 sqrt(a2) / nu) - mu) / sigma   (Re_Delta channel, src/nets.jl:311-331 convention)
__global__ void k_cnn_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma) {
  const double re = delta * delta * sqrt(*a2) / nu;
  *z = (log(re) - mu) / sigma;
}

template <int CP, int COP, bool LAST> static size_t conv_smem() {
  return size_t(3 * kSlots) * (CP / 8) * kRowPlane + size_t(27) * (CP / 8) * COP * 16 + 32;
}

template <int CP, int COP, bool LAST> static void conv_attr() {
  cudaFuncSetAttribute(k_conv3<CP, COP, LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(conv_smem<CP, COP, LAST>()));
}

bool cnn_supported(int n, int D) { return n == kN && D == 3; }

void launch_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma, cudaStream_t st) {
  k_cnn_redelta<<<1, 1, 0, st>>>(a2, z, delta, nu, mu, sigma);
}

void cnn_init() {
  conv_attr<16, 32, false>();
  conv_attr<32, 32, false>();
  conv_attr<32, 16, true>();
}

void launch_cnn_forward(const CnnArgs& a, cudaStream_t st) {
  const long long npts = (long long)kN * kN * kN;
  k_cnn_redelta<<<1, 1, 0, st>>>(a.a2, a.z, a.delta, a.nu, a.mu, a.sigma);
  k_cnn_input<<<unsigned((npts + 255) / 256), 256, 0, st>>>(
      static_cast<const float*>(a.u[0]), static_cast<const float*>(a.u[1]), static_cast<const float*>(a.u[2]), a.z,
      a.act0, npts);
  const int grid = a.nsm > 0 ? a.nsm : 148;
  const TauPtrs none{};
  k_conv3<16, 32, false><<<grid, kConvThreads, conv_smem<16, 32, false>(), st>>>(a.act0, a.w[0], a.b[0], a.act1, none, a.err);
  k_conv3<32, 32, false><<<grid, kConvThreads, conv_smem<32, 32, false>(), st>>>(a.act1, a.w[1], a.b[1], a.act2, none, a.err);
  k_conv3<32, 32, false><<<grid, kConvThreads, conv_smem<32, 32, false>(), st>>>(a.act2, a.w[2], a.b[2], a.act1, none, a.err);
  k_conv3<32, 16, true><<<grid, kConvThreads, conv_smem<32, 16, true>(), st>>>(a.act1, a.w[3], a.b[3], nullptr, a.tau, a.err);
}

}  // namespace sc
