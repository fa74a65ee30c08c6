// CNN closure (new; no reference counterpart): 3x3x3 periodic convolutions on
// the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32
// accumulators in tensor memory).
//
// Network (per LES instance, 128^3): input u (3 physical channels) and the
// standardised log Re_Delta as a constant 4th channel, conv 4->32, GELU,
// conv 32->32, GELU, conv 32->32, GELU, conv 32->6 -> tau (pair order).
//
// Grids of n = 64 and n = 128 points per axis.  One CTA computes one output
// x-row at a time with M = 128 MMAs: at n = 128 the row is the tile; at n = 64
// rows 64..127 of the tile read staged data past the row (in bounds, never
// stored) and only TMEM lanes 0..63 are read back.  The
// nine input rows (y-1..y+1, z-1..z+1) are staged once in shared memory in the
// UMMA K-major no-swizzle layout [row][k-chunk][x+1][8 channels] with a one-voxel
// periodic halo in x, so the 27 taps are 27 descriptors into the same slab:
// the x shift of a tap is a 16-byte offset of the descriptor's start address.
// All weights of the layer stay in shared memory for the CTA's lifetime.
// One elected thread issues the MMAs; tcgen05.commit signals an mbarrier; the
// accumulator (128 lanes x C_out columns) is read back with tcgen05.ld for the
// bias + GELU + BF16 epilogue.  Every mbarrier wait is bounded: on timeout the
// kernel raises an error flag, frees its tensor memory and returns.  The bound
// of the row pipeline's waits is a launch argument (a plan option, so that a
// test can make a wait run out); the last wait for MMAs still in flight before
// the tensor memory is freed always keeps the full default bound.
//
// Split precision (SC_CLOPT_CNN_SPLIT): each operand is stored as two 16-bit
// parts x = hi + lo, and a convolution is three launches of the same kernel,
// A_hi W_hi + A_lo W_hi + A_hi W_lo, accumulated in an FP32 channels-last
// buffer by the epilogue modes kLinear, kAccum and a last mode that applies
// bias and GELU (tanhf) and writes the hi/lo activations (or tau).  Forward
// passes use FP16 parts (kind::f16 with both operands f16); the adjoint's
// input-gradient passes use BF16 parts.  One MMA never mixes the two types.
#include <cuda_bf16.h>
#include <stdint.h>

#include "sc_cnn.h"

namespace sc {

namespace {

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

template <int NOUT, bool F16 = false>
__host__ __device__ constexpr uint32_t make_idesc() {
  // kind::f16: D f32 (bits 4-5 = 1); A and B of one type, both bf16 (bits 7-9
  // and 10-12 = 1) or both f16 (0); both K-major, N >> 3 at bit 17, M >> 4 at
  // bit 24 (M = 128)
  constexpr uint32_t ab = F16 ? 0u : 1u;
  return (1u << 4) | (ab << 7) | (ab << 10) | (uint32_t(NOUT >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

// D += A B (the accumulators are zeroed in tensor memory beforehand), no lanes masked
__device__ __forceinline__ void mma_bf16_acc(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(1u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Polls the mbarrier phase `parity` at most `limit` times (try_wait suspends
// for a hardware-defined time per poll); false when the wait ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  const uint32_t a = smem_u32(bar);
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

// zero 32 lanes x 16 columns of tensor memory (this warp's lane quadrant)
__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
  const uint32_t z = 0;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(z)
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
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
// the same with the library tanhf (a few ulp): the split precision's activation
__device__ __forceinline__ float gelu_exact(float x) {
  const float u = 0.7978845608028654f * x * (1.f + 0.044715f * x * x);
  return 0.5f * x * (1.f + tanhf(u));
}


__device__ __forceinline__ float gelu_grad(float x) {
  const float c = 0.7978845608028654f, a = 0.044715f;
  const float t = tanhf(c * x * (1.f + a * x * x));
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * a * x * x);
}

}  // namespace

// bytes of one k-chunk plane of a staged row: KN + 2 voxels of 16 bytes,
// rounded up to 128 bytes so that every plane is a bulk-copy destination
template <int KN> constexpr int row_plane() { return ((KN + 2) * 16 + 127) / 128 * 128; }

// Epilogue modes: BF16 GELU activations; the same plus the FP32
// pre-activations (kept for the adjoint); FP32 planar tau (last layer);
// FP32 channels-last without bias or activation (the input-gradient
// convolution).  The split precision's passes: kLinear (first pass), kAccum
// (the FP32 channels-last output += this pass), and the last pass kGeluSplit
// (h = (this pass + the accumulated output) scale + bias, written back in
// place as the pre-activation; GELU with tanhf; FP16 hi/lo activations) or
// kTauSplit (tau = (this pass + accumulated) scale + bias, planar).
enum { kGelu = 0, kGeluSave = 1, kTau = 2, kLinear = 3, kAccum = 4, kGeluSplit = 5, kTauSplit = 6 };

struct ConvOut {
  __nv_bfloat16* act;  // kGelu, kGeluSave: BF16 channels-last [n^3][COP]
  float* pre;          // kGeluSave: FP32 channels-last pre-activations; kLinear, kAccum: FP32 channels-last
                       // output; kGeluSplit, kTauSplit: the accumulated passes (kGeluSplit writes h there)
  TauPtrs tau;         // kTau, kTauSplit
  __half* acth;        // kGeluSplit: FP16 channels-last activations, high parts
  __half* actl;        // kGeluSplit: low parts (activation - high part, rounded to FP16)
  float scale;         // kGeluSplit, kTauSplit: factor of the accumulated sum before the bias
};

// One convolution layer.  act_in: BF16 channels-last [n^3][CP]; weights:
// BF16 [27][CP/8][COP][8] (UMMA K-major planes per tap); output per MODE.
//
// Input-stationary MMAs: an output row (y, z) sums the 27 taps over the input
// rows (y + dy, z + dz), so one staged input row (y', z + dz) shifted by dx
// feeds the three output rows y' - 1, y', y' + 1 (dy = +1, 0, -1) at once: one
// MMA of N = 3 C_out per (dz, dx, 16 input channels) against the weights
// stacked in shared memory as [dz][dx][k-chunk][dy = +1, 0, -1][C_out][8],
// instead of three MMAs of N = C_out -- the same FLOPs with a third of the
// A-operand reads, so the tensor pipe rather than the shared-memory operand
// bandwidth sets the pace.  Output row y accumulates in tensor-memory block
// y mod 6 (C_out columns each) and the MMAs of step y' write blocks
// m, m + 1, m + 2 with m = (y' - 1) mod 6, where blocks 6 and 7 stand in for
// blocks 0 and 1: the three rows always form one contiguous range, every MMA
// has the same shape and accumulates (MMAs of mixed shapes or split column
// ranges measured up to 5x slower), and a row of block 0 or 1 is the sum of
// that block and its stand-in.  Row y completes with step y + 1; its blocks are
// read out and zeroed one step later, well before row y + 6 takes them.  A step
// is 9 x CP/16 MMAs; the steps of a run of output rows y0..y1 of one plane go
// from y0 - 1 to y1 + 1.
//
// Each CTA walks a contiguous run of x-rows (y fastest) of one plane at a
// time.  Three warp roles run decoupled within a run, handing off through
// mbarriers (every wait bounded; a wait that runs out raises a shared abort
// flag that ends the other roles' waits too):
//  - warp 0, one thread: for each step y', waits until input row y' is staged
//    and (from the sixth step on) until the block of row y' + 1 was read out
//    and zeroed, issues the MMAs and commits them to step barrier k mod 4;
//  - warp 1: waits for the copies of input row y' + 1, writes its halo and
//    marks it staged, then, once step y' - 1 is done, issues the bulk copies
//    of input row y' + 4 into the ring slot row y' - 1 left;
//  - warps 4-11 (two per tensor-memory lane quadrant): for each row, once the
//    step that completes it is done, read it out, zero its blocks and mark
//    them free, then bias + activation + store.
// The epilogue may lag the MMAs by up to four steps (the accumulator ring and
// the four step barriers), so its latency overlaps the tensor pipe's work.  A
// change of z-plane ends the run with a CTA barrier and restages.
constexpr int kSlots = 5;
constexpr int kConvThreads = 384;

template <int KN, int CP, int COP, int MODE, bool F16>
__global__ void __launch_bounds__(kConvThreads, 1)
k_conv3(const __grid_constant__ ConvMaps maps, const __nv_bfloat16* __restrict__ wgt,
        const float* __restrict__ bias, const ConvOut out, int* __restrict__ err, long long wait_limit) {
  constexpr int kRowPlane = row_plane<KN>();
  constexpr int CPC = CP / 8;              // 16-byte channel chunks
  constexpr int PLANE_ROW = CPC * kRowPlane;
  constexpr int SIN = 3 * kSlots * PLANE_ROW;  // [zr][slot] staged rows
  constexpr int NS = 3 * COP;              // stacked rows per k-chunk plane: the three dy taps
  constexpr int SW = 9 * CPC * NS * 16;
  constexpr uint32_t IDESC = make_idesc<3 * COP, F16>();
  constexpr uint32_t kTmemCols = 8 * COP;  // eight accumulator blocks
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* s_in = sm;
  unsigned char* s_w = sm + SIN;
  uint64_t* cbar = reinterpret_cast<uint64_t*>(sm + SIN + SW);       // [4] MMA steps
  uint64_t* staged = cbar + 4;                                        // [kSlots] row copies landed
  uint64_t* ready = staged + kSlots;                                  // [kSlots] rows staged (halo written)
  uint64_t* zeroed = ready + kSlots;                                  // [6] accumulator blocks free
  uint32_t* tslot = reinterpret_cast<uint32_t*>(zeroed + 6);
  int* abort_flag = reinterpret_cast<int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // epilogue warps: lane quadrant warp % 4 (rows 32 (warp % 4) ..), columns ecol0 .. ecol0 + 15
  const int lane_base = 32 * (warp % 4);
  const int ecol0 = warp >= 8 ? COP / 2 : 0;
  const bool is_epi = warp >= 4 && (COP / 2 == 16 || warp < 8) && lane_base < KN;
  // number of epilogue warps (the arrival count of the zeroed barriers)
  constexpr int NEPI = ((COP / 2 == 16) ? 2 : 1) * (KN >= 128 ? 4 : (KN + 31) / 32);

  // stacked weights: chunk ((dz 3 + dx) CPC + kc) NS + j COP + co holds tap
  // (dz, dy index 2 - j, dx) of the [27][CPC][COP] layout (dy index 0, 1, 2
  // for dy = -1, 0, +1), j = 0, 1, 2 for the output rows y' - 1, y', y' + 1
  for (int d = tid; d < SW / 16; d += blockDim.x) {
    const int co = d % COP, j = (d % NS) / COP, kc = (d / NS) % CPC, g = d / (NS * CPC);
    const int dyi = 2 - j;
    const int src = (((g / 3) * 9 + dyi * 3 + g % 3) * CPC + kc) * COP + co;
    reinterpret_cast<uint4*>(s_w)[d] = __ldg(reinterpret_cast<const uint4*>(wgt) + src);
  }
  constexpr bool kBias = MODE == kGelu || MODE == kGeluSave || MODE == kTau || MODE == kGeluSplit || MODE == kTauSplit;
  constexpr bool kTauOut = MODE == kTau || MODE == kTauSplit;
  float bia[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) bia[c] = (kBias && is_epi && (!kTauOut || c < 6)) ? __ldg(bias + ecol0 + c) : 0.f;
  if (tid == 0) {
    for (int q = 0; q < 4; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(cbar + q)));
    for (int q = 0; q < kSlots; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(staged + q)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(ready + q)));
    }
    for (int q = 0; q < 6; ++q)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(zeroed + q)), "r"(NEPI));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *abort_flag = 0;
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
  bool ok = true;

  // bounded wait that also gives up once another role raised the abort flag;
  // it spins on the non-suspending test_wait (the roles hand off every step,
  // and a suspended try_wait resumed measurably later than the phase completed)
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < wait_limit; ++it) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
      if (done) return true;
      if ((it & 63) == 63 && *reinterpret_cast<volatile int*>(abort_flag)) return false;
    }
    return false;
  };
  auto fail = [&] { *reinterpret_cast<volatile int*>(abort_flag) = 1; };
  auto arrive = [](uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
  };
  // tensor-memory block of output row y (y >= -2); blocks 0 and 1 also
  // accumulate in their stand-ins 6 and 7
  auto acc_blk = [](int y) -> int { return ((y % 6) + 6) % 6; };
  // read out row y's 16 columns of this warp and zero them (epilogue warps)
  auto readout = [&](int y, float* v) {
    const int blk = acc_blk(y);
    const uint32_t ta = tmem + (uint32_t(lane_base) << 16) + uint32_t(blk * COP + ecol0);
    tmem_ld<16>(ta, v);
    tmem_zero16(ta);
    if (blk < 2) {
      float w[16];
      const uint32_t tb = ta + uint32_t(6 * COP);
      tmem_ld<16>(tb, w);
      tmem_zero16(tb);
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] += w[c];
    }
  };
  // bias + activation + store of row prow (z KN + y) from the read-out values
  auto epilogue = [&](int prow, const float* v) {
    if (!is_epi) return;
    const long long vox = (long long)prow * KN + lane_base + tid % 32;
    if (MODE == kGelu || MODE == kGeluSave) {
      __align__(16) __nv_bfloat16 o[16];
      __align__(16) float h[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        h[c] = v[c] + bia[c];
        o[c] = __float2bfloat16_rn(gelu(h[c]));
      }
      uint4* dst = reinterpret_cast<uint4*>(out.act + vox * COP + ecol0);
      dst[0] = reinterpret_cast<uint4*>(o)[0];
      dst[1] = reinterpret_cast<uint4*>(o)[1];
      if (MODE == kGeluSave) {
        float4* ph = reinterpret_cast<float4*>(out.pre + vox * COP + ecol0);
#pragma unroll
        for (int j = 0; j < 4; ++j) ph[j] = reinterpret_cast<float4*>(h)[j];
      }
    } else if (MODE == kTau) {
#pragma unroll
      for (int c = 0; c < 6; ++c) out.tau.p[c][vox] = v[c] + bia[c];
    } else if (MODE == kTauSplit) {
      const float4* pl = reinterpret_cast<const float4*>(out.pre + vox * COP);
      const float4 p0 = pl[0], p1 = pl[1];
      const float pv[6] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y};
#pragma unroll
      for (int c = 0; c < 6; ++c) out.tau.p[c][vox] = (v[c] + pv[c]) * out.scale + bia[c];
    } else if (MODE == kGeluSplit) {
      float4* pl = reinterpret_cast<float4*>(out.pre + vox * COP + ecol0);
      __align__(16) __half hi[16];
      __align__(16) __half lo[16];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float4 p = pl[j];
        const float h[4] = {(v[4 * j] + p.x) * out.scale + bia[4 * j], (v[4 * j + 1] + p.y) * out.scale + bia[4 * j + 1],
                            (v[4 * j + 2] + p.z) * out.scale + bia[4 * j + 2],
                            (v[4 * j + 3] + p.w) * out.scale + bia[4 * j + 3]};
        pl[j] = make_float4(h[0], h[1], h[2], h[3]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float y = gelu_exact(h[e]);
          const __half hh = __float2half_rn(y);
          hi[4 * j + e] = hh;
          lo[4 * j + e] = __float2half_rn(y - __half2float(hh));
        }
      }
      uint4* dh = reinterpret_cast<uint4*>(out.acth + vox * COP + ecol0);
      uint4* dl = reinterpret_cast<uint4*>(out.actl + vox * COP + ecol0);
      dh[0] = reinterpret_cast<uint4*>(hi)[0];
      dh[1] = reinterpret_cast<uint4*>(hi)[1];
      dl[0] = reinterpret_cast<uint4*>(lo)[0];
      dl[1] = reinterpret_cast<uint4*>(lo)[1];
    } else if (MODE == kAccum) {
      float4* pl = reinterpret_cast<float4*>(out.pre + vox * COP + ecol0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float4 p = pl[j];
        pl[j] = make_float4(p.x + v[4 * j], p.y + v[4 * j + 1], p.z + v[4 * j + 2], p.w + v[4 * j + 3]);
      }
    } else {
      float4* pl = reinterpret_cast<float4*>(out.pre + vox * COP + ecol0);
#pragma unroll
      for (int j = 0; j < 4; ++j) pl[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
  };
  // Input rows reach the ring by bulk tensor copies: row yv of the three
  // z-offsets of plane z, CP/8 boxes of 8 channels x (KN + 2) voxels each (x
  // from -1; the copy engine fills x = -1 and x = KN with zeros), completing on
  // the slot's mbarrier.  Thread 32 issues them; warp 1 then waits for them and
  // writes the periodic halo voxels x = -1 and x = KN from x = KN - 1 and 0.
  uint32_t spar = 0;  // bit s: parity of the next wait on staged[s] (same in every thread)
  uint32_t tin = 0;   // thread 32: bit s set while a copy into slot s is in flight
  auto slot_of = [](int yv) { return (yv + KN) % kSlots; };
  auto tma_row = [&](int z, int yv) {
    const int sl = slot_of(yv), yy = (yv + KN) % KN;
    // bytes delivered: 3 rows x CP/8 boxes of (KN + 2) 16-byte voxels (the
    // planes' padding to 128 bytes is not written)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(staged + sl)),
                 "r"(3 * CPC * (KN + 2) * 16)
                 : "memory");
    for (int zr = 0; zr < 3; ++zr) {
      const int zz = (z + zr - 1 + KN) % KN;
      for (int c = 0; c < CPC; ++c) {
        unsigned char* dst = s_in + (zr * kSlots + sl) * PLANE_ROW + c * kRowPlane;
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
            "[%6];" ::"r"(smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(&maps.m[c])), "r"(0), "r"(-1), "r"(yy), "r"(zz), "r"(smem_u32(staged + sl))
            : "memory");
      }
    }
    tin |= 1u << sl;
  };
  // warp 1: wait for row yv's copies (bounded) and write its halo; warp-uniform result
  auto patch_row = [&](int yv) -> bool {
    const int sl = slot_of(yv);
    const bool w = __all_sync(0xffffffffu, wait(staged + sl, (spar >> sl) & 1u));
    if (w && lane < 3 * CPC * 2) {
      const int zr = lane / (2 * CPC), c = (lane / 2) % CPC, side = lane & 1;
      unsigned char* plane = s_in + (zr * kSlots + sl) * PLANE_ROW + c * kRowPlane;
      const uint4 v = reinterpret_cast<const uint4*>(plane)[side ? 1 : KN];
      reinterpret_cast<uint4*>(plane)[side ? KN + 1 : 0] = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    return w;
  };
  const int nrows = KN * KN;
  const int per = (nrows + gridDim.x - 1) / gridDim.x;
  const int rbeg = blockIdx.x * per;
  const int rend = min(rbeg + per, nrows);
  int k0 = 0;                    // global index of the run's first step (step k on cbar[k % 4])
  uint32_t rpar = 0;             // thread 0: bit s, parity of the next wait on ready[s]
  uint32_t zpar = 0;             // thread 0: bit b, parity of the next wait on zeroed[b]
  int last_k = -1;               // thread 0: last committed step
  float v[16];
  for (int r0 = rbeg; r0 < rend && ok;) {
    // one run of output rows y0..y1 of plane z: steps y0 - 1 .. y1 + 1
    const int z = r0 / KN, y0 = r0 % KN;
    const int y1 = min(KN - 1, y0 + (rend - r0) - 1);
    const int zrow = z * KN;
    const int nsteps = y1 - y0 + 3;
    r0 += y1 - y0 + 1;
    // copy input rows y0 - 1 .. y0 + 2 and zero the accumulator blocks
    if (tid == 32)
      for (int yv = y0 - 1; yv <= min(y0 + 2, y1 + 1); ++yv) tma_row(z, yv);
    if (is_epi)
      for (int q = 0; q < 8; ++q) tmem_zero16(tmem + (uint32_t(lane_base) << 16) + uint32_t(q * COP + ecol0));
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    bool mine = true;
    if (tid == 0) {
      // MMA issue
      const uint64_t DA0 = make_desc(smem_u32(s_in), kRowPlane, 128);
      const uint64_t DB0 = make_desc(smem_u32(s_w), NS * 16, 128);
      for (int i = 0; i < nsteps && mine; ++i) {
        const int yv = y0 - 1 + i, kk = k0 + i;
        const int sl = slot_of(yv);
        // every staged row is waited for once, in order
        mine = wait(ready + sl, (rpar >> sl) & 1u);
        rpar ^= 1u << sl;
        if (mine && yv >= y0 + 3) {  // the block of row yv + 1 held row yv - 5 of this run
          const int bq = acc_blk(yv - 5);
          mine = wait(zeroed + bq, (zpar >> bq) & 1u);
          zpar ^= 1u << bq;
        }
        if (!mine) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t sa = uint32_t(sl) * (PLANE_ROW >> 4);
        const uint32_t dcol = tmem + uint32_t(acc_blk(yv - 1) * COP);  // rows yv - 1, yv, yv + 1
#pragma unroll
        for (int g = 0; g < 9 * (CPC / 2); ++g) {
          const int dz = g / (3 * (CPC / 2)), dx = (g / (CPC / 2)) % 3, h = g % (CPC / 2);
          const uint64_t da = DA0 + sa + uint32_t(dz * kSlots * (PLANE_ROW >> 4) + dx + 2 * h * (kRowPlane >> 4));
          const uint64_t db = DB0 + uint32_t(((dz * 3 + dx) * CPC + 2 * h) * NS);
          mma_bf16_acc(dcol, da, db, IDESC);
        }
        mma_commit(cbar + (kk & 3));
        last_k = kk;
      }
      if (!mine) fail();
      // read-outs of this run no step waited for (rows y1 - 3 .. y1, or the
      // whole run if it is short): their phases complete before the run-end
      // barrier, so they are counted here without a wait
      for (int r = max(y0 - 2, y1 - 3); r <= y1; ++r) zpar ^= 1u << acc_blk(r);
    } else if (warp == 1) {
      // staging: complete row y0 - 1, then per step
      // (a copy whose wait ran out stays recorded in flight for the exit path)
      mine = patch_row(y0 - 1);
      __syncwarp();
      if (mine) {
        if (lane == 0) arrive(ready + slot_of(y0 - 1));
        spar ^= 1u << slot_of(y0 - 1);
        if (lane == 0) tin &= ~(1u << slot_of(y0 - 1));
      }
      for (int i = 0; i < nsteps && mine; ++i) {
        const int yv = y0 - 1 + i, kk = k0 + i;
        // complete input row yv + 1 as soon as its copies (issued three steps
        // ago) have landed: the MMA thread may run several steps ahead
        if (yv + 1 <= y1 + 1) {
          mine = patch_row(yv + 1);
          __syncwarp();
          if (mine) {
            if (lane == 0) arrive(ready + slot_of(yv + 1));
            spar ^= 1u << slot_of(yv + 1);
            if (lane == 0) tin &= ~(1u << slot_of(yv + 1));
          }
        }
        // copy input row yv + 4 into the slot input row yv - 1 left, once step
        // yv - 1 (its last reader) is done
        if (mine && yv + 4 <= y1 + 1) {
          if (i > 0) mine = __all_sync(0xffffffffu, wait(cbar + ((kk - 1) & 3), uint32_t((kk - 1) >> 2) & 1u));
          if (mine && lane == 0) tma_row(z, yv + 4);
        }
      }
      if (!mine) fail();
    } else if (is_epi) {
      // read-out, zeroing and epilogue of rows y0 - 2 .. y1 (row r completes with step r + 1)
      for (int r = y0 - 2; r <= y1 && mine; ++r) {
        const int kk = k0 + (r + 1 - (y0 - 1));
        mine = __all_sync(0xffffffffu, wait(cbar + (kk & 3), uint32_t(kk >> 2) & 1u));
        if (!mine) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        readout(r, v);
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) arrive(zeroed + acc_blk(r));
        if (r >= y0) epilogue(zrow + r, v);
      }
      if (!mine) fail();
    }
    k0 += nsteps;
    asm volatile("tcgen05.fence::before_thread_sync;");
    ok = __syncthreads_and(mine) != 0;
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // a wait ran out: give the MMAs still in flight one more bounded wait before
    // the tensor memory they write is released (steps complete in order), and
    // the row copies still in flight one before the CTA's shared memory is
    if (tid == 0 && last_k >= 0) mbar_wait(cbar + (last_k & 3), uint32_t(last_k >> 2) & 1u, kDefaultWaitLimit);
    if (tid == 32)
      for (int q = 0; q < kSlots; ++q)
        if ((tin >> q) & 1u) mbar_wait(staged + q, (spar >> q) & 1u, kDefaultWaitLimit);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

__global__ void k_set_flag(int* f) { *f = 1; }

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

// the same input channels as FP16 high and low parts (split precision): hi = fp16(x), lo = fp16(x - hi)
__device__ __forceinline__ void split_f16(float x, __half& hi, __half& lo) {
  hi = __float2half_rn(x);
  lo = __float2half_rn(x - __half2float(hi));
}
__global__ void k_cnn_input_split(const float* __restrict__ ux, const float* __restrict__ uy,
                                  const float* __restrict__ uz, const double* __restrict__ z, __half* __restrict__ oh,
                                  __half* __restrict__ ol, long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  __align__(16) __half h[16];
  __align__(16) __half l[16];
  split_f16(ux[i], h[0], l[0]);
  split_f16(uy[i], h[1], l[1]);
  split_f16(uz[i], h[2], l[2]);
  split_f16(float(*z), h[3], l[3]);
#pragma unroll
  for (int c = 4; c < 16; ++c) h[c] = l[c] = __float2half_rn(0.f);
  uint4* dh = reinterpret_cast<uint4*>(oh + i * 16);
  uint4* dl = reinterpret_cast<uint4*>(ol + i * 16);
  dh[0] = reinterpret_cast<uint4*>(h)[0];
  dh[1] = reinterpret_cast<uint4*>(h)[1];
  dl[0] = reinterpret_cast<uint4*>(l)[0];
  dl[1] = reinterpret_cast<uint4*>(l)[1];
}

// z = (log(Delta^2 sqrt(a2) / nu) - mu) / sigma   (Re_Delta channel, src/nets.jl:311-331 convention)
__global__ void k_cnn_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma) {
  const double re = delta * delta * sqrt(*a2) / nu;
  *z = (log(re) - mu) / sigma;
}

// ---------------------------------------------------------------------------
// backward pass helpers
// ---------------------------------------------------------------------------
// dL/dtau (6 planar FP32) -> BF16 channels-last [n^3][16] (channels 6..15 zero)
__global__ void k_gtau_cl(TauPtrs g, __nv_bfloat16* __restrict__ out, long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  __align__(16) __nv_bfloat16 o[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) o[c] = __float2bfloat16_rn(c < 6 ? g.p[c][i] : 0.f);
  uint4* dst = reinterpret_cast<uint4*>(out + i * 16);
  dst[0] = reinterpret_cast<uint4*>(o)[0];
  dst[1] = reinterpret_cast<uint4*>(o)[1];
}

// g_pre = BF16(g_post * gelu'(h)), channels-last [n^3][32]
__global__ void k_gelu_bwd_cl(const float* __restrict__ gpost, const float* __restrict__ h,
                              __nv_bfloat16* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = __float2bfloat16_rn(gpost[i] * gelu_grad(h[i]));
}

// split precision: BF16 high and low parts, hi = bf16(x), lo = bf16(x - hi)
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}
__global__ void k_gtau_cl_split(TauPtrs g, __nv_bfloat16* __restrict__ oh, __nv_bfloat16* __restrict__ ol,
                                long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  __align__(16) __nv_bfloat16 h[16];
  __align__(16) __nv_bfloat16 l[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) split_bf16(c < 6 ? g.p[c][i] : 0.f, h[c], l[c]);
  uint4* dh = reinterpret_cast<uint4*>(oh + i * 16);
  uint4* dl = reinterpret_cast<uint4*>(ol + i * 16);
  dh[0] = reinterpret_cast<uint4*>(h)[0];
  dh[1] = reinterpret_cast<uint4*>(h)[1];
  dl[0] = reinterpret_cast<uint4*>(l)[0];
  dl[1] = reinterpret_cast<uint4*>(l)[1];
}
__global__ void k_gelu_bwd_cl_split(const float* __restrict__ gpost, const float* __restrict__ h,
                                    __nv_bfloat16* __restrict__ oh, __nv_bfloat16* __restrict__ ol, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  split_bf16(gpost[i] * gelu_grad(h[i]), oh[i], ol[i]);
}

// FP32 channels-last [n^3][16] -> planar channels 0..3 (dL/dv and the z channel)
__global__ void k_gin_planar(const float* __restrict__ gin, const GinPtrs o, long long npts) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const float4 v = *reinterpret_cast<const float4*>(gin + i * 16);
  o.p[0][i] = v.x; o.p[1][i] = v.y; o.p[2][i] = v.z; o.p[3][i] = v.w;
}

// Weight and bias gradients of one layer (CUDA cores, FP32 accumulation,
// FP64 atomics into the flat parameter gradient):
//   gw[co][ci][t] += sum_v g[v][co] a[v + off(t)][ci],  gb[co] += sum_v g[v][co]
// for co < cout, ci < cin.  Block (tap t, chunk of voxels).  Only the first CI
// (4 | 32) input and CO (8 | 32) output channels are formed, the layer's own
// channels rounded up to the tile, not the padded CP, COP of the activations.
// A group of (CO/8)(CI/4) threads holds 8 x 4 (co, ci) register tiles, so a
// voxel costs three 16-byte shared loads per 32 FMAs; the groups split each
// staged block of VS voxels.  The bias sums run only in the centre-tap blocks.
// The groups' tiles are summed in shared memory by all threads, then one FP64
// atomic per gradient entry and block.
// SPLIT: g = g + glo (BF16 high and low parts) and a = FP16 high + low parts
// (a and alo of type __half); otherwise a is BF16 and glo, alo are unused.
template <int KN, int CP, int COP, int CI, int CO, bool SPLIT>
__global__ void __launch_bounds__(256)
k_conv_wgrad(const __nv_bfloat16* __restrict__ g, const __nv_bfloat16* __restrict__ glo, const void* __restrict__ a,
             const void* __restrict__ alo, int cin, int cout, int vchunk, double* __restrict__ gw,
             double* __restrict__ gb) {
  static_assert(CI % 4 == 0 && CI <= CP && CO % 8 == 0 && CO <= COP, "tile shape");
  constexpr int TCO = 8, TCI = 4, NE = TCO * TCI;
  constexpr int TG = (CO / TCO) * (CI / TCI);  // threads per group
  constexpr int NG = 256 / TG;                  // groups
  constexpr int VS = 128;                       // voxels per stage
  constexpr int LG = CO + 4, LA = CI + 4;       // padded shared rows (16-byte multiples)
  constexpr int STAGE = VS * (LG + LA);         // floats of one staged block
  constexpr int RED = 256 * NE;                 // floats of the groups' tiles
  constexpr long long NPTS = (long long)KN * KN * KN;
  __shared__ __align__(16) float sbuf[STAGE > RED ? STAGE : RED];
  float* sg = sbuf;            // [VS][LG]
  float* sa = sbuf + VS * LG;  // [VS][LA]
  const int t = blockIdx.x;    // tap
  const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
  const bool centre = t == 13;
  const int tid = threadIdx.x, grp = tid / TG, lt = tid % TG;
  const int co0 = TCO * (lt / (CI / TCI)), ci0 = TCI * (lt % (CI / TCI));
  float acc[TCO][TCI] = {};
  float accb[TCO] = {};
  const long long v0 = (long long)blockIdx.y * vchunk;
  const long long v1 = min(v0 + vchunk, NPTS);
  for (long long vb = v0; vb < v1; vb += VS) {
    // stage the g rows and the shifted a rows (16-bit pairs -> FP32)
    for (int i = tid; i < VS * CO / 2; i += 256) {
      const int vv = i / (CO / 2), c = 2 * (i % (CO / 2));
      const long long v = vb + vv;
      float2 f = make_float2(0.f, 0.f);
      if (v < v1) {
        f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(g + v * COP + c));
        if (SPLIT) {
          const float2 l = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(glo + v * COP + c));
          f.x += l.x; f.y += l.y;
        }
      }
      *reinterpret_cast<float2*>(sg + vv * LG + c) = f;
    }
    for (int i = tid; i < VS * CI / 2; i += 256) {
      const int vv = i / (CI / 2), c = 2 * (i % (CI / 2));
      const long long v = vb + vv;
      float2 f = make_float2(0.f, 0.f);
      if (v < v1) {
        const int x = int(v % KN), y = int((v / KN) % KN), z = int(v / ((long long)KN * KN));
        const long long q = ((long long)((z + dz + KN) % KN) * KN + (y + dy + KN) % KN) * KN + (x + dx + KN) % KN;
        if (SPLIT) {
          f = __half22float2(*reinterpret_cast<const __half2*>(static_cast<const __half*>(a) + q * CP + c));
          const float2 l = __half22float2(*reinterpret_cast<const __half2*>(static_cast<const __half*>(alo) + q * CP + c));
          f.x += l.x; f.y += l.y;
        } else {
          f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(static_cast<const __nv_bfloat16*>(a) + q * CP + c));
        }
      }
      *reinterpret_cast<float2*>(sa + vv * LA + c) = f;
    }
    __syncthreads();
    for (int vv = grp; vv < VS; vv += NG) {
      const float4 g0 = *reinterpret_cast<const float4*>(sg + vv * LG + co0);
      const float4 g1 = *reinterpret_cast<const float4*>(sg + vv * LG + co0 + 4);
      const float4 aa = *reinterpret_cast<const float4*>(sa + vv * LA + ci0);
      const float gv[TCO] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
      const float av[TCI] = {aa.x, aa.y, aa.z, aa.w};
#pragma unroll
      for (int i = 0; i < TCO; ++i)
#pragma unroll
        for (int j = 0; j < TCI; ++j) acc[i][j] = fmaf(gv[i], av[j], acc[i][j]);
      if (centre) {
#pragma unroll
        for (int i = 0; i < TCO; ++i) accb[i] += gv[i];
      }
    }
    __syncthreads();
  }
  // the groups' tiles: red[grp][lt][e], e = i TCI + j; entry o = lt NE + e of
  // a group is (co0(lt) + e / TCI, ci0(lt) + e % TCI)
  float* red = sbuf;
#pragma unroll
  for (int e = 0; e < NE; ++e) red[(grp * TG + lt) * NE + e] = acc[e / TCI][e % TCI];
  __syncthreads();
  for (int o = tid; o < TG * NE; o += 256) {
    float sum = 0.f;
    for (int k = 0; k < NG; ++k) sum += red[k * TG * NE + o];
    const int l2 = o / NE, e = o % NE;
    const int co = TCO * (l2 / (CI / TCI)) + e / TCI, ci = TCI * (l2 % (CI / TCI)) + e % TCI;
    if (co < cout && ci < cin) atomicAdd(&gw[((long long)co * cin + ci) * 27 + t], double(sum));
  }
  if (!centre) return;  // uniform per block
  __syncthreads();
  // bias: the threads with ci0 = 0 hold every co once per group
  if (ci0 == 0) {
#pragma unroll
    for (int i = 0; i < TCO; ++i) red[grp * CO + co0 + i] = accb[i];
  }
  __syncthreads();
  if (tid < CO) {
    float sum = 0.f;
    for (int k = 0; k < NG; ++k) sum += red[k * CO + tid];
    if (tid < cout) atomicAdd(&gb[tid], double(sum));
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <int KN, int CP, int COP> static size_t conv_smem() {
  // + the mbarriers (4 steps, 2 x kSlots rows, 6 blocks), the TMEM slot and the abort flag
  return size_t(3 * kSlots) * (CP / 8) * row_plane<KN>() + size_t(27) * (CP / 8) * COP * 16 + 192;
}

template <int KN, int CP, int COP, int MODE, bool F16 = false> static void conv_attr() {
  cudaFuncSetAttribute(k_conv3<KN, CP, COP, MODE, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       int(conv_smem<KN, CP, COP>()));
}

// in: channels-last 16-bit input (BF16, or FP16 when F16); w: packed 16-bit
// weights of the same type.  The tensor maps are encoded with the BF16 element
// type for both: a bulk tensor copy moves 16-bit elements without converting
// them, and its zero fill is the all-zero bit pattern, +0 in either type.
template <int KN, int CP, int COP, int MODE, bool F16 = false>
static void conv_launch(int grid, const void* in, const void* w, const float* b, const ConvOut& o, int* err,
                        long long wait_limit, cudaStream_t st) {
  // one map per 8-channel chunk of the channels-last input [z][y][x][CP]:
  // dims (8 channels, x, y, z), boxes of 8 channels x (KN + 2) voxels of one row
  ConvMaps maps{};
  const unsigned long long dims[4] = {8, KN, KN, KN};
  const unsigned long long str[3] = {CP * 2ull, KN * CP * 2ull, (unsigned long long)KN * KN * CP * 2ull};
  const unsigned box[4] = {8, KN + 2, 1, 1};
  bool enc = true;
  for (int c = 0; c < CP / 8; ++c)
    enc = enc && tma_encode_bf16_4d(&maps.m[c], static_cast<const unsigned char*>(in) + 16 * c, dims, str, box);
  if (!enc) {  // no tensor-map encoder: report it through the closure's error flag
    k_set_flag<<<1, 1, 0, st>>>(err);
    return;
  }
  k_conv3<KN, CP, COP, MODE, F16><<<grid, kConvThreads, conv_smem<KN, CP, COP>(), st>>>(
      maps, static_cast<const __nv_bfloat16*>(w), b, o, err, wait_limit);
}

// One layer in split precision: three passes A_hi W_hi (kLinear), A_lo W_hi
// (kAccum) and A_hi W_lo (FIN), all accumulating in the FP32 buffer o.pre.  The
// dropped A_lo W_lo term is below the representation error of the parts.
template <int KN, int CP, int COP, int FIN, bool F16>
static void conv_split(int grid, const void* in_h, const void* in_l, const void* w_h, const void* w_l, const float* b,
                       const ConvOut& o, int* err, long long wait_limit, cudaStream_t st) {
  conv_launch<KN, CP, COP, kLinear, F16>(grid, in_h, w_h, nullptr, o, err, wait_limit, st);
  conv_launch<KN, CP, COP, kAccum, F16>(grid, in_l, w_h, nullptr, o, err, wait_limit, st);
  conv_launch<KN, CP, COP, FIN, F16>(grid, in_h, w_l, b, o, err, wait_limit, st);
}

bool cnn_supported(int n, int D) { return (n == 64 || n == 128) && D == 3; }

void launch_redelta(const double* a2, double* z, double delta, double nu, double mu, double sigma, cudaStream_t st) {
  k_cnn_redelta<<<1, 1, 0, st>>>(a2, z, delta, nu, mu, sigma);
}

template <int KN> static void cnn_init_n() {
  conv_attr<KN, 16, 32, kGelu>();
  conv_attr<KN, 32, 32, kGelu>();
  conv_attr<KN, 32, 16, kTau>();
  conv_attr<KN, 16, 32, kGeluSave>();
  conv_attr<KN, 32, 32, kGeluSave>();
  conv_attr<KN, 16, 32, kLinear>();
  conv_attr<KN, 32, 32, kLinear>();
  conv_attr<KN, 32, 16, kLinear>();
  // split precision: FP16 forward passes, BF16 input-gradient passes
  conv_attr<KN, 16, 32, kLinear, true>();
  conv_attr<KN, 16, 32, kAccum, true>();
  conv_attr<KN, 16, 32, kGeluSplit, true>();
  conv_attr<KN, 32, 32, kLinear, true>();
  conv_attr<KN, 32, 32, kAccum, true>();
  conv_attr<KN, 32, 32, kGeluSplit, true>();
  conv_attr<KN, 32, 16, kLinear, true>();
  conv_attr<KN, 32, 16, kAccum, true>();
  conv_attr<KN, 32, 16, kTauSplit, true>();
  conv_attr<KN, 16, 32, kAccum>();
  conv_attr<KN, 32, 32, kAccum>();
  conv_attr<KN, 32, 16, kAccum>();
}

void cnn_init() {
  cnn_init_n<64>();
  cnn_init_n<128>();
}

static unsigned nblk(long long n) { return unsigned((n + 255) / 256); }

template <int KN> static void cnn_forward_n(const CnnArgs& a, cudaStream_t st) {
  const long long npts = (long long)KN * KN * KN;
  k_cnn_redelta<<<1, 1, 0, st>>>(a.a2, a.z, a.delta, a.nu, a.mu, a.sigma);
  k_cnn_input<<<nblk(npts), 256, 0, st>>>(static_cast<const float*>(a.u[0]), static_cast<const float*>(a.u[1]),
                                          static_cast<const float*>(a.u[2]), a.z, a.act0, npts);
  const int grid = a.nsm > 0 ? a.nsm : 148;
  ConvOut o1{}, o2{}, o3{}, o4{};
  o1.act = a.act1; o1.pre = a.pre[0];
  o2.act = a.act2; o2.pre = a.pre[1];
  __nv_bfloat16* a3 = a.act3 ? a.act3 : a.act1;
  o3.act = a3; o3.pre = a.pre[2];
  o4.tau = a.tau;
  if (a.pre[0]) {
    conv_launch<KN, 16, 32, kGeluSave>(grid, a.act0, a.w[0], a.b[0], o1, a.err, a.wait_limit, st);
    conv_launch<KN, 32, 32, kGeluSave>(grid, a.act1, a.w[1], a.b[1], o2, a.err, a.wait_limit, st);
    conv_launch<KN, 32, 32, kGeluSave>(grid, a.act2, a.w[2], a.b[2], o3, a.err, a.wait_limit, st);
  } else {
    conv_launch<KN, 16, 32, kGelu>(grid, a.act0, a.w[0], a.b[0], o1, a.err, a.wait_limit, st);
    conv_launch<KN, 32, 32, kGelu>(grid, a.act1, a.w[1], a.b[1], o2, a.err, a.wait_limit, st);
    conv_launch<KN, 32, 32, kGelu>(grid, a.act2, a.w[2], a.b[2], o3, a.err, a.wait_limit, st);
  }
  conv_launch<KN, 32, 16, kTau>(grid, a3, a.w[3], a.b[3], o4, a.err, a.wait_limit, st);
}

// split precision: FP16 hi/lo inputs and weights, three passes per layer,
// exact GELU; layer l accumulates in pre[l] when given (the adjoint keeps h
// there), else in acc; layer 4 always in acc
template <int KN> static void cnn_forward_split_n(const CnnArgs& a, cudaStream_t st) {
  const long long npts = (long long)KN * KN * KN;
  k_cnn_redelta<<<1, 1, 0, st>>>(a.a2, a.z, a.delta, a.nu, a.mu, a.sigma);
  k_cnn_input_split<<<nblk(npts), 256, 0, st>>>(static_cast<const float*>(a.u[0]), static_cast<const float*>(a.u[1]),
                                                static_cast<const float*>(a.u[2]), a.z, a.acth[0], a.actl[0], npts);
  const int grid = a.nsm > 0 ? a.nsm : 148;
  ConvOut o[4] = {};
  for (int l = 0; l < 3; ++l) {
    o[l].pre = a.pre[l] ? a.pre[l] : a.acc;
    o[l].acth = a.acth[l + 1];
    o[l].actl = a.actl[l + 1];
    o[l].scale = 1.f / kSplitScale;
  }
  o[3].pre = a.acc;
  o[3].tau = a.tau;
  o[3].scale = 1.f / kSplitScale;
  conv_split<KN, 16, 32, kGeluSplit, true>(grid, a.acth[0], a.actl[0], a.wh[0], a.wl[0], a.b[0], o[0], a.err,
                                           a.wait_limit, st);
  conv_split<KN, 32, 32, kGeluSplit, true>(grid, a.acth[1], a.actl[1], a.wh[1], a.wl[1], a.b[1], o[1], a.err,
                                           a.wait_limit, st);
  conv_split<KN, 32, 32, kGeluSplit, true>(grid, a.acth[2], a.actl[2], a.wh[2], a.wl[2], a.b[2], o[2], a.err,
                                           a.wait_limit, st);
  conv_split<KN, 32, 16, kTauSplit, true>(grid, a.acth[3], a.actl[3], a.wh[3], a.wl[3], a.b[3], o[3], a.err,
                                          a.wait_limit, st);
}

void launch_cnn_forward(const CnnArgs& a, cudaStream_t st) {
  if (a.split) {
    if (a.n == 64) cnn_forward_split_n<64>(a, st);
    else cnn_forward_split_n<128>(a, st);
    return;
  }
  if (a.n == 64) cnn_forward_n<64>(a, st);
  else cnn_forward_n<128>(a, st);
}

// CI, CO: the layer's channels rounded up to the register tile (4 | 32 inputs, 8 | 32 outputs)
template <int KN, int CP, int COP, int CI, int CO, bool SPLIT = false>
static void wgrad_launch(const __nv_bfloat16* g, const void* act, int cin, int cout, double* gw, double* gb,
                         cudaStream_t st, const __nv_bfloat16* glo = nullptr, const void* alo = nullptr) {
  constexpr long long npts = (long long)KN * KN * KN;
  const int vchunk = KN >= 128 ? 16384 : 4096;  // 27 x 128 | 27 x 64 blocks: about 6 and 3 full waves
  dim3 grid(27, unsigned((npts + vchunk - 1) / vchunk));
  k_conv_wgrad<KN, CP, COP, CI, CO, SPLIT><<<grid, 256, 0, st>>>(g, glo, act, alo, cin, cout, vchunk, gw, gb);
}

template <int KN> static void cnn_backward_n(const CnnBwdArgs& a, cudaStream_t st) {
  const long long npts = (long long)KN * KN * KN;
  const int grid = a.nsm > 0 ? a.nsm : 148;
  // layer 4: g4 = dL/dtau (BF16 [v][16]); input gradient through W4^T; weight gradient against act3
  k_gtau_cl<<<nblk(npts), 256, 0, st>>>(a.gtau, a.gbf, npts);
  wgrad_launch<KN, 32, 16, 32, 8>(a.gbf, a.act[3], 32, 6, a.gw + a.woff[3], a.gw + a.woff[3] + 6 * 32 * 27, st);
  ConvOut o{};
  o.pre = a.gf;
  conv_launch<KN, 16, 32, kLinear>(grid, a.gbf, a.wt[3], nullptr, o, a.err, a.wait_limit, st);
  // layers 3, 2: g_pre = g_post * gelu'(h); input and weight gradients
  for (int l = 2; l >= 1; --l) {
    k_gelu_bwd_cl<<<nblk(npts * 32), 256, 0, st>>>(a.gf, a.pre[l], a.gbf, npts * 32);
    wgrad_launch<KN, 32, 32, 32, 32>(a.gbf, a.act[l], 32, 32, a.gw + a.woff[l], a.gw + a.woff[l] + 32 * 32 * 27, st);
    conv_launch<KN, 32, 32, kLinear>(grid, a.gbf, a.wt[l], nullptr, o, a.err, a.wait_limit, st);
  }
  // layer 1: input gradient into 16 channels (4 used), then planar
  k_gelu_bwd_cl<<<nblk(npts * 32), 256, 0, st>>>(a.gf, a.pre[0], a.gbf, npts * 32);
  wgrad_launch<KN, 16, 32, 4, 32>(a.gbf, a.act[0], 4, 32, a.gw + a.woff[0], a.gw + a.woff[0] + 32 * 4 * 27, st);
  conv_launch<KN, 32, 16, kLinear>(grid, a.gbf, a.wt[0], nullptr, o, a.err, a.wait_limit, st);
  k_gin_planar<<<nblk(npts), 256, 0, st>>>(a.gf, a.gin_planar, npts);
}

// split precision: BF16 hi/lo gradients and transposed weights (three passes
// per input-gradient convolution), weight gradients from the hi + lo sums
template <int KN> static void cnn_backward_split_n(const CnnBwdArgs& a, cudaStream_t st) {
  const long long npts = (long long)KN * KN * KN;
  const int grid = a.nsm > 0 ? a.nsm : 148;
  ConvOut o{};
  o.pre = a.gf;
  k_gtau_cl_split<<<nblk(npts), 256, 0, st>>>(a.gtau, a.gbf, a.gbf_lo, npts);
  wgrad_launch<KN, 32, 16, 32, 8, true>(a.gbf, a.acth[3], 32, 6, a.gw + a.woff[3], a.gw + a.woff[3] + 6 * 32 * 27, st,
                                 a.gbf_lo, a.actl[3]);
  conv_split<KN, 16, 32, kAccum, false>(grid, a.gbf, a.gbf_lo, a.wt[3], a.wtl[3], nullptr, o, a.err, a.wait_limit, st);
  for (int l = 2; l >= 1; --l) {
    k_gelu_bwd_cl_split<<<nblk(npts * 32), 256, 0, st>>>(a.gf, a.pre[l], a.gbf, a.gbf_lo, npts * 32);
    wgrad_launch<KN, 32, 32, 32, 32, true>(a.gbf, a.acth[l], 32, 32, a.gw + a.woff[l], a.gw + a.woff[l] + 32 * 32 * 27, st,
                                   a.gbf_lo, a.actl[l]);
    conv_split<KN, 32, 32, kAccum, false>(grid, a.gbf, a.gbf_lo, a.wt[l], a.wtl[l], nullptr, o, a.err, a.wait_limit,
                                          st);
  }
  k_gelu_bwd_cl_split<<<nblk(npts * 32), 256, 0, st>>>(a.gf, a.pre[0], a.gbf, a.gbf_lo, npts * 32);
  wgrad_launch<KN, 16, 32, 4, 32, true>(a.gbf, a.acth[0], 4, 32, a.gw + a.woff[0], a.gw + a.woff[0] + 32 * 4 * 27, st,
                                 a.gbf_lo, a.actl[0]);
  conv_split<KN, 32, 16, kAccum, false>(grid, a.gbf, a.gbf_lo, a.wt[0], a.wtl[0], nullptr, o, a.err, a.wait_limit, st);
  k_gin_planar<<<nblk(npts), 256, 0, st>>>(a.gf, a.gin_planar, npts);
}

void launch_cnn_backward(const CnnBwdArgs& a, cudaStream_t st) {
  if (a.split) {
    if (a.n == 64) cnn_backward_split_n<64>(a, st);
    else cnn_backward_split_n<128>(a, st);
    return;
  }
  if (a.n == 64) cnn_backward_n<64>(a, st);
  else cnn_backward_n<128>(a, st);
}

}  // namespace sc
