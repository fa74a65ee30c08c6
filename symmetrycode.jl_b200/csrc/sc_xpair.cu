// 3D x sweep with the Navier-Stokes products for N = 810, rows processed in
// pairs on the packed f32x2 pipe (sm_100a).
//
// One 96-thread CTA owns the two rows r, r' = r + 1 of every component.  Each
// complex value in registers and shared memory is a P2 (sc_pair.cuh) holding
// the same point of row r (lane a) and row r' (lane b), so every butterfly,
// twiddle and product runs once for both rows.  Per row pair the sweep does
// two inverse pair transforms and three forward pair transforms:
//   inverse pencil A: u1 + i u2 (Hermitian-extended c2r of both rows)
//   inverse pencil B: u3 (each lane a Hermitian pencil; its imaginary output is 0)
//   forward kinds:    (u1 u1 + i u2 u2), (u3 u3 + i u1 u2), (u2 u3 + i u3 u1)
// 810 = 9 * 9 * 10 with the pass structure of a three-level sweep:
//   Ia  t = 9 q + m2 (81 threads): radix-10 over p of Z[81 p + t] (gathered
//       from the staged rows), twiddle exp(+2 pi i q s_a / 90)           -> X
//   Ib  t = 9 s_a + m2 (90): radix-9 over q, twiddle exp(+2 pi i m2 s1/810)-> Y
//   Ic  t = s1 (90): radix-9 over m2 -> physical x = s1 + 90 s2 in registers
//   F1  the same thread forms the three products at its 9 points, radix-9
//       over m1, twiddle exp(-2 pi i m2 s1' / 810)                        -> W
//   F2  t = 10 s1' + q (90): radix-9 over p, twiddle exp(-2 pi i q s_a/90) -> V
//   F3  t = 9 s1' + s_a (81): radix-10 over q, retained k only           -> Z
//   S   split the paired spectra of each row and store the six product rows.
// Because the last inverse pass leaves every thread holding exactly the points
// its first forward pass needs, the products never go through shared memory.
// Shared memory: three pair slots of PS P2 (16 B) each, 42 KB, five CTAs per
// SM; the staged input rows alias slot 2 until Ia has consumed them.  Element
// index maps (X: 89 s_a + 9 q + m2; Y: 90 s_b + 9 s_a + m2; W: 90 s + m2;
// V: 90 s1' + 9 q + s_a) keep every exchange free of 16-byte bank conflicts
// except the F3 loads (no linear V layout serves both the F2 stores and the
// F3 loads).
#include "sc_fft.cuh"
#include "sc_internal.h"
#include "sc_pair.cuh"

namespace sc {

namespace {

constexpr int kXN = 810, kXT = 96, kXPS = 882;
constexpr size_t kXSmem = size_t(3) * kXPS * sizeof(P2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Paired twiddle exp(-2 pi i j / 810) from the plan's pair table (C, S, NS, pad).
__device__ __forceinline__ TwP twp(const float4* __restrict__ t4, int j) {
  const float4 a = __ldg(t4 + 2 * j), b = __ldg(t4 + 2 * j + 1);
  return {make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y)};
}

// Hermitian extension of one real row from its staged half spectrum (kmax + 1
// modes): Z[k] = U[k] for k <= kmax, conj(U[N - k]) for k >= N - kmax, else 0;
// the mean's imaginary part is dropped (a real row's c2r ignores it).
__device__ __forceinline__ float2 hrow(const float2* r, int k, bool direct, bool mirror) {
  if (direct) {
    float2 x = r[k];
    if (k == 0) x.y = 0.f;
    return x;
  }
  if (mirror) {
    const float2 x = r[kXN - k];
    return make_float2(x.x, -x.y);
  }
  return make_float2(0.f, 0.f);
}

// Which k = 81 p + t are retained (FULL: kmax = 270, known per p).
template <bool FULL>
__device__ __forceinline__ void kclass(int p, int t, int kmax, bool& direct, bool& mirror) {
  const int k = 81 * p + t;
  if (FULL) {
    direct = p <= 2 || (p == 3 && t <= 27);
    mirror = p >= 7 || (p == 6 && t >= 54);
  } else {
    direct = k <= kmax;
    mirror = k >= kXN - kmax;
  }
}

// Products of both rows at this thread's 9 points, first forward radix-9, twiddle.
template <int KIND>
__device__ __forceinline__ void f1_kind(const float2* u1, const float2* u2, const float2* u3,
                                        const TwP* wf, P2* slot, int t) {
  P2 v[9];
#pragma unroll
  for (int m1 = 0; m1 < 9; ++m1) {
    const float2 a = KIND == 0 ? u1[m1] : KIND == 1 ? u3[m1] : u2[m1];
    const float2 b = KIND == 0 ? u1[m1] : u3[m1];
    const float2 c = KIND == 0 ? u2[m1] : u1[m1];
    const float2 d = KIND == 2 ? u3[m1] : u2[m1];
    v[m1] = {mul2(a, b), mul2(c, d)};
  }
  PDFT<9, false>::run(v);
  P2* ws = slot + t;
  ws[0] = v[0];
#pragma unroll
  for (int s = 1; s < 9; ++s) ws[90 * s] = pmul(v[s], wf[s]);
}

// MINB: CTAs per SM the register budget is cut for (5: 128 registers; 4: 168,
// room to keep the DFT constants' register pairs resident)
template <bool FULL, int MINB>
__global__ void __launch_bounds__(kXT, MINB) k_xpair810(const XArgs a, const float4* __restrict__ t4) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  P2* s0 = reinterpret_cast<P2*>(smem_raw);
  P2* s1 = s0 + kXPS;
  P2* s2 = s1 + kXPS;
  const int t = threadIdx.x;
  const long long r0 = (long long)blockIdx.x * 2;
  const bool has1 = r0 + 1 < a.nrows;
  const int K1 = FULL ? 271 : a.K1in, kmax = K1 - 1;
  const int K1o = FULL ? 271 : a.K1out, ko = K1o - 1;
  const long long ldo = a.ldo > 0 ? a.ldo : K1o;

  // L: stage the six rows (u1, u2, u3 of r and r') into slot 2, [c][row][K1]
  float2* rin = reinterpret_cast<float2*>(s2);
  {
    const float2* in0 = static_cast<const float2*>(a.in[0]);
    const float2* in1 = static_cast<const float2*>(a.in[1]);
    const float2* in2 = static_cast<const float2*>(a.in[2]);
    // FULL with both rows: rows r0 (even) and r0 + 1 of a component are 2 x 271
    // contiguous elements starting 4336 r0 / 2 bytes into it
    const bool pair16 =
        FULL && has1 &&
        ((reinterpret_cast<unsigned long long>(in0) | reinterpret_cast<unsigned long long>(in1) |
          reinterpret_cast<unsigned long long>(in2)) & 15) == 0;
    if (pair16) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2* src = (c == 0 ? in0 : c == 1 ? in1 : in2) + r0 * K1;
        float2* dst = rin + 2 * c * K1;
        for (int j = t; j < K1; j += kXT) cp_async16(dst + 2 * j, src + 2 * j);
      }
    } else {
      for (int i = t; i < 6 * K1; i += kXT) {
        const int cr = i / K1, kx = i - cr * K1;
        const float2* src = cr < 2 ? in0 : cr < 4 ? in1 : in2;
        float2* dst = rin + i;
        if ((cr & 1) == 0 || has1) cp_async8(dst, src + (r0 + (cr & 1)) * K1 + kx);
        else *dst = make_float2(0.f, 0.f);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  }
  __syncthreads();

  // Ia: pencil A (u1 + i u2) -> slot 0, pencil B (u3) -> slot 1
  if (t < 81) {
    const int q = t / 9;
    const float2* u1a = rin;           // row r
    const float2* u1b = rin + K1;      // row r'
    const float2* u2a = rin + 2 * K1;
    const float2* u2b = rin + 3 * K1;
    const float2* u3a = rin + 4 * K1;
    const float2* u3b = rin + 5 * K1;
    TwP w[10];  // the pass's twiddles, loaded once and used by both pencils
#pragma unroll
    for (int sa = 1; sa < 10; ++sa) w[sa] = twp(t4, 9 * q * sa);
#pragma unroll 1
    for (int j = 0; j < 2; ++j) {
      P2 v[10];
#pragma unroll
      for (int p = 0; p < 10; ++p) {
        if (FULL && (p == 4 || p == 5)) { v[p] = pzero(); continue; }  // 324 <= k <= 485 never retained
        bool direct, mirror;
        kclass<FULL>(p, t, kmax, direct, mirror);
        const int k = 81 * p + t;
        if (j == 0) {
          const float2 xa = hrow(u1a, k, direct, mirror), ya = hrow(u2a, k, direct, mirror);
          const float2 xb = hrow(u1b, k, direct, mirror), yb = hrow(u2b, k, direct, mirror);
          v[p] = {make_float2(xa.x - ya.y, xb.x - yb.y), make_float2(xa.y + ya.x, xb.y + yb.x)};
        } else {
          const float2 xa = hrow(u3a, k, direct, mirror), xb = hrow(u3b, k, direct, mirror);
          v[p] = {make_float2(xa.x, xb.x), make_float2(xa.y, xb.y)};
        }
      }
      PDFT<10, true>::run(v);
      P2* xs = (j == 0 ? s0 : s1) + t;
      xs[0] = v[0];
#pragma unroll
      for (int sa = 1; sa < 10; ++sa) xs[89 * sa] = pmulc(v[sa], w[sa]);
    }
  }
  __syncthreads();
  // Ib: A: slot 0 -> slot 2 (the staged rows are consumed); B: slot 1 in place
  {
    const int sa = t / 9, m2 = t - 9 * sa;
    TwP w[9];
    if (t < 90) {
#pragma unroll
      for (int sb = 0; sb < 9; ++sb) w[sb] = twp(t4, m2 * (sa + 10 * sb));
    }
#pragma unroll 1
    for (int j = 0; j < 2; ++j) {
      P2 v[9];
      if (t < 90) {
        const P2* xs = (j == 0 ? s0 : s1) + 89 * sa + m2;
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = xs[9 * q];
        PDFT<9, true>::run(v);
#pragma unroll
        for (int sb = 0; sb < 9; ++sb) v[sb] = pmulc(v[sb], w[sb]);
      }
      if (j == 1) __syncthreads();  // every read of slot 1 is done before it is overwritten
      if (t < 90) {
        P2* ys = (j == 0 ? s2 : s1) + t;
#pragma unroll
        for (int sb = 0; sb < 9; ++sb) ys[90 * sb] = v[sb];
      }
    }
  }
  __syncthreads();
  // Ic + F1: physical velocities of both rows at x = t + 90 s2, then the products
  {
    float2 u1[9], u2[9], u3[9];
    TwP wf[9];
    if (t < 90) {
#pragma unroll
      for (int s = 1; s < 9; ++s) wf[s] = twp(t4, t * s);
      P2 v[9];
      const P2* ya = s2 + 9 * t;
#pragma unroll
      for (int m2 = 0; m2 < 9; ++m2) v[m2] = ya[m2];
      PDFT<9, true>::run(v);
#pragma unroll
      for (int s = 0; s < 9; ++s) { u1[s] = v[s].re; u2[s] = v[s].im; }
      const P2* yb = s1 + 9 * t;
#pragma unroll
      for (int m2 = 0; m2 < 9; ++m2) v[m2] = yb[m2];
      PDFT<9, true>::run(v);
#pragma unroll
      for (int s = 0; s < 9; ++s) u3[s] = v[s].re;
      f1_kind<0>(u1, u2, u3, wf, s0, t);  // slot 0 is free
    }
    __syncthreads();
    if (t < 90) {
      f1_kind<1>(u1, u2, u3, wf, s1, t);
      f1_kind<2>(u1, u2, u3, wf, s2, t);
    }
  }
  __syncthreads();
  // F2, in place per slot
  {
    const int s1i = t / 10, q = t - 10 * s1i;
    TwP w[9];
    if (t < 90) {
#pragma unroll
      for (int s = 1; s < 9; ++s) w[s] = twp(t4, 9 * q * s);
    }
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      P2* sl = j == 0 ? s0 : j == 1 ? s1 : s2;
      P2 v[9];
      if (t < 90) {
        const P2* ws = sl + 90 * s1i + q;
#pragma unroll
        for (int p = 0; p < 9; ++p) v[p] = ws[10 * p];
        PDFT<9, false>::run(v);
#pragma unroll
        for (int s = 1; s < 9; ++s) v[s] = pmul(v[s], w[s]);
      }
      __syncthreads();
      if (t < 90) {
        P2* vs = sl + 90 * s1i + 9 * q;
#pragma unroll
        for (int s = 0; s < 9; ++s) vs[s] = v[s];
      }
    }
  }
  __syncthreads();
  // F3, in place per slot, pruned to the retained modes (outputs s_b = 4, 5,
  // k in [324, 485], are never retained and are not formed)
  {
    const int s1i = t / 9, sa = t - 9 * s1i;
    const int kb = s1i + 9 * sa;
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
      P2* sl = j == 0 ? s0 : j == 1 ? s1 : s2;
      P2 v[10];
      if (t < 81) {
        const P2* vs = sl + 90 * s1i + sa;
#pragma unroll
        for (int q = 0; q < 10; ++q) v[q] = vs[9 * q];
        PDFT<10, false>::run(v);
      }
      __syncthreads();
      if (t < 81) {
#pragma unroll
        for (int sb = 0; sb < 10; ++sb) {
          if (sb == 4 || sb == 5) continue;
          const int k = kb + 81 * sb;
          if (FULL) {
            if (sb <= 2 || (sb == 3 && k <= 270)) sl[k] = v[sb];
            else if (sb >= 7 || (sb == 6 && k >= 540)) sl[270 + (kXN - k)] = v[sb];
          } else {
            if (k <= ko) sl[k] = v[sb];
            else if (k >= kXN - ko) sl[ko + (kXN - k)] = v[sb];
          }
        }
      }
    }
  }
  __syncthreads();
  // S: split each row's paired spectrum Z = X + i Y (X, Y the spectra of two
  // real products): X[k] = (Z[k] + conj Z[-k]) / 2, Y[k] = (Z[k] - conj Z[-k]) / 2i;
  // the 1/n^3 of to_spec rides on the 1/2
  const float hsc = 0.5f * float(a.scale);
  float2* o[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) o[c] = static_cast<float2*>(a.out[c]);
  for (int kx = t; kx < K1o; kx += kXT) {
    const int kc = kx == 0 ? 0 : ko + kx;
    const long long oa = r0 * ldo + kx, ob = oa + ldo;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const P2* zs = b == 0 ? s0 : b == 1 ? s1 : s2;
      const P2 z = zs[kx], zc = zs[kc];
      const float2 xr = mul2(add2(z.re, zc.re), c2(hsc));   // Re X, both rows
      const float2 xi = mul2(sub2(z.im, zc.im), c2(hsc));   // Im X
      const float2 yr = mul2(add2(z.im, zc.im), c2(hsc));   // Re Y
      const float2 yi = mul2(sub2(zc.re, z.re), c2(hsc));   // Im Y
      o[2 * b][oa] = make_float2(xr.x, xi.x);
      o[2 * b + 1][oa] = make_float2(yr.x, yi.x);
      if (has1) {
        o[2 * b][ob] = make_float2(xr.y, xi.y);
        o[2 * b + 1][ob] = make_float2(yr.y, yi.y);
      }
    }
  }
}

}  // namespace

size_t xpair810_twiddle_bytes() { return size_t(kXN) * 2 * sizeof(float4); }

// The pair twiddle table: entry j = exp(-2 pi i j / 810) as (c, c, s, s, -s, -s, 0, 0).
void xpair810_twiddles(const float2* tw, float* out8) {
  for (int j = 0; j < kXN; ++j) {
    const float c = tw[j].x, s = tw[j].y;
    float* e = out8 + 8 * j;
    e[0] = c; e[1] = c; e[2] = s; e[3] = s; e[4] = -s; e[5] = -s; e[6] = 0.f; e[7] = 0.f;
  }
}

bool init_xpair810() {
  cudaFuncSetAttribute(k_xpair810<true, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kXSmem));
  cudaFuncSetAttribute(k_xpair810<false, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kXSmem));
  cudaFuncSetAttribute(k_xpair810<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kXSmem));
  cudaFuncSetAttribute(k_xpair810<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kXSmem));
  return cudaGetLastError() == cudaSuccess;
}

void launch_xpair810(const XArgs& a, const void* twp_table, int minb, cudaStream_t st) {
  const unsigned nb = unsigned((a.nrows + 1) / 2);
  const float4* t4 = static_cast<const float4*>(twp_table);
  const bool full = a.K1in == 271 && a.K1out == 271;
  if (minb == 4) {
    if (full) k_xpair810<true, 4><<<nb, kXT, kXSmem, st>>>(a, t4);
    else k_xpair810<false, 4><<<nb, kXT, kXSmem, st>>>(a, t4);
  } else {
    if (full) k_xpair810<true, 5><<<nb, kXT, kXSmem, st>>>(a, t4);
    else k_xpair810<false, 5><<<nb, kXT, kXSmem, st>>>(a, t4);
  }
}

}  // namespace sc
