// Allocation-free spectrum: sc_spectrum_static (include/symcode.h).
//
// The energy spectrum of sc_spectrum (src/solver.jl:693-699), computed straight
// from the full RFFT layout (n/2+1, n[, n]) without a plan and without any
// device allocation.  Who needs this: a monitor that runs between the time steps
// of a large DNS whose device memory is already committed to the solver's state
// and work buffers.  sc_spectrum would set up a plan there (work buffers of
// several field sizes) and take a stream-ordered buffer for its shell sums on
// every call; either can fail when memory is full, and a pool that has to grow
// or trim holds up the stream the solver steps on.  This entry point touches
// only the caller's field, the caller's host array and a fixed 4 KiB device
// array compiled into the library.
//
// The shell accumulators live in g_shell_scratch.  The first call on each
// device looks up its device address with that device current
// (cudaGetSymbolAddress); that lookup may load the module, so make the first
// call on each device before any stream capture begins.  The address is cached
// per device together with the id of the CUDA context it was looked up in; a
// call in a new context (after cudaDeviceReset, or a primary-context reset by
// another library in the process) repeats the lookup, so its first call comes
// before any capture too.  Every call on a device shares the one array: two
// calls that overlap in time, on other streams or from other host threads,
// race on it and both return wrong sums.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "sc_fft.cuh"
#include "sc_internal.h"
#include "symcode.h"

#define SC_STR2(x) #x
#define SC_STR(x) SC_STR2(x)

namespace {

// Shell sums of the current call; zeroed at the start of every call.
static __device__ __align__(256) double g_shell_scratch[SC_SPECTRUM_STATIC_MAX_SHELLS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
struct ScratchSlot {
  unsigned long long ctx_id;  // context the address belongs to (0: none yet)
  double* ptr;
};
ScratchSlot g_scratch[kMaxDevices] = {};

// Unique id of the calling thread's current CUDA context (ids are never reused
// within a process, unlike context handles).  The driver calls are reached
// through the runtime's entry-point table, so the library needs no -lcuda.
int current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1{}, q2{};
    cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
    cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
    if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
        q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return sc::api_fail(SC_ERR_CUDA, "cudaGetDriverEntryPoint(cuCtxGetCurrent / cuCtxGetId)", "");
    get_current = reinterpret_cast<GetCurrent>(f1);
    get_id = reinterpret_cast<GetId>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return sc::api_fail(SC_ERR_CUDA, "no current CUDA context", "");
  if (get_id(ctx, id) != CUDA_SUCCESS) return sc::api_fail(SC_ERR_CUDA, "cuCtxGetId", "");
  return SC_OK;
}

// Device address of g_shell_scratch in the current device's current context
// (looked up once per device and context).
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "cudaGetDevice", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return sc::api_fail(SC_ERR_UNSUPPORTED, "device ordinal beyond 63", "");
  // initialise the device's primary context and make it current (CUDA >= 12:
  // cudaSetDevice does both; a no-op when it already is)
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "cudaSetDevice", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  unsigned long long id = 0;
  int rc = current_context_id(&id);
  if (rc) return rc;
  ScratchSlot& slot = g_scratch[dev];
  if (!slot.ptr || slot.ctx_id != id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_shell_scratch);
    if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "cudaGetSymbolAddress(shell scratch)", cudaGetErrorString(e));
    slot.ptr = static_cast<double*>(p);
    slot.ctx_id = id;
  }
  *out = slot.ptr;
  return SC_OK;
}

struct StaticSpecArgs {
  const void* u[3];
  int D, n, nshell;
};

// Variant of the compact-cube spectrum kernel: it walks the cube of half-width
// nshell (every mode with |k| < nshell + 1 has |k_i| <= nshell), indexes the
// full RFFT layout directly, and sums each block's shells in shared memory
// before one global atomic per shell.
template <typename R>
__global__ void k_spectrum_static(const StaticSpecArgs a, double* shell) {
  using C = typename sc::V2<R>::T;
  extern __shared__ double ssum[];
  for (int i = threadIdx.x; i < a.nshell; i += blockDim.x) ssum[i] = 0.0;
  __syncthreads();
  const int kw = a.nshell, K1 = kw + 1, K2 = 2 * kw + 1, nx = a.n / 2 + 1;
  const long long nm = (long long)K1 * K2 * (a.D == 3 ? K2 : 1);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long long)gridDim.x * blockDim.x) {
    const int ix = int(i % K1);
    const long long r = i / K1;
    const int py = int(r % K2), pz = a.D == 3 ? int(r / K2) : 0;
    const int iy = py <= kw ? py : py - K2, iz = pz <= kw ? pz : pz - K2;
    const long long k2 = (long long)ix * ix + (long long)iy * iy + (long long)iz * iz;
    int sh = int(sqrt(double(k2)));
    while ((long long)(sh + 1) * (sh + 1) <= k2) ++sh;
    while ((long long)sh * sh > k2) --sh;
    if (sh < 1 || sh > a.nshell) continue;
    const long long yy = iy < 0 ? iy + a.n : iy, zz = iz < 0 ? iz + a.n : iz;
    const long long idx = ix + nx * (yy + (long long)a.n * zz);
    double e = 0;
    for (int c = 0; c < a.D; ++c) {
      const C v = static_cast<const C*>(a.u[c])[idx];
      e += double(v.x) * v.x + double(v.y) * v.y;
    }
    atomicAdd(&ssum[sh - 1], 0.5 * (ix > 0 ? 2.0 : 1.0) * e);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < a.nshell; i += blockDim.x)
    if (ssum[i] != 0.0) atomicAdd(&shell[i], ssum[i]);
}

template <typename R>
void launch_spectrum_static(const StaticSpecArgs& a, double* shell, cudaStream_t st) {
  const long long kw = a.nshell;
  const long long nm = (kw + 1) * (2 * kw + 1) * (a.D == 3 ? (2 * kw + 1) : 1);
  long long nb = (nm + 255) / 256;
  if (nb > 148 * 4) nb = 148 * 4;
  k_spectrum_static<R><<<unsigned(nb), 256, a.nshell * sizeof(double), st>>>(a, shell);
}

}  // namespace

extern "C" {

int sc_spectrum_static(const void* const* u, int n, int D, int dtype, int nshell, double* s, void* stream) {
  if (!u || !s) return sc::api_fail(SC_ERR_INVALID, "null argument", "");
  if (D != 2 && D != 3) return sc::api_fail(SC_ERR_INVALID, "D must be 2 or 3", "");
  if (dtype != SC_FLOAT32 && dtype != SC_FLOAT64) return sc::api_fail(SC_ERR_INVALID, "unknown dtype", "");
  for (int c = 0; c < D; ++c)
    if (!u[c]) return sc::api_fail(SC_ERR_INVALID, "null field component", "");
  if (nshell > SC_SPECTRUM_STATIC_MAX_SHELLS)
    return sc::api_fail(SC_ERR_SIZE, "nshell exceeds the static shell scratch",
                        "at most " SC_STR(SC_SPECTRUM_STATIC_MAX_SHELLS) " shells");
  if (n < 4 || n % 2) return sc::api_fail(SC_ERR_SIZE, "n must be even and >= 4", "");
  if (nshell < 1 || nshell > n / 3)
    return sc::api_fail(SC_ERR_INVALID, "shells beyond n/3 are not retained", "need 1 <= nshell <= n/3");
  double* shell = nullptr;
  int rc = scratch_for_current_device(&shell);
  if (rc) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(shell, 0, nshell * sizeof(double), st);
  if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "cudaMemsetAsync(shell scratch)", cudaGetErrorString(e));
  StaticSpecArgs a{};
  for (int c = 0; c < D; ++c) a.u[c] = u[c];
  a.D = D; a.n = n; a.nshell = nshell;
  if (dtype == SC_FLOAT64) launch_spectrum_static<double>(a, shell, st);
  else launch_spectrum_static<float>(a, shell, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "spectrum_static launch", cudaGetErrorString(e));
  e = cudaMemcpyAsync(s, shell, nshell * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sc::api_fail(SC_ERR_CUDA, "spectrum_static result", cudaGetErrorString(e));
  return SC_OK;
}

}  // extern "C"
