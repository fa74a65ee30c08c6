// C ABI of the B200 pseudo-spectral Navier-Stokes path (declared in include/symcode.h).
//
// The plan object stands in for the reference's `Grid` + `getcache` pair
// (src/solver.jl:131-151, 956-965): it owns the twiddle table, the pencil
// scratch of the five-sweep pipeline and the compact 2/3-cube state buffers of
// the steppers.  The caller owns the fields it passes in.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "sc_fft.cuh"
#include "sc_internal.h"
#include "sc_les.h"
#include "sc_cnn.h"
#include "sc_cnn_cc.h"
#include "symcode.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define SC_CU(call)                                                                      \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(SC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return SC_OK;
}

}  // namespace

namespace sc {
int api_fail(int code, const char* what, const char* detail) {
  return detail && *detail ? fail(code, "%s: %s", what, detail) : fail(code, "%s", what);
}
}  // namespace sc

struct sc_plan {
  int D = 0, n = 0, dtype = 0, dev = 0;
  double l = 0;
  int kc = 0, K1 = 0, K2 = 0;
  size_t csz = 0;   // compact modes per component
  size_t fsz = 0;   // full-layout modes per component
  size_t esz = 0;   // bytes per complex
  size_t ws = 0;
  void* tw = nullptr;
  void* U[3] = {}, *ACC[3] = {}, *S[3] = {};
  void* sig[6] = {};
  void* be[6] = {};
  void* cc[3] = {};
  void* dd[6] = {};
  double* dscal = nullptr;  // [0] forcing A, [1] reduction accumulator
  int* err = nullptr;       // device word set when a bounded wait of a TMA-fed sweep ran out
  void* fa = nullptr, *fb = nullptr;  // full-spectrum scratch (lazy)
  std::vector<void*> allocs;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t g_rk4 = nullptr;
  double k_rk4[5] = {0, 0, 0, 0, 0};
  cudaGraphExec_t g_wray = nullptr;
  double k_wray[3] = {0, 0, 0};
  int use_graph = 1;  // SC_OPT_USE_GRAPH
  long long wait_limit = sc::kDefaultWaitLimit;  // SC_OPT_WAIT_LIMIT
  // kernel variant of each sweep of the product pipeline (SC_OPT_VARIANT_*:
  // z-inverse, y-inverse, x, y-forward, z-forward), chosen by the autotuner
  int variant[5] = {0, 0, 0, 0, 0};
};

// A closure model `model(u, G) -> tau` (src/les.jl:19, src/closures.jl) bound
// to a plan; owns the scratch its evaluation needs.
struct sc_closure {
  sc_plan* p = nullptr;
  int kind = 0;
  double delta = 0;
  double prm[4] = {0, 0, 0, 0};
  void* gc[9] = {};   // compact spectral scratch (gradient / filtered stress)
  void* gp[9] = {};   // physical scratch (gradient / L1)
  void* tp[6] = {};   // physical tau (and S, m1)
  void* th[6] = {};   // compact tau-hat (the closure's stress spectrum)
  void* ut[3] = {};   // compact test-filtered velocity
  void* s2[6] = {};   // compact strain / filtered F[m1]
  void* ph2[6] = {};  // physical M1
  void* ph3[6] = {};  // physical S~ then m2
  void* ph4[3] = {};  // physical test-filtered velocity
  void* bb[12] = {};  // batched-transform scratch (kx, ky, z), stored [ky][z][kx]
  void* cb[12] = {};  // batched-transform scratch (kx, y, z)
  double* dsum = nullptr;  // [<ML>, <MM>, c] (dynamic Smagorinsky); [a2, -, -, z] (CNN)
  // CNN closure
  void* cw[4] = {};   // packed BF16 weights per layer
  void* cbias[4] = {};
  void* act[3] = {};  // BF16 activations
  void* cwt[4] = {};  // packed BF16 transposed, flipped weights (input-gradient convolutions)
  void* tact3 = nullptr;        // adjoint: BF16 input of layer 4
  void* tpre[3] = {};           // adjoint: FP32 pre-activations
  void* tgbf = nullptr;         // adjoint: BF16 gradient scratch
  void* tgf = nullptr;          // adjoint: FP32 gradient scratch
  // split precision (SC_CLOPT_CNN_SPLIT): FP16 hi/lo forward weights (x kSplitScale),
  // BF16 low parts of the transposed weights, FP16 hi/lo activations, FP32 accumulator
  bool cnn_split = false;
  bool split_fits = true;       // the uploaded weights x kSplitScale are FP16 numbers
  void* cwh[4] = {};
  void* cwl[4] = {};
  void* cwtl[4] = {};
  void* sacth[4] = {};
  void* sactl[4] = {};
  void* sacc = nullptr;
  void* tgbfl = nullptr;        // adjoint: BF16 gradient scratch, low parts
  int* err = nullptr;
  double nu = 0, mu = 0, sigma = 1;
  // CUDA-core CNN (FP32/FP64): weights, activations a0 h1 a1 h2 a2 h3 a3, tau, gradients
  void* ccw[4] = {};
  void* ccb[4] = {};
  void* cca[7] = {};
  void* cctau = nullptr;   // [6][npts]
  void* ccg[2] = {};       // [32][npts] gradient ping-pong
  void* ccg0 = nullptr;    // [4][npts]
  double* gw = nullptr;    // flat parameter gradient (FP64)
  long long nparam = 0;
  // pointwise MLP closure
  int mlp_nl = 0;
  int mlp_w[sc::kMlpMaxLayers + 1] = {};
  void* mlp_theta = nullptr;
  double* mlp_z = nullptr;  // [sum |G|^2, z] when the Re_Delta channel is used
  std::vector<void*> allocs;
};

// Batched LES: several independent instances (own plan, state, closure, nu,
// dt, forcing) advanced by one CUDA graph per step with one branch per instance.
struct sc_les_batch {
  std::vector<sc_les_instance> inst;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
  std::vector<int> active;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t graph = nullptr;
  double* energy = nullptr;  // [ninst] FP64 energies of the last guard
  int* status = nullptr;     // [ninst] 0 ok, SC_ERR_DIVERGED
  int dev = 0;
  // fused a-posteriori reductions (sc_les_batch_set_snapshots): every `snap_every`
  // steps the snapshot graph (the step graph plus the reductions) runs instead
  cudaGraphExec_t snap_graph = nullptr;
  int snap_every = 0, nshell = 0, max_snap = 0;
  long long steps_done = 0;  // steps since the snapshots were configured
  int nsnap = 0;             // snapshots recorded (host count; the device keeps its own)
  double* scratch = nullptr; // [ninst][stride] reductions of the current snapshot
  double* snaps = nullptr;   // [max_snap][ninst][stride]
  int* dcount = nullptr;     // device snapshot counter
};

namespace {

int plan_alloc(sc_plan* p, void** out, size_t bytes) {
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SC_ERR_OOM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  }
  p->allocs.push_back(ptr);
  p->ws += bytes;
  *out = ptr;
  return SC_OK;
}

void plan_free(sc_plan* p) {
  if (p->g_rk4) cudaGraphExecDestroy(p->g_rk4);
  if (p->g_wray) cudaGraphExecDestroy(p->g_wray);
  for (void* a : p->allocs) cudaFree(a);
  p->allocs.clear();
  if (p->cap) cudaStreamDestroy(p->cap);
}

// Host image of a twiddle buffer: exp(-2 pi i m / n) from long double, and for
// FP32 n = 810 the x sweep's pair table after it (sc::twiddle_buffer_bytes).
template <typename R>
std::vector<unsigned char> twiddle_image(int n) {
  using C = typename sc::V2<R>::T;
  std::vector<unsigned char> img(sc::twiddle_buffer_bytes(n, sizeof(C)));
  C* h = reinterpret_cast<C*>(img.data());
  for (int m = 0; m < n; ++m) {
    const long double pi = 3.141592653589793238462643383279502884L;
    const long double th = 2.0L * pi * (long double)m / (long double)n;
    h[m].x = (R)cosl(th);
    h[m].y = (R)(-sinl(th));
  }
  if (img.size() > sizeof(C) * (size_t)n)
    sc::xpair810_twiddles(reinterpret_cast<const float2*>(h), reinterpret_cast<float*>(h + n));
  return img;
}

template <typename R>
int upload_twiddles(sc_plan* p) {
  const std::vector<unsigned char> img = twiddle_image<R>(p->n);
  SC_CU(cudaMemcpy(p->tw, img.data(), img.size(), cudaMemcpyHostToDevice));
  return SC_OK;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// column-sweep geometry of the 3D transforms
// ---------------------------------------------------------------------------
// Between the z and y sweeps a field lives as (kx, ky, z), stored [ky][z][kx]:
// element kx + K1 (z + n ky).  The compact cube is [kz][ky][kx], so every z
// line of it spans all kz planes (one plane = K1 (2k+1) elements, 1.17 MB at
// 810^3 FP32) and touches hundreds of 2 MB pages.  With z innermost in the
// intermediate, each z sweep has one such page-spread side instead of two and
// each y sweep gets one: at 810^3 the four sweeps of one right-hand side take
// about 8.1 ms instead of 9.0 ms with a [z][ky][kx] intermediate.
// `ld` (default K1): row length of the intermediates' x axis.  The product
// pipeline pads it to an even count (272 at 810^3) so that every row of the
// intermediates it feeds to the TMA-fed sweeps starts on a 16-byte boundary.
// Inverse z: compact cube (K1 x K2 x K2) -> intermediate, k = 0 masked.
sc::ColArgs z_inverse_args(int K1, int K2, int n, int kc, int ldo = 0) {
  sc::ColArgs a{};
  const long long lo = ldo > 0 ? ldo : K1;
  a.K1 = K1; a.ncols = K2;
  a.in_cs = K1; a.in_es = (long long)K1 * K2; a.out_cs = lo * n; a.out_es = lo;
  a.kpos = kc + 1; a.kneg = kc; a.zero_origin = 1;
  return a;
}
// Inverse y: intermediate -> physical-(y, z) rows [z][y][kx] (row length K1).
sc::ColArgs y_inverse_args(int K1, int n, int kc, int ldi = 0) {
  sc::ColArgs b{};
  const long long li = ldi > 0 ? ldi : K1;
  b.K1 = K1; b.ncols = n;
  b.in_cs = li; b.in_es = li * n; b.out_cs = (long long)K1 * n; b.out_es = K1;
  b.kpos = kc + 1; b.kneg = kc;
  return b;
}
// Forward y: rows [z][y][kx] (x extent K1) -> intermediate (ky pruned to 2 kout + 1).
sc::ColArgs y_forward_args(int K1, int n, int kout, int ld = 0) {
  sc::ColArgs f{};
  const long long l = ld > 0 ? ld : K1;
  f.K1 = K1; f.ncols = n;
  f.in_cs = l * n; f.in_es = l; f.out_cs = l; f.out_es = l * n;
  f.kpos = kout + 1; f.kneg = kout;
  return f;
}
// Forward z: intermediate -> compact cube of half-width kout (x extent K1 = kout + 1).
sc::ColArgs z_forward_args(int K1, int n, int kout, int ldi = 0) {
  sc::ColArgs g{};
  const int K2 = 2 * kout + 1;
  const long long li = ldi > 0 ? ldi : K1;
  g.K1 = K1; g.ncols = K2;
  g.in_cs = li * n; g.in_es = li; g.out_cs = K1; g.out_es = (long long)K1 * K2;
  g.kpos = kout + 1; g.kneg = kout;
  return g;
}
int even_up(int k) { return k + (k & 1); }

// ---------------------------------------------------------------------------
// the five-sweep product pipeline: compact u -> compact F[u_i u_j]/n^D in p->sig
// ---------------------------------------------------------------------------
// `ev` (optional): events recorded after each launch, ev[0] before the first.
// Output: the product spectra on the compact cube of half-width `kout` <= kc
// (x extent kout+1, y/z extent 2 kout+1) in `sig` (default: the plan's).
template <typename R>
int products(sc_plan* p, void* const* u, cudaStream_t st, cudaEvent_t* ev = nullptr, int kout = -1,
             void* const* sig = nullptr) {
  const int n = p->n, K1 = p->K1, K2 = p->K2, kc = p->kc;
  if (kout < 0) kout = kc;
  if (!sig) sig = p->sig;
  const int K1o = kout + 1;
  int iev = 0;
  auto mark = [&]() { if (ev) cudaEventRecord(ev[iev++], st); };
  mark();
  sc::ColArgs a{};
  if (p->D == 3) {
    // intermediates B = z-inverse output, D = x-sweep output, E = y-forward
    // output have even row lengths (the buffers are allocated for K1 + 1)
    const int ld = even_up(K1), ldo = even_up(K1o);
    auto bounded = [&](sc::ColArgs& c, int v) { c.variant = v; c.wait_limit = p->wait_limit; c.err = p->err; };
    a = z_inverse_args(K1, K2, n, kc, ld);
    for (int c = 0; c < 3; ++c) { a.in[c] = u[c]; a.out[c] = p->be[c]; }
    a.ncomp = 3;
    bounded(a, p->variant[0]);
    if (!sc::launch_col_inv<R>(n, a, p->tw, st)) return fail(SC_ERR_SIZE, "unsupported n=%d", n);
    mark();
    sc::ColArgs b = y_inverse_args(K1, n, kc, ld);
    for (int c = 0; c < 3; ++c) { b.in[c] = p->be[c]; b.out[c] = p->cc[c]; }
    b.ncomp = 3;
    bounded(b, p->variant[1]);
    sc::launch_col_inv<R>(n, b, p->tw, st);
    mark();
    sc::XArgs x{};
    for (int c = 0; c < 3; ++c) x.in[c] = p->cc[c];
    for (int c = 0; c < 6; ++c) x.out[c] = p->dd[c];
    x.D = 3; x.K1in = K1; x.K1out = K1o; x.nrows = (long long)n * n; x.scale = 1.0 / ((double)n * n * n);
    x.ldo = ldo;
    x.variant = p->variant[2];
    sc::launch_xsweep_ns<R>(n, x, p->tw, st);
    mark();
    sc::ColArgs f = y_forward_args(K1o, n, kout, ldo);
    for (int c = 0; c < 6; ++c) { f.in[c] = p->dd[c]; f.out[c] = p->be[c]; }
    f.ncomp = 6;
    bounded(f, p->variant[3]);
    sc::launch_col_fwd<R>(n, f, p->tw, st);
    mark();
    sc::ColArgs g = z_forward_args(K1o, n, kout, ldo);
    for (int c = 0; c < 6; ++c) { g.in[c] = p->be[c]; g.out[c] = sig[c]; }
    g.ncomp = 6;
    bounded(g, p->variant[4]);
    sc::launch_col_fwd<R>(n, g, p->tw, st);
    mark();
  } else {
    for (int c = 0; c < 2; ++c) { a.in[c] = u[c]; a.out[c] = p->cc[c]; }
    a.ncomp = 2; a.K1 = K1; a.ncols = 1;
    a.in_cs = 0; a.in_es = K1; a.out_cs = 0; a.out_es = K1;
    a.kpos = kc + 1; a.kneg = kc; a.zero_origin = 1;
    if (!sc::launch_col_inv<R>(n, a, p->tw, st)) return fail(SC_ERR_SIZE, "unsupported n=%d", n);
    mark();
    sc::XArgs x{};
    for (int c = 0; c < 2; ++c) x.in[c] = p->cc[c];
    for (int c = 0; c < 3; ++c) x.out[c] = p->dd[c];
    x.D = 2; x.K1in = K1; x.K1out = K1o; x.nrows = n; x.scale = 1.0 / ((double)n * n);
    sc::launch_xsweep_ns<R>(n, x, p->tw, st);
    mark();
    sc::ColArgs f{};
    for (int c = 0; c < 3; ++c) { f.in[c] = p->dd[c]; f.out[c] = sig[c]; }
    f.ncomp = 3; f.K1 = K1o; f.ncols = 1;
    f.in_cs = 0; f.in_es = K1o; f.out_cs = 0; f.out_es = K1o;
    f.kpos = kout + 1; f.kneg = kout;
    sc::launch_col_fwd<R>(n, f, p->tw, st);
    mark();
  }
  return check_launch("product pipeline");
}

// ---------------------------------------------------------------------------
// batched transforms between the compact cube and physical space
// (to_phys!(twothirds(.)) and to_spec! of src/solver.jl:210-215, 371-389)
// ---------------------------------------------------------------------------
template <typename R>
int c2p_batch(sc_plan* p, void* const* bb, void* const* cb, void* const* in, void* const* out, int m,
              cudaStream_t st) {
  const int n = p->n, K1 = p->K1, K2 = p->K2, kc = p->kc;
  for (int c0 = 0; c0 < m; c0 += 12) {
    const int mc = m - c0 < 12 ? m - c0 : 12;
    sc::ColArgs a{};
    if (p->D == 3) {
      a = z_inverse_args(K1, K2, n, kc);
      for (int c = 0; c < mc; ++c) { a.in[c] = in[c0 + c]; a.out[c] = bb[c]; }
      a.ncomp = mc;
      sc::launch_col_inv<R>(n, a, p->tw, st);
      sc::ColArgs b = y_inverse_args(K1, n, kc);
      for (int c = 0; c < mc; ++c) { b.in[c] = bb[c]; b.out[c] = cb[c]; }
      b.ncomp = mc;
      sc::launch_col_inv<R>(n, b, p->tw, st);
    } else {
      for (int c = 0; c < mc; ++c) { a.in[c] = in[c0 + c]; a.out[c] = cb[c]; }
      a.ncomp = mc; a.K1 = K1; a.ncols = 1;
      a.in_cs = 0; a.in_es = K1; a.out_cs = 0; a.out_es = K1;
      a.kpos = kc + 1; a.kneg = kc; a.zero_origin = 1;
      sc::launch_col_inv<R>(n, a, p->tw, st);
    }
    sc::XPlainArgs x{};
    for (int c = 0; c < mc; ++c) { x.in[c] = cb[c]; x.out[c] = out[c0 + c]; }
    x.ncomp = mc; x.K1 = K1; x.nrows = p->D == 3 ? (long long)n * n : n; x.scale = 1.0;
    sc::launch_x_c2r<R>(n, x, p->tw, st);
  }
  return check_launch("compact to physical");
}

template <typename R>
int p2c_batch(sc_plan* p, void* const* bb, void* const* cb, void* const* in, void* const* out, int m,
              cudaStream_t st) {
  const int n = p->n, K1 = p->K1, K2 = p->K2, kc = p->kc;
  for (int c0 = 0; c0 < m; c0 += 12) {
    const int mc = m - c0 < 12 ? m - c0 : 12;
    sc::XPlainArgs x{};
    for (int c = 0; c < mc; ++c) { x.in[c] = in[c0 + c]; x.out[c] = cb[c]; }
    x.ncomp = mc; x.K1 = K1; x.nrows = p->D == 3 ? (long long)n * n : n;
    x.scale = 1.0 / std::pow((double)n, p->D);
    sc::launch_x_r2c<R>(n, x, p->tw, st);
    sc::ColArgs f{};
    if (p->D == 3) {
      f = y_forward_args(K1, n, kc);
      for (int c = 0; c < mc; ++c) { f.in[c] = cb[c]; f.out[c] = bb[c]; }
      f.ncomp = mc;
      sc::launch_col_fwd<R>(n, f, p->tw, st);
      sc::ColArgs g = z_forward_args(K1, n, kc);
      for (int c = 0; c < mc; ++c) { g.in[c] = bb[c]; g.out[c] = out[c0 + c]; }
      g.ncomp = mc;
      sc::launch_col_fwd<R>(n, g, p->tw, st);
    } else {
      for (int c = 0; c < mc; ++c) { f.in[c] = cb[c]; f.out[c] = out[c0 + c]; }
      f.ncomp = mc; f.K1 = K1; f.ncols = 1;
      f.in_cs = 0; f.in_es = K1; f.out_cs = 0; f.out_es = K1;
      f.kpos = kc + 1; f.kneg = kc;
      sc::launch_col_fwd<R>(n, f, p->tw, st);
    }
  }
  return check_launch("physical to compact");
}

sc::LesSpecArgs spec_args(sc_plan* p) {
  sc::LesSpecArgs a{};
  a.kc = p->kc;
  a.nmodes = (long long)p->csz;
  a.kfac = 2.0 * M_PI / p->l;
  a.scale = 1.0;
  return a;
}

sc::LesPhysArgs phys_args(sc_plan* p) {
  sc::LesPhysArgs a{};
  a.npts = (long long)std::pow((double)p->n, p->D);
  return a;
}

// ---------------------------------------------------------------------------
// CUDA-core CNN closure (FP32/FP64): forward with stored activations, backward
// ---------------------------------------------------------------------------
static const int kCcCin[4] = {4, 32, 32, 32}, kCcCout[4] = {32, 32, 32, 6};

int num_sms_api() {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm > 0 ? nsm : 148;
}

long long cc_layer_offset(int l) {  // offset of layer l in the flat parameter vector [w, b]
  long long o = 0;
  for (int i = 0; i < l; ++i) o += (long long)kCcCout[i] * kCcCin[i] * 27 + kCcCout[i];
  return o;
}

template <typename R>
int cc_forward(sc_closure* cl, void* const* u, cudaStream_t st) {
  sc_plan* p = cl->p;
  const long long np = phys_args(p).npts;
  int rc = c2p_batch<R>(p, cl->bb, cl->cb, u, cl->gp, 3, st);  // v = T(u)
  if (rc) return rc;
  SC_CU(cudaMemsetAsync(cl->dsum, 0, sizeof(double), st));
  sc::launch_spectral_energy<R>(u, 3, 3, p->n, p->K1, p->K2, 1, p->kc, 2.0 * M_PI / p->l, 1, cl->dsum, st);
  sc::launch_redelta(cl->dsum, cl->dsum + 3, cl->delta, cl->nu, cl->mu, cl->sigma, st);
  R* const* A = reinterpret_cast<R* const*>(cl->cca);
  sc::launch_cc_input<R>(static_cast<const R*>(cl->gp[0]), static_cast<const R*>(cl->gp[1]),
                         static_cast<const R*>(cl->gp[2]), cl->dsum + 3, A[0], np, st);
  const R* inp = A[0];
  for (int l = 0; l < 4; ++l) {
    sc::ConvArgs c{};
    c.in = inp; c.w = cl->ccw[l]; c.b = cl->ccb[l];
    c.out = l < 3 ? (void*)A[1 + 2 * l] : cl->cctau;
    c.n = p->n; c.cin = kCcCin[l]; c.cout = kCcCout[l];
    sc::launch_conv_fwd<R>(c, st);
    if (l < 3) {
      sc::launch_gelu<R>(A[1 + 2 * l], A[2 + 2 * l], (long long)kCcCout[l] * np, st);
      inp = A[2 + 2 * l];
    }
  }
  return check_launch("cnn forward (CUDA cores)");
}

// Given g_tau (dL/dtau, planar [6][npts]) after cc_forward at the same u:
// parameter gradients accumulate into cl->gw; dL/dv (3 planar) is left in
// ccg0[0..2], dL/dz in cl->dsum[1].
template <typename R>
int cc_backward(sc_closure* cl, const R* gtau, cudaStream_t st) {
  sc_plan* p = cl->p;
  const long long np = phys_args(p).npts;
  R* const* A = reinterpret_cast<R* const*>(cl->cca);
  R* g0 = static_cast<R*>(cl->ccg[0]);
  R* g1 = static_cast<R*>(cl->ccg[1]);
  const R* gout = gtau;
  R* gin = g0;
  for (int l = 3; l >= 0; --l) {
    sc::ConvArgs c{};
    c.in = l > 0 ? (const void*)A[2 * l] : (const void*)A[0];
    c.w = cl->ccw[l];
    c.out = const_cast<R*>(gout);
    c.in_grad = l > 0 ? (void*)gin : cl->ccg0;
    c.n = p->n; c.cin = kCcCin[l]; c.cout = kCcCout[l];
    const long long off = cc_layer_offset(l);
    sc::launch_conv_bwd<R>(c, cl->gw + off, cl->gw + off + (long long)kCcCout[l] * kCcCin[l] * 27, st);
    if (l > 0) {
      sc::launch_gelu_bwd<R>(A[2 * l - 1], gin, (long long)kCcCin[l] * np, st);  // pre-activation h_l
      gout = gin;
      gin = (gin == g0) ? g1 : g0;
    }
  }
  SC_CU(cudaMemsetAsync(cl->dsum + 1, 0, sizeof(double), st));
  sc::launch_sum<R>(static_cast<const R*>(cl->ccg0) + 3 * np, np, cl->dsum + 1, st);
  return check_launch("cnn backward (CUDA cores)");
}

sc::MlpArgs mlp_args(sc_closure* cl, const void* const* G, void* const* tau) {
  sc_plan* p = cl->p;
  sc::MlpArgs a{};
  const int D = p->D;
  for (int c = 0; c < D * D; ++c) a.G[c] = G[c];
  for (int c = 0; c < (D == 3 ? 6 : 3); ++c) a.tau[c] = tau[c];
  a.npts = phys_args(p).npts;
  a.D = D; a.nl = cl->mlp_nl;
  for (int l = 0; l <= cl->mlp_nl; ++l) a.w[l] = cl->mlp_w[l];
  a.theta = cl->mlp_theta;
  a.delta = cl->delta;
  a.mode = cl->kind == sc::kTbnn ? 1 : 0;
  return a;
}

// The split-precision fields of a forward pass (pre[] as the caller set it).
void tc_split_args(const sc_closure* cl, sc::CnnArgs& a) {
  if (!cl->cnn_split) return;
  a.split = true;
  for (int l = 0; l < 4; ++l) {
    a.wh[l] = static_cast<const __half*>(cl->cwh[l]);
    a.wl[l] = static_cast<const __half*>(cl->cwl[l]);
    a.acth[l] = static_cast<__half*>(cl->sacth[l]);
    a.actl[l] = static_cast<__half*>(cl->sactl[l]);
  }
  a.acc = static_cast<float*>(cl->sacc);
}

// Tensor-core CNN for the adjoint: forward at u keeping every layer input and
// the pre-activations (v in gp[0..2], tau in tp), and backward from dL/dtau
// (planar FP32 in cctau) to dL/dv (ccg0[0..2]), dL/dz (dsum[1]) and the
// parameter gradient (cl->gw).  The backward differentiates the network with
// the BF16 roundings of weights and activations taken as identities.
int tc_forward(sc_closure* cl, void* const* u, cudaStream_t st) {
  sc_plan* p = cl->p;
  int rc = c2p_batch<float>(p, cl->bb, cl->cb, u, cl->gp, 3, st);
  if (rc) return rc;
  SC_CU(cudaMemsetAsync(cl->dsum, 0, sizeof(double), st));
  sc::launch_spectral_energy<float>(u, 3, 3, p->n, p->K1, p->K2, 1, p->kc, 2.0 * M_PI / p->l, 1, cl->dsum, st);
  sc::CnnArgs a{};
  a.n = p->n;
  for (int c = 0; c < 3; ++c) a.u[c] = cl->gp[c];
  for (int l = 0; l < 4; ++l) {
    a.w[l] = static_cast<const __nv_bfloat16*>(cl->cw[l]);
    a.b[l] = static_cast<const float*>(cl->cbias[l]);
  }
  a.act0 = static_cast<__nv_bfloat16*>(cl->act[0]);
  a.act1 = static_cast<__nv_bfloat16*>(cl->act[1]);
  a.act2 = static_cast<__nv_bfloat16*>(cl->act[2]);
  a.act3 = static_cast<__nv_bfloat16*>(cl->tact3);
  for (int l = 0; l < 3; ++l) a.pre[l] = static_cast<float*>(cl->tpre[l]);
  for (int c = 0; c < 6; ++c) a.tau.p[c] = static_cast<float*>(cl->tp[c]);
  a.a2 = cl->dsum; a.z = cl->dsum + 3;
  a.delta = cl->delta; a.nu = cl->nu; a.mu = cl->mu; a.sigma = cl->sigma;
  a.err = cl->err;
  a.nsm = num_sms_api();
  a.wait_limit = p->wait_limit;
  tc_split_args(cl, a);
  sc::launch_cnn_forward(a, st);
  return check_launch("cnn forward (tensor cores, adjoint)");
}

int tc_backward(sc_closure* cl, cudaStream_t st) {
  sc_plan* p = cl->p;
  const long long np = phys_args(p).npts;
  sc::CnnBwdArgs b{};
  b.n = p->n;
  for (int c = 0; c < 6; ++c) b.gtau.p[c] = static_cast<float*>(cl->cctau) + (size_t)c * np;
  for (int l = 0; l < 4; ++l) b.wt[l] = static_cast<const __nv_bfloat16*>(cl->cwt[l]);
  b.act[0] = static_cast<const __nv_bfloat16*>(cl->act[0]);
  b.act[1] = static_cast<const __nv_bfloat16*>(cl->act[1]);
  b.act[2] = static_cast<const __nv_bfloat16*>(cl->act[2]);
  b.act[3] = static_cast<const __nv_bfloat16*>(cl->tact3);
  for (int l = 0; l < 3; ++l) b.pre[l] = static_cast<const float*>(cl->tpre[l]);
  b.gbf = static_cast<__nv_bfloat16*>(cl->tgbf);
  b.gf = static_cast<float*>(cl->tgf);
  for (int c = 0; c < 4; ++c) b.gin_planar.p[c] = static_cast<float*>(cl->ccg0) + (size_t)c * np;
  b.gw = cl->gw;
  for (int l = 0; l < 4; ++l) b.woff[l] = cc_layer_offset(l);
  b.err = cl->err;
  b.nsm = num_sms_api();
  b.wait_limit = p->wait_limit;
  if (cl->cnn_split) {
    b.split = true;
    for (int l = 0; l < 4; ++l) {
      b.wtl[l] = static_cast<const __nv_bfloat16*>(cl->cwtl[l]);
      b.acth[l] = static_cast<const __half*>(cl->sacth[l]);
      b.actl[l] = static_cast<const __half*>(cl->sactl[l]);
    }
    b.gbf_lo = static_cast<__nv_bfloat16*>(cl->tgbfl);
  }
  sc::launch_cnn_backward(b, st);
  SC_CU(cudaMemsetAsync(cl->dsum + 1, 0, sizeof(double), st));
  sc::launch_sum<float>(static_cast<const float*>(cl->ccg0) + 3 * np, np, cl->dsum + 1, st);
  return check_launch("cnn backward (tensor cores)");
}

// Closure stress of the compact state u into cl->th (compact), i.e. the
// spectrum to_spec!(model(u, G)) that les! adds to sigma (src/les.jl:19-27).
// Bardina and dynamic Smagorinsky read the product spectra F[u_i u_j]/n^D from
// p->sig, which the caller has just computed for the same u.
template <typename R>
int closure_tauhat(sc_closure* cl, void* const* u, cudaStream_t st, void* const* tau_phys_out = nullptr) {
  sc_plan* p = cl->p;
  const int D = p->D, NP = D == 3 ? 6 : 3;
  int rc = SC_OK;
  if (cl->kind == sc::kMlp || cl->kind == sc::kTbnn) {
    sc::LesSpecArgs g = spec_args(p);
    for (int c = 0; c < D; ++c) g.in[c] = u[c];
    for (int c = 0; c < D * D; ++c) g.out[c] = cl->gc[c];
    sc::launch_grad<R>(g, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->gc, cl->gp, D * D, st))) return rc;
    sc::launch_mlp<R>(mlp_args(cl, (const void* const*)cl->gp, cl->tp), cl->mlp_z, cl->nu, cl->mu, cl->sigma, st);
    if ((rc = check_launch("mlp closure"))) return rc;
  } else if (cl->kind == sc::kClark || cl->kind == sc::kSmagorinsky || cl->kind == sc::kVerstappen) {
    sc::LesSpecArgs g = spec_args(p);
    for (int c = 0; c < D; ++c) g.in[c] = u[c];
    for (int c = 0; c < D * D; ++c) g.out[c] = cl->gc[c];
    sc::launch_grad<R>(g, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->gc, cl->gp, D * D, st))) return rc;
    sc::LesPhysArgs a = phys_args(p);
    for (int c = 0; c < D * D; ++c) a.in[c] = cl->gp[c];
    for (int c = 0; c < NP; ++c) a.out[c] = cl->tp[c];
    a.kind = cl->kind; a.delta = cl->delta; a.p0 = cl->prm[0];
    sc::launch_closure_pt<R>(a, D, st);
  } else if (cl->kind == sc::kBardina) {
    const double dt_ = cl->prm[0] * cl->delta;
    sc::LesSpecArgs f = spec_args(p);
    for (int c = 0; c < D; ++c) { f.in[c] = u[c]; f.out[c] = cl->ut[c]; }
    f.ncomp = D; f.delta = dt_;
    sc::launch_spec_filter<R>(f, D, st);
    sc::LesSpecArgs h = spec_args(p);
    for (int c = 0; c < NP; ++c) { h.in[c] = p->sig[c]; h.out[c] = cl->gc[c]; }
    h.ncomp = NP; h.delta = dt_;
    sc::launch_spec_filter<R>(h, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->gc, cl->gp, NP, st))) return rc;
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->ut, cl->ph4, D, st))) return rc;
    sc::LesPhysArgs a = phys_args(p);
    for (int c = 0; c < NP; ++c) { a.in[c] = cl->gp[c]; a.out[c] = cl->tp[c]; }
    for (int c = 0; c < D; ++c) a.in2[c] = cl->ph4[c];
    a.kind = 1;  // trace-free
    sc::launch_sub_products<R>(a, D, st);
  } else if (cl->kind == sc::kDynSmagorinsky) {
    const double dtl = 2.0 * cl->delta, ddb = std::sqrt(dtl * dtl + cl->delta * cl->delta);
    sc::LesSpecArgs f = spec_args(p);  // u~ = P G~ u
    for (int c = 0; c < D; ++c) { f.in[c] = u[c]; f.out[c] = cl->ut[c]; }
    f.ncomp = D; f.delta = dtl;
    sc::launch_spec_filter<R>(f, D, st);
    sc::LesSpecArgs h = spec_args(p);  // P G~ sigma
    for (int c = 0; c < NP; ++c) { h.in[c] = p->sig[c]; h.out[c] = cl->gc[c]; }
    h.ncomp = NP; h.delta = dtl;
    sc::launch_spec_filter<R>(h, D, st);
    sc::LesSpecArgs sr = spec_args(p);  // S-hat
    for (int c = 0; c < D; ++c) sr.in[c] = u[c];
    for (int c = 0; c < NP; ++c) sr.out[c] = cl->s2[c];
    sc::launch_strain<R>(sr, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->gc, cl->gp, NP, st))) return rc;   // L1
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->ut, cl->ph4, D, st))) return rc;   // u~
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->s2, cl->tp, NP, st))) return rc;   // S
    sc::LesSpecArgs h2 = spec_args(p);  // P G~ P S-hat, in place
    for (int c = 0; c < NP; ++c) { h2.in[c] = cl->s2[c]; h2.out[c] = cl->s2[c]; }
    h2.ncomp = NP; h2.delta = dtl;
    sc::launch_spec_filter<R>(h2, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->s2, cl->ph3, NP, st))) return rc;  // S~
    sc::LesPhysArgs m1 = phys_args(p);  // m1 = smag(S, Delta), in place
    for (int c = 0; c < NP; ++c) { m1.in[c] = cl->tp[c]; m1.out[c] = cl->tp[c]; }
    m1.delta = cl->delta;
    sc::launch_smag_tensor<R>(m1, D, st);
    sc::LesPhysArgs m2 = phys_args(p);  // m2 = smag(S~, sqrt(5) Delta), in place
    for (int c = 0; c < NP; ++c) { m2.in[c] = cl->ph3[c]; m2.out[c] = cl->ph3[c]; }
    m2.delta = ddb;
    sc::launch_smag_tensor<R>(m2, D, st);
    if ((rc = p2c_batch<R>(p, cl->bb, cl->cb, cl->tp, cl->th, NP, st))) return rc;   // F[m1]
    sc::LesSpecArgs h3 = spec_args(p);  // P G~ F[m1]
    for (int c = 0; c < NP; ++c) { h3.in[c] = cl->th[c]; h3.out[c] = cl->s2[c]; }
    h3.ncomp = NP; h3.delta = dtl;
    sc::launch_spec_filter<R>(h3, D, st);
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, cl->s2, cl->ph2, NP, st))) return rc;  // M1
    SC_CU(cudaMemsetAsync(cl->dsum, 0, 3 * sizeof(double), st));
    sc::LesPhysArgs ml = phys_args(p);
    for (int c = 0; c < NP; ++c) { ml.in[c] = cl->gp[c]; ml.in3[c] = cl->ph2[c]; ml.in4[c] = cl->ph3[c]; }
    for (int c = 0; c < D; ++c) ml.in2[c] = cl->ph4[c];
    sc::launch_dynsmag_mlmm<R>(ml, D, cl->dsum, st);
    sc::LesSpecArgs sc_ = spec_args(p);  // tau-hat = c P F[m1]
    for (int c = 0; c < NP; ++c) { sc_.in[c] = cl->th[c]; sc_.out[c] = cl->th[c]; }
    sc_.ncomp = NP; sc_.delta = 0; sc_.dscale = cl->dsum + 2;
    sc::launch_spec_filter<R>(sc_, D, st);
    if (tau_phys_out) return c2p_batch<R>(p, cl->bb, cl->cb, cl->th, tau_phys_out, NP, st);
    return check_launch("dynamic Smagorinsky");
  } else if (cl->kind == sc::kCnn) {
    if ((rc = c2p_batch<R>(p, cl->bb, cl->cb, u, cl->gp, D, st))) return rc;  // u (physical)
    SC_CU(cudaMemsetAsync(cl->dsum, 0, sizeof(double), st));
    sc::launch_spectral_energy<R>(u, D, D, p->n, p->K1, p->K2, 1, p->kc, 2.0 * M_PI / p->l, 1, cl->dsum, st);
    sc::CnnArgs a{};
    a.n = p->n;
    for (int c = 0; c < 3; ++c) a.u[c] = cl->gp[c];
    for (int l = 0; l < 4; ++l) {
      a.w[l] = static_cast<const __nv_bfloat16*>(cl->cw[l]);
      a.b[l] = static_cast<const float*>(cl->cbias[l]);
    }
    a.act0 = static_cast<__nv_bfloat16*>(cl->act[0]);
    a.act1 = static_cast<__nv_bfloat16*>(cl->act[1]);
    a.act2 = static_cast<__nv_bfloat16*>(cl->act[2]);
    for (int c = 0; c < 6; ++c) a.tau.p[c] = static_cast<float*>(cl->tp[c]);
    a.a2 = cl->dsum; a.z = cl->dsum + 3;
    a.delta = cl->delta; a.nu = cl->nu; a.mu = cl->mu; a.sigma = cl->sigma;
    a.err = cl->err;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    a.nsm = nsm;
    a.wait_limit = p->wait_limit;
    tc_split_args(cl, a);
    sc::launch_cnn_forward(a, st);
    if ((rc = check_launch("cnn closure"))) return rc;
  } else if (cl->kind == sc::kCnnFp) {
    if ((rc = cc_forward<R>(cl, u, st))) return rc;
    void* tslice[6];
    for (int c = 0; c < 6; ++c) tslice[c] = static_cast<R*>(cl->cctau) + (size_t)c * phys_args(p).npts;
    if (tau_phys_out) {
      for (int c = 0; c < 6; ++c)
        SC_CU(cudaMemcpyAsync(tau_phys_out[c], tslice[c], (size_t)phys_args(p).npts * sizeof(R),
                              cudaMemcpyDeviceToDevice, st));
      return check_launch("closure");
    }
    return p2c_batch<R>(p, cl->bb, cl->cb, tslice, cl->th, NP, st);
  } else {
    return fail(SC_ERR_UNSUPPORTED, "closure kind %d has no evaluation in this build", cl->kind);
  }
  // tp holds the physical stress
  if (tau_phys_out) {
    for (int c = 0; c < NP; ++c)
      SC_CU(cudaMemcpyAsync(tau_phys_out[c], cl->tp[c], (size_t)phys_args(p).npts * sizeof(R),
                            cudaMemcpyDeviceToDevice, st));
    return check_launch("closure");
  }
  return p2c_batch<R>(p, cl->bb, cl->cb, cl->tp, cl->th, NP, st);
}

template <typename R>
sc::EpiArgs epi_base(sc_plan* p, void* const* us, double visc) {
  sc::EpiArgs e{};
  for (int c = 0; c < 6; ++c) e.sig[c] = p->sig[c];
  for (int c = 0; c < p->D; ++c) e.us[c] = us[c];
  e.D = p->D; e.K1 = p->K1; e.K2 = p->K2; e.kc = p->kc;
  e.kfac = 2.0 * M_PI / p->l;
  e.visc = visc;
  return e;
}

template <typename R>
void add_closure_stress(sc::EpiArgs& e, sc_closure* cl, int D) {
  if (!cl || cl->kind == sc::kNoClosure) return;
  for (int c = 0; c < (D == 3 ? 6 : 3); ++c) e.sig2[c] = cl->th[c];
  e.has_sig2 = 1;
}

template <typename R>
int stage_rhs(sc_plan* p, sc_closure* cl, void* const* us, cudaStream_t st) {
  int rc = products<R>(p, us, st);
  if (rc) return rc;
  if (cl && cl->kind != sc::kNoClosure) return closure_tauhat<R>(cl, us, st);
  return SC_OK;
}

template <typename R>
int rk4_step(sc_plan* p, double dt, double visc, const sc_forcing* frc, cudaStream_t st, sc_closure* cl = nullptr) {
  const bool forced = frc != nullptr && frc->enabled;
  for (int s = 0; s < 4; ++s) {
    void* const* us = s == 0 ? p->U : p->S;
    if (forced) sc::launch_band_forcing<R>(us, p->D, p->K1, p->K2, p->kc, frc->eps, p->dscal, st);
    int rc = stage_rhs<R>(p, cl, us, st);
    if (rc) return rc;
    sc::EpiArgs e = epi_base<R>(p, us, visc);
    add_closure_stress<R>(e, cl, p->D);
    e.proj_k = 1;
    e.forcing = forced ? p->dscal : nullptr;
    static const double wa[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
    static const double cbv[3] = {0.5, 0.5, 1.0};
    // The accumulator ACC = U + dt sum_j wa[j] k_j is first written at stage 1,
    // from the stage input S = U + cbv[0] dt k1 that stage reads anyway:
    // ACC = U + (wa[0] / cbv[0]) (S - U) + wa[1] dt k2.  Stage 0 writes only S.
    for (int c = 0; c < p->D; ++c) {
      e.base_a[c] = s <= 1 ? nullptr : p->ACC[c];
      e.out_a[c] = s == 0 ? nullptr : (s == 3 ? p->U[c] : p->ACC[c]);
      if (s < 3) { e.base_b[c] = p->U[c]; e.out_b[c] = p->S[c]; }
    }
    e.mix_a = s == 1;
    e.mix = wa[0] / cbv[0];
    e.ca = wa[s] * dt;
    e.has_b = s < 3;
    e.cb = s < 3 ? cbv[s] * dt : 0.0;
    sc::launch_epilogue<R>(e, st);
  }
  return check_launch("rk4 step");
}

template <typename R>
int wray3_step(sc_plan* p, double dt, double visc, cudaStream_t st, sc_closure* cl = nullptr) {
  static const double a[3] = {8.0 / 15, 5.0 / 12, 3.0 / 4};
  static const double b[2] = {1.0 / 4, 0.0};
  for (int s = 0; s < 3; ++s) {
    int rc = stage_rhs<R>(p, cl, p->U, st);
    if (rc) return rc;
    sc::EpiArgs e = epi_base<R>(p, p->U, visc);
    add_closure_stress<R>(e, cl, p->D);
    e.proj_a = 1;
    for (int c = 0; c < p->D; ++c) {
      e.base_a[c] = s == 0 ? p->U[c] : p->S[c];
      e.out_a[c] = p->U[c];
      e.base_b[c] = s == 0 ? p->U[c] : p->S[c];
      e.out_b[c] = p->S[c];
    }
    e.ca = a[s] * dt;
    e.has_b = (s < 2 && (s == 0 || b[s] != 0.0)) ? 1 : 0;
    e.cb = s < 2 ? b[s] * dt : 0.0;
    sc::launch_epilogue<R>(e, st);
  }
  return check_launch("wray3 step");
}

template <typename R>
int pack_state(sc_plan* p, const void* const* u, void* const* dst, cudaStream_t st) {
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) { a.src[c] = u[c]; a.dst[c] = dst[c]; }
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  sc::launch_pack<R>(a, st);
  return check_launch("pack");
}

template <typename R>
int unpack_state(sc_plan* p, void* const* src, void* const* u, cudaStream_t st) {
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) { a.src[c] = src[c]; a.dst[c] = u[c]; }
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  sc::launch_unpack<R>(a, st);
  return check_launch("unpack");
}

int check_ptrs(const void* const* u, int k) {
  if (!u) return fail(SC_ERR_INVALID, "null field array");
  for (int c = 0; c < k; ++c)
    if (!u[c]) return fail(SC_ERR_INVALID, "null component pointer %d", c);
  return SC_OK;
}

int ensure_device(sc_plan* p) {
  int cur = -1;
  SC_CU(cudaGetDevice(&cur));
  if (cur != p->dev) SC_CU(cudaSetDevice(p->dev));
  return SC_OK;
}

template <typename R>
int run_rk4_graph(sc_plan* p, double dt, double visc, int nsteps, const sc_forcing* frc, cudaStream_t st,
                  sc_closure* cl = nullptr) {
  double key[5] = {dt, visc, (frc && frc->enabled) ? 1.0 : 0.0, (frc && frc->enabled) ? frc->eps : 0.0, 0.0};
  std::memcpy(&key[4], &cl, sizeof(cl));
  if (!p->g_rk4 || std::memcmp(key, p->k_rk4, sizeof(key)) != 0) {
    if (p->g_rk4) { cudaGraphExecDestroy(p->g_rk4); p->g_rk4 = nullptr; }
    cudaGraph_t g;
    SC_CU(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    int rc = rk4_step<R>(p, dt, visc, frc, p->cap, cl);
    cudaError_t e = cudaStreamEndCapture(p->cap, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(SC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&p->g_rk4, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { p->g_rk4 = nullptr; return fail(SC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    std::memcpy(p->k_rk4, key, sizeof(key));
  }
  for (int i = 0; i < nsteps; ++i) SC_CU(cudaGraphLaunch(p->g_rk4, st));
  return SC_OK;
}

template <typename R>
int run_rk4(sc_plan* p, double dt, double visc, int nsteps, const sc_forcing* frc, cudaStream_t st,
            sc_closure* cl = nullptr) {
  if (p->use_graph) return run_rk4_graph<R>(p, dt, visc, nsteps, frc, st, cl);
  for (int i = 0; i < nsteps; ++i) {
    int rc = rk4_step<R>(p, dt, visc, frc, st, cl);
    if (rc) return rc;
  }
  return SC_OK;
}

template <typename R>
int run_wray_graph(sc_plan* p, double dt, double visc, cudaStream_t st, sc_closure* cl = nullptr) {
  double key[3] = {dt, visc, 0.0};
  std::memcpy(&key[2], &cl, sizeof(cl));
  if (!p->g_wray || std::memcmp(key, p->k_wray, sizeof(key)) != 0) {
    if (p->g_wray) { cudaGraphExecDestroy(p->g_wray); p->g_wray = nullptr; }
    cudaGraph_t g;
    SC_CU(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    int rc = wray3_step<R>(p, dt, visc, p->cap, cl);
    cudaError_t e = cudaStreamEndCapture(p->cap, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(SC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&p->g_wray, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { p->g_wray = nullptr; return fail(SC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    std::memcpy(p->k_wray, key, sizeof(key));
  }
  SC_CU(cudaGraphLaunch(p->g_wray, st));
  return SC_OK;
}

template <typename R>
int ensure_full_scratch(sc_plan* p) {
  if (p->fa) return SC_OK;
  const size_t bytes = p->fsz * p->esz;
  int rc = plan_alloc(p, &p->fa, bytes);
  if (rc) return rc;
  return plan_alloc(p, &p->fb, bytes);
}

template <typename R>
int to_phys_impl(sc_plan* p, const void* spec, void* phys, cudaStream_t st) {
  int rc = ensure_full_scratch<R>(p);
  if (rc) return rc;
  const int n = p->n, Kf = n / 2 + 1;
  const void* cur = spec;
  if (p->D == 3) {
    sc::ColArgs a{};
    a.in[0] = spec; a.out[0] = p->fa; a.ncomp = 1; a.K1 = Kf; a.ncols = n;
    a.in_cs = Kf; a.in_es = (long long)Kf * n; a.out_cs = Kf; a.out_es = (long long)Kf * n;
    a.kpos = n / 2; a.kneg = n / 2;
    sc::launch_col_inv<R>(n, a, p->tw, st);
    sc::ColArgs b{};
    b.in[0] = p->fa; b.out[0] = p->fb; b.ncomp = 1; b.K1 = Kf; b.ncols = n;
    b.in_cs = (long long)Kf * n; b.in_es = Kf; b.out_cs = (long long)Kf * n; b.out_es = Kf;
    b.kpos = n / 2; b.kneg = n / 2;
    sc::launch_col_inv<R>(n, b, p->tw, st);
    cur = p->fb;
  } else {
    sc::ColArgs b{};
    b.in[0] = spec; b.out[0] = p->fb; b.ncomp = 1; b.K1 = Kf; b.ncols = 1;
    b.in_cs = 0; b.in_es = Kf; b.out_cs = 0; b.out_es = Kf;
    b.kpos = n / 2; b.kneg = n / 2;
    sc::launch_col_inv<R>(n, b, p->tw, st);
    cur = p->fb;
  }
  sc::XPlainArgs x{};
  x.in[0] = cur; x.out[0] = phys; x.ncomp = 1; x.K1 = Kf;
  x.nrows = p->D == 3 ? (long long)n * n : n;
  x.scale = 1.0;
  sc::launch_x_c2r<R>(n, x, p->tw, st);
  return check_launch("to_phys");
}

template <typename R>
int to_spec_impl(sc_plan* p, const void* phys, void* spec, cudaStream_t st) {
  int rc = ensure_full_scratch<R>(p);
  if (rc) return rc;
  const int n = p->n, Kf = n / 2 + 1;
  sc::XPlainArgs x{};
  x.in[0] = phys; x.out[0] = p->D == 3 ? p->fa : p->fb; x.ncomp = 1; x.K1 = Kf;
  x.nrows = p->D == 3 ? (long long)n * n : n;
  x.scale = 1.0 / std::pow((double)n, p->D);
  sc::launch_x_r2c<R>(n, x, p->tw, st);
  if (p->D == 3) {
    sc::ColArgs a{};
    a.in[0] = p->fa; a.out[0] = p->fb; a.ncomp = 1; a.K1 = Kf; a.ncols = n;
    a.in_cs = (long long)Kf * n; a.in_es = Kf; a.out_cs = (long long)Kf * n; a.out_es = Kf;
    a.kpos = n / 2; a.kneg = n / 2;
    sc::launch_col_fwd<R>(n, a, p->tw, st);
    sc::ColArgs b{};
    b.in[0] = p->fb; b.out[0] = spec; b.ncomp = 1; b.K1 = Kf; b.ncols = n;
    b.in_cs = Kf; b.in_es = (long long)Kf * n; b.out_cs = Kf; b.out_es = (long long)Kf * n;
    b.kpos = n / 2; b.kneg = n / 2;
    sc::launch_col_fwd<R>(n, b, p->tw, st);
  } else {
    sc::ColArgs b{};
    b.in[0] = p->fb; b.out[0] = spec; b.ncomp = 1; b.K1 = Kf; b.ncols = 1;
    b.in_cs = 0; b.in_es = Kf; b.out_cs = 0; b.out_es = Kf;
    b.kpos = n / 2; b.kneg = n / 2;
    sc::launch_col_fwd<R>(n, b, p->tw, st);
  }
  return check_launch("to_spec");
}

template <typename R>
int energy_impl(sc_plan* p, const void* const* u, int compact, int weight_k2, double* out, cudaStream_t st,
                int mask23 = 0) {
  SC_CU(cudaMemsetAsync(p->dscal + 1, 0, sizeof(double), st));
  const int K1 = compact ? p->K1 : p->n / 2 + 1;
  const int K2 = compact ? p->K2 : p->n;
  sc::launch_spectral_energy<R>(u, p->D, p->D, p->n, K1, K2, compact, p->kc, 2.0 * M_PI / p->l, weight_k2,
                                p->dscal + 1, st, mask23);
  int rc = check_launch("energy");
  if (rc) return rc;
  double h = 0;
  SC_CU(cudaMemcpyAsync(&h, p->dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  SC_CU(cudaStreamSynchronize(st));
  *out = h;
  return SC_OK;
}

template <typename R>
int filter_impl(sc_plan* dns, sc_plan* les, const void* const* u, const double* deltas, int nd,
                void* const* ubar, void* const* tau, cudaStream_t st) {
  const int D = dns->D;
  int rc = pack_state<R>(dns, u, dns->S, st);
  if (rc) return rc;
  rc = products<R>(dns, dns->S, st, nullptr, les->kc, dns->sig);
  if (rc) return rc;
  for (int d = 0; d < nd; ++d) {
    sc::FilterArgs f{};
    for (int c = 0; c < D; ++c) { f.udns[c] = dns->S[c]; f.ubar[c] = les->S[c]; }
    for (int c = 0; c < (D == 3 ? 6 : 3); ++c) { f.sig1[c] = dns->sig[c]; f.tau[c] = les->sig[c]; }
    f.D = D; f.kcd = dns->kc; f.kcl = les->kc; f.kfac = 2.0 * M_PI / les->l;
    f.delta = (deltas[d] > 0) ? deltas[d] : 0.0;
    f.pass = 0;
    sc::launch_filter<R>(f, st);
    rc = products<R>(les, les->S, st);
    if (rc) return rc;
    f.pass = 1;
    sc::launch_filter<R>(f, st);
    rc = unpack_state<R>(les, les->S, ubar + (size_t)D * d, st);
    if (rc) return rc;
    sc::PackArgs pa{};
    const int nt = D == 3 ? 6 : 3;
    for (int c = 0; c < nt; ++c) { pa.src[c] = les->sig[c]; pa.dst[c] = tau[(size_t)nt * d + c]; }
    pa.ncomp = nt; pa.D = D; pa.n = les->n; pa.kc = les->kc;
    sc::launch_unpack<R>(pa, st);
    rc = check_launch("filter");
    if (rc) return rc;
  }
  return SC_OK;
}

#define SC_DTYPE_DISPATCH(p, FN, ...) \
  ((p)->dtype == SC_FLOAT64 ? FN<double>(__VA_ARGS__) : FN<float>(__VA_ARGS__))

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

int sc_abi_version(void) { return SC_ABI_VERSION; }
const char* sc_last_error_string(void) { return g_err.c_str(); }
int sc_fft_size_supported(int n) { return sc::fft_size_supported(n) ? 1 : 0; }

int sc_plan_create(sc_plan** out, int D, int n, double l, int dtype, size_t* workspace_bytes) {
  if (!out) return fail(SC_ERR_INVALID, "plan output pointer is null");
  *out = nullptr;
  if (D != 2 && D != 3) return fail(SC_ERR_INVALID, "D must be 2 or 3 (got %d)", D);
  if (n % 2 != 0) return fail(SC_ERR_SIZE, "Only even number of grid points supported (n=%d)", n);
  if (!sc::fft_size_supported(n)) return fail(SC_ERR_SIZE, "n=%d is not a supported 2^a 3^b 5^c size", n);
  if (!(l > 0)) return fail(SC_ERR_INVALID, "domain length must be positive");
  if (dtype != SC_FLOAT32 && dtype != SC_FLOAT64) return fail(SC_ERR_INVALID, "dtype must be 0 (f32) or 1 (f64)");
  sc_plan* p = new sc_plan();
  p->D = D; p->n = n; p->l = l; p->dtype = dtype;
  SC_CU(cudaGetDevice(&p->dev));
  p->kc = n / 3; p->K1 = p->kc + 1; p->K2 = 2 * p->kc + 1;
  p->esz = dtype == SC_FLOAT64 ? 16 : 8;
  p->csz = (size_t)p->K1 * p->K2 * (D == 3 ? p->K2 : 1);
  p->fsz = (size_t)(n / 2 + 1) * n * (D == 3 ? n : 1);
  // (kx, y[, z]) and (kx, ky, z) scratch; in 3D the x extent is padded to an
  // even count for the product pipeline's intermediates
  const size_t K1x = D == 3 ? (size_t)even_up(p->K1) : (size_t)p->K1;
  const size_t plane = K1x * n * (D == 3 ? n : 1);
  const size_t mid = K1x * p->K2 * n;
  int rc = SC_OK;
  bool ok = (dtype == SC_FLOAT64) ? sc::init_kernels<double>(n) : sc::init_kernels<float>(n);
  if (!ok) { rc = fail(SC_ERR_CUDA, "kernel attribute setup failed for n=%d", n); goto bad; }
  if ((rc = plan_alloc(p, &p->tw, sc::twiddle_buffer_bytes(n, p->esz)))) goto bad;
  for (int c = 0; c < D; ++c) {
    if ((rc = plan_alloc(p, &p->U[c], p->csz * p->esz))) goto bad;
    if ((rc = plan_alloc(p, &p->ACC[c], p->csz * p->esz))) goto bad;
    if ((rc = plan_alloc(p, &p->S[c], p->csz * p->esz))) goto bad;
  }
  for (int c = 0; c < (D == 3 ? 6 : 3); ++c) {
    if ((rc = plan_alloc(p, &p->sig[c], p->csz * p->esz))) goto bad;
    if ((rc = plan_alloc(p, &p->dd[c], plane * p->esz))) goto bad;
    if (D == 3 && (rc = plan_alloc(p, &p->be[c], mid * p->esz))) goto bad;
  }
  for (int c = 0; c < D; ++c)
    if ((rc = plan_alloc(p, &p->cc[c], plane * p->esz))) goto bad;
  if ((rc = plan_alloc(p, (void**)&p->dscal, 16 * sizeof(double)))) goto bad;
  if ((rc = plan_alloc(p, (void**)&p->err, sizeof(int)))) goto bad;
  if (cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking) != cudaSuccess) {
    rc = fail(SC_ERR_CUDA, "stream creation failed");
    goto bad;
  }
  rc = dtype == SC_FLOAT64 ? upload_twiddles<double>(p) : upload_twiddles<float>(p);
  if (rc) goto bad;
  if (cudaMemset(p->dscal, 0, 16 * sizeof(double)) != cudaSuccess ||
      cudaMemset(p->err, 0, sizeof(int)) != cudaSuccess) {
    rc = fail(SC_ERR_CUDA, "memset");
    goto bad;
  }
  if (workspace_bytes) *workspace_bytes = p->ws;
  *out = p;
  return SC_OK;
bad:
  plan_free(p);
  delete p;
  return rc;
}

int sc_plan_destroy(sc_plan* p) {
  if (!p) return SC_OK;
  ensure_device(p);
  plan_free(p);
  delete p;
  return SC_OK;
}

int sc_plan_info(const sc_plan* p, int* D, int* n, int* dtype, int* kcut) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (D) *D = p->D;
  if (n) *n = p->n;
  if (dtype) *dtype = p->dtype;
  if (kcut) *kcut = p->kc;
  return SC_OK;
}

int sc_to_phys(sc_plan* p, const void* spec, void* phys, void* stream) {
  if (!p || !spec || !phys) return fail(SC_ERR_INVALID, "null argument");
  int rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, to_phys_impl, p, spec, phys, as_stream(stream));
}

int sc_to_spec(sc_plan* p, const void* phys, void* spec, void* stream) {
  if (!p || !spec || !phys) return fail(SC_ERR_INVALID, "null argument");
  int rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, to_spec_impl, p, phys, spec, as_stream(stream));
}

int sc_rhs(sc_plan* p, const void* const* u, void* const* du, double visc, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = check_ptrs((const void* const*)du, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  auto body = [&](auto tag) -> int {
    using R = decltype(tag);
    int r = pack_state<R>(p, u, p->S, st);
    if (r) return r;
    r = products<R>(p, p->S, st);
    if (r) return r;
    sc::EpiArgs e = epi_base<R>(p, p->S, visc);
    for (int c = 0; c < p->D; ++c) { e.base_a[c] = nullptr; e.out_a[c] = p->ACC[c]; }
    e.ca = 1.0;
    sc::launch_epilogue<R>(e, st);
    r = check_launch("rhs epilogue");
    if (r) return r;
    return unpack_state<R>(p, p->ACC, du, st);
  };
  return p->dtype == SC_FLOAT64 ? body(double()) : body(float());
}

int sc_state_load(sc_plan* p, const void* const* u, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, pack_state, p, u, p->U, as_stream(stream));
}

int sc_state_store(sc_plan* p, void* const* u, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  int rc = check_ptrs((const void* const*)u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, unpack_state, p, p->U, u, as_stream(stream));
}

int sc_state_rk4(sc_plan* p, double dt, double visc, int nsteps, const sc_forcing* frc, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (nsteps < 0) return fail(SC_ERR_INVALID, "nsteps must be >= 0");
  if (frc && frc->enabled && !(frc->eps >= 0)) return fail(SC_ERR_INVALID, "forcing eps must be >= 0");
  int rc = ensure_device(p);
  if (rc) return rc;
  if (nsteps == 0) return SC_OK;
  return SC_DTYPE_DISPATCH(p, run_rk4, p, dt, visc, nsteps, frc, as_stream(stream));
}

int sc_state_rk4_launches_per_step(const sc_plan* p, int forced) {
  if (!p) return 0;
  // per stage: [band forcing] + 5 sweeps (3D) or 3 sweeps (2D) + epilogue
  return 4 * ((forced ? 1 : 0) + (p->D == 3 ? 5 : 3) + 1);
}

int sc_rk4_steps(sc_plan* p, void* const* u, double dt, double visc, int nsteps, const sc_forcing* frc,
                 void* stream) {
  int rc = sc_state_load(p, (const void* const*)u, stream);
  if (rc) return rc;
  rc = sc_state_rk4(p, dt, visc, nsteps, frc, stream);
  if (rc) return rc;
  return sc_state_store(p, u, stream);
}

int sc_wray3_step(sc_plan* p, void* const* u, double dt, double visc, void* stream) {
  int rc = sc_state_load(p, (const void* const*)u, stream);
  if (rc) return rc;
  rc = SC_DTYPE_DISPATCH(p, run_wray_graph, p, dt, visc, as_stream(stream));
  if (rc) return rc;
  return sc_state_store(p, u, stream);
}

int sc_state_profile_rhs(sc_plan* p, double visc, int reps, double* ms, int* nkernels, void* stream) {
  if (!p || !ms || !nkernels || reps < 1) return fail(SC_ERR_INVALID, "bad argument");
  int rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const int nk = (p->D == 3 ? 5 : 3) + 1;
  cudaEvent_t ev[8];
  for (int i = 0; i <= nk; ++i) SC_CU(cudaEventCreate(&ev[i]));
  for (int i = 0; i < nk; ++i) ms[i] = 0;
  auto body = [&](auto tag) -> int {
    using R = decltype(tag);
    for (int r = 0; r < reps; ++r) {
      int q = products<R>(p, p->U, st, ev);
      if (q) return q;
      sc::EpiArgs e = epi_base<R>(p, p->U, visc);
      for (int c = 0; c < p->D; ++c) { e.base_a[c] = nullptr; e.out_a[c] = p->ACC[c]; }
      e.ca = 1.0;
      sc::launch_epilogue<R>(e, st);
      cudaEventRecord(ev[nk], st);
      SC_CU(cudaEventSynchronize(ev[nk]));
      for (int i = 0; i < nk; ++i) {
        float t = 0;
        SC_CU(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
        ms[i] += t / reps;
      }
    }
    return check_launch("profile");
  };
  rc = p->dtype == SC_FLOAT64 ? body(double()) : body(float());
  for (int i = 0; i <= nk; ++i) cudaEventDestroy(ev[i]);
  *nkernels = nk;
  return rc;
}

}  // extern "C"

namespace {
template <typename R>
int microbench_impl(int kernel, int n, long long count, int reps, double* ms, double* bytes) {
  const int variant = kernel >> 8;  // autotuner variant of the sweep (sc_plan_num_variants)
  kernel &= 0xff;
  const int kc = n / 3, K1 = kc + 1, K2 = 2 * kc + 1;
  const size_t esz = sizeof(typename sc::V2<R>::T);
  std::vector<void*> bufs;
  auto alloc = [&](size_t elems) -> void* {
    void* ptr = nullptr;
    if (cudaMalloc(&ptr, elems * esz) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    cudaMemset(ptr, 0, elems * esz);
    bufs.push_back(ptr);
    return ptr;
  };
  auto cleanup = [&]() { for (void* b : bufs) cudaFree(b); };
  const std::vector<unsigned char> timg = twiddle_image<R>(n);  // the solver's twiddles
  void* tw = alloc((timg.size() + esz - 1) / esz);
  if (!tw) { cleanup(); return fail(SC_ERR_OOM, "microbench allocation failed"); }
  cudaMemcpy(tw, timg.data(), timg.size(), cudaMemcpyHostToDevice);
  if (!(esz == 8 ? sc::init_kernels<float>(n) : sc::init_kernels<double>(n))) { cleanup(); return fail(SC_ERR_SIZE, "n"); }
  sc::ColArgs ca{};
  sc::XArgs xa{};
  double b = 0;
  const int ld = even_up(K1);
  int* err = static_cast<int*>(alloc(1));
  const int nin = kernel == 1 ? 6 : 3, nout = kernel == 0 ? 3 : 6;
  if (kernel == 0 || kernel == 1) {
    // y-inverse (3 comps) / y-forward (6 comps) of the solver over `count` z
    // planes: the (kx, ky, z) side is a full-size intermediate, so its lines
    // keep the solver's strides
    // (the product pipeline's padded row length on the intermediate side)
    if (count > n) { cleanup(); return fail(SC_ERR_INVALID, "count exceeds the %d z planes", n); }
    const size_t mid = (size_t)ld * n * K2;
    ca = kernel == 0 ? y_inverse_args(K1, n, kc, ld) : y_forward_args(K1, n, kc, ld);
    for (int c = 0; c < nin; ++c) ca.in[c] = alloc(kernel == 0 ? mid : (size_t)ld * n * count);
    for (int c = 0; c < nout; ++c) ca.out[c] = alloc(kernel == 0 ? (size_t)K1 * n * count : mid);
    ca.ncomp = nout; ca.ncols = (int)count;
    b = (double)(nin + nout) / 2 * esz * K1 * count * (K2 + n);
  } else if (kernel == 3 || kernel == 4) {
    // z-inverse / z-forward of the solver, one component, over the first
    // `count` ky columns of a full-size cube and intermediate
    if (count > K2) { cleanup(); return fail(SC_ERR_INVALID, "count exceeds the %d ky columns", K2); }
    const size_t cube = (size_t)K1 * K2 * K2, mid = (size_t)ld * n * K2;
    ca = kernel == 3 ? z_inverse_args(K1, K2, n, kc, ld) : z_forward_args(K1, n, kc, ld);
    ca.in[0] = alloc(kernel == 3 ? cube : mid);
    ca.out[0] = alloc(kernel == 3 ? mid : cube);
    ca.ncomp = 1; ca.ncols = (int)count;
    b = (double)esz * K1 * count * (K2 + n);
  } else if (kernel == 2) {  // 3D x sweep over `count` rows
    for (int c = 0; c < 3; ++c) xa.in[c] = alloc((size_t)K1 * count);
    for (int c = 0; c < 6; ++c) xa.out[c] = alloc((size_t)K1 * count);
    xa.D = 3; xa.K1in = K1; xa.K1out = K1; xa.nrows = count; xa.scale = 1.0 / ((double)n * n * n);
    xa.variant = variant;
    b = 9.0 * K1 * count * esz;
  } else {
    cleanup();
    return fail(SC_ERR_INVALID, "unknown microbench kernel %d", kernel);
  }
  for (void* q : bufs) if (!q) { cleanup(); return fail(SC_ERR_OOM, "microbench allocation failed"); }
  ca.variant = variant;
  ca.wait_limit = sc::kDefaultWaitLimit;
  ca.err = err;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0); cudaEventCreate(&e1);
  auto launch = [&]() {
    if (kernel == 0 || kernel == 3) sc::launch_col_inv<R>(n, ca, tw, 0);
    else if (kernel == 1 || kernel == 4) sc::launch_col_fwd<R>(n, ca, tw, 0);
    else sc::launch_xsweep_ns<R>(n, xa, tw, 0);
  };
  launch();
  cudaEventRecord(e0, 0);
  for (int r = 0; r < reps; ++r) launch();
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  int rc = check_launch("microbench");
  int h = 0;
  if (!rc && err) cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
  if (!rc && h) rc = fail(SC_ERR_TIMEOUT, "a bounded wait of the TMA-fed sweep ran out");
  cleanup();
  if (rc) return rc;
  *ms = t / reps;
  *bytes = b;
  return SC_OK;
}
}  // namespace

extern "C" {

int sc_microbench(int kernel, int n, int dtype, long long count, int reps, double* ms, double* bytes) {
  if (!ms || !bytes || reps < 1 || count < 1 || kernel < 0) return fail(SC_ERR_INVALID, "bad argument");
  if (!sc::fft_size_supported(n)) return fail(SC_ERR_SIZE, "unsupported n=%d", n);
  return dtype == SC_FLOAT64 ? microbench_impl<double>(kernel, n, count, reps, ms, bytes)
                             : microbench_impl<float>(kernel, n, count, reps, ms, bytes);
}

int sc_state_energy(sc_plan* p, double* e, void* stream) {
  if (!p || !e) return fail(SC_ERR_INVALID, "null argument");
  int rc = ensure_device(p);
  if (rc) return rc;
  double s = 0;
  rc = SC_DTYPE_DISPATCH(p, energy_impl, p, (const void* const*)p->U, 1, 0, &s, as_stream(stream));
  if (rc) return rc;
  *e = 0.5 * s;
  return SC_OK;
}

int sc_energy(sc_plan* p, const void* const* u, double* e, void* stream) {
  if (!p || !e) return fail(SC_ERR_INVALID, "null argument");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  double s = 0;
  rc = SC_DTYPE_DISPATCH(p, energy_impl, p, u, 0, 0, &s, as_stream(stream));
  if (rc) return rc;
  *e = 0.5 * s;
  return SC_OK;
}

int sc_dissipation(sc_plan* p, const void* const* u, double visc, double* d, void* stream) {
  if (!p || !d) return fail(SC_ERR_INVALID, "null argument");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  double s = 0;
  rc = SC_DTYPE_DISPATCH(p, energy_impl, p, u, 0, 1, &s, as_stream(stream));
  if (rc) return rc;
  *d = visc * s;
  return SC_OK;
}

int sc_filter_sfs(sc_plan* dns, sc_plan* les, const void* const* u, const double* deltas, int ndelta,
                  void* const* ubar, void* const* tau, void* stream) {
  if (!dns || !les || !deltas || ndelta < 1 || !ubar || !tau) return fail(SC_ERR_INVALID, "bad argument");
  if (dns == les) return fail(SC_ERR_INVALID, "the DNS and LES plans must be distinct objects");
  if (dns->D != les->D || dns->dtype != les->dtype || dns->dev != les->dev)
    return fail(SC_ERR_INVALID, "DNS and LES plans differ in dimension, precision or device");
  if (std::fabs(dns->l - les->l) > 1e-12 * dns->l) return fail(SC_ERR_INVALID, "DNS and LES domain lengths differ");
  if (les->n > dns->n) return fail(SC_ERR_INVALID, "LES grid (n=%d) finer than the DNS grid (n=%d)", les->n, dns->n);
  int rc = check_ptrs(u, dns->D);
  if (!rc) rc = check_ptrs((const void* const*)ubar, dns->D * ndelta);
  if (!rc) rc = check_ptrs((const void* const*)tau, (dns->D == 3 ? 6 : 3) * ndelta);
  if (!rc) rc = ensure_device(dns);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(dns, filter_impl, dns, les, u, deltas, ndelta, ubar, tau, as_stream(stream));
}

int sc_filter_reynolds(sc_plan* les, const void* const* ubar, double visc, double delta, double* out, void* stream) {
  if (!les || !out || !(visc > 0)) return fail(SC_ERR_INVALID, "bad argument");
  int rc = check_ptrs(ubar, les->D);
  if (!rc) rc = ensure_device(les);
  if (rc) return rc;
  double a2 = 0;
  rc = SC_DTYPE_DISPATCH(les, energy_impl, les, ubar, 0, 1, &a2, as_stream(stream), 1);
  if (rc) return rc;
  *out = delta * delta * std::sqrt(a2) / visc;
  return SC_OK;
}

int sc_closure_create(sc_closure** out, sc_plan* p, int kind, double delta, const double* params, int nparams) {
  if (!out || !p) return fail(SC_ERR_INVALID, "null argument");
  *out = nullptr;
  if (kind < sc::kNoClosure || kind > sc::kBardina)
    return fail(kind == sc::kCnn ? SC_ERR_UNSUPPORTED : SC_ERR_INVALID,
                kind == sc::kCnn ? "the CNN closure is created with sc_cnn_closure_create" : "unknown closure kind %d",
                kind);
  if (kind == sc::kVerstappen && p->D != 3) return fail(SC_ERR_INVALID, "Q-R model is only defined in 3D");
  if (kind != sc::kNoClosure && !(delta > 0)) return fail(SC_ERR_INVALID, "filter width must be positive");
  if (nparams < 0 || nparams > 4 || (nparams > 0 && !params)) return fail(SC_ERR_INVALID, "bad params");
  int rc = ensure_device(p);
  if (rc) return rc;
  sc_closure* cl = new sc_closure();
  cl->p = p; cl->kind = kind; cl->delta = delta;
  for (int i = 0; i < nparams; ++i) cl->prm[i] = params[i];
  if (kind == sc::kSmagorinsky && nparams < 1) cl->prm[0] = 0.17;
  if (kind == sc::kVerstappen && nparams < 1) cl->prm[0] = 0.345;
  if (kind == sc::kBardina && nparams < 1) cl->prm[0] = 2.0;
  const int D = p->D, NP = D == 3 ? 6 : 3;
  const size_t cb = p->csz * p->esz;
  const size_t pb = (size_t)std::pow((double)p->n, D) * (p->esz / 2);
  const size_t mid = (D == 3 ? (size_t)p->K1 * p->K2 * p->n : 0) * p->esz;
  const size_t plane = (size_t)p->K1 * p->n * (D == 3 ? p->n : 1) * p->esz;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  if (kind != sc::kNoClosure) {
    for (int c = 0; c < D * D && !rc; ++c) rc = A(&cl->gc[c], cb);
    for (int c = 0; c < D * D && !rc; ++c) rc = A(&cl->gp[c], pb);
    for (int c = 0; c < NP && !rc; ++c) rc = A(&cl->tp[c], pb);
    for (int c = 0; c < NP && !rc; ++c) rc = A(&cl->th[c], cb);
    for (int c = 0; c < D && !rc; ++c) rc = A(&cl->ut[c], cb);
    for (int c = 0; c < NP && !rc; ++c) rc = A(&cl->s2[c], cb);
    for (int c = 0; c < NP && !rc; ++c) rc = A(&cl->ph2[c], pb);
    for (int c = 0; c < NP && !rc; ++c) rc = A(&cl->ph3[c], pb);
    for (int c = 0; c < D && !rc; ++c) rc = A(&cl->ph4[c], pb);
    for (int c = 0; c < 12 && !rc; ++c) rc = A(&cl->cb[c], plane);
    for (int c = 0; c < 12 && !rc && D == 3; ++c) rc = A(&cl->bb[c], mid);
    if (!rc) rc = A((void**)&cl->dsum, 4 * sizeof(double));
  }
  if (rc) {
    for (void* a : cl->allocs) cudaFree(a);
    delete cl;
    return rc;
  }
  *out = cl;
  return SC_OK;
}

static uint16_t host_bf16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  if ((x & 0x7f800000u) == 0x7f800000u) return uint16_t((x >> 16) | ((x & 0xffffu) ? 0x40u : 0u));  // inf/nan
  const uint32_t lsb = (x >> 16) & 1u;
  x += 0x7fffu + lsb;  // round to nearest even
  return uint16_t(x >> 16);
}

static float host_bf16_value(uint16_t b) {
  const uint32_t x = uint32_t(b) << 16;
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}

}  // extern "C"

namespace {
// Upload theta (PyTorch order per layer: w[Cout][Cin][27] then b[Cout]) to the
// tensor-core CNN: BF16 forward weights in the UMMA K-major layout
// [27][CP/8][COP][8], FP32 biases, and the input-gradient convolution's
// weights W'[ci][co][t'] = W[co][ci][26 - t'] (transposed and flipped) in the
// same layout with the roles of CP and COP exchanged.
int tc_upload_params(sc_closure* cl, const double* theta) {
  static const int cin[4] = {4, 32, 32, 32}, cout[4] = {32, 32, 32, 6}, cp[4] = {16, 32, 32, 32},
                   cop[4] = {32, 32, 32, 16};
  bool fits = true;  // every weight x kSplitScale is an FP16 number
  for (int l = 0; l < 4; ++l) {
    const long long o = cc_layer_offset(l), nw = (long long)cout[l] * cin[l] * 27;
    const int cpc = cp[l] / 8;
    const size_t nwp = (size_t)27 * cp[l] * cop[l];
    // BF16 forward and transposed weights; for the split precision also the
    // FP16 high and low parts of theta x kSplitScale (forward) and the BF16
    // low parts theta - bf16(theta) of the transposed weights
    std::vector<uint16_t> wp(nwp, 0), wt(nwp, 0), wh(nwp, 0), wl(nwp, 0), wtl(nwp, 0);
    for (int t = 0; t < 27; ++t)
      for (int kc = 0; kc < cpc; ++kc)
        for (int nn = 0; nn < cout[l]; ++nn)
          for (int j = 0; j < 8; ++j) {
            const int ci = 8 * kc + j;
            if (ci >= cin[l]) continue;
            const double x = theta[o + ((long long)nn * cin[l] + ci) * 27 + t];
            const size_t d = (((size_t)t * cpc + kc) * cop[l] + nn) * 8 + j;
            wp[d] = host_bf16(float(x));
            const double xs = x * double(sc::kSplitScale);
            if (!(std::fabs(xs) < 6.5e4)) fits = false;
            const __half hh = __float2half_rn(float(xs));
            const __half hl = __float2half_rn(float(xs - double(__half2float(hh))));
            std::memcpy(&wh[d], &hh, 2);
            std::memcpy(&wl[d], &hl, 2);
          }
    const int cpc2 = cop[l] / 8;  // input-gradient convolution: CP' = cop, COP' = cp
    for (int t2 = 0; t2 < 27; ++t2)
      for (int kc = 0; kc < cpc2; ++kc)
        for (int nn = 0; nn < cin[l]; ++nn)
          for (int j = 0; j < 8; ++j) {
            const int k = 8 * kc + j;  // a forward output channel
            if (k >= cout[l]) continue;
            const double x = theta[o + ((long long)k * cin[l] + nn) * 27 + (26 - t2)];
            const size_t d = (((size_t)t2 * cpc2 + kc) * cp[l] + nn) * 8 + j;
            wt[d] = host_bf16(float(x));
            wtl[d] = host_bf16(float(x - double(host_bf16_value(wt[d]))));
          }
    std::vector<float> bp(cop[l], 0.f);
    for (int nn = 0; nn < cout[l]; ++nn) bp[nn] = float(theta[o + nw + nn]);
    SC_CU(cudaMemcpy(cl->cw[l], wp.data(), wp.size() * 2, cudaMemcpyHostToDevice));
    SC_CU(cudaMemcpy(cl->cwt[l], wt.data(), wt.size() * 2, cudaMemcpyHostToDevice));
    SC_CU(cudaMemcpy(cl->cwh[l], wh.data(), wh.size() * 2, cudaMemcpyHostToDevice));
    SC_CU(cudaMemcpy(cl->cwl[l], wl.data(), wl.size() * 2, cudaMemcpyHostToDevice));
    SC_CU(cudaMemcpy(cl->cwtl[l], wtl.data(), wtl.size() * 2, cudaMemcpyHostToDevice));
    SC_CU(cudaMemcpy(cl->cbias[l], bp.data(), bp.size() * 4, cudaMemcpyHostToDevice));
  }
  cl->split_fits = fits;
  if (cl->cnn_split && !fits) return fail(SC_ERR_INVALID, "a CNN weight is beyond the FP16 range of the split precision");
  return SC_OK;
}

// the tensor-core CNN's adjoint buffers, on first use
int tc_adjoint_buffers(sc_closure* cl) {
  if (cl->tgf) return SC_OK;
  const size_t np = (size_t)cl->p->n * cl->p->n * cl->p->n;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  int rc = A(&cl->tact3, np * 32 * 2);
  for (int l = 0; l < 3 && !rc; ++l) rc = A(&cl->tpre[l], np * 32 * 4);
  if (!rc) rc = A(&cl->tgbf, np * 32 * 2);
  if (!rc) rc = A(&cl->cctau, np * 6 * 4);
  if (!rc) rc = A(&cl->ccg0, np * 4 * 4);
  if (!rc) rc = A(&cl->tgbfl, np * 32 * 2);
  if (!rc) rc = A(&cl->tgf, np * 32 * 4);  // last: marks the set complete
  return rc;
}

// the split precision's activation buffers, on first use
int tc_split_buffers(sc_closure* cl) {
  if (cl->sacc) return SC_OK;
  const size_t np = (size_t)cl->p->n * cl->p->n * cl->p->n;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  int rc = SC_OK;
  for (int l = 0; l < 4 && !rc; ++l) {
    const size_t ch = l == 0 ? 16 : 32;
    rc = A(&cl->sacth[l], np * ch * 2);
    if (!rc) rc = A(&cl->sactl[l], np * ch * 2);
  }
  if (!rc) rc = A(&cl->sacc, np * 32 * 4);  // last: marks the set complete
  return rc;
}
}  // namespace

extern "C" {

int sc_cnn_closure_create(sc_closure** out, sc_plan* p, double delta, double visc, const float* const* weights,
                          const float* const* biases, double mu, double sigma) {
  if (!out || !p || !weights || !biases) return fail(SC_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->dtype != SC_FLOAT32 || !sc::cnn_supported(p->n, p->D))
    return fail(SC_ERR_UNSUPPORTED, "the tensor-core CNN closure runs on FP32 3D plans with n = 64 or 128");
  if (!(delta > 0) || !(visc > 0) || !(sigma > 0)) return fail(SC_ERR_INVALID, "delta, visc and sigma must be positive");
  for (int l = 0; l < 4; ++l)
    if (!weights[l] || !biases[l]) return fail(SC_ERR_INVALID, "missing weights of layer %d", l);
  sc_closure* cl = nullptr;
  int rc = sc_closure_create(&cl, p, sc::kClark, delta, nullptr, 0);  // allocates the common scratch
  if (rc) return rc;
  cl->kind = sc::kCnn;
  cl->nu = visc; cl->mu = mu; cl->sigma = sigma;
  cl->nparam = cc_layer_offset(4);
  static const int cp[4] = {16, 32, 32, 32}, cop[4] = {32, 32, 32, 16};
  const size_t npts = (size_t)p->n * p->n * p->n;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  for (int l = 0; l < 4 && !rc; ++l) {
    const size_t nwp = (size_t)27 * cp[l] * cop[l];
    rc = A(&cl->cw[l], nwp * 2);
    if (!rc) rc = A(&cl->cwt[l], nwp * 2);
    if (!rc) rc = A(&cl->cwh[l], nwp * 2);
    if (!rc) rc = A(&cl->cwl[l], nwp * 2);
    if (!rc) rc = A(&cl->cwtl[l], nwp * 2);
    if (!rc) rc = A(&cl->cbias[l], cop[l] * 4);
  }
  if (!rc) rc = A(&cl->act[0], npts * 16 * 2);
  if (!rc) rc = A(&cl->act[1], npts * 32 * 2);
  if (!rc) rc = A(&cl->act[2], npts * 32 * 2);
  if (!rc) rc = A((void**)&cl->err, sizeof(int));
  if (!rc) rc = A((void**)&cl->gw, cl->nparam * sizeof(double));
  if (!rc && cudaMemset(cl->err, 0, sizeof(int)) != cudaSuccess) rc = fail(SC_ERR_CUDA, "memset");
  if (!rc) {
    std::vector<double> theta(cl->nparam);
    for (int l = 0; l < 4; ++l) {
      const long long o = cc_layer_offset(l), nw = (long long)kCcCout[l] * kCcCin[l] * 27;
      for (long long i = 0; i < nw; ++i) theta[o + i] = weights[l][i];
      for (int i = 0; i < kCcCout[l]; ++i) theta[o + nw + i] = biases[l][i];
    }
    rc = tc_upload_params(cl, theta.data());
  }
  if (!rc) {
    sc::cnn_init();
    if (cudaGetLastError() != cudaSuccess) rc = fail(SC_ERR_CUDA, "CNN kernel setup");
  }
  if (rc) { sc_closure_destroy(cl); return rc; }
  *out = cl;
  return SC_OK;
}

int sc_cnn_fp_closure_create(sc_closure** out, sc_plan* p, double delta, double visc, const float* const* weights,
                             const float* const* biases, double mu, double sigma) {
  if (!out || !p || !weights || !biases) return fail(SC_ERR_INVALID, "null argument");
  *out = nullptr;
  if (p->D != 3) return fail(SC_ERR_UNSUPPORTED, "the CNN closure is 3D");
  if (!(delta > 0) || !(visc > 0) || !(sigma > 0)) return fail(SC_ERR_INVALID, "delta, visc and sigma must be positive");
  for (int l = 0; l < 4; ++l)
    if (!weights[l] || !biases[l]) return fail(SC_ERR_INVALID, "missing weights of layer %d", l);
  sc_closure* cl = nullptr;
  int rc = sc_closure_create(&cl, p, sc::kClark, delta, nullptr, 0);
  if (rc) return rc;
  cl->kind = sc::kCnnFp;
  cl->nu = visc; cl->mu = mu; cl->sigma = sigma;
  const size_t es = p->esz / 2;  // bytes per real
  const size_t np = (size_t)p->n * p->n * p->n;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  cl->nparam = cc_layer_offset(4);
  for (int l = 0; l < 4 && !rc; ++l) {
    const size_t nw = (size_t)kCcCout[l] * kCcCin[l] * 27;
    rc = A(&cl->ccw[l], nw * es);
    if (!rc) rc = A(&cl->ccb[l], kCcCout[l] * es);
  }
  static const int chans[7] = {4, 32, 32, 32, 32, 32, 32};
  for (int i = 0; i < 7 && !rc; ++i) rc = A(&cl->cca[i], chans[i] * np * es);
  if (!rc) rc = A(&cl->cctau, 6 * np * es);
  for (int i = 0; i < 2 && !rc; ++i) rc = A(&cl->ccg[i], 32 * np * es);
  if (!rc) rc = A(&cl->ccg0, 4 * np * es);
  if (!rc) rc = A((void**)&cl->gw, cl->nparam * sizeof(double));
  if (rc) { sc_closure_destroy(cl); return rc; }
  std::vector<double> theta(cl->nparam);
  for (int l = 0; l < 4; ++l) {
    const long long o = cc_layer_offset(l), nw = (long long)kCcCout[l] * kCcCin[l] * 27;
    for (long long i = 0; i < nw; ++i) theta[o + i] = weights[l][i];
    for (int i = 0; i < kCcCout[l]; ++i) theta[o + nw + i] = biases[l][i];
  }
  rc = sc_closure_set_params(cl, theta.data());
  if (rc) { sc_closure_destroy(cl); return rc; }
  *out = cl;
  return SC_OK;
}

}  // extern "C"

namespace {
int pointwise_net_create(sc_closure** out, sc_plan* p, int kind, double delta, double visc, int nlayers,
                         const int* widths, const double* theta, int use_redelta, double mu, double sigma) {
  if (!out || !p || !widths || !theta) return fail(SC_ERR_INVALID, "null argument");
  *out = nullptr;
  const int D = p->D, NP = D == 3 ? 6 : 3;
  const int nin = kind == sc::kTbnn ? (D == 3 ? 5 : 2) : D * D;  // invariants or gradient channels
  const int nout = kind == sc::kTbnn ? (D == 3 ? 7 : 2) : NP;    // basis coefficients or stress
  if (nlayers < 1 || nlayers > sc::kMlpMaxLayers) return fail(SC_ERR_INVALID, "1 <= nlayers <= %d", sc::kMlpMaxLayers);
  if (widths[0] != nin + (use_redelta ? 1 : 0))
    return fail(SC_ERR_INVALID, "widths[0] must be %d (+1 with the Re_Delta channel)", nin);
  if (widths[nlayers] != nout) return fail(SC_ERR_INVALID, "the last width must be %d", nout);
  for (int l = 0; l <= nlayers; ++l)
    if (widths[l] < 1 || widths[l] > sc::kMlpMaxWidth) return fail(SC_ERR_INVALID, "widths must be 1..%d", sc::kMlpMaxWidth);
  if (!(delta > 0) || (use_redelta && (!(visc > 0) || !(sigma > 0))))
    return fail(SC_ERR_INVALID, "delta (and with Re_Delta: visc, sigma) must be positive");
  sc_closure* cl = nullptr;
  int rc = sc_closure_create(&cl, p, sc::kClark, delta, nullptr, 0);
  if (rc) return rc;
  cl->kind = kind;
  cl->nu = visc; cl->mu = mu; cl->sigma = sigma;
  cl->mlp_nl = nlayers;
  long long np_ = 0;
  for (int l = 0; l < nlayers; ++l) {
    cl->mlp_w[l] = widths[l];
    np_ += (long long)widths[l] * widths[l + 1] + (l < nlayers - 1 ? widths[l + 1] : 0);
  }
  cl->mlp_w[nlayers] = widths[nlayers];
  cl->nparam = np_;
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e)); }
    cl->allocs.push_back(*ptr);
    return SC_OK;
  };
  rc = A(&cl->mlp_theta, np_ * (p->esz / 2));
  if (!rc && use_redelta) rc = A((void**)&cl->mlp_z, 2 * sizeof(double));
  if (!rc) rc = sc_closure_set_params(cl, theta);
  if (rc) { sc_closure_destroy(cl); return rc; }
  *out = cl;
  return SC_OK;
}
}  // namespace

extern "C" {

int sc_mlp_closure_create(sc_closure** out, sc_plan* p, double delta, double visc, int nlayers, const int* widths,
                          const double* theta, int use_redelta, double mu, double sigma) {
  return pointwise_net_create(out, p, sc::kMlp, delta, visc, nlayers, widths, theta, use_redelta, mu, sigma);
}

int sc_tbnn_closure_create(sc_closure** out, sc_plan* p, double delta, double visc, int nlayers, const int* widths,
                           const double* theta, int use_redelta, double mu, double sigma) {
  return pointwise_net_create(out, p, sc::kTbnn, delta, visc, nlayers, widths, theta, use_redelta, mu, sigma);
}

int sc_closure_num_params(const sc_closure* cl, long long* n) {
  if (!cl || !n) return fail(SC_ERR_INVALID, "null argument");
  *n = (cl->kind == sc::kCnnFp || cl->kind == sc::kCnn || cl->kind == sc::kMlp || cl->kind == sc::kTbnn) ? cl->nparam
                                                                                                         : 0;
  return SC_OK;
}

int sc_closure_set_params(sc_closure* cl, const double* theta) {
  if (!cl || !theta) return fail(SC_ERR_INVALID, "null argument");
  if (cl->kind == sc::kCnn) return tc_upload_params(cl, theta);
  if (cl->kind == sc::kMlp || cl->kind == sc::kTbnn) {
    if (cl->p->dtype == SC_FLOAT64) {
      SC_CU(cudaMemcpy(cl->mlp_theta, theta, cl->nparam * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> f(theta, theta + cl->nparam);
      SC_CU(cudaMemcpy(cl->mlp_theta, f.data(), cl->nparam * 4, cudaMemcpyHostToDevice));
    }
    return SC_OK;
  }
  if (cl->kind != sc::kCnnFp) return fail(SC_ERR_UNSUPPORTED, "only the CNN closures have a parameter vector");
  const bool f64 = cl->p->dtype == SC_FLOAT64;
  for (int l = 0; l < 4; ++l) {
    const long long o = cc_layer_offset(l), nw = (long long)kCcCout[l] * kCcCin[l] * 27, nb_ = kCcCout[l];
    if (f64) {
      SC_CU(cudaMemcpy(cl->ccw[l], theta + o, nw * 8, cudaMemcpyHostToDevice));
      SC_CU(cudaMemcpy(cl->ccb[l], theta + o + nw, nb_ * 8, cudaMemcpyHostToDevice));
    } else {
      std::vector<float> w(theta + o, theta + o + nw), b(theta + o + nw, theta + o + nw + nb_);
      SC_CU(cudaMemcpy(cl->ccw[l], w.data(), nw * 4, cudaMemcpyHostToDevice));
      SC_CU(cudaMemcpy(cl->ccb[l], b.data(), nb_ * 4, cudaMemcpyHostToDevice));
    }
  }
  // cached step graphs captured the old weights by pointer, which stay valid
  return SC_OK;
}

int sc_closure_set_option(sc_closure* cl, int option, long long value) {
  if (!cl) return fail(SC_ERR_INVALID, "null argument");
  if (option != SC_CLOPT_CNN_SPLIT) return fail(SC_ERR_INVALID, "unknown closure option %d", option);
  if (cl->kind != sc::kCnn)
    return fail(SC_ERR_UNSUPPORTED, "the split precision is an option of the tensor-core CNN closure");
  if (value != 0 && value != 1) return fail(SC_ERR_INVALID, "SC_CLOPT_CNN_SPLIT takes 0 or 1");
  sc_plan* p = cl->p;
  ensure_device(p);
  if (value && !cl->split_fits)
    return fail(SC_ERR_INVALID, "a CNN weight is beyond the FP16 range of the split precision");
  if (value) {
    const int rc = tc_split_buffers(cl);
    if (rc) return rc;
  }
  cl->cnn_split = value != 0;
  // cached step graphs hold the other precision's launches
  if (p->g_rk4) { cudaGraphExecDestroy(p->g_rk4); p->g_rk4 = nullptr; }
  if (p->g_wray) { cudaGraphExecDestroy(p->g_wray); p->g_wray = nullptr; }
  return SC_OK;
}

int sc_plan_status(sc_plan* p, int* status) {
  if (!p || !status) return fail(SC_ERR_INVALID, "null argument");
  ensure_device(p);
  int h = 0;
  SC_CU(cudaMemcpy(&h, p->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) SC_CU(cudaMemset(p->err, 0, sizeof(int)));
  *status = h ? SC_ERR_TIMEOUT : SC_OK;
  return SC_OK;
}

int sc_closure_status(sc_closure* cl, int* status) {
  if (!cl || !status) return fail(SC_ERR_INVALID, "null argument");
  *status = 0;
  if (!cl->err) return SC_OK;
  int h = 0;
  SC_CU(cudaMemcpy(&h, cl->err, sizeof(int), cudaMemcpyDeviceToHost));
  *status = h ? SC_ERR_TIMEOUT : SC_OK;
  return SC_OK;
}

int sc_closure_destroy(sc_closure* cl) {
  if (!cl) return SC_OK;
  sc_plan* p = cl->p;
  if (p) {
    ensure_device(p);
    // cached step graphs may reference this closure's buffers
    if (p->g_rk4) { cudaGraphExecDestroy(p->g_rk4); p->g_rk4 = nullptr; }
    if (p->g_wray) { cudaGraphExecDestroy(p->g_wray); p->g_wray = nullptr; }
  }
  for (void* a : cl->allocs) cudaFree(a);
  delete cl;
  return SC_OK;
}

int sc_closure_eval(sc_closure* cl, const void* const* u, const void* const* G, void* const* tau, void* stream) {
  if (!cl) return fail(SC_ERR_INVALID, "null closure");
  sc_plan* p = cl->p;
  const int D = p->D, NP = D == 3 ? 6 : 3;
  int rc = check_ptrs((const void* const*)tau, NP);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  if (cl->kind == sc::kNoClosure) return fail(SC_ERR_INVALID, "the empty closure has no stress");
  cudaStream_t st = as_stream(stream);
  auto body = [&](auto tag) -> int {
    using R = decltype(tag);
    if (cl->kind == sc::kMlp || cl->kind == sc::kTbnn) {
      int r = check_ptrs(G, D * D);
      if (r) return r;
      sc::launch_mlp<R>(mlp_args(cl, G, tau), cl->mlp_z, cl->nu, cl->mu, cl->sigma, st);
      return check_launch("mlp closure");
    }
    if (cl->kind == sc::kClark || cl->kind == sc::kSmagorinsky || cl->kind == sc::kVerstappen) {
      int r = check_ptrs(G, D * D);
      if (r) return r;
      sc::LesPhysArgs a = phys_args(p);
      for (int c = 0; c < D * D; ++c) a.in[c] = G[c];
      for (int c = 0; c < NP; ++c) a.out[c] = tau[c];
      a.kind = cl->kind; a.delta = cl->delta; a.p0 = cl->prm[0];
      sc::launch_closure_pt<R>(a, D, st);
      return check_launch("closure");
    }
    int r = check_ptrs(u, D);
    if (r) return r;
    if ((r = pack_state<R>(p, u, p->S, st))) return r;
    if ((r = products<R>(p, p->S, st))) return r;
    if ((r = closure_tauhat<R>(cl, p->S, st, tau))) return r;
    if (cl->err) {
      int h = 0;
      SC_CU(cudaMemcpyAsync(&h, cl->err, sizeof(int), cudaMemcpyDeviceToHost, st));
      SC_CU(cudaStreamSynchronize(st));
      if (h) return fail(SC_ERR_TIMEOUT, "a bounded wait of the CNN kernel ran out");
    }
    return SC_OK;
  };
  return p->dtype == SC_FLOAT64 ? body(double()) : body(float());
}

int sc_les_rhs(sc_plan* p, sc_closure* cl, const void* const* u, void* const* du, double visc, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = check_ptrs((const void* const*)du, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  auto body = [&](auto tag) -> int {
    using R = decltype(tag);
    int r = pack_state<R>(p, u, p->S, st);
    if (r) return r;
    if ((r = stage_rhs<R>(p, cl, p->S, st))) return r;
    sc::EpiArgs e = epi_base<R>(p, p->S, visc);
    add_closure_stress<R>(e, cl, p->D);
    for (int c = 0; c < p->D; ++c) { e.base_a[c] = nullptr; e.out_a[c] = p->ACC[c]; }
    e.ca = 1.0;
    sc::launch_epilogue<R>(e, st);
    if ((r = check_launch("les rhs"))) return r;
    return unpack_state<R>(p, p->ACC, du, st);
  };
  return p->dtype == SC_FLOAT64 ? body(double()) : body(float());
}

int sc_state_les_rk4(sc_plan* p, sc_closure* cl, double dt, double visc, int nsteps, const sc_forcing* frc,
                     void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  if (nsteps < 0) return fail(SC_ERR_INVALID, "nsteps must be >= 0");
  int rc = ensure_device(p);
  if (rc || nsteps == 0) return rc;
  return SC_DTYPE_DISPATCH(p, run_rk4, p, dt, visc, nsteps, frc, as_stream(stream), cl);
}

int sc_les_rk4_steps(sc_plan* p, sc_closure* cl, void* const* u, double dt, double visc, int nsteps,
                     const sc_forcing* frc, void* stream) {
  int rc = sc_state_load(p, (const void* const*)u, stream);
  if (rc) return rc;
  rc = sc_state_les_rk4(p, cl, dt, visc, nsteps, frc, stream);
  if (rc) return rc;
  return sc_state_store(p, u, stream);
}

int sc_les_wray3_step(sc_plan* p, sc_closure* cl, void* const* u, double dt, double visc, void* stream) {
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  int rc = sc_state_load(p, (const void* const*)u, stream);
  if (rc) return rc;
  rc = SC_DTYPE_DISPATCH(p, run_wray_graph, p, dt, visc, as_stream(stream), cl);
  if (rc) return rc;
  return sc_state_store(p, u, stream);
}

}  // extern "C"

namespace {
template <typename R>
int vmax_impl(sc_plan* p, void* const* uc, double* vmax, cudaStream_t st) {
  // y/z inverse of the D components (zero-padded, k = 0 masked) into the pencil scratch
  const int n = p->n, K1 = p->K1, K2 = p->K2, kc = p->kc, D = p->D;
  if (D == 3) {
    sc::ColArgs a = z_inverse_args(K1, K2, n, kc);
    for (int c = 0; c < 3; ++c) { a.in[c] = uc[c]; a.out[c] = p->be[c]; }
    a.ncomp = 3;
    sc::launch_col_inv<R>(n, a, p->tw, st);
    sc::ColArgs b = y_inverse_args(K1, n, kc);
    for (int c = 0; c < 3; ++c) { b.in[c] = p->be[c]; b.out[c] = p->cc[c]; }
    b.ncomp = 3;
    sc::launch_col_inv<R>(n, b, p->tw, st);
  } else {
    sc::ColArgs a{};
    for (int c = 0; c < 2; ++c) { a.in[c] = uc[c]; a.out[c] = p->cc[c]; }
    a.ncomp = 2; a.K1 = K1; a.ncols = 1;
    a.in_cs = 0; a.in_es = K1; a.out_cs = 0; a.out_es = K1;
    a.kpos = kc + 1; a.kneg = kc; a.zero_origin = 1;
    sc::launch_col_inv<R>(n, a, p->tw, st);
  }
  SC_CU(cudaMemsetAsync(p->dscal + 2, 0, sizeof(double), st));
  sc::XPlainArgs x{};
  for (int c = 0; c < D; ++c) x.in[c] = p->cc[c];
  x.ncomp = D; x.K1 = K1; x.nrows = D == 3 ? (long long)n * n : n;
  sc::launch_x_vmax<R>(n, x, p->tw, reinterpret_cast<unsigned long long*>(p->dscal + 2), st);
  int rc = check_launch("vmax");
  if (rc) return rc;
  double h = 0;
  SC_CU(cudaMemcpyAsync(&h, p->dscal + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  SC_CU(cudaStreamSynchronize(st));
  *vmax = h;
  return SC_OK;
}

template <typename R>
int clamp_impl(sc_plan* p, void* const* uc, double* eref_host, int mode, cudaStream_t st) {
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) a.dst[c] = uc[c];
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  if (mode == 1) SC_CU(cudaMemcpyAsync(p->dscal + 4, eref_host, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
  sc::launch_shell_clamp<R>(a, p->dscal + 4, mode, st);
  int rc = check_launch("shell clamp");
  if (rc) return rc;
  if (mode == 0) {
    SC_CU(cudaMemcpyAsync(eref_host, p->dscal + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SC_CU(cudaStreamSynchronize(st));
  }
  return SC_OK;
}

template <typename R>
int spectrum_impl(sc_plan* p, void* const* uc, int nshell, double* out, cudaStream_t st) {
  double* d = nullptr;
  SC_CU(cudaMallocAsync((void**)&d, nshell * sizeof(double), st));
  cudaMemsetAsync(d, 0, nshell * sizeof(double), st);
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) a.src[c] = uc[c];
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  sc::launch_spectrum<R>(a, nshell, d, st);
  int rc = check_launch("spectrum");
  cudaMemcpyAsync(out, d, nshell * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  SC_CU(cudaStreamSynchronize(st));
  return rc;
}
}  // namespace

extern "C" {

int sc_propose_timestep(sc_plan* p, const void* const* u, double visc, double* dt, void* stream) {
  if (!p || !dt || !(visc > 0)) return fail(SC_ERR_INVALID, "bad argument");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  double vmax = 0;
  rc = SC_DTYPE_DISPATCH(p, pack_state, p, u, p->S, st);
  if (!rc) rc = SC_DTYPE_DISPATCH(p, vmax_impl, p, p->S, &vmax, st);
  if (rc) return rc;
  const double h = p->l / p->n;
  const double dconv = h / vmax, ddiff = h * h / p->D / 2 / visc;
  *dt = dconv < ddiff ? dconv : ddiff;
  return SC_OK;
}

int sc_shell_energies(sc_plan* p, const void* const* u, double* eref, void* stream) {
  if (!p || !eref) return fail(SC_ERR_INVALID, "bad argument");
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  rc = SC_DTYPE_DISPATCH(p, pack_state, p, u, p->S, st);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, clamp_impl, p, p->S, eref, 0, st);
}

int sc_maintain_shell_energy(sc_plan* p, void* const* u, const double* eref, void* stream) {
  if (!p || !eref) return fail(SC_ERR_INVALID, "bad argument");
  int rc = check_ptrs((const void* const*)u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  double e[2] = {eref[0], eref[1]};
  rc = SC_DTYPE_DISPATCH(p, pack_state, p, (const void* const*)u, p->S, st);
  if (!rc) rc = SC_DTYPE_DISPATCH(p, clamp_impl, p, p->S, e, 1, st);
  if (!rc) rc = SC_DTYPE_DISPATCH(p, unpack_state, p, p->S, u, st);
  if (!rc) SC_CU(cudaStreamSynchronize(st));
  return rc;
}

int sc_state_maintain_shell_energy(sc_plan* p, const double* eref, void* stream) {
  if (!p || !eref) return fail(SC_ERR_INVALID, "bad argument");
  int rc = ensure_device(p);
  if (rc) return rc;
  double e[2] = {eref[0], eref[1]};
  rc = SC_DTYPE_DISPATCH(p, clamp_impl, p, p->U, e, 1, as_stream(stream));
  if (!rc) SC_CU(cudaStreamSynchronize(as_stream(stream)));
  return rc;
}

int sc_spectrum(sc_plan* p, const void* const* u, int nshell, double* s, void* stream) {
  if (!p || !s || nshell < 1) return fail(SC_ERR_INVALID, "bad argument");
  if (nshell > p->kc) return fail(SC_ERR_INVALID, "shells beyond n/3 are not retained (nshell <= %d)", p->kc);
  int rc = check_ptrs(u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  rc = SC_DTYPE_DISPATCH(p, pack_state, p, u, p->S, st);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, spectrum_impl, p, p->S, nshell, s, st);
}

int sc_les_diagnostics(sc_plan* p, sc_closure* cl, const void* const* u, const void* const* uref, double visc,
                       int nshell, double* out, double* spec, double* transfer, void* stream) {
  if (!p || !out || !spec || !transfer || nshell < 1) return fail(SC_ERR_INVALID, "bad argument");
  if (nshell > p->kc) return fail(SC_ERR_INVALID, "shells beyond n/3 are not retained (nshell <= %d)", p->kc);
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  if (cl && cl->kind == sc::kNoClosure) cl = nullptr;
  int rc = check_ptrs(u, p->D);
  if (!rc && uref) rc = check_ptrs(uref, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  auto body = [&](auto tag) -> int {
    using R = decltype(tag);
    double s = 0;
    int r = energy_impl<R>(p, u, 0, 0, &s, st);
    if (r) return r;
    out[1] = 0.5 * s;
    if ((r = energy_impl<R>(p, u, 0, 1, &s, st))) return r;
    out[2] = visc * s;
    if ((r = pack_state<R>(p, u, p->S, st))) return r;
    if ((r = spectrum_impl<R>(p, p->S, nshell, spec, st))) return r;
    // e_post and the closure terms accumulate into dscal[1..2] and a shell buffer
    double* d = nullptr;
    SC_CU(cudaMallocAsync((void**)&d, (3 + nshell) * sizeof(double), st));
    cudaMemsetAsync(d, 0, (3 + nshell) * sizeof(double), st);
    sc::DiagArgs a{};
    a.D = p->D; a.n = p->n; a.kc = p->kc; a.kfac = 2.0 * M_PI / p->l;
    for (int c = 0; c < p->D; ++c) a.u[c] = u[c];
    if (uref) {
      for (int c = 0; c < p->D; ++c) a.uref[c] = uref[c];
      sc::launch_epost<R>(a, d, st);
    }
    if (cl) {
      if ((r = products<R>(p, p->S, st))) { cudaFreeAsync(d, st); return r; }
      if ((r = closure_tauhat<R>(cl, p->S, st))) { cudaFreeAsync(d, st); return r; }
      sc::DiagArgs b = a;
      for (int c = 0; c < p->D; ++c) b.u[c] = p->S[c];
      for (int c = 0; c < (p->D == 3 ? 6 : 3); ++c) b.th[c] = cl->th[c];
      sc::launch_sfs_diag<R>(b, nshell, d + 2, d + 3, st);
    }
    r = check_launch("les diagnostics");
    std::vector<double> h(3 + nshell);
    cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    SC_CU(cudaStreamSynchronize(st));
    if (r) return r;
    out[0] = uref ? std::sqrt(h[0]) / std::sqrt(h[1]) : 0.0;
    out[3] = -h[2];
    for (int i = 0; i < nshell; ++i) transfer[i] = h[3 + i];
    return SC_OK;
  };
  return p->dtype == SC_FLOAT64 ? body(double()) : body(float());
}

size_t sc_rollout_traj_bytes(const sc_plan* p, int nsteps) {
  if (!p || nsteps < 1) return 0;
  return (size_t)nsteps * p->D * p->csz * p->esz;
}

}  // extern "C"

namespace {

// Stage derivative F(u) = P[div(stress(u) + closure)] of the compact state u into k.
template <typename R>
int stage_F(sc_plan* p, sc_closure* cl, void* const* u, void* const* k, double visc, cudaStream_t st) {
  int rc = stage_rhs<R>(p, cl, u, st);
  if (rc) return rc;
  sc::EpiArgs e = epi_base<R>(p, u, visc);
  add_closure_stress<R>(e, cl, p->D);
  e.proj_k = 1;
  for (int c = 0; c < p->D; ++c) { e.base_a[c] = nullptr; e.out_a[c] = k[c]; }
  e.ca = 1.0;
  sc::launch_epilogue<R>(e, st);
  return check_launch("stage derivative");
}

// Adjoint of one stage: mu = (dF/du)^T lam at u; parameter gradients of the
// closure accumulate into cl->gw.  Scratch: closure buffers (gp, s2, ph2, th).
template <typename R>
int stage_adjoint(sc_plan* p, sc_closure* cl, void* const* u, void* const* lam, void* const* mu, double visc,
                  cudaStream_t st) {
  const int D = p->D, NP = D == 3 ? 6 : 3;
  const long long np = phys_args(p).npts;
  const double N = double(np);
  void* const* lsig = cl->s2;  // compact [NP]
  sc::AdjSpecArgs as{};
  for (int c = 0; c < D; ++c) { as.lam[c] = lam[c]; as.u[c] = u[c]; as.mu[c] = mu[c]; }
  for (int c = 0; c < NP; ++c) as.lsig[c] = lsig[c];
  as.D = D; as.kc = p->kc; as.kfac = 2.0 * M_PI / p->l; as.visc = visc;
  sc::launch_adj_spec<R>(as, st);
  const bool tc = cl && cl->kind == sc::kCnn;
  const bool cnn = cl && (cl->kind == sc::kCnnFp || tc);
  int rc = SC_OK;
  // physical velocity of the stage (and the CNN activations) at u
  if (tc) rc = tc_forward(cl, u, st);  // v in gp[0..2]
  else if (cnn) rc = cc_forward<R>(cl, u, st);
  else rc = c2p_batch<R>(p, cl->bb, cl->cb, u, cl->gp, D, st);
  if (rc) return rc;
  // m = T(lsig) / N, physical: into the CNN tau buffer (as dL/dtau) or gp[3..]
  void* m[6];
  for (int c = 0; c < NP; ++c)
    m[c] = cnn ? (void*)(static_cast<R*>(cl->cctau) + (size_t)c * np) : cl->gp[3 + c];
  {
    // c2p with the 1/N factor folded into the x-direction c2r
    const int n = p->n, K1 = p->K1, K2 = p->K2, kc = p->kc;
    for (int c0 = 0; c0 < NP; c0 += 12) {
      const int mc = NP - c0 < 12 ? NP - c0 : 12;
      sc::ColArgs a = z_inverse_args(K1, K2, n, kc);
      for (int c = 0; c < mc; ++c) { a.in[c] = lsig[c0 + c]; a.out[c] = cl->bb[c]; }
      a.ncomp = mc;
      sc::launch_col_inv<R>(n, a, p->tw, st);
      sc::ColArgs b = y_inverse_args(K1, n, kc);
      for (int c = 0; c < mc; ++c) { b.in[c] = cl->bb[c]; b.out[c] = cl->cb[c]; }
      b.ncomp = mc;
      sc::launch_col_inv<R>(n, b, p->tw, st);
      sc::XPlainArgs x{};
      for (int c = 0; c < mc; ++c) { x.in[c] = cl->cb[c]; x.out[c] = m[c0 + c]; }
      x.ncomp = mc; x.K1 = K1; x.nrows = (long long)n * n; x.scale = 1.0 / N;
      sc::launch_x_c2r<R>(n, x, p->tw, st);
    }
    if ((rc = check_launch("adjoint stress to physical"))) return rc;
  }
  if (tc && (rc = tc_backward(cl, st))) return rc;
  if (cnn && !tc && (rc = cc_backward<R>(cl, static_cast<const R*>(cl->cctau), st))) return rc;
  sc::AdjPhysArgs ap{};
  for (int c = 0; c < D; ++c) {
    ap.v[c] = cl->gp[c];
    ap.add[c] = cnn ? (const void*)(static_cast<R*>(cl->ccg0) + (size_t)c * np) : nullptr;
    ap.lv[c] = cl->ph2[c];
  }
  for (int c = 0; c < NP; ++c) ap.m[c] = m[c];
  ap.D = D; ap.npts = np; ap.inv_npts = 1.0;
  sc::launch_adj_products<R>(ap, st);
  if ((rc = p2c_batch<R>(p, cl->bb, cl->cb, cl->ph2, cl->th, D, st))) return rc;
  sc::AdjAccArgs aa{};
  for (int c = 0; c < D; ++c) { aa.mu[c] = mu[c]; aa.x[c] = cl->th[c]; aa.u[c] = u[c]; }
  aa.lamz = cnn ? cl->dsum + 1 : nullptr;
  aa.a2 = cl->dsum;
  aa.sigma = cnn ? cl->sigma : 1.0;
  aa.scale = N; aa.kfac = 2.0 * M_PI / p->l; aa.D = D; aa.kc = p->kc;
  sc::launch_adj_acc<R>(aa, st);
  return check_launch("stage adjoint");
}

struct RolloutBufs {
  std::vector<void*> all;
  void* u[4][3];   // stage inputs
  void* k[3];      // stage derivative scratch
  void* lam[3], *lk[3], *mu[3];
  void* ck = nullptr;  // checkpoints
  void* seg = nullptr; // segment states
  double* dloss = nullptr;
};

template <typename R>
int rollout_impl(sc_plan* p, sc_closure* cl, const void* const* u0, const void* traj, double dt, double visc,
                 int nsteps, int ck, double* loss, double* grad, void* rec, cudaStream_t st) {
  const int D = p->D;
  const size_t cbytes = p->csz * p->esz;  // one compact component
  const size_t sbytes = D * cbytes;       // one compact state
  RolloutBufs B{};
  auto A = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMallocAsync(ptr, bytes, st);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(SC_ERR_OOM, "rollout scratch: %s", cudaGetErrorString(e)); }
    B.all.push_back(*ptr);
    return SC_OK;
  };
  auto freeall = [&]() { for (void* a : B.all) cudaFreeAsync(a, st); };
  // a CUDA error in the body frees the rollout buffers before it returns
#define SC_CU_FREE(call)                                                                     \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      freeall();                                                                             \
      return fail(SC_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));                     \
    }                                                                                        \
  } while (0)
  int rc = SC_OK;
  const bool adj = grad != nullptr;
  const int nck = adj ? nsteps / ck + 1 : 0;
  for (int s_ = 0; s_ < 4 && !rc; ++s_)
    for (int c = 0; c < D && !rc; ++c) rc = A(&B.u[s_][c], cbytes);
  for (int c = 0; c < D && !rc; ++c) {
    rc = A(&B.k[c], cbytes);
    if (!rc) rc = A(&B.lam[c], cbytes);
    if (!rc) rc = A(&B.lk[c], cbytes);
    if (!rc) rc = A(&B.mu[c], cbytes);
  }
  if (!rc && adj) rc = A(&B.ck, nck * sbytes);
  // the working state lives in segment slot 0 in every mode
  if (!rc) rc = A(&B.seg, (adj ? ck + 1 : 1) * sbytes);
  if (!rc) rc = A((void**)&B.dloss, 2 * sizeof(double));  // [loss, scratch]
  if (rc) { freeall(); return rc; }
  auto state_ptrs = [&](void* base, long long idx, void** out3) {
    for (int c = 0; c < D; ++c) out3[c] = static_cast<char*>(base) + (size_t)idx * sbytes + c * cbytes;
  };
  auto traj_ptrs = [&](int step, const void** out3) {  // target after `step` steps (1-based)
    for (int c = 0; c < D; ++c)
      out3[c] = static_cast<const char*>(traj) + (size_t)(step - 1) * sbytes + c * cbytes;
  };
  // one RK4 step of the state in x (in place) using B.u / B.k
  auto step = [&](void* const* x) -> int {
    const long long nm = (long long)p->csz;
    for (int c = 0; c < D; ++c) SC_CU(cudaMemcpyAsync(B.u[0][c], x[c], cbytes, cudaMemcpyDeviceToDevice, st));
    static const double cst[3] = {0.5, 0.5, 1.0};
    static const double w[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
    for (int s_ = 0; s_ < 4; ++s_) {
      int r = stage_F<R>(p, cl, B.u[s_], B.k, visc, st);
      if (r) return r;
      sc::launch_axpby<R>(x, (const void* const*)B.k, w[s_] * dt, 1.0, D, nm, st);  // x += w dt k
      if (s_ < 3) {
        for (int c = 0; c < D; ++c) SC_CU(cudaMemcpyAsync(B.u[s_ + 1][c], B.u[0][c], cbytes, cudaMemcpyDeviceToDevice, st));
        sc::launch_axpby<R>(B.u[s_ + 1], (const void* const*)B.k, cst[s_] * dt, 1.0, D, nm, st);
      }
    }
    return check_launch("rollout step");
  };
  // forward rollout: loss, checkpoints / trajectory record
  void* x[3];
  state_ptrs(B.seg, 0, x);
  if ((rc = pack_state<R>(p, u0, x, st))) { freeall(); return rc; }
  SC_CU_FREE(cudaMemsetAsync(B.dloss, 0, sizeof(double), st));
  if (adj) SC_CU_FREE(cudaMemcpyAsync(B.ck, x[0], sbytes, cudaMemcpyDeviceToDevice, st));
  for (int s_ = 1; s_ <= nsteps && !rc; ++s_) {
    rc = step(x);
    if (rc) break;
    if (rec) SC_CU_FREE(cudaMemcpyAsync(static_cast<char*>(rec) + (size_t)(s_ - 1) * sbytes, x[0], sbytes,
                                   cudaMemcpyDeviceToDevice, st));
    if (traj) {
      const void* t3[3];
      traj_ptrs(s_, t3);
      sc::launch_mse<R>((const void* const*)x, t3, nullptr, 0.0, D, p->kc, B.dloss, st);
    }
    if (adj && s_ % ck == 0)
      SC_CU_FREE(cudaMemcpyAsync(static_cast<char*>(B.ck) + (size_t)(s_ / ck) * sbytes, x[0], sbytes,
                            cudaMemcpyDeviceToDevice, st));
  }
  if (!rc && adj) {
    SC_CU_FREE(cudaMemsetAsync(cl ? (void*)cl->gw : nullptr, 0, cl ? cl->nparam * sizeof(double) : 0, st));
    sc::launch_axpby<R>(B.lam, nullptr, 0.0, 0.0, D, (long long)p->csz, st);  // lam = 0
    const double coef = 2.0 / nsteps;
    for (int seg = (nsteps - 1) / ck; seg >= 0 && !rc; --seg) {
      const int c0 = seg * ck, c1 = std::min(nsteps, c0 + ck);
      // recompute u_{c0} .. u_{c1} into the segment buffer
      SC_CU_FREE(cudaMemcpyAsync(B.seg, static_cast<char*>(B.ck) + (size_t)seg * sbytes, sbytes, cudaMemcpyDeviceToDevice, st));
      for (int s_ = c0 + 1; s_ <= c1 && !rc; ++s_) {
        void* xs[3];
        state_ptrs(B.seg, s_ - c0, xs);
        SC_CU_FREE(cudaMemcpyAsync(xs[0], static_cast<char*>(B.seg) + (size_t)(s_ - c0 - 1) * sbytes, sbytes,
                              cudaMemcpyDeviceToDevice, st));
        rc = step(xs);
      }
      for (int s_ = c1; s_ > c0 && !rc; --s_) {
        void* us[3];
        state_ptrs(B.seg, s_ - c0, us);
        const void* t3[3];
        traj_ptrs(s_, t3);
        // lam += dL/du_s = coef (u_s - u*_s)
        sc::launch_mse<R>((const void* const*)us, t3, B.mu, coef, D, p->kc, B.dloss + 1, st);
        sc::launch_axpby<R>(B.lam, (const void* const*)B.mu, 1.0, 1.0, D, (long long)p->csz, st);
        // step adjoint at u_{s-1}: recompute the stage inputs, then transpose stages 4..1
        void* un[3];
        state_ptrs(B.seg, s_ - c0 - 1, un);
        for (int c = 0; c < D; ++c) SC_CU_FREE(cudaMemcpyAsync(B.u[0][c], un[c], cbytes, cudaMemcpyDeviceToDevice, st));
        static const double cst[3] = {0.5, 0.5, 1.0};
        for (int q = 0; q < 3 && !rc; ++q) {
          rc = stage_F<R>(p, cl, B.u[q], B.k, visc, st);
          if (rc) break;
          for (int c = 0; c < D; ++c) SC_CU_FREE(cudaMemcpyAsync(B.u[q + 1][c], B.u[0][c], cbytes, cudaMemcpyDeviceToDevice, st));
          sc::launch_axpby<R>(B.u[q + 1], (const void* const*)B.k, cst[q] * dt, 1.0, D, (long long)p->csz, st);
        }
        if (rc) break;
        // lam_n accumulates in B.lam (identity part already there)
        static const double wq[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
        // lk = w4 dt lam
        for (int c = 0; c < D; ++c) SC_CU_FREE(cudaMemcpyAsync(B.lk[c], B.lam[c], cbytes, cudaMemcpyDeviceToDevice, st));
        sc::launch_axpby<R>(B.lk, nullptr, 0.0, wq[3] * dt, D, (long long)p->csz, st);
        // keep a copy of lam (dL/du_{n+1}) in B.k for the stage combinations
        for (int c = 0; c < D; ++c) SC_CU_FREE(cudaMemcpyAsync(B.k[c], B.lam[c], cbytes, cudaMemcpyDeviceToDevice, st));
        for (int q = 3; q >= 0 && !rc; --q) {
          rc = stage_adjoint<R>(p, cl, B.u[q], B.lk, B.mu, visc, st);
          if (rc) break;
          sc::launch_axpby<R>(B.lam, (const void* const*)B.mu, 1.0, 1.0, D, (long long)p->csz, st);  // lam_n += mu
          if (q > 0) {
            // lk_{q-1} = w_{q-1} dt lam_{n+1} + c_{q-1} dt mu
            for (int c = 0; c < D; ++c) SC_CU_FREE(cudaMemcpyAsync(B.lk[c], B.k[c], cbytes, cudaMemcpyDeviceToDevice, st));
            sc::launch_axpby<R>(B.lk, (const void* const*)B.mu, cst[q - 1] * dt, wq[q - 1] * dt, D,
                                (long long)p->csz, st);
          }
        }
      }
    }
  }
  double h = 0;
  if (!rc) {
    SC_CU_FREE(cudaMemcpyAsync(&h, B.dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (adj && cl && cl->gw) SC_CU_FREE(cudaMemcpyAsync(grad, cl->gw, cl->nparam * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  freeall();
  SC_CU(cudaStreamSynchronize(st));
  if (loss) *loss = traj ? h / nsteps : 0.0;
  return rc;
}
#undef SC_CU_FREE
}  // namespace

extern "C" {

int sc_rollout_record(sc_plan* p, sc_closure* cl, const void* const* u0, double dt, double visc, int nsteps,
                      void* traj, void* stream) {
  if (!p || !traj || nsteps < 1) return fail(SC_ERR_INVALID, "bad argument");
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  int rc = check_ptrs(u0, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, rollout_impl, p, cl, u0, nullptr, dt, visc, nsteps, 1, nullptr, nullptr, traj,
                           as_stream(stream));
}

int sc_rollout_loss(sc_plan* p, sc_closure* cl, const void* const* u0, const void* traj, double dt, double visc,
                    int nsteps, double* loss, void* stream) {
  if (!p || !traj || !loss || nsteps < 1) return fail(SC_ERR_INVALID, "bad argument");
  if (cl && cl->p != p) return fail(SC_ERR_INVALID, "closure belongs to another plan");
  int rc = check_ptrs(u0, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, rollout_impl, p, cl, u0, traj, dt, visc, nsteps, 1, loss, nullptr, nullptr,
                           as_stream(stream));
}

int sc_rollout_adjoint(sc_plan* p, sc_closure* cl, const void* const* u0, const void* traj, double dt, double visc,
                       int nsteps, int ckpt_every, double* loss, double* grad, void* stream) {
  if (!p || !traj || !grad || nsteps < 1 || ckpt_every < 1) return fail(SC_ERR_INVALID, "bad argument");
  if (!cl || cl->p != p || (cl->kind != sc::kCnnFp && cl->kind != sc::kCnn))
    return fail(SC_ERR_INVALID, "the adjoint needs a CNN closure of this plan");
  int rc = check_ptrs(u0, p->D);
  if (!rc) rc = ensure_device(p);
  if (!rc && cl->kind == sc::kCnn) rc = tc_adjoint_buffers(cl);
  if (rc) return rc;
  return SC_DTYPE_DISPATCH(p, rollout_impl, p, cl, u0, traj, dt, visc, nsteps, ckpt_every, loss, grad, nullptr,
                           as_stream(stream));
}

int sc_rollout_adjoint_batch(int njobs, const sc_rollout_job* jobs, int* status, void* stream) {
  if (njobs < 1 || !jobs || !status) return fail(SC_ERR_INVALID, "bad argument");
  for (int i = 0; i < njobs; ++i)
    for (int j = 0; j < i; ++j)
      if (jobs[i].plan == jobs[j].plan || jobs[i].closure == jobs[j].closure)
        return fail(SC_ERR_INVALID, "jobs %d and %d share a plan or closure", j, i);
  // jobs start after the work already on the caller's stream
  cudaEvent_t ready;
  SC_CU(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  SC_CU(cudaEventRecord(ready, as_stream(stream)));
  std::vector<std::string> errs(njobs);
  auto run = [&](int i) {
    const sc_rollout_job& J = jobs[i];
    cudaStream_t js = nullptr;
    int rc = J.plan ? ensure_device(J.plan) : fail(SC_ERR_INVALID, "null plan");
    if (!rc && cudaStreamCreateWithFlags(&js, cudaStreamNonBlocking) != cudaSuccess)
      rc = fail(SC_ERR_CUDA, "cudaStreamCreateWithFlags failed");
    if (!rc && cudaStreamWaitEvent(js, ready, 0) != cudaSuccess) rc = fail(SC_ERR_CUDA, "cudaStreamWaitEvent failed");
    if (!rc)
      rc = sc_rollout_adjoint(J.plan, J.closure, J.u0, J.traj, J.dt, J.visc, J.nsteps, J.ckpt_every, J.loss, J.grad,
                              js);
    if (js) cudaStreamDestroy(js);
    status[i] = rc;
    if (rc) errs[i] = g_err;  // the error text is per host thread
  };
  std::vector<std::thread> th;
  th.reserve(njobs - 1);
  for (int i = 1; i < njobs; ++i) th.emplace_back(run, i);
  run(0);
  for (auto& t : th) t.join();
  cudaEventDestroy(ready);
  for (int i = 0; i < njobs; ++i)
    if (status[i]) return fail(status[i], "job %d: %s", i, errs[i].c_str());
  return SC_OK;
}

int sc_plan_num_variants(const sc_plan* p, int sweep, int* count) {
  if (!p || !count || sweep < 0 || sweep > 4) return fail(SC_ERR_INVALID, "bad argument");
  *count = 1;
  if (p->dtype != SC_FLOAT32 || !sc::fast_supported(p->n)) return SC_OK;
  if (p->D != 3) return SC_OK;
  *count = sweep == 2 ? sc::xsweep_variants(p->n, p->D) : sc::col2_variants(p->n);
  // the z inverse reads the compact cube, whose rows (271 complex at 810^3)
  // are not 16-byte strided: no TMA-fed variants
  if (sweep == 0 && p->n == 810) *count -= sc::kColTmaConfigs;
  return SC_OK;
}

int sc_plan_set_option(sc_plan* p, int option, long long value) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (option == SC_OPT_USE_GRAPH) { p->use_graph = value ? 1 : 0; return SC_OK; }
  if (option == SC_OPT_WAIT_LIMIT) {
    p->wait_limit = value < 0 ? sc::kDefaultWaitLimit : value;
    // the plan's own step graphs carry the bound of their column sweeps
    if (p->g_rk4) { cudaGraphExecDestroy(p->g_rk4); p->g_rk4 = nullptr; }
    if (p->g_wray) { cudaGraphExecDestroy(p->g_wray); p->g_wray = nullptr; }
    return SC_OK;
  }
  if (option >= SC_OPT_VARIANT_ZINV && option <= SC_OPT_VARIANT_ZFWD) {
    const int sweep = option - SC_OPT_VARIANT_ZINV;
    int nv = 0;
    sc_plan_num_variants(p, sweep, &nv);
    if (value < 0 || value >= nv) return fail(SC_ERR_INVALID, "sweep %d has %d variants", sweep, nv);
    p->variant[sweep] = int(value);
    // cached step graphs hold the old launches
    if (p->g_rk4) { cudaGraphExecDestroy(p->g_rk4); p->g_rk4 = nullptr; }
    if (p->g_wray) { cudaGraphExecDestroy(p->g_wray); p->g_wray = nullptr; }
    return SC_OK;
  }
  return fail(SC_ERR_INVALID, "unknown option %d", option);
}

}  // extern "C"

namespace {
__global__ void k_guard(const double* e, int* status, int n, double limit) {
  const int i = threadIdx.x;
  if (i < n) {
    const double v = e[i];
    if (!(v <= limit)) status[i] = SC_ERR_DIVERGED;  // also catches NaN
  }
}

// Record stride of one instance's snapshot: ke, eps_visc, eps_sfs, spectrum
// (nshell shells), shell transfer (nshell shells).
int snap_stride(int nshell) { return 3 + 2 * nshell; }

// The per-instance reductions of one snapshot into b->scratch, on the
// instance's stream (the quantities of sc_les_diagnostics, src/les.jl:94-148,
// without e_post, which needs a reference trajectory).
template <typename R>
int snapshot_reductions(sc_les_batch* b, int i, cudaStream_t st) {
  const sc_les_instance& in = b->inst[i];
  sc_plan* p = in.plan;
  const int stride = snap_stride(b->nshell);
  double* d = b->scratch + (size_t)i * stride;
  cudaMemsetAsync(d, 0, stride * sizeof(double), st);
  const double kfac = 2.0 * M_PI / p->l;
  sc::launch_spectral_energy<R>((const void* const*)p->U, p->D, p->D, p->n, p->K1, p->K2, 1, p->kc, kfac, 0, d, st);
  sc::launch_spectral_energy<R>((const void* const*)p->U, p->D, p->D, p->n, p->K1, p->K2, 1, p->kc, kfac, 1, d + 1,
                                st);
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) a.src[c] = p->U[c];
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  sc::launch_spectrum<R>(a, b->nshell, d + 3, st);
  sc_closure* cl = in.closure && in.closure->kind != sc::kNoClosure ? in.closure : nullptr;
  if (cl) {
    int rc = products<R>(p, p->U, st);
    if (!rc) rc = closure_tauhat<R>(cl, p->U, st);
    if (rc) return rc;
    sc::DiagArgs g{};
    g.D = p->D; g.n = p->n; g.kc = p->kc; g.kfac = kfac;
    for (int c = 0; c < p->D; ++c) g.u[c] = p->U[c];
    for (int c = 0; c < (p->D == 3 ? 6 : 3); ++c) g.th[c] = cl->th[c];
    sc::launch_sfs_diag<R>(g, b->nshell, d + 2, d + 3 + b->nshell, st);
  }
  return check_launch("snapshot reductions");
}

// Append the snapshot scratch to the record (ke = sum/2, eps_visc = visc sum,
// eps_sfs sign as sc_les_diagnostics) at the device counter, then count it.
__global__ void k_snap_append(const double* scratch, double* snaps, int* count, const double* visc, int ninst,
                              int stride, int max_snap) {
  const int c = *count;
  if (c < max_snap) {
    for (int j = threadIdx.x; j < ninst * stride; j += blockDim.x) {
      const int i = j / stride, q = j - i * stride;
      double v = scratch[j];
      if (q == 0) v *= 0.5;
      else if (q == 1) v *= visc[i];
      else if (q == 2) v = -v;
      snaps[(size_t)c * ninst * stride + j] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && c < max_snap) *count = c + 1;
}

int batch_capture_one(sc_les_batch* b, bool snapshot, cudaGraphExec_t* out);

int batch_capture(sc_les_batch* b) {
  int rc = batch_capture_one(b, false, &b->graph);
  if (!rc && b->snap_every > 0) rc = batch_capture_one(b, true, &b->snap_graph);
  return rc;
}

int batch_capture_one(sc_les_batch* b, bool snapshot, cudaGraphExec_t* out) {
  if (*out) { cudaGraphExecDestroy(*out); *out = nullptr; }
  const int ni = (int)b->inst.size();
  cudaGraph_t g;
  SC_CU(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
  int rc = SC_OK;
  cudaEventRecord(b->fork, b->origin);
  for (int i = 0; i < ni && !rc; ++i) {
    if (!b->active[i]) continue;
    const sc_les_instance& in = b->inst[i];
    cudaStreamWaitEvent(b->streams[i], b->fork, 0);
    sc_forcing f{in.forced, in.eps};
    rc = in.plan->dtype == SC_FLOAT64
             ? rk4_step<double>(in.plan, in.dt, in.visc, &f, b->streams[i], in.closure)
             : rk4_step<float>(in.plan, in.dt, in.visc, &f, b->streams[i], in.closure);
    if (rc) break;
    cudaMemsetAsync(b->energy + i, 0, sizeof(double), b->streams[i]);
    sc_plan* p = in.plan;
    if (p->dtype == SC_FLOAT64)
      sc::launch_spectral_energy<double>((const void* const*)p->U, p->D, p->D, p->n, p->K1, p->K2, 1, p->kc,
                                         2.0 * M_PI / p->l, 0, b->energy + i, b->streams[i]);
    else
      sc::launch_spectral_energy<float>((const void* const*)p->U, p->D, p->D, p->n, p->K1, p->K2, 1, p->kc,
                                        2.0 * M_PI / p->l, 0, b->energy + i, b->streams[i]);
    if (snapshot)
      rc = p->dtype == SC_FLOAT64 ? snapshot_reductions<double>(b, i, b->streams[i])
                                  : snapshot_reductions<float>(b, i, b->streams[i]);
    cudaEventRecord(b->events[i], b->streams[i]);
    cudaStreamWaitEvent(b->origin, b->events[i], 0);
  }
  // energy is accumulated as sum |u|^2 (RFFT weights); the guard limit is 2 * 1e5
  k_guard<<<1, 256, 0, b->origin>>>(b->energy, b->status, ni, 2.0e5);
  if (snapshot)
    k_snap_append<<<1, 256, 0, b->origin>>>(b->scratch, b->snaps, b->dcount, b->scratch + (size_t)ni * snap_stride(b->nshell),
                                            ni, snap_stride(b->nshell), b->max_snap);
  cudaError_t e = cudaStreamEndCapture(b->origin, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(SC_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { *out = nullptr; return fail(SC_ERR_CUDA, "batch instantiate: %s", cudaGetErrorString(e)); }
  return SC_OK;
}

void snap_free(sc_les_batch* b) {
  if (b->snap_graph) cudaGraphExecDestroy(b->snap_graph);
  if (b->scratch) cudaFree(b->scratch);
  if (b->snaps) cudaFree(b->snaps);
  if (b->dcount) cudaFree(b->dcount);
  b->snap_graph = nullptr; b->scratch = nullptr; b->snaps = nullptr; b->dcount = nullptr;
  b->snap_every = b->nshell = b->max_snap = b->nsnap = 0;
  b->steps_done = 0;
}

void batch_free(sc_les_batch* b) {
  snap_free(b);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (auto s : b->streams) cudaStreamDestroy(s);
  for (auto e : b->events) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  if (b->energy) cudaFree(b->energy);
  if (b->status) cudaFree(b->status);
}
}  // namespace

extern "C" {

int sc_les_batch_create(sc_les_batch** out, const sc_les_instance* inst, int ninst) {
  if (!out || !inst || ninst < 1 || ninst > 256) return fail(SC_ERR_INVALID, "bad argument");
  *out = nullptr;
  int dev = inst[0].plan ? inst[0].plan->dev : 0;
  for (int i = 0; i < ninst; ++i) {
    if (!inst[i].plan) return fail(SC_ERR_INVALID, "instance %d has no plan", i);
    if (inst[i].plan->dev != dev) return fail(SC_ERR_INVALID, "instances must share one device");
    if (inst[i].closure && inst[i].closure->p != inst[i].plan)
      return fail(SC_ERR_INVALID, "instance %d: closure belongs to another plan", i);
    for (int j = 0; j < i; ++j)
      if (inst[j].plan == inst[i].plan) return fail(SC_ERR_INVALID, "instances %d and %d share a plan", j, i);
  }
  SC_CU(cudaSetDevice(dev));
  sc_les_batch* b = new sc_les_batch();
  b->inst.assign(inst, inst + ninst);
  b->active.assign(ninst, 1);
  b->dev = dev;
  int rc = SC_OK;
  if (cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc((void**)&b->energy, ninst * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&b->status, ninst * sizeof(int)) != cudaSuccess)
    rc = fail(SC_ERR_CUDA, "batch resources");
  for (int i = 0; i < ninst && !rc; ++i) {
    cudaStream_t s;
    cudaEvent_t e;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      rc = fail(SC_ERR_CUDA, "batch streams");
      break;
    }
    b->streams.push_back(s);
    b->events.push_back(e);
  }
  if (!rc && cudaMemset(b->status, 0, ninst * sizeof(int)) != cudaSuccess) rc = fail(SC_ERR_CUDA, "memset");
  if (!rc) rc = batch_capture(b);
  if (rc) { batch_free(b); delete b; return rc; }
  *out = b;
  return SC_OK;
}

int sc_les_batch_run(sc_les_batch* b, int nsteps, void* stream) {
  if (!b || nsteps < 0) return fail(SC_ERR_INVALID, "bad argument");
  SC_CU(cudaSetDevice(b->dev));
  for (int i = 0; i < nsteps; ++i) {
    ++b->steps_done;
    const bool snap = b->snap_every > 0 && b->steps_done % b->snap_every == 0 && b->nsnap < b->max_snap;
    SC_CU(cudaGraphLaunch(snap ? b->snap_graph : b->graph, as_stream(stream)));
    if (snap) ++b->nsnap;
  }
  return SC_OK;
}

int sc_random_field(sc_plan* p, unsigned long long seed, const void* const* draws, double kpeak, double totalenergy,
                    void* const* u_hat, void* stream) {
  if (!p || !(kpeak > 0) || !(totalenergy >= 0)) return fail(SC_ERR_INVALID, "bad argument");
  if (draws) {
    int rc = check_ptrs(draws, p->D);
    if (rc) return rc;
  }
  if (u_hat) {
    int rc = check_ptrs((const void* const*)u_hat, p->D);
    if (rc) return rc;
  }
  int rc = ensure_device(p);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const int D = p->D, n = p->n;
  // peak_profile(k, kpeak) = k^4 exp(-2 (k / kpeak)^2) on shells 0 .. floor(sqrt(D) n / 2)
  const int smax = int(std::floor(std::sqrt(double(D)) * (n / 2)));
  std::vector<double> target(smax + 1);
  double tot = 0;
  for (int s_ = 0; s_ <= smax; ++s_) {
    const double k = s_;
    target[s_] = k * k * k * k * std::exp(-2.0 * (k / kpeak) * (k / kpeak));
    tot += target[s_];
  }
  for (double& v : target) v = tot > 0 ? totalenergy * v / tot : 0.0;
  const size_t cb = p->csz * 16;  // one FP64 compact component
  void* w[3] = {nullptr, nullptr, nullptr};
  double* dbuf = nullptr;  // [eshell (smax + 1) | target (smax + 1)]
  auto release = [&]() {
    for (int c = 0; c < 3; ++c)
      if (w[c]) cudaFreeAsync(w[c], st);
    if (dbuf) cudaFreeAsync(dbuf, st);
  };
  for (int c = 0; c < D; ++c)
    if (cudaMallocAsync(&w[c], cb, st) != cudaSuccess) { cudaGetLastError(); release(); return fail(SC_ERR_OOM, "randomfield scratch"); }
  if (cudaMallocAsync((void**)&dbuf, 2 * (smax + 1) * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    release();
    return fail(SC_ERR_OOM, "randomfield scratch");
  }
  cudaError_t e = cudaMemsetAsync(dbuf, 0, (smax + 1) * sizeof(double), st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dbuf + smax + 1, target.data(), (smax + 1) * sizeof(double), cudaMemcpyHostToDevice, st);
  for (int c = 0; c < D && e == cudaSuccess; ++c)
    if (draws) e = cudaMemcpyAsync(w[c], draws[c], cb, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) { release(); return fail(SC_ERR_CUDA, "randomfield: %s", cudaGetErrorString(e)); }
  if (!draws) sc::launch_random_draws(w, D, p->K1, p->kc, seed, st);
  if (p->dtype == SC_FLOAT64)
    sc::launch_random_finish<double>(w, p->U, D, n, p->K1, p->kc, dbuf, dbuf + smax + 1, st);
  else
    sc::launch_random_finish<float>(w, p->U, D, n, p->K1, p->kc, dbuf, dbuf + smax + 1, st);
  rc = check_launch("randomfield");
  if (!rc && u_hat) rc = SC_DTYPE_DISPATCH(p, unpack_state, p, p->U, u_hat, st);
  release();
  e = cudaStreamSynchronize(st);  // the host target array is read by the copy above
  if (!rc && e != cudaSuccess) rc = fail(SC_ERR_CUDA, "randomfield: %s", cudaGetErrorString(e));
  return rc;
}

int sc_les_batch_set_snapshots(sc_les_batch* b, int every, int nshell, int max_snap) {
  if (!b || every < 0 || (every > 0 && (nshell < 1 || max_snap < 1))) return fail(SC_ERR_INVALID, "bad argument");
  for (const sc_les_instance& in : b->inst)
    if (every > 0 && nshell > in.plan->kc)
      return fail(SC_ERR_INVALID, "shells beyond n/3 are not retained (nshell <= %d)", in.plan->kc);
  SC_CU(cudaSetDevice(b->dev));
  snap_free(b);
  if (every == 0) return SC_OK;
  const int ni = (int)b->inst.size();
  const size_t stride = snap_stride(nshell);
  b->snap_every = every; b->nshell = nshell; b->max_snap = max_snap;
  // scratch: [ninst][stride] reductions, then [ninst] viscosities
  if (cudaMalloc((void**)&b->scratch, (ni * stride + ni) * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&b->snaps, (size_t)max_snap * ni * stride * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&b->dcount, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    snap_free(b);
    return fail(SC_ERR_OOM, "snapshot record");
  }
  std::vector<double> visc(ni);
  for (int i = 0; i < ni; ++i) visc[i] = b->inst[i].visc;
  SC_CU(cudaMemcpy(b->scratch + ni * stride, visc.data(), ni * sizeof(double), cudaMemcpyHostToDevice));
  SC_CU(cudaMemset(b->dcount, 0, sizeof(int)));
  SC_CU(cudaMemset(b->snaps, 0, (size_t)max_snap * ni * stride * sizeof(double)));
  int rc = batch_capture_one(b, true, &b->snap_graph);
  if (rc) snap_free(b);
  return rc;
}

int sc_les_batch_snapshots(sc_les_batch* b, int* nsnap, double* out, void* stream) {
  if (!b || !nsnap) return fail(SC_ERR_INVALID, "bad argument");
  *nsnap = b->nsnap;
  if (!out || b->nsnap == 0) return SC_OK;
  SC_CU(cudaSetDevice(b->dev));
  const size_t n = (size_t)b->nsnap * b->inst.size() * snap_stride(b->nshell);
  SC_CU(cudaMemcpyAsync(out, b->snaps, n * sizeof(double), cudaMemcpyDeviceToHost, as_stream(stream)));
  SC_CU(cudaStreamSynchronize(as_stream(stream)));
  return SC_OK;
}

int sc_les_batch_status(sc_les_batch* b, int* status, double* energy, int freeze, void* stream) {
  if (!b || !status) return fail(SC_ERR_INVALID, "bad argument");
  SC_CU(cudaSetDevice(b->dev));
  const int ni = (int)b->inst.size();
  std::vector<double> e(ni);
  SC_CU(cudaMemcpyAsync(status, b->status, ni * sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream)));
  SC_CU(cudaMemcpyAsync(e.data(), b->energy, ni * sizeof(double), cudaMemcpyDeviceToHost, as_stream(stream)));
  SC_CU(cudaStreamSynchronize(as_stream(stream)));
  if (energy)
    for (int i = 0; i < ni; ++i) energy[i] = 0.5 * e[i];
  if (freeze) {
    bool changed = false;
    for (int i = 0; i < ni; ++i)
      if (status[i] != 0 && b->active[i]) { b->active[i] = 0; changed = true; }
    if (changed) return batch_capture(b);
  }
  return SC_OK;
}

int sc_les_batch_destroy(sc_les_batch* b) {
  if (!b) return SC_OK;
  cudaSetDevice(b->dev);
  batch_free(b);
  delete b;
  return SC_OK;
}

int sc_twothirds(sc_plan* p, void* const* f, int ncomp, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  if (ncomp < 1 || ncomp > sc::kMaxComp) return fail(SC_ERR_INVALID, "ncomp must be 1..%d", sc::kMaxComp);
  int rc = check_ptrs((const void* const*)f, ncomp);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  sc::PackArgs a{};
  for (int c = 0; c < ncomp; ++c) a.dst[c] = f[c];
  a.ncomp = ncomp; a.D = p->D; a.n = p->n; a.kc = p->kc;
  if (p->dtype == SC_FLOAT64) sc::launch_twothirds_full<double>(a, as_stream(stream));
  else sc::launch_twothirds_full<float>(a, as_stream(stream));
  return check_launch("twothirds");
}

int sc_project(sc_plan* p, void* const* u, void* stream) {
  if (!p) return fail(SC_ERR_INVALID, "null plan");
  int rc = check_ptrs((const void* const*)u, p->D);
  if (!rc) rc = ensure_device(p);
  if (rc) return rc;
  sc::PackArgs a{};
  for (int c = 0; c < p->D; ++c) a.dst[c] = u[c];
  a.ncomp = p->D; a.D = p->D; a.n = p->n; a.kc = p->kc;
  if (p->dtype == SC_FLOAT64) sc::launch_project_full<double>(a, 2.0 * M_PI / p->l, as_stream(stream));
  else sc::launch_project_full<float>(a, 2.0 * M_PI / p->l, as_stream(stream));
  return check_launch("project");
}

}  // extern "C"
