/*
 * symcode.h -- C ABI of the B200 (sm_100a) pseudo-spectral Navier-Stokes hot
 * path of SymmetryCode.jl.
 *
 * Every entry point replaces one call of the reference's Julia solver/closure
 * API (cited per function as file:line of the reference project) and is what
 * a Julia `ccall` shim binds (see symmetrycode.jl_b200/julia/SymCodeB200.jl).
 *
 * Conventions (identical to the reference's arrays):
 *  - A spectral scalar field is a contiguous array of interleaved complex
 *    numbers (re, im) of the plan's precision, shape (n/2+1, n[, n]) in
 *    column-major order (x fastest, x is the halved RFFT axis): the element
 *    with integer wavenumber index (ix, iy, iz) (0-based) is at linear index
 *    ix + (n/2+1) * (iy + n * iz).  `Complex{Float32/Float64}` CuArrays have
 *    exactly this layout.
 *  - A vector field is passed as an array of D device pointers (x, y[, z]);
 *    a symmetric tensor field as 3 (2D) or 6 (3D) pointers in the order
 *    xx, yy[, zz], xy[, yz, zx]; a velocity-gradient field as D*D pointers in
 *    the order xx, yx, zx, xy, yy, zy, xz, yz, zz (G_ab = d u_a / d x_b).
 *  - A physical scalar field is a real array of shape (n, n[, n]), x fastest.
 *  - Normalisation: u_hat = F[u] / n^D (src/solver.jl:204-215).
 *  - All pointers are device pointers unless stated otherwise; `stream` is a
 *    cudaStream_t (NULL = legacy default stream).  Calls are stream-ordered and
 *    asynchronous unless documented as synchronous.
 *  - Every call returns an sc_status; on error sc_last_error_string() (per
 *    thread) describes it.  No exception crosses the ABI.
 *  - A plan is not thread-safe: use one plan per stream/thread.
 */
#ifndef SYMCODE_H
#define SYMCODE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_ABI_VERSION 1

#if defined(__GNUC__)
#define SC_API __attribute__((visibility("default")))
#else
#define SC_API
#endif

typedef struct sc_plan sc_plan;

typedef enum sc_dtype { SC_FLOAT32 = 0, SC_FLOAT64 = 1 } sc_dtype;

typedef enum sc_status {
  SC_OK = 0,
  SC_ERR_INVALID = 1,      /* bad argument (null pointer, D not 2/3, ...) */
  SC_ERR_SIZE = 2,         /* n odd or not 2^a 3^b 5^c in the supported set */
  SC_ERR_CUDA = 3,         /* CUDA runtime error */
  SC_ERR_OOM = 4,          /* device allocation failed */
  SC_ERR_DIVERGED = 5,     /* blow-up guard tripped (energy > limit or non-finite) */
  SC_ERR_UNSUPPORTED = 6,  /* valid request outside what this build implements */
  SC_ERR_TIMEOUT = 7       /* a bounded device-side wait ran out (kernel returned early) */
} sc_status;

/* Linear band forcing of the RK4 stepper: f_hat = A u_hat on 1 <= |k|^2 < 9
 * (shells 1 and 2, the shells the reference clamps in maintain_shell_energy!,
 * src/solver.jl:1146-1152, src/data.jl:49,65) with A = eps / (2 E_band)
 * recomputed from every stage input in FP64, so energy enters at rate eps. */
typedef struct sc_forcing {
  int enabled;
  double eps;
} sc_forcing;

/* ---- library ------------------------------------------------------------ */
SC_API int sc_abi_version(void);
SC_API const char* sc_last_error_string(void);
/* 1 if n is a grid size this build has FFT kernels for (even, 2^a 3^b 5^c). */
SC_API int sc_fft_size_supported(int n);

/* ---- plan: Grid{D}(; l, n) + getcache(grid) ------------------------------
 * Replaces `Grid{D}(; l, n, backend)` (src/solver.jl:131-151) together with
 * `getcache(grid)` (src/solver.jl:956-965) and the cuFFT plan of `getplan`
 * (src/solver.jl:432).  Allocates all scratch on the current device; no
 * allocation happens in any later call except the first sc_to_phys/sc_to_spec
 * (full-spectrum scratch) and the first sc_rk4_steps/sc_wray3_step (graph). */
SC_API int sc_plan_create(sc_plan** plan, int D, int n, double l, int dtype, size_t* workspace_bytes);
SC_API int sc_plan_destroy(sc_plan* plan);
SC_API int sc_plan_info(const sc_plan* plan, int* D, int* n, int* dtype, int* kcut);

/* ---- FFT wrappers --------------------------------------------------------
 * to_phys! (src/solver.jl:210-211): phys = c2r(spec) * n^D (unnormalised
 * inverse).  Unlike the reference's c2r the input is preserved.  Imaginary
 * parts of the kx = 0 and kx = n/2 planes that break Hermitian symmetry are
 * treated as the c2r transform does (only the real part of the row DC and
 * Nyquist bins is used). */
SC_API int sc_to_phys(sc_plan* plan, const void* spec, void* phys, void* stream);
/* to_spec! (src/solver.jl:214-215): spec = r2c(phys) / n^D. */
SC_API int sc_to_spec(sc_plan* plan, const void* phys, void* spec, void* stream);

/* ---- spectral point kernels (in place, full layout) ---------------------- */
/* twothirds! (src/solver.jl:371-389) on `ncomp` scalar fields. */
SC_API int sc_twothirds(sc_plan* plan, void* const* fields, int ncomp, void* stream);
/* project! (src/solver.jl:350-368). */
SC_API int sc_project(sc_plan* plan, void* const* u_hat, void* stream);

/* ---- Navier-Stokes right-hand side ----------------------------------------
 * convectiondiffusion!(du, u, grid, cache; visc) (src/solver.jl:949-953):
 * du_i = -i k_j (F[(P u_i)(P u_j)]/n^D - visc i (k_j u_i + k_i u_j)), P the
 * 2/3 rule.  Output: du on the retained modes (|k_i| <= n/3, k != 0), zero
 * elsewhere -- i.e. twothirds!(du) of the reference's du, which is all that
 * ever reaches the retained modes of the state. */
SC_API int sc_rhs(sc_plan* plan, const void* const* u_hat, void* const* du_hat, double visc, void* stream);

/* ---- time steppers (state in full layout, advanced in place) -------------
 * wray3!(convectiondiffusion!, u, dt, grid, cache; visc) (src/solver.jl:968-1012):
 * one low-storage Wray RK3 step, projecting after every stage.  The state is
 * kept on the 2/3 cube (modes outside it are set to zero); its retained modes
 * follow the reference's exactly. */
SC_API int sc_wray3_step(sc_plan* plan, void* const* u_hat, double dt, double visc, void* stream);
/* New (no reference counterpart): `nsteps` classical RK4 steps,
 * u_{n+1} = P(u_n + dt/6 (k1 + 2 k2 + 2 k3 + k4)), k_s = P(rhs(u_s)) + forcing,
 * with the optional linear band forcing.  Same state convention as
 * sc_wray3_step.  One RK4 step is captured in a CUDA graph and replayed. */
SC_API int sc_rk4_steps(sc_plan* plan, void* const* u_hat, double dt, double visc, int nsteps,
                 const sc_forcing* forcing, void* stream);

/* ---- initial field ---------------------------------------------------------
 * randomfield(peak_profile, g; kpeak, totalenergy) (src/solver.jl:576-641,
 * :523) on the device, in FP64: complex normal coefficients on the retained
 * 2/3 cube (each part N(0, 1/2)), symmetrize! of the kx = 0 plane, project!,
 * twothirds!, and the rescale of every shell floor|k| = s to
 * totalenergy * s^4 exp(-2 (s/kpeak)^2) / sum_s (...).  The result becomes the
 * plan's state (as sc_state_load) and, when u_hat is not NULL, is written to
 * u_hat in the full layout.  draws: D device arrays of the coefficients in the
 * compact layout (complex FP64, (K2, K2, K1) x-fastest; the caller's own
 * generator), or NULL for the device's counter-based generator keyed by seed
 * (splitmix64 + Box-Muller; Julia's Xoshiro stream is not reproduced).
 * Synchronous. */
SC_API int sc_random_field(sc_plan* plan, unsigned long long seed, const void* const* draws, double kpeak,
                           double totalenergy, void* const* u_hat, void* stream);

/* ---- device-resident state (compact 2/3 cube held by the plan) ----------- */
/* Gather the retained modes of u_hat into the plan's state. */
SC_API int sc_state_load(sc_plan* plan, const void* const* u_hat, void* stream);
/* Scatter the plan's state back to the full layout (zeros outside the 2/3 cube). */
SC_API int sc_state_store(sc_plan* plan, void* const* u_hat, void* stream);
/* sc_rk4_steps on the plan's state, without the load/store. */
SC_API int sc_state_rk4(sc_plan* plan, double dt, double visc, int nsteps, const sc_forcing* forcing, void* stream);
/* energy(u) (src/solver.jl:643-646) of the plan's state, FP64, synchronous. */
SC_API int sc_state_energy(sc_plan* plan, double* energy, void* stream);
/* Profiling hook: run the right-hand side of the plan's state `reps` times
 * with CUDA events between its kernels and return the mean time (ms) of each
 * kernel in launch order -- 3D: z-inverse, y-inverse, x sweep, y-forward,
 * z-forward, epilogue; 2D: y-inverse, x sweep, y-forward, epilogue.
 * `ms` must hold 8 doubles.  Synchronous. */
SC_API int sc_state_profile_rhs(sc_plan* plan, double visc, int reps, double* ms, int* nkernels, void* stream);
/* Microbenchmark of one sweep kernel on zero-filled synthetic buffers of the
 * right shape (allocated and freed inside; legacy default stream):
 * kernel 0 = y-inverse sweep (3 comps) over `count` z planes, 1 = y-forward
 * sweep (6 comps) over `count` z planes, 2 = the 3D x sweep with products over
 * `count` rows, 3 / 4 = z-inverse / z-forward sweep of one component over the
 * first `count` ky columns of a full-size cube (count <= 2 (n/3) + 1).  Returns the mean ms per launch over `reps` launches and the
 * algorithmic bytes of one launch.  Synchronous; used by the profiles and the
 * tile autotuning, not by the solver. */
SC_API int sc_microbench(int kernel, int n, int dtype, long long count, int reps, double* ms, double* bytes);
/* Number of kernels one sc_state_rk4 step launches (for launch accounting). */
SC_API int sc_state_rk4_launches_per_step(const sc_plan* plan, int forced);

/* ---- LES closures and the LES right-hand side --------------------------------
 * A closure is the reference's closure object `model(u, G) -> tau`
 * (src/les.jl:19), bound to a plan.  Kinds and parameters:
 *   SC_CLOSURE_NONE        no model (les! reduces to convectiondiffusion!)
 *   SC_CLOSURE_CLARK       create_clark(Delta, g): tau = Delta^2/12 G G^T (src/closures.jl:37-42,64)
 *   SC_CLOSURE_SMAGORINSKY create_smagorinsky(C_s, Delta, g), params[0] = C_s (default 0.17)
 *   SC_CLOSURE_VERSTAPPEN  create_verstappen(C, Delta, g), params[0] = C (3D only; default 0.345)
 *   SC_CLOSURE_DYNAMIC_SMAGORINSKY  create_dynamic_smagorinsky(Delta, g) (src/closures.jl:188-272):
 *                          Germano-Lilly with a Gaussian(2 Delta) test filter, global FP64 averages
 *   SC_CLOSURE_BARDINA     create_bardina(s, Delta, g), params[0] = s (default 2; src/closures.jl:81-115)
 * Closure scratch is allocated at creation; evaluation allocates nothing. */
#define SC_CLOSURE_NONE 0
#define SC_CLOSURE_CLARK 1
#define SC_CLOSURE_SMAGORINSKY 2
#define SC_CLOSURE_VERSTAPPEN 3
#define SC_CLOSURE_DYNAMIC_SMAGORINSKY 4
#define SC_CLOSURE_BARDINA 5
#define SC_CLOSURE_CNN 6
#define SC_CLOSURE_CNN_FP 7
typedef struct sc_closure sc_closure;
SC_API int sc_closure_create(sc_closure** closure, sc_plan* plan, int kind, double delta, const double* params,
                             int nparams);
SC_API int sc_closure_destroy(sc_closure* closure);
/* CNN closure (new; no reference counterpart; the batched 128^3 LES closure): input u (3
 * physical channels) plus the standardised log Re_Delta, (log(Delta^2
 * sqrt(<|grad u|^2>)/visc) - mu)/sigma, as a 4th constant channel (the
 * convention of fullchain, src/nets.jl:311-331); four 3x3x3 periodic
 * convolutions 4->32->32->32->6 with GELU between them (NNlib's tanh form,
 * src/nets.jl:187; hardware tanh.approx.f32 in this BF16 path); output tau in
 * pair order.  BF16 weights and activations, FP32 accumulation on tcgen05
 * tensor cores.  weights[l]: host FP32 (C_out, C_in, 3, 3, 3) (rounded to BF16
 * here), biases[l]: host FP32 (C_out).  FP32 3D plans with n = 64 or 128.
 * sc_closure_set_option(SC_CLOPT_CNN_SPLIT) switches it to three passes over
 * hi/lo operand parts per convolution (about FP32 accuracy). */
SC_API int sc_cnn_closure_create(sc_closure** closure, sc_plan* plan, double delta, double visc,
                                 const float* const* weights, const float* const* biases, double mu, double sigma);
/* The same CNN on CUDA cores in the plan's precision (FP32 or FP64, any 3D
 * grid), without BF16 rounding: the closure the a-posteriori adjoint
 * differentiates, and the FP64 per-instance reference of the tensor-core CNN. */
SC_API int sc_cnn_fp_closure_create(sc_closure** closure, sc_plan* plan, double delta, double visc,
                                    const float* const* weights, const float* const* biases, double mu,
                                    double sigma);
/* Flat parameter vector of the FP32/FP64 CNN closure, layer by layer [w (C_out, C_in, 27), b (C_out)]. */
/* fullchain(setup, mlp(...)) (src/nets.jl:311-331, 248-296): a pointwise MLP
 * closure in the plan's precision.  Input: the velocity gradient G normalised
 * by (|G| + eps) pointwise, channels d_b u_a with a fastest, plus the
 * standardised log Re_Delta channel when use_redelta (append_redelta,
 * src/data.jl:689-695, with mu, sigma); layers widths[0] -> ... -> widths[nlayers]
 * (widths[0] = D^2 (+1), widths[nlayers] = 6 | 3, each <= 128) with GELU (NNlib's
 * tanh form) on all but the last, which has no bias; trace removed; tau =
 * output * Delta^2 |G|^2.  theta: per layer W[c_out][c_in] (the memory order of
 * Lux's (c_in, c_out) PointwiseConv weight), then b[c_out] (not for the last).
 * Kind SC_CLOSURE_MLP. */
#define SC_CLOSURE_MLP 8
SC_API int sc_mlp_closure_create(sc_closure** closure, sc_plan* plan, double delta, double visc, int nlayers,
                                 const int* widths, const double* theta, int use_redelta, double mu, double sigma);
/* tbnn(net, ps, st, Delta, g; use_redelta, redelta_norm, visc) (src/nets.jl:560-588)
 * with the tensor basis of tb_kernel! (src/nets.jl:393-505): the normalised
 * gradient's invariants tr(SS), tr(RR) [, tr(SSS), tr(SRR), tr(SSRR)] (+ Re_Delta)
 * feed the same pointwise MLP (widths[0] = 2 | 5 (+1), widths[nlayers] = 2 | 7
 * basis coefficients); tau = sum_k w_k B_k * Delta^2 |G|^2 with the deviatoric
 * basis dev(S), dev(SR - RS) (2D) or dev(S), dev(SS), dev(RR), dev(SR - RS),
 * dev(RSR), dev(RSS - SSR), dev(RSRR - RRSR) (3D).  Kind SC_CLOSURE_TBNN. */
#define SC_CLOSURE_TBNN 9
SC_API int sc_tbnn_closure_create(sc_closure** closure, sc_plan* plan, double delta, double visc, int nlayers,
                                  const int* widths, const double* theta, int use_redelta, double mu, double sigma);
SC_API int sc_closure_num_params(const sc_closure* closure, long long* nparams);
SC_API int sc_closure_set_params(sc_closure* closure, const double* theta);
/* Synchronous: SC_ERR_TIMEOUT if a bounded wait of the closure's kernels ran out. */
SC_API int sc_closure_status(sc_closure* closure, int* status);
/* Closure options (no reference counterpart; the reference's networks run in
 * the precision of their weights).  SC_CLOPT_CNN_SPLIT (tensor-core CNN
 * closure only): 1 evaluates every convolution as three tcgen05 passes over
 * split operands, x = hi + lo with hi the nearest 16-bit number to x and lo the
 * nearest to x - hi, A_hi W_hi + A_lo W_hi + A_hi W_lo accumulated in FP32 (FP16
 * parts in the forward pass, weights stored x 64 so that their low parts stay
 * normal FP16 numbers; BF16 parts for the adjoint's input-gradient
 * convolutions, whose gradients need BF16's exponent range), with GELU from
 * tanhf and the weight gradients from the hi + lo sums: about FP32 accuracy at
 * three times the convolutions' tensor-core work.  0 (default): BF16 operands,
 * one pass.  SC_ERR_INVALID when a weight x 64 is beyond the FP16 range.
 * Allocates the split activations on the first switch; cached step graphs of
 * the closure's plan are rebuilt (LES batches and graphs captured by the caller
 * keep the precision they were captured with). */
#define SC_CLOPT_CNN_SPLIT 1
SC_API int sc_closure_set_option(sc_closure* closure, int option, long long value);
/* model(u, G): the packed physical stress tau (3|6 fields, pair order) from
 * the spectral velocity u_hat (full layout) and the physical velocity
 * gradient G (D*D fields, G[a + D b] = d u_a / d x_b; Clark, Smagorinsky and
 * Verstappen read only G, Bardina and dynamic Smagorinsky only u_hat). */
SC_API int sc_closure_eval(sc_closure* closure, const void* const* u_hat, const void* const* G_phys,
                           void* const* tau_phys, void* stream);
/* les!(du, u, grid, cache; model, visc) (src/les.jl:4-33): du = div(stress(u)
 * + F[model(u, G)]) with G = to_phys(twothirds(vectorgradient(u))); output on
 * the retained modes as sc_rhs.  closure = NULL gives convectiondiffusion!. */
SC_API int sc_les_rhs(sc_plan* plan, sc_closure* closure, const void* const* u_hat, void* const* du_hat, double visc,
                      void* stream);
/* wray3!(les!, u, dt, grid, cache; model, visc) (src/les.jl:216-219). */
SC_API int sc_les_wray3_step(sc_plan* plan, sc_closure* closure, void* const* u_hat, double dt, double visc,
                             void* stream);
/* RK4 steps of the LES (new), optional band forcing; graph-captured. */
SC_API int sc_les_rk4_steps(sc_plan* plan, sc_closure* closure, void* const* u_hat, double dt, double visc,
                            int nsteps, const sc_forcing* forcing, void* stream);
/* sc_les_rk4_steps on the plan's device-resident state. */
SC_API int sc_state_les_rk4(sc_plan* plan, sc_closure* closure, double dt, double visc, int nsteps,
                            const sc_forcing* forcing, void* stream);

/* ---- batched LES ----------------------------------------------------------------
 * No reference counterpart (the reference runs one LES per process,
 * src/les.jl:56-186).  Each instance owns a plan (its device-resident state is
 * loaded with sc_state_load), an optional closure, nu, dt and forcing.  One RK4
 * step of every active instance is captured into one CUDA graph (one branch
 * per instance, so instances run concurrently) followed by an FP64 energy
 * guard; sc_les_batch_run replays it.  An instance whose energy exceeds 1e5 or
 * is not finite gets status SC_ERR_DIVERGED (the blow-up guard of solve_les!,
 * src/les.jl:224-237); sc_les_batch_status(..., freeze = 1) drops such
 * instances from later steps without stopping the others. */
typedef struct sc_les_instance {
  sc_plan* plan;
  sc_closure* closure;
  double visc;
  double dt;
  int forced;
  double eps;
} sc_les_instance;
typedef struct sc_les_batch sc_les_batch;
SC_API int sc_les_batch_create(sc_les_batch** batch, const sc_les_instance* instances, int ninstances);
SC_API int sc_les_batch_run(sc_les_batch* batch, int nsteps, void* stream);
/* Synchronous: per-instance status and energy (energy may be NULL). */
SC_API int sc_les_batch_status(sc_les_batch* batch, int* status, double* energy, int freeze, void* stream);
SC_API int sc_les_batch_destroy(sc_les_batch* batch);
/* The a-posteriori reductions of solve_les!'s reduce! (src/les.jl:94-148),
 * fused into the batched stepper: every `every` steps of sc_les_batch_run the
 * step graph also reduces, for every active instance, its kinetic energy,
 * viscous dissipation (FP64 sums, as sc_les_diagnostics), SFS dissipation,
 * spectrum and shell transfer (shells 1..nshell) into a device record of at
 * most max_snap snapshots, with no host round trip during the run; e_post,
 * which needs a reference trajectory, stays with sc_les_diagnostics.
 * every = 0 turns it off; calling it again starts a new record.
 * sc_les_batch_snapshots returns the number recorded and (out != NULL) the
 * record [nsnap][ninstances][3 + 2 nshell] = (ke, eps_visc, eps_sfs,
 * spectrum[nshell], transfer[nshell]); synchronous.  Frozen (diverged)
 * instances keep their last values. */
SC_API int sc_les_batch_set_snapshots(sc_les_batch* batch, int every, int nshell, int max_snap);
SC_API int sc_les_batch_snapshots(sc_les_batch* batch, int* nsnap, double* out, void* stream);

/* ---- plan options ---------------------------------------------------------------- */
#define SC_OPT_USE_GRAPH 1 /* 1 (default): steppers replay a captured CUDA graph; 0: launch eagerly */
/* Bound of the device-side waits of the plan's tensor-core CNN closures and
 * of its TMA-fed column sweeps (polls of an mbarrier before a wait gives up).
 * A CNN kernel whose wait runs out sets the closure's error flag --
 * sc_closure_status then reports SC_ERR_TIMEOUT -- frees its tensor memory and
 * returns; a column sweep sets the plan's error word (sc_plan_status) and
 * returns.  A negative value restores the default (2^26 polls); 0 makes
 * every such wait give up at once, which lets a test exercise the timeout path
 * without hanging or faulting anything; the kernels' last wait for work still
 * in flight (tensor-core MMAs, bulk copies into shared memory) always keeps
 * the default bound.  Takes effect at the next evaluation (not in step graphs
 * captured before the change). */
#define SC_OPT_WAIT_LIMIT 2
/* Kernel variant of one sweep of the 3D product pipeline of an FP32 plan
 * (value 0 .. sc_plan_num_variants - 1; 0 is the default): the candidates of
 * the autotuner (symcode.autotune), which times every variant of every sweep
 * on the plan's own buffers and keeps the fastest.  The variants are the same
 * transforms by other tile widths, splits N = N1 N2 or x-sweep kernels, and at
 * n = 810 persistent column sweeps fed by tensor-memory-access bulk copies
 * (variants 4-6 of the y-inverse, y-forward and z-forward sweeps); the
 * steppers' cached graphs are rebuilt after a change.  No reference
 * counterpart (the reference's plan choice is cuFFT/FFTW planning,
 * src/solver.jl:432). */
#define SC_OPT_VARIANT_ZINV 3
#define SC_OPT_VARIANT_YINV 4
#define SC_OPT_VARIANT_X 5
#define SC_OPT_VARIANT_YFWD 6
#define SC_OPT_VARIANT_ZFWD 7
SC_API int sc_plan_set_option(sc_plan* plan, int option, long long value);
/* Number of variants of sweep 0..4 (z-inverse, y-inverse, x, y-forward,
 * z-forward) for this plan (1 where there is no choice: FP64 plans, 2D, sizes
 * without the FP32 two-level engine). */
SC_API int sc_plan_num_variants(const sc_plan* plan, int sweep, int* count);
/* Synchronous: SC_ERR_TIMEOUT in *status if a bounded wait of the plan's
 * TMA-fed column sweeps ran out since the last call (their outputs are then
 * invalid), else SC_OK; reading clears the record. */
SC_API int sc_plan_status(sc_plan* plan, int* status);

/* ---- a-posteriori training: rollout, loss and hand-written adjoint ----------
 * New (the reference trains a-priori only, src/training.jl:3-109).  A rollout
 * is `nsteps` RK4 steps (projected stage derivatives, no forcing) of the LES
 * with `closure` from u0 (full layout).  A trajectory is `nsteps` compact
 * states (retained modes, the plan's precision) on the device, size
 * sc_rollout_traj_bytes.  The loss is the trajectory MSE
 *   L = 1/nsteps sum_s <u_s - u*_s, u_s - u*_s>,
 * <a, b> = sum over the half spectrum of w Re(conj a b) (the physical mean of
 * the product).  sc_rollout_adjoint returns L and dL/dtheta (host, FP64,
 * sc_closure_num_params entries) by the discrete adjoint of the RK4 steps and
 * of the LES right-hand side (FFT transposes, product and viscous terms,
 * projection, the CNN's convolutions and GELUs and its Re_Delta channel),
 * recomputing the states from checkpoints every `ckpt_every` steps.
 * All three are synchronous. */
SC_API size_t sc_rollout_traj_bytes(const sc_plan* plan, int nsteps);
SC_API int sc_rollout_record(sc_plan* plan, sc_closure* closure, const void* const* u0, double dt, double visc,
                             int nsteps, void* traj, void* stream);
SC_API int sc_rollout_loss(sc_plan* plan, sc_closure* closure, const void* const* u0, const void* traj, double dt,
                           double visc, int nsteps, double* loss, void* stream);
SC_API int sc_rollout_adjoint(sc_plan* plan, sc_closure* closure, const void* const* u0, const void* traj,
                              double dt, double visc, int nsteps, int ckpt_every, double* loss, double* grad,
                              void* stream);
/* A batch of training rollouts (the a-posteriori training step over several
 * LES instances): job i is sc_rollout_adjoint(plan, closure, u0, traj, dt,
 * visc, nsteps, ckpt_every, loss, grad).  The jobs run concurrently, each from
 * its own host thread on its own stream, after the work already queued on
 * `stream`; every job needs its own plan and closure.  status[i] receives each
 * job's sc_status; the call returns the first non-zero one.  Synchronous. */
typedef struct sc_rollout_job {
  sc_plan* plan;
  sc_closure* closure;
  const void* u0[3];
  const void* traj;
  double dt, visc;
  int nsteps, ckpt_every;
  double* loss; /* host, 1 */
  double* grad; /* host, sc_closure_num_params */
} sc_rollout_job;
SC_API int sc_rollout_adjoint_batch(int njobs, const sc_rollout_job* jobs, int* status, void* stream);

/* ---- DNS -> LES filter ------------------------------------------------------
 * sfs!(; tau, ubar, u, g_dns, g_les, Delta) (src/data.jl:625-642) for `ndelta`
 * filter widths at once (the DNS products are computed once and shared):
 *   ubar = twothirds(G_Delta cutoff(u)),
 *   tau  = tracefree(twothirds(G_Delta cutoff(sigma_dns) - sigma_les(ubar))),
 * cutoff! / gaussianfilter! as in src/filtering.jl:28-67.  `deltas[d]` is the
 * physical width (Delta_factor * l / n_les in the reference, src/experiment.jl:164);
 * deltas[d] <= 0 means no Gaussian (the reference's Delta = nothing).
 * u_hat: DNS full layout (D pointers).  ubar_hat: ndelta*D LES full-layout
 * fields (d-major); tau_hat: ndelta*(3|6) LES full-layout fields, pair order
 * xx, yy[, zz], xy[, yz, zx].  The two plans must be distinct, same D, l,
 * precision and device, n_les <= n_dns. */
SC_API int sc_filter_sfs(sc_plan* dns, sc_plan* les, const void* const* u_hat, const double* deltas, int ndelta,
                         void* const* ubar_hat, void* const* tau_hat, void* stream);
/* filter_reynolds(ubar, g, visc, Delta) (src/solver.jl:768-774):
 * Delta^2 sqrt(sum_ab getenergy(twothirds(d_b ubar_a))) / visc.  Synchronous. */
SC_API int sc_filter_reynolds(sc_plan* les, const void* const* ubar_hat, double visc, double delta, double* re,
                              void* stream);

/* ---- CFL step, forcing by shell clamp, spectrum ------------------------------- */
/* propose_timestep(u, grid, visc, cache) (src/solver.jl:931-947):
 * min(h / max|P u|, h^2 / (2 D visc)); the caller multiplies by cfl.  Synchronous. */
SC_API int sc_propose_timestep(sc_plan* plan, const void* const* u_hat, double visc, double* dt, void* stream);
/* energy_shells(grid, [1, 2], u) (src/solver.jl:1135-1140): the reference
 * energies of shells 1 <= |k| < 2 and 2 <= |k| < 3 (eref[0..1]).  Synchronous. */
SC_API int sc_shell_energies(sc_plan* plan, const void* const* u_hat, double* eref, void* stream);
/* maintain_shell_energy!(u, shells) (src/solver.jl:1146-1152): rescale those
 * shells of u_hat (retained modes) to eref.  Synchronous. */
SC_API int sc_maintain_shell_energy(sc_plan* plan, void* const* u_hat, const double* eref, void* stream);
SC_API int sc_state_maintain_shell_energy(sc_plan* plan, const double* eref, void* stream);
/* spectrum(u, grid) (src/solver.jl:693-699) on shells 1..nshell (nshell <= n/3):
 * s[i-1] = 1/2 sum_{i <= |k| < i+1} |u_hat|^2 with the RFFT double count.  Synchronous. */
SC_API int sc_spectrum(sc_plan* plan, const void* const* u_hat, int nshell, double* s, void* stream);

/* The a-posteriori reductions of one LES state in solve_les!'s reduce!
 * (src/les.jl:94-148): out[0] = e_post = ||u - twothirds(u_ref)|| / ||twothirds(u_ref)||
 * (0 when u_ref is null), out[1] = kinetic energy, out[2] = viscous
 * dissipation (get_dissipation!), out[3] = eps_sfs = -mean(tau_dev : S) with
 * the closure re-evaluated on u (0 without a closure); spec[0..nshell-1] =
 * spectrum(u); transfer[i-1] = sum over shell i of Re(conj(u) . (-i k_j tau_dev_ij))
 * (zeros without a closure).  1 <= nshell <= n/3.  Synchronous. */
SC_API int sc_les_diagnostics(sc_plan* plan, sc_closure* closure, const void* const* u_hat,
                              const void* const* uref_hat, double visc, int nshell, double* out, double* spec,
                              double* transfer, void* stream);

/* ---- diagnostics (FP64 on the device; synchronous, result to host) ------- */
/* energy(u) (src/solver.jl:643-646): 1/2 sum_i getenergy(u_i). */
SC_API int sc_energy(sc_plan* plan, const void* const* u_hat, double* energy, void* stream);
/* get_dissipation! (src/solver.jl:808-811): visc sum k^2 |u|^2 (RFFT double count). */
SC_API int sc_dissipation(sc_plan* plan, const void* const* u_hat, double visc, double* diss, void* stream);

/* ---- allocation-free spectrum (no counterpart in the reference) ----------- */
/* The spectrum of sc_spectrum (shells 1..nshell, 1 <= nshell <= n/3) read
 * straight from the full RFFT layout u_hat[c] (n/2+1, n[, n]), with no plan and
 * no device allocation: the shell sums go to a fixed device array of
 * SC_SPECTRUM_STATIC_MAX_SHELLS doubles (4 KiB) inside the library, zeroed by
 * each call; a larger nshell returns SC_ERR_SIZE.  For callers that may not
 * allocate, such as a monitor between the time steps of a run whose device
 * memory is taken by the solver: sc_spectrum there would set up a plan's work
 * buffers and take a stream-ordered shell buffer per call.  The first call on
 * each device looks up the array's address with that device current; make it
 * before any stream capture begins.  The address is kept per device and CUDA
 * context, so the first call after a context reset (cudaDeviceReset) looks it
 * up again and also belongs before any capture.  Calls on one device share the array, so
 * calls that overlap in time (other streams or host threads) race.
 * Synchronous on stream. */
#define SC_SPECTRUM_STATIC_MAX_SHELLS 512
SC_API int sc_spectrum_static(const void* const* u_hat, int n, int D, int dtype, int nshell, double* s,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SYMCODE_H */
