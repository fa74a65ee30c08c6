"""Host-side mirror of SymmetryCode.jl's solver API over the B200 C ABI.

Each function here has the name of the reference function it replaces (an
in-place Julia ``f!`` becomes ``f_``), the same argument meaning and the same
array layout, and runs the hand-written sm_100a kernels of ``libsymcode.so``
through ctypes.  torch provides device memory and streams only.

Field layout: a spectral scalar field of a ``Grid`` is a contiguous complex
torch tensor of shape ``(n, n/2+1)`` (2D) or ``(n, n, n/2+1)`` (3D) -- in
memory the reference's column-major ``(n/2+1, n[, n])`` array; vector fields
are lists ``[x, y(, z)]``, symmetric tensors ``[xx, yy(, zz), xy(, yz, zx)]``.
"""

from __future__ import annotations

import ctypes as ct
import math

import torch

from . import autotune, fields  # noqa: F401
from ._lib import (SC_CLOPT_CNN_SPLIT, SC_FLOAT32, SC_FLOAT64, SymcodeError, check, header_functions, lib,
                   ptr_array, sc_forcing, sc_les_instance)

__all__ = [
    "Grid", "SymcodeError", "scalarfield", "vectorfield", "tensorfield", "spacescalarfield",
    "spacevectorfield", "to_phys_", "to_spec_", "twothirds_", "project_", "convectiondiffusion_",
    "wray3_", "rk4_", "energy", "get_dissipation", "lib", "header_functions", "sfs_", "filter_reynolds",
    "State", "LesBatch", "propose_timestep", "energy_shells", "maintain_shell_energy_", "spectrum",
    "turbulence_statistics", "set_option", "Closure", "create_clark", "create_smagorinsky", "create_verstappen",
    "create_dynamic_smagorinsky", "create_bardina", "create_cnn_closure", "kaiming_cnn_weights",
    "create_cnn_fp_closure", "closure_num_params", "closure_set_params", "closure_set_option", "SC_CLOPT_CNN_SPLIT",
    "pack_cnn_params", "rollout_record",
    "rollout_loss", "rollout_adjoint", "les_", "les_wray3_", "les_rk4_", "fields",
]


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ct.c_void_p(stream.cuda_stream)


class Grid:
    """``Grid{D}(; l, n)`` + ``getcache(grid)`` (src/solver.jl:131-151, 956-965).

    Creates the device plan (twiddles and all pencil scratch) on ``device``.
    ``dtype`` is the real precision of the fields (torch.float32 / float64).
    """

    def __init__(self, D, n, l=2 * math.pi, dtype=torch.float64, device="cuda"):
        if n % 2 != 0:
            raise AssertionError("Only even number of grid points supported.")
        if D not in (2, 3):
            raise ValueError("D must be 2 or 3")
        if not torch.cuda.is_available():
            raise RuntimeError("symcode needs a CUDA device (sm_100a); none is available")
        self.D, self.n, self.l = D, n, float(l)
        self.dtype = dtype
        self.cdtype = torch.complex64 if dtype == torch.float32 else torch.complex128
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        L = lib()
        plan = ct.c_void_p()
        ws = ct.c_size_t()
        with torch.cuda.device(self.device):
            check(L.sc_plan_create(ct.byref(plan), D, n, self.l,
                                   SC_FLOAT32 if dtype == torch.float32 else SC_FLOAT64, ct.byref(ws)))
        self._plan = plan
        self.workspace_bytes = ws.value

    # reference accessors (src/solver.jl:155-202)
    @property
    def tensordim(self):
        return 3 if self.D == 2 else 6

    @property
    def spacing(self):
        return self.l / self.n

    @property
    def volume(self):
        return (self.l / self.n) ** self.D

    @property
    def ndrange(self):
        return (self.n // 2 + 1,) + (self.n,) * (self.D - 1)

    @property
    def space_ndrange(self):
        return (self.n,) * self.D

    @property
    def spec_shape(self):
        return tuple(reversed(self.ndrange))

    @property
    def phys_shape(self):
        return (self.n,) * self.D

    @property
    def plan(self):
        return self._plan

    def close(self):
        if getattr(self, "_plan", None):
            with torch.cuda.device(self.device):
                lib().sc_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers ---------------------------------------------------------
    def _check_spec(self, t):
        if t.dtype != self.cdtype or tuple(t.shape) != self.spec_shape or not t.is_contiguous() or t.device != self.device:
            raise ValueError(f"expected contiguous {self.cdtype} tensor of shape {self.spec_shape} on {self.device}, "
                             f"got {t.dtype} {tuple(t.shape)} on {t.device}")
        return t.data_ptr()

    def _check_phys(self, t):
        if t.dtype != self.dtype or tuple(t.shape) != self.phys_shape or not t.is_contiguous() or t.device != self.device:
            raise ValueError(f"expected contiguous {self.dtype} tensor of shape {self.phys_shape} on {self.device}")
        return t.data_ptr()


# --------------------------------------------------------------------------
# field allocators (src/solver.jl:245-300)
# --------------------------------------------------------------------------

def scalarfield(g: Grid):
    return torch.zeros(g.spec_shape, dtype=g.cdtype, device=g.device)


def vectorfield(g: Grid):
    return [scalarfield(g) for _ in range(g.D)]


def tensorfield(g: Grid):
    return [scalarfield(g) for _ in range(g.tensordim)]


def spacescalarfield(g: Grid):
    return torch.zeros(g.phys_shape, dtype=g.dtype, device=g.device)


def spacevectorfield(g: Grid):
    return [spacescalarfield(g) for _ in range(g.D)]


# --------------------------------------------------------------------------
# solver calls
# --------------------------------------------------------------------------

def to_phys_(phys, spec, g: Grid, stream=None):
    """``to_phys!(phys, spec, plan, g)`` (src/solver.jl:210-211); ``spec`` is preserved."""
    check(lib().sc_to_phys(g.plan, ct.c_void_p(g._check_spec(spec)), ct.c_void_p(g._check_phys(phys)),
                           _stream_ptr(stream)))
    return phys


def to_spec_(spec, phys, g: Grid, stream=None):
    """``to_spec!(spec, phys, plan, g)`` (src/solver.jl:214-215)."""
    check(lib().sc_to_spec(g.plan, ct.c_void_p(g._check_phys(phys)), ct.c_void_p(g._check_spec(spec)),
                           _stream_ptr(stream)))
    return spec


def twothirds_(fields, g: Grid, stream=None):
    """``apply!(twothirds!, g, (u, g))`` on one or several scalar fields (src/solver.jl:371-389)."""
    if isinstance(fields, torch.Tensor):
        fields = [fields]
    pp, _keep = ptr_array([g._check_spec(f) for f in fields])
    check(lib().sc_twothirds(g.plan, pp, len(fields), _stream_ptr(stream)))
    return fields


def project_(u, g: Grid, stream=None):
    """``apply!(project!, g, (u, g))`` (src/solver.jl:350-368)."""
    pp, _keep = ptr_array([g._check_spec(c) for c in u])
    check(lib().sc_project(g.plan, pp, _stream_ptr(stream)))
    return u


def convectiondiffusion_(du, u, g: Grid, visc, stream=None):
    """``convectiondiffusion!(du, u, grid, cache; visc)`` (src/solver.jl:949-953).

    ``du`` receives the right-hand side on the modes the 2/3 rule keeps
    (``twothirds!`` of the reference's ``du``), zero elsewhere.
    """
    pu, _k1 = ptr_array([g._check_spec(c) for c in u])
    pd, _k2 = ptr_array([g._check_spec(c) for c in du])
    check(lib().sc_rhs(g.plan, pu, pd, float(visc), _stream_ptr(stream)))
    return du


def wray3_(u, dt, g: Grid, visc, stream=None):
    """``wray3!(convectiondiffusion!, u, Δt, grid, cache; visc)`` (src/solver.jl:968-1012)."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    check(lib().sc_wray3_step(g.plan, pu, float(dt), float(visc), _stream_ptr(stream)))
    return u


def rk4_(u, dt, g: Grid, visc, nsteps=1, eps=None, stream=None):
    """``nsteps`` RK4 steps with optional linear band forcing at injection rate ``eps`` (new)."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    f = sc_forcing(1 if eps is not None else 0, float(eps) if eps is not None else 0.0)
    check(lib().sc_rk4_steps(g.plan, pu, float(dt), float(visc), int(nsteps), ct.byref(f), _stream_ptr(stream)))
    return u


def energy(u, g: Grid, stream=None):
    """``energy(u)`` (src/solver.jl:643-646), accumulated in FP64 on the device."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    out = ct.c_double()
    check(lib().sc_energy(g.plan, pu, ct.byref(out), _stream_ptr(stream)))
    return out.value


def get_dissipation(u, visc, g: Grid, stream=None):
    """``get_dissipation!`` (src/solver.jl:808-811), FP64 on the device."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    out = ct.c_double()
    check(lib().sc_dissipation(g.plan, pu, float(visc), ct.byref(out), _stream_ptr(stream)))
    return out.value


def sfs_(ubar, tau, u, g_dns: Grid, g_les: Grid, deltas, stream=None):
    """``sfs!(; τ, ubar, u, g_dns, g_les, Δ)`` (src/data.jl:625-642) for one or several widths.

    ``deltas``: a float or a list (``None`` = no Gaussian).  For a list, ``ubar``
    and ``tau`` are lists (one vector / tensor field per width).
    """
    single = not isinstance(deltas, (list, tuple))
    ds = [deltas] if single else list(deltas)
    ub = [ubar] if single else ubar
    ta = [tau] if single else tau
    if len(ub) != len(ds) or len(ta) != len(ds):
        raise ValueError("one ubar and one tau field per filter width")
    dv = (ct.c_double * len(ds))(*[(-1.0 if d is None else float(d)) for d in ds])
    pu, _k1 = ptr_array([g_dns._check_spec(c) for c in u])
    pb, _k2 = ptr_array([g_les._check_spec(c) for f in ub for c in f])
    pt, _k3 = ptr_array([g_les._check_spec(c) for f in ta for c in f])
    check(lib().sc_filter_sfs(g_dns.plan, g_les.plan, pu, dv, len(ds), pb, pt, _stream_ptr(stream)))
    return ubar, tau


def filter_reynolds(ubar, g: Grid, visc, delta, stream=None):
    """``filter_reynolds(ubar, g, visc, Δ)`` (src/solver.jl:768-774)."""
    pu, _k = ptr_array([g._check_spec(c) for c in ubar])
    out = ct.c_double()
    check(lib().sc_filter_reynolds(g.plan, pu, float(visc), float(delta), ct.byref(out), _stream_ptr(stream)))
    return out.value


# --------------------------------------------------------------------------
# closures (src/closures.jl) and the LES right-hand side (src/les.jl:4-33)
# --------------------------------------------------------------------------
CLOSURE_NONE, CLOSURE_CLARK, CLOSURE_SMAGORINSKY, CLOSURE_VERSTAPPEN = 0, 1, 2, 3
CLOSURE_DYNAMIC_SMAGORINSKY, CLOSURE_BARDINA, CLOSURE_CNN = 4, 5, 6


class Closure:
    """A closure model bound to a Grid; ``closure(u, G)`` returns the packed
    physical stress like the reference's ``model(u, G)`` (src/les.jl:19)."""

    def __init__(self, g: Grid, kind, delta=0.0, params=()):
        self.g, self.kind, self.delta = g, kind, float(delta)
        ptr = ct.c_void_p()
        pa = (ct.c_double * max(1, len(params)))(*params) if params else None
        with torch.cuda.device(g.device):
            check(lib().sc_closure_create(ct.byref(ptr), g.plan, int(kind), float(delta), pa, len(params)))
        self._ptr = ptr

    @property
    def ptr(self):
        return self._ptr

    def __call__(self, u, G=None, stream=None):
        g = self.g
        tau = [torch.zeros(g.phys_shape, dtype=g.dtype, device=g.device) for _ in range(g.tensordim)]
        pu, _k1 = ptr_array([g._check_spec(c) for c in u]) if u is not None else (None, None)
        pg, _k2 = ptr_array([g._check_phys(c) for c in G]) if G is not None else (None, None)
        pt, _k3 = ptr_array([g._check_phys(c) for c in tau])
        check(lib().sc_closure_eval(self._ptr, pu, pg, pt, _stream_ptr(stream)))
        return torch.stack(tau, 0)

    def close(self):
        if getattr(self, "_ptr", None):
            with torch.cuda.device(self.g.device):
                lib().sc_closure_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_clark(delta, g: Grid):
    """``create_clark(Δ, g)`` (src/closures.jl:64)."""
    return Closure(g, CLOSURE_CLARK, delta)


def create_smagorinsky(CS, delta, g: Grid):
    """``create_smagorinsky(CS, Δ, g)`` (src/closures.jl:65-66)."""
    return Closure(g, CLOSURE_SMAGORINSKY, delta, (CS,))


def create_verstappen(C, delta, g: Grid):
    """``create_verstappen(C, Δ, g)`` (src/closures.jl:68-71); 3D only."""
    return Closure(g, CLOSURE_VERSTAPPEN, delta, (C,))


def create_dynamic_smagorinsky(delta, g: Grid):
    """``create_dynamic_smagorinsky(Δ, g)`` (src/closures.jl:188-272)."""
    return Closure(g, CLOSURE_DYNAMIC_SMAGORINSKY, delta)


def create_bardina(s, delta, g: Grid):
    """``create_bardina(s, Δ, g)`` (src/closures.jl:81-115)."""
    return Closure(g, CLOSURE_BARDINA, delta, (s,))


def kaiming_cnn_weights(seed, layers=((4, 32), (32, 32), (32, 32), (32, 6))):
    """Seeded Kaiming-normal weights (std sqrt(2 / fan_in), fan_in = 27 C_in)
    for the CNN closure, PyTorch conv3d layout (C_out, C_in, 3, 3, 3), zero biases."""
    import numpy as np
    rng = np.random.Generator(np.random.PCG64(seed))
    ws, bs = [], []
    for cin, cout in layers:
        ws.append((rng.standard_normal((cout, cin, 3, 3, 3)) * (2.0 / (27 * cin)) ** 0.5).astype(np.float32))
        bs.append(np.zeros(cout, dtype=np.float32))
    return ws, bs


def create_cnn_closure(delta, visc, g: Grid, weights, biases, mu=0.0, sigma=1.0, split=False):
    """The tensor-core CNN closure (``sc_cnn_closure_create``); FP32, 3D, n = 64 or 128.
    ``split=True`` switches it to the split precision (``SC_CLOPT_CNN_SPLIT``):
    three tensor-core passes over hi/lo operand parts per convolution, about
    FP32 accuracy."""
    import numpy as np
    ws = [np.ascontiguousarray(w, dtype=np.float32) for w in weights]
    bs = [np.ascontiguousarray(b, dtype=np.float32) for b in biases]
    FP = ct.POINTER(ct.c_float)
    wa = (FP * 4)(*[w.ctypes.data_as(FP) for w in ws])
    ba = (FP * 4)(*[b.ctypes.data_as(FP) for b in bs])
    cl = Closure.__new__(Closure)
    cl.g, cl.kind, cl.delta = g, CLOSURE_CNN, float(delta)
    ptr = ct.c_void_p()
    with torch.cuda.device(g.device):
        check(lib().sc_cnn_closure_create(ct.byref(ptr), g.plan, float(delta), float(visc), wa, ba, float(mu),
                                          float(sigma)))
    cl._ptr = ptr
    if split:
        closure_set_option(cl, SC_CLOPT_CNN_SPLIT, 1)
    return cl


def closure_set_option(cl, option, value):
    """``sc_closure_set_option``: ``SC_CLOPT_CNN_SPLIT`` (1) = 1 evaluates the
    tensor-core CNN in split precision, 0 in BF16."""
    with torch.cuda.device(cl.g.device):
        check(lib().sc_closure_set_option(cl.ptr, int(option), int(value)))


def create_cnn_fp_closure(delta, visc, g: Grid, weights, biases, mu=0.0, sigma=1.0):
    """The CNN closure on CUDA cores in the grid's precision (``sc_cnn_fp_closure_create``)."""
    import numpy as np
    ws = [np.ascontiguousarray(w, dtype=np.float32) for w in weights]
    bs = [np.ascontiguousarray(b, dtype=np.float32) for b in biases]
    FP = ct.POINTER(ct.c_float)
    wa = (FP * 4)(*[w.ctypes.data_as(FP) for w in ws])
    ba = (FP * 4)(*[b.ctypes.data_as(FP) for b in bs])
    cl = Closure.__new__(Closure)
    cl.g, cl.kind, cl.delta = g, 7, float(delta)
    ptr = ct.c_void_p()
    with torch.cuda.device(g.device):
        check(lib().sc_cnn_fp_closure_create(ct.byref(ptr), g.plan, float(delta), float(visc), wa, ba, float(mu),
                                             float(sigma)))
    cl._ptr = ptr
    return cl


CLOSURE_MLP, CLOSURE_TBNN = 8, 9


def create_mlp_closure(delta, visc, g: Grid, weights, biases, use_redelta=False, mu=0.0, sigma=1.0):
    """``fullchain(setup, mlp(...))`` (src/nets.jl:311-331): pointwise MLP closure.
    ``weights[l]``: (c_out, c_in); ``biases[l]``: (c_out,) for all layers but the last."""
    return _pointwise_net(lib().sc_mlp_closure_create, CLOSURE_MLP, delta, visc, g, weights, biases, use_redelta,
                          mu, sigma)


def create_tbnn_closure(delta, visc, g: Grid, weights, biases, use_redelta=False, mu=0.0, sigma=1.0):
    """``tbnn`` (src/nets.jl:560-588): invariants -> MLP -> tensor-basis coefficients."""
    return _pointwise_net(lib().sc_tbnn_closure_create, CLOSURE_TBNN, delta, visc, g, weights, biases, use_redelta,
                          mu, sigma)


def _pointwise_net(fn, kind, delta, visc, g: Grid, weights, biases, use_redelta, mu, sigma):
    import numpy as np
    nl = len(weights)
    widths = [int(np.shape(weights[0])[1])] + [int(np.shape(w)[0]) for w in weights]
    parts = []
    for l, w in enumerate(weights):
        parts.append(np.asarray(w, dtype=np.float64).ravel())
        if l < nl - 1:
            parts.append(np.asarray(biases[l], dtype=np.float64).ravel())
    theta = np.ascontiguousarray(np.concatenate(parts))
    wa = (ct.c_int * (nl + 1))(*widths)
    cl = Closure.__new__(Closure)
    cl.g, cl.kind, cl.delta = g, kind, float(delta)
    ptr = ct.c_void_p()
    with torch.cuda.device(g.device):
        check(fn(ct.byref(ptr), g.plan, float(delta), float(visc), nl, wa,
                 theta.ctypes.data_as(ct.POINTER(ct.c_double)), int(bool(use_redelta)), float(mu), float(sigma)))
    cl._ptr = ptr
    return cl


def closure_num_params(cl):
    n = ct.c_longlong()
    check(lib().sc_closure_num_params(cl.ptr, ct.byref(n)))
    return n.value


def closure_set_params(cl, theta):
    import numpy as np
    th = np.ascontiguousarray(theta, dtype=np.float64)
    check(lib().sc_closure_set_params(cl.ptr, th.ctypes.data_as(ct.POINTER(ct.c_double))))


def pack_cnn_params(weights, biases):
    """Flat parameter vector [w1, b1, ..., w4, b4] of ``sc_closure_set_params``."""
    import numpy as np
    return np.concatenate([np.concatenate([np.ravel(w), np.ravel(b)]) for w, b in zip(weights, biases)]).astype(np.float64)


def rollout_record(g: Grid, cl, u0, dt, visc, nsteps, stream=None):
    """Trajectory of ``nsteps`` RK4 steps (compact states on the device)."""
    nb = lib().sc_rollout_traj_bytes(g.plan, int(nsteps))
    traj = torch.empty(nb, dtype=torch.uint8, device=g.device)
    pu, _k = ptr_array([g._check_spec(c) for c in u0])
    check(lib().sc_rollout_record(g.plan, _cl(cl), pu, float(dt), float(visc), int(nsteps),
                                  ct.c_void_p(traj.data_ptr()), _stream_ptr(stream)))
    return traj


def rollout_loss(g: Grid, cl, u0, traj, dt, visc, nsteps, stream=None):
    pu, _k = ptr_array([g._check_spec(c) for c in u0])
    out = ct.c_double()
    check(lib().sc_rollout_loss(g.plan, _cl(cl), pu, ct.c_void_p(traj.data_ptr()), float(dt), float(visc),
                                int(nsteps), ct.byref(out), _stream_ptr(stream)))
    return out.value


def rollout_adjoint(g: Grid, cl, u0, traj, dt, visc, nsteps, ckpt_every=5, stream=None):
    """(loss, dloss/dtheta) of the trajectory MSE by the hand-written adjoint."""
    import numpy as np
    pu, _k = ptr_array([g._check_spec(c) for c in u0])
    grad = np.zeros(closure_num_params(cl), dtype=np.float64)
    out = ct.c_double()
    check(lib().sc_rollout_adjoint(g.plan, _cl(cl), pu, ct.c_void_p(traj.data_ptr()), float(dt), float(visc),
                                   int(nsteps), int(ckpt_every), ct.byref(out),
                                   grad.ctypes.data_as(ct.POINTER(ct.c_double)), _stream_ptr(stream)))
    return out.value, grad


def rollout_adjoint_batch(jobs, stream=None):
    """Several training rollouts at once (``sc_rollout_adjoint_batch``): each job is a
    dict(grid, closure, u0, traj, dt, visc, nsteps, ckpt_every); returns a list of
    (loss, dloss/dtheta).  Jobs run concurrently, one stream each; every job needs
    its own grid (plan) and closure."""
    import numpy as np
    from ._lib import sc_rollout_job
    n = len(jobs)
    arr = (sc_rollout_job * n)()
    keep, outs = [], []
    for i, j in enumerate(jobs):
        g = j["grid"]
        u0 = [g._check_spec(c) for c in j["u0"]]  # device addresses (validated)
        keep.append(j["u0"])
        grad = np.zeros(closure_num_params(j["closure"]), dtype=np.float64)
        loss = ct.c_double()
        outs.append((loss, grad))
        J = arr[i]
        J.plan, J.closure = g.plan, _cl(j["closure"])
        for c in range(3):
            J.u0[c] = u0[c] if c < len(u0) else None
        J.traj = j["traj"].data_ptr()
        J.dt, J.visc = float(j["dt"]), float(j["visc"])
        J.nsteps, J.ckpt_every = int(j["nsteps"]), int(j.get("ckpt_every", 5))
        J.loss = ct.pointer(loss)
        J.grad = grad.ctypes.data_as(ct.POINTER(ct.c_double))
    status = (ct.c_int * n)()
    check(lib().sc_rollout_adjoint_batch(n, arr, status, _stream_ptr(stream)))
    return [(l.value, g) for l, g in outs]


def _cl(model):
    return model.ptr if model is not None else None


def les_(du, u, g: Grid, model, visc, stream=None):
    """``les!(du, u, grid, cache; model, visc)`` (src/les.jl:4-33), retained modes."""
    pu, _k1 = ptr_array([g._check_spec(c) for c in u])
    pd, _k2 = ptr_array([g._check_spec(c) for c in du])
    check(lib().sc_les_rhs(g.plan, _cl(model), pu, pd, float(visc), _stream_ptr(stream)))
    return du


def les_wray3_(u, dt, g: Grid, model, visc, stream=None):
    """``wray3!(les!, u, Δt, grid, cache; model, visc)`` (src/les.jl:216-219)."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    check(lib().sc_les_wray3_step(g.plan, _cl(model), pu, float(dt), float(visc), _stream_ptr(stream)))
    return u


def les_rk4_(u, dt, g: Grid, model, visc, nsteps=1, eps=None, stream=None):
    """RK4 steps of the LES with closure ``model`` (new)."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    f = sc_forcing(1 if eps is not None else 0, float(eps) if eps is not None else 0.0)
    check(lib().sc_les_rk4_steps(g.plan, _cl(model), pu, float(dt), float(visc), int(nsteps), ct.byref(f),
                                 _stream_ptr(stream)))
    return u


class LesBatch:
    """Batched LES (``sc_les_batch_*``): instances = list of dicts with keys
    ``grid`` (its State already loaded), ``closure`` (or None), ``visc``, ``dt``,
    ``eps`` (None = unforced).  One CUDA graph advances all of them per step."""

    def __init__(self, instances):
        n = len(instances)
        arr = (sc_les_instance * n)()
        for i, d in enumerate(instances):
            eps = d.get("eps")
            arr[i] = sc_les_instance(d["grid"].plan.value, _cl(d.get("closure")).value if d.get("closure") else None,
                                     float(d["visc"]), float(d["dt"]), 1 if eps is not None else 0,
                                     float(eps or 0.0))
        self.n = n
        self.instances = instances
        ptr = ct.c_void_p()
        check(lib().sc_les_batch_create(ct.byref(ptr), arr, n))
        self._ptr = ptr

    def run(self, nsteps, stream=None):
        check(lib().sc_les_batch_run(self._ptr, int(nsteps), _stream_ptr(stream)))

    def status(self, freeze=False, stream=None):
        st = (ct.c_int * self.n)()
        en = (ct.c_double * self.n)()
        check(lib().sc_les_batch_status(self._ptr, st, en, 1 if freeze else 0, _stream_ptr(stream)))
        return list(st), list(en)

    def set_snapshots(self, every, nshell, max_snap):
        """Fuse reduce!'s reductions (src/les.jl:94-148) into the stepper: every
        `every` steps, record each instance's ke, eps_visc, eps_sfs, spectrum and
        shell transfer on the device (``sc_les_batch_set_snapshots``)."""
        self.nshell = int(nshell)
        check(lib().sc_les_batch_set_snapshots(self._ptr, int(every), int(nshell), int(max_snap)))

    def snapshots(self, stream=None):
        """The record so far: a list over snapshots of a list over instances of
        dicts (ke, eps_visc, eps_sfs, spectrum, transfer)."""
        import numpy as np
        ns = ct.c_int()
        check(lib().sc_les_batch_snapshots(self._ptr, ct.byref(ns), None, _stream_ptr(stream)))
        if ns.value == 0:
            return []
        stride = 3 + 2 * self.nshell
        buf = np.zeros(ns.value * self.n * stride, dtype=np.float64)
        check(lib().sc_les_batch_snapshots(self._ptr, ct.byref(ns), buf.ctypes.data_as(ct.POINTER(ct.c_double)),
                                           _stream_ptr(stream)))
        rec = buf.reshape(ns.value, self.n, stride)
        return [[{"ke": r[0], "eps_visc": r[1], "eps_sfs": r[2], "spectrum": r[3:3 + self.nshell].copy(),
                  "transfer": r[3 + self.nshell:].copy()} for r in snap] for snap in rec]

    def close(self):
        if getattr(self, "_ptr", None):
            lib().sc_les_batch_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_field(g: Grid, seed=0, kpeak=4.0, totalenergy=1.0, draws=None, out=None, stream=None):
    """``randomfield(peak_profile, g; kpeak, totalenergy)`` (src/solver.jl:576-641) on
    the device (``sc_random_field``).  The field becomes the plan's state; it is
    also returned in the full layout (``out`` or new tensors).  ``draws``:
    complex128 device tensors of the normal coefficients on the compact 2/3
    cube (``fields.compact_shape``), or None for the device generator (seed)."""
    out = vectorfield(g) if out is None else out
    pd, _k1 = ptr_array([c.data_ptr() for c in draws]) if draws is not None else (None, None)
    po, _k2 = ptr_array([g._check_spec(c) for c in out])
    check(lib().sc_random_field(g.plan, int(seed), pd, float(kpeak), float(totalenergy), po, _stream_ptr(stream)))
    return out


def set_option(g: Grid, option, value):
    """``sc_plan_set_option``: ``SC_OPT_USE_GRAPH`` (1) replays captured CUDA
    graphs in the steppers (default) or launches eagerly (0);
    ``SC_OPT_WAIT_LIMIT`` (2) bounds the device waits of the tensor-core CNN
    and of the TMA-fed column sweeps (polls; negative: the default);
    ``SC_OPT_VARIANT_*`` (3..7) pick a sweep's kernel variant (``autotune``)."""
    check(lib().sc_plan_set_option(g.plan, int(option), int(value)))


def plan_status(g: Grid):
    """``sc_plan_status``: SC_ERR_TIMEOUT (7) if a bounded wait of the plan's
    TMA-fed column sweeps ran out since the last call, else 0 (synchronous;
    reading clears the record)."""
    st = ct.c_int()
    check(lib().sc_plan_status(g.plan, ct.byref(st)))
    return st.value


def propose_timestep(u, g: Grid, visc, stream=None):
    """``propose_timestep(u, grid, visc, cache)`` (src/solver.jl:931-947)."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    out = ct.c_double()
    check(lib().sc_propose_timestep(g.plan, pu, float(visc), ct.byref(out), _stream_ptr(stream)))
    return out.value


def energy_shells(g: Grid, u, stream=None):
    """``energy_shells(grid, [1, 2], u)`` (src/solver.jl:1135-1140): reference shell energies."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    e = (ct.c_double * 2)()
    check(lib().sc_shell_energies(g.plan, pu, e, _stream_ptr(stream)))
    return [e[0], e[1]]


def maintain_shell_energy_(u, eref, g: Grid, stream=None):
    """``maintain_shell_energy!(u, shells)`` (src/solver.jl:1146-1152) for shells 1 and 2."""
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    e = (ct.c_double * 2)(*eref)
    check(lib().sc_maintain_shell_energy(g.plan, pu, e, _stream_ptr(stream)))
    return u


def spectrum(u, g: Grid, nshell=None, stream=None):
    """``spectrum(u, grid)`` (src/solver.jl:693-699) on shells 1..nshell (default n÷3)."""
    nshell = nshell or g.n // 3
    pu, _k = ptr_array([g._check_spec(c) for c in u])
    s = (ct.c_double * nshell)()
    check(lib().sc_spectrum(g.plan, pu, int(nshell), s, _stream_ptr(stream)))
    return list(s)


def les_diagnostics(u, g: Grid, model=None, uref=None, visc=0.0, nshell=None, stream=None):
    """The a-posteriori reductions of ``solve_les!``'s ``reduce!`` (src/les.jl:94-148):
    dict(e_post, ke, eps_visc, eps_sfs, spectrum, transfer)."""
    nshell = nshell or g.n // 3
    pu, _k1 = ptr_array([g._check_spec(c) for c in u])
    pr, _k2 = ptr_array([g._check_spec(c) for c in uref]) if uref is not None else (None, None)
    out = (ct.c_double * 4)()
    spec = (ct.c_double * nshell)()
    tr = (ct.c_double * nshell)()
    check(lib().sc_les_diagnostics(g.plan, _cl(model), pu, pr, float(visc), int(nshell), out, spec, tr,
                                   _stream_ptr(stream)))
    return dict(e_post=out[0], ke=out[1], eps_visc=out[2], eps_sfs=out[3], spectrum=list(spec), transfer=list(tr))


def turbulence_statistics(u, visc, g: Grid):
    """``turbulence_statistics`` (src/solver.jl:836-852) from the device FP64 reductions."""
    e = energy(u, g)
    diss = get_dissipation(u, visc, g)
    uavg = math.sqrt(2 * e / g.D)
    l_kol = (visc ** 3 / diss) ** 0.25
    l_tay = math.sqrt(15 * visc / diss) * uavg
    l_int = uavg ** 3 / diss
    return dict(e=e, uavg=uavg, diss=diss, l_int=l_int, l_tay=l_tay, l_kol=l_kol, t_int=l_int / uavg,
                t_tay=l_tay / uavg, t_kol=math.sqrt(visc / diss), Re_int=l_int * uavg / visc,
                Re_tay=l_tay * uavg / visc, kmax_eta=(math.pi * g.n / g.l) * l_kol)


class State:
    """Device-resident compact state of a plan (sc_state_* entry points)."""

    def __init__(self, g: Grid):
        self.g = g

    def load(self, u, stream=None):
        pu, _k = ptr_array([self.g._check_spec(c) for c in u])
        check(lib().sc_state_load(self.g.plan, pu, _stream_ptr(stream)))

    def store(self, u, stream=None):
        pu, _k = ptr_array([self.g._check_spec(c) for c in u])
        check(lib().sc_state_store(self.g.plan, pu, _stream_ptr(stream)))

    def rk4(self, dt, visc, nsteps=1, eps=None, stream=None):
        f = sc_forcing(1 if eps is not None else 0, float(eps) if eps is not None else 0.0)
        check(lib().sc_state_rk4(self.g.plan, float(dt), float(visc), int(nsteps), ct.byref(f), _stream_ptr(stream)))

    def energy(self, stream=None):
        out = ct.c_double()
        check(lib().sc_state_energy(self.g.plan, ct.byref(out), _stream_ptr(stream)))
        return out.value

    def profile_rhs(self, visc, reps=3, stream=None):
        """Mean ms per kernel of one right-hand side (sc_state_profile_rhs)."""
        ms = (ct.c_double * 8)()
        nk = ct.c_int()
        check(lib().sc_state_profile_rhs(self.g.plan, float(visc), int(reps), ms, ct.byref(nk), _stream_ptr(stream)))
        return list(ms[: nk.value])

    def les_rk4(self, model, dt, visc, nsteps=1, eps=None, stream=None):
        f = sc_forcing(1 if eps is not None else 0, float(eps) if eps is not None else 0.0)
        check(lib().sc_state_les_rk4(self.g.plan, _cl(model), float(dt), float(visc), int(nsteps), ct.byref(f),
                                     _stream_ptr(stream)))

    def launches_per_step(self, forced):
        return lib().sc_state_rk4_launches_per_step(self.g.plan, 1 if forced else 0)
