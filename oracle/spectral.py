"""Grid, spectral point kernels, NS right-hand side, steppers, forcing, initial
fields and diagnostics: FP64 restatement of ``src/solver.jl`` (reference).

Test infrastructure only (see ``oracle/__init__.py``).

Layout: a spectral scalar field of a ``D``-dimensional grid with ``n`` points
per side is a complex128 array of shape ``(n, n/2+1)`` (2D) or
``(n, n, n/2+1)`` (3D), indexed ``[iy, ix]`` / ``[iz, iy, ix]``; this is the
memory layout of the reference's column-major ``(n/2+1, n[, n])`` arrays.  A
vector field is a list of ``D`` such arrays (x, y[, z]); a symmetric tensor
field is a list in the reference's order xx, yy, zz, xy, yz, zx (3D) or
xx, yy, xy (2D).
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

__all__ = [
    "Grid", "WORKERS", "wavenumbers_int", "wavenumbers_full", "k2_int", "k2_full",
    "to_phys", "to_spec", "dealias_phys", "twothirds", "project", "symmetrize",
    "nonlinearity", "viscosity", "stress", "tensordivergence", "vectordivergence",
    "convectiondiffusion", "wray3", "forwardeuler", "propose_timestep",
    "band_mask", "band_energy", "linear_forcing_coeff", "rk4_step", "rk4_rhs",
    "energy", "getenergy", "spectralsum", "get_dissipation", "energy_shells",
    "maintain_shell_energy", "peak_profile", "random_field", "random_field_compact",
    "retained_shape", "pack_retained", "unpack_retained", "vectorgradient",
    "strainrate", "make_tracefree", "turbulence_statistics", "taylorgreen",
    "pairs", "rel_l2", "SYM_PAIRS_3D", "SYM_PAIRS_2D", "spectrum",
]

WORKERS = int(os.environ.get("SC_ORACLE_WORKERS", os.cpu_count() or 1))

SYM_PAIRS_3D = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]  # xx yy zz xy yz zx
SYM_PAIRS_2D = [(0, 0), (1, 1), (0, 1)]  # xx yy xy


def pairs(D):
    """Symmetric-tensor component order (``tensorfield``, src/solver.jl:254-262)."""
    return SYM_PAIRS_3D if D == 3 else SYM_PAIRS_2D


@dataclass(frozen=True)
class Grid:
    """Periodic box ``[0, l)^D`` with ``n`` points per side (src/solver.jl:131-151).

    ``n`` must be even, exactly as ``Grid{D}(; l, n)`` asserts (src/solver.jl:148).
    """

    D: int
    n: int
    l: float = 2 * math.pi

    def __post_init__(self):
        if self.n % 2 != 0:
            raise AssertionError("Only even number of grid points supported.")
        if self.D not in (2, 3):
            raise ValueError("D must be 2 or 3")

    @property
    def tensordim(self):  # src/solver.jl:159-160
        return 3 if self.D == 2 else 6

    @property
    def spacing(self):  # src/solver.jl:163
        return self.l / self.n

    @property
    def volume(self):  # src/solver.jl:166
        return (self.l / self.n) ** self.D

    @property
    def ndrange(self):
        """Julia-order spectral shape ``(n/2+1, n[, n])`` (src/solver.jl:198-199)."""
        return (self.n // 2 + 1,) + (self.n,) * (self.D - 1)

    @property
    def space_ndrange(self):  # src/solver.jl:202
        return (self.n,) * self.D

    @property
    def spec_shape(self):
        """numpy C-order shape with the same memory layout as ``ndrange``."""
        return tuple(reversed(self.ndrange))

    @property
    def phys_shape(self):
        return (self.n,) * self.D

    @property
    def kcut(self):  # src/solver.jl:374
        return self.n // 3

    @property
    def fft_fac(self):  # get_fft_fac, src/solver.jl:207
        return self.n ** self.D


def _fftfreq_int(n):
    """``fftfreq_int`` (src/solver.jl:167): 0..n/2-1, -n/2..-1."""
    i = np.arange(n)
    return np.where(i <= (n - 1) // 2, i, i - n)


def wavenumbers_int(g: Grid):
    """Broadcastable integer wavenumbers (kx, ky[, kz]) (src/solver.jl:170-172)."""
    kx = np.arange(g.n // 2 + 1)
    ky = _fftfreq_int(g.n)
    if g.D == 2:
        return kx[None, :], ky[:, None]
    return kx[None, None, :], ky[None, :, None], ky[:, None, None]


def wavenumbers_full(g: Grid):
    """``2π/l`` times the integer wavenumbers (src/solver.jl:178-184)."""
    f = 2 * math.pi / g.l
    return tuple(f * k.astype(np.float64) for k in wavenumbers_int(g))


def k2_int(g: Grid):
    ks = wavenumbers_int(g)
    return sum(k * k for k in ks)


def k2_full(g: Grid):
    ks = wavenumbers_full(g)
    return sum(k * k for k in ks)


# --------------------------------------------------------------------------
# FFT wrappers (src/solver.jl:204-232)
# --------------------------------------------------------------------------

def to_phys(spec, g: Grid):
    """``to_phys!``: unnormalised inverse RFFT (``ldiv!`` times ``n^D``), src/solver.jl:210-211."""
    return sfft.irfftn(spec, s=g.phys_shape, norm="forward", workers=WORKERS)


def to_spec(phys, g: Grid):
    """``to_spec!``: RFFT divided by ``n^D``, src/solver.jl:214-215."""
    return sfft.rfftn(phys, norm="forward", workers=WORKERS)


def dealias_phys(phys, g: Grid):
    """``dealias_phys!`` (src/solver.jl:218-223): r2c, 2/3 rule, normalised c2r.

    The reference runs ``mul!`` (unscaled forward) then ``ldiv!`` (inverse
    divided by ``n^D``) so the two scalings cancel.
    """
    spec = sfft.rfftn(phys, workers=WORKERS)
    spec = twothirds(spec, g)
    return sfft.irfftn(spec, s=g.phys_shape, workers=WORKERS)


# --------------------------------------------------------------------------
# Spectral point kernels
# --------------------------------------------------------------------------

def _retained_mask(g: Grid):
    ks = wavenumbers_int(g)
    kc = g.kcut
    m = np.ones(g.spec_shape, dtype=bool)
    for k in ks:
        m &= np.abs(k) <= kc
    nonzero = np.zeros(g.spec_shape, dtype=bool)
    for k in ks:
        nonzero |= k != 0
    return m & nonzero


def twothirds(u, g: Grid):
    """``twothirds!`` (src/solver.jl:371-389): keep |k_i| <= n÷3 for all i, and zero k = 0."""
    return np.where(_retained_mask(g), u, 0)


def project(u, g: Grid):
    """``project!`` (src/solver.jl:350-368): Leray projection, k = 0 left intact."""
    ks = wavenumbers_full(g)
    k2 = sum(k * k for k in ks)
    kdotu = sum(k * c for k, c in zip(ks, u))
    with np.errstate(invalid="ignore", divide="ignore"):
        p = kdotu / k2
    zero = np.zeros(g.spec_shape, dtype=bool)
    zero[(0,) * g.D] = True
    p = np.where(zero, 0, p)
    return [c - k * p for k, c in zip(ks, u)]


def symmetrize(u, g: Grid):
    """``symmetrize!`` (src/solver.jl:398-430): Hermitian fix on the kx = 0 and kx = n/2 planes.

    On those planes each mode whose partner ``(-ky, -kz)`` comes earlier in
    (iy, iz) lexicographic order copies the partner's conjugate; self-conjugate
    modes keep only their real part.
    """
    n = g.n
    out = np.array(u, copy=True)
    idx = np.arange(n)
    pidx = (-idx) % n  # partner index: n+2-i (1-based) except the self-conjugate 0 and n/2
    for ix in (0, n // 2):
        if g.D == 2:
            P = u[:, ix]
            Q = P.copy()
            selfm = pidx == idx
            write = idx > pidx
            Q[write] = np.conj(P[pidx[write]])
            Q[selfm] = P[selfm].real
            out[:, ix] = Q
        else:
            P = u[:, :, ix]  # [iz, iy]
            Q = P.copy()
            iz, iy = np.meshgrid(idx, idx, indexing="ij")
            piz, piy = pidx[iz], pidx[iy]
            selfm = (iy == piy) & (iz == piz)
            write = (iy > piy) | ((iy == piy) & (iz > piz))
            Q[write] = np.conj(P[piz[write], piy[write]])
            Q[selfm] = P[selfm].real
            out[:, :, ix] = Q
    return out


def vectordivergence(u, g: Grid):
    """``vectordivergence!`` (src/solver.jl:484-493)."""
    ks = wavenumbers_full(g)
    return sum(1j * k * c for k, c in zip(ks, u))


def nonlinearity(u, g: Grid):
    """``nonlinearity!`` (src/solver.jl:434-456).

    ``σ_ij = F[(P u_i)(P u_j)] / n^D`` for the symmetric pairs, with P the 2/3
    rule; the outputs are *not* truncated.
    """
    v = [to_phys(twothirds(c, g), g) for c in u]
    return [to_spec(v[i] * v[j], g) for (i, j) in pairs(g.D)]


def viscosity(sigma, u, visc, g: Grid):
    """``viscosity!`` (src/solver.jl:458-476): σ_ij -= ν i (k_j u_i + k_i u_j) on unmasked u."""
    ks = wavenumbers_full(g)
    out = []
    for s, (i, j) in zip(sigma, pairs(g.D)):
        if i == j:
            out.append(s - 2 * visc * 1j * ks[i] * u[i])
        else:
            out.append(s - visc * 1j * (ks[j] * u[i] + ks[i] * u[j]))
    return out


def stress(u, visc, g: Grid):
    """``stress!`` (src/solver.jl:478-482)."""
    return viscosity(nonlinearity(u, g), u, visc, g)


def _sym_index(D):
    pr = pairs(D)
    idx = {}
    for c, (i, j) in enumerate(pr):
        idx[(i, j)] = c
        idx[(j, i)] = c
    return idx


def tensordivergence(sigma, g: Grid):
    """``tensordivergence!`` (src/solver.jl:509-521): du_i = -i k_j σ_ij."""
    ks = wavenumbers_full(g)
    idx = _sym_index(g.D)
    return [sum(-1j * ks[j] * sigma[idx[(i, j)]] for j in range(g.D)) for i in range(g.D)]


def convectiondiffusion(u, g: Grid, visc):
    """``convectiondiffusion!`` (src/solver.jl:949-953)."""
    return tensordivergence(stress(u, visc, g), g)


def forwardeuler(f, u, g: Grid, dt, **kw):
    """``forwardeuler!`` (src/solver.jl:894-901)."""
    du = f(u, g, **kw)
    return project([c + dt * d for c, d in zip(u, du)], g)


def wray3(f, u, dt, g: Grid, **kw):
    """``wray3!`` (src/solver.jl:968-1012): low-storage Wray RK3, projecting after each stage."""
    a = (8 / 15, 5 / 12, 3 / 4)
    b = (1 / 4, 0.0)
    ustart = [c.copy() for c in u]
    u = [c.copy() for c in u]
    for i in range(3):
        du = f(u, g, **kw)
        if i > 0:
            u = [c.copy() for c in ustart]
        u = [c + a[i] * dt * d for c, d in zip(u, du)]
        u = project(u, g)
        if i < 2:
            ustart = [c + b[i] * dt * d for c, d in zip(ustart, du)]
    return u


def propose_timestep(u, g: Grid, visc):
    """``propose_timestep`` (src/solver.jl:931-947): CFL-type bound (times ``cfl`` by the caller)."""
    v = [to_phys(twothirds(c, g), g) for c in u]
    vmax = np.sqrt(sum(c * c for c in v)).max()
    h = g.l / g.n
    return min(h / vmax, h * h / g.D / 2 / visc)


# --------------------------------------------------------------------------
# Energy, dissipation, shells (src/solver.jl:643-811, 1080-1152)
# --------------------------------------------------------------------------

def getenergy(c):
    """``getenergy`` (src/solver.jl:702): Σ|û|² counting interior kx twice."""
    K = c.shape[-1]
    return float(np.sum(np.abs(c) ** 2) + np.sum(np.abs(c[..., 1:K - 1]) ** 2))


def spectralsum(f, c):
    """``spectralsum`` (src/solver.jl:705)."""
    K = c.shape[-1]
    return f(c).sum() + f(c[..., 1:K - 1]).sum()


def energy(u):
    """``energy`` (src/solver.jl:643-646): ½ Σ_i getenergy(u_i)."""
    return sum(getenergy(c) for c in u) / 2


def get_dissipation(u, visc, g: Grid):
    """``get_dissipation!`` (src/solver.jl:808-811): ν Σ k²|û|² with the RFFT double count."""
    k2 = k2_full(g)
    d = visc * k2 * sum(np.abs(c) ** 2 for c in u)
    K = d.shape[-1]
    return float(d.sum() + d[..., 1:K - 1].sum())


def turbulence_statistics(u, visc, g: Grid):
    """3D K41 statistics (src/solver.jl:836-852)."""
    u = [twothirds(c, g) for c in u]
    e = sum(getenergy(c) for c in u) / 2
    diss = get_dissipation(u, visc, g)
    uavg = math.sqrt(2 * e / g.D)
    l_kol = (visc ** 3 / diss) ** 0.25
    l_tay = math.sqrt(15 * visc / diss) * uavg
    l_int = uavg ** 3 / diss
    return dict(e=e, uavg=uavg, diss=diss, l_int=l_int, l_tay=l_tay, l_kol=l_kol,
                t_int=l_int / uavg, t_tay=l_tay / uavg, t_kol=math.sqrt(visc / diss),
                Re_int=l_int * uavg / visc, Re_tay=l_tay * uavg / visc,
                kmax_eta=(math.pi * g.n / g.l) * l_kol)


def _shell_masks(g: Grid, i):
    k2 = k2_int(g)
    inds = (k2 >= i * i) & (k2 < (i + 1) * (i + 1))
    K = g.n // 2 + 1
    interior = np.zeros(g.spec_shape, dtype=bool)
    interior[..., 1:K - 1] = True
    return inds, inds & interior


def energy_shells(g: Grid, shells, u):
    """``energy_shells`` (src/solver.jl:1135-1140) with ``getshells`` (src/solver.jl:1080-1129)."""
    out = []
    for i in shells:
        inds, conj = _shell_masks(g, i)
        eref = sum(np.sum(np.abs(c[inds]) ** 2) + np.sum(np.abs(c[conj]) ** 2) for c in u) / 2
        out.append((inds, conj, float(eref)))
    return out


def maintain_shell_energy(u, shells):
    """``maintain_shell_energy!`` (src/solver.jl:1146-1152)."""
    u = [c.copy() for c in u]
    for inds, conj, eref in shells:
        es = sum(np.sum(np.abs(c[inds]) ** 2) + np.sum(np.abs(c[conj]) ** 2) for c in u) / 2
        f = math.sqrt(eref / es)
        for c in u:
            c[inds] *= f
    return u


def spectrum(u, g: Grid, nshell=None):
    """``spectrum`` with ``spectral_stuff`` shells 1..n÷3 (src/solver.jl:664-699):
    s_i = ½ Σ_{i <= |k| < i+1} |û|² over the RFFT array plus the conjugate interior."""
    nshell = nshell or g.n // 3
    k2 = k2_int(g)
    K = g.n // 2 + 1
    w = np.ones(g.spec_shape)
    w[..., 1:K - 1] = 2.0
    e = sum(np.abs(c) ** 2 for c in u) * w / 2
    out = []
    for i in range(1, nshell + 1):
        m = (k2 >= i * i) & (k2 < (i + 1) * (i + 1))
        out.append(float(e[m].sum()))
    return out


# --------------------------------------------------------------------------
# RK4 with linear band forcing (new stepper; no reference counterpart)
# --------------------------------------------------------------------------

def band_mask(g: Grid, kmin2=1, kmax2=9):
    """Forced band ``1 <= |k|^2 < 9`` (integer k): shells 1 and 2, the modes
    ``maintain_shell_energy!`` clamps in the reference (src/data.jl:49,65)."""
    k2 = k2_int(g)
    return (k2 >= kmin2) & (k2 < kmax2)


def band_energy(u, g: Grid):
    """½ Σ_band |û|², interior kx counted twice (as ``getenergy``)."""
    m = band_mask(g)
    K = g.n // 2 + 1
    w = np.ones(g.spec_shape)
    w[..., 1:K - 1] = 2.0
    return float(sum(np.sum((w * np.abs(c) ** 2)[m]) for c in u) / 2)


def linear_forcing_coeff(u, g: Grid, eps):
    """A = ε / (2 E_f): the band forcing f = A û injects energy at rate ε."""
    ef = band_energy(u, g)
    return eps / (2 * ef) if ef > 0 else 0.0


def rk4_rhs(u, g: Grid, visc, eps=None):
    """RK4 stage derivative: P(twothirds(convectiondiffusion(u))) + A u|band.

    The truncation keeps the state inside the 2/3 cube; the retained modes are
    those of the reference's untruncated state (aliased modes never feed back:
    every product input is truncated and the other terms are diagonal in k).
    """
    du = convectiondiffusion(u, g, visc)
    du = project([twothirds(c, g) for c in du], g)
    if eps is not None:
        A = linear_forcing_coeff(u, g, eps)
        m = band_mask(g)
        du = [d + np.where(m, A * c, 0) for d, c in zip(du, u)]
    return du


def rk4_step(u, dt, g: Grid, visc, eps=None):
    """Classical RK4: u_{n+1} = P(u_n + dt/6 (k1 + 2k2 + 2k3 + k4)) with projected stage derivatives."""
    k1 = rk4_rhs(u, g, visc, eps)
    k2 = rk4_rhs([c + 0.5 * dt * d for c, d in zip(u, k1)], g, visc, eps)
    k3 = rk4_rhs([c + 0.5 * dt * d for c, d in zip(u, k2)], g, visc, eps)
    k4 = rk4_rhs([c + dt * d for c, d in zip(u, k3)], g, visc, eps)
    return [c + dt / 6 * (a + 2 * b + 2 * cc + d) for c, a, b, cc, d in zip(u, k1, k2, k3, k4)]


# --------------------------------------------------------------------------
# Initial conditions (src/solver.jl:523-641)
# --------------------------------------------------------------------------

def peak_profile(k, kpeak):
    """``peak_profile`` (src/solver.jl:523)."""
    return k ** 4 * math.exp(-2 * (k / kpeak) ** 2)


def retained_shape(D, n):
    """Compact 2/3-cube shape, numpy C-order: (K2, K2, K1) or (K2, K1),
    K1 = n÷3 + 1 (kx = 0..n÷3), K2 = 2(n÷3) + 1 (k = 0..n÷3 then -n÷3..-1)."""
    k = n // 3
    return (2 * k + 1,) * (D - 1) + (k + 1,)


def _compact_to_fft_index(n):
    k = n // 3
    p = np.arange(2 * k + 1)
    return np.where(p <= k, p, p + n - (2 * k + 1))


def pack_retained(c, g: Grid):
    """Gather the 2/3 cube (kx <= n÷3, |ky|,|kz| <= n÷3) into the compact layout."""
    f = _compact_to_fft_index(g.n)
    k = g.n // 3
    if g.D == 2:
        return np.ascontiguousarray(c[np.ix_(f, np.arange(k + 1))])
    return np.ascontiguousarray(c[np.ix_(f, f, np.arange(k + 1))])


def unpack_retained(cc, g: Grid):
    """Scatter a compact 2/3 cube back to the full RFFT layout (zeros elsewhere)."""
    out = np.zeros(g.spec_shape, dtype=cc.dtype)
    f = _compact_to_fft_index(g.n)
    k = g.n // 3
    if g.D == 2:
        out[np.ix_(f, np.arange(k + 1))] = cc
    else:
        out[np.ix_(f, f, np.arange(k + 1))] = cc
    return out


def random_field_compact(D, n, seed, kpeak=4.0, totalenergy=1.0, profile=None, dtype=np.complex128):
    """Seeded solenoidal random field with shell spectrum E(k) ∝ profile(k), compact 2/3 layout.

    Follows ``randomfield`` (src/solver.jl:576-641) step by step -- complex
    normal draws, ``symmetrize!``, ``project!``, ``twothirds!``, per-shell
    rescale of ``kleft <= |k| < kleft+1`` to ``totalenergy·profile/Σprofile``
    over ``0..floor(√D·n/2)``, ``twothirds!`` -- but draws only on the retained
    2/3 cube (the reference's draws outside it are zeroed by ``twothirds!``)
    with numpy ``PCG64(seed)``: per component x, y[, z], re then im, each
    N(0, ½) (Julia complex ``randn``), over the compact array in C order.
    Julia's Xoshiro stream is not reproduced: oracle and CUDA path consume the
    same bytes.
    """
    if profile is None:
        def profile(k):
            return peak_profile(k, kpeak)
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = retained_shape(D, n)
    s = math.sqrt(0.5)
    u = []
    for _ in range(D):
        re = rng.standard_normal(shape)
        im = rng.standard_normal(shape)
        u.append((re + 1j * im) * s)
    k = n // 3
    K2 = 2 * k + 1
    pidx = np.concatenate([[0], np.arange(K2 - 1, 0, -1)])  # compact index of -k
    idx = np.arange(K2)
    # symmetrize! on the kx = 0 plane (kx = n/2 is outside the 2/3 cube)
    for c in u:
        if D == 2:
            P = c[:, 0].copy()
            fy = _compact_to_fft_index(n)
            write = fy > ((-fy) % n)
            Q = P.copy()
            Q[write] = np.conj(P[pidx[write]])
            Q[idx == 0] = P[0].real
            c[:, 0] = Q
        else:
            P = c[:, :, 0].copy()
            fy = _compact_to_fft_index(n)
            FZ, FY = np.meshgrid(fy, fy, indexing="ij")
            PFZ, PFY = (-FZ) % n, (-FY) % n
            write = (FY > PFY) | ((FY == PFY) & (FZ > PFZ))
            IZ, IY = np.meshgrid(idx, idx, indexing="ij")
            Q = P.copy()
            Q[write] = np.conj(P[pidx[IZ[write]], pidx[IY[write]]])
            Q[0, 0] = P[0, 0].real
            c[:, :, 0] = Q
    # wavenumbers on the compact cube
    kk = np.where(idx <= k, idx, idx - K2).astype(np.float64)
    kxs = np.arange(k + 1, dtype=np.float64)
    if D == 2:
        KS = [kxs[None, :], kk[:, None]]
    else:
        KS = [kxs[None, None, :], kk[None, :, None], kk[:, None, None]]
    k2 = sum(a * a for a in KS)
    with np.errstate(invalid="ignore", divide="ignore"):
        p = sum(a * c for a, c in zip(KS, u)) / k2
    p.flat[0] = 0
    u = [c - a * p for a, c in zip(KS, u)]
    for c in u:  # twothirds!: zero k = 0
        c.flat[0] = 0
    # per-shell rescale
    w = np.ones(shape)
    w[..., 1:] = 2.0  # interior kx double count (kx = n/2 is not retained)
    E = sum(np.abs(c) ** 2 for c in u) / 2
    k2i = np.rint(k2).astype(np.int64)
    shell = np.floor(np.sqrt(k2i)).astype(np.int64)
    # guard floating sqrt at perfect squares
    shell = np.where((shell + 1) ** 2 <= k2i, shell + 1, shell)
    shell = np.where(shell ** 2 > k2i, shell - 1, shell)
    kdiag = int(math.floor(math.sqrt(D) * (n // 2)))
    prof = np.array([profile(kk_) for kk_ in range(kdiag + 1)])
    eshell = np.bincount(shell.ravel(), weights=(w * E).ravel(), minlength=kdiag + 1)
    e0 = totalenergy * prof / prof.sum()
    with np.errstate(invalid="ignore", divide="ignore"):
        fac = np.where(eshell[: kdiag + 1] > 0, np.sqrt(e0 / eshell[: kdiag + 1]), 0.0)
    f = fac[shell]
    u = [(c * f).astype(dtype) for c in u]
    return u


def random_field(g: Grid, seed, kpeak=4.0, totalenergy=1.0, profile=None):
    """Full-layout version of :func:`random_field_compact`."""
    uc = random_field_compact(g.D, g.n, seed, kpeak, totalenergy, profile)
    return [unpack_retained(c, g) for c in uc]


def taylorgreen(g: Grid, V0=1.0, doproject=True):
    """``taylorgreen`` (src/solver.jl:537-570), cell-centred points."""
    n, l = g.n, g.l
    h = l / n
    x = np.linspace(h / 2, l - h / 2, n)
    if g.D == 2:
        Y, X = np.meshgrid(x, x, indexing="ij")
        ux = -V0 * np.sin(2 * np.pi * X / l) * np.cos(2 * np.pi * Y / l)
        uy = V0 * np.cos(2 * np.pi * X / l) * np.sin(2 * np.pi * Y / l)
        u = [to_spec(ux, g), to_spec(uy, g)]
    else:
        Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
        ux = V0 * np.sin(2 * np.pi * X / l) * np.cos(2 * np.pi * Y / l) * np.cos(2 * np.pi * Z / l)
        uy = -V0 * np.cos(2 * np.pi * X / l) * np.sin(2 * np.pi * Y / l) * np.cos(2 * np.pi * Z / l)
        u = [to_spec(ux, g), to_spec(uy, g), np.zeros(g.spec_shape, complex)]
    return project(u, g) if doproject else u


# --------------------------------------------------------------------------
# Gradients and tensors (src/solver.jl:320-332, 711-794)
# --------------------------------------------------------------------------

def vectorgradient(u, g: Grid):
    """``vectorgradient!`` (src/solver.jl:711-733): G_ab = i k_b u_a, returned as a dict keyed 'xy' etc."""
    ks = wavenumbers_full(g)
    names = "xyz"[: g.D]
    return {names[a] + names[b]: 1j * ks[b] * u[a] for a in range(g.D) for b in range(g.D)}


def strainrate(u, g: Grid):
    """``strainrate!`` (src/solver.jl:776-794)."""
    ks = wavenumbers_full(g)
    out = []
    for (i, j) in pairs(g.D):
        if i == j:
            out.append(1j * ks[i] * u[i])
        else:
            out.append(1j * (ks[j] * u[i] + ks[i] * u[j]) / 2)
    return out


def make_tracefree(tau, D):
    """``make_tracefree!`` (src/solver.jl:320-332)."""
    tau = [t.copy() for t in tau]
    tr = sum(tau[i] for i in range(D)) / D
    for i in range(D):
        tau[i] = tau[i] - tr
    return tau


def rel_l2(a, b):
    """Relative L2 distance ||a - b|| / ||b|| over a list of arrays."""
    if isinstance(a, np.ndarray):
        a, b = [a], [b]
    num = math.sqrt(sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b)))
    den = math.sqrt(sum(float(np.sum(np.abs(y) ** 2)) for y in b))
    return num / den if den > 0 else num
