"""Full-size FP64 oracle on the compact 2/3 cube: RHS, RK4 step and sfs! at 810^3.

Test infrastructure only (see ``oracle/__init__.py``).  The same arithmetic as
:mod:`oracle.spectral` / :mod:`oracle.filtering` (``rk4_rhs``, ``rk4_step``,
``sfs``), restated so that an 810^3 grid fits in host memory and runs in about
a minute on 16 cores:

* the state is held on the retained 2/3 cube only (``kx <= n÷3``,
  ``|ky|, |kz| <= n÷3``, FFT order, numpy shape ``(2k+1, 2k+1, k+1)`` indexed
  ``[iz, iy, ix]``), the layout ``random_field_compact`` produces;
* one full RFFT buffer is reused for every inverse transform: it is zero
  outside the four retained corner blocks, so a scatter is four slice copies;
* every product ``v_i v_j`` is transformed and immediately cut back to the
  cube the caller needs, so at most one full spectrum is alive at a time.

Peak host memory at 810^3 is about 45 GB (three physical velocities, one
product, one full spectrum, the six product cubes and the RK4 buffers).

Reference functions followed (file:line of the reference):
``nonlinearity!`` src/solver.jl:434-456, ``viscosity!`` :458-476,
``tensordivergence!`` :509-521, ``project!`` :350-368, ``twothirds!``
:371-389, ``cutoff!`` src/filtering.jl:28-34, ``gaussianfilter!`` :44-67,
``sfs!`` src/data.jl:625-642, ``make_tracefree!`` src/solver.jl:320-332; the
RK4 stepper and the linear band forcing are the new stepper of
``oracle.spectral.rk4_step``.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft

__all__ = ["CompactOracle"]

_PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]  # xx yy zz xy yz zx


def _blocks(n, kw):
    """Slices of the four corner blocks of a half-width-``kw`` cube (FFT order
    along y and z) in the full ``(n, n, n/2+1)`` array and in the cube."""
    lo_full, hi_full = slice(0, kw + 1), slice(n - kw, n)
    lo_cube, hi_cube = slice(0, kw + 1), slice(kw + 1, 2 * kw + 1)
    out = []
    for zf, zc in ((lo_full, lo_cube), (hi_full, hi_cube)):
        for yf, yc in ((lo_full, lo_cube), (hi_full, hi_cube)):
            out.append(((zf, yf, slice(0, kw + 1)), (zc, yc, slice(None))))
    return out


class CompactOracle:
    """FP64 3D oracle of one grid ``n`` (``l = 2π``) on the compact 2/3 cube.

    Pointwise work runs on z-slab chunks in a thread pool (numpy releases the
    GIL inside ufuncs); every chunk does the same arithmetic in the same order
    as the whole-array expressions of :mod:`oracle.spectral`.
    """

    def __init__(self, n, workers=None):
        if n % 2:
            raise AssertionError("Only even number of grid points supported.")
        self.n = n
        self.k = n // 3
        self.workers = workers or int(os.environ.get("SC_ORACLE_WORKERS", os.cpu_count() or 1))
        k = self.k
        kk = np.concatenate([np.arange(k + 1), np.arange(-k, 0)]).astype(np.float64)
        self.kx = np.arange(k + 1, dtype=np.float64)[None, None, :]
        self.ky = kk[None, :, None]
        self.kz = kk[:, None, None]
        self.k2 = self.kx ** 2 + self.ky ** 2 + self.kz ** 2
        self._full = None
        self._pool = ThreadPoolExecutor(self.workers)

    def _map(self, fn, n0):
        """fn(slice) over ``workers`` contiguous chunks of range(n0), in parallel."""
        b = np.linspace(0, n0, min(self.workers, n0) + 1).astype(int)
        list(self._pool.map(lambda i: fn(slice(b[i], b[i + 1])), range(len(b) - 1)))

    # ------------------------------------------------------------------ layout
    @property
    def shape(self):
        return (2 * self.k + 1, 2 * self.k + 1, self.k + 1)

    def full_buffer(self):
        if self._full is None:
            self._full = np.zeros((self.n, self.n, self.n // 2 + 1), dtype=np.complex128)
        return self._full

    def release(self):
        self._full = None

    def scatter(self, cube, out):
        """Write a compact cube into the retained blocks of a full spectrum
        (the rest of ``out`` is left as it is: zero for the shared buffer)."""
        for (f, c) in _blocks(self.n, self.k):
            out[f] = cube[c]

    def gather(self, full, kw=None):
        """Cut the cube of half-width ``kw`` (default ``n÷3``) out of a full spectrum."""
        kw = self.k if kw is None else kw
        cube = np.empty((2 * kw + 1, 2 * kw + 1, kw + 1), dtype=full.dtype)
        for (f, c) in _blocks(self.n, kw):
            cube[c] = full[f]
        return cube

    # ------------------------------------------------------------ operators
    def to_phys(self, cube):
        """``to_phys!`` of ``twothirds!(cube)``: Σ_k û e^{ikx} (src/solver.jl:210-211, 371-389)."""
        buf = self.full_buffer()
        self.scatter(cube, buf)
        buf[0, 0, 0] = 0  # twothirds! also zeroes k = 0
        return sfft.irfftn(buf, s=(self.n,) * 3, norm="forward", workers=self.workers)

    def products(self, u, kw=None):
        """``nonlinearity!`` (src/solver.jl:434-456): σ_ij = F[(P u_i)(P u_j)]/n^3
        in the pair order xx yy zz xy yz zx, cut to the cube of half-width kw."""
        v = [self.to_phys(c) for c in u]
        tmp = np.empty_like(v[0])
        sig = []
        for (i, j) in _PAIRS:
            self._map(lambda z: np.multiply(v[i][z], v[j][z], out=tmp[z]), self.n)
            s = sfft.rfftn(tmp, norm="forward", workers=self.workers)
            sig.append(self.gather(s, kw))
            del s
        return sig

    def convectiondiffusion(self, u, visc, sig=None):
        """``convectiondiffusion!`` (src/solver.jl:949-953) on the retained modes:
        du_i = -i k_j (σ_ij - ν i (k_j u_i + k_i u_j)) (``viscosity!`` :458-476,
        ``tensordivergence!`` :509-521), then ``twothirds!``."""
        sig = self.products(u) if sig is None else sig
        ks = (self.kx, self.ky, self.kz)
        idx = {}
        for c, (i, j) in enumerate(_PAIRS):
            idx[(i, j)] = c
            idx[(j, i)] = c
        du = [np.empty(self.shape, dtype=np.complex128) for _ in range(3)]

        def chunk(z):
            kz = ks[2][z]
            kc = (ks[0], ks[1], kz)
            for i in range(3):
                acc = np.zeros(du[i][z].shape, dtype=np.complex128)
                for j in range(3):
                    s = sig[idx[(i, j)]][z]
                    visc_ij = visc * 1j * (kc[j] * u[i][z] + kc[i] * u[j][z])
                    acc += -1j * kc[j] * (s - visc_ij)
                du[i][z] = acc
        self._map(chunk, self.shape[0])
        for c in du:
            c[0, 0, 0] = 0
        return du

    def project(self, u):
        """``project!`` (src/solver.jl:350-368): Leray projection, k = 0 left intact."""
        out = [np.empty_like(c) for c in u]

        def chunk(z):
            ks = (self.kx, self.ky, self.kz[z])
            kdotu = ks[0] * u[0][z] + ks[1] * u[1][z] + ks[2] * u[2][z]
            with np.errstate(invalid="ignore", divide="ignore"):
                p = kdotu / self.k2[z]
            if z.start == 0:
                p[0, 0, 0] = 0
            for c, (k, uc) in enumerate(zip(ks, u)):
                out[c][z] = uc[z] - k * p
        self._map(chunk, self.shape[0])
        return out

    def band_mask(self):
        """Forced band 1 <= |k|^2 < 9 (integer k)."""
        if getattr(self, "_band", None) is None:
            self._band = (self.k2 >= 1) & (self.k2 < 9)
        return self._band

    def energy(self, u, mask=None):
        """½ Σ|û|² with interior kx counted twice (``getenergy``, src/solver.jl:702)."""
        w = np.ones(self.shape)
        w[..., 1:] = 2.0  # kx = n/2 is outside the cube
        e = 0.0
        for c in u:
            a = w * (c.real ** 2 + c.imag ** 2)
            e += float(a[mask].sum() if mask is not None else a.sum())
        return e / 2

    def rk4_rhs(self, u, visc, eps=None):
        """The RK4 stage derivative of ``oracle.spectral.rk4_rhs``:
        P(twothirds(convectiondiffusion(u))) + A u on the band, A = ε / (2 E_band)."""
        du = self.project(self.convectiondiffusion(u, visc))
        if eps is not None:
            # the band 1 <= |k|^2 < 9 lies within |k_i| <= 2: work on its index list
            bi = self.band_index()
            w = np.where(bi[2] > 0, 2.0, 1.0)  # interior kx counted twice
            ef = sum(float(np.sum(w * np.abs(c[bi]) ** 2)) for c in u) / 2
            A = eps / (2 * ef) if ef > 0 else 0.0
            for d, c in zip(du, u):
                d[bi] += A * c[bi]
        return du

    def band_index(self):
        """Index arrays (iz, iy, ix) of the band 1 <= |k|^2 < 9 in the cube."""
        if getattr(self, "_band_idx", None) is None:
            self._band_idx = np.nonzero(self.band_mask())
        return self._band_idx

    def _axpy(self, y, x, a, out=None):
        """out = y + a x (out defaults to y, in place), per component, in parallel."""
        out = y if out is None else out

        def chunk(z):
            for o, yc, xc in zip(out, y, x):
                o[z] = yc[z] + a * xc[z]
        self._map(chunk, self.shape[0])
        return out

    def rk4_step(self, u, dt, visc, eps=None):
        """Classical RK4 step of ``oracle.spectral.rk4_step``:
        u + dt/6 (k1 + 2 k2 + 2 k3 + k4), stage inputs u + c_q dt k_q."""
        ks = [self.rk4_rhs(u, visc, eps)]
        for cs in (0.5, 0.5, 1.0):
            stage = self._axpy(u, ks[-1], cs * dt, out=[np.empty_like(c) for c in u])
            ks.append(self.rk4_rhs(stage, visc, eps))
            del stage
        out = [np.empty_like(c) for c in u]

        def chunk(z):
            for c in range(3):
                out[c][z] = u[c][z] + dt / 6 * (ks[0][c][z] + 2 * ks[1][c][z] + 2 * ks[2][c][z] + ks[3][c][z])
        self._map(chunk, self.shape[0])
        return out

    # --------------------------------------------------------------- filter
    def sfs(self, u, n_les, deltas):
        """``sfs!`` (src/data.jl:625-642) from the compact DNS state to an
        ``n_les`` grid, for every Δ in ``deltas`` (``None``: no Gaussian).  Returns
        a list of ``(ubar, tau, scale)`` with ubar and tau in the full LES RFFT
        layout ``(nb, nb, nb/2+1)`` (numpy C order, the layout of
        ``oracle.filtering.sfs``) and ``scale`` the L2 norm of the filtered DNS
        products P_les G C(σ_dns), the first of the two terms τ cancels."""
        nb = n_les
        kw = nb // 2
        sig = self.products(u, kw)
        ub_cube = [self._cube_from_compact(c, kw) for c in u]
        out = []
        for delta in deltas:
            ubar = [self._twothirds_les(self._gauss(self._cutoff(c, kw, nb), delta, nb), nb) for c in ub_cube]
            sbar1 = [self._gauss(self._cutoff(s, kw, nb), delta, nb) for s in sig]
            sbar2 = self._les_products(ubar, nb)
            tau = [self._twothirds_les(a - b, nb) for a, b in zip(sbar1, sbar2)]
            tr = (tau[0] + tau[1] + tau[2]) / 3
            tau = [t - tr if i < 3 else t for i, t in enumerate(tau)]
            scale = float(np.sqrt(sum(np.sum(np.abs(self._twothirds_les(a, nb)) ** 2) for a in sbar1)))
            out.append((ubar, tau, scale))
        return out

    def _cube_from_compact(self, c, kw):
        """The half-width-kw cube of a compact state (kw <= n÷3)."""
        k = self.k
        cube = np.zeros((2 * kw + 1, 2 * kw + 1, kw + 1), dtype=np.complex128)
        sel = np.concatenate([np.arange(kw + 1), np.arange(2 * k + 1 - kw, 2 * k + 1)])
        cube[...] = c[np.ix_(sel, sel, np.arange(kw + 1))]
        return cube

    @staticmethod
    def _cutoff(cube, kw, nb):
        """``cutoff!`` (src/filtering.jl:9-34): coarse (nb, nb, nb/2+1) from the
        half-width-kw cube (kw = nb/2; coarse index i <-> wavenumber i or i - nb)."""
        idx = np.concatenate([np.arange(nb // 2), np.arange(kw + 1, 2 * kw + 1)])
        return np.ascontiguousarray(cube[np.ix_(idx, idx, np.arange(nb // 2 + 1))])

    @staticmethod
    def _les_k(nb):
        f = np.arange(nb)
        ky = np.where(f <= (nb - 1) // 2, f, f - nb).astype(np.float64)
        kx = np.arange(nb // 2 + 1, dtype=np.float64)
        return kx[None, None, :], ky[None, :, None], ky[:, None, None]

    @classmethod
    def _gauss(cls, c, delta, nb):
        """``gaussianfilter!`` (src/filtering.jl:44-67): × exp(-Δ²k²/24) except k² < 9."""
        if delta is None:
            return c
        kx, ky, kz = cls._les_k(nb)
        k2 = kx ** 2 + ky ** 2 + kz ** 2
        w = np.where(k2 < 9.0, 1.0, np.exp(-delta ** 2 * k2 / 24))
        return c * w

    @classmethod
    def _twothirds_les(cls, c, nb):
        kx, ky, kz = cls._les_k(nb)
        kc = nb // 3
        m = (np.abs(kx) <= kc) & (np.abs(ky) <= kc) & (np.abs(kz) <= kc)
        m = m & ~((kx == 0) & (ky == 0) & (kz == 0))
        return np.where(m, c, 0)

    @staticmethod
    def _les_products(ubar, nb):
        v = [sfft.irfftn(twothirds_c, s=(nb,) * 3, norm="forward") for twothirds_c in ubar]
        return [sfft.rfftn(v[i] * v[j], norm="forward") for (i, j) in _PAIRS]
