"""FP64 CPU oracle for the pseudo-spectral Navier-Stokes hot path of SymmetryCode.jl.

TEST INFRASTRUCTURE ONLY.  This package is the checker: it is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` leg and
``--impl reference`` arm of ``bench.py``, and by nothing else.  The product
path (``symmetrycode.jl_b200``) never imports it and fails loudly when its CUDA
library is missing.

It is a line-by-line restatement in numpy + ``scipy.fft`` (pocketfft, FP64) of
the reference's Julia functions; every function cites the reference file:line
it follows.  The reference itself (Julia, KernelAbstractions, FFTW/cuFFT)
cannot run in this environment (no Julia toolchain), so parity is pinned by the
reference's own known-answer tests (``test/test_fft.jl``,
``test/test_solver_kernels.jl``, ``test/test_grid.jl``,
``test/test_closures.jl``, ``test/test_tensor_helpers.jl``), ported to
``tests/test_oracle_known_answers.py``.  Everything those tests do not reach
(RHS values, Wray3, RK4, forcing, the SFS filter, dynamic Smagorinsky, les!)
is **parity unpinned** against the reference and is instead checked through
physical/mathematical properties (Galerkin energy conservation of the
dealiased nonlinear term, Taylor-Green analytic RHS, RK order of convergence,
Hermitian symmetry, divergence-free output).

Two further modules serve the production size 810^3: ``oracle.triad`` (exact
triad sums of sparse fields, no FFT) and ``oracle.compact`` (the same FFT
oracle on the compact 2/3 cube, lean enough to run 810^3 in host memory).
Both are checked against the restatement above by CPU tests
(``tests/test_oracle_sparse_compact.py``); they are imported explicitly, not
re-exported here.

Array convention: the reference stores spectral fields column-major with shape
``(n/2+1, n, n)`` (x fastest, x is the halved RFFT axis).  Here numpy C-order
arrays of shape ``(n, n, n/2+1)`` indexed ``[iz, iy, ix]`` have the identical
memory layout, so the same bytes can be handed to the C ABI.
"""

from .spectral import *  # noqa: F401,F403
from .filtering import *  # noqa: F401,F403
from .closures import *  # noqa: F401,F403
from .les import *  # noqa: F401,F403
from .cnn import *  # noqa: F401,F403
