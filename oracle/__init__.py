"""CPU oracle for the TorChannel IMEX time step -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy FP64, the reference algorithm of
gmcavallazzi/torChannel's solver step (``solver.py``, ``operators.py``,
``tridiag.py``, ``projection_fft.py``, ``projection.py``, ``utils.py``,
``turbstats.py``).  Every function cites the reference file:line it follows.

It is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
may import it.  The ``torchannel_b200`` package never imports it and has no CPU
fallback.

Parity pin: the restatement is checked against golden vectors that
``tests/golden/make_golden.py`` produced by importing and running the
reference itself (``tests/golden/*.npz``); see ``tests/test_oracle_golden.py``.

Arrays use the reference layout: ``u`` (nx+1, ny+2, nz+2), ``v`` (nx+2, ny+1,
nz+2), ``w`` (nx+2, ny+2, nz+1), ``p`` (nx+2, ny+2, nz+2), C order with z
fastest, ghosts included.
"""

from .grid import generate_grid, generate_hybrid_grid  # noqa: F401
from . import ops, poisson, stats, step  # noqa: F401
