"""CPU oracle for the famrdp_jax RHS + TVD-RK3 step path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
package.  It is used by ``tests/`` (as the parity checker), by
``__graft_entry__.smoke()`` (as the checker of one small GPU call) and by
``bench.py`` (the timed ``cpu_baseline`` leg and ``--impl reference``).

``oracle.ref`` restates the reference (LucasLu123/famrdp-jax, pure Python/JAX)
line by line in FP64, once, over an array-backend adapter:

* ``NP``    -- NumPy FP64 (the parity oracle; single-threaded elementwise work);
* ``TORCH`` -- PyTorch-CPU FP64 (the same code; multithreaded; provides
  autograd in place of ``jax.grad``).

JAX itself is not installed in this image, so the reference cannot be
imported here.  Parity is pinned by (a) the reference's own known-answer
tests restated in ``tests/test_oracle_kat.py`` and (b) the reference's
Fortran-generated metric golden data (``tests/golden/test3_metric.npz``).
"""
from oracle.ref import NP, TORCH  # noqa: F401
