"""TEST INFRASTRUCTURE -- the parity oracle for the cola_halo hot path.

Nothing in the product imports this package.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it, and
only as the checker (never as the thing measured or shipped).

* ``oracle/_ref/libcolaref.so`` -- the reference's own pm.c, cola.c, lpt.c,
  power.c, move.c, comm.c, msg.c, timer.c compiled unchanged against the
  project's single-rank MPI / FFTW3f-MPI / GSL shims (``oracle/Makefile``).
* ``oracle/ref.py`` -- ctypes binding of that library.
* ``oracle/restate.py`` -- an independent numpy restatement of the same
  algorithm, each function citing the reference file:line it follows.
"""
