"""CPU oracle of the guarded SIMP-floor solve -- test infrastructure only.

A numpy / scipy restatement of the reference's algorithm for this path (the
matrix-free hex8 operator, the Galerkin GMG hierarchy with its smoothers,
safeguarded corrections and inner Krylov wrappers, FGMRES, PCG and the guarded
floor policy), each function citing the reference file:line it follows.

Parity status: pinned.  ``tests/test_oracle.py`` checks this restatement
against fixtures produced by running the reference's own unmodified Python on
the host (``tests/golden/make_golden.py``): structure (KE, edof, P, free DOFs,
level operators) to round-off, preconditioner applies and full solves, and the
cantilever boundary conditions.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker / the timed CPU
baseline; the product path (``gpu_fem`` over libsimpfem) never touches it.
"""
