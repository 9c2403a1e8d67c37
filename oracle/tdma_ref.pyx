# cython: language_level=3
# Test infrastructure, not product code.
#
# Exposes the reference's own Thomas solver (SparseSolvers.TDMA.solve,
# SparseSolvers.pyx:24-44, a cdef method that Python cannot call) to the
# checker.  The reference module itself is cythonized from where it lies
# by oracle/build_ref.py; this wrapper only cimports it.
cimport SparseSolvers


def tdma_solve(double[::1] x, double[::1] a, double[::1] b, double[::1] c):
    """Solve one tridiagonal system in place with the reference TDMA."""
    cdef SparseSolvers.TDMA t = SparseSolvers.TDMA()
    t.initialize(x.shape[0])
    t.solve(&x[0], &a[0], &b[0], &c[0])
    t.destroy()


def tdma_known_answer():
    """The reference's only known-answer test (SparseSolvers.pyx:49-60)."""
    SparseSolvers.TDMA().test()
