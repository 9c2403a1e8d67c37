"""CPU oracle for the PyCLES hot path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product package imports this directory.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
use it, and only as the checker.

* ``port``     -- numpy restatement of the reference algorithms (each function
                  cites the reference file:line it follows).
* ``ref``      -- ctypes binding to the reference's own C kernels, compiled in
                  place by ``build_ref.py`` into ``oracle/_ref/``.  Used to pin
                  ``port`` and to generate the golden fixtures.
* ``glue``     -- restatement of the Cython glue that calls the kernels
                  (PressureSolver, PressureFFTParallel, TimeStepping,
                  PrognosticVariables.update_all_bcs, HorizontalMean,
                  ClausiusClapeyron, ReferenceState) plus a single-rank
                  ``Simulation3d.run`` stage loop over the hot-path components.

Parity pins: the reference's C kernels (advection, flux divergence,
thermodynamics, halo buffers) through ``ref``; the reference TDMA's
known-answer test (SparseSolvers.pyx:49-60) through the cythonized module.
The FFT/ODE arithmetic at the boundary is scipy's (fftpack, odeint), as in
the reference; the reference pins no version of it.
"""
