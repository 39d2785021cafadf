"""CPU oracle: a plain NumPy/SciPy restatement of the reference DGFS algorithms.

THIS PACKAGE IS TEST INFRASTRUCTURE.  It is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product path
(``dgfs1d_gpu_b200``) never imports, calls or falls back to anything here.

Every function cites the reference file:line it restates (paths relative to
the dgfs1D_gpu project root).  The reference computes every operator with
PyCUDA kernels and cuFFT; here the kernels' arithmetic is restated element by
element in float64 and cuFFT is replaced by pocketfft (``scipy.fft``) with the
cuFFT conventions: CUFFT_FORWARD = unnormalised e^{-i}, CUFFT_INVERSE =
unnormalised e^{+i} (i.e. ``n * ifftn``).

Pinning: ``tests/golden`` holds vectors produced from the reference itself in
a container where it is checked out -- its pure-Python setup code (quadrature,
velocity mesh, spherical designs, prefactors, DG basis) imported directly, and
its Mako CUDA kernels rendered and executed on the CPU with the same
pocketfft stand-in for cuFFT (``tests/golden/make_golden.py``).  The oracle is
checked against those vectors by ``tests/test_oracle_golden.py``.
"""
