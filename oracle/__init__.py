"""CPU oracle for the dnsbox pseudospectral time step -- TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy FP64 (and, for tiny grids, in plain C with
naive separable DFTs), the reference algorithm of DavetheSlayer/dnsbox for the
hot path: ``rhs_nonlinear`` (rhs.f90:18-135), ``rhs_Eband`` (rhs.f90:137-168),
``rhs_int_fact`` (rhs.f90:8-16), the integrating-factor Heun step
(dnsboxheun.f90:85-126), the IF-AB2 step (dnsbox.f90:87-191), the state
operators of state.f90 and ``io_Courant`` (io.f90:664-676), and the adjoint
chain of rhsAdj.f90.

It is the checker, never the thing measured or shipped: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs
of ``bench.py`` may import it.  The product (``dnsbox_b200``) never imports it
and has no CPU fallback.

Pinning: the reference (Fortran + MPI + p3dfft + FFTW + HDF5) cannot be built in
this image.  The oracle is pinned against (a) golden vectors produced by running
the reference's own NumPy prototype ``python/dnsbox.py`` (``nonLinear``,
``timeStep``, ``stats``) unmodified under a Python-3 compatibility shim
(``tests/golden/make_golden.py``), and (b) the reference's known-answer tests:
the Beltrami analytic solution (state.f90:287-348), the FFT round trip
(single/test.f90:10-31) and the divergence check (single/test.f90:57-62).  The
FFT arithmetic itself lives in p3dfft/FFTW (un-vendored, unpinned versions);
FFT-level parity is defined against pocketfft (``scipy.fft``) and the
independent naive-DFT C restatement in ``naive_rhs.c``.
"""
