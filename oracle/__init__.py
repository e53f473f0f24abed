"""CPU FP64 oracle for the 3D-RISM solute hot path of bgy3d.

TEST INFRASTRUCTURE ONLY.  Nothing under ``oracle/`` is part of the
product: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import it, and only as the checker (or the timed
CPU restatement), never as the computation being measured or shipped.

The reference (C99 + Fortran 2008 + Guile, on PETSc/FFTW-MPI) cannot be
built in this environment (no gfortran, Guile, PETSc, FFTW or MPI), so
this package restates its algorithm in NumPy/SciPy:

* ``closures``  -- closures.f90 (HNC/KH/PY/PSE-n closures, their
  differentials and the chemical-potential integrands);
* ``rism1d``    -- rism.f90 / drism.f90 / fft.f90 / bessel.f90: the 1D
  RISM/DRISM pure-solvent solve that produces chi(k), and the 1D
  solute-solvent solve;
* ``hnc3d``     -- hnc3d.c / bgy3d-solutes.c / bgy3d-vec.c /
  bgy3d-force.h: the 3D solute solve ``hnc3d_solute_solve``;
* ``newton``    -- a Newton-GMRES driver standing in for PETSc
  SNESNEWTONLS + KSPGMRES (bgy3d-snes.c); only the fixed point matters.

Parity is pinned against the reference's published values: README:16
(1D water mu = -7.869294), README:28/30 (3D water mu = -6.349052 with
renormalisation, -6.297170 without), test/out/water.hnc3d.g2 and the six
test/out/*.hnc3d.g1 (3D pure solvent and solutes, every printed digit).
The charged-ion regression test/out/run-ions-out (9 ions x 6 closures, 1D
and 3D) is reproduced up to one constant per closure and dimension, the
same for every ion (|offset| < 2.5e-3 in 1D, < 3e-2 in 3D, from the
long-range treatment of the revision that printed it); after removing it
every ion agrees to the 4 printed decimals.  See
tests/test_oracle_goldens.py.
"""
