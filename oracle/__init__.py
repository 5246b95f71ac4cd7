"""CPU oracle for the toporecon PDHG hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the algorithms that the reference
(MRI-Research/MultiNodeMRI-MICCAI26, ``toporecon``) runs on its hot path:

* ``oracle.nufft``    -- the Kaiser-Bessel NUFFT that the reference obtains from
  SigPy 0.1.27 (``src/toporecon/nufft_backend.py:101-116`` calls
  ``sp.nufft`` / ``sp.nufft_adjoint`` with default ``oversamp=1.25, width=4``),
  restated from SigPy's published method, plus an FP64 direct NUDFT.
* ``oracle.wavelets`` -- the db1 echo Haar pair of ``algorithms/tvmw.py:312-375``
  and a PyWavelets-convention ``zero``-mode db6 ``wavedec3``/``waverec3`` that
  the reference obtains from ptwt (``algorithms/tvmw.py:196-206``).
* ``oracle.pdhg``     -- the TVM / TVME / TVMW PDHG iterations and stopping
  rules of ``algorithms/tvm.py:227-472``, ``algorithms/tvme.py:208-557`` and
  ``algorithms/tvmw.py:385-786`` collapsed onto one device.
* ``oracle.cgrid``    -- an OpenMP C restatement of the KB interpolation and
  gridding loops (``oracle/kbgrid.c``), used for speed and as the CPU baseline.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline
and ``--impl reference`` legs) may import this package, and only as the reference side of a comparison
or as the timed CPU baseline.  The product path never calls it.

Parity status.  The reference's own tests pin nothing on this path (its unit
tests cover CFL I/O, the dataset contract, trajectory scaling and stitching
only).  The PDHG restatement is pinned against golden vectors produced by
importing the reference's own ``TvmReconstructor`` / ``TvmeReconstructor`` /
``TvmwReconstructor`` with SigPy, ptwt and mpi4py replaced by shims
(``tests/golden/make_golden.py``).  The NUFFT convention (SigPy 0.1.27) and the
db6 wavelet convention (ptwt / PyWavelets) cannot be run in this container:
for those two pieces parity is UNPINNED against the third-party libraries and
is anchored only on the FP64 direct NUDFT, adjointness and perfect-
reconstruction properties.
"""
