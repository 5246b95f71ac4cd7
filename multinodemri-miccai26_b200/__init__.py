"""toporecon_b200: a Blackwell (sm_100a) backend for toporecon's PDHG reconstruction loop.

Import name: this directory is the package ``multinodemri-miccai26_b200``
(load it with ``importlib.import_module("multinodemri-miccai26_b200")`` or run
``python -m multinodemri-miccai26_b200 reconstruct ...``).

Public pieces:
  nufft_backend   NufftBackend contract, B200NufftBackend, create_nufft_backend
  solver          PdhgSolver (TVM / TVME / TVMW on one GPU)
  algorithms      TvmReconstructor, TvmeReconstructor, TvmwReconstructor + CLI mains
  synthetic       seeded synthetic cones datasets
  warmstart       learned PDHG warm start (3-D complex conv encoder-decoder)
"""

from . import _lib, synthetic  # noqa: F401

__all__ = ["_lib", "synthetic"]
__version__ = "0.1.0"
