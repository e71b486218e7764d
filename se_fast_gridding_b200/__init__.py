"""se_fast_gridding_b200 -- Spectral Ewald fast Gaussian gridding on B200.

A from-scratch sm_100a implementation of the SE_fast_gridding hot path
(spread -> periodic fold -> FFT -> Green's function scaling -> inverse FFT ->
unfold -> interpolate), behind two C ABIs in libse_gpu.so:

  include/se_fgg_gpu.h  the reference's own API (SE_FGG_*, scaling, ...) plus
                        include/fftw3.h, so unchanged callers link against it
  include/se_gpu.h      the device-resident API (plans, batches)

Python modules: ``solver`` (torch-facing plans and batches), ``fgg`` (the
reference interface), ``serve`` (continuous-batching request loop),
``shard`` (assignment of independent systems to ranks).
"""
from ._lib import SEError, build, lib  # noqa: F401

__all__ = ["SEError", "build", "lib"]
