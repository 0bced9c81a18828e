"""atmdyn: B200 (sm_100a) dynamical core of felix-goddard/atmosphere-model.

The CUDA library libatmdyn.so implements the reference's dycore step (the
C-grid and D-grid flux-form semi-Lagrangian sweeps with PPM, the vertical
PPM remap and the periodic halo fill) behind the C ABI of include/atmdyn.h.
This package is its host side: the ctypes binding (:mod:`atmdyn.dycore`),
the time loop of the reference (:mod:`atmdyn.model`), seeded initial
conditions (:mod:`atmdyn.ic`), the namelist and netCDF-3 file formats
(:mod:`atmdyn.io`), the autograd binding of the adjoint
(:mod:`atmdyn.adjoint`) and the batched ensemble (:mod:`atmdyn.ensemble`).
"""
from . import ic, model  # noqa: F401
from ._lib import AtmError, load, build  # noqa: F401
from .dycore import Dycore, device_pow_log  # noqa: F401

__version__ = '0.1'
