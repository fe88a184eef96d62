"""B200-native LES time step (pseudo-spectral ABL LES of fmargairaz/new-repo).

The operators run as hand-written sm_100a CUDA kernels in ``liblesgpu.so``
behind the C ABI of ``include/lesgpu.h``; ``LES`` mirrors the reference's
module entry points on top of it.
"""
from .capi import FIELDS, PLANES, LesError, load  # noqa: F401
from .les import LES, RunParams, inversion_noise, log_law_noise, read_namelist, scalar_linear_noise  # noqa: F401

__all__ = ["LES", "RunParams", "LesError", "read_namelist", "log_law_noise", "scalar_linear_noise", "inversion_noise", "FIELDS", "PLANES", "load"]
