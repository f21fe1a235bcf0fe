"""vsmc_b200 -- the vSMC SMC step (move + log-weight, normalisation/ESS, six
resampling schemes, Philox4x32-10 / Threefry4x64-20 streams) on B200.

The product is the C-ABI library libvsmc_cuda.so (include/vsmc_cuda.h) with
its C++ facade (include/vsmc_b200/); this package builds it
(``vsmc_b200.build``) and binds it for Python callers (``vsmc_b200.capi``).
"""
from . import build  # noqa: F401

__all__ = ["build", "capi"]
