"""bem_b200 -- B200-native dense PMCHWT path (assembly, complex LU, far field /
Mueller) behind the C ABI of libbemdense.so."""
from ._lib import (BemError, BemLibraryMissing, LIB_PATH, PREC_FP32_REFINE, PREC_FP64,  # noqa: F401
                   lib)
from .api import *  # noqa: F401,F403
