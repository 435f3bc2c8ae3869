"""B200-native MOAO tomographic-reconstructor path (covariance generation,
Cholesky reconstructor, Cee/Cvv, intersample PSF) behind the reference's
interface. See ``moao_b200.api`` for the entry points."""
from .api import (Cee_Cvv, Context, Intersample, MoaoError, NotSPDError, Tomo, default_context,
                  intersample_inputs, matcov_tile, reconstructor)
from ._lib import LIB_PATH, lib

__all__ = ["Cee_Cvv", "Context", "Intersample", "MoaoError", "NotSPDError", "Tomo",
           "default_context", "intersample_inputs", "matcov_tile", "reconstructor", "LIB_PATH",
           "lib"]
