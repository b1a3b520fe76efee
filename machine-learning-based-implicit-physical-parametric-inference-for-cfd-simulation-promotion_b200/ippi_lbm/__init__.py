"""ippi_lbm -- Python host side of the B200 D2Q9 time step.

``Lattice`` wraps one lattice of the C ABI (libippi_lbm.so, include/ippi_lbm.h);
``scenes`` builds the benchmark inputs.  The reference's own C++ API (Mesh,
Lattice, main.cpp) is mirrored in C++ by ../host/ over the same ABI.
"""
from ._lib import (BC_CHANNEL, BC_REF_NEE, BF16, BGK, DELTA_BILINEAR, DELTA_PESKIN4, F16, F32,
                   F64, FIELD_AVG_RHO, FIELD_AVG_U, FIELD_AVG_V, FIELD_F, FIELD_FLAGS,
                   FIELD_NNFLAG, FIELD_RHO, FIELD_TAU, FIELD_UX, FIELD_UY, LES_NONE,
                   LES_CSM, LES_DYNAMIC, LES_FIELD, LES_LEARNED, LES_SMAGORINSKY, LES_WALE, MRT, RR,
                   DivergedError, IppiError, lib)
from . import scenes
from .lattice import Lattice

__all__ = ["Lattice", "lib", "IppiError", "DivergedError", "BGK", "MRT", "RR", "F64", "F32",
           "F16", "BF16", "BC_REF_NEE", "BC_CHANNEL", "LES_NONE", "LES_SMAGORINSKY",
           "DELTA_BILINEAR", "DELTA_PESKIN4", "FIELD_F", "FIELD_RHO", "FIELD_UX", "FIELD_UY",
           "FIELD_TAU", "FIELD_AVG_U", "FIELD_AVG_V", "FIELD_AVG_RHO", "FIELD_FLAGS",
           "FIELD_NNFLAG", "LES_LEARNED", "LES_FIELD", "LES_WALE", "LES_CSM", "LES_DYNAMIC"]
