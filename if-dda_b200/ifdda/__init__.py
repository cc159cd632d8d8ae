"""ifdda -- host-side mirror of IF-DDA's cdmlib solve path on top of
libifdda_gpu.so (sm_100a).

Routine names and argument meaning follow the reference:
  greencalculfft      cdmlib/calculgreenfft.f:1-104     -> GreenSpectrum
  produitfftmatvectopt cdmlib/produitfftmatvectopt.f:3-121 -> GreenSpectrum.matvec(tabdip=None)
  produitfftmatvect3  cdmlib/produitfftmatvect3.f:2-127  -> GreenSpectrum.matvec(tabdip=...)
  inverserigopt       cdmlib/inverserigopt.f:1-1085      -> GreenSpectrum.inverserig(tabdip=None)
  inverserig          cdmlib/inverserig.f:1-1090         -> GreenSpectrum.inverserig(tabdip=...)
  local_macro         cdmlib/local-macro.f:3-71          -> Context.local_macro
  cross sections      cdmlib/cdmlib.f:2730-2746          -> Context.cross_sections
  ondeplane(kxky)     cdmlib/ondeplane.f, ondeplanekxky.f -> Context.planewaves
"""
from .api import (Context, GreenSpectrum, SolveResult, IFDDA_FP64, IFDDA_MIXED, IFDDA_FP32,  # noqa: F401
                  IfddaError)
from . import _capi  # noqa: F401
