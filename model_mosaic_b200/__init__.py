"""model_mosaic_b200: model_mosaic's forward-model hot path (USFFT Radon
R/RT, Fresnel D/DT, psi and |.|^2 stages) as hand-written sm_100a CUDA
behind a C-ABI (include/mosaic.h), with the reference's Python classes on top.
"""
from model_mosaic_b200._ffi import lib, MosaicError  # noqa: F401


def __getattr__(name):
    # lazy: importing the package must not need a GPU
    if name == "TomoReal":
        from model_mosaic_b200.processing.tomo import TomoReal
        return TomoReal
    if name == "TomoLargeReal":
        from model_mosaic_b200.processing.tomo_large import TomoLargeReal
        return TomoLargeReal
    if name == "Propagation":
        from model_mosaic_b200.processing.propagation import Propagation
        return Propagation
    if name == "PropagationLarge":
        from model_mosaic_b200.processing.propagation_large import PropagationLarge
        return PropagationLarge
    raise AttributeError(name)
