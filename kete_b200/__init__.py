"""kete_b200 -- kete's orbit-propagation hot path, B200-native.

Drop-in GPU versions of kete's ``propagate_two_body``, ``propagate_n_body``,
``fov_state_check``, ``hg_apparent_mag`` and ``NeatmParams.evaluate``, computed in FP64
by hand-written sm_100a CUDA kernels in ``libketeb200.so`` (C ABI: include/kete_b200.h).
"""
from . import autodiff, flux, fov, spice, state_transition
from .fov import (ConeFOV, NeosCmos, NeosVisit, OmniDirectionalFOV, RectangleFOV, WiseCmos,
                  ZtfCcdQuad, ZtfField, fov_spk_check, fov_state_check, fov_static_check)
from ._lib import KeteB200Error, init
from .propagation import (
    NonGravModel,
    propagate_n_body,
    propagate_n_body_arrays,
    propagate_n_body_long,
    propagate_n_body_long_arrays,
    propagate_two_body,
    propagate_two_body_arrays,
    radau_central_arrays,
    spk_accel_arrays,
    vec_accel_arrays,
)
from .state import Frames, SimultaneousStates, State
from .state_transition import compute_stm, propagate_covariance, propagate_covariance_n_body

__all__ = [
    "autodiff",
    "flux",
    "fov",
    "RectangleFOV",
    "ConeFOV",
    "OmniDirectionalFOV",
    "WiseCmos",
    "NeosCmos",
    "NeosVisit",
    "ZtfCcdQuad",
    "ZtfField",
    "fov_state_check",
    "fov_spk_check",
    "fov_static_check",
    "spice",
    "init",
    "KeteB200Error",
    "NonGravModel",
    "propagate_n_body",
    "propagate_n_body_arrays",
    "propagate_n_body_long",
    "propagate_n_body_long_arrays",
    "propagate_two_body",
    "propagate_two_body_arrays",
    "radau_central_arrays",
    "spk_accel_arrays",
    "vec_accel_arrays",
    "Frames",
    "SimultaneousStates",
    "State",
    "state_transition",
    "compute_stm",
    "propagate_covariance",
    "propagate_covariance_n_body",
]
