"""unicycle_b200: B200 (sm_100a) implementation of Unicycle's 3-D quasi-dynamic
boundary-integral hot path behind a C ABI (include/ucg.h, libucg.so).

    from unicycle_b200 import Simulation, configs
"""
from . import configs  # noqa: F401  (pure numpy; no device needed)
from ._lib import UcgError, load  # noqa: F401
from ._lib import (UCG_OKADA_FP64, UCG_OKADA_REF32IO, UCG_PREC_FP64,  # noqa: F401
                   UCG_PREC_HMATRIX, UCG_PREC_HMATRIX_SPLIT, UCG_PREC_SPLIT_BF16,
                   UCG_PREC_SPLIT_PAIR)
from .simulation import Simulation  # noqa: F401
from .ensemble import Ensemble  # noqa: F401
from .stepmodel import StepModel  # noqa: F401
from .deck import Deck, write_deck  # noqa: F401

__all__ = ["Simulation", "Ensemble", "StepModel", "Deck", "write_deck", "configs", "UcgError", "load"]
