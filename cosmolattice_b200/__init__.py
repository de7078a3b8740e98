"""B200-native lattice time evolution for CosmoLattice models.

Product path: the CUDA library ``lib/libclb200.so`` behind the C ABI in ``include/clb200.h``;
this package is its host side (parameters, models, initial conditions, evolver and measurer
shaped like the reference's CosmoInterface API).
"""
from . import _capi
from .lattice import Evolver, Lattice, Measurer, ModelInitializer, run
from .models import MODELS, CouplingsManager, Model, lphi4, lphi4_1f
from .params import ParameterParser, RunParameters, RunParametersInconsistent, RunParametersMissing

__all__ = [
    "_capi", "Evolver", "Lattice", "Measurer", "ModelInitializer", "run", "MODELS", "CouplingsManager",
    "Model", "lphi4", "lphi4_1f", "ParameterParser", "RunParameters", "RunParametersInconsistent",
    "RunParametersMissing",
]
