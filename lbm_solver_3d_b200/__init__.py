"""B200-native (sm_100a) D3Q19 TRT + squirmer lattice Boltzmann hot path."""
from .params import Params, ParamError  # noqa: F401
