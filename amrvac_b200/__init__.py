"""B200-native finite-volume block update for MPI-AMRVAC.

The product is the C ABI library ``libamrvac_gpu.so`` (CUDA, sm_100a) declared
in ``include/amrvac_gpu.h``; this package is its thin Python host layer.
"""
from . import _lib  # noqa: F401
from .api import Context, srl_maps  # noqa: F401
from .ensemble import Ensemble, Instance  # noqa: F401
from .config import config_from_par, make_cfg, parse_namelists, read_par_files  # noqa: F401

__all__ = ["Context", "Ensemble", "Instance", "make_cfg", "config_from_par", "parse_namelists", "read_par_files", "srl_maps"]
