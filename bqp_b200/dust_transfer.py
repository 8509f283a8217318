"""Import-compatible stand-in for the reference's ``dust_transfer`` module.

``from bqp_b200 import dust_transfer as dt`` gives the propagator names of
dust_transfer/python/dust_transfer/__init__.py.  The transfer optimizer
(``TransferProblem``) is not part of this package.
"""
from .api import MU_EARTH_KM3_S2, eci_to_kep, kep_to_eci, propagate, propagate_final

__all__ = ["MU_EARTH_KM3_S2", "propagate", "propagate_final", "kep_to_eci", "eci_to_kep"]
