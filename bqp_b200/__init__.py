"""bqp_b200 -- batched orbit propagator for one NVIDIA B200 (sm_100a).

A drop-in for the Lightyear propagator of tdude78/bqp's ``dust_transfer``:
``propagate``, ``propagate_final``, ``kep_to_eci``, ``eci_to_kep`` with the
reference's arguments and results, plus batch entry points.  The numerics run
in the CUDA kernels of ``libbqp_b200.so`` (C ABI: include/bqp_prop.h).
"""
from .api import (MU_EARTH_KM3_S2, eci_to_kep, kep_to_eci, propagate, propagate_batch_final,
                  propagate_batch_sampled, propagate_final)

__all__ = ["MU_EARTH_KM3_S2", "propagate", "propagate_final", "kep_to_eci", "eci_to_kep",
           "propagate_batch_final", "propagate_batch_sampled"]
__version__ = "0.1.0"
