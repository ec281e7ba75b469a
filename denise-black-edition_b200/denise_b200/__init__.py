"""B200 P-SV propagator and FWI adjoint gradient (host-side Python mirror).

The compute path is the CUDA library ``lib/libdenise_b200.so`` behind the C
ABI of ``include/denise_b200.h``; this package binds it with ctypes and adds
the synthetic workloads, the serving loop and helpers.  Importing it fails if
the library has not been built - nothing here computes wavefields on the CPU.
"""
from ._lib import (ACC_F32, ACC_F64, ARITH_EXACT, ARITH_FMA, DeniseError, MODE_ADJOINT, MODE_FORWARD,
                   MODE_OBJECTIVE, SEC_CURL, SEC_DIV, SEC_P, SEC_VX, SEC_VY, SNAP_BF16, SNAP_F16, SNAP_F32,
                   device_count)
from .api import (FIELDS, Model, PsvParams, Shot, average_materials, cfl_limit, device_memory, device_trim,
                  holbergcoeff, last_run_stats, model_footprint, pml_profiles, prepare_visc, run, run_plain,
                  shot_footprint, tdfilt, wavelet)

__all__ = [n for n in dir() if not n.startswith("_")]
