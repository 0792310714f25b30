"""B200 (sm_100a) conjunction screening: a drop-in for mizuba's
``conjunctions(pj, conj_thresh, conj_det_interval)`` hot path."""

from enum import IntEnum

from .polyjectory import polyjectory
from .conjunctions import (conjunctions, device_conjunctions, get_tmpdir, release_scratch, scratch_bytes,
                          set_tmpdir, to_device)
from .autotune import autotune
from .sgp4 import gpe_dtype, make_sgp4_polyjectory, sgp4_pj_status, sgp4_propagate


class otype(IntEnum):
    # Codes of mizuba/__init__.py:61-66.
    PRIMARY = 1
    SECONDARY = 2
    MASKED = 4


__all__ = ["polyjectory", "conjunctions", "device_conjunctions", "otype", "to_device", "get_tmpdir", "set_tmpdir", "autotune",
           "release_scratch", "scratch_bytes", "gpe_dtype", "make_sgp4_polyjectory", "sgp4_pj_status",
           "sgp4_propagate"]
