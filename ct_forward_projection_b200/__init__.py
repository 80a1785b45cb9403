"""B200-native polyenergetic cone-beam CT forward projector.

The compute path is libctfp.so (include/ctfp.h), hand-written CUDA for sm_100a;
`Projector` (projector.py) is the Python host mirror of the C ABI, and the
drop-in C++ classes live in compat/.
"""
from .projector import (Batch, Projector, build_det_response, build_grid_table, compute_paras, finalize_counts,
                        labels_to_density, sample_volume, scintillator_thickness)

__all__ = ["Batch", "Projector", "build_det_response", "build_grid_table", "compute_paras", "finalize_counts",
           "labels_to_density", "sample_volume", "scintillator_thickness"]
__version__ = "0.1.0"
