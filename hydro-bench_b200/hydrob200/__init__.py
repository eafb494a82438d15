"""hydrob200: B200-native (sm_100a) shallow-water timestep of hydro-bench's
hydro-cal solver (CalculateFlux + UpdateCell) behind a C ABI."""
from ._lib import HydroError, VARIANT_H, VARIANT_F, FP64, FP32, SPLIT, LIB_PATH  # noqa: F401
from .solver import Deck, Solver, Batch, RefLayoutMesh, take_ref_device_errors, launch_shapes  # noqa: F401
