"""hb_ref_step_static: the one-call timestep that allocates no device memory.

It serves callers that cannot call cudaMalloc (the device allocator belongs to
a host framework, or the memory budget is fixed at start-up): its flux-to-update
scratch is a fixed array inside the library. These tests drive it through the C
ABI on the caller's own reference-layout arrays and check, over two calls in a
row, that it gives exactly what the existing pair hb_ref_calculate_flux +
hb_ref_update_cell gives (fp64: bit for bit, the tolerance of every fp64 parity
test here). Collected last so that a stop at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

import hydrob200 as hb
from hydrob200 import _lib

pytestmark = pytest.mark.gpu

FIELDS = ("H", "U", "V", "Z", "W", "FLUX0", "FLUX1", "FLUX2", "FLUX3", "KLAS")


def _same(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.array_equal(a.view(np.uint64), b.view(np.uint64)) or np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("name,variant", [("stress_a", "H"), ("stress_a", "F"), ("breach", "H"), ("f1", "H")])
def test_static_step_matches_existing_entry_points(deck_dir, name, variant):
    import torch
    lib = _lib.lib()
    deck = hb.Deck(deck_dir[name])
    assert deck.cells <= _lib.REF_STEP_STATIC_MAX_CELLS
    ref = hb.RefLayoutMesh(deck, variant=variant)     # existing entry points
    new = hb.RefLayoutMesh(deck, variant=variant)     # allocation-free entry point
    v = 0 if variant == "H" else 1
    stream = torch.cuda.current_stream().cuda_stream
    for call, (kt, jt) in enumerate([(1, 0), (2, 0)]):
        ref.calculate_flux(kt, jt, stream)
        ref.update_cell(stream)
        _lib.check(lib.hb_ref_step_static(C.byref(new.view), kt, jt, v, stream))
        a, b = ref.dump(), new.dump()
        for k in FIELDS:
            assert _same(a[k], b[k]), f"{name}/{variant} call {call + 1}: {k} differs"
    assert hb.take_ref_device_errors() == 0


def test_static_step_takes_no_device_memory(deck_dir):
    """The property the entry point exists for: once the library is loaded and
    the first call has looked up the array's address, further calls change
    the device's free memory by nothing (every other buffer here is the
    caller's, allocated before the measurement)."""
    import torch
    lib = _lib.lib()
    deck = hb.Deck(deck_dir["f1"])
    new = hb.RefLayoutMesh(deck)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(lib.hb_ref_step_static(C.byref(new.view), 1, 0, 0, stream))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for kt in range(2, 12):
        _lib.check(lib.hb_ref_step_static(C.byref(new.view), kt, 0, 0, stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_step_rejects_meshes_beyond_capacity():
    view = _lib.RefMeshView()
    view.CELL = _lib.REF_STEP_STATIC_MAX_CELLS + 1
    view.NDAYS = 1
    status = _lib.lib().hb_ref_step_static(C.byref(view), 1, 0, 0, None)
    assert status == 9   # HB_E_TOO_LARGE, before anything is launched
