"""CPU-side checks of the drop-in boundary: the C-ABI library loads and exports
every symbol include/rtm_b200.h declares; argument validation needs no GPU;
the reference-level Python API keeps the reference's names."""
import ctypes
import inspect
import os

import numpy as np
import pytest

from taichirtm_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert "rtm_forward" in names and "rtm_backward" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert b"sm_100a" in L.rtm_version()


def test_plan_create_rejects_bad_geometry_without_gpu():
    """Validation runs before any device call."""
    L = _lib.lib()
    g = _lib.RtmGrid(10, 10, 1.0, 1.0, 1000.0, 5, 2, 3)
    src = np.array([[20, 3]], np.int32)  # outside the 10-row window
    rec = np.array([[1, 1]], np.int32)
    shot = (_lib.RtmShot * 1)(_lib.RtmShot(0, 10, 1, src.ctypes.data_as(_lib.I32P), 1,
                                           rec.ctypes.data_as(_lib.I32P)))
    h = ctypes.c_void_p()
    rc = L.rtm_plan_create(ctypes.byref(g), 1, shot, None, ctypes.byref(h))
    assert rc == -1 and not h.value
    assert b"source" in L.rtm_last_error()
    g2 = _lib.RtmGrid(10, 10, 1.0, 1.0, 1000.0, 5, 20, 3)  # sponge wider than the grid
    rc = L.rtm_plan_create(ctypes.byref(g2), 1, shot, None, ctypes.byref(h))
    assert rc == -1


def test_reference_names_exported():
    import taichirtm_b200 as T
    for n in ["ReverseTimeMigration", "init_taichi", "reset_taichi", "ForwardModeling",
              "BackwardModeling", "load_rtm_results", "stack_rtm_images", "compute_display_limits",
              "prepare_image_data", "create_visualization_data", "save_stacked_results"]:
        assert hasattr(T, n), n
    sig = inspect.signature(T.ForwardModeling.run)
    assert list(sig.parameters)[1:] == ["save", "display_callback", "stability_check_interval"]
    sig = inspect.signature(T.BackwardModeling.run_calc)
    ref = ["import_fwdata_u", "import_fwdata_v", "import_fwdata_w", "isnaps_field", "num_snaps",
           "isnap_interval", "method", "display_callback", "stability_check_interval"]
    names = list(sig.parameters)[1:]
    assert names[:len(ref)] == ref
    # extensions only as keyword-only parameters with defaults after the reference's
    for n in names[len(ref):]:
        prm = sig.parameters[n]
        assert prm.kind is inspect.Parameter.KEYWORD_ONLY and prm.default is not inspect.Parameter.empty, n


def test_product_has_no_oracle_dependency():
    """The product package never imports the oracle (test infrastructure)."""
    root = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "taichirtm_b200")
    for dirpath, _, files in os.walk(root):
        for f in files:
            if f.endswith(".py"):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "from oracle" not in text, f


def test_memory_estimates_match_reference_formulae():
    from taichirtm_b200 import BackwardModeling, ForwardModeling
    assert ForwardModeling.estimate_memory_bytes(100, 50, 200, 1, 10) == 17 * 100 * 50 * 4 + 3 * 10 * 200 * 4
    assert BackwardModeling.estimate_memory_bytes(100, 50, 200, 2, 10) == 20 * 100 * 50 * 4 + 3 * 2 * 200 * 4
