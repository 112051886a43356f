"""libpq3d.so loads and exports every entry point include/pq3d.h declares (no GPU needed)."""
import ctypes

from pyquake3d_b200 import _lib


def test_library_exports_header_symbols():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _lib.exported_symbols()
    assert "TDstressFS_C" in names and "TDstressEachSourceAtReceiver_C" in names
    assert len(names) >= 17
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_record_layouts_match():
    L = _lib.load()   # raises on any layout mismatch
    assert L.pq3d_src_record_bytes() == 33 * 8
