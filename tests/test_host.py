"""Host-side checks that need no GPU: the C-ABI library loads and exports
every symbol the header declares, argument validation that happens before
any device work, and the Python front end's own validation."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from vortrace_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "vortrace_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(vt_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    lib = L.load()
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(L.EXPORTS) == syms


def test_abi_and_verbose():
    lib = L.load()
    assert lib.vt_abi_version() == 2
    import vortrace_b200 as vt
    vt.set_verbose(True)
    assert vt.get_verbose() is True
    vt.set_verbose(False)
    assert vt.get_verbose() is False


def test_create_rejects_size_mismatch():
    # src/bindings.cpp:53-56 / src/pointcloud.cpp:18-22 wording
    lib = L.load()
    pos = np.zeros((4, 3))
    f = np.ones(3)
    sb = np.array([0, 1, 0, 1, 0, 1], float)
    h = C.c_void_p()
    rc = lib.vt_cloud_create(L.dptr(pos), 4, L.dptr(f), 3, 1, L.dptr(sb), None, 0, 0,
                             C.byref(h))
    assert rc == L.VT_ERR_INVALID
    assert lib.vt_last_error() == b"Input sizes must match: pos has 4 rows but fields has 3"
    assert not h.value


def test_python_validation_before_device():
    import vortrace_b200 as vt
    with pytest.raises(ValueError, match="fields must be 1D"):
        vt.ProjectionCloud(np.zeros((3, 3)), np.zeros((3, 1, 1)), boundbox=[0, 1] * 3)
    with pytest.raises(ValueError, match="Input sizes must match"):
        vt.ProjectionCloud(np.zeros((3, 3)), np.zeros(4), boundbox=[0, 1] * 3)


def test_null_handles():
    lib = L.load()
    assert lib.vt_cloud_build_tree(None) == L.VT_ERR_INVALID
    info = L.CloudInfo()
    assert lib.vt_cloud_get_info(None, C.byref(info)) == L.VT_ERR_INVALID
    assert lib.vt_segments_count(None) == 0
    lib.vt_cloud_destroy(None)
    lib.vt_segments_free(None)


def test_grid_io_round_trip(tmp_path):
    from vortrace_b200 import io as vio
    data = np.arange(12.0).reshape(3, 4)
    vio.save_grid(tmp_path / "g.npz", data, extent=[0, 1, 2, 3], metadata={"npix": 4, "f": "rho"})
    d, meta = vio.load_grid(tmp_path / "g.npz")
    np.testing.assert_array_equal(d, data)
    assert meta["npix"] == 4 and meta["f"] == "rho"
    np.testing.assert_array_equal(meta["extent"], [0, 1, 2, 3])
    with pytest.raises(ValueError, match="Unknown format"):
        vio.save_grid(tmp_path / "g.bin", data, fmt="bin")
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError, match="h5py is required"):
            vio.save_grid(tmp_path / "g.h5", data, fmt="hdf5")
