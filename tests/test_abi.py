"""The C-ABI library loads and exports every entry point declared in include/*.h
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:m2cg_status|void|const char\*)\s+(m2cg_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("m2cg_create", "m2cg_advance", "m2cg_compute_residual", "m2cg_riemann_batch",
                 "m2cg_batch_create", "m2cg_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from m2c_b200 import gpu
    if not os.path.exists(gpu.LIB_PATH):
        pytest.fail("libm2c_gpu.so is not built: run m2c_b200/build.py")
    lib = ctypes.CDLL(gpu.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"exported symbols missing: {missing}"


def test_defaults_match_reference_iodata():
    """m2cg_default_* fill the reference's IoData defaults; the Python mirror agrees."""
    from m2c_b200 import abi, gpu
    L = gpu.lib()
    s = abi.Scheme()
    L.m2cg_default_scheme(ctypes.byref(s))
    py = abi.scheme()
    for name, _ in abi.Scheme._fields_:
        assert getattr(s, name) == getattr(py, name), name
    m = abi.Material()
    L.m2cg_default_material(ctypes.byref(m))
    pm = abi.material()
    for name, _ in abi.Material._fields_:
        assert getattr(m, name) == getattr(pm, name), name


def test_batch_create_rejects_bad_arguments_before_any_device_call():
    """m2cg_batch_create validates its arguments on the host first: a tube
    shorter than 4 cells, viscous materials, and a persistent launch asked
    for with a block size other than its 128 threads are refused with
    M2CG_ERR_ARG / M2CG_ERR_UNSUPPORTED and a message, without a GPU."""
    import numpy as np
    from m2c_b200 import abi, cases, gpu
    s = cases.tube_scheme()
    lens, mats, VL, VR, _ = cases.tubes(3, seed=2)
    with pytest.raises(gpu.M2CError, match="128 threads"):
        gpu.Batch(s, lens, mats, VL, VR, cells_per_block=256, threads_per_block=256, use_graph=2)
    short = np.array(lens)
    short[1] = 3
    with pytest.raises(gpu.M2CError, match="at least 4 cells"):
        gpu.Batch(s, short, mats, VL, VR)
    visc = list(mats)
    visc[2] = abi.material(visc[2].gamma, visc[2].p_c, mu=1e-3)
    with pytest.raises(gpu.M2CError, match="viscous"):
        gpu.Batch(s, lens, visc, VL, VR)
