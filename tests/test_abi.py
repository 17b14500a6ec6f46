"""C ABI of libaero3d.so: exports, host-side grid parity, argument and no-device errors."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aero3d.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(a3d_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(aero):
    from importlib import import_module
    lib = import_module("3d_aero_lab_b200._lib").lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_python_prototypes_cover_header():
    from importlib import import_module
    protos = import_module("3d_aero_lab_b200._lib").PROTOS
    assert set(declared_functions()) <= set(protos)


def test_struct_layout_matches_header():
    from importlib import import_module
    abi = import_module("3d_aero_lab_b200.abi")
    # 18 doubles per surface; engine: 3 doubles + 2 int32 + double + 302 floats
    assert C.sizeof(abi.a3d_surface) == 18 * 8
    assert C.sizeof(abi.a3d_engine) == 3 * 8 + 8 + 8 + 302 * 4
    assert C.sizeof(abi.a3d_exit) == 8 + 3 * 8
    assert C.sizeof(abi.a3d_shape) == 8 * 8 + 3 * 18 * 8 + 4 * 8 + 8 + 2 * C.sizeof(abi.a3d_engine) + 2 * 32


@pytest.mark.parametrize("typ,cells", [("fighter", 30000), ("fighter", 4.0e6), ("interceptor", 50000),
                                       ("airliner", 150e3), ("airliner", 1.2e8), ("fighter", 500)])
def test_grid_matches_oracle_exactly(aero, ref, typ, cells):
    """cfdGrid (src/air_cfd.js:21-44) on the host side of the library vs the oracle, bit for bit."""
    sh = aero.shape_of(aero.build_aircraft(typ))
    g = aero.cfd_grid(sh, cells)
    o = ref.grid(sh, cells)
    assert (g.NX, g.NY, g.NZ) == (o.NX, o.NY, o.NZ)
    assert np.array_equal(g.X.f, o.xf) and np.array_equal(g.Y.f, o.yf) and np.array_equal(g.Z.f, o.zf)
    assert g.h == o.h
    assert abs(g.N / cells - 1) < 0.06


def test_bad_arguments_are_reported(aero):
    from importlib import import_module
    L = import_module("3d_aero_lab_b200._lib")
    lib = L.lib()
    sh = aero.shape_of(aero.build_aircraft("fighter"))
    xf = np.zeros(4)
    dims = np.zeros(3, np.int32)
    h = C.c_double()
    core = np.zeros(5)
    rc = lib.a3d_grid_build(C.byref(sh), 30000.0, 3, xf, xf, xf, dims, C.byref(h), core)
    assert rc == 1 and b"capacity" in lib.a3d_last_error()
    rc = lib.a3d_grid_build(C.byref(sh), -5.0, 3, xf, xf, xf, dims, C.byref(h), core)
    assert rc == 1
    with pytest.raises(L.AeroError):
        L.check(rc)


def test_no_device_fails_loudly_without_fallback(aero):
    """Without a GPU the solver refuses to run (A3D_ERR_NODEVICE); it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from importlib import import_module
    L = import_module("3d_aero_lab_b200._lib")
    sh = aero.shape_of(aero.build_aircraft("fighter"))
    g = aero.cfd_grid(sh, 2000)
    with pytest.raises(L.AeroError) as e:
        aero.cfd_geom(sh, g, 0.0)
    assert e.value.status == 8
    with pytest.raises(L.AeroError):
        aero.CfdGPU(g, shape=sh)


def test_slab_and_chunk_entry_points_check_their_arguments():
    """The z-chunk and z-slab entry points refuse null handles with a status, on any machine."""
    from importlib import import_module
    L = import_module("3d_aero_lab_b200._lib")
    lib = L.lib()
    i32 = C.c_int32()
    calls = [lib.a3d_solver_set_chunks(None, 0), lib.a3d_solver_get_chunks(None, C.byref(i32)),
             lib.a3d_solver_get_kernel(None, C.byref(i32), C.byref(i32)), lib.a3d_solver_stage(None, 1),
             lib.a3d_solver_set_owned(None, 0, 1), lib.a3d_solver_copy_planes(None, 0, None, 0, 1, 0),
             lib.a3d_solver_set_neighbors(None, None, None), lib.a3d_solver_sync_neighbors(None),
             lib.a3d_solver_residual_parts(None, np.zeros(2))]
    for rc in calls:
        assert rc != 0
        assert lib.a3d_last_error()


def test_grid_levels_are_the_apps(aero):
    """cfdGrid(ac, level) with the app's CFD_GRIDS (src/air_cfd.js:10)."""
    sh = aero.shape_of(aero.build_aircraft("fighter"))
    for level, cells in (("coarse", 150e3), ("medium", 380e3), ("fine", 820e3)):
        a, b = aero.cfd_grid(sh, level), aero.cfd_grid(sh, cells)
        assert (a.NX, a.NY, a.NZ) == (b.NX, b.NY, b.NZ) and abs(a.N / cells - 1) < 0.06


def test_every_entry_point_refuses_null_arguments():
    """Every declared function called with null pointers and zero sizes returns A3D_ERR_ARG with
    a message, on any machine (the argument checks come before any device work); the destroy
    functions accept a null handle like free()."""
    from importlib import import_module
    L = import_module("3d_aero_lab_b200._lib")
    L.lib()
    raw = C.CDLL(L.LIB_PATH)  # separate function objects: pointer arguments as plain void*
    raw.a3d_last_error.restype = C.c_char_p
    destroy = {"a3d_solver_destroy", "a3d_batch_destroy", "a3d_server_destroy"}
    checked = 0
    for name in declared_functions():
        if name in ("a3d_last_error", "a3d_abi_version"):
            continue
        _, args = L.PROTOS[name]
        types, vals = [], []
        for t in args:
            if t is C.c_double:
                types.append(t); vals.append(0.0)
            elif t in (C.c_int, C.c_int32, C.c_int64):
                types.append(t); vals.append(0)
            else:
                types.append(C.c_void_p); vals.append(None)
        f = raw[name]
        f.argtypes, f.restype = types, C.c_int
        rc = f(*vals)
        if name in destroy:
            assert rc == 0, name
        else:
            assert rc == 1, (name, rc)
            assert raw.a3d_last_error().startswith(b"bad argument"), name
        checked += 1
    assert checked == len(declared_functions()) - 2
