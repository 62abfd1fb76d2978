"""CPU-side checks of the C ABI library and the host mirror (no kernel launches)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "tigre_b200.h")
COMPAT = os.path.join(ROOT, "include", "tigre_b200_compat.hpp")


def _declared(path, pattern):
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"//[^\n]*", "", txt)
    return sorted(set(re.findall(pattern, txt)))


def test_library_exports_every_declared_symbol(native_lib):
    names = _declared(HEADER, r"\b(tigre_[a-z0-9_]+)\s*\(")
    assert len(names) >= 24
    for n in names:
        assert hasattr(native_lib, n), n


def test_compat_symbols_have_reference_mangling():
    from tigre_b200._native import LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", LIB_PATH], capture_output=True, text=True).stdout
    for sig in ["siddon_ray_projection(float*, Geometry, float**, float const*, int, GpuIds const&)",
                "interpolation_projection(float*, Geometry, float**, float const*, int, GpuIds const&)",
                "voxel_backprojection(float*, Geometry, float*, float const*, int, GpuIds const&)",
                "voxel_backprojection2(float*, Geometry, float*, float const*, int, GpuIds const&)",
                "pocs_tv(float*, float*, float, long const*, int, GpuIds const&)",
                "siddon_ray_projection_parallel(float*, Geometry, float**, float const*, int, GpuIds const&)",
                "voxel_backprojection_parallel(float*, Geometry, float*, float const*, int, GpuIds const&)"]:
        assert sig in out, sig


def test_geometry_struct_layout_matches_reference():
    from tigre_b200._native import TigreGeometry
    # sizeof/offsetof of struct Geometry (types_TIGRE.hpp:48-85) as g++ lays it out on LP64
    assert C.sizeof(TigreGeometry) == 184
    assert TigreGeometry.offOrigX.offset == 40 and TigreGeometry.nDetecU.offset == 72
    assert TigreGeometry.COR.offset == 168 and TigreGeometry.accuracy.offset == 180


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_host_api_reports_no_device_instead_of_exiting():
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    g = cone_geometry((8, 8, 8), (8.0, 8.0, 8.0), (8, 8), (1.0, 1.0))
    with pytest.raises(ValueError, match="code 2"):
        tigre.Ax(np.zeros((8, 8, 8), np.float32), g, np.zeros(2, np.float32))
    from tigre_b200.utilities.errors import TigreCudaCallError
    with pytest.raises(TigreCudaCallError):
        tigre.Atb(np.zeros((2, 8, 8), np.float32), g, np.zeros(2, np.float32), "matched")


def test_plan_rejects_bad_geometry(native_lib):
    from tigre_b200 import _native as N
    from tigre_b200.utilities.geometry import cone_geometry
    g = N.checked_geometry(cone_geometry((8, 8, 8), (8.0, 8.0, 8.0), (8, 8), (1.0, 1.0)), np.zeros(3, np.float32))
    cg = N.CGeometry(g, 3)
    cg.s.dVoxelX = 0.0
    h = C.c_void_p()
    ang = np.zeros((3, 3), np.float32)
    rc = native_lib.tigre_plan_create(C.byref(cg.s), ang.ctypes.data, 3, 0, C.byref(h))
    assert rc != 0 and not h.value


def test_check_geo_expands_per_angle_fields():
    from tigre_b200.utilities.geometry import cone_geometry
    g = cone_geometry((4, 5, 6), (4.0, 5.0, 6.0), (7, 8), (1.0, 1.0))
    g.check_geo(np.linspace(0, 1, 5))
    assert g.angles.shape == (5, 3)
    assert g.DSO.shape == (5,) and g.offOrigin.shape == (5, 3) and g.offDetector.shape == (5, 2)
    assert g.rotDetector.shape == (5, 3) and g.COR.shape == (5,) and g.accuracy == 0.5
    g.cast_to_single()
    assert g.DSO.dtype == np.float32 and g.nVoxel.dtype.kind == "i"
    bad = cone_geometry((4, 5, 6), (4.0, 5.0, 7.0), (7, 8), (1.0, 1.0))
    bad.dVoxel = np.array([1.0, 1.0, 1.0])
    with pytest.raises(AttributeError):
        bad.check_geo(np.zeros(2))


def test_ax_input_validation():
    import tigre_b200 as tigre
    from tigre_b200.utilities.geometry import cone_geometry
    g = cone_geometry((4, 5, 6), (4.0, 5.0, 6.0), (7, 8), (1.0, 1.0))
    with pytest.raises(TypeError):
        tigre.Ax(np.zeros((4, 5, 6), np.float64), g, np.zeros(2))
    with pytest.raises(ValueError):
        tigre.Ax(np.zeros((4, 5, 7), np.float32), g, np.zeros(2))
    with pytest.raises(ValueError):
        tigre.Atb(np.zeros((3, 7, 8), np.float32), g, np.zeros(2))


def test_options_round_trip_without_a_device(native_lib):
    from tigre_b200 import _native as N
    assert native_lib.tigre_get_option(N.OPT_HOST_STAGING) == -1
    assert native_lib.tigre_get_option(N.OPT_BP_SKIP_COPY) == -1
    with N.option(N.OPT_HOST_CHUNK_VIEWS, 7):
        assert native_lib.tigre_get_option(N.OPT_HOST_CHUNK_VIEWS) == 7
    assert native_lib.tigre_get_option(N.OPT_HOST_CHUNK_VIEWS) == 0
    assert native_lib.tigre_set_option(99, 1) == -1
    assert "unknown option" in N.last_error()
