"""TIGRE's unmodified Cython extensions linked to libtigre_b200.so (tests/dropin/build.py),
without a GPU: every call reports the missing device through the reference's own error
path instead of exiting the process, and the void regulariser entry points fill their
output with NaN rather than return uninitialised memory."""
import os

import numpy as np
import pytest

from tests.conftest import has_gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(HERE, "dropin", "_build")

pytestmark = pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")


@pytest.fixture(scope="module")
def T():
    from oracle import reference_package as RP
    if not RP.available("ours"):
        pytest.skip("drop-in build absent (tests/dropin/build.py needs the TIGRE source tree)")
    return RP.load("ours")


def test_reference_calls_report_errors_instead_of_exiting(T):
    from tests import geometries as G
    from tests.test_dropin_gpu import _ref_geometry
    from tigre.utilities.errors import TigreCudaCallError
    g = _ref_geometry(T, G.c1_geometry())
    ang = G.angles(4)
    with pytest.raises(ValueError, match="Call to Ax failed"):
        T.Ax(np.zeros((64, 64, 64), np.float32), g, ang, "Siddon")
    with pytest.raises(TigreCudaCallError):
        T.Atb(np.zeros((4, 128, 128), np.float32), g, ang, "matched")


def test_void_regularisers_return_nan_on_failure(T):
    from _minTV import minTV
    from _AwminTV import AwminTV
    img = np.ones((4, 5, 6), np.float32)
    assert np.isnan(minTV(img, 0.01, 2)).all()
    assert np.isnan(AwminTV(img, 0.01, 2)).all()
