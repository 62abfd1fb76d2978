"""Failure detection without a GPU fault: a bounded wait that runs out is reported, and the
device stays usable.

TIGRE_OPT_BP_SKIP_COPY makes the TMA-staged backprojector issue no copy (and no arrival) for
one view of each launch, so every block's bounded mbarrier wait for that view runs out with
nothing in flight.  The threads then wait no more, no further copy is issued, thread 0
waits for the copy of the next view that was already issued, and the block writes nothing,
sets TIGRE_STATUS_WAIT_EXPIRED in the plan status word and exits;
the device call returns normally (the status is the report), the host call returns
TIGRE_ERR_CUDA.  Afterwards the same plan and the host entry points give correct results.
"""
import numpy as np
import pytest

from tests import geometries as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _case():
    geo = G.c1_geometry()
    ang = G.angles(12)
    img = G.phantom((64, 64, 64), seed=6)
    return geo, ang, img, O.ax(img, geo, ang, "Siddon")


@pytest.mark.parametrize("view", [0, 5, 11])
def test_expired_wait_sets_status_on_the_device_api(view):
    import torch
    from tigre_b200 import _native as N, projectors as P
    geo, ang, img, proj = _case()
    dproj = torch.from_numpy(proj).cuda()
    with N.option(N.OPT_BP_SKIP_COPY, view):
        plan = N.get_plan(N.checked_geometry(geo, ang), 0)
        assert plan.status() == 0
        P.atb(dproj, plan, "matched")
        st = plan.status()
        assert st & N.STATUS_WAIT_EXPIRED, st
    # the context is intact: a fresh plan backprojects correctly and reports nothing
    plan = N.get_plan(N.checked_geometry(geo, ang), 0)
    got = P.atb(dproj, plan, "matched").cpu().numpy()
    mx, l2 = G.rel_err(got, O.atb(proj, geo, ang, "matched"))
    assert mx <= TOL and l2 <= TOL, (mx, l2)
    assert plan.status() == 0


def test_expired_wait_fails_the_host_call():
    import tigre_b200 as tigre
    from tigre_b200 import _native as N
    from tigre_b200.utilities.errors import TigreCudaCallError
    geo, ang, img, proj = _case()
    with N.option(N.OPT_BP_SKIP_COPY, 2):
        with pytest.raises(TigreCudaCallError) as e:
            tigre.Atb(proj, geo, ang, "FDK")
        assert e.value.error_index == 1
        assert "bounded wait expired" in str(e.value)
    got = tigre.Atb(proj, geo, ang, "FDK")
    mx, l2 = G.rel_err(got, O.atb(proj, geo, ang, "FDK"))
    assert mx <= TOL and l2 <= TOL, (mx, l2)
    # a failed call does not leave its status behind for the next one
    got2 = tigre.Atb(proj, geo, ang, "matched")
    mx, l2 = G.rel_err(got2, O.atb(proj, geo, ang, "matched"))
    assert mx <= TOL and l2 <= TOL, (mx, l2)


def test_projection_after_failed_backprojection_succeeds():
    """The status word is per call: a projection on the same cached plan after a failed
    backprojection reports no error (each host call clears the word before its launches)."""
    import tigre_b200 as tigre
    from tigre_b200 import _native as N
    from tigre_b200.utilities.errors import TigreCudaCallError
    geo, ang, img, proj = _case()
    with N.option(N.OPT_BP_SKIP_COPY, 1):
        with pytest.raises(TigreCudaCallError):
            tigre.Atb(proj, geo, ang, "matched")
        got = tigre.Ax(img, geo, ang, "Siddon")
    mx, l2 = G.rel_err(got, proj)
    assert mx <= TOL and l2 <= TOL, (mx, l2)
