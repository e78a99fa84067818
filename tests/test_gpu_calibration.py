"""The device primitive-cost calibration (rtb_calibrate_costs), run with a short protocol:
sphere-normalised weights come out positive and ordered the way the operations' work is
(affine tests above the plain sphere, one child box below an interior step of two), and
the protocol's limits return errors instead of running."""
import ctypes as C

import pytest

from rtb200 import calibrate as K
from rtb200 import native as N
from rtb200.tracer import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def test_quick_calibration(ctx):
    cal = K.calibrate(ctx, K.default_params(ctx.device_info().sm_count, quick=True))
    w = cal.weights
    assert w["sphere"] == 1.0
    for k, v in w.items():
        assert v > 0.0, k
    assert w["affineSphere"] > w["sphere"] and w["affineBox"] > w["sphere"]
    assert w["interiorTraversal"] > w["nodeAabb"]
    assert len(cal.per_profile) == 3 and all(s > 0 for s in cal.sphere_ns)
    cfg = cal.build_config()
    assert cfg.box_weight == w["box"]


def test_calibration_limits(ctx):
    w = K.calibration_workload(records=256, profiles=1)
    p = K.default_params(ctx.device_info().sm_count, quick=True)
    p.max_launch_ms = 1e-6  # every launch takes longer
    with pytest.raises(N.RtbError) as e:
        K.calibrate(ctx, p, w)
    assert e.value.status == 8  # RTB_ERR_LIMIT
    bad = N.CalibrationParams(p.blocks, 512, 16, 4, 4, 3, 1, 0, 250.0)  # too many threads
    with pytest.raises(ValueError):
        K.calibrate(ctx, bad, w)
