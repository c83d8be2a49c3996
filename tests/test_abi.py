"""CPU checks of the C ABI: the library loads and exports every entry
point include/espice_lanes.h, include/espice_mlp.h and
include/espice_points.h declare (no compute without a GPU)."""

import os
import re

from espice_b200 import lanes, mlp, points

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    with open(os.path.join(ROOT, "include", header)) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"\b(esl_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_listed():
    assert declared("espice_lanes.h") == sorted(lanes.EXPORTS)
    assert declared("espice_mlp.h") == sorted(mlp.EXPORTS)
    assert declared("espice_points.h") == sorted(points.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = lanes.lib()
    missing = [s for h in ("espice_lanes.h", "espice_mlp.h", "espice_points.h") for s in declared(h) if not hasattr(lib, s)]
    assert not missing, missing


def test_no_device_is_reported_not_faked():
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    from espice_b200 import decks
    fr, _, _ = decks.grid_diodes(points=4)
    with pytest.raises(lanes.LaneError) as e:
        lanes.DcLanes(fr)
    assert e.value.code == lanes.ESL_NO_DEVICE
    with pytest.raises(mlp.MlpError) as e:
        mlp.Mlp(4, 32, 2, 4)
    assert e.value.code == 5  # ESL_MLP_NO_DEVICE


def test_points_config_checked_before_the_device():
    """esl_points_create refuses a bad configuration with INVALID_ARGUMENT
    before it looks for a device, and reports a missing device as FAILED."""
    import torch
    import pytest
    from espice_b200 import decks
    fr, slots, _ = decks.grid_diodes(points=4)
    bad = [
        dict(analysis=points.TRAN, results=[("x1", points.RESULT_UNKNOWN, 1)]),
        dict(analysis=points.OP, results=[("m", points.RESULT_MEASURE, 0)]),
        dict(analysis=points.OP, results=[("x1", points.RESULT_UNKNOWN, fr.n)]),
        dict(analysis=points.OP, results=[("x1", points.RESULT_UNKNOWN, 1), ("X1", points.RESULT_UNKNOWN, 2)]),
        dict(analysis=2, results=[]),
    ]
    for kw in bad:
        with pytest.raises(points.PointsError) as e:
            points.Points(fr, slots, **kw)
        assert e.value.code == points.PTS_INVALID_ARGUMENT, kw
    if not torch.cuda.is_available():
        with pytest.raises(points.PointsError) as e:
            points.Points(fr, slots, points.OP, [("x1", points.RESULT_UNKNOWN, 1)])
        assert e.value.code == points.PTS_FAILED


def test_analog_block_live_parameter_columns():
    """The analog block's 16 live parameters (temperature in kelvin) taken
    through its slot-to-column map are its 248 expanded lane values."""
    import numpy as np

    from espice_b200 import decks
    fr, expand = decks.analog_block()
    p, _ = decks.analog_block_params(seed=9, points=64)
    assert len(expand.cols) == len(expand.slots)
    assert np.array_equal(expand.lane_params(p)[:, expand.cols], expand(p))
