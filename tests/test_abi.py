"""CPU checks of the C ABI: the library loads and exports every entry
point include/espice_lanes.h declares (no compute without a GPU)."""

import os
import re

from espice_b200 import lanes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    with open(os.path.join(ROOT, "include", "espice_lanes.h")) as fh:
        text = fh.read()
    return sorted(set(re.findall(r"\b(esl_[a-z_]+)\s*\(", text)))


def test_header_declarations_listed():
    assert declared() == sorted(lanes.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = lanes.lib()
    missing = [s for s in declared() if not hasattr(lib, s)]
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
