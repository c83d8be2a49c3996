"""B200 sweep-lane Newton: the reference's GPU sweep-lane hot path (device
eval and stamp, Jacobian assembly, Gilbert-Peierls refactor on a frozen
pivot tape, forward/back solves, the Newton loop) as one fused sm_100a
kernel behind a C ABI (include/espice_lanes.h)."""

from .circuit import Circuit, Frozen, Slot  # noqa: F401
