"""Seeded synthetic decks of the sweep-lane workloads (the reference has no
public suite for this path; these stand in with the stated shapes, sizes and
value distributions, and fixed seeds).

grid_diodes: an 8x8 resistor grid (R log-uniform in [100, 10k] ohm), 16
diodes (IS = 1e-14 A, N = 1, RS = 10 ohm) from seeded grid nodes to ground
and one voltage source at the corner node, swept 0..5 V in 256 points. About
82 unknowns with the diodes' internal nodes and the source's branch row.
"""

from __future__ import annotations

import numpy as np

from .circuit import Circuit


def grid_diodes(seed: int = 1, rows: int = 8, cols: int = 8, n_diodes: int = 16,
                points: int = 256, v_stop: float = 5.0):
    """Returns (frozen circuit, [source dc slot], sweep values [points][1])."""
    rng = np.random.default_rng(seed)
    c = Circuit()
    name = lambda r, k: f"n{r}_{k}"  # noqa: E731
    c.V("vin", name(0, 0), "0", dc=0.0)
    for r in range(rows):
        for k in range(cols):
            if k + 1 < cols:
                c.R(f"rh{r}_{k}", name(r, k), name(r, k + 1), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
            if r + 1 < rows:
                c.R(f"rv{r}_{k}", name(r, k), name(r + 1, k), float(np.exp(rng.uniform(np.log(100), np.log(1e4)))))
    nodes = rng.choice(rows * cols, size=n_diodes, replace=False)
    for i, nd in enumerate(sorted(int(v) for v in nodes)):
        c.D(f"d{i}", name(nd // cols, nd % cols), "0", is_=1e-14, n=1.0, rs=10.0)
    fr = c.freeze()
    slot = fr.slot("vin", "dc")
    values = np.linspace(0.0, v_stop, points).reshape(-1, 1)
    return fr, [slot], values
