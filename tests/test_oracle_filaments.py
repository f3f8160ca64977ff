"""The oracle's filament forces against golden vectors from the reference's own chain_bending /
chain_tension (python/simulate.py:14-88, assembled as at :130-142; tests/golden/
make_filament_golden.py): bit-exact. CPU only."""
import os

import numpy as np
import pytest

from oracle import hignn_oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "filament_forces.npz")


@pytest.mark.parametrize("case", ["chains", "short", "pairs", "single"])
def test_filament_forces_match_reference(case):
    g = np.load(GOLD)
    nf, nc, L, kt, kb = g[f"{case}_params"]
    f = O.filament_forces(g[f"{case}_x"], g[f"{case}_f0"], int(nf), int(nc), L, kt, kb)
    assert f.dtype == np.float32
    assert np.array_equal(f, g[f"{case}_f"])
