"""The oracle still reproduces the committed golden fixtures (regression guard)."""
import numpy as np
import pytest

from oracle import np_oracle as O
from tests.conftest import load_case
from tests.golden.make_fixtures import BASE, CASES, make


@pytest.mark.parametrize("name", sorted(CASES))
def test_fixture_regenerates(name):
    ref = load_case(name)
    new = make(name, CASES[name])
    for k, v in ref.items():
        if k == "config" or k.startswith("sens_"):
            continue
        a, b = np.asarray(new[k]), np.asarray(v)
        assert a.shape == b.shape, k
        scale = max(1.0, float(np.max(np.abs(b)))) if b.size else 1.0
        assert np.max(np.abs(a - b), initial=0.0) <= 1e-13 * scale, k


def test_fixture_cases_cover_every_orbit_branch():
    seen = set()
    for name, over in CASES.items():
        c = O.OracleConfig(**{**BASE, **over})
        g = O.compute_grids(c, O.ToomreZang.from_config(c))
        e, L2 = g.e, g.L2_m
        if (np.abs(e) < 1e-10).any():
            seen.add("circular")
        if ((e >= 1e-10) & (e < 0.01)).any():
            seen.add("epicyclic")
        if ((e >= 0.01) & (L2 > 1e-12)).any():
            seen.add("general")
        if ((e >= 0.01) & (L2 <= 1e-12)).any():
            seen.add("radial")
        if (g.SGNL < 0).any():
            seen.add("retrograde")
    assert seen == {"circular", "epicyclic", "general", "radial", "retrograde"}
