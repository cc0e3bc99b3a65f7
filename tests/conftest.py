"""Shared fixtures.  `-m gpu` tests need a CUDA device and the built library;
everything else runs on the CPU (library loading, host table builder, input
formats, oracle pinning, multi-process host logic)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def assets_root():
    from ompmc_b200 import assets
    return assets.require_assets()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))
    return load


CASES = {
    "water30": dict(media=["H2O521ICRU"], collimator=(-5.0, 5.0, -5.0, 5.0)),
    "slab64": dict(media=["H2O521ICRU", "LUNG521ICRU", "ICRPBONE521ICRU"], collimator=(-2.5, 2.5, -2.5, 2.5)),
    "ctsmall": dict(media=["AIR521ICRU", "LUNG521ICRU", "ICRUTISSUE521ICRU", "ICRPBONE521ICRU"],
                    collimator=(-5.0, 5.0, -5.0, 5.0)),
}


def case_phantom(name):
    from ompmc_b200 import assets as A
    if name == "water30":
        return A.water_cube(30, 1.0)
    if name == "slab64":
        return A.slab_phantom(64, 0.25)
    if name == "ctsmall":
        return A.ct_phantom(32, 32, 24, 1.2, seed=7)
    raise KeyError(name)


def z_outliers_allowed(n):
    """Voxels that may lie beyond |z| = 3 in a z-test over n voxels: 1 % of
    them, or for small n the 99.9 % Poisson quantile of the count expected
    when z follows a Student t of about 50 degrees of freedom (0.5 % of the
    voxels), whichever is larger."""
    from scipy.stats import poisson
    return max(int(0.01 * n), int(poisson.ppf(0.999, 0.005 * n)))


_engines = {}


@pytest.fixture(scope="session")
def engine_for(assets_root):
    """Engine (FP64 + FP32 tables resident) for a named golden case."""
    from ompmc_b200.engine import Engine, Tables

    def get(name, data="data", **kw):
        """data: the data folder under the assets root (`data_spin`: the
        synthetic, non-constant spin file)."""
        key = (name, data, tuple(sorted(kw.items())))
        if key not in _engines:
            if data == "data_spin":
                from ompmc_b200 import assets as A
                A.stage_spin_variant(assets_root)
            t = Tables.from_assets(CASES[name]["media"], assets_root, data=data)
            _engines[key] = Engine(t, case_phantom(name), **kw)
        return _engines[key]
    yield get
    for e in _engines.values():
        e.close()
    _engines.clear()
