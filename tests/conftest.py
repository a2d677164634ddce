"""Shared test fixtures.

Marker `gpu`: needs a B200 (run with `-m gpu`); everything else runs on CPU.
The CPU oracle (oracle/) is the checker; it is built on first use.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (run with -m gpu)")


def make_system(name, ncell=None, seed=2026):
    """Normalised AO system for a named workload (optionally on fewer cells)."""
    import pyoracle
    from william_ci_b200 import system as S
    cell, basis = S.workload(name, seed=seed)
    if ncell is not None:
        cell = S.scaled_down(cell, ncell)
    sysm = S.build_system(cell, basis)
    pyoracle.normalize(sysm)
    return sysm


@pytest.fixture(scope="session")
def systems():
    cache = {}

    def get(name, ncell=None):
        key = (name, tuple(ncell) if ncell else None)
        if key not in cache:
            cache[key] = make_system(name, ncell)
        return cache[key]
    return get


def random_density(n, seed=0):
    rng = np.random.default_rng(seed)
    P = rng.standard_normal((n, n)) * 0.3
    return P + P.T
