"""Shared fixtures: the package (whose directory name is not an identifier), the
oracle bindings, golden fixtures and GPU availability."""
from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))


def load_pkg():
    name = "hydro_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, ROOT / "scalable-fpga-hydrodynamics_b200" / "__init__.py",
        submodule_search_locations=[str(ROOT / "scalable-fpga-hydrodynamics_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running (minutes)")


@pytest.fixture(scope="session")
def hb():
    return load_pkg()


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc

    return orc.Oracle()


@pytest.fixture(scope="session")
def orc():
    import oracle as orc_mod

    return orc_mod


@pytest.fixture(scope="session")
def kat():
    return json.loads((GOLDEN / "kat_logs.json").read_text())


@pytest.fixture(scope="session")
def ref_runs():
    meta = json.loads((GOLDEN / "ref_runs.json").read_text())
    arrays = dict(np.load(GOLDEN / "ref_runs.npz"))
    return meta, arrays


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    hb = load_pkg()
    hb.build()
    return torch
