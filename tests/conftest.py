"""Shared test setup.

The package directory is ``marinehydro.jl_b200/`` (a name with a dot, so it is
loaded by path and registered as ``marinehydro_b200``).  ``-m gpu`` selects
the tests that need a B200; everything else runs on the CPU.
"""
from __future__ import annotations

import importlib.util
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def load_package():
    name = "marinehydro_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "marinehydro.jl_b200"
    spec = importlib.util.spec_from_file_location(
        name, pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def mh():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def gpu(mh):
    """A context on device 0; GPU tests are skipped where no device is visible."""
    if mh.device_count() == 0:
        pytest.skip("no CUDA device visible")
    ctx = mh.Context(0)
    yield ctx
    ctx.close()


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture
def series_fp64(gpu):
    """The mixed path's wave pass with its Horner series in FP64 (level 0)
    for the duration of a test: the tests that check the frequency-batched
    kernels against the one-frequency FP64 path to 1e-8 or tighter run the
    kernels' FP64 form; the default FP32 series (level 1) has its own bounds."""
    gpu.set_wave_series_fp32(0)
    yield gpu
    gpu.set_wave_series_fp32(1)
