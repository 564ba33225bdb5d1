"""The reference's own test module (python/tests/test_core.py), run unchanged through the import
aliases of ``boltzmann_b200.alias``.

The module is loaded from the reference checkout where one exists (``BOLTZMANN_REFERENCE``, else
``../reference`` beside this repository; it is not copied here, so the test is skipped on a
machine without it). Its three parameter tests are pure Python and must pass on the host as they
are. Its four simulation tests need the CUDA device: on a host without one, each must fail loudly
with the backend's PanicException (there is no CPU fallback); their bodies run on the GPU in
``tests/test_gpu_api.py`` through the same ``boltzmann.core`` alias.
"""

from __future__ import annotations

import importlib.util
import sys

import pytest

from oracle.build import reference_root

SUITE = reference_root() / "python" / "tests" / "test_core.py"
PARAMETER_TESTS = ["test_check_lbm_params", "test_calc_lbm_params_lu", "test_calc_lbm_params_si"]
SIMULATION_TESTS = ["test_simulation_1", "test_simulation_2", "test_simulation_3",
                    "test_simulation_serde"]


@pytest.fixture(scope="module")
def suite():
    if not SUITE.exists():
        pytest.skip("the reference checkout is not on this machine")
    from boltzmann_b200 import alias

    alias.install()
    spec = importlib.util.spec_from_file_location("reference_test_core", SUITE)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert mod.Simulation is sys.modules["boltzmann_b200.core"].Simulation
    return mod


def test_suite_lists_the_expected_tests(suite):
    names = {n for n in dir(suite) if n.startswith("test_")}
    assert names == set(PARAMETER_TESTS) | set(SIMULATION_TESTS)


@pytest.mark.parametrize("name", PARAMETER_TESTS)
def test_reference_parameter_test_passes(suite, name):
    getattr(suite, name)()


@pytest.mark.parametrize("name", SIMULATION_TESTS)
def test_reference_simulation_test_needs_the_device(suite, name):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: the GPU suite runs these")
    from boltzmann_b200.core import PanicException

    with pytest.raises(PanicException):
        getattr(suite, name)()
