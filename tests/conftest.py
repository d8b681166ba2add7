import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


def pytest_collection_modifyitems(config, items):
    """A GPU test that stops making progress fails after 15 minutes instead of
    holding the device (pytest-timeout, when installed)."""
    try:
        import pytest_timeout  # noqa: F401
    except ImportError:
        return
    for item in items:
        if item.get_closest_marker("gpu") and not item.get_closest_marker("timeout"):
            item.add_marker(pytest.mark.timeout(900))


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build_oracle()
    return oracle


@pytest.fixture(scope="session")
def legacy_oracle_gf(oracle_mod):
    """Nemoh-2 settings of the reference's golden tests
    (pytest/test_consistency_with_Nemoh_2.py:24-33)."""
    return oracle_mod.OracleDelhommeau(tabulation_nr=328, tabulation_nz=46, tabulation_grid_shape="legacy",
                                       tabulation_nb_integration_points=251, gf_singularities="high_freq")


@pytest.fixture(scope="session")
def default_oracle_gf(oracle_mod):
    """Reference defaults (green_functions/delhommeau.py:30-41)."""
    return oracle_mod.OracleDelhommeau()


def hemisphere_volume(mesh):
    """Volume enclosed by an immersed mesh and the plane z=0 (divergence theorem on z)."""
    return float(np.sum(mesh.faces_areas * mesh.faces_normals[:, 2] * mesh.faces_centers[:, 2]))
