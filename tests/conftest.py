import pytest

from tests.helpers import golden  # noqa: F401  (re-exported for convenience)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests against the oracle")


@pytest.fixture(scope="session")
def lib():
    from cmpmc_b200 import _ffi
    return _ffi.load()


@pytest.fixture(scope="session")
def ge_lattice():
    import cmpmc_b200 as cm
    return cm.CrystalLattice(cm.materials.Germanium())
