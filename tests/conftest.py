"""Shared pytest set-up: the `gpu` marker, the oracle (checker) fixture and the
product package loader."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def pkg():
    import __graft_entry__

    mod = __graft_entry__.load_package()
    mod.lib()
    return mod


@pytest.fixture(scope="session")
def host_ctx(pkg):
    ctx = pkg.Context(-1)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def gpu_ctx(pkg):
    ctx = pkg.Context(0)
    yield ctx
    ctx.close()
