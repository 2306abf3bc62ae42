"""Shared test setup: builds the native library and the oracle (incremental),
registers the `gpu` marker and puts the packages on sys.path."""
import faulthandler
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
PKG = os.path.join(ROOT, "map_b200")


faulthandler.enable()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    import importlib
    importlib.import_module("map_b200.build").build()
    from oracle import build_oracle
    build_oracle.build_oracle()
    build_oracle.build_ref_util()
    yield


@pytest.fixture(scope="session")
def M(_built):
    from map_b200 import map as M
    return M


@pytest.fixture()
def fresh(M):
    """Resets engine switches after a test that changes them."""
    yield M
    M.set_border(M.BORDER_BLOCK_MIRROR)
    M.set_exec_mode(M.EXEC_FUSED)
    M.set_paired_cells(True)
    M.set_flow_jump_cells(-1)
    M.set_algebraic_rewrite(True)
    M.set_prediction(True)
    M.set_default_blocksize([256, 256])
