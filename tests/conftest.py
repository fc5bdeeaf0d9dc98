"""Shared fixtures: the product library, the oracle restatement and (when built)
the library compiled from the reference sources."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE_TREE = os.environ.get("KARAM_REFERENCE_TREE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests proper")


@pytest.fixture(scope="session")
def product():
    from karam_b200 import build
    build.build()
    import karam_b200
    return karam_b200


@pytest.fixture(scope="session")
def port():
    from oracle import pyoracle
    pyoracle.build("port")
    return pyoracle.Oracle("port")


@pytest.fixture(scope="session")
def ref():
    """The oracle built from the reference's own sources. Built here when the
    reference tree is present; elsewhere the prebuilt library is used if it
    travelled with the repository."""
    from oracle import pyoracle
    if os.path.isdir(REFERENCE_TREE):
        pyoracle.build("ref")
    if not pyoracle.available("ref"):
        pytest.skip("reference-built oracle not available")
    return pyoracle.Oracle("ref")


@pytest.fixture(scope="session")
def ctx(product):
    return product.Context(0)
