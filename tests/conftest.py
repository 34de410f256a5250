"""Shared pytest setup: the `gpu` marker, import paths, and small LP builders."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ps26119-solver_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

REFERENCE_DATA = "/root/reference/data"  # present only where the reference sources are mounted


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    # GPU tests without a device are skipped, never silently passed on a CPU path.
    try:
        import torch
        have = torch.cuda.is_available()
    except Exception:
        have = False
    if have:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ref():
    import reference
    if not reference.available():
        pytest.skip("oracle/_ref not built (make -C oracle ref)")
    return reference


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not oracle.available():
        pytest.skip("oracle/liboracle.so not built (make -C oracle oracle)")
    return oracle
