"""Shared pytest setup: the `gpu` marker, import paths, and small LP builders."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ps26119-solver_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

# The reference sources ($PS26119_REFERENCE_DIR, else a "reference" directory beside this repository);
# their data files are present only where the sources are mounted.
REFERENCE_DIR = os.environ.get("PS26119_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")
REFERENCE_DATA = os.path.join(REFERENCE_DIR, "data")


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


def _build_host_probe(out_dir, defines=()):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "ps26119-solver_b200")
    csrc = os.path.join(pkg, "csrc")
    units = ("solver.cpp", "certify.cpp", "io.cpp")
    objs = [os.path.join(pkg, "_build", u + ".o") for u in units]
    if defines or not all(os.path.exists(o) for o in objs):
        objs = [os.path.join(csrc, u) for u in units]
    exe = str(out_dir / "host_probe")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", *[f"-D{d}" for d in defines], "-I", csrc, "-I",
           "/usr/local/cuda/include", os.path.join(root, "tests", "native", "host_probe.cpp"), *objs, "-o", exe,
           "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.fixture(scope="session")
def host_probe(tmp_path_factory):
    """tests/native/host_probe.cpp linked with the library's host objects (compiled from the
    library's sources when the build's objects are absent): the library's presolve, postsolve,
    check_solution and certified bound on model files, on the CPU."""
    return _build_host_probe(tmp_path_factory.mktemp("probe"))


@pytest.fixture(scope="session")
def host_probe_no_buckets(tmp_path_factory):
    """The host probe built from the library's sources with the row-block bucketing limited to
    4,096 entries, so that larger models take the passes' forms without scratch."""
    return _build_host_probe(tmp_path_factory.mktemp("probe_nb"), defines=("PS26119_BUCKET_MAX_ENTRIES=4096",))
