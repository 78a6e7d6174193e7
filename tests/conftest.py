import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    """The reference's own ED library, compiled as the CPU oracle."""
    from oracle import ref, refpath
    if not ref.available() and refpath.reference_root() is not None:
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle", "ref_build")] + refpath.make_args(),
                       check=True)
    if not ref.available():
        pytest.skip("oracle library not built")
    ref.lib()
    return ref


@pytest.fixture(scope="session")
def qed():
    """The product library (built in-tree); fails loudly when missing."""
    import pyqcm_b200
    from pyqcm_b200 import build
    if not os.path.exists(pyqcm_b200.LIB_PATH):
        build.build()
    pyqcm_b200.lib()
    return pyqcm_b200


_counter = [1000]


@pytest.fixture
def fresh():
    """Fresh (model name suffix, label) pairs: both libraries keep global registries."""
    def make():
        _counter[0] += 1
        return f"_{_counter[0]}", _counter[0]
    return make
