import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtbr.so")


def _cuda_available() -> bool:
    try:
        import torch  # noqa: F401  (only to ask the driver; the product does not use torch)
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc
    if not os.path.exists(orc.LIB):
        orc.build(ref=False)
    return orc.Oracle()


@pytest.fixture(scope="session")
def ref_harness():
    from oracle import oracle as orc
    if not os.path.exists(orc.REF_LIB):
        if not os.path.isdir(orc.REF_SRC):
            pytest.skip("reference tree not available (fixtures cover this case)")
        orc.build(ref=True)
    return orc.RefHarness()


@pytest.fixture(scope="session")
def ctx():
    from turboransac_b200 import Context, build
    build.build()
    return Context(0, 2 << 30)
