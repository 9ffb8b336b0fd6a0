import json
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = ROOT / "tests" / "golden" / "golden.json"
GOLDEN_LARGE = ROOT / "tests" / "golden" / "golden_large.json"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and liblgpu.so")


@pytest.fixture(scope="session")
def ref():
    import lgref

    if not lgref.LIB_PATH.exists():
        lgref.build()
    return lgref


@pytest.fixture(scope="session")
def lg():
    import __graft_entry__ as g

    return g.load_package()


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())


@pytest.fixture(scope="session")
def golden_large():
    return json.loads(GOLDEN_LARGE.read_text())


@pytest.fixture(scope="session")
def ctx(lg):
    c = lg.Context(0)
    yield c
    c.close()
