import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the device engine")


@pytest.fixture(scope="session")
def lib():
    from fevc_b200 import abi, build

    build.build()
    return abi.load()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.library()
    return oracle


@pytest.fixture(scope="session")
def golden():
    import json

    d = ROOT / "tests" / "golden"
    return {"prep": json.loads((d / "prep_cases.json").read_text()),
            "jla": json.loads((d / "jla_cases.json").read_text())}


@pytest.fixture(scope="session")
def has_gpu(lib):
    return lib.fevcb_device_count() > 0
