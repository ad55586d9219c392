import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")], stdout=subprocess.DEVNULL)
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden_decode():
    return load_golden("decode_golden.json")


@pytest.fixture(scope="session")
def golden_encode():
    return load_golden("encode_golden.json")


@pytest.fixture(scope="session")
def golden_tables():
    return load_golden("tables_golden.json")


@pytest.fixture(scope="session")
def golden_misc():
    return load_golden("misc_golden.json")


@pytest.fixture(scope="session")
def wl():
    """The product bindings; GPU tests need the built library."""
    import wimax_ldpc_lib_b200 as wl
    wl.lib()
    return wl


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test without a CUDA device"
    return torch
