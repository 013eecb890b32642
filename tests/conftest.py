import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def orc():
    from oracle import build_oracle, oracle
    build_oracle.build_oracle()
    oracle.set_fp_mode(oracle.FP_HOST)
    return oracle


@pytest.fixture(scope="session")
def ref(orc):
    """the reference's own per-candidate functions (oracle/_ref), or skip"""
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref/libfastrrt_ref.so not built")
    return orc


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import fastrrt_b200
    fastrrt_b200.lib()
    return fastrrt_b200
