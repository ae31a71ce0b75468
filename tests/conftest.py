import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_blocks.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle

    if not os.path.exists(oracle.REF_SO):
        pytest.skip("compiled reference (oracle/_ref) not present")
    return oracle.Reference()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def lc():
    import leco_b200

    leco_b200.lib()
    return leco_b200


@pytest.fixture(scope="session")
def dev():
    import torch

    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch.device("cuda:0")


def golden_cases(golden):
    """Yields (key, codec, s, n, family) for every per-block golden case."""
    names = {"leco": 0, "for": 1, "delta": 2, "poly2": 3}
    for k in golden.files:
        if not k.endswith("__image"):
            continue
        key = k[: -len("__image")]
        cname, t, nn, fam = key.split("_", 3)
        yield key, names[cname], int(t[1:]) // 8, int(nn[1:]), fam
