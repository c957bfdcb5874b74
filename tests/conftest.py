import os
import sys

import numpy as np
import pytest

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


class FixtureLove:
    """Love-number object rebuilt from the arrays stored in a golden fixture."""

    def __init__(self, fx, prefix="love_"):
        for key in ("s", "r", "rprime", "rT", "rprimeT", "he", "ke", "hTE", "kTE", "nmod", "le", "lTE", "rl",
                    "rlT"):
            if prefix + key in fx:
                setattr(self, key, np.asarray(fx[prefix + key]))
        self.max_modes = int(self.s.shape[0])


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def golden():
    return load_golden
