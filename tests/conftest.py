import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a)")
    config.addinivalue_line("markers", "large: full-size configuration (720k / 2.9M cells)")


def _ensure_built():
    from oplus2_matlab_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from oplus2_matlab_b200 import build
        build.build()


_ensure_built()


@pytest.fixture
def op2():
    """A fresh OP2 session on cuda:0: op_init, errors returned instead of
    exiting, default strategy and reduction restored, op_exit afterwards."""
    from oplus2_matlab_b200 import api
    api.set_error_mode(api.ERRORS_RETURN)
    api.clear_error()
    api.op_init([], 0)
    assert api.last_error() == "", api.last_error()
    old_s = api.set_strategy(api.STRATEGY_AUTO)
    old_r = api.set_reduction(api.REDUCE_TREE)
    yield api
    err = api.last_error()
    api.op_exit()
    api.set_strategy(old_s)
    api.set_reduction(old_r)
    api.clear_error()
    assert err == "", err


def scratch_dir():
    """A private scratch directory inside the repository (tests/golden/_scratch
    is git-ignored)."""
    import tempfile
    base = os.path.join(GOLDEN, "_scratch")
    os.makedirs(base, exist_ok=True)
    return tempfile.mkdtemp(dir=base)


def load_golden(name):
    import json
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)
