import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), os.path.join(ROOT, "turbo-cat_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

# the oracle is the checker; build it if this checkout has not yet
if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def engine():
    from turbocat import _capi

    return _capi.Engine(int(os.environ.get("TURBOCAT_DEVICE", "0")))


@pytest.fixture(scope="session")
def capi():
    from turbocat import _capi

    return _capi
