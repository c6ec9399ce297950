import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libwamgpu.so")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "coarse_st6_protocol.json")) as f:
        return json.load(f)


def coarse_st6_config():
    """The configuration of the reference's own coarse ST6 run (const/WAM_User)."""
    from wam_b200.model import make_config
    return make_config(12, 25, 0.04177248, 2, 600, 300, 55555.5547, shallow_run=True, spherical_run=True,
                       lcflx=True, betamax=1.3, cdfac=1.08)
