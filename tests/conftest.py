import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


_REPORT = []


def report(line):
    """A line for the session's closing summary (figures of the parity runs:
    points checked, escalation counts), so that a quiet run shows them."""
    _REPORT.append(line)


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if _REPORT:
        terminalreporter.write_sep("-", "parity figures")
        for line in _REPORT:
            terminalreporter.write_line(line)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def inputs():
    from tests.golden.fixtures import Inputs
    return Inputs()


@pytest.fixture(scope="session")
def ref_outputs():
    from tests.golden.fixtures import Outputs
    return Outputs()


@pytest.fixture(scope="session")
def oracle_ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")
    return ref
