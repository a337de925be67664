import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def built_lib():
    from tensorray_b200 import build
    return build.build()


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    """Print the measured GPU-vs-oracle errors of the parity tests."""
    try:
        from tests.helpers import PARITY_LOG
    except Exception:
        return
    if not PARITY_LOG:
        return
    tr = terminalreporter
    tr.write_sep("-", "parity errors (CUDA path vs oracle, same samples)")
    for label, what, val, extra in PARITY_LOG:
        tr.write_line(f"{label:<48} {what:<14} {val:.3e}  {extra}")
