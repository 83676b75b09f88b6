import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# Parity figures recorded by the tests (name -> dict), printed as one JSON line
# each at the end of the session, so that a quiet run (-q) still shows them,
# and written to $XPBD_PARITY_JSON when that is set.
_PARITY: dict = {}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) and the built libxpbd_b200.so")


@pytest.fixture
def parity_record():
    """record(name, **figures): keep a test's measured errors for the session summary."""
    def record(name, **figures):
        _PARITY[name] = {k: (float(v) if hasattr(v, "__float__") and not isinstance(v, (bool, int)) else v)
                         for k, v in figures.items()}
    return record


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    if not _PARITY:
        return
    terminalreporter.write_sep("-", "parity figures")
    for name, figs in _PARITY.items():
        terminalreporter.write_line(json.dumps({"parity": name, **figs}, default=str))
    out = os.environ.get("XPBD_PARITY_JSON")
    if out:
        Path(out).write_text(json.dumps(_PARITY, indent=1, default=str))
