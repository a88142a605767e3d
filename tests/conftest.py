import json
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "tests"))
sys.path.insert(0, str(REPO / "how-mhd-kokkos_b200"))

# Achieved parity figures (max relative dt error, relative L1 per variable,
# ...) that tests report through the `parity_record` fixture: printed at the
# end of the session and, when HOW_PARITY_RECORD names a file, written there
# as JSON.
_RECORDS = []


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:   # noqa: BLE001
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture
def parity_record(request):
    """Call with keyword figures; they are stored under the test's id."""
    def rec(**kw):
        row = {"test": request.node.nodeid}
        for k, v in kw.items():
            try:
                import numpy as np
                if isinstance(v, np.ndarray):
                    v = v.tolist()
                elif isinstance(v, np.generic):
                    v = v.item()
            except ImportError:
                pass
            row[k] = v
        _RECORDS.append(row)
    return rec


def pytest_terminal_summary(terminalreporter):
    if not _RECORDS:
        return
    terminalreporter.write_sep("-", "achieved parity figures")
    for r in _RECORDS:
        terminalreporter.write_line(json.dumps(r))
    out = os.environ.get("HOW_PARITY_RECORD")
    if out:
        Path(out).parent.mkdir(parents=True, exist_ok=True)
        Path(out).write_text(json.dumps(_RECORDS, indent=1))
