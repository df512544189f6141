import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "qphix-codegen_b200"), os.path.join(REPO, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from qphix_b200 import _lib
    _lib.lib()
    return torch.device("cuda:0")


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    """Print the worst error of every parity check that ran (tests record
    them through helpers.record); QB200_PARITY_JSON names a file to write
    the same table to."""
    mod = sys.modules.get("helpers")
    table = getattr(mod, "PARITY", None) if mod is not None else None
    if not table:
        return
    terminalreporter.write_sep("-", "worst parity errors (per component, relative)")
    for name in sorted(table):
        err, tol = table[name]
        terminalreporter.write_line("%-72s %.3e%s" % (name, err, "" if tol is None else "  (bound %.0e)" % tol))
    path = os.environ.get("QB200_PARITY_JSON")
    if path:
        import json
        with open(path, "w") as f:
            json.dump({k: {"worst": v[0], "bound": v[1]} for k, v in table.items()}, f, indent=1, sort_keys=True)
