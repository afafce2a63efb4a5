import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "meraxes-devs_qyxnew_b200", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_sessionfinish(session, exitstatus):
    """Write the error table of the configuration-level parity tests (helpers.record) to the file
    RG_PARITY_TABLE names, if any."""
    path = os.environ.get("RG_PARITY_TABLE")
    if not path:
        return
    helpers = sys.modules.get("helpers")
    rows = getattr(helpers, "PARITY_ROWS", None) if helpers else None
    if not rows:
        return
    lines = ["| configuration | output | measure | value | gate |", "|---|---|---|---|---|"]
    for cfg, out, measure, value, gate in rows:
        lines.append(f"| {cfg} | {out} | {measure} | {value:.3e} | {gate} |")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
