import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle():
    import build_ref
    import pyoracle
    build_ref.build_oracle()
    return pyoracle.Oracle()


def pytest_terminal_summary(terminalreporter):
    """Parity evidence: for every field the condition-aware bound checked, its norm-wise error and how
    many values needed the input-rounding sensitivity term on top of the plain norm-wise tolerance."""
    try:
        from helpers import NORM_LOG, SLACK_LOG
    except ImportError:
        return
    for line in NORM_LOG:
        terminalreporter.write_line(line)
    if not SLACK_LOG:
        return
    tr = terminalreporter
    tot = sum(e[3] for e in SLACK_LOG)
    slack = sum(e[2] for e in SLACK_LOG)
    worst = max(SLACK_LOG, key=lambda e: e[2] / max(e[3], 1))
    tr.write_sep("-", "parity bound: %d fields, %d of %d values (%.4f%%) needed the sensitivity term; "
                      "most in one field: %s (%d of %d)" % (len(SLACK_LOG), slack, tot, 100.0 * slack / max(tot, 1),
                                                            worst[0], worst[2], worst[3]))
    for what, nerr, ns, nt, ratio in sorted(SLACK_LOG, key=lambda e: -e[2] / max(e[3], 1))[:40]:
        tr.write_line("  %-60s norm-wise %.2e  slack %d/%d  max err/tol %.2f" % (what[:60], nerr, ns, nt, ratio))
