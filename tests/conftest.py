"""Shared pytest configuration.

Markers:
  gpu   needs a CUDA device (a B200); runs the sm_100a kernels through the C ABI.
  slow  longer CPU work (still a few seconds to a minute).

The ``report`` fixture collects lines printed in the terminal summary, as the
reference's own conftest does for its verification diagnostics.
"""

from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

_REPORTS = pytest.StashKey[list]()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer-running CPU test")


@pytest.fixture(scope="session")
def report(pytestconfig):
    lines = pytestconfig.stash.setdefault(_REPORTS, [])
    return lines.append


def pytest_terminal_summary(terminalreporter, exitstatus, config):
    lines = config.stash.get(_REPORTS, [])
    if not lines:
        return
    terminalreporter.write_sep("=", "verification report")
    for line in lines:
        terminalreporter.write_line(line)
