import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(REPO, "c3d-2015_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def pytest_terminal_summary(terminalreporter):
    """Tie exemptions of the closure parity checks that ran: cells checked, cells exempted
    as rounding ties, and how many of those differ from the oracle in iteration count."""
    mod = sys.modules.get("oracle_lib")
    log = getattr(mod, "TIE_LOG", None)
    if not log:
        return
    terminalreporter.section("rounding-tie exemptions")
    for label, n, ties, differ in log:
        terminalreporter.write_line(f"{label}: {ties} tie cells of {n}, {differ} of them with "
                                    f"another iteration count")


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import Oracle
    return Oracle()


def write_deck(tmp_path, **kw):
    from oracle_lib import deck_text
    d = tmp_path / "input.deck"
    d.write_text(deck_text(**kw))
    return str(d)
