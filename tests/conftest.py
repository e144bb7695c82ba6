"""Shared pytest setup: the `gpu` marker and repository paths."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def pytest_sessionstart(session):
    # the oracle (CPU checker) may use every host core
    try:
        from oracle import oracle as O
        O.set_threads(os.cpu_count() or 1)
    except Exception:  # the oracle library is built by __graft_entry__.build()
        pass
