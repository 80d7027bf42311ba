import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built libturbo_hot.so")


def pytest_terminal_summary(terminalreporter):
    from tests.helpers import ELEM_FLOOR, ELEMENTWISE_REPORT
    if not ELEMENTWISE_REPORT:
        return
    terminalreporter.write_sep("-", f"element-wise gradient errors (entries >= {ELEM_FLOOR:g} of the largest)")
    for what, n, worst in ELEMENTWISE_REPORT:
        terminalreporter.write_line(f"{what:60s} {n:10d} entries  worst rel err {worst:.3e}")
