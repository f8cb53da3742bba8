import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libstopeps_gpu.so")


# Device paths added most recently run after the established parity suite, so
# that under ``-x`` a failure of theirs is reported without hiding the results
# of the paths before them; among themselves they run in the listed order
# (the smallest changes to established paths first).
# The order is otherwise unchanged.
LATE_MODULES = ("test_gpu_site_fields.py", "test_gpu_repair.py", "test_gpu_adjoint.py",
                "test_gpu_variational.py", "test_gpu_diagonal.py")


def pytest_collection_modifyitems(config, items):
    def rank(item):
        name = os.path.basename(str(item.fspath))
        return LATE_MODULES.index(name) + 1 if name in LATE_MODULES else 0
    items.sort(key=rank)


@pytest.fixture(scope="session")
def sps():
    import __graft_entry__ as g
    return g.load_package()
