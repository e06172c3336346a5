import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(REPO, "tests", "golden")


@pytest.fixture(scope="session")
def parity_log():
    """record(name, **values): print a measured error figure and, when MC_PARITY_LOG names a
    file, append it there as one JSON line (the figures quoted beside each bar)."""
    import json

    path = os.environ.get("MC_PARITY_LOG")

    def record(name, **values):
        line = json.dumps({"test": name, **{k: (float(v) if not isinstance(v, (str, list, dict)) else v)
                                            for k, v in values.items()}})
        print(line)
        if path:
            with open(path, "a") as fh:
                fh.write(line + "\n")

    return record
