import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "k-wave-swift_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")


_TUNE_CACHE = None


@pytest.fixture(autouse=True)
def _private_tune_cache(request, tmp_path_factory, monkeypatch):
    """GPU tests keep the operator-pass autotuner's choices in a cache of their own (unless the run
    names one), so the small problems they tune do not land in the user's default cache."""
    global _TUNE_CACHE
    if request.node.get_closest_marker("gpu") is None or os.environ.get("KW_TUNE_CACHE"):
        yield
        return
    if _TUNE_CACHE is None:
        _TUNE_CACHE = str(tmp_path_factory.mktemp("tune") / "tune.json")
    monkeypatch.setenv("KW_TUNE_CACHE", _TUNE_CACHE)
    yield
