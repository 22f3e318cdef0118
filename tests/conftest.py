import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# the autotuner's disk cache of this test session stays in a scratch file
if "HITB200_TUNE_CACHE" not in os.environ:
    import tempfile

    os.environ["HITB200_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="hitb200_tune_"),
                                                    "tuning.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import pytest

    try:
        import torch

        has_cuda = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_cuda = False
    if has_cuda:
        return
    skip = pytest.mark.skip(reason="needs a CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
