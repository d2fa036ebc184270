"""Shared test set-up: the `gpu` marker and the two libraries under test.

`libzf.so` (the product, include/zf.h) with its C host driver `zf_run`, and
`oracle/liboracle.so` (the CPU restatement of the reference that the
parity tests compare against) are built on first use.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests proper")


def _ensure_built():
    if not all(os.path.exists(os.path.join(ROOT, "zebraflow_b200", f)) for f in ("libzf.so", "zf_run")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "zebraflow_b200", "csrc")],
                       check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return has_gpu()
