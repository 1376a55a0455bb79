import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from zlatko_b200 import build

    build.build()
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libccr_ref.so")
    oracle_lib = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
    if os.path.isdir("/root/reference") or not os.path.exists(ref_lib) or not os.path.exists(oracle_lib):
        # The GPU box has no reference sources: it uses the prebuilt oracle libraries that travel with the repo.
        targets = ["ref"] if os.path.isdir("/root/reference") else []
        if os.path.exists(os.path.join(ROOT, "oracle", "fused_oracle.c")):
            targets.append("restatement")
        if targets:
            subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle")] + targets, check=True)


_ensure_built()


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from zlatko_b200.gpu import Context

    c = Context(0)
    yield c
    c.close()
