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
    # The plain-C restatement builds anywhere; the reference library only where its sources are (elsewhere the
    # prebuilt copy that travels with the repository, if any, is used).
    # The reference's sources: ZK_REFERENCE_DIR, else where the build container mounts them.
    reference = os.environ.get("ZK_REFERENCE_DIR", "/root/reference")
    targets = ["restatement"] + (["ref"] if os.path.isdir(reference) else [])
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), f"REF={reference}"] + targets, check=True)


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
