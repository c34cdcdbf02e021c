"""pytest configuration: the gpu marker, and in-tree builds of the CUDA
library and the oracle when they are missing (they travel prebuilt to GPU
machines)."""
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (the parity tests of the kernels)")
    lib = ROOT / "restir_b200" / "librestir_gpu.so"
    if not lib.exists():
        subprocess.run([sys.executable, "-m", "restir_b200.build"], cwd=ROOT, check=True)
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        cuda = torch.cuda.is_available()
    except Exception:
        cuda = False
    if cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
