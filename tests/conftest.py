"""Shared fixtures: import paths, the `gpu` marker, small meshes."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "amr-demo_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ag():
    import amrgpu
    amrgpu.lib()
    return amrgpu


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.restatement()
    return O
