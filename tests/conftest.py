import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def reference_root():
    """The reference's source tree, for the CPU tests that read its headers, scenes and unit-test
    files: $POLYTOPE_REFERENCE, else the tree oracle/Makefile built oracle/_ref from (recorded in
    oracle/_ref/ref_root.txt).  None when neither names an existing directory (those tests skip)."""
    root = os.environ.get("POLYTOPE_REFERENCE")
    if not root:
        try:
            with open(os.path.join(ROOT, "oracle", "_ref", "ref_root.txt")) as f:
                root = f.read().strip()
        except OSError:
            return None
    return root if root and os.path.isdir(root) else None


def reference_path(*parts):
    """A path inside the reference tree, or a path that does not exist when the tree is absent."""
    root = reference_root()
    return os.path.join(root, *parts) if root else os.path.join(ROOT, "_no_reference_tree", *parts)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_bit_equal(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    ba, bb = bits(a), bits(b)
    bad = np.nonzero(ba.ravel() != bb.ravel())[0]
    assert bad.size == 0, f"{what}: {bad.size} mismatches, first at {bad[:5]}: {a.ravel()[bad[:5]]} vs {b.ravel()[bad[:5]]}"


@pytest.fixture(scope="session")
def cuda_device():
    """GPU tests fail (not skip) without a device: they only run where one is expected."""
    import torch
    assert torch.cuda.is_available(), "gpu-marked test needs a CUDA device"
    return torch.device("cuda:0")
