import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden', 'reference_golden.npz')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200) and the built extension')


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason='no CUDA GPU here')
    for it in items:
        if 'gpu' in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope='session')
def golden():
    return dict(np.load(GOLDEN))


def ref_core():
    """The reference's compiled core (oracle/build_ref.sh), or None where it was not built."""
    d = os.path.join(ROOT, 'oracle', '_ref')
    if not os.path.isdir(d) or not any(f.startswith('_core') for f in os.listdir(d)):
        return None
    if d not in sys.path:
        sys.path.insert(0, d)
    import _core
    return _core
