import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a) and the built CUDA library')


def golden_cases():
    return sorted(fn[:-4] for fn in os.listdir(GOLDEN) if fn.endswith('.npz') and fn not in ('mesh_kernels.npz',
                                                                                              'utils.npz'))


@pytest.fixture(scope='session')
def golden_dir():
    return GOLDEN
