import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
GOLDEN = Path(__file__).resolve().parent / 'golden'


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200, sm_100a)')


def load_golden(name):
    return dict(np.load(GOLDEN / f'{name}.npz'))


def fluid_mask(case):
    from oracle_port import TYPES
    g = np.asarray(case['geometry'])
    fl = np.zeros(g.shape, bool)
    for k, (t, *_rest) in case['labels'].items():
        if TYPES[t] in (0x1, 0x2, 0x4, 0x8, 0x40):   # VD, GV, PB, VB, HF carry populations
            fl |= g == k
    return fl
