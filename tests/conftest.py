import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200)')


@pytest.fixture(scope='session')
def panda():
    from rtcollisiondetection_b200 import scenes
    return scenes.load_panda()


@pytest.fixture(scope='session')
def small_scene():
    from rtcollisiondetection_b200 import scenes
    return scenes.discrete_small()


@pytest.fixture(scope='session')
def ctx():
    from rtcollisiondetection_b200 import rtcd
    c = rtcd.Context(0)
    yield c
    c.close()
