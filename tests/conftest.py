"""Test configuration: the ``gpu`` marker and import paths.

Tests marked ``gpu`` run the CUDA path on a B200 and compare it with the CPU
oracles under oracle/; everything else runs on the CPU.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size parity run (tens of seconds of CPU oracle)")
