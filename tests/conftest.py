"""Shared test set-up: repository root on sys.path, the `gpu` marker, and the CPU checkers
(oracle/liboracle_gauss.so, tests/native/libhostlogic.so) built on demand."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

HOSTLOGIC = os.path.join(ROOT, "tests", "native", "libhostlogic.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def build_checkers() -> None:
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle_gauss.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    if not os.path.exists(HOSTLOGIC):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                        "-I" + os.path.join(ROOT, "diplib_b200", "csrc"), "-o", HOSTLOGIC,
                        os.path.join(ROOT, "tests", "native", "host_logic_shim.cpp")], check=True)


build_checkers()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
