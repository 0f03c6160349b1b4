"""The C++ drop-in: the dip::GaussFIR device branch a DIPlib maintainer adds (the code INTEGRATION.md
quotes, in tests/native/gaussfir_dropin.cpp) compiled against DIPlib's own headers and linked with
the reference build and libdipcu.so.  The program forges dip::Images in device memory through a
cudaMalloc-backed dip::ExternalInterface, runs the branch -- 1D to 3D, sfloat, uint8, uint16, sint32
and dfloat input, a tensor image, a protected integer output, an in-place call, mixed boundary
conditions -- and compares each result with the host dip::GaussFIR of the reference build, then
checks that bad arguments throw the reference's errors."""
from __future__ import annotations

import os
import subprocess

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

PROGRAM = os.path.join(ROOT, "tests", "native", "gaussfir_dropin")


def test_gaussfir_device_branch_matches_host_dip_gaussfir(cuda):
    if not os.path.exists(PROGRAM):
        pytest.skip("tests/native/gaussfir_dropin is built only where the DIPlib reference tree is present")
    r = subprocess.run([PROGRAM], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "ALL OK" in r.stdout
