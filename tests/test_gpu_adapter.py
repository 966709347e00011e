"""The reference's own scenarios (two bodies under SyplecticEuler, 3D FMM vs
NaiveUpdate) run by the reference's classes with the GPU update methods of
nbody-fmm_b200/cpp/gpu_fmm.hpp plugged in (oracle/adapter_check.cpp)."""
import os
import subprocess

import pytest
from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_reference_classes_drive_gpu_update_methods():
    exe = os.path.join(ROOT, "oracle", "_ref", "adapter_check")
    if not os.path.exists(exe):
        pytest.skip("adapter_check not built (needs the reference sources)")
    r = subprocess.run([exe], capture_output=True, timeout=300)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
