"""Drop-in proof: the reference's own fv::Simulation and TimeScheme (compiled from its sources) step a state with the GPU
residual passed through its ResidualFn seam (oracle/ref/dropin_check.cpp, include/fenice_gpu.hpp); the result must be the
reference's own run, bit for bit (states, every dt and wave speed)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "dropin_check")


@pytest.mark.skipif(not os.path.exists(EXE), reason="the drop-in check needs the reference's sources at build time (oracle/ref/Makefile dropin)")
@pytest.mark.parametrize("case,steps", [("vortex", 12), ("tgv", 3), ("riemann", 6), ("cylinder", 20), ("sources", 10), ("sources_rk3", 5)])
def test_reference_time_scheme_drives_gpu_residual(case, steps):
    r = subprocess.run([EXE, case, str(steps)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bit-identical" in r.stdout
