"""Checkpoint interop on the GPU: a run on the device resumes from the reference's own checkpoint (step 7, with the
MUSCL-Hancock lagged speed where the scheme has one, and the pose and state of a moving immersed body: a 2-D body driven by
the flow with a driven rotation, a 3-D sphere in prescribed motion, a 3-D sphere driven by the flow) and reaches the
reference's uninterrupted step-15 state bit for bit; a checkpoint written by the device run and read back resumes it
exactly; the dump_state file round-trips; a moving-body run refuses a checkpoint without the body's pose."""
import json
import os

import numpy as np
import pytest

from fenice_b200 import Run
from fenice_b200 import checkpoint as ck

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FINAL = np.load(os.path.join(GOLD, "ckpt_final.npz"))
NAMES = ["hancock_2d", "weno5_rk3_3d", "free_circle_rk2_2d", "prescribed_sphere_3d", "free_sphere_3d"]


def bits_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
def test_device_resumes_from_the_reference_checkpoint(name):
    run = Run(json.loads(str(FINAL[f"{name}/params"])))
    step = ck.load_checkpoint(os.path.join(GOLD, f"ckpt_{name}.npz"), run)
    assert step == 7
    total = int(FINAL[f"{name}/step"])
    assert run.run(1e30, max_steps=total - step) == total - step
    ref = FINAL[f"{name}/U"]
    assert bits_equal(run.state()[:, :ref.shape[1]], ref)
    assert run.t == float(FINAL[f"{name}/t"])


@pytest.mark.parametrize("name", NAMES)
def test_device_checkpoint_round_trip(name, tmp_path):
    params = json.loads(str(FINAL[f"{name}/params"]))
    start = Run(params)
    ck.load_checkpoint(os.path.join(GOLD, f"ckpt_{name}.npz"), start)
    whole = Run(params)
    ck.load_checkpoint(os.path.join(GOLD, f"ckpt_{name}.npz"), whole)
    whole.run(1e30, max_steps=6)
    start.run(1e30, max_steps=3)
    path = str(tmp_path / "c.npz")
    ck.save_checkpoint(path, start, 10)
    resumed = Run(params)
    assert ck.load_checkpoint(path, resumed) == 10
    resumed.run(1e30, max_steps=3)
    assert bits_equal(resumed.state(), whole.state()) and resumed.t == whole.t
    dump = str(tmp_path / "d.npz")
    ck.dump_state(dump, resumed, 13)
    U, t, s = ck.read_dump(dump)
    assert bits_equal(U, resumed.state()) and t == resumed.t and s == 13


def test_moving_body_refuses_a_checkpoint_without_its_pose(tmp_path):
    """SimulationRestart.cpp:103: a run with a moving body does not resume from a file without body_pose."""
    name = "free_circle_rk2_2d"
    a = ck.read_checkpoint(os.path.join(GOLD, f"ckpt_{name}.npz"))
    del a["body_pose"]
    path = str(tmp_path / "static.npz")
    ck.write_checkpoint(path, a)
    run = Run(json.loads(str(FINAL[f"{name}/params"])))
    with pytest.raises(ValueError, match="no pose of the moving body"):
        ck.load_checkpoint(path, run)
