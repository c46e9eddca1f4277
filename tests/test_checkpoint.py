"""Checkpoint interop with the reference (fenice_b200.checkpoint): the reference's own checkpoints
(tests/golden/ckpt_*.npz, written by its solver through tests/golden/make_checkpoint.py) are read here, a checkpoint
written here has the reference's keys, types and shapes, and, where the reference is compiled (oracle/_ref), the
reference resumes from a checkpoint written here and reaches its uninterrupted run's final state bit for bit."""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from fenice_b200 import checkpoint as ck
from fenice_b200 import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
FENICE = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "fenice")
NAMES = ["hancock_2d", "weno5_rk3_3d", "free_circle_rk2_2d", "prescribed_sphere_3d", "free_sphere_3d"]
MOVING = {"free_circle_rk2_2d": 13, "prescribed_sphere_3d": 14, "free_sphere_3d": 21}
FINAL = np.load(os.path.join(GOLD, "ckpt_final.npz"))


def ref_ckpt(name):
    return ck.read_checkpoint(os.path.join(GOLD, f"ckpt_{name}.npz"))


@pytest.mark.parametrize("name", NAMES)
def test_reads_the_reference_checkpoint(name):
    a = ref_ckpt(name)
    assert int(a["format_version"]) == 1 and int(a["step"]) == 7
    p = P.resolve(json.loads(str(FINAL[f"{name}/params"])))
    assert a["U"].shape == (int(p["nx"]) * int(p["ny"]) * int(p["nz"]), 5 if int(p["nz"]) > 1 else 4)
    assert ("S" in a) == (name == "hancock_2d") and (name != "hancock_2d" or float(a["S"]) > 0)


@pytest.mark.parametrize("name", NAMES)
def test_written_checkpoint_has_the_reference_layout(name, tmp_path):
    a = ref_ckpt(name)
    p = P.resolve(json.loads(str(FINAL[f"{name}/params"])))
    U5 = np.zeros((a["U"].shape[0], 5))
    U5[:, :a["U"].shape[1]] = a["U"]
    mine = ck.checkpoint_arrays(U5, float(a["t"]), int(a["step"]), p, float(a["S"]) if "S" in a else 0.0, body_pose=a.get("body_pose"))
    assert ("body_pose" in a) == (name in MOVING) and (name not in MOVING or a["body_pose"].shape == (MOVING[name],))
    path = str(tmp_path / "mine.npz")
    ck.write_checkpoint(path, mine)
    b = np.load(path)
    assert set(b.files) == set(a)
    for k in a:
        assert b[k].dtype.kind == a[k].dtype.kind and b[k].shape == (a[k].shape if k not in ("collection_time", "collection_file") else b[k].shape), k
        if k not in ("collection_time", "collection_file"):
            assert np.array_equal(b[k], a[k]), k
    with pytest.raises(ValueError, match="newer"):
        bad = dict(mine, format_version=np.array(2, dtype=np.int64))
        ck.write_checkpoint(path, bad)
        ck.read_checkpoint(path)


@pytest.mark.skipif(not os.path.exists(FENICE), reason="the reference is not compiled here (oracle/_ref)")
@pytest.mark.parametrize("name", NAMES)
def test_reference_resumes_from_a_checkpoint_written_here(name):
    """The reference's solver, resumed (resume = true) from a checkpoint written by fenice_b200.checkpoint with its own
    step-7 state, runs 8 steps to its uninterrupted run's step-15 state, bit for bit."""
    a = ref_ckpt(name)
    p = P.resolve(json.loads(str(FINAL[f"{name}/params"])))
    U5 = np.zeros((a["U"].shape[0], 5))
    U5[:, :a["U"].shape[1]] = a["U"]
    tmp = tempfile.mkdtemp(prefix="fvg_ckpt_test_")
    try:
        with open(os.path.join(tmp, "case.toml"), "w") as f:
            f.write(str(FINAL[f"{name}/case_toml"]))
        out = os.path.join(tmp, "out")
        dest = os.path.join(out, str(FINAL[f"{name}/ckpt_relpath"]))
        os.makedirs(os.path.dirname(dest))
        ck.write_checkpoint(dest, ck.checkpoint_arrays(U5, float(a["t"]), int(a["step"]), p, float(a["S"]) if "S" in a else 0.0,
                                                       body_pose=a.get("body_pose")))
        sets = json.loads(str(FINAL[f"{name}/sets"]))   # the case's own --set keys (its mesh, schemes, sides, body)
        cmd = [FENICE, "--case", os.path.join(tmp, "case.toml"), "--no-logo", "--threads", "2"]
        for k, v in sets.items():
            if k not in ("t_end", "save_interval"):
                cmd += ["--set", f"{k}={v}"]
        cmd += ["--set", "t_end=1e9", "--set", "save_interval=1000000000", "--set", "max_steps=8", "--set", f"output_root={out}",
                "--set", "resume=true", "--set", f"dump_state={os.path.join(tmp, 'resumed.npz')}"]
        subprocess.run(cmd, capture_output=True, text=True, check=True)
        d = np.load(os.path.join(tmp, "resumed.npz"))
        assert int(d["step"]) == int(FINAL[f"{name}/step"])
        assert float(d["t"]) == float(FINAL[f"{name}/t"])
        assert np.array_equal(d["U"].view(np.uint64), FINAL[f"{name}/U"].view(np.uint64))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
