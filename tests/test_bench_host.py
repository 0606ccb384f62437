"""bench.py's host-side workload plumbing (no GPU): the timed tool paths repeat
the configured frames, the error-bar paths are the configured start and the
in-contact start with their own seeds, and the training set per workload."""
import numpy as np

import bench
import multigridsoftbody_b200 as mg


def test_timed_paths_repeat_the_configured_frames():
    _, _, _, tool, desc, _ = bench.make_workload("beam", mg)
    a0, b0, r0 = tool(0)
    assert np.allclose(tool(225)[0], a0) and np.allclose(tool(450)[1], b0)   # 225-frame period
    assert 1.4 < float(a0[0, 2]) < 1.6 and float(r0[0]) == np.float32(0.3)
    z = [float(tool(f)[0][0, 2]) for f in range(225)]
    assert z[-1] < -2.8                                                        # down to z = -3 (frame 300)
    assert "frames 75-300" in desc


def test_accuracy_paths_configured_and_in_contact():
    paths = bench.accuracy_paths("beam", 1)
    assert [label for label, _ in paths] == ["config-1 path from z=3", "in contact from z=1.5"]
    z0 = [float(t(0)[0][0, 2]) for _, t in paths]
    assert 2.9 < z0[0] < 3.1 and 1.4 < z0[1] < 1.6
    held = bench.accuracy_paths("beam", 301)
    assert not np.allclose(held[0][1](5)[0], paths[0][1](5)[0])               # another tool seed
    assert len(bench.accuracy_paths("blob", 1)) == 1


def test_train_runs_per_workload():
    assert bench.TRAIN_RUNS["blob"][0] == 32 and bench.TRAIN_RUNS["beam"][0] == 8
