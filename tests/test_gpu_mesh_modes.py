"""The interval stage switches from the level-ordered form (one warp per
cell) to group mode (one warp per sibling group over register tapes) once a
level has many cells; the benchmark shapes cross that threshold, the small
test shapes do not.  These tests rerun the mesh parity tests of
test_gpu_mesh.py in a child process whose threshold is lowered through
LFB_GROUP_MODE_CELLS, so that group mode (alone, and after level-ordered
levels) is checked against the oracle on the same shapes."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("cells", [1, 64])
def test_mesh_parity_in_group_mode(gpu, cells):
    env = dict(os.environ, LFB_GROUP_MODE_CELLS=str(cells))
    r = subprocess.run(
        [sys.executable, "-m", "pytest", os.path.join(HERE, "test_gpu_mesh.py"),
         "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"],
        env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
