"""The interval stage runs each octree level in one of three forms: one
block per cell (few cells, long tapes), one warp per cell over
level-ordered lists, or group mode (one warp per sibling group over
register tapes, many cells).  The small test shapes only reach the first
form under the default thresholds; these tests rerun the mesh parity tests
of test_gpu_mesh.py in a child process with the thresholds moved through
LFB_GROUP_MODE_CELLS and LFB_BLOCK_MODE_CELLS, so that every form, alone
and after the others, is checked against the oracle on the same shapes."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("group,block", [(1, 0), (64, 0), (1 << 30, 0), (1 << 30, 1 << 30)])
def test_mesh_parity_in_each_interval_mode(gpu, group, block):
    """group: cells from which group mode runs; block: cells up to which the
    block-per-cell kernel runs (else the warp-per-cell one)."""
    env = dict(os.environ, LFB_GROUP_MODE_CELLS=str(group), LFB_BLOCK_MODE_CELLS=str(block))
    r = subprocess.run(
        [sys.executable, "-m", "pytest", os.path.join(HERE, "test_gpu_mesh.py"),
         "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider"],
        env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
