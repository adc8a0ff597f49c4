"""Whole-region meshes of the benchmark shapes against the CPU oracle
mesher (the reference's DC mesher restated: worker_pool.inl, dc_tree.inl,
dual.hpp, dc_mesher.cpp), at the configured resolution or two octree levels
below it.

* The 64-sphere union (exact operations only) at 64 voxels per unit over
  [-1.5, 1.5]^3 (octree depth 8) and at min_feature 0.1 (depth 5): the
  oracle's exact triangle set.
* The 2000-primitive random CSG of the mesh benchmark (seed 2, 24,908
  clauses, exp / log blends) at depth 8: the oracle meshes with the GPU's
  exp / log results (libm_replay), every other operation being exactly
  rounded on both sides, and must give the GPU's exact triangle set; and
  without the replay, within the bbox-relative Hausdorff bar of 1e-4.
"""
import os

import numpy as np
import pytest

from libfive_b200 import workloads
from libfive_b200.shape import Tape
from libm_replay import with_gpu_libm
from mesh_compare import edge_pairs_ok, hausdorff, oracle_mesh, same_mesh
from oracle_ffi import OracleTape

pytestmark = pytest.mark.gpu

LO, HI = (-1.5, -1.5, -1.5), (1.5, 1.5, 1.5)
THREADS = max(1, os.cpu_count() or 1)


def depth_min_feature(depth):
    """min_feature giving `depth` octree levels over the 3-unit region
    (Region::withResolution, region.hpp:226-231)."""
    return 3.0 / (2 ** depth - 24)


@pytest.mark.parametrize("min_feature", [1.0 / 64, 0.1], ids=["res64", "mf0.1"])
def test_spheres64_full_region(gpu, min_feature):
    s = workloads.spheres_union(64, seed=1)
    v, t, st = Tape(s).render_mesh(LO, HI, min_feature, stats=True)
    assert st.levels == (8 if min_feature < 0.05 else 5)
    ov, ot = oracle_mesh(OracleTape(s), LO, HI, min_feature, threads=THREADS)
    assert len(t) > 0
    assert same_mesh(v, t, ov, ot)
    assert len(v) == len(ov)
    # touching spheres can leave edges shared by four triangles; the GPU
    # mesh pairs its edges exactly where the oracle's does
    assert edge_pairs_ok(t) == edge_pairs_ok(ot)


def test_csg2000_depth8(gpu):
    s = workloads.random_csg(2000, seed=2)
    mf = depth_min_feature(8)
    v, t, st = Tape(s).render_mesh(LO, HI, mf, stats=True)
    assert st.levels == 8
    assert len(t) > 100000
    ora = OracleTape(s)
    ov, ot = oracle_mesh(ora, LO, HI, mf, threads=THREADS)
    assert len(t) == len(ot)
    assert hausdorff(v, t, ov, ot) <= 1e-4 * 3.0
    rv, rt = with_gpu_libm(lambda: oracle_mesh(ora, LO, HI, mf, threads=THREADS))
    assert same_mesh(v, t, rv, rt)
    assert len(v) == len(rv)
