"""Benchmark: dual-contouring meshes per second on a 2000-primitive CSG.

Workload (the single-GPU configuration of the benchmark plan): a random
binary CSG tree of 2000 primitives (spheres, boxes, z-cylinders; centres
U[-1,1]^3, sizes U[0.02,0.2]; unions / smooth blends / differences /
intersections), region [-1.5,1.5]^3 meshed to octree depth 10 (1024^3
cells) with max_err 1e-8.  One step = one complete mesh.  Inputs are
synthetic and seeded (libfive_b200/workloads.py); rank r meshes seed 2 + r.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is meshes/s with the tape resident on
the device (lfb_render_mesh, mesh downloaded to the host each step); `e2e`
builds the device tape from the host tree (flatten + upload) and downloads
the mesh every step.  L2 is flushed (a 512 MiB write) before every timed
step, outside the per-step event pair.
"""
import argparse
import concurrent.futures
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED_BASE = 2
N_PRIMS = 2000
REGION = ((-1.5, -1.5, -1.5), (1.5, 1.5, 1.5))
MIN_FEATURE = 3.0 / 1000.0      # Region::withResolution -> depth 10


def min_feature_for(depth):
    """min_feature giving `depth` levels over the 3-unit region."""
    return 3.0 / (2 ** depth - 24) if depth >= 6 else 3.0 / (2 ** depth - 0.5)
MAX_ERR = 1e-8

# FP32 lane-ops per clause evaluation (value mode / value+gradient mode),
# fixed per opcode; library calls count as 20.
W_VALUE = {"copy": 0, "add": 1, "sub": 1, "neg": 1, "mul": 1, "min": 1, "max": 1,
           "square": 1, "abs": 1, "sqrt": 1, "div": 3, "recip": 3, "exp": 3, "log": 3,
           "const-var": 0}
W_GRAD = {"copy": 0, "add": 4, "sub": 4, "neg": 4, "mul": 7, "min": 5, "max": 5,
          "square": 5, "abs": 5, "sqrt": 7, "div": 11, "recip": 8, "exp": 6, "log": 7,
          "const-var": 0}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true",
                   help="skip the end-to-end pass (profiling runs)")
    p.add_argument("--depth", type=int, default=10,
                   help="octree depth; 10 is the benchmark workload, smaller "
                        "depths are for profiling captures")
    p.add_argument("--workload", default="csg2000",
                   choices=["csg2000", "batch", "eval", "adjoint", "heightmap", "fit",
                            "spheres64", "slice"],
                   help="batch: many trees of mixed size and depth, meshed "
                        "one after another and through lfb_render_meshes")
    p.add_argument("--trees", type=int, default=512, help="batch workload: tree count")
    p.add_argument("--workers", type=int, default=4,
                   help="batch workload: meshes in flight at once")
    p.add_argument("--shapes", type=int, default=64, help="fit workload: shapes")
    p.add_argument("--fit-points", type=int, default=1 << 18,
                   help="fit workload: surface points per shape")
    p.add_argument("--no-remesh", action="store_true",
                   help="fit workload: skip timing the remesh")
    p.add_argument("--points", type=int, default=1 << 22,
                   help="adjoint workload: points (smaller for profiling captures)")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# Process group of an auxiliary workload under torchrun (set by main; None
# on one GPU).  Its only traffic is rank_max.
_AUX_PG = None


def aux_group(world, local):
    """NCCL group for an auxiliary workload when WORLD_SIZE > 1, else None."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return dist


def rank_max(x, pg=None):
    """Max over ranks of a device-timed figure (identity on one GPU); every
    rank calls it at the same points."""
    pg = pg or _AUX_PG
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return t.item()


def rank_seed(rank):
    """Weak scaling: every rank meshes its own seeded shape."""
    return SEED_BASE + rank


def combine_ranks(total_ms, e2e_ms, world, steps, pg, device):
    """Max over ranks of the device-timed totals (one all-reduce; the only
    collective of the run) and the whole-job meshes/s: every rank meshes
    `steps` shapes in the slowest rank's time."""
    import torch
    times = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=device)
    if pg:
        pg.all_reduce(times, op=pg.ReduceOp.MAX)
    total_ms, e2e_ms = times.tolist()
    value = world * steps / (total_ms / 1000.0)
    e2e_value = world * steps / (e2e_ms / 1000.0) if e2e_ms > 0 else None
    return total_ms, e2e_ms, value, e2e_value


def build_shape(seed):
    from libfive_b200 import workloads
    return workloads.random_csg(N_PRIMS, seed=seed)


def tape_weights(shape):
    """Average FP32 lane-ops per clause of the unpruned tape, value / grad."""
    from libfive_b200 import ffi
    from libfive_b200.shape import slot_tape
    lib = ffi.load()
    st = slot_tape(shape)
    names = {}
    for op, _, _, _ in st["clauses"]:
        n = names.setdefault(op, None)
        if n is None:
            for cand in list(W_VALUE) + ["atan2", "pow", "sin", "cos"]:
                if lib.libfive_opcode_enum(cand.encode()) == op:
                    names[op] = cand
                    break
    wv = [W_VALUE.get(names.get(op), 20) for op, _, _, _ in st["clauses"]]
    wg = [W_GRAD.get(names.get(op), 20) for op, _, _, _ in st["clauses"]]
    n = max(1, len(wv))
    return sum(wv) / n, sum(wg) / n, len(st["clauses"])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ffi import OracleTape, load
    return OracleTape, load()


def cpu_mesh_time(shape, cores, stride=1, min_feature=MIN_FEATURE):
    """The oracle (the reference's DC mesher restated, its octree build and
    dual walk run as task pools over all `cores` threads as the reference's
    WorkerPool and Dual walker do) on the whole region.  stride 1: the full
    mesh; returns (seconds, triangles).  stride > 1: only every stride-th of
    the parallel octree tasks (cells five levels below the root) is built;
    returns (estimated seconds of the full mesh: serial top levels + stride
    x the sampled tasks' time, None)."""
    import numpy as np
    OracleTape, lib = _oracle()
    ora = OracleTape(shape)
    ph = np.zeros(3)
    nt = ctypes.c_uint32()
    lo, hi = REGION
    lib.ora_time_mesh(ora.h, *lo, *hi, min_feature, MAX_ERR, cores, stride, ph.ctypes.data,
                      ctypes.byref(nt))
    if stride == 1:
        return float(ph.sum()), int(nt.value)
    return float(ph[0] + stride * ph[1]), None


def mesh_config():
    """The workload's `config`, identical on both arms."""
    return {"workload": "csg2000-depth10-dc", "primitives": N_PRIMS, "seed": SEED_BASE,
            "octree_depth": 10, "region": "[-1.5,1.5]^3", "max_err": MAX_ERR,
            "l2": "flushed (512 MiB write) before every timed step"}


def run_reference(args, world, rank):
    """The reference's CPU mesher (restated: the reference cannot be built
    here) on every host thread, measured on the whole mesh: the K timed steps
    are one complete mesh of the workload (wall time of the full octree
    build, collapse and dual walk), so meshes/s = 1 / that time and each
    step is reported as 1/K of it.  Warm-up steps build a 1/64 sample of the
    octree tasks, untimed."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    shape = build_shape(SEED_BASE)
    for _ in range(args.warmup):
        cpu_mesh_time(shape, cores, stride=64)
    total, tris = cpu_mesh_time(shape, cores)
    value = 1.0 / total
    sample = (f"one whole mesh of the workload ({tris} triangles) on {cores} threads: "
              f"{total:.1f} s, divided evenly over the {args.steps} timed steps")
    print(json.dumps({
        "impl": "reference",
        "metric": "DC meshes/s", "value": value, "unit": "meshes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": mesh_config(),
        "cpu_baseline": {"value": value, "unit": "meshes/s", "cores": cores,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "meshes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def spheres64_summary(lib, cores):
    """The plain configuration's mesh beside the main line: the 64-sphere
    union (seed 1) over [-1.5,1.5]^3 at 64 voxels per unit (depth 8), GPU
    device time per mesh (tape resident, mesh downloaded) and the oracle
    mesher on the whole region on every host core, and whether both give
    the same triangle set."""
    import torch
    from libfive_b200 import workloads
    from libfive_b200.shape import Tape
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from mesh_compare import oracle_mesh, same_mesh
    from oracle_ffi import OracleTape
    shape = workloads.spheres_union(64, seed=1)
    tape = Tape(shape)
    lo, hi = REGION
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    holder = {}

    def once():
        holder["mesh"] = tape.render_mesh(lo, hi, 1.0 / 64, MAX_ERR)

    ms = _timed(once, 10, 3, flush)
    t0 = time.perf_counter()
    ov, ot = oracle_mesh(OracleTape(shape), lo, hi, 1.0 / 64, MAX_ERR, threads=cores)
    dt = time.perf_counter() - t0
    v, t = holder["mesh"]
    return {"gpu_meshes_per_s": 1e3 / ms, "cpu_meshes_per_s": 1.0 / dt, "cores": cores,
            "kind": "port", "triangles": int(len(t)),
            "same_triangles_as_oracle": bool(len(ov) == len(v) and same_mesh(v, t, ov, ot))}


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    from libfive_b200 import ffi
    from libfive_b200.shape import Tape
    lib = ffi.load()
    shape = build_shape(rank_seed(rank))
    tape = Tape(shape)
    wv, wg, n_clauses = tape_weights(shape)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(*REGION)])
    settings = ffi.MeshSettings(MIN_FEATURE if args.depth == 10 else
                                min_feature_for(args.depth), MAX_ERR)

    def mesh_once(t):
        st = ffi.MeshStats()
        m = lib.lfb_render_mesh(t.ptr, region, settings, ctypes.byref(st))
        if not m:
            raise RuntimeError("lfb_render_mesh failed: " + ffi.last_error()[1])
        lib.libfive_mesh_delete(m)
        return st

    for _ in range(args.warmup):
        mesh_once(tape)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = lib.lfb_kernel_launches()
    total_ms, leaf_ms, evals_v, evals_g = 0.0, 0.0, 0, 0
    stats = None
    for _ in range(args.steps):
        flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        stats = mesh_once(tape)
        b.record()
        b.synchronize()
        total_ms += a.elapsed_time(b)
        leaf_ms += stats.ms_leaf
        evals_v += stats.clause_evals
        evals_g += stats.clause_evals_grad
    torch.cuda.synchronize()
    launches = lib.lfb_kernel_launches() - launches0
    if pg:
        pg.barrier()
    clk = clocks.stop()

    # End to end through the public API: flatten + upload the tape, mesh,
    # download and copy into a libfive_mesh, every step.
    e2e_ms, h2d, d2h = 0.0, 0, 0
    for _ in range(0 if args.no_e2e else args.steps):
        flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        t = Tape(shape)
        st = mesh_once(t)
        b.record()
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
        h2d = t.n_clauses * 8 + (t.n_const + t.n_vars) * 4
        d2h = (st.vertices + 1) * 12 + st.triangles * 12
        del t

    total_ms, e2e_ms, value, e2e_value = combine_ranks(total_ms, e2e_ms, world, args.steps,
                                                       pg, "cuda")

    if rank == 0:
        sm_mhz = clk.get("sm_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        peak = sms * 128 * sm_mhz * 1e6 / 1e9          # G lane-ops/s
        ops = (evals_v * wv + evals_g * wg) / args.steps
        achieved = ops / (leaf_ms / args.steps / 1000.0) / 1e9
        # DRAM bytes of one leaf launch, from the committed ncu summary of
        # this workload (dram__bytes_read.sum + dram__bytes_write.sum).
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "k_leaf_groups_csg2000_depth10_dram.md")
        if args.depth == 10 and os.path.exists(tpath):
            for ln in open(tpath):
                if ln.startswith("dram_bytes_per_launch:"):
                    traffic = int(ln.split(":", 1)[1].strip())
        line = {
            "metric": "DC meshes/s", "value": value, "unit": "meshes/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded CSG, seed 2 + rank)",
            "config": mesh_config(),
            "mesh": {"tape_clauses": n_clauses, "octree_depth": stats.levels,
                     "triangles": stats.triangles, "vertices": stats.vertices,
                     "leaf_records": stats.leaves_ambiguous},
            "roofline": {
                "kernel": "leaf stage: k_leaf_groups (corners, edge search; 82 % of the "
                          "stage) + k_leaf_qef + k_edge_rank + k_leaf_vertices",
                "bound": "fp32",
                "achieved": achieved, "peak": peak, "unit": "G lane-ops/s",
                "frac": achieved / peak,
                "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x {sm_mhz:.0f} MHz "
                               "(sampled median SM clock); no measured FP32 figure exists",
                "algorithmic_ops_per_launch": ops,
                "clause_evals_per_launch": (evals_v + evals_g) / args.steps,
                "kernel_ms_per_launch": leaf_ms / args.steps,
                "traffic": traffic,
                "traffic_source": ("ncu capture of the leaf stage's four kernels on this "
                                   "workload, dram__bytes_read.sum + dram__bytes_write.sum "
                                   "(profiles/k_leaf_groups_csg2000_depth10_dram.md), taken "
                                   "before the edge-slot cleanup of k_leaf_groups: an upper "
                                   "bound for the current kernels"
                                   if traffic is not None else None),
            },
            "stages_ms": {"interval": stats.ms_interval, "leaf": stats.ms_leaf,
                          "collapse": stats.ms_collapse, "dual": stats.ms_dual},
            "e2e": {"value": e2e_value, "unit": "meshes/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if not args.no_cpu_baseline and world == 1:
            cores = os.cpu_count() or 1
            est, _ = cpu_mesh_time(shape, cores, stride=8)
            line["cpu_baseline"] = {
                "value": 1.0 / est, "unit": "meshes/s", "cores": cores, "kind": "port",
                "sample": f"1/8 of the whole mesh's parallel octree tasks (every 8th cell "
                          f"five levels below the root) on {cores} threads, scaled x8, plus "
                          f"the serial top levels: {est:.1f} s per mesh estimated"}
            line["spheres64"] = spheres64_summary(lib, cores)
        print(json.dumps(line))
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_batch(args, world, rank, local):
    """Many-tree meshing: `--trees` random CSG trees (primitive counts
    log-uniform in [8, 4000], octree depth 8-11 over [-1.5,1.5]^3), each step
    meshing all of them, timed once as a loop of lfb_render_mesh calls and
    once as one lfb_render_meshes call.  Tapes are built before timing; every
    mesh is downloaded to the host.  Rank r meshes its own trees (seed 11 + r)."""
    import torch
    from libfive_b200 import ffi, workloads
    from libfive_b200.shape import Tape
    torch.cuda.set_device(local)
    lib = ffi.load()
    specs = workloads.batch_specs(args.trees, seed=11 + rank)
    tapes = [Tape(workloads.random_csg(n, seed=sd)) for n, sd, _ in specs]
    jobs = [(t, REGION[0], REGION[1], float(1.0 / res), MAX_ERR)
            for t, (_, _, res) in zip(tapes, specs)]
    region = ffi.Region3(*[ffi.Interval(a, b) for a, b in zip(*REGION)])

    def loop():
        tris = 0
        for t, _, _, mf, me in jobs:
            st = ffi.MeshStats()
            m = lib.lfb_render_mesh(t.ptr, region, ffi.MeshSettings(mf, me), ctypes.byref(st))
            if not m:
                raise RuntimeError("lfb_render_mesh failed: " + ffi.last_error()[1])
            lib.libfive_mesh_delete(m)
            tris += st.triangles
        return tris

    n = len(jobs)
    b_tapes = (ffi.tape_t * n)(*[t.ptr for t, *_ in jobs])
    b_regions = (ffi.Region3 * n)(*[region] * n)
    b_settings = (ffi.MeshSettings * n)(*[ffi.MeshSettings(mf, me) for _, _, _, mf, me in jobs])
    b_stats = (ffi.MeshStats * n)()

    def batch():
        # the same work as loop(): meshes downloaded to the host and freed
        meshes = (ctypes.POINTER(ffi.Mesh) * n)()
        rc = lib.lfb_render_meshes(b_tapes, n, b_regions, b_settings, args.workers, meshes,
                                   b_stats)
        for m in meshes:
            if m:
                lib.libfive_mesh_delete(m)
        if rc != 0:
            raise RuntimeError("lfb_render_meshes failed: " + ffi.last_error()[1])
        inflight[0] = sum(st.ms_total for st in b_stats)
        return sum(st.triangles for st in b_stats)

    inflight = [0.0]
    timings = {}
    for name, fn in (("loop", loop), ("batch", batch)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tris = [fn() for _ in range(args.steps)]
        torch.cuda.synchronize()
        timings[name] = rank_max((time.perf_counter() - t0) / args.steps)
        assert len(set(tris)) == 1

    # The same comparison within each resolution class (one step each,
    # after the warm-up above): small meshes leave the GPU idle between
    # the host's per-level waits, large ones fill it alone.
    by_res = {}
    for res in sorted({r for _, _, r in specs}):
        idx = [i for i, (_, _, r) in enumerate(specs) if r == res]
        sub = [jobs[i] for i in idx]
        m = len(sub)
        s_tapes = (ffi.tape_t * m)(*[t.ptr for t, *_ in sub])
        s_regions = (ffi.Region3 * m)(*[region] * m)
        s_settings = (ffi.MeshSettings * m)(*[ffi.MeshSettings(mf, me) for _, _, _, mf, me in sub])
        s_stats = (ffi.MeshStats * m)()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t, _, _, mf, me in sub:
            mm = lib.lfb_render_mesh(t.ptr, region, ffi.MeshSettings(mf, me), None)
            if not mm:
                raise RuntimeError("lfb_render_mesh failed: " + ffi.last_error()[1])
            lib.libfive_mesh_delete(mm)
        torch.cuda.synchronize()
        t_loop = time.perf_counter() - t0
        meshes = (ctypes.POINTER(ffi.Mesh) * m)()
        t0 = time.perf_counter()
        rc = lib.lfb_render_meshes(s_tapes, m, s_regions, s_settings, args.workers, meshes,
                                   s_stats)
        for mm in meshes:
            if mm:
                lib.libfive_mesh_delete(mm)
        if rc != 0:
            raise RuntimeError("lfb_render_meshes failed: " + ffi.last_error()[1])
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0
        t_loop, t_batch = rank_max(t_loop), rank_max(t_batch)
        by_res[str(res)] = {"trees": m, "ms_loop": t_loop * 1e3, "ms_batch": t_batch * 1e3,
                            "batch_over_loop": t_loop / t_batch}
    if rank == 0:
        n = len(jobs)
        print(json.dumps({
            "metric": "meshes/s (many trees)", "value": world * n / timings["batch"],
            "unit": "meshes/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": timings["batch"] * 1e3, "higher_is_better": True,
            "loop_value": world * n / timings["loop"],
            "batch_over_loop": timings["loop"] / timings["batch"],
            "triangles_per_step": tris[0], "by_resolution": by_res,
            "mean_meshes_in_flight": inflight[0] / (timings["batch"] * 1e3),
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch of %d random CSG trees, 8-4000 primitives, "
                                   "depth 8-11" % n, "workers": args.workers}}))


def _timed(fn, steps, warmup, flush):
    """Device time of `steps` calls of fn (CUDA events on the current stream;
    L2 flushed before each call, outside the events)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    total = 0.0
    for _ in range(steps):
        flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        total += a.elapsed_time(b)
    return total / steps


def run_eval(args, world, rank, local):
    """Point evaluation throughput: the union of 64 spheres (centres
    U[-1,1]^3, radii U[0.1,0.35], seed 1 + rank) on the 128^3 inclusive
    lattice over [-1.5,1.5]^3 (2,097,152 points), values and values +
    derivatives, points resident on the device; e2e passes host arrays."""
    import numpy as np
    import torch
    from libfive_b200 import ffi, workloads
    from libfive_b200.shape import Tape
    torch.cuda.set_device(local)
    shape = workloads.spheres_union(64, seed=1 + rank)
    tape = Tape(shape)
    wv, wg, _ = tape_weights(shape)
    pts = workloads.lattice(128)
    n = len(pts[0])
    x, y, z = (torch.from_numpy(a).cuda() for a in pts)
    f, dx, dy, dz = (torch.empty(n, device="cuda") for _ in range(4))
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    st = lambda: torch.cuda.current_stream().cuda_stream  # noqa: E731
    t_val = _timed(lambda: tape.values(x, y, z, out=f, stream=st()), args.steps, args.warmup, flush)
    t_der = _timed(lambda: tape.derivs(x, y, z, v=f, dx=dx, dy=dy, dz=dz, stream=st()),
                   args.steps, args.warmup, flush)
    hx, hy, hz = (np.ascontiguousarray(a) for a in pts)
    hf = np.empty(n, np.float32)
    t_e2e = _timed(lambda: tape.values(hx, hy, hz, out=hf), args.steps, args.warmup, flush)
    t_val, t_der, t_e2e = rank_max(t_val), rank_max(t_der), rank_max(t_e2e)
    ce = n * tape.n_clauses * world      # clause evaluations of all ranks per step
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle port (ArrayEvaluator / DerivArrayEvaluator restated,
        # 256-point batches) on every host core, over the first 2^18 points
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_ffi import OracleTape
        ora = OracleTape(shape)
        m = 1 << 18
        sub = [np.ascontiguousarray(a[:m]) for a in pts]
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        ora.values(*sub, threads=cores)
        tv = time.perf_counter() - t0
        t0 = time.perf_counter()
        ora.derivs(*sub, threads=cores)
        td = time.perf_counter() - t0
        cpu = {"value": m * tape.n_clauses / tv, "unit": "clause-evals/s", "cores": cores,
               "kind": "port", "sample": "first 2^18 lattice points",
               "deriv_value": m * tape.n_clauses / td}
    sm = torch.cuda.get_device_properties(local).multi_processor_count
    peak = sm * 128 * 1965e6 / 1e9   # G FP32 lane-ops/s at the maximum SM clock
    achieved = ce / world * wv / (t_val / 1e3) / 1e9      # one GPU's kernel
    if rank == 0:
        print(json.dumps({
            "metric": "clause-evals/s", "value": ce / (t_val / 1e3), "unit": "clause-evals/s",
            "compiled": bool(ffi.load().lfb_tape_compiled(tape.ptr)),
            "roofline": {"kernel": "lfb_tape_values" if ffi.load().lfb_tape_compiled(tape.ptr)
                         else "k_values", "bound": "fp32", "achieved": achieved,
                         "peak": peak, "unit": "G lane-ops/s", "frac": achieved / peak,
                         "peak_source": "derived: SMs x 128 FP32 lanes x 1965 MHz",
                         "lane_ops_per_clause": wv},
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_val,
            "higher_is_better": True, "deriv_value": ce / (t_der / 1e3), "ms_deriv": t_der,
            "e2e": {"value": ce / (t_e2e / 1e3), "unit": "clause-evals/s",
                    "h2d_bytes_per_step": 12 * n * world, "d2h_bytes_per_step": 4 * n * world},
            "cpu_baseline": cpu, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64-sphere union, 128^3 lattice", "points": n,
                       "clauses": tape.n_clauses, "l2": "flushed before each step"}}))


def run_adjoint(args, world, rank, local):
    """Gradients of loss = mean f(p)^2 with respect to 1024 free variables
    (256 blended spheres' centres and radii) and the 2^22 points, the points
    sampled area-uniformly from the mesh (64 voxels per unit) of a second
    seed's spheres.
    One step = lfb_eval_loss_grad: the forward pass (f and the checkpoints),
    the seed 2 f / N and the reverse sweep."""
    import numpy as np
    import torch
    from libfive_b200 import workloads
    from libfive_b200.shape import Tape
    torch.cuda.set_device(local)
    # the blend in its overflow-free form: with the stdlib's form, float32
    # exp(-k a) over- or underflows a little off the surface and f and its
    # gradients are inf / NaN at most of the points
    shape, vals = workloads.blended_spheres_vars(256, seed=4 + rank, stable=True)
    tape = Tape(shape, vals)
    target, tvals = workloads.blended_spheres_vars(256, seed=1004 + rank, stable=True)
    v, t = Tape(target, tvals).render_mesh((-1.5,) * 3, (1.5,) * 3, 1.0 / 64)
    tri = v[t.astype(np.int64)].astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
    rng = np.random.Generator(np.random.PCG64(7 + rank))
    n = args.points
    k = rng.choice(len(tri), size=n, p=area / area.sum())
    u, w = rng.random(n), rng.random(n)
    flip = u + w > 1
    u[flip], w[flip] = 1 - u[flip], 1 - w[flip]
    p = tri[k, 0] + u[:, None] * (tri[k, 1] - tri[k, 0]) + w[:, None] * (tri[k, 2] - tri[k, 0])
    x, y, z = (torch.from_numpy(np.ascontiguousarray(p[:, a], np.float32)).cuda() for a in range(3))
    f, seed, gx, gy, gz = (torch.empty(n, device="cuda") for _ in range(5))
    gv = torch.zeros(tape.n_vars, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    loss = torch.zeros(1, device="cuda")

    def step():
        # loss = mean f^2 and its gradients: one forward pass (f and the
        # checkpoints), one backward pass with seed 2 f / n
        s = torch.cuda.current_stream().cuda_stream
        gv.zero_()
        tape.loss_grad(x, y, z, f, gx, gy, gz, gvars=gv, loss=loss, stream=s)

    ms = _timed(step, args.steps, args.warmup, flush)
    ms_fwd = _timed(lambda: tape.values(x, y, z, out=f, stream=torch.cuda.current_stream().cuda_stream),
                    args.steps, args.warmup, flush)
    ms, ms_fwd = rank_max(ms), rank_max(ms_fwd)
    comps = n * (3 + tape.n_vars) * world     # gradient components of all ranks per step
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle port: JacobianEvaluator::gradient (variables) and
        # DerivArrayEvaluator (points) on every host core, first 16 points
        # (each point takes 342 forward passes over the tape for 1024 variables)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_ffi import OracleTape
        ora = OracleTape(shape, vals)
        m = 16
        sub = [np.ascontiguousarray(t_.cpu().numpy()[:m]) for t_ in (x, y, z)]
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        ora.jacobian(*sub, threads=cores)
        ora.derivs(*sub, threads=cores)
        dt = time.perf_counter() - t0
        cpu = {"value": m * (3 + tape.n_vars) / dt, "unit": "gradient components/s",
               "cores": cores, "kind": "port", "sample": "first 16 points"}
    if rank == 0:
        print(json.dumps({
            "metric": "grads/s", "cpu_baseline": cpu, "value": comps / (ms / 1e3), "unit": "gradient components/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "loss_grads_per_s": 1e3 / ms,
            "ms_forward": ms_fwd, "step_over_forward": ms / ms_fwd, "dtype": "f32",
            "roofline": reverse_mode_roofline(shape, n, ms),
            "data": "synthetic",
            "finite_gradients": float(torch.isfinite(gv).float().mean().item()),
            "config": {"workload": "256 blended spheres (overflow-free blend), 1024 free "
                                   "variables, 2^22 surface points",
                       "points": n, "vars": tape.n_vars, "clauses": tape.n_clauses}}))


def hbm_peak():
    """(measured HBM GB/s, source): the copy bandwidth in MEASURED_PEAKS.json
    when present, else the earlier measurement on this kind of GPU."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback: earlier B200 copy measurement"


def reverse_mode_ops_per_point(shape):
    """Algorithmic FP32 lane-ops per point of one loss + gradient step: the
    forward pass (W_VALUE per clause, library calls 20) and the reverse sweep
    (per clause: its local partials, counted as one more W_VALUE, and one
    multiply and one add per operand)."""
    from libfive_b200 import ffi
    from libfive_b200.shape import slot_tape
    lib = ffi.load()
    names = {}
    for cand in list(W_VALUE) + ["atan2", "pow", "sin", "cos"]:
        names[lib.libfive_opcode_enum(cand.encode())] = cand
    ops = 0
    for c in slot_tape(shape)["clauses"]:
        w = W_VALUE.get(names.get(c[0]), 20)
        ops += 2 * w + 2 * lib.libfive_opcode_args(c[0])
    return ops


def reverse_mode_roofline(shape, points, ms, sm_mhz=1965.0):
    """FP32 roofline object of a loss + gradient step over `points` points in
    `ms` (the checkpointed reverse mode recomputes instead of storing, so the
    step is bound by arithmetic, not memory)."""
    import torch
    per_point = reverse_mode_ops_per_point(shape)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = sms * 128 * sm_mhz * 1e6 / 1e9
    achieved = per_point * points / (ms / 1e3) / 1e9
    return {"kernel": "lfb_tape_values + lfb_tape_ckpt_fwd + lfb_tape_ckpt_bwd", "bound": "fp32",
            "achieved": achieved, "peak": peak, "unit": "G lane-ops/s", "frac": achieved / peak,
            "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x {sm_mhz:.0f} MHz",
            "traffic": None, "algorithmic_ops_per_point": per_point}


def run_fit(args, world, rank, local):
    """Batched inverse fitting: `--shapes` (64) shapes, each a CSG of 128
    primitives with 7 free variables each (896; workloads.fit_csg_vars, seed
    21 + 1000 rank + 7 j), fitted to 2^18 points sampled from the surface of
    a copy whose variables are perturbed by N(0, 0.05) (meshed at 128 voxels
    per unit).  One step = one Adam step of every shape (lfb_fit_adam_step:
    reverse-mode gradients of mean f^2, losses, update), points resident on
    the device.  The DC remesh of all shapes at 128 voxels per unit, done
    every 50 steps of the 500-step fit, is timed on its own (one
    lfb_render_meshes call) and folded into the job estimate."""
    import numpy as np
    import torch
    from libfive_b200 import shape as shape_mod
    from libfive_b200 import workloads
    from libfive_b200.fit import BatchedFit
    from libfive_b200.shape import Tape
    torch.cuda.set_device(local)
    n_shapes, n_pts = args.shapes, args.fit_points
    lo, hi = REGION
    t0 = time.perf_counter()
    # seeds 21 + 1000 rank, +7, +14, ...; a seed whose perturbed copy meshes
    # to nothing (a random intersection at the top can leave no solid) is
    # skipped
    shapes, vals, pts, seeds = [], [], [], []
    seed, skipped = 21 + 1000 * rank, 0
    while len(shapes) < n_shapes:
        cand = []
        for _ in range(n_shapes - len(shapes)):
            sh, v, _ = workloads.fit_csg_vars(128, seed=seed)
            cand.append((seed, sh, v, Tape(sh, workloads.perturbed(v, 0.05, seed=seed + 1))))
            seed += 7
        meshes = shape_mod.render_meshes([(c[3], lo, hi, 1.0 / 128) for c in cand], workers=4)
        for (sd, sh, v, _), (mv, mt) in zip(cand, meshes):
            if len(mt) == 0:
                skipped += 1
                continue
            shapes.append(sh)
            vals.append(v)
            seeds.append(sd)
            pts.append(tuple(torch.from_numpy(a).cuda()
                             for a in workloads.surface_points(mv, mt, n_pts, seed=sd + 2)))
        del cand, meshes
    tapes = [Tape(sh, v) for sh, v in zip(shapes, vals)]
    setup_s = time.perf_counter() - t0
    fit = BatchedFit(tapes, pts, lr=1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    first = fit.step().clone()
    torch.cuda.synchronize()
    first_s = time.perf_counter() - t0        # includes compiling the tapes' kernels
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    ms = rank_max(_timed(fit.step, args.steps, args.warmup, flush))
    last = fit.losses.clone()
    torch.cuda.synchronize()
    remesh_s = None
    if not args.no_remesh:
        jobs = [(t, lo, hi, 1.0 / 128) for t in tapes]
        shape_mod.render_meshes(jobs, workers=4)   # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        shape_mod.render_meshes(jobs, workers=4)
        torch.cuda.synchronize()
        remesh_s = rank_max(time.perf_counter() - t0)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle port: JacobianEvaluator::gradient (forward mode, one
        # tape pass per three variables) on every host core, first 16 points
        # of shape 0, extrapolated to one step's gradients of all shapes
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_ffi import OracleTape
        ora = OracleTape(shapes[0], vals[0])
        m = 16
        sub = [np.ascontiguousarray(a.cpu().numpy()[:m]) for a in pts[0]]
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        ora.jacobian(*sub, threads=cores)
        ora.values(*sub, threads=cores)
        dt = time.perf_counter() - t0
        cpu = {"value": m / dt / fit.n_points, "unit": "Adam steps/s", "cores": cores,
               "kind": "port", "sample": "16 points of shape 0 (values + 896-variable "
                                         "gradients), extrapolated to %d points" % fit.n_points}
    n_total = fit.n_points * world
    step_s = ms / 1e3
    job_s = 500 * step_s + (10 * remesh_s if remesh_s is not None else 0.0)
    if rank == 0:
        print(json.dumps({
            "metric": "Adam steps/s (64 shapes x 2^18 points, 896 variables each)",
            "value": 1.0 / step_s, "unit": "Adam steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak",
            "grads_per_s": n_total * tapes[0].n_vars / step_s,
            "ms_remesh_all": remesh_s * 1e3 if remesh_s is not None else None,
            "job_500_steps_s": job_s, "first_step_s": first_s, "setup_s": setup_s,
            "roofline": reverse_mode_roofline(shapes[0], fit.n_points, ms),
            "loss_mean_first": float(first.mean()), "loss_mean_last": float(last.mean()),
            "finite": bool(torch.isfinite(last).all()),
            "cpu_baseline": cpu, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%d CSG shapes x 128 primitives (7 vars each), "
                                   "2^%d surface points each, Adam lr 1e-3"
                                   % (n_shapes, int(round(math.log2(n_pts)))),
                       "clauses": tapes[0].n_clauses, "vars_per_shape": tapes[0].n_vars,
                       "points": fit.n_points, "seeds_skipped_empty": skipped,
                       "l2": "flushed before each step"}}))


def run_spheres_mesh(args, world, rank, local):
    """The plain configuration's meshes: the union of 64 spheres (centres
    U[-1,1]^3, radii U[0.1,0.35], seed 1 + rank) over [-1.5,1.5]^3, meshed
    at 64 voxels per unit (min_feature 1/64: octree depth 8) and at
    min_feature 0.1 (depth 5), max_err 1e-8.  Device time per mesh with the
    tape resident (mesh downloaded to the host), e2e from the host tree
    (flatten + upload + mesh + download), the oracle mesher on the whole
    region on every host core, and whether the two meshes have the same
    triangle set."""
    import torch
    from libfive_b200 import workloads
    from libfive_b200.shape import Tape
    torch.cuda.set_device(local)
    shape = workloads.spheres_union(64, seed=1 + rank)
    tape = Tape(shape)
    lo, hi = REGION
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from mesh_compare import oracle_mesh, same_mesh
    from oracle_ffi import OracleTape
    ora = OracleTape(shape)
    cores = os.cpu_count() or 1
    lines = {}
    for name, mf in (("res64", 1.0 / 64), ("min_feature_0.1", 0.1)):
        holder = {}

        def once(t=None):
            v, tr, st = (t or tape).render_mesh(lo, hi, mf, MAX_ERR, stats=True)
            holder["mesh"], holder["stats"] = (v, tr), st

        ms = _timed(once, args.steps, args.warmup, flush)
        ms_e2e = _timed(lambda: once(Tape(shape)), args.steps, args.warmup, flush)
        ms, ms_e2e = rank_max(ms), rank_max(ms_e2e)
        v, tr = holder["mesh"]
        st = holder["stats"]
        # the leaf kernel's FP32 roofline, as on the main mesh line
        wv, wg, _ = tape_weights(shape)
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        peak = sms * 128 * 1965e6 / 1e9
        leaf_ops = st.clause_evals * wv + st.clause_evals_grad * wg
        achieved = leaf_ops / (st.ms_leaf / 1e3) / 1e9 if st.ms_leaf > 0 else 0.0
        entry = {"ms_per_mesh": ms, "meshes_per_s": world * 1e3 / ms,
                 "e2e_meshes_per_s": world * 1e3 / ms_e2e,
                 "roofline": {"kernel": "k_leaf_groups", "bound": "fp32", "achieved": achieved,
                              "peak": peak, "unit": "G lane-ops/s", "frac": achieved / peak,
                              "peak_source": "derived: SMs x 128 FP32 lanes x 1965 MHz"},
                 "octree_depth": st.levels, "triangles": int(len(tr)),
                 "stages_ms": {"interval": st.ms_interval, "leaf": st.ms_leaf,
                               "collapse": st.ms_collapse, "dual": st.ms_dual}}
        if rank == 0 and not args.no_cpu_baseline:
            t0 = time.perf_counter()
            ov, ot = oracle_mesh(ora, lo, hi, mf, MAX_ERR, threads=cores)
            dt = time.perf_counter() - t0
            entry["cpu_baseline"] = {"value": 1.0 / dt, "unit": "meshes/s", "cores": cores,
                                     "kind": "port", "sample": "the whole mesh"}
            entry["same_triangles_as_oracle"] = bool(len(ov) == len(v) and
                                                     same_mesh(v, tr, ov, ot))
        lines[name] = entry
    if rank == 0:
        main_ = lines["res64"]
        print(json.dumps({
            "metric": "DC meshes/s", "value": main_["meshes_per_s"], "unit": "meshes/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": main_["ms_per_mesh"], "higher_is_better": True, "scaling": "weak",
            "dtype": "f32", "data": "synthetic",
            "e2e": {"value": main_["e2e_meshes_per_s"], "unit": "meshes/s"},
            "cpu_baseline": main_.get("cpu_baseline"), "roofline": main_["roofline"],
            "resolutions": lines,
            "config": {"workload": "64-sphere union, [-1.5,1.5]^3, 64 voxels per unit "
                                   "and min_feature 0.1", "clauses": tape.n_clauses,
                       "max_err": MAX_ERR, "l2": "flushed before each mesh"}}))


def run_heightmap(args, world, rank, local):
    """Height maps: the 64-sphere union (seed 1 + rank) over [-1.5,1.5]^3 at
    512 / 3 voxels per unit (512^3 voxels: a 512 x 512 image with 512 z
    samples), depth and normals, downloaded to the host every step.  The
    CPU line is the oracle's restatement of Heightmap::render on one core
    over the same grid (its work follows the surface, not the voxel count,
    so it is timed at full size)."""
    import numpy as np
    import torch
    from libfive_b200 import workloads
    from libfive_b200.shape import Tape, render_heightmap
    torch.cuda.set_device(local)
    shape = workloads.spheres_union(64, seed=1 + rank)
    tape = Tape(shape)
    lo, hi, res = (-1.5,) * 3, (1.5,) * 3, 512 / 3.0
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    out = {}
    ms = _timed(lambda: out.update(r=render_heightmap(tape, lo, hi, res)), args.steps,
                args.warmup, flush)
    ms = rank_max(ms)
    depth, _ = out["r"]
    voxels = depth.size * 512
    line = {
        "metric": "height-map voxels/s", "value": world * voxels / (ms / 1e3),
        "unit": "voxels/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "filled_pixels": int(np.isfinite(depth).sum()),
        "config": {"workload": "64-sphere union height map, 512^3 voxels",
                   "clauses": tape.n_clauses}}
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_ffi import OracleTape, render_heightmap as oracle_heightmap
        ora = OracleTape(shape)
        t0 = time.perf_counter()
        od, _ = oracle_heightmap(ora, lo, hi, res, workers=1)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": voxels / dt, "unit": "voxels/s", "cores": 1,
                                "kind": "port", "sample": "the same 512^3 grid, once"}
        line["matches_oracle"] = bool(np.array_equal(od, depth))
    if rank == 0:
        print(json.dumps(line))


def run_slice(args, world, rank, local):
    """2D contours: the benchmark's 2000-primitive CSG (seed 2 + rank) cut at
    z = 0 over [-1.5,1.5]^2 with min_feature 3/4096 (a depth-12 quadtree),
    max_err 1e-8, contours downloaded and welded on the host every step.
    The CPU line is the oracle's restatement of Contours::render on one
    core, once, on the same slice; `matches_oracle` compares the contours
    point for point as cyclic sequences."""
    import torch
    from libfive_b200.shape import Tape, render_slice
    torch.cuda.set_device(local)
    shape = build_shape(SEED_BASE + rank)
    tape = Tape(shape)
    lo, hi, z, mf = (-1.5, -1.5), (1.5, 1.5), 0.0, 3.0 / 4096
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    out = {}
    ms = _timed(lambda: out.update(c=render_slice(tape, lo, hi, z, mf, MAX_ERR)), args.steps,
                args.warmup, flush)
    ms = rank_max(ms)
    cs = out["c"]
    pts = int(sum(len(c) for c in cs))
    line = {
        "metric": "slices/s", "value": world * 1e3 / ms, "unit": "slices/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "contours": len(cs), "points": pts,
        "config": {"workload": "2000-primitive CSG slice z = 0, depth-12 quadtree",
                   "clauses": tape.n_clauses}}
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from mesh_compare import same_contours
        from oracle_ffi import OracleTape, render_contours
        t0 = time.perf_counter()
        want, _ = render_contours(OracleTape(shape), lo, hi, z, mf, MAX_ERR)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "slices/s", "cores": 1,
                                "kind": "port", "sample": "the same slice, once"}
        line["matches_oracle"] = bool(same_contours(cs, want))
    if rank == 0:
        print(json.dumps(line))


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    aux = {"batch": run_batch, "eval": run_eval, "adjoint": run_adjoint,
           "heightmap": run_heightmap, "fit": run_fit, "spheres64": run_spheres_mesh,
           "slice": run_slice}
    if args.workload in aux:
        global _AUX_PG
        _AUX_PG = aux_group(world, local)
        try:
            aux[args.workload](args, world, rank, local)
        finally:
            if _AUX_PG is not None:
                _AUX_PG.destroy_process_group()
    elif args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
