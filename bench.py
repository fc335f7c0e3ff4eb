#!/usr/bin/env python3
"""Benchmark of the CAT-Surface hot path on B200: one hemisphere of Surf2Sphere + SurfWarp.

Step (one hemisphere; ``value``, seconds per hemisphere): CAT_Surf2Sphere of
the 61,442-vertex / 122,880-face folded Fibonacci hull
(``tests/golden/surf2sphere_c2.npz``) -- stages 1-5 (smoothing, inflation,
finger smoothing), the ellipsoid-to-sphere step, 4,999 ordered
area-smoothing sweeps (projection every 1,000) and the final sphere scaling,
all on the GPU -- then CAT_SurfWarp of that surface and sphere to a second,
differently seeded 61,442-vertex hull (``surf2sphere_c3.npz``, with the
upstream binary's sphere): native stencils, type-5 curvature rotation
features, 46-seed + Nelder-Mead rotation search, two runs of two DARTEL steps
on a 256 x 128 sheet in float64 (the reference's default; a float32 DARTEL
exceeds the 1e-3 vertex bound, its error and time are reported beside), the
``-avg`` pole solve and the blend.  Inputs are synthetic and seeded.  The
input surface is resident in HBM when the step starts; the ellipsoid steps
and SurfWarp's mesh inputs use host arrays (the reference computes them on
the host too).  Timed with CUDA events on the launching stream around the
whole step, L2 flushed by a 256 MiB device write before every step, max over
ranks.

``e2e``: the same hemisphere through the public API with files --
``run_cat_surf2sphere_gpu`` (every stage on the GPU) from the surface GIFTI to
the sphere GIFTI, then ``run_cat_surface_gpu_pipeline`` on the four GIFTI
files; two untimed calls, then the mean of three timed ones.

Also on the line: ``batched_rotation`` (8 surfaces of 40,962-163,842 points
x 4,096 uniform quaternions x 2 features in one persistent launch vs one
launch per surface) and ``batched_dartel`` (16 registrations x 2 step maps on
256 x 128 float32 sheets in one graph-captured batched solve vs 16 graphed
one-at-a-time solves).

Multi-GPU runs are independent replicas (a hemisphere is one sequential
Gauss-Seidel chain plus one Nelder-Mead chain); ``value`` is whole-job
seconds per hemisphere.

``--impl reference`` times the reference's CPU algorithm for the path on the
host (the oracle's restatement, the reference's own code being a prebuilt
binary plus the torch CPU path that does not travel): bounded samples of each
stage, scaled to one hemisphere.
"""

from __future__ import annotations

import argparse
from datetime import timedelta
import gc
import json
import os
from pathlib import Path
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"

METRIC = "s/hemisphere Surf2Sphere+SurfWarp @ max vtx err≤1e-3; batched regs/s vs plain"
UNIT = "s/hemisphere"
WORKLOAD = ("Surf2Sphere (stages 1-5 + 4,999 ordered sweeps, 61,442 v / 122,880 f folded hull) + SurfWarp steps=2 runs=2 -avg "
            "to a second 61,442-v hull, 256x128 float64 DARTEL sheet")
SWEEPS = 4999
# dram__bytes_read.sum + dram__bytes_write.sum of areal_dataflow_kernel<CAT, 8> over 200 sweeps of the
# 61,442-vertex hull (9.1 MB + 0.85 MB; ncu summary in profiles/areal_dataflow_61k_hull_200sweeps.md)
SWEEP_DRAM_BYTES = 9.95e6
SHEET = (256, 128)
CHAIN = dict(steps=2, runs=2, avg=True, loop=6, sheet_size=SHEET, rotation_feature_backend="cuda",
             rotation_feature_solver="colored-sor")
# stage counts of one hemisphere, for scaling the CPU samples
DARTEL_STEPS = (CHAIN["runs"] + int(CHAIN["avg"])) * CHAIN["steps"] * CHAIN["loop"] * 3
FEATURE_SIDES = 2 + 2 * (CHAIN["runs"] + int(CHAIN["avg"]))


def parse_args(argv: list[str] | None = None):
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("native", "reference"), default="native")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-batched", action="store_true", help="skip the batched rotation / DARTEL legs")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--profile", action="store_true",
                        help="for profilers: --warmup then --steps hemispheres with the default sweep launch shape, "
                             "no parity, e2e, CPU or batched legs; prints the step times only")
    parser.add_argument("--case", choices=("sweeps", "preprocess", "dartel", "rotation", "rotation-nm", "depth",
                                           "features", "stencil", "warp"),
                        help="for kernel profilers: run one small case of one kernel family three times "
                             "(the third run is the one to capture) and exit")
    return parser.parse_args(argv)


def run_case(name: str) -> int:
    """Small single-kernel cases on cuda:0 for ncu captures (nothing is timed or printed but a summary)."""

    import numpy as np
    import torch

    from cat_surface_gpu_b200 import surf2sphere, synthetic
    from cat_surface_gpu_b200.gifti import GiftiMesh

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    meshes = load_meshes()
    faces = meshes["faces"]
    if name in ("sweeps", "preprocess"):
        topology = surf2sphere.Surf2SphereTopology.from_mesh(GiftiMesh(meshes["surface"], faces))
        plan = topology.plan
        plan_device = plan.to_device(device)
        scratch = None
        if name == "sweeps":
            # 200 of the 4,999 sweeps of the hemisphere mesh: one persistent launch
            base = torch.from_numpy(meshes["prefix"]).to(device)
            for _ in range(3):
                pts = base.clone()
                scratch = surf2sphere.areal_sweeps_device(pts, plan_device, plan, iterations=201, project_every=1000,
                                                          radius=projection_radius(meshes["prefix"]),
                                                          arithmetic="cat", scratch=scratch)
        else:
            # stage 1 of the hemisphere mesh: one persistent launch of 49 passes plus the stage statistics
            from cat_surface_gpu_b200.features import _topology

            rings = _topology(faces, meshes["surface"].shape[0], device)
            faces_device = torch.from_numpy(faces).to(device)
            base = torch.from_numpy(meshes["surface"]).to(device)
            for _ in range(3):
                pts = base.clone()
                scratch = surf2sphere.preprocess_device(pts, faces_device, rings, plan_device, plan, stop_at=1,
                                                        scratch=scratch)
        torch.cuda.synchronize()
        status, where = surf2sphere.read_status(scratch)
        if status != 0:
            raise RuntimeError(f"{name} kernel status {status} at {where}")
    elif name == "dartel":
        # four dartel_steps (k = 0..3, code 1) on two 256 x 128 float64 maps, batched
        from cat_surface_gpu_b200.surface_warp import solve_dartel_maps

        nx, ny = SHEET
        src = torch.as_tensor(np.stack([synthetic.smooth_sheet(ny, nx, 1), synthetic.smooth_sheet(ny, nx, 2)]),
                              device=device)
        tgt = torch.as_tensor(np.stack([synthetic.smooth_sheet(ny, nx, 3), synthetic.smooth_sheet(ny, nx, 4)]),
                              device=device)
        for _ in range(3):
            solve_dartel_maps(src, tgt, loop=4, its=1, device=device, dtype=torch.float64)
        torch.cuda.synchronize()
    elif name in ("depth", "features", "stencil", "warp"):
        # the 61,442-vertex target hemisphere: its stencil (40,962-point resampling sphere, 256 x 128 sheet),
        # one depth feature (heat smoothing at 15 mm, then up to 1,000 SOR sweeps), the two curvature
        # sheets of a DARTEL run (type 5 at 5/9 and 5/27 mm) and the inverse warp of its sphere
        from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere
        from cat_surface_gpu_b200.rotation_feature import compute_rotation_feature
        from cat_surface_gpu_b200.surface_stencil import build_surface_stencil
        from cat_surface_gpu_b200.surface_warp import _surface_sheets, apply_flow_to_stenciled_sphere

        nx, ny = SHEET
        sphere = normalise_sphere(meshes["target_sphere"])
        surface = torch.as_tensor(meshes["target_surface"], device=device)
        st = build_surface_stencil(sphere, meshes["target_faces"], nx=nx, ny=ny, normalize=False,
                                   device=device).to(device)
        flow = torch.as_tensor(0.01 * np.stack([synthetic.smooth_sheet(ny, nx, 1), synthetic.smooth_sheet(ny, nx, 2)]),
                               device=device)
        current = torch.as_tensor(sphere, device=device)
        for _ in range(3):
            if name == "stencil":
                build_surface_stencil(sphere, meshes["target_faces"], nx=nx, ny=ny, normalize=False, device=device)
            elif name == "depth":
                compute_rotation_feature(st, surface, heat_fwhm=15.0)
            elif name == "features":
                _surface_sheets(surface, surface, st, st, (5.0 / 9.0, 5.0 / 27.0), (5, 5), 2, device, torch.float64,
                                False)
            else:
                apply_flow_to_stenciled_sphere(current, flow, st, inverse=True, device=device, dtype=torch.float64)
        torch.cuda.synchronize()
    elif name == "rotation-nm":
        # Nelder-Mead-sized evaluations (csg_rotation_cost_host): 3 candidates of the source hemisphere's
        # 40,962 stencil points against the target's rotation index, five evaluations per run
        from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere
        from cat_surface_gpu_b200.surface_rotation import RotationGridIndexDevice
        from cat_surface_gpu_b200.surface_stencil import build_surface_stencil

        nx, ny = SHEET
        src = build_surface_stencil(normalise_sphere(meshes["binary_sphere"]), meshes["faces"], nx=nx, ny=ny,
                                    normalize=False, device=device)
        tgt = build_surface_stencil(normalise_sphere(meshes["target_sphere"]), meshes["target_faces"], nx=nx,
                                    ny=ny, normalize=False, device=device)
        index = RotationGridIndexDevice.build(tgt.sphere_points, tgt.faces, device=device)
        rng = np.random.default_rng(1)
        inputs = index.prepare_cost_inputs(src.sphere_points.astype(np.float32),
                                           rng.normal(size=src.sphere_points.shape[0]),
                                           rng.normal(size=tgt.sphere_points.shape[0]))
        costing = index._costing(inputs, 64)
        for _ in range(3):
            for _ in range(5):
                costing.evaluate(rng.uniform(-0.3, 0.3, size=(3, 3)), host=True)
        torch.cuda.synchronize()
    else:
        # 256 quaternion candidates on one 102,400-point surface against the resampling sphere
        from cat_surface_gpu_b200.surface_rotation import (RotationGridIndexDevice, batched_costs,
                                                           quaternion_matrices, uniform_quaternions)
        from cat_surface_gpu_b200.surface_stencil import resampling_sphere

        tp, tf = resampling_sphere(6)
        index = RotationGridIndexDevice.build(tp, tf, device=device, grid_size=128, margin=1)
        pts = synthetic.fibonacci_points(102400, np.random.default_rng(1)).astype(np.float32)
        inputs = index.prepare_cost_inputs(pts, np.sin(3 * pts[:, 0]).astype(np.float64),
                                           np.sin(3 * tp[:, 0]))
        mats = quaternion_matrices(uniform_quaternions(256, 2))
        for _ in range(3):
            batched_costs([index], [inputs], matrix_sets=[mats])
        torch.cuda.synchronize()
    print(json.dumps({"case": name, "ok": True}))
    return 0


def dist_env():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def job_seconds_per_unit(local_total_ms: float, units_per_rank: int, world: int, device) -> float:
    """Seconds per unit for the whole job: the slowest rank's timed total (max over ranks)
    divided by the units every rank processed (replicas: each rank runs its own units)."""

    import torch
    import torch.distributed as dist

    total = torch.tensor([float(local_total_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(total, op=dist.ReduceOp.MAX)
    return float(total.item()) / 1e3 / (units_per_rank * world)


def shard_by_cost(costs, world: int, rank: int) -> list[int]:
    """Indices of the units rank ``rank`` of ``world`` processes in a batched leg.

    Units are independent (surfaces, registrations), so a leg shards with no
    exchange step: largest estimated cost first, dealt in snake order
    (ranks 0 .. world-1, then world-1 .. 0, ...) so the ranks' totals stay
    close; each rank's indices in ascending order.
    """

    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    mine = []
    for k, i in enumerate(order):
        slot = k % (2 * world)
        if (slot if slot < world else 2 * world - 1 - slot) == rank:
            mine.append(i)
    return sorted(mine)


def job_throughput(local_units: float, local_ms: float, world: int, device) -> tuple[float, float]:
    """(units of the whole job, the slowest rank's milliseconds): throughput = units / max time."""

    import torch
    import torch.distributed as dist

    units = torch.tensor([float(local_units)], dtype=torch.float64, device=device)
    ms = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    return float(units.item()), float(ms.item())


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi's start-up (driver and NVML initialisation) stalled this process's CUDA
        # calls for hundreds of milliseconds when it overlapped the first timed steps; the timed
        # region starts once the sampler has written its first sample
        deadline = time.perf_counter() + 10.0
        while time.perf_counter() < deadline and self.proc.poll() is None:
            if Path(self.file.name).stat().st_size > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = [line.split(", ") for line in Path(self.file.name).read_text().splitlines() if line.strip()]
        os.unlink(self.file.name)
        sm, sm_max, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in rows:
            try:
                sm.append(float(row[1]))
                sm_max = max(sm_max, float(row[2]))
                for name, flag in zip(names, row[5:9]):
                    if flag.strip() == "Active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": sm_max, "reasons": sorted(reasons), "samples": len(sm)}


def load_meshes():
    import numpy as np

    c2 = np.load(GOLDEN / "surf2sphere_c2.npz")
    c3 = np.load(GOLDEN / "surf2sphere_c3.npz")
    gold = np.load(GOLDEN / "surfwarp_chain_hemisphere_golden.npz")
    return {
        "faces": c2["faces"].astype(np.int32), "surface": c2["surface"], "prefix": c2["prefix"],
        "binary_sphere": c2["final"], "source_area": float(c2["source_area"]),
        "binary_seconds": float(c2["cpu_seconds"]),
        "target_faces": c3["faces"].astype(np.int32), "target_surface": c3["surface"], "target_sphere": c3["final"],
        "chain_final": gold["final_sphere"], "chain_cpu_seconds": float(gold["cpu_seconds"]),
        "chain_final_builder": gold["builder_final_sphere"] if "builder_final_sphere" in gold.files else None,
        "chain_cpu_threads": int(gold["cpu_threads"]),
        "rotation_evaluations": int(gold["rotation_candidates_evaluated"]),
    }


def projection_radius(prefix) -> float:
    import numpy as np

    return float(np.sqrt(np.max(np.sum(prefix.astype(np.float64) ** 2, axis=1))))


def areal_bytes_per_sweep(n: int, f: int) -> int:
    # positions read + written, faces, incident list, offsets (unique elements)
    return n * (12 + 12) + f * 12 + 3 * f * 4 + (n + 1) * 4


def error_stats(reference, candidate) -> dict:
    import numpy as np

    d = np.linalg.norm(np.asarray(candidate, np.float64) - np.asarray(reference, np.float64), axis=1)
    return {"max": float(d.max()), "mean": float(d.mean()), "p99": float(np.quantile(d, 0.99))}


# ---------------------------------------------------------------------------------------------- CPU (oracle) leg


_ROTATION = {}


def _rotation_worker_init(points, faces, values, grid) -> None:
    """Worker set-up of the rotation sample: the target sphere, its features and its grid."""

    _ROTATION.update(points=points, faces=faces, values=values, grid=grid)


def _rotation_worker_cost(angle):
    from oracle import rotation as orot

    r = _ROTATION
    return float(orot.cost_batch(r["points"], r["faces"], r["values"], r["points"].astype("float32"), r["values"],
                                 angle[None, :], grid=r["grid"])[0])


class CpuSampler:
    """Bounded samples of every stage of the oracle port, scaled to one hemisphere.

    Nothing of this package runs here: stages 1-5, the sweeps and the depth
    SOR are the oracle's C restatements, DARTEL, the stencils (``oracle.stencil``),
    the curvature features and the rotation costs its NumPy restatements.  The
    rotation sample -- the reference search's 46 seed costs -- runs on a
    process pool over all host cores, as the reference evaluates its seeds as
    one batch on all threads; every other stage runs on one thread (the
    sweeps and SOR are sequential Gauss-Seidel chains).  ``sample()`` returns,
    per stage, the measured seconds, the fraction of the hemisphere's work the
    sample covers and the seconds scaled to the whole hemisphere.
    """

    SWEEP_SAMPLE = 300
    DARTEL_KS = (0, 3, 5)  # dartel_steps of the smallest, a middle and the largest squaring count
    STENCIL_ROWS = 4096    # of the 40,962 resampling points
    STENCIL_CELLS = 4096   # of the 32,768 sheet cells

    def __init__(self, meshes):
        import multiprocessing

        import numpy as np

        from oracle import features as of, rotation as orot, stencil as ost

        self.meshes = meshes
        self.cores = max(1, os.cpu_count() or 1)
        self.resampling = ost.tetrahedral_sphere(6)
        points, faces = self.resampling
        sphere_points, indices, weights, _ = ost.surface_stencil(meshes["target_sphere"], meshes["target_faces"],
                                                                 points)
        nx, ny = SHEET
        self.stencil = (sphere_points, indices, weights, ost.sheet_stencil(sphere_points, faces, nx, ny))
        rng = np.random.default_rng(7)
        self.rows = np.sort(rng.choice(points.shape[0], self.STENCIL_ROWS, replace=False))
        self.cells = np.sort(rng.choice(nx * ny, self.STENCIL_CELLS, replace=False))
        mapped = of.resample_vertices(meshes["target_surface"], indices, weights)
        values = of.curvature_type5(mapped, faces, 10.0)
        grid = orot.build_grid(sphere_points, faces)
        self.pool = multiprocessing.get_context("spawn").Pool(
            self.cores, initializer=_rotation_worker_init, initargs=(sphere_points, faces, values, grid))
        self.seeds = orot.seed_angles()
        self.pool.map(_rotation_worker_cost, list(self.seeds[:self.cores]))  # import and first-touch in every worker

    def close(self) -> None:
        self.pool.close()
        self.pool.join()

    def sample(self) -> dict:
        import numpy as np

        from oracle import areal as oa, dartel as od, depth as odepth, features as of, preprocess as opre
        from oracle import stencil as ost
        from cat_surface_gpu_b200 import synthetic

        m = self.meshes
        stages = {}

        def timed(name, fraction, fn):
            start = time.perf_counter()
            result = fn()
            seconds = time.perf_counter() - start
            stages[name] = {"measured_s": seconds, "fraction": fraction, "scaled_s": seconds / fraction}
            return result

        timed("stages_1_5", 1.0, lambda: opre.preprocess(m["surface"], m["faces"], 5))
        timed("sweeps", self.SWEEP_SAMPLE / SWEEPS, lambda: oa.areal_sweeps(
            m["prefix"], m["faces"], iterations=self.SWEEP_SAMPLE + 1, project_every=1000,
            radius=projection_radius(m["prefix"])))
        nx, ny = SHEET
        src = synthetic.smooth_sheet(ny, nx, 1).astype(np.float64)
        tgt = synthetic.smooth_sheet(ny, nx, 2).astype(np.float64)

        def dartel():
            vel = np.zeros((2, ny, nx), dtype=np.float64)
            for k in self.DARTEL_KS:
                vel, _ = od.dartel_step(src, tgt, vel, k)

        timed("dartel", len(self.DARTEL_KS) / DARTEL_STEPS, dartel)
        points, faces = self.resampling

        sp, si, sw, sheet = self.stencil
        timed("stencil_surface", len(self.rows) / points.shape[0] / STENCILS, lambda: ost.surface_stencil(
            m["target_sphere"], m["target_faces"], points, rows=self.rows))
        timed("stencil_sheet", len(self.cells) / (nx * ny) / STENCILS,
              lambda: ost.sheet_stencil(sp, faces, nx, ny, cells=self.cells))
        mapped = of.resample_vertices(m["target_surface"], si, sw)
        timed("features", 1.0 / FEATURE_SIDES, lambda: of.curvature_type5_to_sheet_many(
            mapped, faces, (5.0 / 9.0, 5.0 / 27.0), sheet[0], sheet[1]))

        def depth_setup():
            smoothed = of.smooth_geometry(mapped, faces, 10.0)
            return odepth.System(smoothed, faces), odepth.colour_groups(faces, smoothed.shape[0])

        system, groups = timed("depth_setup", 0.5, depth_setup)  # one of the two sides
        timed("depth_sor", DEPTH_SAMPLE_SWEEPS / (2 * DEPTH_SWEEPS), lambda: system.sor(groups, DEPTH_SAMPLE_SWEEPS))
        seeds = list(self.seeds[:min(len(self.seeds), self.cores)])  # one seed cost per process
        timed("rotation", len(seeds) / m["rotation_evaluations"], lambda: self.pool.map(_rotation_worker_cost, seeds))
        total = sum(v["scaled_s"] for v in stages.values())
        measured = sum(v["measured_s"] for v in stages.values())
        return {"total": total, "measured_s": measured, "stages": stages}


DEPTH_SWEEPS, DEPTH_SAMPLE_SWEEPS = 1000, 20
STENCILS = 5 + int(CHAIN["runs"] > 1)
CPU_SAMPLE = ("oracle port, nothing of this package: stages 1-5 in full and 300 of 4,999 sweeps (C, 1 thread); "
              "dartel_steps k = 0, 3, 5 of the 108 per hemisphere (NumPy); 4,096 of the 40,962 surface rows and "
              "4,096 of the 32,768 sheet cells of 1 of the 6 stencils (NumPy restatement of the helper); 1 of 8 "
              "curvature sheet pairs; depth features: one side's set-up of 2, 20 of the 2 x 1,000 SOR sweeps (C); "
              "min(46, cores) of the reference search's 163 rotation costs (NumPy, one per host core); each stage "
              "scaled by the fraction of the hemisphere's work it covers")


def workload_config(meshes) -> dict:
    """The keys that describe the benchmarked workload; both arms report them unchanged."""

    return {"workload": WORKLOAD, "n_vertices": int(meshes["prefix"].shape[0]),
            "n_faces": int(meshes["faces"].shape[0]), "sweeps": SWEEPS, "project_every": 1000,
            "sheet": list(SHEET), "dartel_dtype": "float64",
            "surfwarp": {k: v for k, v in CHAIN.items() if k != "sheet_size"}}


def run_reference(args):
    """The reference arm: the oracle port on the host cores, bounded samples scaled to one hemisphere.

    ``ms_per_step`` is the wall time of one sample as it was measured;
    ``value`` is that sample scaled to a whole hemisphere stage by stage
    (the ``cpu_baseline.stages_s`` breakdown says what was measured and what
    scaled), so the ratio against the native arm is a model ratio.
    """

    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    meshes = load_meshes()
    sampler = CpuSampler(meshes)
    try:
        for _ in range(args.warmup):
            sampler.sample()
        samples = [sampler.sample() for _ in range(args.steps)]
    finally:
        sampler.close()
    value = statistics.mean(s["total"] for s in samples)
    measured = statistics.mean(s["measured_s"] for s in samples)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": measured * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {**workload_config(meshes), "parallelism": f"oracle port; rotation seeds on {sampler.cores} "
                                                             "processes, other stages one thread"},
        "extrapolated": True,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": sampler.cores, "kind": "port", "sample": CPU_SAMPLE,
                         "measured_s_per_step": measured, "stages_s": samples[-1]["stages"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "development_box_timings": {
            "reference_torch_cpu_chain_s": meshes["chain_cpu_seconds"],
            "reference_torch_cpu_chain_threads": meshes["chain_cpu_threads"],
            "reference_binary_surf2sphere_s": meshes["binary_seconds"],
            "note": "timed when the goldens were made, on an 8-vCPU development container, not on this host"},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------------- GPU legs


class Hemisphere:
    """Device-resident inputs of the hemisphere chain and its step."""

    def __init__(self, meshes, device, dartel_dtype, autotune_launch: bool = True):
        import torch

        from cat_surface_gpu_b200 import surf2sphere
        from cat_surface_gpu_b200.features import _topology
        from cat_surface_gpu_b200.gifti import GiftiMesh

        self.meshes, self.device, self.dartel_dtype = meshes, device, dartel_dtype
        faces = meshes["faces"]
        self.topology = surf2sphere.Surf2SphereTopology.from_mesh(GiftiMesh(meshes["surface"], faces))
        self.plan = self.topology.plan
        self.plan_device = self.plan.to_device(device)
        self.faces_device = torch.from_numpy(faces).to(device)
        self.rings = _topology(faces, meshes["surface"].shape[0], device)
        self.pristine = torch.from_numpy(meshes["surface"]).to(device)
        self.points = torch.empty_like(self.pristine)
        self.prefix_copy = torch.empty_like(self.pristine)
        prefix_radius = projection_radius(meshes["prefix"])
        self.launch = surf2sphere.tuned_areal_launch(torch.from_numpy(meshes["prefix"]).to(device), self.plan_device,
                                                     self.plan, arithmetic="cat", radius=prefix_radius) \
            if autotune_launch else surf2sphere.sweep_launch_default(device)
        self.scratch = None
        self.pre_scratch = None
        self.meshes_in = (GiftiMesh(meshes["surface"], faces),
                          GiftiMesh(meshes["target_surface"], meshes["target_faces"]),
                          GiftiMesh(meshes["target_sphere"], meshes["target_faces"]))

    def step(self, dartel_dtype=None):
        import torch

        from cat_surface_gpu_b200 import surf2sphere
        from cat_surface_gpu_b200.gifti import GiftiMesh
        from cat_surface_gpu_b200.gpu_pipeline import register_meshes

        stream = torch.cuda.current_stream()
        events = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        area = self.meshes["source_area"]
        self.points.copy_(self.pristine)
        events[0].record(stream)
        self.pre_scratch = surf2sphere.preprocess_device(self.points, self.faces_device, self.rings, self.plan_device,
                                                         self.plan, stop_at=5, scratch=self.pre_scratch)
        events[1].record(stream)
        surf2sphere.ellipsoid_to_sphere_device(self.points, area)
        self.prefix_copy.copy_(self.points)  # kept for the parity check against the binary's stage-5 output
        radius = surf2sphere.projection_radius_device(self.points)
        events[2].record(stream)
        self.scratch = surf2sphere.areal_sweeps_device(
            self.points, self.plan_device, self.plan, iterations=SWEEPS + 1, project_every=1000, radius=radius,
            arithmetic="cat", launch=self.launch, scratch=self.scratch)
        events[3].record(stream)
        sphere = surf2sphere.ellipsoid_to_sphere_device(self.points, area).cpu().numpy()
        prefix = self.prefix_copy
        surface, target_surface, target_sphere = self.meshes_in
        final, angle, cost, timings = register_meshes(
            surface, GiftiMesh(sphere, self.meshes["faces"]), target_surface, target_sphere, device=self.device,
            dartel_dtype=dartel_dtype or self.dartel_dtype, stencil_threads=min(64, os.cpu_count() or 8), **CHAIN)
        timings["events"] = events
        return final, sphere, prefix, timings

    def check_status(self):
        from cat_surface_gpu_b200 import surf2sphere

        for scratch, what in ((self.pre_scratch, "preprocess"), (self.scratch, "sweep")):
            status, where = surf2sphere.read_status(scratch)
            if status != 0:
                raise RuntimeError(f"{what} kernel status {status} at {where}")


def hemisphere_e2e(meshes, device, dartel_dtype, workdir: Path) -> tuple[float, int, int, dict]:
    """One hemisphere through the public API with host buffers and GIFTI files; returns (s, h2d, d2h, split).

    ``run_cat_surf2sphere_gpu`` (every stage on the GPU) from the surface
    file to the sphere file, then ``run_cat_surface_gpu_pipeline`` on the four
    GIFTI files.
    """

    import torch

    from cat_surface_gpu_b200.gpu_pipeline import run_cat_surface_gpu_pipeline
    from cat_surface_gpu_b200.surf2sphere import run_cat_surf2sphere_gpu

    torch.cuda.synchronize()
    start = time.perf_counter()
    sphere = run_cat_surf2sphere_gpu(workdir / "source_surface.gii", workdir / "source_sphere.gii", stop_at=10,
                                     preprocess_kernel="triton", device=device)
    torch.cuda.synchronize()
    split = time.perf_counter()
    result = run_cat_surface_gpu_pipeline(
        workdir / "source_surface.gii", workdir / "source_sphere.gii", workdir / "target_surface.gii",
        workdir / "target_sphere.gii", workdir / "registered.gii", device=device, dartel_dtype=dartel_dtype,
        stencil_threads=min(64, os.cpu_count() or 8), **CHAIN)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - start
    parts = {"surf2sphere_s": split - start, "surfwarp_s": seconds - (split - start)}
    parts.update({f"surf2sphere.{k}": float(v) for k, v in sphere.timings.items()})
    parts.update({f"surfwarp.{k}": float(v) for k, v in result.timings.items()})
    surface = meshes["surface"]
    # inputs copied to the device: the surface twice (Surf2Sphere, SurfWarp), the sphere, the target mesh
    h2d = 2 * surface.nbytes + sphere.vertices.nbytes + meshes["target_surface"].nbytes + meshes["target_sphere"].nbytes
    h2d += 2 * meshes["faces"].nbytes + meshes["target_faces"].nbytes
    d2h = sphere.vertices.nbytes + result.vertices.nbytes
    return seconds, int(h2d), int(d2h), parts


def batched_rotation_leg(device, world: int = 1, rank: int = 0) -> dict:
    """8 surfaces x 4,096 quaternions x 2 features in one persistent launch.

    Compared with one launch per surface and with one launch per (surface,
    candidate) -- the one-candidate-at-a-time form ("plain"), timed on 32
    candidates per surface and scaled.  Source points are the surfaces'
    unit-sphere vertex directions (the jittered Fibonacci points their folded
    hulls are built on); the cost reads only points and features, not faces.
    """

    import numpy as np
    import torch

    from cat_surface_gpu_b200 import autotune, synthetic
    from cat_surface_gpu_b200.surface_rotation import (RotationGridIndex, batched_costs, quaternion_matrices,
                                                       uniform_quaternions)
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere

    rng = np.random.default_rng(2024)
    all_sizes = sorted(int(v) for v in rng.integers(40962, 163843, size=8))
    mine = shard_by_cost(all_sizes, world, rank)
    sizes = [all_sizes[i] for i in mine]
    tp, tf = resampling_sphere(6)
    index = RotationGridIndex.from_geometry(tp, tf, grid_size=128, margin=1,
                                            include_dense_candidate_table=False).to(device)

    def features(points, seed):
        # curvature proxy (-sum l(l+1) c Y) and depth proxy (max r - r) of a seeded radial fold, z-scored
        r_rng, c_rng = np.random.default_rng(seed), np.random.default_rng(seed)
        fold = synthetic.real_sph_harm_sum(points, range(8, 41), 0.15, r_rng)
        curv = np.zeros(points.shape[0])
        for degree in range(8, 41):
            curv -= degree * (degree + 1) * synthetic.real_sph_harm_sum(points, range(degree, degree + 1), 0.15,
                                                                        c_rng)
        depth = fold.max() - fold
        out = np.stack([curv, depth])
        out = (out - out.mean(axis=1, keepdims=True)) / out.std(axis=1, keepdims=True)
        return out.astype(np.float32).astype(np.float64)

    target_values = features(tp, 7)
    inputs, mats = [], []
    for i, n in zip(mine, sizes):
        pts = synthetic.fibonacci_points(n, np.random.default_rng(100 + i)).astype(np.float32)
        inputs.append(index.prepare_cost_inputs(pts, features(pts.astype(np.float64), 200 + i), target_values))
        mats.append(quaternion_matrices(uniform_quaternions(4096, 300 + i)))
    indices = [index] * len(sizes)
    key = (tuple(sizes), 4096, 2)
    shape = autotune.tune("rotation_cost", key, autotune.rotation_candidates(device),
                          lambda s: batched_costs(indices, inputs, matrix_sets=mats, **s), repeats=1, warmup=1)

    def batched():
        return batched_costs(indices, inputs, matrix_sets=mats, **shape)

    def per_surface():
        return [batched_costs([index], [inp], matrix_sets=[m], **shape)[0] for inp, m in zip(inputs, mats)]

    # one launch per (surface, candidate): how a one-candidate-at-a-time search costs them;
    # timed on the first 32 candidates of every surface and scaled to 4,096
    sample = 32

    def per_candidate():
        return [[batched_costs([index], [inp], matrix_sets=[m[c:c + 1]], **shape)[0] for c in range(sample)]
                for inp, m in zip(inputs, mats)]

    together = batched()
    alone = per_surface()
    single = per_candidate()
    identical = all(torch.equal(a, b) for a, b in zip(together, alone)) and all(
        torch.equal(a[:sample], torch.cat(b)) for a, b in zip(together, single))
    batched_ms = autotune.time_call(batched, repeats=3, warmup=1)
    plain_ms = autotune.time_call(per_surface, repeats=3, warmup=1)
    candidate_ms = autotune.time_call(per_candidate, repeats=2, warmup=1) * 4096 / sample
    evaluations, job_ms = job_throughput(4096 * sum(sizes), batched_ms, world, device)
    # algorithmic bytes per (candidate, point): point 12 + 2 source features 16 + 3 target ids 12
    # + 3 x 2 target features 48 + 36 bytes per scanned candidate triangle (mean CSR width of the grid)
    offsets = index.candidate_offsets.cpu().numpy().astype(np.int64)
    width = np.diff(offsets)
    mean_width = float(width[width > 0].mean())
    bytes_per_eval = 12 + 16 + 12 + 48 + 36 * mean_width
    return {
        "surfaces": all_sizes, "ranks": world, "surfaces_on_rank0": sizes if rank == 0 else None,
        "candidates_per_surface": 4096, "features": 2, "autotuned_shape": shape,
        "batched_ms": batched_ms, "per_surface_ms": plain_ms, "speedup_vs_per_surface": plain_ms / batched_ms,
        "one_candidate_per_launch_ms": candidate_ms, "one_candidate_per_launch_sample": sample,
        "speedup_vs_plain": candidate_ms / batched_ms,
        "point_evaluations_per_s": evaluations / (job_ms / 1e3), "costs_identical_to_plain": bool(identical),
        "kernel_gbs_algorithmic": evaluations * bytes_per_eval / (job_ms / 1e3) / 1e9 / world,
        "bytes_per_evaluation": bytes_per_eval, "mean_cell_width": mean_width,
    }


def batched_dartel_leg(device, repeats: int = 5) -> dict:
    """16 registrations x 2 step maps (256 x 128 float32): one graphed batched solve vs 16 graphed solves."""

    import numpy as np
    import torch

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.surface_stencil import resampling_sphere
    from cat_surface_gpu_b200.surface_warp import apply_flow_to_sphere, solve_dartel_maps, solve_dartel_registrations

    nx, ny = SHEET
    regs, steps = 16, 2
    template = np.stack([synthetic.smooth_sheet(ny, nx, 5000 + s) for s in range(steps)])
    src = np.stack([[synthetic.smooth_sheet(ny, nx, 6000 + 2 * r + s) for s in range(steps)] for r in range(regs)])
    s_dev = torch.as_tensor(src, dtype=torch.float32, device=device)
    t_dev = torch.as_tensor(np.broadcast_to(template, src.shape).copy(), dtype=torch.float32, device=device)
    flows, _ = solve_dartel_registrations(s_dev, t_dev, dtype=torch.float32, cuda_graph=True)  # capture
    plain_flows = [solve_dartel_maps(s_dev[r], t_dev[r], dtype=torch.float32, cuda_graph=True).flow
                   for r in range(regs)]  # capture
    torch.cuda.synchronize()
    batch_lat, plain_lat = [], []
    stream = torch.cuda.current_stream()
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        flows, _ = solve_dartel_registrations(s_dev, t_dev, dtype=torch.float32, cuda_graph=True)
        e1.record(stream)
        e1.synchronize()
        batch_lat.append(e0.elapsed_time(e1))
        events = [torch.cuda.Event(enable_timing=True) for _ in range(regs + 1)]
        events[0].record(stream)
        for r in range(regs):
            plain_flows[r] = solve_dartel_maps(s_dev[r], t_dev[r], dtype=torch.float32, cuda_graph=True).flow
            events[r + 1].record(stream)
        events[-1].synchronize()
        plain_lat.extend(events[r].elapsed_time(events[r + 1]) for r in range(regs))
    unit = torch.from_numpy(np.array(resampling_sphere(5)[0], dtype=np.float32)).to(device)
    errors = [float(torch.linalg.vector_norm(apply_flow_to_sphere(unit, flows[r], device=device)
                                             - apply_flow_to_sphere(unit, plain_flows[r], device=device),
                                             dim=1).max()) for r in range(regs)]
    batch_s = statistics.mean(batch_lat) / 1e3
    plain_s = sum(plain_lat) / repeats / 1e3
    return {
        "registrations": regs, "step_maps": steps, "sheet": [nx, ny], "dtype": "float32", "cuda_graphs": True,
        "batched_regs_per_s": regs / batch_s, "plain_regs_per_s": regs / plain_s,
        "speedup_vs_plain": plain_s / batch_s,
        "batched_latency_ms": {"p50": float(np.percentile(batch_lat, 50)), "p99": float(np.percentile(batch_lat, 99))},
        "plain_latency_ms": {"p50": float(np.percentile(plain_lat, 50)), "p99": float(np.percentile(plain_lat, 99))},
        "max_vertex_error_vs_plain": max(errors),
        "maps": "seeded smooth sheets standing in for the curvature maps of 16 uneven meshes",
    }


def _registration_subject(spec):
    """Worker of the registration leg: one subject mesh and its sphere (spawned process)."""

    from cat_surface_gpu_b200 import synthetic

    return synthetic.folded_hull_and_sphere(*spec)


def batched_registration_leg(device, repeats: int = 3, world: int = 1, rank: int = 0) -> dict:
    """16 subject meshes (folded hulls of 40,962-163,842 vertices) registered to one 61,442-vertex template.

    A registration: the curvature sheets of both surfaces on their stencils,
    one DARTEL run of two steps (256 x 128, float64, graph-captured solve)
    and the inverse warp of the subject's sphere; each subject's stencil is
    built once beforehand (``prep_s``), as a serving system builds it when a
    subject arrives.  Batched: all 16 through one batched solve; plain: one
    registration at a time.  The first two subjects are compared with the
    reference's CPU registration (``registration_golden.npz``).  The
    checkpointed adjoint (k = 7) of the DARTEL data term is timed on the
    registrations' step maps: one batched gradient of all 16 vs one at a time.
    """

    import multiprocessing

    import numpy as np
    import torch

    from cat_surface_gpu_b200 import synthetic
    from cat_surface_gpu_b200.dartel_adjoint import dartel_data_term
    from cat_surface_gpu_b200.gpu_pipeline import normalise_sphere
    from cat_surface_gpu_b200.surface_stencil import build_surface_stencil
    from cat_surface_gpu_b200.surface_warp import (_surface_sheets, apply_flow_to_stenciled_sphere,
                                                   solve_dartel_from_surfaces, solve_dartel_from_surfaces_many)

    all_specs = synthetic.registration_subjects()
    mine = shard_by_cost([n for n, _ in all_specs], world, rank)
    specs = [all_specs[i] for i in mine]
    with multiprocessing.get_context("spawn").Pool(min(len(specs), max(1, os.cpu_count() or 1))) as pool:
        subjects = pool.map(_registration_subject, specs)
    target = np.load(GOLDEN / "surf2sphere_c3.npz")
    nx, ny = SHEET
    steps, loop = 2, 6
    fwhm = tuple(5.0 / (3.0 ** (steps + i)) for i in range(steps))
    tgt_stencil = build_surface_stencil(target["final"], target["faces"], nx=nx, ny=ny, device=device).to(device)
    tgt_surface = torch.as_tensor(target["surface"], device=device)
    start = time.perf_counter()
    prepared = []
    for vertices, faces, sphere in subjects:
        current = normalise_sphere(sphere)
        stencil = build_surface_stencil(current, faces, nx=nx, ny=ny, normalize=False, device=device).to(device)
        prepared.append((torch.as_tensor(vertices, device=device), stencil, torch.as_tensor(current, device=device)))
    torch.cuda.synchronize(device)
    prep_s = time.perf_counter() - start

    def batched():
        flows = solve_dartel_from_surfaces_many([(v, tgt_surface, st, tgt_stencil, fwhm) for v, st, _ in prepared],
                                                curvtypes=(5, 5, 2), n_steps=steps, loop=loop, device=device,
                                                dtype=torch.float64, cuda_graph=True)
        return [apply_flow_to_stenciled_sphere(cur, f, st, inverse=True, device=device, dtype=torch.float64)
                for (_, st, cur), f in zip(prepared, flows)]

    def plain(r):
        v, st, cur = prepared[r]
        flow = solve_dartel_from_surfaces(v, tgt_surface, st, tgt_stencil, fwhm=fwhm, curvtypes=(5, 5, 2),
                                          n_steps=steps, loop=loop, device=device, dtype=torch.float64,
                                          cuda_graph=True).flow
        return apply_flow_to_stenciled_sphere(cur, flow, st, inverse=True, device=device, dtype=torch.float64)

    warped = batched()  # capture the batched graph
    alone = [plain(r) for r in range(len(prepared))]  # capture the single-registration graph
    torch.cuda.synchronize(device)
    stream = torch.cuda.current_stream(device)
    batch_ms, plain_ms = [], []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        warped = batched()
        e1.record(stream)
        e1.synchronize()
        batch_ms.append(e0.elapsed_time(e1))
        events = [torch.cuda.Event(enable_timing=True) for _ in range(len(prepared) + 1)]
        events[0].record(stream)
        for r in range(len(prepared)):
            alone[r] = plain(r)
            events[r + 1].record(stream)
        events[-1].synchronize()
        plain_ms.extend(events[r].elapsed_time(events[r + 1]) for r in range(len(prepared)))
    regs, job_batch_ms = job_throughput(len(prepared), statistics.mean(batch_ms), world, device)
    _, job_plain_ms = job_throughput(0, sum(plain_ms) / repeats, world, device)
    batch_s, plain_s = job_batch_ms / 1e3, job_plain_ms / 1e3
    golden = np.load(GOLDEN / "registration_golden.npz")
    # the golden's two subjects are the two smallest; check the ones this rank registered
    vs_cpu = {f"subject_{k}": error_stats(golden[f"warped_{k}"], warped[mine.index(k)].cpu().numpy())
              for k in range(2) if k in mine}
    vs_plain = max(float(torch.linalg.vector_norm(a - b, dim=1).max()) for a, b in zip(warped, alone))

    # checkpointed adjoint of the data term on the registrations' step maps
    sheets = [_surface_sheets(v, tgt_surface, st, tgt_stencil, fwhm, (5, 5, 2), steps, device, torch.float64, True)
              for v, st, _ in prepared]
    src = torch.cat([a for a, _ in sheets]).contiguous()
    tgt = torch.cat([b for _, b in sheets]).contiguous()
    gen = torch.Generator(device=device).manual_seed(9)
    velocity = (0.3 * torch.randn((src.shape[0], 2, ny, nx), generator=gen, device=device, dtype=torch.float64))

    def gradient(v, s, t):
        v = v.detach().requires_grad_(True)
        dartel_data_term(v, s, t, k=7).sum().backward()
        return v.grad

    for _ in range(2):
        gradient(velocity, src, tgt)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    together = gradient(velocity, src, tgt)
    e1.record(stream)
    e1.synchronize()
    adjoint_batched_ms = e0.elapsed_time(e1)
    e0.record(stream)
    single = [gradient(velocity[i:i + steps], src[i:i + steps], tgt[i:i + steps]) for i in range(0, src.shape[0], steps)]
    e1.record(stream)
    e1.synchronize()
    adjoint_plain_ms = e0.elapsed_time(e1)
    # the adjoint scatters the value part with float64 atomics, so the two agree to rounding, not bit for bit
    apart = torch.cat(single)
    adjoint_rel = float((together - apart).abs().max() / together.abs().max().clamp_min(1e-300))
    return {
        "registrations": int(regs), "ranks": world, "subject_vertices": [n for n, _ in all_specs],
        "template_vertices": int(
            target["surface"].shape[0]), "sheet": [nx, ny], "dtype": "float64", "steps": steps, "loop": loop,
        "cuda_graphs": True, "prep_s": prep_s,
        "batched_regs_per_s": regs / batch_s, "plain_regs_per_s": regs / plain_s,
        "speedup_vs_plain": plain_s / batch_s,
        "batched_latency_ms": {"p50": float(np.percentile(batch_ms, 50)), "p99": float(np.percentile(batch_ms, 99))},
        "plain_latency_ms": {"p50": float(np.percentile(plain_ms, 50)), "p99": float(np.percentile(plain_ms, 99))},
        "vertex_error_vs_cpu_reference": vs_cpu,
        "max_vertex_error_vs_plain": vs_plain,
        "adjoint": {"k": 7, "maps": int(src.shape[0]), "batched_ms": adjoint_batched_ms,
                    "one_registration_at_a_time_ms": adjoint_plain_ms,
                    "batched_gradients_per_s": len(prepared) / (adjoint_batched_ms / 1e3),
                    "plain_gradients_per_s": len(prepared) / (adjoint_plain_ms / 1e3),
                    "max_rel_difference_vs_one_at_a_time": adjoint_rel},
    }


def run_native(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from cat_surface_gpu_b200 import _native, surf2sphere
    from cat_surface_gpu_b200.gifti import GiftiMesh, write_gifti_mesh

    world, rank, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    meshes = load_meshes()
    n, f = meshes["prefix"].shape[0], meshes["faces"].shape[0]
    hemi = Hemisphere(meshes, device, torch.float64, autotune_launch=not args.profile)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        hemi.step()
    barrier()
    hemi.check_status()
    # Python's cyclic collector: a full collection over the ~170k objects of torch and the
    # package pauses 50-100 ms in whichever step it lands; collect once and freeze what exists
    gc.collect()
    gc.freeze()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    step_ms, kernel_ms, pre_ms, stage = [], [], [], []
    final = sphere = prefix = None
    launches_before = _native.kernel_launches()
    if args.profile:  # profilers can restrict a capture to this range (ncu --nvtx --nvtx-include "timed/")
        torch.cuda.nvtx.range_push("timed")
    for index in range(args.steps):
        flush.fill_(index & 0xFF)
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        final, sphere, prefix, timings = hemi.step()
        s1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(s0.elapsed_time(s1))
        ev = timings.pop("events")
        pre_ms.append(ev[0].elapsed_time(ev[1]))
        kernel_ms.append(ev[2].elapsed_time(ev[3]))
        stage.append(timings)
    barrier()
    if args.profile:
        torch.cuda.nvtx.range_pop()
    launches = _native.kernel_launches() - launches_before
    clocks = sampler.stop() if sampler else None
    hemi.check_status()
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "step_ms": step_ms, "sweeps_kernel_ms": kernel_ms,
                              "preprocess_ms": pre_ms, "gpu_launches": launches}))
        if world > 1:
            dist.destroy_process_group()
        return 0
    value = job_seconds_per_unit(sum(step_ms), args.steps, world, device)
    total_s = value * args.steps * world

    # parity (untimed): the chain against the reference's CPU chain (float64 DARTEL, like the timed chain),
    # the sweeps against the upstream binary, and a float32-DARTEL chain against the float64 one
    parity = {"chain_vs_cpu_reference": error_stats(meshes["chain_final"], final),
              # the reference's CPU chain on this package's stencils instead of its helper's float32 ones
              "chain_vs_cpu_reference_same_stencils": (error_stats(meshes["chain_final_builder"], final)
                                                       if meshes["chain_final_builder"] is not None else None),
              "surf2sphere_vs_binary": error_stats(meshes["binary_sphere"], sphere),
              "stages_1_5_vs_binary": error_stats(meshes["prefix"], prefix.cpu().numpy())}
    hemi.step(dartel_dtype=torch.float32)  # warm (graph capture for float32)
    torch.cuda.synchronize()
    f0 = time.perf_counter()
    final32, _, _, timings32 = hemi.step(dartel_dtype=torch.float32)
    torch.cuda.synchronize()
    parity["chain_dartel_f32_vs_f64"] = error_stats(final, final32)
    parity["chain_dartel_f32_seconds"] = time.perf_counter() - f0

    e2e = None
    if not args.no_e2e:
        with tempfile.TemporaryDirectory(prefix="bench_e2e_") as tmp:
            work = Path(tmp)
            write_gifti_mesh(work / "source_surface.gii", GiftiMesh(meshes["surface"], meshes["faces"]))
            write_gifti_mesh(work / "target_surface.gii", GiftiMesh(meshes["target_surface"], meshes["target_faces"]))
            write_gifti_mesh(work / "target_sphere.gii", GiftiMesh(meshes["target_sphere"], meshes["target_faces"]))
            for _ in range(2):  # warm-up: the host paths and the first page-locked allocations
                hemisphere_e2e(meshes, device, torch.float64, work)
            runs = [hemisphere_e2e(meshes, device, torch.float64, work) for _ in range(3)]
        e2e = {"value": job_seconds_per_unit(1e3 * sum(r[0] for r in runs), len(runs), world, device), "unit": UNIT,
               "h2d_bytes_per_step": runs[0][1], "d2h_bytes_per_step": runs[0][2],
               "split_s": {k: sum(r[3].get(k, 0.0) for r in runs) / len(runs) for k in runs[0][3]}}

    batched = {}
    if not args.no_batched:
        batched["batched_rotation"] = batched_rotation_leg(device, world, rank)
        batched["batched_dartel"] = batched_dartel_leg(device)
        batched["batched_registration"] = batched_registration_leg(device, world=world, rank=rank)

    if rank == 0:
        kernel_s = statistics.mean(kernel_ms) / 1e3
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        peak_source = "measured" if "hbm_gbs" in peaks else "fallback"
        achieved = areal_bytes_per_sweep(n, f) * SWEEPS / kernel_s / 1e9
        # one wavefront runs every sweep (the projections ride in it)
        wavefront_steps = (SWEEPS - 1) * hemi.plan.level_stride + hemi.plan.n_levels
        stages = {k: statistics.mean(t[k] for t in stage) for k in stage[0] if isinstance(stage[0][k], float)}
        stages["sweeps_kernel_s"] = kernel_s
        stages["preprocess_kernels_s"] = statistics.mean(pre_ms) / 1e3
        cpu_baseline = None
        if world == 1 and not args.no_cpu_baseline:
            sampler = CpuSampler(meshes)
            try:
                sample = sampler.sample()
            finally:
                sampler.close()
            cpu_baseline = {"value": sample["total"], "unit": UNIT, "cores": sampler.cores, "kind": "port",
                            "sample": CPU_SAMPLE, "measured_s": sample["measured_s"], "extrapolated": True,
                            "stages_s": sample["stages"],
                            "development_box_timings": {
                                "reference_torch_cpu_chain_s": meshes["chain_cpu_seconds"],
                                "reference_torch_cpu_threads": meshes["chain_cpu_threads"],
                                "reference_binary_surf2sphere_s": meshes["binary_seconds"]}}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps,
            "step_ms_each": [round(ms, 3) for ms in step_ms],
            "dartel_s_each": [round(t.get("dartel_total_seconds", 0.0), 4) for t in stage],
            "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {**workload_config(meshes),
                       "levels": hemi.plan.n_levels, "wavefront_stride": hemi.plan.level_stride,
                       "wavefront_steps": wavefront_steps,
                       "sweep_launch": hemi.launch,
                       "l2": "flushed before every timed step by a 256 MiB device write",
                       "python_gc": "collected and frozen after the warm-up (gc.freeze)",
                       "parallelism": f"replicas x{world}"},
            "stages_s": stages,
            "roofline": {
                "kernel": "areal_sweeps (persistent wavefront)", "bound": "hbm", "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "traffic": SWEEP_DRAM_BYTES,
                "traffic_source": "ncu capture of a 200-sweep launch on the same mesh (not scaled: the working set "
                                  "is read once per launch)", "peak_source": peak_source,
                "note": "algorithmic bytes = 4,999 x (24 N + 24 F + 4 (N+1)); the sweep chain is bound by the "
                        "latency of its dependency chain (working set L2-resident); peak = "
                        f"{peak_source} HBM copy bandwidth; traffic = DRAM bytes of one ncu capture of a 200-sweep "
                        "launch on the same mesh: the working set is read once per launch, so a 4,999-sweep "
                        "launch moves the same bytes",
                "kernel_ms": kernel_s * 1e3, "us_per_wavefront_step": kernel_s / wavefront_steps * 1e6,
            },
            "cpu_baseline": cpu_baseline,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
            "parity": parity,
            **batched,
            "published_reference": {"value": 3.7084 + 19.4, "unit": "s",
                                    "what": "reference GPU area smoothing 3.71 s + SurfWarp 19.4 s on RTX 2080 Ti, "
                                            "anatomical LH mesh (docs/BENCHMARKS.md)"},
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.case:
        return run_case(args.case)
    if args.impl == "reference":
        return run_reference(args)
    return run_native(args)


if __name__ == "__main__":
    raise SystemExit(main())
