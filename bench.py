"""Benchmark: JointRecon outer iterations per second on the 256x224x176, 32-coil, 64-shot
DISORDER workload (16x16 tiles, accel 2, random-walk + jump motion, 8 CG iterations and one LM
step per outer iteration), on motionest's sm_100a kernels.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl motionest|reference]
                  [--workload large|medium|slab|small] [--batch B] [--jacobian reference|exact]
                  [--no-e2e] [--no-cpu] [--no-plain] [--noise S] [--pyramid] [--sharded]
                  [--replicas] [--no-graph] [--multi] [--dft] [--dft-only]

One "step" = one JointRecon outer iteration exactly as joint_recon.py:93-102 runs it: CG image
step (max_cg_iter=8), one LM motion step, x *= M, and the objective.  Inputs are synthetic and
seeded (no dataset exists for this path).  Every volume is larger than L2 (coil maps alone are
2.6 GB), so no L2 flush is needed between steps.

--impl reference times the reference algorithm on the host CPU: the oracle port (a NumPy/SciPy
restatement of the reference, pinned to its outputs) with all host threads.  Each step is a
bounded sample of the same workload (one shot's transform, adjoint, derivative and 32-coil 3-D
FFT pairs), extrapolated to one outer iteration by the reference's own operation counts; the
line also carries that model checked against whole outer iterations timed end to end on the
64x64x48 / 8-coil / 16-shot workload (all threads and one thread).

The line also carries "plain": the same reconstruction with one shot per launch (the
reference's per-shot loop on the same kernels) and the reference's order of operations for
each CG solve's initial residual (right-hand side and A x formed separately; the fast form
takes b - A x from one pass, left by the previous objective) over the same iterations, its
iterations per second, fast/plain, and how far its image and transforms are from the batched
run's.

With --gpus N > 1 (torchrun) the ranks run one reconstruction split by shots
(motionest.sharded: one all-reduce of the image per normal operator), "scaling": "strong", and
value = that reconstruction's iterations / max rank time.  With --replicas every rank instead
runs an independent replica of the workload (no collective on the data path), "scaling":
"weak", and value = total iterations / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (shape, coils, shots, tile, accel, ellipsoids, cg iters)
    "large": ((256, 224, 176), 32, 64, (16, 16), 2, 40, 8),
    "medium": ((128, 112, 88), 16, 32, (8, 8), 2, 20, 8),
    # the large workload's planes (same samples per shot, coils, shots) on 32 readout points:
    # small enough for full ncu captures, same per-plane kernel behaviour
    "slab": ((256, 224, 32), 32, 64, (16, 16), 2, 40, 8),
    "small": ((64, 64, 48), 8, 16, (4, 4), 1, 10, 5),
    # the precision workload's size: 256x256x192 (line lengths 256 / 256 / 192)
    "precision": ((256, 256, 192), 32, 64, (16, 16), 2, 40, 8),
}
METRIC = "JointRecon iter/s (CG+LM, 64 shots, 32 coils)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="motionest", choices=["motionest", "reference"])
    ap.add_argument("--workload", default="large", choices=list(WORKLOADS))
    ap.add_argument("--batch", type=int, default=0, help="shots per launch (0 = all)")
    ap.add_argument("--jacobian", default="reference", choices=["reference", "exact"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1 ranks, one independent reconstruction per rank (weak "
                         "scaling); default: one reconstruction split by shots over the ranks")
    ap.add_argument("--sharded", action="store_true",
                    help="one reconstruction split by shots over the ranks (the default for "
                         "N > 1); on one GPU, runs it through the one-rank communicator")
    ap.add_argument("--multi", action="store_true",
                    help="also time 12 reconstructions of uneven size (64^3, 96x96x72, "
                         "128x128x96, 192x192x144, 3 each; coils, shots and tiles from a seed; "
                         "continuous intra-shot motion) one at a time and all together "
                         "(motionest.multi.MultiRecon)")
    ap.add_argument("--dft", action="store_true",
                    help="also time the split-precision tensor-core row DFT against the "
                         "register FFT on 2^20 rows of 224 and of 256 points")
    ap.add_argument("--dft-only", action="store_true",
                    help="only the DFT comparison of --dft (one JSON object), no reconstruction")
    ap.add_argument("--no-graph", action="store_true",
                    help="run the CG solves of the timed reconstruction as a host loop instead "
                         "of CUDA graphs (the plain arm always uses the host loop)")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain (one shot per launch) comparison run")
    ap.add_argument("--noise", type=float, default=1e-3,
                    help="noise std per real component, relative to max|k| (default 1e-3)")
    ap.add_argument("--plain-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--pyramid", action="store_true",
                    help="also time pyramid_reconstruction end to end (3 levels, 20 base "
                         "iterations: 80 at x0.25, 40 at x0.5, then 100 CG iterations at x1)")
    return ap.parse_args()


def config_dict(name, extra=None):
    shape, C, S, tile, accel, nell, cg = WORKLOADS[name]
    d = {"workload": f"DISORDER JointRecon {shape[0]}x{shape[1]}x{shape[2]}, {C} coils, {S} shots, "
                     f"tiles {tile[0]}x{tile[1]}, accel {accel}, {cg} CG + 1 LM per iteration",
         "shape": list(shape), "coils": C, "shots": S, "tile": list(tile), "accel": accel,
         "cg_iters": cg, "lm_steps": 1, "ellipsoids": nell, "noise_rel_sigma": None,
         "l2": "no flush: every input exceeds L2 (maps 2.6 GB)"}
    if extra:
        d.update(extra)
    return d


# ------------------------------------------------------------------------------ CPU arm
def iteration_model(t, S, k, cg_applications=None):
    """Seconds of one outer iteration by the reference's operation counts
    (image_estimation.py:93-163, transform_estimation.py:39-135, joint_recon.py:108-115), from the
    per-shot unit times t: T, TH, dT, and F / Fi (one 3-D FFT pair over all coils).  The CG step
    applies the normal operator k + 1 times (A x, then k iterations) unless it stops early, in
    which case `cg_applications` gives the count."""
    normal = t["T"] + t["F"] + t["Fi"] + t["TH"]
    napp = (k + 1) if cg_applications is None else cg_applications
    return (S * (t["Fi"] + t["TH"])                                  # b
            + napp * S * normal                                      # A applications
            + S * (2 * (t["T"] + t["F"]) + 6 * (t["dT"] + t["F"]))   # LM
            + S * (t["T"] + t["F"]))                                 # objective


class UnitSample:
    """The reference's per-shot unit operations on the oracle port at `shape` with C coils: the
    inputs are made once, and run() times one shot's T, T^H and dT and the coil 3-D FFT pair."""

    def __init__(self, shape, C, threads, seed=0):
        from oracle import Oracle, transform_grids
        self.O = Oracle(np.complex64, workers=threads)
        rng = np.random.default_rng(seed)
        self.x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
        self.p = np.array([0.5, -0.3, 0.2, 0.02, -0.03, 0.04])
        self.kg, self.rk = transform_grids(shape, [1, 1, 1])
        self.coil = (rng.standard_normal((C,) + shape).astype(np.float32)
                     + 1j * rng.standard_normal((C,) + shape).astype(np.float32)).astype(np.complex64)

    def run(self):
        O, x, p, kg, rk, coil = self.O, self.x, self.p, self.kg, self.rk, self.coil
        t = {}
        for name, fn in (("T", lambda: O.rigid_apply(x, p, kg, rk)),
                         ("TH", lambda: O.rigid_adjoint(x, p, kg, rk)),
                         ("dT", lambda: O.rigid_derivative(x, p, 4, kg, rk)),
                         ("F", lambda: O.fft(coil, (-3, -2, -1))),
                         ("Fi", lambda: O.ifft(coil, (-3, -2, -1)))):
            t0 = time.perf_counter()
            fn()
            t[name] = time.perf_counter() - t0
        return t


def unit_times(shape, C, threads, seed=0):
    return UnitSample(shape, C, threads, seed).run()


def cpu_reference_sample(name, threads, sample=None):
    """Time the reference algorithm's unit operations at full size on the host CPU (the oracle
    port, scipy.fft with `threads` workers) and extrapolate one outer iteration.  Returns
    (iterations per second, seconds the timed operations took, unit times)."""
    shape, C, S, tile, accel, nell, k = WORKLOADS[name]
    sample = sample or UnitSample(shape, C, threads)
    t = sample.run()
    return 1.0 / iteration_model(t, S, k), sum(t.values()), t


def config0_check(threads):
    """The extrapolation model checked on the 64x64x48 / 8-coil / 16-shot workload, where a
    whole outer iteration of the port is cheap enough to run: the second outer iteration of the
    oracle's JointRecon on the fixture inputs (tests/golden/config0.npz), timed end to end,
    against the model built from unit times at that size with the CG count that iteration
    actually ran."""
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import config_inputs as ci
    from oracle import Oracle, transform_grids
    ksp, mps, masks, _ = ci.load(ROOT / "tests" / "golden")
    kg, rk = transform_grids(ci.SHAPE, [1, 1, 1])
    O = Oracle(np.complex64, workers=threads)
    k_u, m_u, mask_u, max_norm, P, M = O.joint_setup(ksp, mps, masks)
    S = ci.NSHOTS
    x = np.zeros(ci.SHAPE, np.complex64)
    t = np.zeros((S, 6))
    damp, flags = np.ones(S), np.zeros(S, bool)
    secs, apps = [], []
    for _ in range(2):
        t0 = time.perf_counter()
        x, iters = O.estimate_image_cg(k_u, m_u, mask_u, t, kg, rk, P, M, x0=x,
                                       max_iter=ci.CG_ITERS, return_iters=True)
        x = O.estimate_transform(k_u, m_u, mask_u, x, kg, rk, damp, flags, t) * M
        O.objective(k_u, m_u, mask_u, x, t, kg, rk)
        secs.append(time.perf_counter() - t0)
        apps.append(iters + 1)
    model = iteration_model(unit_times(ci.SHAPE, ci.NCOILS, threads), S, ci.CG_ITERS, apps[-1])
    return {"workload": "64x64x48, 8 coils, 16 shots, DISORDER 4x4, 5 CG + 1 LM",
            "threads": threads, "measured_s_per_iter": secs[-1], "modelled_s_per_iter": model,
            "model_over_measured": model / secs[-1], "cg_applications": apps[-1]}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    shape, C = WORKLOADS[args.workload][:2]
    sample = UnitSample(shape, C, threads)  # inputs made once, outside the timed steps
    steps = []
    for _ in range(args.warmup + args.steps):
        steps.append(cpu_reference_sample(args.workload, threads, sample))
    timed = steps[args.warmup:]
    v = float(np.median([s[0] for s in timed]))
    sample_ms = 1000.0 * float(np.median([s[1] for s in timed]))
    # the extrapolation validated where a whole iteration can be timed, with all threads and
    # with one (scipy.fft's default, as the reference calls it)
    check = [config0_check(threads), config0_check(1)]
    sample.O.workers = 1
    w1 = cpu_reference_sample(args.workload, 1, sample)[0]
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample_ms,
        "step": "one bounded sample: the reference's per-shot unit operations (T, T^H, dT, and "
                "the coil 3-D FFT pair) timed at full size; value extrapolates one outer "
                "iteration from them by the reference's operation counts",
        "extrapolated_ms_per_iteration": 1000.0 / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic", "config": config_dict(args.workload),
        "cpu_baseline": {"value": v, "unit": "iter/s", "cores": threads, "kind": "port",
                         "sample": "oracle port of the reference on the host CPU (scipy.fft, "
                                   f"{threads} workers): one shot's T, T^H, dT and the "
                                   "coil 3-D FFT pair at full size, extrapolated to one outer "
                                   f"iteration; {sample_ms / 1000.0:.1f} s of CPU work per step",
                         "value_workers_1": w1},
        "model_check": check,
        "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------------------ GPU arm
MULTI_SHAPES = [(64, 64, 64), (96, 96, 72), (128, 128, 96), (192, 192, 144)]


def multi_problems(seed=11):
    """The 12-instance mix: 3 of each shape, coils in 8..32, shots in 16..128 (at most 2048
    samples per shot and plane), DISORDER tiles 4x4..16x16 dividing the plane, accel 1,
    continuous intra-shot motion (4 segments per shot, drift up to 2 deg / 2 voxels)."""
    from motionest.simulation import make_workload
    from motionest.utils import compute_transform_grids_voxel
    rng = np.random.default_rng(seed)
    out = []
    for k, shape in enumerate(MULTI_SHAPES * 3):
        X, Y, _ = shape
        C = int(rng.choice([8, 16, 32]))
        shots = [s for s in (16, 32, 64, 128) if X * Y // s <= 2048]
        S = int(rng.choice(shots))
        tile = int(rng.choice([t for t in (4, 8, 16) if X % t == 0 and Y % t == 0]))
        wl = make_workload(shape, C, S, (tile, tile), 1, motion="continuous", n_ellipsoids=10,
                           seed=100 + k)
        kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
        out.append(dict(ksp=wl["ksp"], mps=wl["mps"], masks=wl["masks"], kgrid=kg, rkgrid=rk,
                        desc=f"{X}x{Y}x{shape[2]}/{C}c/{S}s/{tile}x{tile}"))
    return out


def time_multi(iters=2, cg=8):
    """Outer iterations of the 12 instances one reconstruction at a time (each JointRecon with
    graph CG, shots per launch from the autotuner) against MultiRecon advancing all 12
    together; both timed with CUDA events after one warm-up iteration."""
    import torch
    from motionest.joint_recon import JointRecon
    from motionest.multi import MultiRecon
    probs = multi_problems()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seq_ms = 0.0
    for p in probs:
        app = JointRecon(p["ksp"], p["mps"], p["masks"], p["kgrid"], p["rkgrid"], max_cg_iter=cg,
                         cg_graph=True, batch="auto")
        app.step()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(iters):
            app.step()
            app._compute_objective()
        e1.record()
        torch.cuda.synchronize()
        seq_ms += e0.elapsed_time(e1)
        app._graph.close()
        del app
    # the rigid transform of every instance's shots: one me_rigid_apply per instance against one
    # me_rigid_apply_multi over all 12 (each step one persistent launch per line length)
    from motionest import _lib
    from motionest.multi import apply_transforms
    from motionest.utils import DeviceGrid
    jobs = []
    for p in probs:
        X, Y, Z = p["ksp"].shape[1:]
        S = p["masks"].shape[0]
        jobs.append(dict(x=torch.randn((Z, X, Y), dtype=torch.complex64, device="cuda"),
                         out=torch.empty((S, Z, X, Y), dtype=torch.complex64, device="cuda"),
                         params=torch.as_tensor(np.random.default_rng(S).uniform(-0.05, 0.05,
                                                                                 (S, 6))).cuda(),
                         grid=DeviceGrid(p["kgrid"], p["rkgrid"], (X, Y, Z))))

    def one_by_one():
        for jb in jobs:
            Z, X, Y = jb["x"].shape
            _lib.call("me_rigid_apply", _lib.ptr(jb["x"]), 0, _lib.ptr(jb["out"]), X * Y * Z,
                      jb["out"].shape[0], _lib.MeLayout(Y, 1, X * Y), jb["grid"].ref,
                      _lib.ptr(jb["params"]), 6, 0, _lib.stream_ptr())

    t_apply = {}
    for name, fn in (("one_at_a_time_ms", one_by_one),
                     ("multi_ms", lambda: apply_transforms(jobs))):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        t_apply[name] = e0.elapsed_time(e1) / 3
    del jobs
    mr = MultiRecon(probs, max_cg_iter=cg)
    mr.step()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(iters):
        mr.step()
    e1.record()
    torch.cuda.synchronize()
    par_ms = e0.elapsed_time(e1)
    mr.close()
    return {"instances": [p["desc"] for p in probs], "outer_iterations": iters,
            "cg_iters": cg, "one_at_a_time_s": seq_ms / 1000.0, "together_s": par_ms / 1000.0,
            "speedup": seq_ms / par_ms, "transform_apply": t_apply,
            "note": "12 reconstructions x outer iterations; one at a time = the sum of each "
                    "instance's own timed iterations; together = MultiRecon, every instance on "
                    "its own stream, CG solves as CUDA graphs"}


def time_dft(rows=1 << 20, reps=5):
    """Orthonormal forward DFTs of `rows` contiguous complex64 rows: the register FFT
    (me_fft_axis) against the split-precision TF32 tensor-core DFT (me_dft_rows_split), CUDA
    events over `reps` launches each after a warm-up, inputs and outputs (2 GB each) above L2;
    relative L2 error of each against FP64 on 512 sampled rows."""
    import torch
    from motionest import _lib
    st = _lib.stream_ptr()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {}
    for n in (224, 256):
        x = torch.randn(rows, n, dtype=torch.complex64, device="cuda")
        y = torch.empty_like(x)
        lay = _lib.MeLayout(n, 1, 1)
        runs = {"register_fft": lambda: _lib.call("me_fft_axis", _lib.ptr(x), 0, _lib.ptr(y), 0, 1,
                                                  rows, n, 1, lay, 1, 0, st),
                "split_tf32_mma": lambda: _lib.call("me_dft_rows_split", _lib.ptr(x), _lib.ptr(y),
                                                    rows, n, 0, st)}
        sel = np.random.default_rng(n).choice(rows, 512, replace=False)
        ref = np.fft.fft(x[sel].cpu().numpy().astype(np.complex128), axis=1, norm="ortho")
        res = {}
        for name, fn in runs.items():
            fn()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            got = y[sel].cpu().numpy()
            err = float(np.max(np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)))
            res[name] = {"ms": ms, "gbs": rows * n * 16 / ms / 1e6, "max_rel_err_vs_fp64": err}
        res["split_over_register_time"] = res["split_tf32_mma"]["ms"] / res["register_fft"]["ms"]
        out[str(n)] = res
        del x, y
    return out


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1].split()[0]), float(parts[2].split()[0]), parts[4:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, flags in rows:
            for n, f in zip(names, flags[1:]):
                if f.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1],
                "reasons": sorted(reasons), "samples": len(rows)}


def rank_max(x, device):
    """Max of x over the ranks of the default process group (x itself when there is none or
    it has one rank): the job's time is its slowest rank's.  Every rank must call it."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, max_ms):
    """Outer iterations per second of the whole job: every rank ran `steps` iterations of its
    own replica, and the job took the slowest rank's max_ms milliseconds."""
    return world * steps / (max_ms / 1000.0)


# The kernel variants that make the plain form: cp.async staging instead of TMA tensor and bulk
# copies, and the LM statistics through seven written K regions and a second kernel.  The
# library reads them once per process, so that arm runs in a child process.
PLAIN_ENV = {"ME_NO_TMA": "1", "ME_NO_BULK": "1", "ME_LM_TWO_PASS": "1"}


def plain_child(args):
    """The plain form of the timed reconstruction, in this (child) process: one shot per launch,
    host-loop CG and the kernel variants of PLAIN_ENV, on the same seeded data; its last
    `steps` iterations timed with CUDA events.  Writes the time, image and transforms to
    args.plain_child (an .npz file)."""
    import torch
    from motionest.joint_recon import JointRecon
    from motionest.simulation import make_workload
    from motionest.utils import compute_transform_grids_voxel
    shape, C, S, tile, accel, nell, k = WORKLOADS[args.workload]
    wl = make_workload(shape, C, S, tile, accel, motion="walk", n_ellipsoids=nell, seed=1,
                       noise=args.noise)
    kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
    app = JointRecon(wl["ksp"], wl["mps"], wl["masks"], kg, rk, max_cg_iter=k, max_nm_iter=1,
                     max_joint_iter=args.steps, jacobian=args.jacobian, batch=1,
                     fused_residual=False)
    for _ in range(args.warmup):
        app.step()
        app._compute_objective()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    objs = []
    for _ in range(args.steps):
        app.step()
        objs.append(app._compute_objective())
    e1.record()
    torch.cuda.synchronize()
    np.savez(args.plain_child, ms=e0.elapsed_time(e1), x=app.x.cpu().numpy(),
             t=app.t.cpu().numpy(), objs=np.array(objs))


def run_plain_child(args):
    """Run plain_child in a child process with the plain kernel variants; returns its npz."""
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    cmd = [sys.executable, str(Path(__file__).resolve()), "--workload", args.workload,
           "--steps", str(args.steps), "--warmup", str(args.warmup), "--jacobian", args.jacobian,
           "--noise", repr(args.noise), "--plain-child", path]
    env = dict(os.environ, **PLAIN_ENV)
    env.pop("WORLD_SIZE", None)
    try:
        subprocess.run(cmd, env=env, check=True, stdout=subprocess.DEVNULL, timeout=1800)
        with np.load(path) as z:
            return {key: z[key] for key in z.files}
    finally:
        os.unlink(path)


def main():
    args = parse()
    if args.plain_child:
        plain_child(args)
        return
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and not args.replicas:
        args.sharded = True
    # the sharded reconstruction's CG exchanges through the host-side communicator: no graph
    args.graph = not args.no_graph and not args.sharded
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    if args.dft_only:
        print(json.dumps({"dft": time_dft()}), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from motionest import _lib
    from motionest.joint_recon import JointRecon
    from motionest.simulation import make_workload
    from motionest.utils import compute_transform_grids_voxel

    shape, C, S, tile, accel, nell, k = WORKLOADS[args.workload]
    # replicas reconstruct their own data; the ranks of a sharded reconstruction share it
    wl = make_workload(shape, C, S, tile, accel, motion="walk", n_ellipsoids=nell,
                       seed=1 if args.sharded else 1 + rank, noise=args.noise)
    kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
    batch = args.batch or None
    Recon = JointRecon
    jobs = world  # reconstructions the job runs at once
    if args.sharded:
        from motionest.sharded import ShardedJointRecon, SoloComm, TorchComm
        comm = TorchComm() if world > 1 else SoloComm()

        def Recon(*a, **kw):
            return ShardedJointRecon(*a, comm=comm, **kw)
        jobs = 1
    app = Recon(wl["ksp"], wl["mps"], wl["masks"], kg, rk, max_cg_iter=k, max_nm_iter=1,
                max_joint_iter=args.steps, jacobian=args.jacobian, batch=batch,
                **({"cg_graph": True} if args.graph else {}))

    def step():
        app.step()
        return app._compute_objective()

    for _ in range(args.warmup):
        step()
    lib = _lib.load()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    n0 = lib.me_launch_count()
    cg0 = len(app.cg_iterations)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    ev0.record()
    objs = [step() for _ in range(args.steps)]
    ev1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = lib.me_launch_count() - n0
    clk = clocks.stop()
    cg_counts = app.cg_iterations[cg0:]
    ms = rank_max(ms, "cuda")
    if world > 1:
        dist.barrier()
    ms_per_step = ms / args.steps
    value = whole_job_rate(jobs, args.steps, ms)

    # roofline of the dominant unit: one application of the SENSE normal operator, plus the
    # kernel classes inside it, each timed with CUDA events on the launching (current) stream
    pb = app.pb  # this rank's shots (all of them unless sharded)
    Sl = pb.nshots
    p = torch.randn_like(app.x)
    out = torch.empty_like(app.x)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1000.0

    X, Y, Z = shape
    V = X * Y * Z
    t_normal = timed(lambda: pb.normal(p, out))
    # sharded: the same operator with its all-reduce over the ranks (every rank takes part)
    t_normal_reduced = timed(lambda: app._reduced.normal(p, out)) if args.sharded else None
    # one more application inside its own NVTX range, so that a profiler can take exactly the
    # launches of one normal operator (--nvtx-include "normal_op/")
    torch.cuda.nvtx.range_push("normal_op")
    pb.normal(p, out)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    U = torch.empty((Sl, Z, X, Y), dtype=torch.complex64, device=p.device)
    lay = _lib.MeLayout(Y, 1, X * Y)
    st = _lib.stream_ptr()
    t_apply = timed(lambda: _lib.call("me_rigid_apply", _lib.ptr(p), 0, _lib.ptr(U), V, Sl, lay,
                                      pb.grid.ref, _lib.ptr(pb.transforms), 6, 0, st))
    # the SENSE kernels alone, on the shots' transformed volumes just formed: one launch each
    Kb = torch.empty_like(pb.ydat)
    t_sense_fwd = timed(lambda: _lib.call("me_sense_forward_volumes", pb.ref, _lib.ptr(U), V, 0,
                                          Sl, _lib.ptr(Kb), st), reps=5)
    t_sense_adj = timed(lambda: _lib.call("me_sense_adjoint_volumes", pb.ref, _lib.ptr(Kb), 0,
                                          Sl, _lib.ptr(U), V, st), reps=5)
    del U, Kb
    t_lm = timed(lambda: pb.lm_stats(app.x, 0 if args.jacobian == "reference" else 1))
    t_pass = t_apply / 10.0
    mps_bytes = C * 8 * V
    kernels = {
        "rigid_pass": {"seconds_per_launch": t_pass, "algorithmic_bytes": Sl * 2 * 8 * V,
                       "achieved_gbs": Sl * 2 * 8 * V / t_pass / 1e9,
                       "note": f"one FFT-chirp-IFFT line pass over {Sl} shots' volumes"},
        "sense_forward": {"seconds_per_launch": t_sense_fwd,
                          "algorithmic_bytes": Sl * (mps_bytes + 8 * V),
                          "achieved_gbs": Sl * (mps_bytes + 8 * V) / t_sense_fwd / 1e9,
                          "note": f"one launch over {Sl} shots' transformed volumes "
                                  "(me_sense_forward_volumes), mean of 5"},
        "sense_adjoint": {"seconds_per_launch": t_sense_adj,
                          "algorithmic_bytes": Sl * (mps_bytes + 8 * V) + 8 * V,
                          "achieved_gbs": (Sl * (mps_bytes + 8 * V) + 8 * V) / t_sense_adj / 1e9,
                          "note": f"one launch over {Sl} shots' sampled k-space "
                                  "(me_sense_adjoint_volumes), mean of 5"},
        "lm_statistics": {"seconds_per_launch": t_lm,
                          "note": "one call: T x and its six partials for every shot (shared-"
                                  "prefix Jacobian passes) and the 28 Gauss-Newton sums of the "
                                  "seven volumes' forward model, contracted in registers"},
    }
    bytes_normal = Sl * (C * 8 * V + 2 * 8 * V) + Sl * X * Y
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_normal / t_normal / 1e9
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of all launches of one
    # normal-operator application, captured with ncu on the 256x224x32 slab (64 shots, 32 coils)
    # and scaled by the plane count, since every kernel's traffic is per plane: 39.90 GB for
    # 32 planes, of which the 20 line passes 35.6 GB, the forward 1.80 GB, the adjoint 1.60 GB
    # and the shot sum 0.95 GB.  Known only for the workloads with those planes.
    traffic = None
    if (X, Y, C, Sl) == (256, 224, 32, 64):
        traffic = 39.90e9 / 32 * Z

    result = {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if args.sharded else "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic",
        "config": config_dict(args.workload, {
            "parallelism": ("shots sharded" if args.sharded else "replicas") if world > 1
            else "single", "noise_rel_sigma": args.noise,
            "batch_shots": batch or S, "jacobian": args.jacobian, "cg_graph": args.graph,
            "cg_iterations_timed": cg_counts, "objective_last": objs[-1]}),
        "gpu_launches": int(launches),
        "clocks": clk,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_note": "ncu DRAM bytes of one application on the 32-plane slab, "
                                     "scaled by planes; mostly the line passes' volume traffic, "
                                     "which the algorithmic model leaves out"
                     if traffic else None,
                     "kernel": "SENSE normal operator (one application, "
                               + ("this rank's shots)" if args.sharded and world > 1
                                  else "all shots)"),
                     "algorithmic_bytes": bytes_normal, "seconds": t_normal,
                     "seconds_with_allreduce": t_normal_reduced,
                     "kernels": kernels,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks
                     else "fallback 6650 GB/s"},
    }

    # fast vs plain at equal error: the same reconstruction with one shot per launch (the
    # reference's per-shot loop) over the same iterations, timed with events on its last
    # `steps` iterations, and compared iterate for iterate with the batched run above
    if not args.no_plain:
        app_p = Recon(wl["ksp"], wl["mps"], wl["masks"], kg, rk, max_cg_iter=k, max_nm_iter=1,
                      max_joint_iter=args.steps, jacobian=args.jacobian, batch=1,
                      fused_residual=False)
        for _ in range(args.warmup):
            app_p.step()
            app_p._compute_objective()
        torch.cuda.synchronize()
        e0.record()
        objs_p = []
        for _ in range(args.steps):
            app_p.step()
            objs_p.append(app_p._compute_objective())
        e1.record()
        torch.cuda.synchronize()
        ms_p = rank_max(e0.elapsed_time(e1), "cuda")
        plain_value = whole_job_rate(jobs, args.steps, ms_p)
        dx = float(torch.linalg.vector_norm(app_p.x - app.x) / torch.linalg.vector_norm(app.x))
        dt = float((app_p.t - app.t).abs().max())
        result["plain"] = {
            "value": plain_value, "unit": "iter/s", "batch_shots": 1,
            "fast_over_plain": value / plain_value,
            "x_rel_l2_vs_fast": dx, "t_max_abs_diff_vs_fast": dt,
            "objective_last": objs_p[-1],
            "note": "same kernels, one shot per launch (the reference's per-shot loop), the "
                    "CG loop driven from the host, and each solve's initial residual as the "
                    "right-hand side minus A x (two operator passes, as the reference); the same "
                    f"{args.warmup + args.steps} iterations from the same data as the fast run"}
        del app_p
        # the plain form of the same kernels as well: also cp.async staging and the two-kernel
        # LM statistics (one rank; a child process reads the kernel variants at start-up)
        pc = None
        if world == 1 and not args.sharded:
            try:
                pc = run_plain_child(args)
            except (subprocess.SubprocessError, OSError, ValueError) as exc:
                result["plain"]["unstaged"] = {"error": f"child run failed: {exc}"}
        if pc is not None:
            pv = whole_job_rate(jobs, args.steps, float(pc["ms"]))
            xf = app.x.cpu().numpy()
            result["plain"]["unstaged"] = {
                "value": pv, "unit": "iter/s", "fast_over_plain": value / pv,
                "x_rel_l2_vs_fast": float(np.linalg.norm(pc["x"] - xf) / np.linalg.norm(xf)),
                "t_max_abs_diff_vs_fast": float(np.abs(pc["t"] - app.t.cpu().numpy()).max()),
                "note": "one shot per launch, host-loop CG, initial residuals as b - A x, and "
                        "the kernels' plain variants: "
                        "cp.async staging instead of TMA tensor and bulk copies, LM statistics "
                        "through seven written K regions and a second kernel; a child process "
                        "on the same data and iterations"}

    # end to end through the public API from pinned host buffers
    if not args.no_e2e:
        ksp_h = wl["ksp"].cpu().pin_memory()
        mps_h = wl["mps"].cpu().pin_memory()
        masks = wl["masks"]
        J = 2
        torch.cuda.synchronize()
        e0.record()
        t0 = time.perf_counter()
        # host-loop CG: building a CG graph costs more than it saves over two iterations
        app2 = Recon(ksp_h, mps_h, masks, kg, rk, max_cg_iter=k, max_nm_iter=1,
                     max_joint_iter=J, jacobian=args.jacobian, batch=batch)
        x2, t2 = app2.run()
        x_host = x2.cpu()
        t_host = t2.cpu()
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e2e_s = max(e0.elapsed_time(e1) / 1000.0, wall)
        h2d = ksp_h.numel() * 8 + mps_h.numel() * 8 + masks.size
        d2h = x_host.numel() * 8 + t_host.numel() * 8
        result["e2e"] = {"value": jobs * J / e2e_s, "unit": "iter/s", "h2d_bytes_per_step": h2d,
                         "d2h_bytes_per_step": d2h,
                         "note": f"JointRecon(host arrays) + run({J} iterations) + read back, "
                                 f"{e2e_s:.2f} s per call"}
        del app2

    if args.multi:
        result["multi"] = time_multi()
    if args.dft:
        result["dft"] = time_dft()

    if args.pyramid:
        from motionest.pyramid import pyramid_reconstruction
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xp, tp = pyramid_reconstruction(wl["ksp"], wl["mps"], wl["masks"], S, n_spatial_levels=3,
                                        n_joint_iters=20, verbose=False)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        gt = wl["gt"].cpu().numpy()
        err = float(np.linalg.norm(np.abs(xp) - np.abs(gt)) / np.linalg.norm(np.abs(gt)))
        t_true = wl["t"] - wl["t"].mean(axis=0, keepdims=True)
        result["pyramid"] = {
            "seconds": secs, "levels": [0.25, 0.5, 1.0], "outer_iterations": [80, 40, 0],
            "final_cg_iterations": 100,
            "noise_rel_sigma": args.noise,
            "image_rel_err_vs_truth": err,
            "motion_rmse_deg": float(np.degrees(np.sqrt(np.mean((tp[:, 3:] - t_true[:, 3:]) ** 2)))),
            "motion_rmse_vox": float(np.sqrt(np.mean((tp[:, :3] - t_true[:, :3]) ** 2))),
            "note": "end to end through pyramid_reconstruction from device arrays, wall clock; "
                    "errors compare magnitudes with the phantom and mean-removed motion with "
                    "the simulated motion (at the default noise the data are noise-dominated)"}

    if rank == 0 and world == 1 and not args.no_cpu:
        v, sample_s, t = cpu_reference_sample(args.workload, os.cpu_count() or 1)
        result["cpu_baseline"] = {"value": v, "unit": "iter/s", "cores": os.cpu_count() or 1,
                                  "kind": "port",
                                  "sample": "one shot's T, T^H, dT and 32-coil 3-D FFT pair at "
                                            "full size on the oracle port, extrapolated to one "
                                            f"outer iteration ({sample_s:.1f} s of timed CPU "
                                            "work)"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
