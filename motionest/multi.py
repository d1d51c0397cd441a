"""Several independent reconstructions of uneven size on one GPU at once.

The reference reconstructs one acquisition at a time (joint_recon.py:88-106).  MultiRecon holds
any number of JointRecon instances -- different image sizes, coil and shot counts, DISORDER
tilings -- each with its own CUDA stream and each CG solve as one CUDA graph (CgGraph: the
stopping test runs on the device), and advances all of them by one outer iteration per step():
every instance's work is enqueued back to back on its stream with no host synchronisation in
between, so the GPU runs the small instances' kernels beside the large ones' instead of one
reconstruction after another.  One synchronisation per step then collects the CG iteration
counts and objectives.  Shots per launch come from the launch-shape autotuner
(motionest/autotune.py) unless given.

Every instance computes exactly what a JointRecon of it alone computes (same kernels, same
order on its stream), so the results do not depend on what runs beside it.
"""
import torch

from . import _lib
from ._lib import ptr
from .joint_recon import JointRecon


def apply_transforms(jobs):
    """out = T(params) x for several reconstructions at once (me_rigid_apply_multi: each shear
    step is one persistent launch per line length over all jobs' volumes and line tiles).

    jobs: list of dicts with `x` (a zxy image [Z, X, Y], shared by all of the job's volumes),
    `out` ([nvol, Z, X, Y] complex64), `params` ([nvol, 6] float64) and `grid` (a DeviceGrid
    of the image's shape), all on the current CUDA device.  Up to 16 jobs."""
    arr = (_lib.MeRigidJob * len(jobs))()
    for i, jb in enumerate(jobs):
        Z, X, Y = jb["x"].shape
        out = jb["out"]
        arr[i].in_ = jb["x"].data_ptr()
        arr[i].in_vol_stride = 0
        arr[i].out = out.data_ptr()
        arr[i].out_vol_stride = X * Y * Z
        arr[i].nvol = out.shape[0]
        arr[i].lay = _lib.MeLayout(Y, 1, X * Y)
        arr[i].grid = _lib.ctypes.addressof(jb["grid"].struct)
        arr[i].params = jb["params"].data_ptr()
        arr[i].pstride = 6
    _lib.call("me_rigid_apply_multi", arr, len(jobs), _lib.stream_ptr())
    return [jb["out"] for jb in jobs]


class MultiRecon:
    """problems: list of dicts with ksp, mps, masks (centred, as JointRecon takes them), kgrid,
    rkgrid and optionally t0; joint_kwargs go to every JointRecon (max_cg_iter, max_nm_iter,
    jacobian, batch, ...)."""

    def __init__(self, problems, **joint_kwargs):
        _lib.require_cuda()
        kw = dict(joint_kwargs)
        kw["cg_graph"] = True
        kw.setdefault("batch", "auto")
        self.apps, self.streams = [], []
        for p in problems:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                app = JointRecon(p["ksp"], p["mps"], p["masks"], p["kgrid"], p["rkgrid"],
                                 t0=p.get("t0"), **kw)
            self.apps.append(app)
            self.streams.append(s)
        for s in self.streams:
            torch.cuda.current_stream().wait_stream(s)
        self.objective_history = [[] for _ in self.apps]

    def step(self):
        """One outer iteration of every instance; returns their objectives."""
        objs = []
        cur = torch.cuda.current_stream()
        for app, s in zip(self.apps, self.streams):
            s.wait_stream(cur)
            with torch.cuda.stream(s):
                app.step(sync=False)
                objs.append(app.objective_tensor())
        for s in self.streams:
            cur.wait_stream(s)
        out = []
        for app, o, h in zip(self.apps, objs, self.objective_history):
            app.collect()
            h.append(float(o.item()))
            out.append(h[-1])
        return out

    def run(self, iterations):
        for _ in range(iterations):
            self.step()
        return [(app.image(), app.t) for app in self.apps]

    def close(self):
        for app in self.apps:
            if app._graph is not None:
                app._graph.close()
