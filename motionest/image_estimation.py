"""CG-SENSE image step with the reference's interface (image_estimation.py:10-165)."""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._arrays import like_input, to_device
from ._lib import ptr
from .problem import SenseProblem, xyz_to_zxy, zxy_to_xyz


def cg_solve(pb, x, max_iter, tol, b=None):
    """Preconditioned CG on A = M sum_s T_s^H C^H F^H M_s F C T_s, in place on the zxy image x.

    Same recurrences and stopping rule as image_estimation.py:131-163 (r = b - A x, z = P r,
    p = z; alpha = <r,z>/<p,Ap>; stop when sqrt|<r',z'>| < tol; beta = <r',z'>/<r,z>), with the
    inner products accumulated in float64 on the device.  Returns the number of A applications
    inside the loop."""
    n = x.numel()
    if b is None:
        b = pb.rhs(pb.empty_image())
    r = torch.empty_like(x)
    p = torch.empty_like(x)
    Ap = torch.empty_like(x)
    s = torch.zeros(8, dtype=torch.float64, device=x.device)
    w = ptr(pb.cg_work)
    st = _lib.stream_ptr()
    pb.normal(x, Ap)
    _lib.call("me_cg_init", ptr(b), ptr(Ap), ptr(pb.P), ptr(r), ptr(p), ptr(s), n, w, st)
    iters = 0
    for _ in range(max_iter):
        pb.normal(p, Ap)
        _lib.call("me_cg_pap", ptr(p), ptr(Ap), ptr(s), n, w, st)
        _lib.call("me_cg_update", ptr(x), ptr(r), ptr(p), ptr(Ap), ptr(pb.P), ptr(s), n, w, st)
        iters += 1
        rz_new = float(s[2].item())
        if pb.agree_stop(math.sqrt(abs(rz_new)) < tol):
            break
        _lib.call("me_cg_direction", ptr(p), ptr(r), ptr(pb.P), ptr(s), n, st)
    return iters


class CgGraph:
    """cg_solve as one CUDA graph (me_cg_graph_create): the right-hand side, A x, the CG
    initialisation and the iterations with their stopping test, all on the device, over fixed
    buffers.  The image x (zxy) is solved in place on every run(); the problem's transforms
    are re-read on every run, so the graph serves every outer iteration of a reconstruction
    whose transform tensor is updated in place."""

    def __init__(self, pb, x, max_iter, tol):
        self.pb = pb
        self.x = x
        n = x.numel()
        dev = x.device
        self.b = torch.empty_like(x)
        self.r = torch.empty_like(x)
        self.p = torch.empty_like(x)
        self.Ap = torch.empty_like(x)
        self.s = torch.zeros(8, dtype=torch.float64, device=dev)
        self.iters = torch.zeros(1, dtype=torch.int32, device=dev)
        self.max_iter = int(max_iter)
        self._handle = None
        w = ptr(pb.cg_work)
        stream = torch.cuda.Stream(device=dev)
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            st = _lib.stream_ptr(stream)
            # every captured call runs once first, on scratch, so no first use is captured
            xs = x.clone()
            pb.rhs(self.b)
            pb.normal(xs, self.Ap)
            _lib.call("me_cg_init", ptr(self.b), ptr(self.Ap), ptr(pb.P), ptr(self.r),
                      ptr(self.p), ptr(self.s), n, w, st)
            _lib.call("me_cg_pap", ptr(self.p), ptr(self.Ap), ptr(self.s), n, w, st)
            _lib.call("me_cg_update", ptr(xs), ptr(self.r), ptr(self.p), ptr(self.Ap),
                      ptr(pb.P), ptr(self.s), n, w, st)
            _lib.call("me_cg_direction", ptr(self.p), ptr(self.r), ptr(pb.P), ptr(self.s), n, st)
            del xs
            h = ctypes.c_void_p()
            _lib.call("me_cg_graph_create", pb.ref, ptr(x), ptr(self.b), ptr(self.r),
                      ptr(self.p), ptr(self.Ap), ptr(self.s), ptr(self.iters), self.max_iter,
                      float(tol), pb.batch, ptr(pb.work), w, st, ctypes.byref(h))
            self._handle = h
        torch.cuda.current_stream().wait_stream(stream)
        self._stream = stream

    def launch(self):
        """Enqueue the solve on the current stream (no host synchronisation)."""
        _lib.call("me_cg_graph_launch", self._handle, _lib.stream_ptr())

    def count(self):
        """CG iterations the last solve took (one host read)."""
        it = int(self.iters.item())
        _lib.load().me_cg_graph_account(self._handle, it)
        return it

    def run(self):
        """Solve in place on x; returns the CG iterations taken."""
        self.launch()
        return self.count()

    def close(self):
        if self._handle is not None:
            torch.cuda.synchronize(self.x.device)
            _lib.call("me_cg_graph_destroy", self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def estimate_image_cg(ksp, mps, shot_mask, transforms, kgrid, rkgrid, P, M, x0=None,
                      max_iter=100, tol=1e-6, show_pbar=True, batch=None):
    """Reconstruct the image by preconditioned CG-SENSE given the per-shot transforms.

    Arguments and semantics as the reference's estimate_image_cg: uncentred ksp/mps
    [ncoils, X, Y, Z] complex64, shot_mask [nshots, X, Y, 1] bool, transforms [nshots, 6],
    P and M image-space [X, Y, Z].  `batch` (extra) = shots per kernel launch (default: all).
    Returns x [X, Y, Z] complex64 as the caller's array kind (NumPy in -> NumPy out)."""
    _lib.require_cuda()
    ksp_t = to_device(ksp, torch.complex64)
    mps_t = to_device(mps, torch.complex64)
    t = to_device(np.asarray(transforms, dtype=np.float64) if not isinstance(transforms, torch.Tensor)
                  else transforms, torch.float64)
    planes = _host_mask(shot_mask)
    pb = SenseProblem(ksp_t, mps_t, planes, kgrid, rkgrid, t, P=_host(P), M=_host(M), batch=batch)
    x = pb.empty_image()
    if x0 is None:
        x.zero_()
    else:
        x.copy_(xyz_to_zxy(to_device(x0, torch.complex64)))
    cg_solve(pb, x, max_iter, tol)
    return like_input(zxy_to_xyz(x), ksp)


def _host(a):
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    if hasattr(a, "get"):
        return a.get()
    return np.asarray(a)


def _host_mask(m):
    return _host(m).astype(bool)
