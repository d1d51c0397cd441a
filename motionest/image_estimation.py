"""CG-SENSE image step with the reference's interface (image_estimation.py:10-165)."""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._arrays import like_input, to_device
from ._lib import ptr
from .problem import SenseProblem, xyz_to_zxy, zxy_to_xyz


def cg_solve(pb, x, max_iter, tol, b=None, fused=True, r=None, r_ready=False):
    """Preconditioned CG on A = M sum_s T_s^H C^H F^H M_s F C T_s, in place on the zxy image x.

    Same recurrences and stopping rule as image_estimation.py:131-163 (r = b - A x, z = P r,
    p = z; alpha = <r,z>/<p,Ap>; stop when sqrt|<r',z'>| < tol; beta = <r',z'>/<r,z>), with the
    inner products accumulated in float64 on the device.  Returns the number of A applications
    inside the loop.

    The initial residual b - A x: with `fused` (and no `b`) one pass over the shots forms it
    (SenseProblem.residual: forward model, y - K at the samples, adjoint); otherwise the
    right-hand side and A x are formed separately and subtracted, as the reference does.  `r`
    is an optional buffer for the residual; with `r_ready` it already holds b - A x for this x
    and the problem's transforms, and the solve starts from it."""
    n = x.numel()
    if r is None:
        r = torch.empty_like(x)
    p = torch.empty_like(x)
    Ap = torch.empty_like(x)
    s = torch.zeros(8, dtype=torch.float64, device=x.device)
    w = ptr(pb.cg_work)
    st = _lib.stream_ptr()
    if r_ready or (fused and b is None):
        if not r_ready:
            pb.residual(x, r)
        _lib.call("me_cg_init", ptr(r), None, ptr(pb.P), ptr(r), ptr(p), ptr(s), n, w, st)
    else:
        if b is None:
            b = pb.rhs(pb.empty_image())
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
    """cg_solve as one CUDA graph (me_cg_graph_create): the CG initialisation and the
    iterations with their stopping test, all on the device, over fixed buffers, preceded by the
    initial residual.  With `fused` the graph starts from the residual b - A x that launch()
    forms in one pass (SenseProblem.residual) just before it, or that the caller has already
    put into `r`; otherwise the right-hand side and A x are part of the graph, as in the
    reference.  The image x (zxy) is solved in place on every run(); the problem's transforms
    are re-read on every run, so the graph serves every outer iteration of a reconstruction
    whose transform tensor is updated in place."""

    def __init__(self, pb, x, max_iter, tol, fused=True, r=None):
        self.pb = pb
        self.x = x
        self.fused = fused
        n = x.numel()
        dev = x.device
        self.b = None if fused else torch.empty_like(x)
        self.r = torch.empty_like(x) if r is None else r
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
            # (r too: with `fused` it may already hold a residual the caller formed)
            xs = x.clone()
            rs = torch.empty_like(x)
            pb.normal(xs, self.Ap)
            if fused:
                # the residual pass itself runs outside the graph; only the initialisation
                # from a given residual is captured
                rs.copy_(self.Ap)
                _lib.call("me_cg_init", ptr(rs), None, ptr(pb.P), ptr(rs), ptr(self.p),
                          ptr(self.s), n, w, st)
            else:
                pb.rhs(self.b)
                _lib.call("me_cg_init", ptr(self.b), ptr(self.Ap), ptr(pb.P), ptr(rs),
                          ptr(self.p), ptr(self.s), n, w, st)
            _lib.call("me_cg_pap", ptr(self.p), ptr(self.Ap), ptr(self.s), n, w, st)
            _lib.call("me_cg_update", ptr(xs), ptr(rs), ptr(self.p), ptr(self.Ap),
                      ptr(pb.P), ptr(self.s), n, w, st)
            _lib.call("me_cg_direction", ptr(self.p), ptr(rs), ptr(pb.P), ptr(self.s), n, st)
            del xs, rs
            h = ctypes.c_void_p()
            _lib.call("me_cg_graph_create", pb.ref, ptr(x),
                      None if fused else ptr(self.b), ptr(self.r),
                      ptr(self.p), ptr(self.Ap), ptr(self.s), ptr(self.iters), self.max_iter,
                      float(tol), pb.batch, ptr(pb.work), w, st, ctypes.byref(h))
            self._handle = h
        torch.cuda.current_stream().wait_stream(stream)
        self._stream = stream

    def launch(self, r_ready=False):
        """Enqueue the solve on the current stream (no host synchronisation).  With `fused`,
        first the initial residual into r, unless `r_ready` says r already holds it for the
        current x and transforms."""
        if self.fused and not r_ready:
            self.pb.residual(self.x, self.r)
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
