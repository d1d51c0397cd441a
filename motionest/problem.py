"""Device-resident SENSE problem: everything the CG and LM steps read, in the layouts the
kernels want, plus the me_sense struct that describes it to libmotionest.so.

Built once per reconstruction (JointRecon.__init__ does what joint_recon.py:62-85 does:
uncentre, normalise, P and M) and then reused by every CG iteration, LM step and objective
evaluation, so no per-iteration host work or layout change happens.

Layouts (see include/motionest.h): images [Z][X][Y] ("zxy"), maps [Z][C][X][Y], measured data
as per-shot sample lists in hybrid space [Z][C][n_s].
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import ptr
from .sampling import SampleLists, plane_masks
from .utils import DeviceGrid


def xyz_to_zxy(v):
    return v.permute(2, 0, 1).contiguous()


def zxy_to_xyz(v):
    return v.permute(1, 2, 0).contiguous()


def hybrid_kspace(ksp_u, stream=None):
    """Orthonormal IFFT along z of uncentred k-space [C, X, Y, Z] (one launch, my kernels)."""
    C, X, Y, Z = ksp_u.shape
    out = torch.empty_like(ksp_u)
    lay = _lib.MeLayout(Y * Z, Z, 1)
    _lib.call("me_fft_axis", ptr(ksp_u), X * Y * Z, ptr(out), X * Y * Z, C, X, Y, Z, lay, 2, 1,
              _lib.stream_ptr(stream))
    return out


def max_abs_image(ksp_h, stream=None):
    """max |IFFT_xyz(ksp)| given the hybrid (IFFT_z) k-space: the normaliser of
    joint_recon.py:67.  Transforms one coil at a time through a single scratch volume."""
    C, X, Y, Z = ksp_h.shape
    vox = X * Y * Z
    tmp = torch.empty((X, Y, Z), dtype=torch.complex64, device=ksp_h.device)
    lay = _lib.MeLayout(Y * Z, Z, 1)
    best = torch.zeros(C, dtype=torch.float32, device=ksp_h.device)
    work = torch.empty(_lib.load().me_cg_workspace_bytes(vox), dtype=torch.uint8,
                       device=ksp_h.device)
    st = _lib.stream_ptr(stream)
    for c in range(C):
        src = ksp_h[c]
        _lib.call("me_fft_axis", ptr(src), 0, ptr(tmp), 0, 1, X, Y, Z, lay, 0, 1, st)
        _lib.call("me_fft_axis", ptr(tmp), 0, ptr(tmp), 0, 1, X, Y, Z, lay, 1, 1, st)
        _lib.call("me_max_abs", ptr(tmp), vox, ctypes.c_void_p(best.data_ptr() + 4 * c),
                  ptr(work), st)
    return best.max()


class SenseProblem:
    """Device data of one reconstruction and the C-ABI operators on it.

    ksp_u, mps_u: uncentred [C, X, Y, Z] complex64 CUDA tensors (ksp already normalised);
    planes: uncentred [S, X, Y] bool masks (host); transforms: [S, 6] float64 CUDA tensor
    (the problem keeps a reference and always reads its current values)."""

    def __init__(self, ksp_u, mps_u, planes, kgrid, rkgrid, transforms, P=None, M=None,
                 batch=None, lm_batch=None, grid=None):
        _lib.require_cuda()
        C, X, Y, Z = mps_u.shape
        self.shape = (X, Y, Z)
        self.ncoils = C
        self.vox = X * Y * Z
        dev = mps_u.device
        self.device = dev
        planes = plane_masks(planes)
        if planes.shape[1:] != (X, Y):
            raise ValueError(f"mask plane {planes.shape[1:]} does not match the image {(X, Y)}")
        self.nshots = planes.shape[0]
        self.samples = SampleLists(planes)
        sm = self.samples
        self._keep = []

        def up_i32(a):
            t = torch.as_tensor(a, dtype=torch.int32).to(dev)
            self._keep.append(t)
            return t

        self.shot_off = up_i32(sm.shot_off)
        self.kx = up_i32(sm.kx if sm.total else np.zeros(1, np.int32))
        self.ky = up_i32(sm.ky if sm.total else np.zeros(1, np.int32))
        self.ky_off = up_i32(sm.ky_off)
        self.ky_order = up_i32(sm.ky_order if sm.ky_order.size else np.zeros(1, np.int32))
        self.grid = grid if grid is not None else DeviceGrid(kgrid, rkgrid, (X, Y, Z))
        self.mps = mps_u.permute(3, 0, 1, 2).contiguous()  # [Z][C][X][Y]
        if P is None or M is None:
            self.P = torch.empty((Z, X, Y), dtype=torch.float32, device=dev)
            self.M = torch.empty((Z, X, Y), dtype=torch.uint8, device=dev)
            _lib.call("me_sense_precond", ptr(self.mps), X, Y, Z, C, ptr(self.P), ptr(self.M),
                      _lib.stream_ptr())
        else:
            self.P = xyz_to_zxy(torch.as_tensor(P).to(dev, torch.float32))
            self.M = xyz_to_zxy(torch.as_tensor(M).to(dev).to(torch.uint8))
        self.transforms = transforms
        total = max(sm.total, 1)
        self.ydat = torch.empty(total * C * Z, dtype=torch.complex64, device=dev)
        self._build_struct()
        if ksp_u is not None:
            self.set_kspace(ksp_u)
        lib = _lib.load()
        self.work = torch.empty(0, dtype=torch.uint8, device=dev)
        self.batch = self.lm_batch = 1
        auto = batch == "auto"
        self.set_batches(self.nshots if auto else (batch or self.nshots), lm_batch or 8)
        self.cg_work = torch.empty(lib.me_cg_workspace_bytes(self.vox), dtype=torch.uint8,
                                   device=dev)
        if auto:
            from .autotune import tune
            tune(self)

    def set_batches(self, batch, lm_batch):
        """Shots per launch for the SENSE operators and for the LM statistics; grows the
        workspace when needed (results do not depend on either)."""
        lib = _lib.load()
        self.batch = max(1, min(int(batch), self.nshots))
        self.lm_batch = max(1, min(int(lm_batch), self.nshots))
        wb = max(lib.me_sense_workspace_bytes(self.ref, self.batch),
                 lib.me_lm_workspace_bytes(self.ref, self.lm_batch))
        if wb < 0:
            raise ValueError(lib.me_last_error().decode())
        if self.work.numel() < wb:
            self.work = torch.empty(0, dtype=torch.uint8, device=self.device)
            self.work = torch.empty(int(wb), dtype=torch.uint8, device=self.device)

    def _build_struct(self):
        sm = self.samples
        X, Y, Z = self.shape
        s = _lib.MeSense()
        s.nx, s.ny, s.nz, s.ncoils, s.nshots = X, Y, Z, self.ncoils, self.nshots
        s.mps = self.mps.data_ptr()
        s.samples.nshots, s.samples.nx, s.samples.ny = sm.nshots, sm.nx, sm.ny
        s.samples.max_per_shot = sm.max_per_shot
        s.samples.shot_off = self.shot_off.data_ptr()
        s.samples.kx = self.kx.data_ptr()
        s.samples.ky = self.ky.data_ptr()
        s.samples.ky_off = self.ky_off.data_ptr()
        s.samples.ky_order = self.ky_order.data_ptr()
        s.ydat = self.ydat.data_ptr()
        s.P = self.P.data_ptr()
        s.M = self.M.data_ptr()
        s.grid = ctypes.addressof(self.grid.struct)
        s.transforms = self.transforms.data_ptr()
        self.struct = s
        self.ref = ctypes.byref(s)

    def set_transforms(self, t):
        self.transforms = t
        self.struct.transforms = t.data_ptr()

    def set_kspace(self, ksp_u):
        """ydat = the shots' samples of IFFT_z(ksp) (uncentred, normalised k-space)."""
        kh = hybrid_kspace(ksp_u)
        _lib.call("me_sense_gather", self.ref, ptr(kh), ptr(self.ydat), _lib.stream_ptr())

    def agree_stop(self, stop):
        """The CG stopping decision (one process decides alone)."""
        return stop

    # ------------------------------------------------------------------ operators (zxy)
    def empty_image(self):
        X, Y, Z = self.shape
        return torch.empty((Z, X, Y), dtype=torch.complex64, device=self.device)

    def _unmasked(self):
        """The problem description with the support mask M left out."""
        s = _lib.MeSense.from_buffer_copy(self.struct)
        s.M = None
        return s

    def normal(self, p, out, batch=None, masked=True):
        ref = self.ref if masked else ctypes.byref(self._unmasked())
        _lib.call("me_sense_normal", ref, ptr(p), ptr(out), batch or self.batch,
                  ptr(self.work), _lib.stream_ptr())
        return out

    def rhs(self, out, batch=None, masked=True):
        ref = self.ref if masked else ctypes.byref(self._unmasked())
        _lib.call("me_sense_rhs", ref, ptr(out), batch or self.batch, ptr(self.work),
                  _lib.stream_ptr())
        return out

    def residual(self, x, out, energies=None, batch=None):
        """out = b - A x, the CG's initial residual, from one pass over the shots
        (me_sense_residual); with `energies` ([nshots] float64) also each shot's
        ||M_s (F C T_s x - y)||^2 at the problem's transforms."""
        e = ptr(energies) if energies is not None else None
        _lib.call("me_sense_residual", self.ref, ptr(x), ptr(out), e, batch or self.batch,
                  ptr(self.work), _lib.stream_ptr())
        return out

    def residual_norms(self, x, transforms, out=None, batch=None):
        if out is None:
            out = torch.empty(self.nshots, dtype=torch.float64, device=self.device)
        _lib.call("me_sense_residual_norms", self.ref, ptr(x), ptr(transforms), ptr(out),
                  batch or self.batch, ptr(self.work), _lib.stream_ptr())
        return out

    def forward(self, x, transforms, out=None, batch=None):
        """Per-shot sampled hybrid k-space M_s F_xy C T_s x (ydat layout)."""
        if out is None:
            out = torch.empty_like(self.ydat)
        _lib.call("me_sense_forward", self.ref, ptr(x), ptr(transforms), ptr(out),
                  batch or self.batch, ptr(self.work), _lib.stream_ptr())
        return out

    def scatter(self, K, ksp_h):
        """ksp_h[c, kx, ky, z] += K at every shot's samples (duplicates add up)."""
        _lib.call("me_sense_scatter", self.ref, ptr(K), ptr(ksp_h), _lib.stream_ptr())
        return ksp_h

    def lm_gradient(self, x, jac_mode, out=None, batch=None):
        """[S, 7] float64: e0 and the gradient g of each shot (me_lm_gradient), with a
        workspace of its own (the LM workspace, which CG graphs may hold, is left alone)."""
        if out is None:
            out = torch.empty((self.nshots, 7), dtype=torch.float64, device=self.device)
        b = batch or self.lm_batch
        need = _lib.load().me_lm_gradient_workspace_bytes(self.ref, b)
        if need < 0:
            raise ValueError(_lib.load().me_last_error().decode())
        if getattr(self, "_grad_work", None) is None or self._grad_work.numel() < need:
            self._grad_work = torch.empty(int(need), dtype=torch.uint8, device=self.device)
        _lib.call("me_lm_gradient", self.ref, ptr(x), int(jac_mode), ptr(out), b,
                  ptr(self._grad_work), _lib.stream_ptr())
        return out

    def lm_stats(self, x, jac_mode, out=None, batch=None):
        if out is None:
            out = torch.empty((self.nshots, 28), dtype=torch.float64, device=self.device)
        _lib.call("me_lm_normal_equations", self.ref, ptr(x), int(jac_mode), ptr(out),
                  batch or self.lm_batch, ptr(self.work), _lib.stream_ptr())
        return out

    def apply_transform(self, x, params, out=None, inverse=False):
        """out = T(params) x on a zxy image (params: [6] float64 CUDA tensor)."""
        X, Y, Z = self.shape
        out = x if out is None else out
        lay = _lib.MeLayout(Y, 1, X * Y)
        _lib.call("me_rigid_apply", ptr(x), 0, ptr(out), 0, 1, lay, self.grid.ref, ptr(params), 0,
                  int(inverse), _lib.stream_ptr())
        return out


def fft_axes(v, axes, inverse, out=None):
    """Orthonormal (I)FFT of a [..., X, Y, Z] complex64 CUDA tensor along the given spatial
    axes (0, 1, 2 = X, Y, Z), batched over the leading dims, with libmotionest's line kernels."""
    v = v.contiguous()
    X, Y, Z = v.shape[-3:]
    nvol = v.numel() // (X * Y * Z)
    out = torch.empty_like(v) if out is None else out
    lay = _lib.MeLayout(Y * Z, Z, 1)
    src = v
    for a in axes:
        _lib.call("me_fft_axis", ptr(src), X * Y * Z, ptr(out), X * Y * Z, nvol, X, Y, Z, lay, a,
                  int(inverse), _lib.stream_ptr())
        src = out
    if not axes:
        out.copy_(v)
    return out


def centred_fft(v, inverse=False):
    """SigPy-style centred orthonormal 3-D (I)FFT over the last three axes."""
    ax = (-3, -2, -1)
    u = torch.fft.ifftshift(v, dim=ax).contiguous()
    return torch.fft.fftshift(fft_axes(u, (0, 1, 2), inverse), dim=ax)


def centred_resize(v, oshape):
    """Centred crop / zero-pad (SigPy's resize convention, used at pyramid.py:65-67)."""
    ishape = tuple(v.shape)
    oshape = tuple(oshape)
    if ishape == oshape:
        return v
    ish = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)]
    osh = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)]
    cp = [min(i - a, o - b) for i, a, o, b in zip(ishape, ish, oshape, osh)]
    out = torch.zeros(oshape, dtype=v.dtype, device=v.device)
    out[tuple(slice(b, b + c) for b, c in zip(osh, cp))] = \
        v[tuple(slice(a, a + c) for a, c in zip(ish, cp))]
    return out
