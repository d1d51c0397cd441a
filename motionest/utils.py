"""Transform grids (utils.py:107-137 of the reference) and their device form."""
import ctypes

import numpy as np
import torch

from . import _lib
from ._arrays import as_float64_host


def compute_transform_grids_voxel(shape, voxel_size, downsample_res=None, xp=np):
    """fftshifted spatial and spectral grids for the shear-based rigid transform.

    Same outputs as the reference (utils.py:107-137): kgrid = {'x','y','z'} float64 vectors
    shaped (X,1,1), (1,Y,1), (1,1,Z) over the (downsampled) sample counts, and
    rkgrid['tan'|'sin'][axis] products of the full-resolution r grid with the k grid.
    `xp` may be numpy or torch (torch returns float64 CUDA tensors)."""
    nx, ny, nz = shape
    vx, vy, vz = voxel_size
    if downsample_res is None:
        downsample_res = shape
    ds_x, ds_y, ds_z = downsample_res
    fs = np.fft.fftshift
    rx = fs((np.linspace(-nx // 2, nx // 2, ds_x, endpoint=False) * vx).reshape(-1, 1, 1))
    ry = fs((np.linspace(-ny // 2, ny // 2, ds_y, endpoint=False) * vy).reshape(1, -1, 1))
    rz = fs((np.linspace(-nz // 2, nz // 2, ds_z, endpoint=False) * vz).reshape(1, 1, -1))
    kx = fs(np.linspace(-np.pi, np.pi, ds_x, endpoint=False).reshape((-1, 1, 1)))
    ky = fs(np.linspace(-np.pi, np.pi, ds_y, endpoint=False).reshape((1, -1, 1)))
    kz = fs(np.linspace(-np.pi, np.pi, ds_z, endpoint=False).reshape((1, 1, -1)))
    kgrid = {"x": kx, "y": ky, "z": kz}
    rkgrid = {"tan": {"x": rz * ky, "y": rx * kz, "z": ry * kx},
              "sin": {"x": ry * kz, "y": rz * kx, "z": rx * ky}}
    if xp is torch:
        dev = torch.device("cuda", torch.cuda.current_device())
        conv = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)  # noqa: E731
        kgrid = {k: conv(v) for k, v in kgrid.items()}
        rkgrid = {m: {k: conv(v) for k, v in d.items()} for m, d in rkgrid.items()}
    return kgrid, rkgrid


class DeviceGrid:
    """kgrid/rkgrid uploaded once as float64 CUDA tensors, plus the me_grid struct that points
    at them.  Keeps the tensors alive as long as the struct is used."""

    def __init__(self, kgrid, rkgrid, shape=None):
        dev = torch.device("cuda", torch.cuda.current_device())
        self.tensors = []

        def up(a):
            t = torch.as_tensor(as_float64_host(a), dtype=torch.float64).to(dev).contiguous()
            self.tensors.append(t)
            return t

        ks = [up(kgrid[a]) for a in "xyz"]
        dims = tuple(int(k.numel()) for k in ks)
        if shape is not None and tuple(shape) != dims:
            raise ValueError(f"grid sizes {dims} do not match the volume shape {tuple(shape)}")
        self.shape = dims
        g = _lib.MeGrid()
        g.nx, g.ny, g.nz = dims
        for i, k in enumerate(ks):
            g.k[i] = k.data_ptr()
        for m, field, stf in (("tan", g.tan_rk, g.tan_st), ("sin", g.sin_rk, g.sin_st)):
            for i, a in enumerate("xyz"):
                t = up(rkgrid[m][a])
                if t.dim() != 3:
                    t = t.reshape((1,) * (3 - t.dim()) + tuple(t.shape))
                for d in range(3):
                    if t.shape[d] not in (1, dims[d]):
                        raise ValueError(f"rkgrid['{m}']['{a}'] shape {tuple(t.shape)} does not "
                                         f"broadcast to {dims}")
                field[i] = t.data_ptr()
                for d in range(3):
                    stf[i][d] = t.stride(d) if t.shape[d] > 1 else 0
                self.tensors.append(t)
        # separable / uniform structure (lets the kernels use chirp recurrences)
        knp = [as_float64_host(kgrid[a]).reshape(-1) for a in "xyz"]
        for a in range(3):
            g.k_uniform[a] = int(_is_uniform_fftshift(knp[a]))
        shear_axis = {"tan": (1, 2, 0), "sin": (2, 0, 1)}
        for m, field in (("tan", g.tan_r), ("sin", g.sin_r)):
            for i, a in enumerate("xyz"):
                ax = shear_axis[m][i]
                r = _separable_factor(as_float64_host(rkgrid[m][a]), knp[ax], ax)
                if r is not None and g.k_uniform[ax]:
                    t = up(r)
                    field[i] = t.data_ptr()
        self.struct = g
        self.ref = ctypes.byref(self.struct)


def _is_uniform_fftshift(k):
    """k == 2 pi (m(n) - N/2) / N with m(n) = (n - N//2) mod N (fftshifted linspace)."""
    n = k.size
    m = (np.arange(n) - n // 2) % n
    ref = 2.0 * np.pi * (m - n / 2.0) / n
    return bool(np.allclose(k, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max())))


def _separable_factor(plane, kvec, ax):
    """If the 3-D broadcast plane equals r[o] * kvec[n] (n along axis `ax`, o along its other
    non-broadcast axis), return r as a full-length vector over axis o; else None."""
    p = np.asarray(plane, dtype=np.float64)
    if p.ndim != 3:
        return None
    axes = [d for d in range(3) if p.shape[d] > 1 and d != ax]
    if len(axes) != 1 or p.shape[ax] != kvec.size:
        return None
    o = axes[0]
    q = np.moveaxis(p, (ax, o), (0, 1)).reshape(p.shape[ax], p.shape[o], -1)
    if q.shape[2] != 1:
        return None
    q = q[..., 0]
    i = int(np.argmax(np.abs(kvec)))
    if kvec[i] == 0:
        return None
    r = q[i] / kvec[i]
    if not np.allclose(np.outer(kvec, r), q, rtol=1e-13, atol=1e-13 * max(1.0, np.abs(q).max())):
        return None
    return r


_grid_cache = {}


def device_grid(kgrid, rkgrid, shape=None):
    """DeviceGrid for (kgrid, rkgrid), cached by the identity of the dicts' arrays."""
    key = (id(kgrid), id(rkgrid), torch.cuda.current_device())
    hit = _grid_cache.get(key)
    if hit is not None and hit[0] is kgrid and hit[1] is rkgrid:
        return hit[2]
    dg = DeviceGrid(kgrid, rkgrid, shape)
    if len(_grid_cache) > 64:
        _grid_cache.clear()
    _grid_cache[key] = (kgrid, rkgrid, dg)
    return dg
