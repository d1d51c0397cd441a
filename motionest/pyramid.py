"""Coarse-to-fine driver with the reference's interface (pyramid.py:24-118)."""
import numpy as np
import torch

from . import _lib
from ._arrays import to_device
from .image_estimation import _host_mask, cg_solve
from .joint_recon import JointRecon
from .problem import SenseProblem, centred_fft, centred_resize, hybrid_kspace, max_abs_image, \
    xyz_to_zxy, zxy_to_xyz
from .utils import compute_transform_grids_voxel

AX3 = (-3, -2, -1)


def aggregate_sampling_masks(A, bin_factor):
    """Masks of `bin_factor` consecutive shots summed into one motion state
    (pyramid.py:120-123): [nshots, ...] -> [nshots // bin_factor, ...] sample counts."""
    A = np.asarray(A)
    nb = A.shape[0] // bin_factor
    return A.reshape((nb, bin_factor) + A.shape[1:]).sum(1)


def aggregate_transforms(T, bin_factor):
    """Transforms of `bin_factor` consecutive shots summed per motion state (pyramid.py:125-128);
    divide by bin_factor for the bin's mean transform."""
    T = np.asarray(T)
    nb = T.shape[0] // bin_factor
    return T.reshape(nb, bin_factor, 6).sum(1)


def pyramid_reconstruction(ksp, mps, A, nshots, n_spatial_levels=3, n_temporal_levels=3,
                           n_joint_iters=100, save_path=None, sampling="disorder",
                           verbose=True, temporal=False, **joint_kwargs):
    """Multi-resolution joint reconstruction, as the reference's pyramid_reconstruction.

    Coarse levels (factor 4, then 2, ...) crop k-space and masks in x and y (z kept for
    DISORDER), resample the maps by centred FFT / crop / IFFT, and run JointRecon for
    n_joint_iters * factor outer iterations starting from the previous level's transforms
    (carried unscaled, with the full-resolution r grid and the downsampled k grid, as
    pyramid.py:72-73 does).  The full-resolution level is image-only CG with the reference's
    default 100 iterations.  Returns (x [X, Y, Z] complex NumPy, centred; t [nshots, 6]).
    Convergence plots are not drawn (save_path is accepted and ignored).  joint_kwargs (extra)
    are passed to JointRecon.

    Temporal levels: the reference sketches them but leaves them disabled (pyramid.py:80-95),
    so by default n_temporal_levels is unused, as there.  temporal=True (extra) runs them at the
    coarsest spatial level, before its per-shot JointRecon: for factors 2^(L-1), ..., 2 (L =
    n_temporal_levels; factors that do not divide nshots are skipped) the shots are merged
    into nshots / factor motion states -- masks summed (aggregate_sampling_masks), the bin's
    mean transform as the start (aggregate_transforms / factor) -- reconstructed jointly for
    the level's iterations, and every shot then starts from its bin's estimate."""
    _lib.require_cuda()
    ksp_t = to_device(ksp, torch.complex64)
    mps_t = to_device(mps, torch.complex64)
    A_np = _host_mask(A)
    full = tuple(ksp_t.shape[1:])
    ncoils = ksp_t.shape[0]
    t_est = torch.zeros((nshots, 6), dtype=torch.float64, device=ksp_t.device)
    for sl in range(n_spatial_levels - 1):
        f = 2 ** (n_spatial_levels - sl - 1)
        if sampling == "disorder":
            ds = (int(full[0] // f), int(full[1] // f), full[2])
        elif sampling == "sequential":
            ds = (int(full[0] // f), full[1], full[2])
        else:
            raise ValueError("sampling must be 'disorder' or 'sequential'")
        if verbose:
            print(f"Spatial Level {sl + 1}/{n_spatial_levels} Downsampling by a factor of {f}")
        mps_res = centred_fft(centred_resize(centred_fft(mps_t), (ncoils, *ds)), inverse=True)
        ksp_res = centred_resize(ksp_t, (ncoils, *ds))
        A_res = _np_resize(A_np, (nshots, *ds[:2], 1))
        kgrid, rkgrid = compute_transform_grids_voxel(full, [1, 1, 1], ds)
        if temporal and sl == 0:
            t_est = _temporal_levels(ksp_res, mps_res, A_res, kgrid, rkgrid, t_est, nshots,
                                     n_temporal_levels, int(n_joint_iters * f), verbose,
                                     joint_kwargs)
        app = JointRecon(ksp_res, mps_res, A_res, kgrid, rkgrid, t0=t_est,
                         max_joint_iter=int(n_joint_iters * f), **joint_kwargs)
        _, t_est = app.run()
        del app
    if verbose:
        print("Final level of the pyramid - full resolution, image estimation only!")
    ksp_u = torch.fft.ifftshift(ksp_t, dim=AX3).contiguous()
    mps_u = torch.fft.ifftshift(mps_t, dim=AX3).contiguous()
    planes_u = np.fft.ifftshift(A_np.reshape(A_np.shape[:3]), axes=(-2, -1))
    max_norm = float(max_abs_image(hybrid_kspace(ksp_u)).item())
    ksp_u.div_(max_norm)
    kgrid, rkgrid = compute_transform_grids_voxel(full, [1, 1, 1], None)
    pb = SenseProblem(ksp_u, mps_u, planes_u, kgrid, rkgrid, t_est,
                      batch=joint_kwargs.get("batch"))
    x = pb.empty_image().zero_()
    cg_solve(pb, x, 100, 1e-6)
    x = torch.fft.fftshift(zxy_to_xyz(x) * max_norm, dim=AX3)
    return x.cpu().numpy(), t_est.cpu().numpy()


def _temporal_levels(ksp_res, mps_res, A_res, kgrid, rkgrid, t_est, nshots, levels, iters,
                     verbose, joint_kwargs):
    """Coarse-to-fine over motion-state bins (see pyramid_reconstruction); returns the per-shot
    transforms to start the per-shot level from."""
    for tl in range(levels - 1):
        tf = 2 ** (levels - tl - 1)
        if nshots % tf:
            continue
        if verbose:
            print(f"Temporal Level {tl + 1}/{levels}: {nshots // tf} motion states of {tf} shots")
        A_eff = aggregate_sampling_masks(A_res, tf) > 0
        T_eff = aggregate_transforms(t_est.cpu().numpy(), tf) / tf
        app = JointRecon(ksp_res, mps_res, A_eff, kgrid, rkgrid, t0=T_eff, max_joint_iter=iters,
                         **joint_kwargs)
        _, T_b = app.run()
        t_est = torch.repeat_interleave(T_b, tf, dim=0).contiguous()
        del app
    return t_est


def _np_resize(a, oshape):
    ishape = a.shape
    if tuple(ishape) == tuple(oshape):
        return a
    ish = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)]
    osh = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)]
    cp = [min(i - x, o - y) for i, x, o, y in zip(ishape, ish, oshape, osh)]
    out = np.zeros(oshape, dtype=a.dtype)
    out[tuple(slice(y, y + c) for y, c in zip(osh, cp))] = a[tuple(slice(x, x + c) for x, c in zip(ish, cp))]
    return out
