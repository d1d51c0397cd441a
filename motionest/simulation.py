"""Seeded synthetic inputs and the motion-corrupted forward model.

generate_corrupted_kspace keeps the reference's interface (simulation.py:65-85): centred
image, maps and masks in, centred k-space out, y = fftshift sum_s M_s F (C T_s x).  It runs on
libmotionest's kernels: the shots' samples are computed in hybrid space by the SENSE forward
kernel, scattered (duplicates across shots add up, as `ksp += temp` does), and FFT'd along z.

The phantom / coil / motion generators produce the workloads the benchmarks are quoted on:
a sum of random soft ellipsoids with intensities U[0.1, 1] times a smooth degree-2 polynomial
phase, Gaussian-bump coils on a ring normalised to unit root-sum-of-squares, and uniform random
motion, a random walk with abrupt jumps, or continuous intra-shot motion.
"""
import numpy as np
import torch

from . import _lib
from ._arrays import to_device
from .image_estimation import _host_mask
from .problem import SenseProblem, fft_axes, xyz_to_zxy
from .sampling import disorder_masks
from .utils import compute_transform_grids_voxel

AX3 = (-3, -2, -1)


def _axes(shape, device):
    X, Y, Z = shape
    gx = torch.linspace(-1, 1, X, device=device, dtype=torch.float32).view(X, 1, 1)
    gy = torch.linspace(-1, 1, Y, device=device, dtype=torch.float32).view(1, Y, 1)
    gz = torch.linspace(-1, 1, Z, device=device, dtype=torch.float32).view(1, 1, Z)
    return gx, gy, gz


def phantom(shape, n_ellipsoids=10, seed=0, device=None):
    """Centred complex64 phantom: sum of n random ellipsoids (intensity U[0.1, 1]) times
    exp(i * random degree-2 polynomial)."""
    device = device or ("cuda" if torch.cuda.is_available() else "cpu")
    rng = np.random.default_rng(seed)
    gx, gy, gz = _axes(shape, device)
    mag = torch.zeros(shape, dtype=torch.float32, device=device)
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.45, 0.45, 3)
        a = rng.uniform(0.08, 0.45, 3)
        ang = rng.uniform(0, np.pi)
        ca, sa = float(np.cos(ang)), float(np.sin(ang))
        u = ((gx - c[0]) * ca + (gy - c[1]) * sa) / a[0]
        v = (-(gx - c[0]) * sa + (gy - c[1]) * ca) / a[1]
        w = (gz - c[2]) / a[2]
        inside = (u * u + v * v + w * w) <= 1.0
        mag = mag + float(rng.uniform(0.1, 1.0)) * inside
    q = rng.normal(0, 0.6, 10)
    ph = (q[0] * gx + q[1] * gy + q[2] * gz + q[3] * gx * gx + q[4] * gy * gy + q[5] * gz * gz
          + q[6] * gx * gy + q[7] * gx * gz + q[8] * gy * gz + q[9])
    return torch.polar(mag, ph).to(torch.complex64)


def coil_maps(shape, ncoils, seed=0, unit_rss=True, device=None):
    """Centred [C, X, Y, Z] Gaussian-bump sensitivities centred on a ring in the x-y plane with
    a ring-angle phase; normalised to unit root-sum-of-squares unless unit_rss=False (then
    P and M of the reconstruction are no longer trivial)."""
    device = device or ("cuda" if torch.cuda.is_available() else "cpu")
    rng = np.random.default_rng(seed + 7919)
    gx, gy, gz = _axes(shape, device)
    maps = []
    for c in range(ncoils):
        ang = 2 * np.pi * c / ncoils + rng.uniform(-0.1, 0.1)
        ring = 1.2 if ncoils <= 16 else (1.2 if c % 2 == 0 else 0.9)
        cx, cy = ring * np.cos(ang), ring * np.sin(ang)
        cz = rng.uniform(-0.5, 0.5)
        width = rng.uniform(0.7, 1.1)
        mag = torch.exp(-((gx - cx) ** 2 + (gy - cy) ** 2 + 0.6 * (gz - cz) ** 2) / width)
        maps.append(torch.polar(mag, torch.full_like(mag, float(ang)) + 0.4 * gz))
    m = torch.stack(maps)
    if unit_rss:
        m = m / torch.sqrt(torch.sum(m.abs() ** 2, dim=0, keepdim=True))
    else:
        m = m * 1.6
    return m.to(torch.complex64)


def motion_uniform(nshots, rot_deg=3.0, trans_vox=2.0, seed=0):
    """[S, 6] float64: translations U[-trans, trans] voxels, rotations U[-rot, rot] degrees
    (in radians)."""
    rng = np.random.default_rng(seed + 104729)
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-trans_vox, trans_vox, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-rot_deg, rot_deg, (nshots, 3)))
    return t


def motion_random_walk(nshots, step_deg=0.3, step_vox=0.3, jumps=3, jump_deg=8.0, jump_vox=6.0,
                       seed=0):
    """[S, 6] float64: a random walk (Gaussian steps) plus `jumps` abrupt jumps of up to
    jump_deg / jump_vox, centred to zero mean."""
    rng = np.random.default_rng(seed + 1299709)
    steps = np.zeros((nshots, 6))
    steps[:, :3] = rng.normal(0, step_vox, (nshots, 3))
    steps[:, 3:] = rng.normal(0, step_deg, (nshots, 3))
    for s in rng.choice(np.arange(1, nshots), size=min(jumps, nshots - 1), replace=False):
        steps[s, :3] += rng.uniform(-jump_vox, jump_vox, 3)
        steps[s, 3:] += rng.uniform(-jump_deg, jump_deg, 3)
    t = np.cumsum(steps, axis=0)
    t -= t.mean(axis=0, keepdims=True)
    t[:, 3:] = np.deg2rad(t[:, 3:])
    return t


def motion_continuous(nshots, segments=4, drift_deg=2.0, drift_vox=2.0, rot_deg=3.0,
                      trans_vox=2.0, seed=0):
    """[nshots * segments, 6] float64 per-segment transforms of continuous intra-shot motion:
    shot s has a pose drawn like motion_uniform (U[-rot_deg, rot_deg] degrees, U[-trans_vox,
    trans_vox] voxels) and drifts linearly through it over its `segments` segments by a seeded
    total of up to drift_deg / drift_vox per parameter (segment k sits at pose + drift *
    (k / (segments - 1) - 1/2)); centred to zero mean over all segments."""
    rng = np.random.default_rng(seed + 15485863)
    base = motion_uniform(nshots, rot_deg, trans_vox, seed)
    drift = np.zeros((nshots, 6))
    drift[:, :3] = rng.uniform(-drift_vox, drift_vox, (nshots, 3))
    drift[:, 3:] = np.deg2rad(rng.uniform(-drift_deg, drift_deg, (nshots, 3)))
    frac = (np.arange(segments) / max(segments - 1, 1) - 0.5)[None, :, None]
    t = (base[:, None, :] + drift[:, None, :] * frac).reshape(nshots * segments, 6)
    return t - t.mean(axis=0, keepdims=True)


def generate_corrupted_kspace(gt_img, mps, A, transforms):
    """y = fftshift sum_s M_s F (C T_s ifftshift(x)) (simulation.py:65-85), on the GPU.
    Returns a complex64 CUDA tensor [C, X, Y, Z] (centred)."""
    _lib.require_cuda()
    gt = torch.fft.ifftshift(to_device(gt_img, torch.complex64)).contiguous()
    mps_u = torch.fft.ifftshift(to_device(mps, torch.complex64), dim=AX3).contiguous()
    planes = np.fft.ifftshift(_host_mask(A).reshape(np.shape(A)[:3]), axes=(-2, -1))
    t = torch.as_tensor(np.asarray(transforms if not isinstance(transforms, torch.Tensor)
                                   else transforms.cpu(), dtype=np.float64)).cuda()
    kgrid, rkgrid = compute_transform_grids_voxel(tuple(gt.shape), [1, 1, 1])
    pb = SenseProblem(None, mps_u, planes, kgrid, rkgrid, t)
    K = pb.forward(xyz_to_zxy(gt), t)
    C = mps_u.shape[0]
    ksp_h = torch.zeros((C,) + tuple(gt.shape), dtype=torch.complex64, device=gt.device)
    pb.scatter(K, ksp_h)
    ksp = fft_axes(ksp_h, (2,), inverse=False)
    return torch.fft.fftshift(ksp, dim=AX3)


def add_noise(ksp, rel_sigma=1e-3, seed=0):
    """ksp + complex Gaussian noise of std rel_sigma * max|ksp| per real component."""
    g = torch.Generator(device=ksp.device).manual_seed(int(seed))
    std = float(rel_sigma * ksp.abs().max().item())
    n = torch.randn(ksp.shape + (2,), generator=g, device=ksp.device, dtype=torch.float32)
    return ksp + std * torch.view_as_complex(n)


def make_workload(shape, ncoils, nshots, tile, accel, motion="uniform", n_ellipsoids=10, seed=0,
                  noise=1e-3, unit_rss=True, rot_deg=3.0, trans_vox=2.0, segments=4):
    """Seeded synthetic reconstruction problem: dict with centred gt, mps, masks (host), t, ksp.

    motion: 'uniform' (U[-rot_deg, rot_deg] / U[-trans_vox, trans_vox] per shot), 'walk' (random
    walk plus jumps), or 'continuous': intra-shot motion with `segments` states per shot, as the
    reference's --continuous experiments corrupt the data (simulation.py:372-373,404-410): the
    k-space is generated with the DISORDER order binned into nshots * segments corruption
    states, each with its own transform (motion_continuous), while the reconstruction masks bin
    it into nshots.  Then t holds the per-segment transforms and `masks_corruption` the
    corruption masks."""
    X, Y, Z = shape
    gt = phantom(shape, n_ellipsoids, seed)
    mps = coil_maps(shape, ncoils, seed, unit_rss)
    masks = disorder_masks(X, Y, tile, accel, nshots)
    extra = {}
    if motion == "uniform":
        t = motion_uniform(nshots, rot_deg, trans_vox, seed)
        corrupt = masks
    elif motion == "continuous":
        t = motion_continuous(nshots, segments, 2.0, 2.0, rot_deg, trans_vox, seed)
        corrupt = disorder_masks(X, Y, tile, accel, nshots * segments)
        extra["masks_corruption"] = corrupt
    else:
        t = motion_random_walk(nshots, seed=seed)
        corrupt = masks
    ksp = generate_corrupted_kspace(gt, mps, corrupt, t)
    if noise > 0:
        ksp = add_noise(ksp, noise, seed)
    return dict(gt=gt, mps=mps, masks=masks, t=t, ksp=ksp, **extra)
