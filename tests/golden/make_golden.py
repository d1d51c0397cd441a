"""Generate the golden fixtures in this directory by running the reference itself.

The reference (chiew-group/motion-estimation) is pure Python on CuPy/SigPy and ships no tests,
golden vectors or fixtures.  This script imports its modules UNMODIFIED from a checkout of it
(given by --ref or the ME_REFERENCE environment variable), with the NumPy/SciPy stand-ins in ``_standins/`` in place of
cupy, cupyx.scipy.fft and sigpy, runs them on seeded small inputs on the CPU, and writes
inputs and outputs to ``*.npz`` files next to this script.  The fixtures are what the oracle
and the CUDA path are pinned against; this script is only needed to regenerate them (it is
never run by the tests, and the reference checkout does not exist on the GPU machines).

Usage:  python tests/golden/make_golden.py --ref <reference checkout> [--only name ...]
"""
import argparse
import hashlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(ref):
    sys.path.insert(0, str(HERE / "_standins"))
    sys.path.insert(0, str(ref))
    import image_estimation  # noqa: E402
    import joint_recon  # noqa: E402
    import pyramid  # noqa: E402
    import simulation  # noqa: E402
    import transform  # noqa: E402
    import transform_estimation  # noqa: E402
    import utils  # noqa: E402
    return dict(transform=transform, utils=utils, image_estimation=image_estimation,
                transform_estimation=transform_estimation, joint_recon=joint_recon,
                pyramid=pyramid, simulation=simulation)


def _cvol(rng, shape, dtype=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def _smooth_phantom(rng, shape, n_ell=4):
    """Small smooth complex test object (a few soft ellipsoids times a smooth phase)."""
    X, Y, Z = shape
    gx, gy, gz = np.meshgrid(np.linspace(-1, 1, X), np.linspace(-1, 1, Y), np.linspace(-1, 1, Z),
                             indexing="ij")
    img = np.zeros(shape, np.float64)
    for _ in range(n_ell):
        c = rng.uniform(-0.4, 0.4, 3)
        a = rng.uniform(0.2, 0.5, 3)
        r2 = ((gx - c[0]) / a[0]) ** 2 + ((gy - c[1]) / a[1]) ** 2 + ((gz - c[2]) / a[2]) ** 2
        img += rng.uniform(0.1, 1.0) / (1.0 + np.exp((r2 - 1.0) * 6.0))
    phase = 0.5 * gx + 0.3 * gy * gy - 0.2 * gz * gx
    return (img * np.exp(1j * phase)).astype(np.complex64)


def _coils(rng, shape, ncoils, unit_rss=False):
    """Gaussian-bump coil maps on a ring (not unit RSS unless asked), centred layout."""
    X, Y, Z = shape
    gx, gy, gz = np.meshgrid(np.linspace(-1, 1, X), np.linspace(-1, 1, Y), np.linspace(-1, 1, Z),
                             indexing="ij")
    maps = []
    for c in range(ncoils):
        ang = 2 * np.pi * c / ncoils
        cx, cy = 1.1 * np.cos(ang), 1.1 * np.sin(ang)
        mag = np.exp(-((gx - cx) ** 2 + (gy - cy) ** 2 + 0.5 * gz ** 2) / 1.2)
        maps.append(mag * np.exp(1j * (ang + 0.3 * gz)))
    maps = np.stack(maps)
    if unit_rss:
        maps /= np.sqrt(np.sum(np.abs(maps) ** 2, axis=0, keepdims=True))
    else:
        maps *= 1.6
    return maps.astype(np.complex64)


def _disorder_masks(sim, X, Y, tile, accel, nshots):
    """DISORDER masks [nshots, X, Y] exactly as simulation.py:385-402 builds them."""
    cfg = sim.DisorderConfig(max_line_number=Y - 1, max_partition_number=X - 1,
                             pat_lines_to_measure=Y // accel, block_lin=tile[1],
                             block_par=tile[0], seed=123456)
    order, (L, P) = sim.make_disorder_order(cfg)
    order = np.array(order, dtype=int)
    A = np.zeros((nshots, X, Y), dtype=bool)
    sps = order.shape[0] // nshots
    for s in range(nshots):
        A[s, order[s * sps:(s + 1) * sps, 1], order[s * sps:(s + 1) * sps, 0]] = True
    return order, (L, P), A


def _save(name, **arrays):
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"wrote {path.name}: {os.path.getsize(path) / 1024:.1f} KiB")


def make_grids(R):
    utils = R["utils"]
    out = {}
    cases = [((16, 12, 10), (1, 1, 1), None), ((9, 7, 5), (1, 1, 1), None),
             ((16, 12, 10), (1, 1, 1), (8, 6, 10)), ((12, 10, 8), (1.0, 1.25, 0.8), None)]
    for i, (shape, vox, ds) in enumerate(cases):
        kg, rk = utils.compute_transform_grids_voxel(shape, list(vox), ds, xp=np)
        out[f"c{i}_shape"] = np.array(shape)
        out[f"c{i}_vox"] = np.array(vox, dtype=np.float64)
        out[f"c{i}_ds"] = np.array(ds if ds is not None else shape)
        for a in "xyz":
            out[f"c{i}_k{a}"] = kg[a]
            out[f"c{i}_tan_{a}"] = rk["tan"][a]
            out[f"c{i}_sin_{a}"] = rk["sin"][a]
    out["ncases"] = np.array(len(cases))
    _save("grids", **out)


def make_transform(R):
    utils, tr = R["utils"], R["transform"]
    rng = np.random.default_rng(1001)
    out = {}
    cases = [((16, 12, 10), [1.3, -0.7, 0.4, 0.05, -0.08, 0.11]),
             ((9, 8, 7), [0.6, 1.1, -0.9, -0.04, 0.03, 0.09]),
             ((16, 12, 10), [-2.2, 3.1, 1.7, 0.14, -0.12, 0.13]),
             ((8, 6, 4), [0.0, 0.0, 0.0, 0.0, 0.0, 0.0])]
    for i, (shape, params) in enumerate(cases):
        kg, rk = utils.compute_transform_grids_voxel(shape, [1, 1, 1], xp=np)
        x = _cvol(rng, shape)
        p = np.array(params, dtype=np.float64)
        T = tr.RigidTransformCudaOptimzied(p, kg, rk)
        Ti = tr.RigidTransformCudaOptimzied(p, kg, rk, inverse=True)
        out[f"c{i}_x"] = x
        out[f"c{i}_params"] = p
        out[f"c{i}_apply"] = T.apply(x)
        out[f"c{i}_apply_inv"] = Ti.apply(x)
        out[f"c{i}_adjoint"] = T.adjoint(x)
        dT = tr.RigidTransformDerivativeCuda(shape, p, kg, rk)
        out[f"c{i}_deriv"] = np.stack([dT.apply(x, q) for q in range(6)])
    out["ncases"] = np.array(len(cases))
    _save("transform", **out)


def _small_problem(R, rng, shape, ncoils, nshots, unit_rss=False, tile=(4, 4), accel=1,
                   rot_deg=3.0, trans=1.0, noise=1e-3):
    """Centred (k-space, maps, masks, transforms, ground truth) as the reference's scripts
    build them (simulation.py:385-458)."""
    sim = R["simulation"]
    X, Y, Z = shape
    gt = _smooth_phantom(rng, shape)
    mps = _coils(rng, shape, ncoils, unit_rss)
    _, _, A = _disorder_masks(sim, X, Y, tile, accel, nshots)
    A = A[..., None]
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-trans, trans, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-rot_deg, rot_deg, (nshots, 3)))
    ksp = sim.generate_corrupted_kspace(gt, mps, A, t)
    if noise > 0:
        std = noise * np.max(np.abs(ksp))
        ksp = ksp + (std * (rng.standard_normal(ksp.shape) + 1j * rng.standard_normal(ksp.shape)))
    return gt, mps, A, t, ksp.astype(np.complex64)


def make_forward(R):
    """generate_corrupted_kspace (simulation.py:65-85) on a small DISORDER case."""
    rng = np.random.default_rng(2002)
    gt, mps, A, t, ksp = _small_problem(R, rng, (16, 12, 10), 4, 4, noise=0.0)
    _save("forward", gt=gt, mps=mps, mask=A, transforms=t, ksp=ksp)


def _uncentred(ksp, mps, A):
    ax = (-3, -2, -1)
    kspu = np.fft.ifftshift(ksp, axes=ax).astype(np.complex64)
    mpsu = np.fft.ifftshift(mps, axes=ax).astype(np.complex64)
    Au = np.fft.ifftshift(A, axes=ax)
    return kspu, mpsu, Au


def make_cg(R):
    """estimate_image_cg (image_estimation.py:10-165) on uncentred inputs, as JointRecon calls it."""
    ie, utils = R["image_estimation"], R["utils"]
    out = {}
    rng = np.random.default_rng(3003)
    for i, (unit, iters, x0rand) in enumerate([(False, 5, False), (False, 4, True), (True, 6, False)]):
        shape = (16, 12, 10)
        gt, mps, A, t, ksp = _small_problem(R, rng, shape, 4, 4, unit_rss=unit)
        kspu, mpsu, Au = _uncentred(ksp, mps, A)
        kspu = kspu / np.max(np.abs(np.fft.ifftn(kspu, axes=(-3, -2, -1), norm="ortho")))
        kspu = kspu.astype(np.complex64)
        P = 1 / (np.sum(np.abs(mpsu) ** 2, axis=0) + 1e-3)
        M = np.sum(np.abs(mpsu) ** 2, axis=0) > 0.1
        kg, rk = utils.compute_transform_grids_voxel(shape, [1, 1, 1], xp=np)
        x0 = _cvol(rng, shape) * 0.1 if x0rand else None
        tt = t if i != 2 else np.zeros_like(t)
        x = ie.estimate_image_cg(kspu, mpsu, Au, tt, kg, rk, P, M, x0=x0, max_iter=iters,
                                 show_pbar=False)
        out[f"c{i}_ksp"] = kspu
        out[f"c{i}_mps"] = mpsu
        out[f"c{i}_mask"] = Au
        out[f"c{i}_transforms"] = tt
        out[f"c{i}_P"] = P
        out[f"c{i}_M"] = M
        out[f"c{i}_x0"] = x0 if x0 is not None else np.zeros(shape, np.complex64)
        out[f"c{i}_max_iter"] = np.array(iters)
        out[f"c{i}_x"] = x
    out["ncases"] = np.array(3)
    _save("cg", **out)


def make_lm(R):
    """One estimate_transform call (transform_estimation.py:7-151) with a fixed image."""
    te, ie, utils = R["transform_estimation"], R["image_estimation"], R["utils"]
    rng = np.random.default_rng(4004)
    shape = (16, 12, 10)
    gt, mps, A, t_true, ksp = _small_problem(R, rng, shape, 4, 4)
    kspu, mpsu, Au = _uncentred(ksp, mps, A)
    kspu = (kspu / np.max(np.abs(np.fft.ifftn(kspu, axes=(-3, -2, -1), norm="ortho")))).astype(
        np.complex64)
    kg, rk = utils.compute_transform_grids_voxel(shape, [1, 1, 1], xp=np)
    P = 1 / (np.sum(np.abs(mpsu) ** 2, axis=0) + 1e-3)
    M = np.sum(np.abs(mpsu) ** 2, axis=0) > 0.1
    t0 = t_true + rng.normal(0, 0.3, t_true.shape) * np.array([1, 1, 1, 0.02, 0.02, 0.02])
    t0[0] = 0.0
    img = ie.estimate_image_cg(kspu, mpsu, Au, np.zeros_like(t0), kg, rk, P, M, max_iter=4,
                               show_pbar=False)
    img = img.astype(np.complex64)
    out = dict(ksp=kspu, mps=mpsu, mask=Au)
    # Case 2 starts far from the truth with the true image, so that some shots' steps are
    # rejected (e1 >= e0) and their damping grows (transform_estimation.py:138-144).
    img_true = np.fft.ifftshift(gt).astype(np.complex64)
    rng_far = np.random.default_rng(4245)
    t_far = t_true + 12.0 * np.array([[1, 1, 1, 0.05, 0.05, 0.05]]) * rng_far.standard_normal(
        t_true.shape)
    cases = [(img, t0, np.ones(4)), (img, t0, np.array([1e-4, 3.0, 0.5, 1e3])),
             (img_true, t_far, np.full(4, 1e-4))]
    for i, (image, tstart, damp0) in enumerate(cases):
        t = tstart.copy()
        damp = damp0.copy()
        flags = np.zeros(4, dtype=bool)
        res = np.zeros_like(kspu)
        part = np.zeros((6,) + kspu.shape, dtype=kspu.dtype)
        g = np.zeros(6)
        H = np.zeros((6, 6))
        new = te.estimate_transform(kspu, mpsu, Au, image, kg, rk, damp, flags, res, part, g, H,
                                    transforms=t, max_iter=1)
        out[f"c{i}_image"] = image
        out[f"c{i}_t0"] = tstart
        out[f"c{i}_damp0"] = damp0
        out[f"c{i}_t"] = t
        out[f"c{i}_damp"] = damp
        out[f"c{i}_flags"] = flags
        out[f"c{i}_image_out"] = new
    out["ncases"] = np.array(len(cases))
    _save("lm", **out)


def make_lm_ga(R):
    """estimate_transform with use_ga=True (transform_estimation.py:75-121) on the LM fixture's
    problem, from a start near the truth (small steps) and one far from it."""
    te = R["transform_estimation"]
    d = np.load(HERE / "lm.npz")
    kspu, mpsu, Au = d["ksp"], d["mps"], d["mask"]
    kg, rk = R["utils"].compute_transform_grids_voxel(kspu.shape[1:], [1, 1, 1], xp=np)
    out = {}
    for i in range(int(d["ncases"])):
        t = d[f"c{i}_t0"].copy()
        damp = d[f"c{i}_damp0"].copy()
        flags = np.zeros(4, dtype=bool)
        res = np.zeros_like(kspu)
        part = np.zeros((6,) + kspu.shape, dtype=kspu.dtype)
        new = te.estimate_transform(kspu, mpsu, Au, d[f"c{i}_image"], kg, rk, damp, flags, res,
                                    part, np.zeros(6), np.zeros((6, 6)), transforms=t,
                                    max_iter=1, use_ga=True)
        out[f"c{i}_t"] = t
        out[f"c{i}_damp"] = damp
        out[f"c{i}_flags"] = flags
        out[f"c{i}_image_out"] = new
    out["ncases"] = np.array(int(d["ncases"]))
    _save("lm_ga", **out)


def make_preprocess(R):
    """coil_compression (coil_compression.py:6-46) and rx_espirit_3d (espirit.py:46-239) on a
    small multi-coil phantom: the maps from the reference's ESPIRiT on the centre of its
    k-space, and the compressed maps and k-space."""
    sys.path.insert(0, str(R["_ref"]))
    import coil_compression as cc
    import espirit as es
    rng = np.random.default_rng(8008)
    shape = (16, 16, 12)
    gt = _smooth_phantom(rng, shape)
    mps = _coils(rng, shape, 6, unit_rss=False)
    ksp = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(mps * gt, axes=(-3, -2, -1)),
                                      axes=(-3, -2, -1), norm="ortho"), axes=(-3, -2, -1))
    ksp = (ksp + 1e-3 * np.abs(ksp).max() * (rng.standard_normal(ksp.shape)
                                             + 1j * rng.standard_normal(ksp.shape))
           ).astype(np.complex64)
    calib = np.ascontiguousarray(np.moveaxis(ksp[:, 4:12, 4:12, 2:10], 0, -1))  # [8, 8, 8, C]
    sens = es.rx_espirit_3d(calib, shape, kernel_size=(3, 3, 3), eig_thresh=0.02,
                            mask_thresh=0.99)
    cc_mps, cc_ksp = cc.coil_compression(mps, ksp, perc=0.95)
    _save("preprocess", mps=mps, ksp=ksp, calib=calib, sens=np.asarray(sens).astype(np.complex64),
          cc_mps=np.asarray(cc_mps).astype(np.complex64),
          cc_ksp=np.asarray(cc_ksp).astype(np.complex64))


def make_joint(R):
    """JointRecon (joint_recon.py:10-115): 3 outer iterations on a small DISORDER case."""
    jr, utils = R["joint_recon"], R["utils"]
    rng = np.random.default_rng(5005)
    shape = (16, 12, 10)
    gt, mps, A, t_true, ksp = _small_problem(R, rng, shape, 4, 4)
    kg, rk = utils.compute_transform_grids_voxel(shape, [1, 1, 1], xp=np)
    app = jr.JointRecon(ksp, mps, A, kg, rk, t0=None, max_cg_iter=3, max_nm_iter=1,
                        max_joint_iter=3, xp=np)
    x, t = app.run()
    _save("joint", ksp=ksp, mps=mps, mask=A, t_true=t_true, gt=gt, max_cg_iter=np.array(3),
          max_nm_iter=np.array(1), max_joint_iter=np.array(3), x=x, t=np.asarray(t),
          objective_history=np.asarray(app.objective_history),
          transform_history=np.asarray(app.transform_history))


def make_pyramid(R):
    """pyramid_reconstruction (pyramid.py:24-118) with 3 spatial levels on 16x16x8."""
    pyr = R["pyramid"]
    rng = np.random.default_rng(6006)
    shape = (16, 16, 8)
    gt, mps, A, t_true, ksp = _small_problem(R, rng, shape, 4, 4)
    save = Path("/tmp/_golden_pyramid")
    save.mkdir(exist_ok=True)
    x, t = pyr.pyramid_reconstruction(ksp, mps, A, 4, n_spatial_levels=3, n_joint_iters=2,
                                      save_path=save)
    _save("pyramid", ksp=ksp, mps=mps, mask=A, n_joint_iters=np.array(2), x=x, t=np.asarray(t))


def _ellipsoid_phantom(rng, shape, n_ell):
    """Centred complex64 phantom: n random solid ellipsoids with intensities U[0.1, 1] times
    exp(i * a random degree-2 polynomial) over [-1, 1]^3."""
    X, Y, Z = shape
    gx, gy, gz = np.meshgrid(np.linspace(-1, 1, X), np.linspace(-1, 1, Y), np.linspace(-1, 1, Z),
                             indexing="ij")
    mag = np.zeros(shape)
    for _ in range(n_ell):
        c = rng.uniform(-0.45, 0.45, 3)
        a = rng.uniform(0.08, 0.45, 3)
        ang = rng.uniform(0, np.pi)
        u = ((gx - c[0]) * np.cos(ang) + (gy - c[1]) * np.sin(ang)) / a[0]
        v = (-(gx - c[0]) * np.sin(ang) + (gy - c[1]) * np.cos(ang)) / a[1]
        w = (gz - c[2]) / a[2]
        mag += rng.uniform(0.1, 1.0) * ((u * u + v * v + w * w) <= 1.0)
    q = rng.normal(0, 0.6, 10)
    ph = (q[0] * gx + q[1] * gy + q[2] * gz + q[3] * gx * gx + q[4] * gy * gy + q[5] * gz * gz
          + q[6] * gx * gy + q[7] * gx * gz + q[8] * gy * gz + q[9])
    return (mag * np.exp(1j * ph)).astype(np.complex64)


def make_config0(R):
    """JointRecon on the small CPU workload (64x64x48, 8 coils, 16 shots DISORDER 4x4, 10 outer
    iterations of 5 CG + 1 LM), with the inputs of config_inputs.py; the reference's own run
    time here is recorded beside its outputs."""
    import time

    sys.path.insert(0, str(HERE))
    import config_inputs as ci
    jr, sim, utils = R["joint_recon"], R["simulation"], R["utils"]
    rng = np.random.default_rng(7007)
    X, Y, Z = ci.SHAPE
    S = ci.NSHOTS
    gt = _ellipsoid_phantom(rng, ci.SHAPE, 10)
    mps = ci.coil_maps()
    _, _, A = _disorder_masks(sim, X, Y, ci.TILE, ci.ACCEL, S)
    A = A[..., None]
    t_true = np.zeros((S, 6))
    t_true[:, :3] = rng.uniform(-2.0, 2.0, (S, 3))
    t_true[:, 3:] = np.deg2rad(rng.uniform(-3.0, 3.0, (S, 3)))
    ksp = sim.generate_corrupted_kspace(gt, mps, A, t_true)
    std = 1e-3 * np.max(np.abs(ksp))
    ksp = (ksp + std * (rng.standard_normal(ksp.shape) + 1j * rng.standard_normal(ksp.shape))
           ).astype(np.complex64)
    q, scale = ci.quantise_kspace(ksp)
    ksp_in = ci.dequantise_kspace(q, scale)
    kg, rk = utils.compute_transform_grids_voxel(ci.SHAPE, [1, 1, 1], xp=np)
    t0 = time.perf_counter()
    app = jr.JointRecon(ksp_in, mps, A, kg, rk, t0=None, max_cg_iter=ci.CG_ITERS, max_nm_iter=1,
                        max_joint_iter=ci.OUTER_ITERS, xp=np)
    x, t = app.run()
    secs = time.perf_counter() - t0
    print(f"config0: reference JointRecon took {secs:.1f} s on {os.cpu_count()} cores")
    _save("config0", ksp_f16=q, ksp_scale=np.array(scale), mps_sha256=ci.digest(mps),
          mask_packed=np.packbits(A.ravel()), t_true=t_true, x=x.astype(np.complex64),
          t=np.asarray(t), transform_history=np.asarray(app.transform_history),
          objective_history=np.asarray(app.objective_history), damp=np.asarray(app.damp),
          flags=np.asarray(app.convergence_flags), reference_seconds=np.array(secs),
          reference_cores=np.array(os.cpu_count()))


def make_config0_pyramid(R):
    """pyramid_reconstruction (pyramid.py:24-118) on the 64x64x48 / 8-coil / 16-shot inputs of
    config_inputs.py: 3 spatial levels with n_joint_iters=2 (8 outer iterations at x0.25, 4 at
    x0.5, then 100 CG iterations at full size)."""
    import time

    sys.path.insert(0, str(HERE))
    import config_inputs as ci
    pyr = R["pyramid"]
    ksp, mps, masks, _ = ci.load(HERE)
    save = Path("/tmp/_golden_pyramid0")
    save.mkdir(exist_ok=True)
    t0 = time.perf_counter()
    x, t = pyr.pyramid_reconstruction(ksp, mps, masks, ci.NSHOTS, n_spatial_levels=3,
                                      n_joint_iters=2, save_path=save)
    secs = time.perf_counter() - t0
    print(f"config0 pyramid: reference took {secs:.1f} s")
    _save("config0_pyramid", x=np.asarray(x).astype(np.complex64), t=np.asarray(t),
          reference_seconds=np.array(secs))


# (X partitions, Y lines, tile (par, lin), accel, nshots used by the workload)
DISORDER_CASES = [
    (16, 12, (4, 4), 1, 4),
    (64, 64, (4, 4), 1, 16),
    (256, 224, (16, 16), 2, 64),
    (128, 128, (8, 8), 1, 32),
    (256, 256, (16, 16), 2, 64),
    (96, 96, (8, 8), 1, 64),
    (192, 192, (16, 16), 2, 128),
    (64, 64, (8, 8), 2, 32),
]


def make_disorder(R):
    """DISORDER reorder (simulation.py:201-245) and shot binning (simulation.py:397-402)."""
    sim = R["simulation"]
    out = {}
    for i, (X, Y, tile, accel, nshots) in enumerate(DISORDER_CASES):
        order, (L, P), A = _disorder_masks(sim, X, Y, tile, accel, nshots)
        out[f"c{i}_case"] = np.array([X, Y, tile[0], tile[1], accel, nshots])
        out[f"c{i}_order"] = order.astype(np.int16)
        out[f"c{i}_LP"] = np.array([L, P])
        out[f"c{i}_mask_sha256"] = np.frombuffer(
            hashlib.sha256(np.ascontiguousarray(A).tobytes()).digest(), dtype=np.uint8)
        if X * Y * nshots <= 64 * 64 * 16:
            out[f"c{i}_mask_packed"] = np.packbits(A.ravel())
    out["ncases"] = np.array(len(DISORDER_CASES))
    _save("disorder", **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ME_REFERENCE"),
                    required="ME_REFERENCE" not in os.environ,
                    help="path of the reference checkout (or set ME_REFERENCE)")
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    R = _import_reference(args.ref)
    R["_ref"] = args.ref
    steps = dict(grids=make_grids, transform=make_transform, forward=make_forward, cg=make_cg,
                 lm=make_lm, joint=make_joint, pyramid=make_pyramid, disorder=make_disorder,
                 config0=make_config0, lm_ga=make_lm_ga, preprocess=make_preprocess,
                 config0_pyramid=make_config0_pyramid)
    for name, fn in steps.items():
        if args.only and name not in args.only:
            continue
        fn(R)


if __name__ == "__main__":
    main()
