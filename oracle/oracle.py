"""CPU oracle for the SAMER/DISORDER joint reconstruction path (TEST INFRASTRUCTURE ONLY).

A plain NumPy/SciPy restatement of the reference's algorithm (chiew-group/motion-estimation),
following its op sequence step by step: full 3-D FFTs per coil, per-shot Python loops, the
same precision casts.  Every function cites the reference file:line it restates.

Who may use this module: the tests under ``tests/`` (as the checker), ``__graft_entry__.smoke()``
(as the checker) and ``bench.py``'s CPU-baseline leg (as the timed CPU implementation).  The
``motionest`` package never imports it; its CUDA path fails loudly when the extension is missing.

Pinning: the reference ships no golden vectors or tests.  This oracle is pinned against
fixtures produced by running the reference's own modules, unmodified, on CPU
(``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks it against every one.

Precision: ``dtype=np.complex64`` reproduces the reference's mixed precision (complex64
volumes, complex64 shear chirps, complex128 translation ramps cast back on multiply).
``dtype=np.complex128`` is the FP64 oracle: every volume, factor and FFT in double.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

AX3 = (-3, -2, -1)


class Oracle:
    """Holds the precision and FFT thread count; all the reference's operations hang off it."""

    def __init__(self, dtype=np.complex64, workers=1):
        self.dtype = np.dtype(dtype)
        self.workers = workers
        self.fp64 = self.dtype == np.complex128

    # ------------------------------------------------------------------ FFT helpers
    def fft(self, a, axes):
        return sfft.fftn(a, axes=axes, norm="ortho", workers=self.workers)

    def ifft(self, a, axes):
        return sfft.ifftn(a, axes=axes, norm="ortho", workers=self.workers)

    def _shear(self, arr, v, axis):
        """One shear: FFT along `axis` -> multiply by v -> IFFT (transform.py:278-285)."""
        arr = self.fft(arr, (axis,))
        arr *= v
        return self.ifft(arr, (axis,))

    # ------------------------------------------------------------------ factors
    def shear_factors(self, theta, rk_tan, rk_sin, conj=False):
        """vtan = exp(i tan(theta/2) rk_tan), vsin = exp(-i sin(theta) rk_sin).

        transform.py:275-276 forms them in complex64 (apply); transform.py:344-345 uses the
        complex128 helper transform.py:5-14 and conjugates (adjoint)."""
        if self.fp64 or conj:
            vt = np.exp(1j * np.tan(theta / 2) * rk_tan)
            vs = np.exp(-1j * np.sin(theta) * rk_sin)
            if not self.fp64:
                # complex128 factor multiplied into a complex64 array in place: computed in
                # complex128 and cast back, which `arr *= v` reproduces.
                pass
        else:
            vt = np.exp(1j * np.tan(theta / 2) * rk_tan, dtype=np.complex64)
            vs = np.exp(-1j * np.sin(theta) * rk_sin, dtype=np.complex64)
        if conj:
            vt, vs = vt.conj(), vs.conj()
        return vt, vs

    @staticmethod
    def translation_factor(kgrid, q, conj=False):
        """U = exp(-i (q1 kx + q2 ky + q3 kz)), complex128 (transform.py:257-261)."""
        u = np.exp(-1j * (q[0] * kgrid["x"] + q[1] * kgrid["y"] + q[2] * kgrid["z"]))
        return u.conj() if conj else u

    @staticmethod
    def _steps(params, rkgrid):
        """(theta, rk_tan, rk_sin, tan_axis, sin_axis) per rotation axis (transform.py:267-271)."""
        t1, t2, t3 = params[3], params[4], params[5]
        return [
            (t1, rkgrid["tan"]["x"], rkgrid["sin"]["x"], 1, 2),
            (t2, rkgrid["tan"]["y"], rkgrid["sin"]["y"], 2, 0),
            (t3, rkgrid["tan"]["z"], rkgrid["sin"]["z"], 0, 1),
        ]

    # ------------------------------------------------------------------ operators
    def rigid_apply(self, x, params, kgrid, rkgrid, inverse=False):
        """T x = Tr . Rz . Ry . Rx x (transform.py:263-318)."""
        arr = np.array(x, dtype=self.dtype, copy=True)
        for theta, rk_t, rk_s, ax_t, ax_s in self._steps(params, rkgrid):
            vt, vs = self.shear_factors(theta, rk_t, rk_s)
            arr = self._shear(arr, vt, ax_t)
            arr = self._shear(arr, vs, ax_s)
            arr = self._shear(arr, vt, ax_t)
        U = self.translation_factor(kgrid, params[:3], conj=inverse)
        arr = self.fft(arr, AX3)
        arr *= U
        return self.ifft(arr, AX3)

    def rigid_adjoint(self, x, params, kgrid, rkgrid):
        """T^H x = Rx^H Ry^H Rz^H Tr^H x (transform.py:320-377)."""
        arr = np.array(x, dtype=self.dtype, copy=True)
        U = self.translation_factor(kgrid, params[:3], conj=True)
        arr = self.fft(arr, AX3)
        arr *= U
        arr = self.ifft(arr, AX3)
        for theta, rk_t, rk_s, ax_t, ax_s in self._steps(params, rkgrid)[::-1]:
            vt, vs = self.shear_factors(theta, rk_t, rk_s, conj=True)
            arr = self._shear(arr, vt, ax_t)
            arr = self._shear(arr, vs, ax_s)
            arr = self._shear(arr, vt, ax_t)
        return arr

    def _rotation(self, arr, theta, rk_t, rk_s, ax_t, ax_s):
        """transform.py:392-409."""
        vt, vs = self.shear_factors(theta, rk_t, rk_s)
        arr = self._shear(arr, vt, ax_t)
        arr = self._shear(arr, vs, ax_s)
        return self._shear(arr, vt, ax_t)

    def _rotation_derivative(self, arr, theta, rk_t, rk_s, ax_t, ax_s):
        """Product rule over the three shears (transform.py:433-474)."""
        vt, vs = self.shear_factors(theta, rk_t, rk_s)
        dvt = 1j * ((1 + np.tan(theta / 2) ** 2) / 2) * rk_t * vt
        dvs = -1j * np.cos(theta) * rk_s * vs
        if not self.fp64:
            dvt, dvs = dvt.astype(np.complex64), dvs.astype(np.complex64)
        f = self.fft(arr, (ax_t,))
        s1 = f * dvt
        s1 = self.ifft(s1, (ax_t,))
        s1 = self.fft(s1, (ax_s,))
        s1 *= vs
        s1 = self.ifft(s1, (ax_s,))
        s1 = self.fft(s1, (ax_t,))
        s1 *= vt
        s2 = f * vt
        s2 = self.ifft(s2, (ax_t,))
        s2 = self.fft(s2, (ax_s,))
        s2 *= dvs
        s2 = self.ifft(s2, (ax_s,))
        s2 = self.fft(s2, (ax_t,))
        s2 *= vt
        s3 = f * vt
        s3 = self.ifft(s3, (ax_t,))
        s3 = self.fft(s3, (ax_s,))
        s3 *= vs
        s3 = self.ifft(s3, (ax_s,))
        s3 = self.fft(s3, (ax_t,))
        s3 *= dvt
        out = s1 + s2 + s3
        return self.ifft(out, (ax_t,))

    def _translation(self, arr, kgrid, q, p_idx=None):
        """transform.py:411-431: 3-D FFT, multiply by U (or -i k_p U), 3-D IFFT."""
        U = self.translation_factor(kgrid, q)
        if p_idx is not None:
            U = -1j * kgrid["xyz"[p_idx]] * U
        arr = self.fft(arr, AX3)
        arr *= U
        return self.ifft(arr, AX3)

    def rigid_derivative(self, x, params, p_idx, kgrid, rkgrid, mode="reference"):
        """Partial derivative of the rigid transform with respect to params[p_idx].

        mode='reference' restates RigidTransformDerivativeCuda.apply (transform.py:476-504),
        which differentiates Tr . Rx . Ry . Rz (z applied first).  mode='exact' differentiates
        the operator that rigid_apply implements, Tr . Rz . Ry . Rx (x applied first).
        p_idx outside 0..5 returns a copy of the input, as transform.py:480-504 does."""
        arr = np.array(x, dtype=self.dtype, copy=True)
        st = self._steps(params, rkgrid)
        q = params[:3]
        order = [2, 1, 0] if mode == "reference" else [0, 1, 2]
        if p_idx not in range(6):
            return arr
        rot_p = p_idx - 3
        for a in order:
            theta, rk_t, rk_s, ax_t, ax_s = st[a]
            if a == rot_p:
                arr = self._rotation_derivative(arr, theta, rk_t, rk_s, ax_t, ax_s)
            else:
                arr = self._rotation(arr, theta, rk_t, rk_s, ax_t, ax_s)
        return self._translation(arr, kgrid, q, p_idx if p_idx < 3 else None)

    # ------------------------------------------------------------------ SENSE pieces
    def vdot_real(self, a, b):
        v = np.vdot(a, b).real
        return v

    def cg_rhs(self, ksp, mps, shot_mask, transforms, kgrid, rkgrid, M):
        """b = M sum_s T_s^H sum_c conj(mps_c) F^H (M_s ksp_c) (image_estimation.py:93-103)."""
        b = np.zeros(ksp.shape[1:], dtype=self.dtype)
        mps_c = np.conj(mps)
        for i in range(transforms.shape[0]):
            temp = (shot_mask[i] * ksp).astype(self.dtype)
            temp = self.ifft(temp, AX3)
            b += self.rigid_adjoint(np.sum(mps_c * temp, axis=0), transforms[i], kgrid, rkgrid)
            b *= M
        return b

    def normal_op(self, x_img, mps, shot_mask, transforms, kgrid, rkgrid, M):
        """A x = M sum_s T_s^H C^H F^H M_s F C T_s x (A_func, image_estimation.py:106-129)."""
        out = np.zeros(x_img.shape, dtype=self.dtype)
        mps_c = np.conj(mps)
        for i in range(transforms.shape[0]):
            Ex = self.rigid_apply(x_img, transforms[i], kgrid, rkgrid)
            Ex = mps * Ex
            Ex = self.fft(Ex, AX3)
            Ex *= shot_mask[i]
            Ex = self.ifft(Ex, AX3)
            out += self.rigid_adjoint(np.sum(mps_c * Ex, axis=0), transforms[i], kgrid, rkgrid)
        out *= M
        return out

    def estimate_image_cg(self, ksp, mps, shot_mask, transforms, kgrid, rkgrid, P, M, x0=None,
                          max_iter=100, tol=1e-6, return_iters=False):
        """Preconditioned CG-SENSE (image_estimation.py:10-165)."""
        dt = self.dtype
        img_shape = ksp.shape[1:]
        x = np.zeros(img_shape, dtype=dt) if x0 is None else np.array(x0, dtype=dt)
        b = self.cg_rhs(ksp, mps, shot_mask, transforms, kgrid, rkgrid, M)

        def A_func(x_img, out):  # image_estimation.py:106-129
            out[...] = self.normal_op(x_img, mps, shot_mask, transforms, kgrid, rkgrid, M)

        Ap = np.empty_like(x)
        A_func(x, Ap)  # image_estimation.py:133-138
        r = b - Ap
        z = P * r
        p = z.copy()
        rsold = self.vdot_real(r, z)
        iters = 0
        for it in range(max_iter):  # image_estimation.py:141-163
            A_func(p, Ap)
            iters += 1
            pAp = float(self.vdot_real(p, Ap))
            alpha = rsold / pAp
            x += alpha * p
            r += -alpha * Ap
            z = P * r
            rsnew = self.vdot_real(r, z)
            if np.sqrt(np.abs(rsnew)) < tol:
                break
            beta = rsnew / rsold
            p = z + beta * p
            rsold = rsnew
        x = x.astype(dt, copy=False)
        return (x, iters) if return_iters else x

    def forward_residual(self, ksp, mps, mask_s, image, t, kgrid, rkgrid):
        """r = M_s (F C T(t) x - y) (transform_estimation.py:41-47)."""
        r = mps * self.rigid_apply(image, t, kgrid, rkgrid)
        r = self.fft(r, AX3)
        r = (r - ksp) * mask_s
        return r.astype(self.dtype, copy=False)

    def jacobian(self, ksp_shape, mps, mask_s, image, t, kgrid, rkgrid, mode="reference"):
        """J_p = M_s F C dT/dp x for p = 0..5 (transform_estimation.py:51-56)."""
        J = np.empty((6,) + tuple(ksp_shape), dtype=self.dtype)
        for p in range(6):
            v = mps * self.rigid_derivative(image, t, p, kgrid, rkgrid, mode)
            J[p] = self.fft(v, AX3) * mask_s
        return J

    def geodesic_step(self, ksp, mps, mask_s, image, t_s, J, H, delta, kgrid, rkgrid,
                      jacobian="reference", ga_mode="reference", eps=1e-4):
        """The use_ga branch of transform_estimation.py:75-121 for one shot: returns the
        accelerated next transform and whether the acceleration was kept.  ga_mode='reference'
        restates the branch as written: its accumulator (`residual_buf`, :93-102) is overwritten
        by each partial, because the FFT output aliases it, so after the loop it holds
        (1 + v_5) J_5(t + eps v); 'intended' accumulates sum_p v_p J_p(t + eps v)."""
        v = -delta
        jv = np.zeros_like(J[0])
        for p in range(6):  # :83-86
            jv += (v[p] * J[p]).astype(jv.dtype)
        J_eps = self.jacobian(ksp.shape, mps, mask_s, image, t_s + eps * v, kgrid, rkgrid,
                              jacobian)  # :89-90, :94-99
        if ga_mode == "reference":
            acc = J_eps[5] + (v[5] * J_eps[5]).astype(J_eps.dtype)
        else:
            acc = np.zeros_like(J[0])
            for p in range(6):
                acc += (v[p] * J_eps[p]).astype(acc.dtype)
        jpv = ((acc - jv) / eps).astype(self.dtype)  # :105-106
        rhs = np.array([-self.vdot_real(jpv, J[p]) for p in range(6)])  # :111-112
        a = np.linalg.solve(H, rhs)  # :115
        keep = np.linalg.norm(a) <= np.linalg.norm(v)  # :118-123
        return t_s + (v + 0.5 * a if keep else v), keep

    def estimate_transform(self, ksp, mps, shot_mask, image, kgrid, rkgrid, damp,
                           convergence_flags, transforms, tol=1e-6, jacobian="reference",
                           record=None, use_ga=False, ga_mode="reference"):
        """One Levenberg-Marquardt sweep over shots, then mean removal
        (transform_estimation.py:7-151; use_ga adds the geodesic acceleration of :75-121).
        Mutates transforms, damp and convergence_flags in place and returns the re-centred
        image."""
        nshots = shot_mask.shape[0]
        for s in range(nshots):
            r = self.forward_residual(ksp, mps, shot_mask[s], image, transforms[s], kgrid, rkgrid)
            e0 = self.vdot_real(r, r)
            J = self.jacobian(ksp.shape, mps, shot_mask[s], image, transforms[s], kgrid, rkgrid,
                              jacobian)
            g = np.array([self.vdot_real(r, J[p]) for p in range(6)], dtype=np.float64)
            H = np.zeros((6, 6))
            for i in range(6):
                for j in range(i, 6):
                    val = self.vdot_real(J[i], J[j])
                    H[i, j] = val + (damp[s] if i == j else 0.0)
                    H[j, i] = H[i, j]
            delta = np.linalg.solve(H, g)
            nxt = transforms[s] - delta
            if use_ga:
                nxt, _ = self.geodesic_step(ksp, mps, shot_mask[s], image, transforms[s], J, H,
                                            delta, kgrid, rkgrid, jacobian, ga_mode)
            r1 = self.forward_residual(ksp, mps, shot_mask[s], image, nxt, kgrid, rkgrid)
            e1 = self.vdot_real(r1, r1)
            if record is not None:
                record.append(dict(shot=s, e0=float(e0), e1=float(e1), g=g, H=H, delta=delta))
            if e1 < e0:  # transform_estimation.py:138-144
                if np.all(np.abs(transforms[s] - nxt) < tol):
                    convergence_flags[s] = True
                transforms[s] = nxt.copy()
                damp[s] = max(damp[s] / 5, 1e-4)
            else:
                damp[s] = min(damp[s] * 1.5, 1e16)
        mean = np.mean(transforms, axis=0)  # transform_estimation.py:147-150
        out = self.rigid_apply(image, mean, kgrid, rkgrid)
        transforms -= mean
        return out

    def objective(self, ksp, mps, shot_mask, x, t, kgrid, rkgrid):
        """sum_s ||M_s (F C T_s x - y)||^2 (joint_recon.py:108-115)."""
        total = 0.0
        for s in range(shot_mask.shape[0]):
            r = self.forward_residual(ksp, mps, shot_mask[s], x, t[s], kgrid, rkgrid)
            total += float(self.vdot_real(r, r))
        return total

    # ------------------------------------------------------------------ drivers
    def joint_setup(self, ksp, mps, shot_mask):
        """JointRecon.__init__ (joint_recon.py:62-85): uncentre, normalise, P and M."""
        dt = self.dtype
        ksp = np.fft.ifftshift(np.asarray(ksp), axes=AX3).astype(dt)
        mps = np.fft.ifftshift(np.asarray(mps), axes=AX3).astype(dt)
        mask = np.fft.ifftshift(np.asarray(shot_mask), axes=AX3).astype(bool)
        max_norm = np.max(np.abs(self.ifft(ksp, AX3)))
        ksp = (ksp / max_norm).astype(dt)
        rss = np.sum(np.abs(mps) ** 2, axis=0)
        P = 1 / (rss + 1e-3)
        M = rss > 0.1
        return ksp, mps, mask, max_norm, P, M

    def joint_recon(self, ksp, mps, shot_mask, kgrid, rkgrid, t0=None, max_cg_iter=3,
                    max_nm_iter=1, max_joint_iter=100, jacobian="reference"):
        """JointRecon(...).run() (joint_recon.py:38-115).  Returns (x, t, objective_history,
        transform_history)."""
        ksp, mps, mask, max_norm, P, M = self.joint_setup(ksp, mps, shot_mask)
        nshots = len(mask)
        x = np.zeros(ksp.shape[1:], dtype=self.dtype)
        t = np.zeros((nshots, 6)) if t0 is None else np.array(t0, dtype=np.float64)
        damp = np.ones(nshots)
        flags = np.zeros(nshots, dtype=bool)
        th, oh = [], []
        for _ in range(max_joint_iter):
            x = self.estimate_image_cg(ksp, mps, mask, t, kgrid, rkgrid, P, M, x0=x,
                                       max_iter=max_cg_iter)
            for _ in range(max_nm_iter):
                x = self.estimate_transform(ksp, mps, mask, x, kgrid, rkgrid, damp, flags, t,
                                            jacobian=jacobian)
                x *= M
            th.append(t.copy())
            oh.append(self.objective(ksp, mps, mask, x, t, kgrid, rkgrid))
        x = np.fft.fftshift(x * max_norm)
        return x, t, np.array(oh), np.stack(th)

    def pyramid_reconstruction(self, ksp, mps, A, nshots, n_spatial_levels=3, n_joint_iters=100,
                               sampling="disorder", max_cg_iter=3, n_temporal_levels=3,
                               temporal=False):
        """Coarse-to-fine driver (pyramid.py:24-118); plots dropped.  temporal=True runs the
        temporal levels the reference sketches but leaves disabled (pyramid.py:80-95,120-127)
        at the coarsest spatial level, the way motionest.pyramid completes them: for factors
        2^(L-1) .. 2, merged motion states (masks of `factor` consecutive shots summed, the
        bin's mean transform as the start), then every shot takes its bin's estimate."""
        full = ksp.shape[1:]
        t_est = np.zeros((nshots, 6))
        ncoils = ksp.shape[0]
        for sl in range(n_spatial_levels - 1):
            f = 2 ** (n_spatial_levels - sl - 1)
            if sampling == "disorder":
                ds = (int(full[0] // f), int(full[1] // f), full[2])
            else:
                ds = (int(full[0] // f), full[1], full[2])
            mps_res = centred_ifft(resize(centred_fft(mps, AX3), (ncoils, *ds)), AX3)
            ksp_res = resize(ksp, (ncoils, *ds))
            A_res = resize(A, (nshots, *ds[:2], 1))
            kg, rk = transform_grids(full, [1, 1, 1], ds)
            if temporal and sl == 0:
                for tl in range(n_temporal_levels - 1):
                    tf = 2 ** (n_temporal_levels - tl - 1)
                    if nshots % tf:
                        continue
                    nb = nshots // tf
                    A_eff = A_res.reshape((nb, tf) + A_res.shape[1:]).sum(1) > 0
                    T_eff = t_est.reshape(nb, tf, 6).sum(1) / tf
                    _, T_b, _, _ = self.joint_recon(ksp_res, mps_res, A_eff, kg, rk, t0=T_eff,
                                                    max_cg_iter=max_cg_iter,
                                                    max_joint_iter=int(n_joint_iters * f))
                    t_est = np.repeat(T_b, tf, axis=0)
            _, t_est, _, _ = self.joint_recon(ksp_res, mps_res, A_res, kg, rk, t0=t_est,
                                              max_cg_iter=max_cg_iter,
                                              max_joint_iter=int(n_joint_iters * f))
        ksp_u, mps_u, mask_u, max_norm, P, M = self.joint_setup(ksp, mps, A)
        kg, rk = transform_grids(full, [1, 1, 1], None)
        x = self.estimate_image_cg(ksp_u, mps_u, mask_u, t_est, kg, rk, P, M,
                                   x0=np.zeros(full, self.dtype))
        return np.fft.fftshift(x * max_norm), t_est

    def corrupted_kspace(self, gt_img, mps, A, transforms):
        """y = fftshift sum_s M_s F (C T_s ifftshift(x)) (simulation.py:65-85)."""
        gt = np.fft.ifftshift(gt_img)
        mps = np.fft.ifftshift(mps, axes=AX3)
        A = np.fft.ifftshift(A, axes=AX3)
        kg, rk = transform_grids(gt.shape, [1, 1, 1])
        ksp = 0
        for s in range(transforms.shape[0]):
            tmp = self.rigid_apply(gt, transforms[s], kg, rk) * mps
            tmp = self.fft(tmp, AX3)
            tmp *= A[s]
            ksp = ksp + tmp
        return np.fft.fftshift(ksp, axes=AX3)


# ---------------------------------------------------------------------- grids and resizing
def transform_grids(shape, voxel_size, downsample_res=None):
    """fftshifted r and k grids (utils.py:107-137)."""
    nx, ny, nz = shape
    vx, vy, vz = voxel_size
    ds_x, ds_y, ds_z = shape if downsample_res is None else downsample_res
    rx = np.fft.fftshift((np.linspace(-nx // 2, nx // 2, ds_x, endpoint=False) * vx).reshape(-1, 1, 1))
    ry = np.fft.fftshift((np.linspace(-ny // 2, ny // 2, ds_y, endpoint=False) * vy).reshape(1, -1, 1))
    rz = np.fft.fftshift((np.linspace(-nz // 2, nz // 2, ds_z, endpoint=False) * vz).reshape(1, 1, -1))
    kx = np.fft.fftshift(np.linspace(-np.pi, np.pi, ds_x, endpoint=False).reshape((-1, 1, 1)))
    ky = np.fft.fftshift(np.linspace(-np.pi, np.pi, ds_y, endpoint=False).reshape((1, -1, 1)))
    kz = np.fft.fftshift(np.linspace(-np.pi, np.pi, ds_z, endpoint=False).reshape((1, 1, -1)))
    kgrid = {"x": kx, "y": ky, "z": kz}
    rkgrid = {"tan": {"x": rz * ky, "y": rx * kz, "z": ry * kx},
              "sin": {"x": ry * kz, "y": rz * kx, "z": rx * ky}}
    return kgrid, rkgrid


def resize(x, oshape):
    """Centred crop / zero-pad, SigPy's resize convention (used at pyramid.py:65-67)."""
    ishape = x.shape
    if tuple(ishape) == tuple(oshape):
        return x
    ish = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)]
    osh = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)]
    cp = [min(i - a, o - b) for i, a, o, b in zip(ishape, ish, oshape, osh)]
    out = np.zeros(oshape, dtype=x.dtype)
    out[tuple(slice(b, b + c) for b, c in zip(osh, cp))] = x[tuple(slice(a, a + c) for a, c in zip(ish, cp))]
    return out


def centred_fft(x, axes):
    """SigPy's centred orthonormal FFT (ifftshift -> fftn -> fftshift), dtype preserved."""
    y = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x, axes=axes), axes=axes, norm="ortho"),
                        axes=axes)
    return y.astype(x.dtype, copy=False)


def centred_ifft(x, axes):
    y = np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(x, axes=axes), axes=axes, norm="ortho"),
                        axes=axes)
    return y.astype(x.dtype, copy=False)
