/*
 * motionest — B200-native SAMER/DISORDER joint motion-corrected MRI reconstruction.
 *
 * C ABI of libmotionest.so: plain pointers and sizes, no torch types.  Every array argument is
 * a DEVICE pointer unless stated otherwise; every call is stream-ordered on the given
 * cudaStream_t (passed as void*; NULL = legacy default stream) and returns ME_OK (0) or an error
 * code, with a message available from me_last_error().  No entry point allocates device memory:
 * scratch is passed in by the caller, sized by the matching *_workspace_bytes() query.
 *
 * The reference (chiew-group/motion-estimation) is pure Python on CuPy; it has no C ABI or
 * FFI.  Each entry point below names the reference function whose computation it replaces, by
 * file:line in that project.  The Python package `motionest` binds these with ctypes and keeps
 * the reference's Python API on top.
 *
 * Conventions
 *  - complex64 data is interleaved (re, im) float32, the NumPy/CuPy/torch complex64 layout.
 *  - Images and coil data are "uncentred" (ifftshift-ed, index 0 = DC), as the reference's
 *    operators expect (image_estimation.py:66).
 *  - FFTs are orthonormal (norm='ortho'), DFT sign exp(-2 pi i k n / N) forward.
 *  - Rigid parameters are float64 [6] = (tx, ty, tz, rx, ry, rz), rotations in radians.
 */
#ifndef MOTIONEST_H
#define MOTIONEST_H

#ifdef __cplusplus
extern "C" {
#endif

#define ME_OK 0
#define ME_ERR_INVALID 1     /* bad argument (shape, size, pointer, mode) */
#define ME_ERR_CUDA 2        /* a CUDA runtime call failed */
#define ME_ERR_UNSUPPORTED 3 /* valid request this build does not handle (e.g. line length) */

#define ME_ABI_VERSION 1

/* Longest supported FFT line (any length up to this whose prime factors are <= 13). */
#define ME_MAX_LINE 512

typedef struct me_c64 {
  float re, im;
} me_c64;

/* Volume layout: element (x, y, z) lives at x*sx + y*sy + z*sz (in complex elements). */
typedef struct me_layout {
  long long sx, sy, sz;
} me_layout;

/* Transform grids as compute_transform_grids_voxel builds them (utils.py:107-137), already on
 * the device as float64.  k[a] is kgrid['x'|'y'|'z'] flattened (length nx|ny|nz).  tan_rk[a] /
 * sin_rk[a] are rkgrid['tan'|'sin']['x'|'y'|'z']; their element strides along x, y, z are given
 * in tan_st[a] / sin_st[a] (0 along a broadcast axis).  The planes are read as given, so any
 * grid the reference accepts is accepted here. */
typedef struct me_grid {
  int nx, ny, nz;
  const double* k[3];
  const double* tan_rk[3];
  const double* sin_rk[3];
  long long tan_st[3][3];
  long long sin_st[3][3];
} me_grid;

/* Per-shot sampling of a [nshots, nx, ny, 1] mask (the mask is constant along z, as the
 * reference's masks are: simulation.py:437, recon.py:165, pyramid.py:67).  For shot s the
 * sampled (kx, ky) points are kx[shot_off[s] .. shot_off[s+1]) and ky[...], sorted by ky;
 * ky_off[s*(ny+1) + v] .. ky_off[s*(ny+1) + v + 1] (relative to shot_off[s]) are the samples
 * with ky == v.  Built on the host from the mask (motionest/sampling.py). */
typedef struct me_samples {
  int nshots, nx, ny;
  int max_per_shot;
  const int* shot_off; /* [nshots + 1] */
  const int* kx;       /* [total] */
  const int* ky;       /* [total] */
  const int* ky_off;   /* [nshots * (ny + 1)] */
} me_samples;

const char* me_last_error(void);
int me_abi_version(void);

/* ------------------------------------------------------------------------------------------
 * 1-D transforms along one axis of a batch of volumes.
 * ---------------------------------------------------------------------------------------- */

/* Orthonormal FFT (inverse != 0: IFFT) along `axis` (0, 1, 2) of nvol volumes, out of place
 * or in place (in == out).  Replaces the per-axis cupyx fft/ifft calls used for the hybrid
 * k-space and the max-norm scan (joint_recon.py:67, image_estimation.py:97). */
int me_fft_axis(const me_c64* in, long long in_vol_stride, me_c64* out, long long out_vol_stride,
                int nvol, int nx, int ny, int nz, me_layout lay, int axis, int inverse,
                void* stream);

/* ------------------------------------------------------------------------------------------
 * Rigid transform operators (transform.py:243-504).
 * `params` is a device float64 array; volume v uses params[v*pstride .. +6) (pstride 0 shares
 * one set).  in == out is allowed; in_vol_stride 0 broadcasts one input to every output.
 * ---------------------------------------------------------------------------------------- */

/* T x = Tr.Rz.Ry.Rx x: RigidTransformCudaOptimzied.apply (transform.py:263-318); inverse != 0
 * conjugates only the translation ramp, as the reference's `inverse` flag does (:308). */
int me_rigid_apply(const me_c64* in, long long in_vol_stride, me_c64* out,
                   long long out_vol_stride, int nvol, me_layout lay, const me_grid* g,
                   const double* params, int pstride, int inverse, void* stream);

/* T^H x: RigidTransformCudaOptimzied.adjoint (transform.py:320-377).  accumulate != 0 computes
 * out += T^H in and overwrites `in` (used as scratch; in != out). */
int me_rigid_adjoint(const me_c64* in, long long in_vol_stride, me_c64* out,
                     long long out_vol_stride, int nvol, me_layout lay, const me_grid* g,
                     const double* params, int pstride, int accumulate, void* stream);

#define ME_JAC_REFERENCE 0 /* d/dp of Tr.Rx.Ry.Rz: RigidTransformDerivativeCuda (transform.py:476-504) */
#define ME_JAC_EXACT 1     /* d/dp of Tr.Rz.Ry.Rx, the operator me_rigid_apply implements */

/* Workspace for me_rigid_derivative / me_rigid_jacobian on one volume (bytes). */
long long me_rigid_jacobian_workspace_bytes(int nx, int ny, int nz);

/* dT/dparams[p_idx] x for one volume: RigidTransformDerivativeCuda.apply(x, p_idx)
 * (transform.py:476-504) in ME_JAC_REFERENCE mode.  p_idx outside 0..5 copies the input, as the
 * reference does.  `work` must hold me_rigid_jacobian_workspace_bytes. */
int me_rigid_derivative(const me_c64* in, me_c64* out, me_layout lay, const me_grid* g,
                        const double* params, int p_idx, int mode, void* work, void* stream);

/* T x and all six partials in one sweep that shares the rotation prefixes:
 * out[0] = T x, out[1 + p] = dT/dp x (p = 0..5), each volume at out + i*out_vol_stride.
 * Replaces the per-shot loop transform_estimation.py:41-56 (its transform work). */
int me_rigid_jacobian(const me_c64* in, me_c64* out, long long out_vol_stride, me_layout lay,
                      const me_grid* g, const double* params, int mode, void* work, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MOTIONEST_H */
