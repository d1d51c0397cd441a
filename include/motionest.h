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

/* Volume layout: element (x, y, z) lives at x*sx + y*sy + z*sz (in complex elements).  The
 * strides must describe a dense permutation of (nx, ny, nz); the stride of an axis of length 1
 * is ignored. */
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
  /* Optional separable description (all NULL / 0 when absent).  k_uniform[a] != 0 states that
   * k[a][n] = 2 pi (m(n) - N/2) / N with m(n) = (n - floor(N/2)) mod N, which is what
   * fftshift(linspace(-pi, pi, N, endpoint=False)) gives.  tan_r[a] / sin_r[a], when set, give
   * the plane as an outer product rk = r[o] * k_pass[n] (n along the shear axis, o along the
   * plane's other non-broadcast axis), with r indexed by that axis.  When both hold, the
   * kernels evaluate the chirps by recurrence along each line instead of per element. */
  const double* tan_r[3];
  const double* sin_r[3];
  int k_uniform[3];
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
  /* Optional (may be NULL): [nshots * ny], each shot's ky bins ordered by decreasing sample
   * count.  The adjoint hands bins to threads in this order, so the threads of a warp walk
   * bins of similar length. */
  const int* ky_order;
} me_samples;

const char* me_last_error(void);
int me_abi_version(void);

/* Number of kernel launches this library has issued since it was loaded (all devices). */
long long me_launch_count(void);

/* Bounded waits.  Kernels that stage data with bulk copies on the TMA engine wait for them on
 * shared-memory barriers; every such wait gives up after about a second, records a fault bit
 * and lets the kernel finish, so a lost copy ends as an error instead of a hung GPU.  No
 * counterpart in the reference (CuPy and cuFFT have no such waits).
 * me_wait_status synchronises the current device, returns the OR of the recorded bits in
 * *status (0: no wait ran out; 1 SENSE forward, 2 SENSE adjoint, 4 line pass, 0x100 the
 * self-test) and clears them.  Results of launches before a non-zero status are not to be
 * trusted.  me_wait_selftest launches one CTA whose barrier never completes (one arrival short
 * of its count) and whose wait gives up after limit_cycles (1 .. 2^31) clock cycles; the next
 * me_wait_status then reports 0x100. */
#define ME_WAIT_SENSE_FWD 0x1u
#define ME_WAIT_SENSE_ADJ 0x2u
#define ME_WAIT_LINE_PASS 0x4u
#define ME_WAIT_SELFTEST 0x100u
int me_wait_status(unsigned* status);
int me_wait_selftest(long long limit_cycles, void* stream);

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

/* One job of me_rigid_apply_multi: the arguments of one me_rigid_apply call (inverse = 0). */
typedef struct me_rigid_job {
  const me_c64* in;
  long long in_vol_stride;
  me_c64* out;
  long long out_vol_stride;
  int nvol;
  me_layout lay;
  const me_grid* grid;
  const double* params;
  int pstride;
} me_rigid_job;

/* T x for up to 16 independent jobs at once -- volumes of different reconstructions, of uneven
 * sizes -- with each of the ten shear steps one persistent launch per distinct line length,
 * over the (job, volume, tile of lines) work items of all jobs of that length.  Every job's line lengths must have compile-time FFTs
 * (ME_FAST_LENGTHS in the sources: 16 ... 256), else ME_ERR_UNSUPPORTED.  Results are
 * bit-identical to one me_rigid_apply per job (transform.py:263-318 for each). */
int me_rigid_apply_multi(const me_rigid_job* jobs, int njobs, void* stream);

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

/* ------------------------------------------------------------------------------------------
 * SENSE operators for one reconstruction problem.
 *
 * Internal layouts (all device memory, complex64 unless noted):
 *   images       [nz][nx][ny]            (z-major "zxy": a readout plane is contiguous)
 *   mps          [nz][ncoils][nx][ny]
 *   ydat, K      per shot s, at offset shot_off[s]*ncoils*nz: [nz][ncoils][n_s], n_s the shot's
 *                sample count -- the measured k-space at the shot's (kx, ky) samples after an
 *                orthonormal inverse FFT along z (hybrid space).  Because every mask is
 *                constant along z, F^H M_s F = F_xy^H M_s F_xy and ||M_s(F v - y)|| =
 *                ||M_s F_xy v - F_z^H y||, so nothing along z is transformed per iteration.
 *   P            [nz][nx][ny] float32    CG preconditioner 1/(sum_c |mps_c|^2 + 1e-3)
 *   M            [nz][nx][ny] uint8      support mask sum_c |mps_c|^2 > 0.1
 *   transforms   [nshots][6] float64
 * `batch` is how many shots one launch of each kernel covers (1 = a plain per-shot loop,
 * nshots = every shot in one launch); results do not depend on it.
 * ---------------------------------------------------------------------------------------- */
typedef struct me_sense {
  int nx, ny, nz, ncoils, nshots;
  const me_c64* mps;
  me_samples samples;
  const me_c64* ydat;
  const float* P;
  const unsigned char* M;
  const me_grid* grid;
  const double* transforms;
} me_sense;

/* Scratch needed by me_sense_normal / me_sense_rhs / me_sense_residual /
 * me_sense_residual_norms for a given batch
 * (bytes), and by me_lm_normal_equations (which holds, per shot of the batch, T x and its six
 * partials, five work volumes, and the seven volumes' sampled k-space). */
long long me_sense_workspace_bytes(const me_sense* pb, int batch);
long long me_lm_workspace_bytes(const me_sense* pb, int batch);

/* Preconditioner and support mask from the maps (joint_recon.py:83,85). */
int me_sense_precond(const me_c64* mps, int nx, int ny, int nz, int ncoils, float* P,
                     unsigned char* M, void* stream);

/* Gather the shot samples of hybrid k-space ksp_h ([ncoils][nx][ny][nz], already inverse
 * FFT'd along z) into the ydat layout above (the masking M_s * ksp of
 * image_estimation.py:94 and transform_estimation.py:45-46, kept sparse). */
int me_sense_gather(const me_sense* pb, const me_c64* ksp_h, me_c64* ydat, void* stream);

/* out = M . sum_s T_s^H sum_c conj(mps_c) F^H M_s F (mps_c T_s p): the CG normal operator,
 * A_func of image_estimation.py:106-129. */
int me_sense_normal(const me_sense* pb, const me_c64* p, me_c64* out, int batch, void* work,
                    void* stream);

/* b = M . sum_s T_s^H sum_c conj(mps_c) F^H (M_s y_c): the CG right-hand side
 * (image_estimation.py:93-103). */
int me_sense_rhs(const me_sense* pb, me_c64* b, int batch, void* work, void* stream);

/* r = M . sum_s T_s^H sum_c conj(mps_c) F^H M_s (y_c - F mps_c T_s x): the CG's initial
 * residual b - A x (image_estimation.py:93-103 and :133-134) from one pass over the shots.  The
 * reference forms b and A x separately and subtracts them; by linearity the same vector comes
 * from one forward model, the sampled difference y - K, and one adjoint, which does the work of
 * one normal-operator application instead of two (and subtracts before the adjoint, where the
 * difference is formed from the samples themselves).  With e != NULL, e[s] (float64, device)
 * receives ||M_s (F C T_s x - y)||^2, bit-identical to me_sense_residual_norms at the problem's
 * own transforms: the summands of JointRecon._compute_objective (joint_recon.py:108-115). */
int me_sense_residual(const me_sense* pb, const me_c64* x, me_c64* r, double* e, int batch,
                      void* work, void* stream);

/* e[s] = ||M_s (F C T(t_s) x - y)||^2 for every shot, float64 on the device, with t read from
 * `transforms` ([nshots][6], device): the residual energies of transform_estimation.py:41-47 and
 * :129-135 and the summands of JointRecon._compute_objective (joint_recon.py:108-115). */
int me_sense_residual_norms(const me_sense* pb, const me_c64* x, const double* transforms,
                            double* e, int batch, void* work, void* stream);

/* K = M_s F_xy C T(t_s) x for every shot, written in the ydat layout (hybrid space): the
 * per-shot forward model of generate_corrupted_kspace (simulation.py:77-82) without its
 * z-FFT. */
int me_sense_forward(const me_sense* pb, const me_c64* x, const double* transforms, me_c64* K,
                     int batch, void* work, void* stream);

/* The SENSE kernels alone, on volumes the caller has already transformed (zxy layout, one
 * volume per shot at vol_stride elements apart).  me_sense_forward_volumes: K = M_s F C u_s for
 * shots shot0 .. shot0 + nshots - 1, steps 2-3 of A_func (image_estimation.py:115-124) without
 * the rigid transform; vol_stride 0 reads one volume for every shot.  K is laid out as ydat,
 * starting at shot shot0's first sample ([shot][z][coil][sample]).
 * me_sense_adjoint_volumes: u_s = C^H F^H M_s K_s for the same shots, steps 4-5 of A_func
 * (image_estimation.py:125-128) without T^H, written (not accumulated) to one volume per shot. */
int me_sense_forward_volumes(const me_sense* pb, const me_c64* vols, long long vol_stride,
                             int shot0, int nshots, me_c64* K, void* stream);
int me_sense_adjoint_volumes(const me_sense* pb, const me_c64* K, int shot0, int nshots,
                             me_c64* vols, long long vol_stride, void* stream);

/* ksp_h[c][kx_j][ky_j][z] += K_s[z][c][j] for every shot in turn (duplicate samples across
 * shots add up, as the reference's `ksp += temp` does, simulation.py:82). */
int me_sense_scatter(const me_sense* pb, const me_c64* K, me_c64* ksp_h, void* stream);

/* Per-shot Gauss-Newton statistics at the current transforms (pb->transforms):
 * stats[s] = {e0, g[0..5], H upper triangle row-major (21)}: 28 float64 per shot, with
 * r = M_s (F C T x - y), J_p = M_s F C dT/dp x, g_p = Re<r, J_p>, H_pq = Re<J_p, J_q>
 * (transform_estimation.py:41-68, without materialising the [6, C, X, Y, Z] Jacobian). */
int me_lm_normal_equations(const me_sense* pb, const me_c64* x, int jac_mode, double* stats,
                           int batch, void* work, void* stream);

/* Gradient-only form of me_lm_normal_equations: grad[s] = {e0, g[0..5]} (7 float64 per shot),
 * g_p = Re<r, J_p> (transform_estimation.py:41-57), computed as Re<C^H F^H M_s r, dT/dp x> in
 * image space: one forward, one adjoint and the partials' sweep per shot instead of a forward
 * of every partial.  Used by the autograd backward, which needs no Gram matrix.  `work` must
 * hold me_lm_gradient_workspace_bytes. */
long long me_lm_gradient_workspace_bytes(const me_sense* pb, int batch);
int me_lm_gradient(const me_sense* pb, const me_c64* x, int jac_mode, double* grad, int batch,
                   void* work, void* stream);

/* Geodesic acceleration (the use_ga branch of transform_estimation.py:75-121): per shot s with
 * LM step v_s = t_next - t (the increment the reference calls v = -delta),
 *   rhs[s][p] = -Re<(J(t_s + eps v_s) v_s - J(t_s) v_s) / eps, J_p(t_s)>,
 * with J = M_s F C dT/dtheta and t = pb->transforms.  `t_eps` holds t + eps v (device [nshots][6]).
 * ga_mode ME_GA_INTENDED forms J(t + eps v) v = sum_p v_p J_p(t + eps v); ME_GA_REFERENCE
 * reproduces what the reference's loop (:93-102) leaves in its accumulator, which every
 * partial overwrites: (1 + v_5) J_5(t + eps v).  The caller then solves (H + damp I) a = rhs and
 * takes v + a / 2 when |a| <= |v| (:115-123).  `work` must hold me_lm_ga_workspace_bytes. */
#define ME_GA_REFERENCE 0
#define ME_GA_INTENDED 1
long long me_lm_ga_workspace_bytes(const me_sense* pb, int batch);
int me_lm_ga_rhs(const me_sense* pb, const me_c64* x, int jac_mode, int ga_mode,
                 const double* t_eps, const double* v, double eps, double* rhs, int batch,
                 void* work, void* stream);

/* Damped solve and proposal: t_next[s] = t[s] - (H_s + damp_s I)^-1 g_s, FP64 LU with partial
 * pivoting (transform_estimation.py:60-71,125). */
int me_lm_propose(const double* stats, const double* damp, const double* t, double* t_next,
                  int nshots, void* stream);

/* Accept / reject per shot (transform_estimation.py:138-144): if e1 < e0 then t = t_next,
 * damp = max(damp/5, 1e-4) and flags |= all(|t - t_next| < tol); else damp = min(1.5 damp,
 * 1e16).  Then the mean transform is subtracted from every shot and written to mean_out
 * (transform_estimation.py:147-150). */
int me_lm_accept(const double* stats, const double* e1, double* t, const double* t_next,
                 double* damp, unsigned char* flags, double tol, double* mean_out, int nshots,
                 void* stream);

/* ------------------------------------------------------------------------------------------
 * CG vector kernels (image_estimation.py:133-163), FP64 accumulation.  `scalars` is a device
 * float64 array of 8 entries holding the CG state: [0] rz_old, [1] pAp, [2] rz_new.
 * ---------------------------------------------------------------------------------------- */
long long me_cg_workspace_bytes(long long n);

/* r = b - Ap; p = P r; scalars[0] = Re<r, P r> (image_estimation.py:133-137).  Ap may be NULL
 * when b already holds the residual (me_sense_residual): then r = b, and b may be r itself. */
int me_cg_init(const me_c64* b, const me_c64* Ap, const float* P, me_c64* r, me_c64* p,
               double* scalars, long long n, void* work, void* stream);

/* scalars[1] = Re<p, Ap> */
int me_cg_pap(const me_c64* p, const me_c64* Ap, double* scalars, long long n, void* work,
              void* stream);

/* alpha = scalars[0] / scalars[1]; x += alpha p; r -= alpha Ap; scalars[2] = Re<r, P r> */
int me_cg_update(me_c64* x, me_c64* r, const me_c64* p, const me_c64* Ap, const float* P,
                 double* scalars, long long n, void* work, void* stream);

/* beta = scalars[2] / scalars[0]; p = P r + beta p; scalars[0] = scalars[2] */
int me_cg_direction(me_c64* p, const me_c64* r, const float* P, double* scalars, long long n,
                    void* stream);

/* The whole CG-SENSE solve of estimate_image_cg (image_estimation.py:89-165) as one CUDA graph:
 * b = the right-hand side (me_sense_rhs), A x, me_cg_init, then a conditional WHILE node whose
 * body is one CG iteration (me_sense_normal, me_cg_pap, me_cg_update, a one-thread kernel that
 * applies the stopping test sqrt|rz_new| < tol and the cap of max_iter iterations on the device,
 * me_cg_direction).  Launching it runs the solve with no host round trip; `iters` (device int)
 * then holds the number of CG iterations taken, the count the host loop returns.  Every pointer
 * and the contents of *pb are captured at creation: the graph keeps reading the same buffers
 * (the transforms are re-read from pb->transforms on every launch).  `stream` must be a created
 * stream, and every library call the graph captures must have run once on this device before
 * (so that no first-use set-up happens during capture).  Creation instantiates a CUDA graph;
 * it makes no device allocation of its own.  Destroy with me_cg_graph_destroy.
 * With b == NULL the prologue leaves out the right-hand side and A x: every launch then starts
 * from the residual b - A x that the caller has put into r beforehand (me_sense_residual on the
 * same stream), and the graph's first step is me_cg_init with r given. */
typedef struct me_cg_graph me_cg_graph;
int me_cg_graph_create(const me_sense* pb, me_c64* x, me_c64* b, me_c64* r, me_c64* p,
                       me_c64* Ap, double* scalars, int* iters, int max_iter, double tol,
                       int batch, void* work, void* cg_work, void* stream, me_cg_graph** out);
int me_cg_graph_launch(me_cg_graph* g, void* stream);
/* Kernels in one pass of the loop body, and adding `iterations` passes to me_launch_count()
 * (the graph's launches are counted as the graph runs them: the prologue on launch, the body by
 * this call once the iteration count is known). */
long long me_cg_graph_body_launches(const me_cg_graph* g);
void me_cg_graph_account(const me_cg_graph* g, int iterations);
int me_cg_graph_destroy(me_cg_graph* g);

/* out[0] = Re<a, b> (float64) */
int me_dot_re(const me_c64* a, const me_c64* b, double* out, long long n, void* work,
              void* stream);

/* Allocation-free variant of me_dot_re, for callers that cannot allocate device memory: a host
 * runtime that reserves all GPU memory itself at start-up, or a serving process whose memory
 * budget forbids device allocations once it is running.  It has no counterpart in the
 * reference.  out[0] = Re<a, b> (float64) as me_dot_re computes it, with the partial sums held
 * in a static 32 KiB device array inside the library (one array per GPU, kept until the process
 * exits) instead of caller scratch, so n is limited to ME_NOALLOC_DOT_MAX_N (2^28) elements;
 * larger n returns ME_ERR_INVALID.  The first call on each device looks up the array's device
 * address and keeps it for the life of the process, so make that first call before any stream
 * capture and do not reset the device (cudaDeviceReset) after it.  All calls share the one
 * array: calls that overlap on the GPU (different streams, no ordering between them) race. */
#define ME_NOALLOC_DOT_CHUNK 65536LL
#define ME_NOALLOC_DOT_PARTIALS 4096
#define ME_NOALLOC_DOT_MAX_N (ME_NOALLOC_DOT_CHUNK * ME_NOALLOC_DOT_PARTIALS)
int me_dot_re_noalloc(const me_c64* a, const me_c64* b, double* out, long long n, void* stream);

/* Orthonormal DFT (inverse != 0: inverse DFT) of nrows contiguous rows of length n (192, 224 or
 * 256) on the tensor cores: two matrix stages of the four-step factorisation n = 16 * n2 as
 * mma.sync TF32 products with FP32 accumulation and every operand split into two TF32 terms
 * (three products per term pair).  The measured alternative to the register FFT of
 * me_fft_axis for the short lines of the rigid-transform and SENSE kernels (transform.py:279-301
 * and image_estimation.py:115-126 do these transforms with cuFFT); out != in. */
int me_dft_rows_split(const me_c64* in, me_c64* out, long long nrows, int n, int inverse,
                      void* stream);

/* out[0] = max |a| (float32) */
int me_max_abs(const me_c64* a, long long n, float* out, void* work, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MOTIONEST_H */
