// Rigid transform operators built from line passes (transform.py:243-504).
//
// T = Tr . Rz . Ry . Rx.  Each rotation R_r is three shears S_tan S_sin S_tan along the axes
// (tan, sin) = (1, 2) for x, (2, 0) for y, (0, 1) for z (transform.py:267-271); each shear is an
// FFT along its axis, a chirp exp(i a rk) and an inverse FFT.  The translation is separable, so
// instead of the reference's 3-D FFT / ramp / 3-D IFFT it becomes three 1-D ramps, two of them
// merged into shear passes along the same axis:
//   z-ramp into the last y-rotation pass (axis 2; Tz commutes with Rz, whose shears act along
//   axes 0 and 1 with phases that do not depend on z), x-ramp into the last z-rotation pass
//   (axis 0), y-ramp as a pass of its own.  10 passes per apply / adjoint.
#include <cstring>
#include <string>

#include "line_pass.cuh"
#include "rigid.cuh"

namespace me {

static const int kTanAxis[3] = {1, 2, 0};
static const int kSinAxis[3] = {2, 0, 1};

// The plane of shear (rot, kind) is indexed by the pass-axis frequency and one other axis.
// The other axis of a rotation's tan shear is its sin shear's pass axis, and the other way round:
//   tan: x->(ax 1, other 2), y->(ax 2, other 0), z->(ax 0, other 1)
//   sin: x->(ax 2, other 1), y->(ax 0, other 2), z->(ax 1, other 0)
static int plane_other_axis(int rot, int kind) {
  return kind == PH_TAN ? kSinAxis[rot] : kTanAxis[rot];
}

Phase shear_phase(const me_grid* g, int rot, int kind, bool deriv, bool conj) {
  Phase p{};
  p.kind = kind;
  p.rot = rot;
  p.deriv = deriv;
  p.conj = conj;
  const int ax = (kind == PH_TAN) ? kTanAxis[rot] : kSinAxis[rot];
  if (kind == PH_TAN) {
    p.plane = g->tan_rk[rot];
    for (int i = 0; i < 3; i++) p.ps[i] = g->tan_st[rot][i];
    p.rvec = g->tan_r[rot];
  } else {
    p.plane = g->sin_rk[rot];
    for (int i = 0; i < 3; i++) p.ps[i] = g->sin_st[rot][i];
    p.rvec = g->sin_r[rot];
  }
  p.oaxis = plane_other_axis(rot, kind);
  p.sep = (p.rvec != nullptr) && g->k_uniform[ax];
  return p;
}

Phase trans_phase(const me_grid* g, int axis, bool deriv, bool conj) {
  Phase p{};
  p.kind = PH_NONE;
  p.trans = 1;
  p.trans_deriv = deriv;
  p.conj = conj;
  p.kv = g->k[axis];
  p.sep = g->k_uniform[axis] != 0;
  return p;
}

static Phase with_trans(Phase p, const me_grid* g, int axis) {
  p.trans = 1;
  p.kv = g->k[axis];
  p.sep = p.sep && g->k_uniform[axis];
  return p;
}

me_layout normalize_layout(const me_grid* g, me_layout lay) {
  // An axis of length 1 is only ever indexed at 0, so its stride carries no information and
  // callers pass anything there (often a stride equal to a neighbour's).  Give it the volume
  // size, which makes it the outermost axis of a dense permutation and never the coalescing
  // axis of a line pass.
  if (!g) return lay;
  const i64 vox = (i64)g->nx * g->ny * g->nz;
  if (g->nx == 1) lay.sx = vox;
  if (g->ny == 1) lay.sy = vox;
  if (g->nz == 1) lay.sz = vox;
  return lay;
}

bool layout_ok(const me_grid* g, me_layout lay) {
  const i64 n[3] = {g->nx, g->ny, g->nz};
  const i64 s[3] = {lay.sx, lay.sy, lay.sz};
  // dense permutation: sorted strides are 1, n_a, n_a*n_b
  int o[3] = {0, 1, 2};
  for (int i = 0; i < 3; i++)
    for (int j = i + 1; j < 3; j++)
      if (s[o[j]] < s[o[i]]) {
        int t = o[i];
        o[i] = o[j];
        o[j] = t;
      }
  return s[o[0]] == 1 && s[o[1]] == n[o[0]] && s[o[2]] == n[o[0]] * n[o[1]];
}

int check_grid(const me_grid* g, me_layout lay) {
  if (!g) return fail("grid is NULL");
  if (g->nx < 1 || g->ny < 1 || g->nz < 1) return fail("grid dims must be positive");
  for (int a = 0; a < 3; a++)
    if (!g->k[a] || !g->tan_rk[a] || !g->sin_rk[a]) return fail("grid pointer is NULL");
  if (!layout_ok(g, lay)) return fail("volume layout must be a dense permutation of (nx,ny,nz)");
  return ME_OK;
}

Rigid::Rigid(const me_grid* g_, me_layout lay, const double* params_, int pstride_,
             cudaStream_t s)
    : g(g_), params(params_), pstride(pstride_), stream(s) {
  lay = normalize_layout(g, lay);
  dims[0] = g->nx;
  dims[1] = g->ny;
  dims[2] = g->nz;
  st[0] = lay.sx;
  st[1] = lay.sy;
  st[2] = lay.sz;
  vox = (i64)g->nx * g->ny * g->nz;
}

int Rigid::pass(int mode, int axis, const float2* in0, const float2* in1, float2* out0,
                float2* out1, i64 in_vs, i64 out_vs, int nvol, const Phase& f0, const Phase& f1,
                int accum) {
  return launch_line_pass(mode, in0, in1, out0, out1, in_vs, out_vs, nvol, dims, st, axis, f0, f1,
                          params, pstride, accum, stream);
}

#define ME_TRY(x)               \
  do {                          \
    int _rc = (x);              \
    if (_rc != ME_OK) return _rc; \
  } while (0)

// The shear steps of T (axis, phase) in the order they run; `inverse` conjugates only the
// translation ramp (transform.py:308).
static int apply_steps(const me_grid* g, bool inverse, int axes[12], Phase phases[12]) {
  int k = 0;
  for (int r = 0; r < 3; r++) {
    const Phase vt = shear_phase(g, r, PH_TAN, false, false);
    const Phase vs = shear_phase(g, r, PH_SIN, false, false);
    axes[k] = kTanAxis[r];
    phases[k++] = vt;
    axes[k] = kSinAxis[r];
    phases[k++] = vs;
    Phase last = vt;
    if (r == 1) last = with_trans(vt, g, 2);  // Tz merged (axis 2)
    if (r == 2) last = with_trans(vt, g, 0);  // Tx merged (axis 0)
    if (inverse && r >= 1) {
      // keep the shear and flip the ramp's sign with a conjugated ramp-only pass instead
      last = vt;
    }
    axes[k] = kTanAxis[r];
    phases[k++] = last;
  }
  if (inverse) {
    axes[k] = 2;
    phases[k++] = trans_phase(g, 2, false, true);
    axes[k] = 0;
    phases[k++] = trans_phase(g, 0, false, true);
    axes[k] = 1;
    phases[k++] = trans_phase(g, 1, false, true);
  } else {
    axes[k] = 1;
    phases[k++] = trans_phase(g, 1, false, false);
  }
  return k;
}

int Rigid::apply(const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol, bool inverse) {
  const Phase none = phase_none();
  int axes[12];
  Phase phases[12];
  const int n = apply_steps(g, inverse, axes, phases);
  const float2* src = in;
  i64 svs = in_vs;
  for (int k = 0; k < n; k++) {
    ME_TRY(pass(PM_SHEAR, axes[k], src, nullptr, out, nullptr, svs, out_vs, nvol, phases[k],
                none, 0));
    src = out;
    svs = out_vs;
  }
  return ME_OK;
}

int Rigid::adjoint(const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol, bool accum) {
  // T^H = Rx^H Ry^H Rz^H Tr^H: the passes of apply in reverse order with conjugated factors
  // (transform.py:320-377).  Without accumulation the first pass reads `in` and the rest run in
  // place on `out`; with accumulation the first nine run in place on `in` (clobbering it) and
  // the last adds into `out`.
  const Phase none = phase_none();
  struct P {
    int axis;
    Phase f;
  };
  P seq[10];
  int k = 0;
  seq[k++] = {1, trans_phase(g, 1, false, true)};
  for (int r = 2; r >= 0; r--) {
    const Phase vt = shear_phase(g, r, PH_TAN, false, true);
    const Phase vs = shear_phase(g, r, PH_SIN, false, true);
    Phase first = vt;
    if (r == 2) first = with_trans(vt, g, 0);
    if (r == 1) first = with_trans(vt, g, 2);
    seq[k++] = {kTanAxis[r], first};
    seq[k++] = {kSinAxis[r], vs};
    seq[k++] = {kTanAxis[r], vt};
  }
  const float2* src = in;
  i64 svs = in_vs;
  float2* work = accum ? const_cast<float2*>(in) : out;
  const i64 wvs = accum ? in_vs : out_vs;
  for (int i = 0; i < k; i++) {
    const bool last = (i == k - 1);
    float2* dst = last ? out : work;
    const i64 dvs = last ? out_vs : wvs;
    ME_TRY(pass(PM_SHEAR, seq[i].axis, src, nullptr, dst, nullptr, svs, dvs, nvol, seq[i].f, none,
                (last && accum) ? 1 : 0));
    src = work;
    svs = wvs;
  }
  return ME_OK;
}

int Rigid::rotation(int r, const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol,
                    int trans_axis) {
  const Phase none = phase_none();
  const Phase vt = shear_phase(g, r, PH_TAN, false, false);
  const Phase vs = shear_phase(g, r, PH_SIN, false, false);
  const Phase vl = (trans_axis == kTanAxis[r]) ? with_trans(vt, g, trans_axis) : vt;
  ME_TRY(pass(PM_SHEAR, kTanAxis[r], in, nullptr, out, nullptr, in_vs, out_vs, nvol, vt, none, 0));
  ME_TRY(pass(PM_SHEAR, kSinAxis[r], out, nullptr, out, nullptr, out_vs, out_vs, nvol, vs, none, 0));
  ME_TRY(pass(PM_SHEAR, kTanAxis[r], out, nullptr, out, nullptr, out_vs, out_vs, nvol, vl, none, 0));
  return ME_OK;
}

int Rigid::rotation_derivative(int r, const float2* in, i64 in_vs, float2* out, i64 out_vs,
                               float2* wa, float2* wb, i64 w_vs, int nvol, int trans_axis) {
  // d(S_t S_s S_t) = S_t S_s S'_t + S_t S'_s S_t + S'_t S_s S_t   (transform.py:433-474)
  const Phase vt = shear_phase(g, r, PH_TAN, false, false);
  const Phase vs = shear_phase(g, r, PH_SIN, false, false);
  const Phase dvt = shear_phase(g, r, PH_TAN, true, false);
  const Phase dvs = shear_phase(g, r, PH_SIN, true, false);
  const Phase none = phase_none();
  const int at = kTanAxis[r], as = kSinAxis[r];
  // wa = S'_t in, wb = S_t in
  ME_TRY(pass(PM_DUAL_OUT, at, in, nullptr, wa, wb, in_vs, w_vs, nvol, dvt, vt, 0));
  // wa = S_s wa + S'_s wb
  ME_TRY(pass(PM_DUAL_IN, as, wa, wb, wa, nullptr, w_vs, w_vs, nvol, vs, dvs, 0));
  // wb = S_s wb
  ME_TRY(pass(PM_SHEAR, as, wb, nullptr, wb, nullptr, w_vs, w_vs, nvol, vs, none, 0));
  // out = S_t wa + S'_t wb (times the translation ramp along `at` when merged: both terms)
  const bool merge = (trans_axis == at);
  ME_TRY(pass(PM_DUAL_IN, at, wa, wb, out, nullptr, w_vs, out_vs, nvol,
              merge ? with_trans(vt, g, at) : vt, merge ? with_trans(dvt, g, at) : dvt, 0));
  return ME_OK;
}

int Rigid::translation(const float2* in, i64 in_vs, float2* out, i64 out_vs, int deriv_axis,
                       int nvol) {
  const Phase none = phase_none();
  const float2* src = in;
  i64 svs = in_vs;
  for (int a = 0; a < 3; a++) {
    const Phase f = trans_phase(g, a, a == deriv_axis, false);
    ME_TRY(pass(PM_SHEAR, a, src, nullptr, out, nullptr, svs, out_vs, nvol, f, none, 0));
    src = out;
    svs = out_vs;
  }
  return ME_OK;
}

int Rigid::derivative(const float2* in, float2* out, int p, int mode, float2* wa, float2* wb) {
  if (p < 0 || p > 5) {
    return check_cuda(cudaMemcpyAsync(out, in, sizeof(float2) * vox, cudaMemcpyDeviceToDevice,
                                      stream),
                      "derivative copy");
  }
  const int ref_order[3] = {2, 1, 0};
  const int exact_order[3] = {0, 1, 2};
  const int* order = (mode == ME_JAC_REFERENCE) ? ref_order : exact_order;
  const float2* src = in;
  for (int i = 0; i < 3; i++) {
    const int r = order[i];
    if (r == p - 3) {
      ME_TRY(rotation_derivative(r, src, 0, out, 0, wa, wb, 0, 1));
    } else {
      ME_TRY(rotation(r, src, 0, out, 0, 1));
    }
    src = out;
  }
  return translation(out, 0, out, 0, p < 3 ? p : -1, 1);
}

int Rigid::jacobian(const float2* in, i64 in_vs, float2* out, i64 out_ks, i64 out_bs, int nvol,
                    int mode, float2* work, i64 work_bs) {
  const int ref_order[3] = {2, 1, 0};
  const int exact_order[3] = {0, 1, 2};
  const int* order = (mode == ME_JAC_REFERENCE) ? ref_order : exact_order;
  float2* wa = work;
  float2* wb = work + vox;
  float2* P[4];
  i64 pvs[4] = {in_vs, work_bs, work_bs, work_bs};
  P[0] = const_cast<float2*>(in);
  P[1] = work + 2 * vox;
  P[2] = work + 3 * vox;
  P[3] = work + 4 * vox;
  for (int i = 0; i < 3; i++) ME_TRY(rotation(order[i], P[i], pvs[i], P[i + 1], work_bs, nvol));
  // rotation partials: D_{3+o_i} = Tr R_{o_2} .. R_{o_{i+1}} dR_{o_i} P_i.  The ramp along the
  // last rotation's tan axis rides in that rotation's final pass; the other two follow.
  const int ta = kTanAxis[order[2]];
  const Phase none = phase_none();
  for (int i = 0; i < 3; i++) {
    const int r = order[i];
    float2* d = out + (i64)(1 + 3 + r) * out_ks;
    ME_TRY(rotation_derivative(r, P[i], pvs[i], d, out_bs, wa, wb, work_bs, nvol,
                               i == 2 ? ta : -1));
    for (int j = i + 1; j < 3; j++)
      ME_TRY(rotation(order[j], d, out_bs, d, out_bs, nvol, j == 2 ? ta : -1));
    for (int a = 0; a < 3; a++) {
      if (a == ta) continue;
      ME_TRY(pass(PM_SHEAR, a, d, nullptr, d, nullptr, out_bs, out_bs, nvol,
                  trans_phase(g, a, false, false), none, 0));
    }
  }
  // translation partials D_p = T_2 T_1 T_0 P_3 with T_p differentiated, the ramps applied in
  // axis order 0, 1, 2; dual-output passes share the undifferentiated prefix:
  //   O0 = T0 P3, O1 = dT0 P3;  O0 = T1 O0, O2 = dT1 O0;  O0 = T2 O0 (= Tr P3), O3 = dT2 O0;
  //   O1 = T2 T1 O1;  O2 = T2 O2.
  float2* O[4];
  for (int k = 0; k < 4; k++) O[k] = out + (i64)k * out_ks;
  Phase tr[3], dtr[3];
  for (int a = 0; a < 3; a++) {
    tr[a] = trans_phase(g, a, false, false);
    dtr[a] = trans_phase(g, a, true, false);
  }
  ME_TRY(pass(PM_DUAL_OUT, 0, P[3], nullptr, O[0], O[1], work_bs, out_bs, nvol, tr[0], dtr[0], 0));
  ME_TRY(pass(PM_DUAL_OUT, 1, O[0], nullptr, O[0], O[2], out_bs, out_bs, nvol, tr[1], dtr[1], 0));
  ME_TRY(pass(PM_DUAL_OUT, 2, O[0], nullptr, O[0], O[3], out_bs, out_bs, nvol, tr[2], dtr[2], 0));
  ME_TRY(pass(PM_SHEAR, 1, O[1], nullptr, O[1], nullptr, out_bs, out_bs, nvol, tr[1], none, 0));
  ME_TRY(pass(PM_SHEAR, 2, O[1], nullptr, O[1], nullptr, out_bs, out_bs, nvol, tr[2], none, 0));
  ME_TRY(pass(PM_SHEAR, 2, O[2], nullptr, O[2], nullptr, out_bs, out_bs, nvol, tr[2], none, 0));
  // T x itself: Tr P3 (now in O0) in exact mode; the applied transform in the reference's
  // convention, whose rotation order differs from the derivative's
  if (mode != ME_JAC_EXACT) ME_TRY(apply(in, in_vs, out, out_bs, nvol, false));
  return ME_OK;
}

}  // namespace me

using namespace me;

extern "C" {

int me_rigid_apply(const me_c64* in, long long in_vs, me_c64* out, long long out_vs, int nvol,
                   me_layout lay, const me_grid* g, const double* params, int pstride,
                   int inverse, void* stream) {
  lay = normalize_layout(g, lay);
  ME_TRY(check_grid(g, lay));
  if (!in || !out || !params) return fail("me_rigid_apply: NULL pointer");
  if (nvol > 1 && out_vs == 0) return fail("me_rigid_apply: nvol > 1 needs out_vol_stride");
  Rigid R(g, lay, params, pstride, (cudaStream_t)stream);
  return R.apply((const float2*)in, in_vs, (float2*)out, out_vs, nvol, inverse != 0);
}

int me_rigid_apply_multi(const me_rigid_job* jobs, int njobs, void* stream) {
  if (njobs < 0 || (njobs > 0 && !jobs)) return fail("me_rigid_apply_multi: bad job list");
  if (njobs > kMaxMultiJobs)
    return fail("me_rigid_apply_multi: at most " + std::to_string(kMaxMultiJobs) + " jobs");
  if (njobs == 0) return ME_OK;
  const Phase none = phase_none();
  int axes[kMaxMultiJobs][12];
  Phase phases[kMaxMultiJobs][12];
  int nsteps = -1;
  for (int j = 0; j < njobs; j++) {
    const me_rigid_job& J = jobs[j];
    const me_layout lay = normalize_layout(J.grid, J.lay);
    ME_TRY(check_grid(J.grid, lay));
    if (!J.in || !J.out || !J.params) return fail("me_rigid_apply_multi: NULL pointer in a job");
    if (J.nvol < 0) return fail("me_rigid_apply_multi: negative volume count");
    if (J.nvol > 1 && J.out_vol_stride == 0)
      return fail("me_rigid_apply_multi: nvol > 1 needs out_vol_stride");
    const int n = apply_steps(J.grid, false, axes[j], phases[j]);
    if (nsteps >= 0 && n != nsteps) return fail("me_rigid_apply_multi: step counts differ");
    nsteps = n;
  }
  for (int k = 0; k < nsteps; k++) {
    PassArgs A[kMaxMultiJobs];
    for (int j = 0; j < njobs; j++) {
      const me_rigid_job& J = jobs[j];
      Rigid R(J.grid, normalize_layout(J.grid, J.lay), J.params, J.pstride,
              (cudaStream_t)stream);
      const float2* src = (k == 0) ? (const float2*)J.in : (const float2*)J.out;
      const i64 svs = (k == 0) ? J.in_vol_stride : J.out_vol_stride;
      ME_TRY(make_pass_args(PM_SHEAR, src, nullptr, (float2*)J.out, nullptr, svs,
                            J.out_vol_stride, J.nvol, R.dims, R.st, axes[j][k], phases[j][k],
                            none, J.params, J.pstride, 0, &A[j]));
    }
    ME_TRY(launch_multi_shear(A, njobs, (cudaStream_t)stream));
  }
  return ME_OK;
}

int me_rigid_adjoint(const me_c64* in, long long in_vs, me_c64* out, long long out_vs, int nvol,
                     me_layout lay, const me_grid* g, const double* params, int pstride,
                     int accumulate, void* stream) {
  lay = normalize_layout(g, lay);
  ME_TRY(check_grid(g, lay));
  if (!in || !out || !params) return fail("me_rigid_adjoint: NULL pointer");
  if (nvol > 1 && out_vs == 0 && !accumulate)
    return fail("me_rigid_adjoint: nvol > 1 needs out_vol_stride");
  if (accumulate && (const void*)in == (const void*)out)
    return fail("me_rigid_adjoint: accumulate needs in != out (in is overwritten as scratch)");
  if (accumulate && nvol > 1 && out_vs == 0)
    return fail("me_rigid_adjoint: cannot accumulate several volumes into one output");
  Rigid R(g, lay, params, pstride, (cudaStream_t)stream);
  return R.adjoint((const float2*)in, in_vs, (float2*)out, out_vs, nvol, accumulate != 0);
}

long long me_rigid_jacobian_workspace_bytes(int nx, int ny, int nz) {
  return 5LL * nx * ny * nz * (long long)sizeof(me_c64);
}

int me_rigid_derivative(const me_c64* in, me_c64* out, me_layout lay, const me_grid* g,
                        const double* params, int p_idx, int mode, void* work, void* stream) {
  lay = normalize_layout(g, lay);
  ME_TRY(check_grid(g, lay));
  if (!in || !out || !params || !work) return fail("me_rigid_derivative: NULL pointer");
  if (mode != ME_JAC_REFERENCE && mode != ME_JAC_EXACT) return fail("bad jacobian mode");
  Rigid R(g, lay, params, 0, (cudaStream_t)stream);
  float2* w = (float2*)work;
  return R.derivative((const float2*)in, (float2*)out, p_idx, mode, w, w + R.vox);
}

int me_rigid_jacobian(const me_c64* in, me_c64* out, long long out_vs, me_layout lay,
                      const me_grid* g, const double* params, int mode, void* work,
                      void* stream) {
  lay = normalize_layout(g, lay);
  ME_TRY(check_grid(g, lay));
  if (!in || !out || !params || !work) return fail("me_rigid_jacobian: NULL pointer");
  if (mode != ME_JAC_REFERENCE && mode != ME_JAC_EXACT) return fail("bad jacobian mode");
  Rigid R(g, lay, params, 0, (cudaStream_t)stream);
  if (out_vs < R.vox) return fail("me_rigid_jacobian: out_vol_stride too small");
  return R.jacobian((const float2*)in, 0, (float2*)out, out_vs, 0, 1, mode, (float2*)work, 0);
}

}  // extern "C"
