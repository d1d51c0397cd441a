// Host-side composition of line passes into the rigid-transform operators.
#pragma once
#include "line_pass.cuh"

namespace me {

Phase shear_phase(const me_grid* g, int rot, int kind, bool deriv, bool conj);
Phase trans_phase(const me_grid* g, int axis, bool deriv, bool conj);
me_layout normalize_layout(const me_grid* g, me_layout lay);
bool layout_ok(const me_grid* g, me_layout lay);
int check_grid(const me_grid* g, me_layout lay);

struct Rigid {
  const me_grid* g;
  const double* params;
  int pstride;
  cudaStream_t stream;
  int dims[3];
  i64 st[3];
  i64 vox;

  Rigid(const me_grid* g, me_layout lay, const double* params, int pstride, cudaStream_t s);
  int pass(int mode, int axis, const float2* in0, const float2* in1, float2* out0, float2* out1,
           i64 in_vs, i64 out_vs, int nvol, const Phase& f0, const Phase& f1, int accum);
  // out = T in (nvol volumes); in may equal out; in_vs may be 0 (broadcast)
  int apply(const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol, bool inverse);
  // out = T^H in, or out += T^H in (accum: in is clobbered)
  int adjoint(const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol, bool accum);
  // The helpers below act on nvol volumes at once, volume v of each buffer at buffer + v * its
  // stride (params + v * pstride gives its transform); a stride of 0 broadcasts one volume.
  // trans_axis >= 0 merges the translation ramp along that axis into the last pass, which
  // must run along it (kTanAxis[r]).
  int rotation(int r, const float2* in, i64 in_vs, float2* out, i64 out_vs, int nvol,
               int trans_axis = -1);
  int rotation_derivative(int r, const float2* in, i64 in_vs, float2* out, i64 out_vs,
                          float2* wa, float2* wb, i64 w_vs, int nvol, int trans_axis = -1);
  int translation(const float2* in, i64 in_vs, float2* out, i64 out_vs, int deriv_axis, int nvol);
  int derivative(const float2* in, float2* out, int p, int mode, float2* wa, float2* wb);
  // For each of nvol volumes v: out_v[0] = T in_v, out_v[1+p] = dT/dp in_v, where out_v[k] =
  // out + v * out_bs + k * out_ks; work holds 5 volumes per v at work + v * work_bs.
  int jacobian(const float2* in, i64 in_vs, float2* out, i64 out_ks, i64 out_bs, int nvol,
               int mode, float2* work, i64 work_bs);
};

}  // namespace me
