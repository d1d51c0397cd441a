// Line passes: FFT along one axis of a batch of volumes, a per-element phase, inverse FFT.
// Every rigid-transform step of the reference (each shear, each translation ramp, and their
// derivatives) is one of these passes.
#pragma once
#include "common.cuh"
#include "fft_smem.cuh"

namespace me {

enum PassMode {
  PM_SHEAR = 0,     // out0 = IFFT(f0 . FFT(in0))
  PM_DUAL_OUT = 1,  // out0 = IFFT(f0 . FFT(in0)), out1 = IFFT(f1 . FFT(in0))
  PM_DUAL_IN = 2,   // out0 = IFFT(f0 . FFT(in0) + f1 . FFT(in1))
  PM_FWD = 3,       // out0 = f0 . FFT(in0)
  PM_INV = 4,       // out0 = IFFT(f0 . in0)
};

enum PhaseKind { PH_NONE = 0, PH_TAN = 1, PH_SIN = 2 };

// f(n, x, y, z) = scale * mult * exp(i (a * rk(x,y,z) + b * k[n])), optionally conjugated, where
//   a = tan(theta/2) (PH_TAN) or -sin(theta) (PH_SIN), theta = params[3 + rot]   (transform.py:275-276)
//   b = -params[axis] when `trans` (translation ramp, transform.py:257-261)
//   mult = i (1 + tan^2(theta/2))/2 rk  or  -i cos(theta) rk when `deriv`  (transform.py:437-438)
//        times -i k[n] when `trans_deriv`                                     (transform.py:428)
struct Phase {
  int kind;
  int rot;
  int deriv;
  int trans;
  int trans_deriv;
  int conj;
  const double* plane;
  i64 ps[3];
  const double* kv;
  // Separable description (see me_grid): rk = rvec[coordinate along oaxis] * k[n] with k
  // uniform along the pass axis; `sep` set when the whole phase can use the line recurrence.
  const double* rvec;
  int oaxis;
  int sep;
};

struct PassArgs {
  const float2* in0;
  const float2* in1;
  float2* out0;
  float2* out1;
  i64 in_vs, out_vs;
  int nvol;
  int dims[3];
  i64 st[3];
  int ax, au, av;  // pass axis; the two other axes, av the one with the smaller stride
  int nlines;
  FastDiv div_av;     // division by dims[av] (line index -> coordinates)
  FastDiv div_tiles;  // division by the compile-time kernels' tiles per volume
  int B;   // lines per CTA
  int es;  // shared-memory row stride (elements)
  int accum;
  float scale;
  const double* params;
  int pstride;
  Phase ph[2];
  FftPlan plan;
};

inline Phase phase_none() {
  Phase p{};
  p.kind = PH_NONE;
  return p;
}

// The PassArgs of one pass (validated; error code and message on failure).
int make_pass_args(int mode, const float2* in0, const float2* in1, float2* out0, float2* out1,
                   i64 in_vs, i64 out_vs, int nvol, const int dims[3], const i64 st[3], int axis,
                   const Phase& f0, const Phase& f1, const double* params, int pstride, int accum,
                   PassArgs* out);

// One shear step of up to kMaxMultiJobs independent jobs (PassArgs of PM_SHEAR passes, line
// lengths with compile-time FFTs) in one persistent launch.
constexpr int kMaxMultiJobs = 16;
int launch_multi_shear(const PassArgs* jobs, int njobs, cudaStream_t stream);

// Launch one pass.  Returns ME_OK or an error code (error message set).
int launch_line_pass(int mode, const float2* in0, const float2* in1, float2* out0, float2* out1,
                     i64 in_vs, i64 out_vs, int nvol, const int dims[3], const i64 st[3], int axis,
                     const Phase& f0, const Phase& f1, const double* params, int pstride,
                     int accum, cudaStream_t stream);

}  // namespace me
