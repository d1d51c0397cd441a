// Line-pass kernels (see line_pass.cuh).  One CTA owns a tile of B lines of one volume, loads
// it into shared memory with coalesced accesses (rows of B consecutive lines along the
// contiguous axis, or whole contiguous lines), runs the FFT, the phase and the inverse FFT
// there, and writes the tile back.  Tiles are disjoint, so in == out is safe.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "fft_reg.cuh"
#include "line_pass.cuh"

namespace me {

ME_WAIT_FAULT_ACCESSOR(line_pass_wait_fault)

// The compile-time kernels handle every length in ME_FAST_LENGTHS; ME_GENERIC_FFT=1 in the
// environment forces the runtime-plan kernel for all lengths (used by the tests to cover it).
static bool fast_passes_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ME_GENERIC_FFT");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

// Resident CTAs per SM the compile-time pass kernels are compiled for.
#ifndef ME_PASS_MINB
#define ME_PASS_MINB 2
#endif
// 1: the two-line-set (dual) modes keep one tile buffer instead of two, so that two CTAs fit
// on an SM (the next tile is then loaded after the current one is stored, not during it, and
// the other CTA's work covers the load).  Measured on the LM statistics at 256x224x176:
// 696 ms against 712 ms with two buffers and one CTA per SM.
#ifndef ME_DUAL_SINGLE_BUFFER
#define ME_DUAL_SINGLE_BUFFER 1
#endif

struct PhaseCoef {
  double a, b, dm;
};

__device__ __forceinline__ PhaseCoef phase_coef(const Phase& P, const double* prm, int ax) {
  PhaseCoef c{0.0, 0.0, 0.0};
  if (P.kind != PH_NONE) {
    const double th = prm[3 + P.rot];
    if (P.kind == PH_TAN) {
      const double t = tan(th * 0.5);
      c.a = t;
      c.dm = 0.5 * (1.0 + t * t);
    } else {
      c.a = -sin(th);
      c.dm = -cos(th);
    }
  }
  if (P.trans) c.b = -prm[ax];
  return c;
}

__device__ __forceinline__ bool phase_is_identity(const Phase& P) {
  return P.kind == PH_NONE && !P.trans && !P.trans_deriv && !P.deriv;
}

// Phase factor for frequency index n along the pass axis at spatial coordinates c[0..2]
// (c[ax] is ignored by the planes, which are constant or broadcast along the pass axis in
// frequency; c[ax] carries n itself).
__device__ __forceinline__ float2 phase_value(const Phase& P, const PhaseCoef& C, int n,
                                              const int c[3], float scale) {
  double rk = 0.0, kn = 0.0;
  if (P.plane) rk = P.plane[c[0] * P.ps[0] + c[1] * P.ps[1] + c[2] * P.ps[2]];
  if (P.kv) kn = P.kv[n];
  float2 e = expi_reduced(C.a * rk + C.b * kn);
  if (P.deriv) e = cscale(mul_i(e), (float)(C.dm * rk));
  if (P.trans_deriv) e = cscale(mul_mi(e), (float)kn);
  if (P.conj) e = cconj(e);
  return cscale(e, scale);
}

// Global element offset of (line l, index n) inside a volume.
__device__ __forceinline__ i64 elem_offset(const PassArgs& A, int l, int n) {
  const int u = l / A.dims[A.av];
  const int v = l - u * A.dims[A.av];
  return (i64)u * A.st[A.au] + (i64)v * A.st[A.av] + (i64)n * A.st[A.ax];
}

__device__ __forceinline__ void line_coords(const PassArgs& A, int l, int n, int c[3]) {
  const int u = l / A.dims[A.av];
  const int v = l - u * A.dims[A.av];
  c[A.au] = u;
  c[A.av] = v;
  c[A.ax] = n;
}

// Load B lines (starting at line l0) of volume `src` into buf lines [dst_line0, dst_line0+B).
__device__ __forceinline__ void load_tile(const PassArgs& A, const float2* __restrict__ src,
                                          int l0, int nl, float2* buf, int dst_line0) {
  const int N = A.plan.n;
  const int B = A.B;
  if (A.st[A.av] == 1) {
    for (int t = threadIdx.x; t < B * N; t += blockDim.x) {
      const int b = t % B, n = t / B;
      float2 v = make_float2(0.f, 0.f);
      if (b < nl) v = src[elem_offset(A, l0 + b, n)];
      buf[n * A.es + dst_line0 + b] = v;
    }
  } else {
    for (int t = threadIdx.x; t < B * N; t += blockDim.x) {
      const int n = t % N, b = t / N;
      float2 v = make_float2(0.f, 0.f);
      if (b < nl) v = src[elem_offset(A, l0 + b, n)];
      buf[n * A.es + dst_line0 + b] = v;
    }
  }
}

__device__ __forceinline__ void store_tile(const PassArgs& A, float2* __restrict__ dst, int l0,
                                           int nl, const float2* buf, int src_line0, bool accum) {
  const int N = A.plan.n;
  const int B = A.B;
  const bool bfast = (A.st[A.av] == 1);
  for (int t = threadIdx.x; t < B * N; t += blockDim.x) {
    int b, n;
    if (bfast) {
      b = t % B;
      n = t / B;
    } else {
      n = t % N;
      b = t / N;
    }
    if (b >= nl) continue;
    const i64 off = elem_offset(A, l0 + b, n);
    float2 v = buf[n * A.es + src_line0 + b];
    if (accum) v = cadd(v, dst[off]);
    dst[off] = v;
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) line_pass_kernel(const PassArgs A) {
  extern __shared__ float2 smem[];
  const int N = A.plan.n;
  const int vol = blockIdx.y;
  const int l0 = blockIdx.x * A.B;
  const int nl = min(A.B, A.nlines - l0);
  const int B = A.B;

  float2* tw = smem;
  float2* b0 = smem + ((N + 1) & ~1);
  float2* b1 = b0 + (i64)N * A.es;

  const double* prm = A.params ? A.params + (i64)vol * A.pstride : nullptr;
  PhaseCoef c0{0, 0, 0}, c1{0, 0, 0};
  if (prm) {
    c0 = phase_coef(A.ph[0], prm, A.ax);
    if (MODE == PM_DUAL_OUT || MODE == PM_DUAL_IN) c1 = phase_coef(A.ph[1], prm, A.ax);
  }
  const bool id0 = phase_is_identity(A.ph[0]);
  const bool id1 = phase_is_identity(A.ph[1]);

  init_twiddles(tw, N);
  const float2* in0 = A.in0 + (i64)vol * A.in_vs;
  load_tile(A, in0, l0, nl, b0, 0);
  if (MODE == PM_DUAL_IN) {
    const float2* in1 = A.in1 + (i64)vol * A.in_vs;
    load_tile(A, in1, l0, nl, b0, B);
  }
  __syncthreads();

  float2* R = b0;
  float2* S = b1;
  if (MODE != PM_INV) {
    const int nlines = (MODE == PM_DUAL_IN) ? 2 * B : B;
    R = fft_lines<false>(b0, b1, A.plan, nlines, A.es, tw);
    S = (R == b0) ? b1 : b0;
  }

  // phase multiply (and combine / split for the dual modes)
  for (int t = threadIdx.x; t < B * N; t += blockDim.x) {
    const int b = t % B, n = t / B;
    int c[3];
    line_coords(A, l0 + min(b, max(nl - 1, 0)), n, c);
    const float2 v0 = R[n * A.es + b];
    const float2 f0 = id0 ? make_float2(A.scale, 0.f) : phase_value(A.ph[0], c0, n, c, A.scale);
    if (MODE == PM_DUAL_OUT) {
      const float2 f1 = id1 ? make_float2(A.scale, 0.f) : phase_value(A.ph[1], c1, n, c, A.scale);
      R[n * A.es + b] = cmul(v0, f0);
      R[n * A.es + B + b] = cmul(v0, f1);
    } else if (MODE == PM_DUAL_IN) {
      const float2 f1 = id1 ? make_float2(A.scale, 0.f) : phase_value(A.ph[1], c1, n, c, A.scale);
      const float2 v1 = R[n * A.es + B + b];
      R[n * A.es + b] = cadd(cmul(v0, f0), cmul(v1, f1));
    } else {
      R[n * A.es + b] = cmul(v0, f0);
    }
  }
  __syncthreads();

  if (MODE != PM_FWD) {
    const int nlines = (MODE == PM_DUAL_OUT) ? 2 * B : B;
    R = fft_lines<true>(R, S, A.plan, nlines, A.es, tw);
  }

  float2* out0 = A.out0 + (i64)vol * A.out_vs;
  store_tile(A, out0, l0, nl, R, 0, A.accum != 0);
  if (MODE == PM_DUAL_OUT) {
    float2* out1 = A.out1 + (i64)vol * A.out_vs;
    store_tile(A, out1, l0, nl, R, B, false);
  }
}

// ------------------------------------------------------------------ compile-time lengths
// Same contract as line_pass_kernel, with the line FFT in registers (fft_reg.cuh): one group
// of G threads per line, B = 256 / G lines per tile, no CTA-wide barrier between FFT stages.
// CTAs are persistent over (volume, tile) work items and prefetch the next tile with
// asynchronous copies into a second buffer while the current one is transformed.

// Chirp of one line by recurrence along its elements n = j + r*R1 (r < R2):
// f = mult(n) * exp(i C (m(n) - N/2)), m(n) = (n - N/2) mod N, C = (a r_o + b) 2 pi / N.
template <int N, int R1, int R2>
struct LineChirp {
  float2 e, step, stepw;  // current factor (output scale folded in), step by R1, step with wrap
  int m;
  float dmr;   // deriv multiplier per unit (m - N/2): dm * r_o * 2 pi / N
  float tdr;   // translation-derivative multiplier per unit: 2 pi / N
  bool deriv, tderiv, conj;
  // A conjugated phase is conjugated once here: conj(e s^r) = conj(e) conj(s)^r, and the
  // i / -i of the derivative multipliers swap.  The two steps are the same for the G lanes of
  // a line: even lanes evaluate the plain step, odd lanes the wrapping one, and the line's
  // first two lanes hand them to the rest (every lane of the warp must call init).
  __device__ __forceinline__ void init(const Phase& P, const PhaseCoef& Cf, double r_o, int j,
                                       float scale, int G) {
    const double d = kTwoPi / N;
    const double C = (P.conj ? -1.0 : 1.0) * (Cf.a * r_o + Cf.b) * d;
    m = ((j - N / 2) % N + N) % N;
    e = cscale(expi_reduced(C * ((double)m - 0.5 * N)), scale);
    const float2 sv = expi_reduced(C * ((j & 1) ? (double)(R1 - N) : (double)R1));
    const int lead = (threadIdx.x & 31) & ~(G - 1);
    step = make_float2(__shfl_sync(0xffffffffu, sv.x, lead), __shfl_sync(0xffffffffu, sv.y, lead));
    stepw = make_float2(__shfl_sync(0xffffffffu, sv.x, lead + 1),
                        __shfl_sync(0xffffffffu, sv.y, lead + 1));
    dmr = (float)(Cf.dm * r_o * d);
    tdr = (float)d;
    deriv = P.deriv != 0;
    tderiv = P.trans_deriv != 0;
    conj = P.conj != 0;
  }
  __device__ __forceinline__ float2 value() const {
    float2 f = e;
    const float mm = (float)m - 0.5f * N;
    if (deriv) f = cscale(conj ? mul_mi(f) : mul_i(f), dmr * mm);
    if (tderiv) f = cscale(conj ? mul_i(f) : mul_mi(f), tdr * mm);
    return f;
  }
  __device__ __forceinline__ void advance() {
    m += R1;
    if (m >= N) {
      m -= N;
      e = cmul(e, stepw);
    } else {
      e = cmul(e, step);
    }
  }
  // V[r] *= f(j + r R1) for the thread's R2 elements, with the branch on the multiplier taken
  // once for the line rather than per element
  __device__ __forceinline__ void apply(float2 (&V)[R2]) {
    if (deriv || tderiv) {
#pragma unroll
      for (int r = 0; r < R2; r++) {
        V[r] = cmul(V[r], value());
        advance();
      }
    } else {
#pragma unroll
      for (int r = 0; r < R2; r++) {
        V[r] = cmul(V[r], e);
        advance();
      }
    }
  }
};

template <int N, int R1, int R2, int MODE>
__global__ void __launch_bounds__(256, ME_PASS_MINB) fast_pass_kernel(const PassArgs A) {
  using F = LineFft<N, R1, R2>;
  using Ch = LineChirp<N, R1, R2>;
  constexpr int G = F::G;
  constexpr int B = 256 / G;
  constexpr int LS = F::LS;
  constexpr bool kDual = (MODE == PM_DUAL_IN || MODE == PM_DUAL_OUT);
  constexpr int NREG = kDual ? 2 * B : B;
  constexpr int NBUF = (kDual && ME_DUAL_SINGLE_BUFFER) ? 1 : 2;  // tile buffers
  extern __shared__ __align__(16) float2 smem[];
  __shared__ i64 lb_s[2][B];  // line base offsets of the tile in each buffer

  const int tiles_per_vol = (A.nlines + B - 1) / B;
  const int total = tiles_per_vol * A.nvol;
  const i64 sa = A.st[A.ax];
  const bool bfast = (A.st[A.av] == 1);
  const int dv = A.dims[A.av];
  const int g = threadIdx.x / G;
  const int j = threadIdx.x % G;
  const bool id0 = phase_is_identity(A.ph[0]);
  const bool id1 = phase_is_identity(A.ph[1]);

  auto line_base = [&](int l) {
    const int u = A.div_av.div(l);
    return (i64)u * A.st[A.au] + (i64)(l - u * dv) * A.st[A.av];
  };
  // issue the loads of work item t into buffer `bufi`; line offsets computed once per line
  // (the caller has synchronised, so lb_s[bufi] is free)
  auto issue = [&](int t, int bufi) {
    const int vol = A.div_tiles.div(t);
    const int l0 = (t - vol * tiles_per_vol) * B;
    const int nl = min(B, A.nlines - l0);
    float2* buf = smem + bufi * NREG * LS;
    if (threadIdx.x < B) lb_s[bufi][threadIdx.x] = line_base(l0 + min((int)threadIdx.x, nl - 1));
    // each thread computes the offsets of the lines it copies itself (no barrier needed)
    const int nsrc = (MODE == PM_DUAL_IN) ? 2 : 1;
    for (int k = 0; k < nsrc; k++) {
      const float2* src = (k == 0 ? A.in0 : A.in1) + (i64)vol * A.in_vs;
      if (bfast) {
        // b = e % B is fixed per thread (256 is a multiple of B)
        const int b = threadIdx.x % B;
        const i64 base = line_base(l0 + min(b, nl - 1));
        float2* dst0 = buf + (k * B + b) * LS;
        for (int n = threadIdx.x / B; n < N; n += 256 / B) {
          if (b < nl) cp_async8(dst0 + n, src + base + n * sa);
          else dst0[n] = make_float2(0.f, 0.f);
        }
      } else {
        // contiguous lines: one line per group of G = 256 / B threads, n fastest
        const int b = threadIdx.x / G;
        const i64 base = line_base(l0 + min(b, nl - 1));
        float2* dst0 = buf + (k * B + b) * LS;
        for (int n = threadIdx.x % G; n < N; n += G) {
          if (b < nl) cp_async8(dst0 + n, src + base + n * sa);
          else dst0[n] = make_float2(0.f, 0.f);
        }
      }
    }
    cp_async_commit();
  };

  int cur = 0;
  // The shear coefficients depend on the volume only: one thread sets them up in shared memory
  // when the CTA moves to another volume (vol is uniform over the CTA, so the barrier is too).
  __shared__ PhaseCoef coef_s[2];
  int coef_vol = -1;
  if ((int)blockIdx.x < total) issue(blockIdx.x, 0);
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    const int vol = A.div_tiles.div(t);
    const int l0 = (t - vol * tiles_per_vol) * B;
    const int nl = min(B, A.nlines - l0);
    cp_async_wait_all();
    __syncthreads();
    if (NBUF == 2 && t + (int)gridDim.x < total) issue(t + gridDim.x, cur ^ 1);
    float2* buf = smem + cur * NREG * LS;

    // per-line phase set-up
    if (vol != coef_vol) {
      if (threadIdx.x < (kDual ? 2 : 1)) {
        PhaseCoef cf{0, 0, 0};
        if (A.params) cf = phase_coef(A.ph[threadIdx.x], A.params + (i64)vol * A.pstride, A.ax);
        coef_s[threadIdx.x] = cf;
      }
      coef_vol = vol;
      __syncthreads();
    }
    const int l = l0 + min(g, nl - 1);
    int c[3];
    {
      const int u = A.div_av.div(l);
      c[A.au] = u;
      c[A.av] = l - u * dv;
      c[A.ax] = 0;
    }
    Ch ch0, ch1;
    const bool sep0 = !id0 && A.ph[0].sep;
    const bool sep1 = kDual && !id1 && A.ph[1].sep;
    const PhaseCoef c0 = coef_s[0];
    const PhaseCoef c1 = kDual ? coef_s[1] : PhaseCoef{0, 0, 0};
    if (sep0) ch0.init(A.ph[0], c0, A.ph[0].rvec ? A.ph[0].rvec[c[A.ph[0].oaxis]] : 0.0, j, A.scale, G);
    if (sep1) ch1.init(A.ph[1], c1, A.ph[1].rvec ? A.ph[1].rvec[c[A.ph[1].oaxis]] : 0.0, j, A.scale, G);
    // V (element n = j + r R1 in slot r) times the factors of phase 0 or 1; which form applies
    // (identity, line chirp, per-element evaluation) is decided once per line
    auto factor0 = [&](float2 (&V)[R2]) {
      if (id0) {
#pragma unroll
        for (int r = 0; r < R2; r++) V[r] = cscale(V[r], A.scale);
      } else if (sep0) {
        ch0.apply(V);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          V[r] = cmul(V[r], phase_value(A.ph[0], c0, j + r * R1, c, A.scale));
        }
      }
    };
    auto factor1 = [&](float2 (&V)[R2]) {
      if (id1) {
#pragma unroll
        for (int r = 0; r < R2; r++) V[r] = cscale(V[r], A.scale);
      } else if (sep1) {
        ch1.apply(V);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          V[r] = cmul(V[r], phase_value(A.ph[1], c1, j + r * R1, c, A.scale));
        }
      }
    };

    float2* L0 = buf + g * LS;
    float2* L1 = buf + (B + g) * LS;
    float2 X[R2];
    if (MODE == PM_INV) {
      F::load_spectrum(L0, j, X);
    } else {
      F::forward(L0, j, X);
    }
    if (MODE == PM_DUAL_IN) {
      float2 Y[R2];
      F::forward(L1, j, Y);
      if (j < R1) {
        factor0(X);
        factor1(Y);
#pragma unroll
        for (int r = 0; r < R2; r++) X[r] = cadd(X[r], Y[r]);
      }
      F::inverse(L0, j, X);
    } else if (MODE == PM_DUAL_OUT) {
      float2 Y[R2];
      if (j < R1) {
#pragma unroll
        for (int r = 0; r < R2; r++) Y[r] = X[r];
        factor0(X);
        factor1(Y);
      }
      F::inverse(L0, j, X);
      F::inverse(L1, j, Y);
    } else {
      if (j < R1) factor0(X);
      if (MODE == PM_FWD) {
        F::store_spectrum(L0, j, X);
      } else {
        F::inverse(L0, j, X);
      }
    }
    __syncthreads();
    // store the tile
    const int nout = (MODE == PM_DUAL_OUT) ? 2 : 1;
    for (int k = 0; k < nout; k++) {
      float2* dst = (k == 0 ? A.out0 : A.out1) + (i64)vol * A.out_vs;
      const bool acc = (k == 0) && A.accum;
      if (bfast) {
        const int b = threadIdx.x % B;
        if (b < nl) {
          const i64 base = lb_s[cur][b];
          const float2* s0 = buf + (k * B + b) * LS;
          for (int n = threadIdx.x / B; n < N; n += 256 / B) {
            float2 v = s0[n];
            if (acc) v = cadd(v, dst[base + n * sa]);
            dst[base + n * sa] = v;
          }
        }
      } else {
        const int b = threadIdx.x / G;
        if (b < nl) {
          const i64 base = lb_s[cur][b];
          const float2* s0 = buf + (k * B + b) * LS;
          for (int n = threadIdx.x % G; n < N; n += G) {
            float2 v = s0[n];
            if (acc) v = cadd(v, dst[base + n * sa]);
            dst[base + n * sa] = v;
          }
        }
      }
    }
    if (NBUF == 1) {
      __syncthreads();  // the store above has read the buffer the next tile goes into
      if (t + (int)gridDim.x < total) issue(t + gridDim.x, 0);
    } else {
      cur ^= 1;
    }
  }
  cp_async_wait_all();
}

// ------------------------------------------------------------------ TMA tile staging
// The same pass with each tile of B = 256 / G lines (16 lines of 16 threads, or 32 of 8) moved
// by the TMA engine: one thread issues tiled tensor loads of the next tile (completing on an
// mbarrier) and tiled tensor stores of the finished one, so no thread issues per-element global
// loads or stores.  Used for the compile-time lengths when the lines of a tile are B
// consecutive lines of one row (dims[av] a multiple of B) and every stride is a multiple of 16
// bytes:
//   strided lines (st[av] == 1): B / 16 sub-tiles [n][16 lines], each with the tensor map's
//     128-byte swizzle (the 16-byte chunk index XOR n mod 8), so that the lanes of a line read
//     and write distinct banks;
//   contiguous lines (st[ax] == 1): tile [B lines][n], dense.
// The FFT reads its line from the tile and hands its outputs back to the same places (a line
// belongs to one thread group); its transposes use a padded scratch region per group.
struct PassTma {
  CUtensorMap in[2];
  CUtensorMap out[2];
  int in_rank[2];   // 3: one volume (or a broadcast input), 4: indexed by volume
  int out_rank[2];
};

template <int N, int B, bool STRIDED>
__device__ __forceinline__ int tile_off(int b, int n) {
  if (STRIDED) {
    const int sub = (B == 16) ? 0 : (b >> 4);  // 16-line sub-tile
    const int bb = b & 15;
    return sub * (16 * N * 8) + n * 128 + ((((bb >> 1) ^ n) & 7) << 4) + ((bb & 1) << 3);
  }
  return (b * N + n) * 8;
}

template <int N, int R1, int R2, int MODE, bool STRIDED>
__global__ void __launch_bounds__(256, ME_PASS_MINB)
    tma_pass_kernel(const __grid_constant__ PassArgs A, const __grid_constant__ PassTma T) {
  using F = LineFft<N, R1, R2>;
  using Ch = LineChirp<N, R1, R2>;
  constexpr int G = F::G;
  constexpr int B = 256 / G;                      // lines per tile, one per thread group
  constexpr int NSUB = STRIDED ? B / 16 : 1;       // tensor copies per tile and operand
  constexpr int LS = F::LS;
  constexpr bool kDual = (MODE == PM_DUAL_IN || MODE == PM_DUAL_OUT);
  constexpr int NT = kDual ? 2 : 1;  // tiles per buffer
  constexpr int NBUF = (kDual && ME_DUAL_SINGLE_BUFFER) ? 1 : 2;
  constexpr int NIN = (MODE == PM_DUAL_IN) ? 2 : 1;
  constexpr int NOUT = (MODE == PM_DUAL_OUT) ? 2 : 1;
  constexpr int TILE = B * N * 8;  // bytes; a multiple of 1024 for every length used here
  constexpr int SUBT = TILE / NSUB;
  static_assert(SUBT % 1024 == 0, "swizzled sub-tiles start on 1024-byte boundaries");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the swizzle pattern repeats every 1024 bytes of shared-memory address
  unsigned char* tiles = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  float2* scratch = reinterpret_cast<float2*>(tiles + NBUF * NT * TILE);
  __shared__ __align__(8) uint64_t full[NBUF];
  __shared__ PhaseCoef coef_s[2];

  const int tiles_per_vol = A.nlines / B;
  const int total = tiles_per_vol * A.nvol;
  const int dv = A.dims[A.av];
  const int g = threadIdx.x / G;
  const int j = threadIdx.x % G;
  const bool id0 = phase_is_identity(A.ph[0]);
  const bool id1 = phase_is_identity(A.ph[1]);

  if (threadIdx.x == 0) {
    for (int i = 0; i < NBUF; i++) mbar_init(&full[i], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto coords = [&](int t, int& vol, int& u, int& v0) {
    vol = A.div_tiles.div(t);
    const int l0 = (t - vol * tiles_per_vol) * B;
    u = A.div_av.div(l0);
    v0 = l0 - u * dv;
  };
  // thread 0: load work item t into buffer bufi, once the stores out of that buffer have read it
  auto issue = [&](int t, int bufi) {
    int vol, u, v0;
    coords(t, vol, u, v0);
    bulk_wait_read_all();
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&full[bufi], NIN * TILE);
#pragma unroll
    for (int k = 0; k < NIN; k++) {
#pragma unroll
      for (int q = 0; q < NSUB; q++) {
        unsigned char* dst = tiles + (bufi * NT + k) * TILE + q * SUBT;
        const int c0 = STRIDED ? v0 + 16 * q : 0, c1 = STRIDED ? 0 : v0;
        if (T.in_rank[k] == 3) {
          tma_load_3d(dst, &T.in[k], c0, c1, u, &full[bufi]);
        } else {
          tma_load_4d(dst, &T.in[k], c0, c1, u, vol, &full[bufi]);
        }
      }
    }
  };

  if (threadIdx.x == 0 && (int)blockIdx.x < total) issue(blockIdx.x, 0);
  int coef_vol = -1;
  int it = 0;
  for (int t = blockIdx.x; t < total; t += gridDim.x, it++) {
    const int cur = (NBUF == 2) ? (it & 1) : 0;
    const unsigned parity = (NBUF == 2) ? ((it >> 1) & 1) : (it & 1);
    int vol, u, v0;
    coords(t, vol, u, v0);
    mbar_wait_bounded(&full[cur], parity, WF_LINE_PASS);
    if (NBUF == 2 && threadIdx.x == 0 && t + (int)gridDim.x < total) issue(t + gridDim.x, cur ^ 1);
    // the shear coefficients depend on the volume only (the barrier before the previous
    // tile's store separates every read of coef_s from this write)
    if (vol != coef_vol) {
      if (threadIdx.x < (kDual ? 2 : 1)) {
        PhaseCoef cf{0, 0, 0};
        if (A.params) cf = phase_coef(A.ph[threadIdx.x], A.params + (i64)vol * A.pstride, A.ax);
        coef_s[threadIdx.x] = cf;
      }
      coef_vol = vol;
      __syncthreads();
    }
    int c[3];
    c[A.au] = u;
    c[A.av] = v0 + g;
    c[A.ax] = 0;
    Ch ch0, ch1;
    const bool sep0 = !id0 && A.ph[0].sep;
    const bool sep1 = kDual && !id1 && A.ph[1].sep;
    const PhaseCoef c0 = coef_s[0];
    const PhaseCoef c1 = kDual ? coef_s[1] : PhaseCoef{0, 0, 0};
    if (sep0) ch0.init(A.ph[0], c0, A.ph[0].rvec ? A.ph[0].rvec[c[A.ph[0].oaxis]] : 0.0, j, A.scale, G);
    if (sep1) ch1.init(A.ph[1], c1, A.ph[1].rvec ? A.ph[1].rvec[c[A.ph[1].oaxis]] : 0.0, j, A.scale, G);
    auto factor0 = [&](float2 (&V)[R2]) {
      if (id0) {
#pragma unroll
        for (int r = 0; r < R2; r++) V[r] = cscale(V[r], A.scale);
      } else if (sep0) {
        ch0.apply(V);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          V[r] = cmul(V[r], phase_value(A.ph[0], c0, j + r * R1, c, A.scale));
        }
      }
    };
    auto factor1 = [&](float2 (&V)[R2]) {
      if (id1) {
#pragma unroll
        for (int r = 0; r < R2; r++) V[r] = cscale(V[r], A.scale);
      } else if (sep1) {
        ch1.apply(V);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          V[r] = cmul(V[r], phase_value(A.ph[1], c1, j + r * R1, c, A.scale));
        }
      }
    };

    unsigned char* tb0 = tiles + (cur * NT) * TILE;
    unsigned char* tb1 = tiles + (cur * NT + 1) * TILE;
    auto load0 = [&](int n) { return *reinterpret_cast<const float2*>(tb0 + tile_off<N, B, STRIDED>(g, n)); };
    auto load1 = [&](int n) { return *reinterpret_cast<const float2*>(tb1 + tile_off<N, B, STRIDED>(g, n)); };
    auto store0 = [&](int, int n, float2 v) { *reinterpret_cast<float2*>(tb0 + tile_off<N, B, STRIDED>(g, n)) = v; };
    auto store1 = [&](int, int n, float2 v) { *reinterpret_cast<float2*>(tb1 + tile_off<N, B, STRIDED>(g, n)) = v; };
    float2* L = scratch + g * LS;
    float2 X[R2];
    F::forward_from(load0, L, j, X);
    if (MODE == PM_DUAL_IN) {
      float2 Y[R2];
      F::forward_from(load1, L, j, Y);
      if (j < R1) {
        factor0(X);
        factor1(Y);
#pragma unroll
        for (int r = 0; r < R2; r++) X[r] = cadd(X[r], Y[r]);
      }
      F::inverse_to(L, j, X, store0);
    } else if (MODE == PM_DUAL_OUT) {
      float2 Y[R2];
      if (j < R1) {
#pragma unroll
        for (int r = 0; r < R2; r++) Y[r] = X[r];
        factor0(X);
        factor1(Y);
      }
      F::inverse_to(L, j, X, store0);
      F::inverse_to(L, j, Y, store1);
    } else {
      if (j < R1) factor0(X);
      F::inverse_to(L, j, X, store0);
    }
    // the tile's generic-proxy writes are ordered before the async-proxy store
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NOUT; k++) {
#pragma unroll
        for (int q = 0; q < NSUB; q++) {
          const unsigned char* src = tiles + (cur * NT + k) * TILE + q * SUBT;
          const int c0s = STRIDED ? v0 + 16 * q : 0, c1s = STRIDED ? 0 : v0;
          if (T.out_rank[k] == 3) {
            tma_store_3d(&T.out[k], src, c0s, c1s, u);
          } else {
            tma_store_4d(&T.out[k], src, c0s, c1s, u, vol);
          }
        }
      }
      bulk_commit();
      if (NBUF == 1 && t + (int)gridDim.x < total) issue(t + gridDim.x, 0);
    }
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// ME_NO_TMA=1 in the environment keeps every pass on the cp.async kernel (for comparisons).
static bool tma_passes_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ME_NO_TMA");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of one operand of a TMA pass (8-byte elements; boxes of 16 strided lines or of B
// contiguous lines); rank 3 when the operand is one volume, else rank 4 with the volume index
// outermost.
static bool encode_pass_map(CUtensorMap* m, const void* base, const PassArgs& A, bool strided,
                            i64 vs, int rank, int B) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const int N = A.dims[A.ax];
  cuuint64_t dims[4];
  cuuint64_t strides[3];
  cuuint32_t box[4];
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (strided) {
    dims[0] = (cuuint64_t)A.dims[A.av];
    dims[1] = (cuuint64_t)N;
    strides[0] = (cuuint64_t)A.st[A.ax] * 8;
    box[0] = 16;
    box[1] = (cuuint32_t)N;
  } else {
    dims[0] = (cuuint64_t)N;
    dims[1] = (cuuint64_t)A.dims[A.av];
    strides[0] = (cuuint64_t)A.st[A.av] * 8;
    box[0] = (cuuint32_t)N;
    box[1] = (cuuint32_t)B;
  }
  dims[2] = (cuuint64_t)A.dims[A.au];
  strides[1] = (cuuint64_t)A.st[A.au] * 8;
  box[2] = 1;
  dims[3] = (cuuint64_t)A.nvol;
  strides[2] = (cuuint64_t)vs * 8;
  box[3] = 1;
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank,
                         const_cast<void*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE,
                         strided ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Whether pass A (mode, tiles of B lines) can run on the TMA kernel; fills the tensor maps.
static bool tma_pass_setup(int mode, const PassArgs& A, int B, bool* strided, PassTma* T) {
  if (!tma_passes_enabled()) return false;
  if (mode != PM_SHEAR && mode != PM_DUAL_OUT && mode != PM_DUAL_IN) return false;
  if (A.accum) return false;
  const int dv = A.dims[A.av];
  if (dv % B != 0) return false;
  const bool s = (A.st[A.av] == 1);
  if (!s && A.st[A.ax] != 1) return false;
  const i64 other = s ? A.st[A.ax] : A.st[A.av];
  if (other % 2 != 0 || A.st[A.au] % 2 != 0) return false;
  const i64 lim = (i64)1 << 36;  // strides below 2^40 bytes
  if (other >= lim || A.st[A.au] >= lim || A.in_vs >= lim || A.out_vs >= lim) return false;
  const int nin = (mode == PM_DUAL_IN) ? 2 : 1, nout = (mode == PM_DUAL_OUT) ? 2 : 1;
  const float2* ins[2] = {A.in0, A.in1};
  float2* outs[2] = {A.out0, A.out1};
  for (int k = 0; k < nin; k++) {
    if ((uintptr_t)ins[k] % 16 != 0) return false;
    const bool one = (A.in_vs == 0 || A.nvol == 1);
    if (!one && A.in_vs % 2 != 0) return false;
    T->in_rank[k] = one ? 3 : 4;
    if (!encode_pass_map(&T->in[k], ins[k], A, s, A.in_vs, T->in_rank[k], B)) return false;
  }
  for (int k = 0; k < nout; k++) {
    if ((uintptr_t)outs[k] % 16 != 0) return false;
    const bool one = (A.nvol == 1);
    if (!one && A.out_vs % 2 != 0) return false;
    T->out_rank[k] = one ? 3 : 4;
    if (!encode_pass_map(&T->out[k], outs[k], A, s, A.out_vs, T->out_rank[k], B)) return false;
  }
  *strided = s;
  return true;
}

template <int N, int R1, int R2, int MODE, bool STRIDED>
static int launch_tma(PassArgs& A, const PassTma& T, cudaStream_t stream) {
  using F = LineFft<N, R1, R2>;
  constexpr bool kDual = (MODE == PM_DUAL_IN || MODE == PM_DUAL_OUT);
  constexpr int NBUF = (kDual && ME_DUAL_SINGLE_BUFFER) ? 1 : 2;
  constexpr int B = 256 / F::G;
  const size_t smem = 1024 + (size_t)NBUF * (kDual ? 2 : 1) * B * N * 8 +
                      sizeof(float2) * (size_t)F::LS * B;
  A.div_tiles.set(A.nlines / B);
  auto kern = tma_pass_kernel<N, R1, R2, MODE, STRIDED>;
  const int rc = check_cuda(allow_smem(kern, smem), "tma pass smem");
  if (rc != ME_OK) return rc;
  static int occ[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 8 && occ[dev] == 0) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, smem);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    occ[dev] = std::max(1, nb) * std::max(1, sms);
  }
  const long long tiles = (long long)(A.nlines / B) * A.nvol;
  const int grid = (int)std::min<long long>(tiles, dev < 8 ? occ[dev] : 148 * 2);
  count_launch();
  kern<<<grid, 256, smem, stream>>>(A, T);
  return check_cuda(cudaGetLastError(), "tma pass launch");
}

template <int N, int R1, int R2, int MODE>
static int launch_fast(PassArgs& A, cudaStream_t stream) {
  using F = LineFft<N, R1, R2>;
  if constexpr (MODE == PM_SHEAR || MODE == PM_DUAL_OUT || MODE == PM_DUAL_IN) {
    PassTma T;
    bool strided = false;
    if (tma_pass_setup(MODE, A, 256 / F::G, &strided, &T))
      return strided ? launch_tma<N, R1, R2, MODE, true>(A, T, stream)
                     : launch_tma<N, R1, R2, MODE, false>(A, T, stream);
  }
  constexpr int B = 256 / F::G;
  constexpr bool kDual = (MODE == PM_DUAL_IN || MODE == PM_DUAL_OUT);
  const size_t smem = sizeof(float2) * (size_t)F::LS * B * (kDual ? 2 : 1) *
                      ((kDual && ME_DUAL_SINGLE_BUFFER) ? 1 : 2);
  A.div_tiles.set((A.nlines + B - 1) / B);
  const int rc = check_cuda(allow_smem(fast_pass_kernel<N, R1, R2, MODE>, smem), "pass smem");
  if (rc != ME_OK) return rc;
  static int occ[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 8 && occ[dev] == 0) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fast_pass_kernel<N, R1, R2, MODE>, 256, smem);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    occ[dev] = std::max(1, nb) * std::max(1, sms);
  }
  const long long tiles = (long long)((A.nlines + B - 1) / B) * A.nvol;
  const int grid = (int)std::min<long long>(tiles, dev < 8 ? occ[dev] : 148 * 2);
  count_launch();
  fast_pass_kernel<N, R1, R2, MODE><<<grid, 256, smem, stream>>>(A);
  return check_cuda(cudaGetLastError(), "fast pass launch");
}

template <int N, int R1, int R2>
static int launch_fast_mode(int mode, PassArgs& A, cudaStream_t stream) {
  switch (mode) {
    case PM_SHEAR: return launch_fast<N, R1, R2, PM_SHEAR>(A, stream);
    case PM_DUAL_OUT: return launch_fast<N, R1, R2, PM_DUAL_OUT>(A, stream);
    case PM_DUAL_IN: return launch_fast<N, R1, R2, PM_DUAL_IN>(A, stream);
    case PM_FWD: return launch_fast<N, R1, R2, PM_FWD>(A, stream);
    default: return launch_fast<N, R1, R2, PM_INV>(A, stream);
  }
}

// Returns ME_OK / error if handled by a compile-time kernel, -1 if N has no such kernel.
static int try_fast(int mode, PassArgs& A, cudaStream_t stream) {
  switch (A.plan.n) {
#define ME_FAST_CASE(N, R1, R2) \
  case N: return launch_fast_mode<N, R1, R2>(mode, A, stream);
    ME_FAST_LENGTHS(ME_FAST_CASE)
#undef ME_FAST_CASE
    default: return -1;
  }
}

static int pick_B(int N) {
  int B = 16;
  while (B > 4 && N * B > 4096) B /= 2;
  return B;
}

template <int MODE>
static int launch_mode(PassArgs& A, cudaStream_t stream) {
  const int N = A.plan.n;
  const bool dual = (MODE == PM_DUAL_IN || MODE == PM_DUAL_OUT);
  A.es = (dual ? 2 * A.B : A.B) + 1;
  const size_t smem = sizeof(float2) * (((N + 1) & ~1) + 2 * (size_t)N * A.es);
  {
    const int rc = check_cuda(allow_smem(line_pass_kernel<MODE>, smem), "line_pass smem");
    if (rc != ME_OK) return rc;
  }
  dim3 grid((A.nlines + A.B - 1) / A.B, A.nvol);
  count_launch();
  line_pass_kernel<MODE><<<grid, 256, smem, stream>>>(A);
  return check_cuda(cudaGetLastError(), "line_pass launch");
}

int make_pass_args(int mode, const float2* in0, const float2* in1, float2* out0, float2* out1,
                   i64 in_vs, i64 out_vs, int nvol, const int dims[3], const i64 st[3], int axis,
                   const Phase& f0, const Phase& f1, const double* params, int pstride, int accum,
                   PassArgs* out) {
  if (axis < 0 || axis > 2) return fail("line pass: axis must be 0, 1 or 2");
  PassArgs A{};
  A.in0 = in0;
  A.in1 = in1;
  A.out0 = out0;
  A.out1 = out1;
  A.in_vs = in_vs;
  A.out_vs = out_vs;
  A.nvol = nvol;
  for (int i = 0; i < 3; i++) {
    A.dims[i] = dims[i];
    A.st[i] = st[i];
  }
  A.ax = axis;
  int o1 = (axis + 1) % 3, o2 = (axis + 2) % 3;
  // av: the other axis with the smaller stride (the coalescing axis)
  if (st[o1] <= st[o2]) {
    A.av = o1;
    A.au = o2;
  } else {
    A.av = o2;
    A.au = o1;
  }
  A.nlines = dims[A.au] * dims[A.av];
  A.div_av.set(dims[A.av]);
  const int N = dims[axis];
  if (N > ME_MAX_LINE) return fail("line pass: line length exceeds ME_MAX_LINE");
  if (!make_plan(N, &A.plan)) {
    set_error("line pass: line length has a prime factor > 13");
    return ME_ERR_UNSUPPORTED;
  }
  A.B = pick_B(N);
  A.accum = accum;
  A.params = params;
  A.pstride = pstride;
  A.ph[0] = f0;
  A.ph[1] = f1;
  switch (mode) {
    case PM_SHEAR:
    case PM_DUAL_OUT:
    case PM_DUAL_IN:
      A.scale = 1.0f / (float)N;
      break;
    default:
      A.scale = (float)(1.0 / sqrt((double)N));
  }
  *out = A;
  return ME_OK;
}

int launch_line_pass(int mode, const float2* in0, const float2* in1, float2* out0, float2* out1,
                     i64 in_vs, i64 out_vs, int nvol, const int dims[3], const i64 st[3], int axis,
                     const Phase& f0, const Phase& f1, const double* params, int pstride,
                     int accum, cudaStream_t stream) {
  if (axis < 0 || axis > 2) return fail("line pass: axis must be 0, 1 or 2");
  if (nvol < 1) return ME_OK;
  PassArgs A;
  const int rc0 = make_pass_args(mode, in0, in1, out0, out1, in_vs, out_vs, nvol, dims, st, axis,
                                 f0, f1, params, pstride, accum, &A);
  if (rc0 != ME_OK) return rc0;
  if (A.nlines == 0) return ME_OK;
  if (fast_passes_enabled()) {
    const int rc = try_fast(mode, A, stream);
    if (rc >= 0) return rc;
  }
  switch (mode) {
    case PM_SHEAR: return launch_mode<PM_SHEAR>(A, stream);
    case PM_DUAL_OUT: return launch_mode<PM_DUAL_OUT>(A, stream);
    case PM_DUAL_IN: return launch_mode<PM_DUAL_IN>(A, stream);
    case PM_FWD: return launch_mode<PM_FWD>(A, stream);
    case PM_INV: return launch_mode<PM_INV>(A, stream);
    default: return fail("line pass: bad mode");
  }
}

// ------------------------------------------------------------------ several jobs in one launch
// One shear step (PM_SHEAR) of several independent jobs -- volumes of different
// reconstructions, of any sizes -- as one persistent launch per distinct line length along the
// step's axis.  Work items are (job, volume, tile of lines) over the jobs of that length; each
// CTA takes items in turn and runs them through the compile-time tile code of the length, the
// same arithmetic as fast_pass_kernel, so the results are bit-identical to separate launches.
// Two tile buffers per CTA: the next item, of whichever job, is loaded while the current one is
// transformed.  (A single launch that switched between the sixteen compiled lengths would carry
// all their register needs at once.)
struct MultiPassArgs {
  int njobs;
  int tile_off[kMaxMultiJobs + 1];  // prefix sums of the jobs' work items
  PassArgs job[kMaxMultiJobs];
};

template <int N, int R1, int R2>
__global__ void __launch_bounds__(256, ME_PASS_MINB)
    multi_shear_kernel(const __grid_constant__ MultiPassArgs M) {
  using F = LineFft<N, R1, R2>;
  using Ch = LineChirp<N, R1, R2>;
  constexpr int G = F::G;
  constexpr int B = 256 / G;
  constexpr int LS = F::LS;
  extern __shared__ __align__(16) float2 smem[];
  __shared__ i64 lb_s[2][B];  // line base offsets of the tile in each buffer
  __shared__ PhaseCoef coef_s;
  const int total = M.tile_off[M.njobs];
  const int g = threadIdx.x / G;
  const int j = threadIdx.x % G;
  auto job_of = [&](int t) {
    int k = 0;
    while (k + 1 < M.njobs && t >= M.tile_off[k + 1]) k++;
    return k;
  };
  // issue the loads of work item t into buffer `bufi` (the caller has synchronised)
  auto issue = [&](int t, int bufi) {
    const int k = job_of(t);
    const PassArgs& A = M.job[k];
    const int tt = t - M.tile_off[k];
    const int tiles_per_vol = (A.nlines + B - 1) / B;
    const int vol = A.div_tiles.div(tt);
    const int l0 = (tt - vol * tiles_per_vol) * B;
    const int nl = min(B, A.nlines - l0);
    const i64 sa = A.st[A.ax];
    const int dv = A.dims[A.av];
    auto line_base = [&](int l) {
      const int u = A.div_av.div(l);
      return (i64)u * A.st[A.au] + (i64)(l - u * dv) * A.st[A.av];
    };
    float2* buf = smem + bufi * B * LS;
    if (threadIdx.x < B) lb_s[bufi][threadIdx.x] = line_base(l0 + min((int)threadIdx.x, nl - 1));
    const float2* src = A.in0 + (i64)vol * A.in_vs;
    if (A.st[A.av] == 1) {
      const int b = threadIdx.x % B;
      const i64 base = line_base(l0 + min(b, nl - 1));
      float2* dst0 = buf + b * LS;
      for (int n = threadIdx.x / B; n < N; n += 256 / B) {
        if (b < nl) cp_async8(dst0 + n, src + base + n * sa);
        else dst0[n] = make_float2(0.f, 0.f);
      }
    } else {
      const int b = threadIdx.x / G;
      const i64 base = line_base(l0 + min(b, nl - 1));
      float2* dst0 = buf + b * LS;
      for (int n = threadIdx.x % G; n < N; n += G) {
        if (b < nl) cp_async8(dst0 + n, src + base + n * sa);
        else dst0[n] = make_float2(0.f, 0.f);
      }
    }
    cp_async_commit();
  };

  int cur = 0, coef_job = -1, coef_vol = -1;
  if ((int)blockIdx.x < total) issue(blockIdx.x, 0);
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    const int k = job_of(t);
    const PassArgs& A = M.job[k];
    const int tt = t - M.tile_off[k];
    const int tiles_per_vol = (A.nlines + B - 1) / B;
    const int vol = A.div_tiles.div(tt);
    const int l0 = (tt - vol * tiles_per_vol) * B;
    const int nl = min(B, A.nlines - l0);
    cp_async_wait_all();
    __syncthreads();
    if (t + (int)gridDim.x < total) issue(t + gridDim.x, cur ^ 1);
    float2* buf = smem + cur * B * LS;
    // the shear coefficients depend on the job and volume only (both uniform over the CTA)
    if (k != coef_job || vol != coef_vol) {
      if (threadIdx.x == 0) {
        PhaseCoef cf{0, 0, 0};
        if (A.params) cf = phase_coef(A.ph[0], A.params + (i64)vol * A.pstride, A.ax);
        coef_s = cf;
      }
      coef_job = k;
      coef_vol = vol;
      __syncthreads();
    }
    const bool id0 = phase_is_identity(A.ph[0]);
    const int dv = A.dims[A.av];
    const int l = l0 + min(g, nl - 1);
    int c[3];
    {
      const int u = A.div_av.div(l);
      c[A.au] = u;
      c[A.av] = l - u * dv;
      c[A.ax] = 0;
    }
    const bool sep0 = !id0 && A.ph[0].sep;
    const PhaseCoef c0 = coef_s;
    Ch ch0;
    if (sep0) ch0.init(A.ph[0], c0, A.ph[0].rvec ? A.ph[0].rvec[c[A.ph[0].oaxis]] : 0.0, j, A.scale, G);
    float2* L0 = buf + g * LS;
    float2 X[R2];
    F::forward(L0, j, X);
    if (j < R1) {
      if (id0) {
#pragma unroll
        for (int r = 0; r < R2; r++) X[r] = cscale(X[r], A.scale);
      } else if (sep0) {
        ch0.apply(X);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          X[r] = cmul(X[r], phase_value(A.ph[0], c0, j + r * R1, c, A.scale));
        }
      }
    }
    F::inverse(L0, j, X);
    __syncthreads();
    float2* dst = A.out0 + (i64)vol * A.out_vs;
    const i64 sa = A.st[A.ax];
    if (A.st[A.av] == 1) {
      const int b = threadIdx.x % B;
      if (b < nl) {
        const float2* s0 = buf + b * LS;
        for (int n = threadIdx.x / B; n < N; n += 256 / B) dst[lb_s[cur][b] + n * sa] = s0[n];
      }
    } else {
      const int b = threadIdx.x / G;
      if (b < nl) {
        const float2* s0 = buf + b * LS;
        for (int n = threadIdx.x % G; n < N; n += G) dst[lb_s[cur][b] + n * sa] = s0[n];
      }
    }
    cur ^= 1;
  }
  cp_async_wait_all();
}

// The multi-job shear step on TMA tiles: the tiles of every job move by tensor loads and
// stores, as in tma_pass_kernel, through each job's own tensor maps.  Used when every job of
// the launch qualifies for tma_pass_kernel with the same tile layout (all strided or all
// contiguous, as the jobs of one shear step in the same volume layout are).
struct MultiTmaJob {
  CUtensorMap in;
  CUtensorMap out;
  int in_rank, out_rank;
};

struct MultiTmaArgs {
  int njobs;
  int tile_off[kMaxMultiJobs + 1];
  PassArgs job[kMaxMultiJobs];
  MultiTmaJob tm[kMaxMultiJobs];
};

template <int N, int R1, int R2, bool STRIDED>
__global__ void __launch_bounds__(256, ME_PASS_MINB)
    tma_multi_shear_kernel(const __grid_constant__ MultiTmaArgs M) {
  using F = LineFft<N, R1, R2>;
  using Ch = LineChirp<N, R1, R2>;
  constexpr int G = F::G;
  constexpr int B = 256 / G;
  constexpr int LS = F::LS;
  constexpr int TILE = B * N * 8;
  constexpr int NSUB = STRIDED ? B / 16 : 1;
  constexpr int SUBT = TILE / NSUB;
  static_assert(SUBT % 1024 == 0, "swizzled sub-tiles start on 1024-byte boundaries");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* tiles = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  float2* scratch = reinterpret_cast<float2*>(tiles + 2 * TILE);
  __shared__ __align__(8) uint64_t full[2];
  __shared__ PhaseCoef coef_s;
  const int total = M.tile_off[M.njobs];
  const int g = threadIdx.x / G;
  const int j = threadIdx.x % G;
  if (threadIdx.x == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto job_of = [&](int t) {
    int k = 0;
    while (k + 1 < M.njobs && t >= M.tile_off[k + 1]) k++;
    return k;
  };
  auto coords = [&](int k, int t, int& vol, int& u, int& v0) {
    const PassArgs& A = M.job[k];
    const int tt = t - M.tile_off[k];
    vol = A.div_tiles.div(tt);
    const int l0 = (tt - vol * (A.nlines / B)) * B;
    u = A.div_av.div(l0);
    v0 = l0 - u * A.dims[A.av];
  };
  // thread 0: load work item t into buffer bufi, once the stores out of that buffer have read it
  auto issue = [&](int t, int bufi) {
    const int k = job_of(t);
    int vol, u, v0;
    coords(k, t, vol, u, v0);
    const MultiTmaJob& J = M.tm[k];
    bulk_wait_read_all();
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&full[bufi], TILE);
#pragma unroll
    for (int q = 0; q < NSUB; q++) {
      unsigned char* dst = tiles + bufi * TILE + q * SUBT;
      const int c0 = STRIDED ? v0 + 16 * q : 0, c1 = STRIDED ? 0 : v0;
      if (J.in_rank == 3) {
        tma_load_3d(dst, &J.in, c0, c1, u, &full[bufi]);
      } else {
        tma_load_4d(dst, &J.in, c0, c1, u, vol, &full[bufi]);
      }
    }
  };

  if (threadIdx.x == 0 && (int)blockIdx.x < total) issue(blockIdx.x, 0);
  int coef_job = -1, coef_vol = -1;
  int it = 0;
  for (int t = blockIdx.x; t < total; t += gridDim.x, it++) {
    const int cur = it & 1;
    const int k = job_of(t);
    const PassArgs& A = M.job[k];
    const MultiTmaJob& J = M.tm[k];
    int vol, u, v0;
    coords(k, t, vol, u, v0);
    mbar_wait_bounded(&full[cur], (it >> 1) & 1, WF_LINE_PASS);
    if (threadIdx.x == 0 && t + (int)gridDim.x < total) issue(t + gridDim.x, cur ^ 1);
    // the shear coefficients depend on the job and volume only (the barrier before the
    // previous tile's store separates every read of coef_s from this write)
    if (k != coef_job || vol != coef_vol) {
      if (threadIdx.x == 0) {
        PhaseCoef cf{0, 0, 0};
        if (A.params) cf = phase_coef(A.ph[0], A.params + (i64)vol * A.pstride, A.ax);
        coef_s = cf;
      }
      coef_job = k;
      coef_vol = vol;
      __syncthreads();
    }
    const bool id0 = phase_is_identity(A.ph[0]);
    int c[3];
    c[A.au] = u;
    c[A.av] = v0 + g;
    c[A.ax] = 0;
    const bool sep0 = !id0 && A.ph[0].sep;
    const PhaseCoef c0 = coef_s;
    Ch ch0;
    if (sep0) ch0.init(A.ph[0], c0, A.ph[0].rvec ? A.ph[0].rvec[c[A.ph[0].oaxis]] : 0.0, j, A.scale, G);
    unsigned char* tb = tiles + cur * TILE;
    float2* L = scratch + g * LS;
    float2 X[R2];
    F::forward_from([&](int n) { return *reinterpret_cast<const float2*>(tb + tile_off<N, B, STRIDED>(g, n)); },
                    L, j, X);
    if (j < R1) {
      if (id0) {
#pragma unroll
        for (int r = 0; r < R2; r++) X[r] = cscale(X[r], A.scale);
      } else if (sep0) {
        ch0.apply(X);
      } else {
#pragma unroll
        for (int r = 0; r < R2; r++) {
          c[A.ax] = j + r * R1;
          X[r] = cmul(X[r], phase_value(A.ph[0], c0, j + r * R1, c, A.scale));
        }
      }
    }
    F::inverse_to(L, j, X, [&](int, int n, float2 v) {
      *reinterpret_cast<float2*>(tb + tile_off<N, B, STRIDED>(g, n)) = v;
    });
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int q = 0; q < NSUB; q++) {
        const unsigned char* src = tb + q * SUBT;
        const int c0s = STRIDED ? v0 + 16 * q : 0, c1s = STRIDED ? 0 : v0;
        if (J.out_rank == 3) {
          tma_store_3d(&J.out, src, c0s, c1s, u);
        } else {
          tma_store_4d(&J.out, src, c0s, c1s, u, vol);
        }
      }
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

template <int N, int R1, int R2, bool STRIDED>
static int launch_tma_multi_n(const MultiTmaArgs& M, cudaStream_t stream) {
  using F = LineFft<N, R1, R2>;
  constexpr int B = 256 / F::G;
  const size_t smem = 1024 + 2 * (size_t)B * N * 8 + sizeof(float2) * (size_t)F::LS * B;
  auto kern = tma_multi_shear_kernel<N, R1, R2, STRIDED>;
  const int rc = check_cuda(allow_smem(kern, smem), "multi shear smem");
  if (rc != ME_OK) return rc;
  int dev = 0, sms = 148, nb = 2;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, smem);
  const int total = M.tile_off[M.njobs];
  const int grid = (int)std::min<long long>(total, (long long)std::max(1, nb) * sms);
  count_launch();
  kern<<<grid, 256, smem, stream>>>(M);
  return check_cuda(cudaGetLastError(), "multi shear launch");
}

template <int N, int R1, int R2>
static int launch_multi_n(const MultiPassArgs& M, cudaStream_t stream) {
  using F = LineFft<N, R1, R2>;
  const size_t smem = 2 * sizeof(float2) * (size_t)F::LS * (256 / F::G);
  const int rc = check_cuda(allow_smem(multi_shear_kernel<N, R1, R2>, smem), "multi shear smem");
  if (rc != ME_OK) return rc;
  int dev = 0, sms = 148, nb = 2;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, multi_shear_kernel<N, R1, R2>, 256, smem);
  const int total = M.tile_off[M.njobs];
  const int grid = (int)std::min<long long>(total, (long long)std::max(1, nb) * sms);
  count_launch();
  multi_shear_kernel<N, R1, R2><<<grid, 256, smem, stream>>>(M);
  return check_cuda(cudaGetLastError(), "multi shear launch");
}

static bool fast_length(int n) {
  switch (n) {
#define ME_FAST_IS(N, R1, R2) \
  case N: return true;
    ME_FAST_LENGTHS(ME_FAST_IS)
#undef ME_FAST_IS
    default: return false;
  }
}

static int tile_lines(int n) {
  switch (n) {
#define ME_TILE_LINES(N, R1, R2) \
  case N: return 256 / LineFft<N, R1, R2>::G;
    ME_FAST_LENGTHS(ME_TILE_LINES)
#undef ME_TILE_LINES
    default: return 0;
  }
}

int launch_multi_shear(const PassArgs* jobs, int njobs, cudaStream_t stream) {
  if (njobs < 1) return ME_OK;
  if (njobs > kMaxMultiJobs) return fail("multi shear: too many jobs in one launch");
  for (int k = 0; k < njobs; k++)
    if (!fast_length(jobs[k].plan.n)) {
      set_error("multi shear: a job's line length has no compile-time FFT");
      return ME_ERR_UNSUPPORTED;
    }
  // one launch per distinct line length, over the jobs of that length in job order
  bool done[kMaxMultiJobs] = {false};
  for (int k0 = 0; k0 < njobs; k0++) {
    if (done[k0]) continue;
    const int n = jobs[k0].plan.n;
    MultiPassArgs M;
    M.njobs = 0;
    M.tile_off[0] = 0;
    long long total = 0;
    for (int k = k0; k < njobs; k++) {
      if (done[k] || jobs[k].plan.n != n) continue;
      done[k] = true;
      const int B = tile_lines(n);
      total += (long long)((jobs[k].nlines + B - 1) / B) * jobs[k].nvol;
      if (total > 0x7fffffffLL) return fail("multi shear: too many work items");
      M.job[M.njobs] = jobs[k];
      M.job[M.njobs].div_tiles.set((jobs[k].nlines + B - 1) / B);
      M.tile_off[++M.njobs] = (int)total;
    }
    if (total == 0) continue;
    // on TMA tiles when every job of this length qualifies
    const int B = tile_lines(n);
    MultiTmaArgs MT;
    bool tma = true, all_strided = true;
    for (int q = 0; q < M.njobs && tma; q++) {
      PassTma T;
      bool strided = false;
      tma = tma_pass_setup(PM_SHEAR, M.job[q], B, &strided, &T);
      if (tma) {
        if (q == 0) all_strided = strided;
        tma = (strided == all_strided);
        MT.job[q] = M.job[q];
        MT.tm[q].in = T.in[0];
        MT.tm[q].out = T.out[0];
        MT.tm[q].in_rank = T.in_rank[0];
        MT.tm[q].out_rank = T.out_rank[0];
      }
    }
    if (tma) {
      MT.njobs = M.njobs;
      for (int q = 0; q <= M.njobs; q++) MT.tile_off[q] = M.tile_off[q];
    }
    int rc = -1;
    switch (n) {
#define ME_MULTI_LAUNCH(N, R1, R2)                                                  \
  case N:                                                                           \
    rc = !tma ? launch_multi_n<N, R1, R2>(M, stream)                                 \
         : all_strided ? launch_tma_multi_n<N, R1, R2, true>(MT, stream)            \
                       : launch_tma_multi_n<N, R1, R2, false>(MT, stream);          \
    break;
      ME_FAST_LENGTHS(ME_MULTI_LAUNCH)
#undef ME_MULTI_LAUNCH
      default: break;
    }
    if (rc != ME_OK) return rc < 0 ? fail("multi shear: unsupported length") : rc;
  }
  return ME_OK;
}

}  // namespace me
