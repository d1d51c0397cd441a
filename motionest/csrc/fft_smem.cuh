// Shared-memory mixed-radix FFT engine for batches of short lines (length <= ME_MAX_LINE).
//
// Lines live in shared memory in an interleaved layout: element n of line b is at
// buf[n * es + b] (es >= number of lines), so consecutive threads touch consecutive lines and
// every stage is bank-conflict free.  Each stage is a self-sorting (Stockham) radix-R pass
// between two buffers; the radices come from a host-computed plan (8, 4, 2 and the odd primes
// 3, 5, 7, 11, 13), so any length whose prime factors are <= 13 is supported with natural-order
// output and no bit reversal.  Twiddles come from a per-CTA table tw[k] = exp(-2*pi*i*k/N).
#pragma once
#include "common.cuh"

namespace me {

constexpr int kMaxStages = 12;

struct FftPlan {
  int n;
  int nst;
  int radix[kMaxStages];
};

// Host: factor n into the stage radices.  Returns false if n has a prime factor > 13.
inline bool make_plan(int n, FftPlan* p) {
  p->n = n;
  p->nst = 0;
  if (n < 1) return false;
  int m = n, p2 = 0;
  while (m % 2 == 0) {
    m /= 2;
    p2++;
  }
  int n8 = p2 / 3, rem = p2 % 3;
  int tmp[kMaxStages];
  int k = 0;
  if (rem == 1 && n8 > 0) {
    n8--;
    for (int i = 0; i < n8; i++) tmp[k++] = 8;
    tmp[k++] = 4;
    tmp[k++] = 4;
  } else {
    for (int i = 0; i < n8; i++) tmp[k++] = 8;
    if (rem == 1) tmp[k++] = 2;
    if (rem == 2) tmp[k++] = 4;
  }
  const int odd[5] = {3, 5, 7, 11, 13};
  for (int i = 0; i < 5; i++) {
    while (m % odd[i] == 0) {
      if (k >= kMaxStages) return false;
      m /= odd[i];
      tmp[k++] = odd[i];
    }
  }
  if (m != 1) return false;
  for (int i = 0; i < k; i++) p->radix[i] = tmp[i];
  p->nst = k;
  return true;
}

// Fill tw[0..n) with exp(-2*pi*i*k/n) (forward twiddles), cooperatively.
__device__ __forceinline__ void init_twiddles(float2* tw, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

template <bool INV>
__device__ __forceinline__ float2 tw_get(const float2* tw, int idx) {
  float2 w = tw[idx];
  if (INV) w.y = -w.y;
  return w;
}

// ---------------------------------------------------------------- small DFT kernels
template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = csub(v1, v3);
  // forward: W4 = -i ; inverse: +i
  float2 t3r = INV ? mul_i(t3) : mul_mi(t3);
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3r);
  v3 = csub(t1, t3r);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
  const float h = 0.70710678118654752440f;
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // twiddles W8^k (forward exp(-i pi k/4)), k = 1..3
  float2 w1 = INV ? make_float2(h, h) : make_float2(h, -h);
  float2 w3 = INV ? make_float2(-h, h) : make_float2(-h, -h);
  o1 = cmul(o1, w1);
  o2 = INV ? mul_i(o2) : mul_mi(o2);
  o3 = cmul(o3, w3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// Generic odd-length DFT via the twiddle table: W_R^m = tw[m * (N/R)].
template <int R, bool INV>
__device__ __forceinline__ void dft_generic(float2* v, const float2* tw, int N) {
  const int step = N / R;
  float2 out[R];
#pragma unroll
  for (int k = 0; k < R; k++) {
    float2 acc = v[0];
#pragma unroll
    for (int r = 1; r < R; r++) {
      const int m = (r * k) % R;
      acc = cadd(acc, cmul(v[r], tw_get<INV>(tw, m * step)));
    }
    out[k] = acc;
  }
#pragma unroll
  for (int k = 0; k < R; k++) v[k] = out[k];
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v, const float2* tw, int N) {
  if constexpr (R == 2) {
    dft2<INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8<INV>(v);
  } else {
    dft_generic<R, INV>(v, tw, N);
  }
}

// One Stockham stage over `nlines` interleaved lines (element n of line b at buf[n*es + b]).
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ in, float2* __restrict__ out,
                                          int N, int Ns, int nlines, int es,
                                          const float2* __restrict__ tw) {
  const int nb = N / R;
  const int total = nb * nlines;
  const int twstep = N / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t % nlines;
    const int j = t / nlines;
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[(j + r * nb) * es + line];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) v[r] = cmul(v[r], tw_get<INV>(tw, r * k * twstep));
    }
    dft<R, INV>(v, tw, N);
    const int d = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[(d + r * Ns) * es + line] = v[r];
  }
}

// Run the whole plan; data starts in `a`, `b` is scratch of the same size.  Returns the buffer
// that holds the result.  Unnormalised (forward: exp(-2 pi i nk/N); INV: exp(+2 pi i nk/N)).
template <bool INV>
__device__ float2* fft_lines(float2* a, float2* b, const FftPlan& P, int nlines, int es,
                             const float2* tw) {
  int Ns = 1;
  for (int s = 0; s < P.nst; s++) {
    const int R = P.radix[s];
    switch (R) {
      case 2: fft_stage<2, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 3: fft_stage<3, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 4: fft_stage<4, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 5: fft_stage<5, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 7: fft_stage<7, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 8: fft_stage<8, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 11: fft_stage<11, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      case 13: fft_stage<13, INV>(a, b, P.n, Ns, nlines, es, tw); break;
      default: break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace me
