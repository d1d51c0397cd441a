// Register-resident small DFTs and the two-stage line FFT used by the compile-time kernels.
//
// A line of length N = R1 * R2 is owned by a group of G threads (G = 16 or 8, inside one
// warp) and lives in a shared-memory region of LS elements.  Forward transform:
//   stage 1: thread j < R2 reads x[j + r R2] (r < R1), does an R1-point DFT in registers and
//            writes Y_j[k] to row j of a padded [R2][S1] table (S1 = R1 rounded up to odd);
//   stage 2: thread j < R1 reads column j (Y_r[j], r < R2), multiplies by W_N^{r j} (from a
//            table in that order), does an R2-point DFT and ends holding X[j + r R1] for
//            r < R2 in registers.
// The inverse transform consumes that register layout directly (inverse R2-point DFT,
// W_N^{-j a}, transpose through the padded table, inverse R1-point DFT) and writes x in natural
// order.  Only __syncwarp is needed between the steps, all index arithmetic is compile-time,
// and every shared-memory access pattern is bank-conflict free (unit or odd strides).
#pragma once
#include "common.cuh"
#include "dft_consts.cuh"

namespace me {

template <int R, bool INV>
__device__ __forceinline__ float2 wr(int m) {
  // W_R^m = exp(-2 pi i m / R) (forward) or its conjugate (inverse); m is a compile-time
  // constant after unrolling, so this folds to immediates.
  const int mm = ((m % R) + R) % R;
  return make_float2(RadixConst<R>::c(mm), INV ? RadixConst<R>::s(mm) : -RadixConst<R>::s(mm));
}

template <int R, bool INV>
struct RDft;

template <bool INV>
struct RDft<1, INV> {
  static __device__ __forceinline__ void run(float2* v) {}
};

template <bool INV>
struct RDft<2, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct RDft<4, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const float2 t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
    const float2 t3r = INV ? mul_i(t3) : mul_mi(t3);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3r);
    v[3] = csub(t1, t3r);
  }
};

// Odd prime R: pair x_p with x_{R-p} (X[k] and X[R-k] share the cos / sin sums).
template <int R, bool INV>
struct RDftPrime {
  static __device__ __forceinline__ void run(float2* v) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
#pragma unroll
    for (int p = 1; p <= H; p++) {
      a[p - 1] = cadd(v[p], v[R - p]);
      b[p - 1] = csub(v[p], v[R - p]);
    }
    const float2 x0 = v[0];
    float2 s0 = x0;
#pragma unroll
    for (int p = 0; p < H; p++) s0 = cadd(s0, a[p]);
    float2 out[R];
    out[0] = s0;
#pragma unroll
    for (int k = 1; k <= H; k++) {
      float2 re = x0, im = make_float2(0.f, 0.f);
#pragma unroll
      for (int p = 1; p <= H; p++) {
        const float c = RadixConst<R>::c((p * k) % R);
        const float s = RadixConst<R>::s((p * k) % R);
        re.x = fmaf(c, a[p - 1].x, re.x);
        re.y = fmaf(c, a[p - 1].y, re.y);
        im.x = fmaf(s, b[p - 1].x, im.x);
        im.y = fmaf(s, b[p - 1].y, im.y);
      }
      // forward: X[k] = re - i im, X[R-k] = re + i im ; inverse: signs swapped
      const float2 iim = mul_i(im);
      out[k] = INV ? cadd(re, iim) : csub(re, iim);
      out[R - k] = INV ? csub(re, iim) : cadd(re, iim);
    }
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = out[k];
  }
};

template <bool INV> struct RDft<3, INV> : RDftPrime<3, INV> {};
template <bool INV> struct RDft<5, INV> : RDftPrime<5, INV> {};
template <bool INV> struct RDft<7, INV> : RDftPrime<7, INV> {};
template <bool INV> struct RDft<11, INV> : RDftPrime<11, INV> {};
template <bool INV> struct RDft<13, INV> : RDftPrime<13, INV> {};

// Composite R = A * B: n = B n1 + n2, k = k1 + A k2,
// X[k1 + A k2] = sum_{n2} W_R^{n2 k1} W_B^{n2 k2} sum_{n1} x[B n1 + n2] W_A^{n1 k1}.
template <int A, int B, bool INV>
struct RDftComp {
  static __device__ __forceinline__ void run(float2* v) {
    constexpr int R = A * B;
    float2 t[R];
#pragma unroll
    for (int n2 = 0; n2 < B; n2++) {
      float2 u[A];
#pragma unroll
      for (int n1 = 0; n1 < A; n1++) u[n1] = v[B * n1 + n2];
      RDft<A, INV>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < A; k1++)
        t[n2 * A + k1] = (n2 * k1 == 0) ? u[k1] : cmul(u[k1], wr<R, INV>(n2 * k1));
    }
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      float2 w[B];
#pragma unroll
      for (int n2 = 0; n2 < B; n2++) w[n2] = t[n2 * A + k1];
      RDft<B, INV>::run(w);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = w[k2];
    }
  }
};

template <bool INV> struct RDft<6, INV> : RDftComp<2, 3, INV> {};
template <bool INV> struct RDft<8, INV> : RDftComp<2, 4, INV> {};
template <bool INV> struct RDft<9, INV> : RDftComp<3, 3, INV> {};
template <bool INV> struct RDft<12, INV> : RDftComp<4, 3, INV> {};
template <bool INV> struct RDft<14, INV> : RDftComp<2, 7, INV> {};
template <bool INV> struct RDft<16, INV> : RDftComp<4, 4, INV> {};

// Second-stage twiddle W_N^{r j} from the plan-ordered table: for each r the R1 threads of a
// line read R1 consecutive entries (one L1 wavefront per warp instead of one sector per
// thread, as indices r j mod N scattered over the natural-order table would need).
template <int N> __device__ __forceinline__ const float2* twp_table();
#define ME_TWP_TABLE(N, R1, R2) \
  template <> __device__ __forceinline__ const float2* twp_table<N>() { return twp##N; }
ME_FAST_LENGTHS(ME_TWP_TABLE)
#undef ME_TWP_TABLE

template <int N, int R1, bool INV>
__device__ __forceinline__ float2 twP(int r, int j) {
  float2 w = __ldg(twp_table<N>() + r * R1 + j);
  if (INV) w.y = -w.y;
  return w;
}

template <int N, int R1, int R2>
struct LineFft {
  static constexpr int S1 = R1 | 1;  // odd row stride of the transpose table
  static constexpr int LS = ((N > R2 * S1 ? N : R2 * S1)) | 1;
  static constexpr int G = (R1 > R2 ? R1 : R2) <= 8 ? 8 : 16;

  // Forward FFT of the natural-order line in L; thread j (< R1) ends with X[j + r R1].
  static __device__ __forceinline__ void forward(float2* L, int j, float2 (&X)[R2]) {
    forward_from([&](int n) { return L[n]; }, L, j, X);
  }

  // Forward FFT of the line x[n] = load(n) (read once, in the first stage); L is the line's
  // work region and may differ from where load() reads.
  template <class Load>
  static __device__ __forceinline__ void forward_from(Load load, float2* L, int j, float2 (&X)[R2]) {
    float2 u[R1];
    if (j < R2) {
#pragma unroll
      for (int r = 0; r < R1; r++) u[r] = load(j + r * R2);
      RDft<R1, false>::run(u);
    }
    __syncwarp();
    if (j < R2) {
#pragma unroll
      for (int r = 0; r < R1; r++) L[j * S1 + r] = u[r];
    }
    __syncwarp();
    if (j < R1) {
#pragma unroll
      for (int r = 0; r < R2; r++) {
        const float2 y = L[r * S1 + j];
        X[r] = (r == 0) ? y : cmul(y, twP<N, R1, false>(r, j));
      }
      RDft<R2, false>::run(X);
    }
  }

  // Inverse FFT from the register layout of forward(); writes x in natural order into L.
  static __device__ __forceinline__ void inverse(float2* L, int j, float2 (&X)[R2]) {
    inverse_to(L, j, X, [&](int b, int n, float2 v) { L[n] = v; });
    __syncwarp();
  }

  // Inverse FFT handing each output to store(b, n, x[n]) (b < R1 the compile-time slot, n = j +
  // b R2, threads j < R2) instead of writing it to L; L is the line's work region.
  template <class Store>
  static __device__ __forceinline__ void inverse_to(float2* L, int j, float2 (&X)[R2], Store store) {
    if (j < R1) {
      RDft<R2, true>::run(X);
#pragma unroll
      for (int a = 1; a < R2; a++) X[a] = cmul(X[a], twP<N, R1, true>(a, j));
    }
    __syncwarp();
    if (j < R1) {
#pragma unroll
      for (int a = 0; a < R2; a++) L[a * S1 + j] = X[a];
    }
    __syncwarp();
    float2 u[R1];
    if (j < R2) {
#pragma unroll
      for (int b = 0; b < R1; b++) u[b] = L[j * S1 + b];
      RDft<R1, true>::run(u);
    }
    __syncwarp();
    if (j < R2) {
#pragma unroll
      for (int b = 0; b < R1; b++) store(b, j + b * R2, u[b]);
    }
  }

  // Natural-order spectrum from registers (thread j holds X[j + r R1]).
  static __device__ __forceinline__ void store_spectrum(float2* L, int j, const float2 (&X)[R2]) {
    __syncwarp();
    if (j < R1) {
#pragma unroll
      for (int r = 0; r < R2; r++) L[j + r * R1] = X[r];
    }
    __syncwarp();
  }

  static __device__ __forceinline__ void load_spectrum(const float2* L, int j, float2 (&X)[R2]) {
    if (j < R1) {
#pragma unroll
      for (int r = 0; r < R2; r++) X[r] = L[j + r * R1];
    }
  }
};

}  // namespace me
