// Row DFTs on the tensor cores with split-precision operands: the measured alternative to the
// register FFT (fft_reg.cuh) for the short lines of the shear and SENSE kernels.
//
// A row of length N = 16 * N2 (N2 even, <= 16) is transformed in two matrix stages (the
// four-step factorisation n = N2 n1 + n2, k = k1 + 16 k2):
//   stage 1  Y[n2][k1] = sum_n1 x[N2 n1 + n2] W16^(n1 k1)      a [rows*N2 x 16] x [16 x 16] product
//   twiddle  Y[n2][k1] *= W_N^(n2 k1)                           (FP32, in the accumulators)
//   stage 2  X[k1 + 16 k2] = sum_n2 Y[n2][k1] W_N2^(n2 k2)     a [rows*16 x N2] x [N2 x N2] product
// Each complex product is a real one on the interleaved (re, im) embedding, [re im] x
// [[Wr, Wi], [-Wi, Wr]], and runs as mma.sync m16n8k8 TF32 with FP32 accumulation.  TF32 keeps
// 10 mantissa bits, so each operand is split a = a_hi + a_lo (a_hi = tf32(a), a_lo =
// tf32(a - a_hi)) and three products are accumulated, a_lo b_hi + a_hi b_lo + a_hi b_hi, which
// recovers close to FP32 accuracy (the error-corrected TF32 scheme of Ootomo and Yokota, 2022).
//
// me_dft_rows_split is a self-contained benchmark entry point: the same transform as
// me_fft_axis along the contiguous axis (orthonormal), so the two can be timed and compared on
// the same rows.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace me {

__device__ __forceinline__ unsigned to_tf32(float a) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return r;
}

__device__ __forceinline__ void split_tf32(float a, unsigned& hi, unsigned& lo) {
  hi = to_tf32(a);
  lo = to_tf32(a - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Split-precision accumulate of one m16n8k8 tile: d += A B from the split operands (b.x the
// TF32 high part, b.y the low part).
__device__ __forceinline__ void mma_split(float (&d)[4], const unsigned (&ah)[4],
                                          const unsigned (&al)[4], uint2 b0, uint2 b1) {
  mma_tf32(d, al, b0.x, b1.x);
  mma_tf32(d, ah, b0.y, b1.y);
  mma_tf32(d, ah, b0.x, b1.x);
}

constexpr int kTcRows = 8;       // rows per tile
constexpr int kTcThreads = 128;  // four warps

// Real embedding of the complex DFT matrix of size R (padded to RP rows / columns, zeros
// outside): B[2n + u][2k + v] with (u, v) = (0, 0): Wr, (1, 0): -Wi, (0, 1): Wi, (1, 1): Wr,
// each entry stored split as (tf32 hi, tf32 lo), rows `ld` entries apart.
__device__ __forceinline__ void init_dft_embedding(uint2* B, int R, int RP, int ld, bool inv) {
  const int W = 2 * RP;
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
    const int row = e / W, col = e - row * W;
    const int n = row >> 1, u = row & 1, k = col >> 1, v = col & 1;
    float val = 0.f;
    if (n < R && k < R) {
      float s, c;
      sincospif(-2.0f * (float)((n * k) % R) / (float)R, &s, &c);
      if (inv) s = -s;
      val = (u == v) ? c : (u == 0 ? s : -s);
    }
    unsigned hi, lo;
    split_tf32(val, hi, lo);
    B[row * ld + col] = make_uint2(hi, lo);
  }
}

template <int N2>
struct DftSplitPlan {
  static constexpr int N = 16 * N2;
  static constexpr int P2 = (N2 + 3) & ~3;  // stage-2 length padded to a multiple of 4
  static constexpr int SP = P2 + 1;         // odd row stride of the stage-1 result (banks)
  // row strides of the DFT embeddings: the four rows a B fragment load touches then fall on
  // two disjoint halves of the banks
  static constexpr int LD1 = 32 + 8, LD2 = 2 * P2 + 8;
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)kTcRows * N + kTcRows * 16 * SP +
                                                   N2 * 16) +
                                 sizeof(uint2) * (32 * LD1 + 2 * P2 * LD2);
};

template <int N2>
__global__ void __launch_bounds__(kTcThreads) dft_rows_split_kernel(const float2* __restrict__ in,
                                                                     float2* __restrict__ out,
                                                                     i64 nrows, int inverse,
                                                                     float scale) {
  static_assert(N2 % 2 == 0 && N2 <= 16, "rows of 16 * N2 points, N2 even");
  using P = DftSplitPlan<N2>;
  constexpr int N = P::N, P2 = P::P2, SP = P::SP, LD1 = P::LD1, LD2 = P::LD2;
  extern __shared__ __align__(16) float2 dsm[];
  float2* xs = dsm;                                              // [rows][N] in, then out
  float2* ys = xs + kTcRows * N;                                 // [rows][k1][n2], stride SP
  uint2* B1 = reinterpret_cast<uint2*>(ys + kTcRows * 16 * SP);  // 16-point DFT embedding
  uint2* B2 = B1 + 32 * LD1;                                     // N2-point DFT embedding
  float2* tw = reinterpret_cast<float2*>(B2 + 2 * P2 * LD2);     // W_N^(n2 k1)
  const bool inv = inverse != 0;
  init_dft_embedding(B1, 16, 16, LD1, inv);
  init_dft_embedding(B2, N2, P2, LD2, inv);
  for (int e = threadIdx.x; e < N2 * 16; e += blockDim.x) {
    const int n2 = e / 16, k1 = e % 16;
    float s, c;
    sincospif(-2.0f * (float)((n2 * k1) % N) / (float)N, &s, &c);
    tw[e] = make_float2(c, inv ? -s : s);
  }
  for (int e = threadIdx.x; e < kTcRows * 16 * SP; e += blockDim.x) ys[e] = make_float2(0.f, 0.f);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const i64 ntiles = (nrows + kTcRows - 1) / kTcRows;
  for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const i64 r0 = t * kTcRows;
    const int nr = (int)min((i64)kTcRows, nrows - r0);
    __syncthreads();
    for (int e = threadIdx.x; e < kTcRows * N; e += blockDim.x)
      xs[e] = (e / N < nr) ? in[r0 * N + e] : make_float2(0.f, 0.f);
    __syncthreads();
    // stage 1: M = rows * N2 pairs (row, n2), K = 32 (n1, re/im), N = 32 (k1, re/im)
    constexpr int MT1 = kTcRows * N2 / 16;
    for (int mt = warp; mt < MT1; mt += kTcThreads / 32) {
      float acc[4][4];
#pragma unroll
      for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int i = 0; i < 4; i++) acc[nt][i] = 0.f;
      const int m_lo = mt * 16 + gid, m_hi = m_lo + 8;
      const int r_lo = m_lo / N2, n2_lo = m_lo % N2, r_hi = m_hi / N2, n2_hi = m_hi % N2;
#pragma unroll
      for (int ks = 0; ks < 4; ks++) {
        // A[m][kk] = component kk % 2 of x[row][N2 (kk / 2) + n2], kk = ks*8 + tig (+4)
        const int kk0 = ks * 8 + tig, kk1 = kk0 + 4;
        const float2 v00 = xs[r_lo * N + N2 * (kk0 >> 1) + n2_lo];
        const float2 v10 = xs[r_hi * N + N2 * (kk0 >> 1) + n2_hi];
        const float2 v01 = xs[r_lo * N + N2 * (kk1 >> 1) + n2_lo];
        const float2 v11 = xs[r_hi * N + N2 * (kk1 >> 1) + n2_hi];
        float a[4];
        a[0] = (kk0 & 1) ? v00.y : v00.x;
        a[1] = (kk0 & 1) ? v10.y : v10.x;
        a[2] = (kk1 & 1) ? v01.y : v01.x;
        a[3] = (kk1 & 1) ? v11.y : v11.x;
        unsigned ah[4], al[4];
#pragma unroll
        for (int i = 0; i < 4; i++) split_tf32(a[i], ah[i], al[i]);
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
          mma_split(acc[nt], ah, al, B1[(ks * 8 + tig) * LD1 + nt * 8 + gid],
                    B1[(ks * 8 + tig + 4) * LD1 + nt * 8 + gid]);
      }
      // accumulator (row, col 2 tig + {0, 1}) of N-tile nt is the complex Y[n2][k1 = 4 nt + tig]
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int k1 = nt * 4 + tig;
        const float2 ylo = cmul(make_float2(acc[nt][0], acc[nt][1]), tw[n2_lo * 16 + k1]);
        const float2 yhi = cmul(make_float2(acc[nt][2], acc[nt][3]), tw[n2_hi * 16 + k1]);
        ys[(r_lo * 16 + k1) * SP + n2_lo] = ylo;
        ys[(r_hi * 16 + k1) * SP + n2_hi] = yhi;
      }
    }
    __syncthreads();
    // stage 2: M = rows * 16 pairs (row, k1), K = 2 P2 (n2, re/im), N = 2 P2 (k2, re/im)
    constexpr int KS2 = 2 * P2 / 8;
    constexpr int NT2 = 2 * P2 / 8;
    for (int mt = warp; mt < kTcRows; mt += kTcThreads / 32) {  // one row per M-tile
      float acc[NT2][4];
#pragma unroll
      for (int nt = 0; nt < NT2; nt++)
#pragma unroll
        for (int i = 0; i < 4; i++) acc[nt][i] = 0.f;
      const float2* yr = ys + mt * 16 * SP;
#pragma unroll
      for (int ks = 0; ks < KS2; ks++) {
        const int kk0 = ks * 8 + tig, kk1 = kk0 + 4;
        const float2 v00 = yr[gid * SP + (kk0 >> 1)];
        const float2 v10 = yr[(gid + 8) * SP + (kk0 >> 1)];
        const float2 v01 = yr[gid * SP + (kk1 >> 1)];
        const float2 v11 = yr[(gid + 8) * SP + (kk1 >> 1)];
        float a[4];
        a[0] = (kk0 & 1) ? v00.y : v00.x;
        a[1] = (kk0 & 1) ? v10.y : v10.x;
        a[2] = (kk1 & 1) ? v01.y : v01.x;
        a[3] = (kk1 & 1) ? v11.y : v11.x;
        unsigned ah[4], al[4];
#pragma unroll
        for (int i = 0; i < 4; i++) split_tf32(a[i], ah[i], al[i]);
#pragma unroll
        for (int nt = 0; nt < NT2; nt++)
          mma_split(acc[nt], ah, al, B2[(ks * 8 + tig) * LD2 + nt * 8 + gid],
                    B2[(ks * 8 + tig + 4) * LD2 + nt * 8 + gid]);
      }
#pragma unroll
      for (int nt = 0; nt < NT2; nt++) {
        const int k2 = nt * 4 + tig;
        if (k2 < N2) {
          xs[mt * N + gid + 16 * k2] = make_float2(acc[nt][0] * scale, acc[nt][1] * scale);
          xs[mt * N + gid + 8 + 16 * k2] = make_float2(acc[nt][2] * scale, acc[nt][3] * scale);
        }
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * N; e += blockDim.x) out[r0 * N + e] = xs[e];
  }
}

template <int N2>
static int launch_dft_split(const float2* in, float2* out, i64 nrows, int inverse,
                            cudaStream_t st) {
  using P = DftSplitPlan<N2>;
  const int rc = check_cuda(allow_smem(dft_rows_split_kernel<N2>, P::SMEM), "dft split smem");
  if (rc != ME_OK) return rc;
  const i64 ntiles = (nrows + kTcRows - 1) / kTcRows;
  const int grid = (int)std::min<i64>(ntiles, 148LL * 8);
  count_launch();
  dft_rows_split_kernel<N2><<<grid, kTcThreads, P::SMEM, st>>>(
      in, out, nrows, inverse, (float)(1.0 / sqrt((double)P::N)));
  return check_cuda(cudaGetLastError(), "dft split launch");
}

}  // namespace me

using namespace me;

extern "C" {

int me_dft_rows_split(const me_c64* in, me_c64* out, long long nrows, int n, int inverse,
                      void* stream) {
  if (!in || !out) return fail("me_dft_rows_split: NULL pointer");
  if (nrows < 0) return fail("me_dft_rows_split: negative row count");
  if (in == out) return fail("me_dft_rows_split: needs out != in");
  if (nrows == 0) return ME_OK;
  cudaStream_t st = (cudaStream_t)stream;
  switch (n) {
    case 192: return launch_dft_split<12>((const float2*)in, (float2*)out, nrows, inverse, st);
    case 224: return launch_dft_split<14>((const float2*)in, (float2*)out, nrows, inverse, st);
    case 256: return launch_dft_split<16>((const float2*)in, (float2*)out, nrows, inverse, st);
    default:
      set_error("me_dft_rows_split: line lengths 192, 224 and 256 only");
      return ME_ERR_UNSUPPORTED;
  }
}

}  // extern "C"
