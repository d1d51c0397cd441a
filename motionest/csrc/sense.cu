// SENSE operators on the sampled k-space of each shot (image_estimation.py:89-129,
// transform_estimation.py:39-68, joint_recon.py:108-115).
//
// Every mask is constant along z, so F^H M_s F = F_xy^H M_s F_xy: nothing is transformed along
// z per iteration, and the data are kept in hybrid space (orthonormal IFFT_z of k-space, done
// once at set-up).  For one readout plane z the forward model of coil c is
//     K_s[j] = (1/sqrt(XY)) sum_x exp(-2 pi i kx_j x / X) FFT_y(mps_c . u)[x, ky_j]
// i.e. a full FFT along y of every x row followed by a sparse DFT along x evaluated only at the
// shot's samples (a few hundred points instead of the X*Y plane).  The adjoint scatters the
// samples back along x for each ky, inverse-FFTs along y, multiplies by conj(mps_c) and sums
// over coils.
//
//   sense_fwd_kernel  CTA = (plane z, coil c, shot): streams the plane's x rows through shared
//                     memory, FFT_y, accumulates its samples in registers; epilogue writes K,
//                     or the residual energy, or the 28 Gauss-Newton statistics (LM).
//   sense_adj_kernel  CTA = (plane z, x-block, shot): loops over coils, builds the H rows from
//                     K, IFFT_y, accumulates conj(mps) . h in registers, writes one image block.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "fft_reg.cuh"
#include "line_pass.cuh"
#include "rigid.cuh"

namespace me {

#define ME_TRY(x)                 \
  do {                            \
    int _rc = (x);                \
    if (_rc != ME_OK) return _rc; \
  } while (0)

enum FwdMode { FWD_K = 0, FWD_RESID = 1, FWD_LM = 2 };

// Resident CTAs per SM the fast SENSE kernels are compiled for (register budget 65536/(256*n)).
#ifndef ME_SENSE_MINB
#define ME_SENSE_MINB 2
#endif
constexpr int kLmStats = 28;  // e0, g[6], H upper triangle[21]
constexpr int kThreads = 256;

__host__ __device__ inline int pad2(int n) { return (n + 1) & ~1; }

struct FwdArgs {
  int X, Y, Z, C;
  const float2* mps;
  const float2* vols;
  i64 vol_stride;
  int shot0;
  const int* shot_off;
  const int* kx;
  const int* ky;
  const float2* ydat;
  float2* kout;  // offsets relative to shot_off[shot0], or absolute when kout_abs
  int kout_abs;
  int vps;       // volumes per shot (compile-time kernels, V = 1): vols holds [shot][vps] volumes
  i64 kout_vs;   // distance between the K regions of a shot's volumes
  double* partial;
  int XR, es;
  float scale;
  int bulk;  // stage rows with bulk copies (bases 16-byte aligned; set on the host)
  FftPlan plan;
};

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* out) {
  __shared__ double red[kThreads / 32][NV > 1 ? NV : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double a = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) red[warp][k] = a;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) a += red[w][threadIdx.x];
    out[threadIdx.x] = a;
  }
}

// Gauss-Newton sums of one sample: |r|^2, Re(conj(r) J_p) and Re(conj(J_p) J_q) for q >= p.
__device__ __forceinline__ void lm_accumulate(double (&st)[kLmStats], float2 r, const float2 (&J)[6]) {
  st[0] += (double)r.x * r.x + (double)r.y * r.y;
#pragma unroll
  for (int p = 0; p < 6; p++) st[1 + p] += (double)r.x * J[p].x + (double)r.y * J[p].y;
  int k = 7;
#pragma unroll
  for (int p = 0; p < 6; p++)
#pragma unroll
    for (int q = p; q < 6; q++) {
      st[k] += (double)J[p].x * J[q].x + (double)J[p].y * J[q].y;
      k++;
    }
}

template <int MPT, int V, int MODE>
__global__ void __launch_bounds__(kThreads) sense_fwd_kernel(const FwdArgs A) {
  extern __shared__ float2 sm[];
  const int z = blockIdx.x, c = blockIdx.y, b = blockIdx.z;
  const int s = A.shot0 + b;
  const int X = A.X, Y = A.Y;
  float2* twY = sm;
  float2* twX = twY + pad2(Y);
  float2* buf0 = twX + pad2(X);
  float2* buf1 = buf0 + (i64)Y * A.es;
  const int L = V * A.XR;

  init_twiddles(twY, Y);
  init_twiddles(twX, X);

  const int soff = A.shot_off[s];
  const int ns = A.shot_off[s + 1] - soff;
  int mkx[MPT], mky[MPT];
  float2 acc[V][MPT];
#pragma unroll
  for (int m = 0; m < MPT; m++) {
    const int j = threadIdx.x + m * kThreads;
    mkx[m] = -1;
    mky[m] = 0;
    if (j < ns) {
      mkx[m] = A.kx[soff + j];
      mky[m] = A.ky[soff + j];
    }
#pragma unroll
    for (int v = 0; v < V; v++) acc[v][m] = make_float2(0.f, 0.f);
  }

  const i64 plane = (i64)X * Y;
  const float2* mrow = A.mps + ((i64)z * A.C + c) * plane;
  const float2* vbase = A.vols + (i64)b * V * A.vol_stride + (i64)z * plane;

  for (int x0 = 0; x0 < X; x0 += A.XR) {
    const int nr = min(A.XR, X - x0);
    __syncthreads();
    for (int t = threadIdx.x; t < A.XR * Y; t += kThreads) {
      const int xr = t / Y, y = t - xr * Y;
      if (xr < nr) {
        const float2 m = mrow[(i64)(x0 + xr) * Y + y];
#pragma unroll
        for (int v = 0; v < V; v++) {
          const float2 u = vbase[(i64)v * A.vol_stride + (i64)(x0 + xr) * Y + y];
          buf0[y * A.es + v * A.XR + xr] = cmul(m, u);
        }
      } else {
#pragma unroll
        for (int v = 0; v < V; v++) buf0[y * A.es + v * A.XR + xr] = make_float2(0.f, 0.f);
      }
    }
    __syncthreads();
    const float2* G = fft_lines<false>(buf0, buf1, A.plan, L, A.es, twY);
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      if (mkx[m] < 0) continue;
      int idx = (int)(((long long)mkx[m] * x0) % X);
      const float2* grow = G + mky[m] * A.es;
      for (int xr = 0; xr < nr; xr++) {
        const float2 w = twX[idx];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v][m] = cadd(acc[v][m], cmul(grow[v * A.XR + xr], w));
        idx += mkx[m];
        if (idx >= X) idx -= X;
      }
    }
  }

  const i64 zc = (i64)z * A.C + c;
  if constexpr (MODE == FWD_K) {
    const i64 rel = A.kout_abs ? (i64)soff : (i64)(soff - A.shot_off[A.shot0]);
    const i64 base = rel * A.C * A.Z + zc * ns;
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int j = threadIdx.x + m * kThreads;
      if (j < ns) A.kout[base + j] = cscale(acc[0][m], A.scale);
    }
  } else if constexpr (MODE == FWD_RESID) {
    const i64 base = (i64)soff * A.C * A.Z + zc * ns;
    double e[1] = {0.0};
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int j = threadIdx.x + m * kThreads;
      if (j < ns) {
        const float2 r = csub(cscale(acc[0][m], A.scale), A.ydat[base + j]);
        e[0] += (double)r.x * r.x + (double)r.y * r.y;
      }
    }
    block_reduce_store<1>(e, A.partial + ((i64)b * A.Z * A.C + zc));
  } else {
    const i64 base = (i64)soff * A.C * A.Z + zc * ns;
    double st[kLmStats];
#pragma unroll
    for (int k = 0; k < kLmStats; k++) st[k] = 0.0;
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int j = threadIdx.x + m * kThreads;
      if (j >= ns) continue;
      const float2 r = csub(cscale(acc[0][m], A.scale), A.ydat[base + j]);
      float2 J[6];
#pragma unroll
      for (int p = 0; p < 6; p++) J[p] = cscale(acc[(p + 1) % V][m], A.scale);
      lm_accumulate(st, r, J);
    }
    block_reduce_store<kLmStats>(st, A.partial + ((i64)b * A.Z * A.C + zc) * kLmStats);
  }
}

struct AdjArgs {
  int X, Y, Z, C;
  const float2* mps;
  const float2* kin;
  int kin_rel;  // kin offsets relative to shot_off[shot0] (K workspace) or absolute (ydat)
  float2* out;
  i64 vol_stride;
  int shot0;
  const int* shot_off;
  const int* kx;
  const int* ky_off;
  const int* ky_order;  // may be null
  int XB, es;
  float scale;
  int bulk;  // stage map rows with bulk copies (bases 16-byte aligned; set on the host)
  FftPlan plan;
};

template <int EPT>
__global__ void __launch_bounds__(kThreads) sense_adj_kernel(const AdjArgs A) {
  extern __shared__ float2 sm[];
  const int z = blockIdx.x, x0 = blockIdx.y * A.XB, b = blockIdx.z;
  const int s = A.shot0 + b;
  const int X = A.X, Y = A.Y;
  const int nr = min(A.XB, X - x0);
  const int soff = A.shot_off[s];
  const int ns = A.shot_off[s + 1] - soff;
  float2* twY = sm;
  float2* twX = twY + pad2(Y);
  float2* Ks = twX + pad2(X);
  float2* buf0 = Ks + pad2(ns);
  float2* buf1 = buf0 + (i64)Y * A.es;
  init_twiddles(twY, Y);
  init_twiddles(twX, X);

  const int* kyo = A.ky_off + (i64)s * (Y + 1);
  const int* kxs = A.kx + soff;
  const i64 kbase0 = (A.kin_rel ? (i64)(soff - A.shot_off[A.shot0]) : (i64)soff) * A.C * A.Z;
  const i64 plane = (i64)X * Y;

  float2 w[EPT];
#pragma unroll
  for (int m = 0; m < EPT; m++) w[m] = make_float2(0.f, 0.f);

  for (int c = 0; c < A.C; c++) {
    __syncthreads();
    const float2* kc = A.kin + kbase0 + ((i64)z * A.C + c) * ns;
    for (int j = threadIdx.x; j < ns; j += kThreads) Ks[j] = kc[j];
    __syncthreads();
    for (int t = threadIdx.x; t < A.XB * Y; t += kThreads) {
      const int xr = t % A.XB, ky = t / A.XB;
      float2 acc = make_float2(0.f, 0.f);
      if (xr < nr) {
        const int x = x0 + xr;
        for (int j = kyo[ky]; j < kyo[ky + 1]; j++) {
          const int idx = (kxs[j] * x) % X;
          acc = cadd(acc, cmulc(Ks[j], twX[idx]));
        }
      }
      buf0[ky * A.es + xr] = acc;
    }
    __syncthreads();
    const float2* R = fft_lines<true>(buf0, buf1, A.plan, A.XB, A.es, twY);
    const float2* mrow = A.mps + ((i64)z * A.C + c) * plane + (i64)x0 * Y;
#pragma unroll
    for (int m = 0; m < EPT; m++) {
      const int e = threadIdx.x + m * kThreads;
      if (e < nr * Y) {
        const int xr = e / Y, y = e - xr * Y;
        w[m] = cadd(w[m], cmulc(R[y * A.es + xr], mrow[e]));
      }
    }
  }
  float2* o = A.out + (i64)b * A.vol_stride + (i64)z * plane + (i64)x0 * Y;
#pragma unroll
  for (int m = 0; m < EPT; m++) {
    const int e = threadIdx.x + m * kThreads;
    if (e < nr * Y) o[e] = cscale(w[m], A.scale);
  }
}

// ---------------------------------------------------------------- compile-time plane widths
// Fast variants of the two kernels above for line lengths Y with a register FFT plan
// (fft_reg.cuh).  Same arguments, layouts and results.

__device__ __forceinline__ void init_twiddles_any(float2* tw, int n) {
  const float2* g = nullptr;
  switch (n) {
#define ME_TW_CASE(N, R1, R2) \
  case N: g = tw##N; break;
    ME_FAST_LENGTHS(ME_TW_CASE)
#undef ME_TW_CASE
    default: break;
  }
  if (g) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) tw[k] = __ldg(g + k);
  } else {
    init_twiddles(tw, n);
  }
}

// (a * b) mod n for 0 <= a, b < n <= 512 (product < 2^18: exact in float).
__device__ __forceinline__ int mulmod(int a, int b, int n, float inv_n) {
  const int p = a * b;
  int q = __float2int_rd((float)p * inv_n);
  int r = p - q * n;
  if (r < 0) r += n;
  if (r >= n) r -= n;
  return r;
}

// Rows per chunk of the forward kernel (one row per thread group) and its shared-memory plan.
template <int Y, int R1, int R2>
struct FwdPlan {
  using F = LineFft<Y, R1, R2>;
  static constexpr int G = F::G;
  static constexpr int NG = kThreads / G;
  static constexpr int RC = NG;
  static constexpr int LS = F::LS;
  static constexpr int STAGE = 2 * RC * Y;  // staged map rows + image rows
  static constexpr int LINES = NG * LS;
};

template <int Y, int R1, int R2, int MPT, int MODE>
__global__ void __launch_bounds__(kThreads, ME_SENSE_MINB) fast_fwd_kernel(const FwdArgs A) {
  static_assert(MODE == FWD_K || MODE == FWD_RESID, "one volume per CTA");
  using P = FwdPlan<Y, R1, R2>;
  using F = typename P::F;
  constexpr int G = P::G, RC = P::RC, LS = P::LS;
  static_assert(RC % 2 == 0, "the two Horner chains take rows in pairs");
  extern __shared__ __align__(16) float2 sm[];
  // shots vary fastest, so the CTAs of all shots of one (z, coil) run together and share the
  // map plane (and each shot's image plane across coils) through L2
  const int bx = blockIdx.x, c = blockIdx.y, z = blockIdx.z;
  const int b = bx / A.vps, vk = bx - b * A.vps;  // shot in the batch, volume of the shot
  const int s = A.shot0 + b;
  const int X = A.X;
  float2* stage = sm;                 // [2][RC][Y]: map rows, then image rows
  float2* lines = stage + P::STAGE;   // one line region per thread group
  float2* twX = lines + P::LINES;
  init_twiddles_any(twX, X);

  const int soff = A.shot_off[s];
  const int ns = A.shot_off[s + 1] - soff;
  // per sample: kx, ky, the twiddle index kx x0 mod X of the current chunk and its step kx RC
  int mkx[MPT], mky[MPT], idx[MPT], dix[MPT];
  float2 acc[MPT];
#pragma unroll
  for (int m = 0; m < MPT; m++) {
    const int jj = threadIdx.x + m * kThreads;
    mkx[m] = -1;
    mky[m] = 0;
    idx[m] = 0;
    dix[m] = 0;
    if (jj < ns) {
      mkx[m] = A.kx[soff + jj];
      mky[m] = A.ky[soff + jj];
      dix[m] = mulmod(mkx[m], RC % X, X, 1.0f / (float)X);
    }
    acc[m] = make_float2(0.f, 0.f);
  }
  const int g = threadIdx.x / G, j = threadIdx.x % G;
  const i64 plane = (i64)X * Y;
  const float2* mrow = A.mps + ((i64)z * A.C + c) * plane;
  const float2* vbase = A.vols + (i64)bx * A.vol_stride + (i64)z * plane;

  // stage rows [x0, x0 + RC) of the map and of the image: the rows of a chunk are contiguous
  // both in the plane and in the stage, so each is one flat copy.  With A.bulk one thread
  // issues the two as bulk copies on the TMA engine (completion counted on `full`); otherwise
  // every thread issues 16-byte cp.async copies.
  __shared__ __align__(8) uint64_t full;
  const bool bulk = A.bulk != 0;
  if (bulk && threadIdx.x == 0) {
    mbar_init(&full, 1);
    fence_mbar_init();
  }
  auto issue = [&](int x0) {
    const float2* ms = mrow + (i64)x0 * Y;
    const float2* us = vbase + (i64)x0 * Y;
    if (bulk) {
      if (threadIdx.x == 0) {
        const unsigned bytes = (unsigned)(min(RC, X - x0) * Y * sizeof(float2));
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full, 2 * bytes);
        bulk_g2s(stage, ms, bytes, &full);
        bulk_g2s(stage + RC * Y, us, bytes, &full);
      }
      return;
    }
    const int nq = min(RC, X - x0) * (Y / 2);  // 16-byte chunks
    for (int q = threadIdx.x; q < nq; q += kThreads) {
      cp_async16(stage + 2 * q, ms + 2 * q);
      cp_async16(stage + RC * Y + 2 * q, us + 2 * q);
    }
    cp_async_commit();
  };

  issue(0);  // the barrier stays untouched by other threads until the __syncthreads below
  unsigned fphase = 0;
  // The Horner steps W^kx and W^2kx do not change between chunks: with few samples per thread
  // they are read from the table once (registers), else once per chunk.
  constexpr bool kHoist = MPT <= 2;
  float2 hst[kHoist ? MPT : 1], hst2[kHoist ? MPT : 1];
  __syncthreads();  // twX is written above by all threads
  if constexpr (kHoist) {
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int kx = mkx[m] < 0 ? 0 : mkx[m];
      const int k2 = 2 * kx >= X ? 2 * kx - X : 2 * kx;
      hst[m] = twX[kx];
      hst2[m] = twX[k2];
    }
  }
  for (int x0 = 0; x0 < X; x0 += RC) {
    const int nr = min(RC, X - x0);
    if (bulk) {
      mbar_wait_bounded(&full, fphase, WF_SENSE_FWD);
      fphase ^= 1;
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    {
      // FFT of map row x image row, the product formed as the first stage loads it; rows past
      // nr transform zeros
      float2* L = lines + g * LS;
      const float2* ms = stage + g * Y;
      const float2* us = stage + (RC + g) * Y;
      const bool live = g < nr;
      float2 Xr[R2];
      F::forward_from([&](int n) { return live ? cmul(ms[n], us[n]) : make_float2(0.f, 0.f); },
                      L, j, Xr);
      F::store_spectrum(L, j, Xr);
    }
    __syncthreads();
    if (x0 + RC < X) issue(x0 + RC);
    // Sample sums over the chunk's rows by Horner's rule, sum_row L[row] W^(kx row), then one
    // table twiddle W^(kx x0) per chunk.  Rows past nr hold zeros (zero lines transform to
    // zero), so every chunk runs all RC rows, in two interleaved chains (even and odd rows,
    // stepping by W^(2 kx)) so that two FMA chains are in flight.
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      if (mkx[m] < 0) continue;
      const float2 st = kHoist ? hst[m] : twX[mkx[m]];
      const float2 w0 = twX[idx[m]];
      const float2* Lk = lines + mky[m];
      int k2 = 2 * mkx[m];
      if (k2 >= X) k2 -= X;
      const float2 st2 = kHoist ? hst2[m] : twX[k2];
      float2 he = Lk[(RC - 2) * LS], ho = Lk[(RC - 1) * LS];
#pragma unroll
      for (int i = RC / 2 - 2; i >= 0; i--) {
        he = cfma(he, st2, Lk[(2 * i) * LS]);
        ho = cfma(ho, st2, Lk[(2 * i + 1) * LS]);
      }
      acc[m] = cfma(cfma(ho, st, he), w0, acc[m]);
      idx[m] += dix[m];
      if (idx[m] >= X) idx[m] -= X;
    }
  }

  const i64 zc = (i64)z * A.C + c;
  if constexpr (MODE == FWD_K) {
    const i64 rel = A.kout_abs ? (i64)soff : (i64)(soff - A.shot_off[A.shot0]);
    const i64 base = rel * A.C * A.Z + zc * ns;
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int jj = threadIdx.x + m * kThreads;
      if (jj < ns) A.kout[(i64)vk * A.kout_vs + base + jj] = cscale(acc[m], A.scale);
    }
  } else {
    const i64 base = (i64)soff * A.C * A.Z + zc * ns;
    double e[1] = {0.0};
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int jj = threadIdx.x + m * kThreads;
      if (jj < ns) {
        const float2 r = csub(cscale(acc[m], A.scale), A.ydat[base + jj]);
        e[0] += (double)r.x * r.x + (double)r.y * r.y;
      }
    }
    block_reduce_store<1>(e, A.partial + ((i64)b * A.Z * A.C + zc));
  }
}

// Gauss-Newton statistics of the LM step straight from the seven volumes of each shot (T x and
// its six partials, [shot][7] in A.vols): the forward model of all seven runs in one CTA per
// (shot, coil, plane), each chunk's map rows staged once for the seven volumes, and the sampled
// values J_v = M_s F C U_v are contracted in registers into e0 = |J_0 - y|^2, g_p = Re<J_0 - y,
// J_p> and H_pq = Re<J_p, J_q> (transform_estimation.py:39-68) instead of being written out.
// The sums per sample and their block reduction are those of lm_stats_kernel, in the same order,
// so the statistics are bit-identical to the two-kernel path.
template <int Y, int R1, int R2, int MPT>
__global__ void __launch_bounds__(kThreads, ME_SENSE_MINB) fast_lm_kernel(const FwdArgs A) {
  using P = FwdPlan<Y, R1, R2>;
  using F = typename P::F;
  constexpr int G = P::G, RC = P::RC, LS = P::LS;
  constexpr int NV = 7;
  static_assert(RC % 2 == 0, "the two Horner chains take rows in pairs");
  extern __shared__ __align__(16) float2 sm[];
  const int b = blockIdx.x, c = blockIdx.y, z = blockIdx.z;
  const int s = A.shot0 + b;
  const int X = A.X;
  float2* stage = sm;                // map rows [RC][Y], then one volume's image rows [RC][Y]
  float2* lines = stage + P::STAGE;  // one line region per thread group
  float2* twX = lines + P::LINES;
  init_twiddles_any(twX, X);

  const int soff = A.shot_off[s];
  const int ns = A.shot_off[s + 1] - soff;
  int mkx[MPT], mky[MPT], idx[MPT], dix[MPT];
  float2 acc[NV][MPT];
#pragma unroll
  for (int m = 0; m < MPT; m++) {
    const int jj = threadIdx.x + m * kThreads;
    mkx[m] = -1;
    mky[m] = 0;
    idx[m] = 0;
    dix[m] = 0;
    if (jj < ns) {
      mkx[m] = A.kx[soff + jj];
      mky[m] = A.ky[soff + jj];
      dix[m] = mulmod(mkx[m], RC % X, X, 1.0f / (float)X);
    }
#pragma unroll
    for (int v = 0; v < NV; v++) acc[v][m] = make_float2(0.f, 0.f);
  }
  const int g = threadIdx.x / G, j = threadIdx.x % G;
  const i64 plane = (i64)X * Y;
  const float2* mrow = A.mps + ((i64)z * A.C + c) * plane;
  const float2* vbase = A.vols + (i64)b * NV * A.vol_stride + (i64)z * plane;

  // stage the image rows [x0, x0 + RC) of volume v, with the map rows too when `map`
  __shared__ __align__(8) uint64_t full;
  const bool bulk = A.bulk != 0;
  if (bulk && threadIdx.x == 0) {
    mbar_init(&full, 1);
    fence_mbar_init();
  }
  auto issue = [&](int x0, int v, bool map) {
    const float2* ms = mrow + (i64)x0 * Y;
    const float2* us = vbase + (i64)v * A.vol_stride + (i64)x0 * Y;
    if (bulk) {
      if (threadIdx.x == 0) {
        const unsigned bytes = (unsigned)(min(RC, X - x0) * Y * sizeof(float2));
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full, map ? 2 * bytes : bytes);
        if (map) bulk_g2s(stage, ms, bytes, &full);
        bulk_g2s(stage + RC * Y, us, bytes, &full);
      }
      return;
    }
    const int nq = min(RC, X - x0) * (Y / 2);
    for (int q = threadIdx.x; q < nq; q += kThreads) {
      if (map) cp_async16(stage + 2 * q, ms + 2 * q);
      cp_async16(stage + RC * Y + 2 * q, us + 2 * q);
    }
    cp_async_commit();
  };

  issue(0, 0, true);  // the barrier stays untouched by other threads until the __syncthreads below
  unsigned fphase = 0;
  constexpr bool kHoist = MPT <= 2;
  float2 hst[kHoist ? MPT : 1], hst2[kHoist ? MPT : 1];
  __syncthreads();  // twX is written above by all threads
  if constexpr (kHoist) {
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      const int kx = mkx[m] < 0 ? 0 : mkx[m];
      const int k2 = 2 * kx >= X ? 2 * kx - X : 2 * kx;
      hst[m] = twX[kx];
      hst2[m] = twX[k2];
    }
  }
  for (int x0 = 0; x0 < X; x0 += RC) {
    const int nr = min(RC, X - x0);
#pragma unroll 1
    for (int v = 0; v < NV; v++) {
      if (bulk) {
        mbar_wait_bounded(&full, fphase, WF_SENSE_FWD);
        fphase ^= 1;
      } else {
        cp_async_wait_all();
      }
      __syncthreads();
      {
        float2* L = lines + g * LS;
        const float2* ms = stage + g * Y;
        const float2* us = stage + (RC + g) * Y;
        const bool live = g < nr;
        float2 Xr[R2];
        F::forward_from([&](int n) { return live ? cmul(ms[n], us[n]) : make_float2(0.f, 0.f); },
                        L, j, Xr);
        F::store_spectrum(L, j, Xr);
      }
      __syncthreads();
      if (v + 1 < NV) {
        issue(x0, v + 1, false);
      } else if (x0 + RC < X) {
        issue(x0 + RC, 0, true);
      }
      // sample sums of volume v over the chunk's rows (as fast_fwd_kernel)
#pragma unroll
      for (int m = 0; m < MPT; m++) {
        if (mkx[m] < 0) continue;
        const float2 st = kHoist ? hst[m] : twX[mkx[m]];
        const float2 w0 = twX[idx[m]];
        const float2* Lk = lines + mky[m];
        int k2 = 2 * mkx[m];
        if (k2 >= X) k2 -= X;
        const float2 st2 = kHoist ? hst2[m] : twX[k2];
        float2 he = Lk[(RC - 2) * LS], ho = Lk[(RC - 1) * LS];
#pragma unroll
        for (int i = RC / 2 - 2; i >= 0; i--) {
          he = cfma(he, st2, Lk[(2 * i) * LS]);
          ho = cfma(ho, st2, Lk[(2 * i + 1) * LS]);
        }
        // the accumulators rotate as a queue, so that volume v's is always acc[0] (v is not a
        // compile-time index); after the seven volumes of a chunk acc[u] is volume u's again
        const float2 nv = cfma(cfma(ho, st, he), w0, acc[0][m]);
#pragma unroll
        for (int u = 0; u < NV - 1; u++) acc[u][m] = acc[u + 1][m];
        acc[NV - 1][m] = nv;
      }
    }
#pragma unroll
    for (int m = 0; m < MPT; m++) {
      if (mkx[m] < 0) continue;
      idx[m] += dix[m];
      if (idx[m] >= X) idx[m] -= X;
    }
  }

  const i64 zc = (i64)z * A.C + c;
  const i64 yb = (i64)soff * A.C * A.Z + zc * ns;
  double st[kLmStats];
#pragma unroll
  for (int k = 0; k < kLmStats; k++) st[k] = 0.0;
#pragma unroll
  for (int m = 0; m < MPT; m++) {
    const int jj = threadIdx.x + m * kThreads;
    if (jj < ns) {
      // K rounded to float before the difference, as the two-kernel path stores it (a
      // contracted multiply-subtract would round differently)
      const float2 k0 = make_float2(__fmul_rn(acc[0][m].x, A.scale), __fmul_rn(acc[0][m].y, A.scale));
      const float2 r = csub(k0, A.ydat[yb + jj]);
      float2 J[6];
#pragma unroll
      for (int p = 0; p < 6; p++) J[p] = cscale(acc[1 + p][m], A.scale);
      lm_accumulate(st, r, J);
    }
  }
  block_reduce_store<kLmStats>(st, A.partial + ((i64)b * A.Z * A.C + zc) * kLmStats);
}

// Adjoint plan: one image row per thread group; the H rows are built by one thread per ky bin
// (and part of the rows), walking its samples with a twiddle recurrence along x.
template <int Y, int R1, int R2>
struct AdjPlan {
  using F = LineFft<Y, R1, R2>;
  static constexpr int G = F::G;
  static constexpr int NG = kThreads / G;
  static constexpr int LS = F::LS;
  static constexpr int NP0 = (kThreads / Y) < 1 ? 1 : (kThreads / Y);
  static constexpr int NPARTS = NP0 >= 16 ? 16 : NP0 >= 8 ? 8 : NP0 >= 4 ? 4 : NP0 >= 2 ? 2 : 1;
  static constexpr int RP = NG / NPARTS;  // rows per H-building thread
  // When one thread per bin leaves threads idle (Y < 256, all rows per thread), each idle
  // thread takes the second half of the rows of one of the heaviest bins (bins come sorted by
  // sample count), halving the longest walk; both halves write their own rows.
  static constexpr int NSPLIT = (NPARTS == 1 && Y < kThreads) ? (kThreads - Y < Y ? kThreads - Y : Y) : 0;
  static constexpr int RH = RP / 2;  // rows of each half of a shared bin
};

template <int Y, int R1, int R2>
__global__ void __launch_bounds__(kThreads, ME_SENSE_MINB) fast_adj_kernel(const AdjArgs A) {
  using P = AdjPlan<Y, R1, R2>;
  using F = typename P::F;
  constexpr int G = P::G, NG = P::NG, LS = P::LS, RP = P::RP, NSPLIT = P::NSPLIT;
  extern __shared__ __align__(16) float2 sm[];
  // shots vary fastest: the CTAs of all shots of one (z, row block) share the map rows in L2
  const int b = blockIdx.x, x0 = blockIdx.y * NG, z = blockIdx.z;
  const int s = A.shot0 + b;
  const int X = A.X;
  const int soff = A.shot_off[s];
  const int ns = A.shot_off[s + 1] - soff;
  const int kcap = (A.XB + 1) & ~1;            // max samples per shot, padded
  float2* mstage = sm;                          // 2 x [NG][Y] maps rows
  float2* Kb = mstage + 2 * NG * Y;             // 2 x kcap samples
  float2* lines = Kb + 2 * kcap;                // NG x LS
  float2* twX = lines + NG * LS;
  // with NSPLIT > 0: per-sample twiddles shared by all coils, conj W^(kx x0), conj W^(kx (x0 +
  // RH)) and conj W^kx
  float2* tw_a = twX + pad2(X);
  float2* tw_b = tw_a + kcap;
  float2* tw_s = tw_b + kcap;
  init_twiddles_any(twX, X);

  const int g = threadIdx.x / G, j = threadIdx.x % G;
  const int x = x0 + g;
  const int nrows = min(NG, X - x0);
  const float inv_x = 1.0f / (float)X;
  const int* kyo = A.ky_off + (i64)s * (Y + 1);
  const int* kxs = A.kx + soff;
  const i64 kbase0 = (A.kin_rel ? (i64)(soff - A.shot_off[A.shot0]) : (i64)soff) * A.C * A.Z;
  const i64 plane = (i64)X * Y;
  if constexpr (NSPLIT > 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kThreads) {
      const int kx = kxs[i];
      tw_s[i] = cconj(twX[kx]);
      tw_a[i] = cconj(twX[mulmod(kx, min(x0, X - 1), X, inv_x)]);
      tw_b[i] = cconj(twX[mulmod(kx, min(x0 + P::RH, X - 1), X, inv_x)]);
    }
  }

  // H-building role: bin hb, rows [hr0, hr0 + RP), or [hr0, hr0 + RH) for a shared bin
  const bool split = (NSPLIT > 0) && (A.ky_order != nullptr);
  int hb = 0, hr0 = 0;
  bool hbuild = false, half = false;
  if ((int)threadIdx.x < Y * P::NPARTS) {
    const int slot = threadIdx.x % Y;
    hb = A.ky_order ? A.ky_order[(i64)s * Y + slot] : slot;
    hr0 = (threadIdx.x / Y) * RP;
    hbuild = true;
    half = split && slot < NSPLIT;
  } else if (split && (int)threadIdx.x - Y < NSPLIT) {
    hb = A.ky_order[(i64)s * Y + (threadIdx.x - Y)];
    hr0 = P::RH;
    hbuild = true;
    half = true;
  }
  const int hlo = hbuild ? kyo[hb] : 0, hhi = hbuild ? kyo[hb + 1] : 0;

  // map rows of coil c into buffer c & 1: with A.bulk one bulk copy on the TMA engine
  // (completion counted on full[c & 1]), otherwise 16-byte cp.async copies; the coil's samples
  // (8-byte aligned only) always by cp.async
  __shared__ __align__(8) uint64_t full[2];
  const bool bulk = A.bulk != 0;
  if (bulk && threadIdx.x == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    fence_mbar_init();
  }
  auto issue = [&](int c) {
    const float2* mr = A.mps + ((i64)z * A.C + c) * plane + (i64)x0 * Y;
    float2* dst = mstage + (c & 1) * NG * Y;
    if (bulk) {
      if (threadIdx.x == 0) {
        const unsigned bytes = (unsigned)(nrows * Y * sizeof(float2));
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full[c & 1], bytes);
        bulk_g2s(dst, mr, bytes, &full[c & 1]);
      }
    } else {
      const int nq = nrows * Y / 2;
      for (int q = threadIdx.x; q < nq; q += kThreads) cp_async16(dst + 2 * q, mr + 2 * q);
    }
    const float2* kc = A.kin + kbase0 + ((i64)z * A.C + c) * ns;
    float2* kd = Kb + (c & 1) * kcap;
    for (int i = threadIdx.x; i < ns; i += kThreads) cp_async8(kd + i, kc + i);
    cp_async_commit();
  };

  // image row accumulators in the inverse FFT's output layout: thread j < R2 owns y = j + b R2
  float2 w[R1];
#pragma unroll
  for (int m = 0; m < R1; m++) w[m] = make_float2(0.f, 0.f);
  float2* L = lines + g * LS;

  if (bulk) __syncthreads();  // the barriers are initialised before any thread waits on them
  issue(0);
  for (int c = 0; c < A.C; c++) {
    cp_async_wait_all();
    if (bulk) mbar_wait_bounded(&full[c & 1], (c >> 1) & 1, WF_SENSE_ADJ);
    __syncthreads();
    if (c + 1 < A.C) issue(c + 1);
    const float2* K = Kb + (c & 1) * kcap;
    if (hbuild) {
      // H[x][ky] += K exp(+2 pi i kx x / X): the term itself steps by conj(W^kx) per row
      float2 h[RP];
#pragma unroll
      for (int r = 0; r < RP; r++) h[r] = make_float2(0.f, 0.f);
      if constexpr (NSPLIT > 0) {
        const float2* tw0 = (hr0 == 0) ? tw_a : tw_b;
        if (half) {
          for (int i = hlo; i < hhi; i++) {
            const float2 st = tw_s[i];
            float2 v = cmul(K[i], tw0[i]);
#pragma unroll
            for (int r = 0; r < P::RH; r++) {
              h[r] = cadd(h[r], v);
              v = cmul(v, st);
            }
          }
#pragma unroll
          for (int r = 0; r < P::RH; r++) lines[(hr0 + r) * LS + hb] = h[r];
        } else {
          for (int i = hlo; i < hhi; i++) {
            const float2 st = tw_s[i];
            float2 v = cmul(K[i], tw0[i]);
#pragma unroll
            for (int r = 0; r < RP; r++) {
              h[r] = cadd(h[r], v);
              v = cmul(v, st);
            }
          }
#pragma unroll
          for (int r = 0; r < RP; r++) lines[(hr0 + r) * LS + hb] = h[r];
        }
      } else {
        for (int i = hlo; i < hhi; i++) {
          const int kx = kxs[i];
          const float2 st = twX[kx];
          float2 v = cmulc(K[i], twX[mulmod(kx, min(x0 + hr0, X - 1), X, inv_x)]);
#pragma unroll
          for (int r = 0; r < RP; r++) {
            h[r] = cadd(h[r], v);
            v = cmulc(v, st);
          }
        }
#pragma unroll
        for (int r = 0; r < RP; r++) lines[(hr0 + r) * LS + hb] = h[r];
      }
    }
    __syncthreads();
    float2 Xr[R2];
    F::load_spectrum(L, j, Xr);
    const float2* ms = mstage + (c & 1) * NG * Y + g * Y;
    F::inverse_to(L, j, Xr, [&](int q, int y, float2 v) { w[q] = cadd(w[q], cmulc(v, ms[y])); });
  }
  if (g < nrows && j < R2) {
    float2* o = A.out + (i64)b * A.vol_stride + (i64)z * plane + (i64)x * Y;
#pragma unroll
    for (int q = 0; q < R1; q++) o[j + q * R2] = cscale(w[q], A.scale);
  }
}

// Gauss-Newton sums from the sampled T x and its six partials, written by the forward kernel
// into seven K regions kvs apart (offsets relative to the batch's first shot); one CTA per
// (z, coil) plane and shot, FP64 sums reduced in a fixed order.
__global__ void __launch_bounds__(kThreads) lm_stats_kernel(const float2* __restrict__ K, i64 kvs,
                                                            const float2* __restrict__ ydat,
                                                            const int* __restrict__ shot_off,
                                                            int shot0, int ZC,
                                                            double* __restrict__ partial) {
  const i64 zc = blockIdx.x;
  const int b = blockIdx.y;
  const int s = shot0 + b;
  const int soff = shot_off[s], ns = shot_off[s + 1] - soff;
  const i64 kb = (i64)(soff - shot_off[shot0]) * ZC + zc * ns;
  const i64 yb = (i64)soff * ZC + zc * ns;
  double st[kLmStats];
#pragma unroll
  for (int k = 0; k < kLmStats; k++) st[k] = 0.0;
  for (int j = threadIdx.x; j < ns; j += kThreads) {
    const float2 r = csub(K[kb + j], ydat[yb + j]);
    float2 J[6];
#pragma unroll
    for (int p = 0; p < 6; p++) J[p] = K[(p + 1) * kvs + kb + j];
    lm_accumulate(st, r, J);
  }
  block_reduce_store<kLmStats>(st, partial + ((i64)b * ZC + zc) * kLmStats);
}

// Geodesic-acceleration direction volumes.  For each shot b of the batch, with its six partial
// volumes U_b[1 + p] (a Jacobian sweep, shot block of `bs` elements) and its step v_b:
//   first pass  (first = 1): D_b = sum_p v_bp U_b[1 + p]          (ga_mode 1, intended), or
//                            D_b = (1 + v_b5) U_b[6]               (ga_mode 0, as the reference
//                            computes it: its accumulator is overwritten by each partial, so only
//                            the last one, scaled by 1 + v_5, survives)
//   second pass (first = 0): D_b = (D_b - sum_p v_bp U_b[1 + p]) / eps
// D_b lives at U_b[7].
__global__ void ga_combine_kernel(float2* __restrict__ U, i64 bs, i64 vox, int nb,
                                  const double* __restrict__ v, int ga_mode, int first,
                                  double eps) {
  const i64 n = (i64)nb * vox;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const int b = (int)(i / vox);
    const i64 e = i - (i64)b * vox;
    float2* u = U + (i64)b * bs + e;
    const double* vb = v + (i64)b * 6;
    float2 d;
    if (first && ga_mode == 0) {
      d = cscale(u[6 * vox], (float)(1.0 + vb[5]));
    } else {
      d = make_float2(0.f, 0.f);
#pragma unroll
      for (int p = 0; p < 6; p++) d = cadd(d, cscale(u[(1 + p) * vox], (float)vb[p]));
      if (!first) d = cscale(csub(u[7 * vox], d), (float)(1.0 / eps));
    }
    u[7 * vox] = d;
  }
}

// rhs partials: -Re<K_D, K_p> for p = 0..5 over one (z, coil) plane of a shot, with the six
// partials' K in regions 0..5 and the direction's in region 6 (kvs apart).
__global__ void __launch_bounds__(kThreads) ga_dots_kernel(const float2* __restrict__ K, i64 kvs,
                                                           const int* __restrict__ shot_off,
                                                           int shot0, int ZC,
                                                           double* __restrict__ partial) {
  const i64 zc = blockIdx.x;
  const int b = blockIdx.y;
  const int s = shot0 + b;
  const int soff = shot_off[s], ns = shot_off[s + 1] - soff;
  const i64 kb = (i64)(soff - shot_off[shot0]) * ZC + zc * ns;
  double st[6];
#pragma unroll
  for (int p = 0; p < 6; p++) st[p] = 0.0;
  for (int j = threadIdx.x; j < ns; j += kThreads) {
    const float2 d = K[6 * kvs + kb + j];
#pragma unroll
    for (int p = 0; p < 6; p++) {
      const float2 jp = K[p * kvs + kb + j];
      st[p] -= (double)d.x * jp.x + (double)d.y * jp.y;
    }
  }
  block_reduce_store<6>(st, partial + ((i64)b * ZC + zc) * 6);
}

// Residual in place over one (z, coil) plane of a shot, and its energy partial: r = K - y for
// the gradient-only statistics (me_lm_gradient), r = y - K (YMK) for the CG's initial residual
// (me_sense_residual).  |r|^2 is the same either way.
template <bool YMK>
__global__ void __launch_bounds__(kThreads) resid_inplace_kernel(float2* __restrict__ K,
                                                                 const float2* __restrict__ ydat,
                                                                 const int* __restrict__ shot_off,
                                                                 int shot0, int ZC,
                                                                 double* __restrict__ partial) {
  const i64 zc = blockIdx.x;
  const int b = blockIdx.y;
  const int s = shot0 + b;
  const int soff = shot_off[s], ns = shot_off[s + 1] - soff;
  const i64 kb = (i64)(soff - shot_off[shot0]) * ZC + zc * ns;
  const i64 yb = (i64)soff * ZC + zc * ns;
  double e[1] = {0.0};
  for (int j = threadIdx.x; j < ns; j += kThreads) {
    const float2 r = YMK ? csub(ydat[yb + j], K[kb + j]) : csub(K[kb + j], ydat[yb + j]);
    K[kb + j] = r;
    e[0] += (double)r.x * r.x + (double)r.y * r.y;
  }
  block_reduce_store<1>(e, partial + ((i64)b * ZC + zc));
}

// Re<W_b, U_b[1 + p]> partials, p = 0..5, over a grid-stride share of the volume of shot b
// (W_b = U_b[7], shot block of bs elements).
__global__ void __launch_bounds__(kThreads) grad_dots_kernel(const float2* __restrict__ U, i64 bs,
                                                             i64 vox, double* __restrict__ partial) {
  const int b = blockIdx.y;
  const float2* u = U + (i64)b * bs;
  double st[6];
#pragma unroll
  for (int p = 0; p < 6; p++) st[p] = 0.0;
  for (i64 i = blockIdx.x * (i64)kThreads + threadIdx.x; i < vox; i += (i64)gridDim.x * kThreads) {
    const float2 w = u[7 * vox + i];
#pragma unroll
    for (int p = 0; p < 6; p++) {
      const float2 d = u[(1 + p) * vox + i];
      st[p] += (double)w.x * d.x + (double)w.y * d.y;
    }
  }
  block_reduce_store<6>(st, partial + ((i64)b * gridDim.x + blockIdx.x) * 6);
}

// grad[shot0 + b] = {sum of the ZC energy partials, sums of the nblk dot partials}, in order.
__global__ void grad_finish_kernel(const double* __restrict__ epart, int ZC,
                                   const double* __restrict__ dpart, int nblk,
                                   double* __restrict__ grad, int shot0) {
  const int b = blockIdx.x;
  if (threadIdx.x > 6) return;
  double a = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < ZC; i++) a += epart[(i64)b * ZC + i];
  } else {
    const int p = threadIdx.x - 1;
    for (int i = 0; i < nblk; i++) a += dpart[((i64)b * nblk + i) * 6 + p];
  }
  grad[(i64)(shot0 + b) * 7 + threadIdx.x] = a;
}

// out[i] = M[i] * ((out[i] if accumulate) + sum_b vols[b][i])
__global__ void sum_volumes_kernel(const float2* __restrict__ vols, i64 vs, int nb,
                                   const unsigned char* __restrict__ M, float2* __restrict__ out,
                                   i64 n, int accumulate) {
  // The running sum starts from out and adds the batch's shots in order, so the sum over all
  // shots is the same sequence of additions whatever the shots-per-launch batch.
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    float2 a = accumulate ? out[i] : make_float2(0.f, 0.f);
    for (int b = 0; b < nb; b++) a = cadd(a, vols[(i64)b * vs + i]);
    if (M && !M[i]) a = make_float2(0.f, 0.f);
    out[i] = a;
  }
}

// stats[shot0 + b][k] = sum over the Z*C partials of batch entry b
__global__ void reduce_partials_kernel(const double* __restrict__ partial, int nparts, int nstat,
                                       double* __restrict__ out, int shot0) {
  const int b = blockIdx.x;
  for (int k = 0; k < nstat; k++) {
    double a = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) a += partial[((i64)b * nparts + i) * nstat + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
      out[(i64)(shot0 + b) * nstat + k] = t;
    }
    __syncthreads();
  }
}

__global__ void precond_kernel(const float2* __restrict__ mps, int C, i64 plane, int Z, float* P,
                               unsigned char* M) {
  const i64 n = plane * Z;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const i64 z = i / plane, r = i - z * plane;
    float a = 0.f;
    for (int c = 0; c < C; c++) {
      const float2 m = mps[(z * C + c) * plane + r];
      a += m.x * m.x + m.y * m.y;
    }
    P[i] = 1.0f / (a + 1e-3f);
    M[i] = a > 0.1f ? 1 : 0;
  }
}

// ydat[shot s][z][c][j] = ksp_h[c][kx_j][ky_j][z]
__global__ void gather_kernel(const float2* __restrict__ ksp, int X, int Y, int Z, int C,
                              const int* shot_off, const int* kx, const int* ky, int nshots,
                              float2* __restrict__ ydat) {
  const i64 total = (i64)shot_off[nshots] * C * Z;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < total; i += (i64)gridDim.x * blockDim.x) {
    const int z = (int)(i % Z);
    const i64 rest = i / Z;
    const int c = (int)(rest % C);
    const int g = (int)(rest / C);  // global sample index
    // find the shot of sample g (binary search on shot_off)
    int lo = 0, hi = nshots;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (shot_off[mid] <= g) lo = mid; else hi = mid;
    }
    const int s = lo, ns = shot_off[s + 1] - shot_off[s], j = g - shot_off[s];
    const float2 v = ksp[(((i64)c * X + kx[g]) * Y + ky[g]) * Z + z];
    ydat[(i64)shot_off[s] * C * Z + ((i64)z * C + c) * ns + j] = v;
  }
}

// ksp_h[c][kx][ky][z] += K[s][z][c][j] for the samples of shot s (no duplicates within a shot)
__global__ void scatter_kernel(const float2* __restrict__ K, int X, int Y, int Z, int C,
                               const int* shot_off, const int* kx, const int* ky, int s,
                               float2* __restrict__ ksp) {
  const int soff = shot_off[s], ns = shot_off[s + 1] - soff;
  const i64 total = (i64)ns * C * Z;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < total; i += (i64)gridDim.x * blockDim.x) {
    const int z = (int)(i % Z);
    const i64 rest = i / Z;
    const int c = (int)(rest % C);
    const int j = (int)(rest / C);
    const int g = soff + j;
    const float2 v = K[(i64)soff * C * Z + ((i64)z * C + c) * ns + j];
    float2* d = ksp + (((i64)c * X + kx[g]) * Y + ky[g]) * Z + z;
    *d = cadd(*d, v);
  }
}

// ------------------------------------------------------------------------------ launchers
static int grid_1d(i64 n) {
  i64 b = (n + kThreads - 1) / kThreads;
  return (int)std::min<i64>(b, 148LL * 16);
}

static int check_problem(const me_sense* pb) {
  if (!pb) return fail("problem is NULL");
  if (pb->nx < 1 || pb->ny < 1 || pb->nz < 1 || pb->ncoils < 1 || pb->nshots < 1)
    return fail("problem dims must be positive");
  if (!pb->mps || !pb->samples.shot_off || !pb->samples.kx || !pb->samples.ky ||
      !pb->samples.ky_off || !pb->grid || !pb->transforms)
    return fail("problem has a NULL pointer");
  if (pb->samples.nshots != pb->nshots || pb->samples.nx != pb->nx || pb->samples.ny != pb->ny)
    return fail("samples do not match the problem dims");
  if (pb->grid->nx != pb->nx || pb->grid->ny != pb->ny || pb->grid->nz != pb->nz)
    return fail("grid does not match the problem dims");
  if (pb->samples.max_per_shot > 8 * kThreads)
    return fail("a shot has more than 2048 samples per plane; unsupported");
  if (pb->nx > ME_MAX_LINE || pb->ny > ME_MAX_LINE) return fail("plane too large");
  return ME_OK;
}

static me_layout zxy_layout(const me_sense* pb) {
  me_layout l;
  l.sx = pb->ny;
  l.sy = 1;
  l.sz = (i64)pb->nx * pb->ny;
  return l;
}

static i64 vox_of(const me_sense* pb) { return (i64)pb->nx * pb->ny * pb->nz; }

static int fwd_rows(int V, int Y) {
  int xr = (V == 1) ? 16 : 4;
  while (xr > 1 && 2 * (i64)Y * (V * xr + 1) * 8 > 160 * 1024) xr /= 2;
  return xr;
}

template <int MPT, int V, int MODE>
static int launch_fwd_t(FwdArgs& A, int nb, cudaStream_t st) {
  A.es = V * A.XR + 1;
  const size_t smem = sizeof(float2) * (pad2(A.Y) + pad2(A.X) + 2 * (size_t)A.Y * A.es);
  ME_TRY(check_cuda(allow_smem(sense_fwd_kernel<MPT, V, MODE>, smem), "sense_fwd smem"));
  dim3 grid(A.Z, A.C, nb);
  count_launch();
  sense_fwd_kernel<MPT, V, MODE><<<grid, kThreads, smem, st>>>(A);
  return check_cuda(cudaGetLastError(), "sense_fwd launch");
}

template <int V, int MODE>
static int launch_fwd_v(FwdArgs& A, int maxps, int nb, cudaStream_t st) {
  if (maxps <= kThreads) return launch_fwd_t<1, V, MODE>(A, nb, st);
  if (maxps <= 2 * kThreads) return launch_fwd_t<2, V, MODE>(A, nb, st);
  if (maxps <= 4 * kThreads) return launch_fwd_t<4, V, MODE>(A, nb, st);
  return launch_fwd_t<8, V, MODE>(A, nb, st);
}

// Row staging by bulk copies (TMA engine) unless ME_NO_BULK=1; used where every staged range
// starts on a 16-byte boundary.
static bool bulk_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ME_NO_BULK");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}
static bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

ME_WAIT_FAULT_ACCESSOR(sense_wait_fault)

// The LM statistics from the fused seven-volume kernel unless ME_LM_TWO_PASS=1 (the forward
// kernel writing seven K regions, then lm_stats_kernel; bit-identical, kept for comparison).
static bool fused_lm_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ME_LM_TWO_PASS");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

static bool fast_sense_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("ME_GENERIC_FFT");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

template <int Y, int R1, int R2, int MPT, int MODE>
static int launch_fast_fwd_t(FwdArgs& A, int nb, cudaStream_t st) {
  using P = FwdPlan<Y, R1, R2>;
  const size_t smem = sizeof(float2) * ((size_t)P::STAGE + P::LINES + pad2(A.X));
  ME_TRY(check_cuda(allow_smem(fast_fwd_kernel<Y, R1, R2, MPT, MODE>, smem), "fwd smem"));
  dim3 grid(nb * A.vps, A.C, A.Z);
  count_launch();
  fast_fwd_kernel<Y, R1, R2, MPT, MODE><<<grid, kThreads, smem, st>>>(A);
  return check_cuda(cudaGetLastError(), "fast sense_fwd launch");
}

template <int Y, int R1, int R2, int MODE>
static int launch_fast_fwd_m(FwdArgs& A, int maxps, int nb, cudaStream_t st) {
  if (maxps <= kThreads) return launch_fast_fwd_t<Y, R1, R2, 1, MODE>(A, nb, st);
  if (maxps <= 2 * kThreads) return launch_fast_fwd_t<Y, R1, R2, 2, MODE>(A, nb, st);
  if (maxps <= 4 * kThreads) return launch_fast_fwd_t<Y, R1, R2, 4, MODE>(A, nb, st);
  return launch_fast_fwd_t<Y, R1, R2, 8, MODE>(A, nb, st);
}

template <int Y, int R1, int R2, int MPT>
static int launch_fast_lm_t(FwdArgs& A, int nb, cudaStream_t st) {
  using P = FwdPlan<Y, R1, R2>;
  const size_t smem = sizeof(float2) * ((size_t)P::STAGE + P::LINES + pad2(A.X));
  ME_TRY(check_cuda(allow_smem(fast_lm_kernel<Y, R1, R2, MPT>, smem), "lm smem"));
  dim3 grid(nb, A.C, A.Z);
  count_launch();
  fast_lm_kernel<Y, R1, R2, MPT><<<grid, kThreads, smem, st>>>(A);
  return check_cuda(cudaGetLastError(), "fast lm launch");
}

// The fused statistics kernel keeps seven accumulators per sample in registers: up to two
// samples per thread (512 per shot); more take the two-kernel path.
template <int Y, int R1, int R2>
static int launch_fast_lm_y(FwdArgs& A, int maxps, int nb, cudaStream_t st) {
  if (maxps <= kThreads) return launch_fast_lm_t<Y, R1, R2, 1>(A, nb, st);
  if (maxps <= 2 * kThreads) return launch_fast_lm_t<Y, R1, R2, 2>(A, nb, st);
  return -1;
}

static int try_fast_lm(FwdArgs& A, int maxps, int nb, cudaStream_t st) {
  switch (A.Y) {
#define ME_LM_CASE(N, R1, R2) \
  case N: return launch_fast_lm_y<N, R1, R2>(A, maxps, nb, st);
    ME_FAST_LENGTHS(ME_LM_CASE)
#undef ME_LM_CASE
    default: return -1;
  }
}

// The compile-time kernels take one volume per CTA (FWD_K, FWD_RESID); the seven-volume LM
// statistics use FWD_K over seven volumes per shot and lm_stats_kernel instead of FWD_LM.
template <int Y, int R1, int R2>
static int launch_fast_fwd_y(FwdArgs& A, int mode, int maxps, int nb, cudaStream_t st) {
  if (mode == FWD_K) return launch_fast_fwd_m<Y, R1, R2, FWD_K>(A, maxps, nb, st);
  if (mode == FWD_RESID) return launch_fast_fwd_m<Y, R1, R2, FWD_RESID>(A, maxps, nb, st);
  return -1;
}

static int try_fast_fwd(FwdArgs& A, int mode, int maxps, int nb, cudaStream_t st) {
  switch (A.Y) {
#define ME_FWD_CASE(N, R1, R2) \
  case N: return launch_fast_fwd_y<N, R1, R2>(A, mode, maxps, nb, st);
    ME_FAST_LENGTHS(ME_FWD_CASE)
#undef ME_FWD_CASE
    default: return -1;
  }
}

template <int Y, int R1, int R2>
static int launch_fast_adj_y(AdjArgs& A, int maxps, int nb, cudaStream_t st) {
  using P = AdjPlan<Y, R1, R2>;
  constexpr int NG = P::NG;
  A.XB = maxps;
  const size_t smem = sizeof(float2) * (2 * (size_t)NG * Y + 2 * (size_t)pad2(maxps) +
                                        (size_t)NG * P::LS + pad2(A.X) +
                                        (P::NSPLIT > 0 ? 3 * (size_t)pad2(maxps) : 0));
  ME_TRY(check_cuda(allow_smem(fast_adj_kernel<Y, R1, R2>, smem), "adj smem"));
  dim3 grid(nb, (A.X + NG - 1) / NG, A.Z);
  count_launch();
  fast_adj_kernel<Y, R1, R2><<<grid, kThreads, smem, st>>>(A);
  return check_cuda(cudaGetLastError(), "fast sense_adj launch");
}

static int try_fast_adj(AdjArgs& A, int maxps, int nb, cudaStream_t st) {
  switch (A.Y) {
#define ME_ADJ_CASE(N, R1, R2) \
  case N: return launch_fast_adj_y<N, R1, R2>(A, maxps, nb, st);
    ME_FAST_LENGTHS(ME_ADJ_CASE)
#undef ME_ADJ_CASE
    default: return -1;
  }
}

static bool has_fast_length(int n) {
  switch (n) {
#define ME_HAS_CASE(N, R1, R2) \
  case N: return true;
    ME_FAST_LENGTHS(ME_HAS_CASE)
#undef ME_HAS_CASE
    default: return false;
  }
}

// Whether the compile-time SENSE kernels serve this problem (they take the K of several
// volumes per shot in one launch, which the LM statistics use).
static bool fast_sense_for(const me_sense* pb) {
  return fast_sense_enabled() && pb->nx <= 512 && has_fast_length(pb->ny);
}

static int launch_fwd(const me_sense* pb, int mode, const float2* vols, i64 vol_stride, int shot0,
                      int nb, float2* kout, double* partial, cudaStream_t st, int kout_abs = 0,
                      int vps = 1, i64 kout_vs = 0) {
  FwdArgs A{};
  A.kout_abs = kout_abs;
  A.vps = vps;
  A.kout_vs = kout_vs;
  A.X = pb->nx;
  A.Y = pb->ny;
  A.Z = pb->nz;
  A.C = pb->ncoils;
  A.mps = (const float2*)pb->mps;
  A.vols = vols;
  A.vol_stride = vol_stride;
  A.shot0 = shot0;
  A.shot_off = pb->samples.shot_off;
  A.kx = pb->samples.kx;
  A.ky = pb->samples.ky;
  A.ydat = (const float2*)pb->ydat;
  A.kout = kout;
  A.partial = partial;
  A.scale = (float)(1.0 / sqrt((double)pb->nx * pb->ny));
  if (!make_plan(pb->ny, &A.plan)) {
    set_error("ny has a prime factor > 13");
    return ME_ERR_UNSUPPORTED;
  }
  const int maxps = pb->samples.max_per_shot;
  A.bulk = bulk_enabled() && al16(A.mps) && al16(A.vols) && vol_stride % 2 == 0 &&
           pb->ny % 2 == 0;
  if (fast_sense_enabled() && pb->nx <= 512) {
    // FWD_LM over the seven volumes of each shot: the fused statistics kernel, or -1 (not
    // handled) for the caller's two-kernel path
    if (mode == FWD_LM && vps == 7) return fused_lm_enabled() ? try_fast_lm(A, maxps, nb, st) : -1;
    const int rc = try_fast_fwd(A, mode, maxps, nb, st);
    if (rc >= 0) return rc;
  }
  if (vps != 1) {
    set_error("several volumes per shot need the compile-time SENSE kernels");
    return ME_ERR_UNSUPPORTED;
  }
  if (mode == FWD_LM) {
    A.XR = fwd_rows(7, pb->ny);
    return launch_fwd_v<7, FWD_LM>(A, maxps, nb, st);
  }
  A.XR = fwd_rows(1, pb->ny);
  if (mode == FWD_K) return launch_fwd_v<1, FWD_K>(A, maxps, nb, st);
  return launch_fwd_v<1, FWD_RESID>(A, maxps, nb, st);
}

static int launch_fwd_abs(const me_sense* pb, const float2* vols, i64 vol_stride, int shot0,
                          int nb, float2* kout, cudaStream_t st) {
  return launch_fwd(pb, FWD_K, vols, vol_stride, shot0, nb, kout, nullptr, st, 1);
}

template <int EPT>
static int launch_adj_t(AdjArgs& A, int maxps, int nb, cudaStream_t st) {
  A.es = A.XB + 1;
  const size_t smem =
      sizeof(float2) * (pad2(A.Y) + pad2(A.X) + pad2(maxps) + 2 * (size_t)A.Y * A.es);
  ME_TRY(check_cuda(allow_smem(sense_adj_kernel<EPT>, smem), "sense_adj smem"));
  dim3 grid(A.Z, (A.X + A.XB - 1) / A.XB, nb);
  count_launch();
  sense_adj_kernel<EPT><<<grid, kThreads, smem, st>>>(A);
  return check_cuda(cudaGetLastError(), "sense_adj launch");
}

static int launch_adj(const me_sense* pb, const float2* kin, int kin_rel, float2* out, i64 vs,
                      int shot0, int nb, cudaStream_t st) {
  AdjArgs A{};
  A.X = pb->nx;
  A.Y = pb->ny;
  A.Z = pb->nz;
  A.C = pb->ncoils;
  A.mps = (const float2*)pb->mps;
  A.kin = kin;
  A.kin_rel = kin_rel;
  A.out = out;
  A.vol_stride = vs;
  A.shot0 = shot0;
  A.shot_off = pb->samples.shot_off;
  A.kx = pb->samples.kx;
  A.ky_off = pb->samples.ky_off;
  A.ky_order = pb->samples.ky_order;
  A.scale = (float)(1.0 / sqrt((double)pb->nx * pb->ny));
  if (!make_plan(pb->ny, &A.plan)) {
    set_error("ny has a prime factor > 13");
    return ME_ERR_UNSUPPORTED;
  }
  A.bulk = bulk_enabled() && al16(A.mps) && pb->ny % 2 == 0;
  if (fast_sense_enabled() && pb->nx <= 512) {
    const int rc = try_fast_adj(A, pb->samples.max_per_shot, nb, st);
    if (rc >= 0) return rc;
  }
  A.XB = std::max(1, std::min(std::min(pb->nx, 32), 4096 / pb->ny));
  const int ept = (A.XB * pb->ny + kThreads - 1) / kThreads;
  const int maxps = pb->samples.max_per_shot;
  if (ept <= 4) return launch_adj_t<4>(A, maxps, nb, st);
  if (ept <= 8) return launch_adj_t<8>(A, maxps, nb, st);
  return launch_adj_t<16>(A, maxps, nb, st);
}

// Blocks per shot of the gradient's image-space dot products, and the partial sums it keeps
// per shot: one energy partial per (z, coil) plane, then six per block.
constexpr int kGradBlocks = 296;
static i64 grad_partials(const me_sense* pb) {
  return (i64)pb->nz * pb->ncoils + 6LL * kGradBlocks;
}

struct Ws {
  float2* U;
  float2* K;
  double* partial;
  i64 kvs;  // elements per K region (one region per volume of a shot)
};

static i64 align256(i64 n) { return (n + 255) & ~255LL; }

static i64 ws_layout(const me_sense* pb, int batch, int vols_per_shot, int extra_vols, Ws* w,
                     void* base, int kvols = 1, i64 min_partials_per_shot = 0) {
  const i64 vox = vox_of(pb);
  const i64 nU = (i64)batch * vols_per_shot * vox + (i64)extra_vols * vox;
  const i64 nK1 = (i64)batch * pb->samples.max_per_shot * pb->ncoils * pb->nz;
  const i64 nK = nK1 * kvols;
  const i64 nP = (i64)batch * std::max<i64>((i64)pb->nz * pb->ncoils * kLmStats,
                                            min_partials_per_shot);
  const i64 bU = align256(nU * 8), bK = align256(nK * 8), bP = align256(nP * 8);
  if (w && base) {
    char* p = (char*)base;
    w->U = (float2*)p;
    w->K = (float2*)(p + bU);
    w->partial = (double*)(p + bU + bK);
    w->kvs = nK1;
  }
  return bU + bK + bP;
}

}  // namespace me

using namespace me;

extern "C" {

long long me_sense_workspace_bytes(const me_sense* pb, int batch) {
  if (check_problem(pb) != ME_OK || batch < 1) return -1;
  batch = std::min(batch, pb->nshots);
  return ws_layout(pb, batch, 1, 0, nullptr, nullptr);
}

long long me_lm_ga_workspace_bytes(const me_sense* pb, int batch) {
  if (check_problem(pb) != ME_OK || batch < 1) return -1;
  batch = std::min(batch, pb->nshots);
  return ws_layout(pb, batch, 13, 0, nullptr, nullptr, 7);
}

long long me_lm_gradient_workspace_bytes(const me_sense* pb, int batch) {
  if (check_problem(pb) != ME_OK || batch < 1) return -1;
  batch = std::min(batch, pb->nshots);
  return ws_layout(pb, batch, 13, 0, nullptr, nullptr, 1, grad_partials(pb));
}

long long me_lm_workspace_bytes(const me_sense* pb, int batch) {
  if (check_problem(pb) != ME_OK || batch < 1) return -1;
  batch = std::min(batch, pb->nshots);
  return ws_layout(pb, batch, 12, 0, nullptr, nullptr, fast_sense_for(pb) ? 7 : 1);
}

int me_sense_precond(const me_c64* mps, int nx, int ny, int nz, int ncoils, float* P,
                     unsigned char* M, void* stream) {
  if (!mps || !P || !M) return fail("me_sense_precond: NULL pointer");
  const i64 plane = (i64)nx * ny;
  count_launch();
  precond_kernel<<<grid_1d(plane * nz), kThreads, 0, (cudaStream_t)stream>>>(
      (const float2*)mps, ncoils, plane, nz, P, M);
  return check_cuda(cudaGetLastError(), "precond launch");
}

int me_sense_gather(const me_sense* pb, const me_c64* ksp_h, me_c64* ydat, void* stream) {
  ME_TRY(check_problem(pb));
  if (!ksp_h || !ydat) return fail("me_sense_gather: NULL pointer");
  const i64 approx = (i64)pb->nshots * pb->samples.max_per_shot * pb->ncoils * pb->nz;
  count_launch();
  gather_kernel<<<grid_1d(approx), kThreads, 0, (cudaStream_t)stream>>>(
      (const float2*)ksp_h, pb->nx, pb->ny, pb->nz, pb->ncoils, pb->samples.shot_off,
      pb->samples.kx, pb->samples.ky, pb->nshots, (float2*)ydat);
  return check_cuda(cudaGetLastError(), "gather launch");
}

int me_sense_normal(const me_sense* pb, const me_c64* p, me_c64* out, int batch, void* work,
                    void* stream) {
  ME_TRY(check_problem(pb));
  if (!p || !out || !work) return fail("me_sense_normal: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 1, 0, &w, work);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, pb->transforms + 6 * (i64)s0, 6, st);
    ME_TRY(R.apply((const float2*)p, 0, w.U, vox, nb, false));
    ME_TRY(launch_fwd(pb, FWD_K, w.U, vox, s0, nb, w.K, nullptr, st));
    ME_TRY(launch_adj(pb, w.K, 1, w.U, vox, s0, nb, st));
    ME_TRY(R.adjoint(w.U, vox, w.U, vox, nb, false));
    count_launch();
    sum_volumes_kernel<<<grid_1d(vox), kThreads, 0, st>>>(w.U, vox, nb, pb->M, (float2*)out, vox,
                                                          s0 > 0);
    ME_TRY(check_cuda(cudaGetLastError(), "sum_volumes launch"));
  }
  return ME_OK;
}

int me_sense_rhs(const me_sense* pb, me_c64* b, int batch, void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!b || !work || !pb->ydat) return fail("me_sense_rhs: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 1, 0, &w, work);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, pb->transforms + 6 * (i64)s0, 6, st);
    ME_TRY(launch_adj(pb, (const float2*)pb->ydat, 0, w.U, vox, s0, nb, st));
    ME_TRY(R.adjoint(w.U, vox, w.U, vox, nb, false));
    count_launch();
    sum_volumes_kernel<<<grid_1d(vox), kThreads, 0, st>>>(w.U, vox, nb, pb->M, (float2*)b, vox,
                                                          s0 > 0);
    ME_TRY(check_cuda(cudaGetLastError(), "sum_volumes launch"));
  }
  return ME_OK;
}

int me_sense_residual(const me_sense* pb, const me_c64* x, me_c64* r, double* e, int batch,
                      void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !r || !work || !pb->ydat) return fail("me_sense_residual: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 1, 0, &w, work);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  const int zc = pb->nz * pb->ncoils;
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, pb->transforms + 6 * (i64)s0, 6, st);
    ME_TRY(R.apply((const float2*)x, 0, w.U, vox, nb, false));
    ME_TRY(launch_fwd(pb, FWD_K, w.U, vox, s0, nb, w.K, nullptr, st));
    // y - K at the shot's samples, in place, with the energy partials of each (z, coil)
    count_launch();
    resid_inplace_kernel<true><<<dim3(zc, nb), kThreads, 0, st>>>(
        w.K, (const float2*)pb->ydat, pb->samples.shot_off, s0, zc, w.partial);
    ME_TRY(check_cuda(cudaGetLastError(), "residual launch"));
    if (e) {
      count_launch();
      reduce_partials_kernel<<<nb, kThreads, 0, st>>>(w.partial, zc, 1, e, s0);
      ME_TRY(check_cuda(cudaGetLastError(), "reduce launch"));
    }
    ME_TRY(launch_adj(pb, w.K, 1, w.U, vox, s0, nb, st));
    ME_TRY(R.adjoint(w.U, vox, w.U, vox, nb, false));
    count_launch();
    sum_volumes_kernel<<<grid_1d(vox), kThreads, 0, st>>>(w.U, vox, nb, pb->M, (float2*)r, vox,
                                                          s0 > 0);
    ME_TRY(check_cuda(cudaGetLastError(), "sum_volumes launch"));
  }
  return ME_OK;
}

int me_sense_residual_norms(const me_sense* pb, const me_c64* x, const double* transforms,
                            double* e, int batch, void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !transforms || !e || !work || !pb->ydat)
    return fail("me_sense_residual_norms: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 1, 0, &w, work);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, transforms + 6 * (i64)s0, 6, st);
    ME_TRY(R.apply((const float2*)x, 0, w.U, vox, nb, false));
    ME_TRY(launch_fwd(pb, FWD_RESID, w.U, vox, s0, nb, nullptr, w.partial, st));
    count_launch();
    reduce_partials_kernel<<<nb, kThreads, 0, st>>>(w.partial, pb->nz * pb->ncoils, 1, e, s0);
    ME_TRY(check_cuda(cudaGetLastError(), "reduce launch"));
  }
  return ME_OK;
}

int me_sense_forward(const me_sense* pb, const me_c64* x, const double* transforms, me_c64* K,
                     int batch, void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !transforms || !K || !work) return fail("me_sense_forward: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 1, 0, &w, work);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, transforms + 6 * (i64)s0, 6, st);
    ME_TRY(R.apply((const float2*)x, 0, w.U, vox, nb, false));
    // K is written with offsets relative to shot_off[s0]; shift the base to the batch's block
    ME_TRY(launch_fwd_abs(pb, w.U, vox, s0, nb, (float2*)K, st));
  }
  return ME_OK;
}

int me_sense_forward_volumes(const me_sense* pb, const me_c64* vols, long long vol_stride,
                             int shot0, int nshots, me_c64* K, void* stream) {
  ME_TRY(check_problem(pb));
  if (!vols || !K) return fail("me_sense_forward_volumes: NULL pointer");
  if (shot0 < 0 || nshots < 1 || shot0 + nshots > pb->nshots)
    return fail("me_sense_forward_volumes: shot range outside the problem");
  if (vol_stride != 0 && vol_stride < vox_of(pb))
    return fail("me_sense_forward_volumes: volume stride must be 0 or at least one volume");
  return launch_fwd(pb, FWD_K, (const float2*)vols, vol_stride, shot0, nshots, (float2*)K,
                    nullptr, (cudaStream_t)stream);
}

int me_sense_adjoint_volumes(const me_sense* pb, const me_c64* K, int shot0, int nshots,
                             me_c64* vols, long long vol_stride, void* stream) {
  ME_TRY(check_problem(pb));
  if (!vols || !K) return fail("me_sense_adjoint_volumes: NULL pointer");
  if (shot0 < 0 || nshots < 1 || shot0 + nshots > pb->nshots)
    return fail("me_sense_adjoint_volumes: shot range outside the problem");
  if (vol_stride < vox_of(pb))
    return fail("me_sense_adjoint_volumes: volume stride must be at least one volume");
  return launch_adj(pb, (const float2*)K, 1, (float2*)vols, vol_stride, shot0, nshots,
                    (cudaStream_t)stream);
}

int me_sense_scatter(const me_sense* pb, const me_c64* K, me_c64* ksp_h, void* stream) {
  ME_TRY(check_problem(pb));
  if (!K || !ksp_h) return fail("me_sense_scatter: NULL pointer");
  const i64 per = (i64)pb->samples.max_per_shot * pb->ncoils * pb->nz;
  for (int s = 0; s < pb->nshots; s++) {
    count_launch();
    scatter_kernel<<<grid_1d(per), kThreads, 0, (cudaStream_t)stream>>>(
        (const float2*)K, pb->nx, pb->ny, pb->nz, pb->ncoils, pb->samples.shot_off,
        pb->samples.kx, pb->samples.ky, s, (float2*)ksp_h);
    ME_TRY(check_cuda(cudaGetLastError(), "scatter launch"));
  }
  return ME_OK;
}

int me_lm_normal_equations(const me_sense* pb, const me_c64* x, int jac_mode, double* stats,
                           int batch, void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !stats || !work || !pb->ydat) return fail("me_lm_normal_equations: NULL pointer");
  if (jac_mode != ME_JAC_REFERENCE && jac_mode != ME_JAC_EXACT) return fail("bad jacobian mode");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  const bool fast = fast_sense_for(pb);
  ws_layout(pb, batch, 12, 0, &w, work, fast ? 7 : 1);
  const i64 vox = vox_of(pb);
  const me_layout lay = zxy_layout(pb);
  float2* jwork = w.U + (i64)batch * 7 * vox;
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    {
      // T x and its six partials for the batch's shots at once: [shot][7] volumes in U, five
      // work volumes per shot after them
      Rigid R(pb->grid, lay, pb->transforms + 6 * (i64)s0, 6, st);
      ME_TRY(R.jacobian((const float2*)x, 0, w.U, vox, 7 * vox, nb, jac_mode, jwork, 5 * vox));
    }
    const int rcf = fast ? launch_fwd(pb, FWD_LM, w.U, vox, s0, nb, nullptr, w.partial, st, 0, 7)
                         : -1;
    if (rcf >= 0) {
      // fused: the statistics of the seven volumes contracted in registers
      ME_TRY(rcf);
    } else if (fast) {
      // the seven volumes of every shot through the one-volume forward kernel, then the sums
      ME_TRY(launch_fwd(pb, FWD_K, w.U, vox, s0, nb, w.K, nullptr, st, 0, 7, w.kvs));
      const int zc = pb->nz * pb->ncoils;
      count_launch();
      lm_stats_kernel<<<dim3(zc, nb), kThreads, 0, st>>>(w.K, w.kvs, (const float2*)pb->ydat,
                                                          pb->samples.shot_off, s0, zc, w.partial);
      ME_TRY(check_cuda(cudaGetLastError(), "lm stats launch"));
    } else {
      ME_TRY(launch_fwd(pb, FWD_LM, w.U, vox, s0, nb, nullptr, w.partial, st));
    }
    count_launch();
    reduce_partials_kernel<<<nb, kThreads, 0, st>>>(w.partial, pb->nz * pb->ncoils, kLmStats,
                                                     stats, s0);
    ME_TRY(check_cuda(cudaGetLastError(), "reduce launch"));
  }
  return ME_OK;
}

int me_lm_gradient(const me_sense* pb, const me_c64* x, int jac_mode, double* grad, int batch,
                   void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !grad || !work || !pb->ydat) return fail("me_lm_gradient: NULL pointer");
  if (jac_mode != ME_JAC_REFERENCE && jac_mode != ME_JAC_EXACT) return fail("bad jacobian mode");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 13, 0, &w, work, 1, grad_partials(pb));
  const i64 vox = vox_of(pb);
  const i64 bs = 8 * vox;  // per shot: T x, six partials, W = C^H F^H M_s r
  const me_layout lay = zxy_layout(pb);
  float2* jwork = w.U + (i64)batch * bs;
  const int zc = pb->nz * pb->ncoils;
  const int nblk = kGradBlocks;
  double* dpart = w.partial + (i64)batch * zc;  // after the energy partials of the batch
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    Rigid R(pb->grid, lay, pb->transforms + 6 * (i64)s0, 6, st);
    ME_TRY(R.jacobian((const float2*)x, 0, w.U, vox, bs, nb, jac_mode, jwork, 5 * vox));
    // r = M_s F C T x - y at the shot's samples, then W = C^H F^H M_s r in image space
    ME_TRY(launch_fwd(pb, FWD_K, w.U, bs, s0, nb, w.K, nullptr, st));
    count_launch();
    resid_inplace_kernel<false><<<dim3(zc, nb), kThreads, 0, st>>>(
        w.K, (const float2*)pb->ydat, pb->samples.shot_off, s0, zc, w.partial);
    ME_TRY(check_cuda(cudaGetLastError(), "residual launch"));
    ME_TRY(launch_adj(pb, w.K, 1, w.U + 7 * vox, bs, s0, nb, st));
    // g_p = Re<r, M_s F C dT/dp x> = Re<W, dT/dp x>
    count_launch();
    grad_dots_kernel<<<dim3(nblk, nb), kThreads, 0, st>>>(w.U, bs, vox, dpart);
    ME_TRY(check_cuda(cudaGetLastError(), "gradient dots launch"));
    count_launch();
    grad_finish_kernel<<<nb, 32, 0, st>>>(w.partial, zc, dpart, nblk, grad, s0);
    ME_TRY(check_cuda(cudaGetLastError(), "gradient finish launch"));
  }
  return ME_OK;
}

int me_lm_ga_rhs(const me_sense* pb, const me_c64* x, int jac_mode, int ga_mode,
                 const double* t_eps, const double* v, double eps, double* rhs, int batch,
                 void* work, void* stream) {
  ME_TRY(check_problem(pb));
  if (!x || !t_eps || !v || !rhs || !work || !pb->ydat) return fail("me_lm_ga_rhs: NULL pointer");
  if (jac_mode != ME_JAC_REFERENCE && jac_mode != ME_JAC_EXACT) return fail("bad jacobian mode");
  if (ga_mode != ME_GA_REFERENCE && ga_mode != ME_GA_INTENDED) return fail("bad GA mode");
  if (!(eps > 0.0)) return fail("me_lm_ga_rhs: eps must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  batch = std::max(1, std::min(batch, pb->nshots));
  Ws w;
  ws_layout(pb, batch, 13, 0, &w, work, 7);
  const i64 vox = vox_of(pb);
  const i64 bs = 8 * vox;  // per shot: T x, six partials, the direction D
  const me_layout lay = zxy_layout(pb);
  float2* jwork = w.U + (i64)batch * bs;
  const int zc = pb->nz * pb->ncoils;
  for (int s0 = 0; s0 < pb->nshots; s0 += batch) {
    const int nb = std::min(batch, pb->nshots - s0);
    const double* vb = v + 6 * (i64)s0;
    for (int pass = 0; pass < 2; pass++) {
      // partials at theta + eps v first, then at theta
      const double* prm = (pass == 0 ? t_eps : pb->transforms) + 6 * (i64)s0;
      Rigid R(pb->grid, lay, prm, 6, st);
      ME_TRY(R.jacobian((const float2*)x, 0, w.U, vox, bs, nb, jac_mode, jwork, 5 * vox));
      count_launch();
      ga_combine_kernel<<<grid_1d((i64)nb * vox), kThreads, 0, st>>>(w.U, bs, vox, nb, vb, ga_mode,
                                                                      pass == 0, eps);
      ME_TRY(check_cuda(cudaGetLastError(), "ga combine launch"));
    }
    // M_s F C of the six partials at theta and of D, one volume at a time per shot
    for (int k = 0; k < 7; k++)
      ME_TRY(launch_fwd(pb, FWD_K, w.U + (k < 6 ? 1 + k : 7) * vox, bs, s0, nb, w.K + k * w.kvs,
                        nullptr, st));
    count_launch();
    ga_dots_kernel<<<dim3(zc, nb), kThreads, 0, st>>>(w.K, w.kvs, pb->samples.shot_off, s0, zc,
                                                       w.partial);
    ME_TRY(check_cuda(cudaGetLastError(), "ga dots launch"));
    count_launch();
    reduce_partials_kernel<<<nb, kThreads, 0, st>>>(w.partial, zc, 6, rhs, s0);
    ME_TRY(check_cuda(cudaGetLastError(), "reduce launch"));
  }
  return ME_OK;
}

}  // extern "C"
