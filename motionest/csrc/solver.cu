// CG vector kernels with FP64 reductions (image_estimation.py:133-163) and the per-shot
// Levenberg-Marquardt solve / accept / mean-removal kernels (transform_estimation.py:60-150).
//
// Reductions are two-stage and deterministic: a grid of kRedBlocks blocks writes one partial
// per block into caller-provided scratch, then one block sums the partials in a fixed order.
// The CG scalars stay on the device, so a CG iteration needs no host round trip except the
// reference's stopping test.
#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"

namespace me {

#define ME_TRY_CUDA(call, what)                         \
  do {                                                  \
    const int _rc = check_cuda((call), (what));         \
    if (_rc != ME_OK) return _rc;                       \
  } while (0)

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 8;

__device__ __forceinline__ double block_sum(double a) {
  __shared__ double red[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRedThreads / 32; w++) t += red[w];
  return t;
}

__device__ __forceinline__ float block_max(float a) {
  __shared__ float red[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a = fmaxf(a, __shfl_down_sync(0xffffffffu, a, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  float t = 0.f;
  if (threadIdx.x == 0)
    for (int w = 0; w < kRedThreads / 32; w++) t = fmaxf(t, red[w]);
  return t;
}

#define GRID_LOOP(i, n) \
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < (n); i += (i64)gridDim.x * blockDim.x)

__global__ void final_sum_kernel(const double* __restrict__ part, int nparts, double* out) {
  double a = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) a += part[i];
  a = block_sum(a);
  if (threadIdx.x == 0) *out = a;
}

// CG update finaliser: scalars[2] = rz_new, scalars[3] = beta = rz_new / rz_old,
// scalars[0] = rz_new.
__global__ void final_update_kernel(const double* __restrict__ part, int nparts, double* s) {
  double a = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) a += part[i];
  a = block_sum(a);
  if (threadIdx.x == 0) {
    s[2] = a;
    s[3] = a / s[0];
    s[0] = a;
  }
}

__global__ void cg_init_kernel(const float2* __restrict__ b, const float2* __restrict__ Ap,
                               const float* __restrict__ P, float2* __restrict__ r,
                               float2* __restrict__ p, i64 n, double* part) {
  double acc = 0.0;
  GRID_LOOP(i, n) {
    const float2 ri = csub(b[i], Ap[i]);
    const float w = P[i];
    r[i] = ri;
    p[i] = cscale(ri, w);
    acc += (double)w * ((double)ri.x * ri.x + (double)ri.y * ri.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// cg_init_kernel with the residual given: r already holds b - A x (r is read, not written).
__global__ void cg_init_given_kernel(const float2* __restrict__ r, const float* __restrict__ P,
                                     float2* __restrict__ p, i64 n, double* part) {
  double acc = 0.0;
  GRID_LOOP(i, n) {
    const float2 ri = r[i];
    const float w = P[i];
    p[i] = cscale(ri, w);
    acc += (double)w * ((double)ri.x * ri.x + (double)ri.y * ri.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void dot_re_kernel(const float2* __restrict__ a, const float2* __restrict__ b, i64 n,
                              double* part) {
  double acc = 0.0;
  GRID_LOOP(i, n) {
    const float2 u = a[i], v = b[i];
    acc += (double)u.x * v.x + (double)u.y * v.y;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void cg_update_kernel(float2* __restrict__ x, float2* __restrict__ r,
                                 const float2* __restrict__ p, const float2* __restrict__ Ap,
                                 const float* __restrict__ P, const double* __restrict__ s, i64 n,
                                 double* part) {
  const float alpha = (float)(s[0] / s[1]);
  double acc = 0.0;
  GRID_LOOP(i, n) {
    const float2 pi = p[i], api = Ap[i];
    float2 xi = x[i], ri = r[i];
    xi.x += alpha * pi.x;
    xi.y += alpha * pi.y;
    ri.x -= alpha * api.x;
    ri.y -= alpha * api.y;
    x[i] = xi;
    r[i] = ri;
    acc += (double)P[i] * ((double)ri.x * ri.x + (double)ri.y * ri.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void cg_direction_kernel(float2* __restrict__ p, const float2* __restrict__ r,
                                    const float* __restrict__ P, const double* __restrict__ s,
                                    i64 n) {
  const float beta = (float)s[3];
  GRID_LOOP(i, n) {
    const float2 ri = r[i], pi = p[i];
    const float w = P[i];
    p[i] = make_float2(w * ri.x + beta * pi.x, w * ri.y + beta * pi.y);
  }
}

__global__ void max_abs_kernel(const float2* __restrict__ a, i64 n, float* part) {
  float m = 0.f;
  GRID_LOOP(i, n) {
    const float2 v = a[i];
    m = fmaxf(m, sqrtf(v.x * v.x + v.y * v.y));
  }
  m = block_max(m);
  if (threadIdx.x == 0) part[blockIdx.x] = m;
}

__global__ void final_max_kernel(const float* __restrict__ part, int nparts, float* out) {
  float m = 0.f;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) m = fmaxf(m, part[i]);
  m = block_max(m);
  if (threadIdx.x == 0) *out = m;
}

// ---------------------------------------------------------------- Levenberg-Marquardt
// stats[s] = {e0, g[6], H upper triangle (row-major, 21)}
__global__ void lm_propose_kernel(const double* __restrict__ stats, const double* __restrict__ damp,
                                  const double* __restrict__ t, double* __restrict__ t_next,
                                  int nshots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nshots) return;
  const double* st = stats + (i64)s * 28;
  double H[6][7];
  int k = 7;
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) {
      H[i][j] = st[k];
      H[j][i] = st[k];
      k++;
    }
  for (int i = 0; i < 6; i++) {
    H[i][i] += damp[s];
    H[i][6] = st[1 + i];
  }
  // Gaussian elimination with partial pivoting (the LAPACK gesv algorithm numpy.linalg.solve
  // calls) on the augmented 6x7 system.
  for (int c = 0; c < 6; c++) {
    int piv = c;
    double best = fabs(H[c][c]);
    for (int i = c + 1; i < 6; i++)
      if (fabs(H[i][c]) > best) {
        best = fabs(H[i][c]);
        piv = i;
      }
    if (piv != c)
      for (int j = 0; j < 7; j++) {
        const double tmp = H[c][j];
        H[c][j] = H[piv][j];
        H[piv][j] = tmp;
      }
    const double inv = 1.0 / H[c][c];
    for (int i = c + 1; i < 6; i++) {
      const double f = H[i][c] * inv;
      for (int j = c; j < 7; j++) H[i][j] -= f * H[c][j];
    }
  }
  double d[6];
  for (int i = 5; i >= 0; i--) {
    double a = H[i][6];
    for (int j = i + 1; j < 6; j++) a -= H[i][j] * d[j];
    d[i] = a / H[i][i];
  }
  for (int i = 0; i < 6; i++) t_next[(i64)s * 6 + i] = t[(i64)s * 6 + i] - d[i];
}

__global__ void lm_accept_kernel(const double* __restrict__ stats, const double* __restrict__ e1,
                                 double* __restrict__ t, const double* __restrict__ t_next,
                                 double* __restrict__ damp, unsigned char* __restrict__ flags,
                                 double tol, double* __restrict__ mean_out, int nshots) {
  for (int s = threadIdx.x; s < nshots; s += blockDim.x) {
    const double e0 = stats[(i64)s * 28];
    if (e1[s] < e0) {
      bool conv = true;
      for (int i = 0; i < 6; i++) conv = conv && fabs(t[s * 6 + i] - t_next[s * 6 + i]) < tol;
      if (conv && flags) flags[s] = 1;
      for (int i = 0; i < 6; i++) t[s * 6 + i] = t_next[s * 6 + i];
      damp[s] = fmax(damp[s] / 5.0, 1e-4);
    } else {
      damp[s] = fmin(damp[s] * 1.5, 1e16);
    }
  }
  __syncthreads();
  __shared__ double mean[6];
  if (threadIdx.x < 6) {
    double a = 0.0;
    for (int s = 0; s < nshots; s++) a += t[s * 6 + threadIdx.x];
    mean[threadIdx.x] = a / nshots;
    if (mean_out) mean_out[threadIdx.x] = mean[threadIdx.x];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nshots * 6; i += blockDim.x) t[i] -= mean[i % 6];
}

}  // namespace me

using namespace me;

extern "C" {

long long me_cg_workspace_bytes(long long n) { return (long long)kRedBlocks * 8 + 256; }

static int red_grid(i64 n) {
  return (int)std::max<i64>(1, std::min<i64>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads));
}

int me_cg_init(const me_c64* b, const me_c64* Ap, const float* P, me_c64* r, me_c64* p,
               double* scalars, long long n, void* work, void* stream) {
  if (!b || !P || !r || !p || !scalars || !work) return fail("me_cg_init: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int g = red_grid(n);
  if (!Ap && b != r) {
    ME_TRY_CUDA(cudaMemcpyAsync(r, b, (size_t)n * sizeof(me_c64), cudaMemcpyDeviceToDevice, st),
                "me_cg_init: copy of the given residual");
  }
  count_launch();
  if (Ap) {
    cg_init_kernel<<<g, kRedThreads, 0, st>>>((const float2*)b, (const float2*)Ap, P,
                                              (float2*)r, (float2*)p, n, (double*)work);
  } else {
    cg_init_given_kernel<<<g, kRedThreads, 0, st>>>((const float2*)r, P, (float2*)p, n,
                                                    (double*)work);
  }
  count_launch();
  final_sum_kernel<<<1, kRedThreads, 0, st>>>((const double*)work, g, scalars);
  return check_cuda(cudaGetLastError(), "cg_init launch");
}

int me_cg_pap(const me_c64* p, const me_c64* Ap, double* scalars, long long n, void* work,
              void* stream) {
  if (!p || !Ap || !scalars || !work) return fail("me_cg_pap: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int g = red_grid(n);
  count_launch();
  dot_re_kernel<<<g, kRedThreads, 0, st>>>((const float2*)p, (const float2*)Ap, n, (double*)work);
  count_launch();
  final_sum_kernel<<<1, kRedThreads, 0, st>>>((const double*)work, g, scalars + 1);
  return check_cuda(cudaGetLastError(), "cg_pap launch");
}

int me_cg_update(me_c64* x, me_c64* r, const me_c64* p, const me_c64* Ap, const float* P,
                 double* scalars, long long n, void* work, void* stream) {
  if (!x || !r || !p || !Ap || !P || !scalars || !work) return fail("me_cg_update: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int g = red_grid(n);
  count_launch();
  cg_update_kernel<<<g, kRedThreads, 0, st>>>((float2*)x, (float2*)r, (const float2*)p,
                                              (const float2*)Ap, P, scalars, n, (double*)work);
  count_launch();
  final_update_kernel<<<1, kRedThreads, 0, st>>>((const double*)work, g, scalars);
  return check_cuda(cudaGetLastError(), "cg_update launch");
}

int me_cg_direction(me_c64* p, const me_c64* r, const float* P, double* scalars, long long n,
                    void* stream) {
  if (!p || !r || !P || !scalars) return fail("me_cg_direction: NULL pointer");
  count_launch();
  cg_direction_kernel<<<red_grid(n), kRedThreads, 0, (cudaStream_t)stream>>>(
      (float2*)p, (const float2*)r, P, scalars, n);
  return check_cuda(cudaGetLastError(), "cg_direction launch");
}

int me_dot_re(const me_c64* a, const me_c64* b, double* out, long long n, void* work,
              void* stream) {
  if (!a || !b || !out || !work) return fail("me_dot_re: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int g = red_grid(n);
  count_launch();
  dot_re_kernel<<<g, kRedThreads, 0, st>>>((const float2*)a, (const float2*)b, n, (double*)work);
  count_launch();
  final_sum_kernel<<<1, kRedThreads, 0, st>>>((const double*)work, g, out);
  return check_cuda(cudaGetLastError(), "dot launch");
}

// ---------------------------------------------------------------------------------------
// Allocation-free FP64 inner product.  The partial sums live in this file-scope device array
// instead of caller-provided scratch: one partial per ME_NOALLOC_DOT_CHUNK elements, at most
// ME_NOALLOC_DOT_PARTIALS partials (32 KiB per device, held for the life of the process).
// In host code the array's name is only a stand-in for its device address; the address is
// looked up with cudaGetSymbolAddress once per device, with that device current.
static __device__ __align__(256) double g_noalloc_dot_partials[ME_NOALLOC_DOT_PARTIALS];

static std::mutex g_noalloc_mutex;
static double* g_noalloc_ptr[64] = {nullptr};

static int noalloc_partials(double** out) {
  int dev = 0;
  ME_TRY_CUDA(cudaGetDevice(&dev), "me_dot_re_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail("me_dot_re_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    ME_TRY_CUDA(cudaGetSymbolAddress(&p, g_noalloc_dot_partials),
                "me_dot_re_noalloc: cudaGetSymbolAddress");
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return ME_OK;
}

int me_dot_re_noalloc(const me_c64* a, const me_c64* b, double* out, long long n, void* stream) {
  if (!a || !b || !out) return fail("me_dot_re_noalloc: NULL pointer");
  if (n < 0) return fail("me_dot_re_noalloc: negative length");
  if (n > ME_NOALLOC_DOT_MAX_N)
    return fail("me_dot_re_noalloc: n exceeds ME_NOALLOC_DOT_MAX_N (the static scratch holds " +
                std::to_string(ME_NOALLOC_DOT_PARTIALS) + " partial sums of " +
                std::to_string(ME_NOALLOC_DOT_CHUNK) + " elements); use me_dot_re");
  double* part = nullptr;
  const int rc = noalloc_partials(&part);
  if (rc != ME_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // every block writes its own partial, so nothing in the shared array needs clearing
  const int g = (int)std::max<long long>(1, (n + ME_NOALLOC_DOT_CHUNK - 1) / ME_NOALLOC_DOT_CHUNK);
  count_launch();
  dot_re_kernel<<<g, kRedThreads, 0, st>>>((const float2*)a, (const float2*)b, n, part);
  count_launch();
  final_sum_kernel<<<1, kRedThreads, 0, st>>>(part, g, out);
  return check_cuda(cudaGetLastError(), "me_dot_re_noalloc launch");
}

int me_max_abs(const me_c64* a, long long n, float* out, void* work, void* stream) {
  if (!a || !out || !work) return fail("me_max_abs: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const int g = red_grid(n);
  count_launch();
  max_abs_kernel<<<g, kRedThreads, 0, st>>>((const float2*)a, n, (float*)work);
  count_launch();
  final_max_kernel<<<1, kRedThreads, 0, st>>>((const float*)work, g, out);
  return check_cuda(cudaGetLastError(), "max_abs launch");
}

int me_lm_propose(const double* stats, const double* damp, const double* t, double* t_next,
                  int nshots, void* stream) {
  if (!stats || !damp || !t || !t_next) return fail("me_lm_propose: NULL pointer");
  if (nshots < 1) return ME_OK;
  count_launch();
  lm_propose_kernel<<<(nshots + 63) / 64, 64, 0, (cudaStream_t)stream>>>(stats, damp, t, t_next,
                                                                        nshots);
  return check_cuda(cudaGetLastError(), "lm_propose launch");
}

int me_lm_accept(const double* stats, const double* e1, double* t, const double* t_next,
                 double* damp, unsigned char* flags, double tol, double* mean_out, int nshots,
                 void* stream) {
  if (!stats || !e1 || !t || !t_next || !damp) return fail("me_lm_accept: NULL pointer");
  if (nshots < 1) return ME_OK;
  count_launch();
  lm_accept_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(stats, e1, t, t_next, damp, flags, tol,
                                                       mean_out, nshots);
  return check_cuda(cudaGetLastError(), "lm_accept launch");
}

}  // extern "C"
