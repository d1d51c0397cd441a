// Error state, version and the plain per-axis FFT entry point.
#include <atomic>
#include <string>

#include "line_pass.cuh"
#include "rigid.cuh"

namespace me {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(const std::string& msg) {
  g_last_error = msg;
  return ME_ERR_INVALID;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return ME_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return ME_ERR_CUDA;
}

int sense_wait_fault(unsigned* out);
int line_pass_wait_fault(unsigned* out);
ME_WAIT_FAULT_ACCESSOR(capi_wait_fault)

// A barrier that one arrival short of its count never completes: every thread's bounded wait
// runs out after `limit` cycles and records WF_SELFTEST.  Nothing else is in flight.
__global__ void wait_selftest_kernel(long long limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 2);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive(&bar);
  mbar_wait_bounded(&bar, 0, WF_SELFTEST, limit);
}

}  // namespace me

using namespace me;

#define ME_CHECK_RC(x)            \
  do {                            \
    int _rc = (x);                \
    if (_rc != ME_OK) return _rc; \
  } while (0)

extern "C" {

const char* me_last_error(void) { return g_last_error.c_str(); }

int me_abi_version(void) { return ME_ABI_VERSION; }

long long me_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int me_wait_status(unsigned* status) {
  if (!status) return fail("me_wait_status: NULL pointer");
  unsigned a = 0, b = 0, c = 0;
  ME_CHECK_RC(sense_wait_fault(&a));
  ME_CHECK_RC(line_pass_wait_fault(&b));
  ME_CHECK_RC(capi_wait_fault(&c));
  *status = a | b | c;
  return ME_OK;
}

int me_wait_selftest(long long limit_cycles, void* stream) {
  if (limit_cycles < 1 || limit_cycles > kWaitCycles)
    return fail("me_wait_selftest: limit_cycles must be in [1, 2^31]");
  count_launch();
  wait_selftest_kernel<<<1, 64, 0, (cudaStream_t)stream>>>(limit_cycles);
  return check_cuda(cudaGetLastError(), "wait selftest launch");
}

int me_fft_axis(const me_c64* in, long long in_vs, me_c64* out, long long out_vs, int nvol,
                int nx, int ny, int nz, me_layout lay, int axis, int inverse, void* stream) {
  if (!in || !out) return fail("me_fft_axis: NULL pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("me_fft_axis: dims must be positive");
  me_grid g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  lay = normalize_layout(&g, lay);
  if (!layout_ok(&g, lay)) return fail("me_fft_axis: layout must be a dense permutation");
  if (nvol > 1 && out_vs == 0) return fail("me_fft_axis: nvol > 1 needs out_vol_stride");
  const int dims[3] = {nx, ny, nz};
  const i64 st[3] = {lay.sx, lay.sy, lay.sz};
  const Phase none = phase_none();
  return launch_line_pass(inverse ? PM_INV : PM_FWD, (const float2*)in, nullptr, (float2*)out,
                          nullptr, in_vs, out_vs, nvol, dims, st, axis, none, none, nullptr, 0, 0,
                          (cudaStream_t)stream);
}

}  // extern "C"
