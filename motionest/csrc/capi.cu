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

}  // namespace me

using namespace me;

extern "C" {

const char* me_last_error(void) { return g_last_error.c_str(); }

int me_abi_version(void) { return ME_ABI_VERSION; }

long long me_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

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
