// CG-SENSE as one CUDA graph (image_estimation.py:89-165): the right-hand side, A x, the CG
// initialisation and then up to max_iter CG iterations with the reference's stopping test
// sqrt|<r, z>| < tol (:156), all in a single graph launch.  Without b the graph starts from the
// initial residual the caller computed into r (me_sense_residual).
//
// The loop is a conditional WHILE node.  Its body is one CG iteration captured from the same
// C-ABI calls the host loop makes (normal operator, <p, Ap>, the x / r update, the new
// direction); a one-thread kernel in the body evaluates the stopping test and the iteration cap
// on the device and sets the node's condition, so no host round trip happens between
// iterations.  The loop always ends: the cap is checked on every pass, whatever the residual
// (a NaN residual fails the tolerance test and stops at the cap).
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"

namespace me {

__global__ void cg_graph_begin_kernel(int* iters) { *iters = 0; }

__global__ void cg_graph_decide_kernel(const double* __restrict__ s, int* iters, int max_iter,
                                       double tol, cudaGraphConditionalHandle h) {
  const int it = *iters + 1;
  *iters = it;
  const bool converged = sqrt(fabs(s[2])) < tol;
  cudaGraphSetConditional(h, (converged || it >= max_iter) ? 0u : 1u);
}

}  // namespace me

using namespace me;

struct me_cg_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long prologue_launches = 0;
  long long body_launches = 0;
};

extern "C" {

int me_cg_graph_create(const me_sense* pb, me_c64* x, me_c64* b, me_c64* r, me_c64* p,
                       me_c64* Ap, double* scalars, int* iters, int max_iter, double tol,
                       int batch, void* work, void* cg_work, void* stream, me_cg_graph** out) {
  if (!pb || !x || !r || !p || !Ap || !scalars || !iters || !work || !cg_work || !out)
    return fail("me_cg_graph_create: NULL pointer");
  if (max_iter < 0) return fail("me_cg_graph_create: max_iter must be >= 0");
  cudaStream_t st = (cudaStream_t)stream;
  if (st == nullptr) return fail("me_cg_graph_create: needs a created stream (not the legacy default)");
  const long long n = (long long)pb->nx * pb->ny * pb->nz;
  // load the two loop kernels now: a module's first use must not fall inside the capture
  cudaFuncAttributes fa;
  int rc0 = check_cuda(cudaFuncGetAttributes(&fa, cg_graph_begin_kernel), "cg kernel load");
  if (rc0 == ME_OK) rc0 = check_cuda(cudaFuncGetAttributes(&fa, cg_graph_decide_kernel), "cg kernel load");
  if (rc0 != ME_OK) return rc0;
  me_cg_graph* g = new me_cg_graph();
  auto bail = [&](int rc) {
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st, &junk);
      if (junk) cudaGraphDestroy(junk);
    }
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return rc;
  };
  int rc = check_cuda(cudaGraphCreate(&g->graph, 0), "cudaGraphCreate");
  if (rc != ME_OK) return bail(rc);
  cudaGraphConditionalHandle h;
  rc = check_cuda(cudaGraphConditionalHandleCreate(&h, g->graph, max_iter > 0 ? 1u : 0u,
                                                   cudaGraphCondAssignDefault),
                  "cudaGraphConditionalHandleCreate");
  if (rc != ME_OK) return bail(rc);

  // prologue: b, A x, r = b - A x (or, with b == NULL, r as the caller left it), p = z = P r,
  // <r, z>, iteration counter
  rc = check_cuda(cudaStreamBeginCaptureToGraph(st, g->graph, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal),
                  "cudaStreamBeginCaptureToGraph");
  if (rc != ME_OK) return bail(rc);
  const long long c0 = me_launch_count();
  if (b) {
    if ((rc = me_sense_rhs(pb, b, batch, work, stream)) != ME_OK) return bail(rc);
    if ((rc = me_sense_normal(pb, x, Ap, batch, work, stream)) != ME_OK) return bail(rc);
    if ((rc = me_cg_init(b, Ap, pb->P, r, p, scalars, n, cg_work, stream)) != ME_OK)
      return bail(rc);
  } else if ((rc = me_cg_init(r, nullptr, pb->P, r, p, scalars, n, cg_work, stream)) != ME_OK) {
    return bail(rc);
  }
  count_launch();
  cg_graph_begin_kernel<<<1, 1, 0, st>>>(iters);
  if ((rc = check_cuda(cudaGetLastError(), "cg begin launch")) != ME_OK) return bail(rc);
  g->prologue_launches = me_launch_count() - c0;

  // the WHILE node after the prologue
  cudaStreamCaptureStatus cs;
  cudaGraph_t cap = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  rc = check_cuda(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cap, &deps, &ndeps),
                  "cudaStreamGetCaptureInfo");
  if (rc != ME_OK) return bail(rc);
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cond;
  rc = check_cuda(cudaGraphAddNode(&cond, cap, deps, ndeps, &cp), "cudaGraphAddNode (while)");
  if (rc != ME_OK) return bail(rc);
  rc = check_cuda(cudaStreamUpdateCaptureDependencies(st, &cond, 1,
                                                      cudaStreamSetCaptureDependencies),
                  "cudaStreamUpdateCaptureDependencies");
  if (rc != ME_OK) return bail(rc);
  cudaGraph_t whole = nullptr;
  rc = check_cuda(cudaStreamEndCapture(st, &whole), "cudaStreamEndCapture");
  if (rc != ME_OK) return bail(rc);

  // body: one CG iteration (image_estimation.py:141-163)
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  rc = check_cuda(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                                cudaStreamCaptureModeThreadLocal),
                  "cudaStreamBeginCaptureToGraph (body)");
  if (rc != ME_OK) return bail(rc);
  const long long c1 = me_launch_count();
  if ((rc = me_sense_normal(pb, p, Ap, batch, work, stream)) != ME_OK) return bail(rc);
  if ((rc = me_cg_pap(p, Ap, scalars, n, cg_work, stream)) != ME_OK) return bail(rc);
  if ((rc = me_cg_update(x, r, p, Ap, pb->P, scalars, n, cg_work, stream)) != ME_OK)
    return bail(rc);
  count_launch();
  cg_graph_decide_kernel<<<1, 1, 0, st>>>(scalars, iters, max_iter, tol, h);
  if ((rc = check_cuda(cudaGetLastError(), "cg decide launch")) != ME_OK) return bail(rc);
  if ((rc = me_cg_direction(p, r, pb->P, scalars, n, stream)) != ME_OK) return bail(rc);
  g->body_launches = me_launch_count() - c1;
  rc = check_cuda(cudaStreamEndCapture(st, &body), "cudaStreamEndCapture (body)");
  if (rc != ME_OK) return bail(rc);

  // the captured calls counted their kernels; they run only when the graph is launched
  count_launches(-(g->prologue_launches + g->body_launches));
  rc = check_cuda(cudaGraphInstantiate(&g->exec, g->graph, 0), "cudaGraphInstantiate");
  if (rc != ME_OK) return bail(rc);
  *out = g;
  return ME_OK;
}

int me_cg_graph_launch(me_cg_graph* g, void* stream) {
  if (!g || !g->exec) return fail("me_cg_graph_launch: no graph");
  count_launches(g->prologue_launches);
  return check_cuda(cudaGraphLaunch(g->exec, (cudaStream_t)stream), "cudaGraphLaunch");
}

long long me_cg_graph_body_launches(const me_cg_graph* g) { return g ? g->body_launches : -1; }

void me_cg_graph_account(const me_cg_graph* g, int iterations) {
  if (!g) return;
  count_launches(g->body_launches * (long long)iterations);
}

int me_cg_graph_destroy(me_cg_graph* g) {
  if (!g) return ME_OK;
  int rc = ME_OK;
  if (g->exec) rc = check_cuda(cudaGraphExecDestroy(g->exec), "cudaGraphExecDestroy");
  if (g->graph) {
    const int rc2 = check_cuda(cudaGraphDestroy(g->graph), "cudaGraphDestroy");
    if (rc == ME_OK) rc = rc2;
  }
  delete g;
  return rc;
}

}  // extern "C"
