// api_graph.cu -- CUDA graphs of RK steps, and ensembles of them.
//
// gf_rk_graph_create records the launches of gf_rk_advance (nsteps steps
// of one problem) by stream capture on a library-owned stream -- the
// legacy default stream cannot be captured -- and instantiates them;
// gf_graph_launch replays them on the problem's stream with one call.
// gf_graph_ensemble joins graphs of independent problems as child nodes
// without dependencies, so one launch advances every member and the GPU
// runs the members concurrently (config-5 style ensembles of small grids,
// each too small to fill the B200 by itself).  The graphs keep raw device
// pointers: the state, velocity and problem must outlive the graph.
#include "gf_common.cuh"
#include "rk_common.cuh"

struct gf_graph {
  gf_context *ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nodes = 0;  // kernel and copy nodes (top level or in child graphs)
};

namespace {
int count_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
  return (int)n;
}
}  // namespace

extern "C" int gf_rk_graph_create(gf_problem_t prob, int dtype, const gf_rk_traits *tr,
                                  void *const *u, const void *const *c, double dt, int nsteps,
                                  gf_graph_t *out) {
  if (!prob || !out) return GF_ERR_ARG;
  *out = nullptr;
  gf_context *ctx = prob->ctx;
  GF_REQUIRE(ctx, dtype == GF_F64 || dtype == GF_F32, "unknown dtype %d", dtype);
  GF_REQUIRE(ctx, nsteps >= 1, "nsteps must be >= 1");
  int rc = gfrk::check_traits(prob, tr, (const void *const *)u, c);
  if (rc) return rc;
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  // the stepper's work buffers are allocated before capture, so that no
  // allocation happens while the stream is being recorded
  bool ok = dtype == GF_F64 ? gfrk::Stepper<double>(prob, tr, c).alloc()
                            : gfrk::Stepper<float>(prob, tr, c).alloc();
  if (!ok) return gf_fail(ctx, GF_ERR_NOMEM, "RK work allocation failed");
  cudaStream_t cs = nullptr;
  GF_CUDA(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaStream_t saved = ctx->stream;
  ctx->stream = cs;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    rc = gf_rk_advance(prob, dtype, tr, u, c, 0.0, dt, nsteps);
    e = cudaStreamEndCapture(cs, &g);
  }
  ctx->stream = saved;
  cudaStreamDestroy(cs);
  if (rc != GF_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (rc != GF_OK) return rc;
    return gf_fail(ctx, GF_ERR_CUDA, "RK step capture failed: %s", cudaGetErrorString(e));
  }
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return gf_fail(ctx, GF_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  }
  gf_graph *gr = new gf_graph();
  gr->ctx = ctx;
  gr->graph = g;
  gr->exec = x;
  gr->nodes = count_nodes(g);
  *out = gr;
  return GF_OK;
}

extern "C" int gf_graph_ensemble(int n, const gf_graph_t *parts, gf_graph_t *out) {
  if (!parts || !out || n < 1) return GF_ERR_ARG;
  *out = nullptr;
  for (int i = 0; i < n; i++)
    if (!parts[i]) return GF_ERR_ARG;
  gf_context *ctx = parts[0]->ctx;
  for (int i = 1; i < n; i++)
    GF_REQUIRE(ctx, parts[i]->ctx->device == ctx->device, "ensemble members on different devices");
  GF_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaGraph_t g = nullptr;
  GF_CUDA(ctx, cudaGraphCreate(&g, 0));
  int nodes = 0;
  for (int i = 0; i < n; i++) {
    cudaGraphNode_t node;
    cudaError_t e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, parts[i]->graph);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return gf_fail(ctx, GF_ERR_CUDA, "ensemble member %d: %s", i, cudaGetErrorString(e));
    }
    nodes += parts[i]->nodes;
  }
  cudaGraphExec_t x = nullptr;
  cudaError_t e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return gf_fail(ctx, GF_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  }
  gf_graph *gr = new gf_graph();
  gr->ctx = ctx;
  gr->graph = g;
  gr->exec = x;
  gr->nodes = nodes;
  *out = gr;
  return GF_OK;
}

extern "C" int gf_graph_launch(gf_graph_t g) {
  if (!g) return GF_ERR_ARG;
  GF_CUDA(g->ctx, cudaGraphLaunch(g->exec, g->ctx->stream));
  return GF_OK;
}

extern "C" int gf_graph_nodes(gf_graph_t g) { return g ? g->nodes : GF_ERR_ARG; }

extern "C" int gf_graph_destroy(gf_graph_t g) {
  if (!g) return GF_ERR_ARG;
  cudaStreamSynchronize(g->ctx->stream);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return GF_OK;
}
