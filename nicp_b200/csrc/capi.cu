// capi.cu -- the C ABI of include/nicp_gpu.h: contexts, device clouds, the
// workspace, frame and pair batching, CUDA-graph capture of the Gauss-Newton
// loop, and the host side of Aligner::align.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "abi_guard.hpp"
#include "common.cuh"
#include "host_math.hpp"
#include "kernels.hpp"
#include "nicp_gpu.h"

using namespace nicp;

namespace {

struct GraphEntry {
  std::string key;
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels = 0;
  std::vector<Profiler::Rec> recs;
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Offsets into one device allocation, assigned in two passes (size, then place).
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    off = align_up(off, 256);
    size_t r = off;
    off += bytes;
    return r;
  }
};

}  // namespace

struct nicp_ctx {
  int device = 0;
  int sm_count = 148;
  int sweep_ctas_per_sm[3] = {0, 0, 0};  // per moment precision, queried on first use
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  Profiler prof;
  char *ws = nullptr;
  size_t ws_cap = 0;
  char *pin_up = nullptr;
  size_t pin_up_cap = 0;
  cudaEvent_t pin_up_ev = nullptr;
  cudaStream_t copy_stream = nullptr;   // depth staging copies, overlapped with the build kernels
  std::vector<cudaEvent_t> copy_ev;     // one per build chunk: its frames are staged
  cudaEvent_t copy_start = nullptr;     // the compute stream's tail when staging begins
  char *pin_down = nullptr;
  size_t pin_down_cap = 0;
  size_t cloud_bytes = 0;
  std::vector<GraphEntry> graphs;
  nicp_cloud *scratch_cloud = nullptr;
  unsigned long long h2d_bytes = 0, d2h_bytes = 0;  // host<->device traffic issued by the library
  // launch shapes of the alignment loop; the autotuner picks them per
  // resolution mix (results do not depend on them)
  struct Launch {
    int zb_ppt = kZbufDefaultPPT;  // z-buffer points per thread
    int corr_ctas = 0;             // fused kernel CTAs per SM (0: as many as fit)
  };
  Launch launch;
  bool autotune = false;
  std::map<std::string, Launch> tuned;
  // k_stats launch shape per frame-size mix of a build chunk (autotuned),
  // and the shape of the last build
  std::map<std::string, int> stats_tuned;
  int stats_shape = 0;
  std::map<std::string, std::vector<float>> tune_ms;  // trial times per resolution mix
};

struct nicp_cloud {
  nicp_ctx *ctx = nullptr;
  char *mem = nullptr;
  size_t bytes = 0;
  int capacity = 0;  // points
  int rows = 0, cols = 0;
  bool has_eig = false, has_gauss = false;      // storage reserved
  bool eig_valid = false, gauss_valid = false;  // written by the last build
  // information matrices Omega = d1 I + (d0 - d1) n n^T with (d0, d1) per
  // class in omd (point flat / non-flat, normal flat / non-flat): true for
  // clouds built with such parameters, false for uploaded ones
  bool omega_structured = false;
  float omd[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // false while Omega is implicit: a structured cloud built without Stats
  // (the stats kernel leaves omg unwritten; the fused kernel rebuilds Omega
  // from the normal, the class code and omd).  cloud_ensure_omg writes the
  // matrices out for a reader that needs them.
  mutable bool omg_valid = true;
  float4 *pts = nullptr, *nrm = nullptr, *omg = nullptr;
  float *eig = nullptr;
  float4 *gauss = nullptr;  // 3 float4 per point: mean, then the 9 covariance entries row-major
  int *count = nullptr;
  int32_t *index = nullptr;
};

// ------------------------------------------------------------------ helpers
static int fail(nicp_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}

// Every call on a context runs on the context's device, whatever device the
// calling thread has current, and gives the thread its previous device back
// on return: workspaces, clouds and kernels of a context never land on
// another GPU, and a thread that drives contexts on several GPUs needs no
// cudaSetDevice of its own.
class DeviceScope {
 public:
  explicit DeviceScope(const nicp_ctx *ctx) {
    if (!ctx) return;
    if (cudaGetDevice(&prev_) != cudaSuccess) {
      cudaGetLastError();
      prev_ = -1;
    }
    if (prev_ != ctx->device) {
      ok_ = cudaSetDevice(ctx->device) == cudaSuccess;
      if (!ok_) cudaGetLastError();
      switched_ = ok_ && prev_ >= 0;
    }
  }
  ~DeviceScope() {
    if (switched_) cudaSetDevice(prev_);
  }
  DeviceScope(const DeviceScope &) = delete;
  DeviceScope &operator=(const DeviceScope &) = delete;
  bool ok() const { return ok_; }

 private:
  int prev_ = -1;
  bool switched_ = false, ok_ = true;
};

#define NICP_ON_DEVICE(ctx_expr)             \
  DeviceScope device_scope_(ctx_expr);        \
  if (!device_scope_.ok()) return NICP_ECUDA

#define CK(ctx, call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail((ctx), NICP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Writes out a cloud's implicit information matrices (see omg_valid), on the
// stream of the context whose kernels will read them.
static int cloud_ensure_omg(nicp_ctx *ctx, const nicp_cloud *c) {
  if (!c || c->omg_valid) return NICP_OK;
  launch_materialize_omg(c->pts, c->nrm, c->omg, c->count, c->capacity, c->omd, ctx->stream);
  CK(ctx, cudaGetLastError());
  c->omg_valid = true;
  return NICP_OK;
}

static int ensure_ws(nicp_ctx *ctx, size_t bytes) {
  if (bytes <= ctx->ws_cap) return NICP_OK;
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto &g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
  if (ctx->ws) cudaFree(ctx->ws);
  ctx->ws = nullptr;
  ctx->ws_cap = 0;
  size_t cap = align_up(bytes + bytes / 4, 1 << 20);
  if (cudaMalloc(&ctx->ws, cap) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, NICP_ENOMEM, "workspace allocation of " + std::to_string(cap) + " bytes failed");
  }
  ctx->ws_cap = cap;
  return NICP_OK;
}

// Pinned upload staging: waits until the previous upload has been consumed.
static int pin_up(nicp_ctx *ctx, size_t bytes, char **out) {
  CK(ctx, cudaEventSynchronize(ctx->pin_up_ev));
  if (bytes > ctx->pin_up_cap) {
    if (ctx->pin_up) cudaFreeHost(ctx->pin_up);
    ctx->pin_up = nullptr;
    size_t cap = align_up(bytes + bytes / 4, 1 << 16);
    CK(ctx, cudaMallocHost(&ctx->pin_up, cap));
    ctx->pin_up_cap = cap;
  }
  *out = ctx->pin_up;
  return NICP_OK;
}

static int pin_down(nicp_ctx *ctx, size_t bytes, char **out) {
  if (bytes > ctx->pin_down_cap) {
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->pin_down) cudaFreeHost(ctx->pin_down);
    ctx->pin_down = nullptr;
    size_t cap = align_up(bytes + bytes / 4, 1 << 16);
    CK(ctx, cudaMallocHost(&ctx->pin_down, cap));
    ctx->pin_down_cap = cap;
  }
  *out = ctx->pin_down;
  return NICP_OK;
}

static int cloud_reserve(nicp_cloud *c, int capacity, int rows, int cols, bool eig, bool gauss = false) {
  nicp_ctx *ctx = c->ctx;
  size_t P = (size_t)rows * cols;
  if (capacity < 1) capacity = 1;
  if (capacity <= c->capacity && P <= (size_t)c->rows * c->cols && (!eig || c->has_eig) && (!gauss || c->has_gauss)) {
    c->rows = rows;
    c->cols = cols;
    return NICP_OK;
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  if (c->mem) {
    cudaFree(c->mem);
    ctx->cloud_bytes -= c->bytes;
  }
  c->mem = nullptr;
  Layout L;
  size_t o_pts = L.take(16 * (size_t)capacity), o_nrm = L.take(16 * (size_t)capacity);
  size_t o_omg = L.take(48 * (size_t)capacity);
  size_t o_eig = eig ? L.take(4 * kStatsWords * (size_t)capacity) : 0;
  size_t o_gauss = gauss ? L.take(48 * (size_t)capacity) : 0;
  size_t o_cnt = L.take(2 * sizeof(int));  // points, points with a normal
  size_t o_idx = L.take(4 * std::max<size_t>(P, 1));
  if (cudaMalloc(&c->mem, L.off) != cudaSuccess) {
    cudaGetLastError();
    c->capacity = 0;
    return fail(ctx, NICP_ENOMEM, "cloud allocation failed");
  }
  c->bytes = L.off;
  ctx->cloud_bytes += c->bytes;
  c->capacity = capacity;
  c->rows = rows;
  c->cols = cols;
  c->has_eig = eig;
  c->has_gauss = gauss;
  c->eig_valid = c->gauss_valid = false;
  c->pts = (float4 *)(c->mem + o_pts);
  c->nrm = (float4 *)(c->mem + o_nrm);
  c->omg = (float4 *)(c->mem + o_omg);
  c->eig = eig ? (float *)(c->mem + o_eig) : nullptr;
  c->gauss = gauss ? (float4 *)(c->mem + o_gauss) : nullptr;
  c->count = (int *)(c->mem + o_cnt);
  c->index = (int32_t *)(c->mem + o_idx);
  CK(ctx, cudaMemsetAsync(c->count, 0, 2 * sizeof(int), ctx->stream));
  return NICP_OK;
}

static bool valid_camera(const nicp_camera *c) {
  return c && c->rows > 0 && c->cols > 0 && c->scaling > 0 && std::isfinite(c->fx) && std::isfinite(c->fy) &&
         cam_rows(*c) > 0 && cam_cols(*c) > 0;
}

static CorrParams corr_params(const nicp_corr_params &p) {
  CorrParams c;
  c.sq_thr = p.inlier_distance_threshold * p.inlier_distance_threshold;
  c.cos_thr = p.inlier_normal_angular_threshold;
  c.flat_thr = p.flat_curvature_threshold;
  c.min_ratio = 1.0f / p.inlier_curvature_ratio_threshold;
  c.max_ratio = p.inlier_curvature_ratio_threshold;
  c.demoted = p.demoted_to_gicp;
  c.row_limit_threads = std::max(1, p.parity_threads);
  c.row_search = std::max(0, p.row_search_region);
  c.col_search = std::max(0, p.col_search_region);
  return c;
}

static LinParams lin_params(const nicp_lin_params &p) {
  LinParams l;
  l.max_chi2 = p.inlier_max_chi2;
  l.robust = p.robust_kernel;
  l.z_scaling = p.z_scaling;
  l.scale = p.scale;
  l.demoted = p.demoted_to_gicp;
  return l;
}

static void rows12(const HM4 &M, float *o) {
  for (int i = 0; i < 12; i++) o[i] = M.a[i];
}

// ------------------------------------------------------------------ defaults
extern "C" void nicp_default_camera(nicp_camera *c) {
  // PinholePointProjector() and PointProjector() constructors
  c->fx = 1.0f; c->fy = 1.0f; c->cx = 0.5f; c->cy = 0.5f;
  c->scaling = 1.0f;
  c->rows = 0; c->cols = 0;
  c->min_distance = 0.01f; c->max_distance = 6.0f;
  c->baseline = 0.075f; c->alpha = 0.1f;
}

extern "C" void nicp_default_cloud_params(nicp_cloud_params *p) {
  p->depth_scale = 0.001f;
  p->world_radius = 0.1f;
  p->min_image_radius = 10; p->max_image_radius = 30; p->min_points = 50;
  p->curvature_threshold = 0.02f;
  const float pf[3] = {1000.0f, 0.001f, 0.001f}, pn[3] = {1.0f, 0.1f, 0.1f};
  const float nf[3] = {1000.0f, 0.001f, 0.001f}, nn[3] = {0.1f, 1.0f, 1.0f};
  for (int i = 0; i < 3; i++) {
    p->pim_flat[i] = pf[i]; p->pim_nonflat[i] = pn[i];
    p->nim_flat[i] = nf[i]; p->nim_nonflat[i] = nn[i];
  }
  p->pim_curvature_threshold = 0.02f;
  p->nim_curvature_threshold = 0.02f;
  p->moments_precision = NICP_MOMENTS_F64;
  p->keep_gaussians = 0;
  p->keep_stats = 0;
}

extern "C" void nicp_default_corr_params(nicp_corr_params *p) {
  p->inlier_distance_threshold = 1.0f;
  p->inlier_normal_angular_threshold = cosf((float)(M_PI / 6));
  p->flat_curvature_threshold = 0.2f;
  p->inlier_curvature_ratio_threshold = 1.3f;
  p->demoted_to_gicp = 0;
  p->parity_threads = 1;
  p->row_search_region = p->col_search_region = 0;
}

extern "C" void nicp_default_lin_params(nicp_lin_params *p) {
  p->inlier_max_chi2 = 9e3f;
  p->robust_kernel = 1;
  p->z_scaling = 0;
  p->scale = 1.0f;
  p->demoted_to_gicp = 0;
  p->cross_block_f32 = 0;
}

extern "C" void nicp_default_align_params(nicp_align_params *p) {
  p->outer_iterations = 10;
  p->inner_iterations = 1;
  p->lambda = 1e3f;
  p->min_inliers = 100;
  p->translational_min_eigen_ratio = 50.0f;
  p->rotational_min_eigen_ratio = 50.0f;
  p->compute_statistics = 1;
  p->early_exit_eps = 0.0;
}

// ------------------------------------------------------------------ context
extern "C" int nicp_ctx_create(int device, void *stream, nicp_ctx **out) {
  NICP_ABI_TRY
  if (!out) return NICP_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return NICP_ECUDA;
  }
  if (device < 0 || device >= n) return NICP_EINVAL;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) return NICP_ECUDA;
  auto *ctx = new nicp_ctx();
  ctx->device = device;
  // the stream and event belong to `device`; the caller's device is current again on return
  DeviceScope on_device(ctx);
  if (!on_device.ok()) {
    delete ctx;
    return NICP_ECUDA;
  }
  ctx->sm_count = prop.multiProcessorCount > 0 ? prop.multiProcessorCount : 148;
  if (stream) {
    ctx->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return NICP_ECUDA;
    }
    ctx->own_stream = true;
  }
  if (cudaEventCreateWithFlags(&ctx->pin_up_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return NICP_ECUDA;
  }
  *out = ctx;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_ctx_destroy(nicp_ctx *ctx) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);  // staging copies write into ws
  if (ctx->scratch_cloud) nicp_cloud_destroy(ctx->scratch_cloud);
  for (auto &g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->pin_up) cudaFreeHost(ctx->pin_up);
  if (ctx->pin_down) cudaFreeHost(ctx->pin_down);
  cudaEventDestroy(ctx->pin_up_ev);
  for (cudaEvent_t e : ctx->copy_ev) cudaEventDestroy(e);
  if (ctx->copy_start) cudaEventDestroy(ctx->copy_start);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" const char *nicp_ctx_last_error(const nicp_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" int nicp_ctx_synchronize(nicp_ctx *ctx) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" void *nicp_ctx_stream(nicp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" size_t nicp_ctx_device_bytes(const nicp_ctx *ctx) { return ctx ? ctx->ws_cap + ctx->cloud_bytes : 0; }

extern "C" int nicp_ctx_set_profiling(nicp_ctx *ctx, int enable) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  ctx->prof.enabled = enable != 0;
  ctx->prof.recs.clear();
  ctx->prof.next = 0;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_ctx_set_autotune(nicp_ctx *ctx, int enable) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  ctx->autotune = enable != 0;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_ctx_launch_shape(const nicp_ctx *ctx, int *zbuffer_points_per_thread, int *corr_ctas_per_sm,
                                     int *tuned_mixes, int *stats_threads, int *stats_ctas_per_sm) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  if (zbuffer_points_per_thread) *zbuffer_points_per_thread = ctx->launch.zb_ppt;
  if (stats_threads) *stats_threads = stats_shape_threads(ctx->stats_shape);
  if (stats_ctas_per_sm) *stats_ctas_per_sm = stats_shape_min_ctas(ctx->stats_shape);
  if (corr_ctas_per_sm) *corr_ctas_per_sm = ctx->launch.corr_ctas;
  if (tuned_mixes) *tuned_mixes = (int)ctx->tuned.size();
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_ctx_read_profile(nicp_ctx *ctx, int kernel, double *total_ms, int *launches) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || kernel < 0 || kernel >= NICP_K_COUNT) return NICP_EINVAL;
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  double t = 0;
  int n = 0;
  std::vector<Profiler::Rec> keep;
  for (auto &r : ctx->prof.recs) {
    if (r.kernel != kernel) {
      keep.push_back(r);
      continue;
    }
    float ms = 0;
    CK(ctx, cudaEventElapsedTime(&ms, r.a, r.b));
    t += ms;
    n += r.nkernels;
  }
  ctx->prof.recs.swap(keep);
  if (ctx->prof.recs.empty()) ctx->prof.next = 0;
  if (total_ms) *total_ms = t;
  if (launches) *launches = n;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" unsigned long long nicp_ctx_kernel_launches(const nicp_ctx *ctx) { return ctx ? ctx->prof.launches : 0; }

extern "C" int nicp_ctx_transfer_bytes(const nicp_ctx *ctx, unsigned long long *h2d, unsigned long long *d2h) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx) return NICP_EINVAL;
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" const char *nicp_kernel_name(int k) {
  static const char *names[NICP_K_COUNT] = {"unproject", "moments_bands", "moments_sweep", "stats_omega",
                                            "zbuffer",   "resolve",      "corr_lin",     "corr_list",
                                            "lin_list",  "solve",        "transform"};
  return (k >= 0 && k < NICP_K_COUNT) ? names[k] : "?";
}

// ------------------------------------------------------------------ clouds
extern "C" int nicp_cloud_create(nicp_ctx *ctx, nicp_cloud **out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !out) return NICP_EINVAL;
  auto *c = new nicp_cloud();
  c->ctx = ctx;
  *out = c;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_destroy(nicp_cloud *c) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c) return NICP_EINVAL;
  if (c->mem) {
    cudaStreamSynchronize(c->ctx->stream);
    cudaFree(c->mem);
    c->ctx->cloud_bytes -= c->bytes;
  }
  delete c;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_size(nicp_cloud *c, int *n) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c || !n) return NICP_EINVAL;
  if (!c->mem) { *n = 0; return NICP_OK; }
  nicp_ctx *ctx = c->ctx;
  CK(ctx, cudaMemcpyAsync(n, c->count, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_normal_count(nicp_cloud *c, int *n) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c || !n) return NICP_EINVAL;
  if (!c->mem) { *n = 0; return NICP_OK; }
  nicp_ctx *ctx = c->ctx;
  CK(ctx, cudaMemcpyAsync(n, c->count + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_download(nicp_cloud *c, float *p4, float *n4, float *curv, float *op9, float *on9, float *ev3,
                                   float *U9) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c) return NICP_EINVAL;
  nicp_ctx *ctx = c->ctx;
  int n = 0;
  int rc = nicp_cloud_size(c, &n);
  if (rc) return rc;
  if (n == 0) return NICP_OK;
  if ((ev3 || U9) && !c->eig_valid) return fail(ctx, NICP_ESTATE, "cloud was built without keep_stats");
  if ((rc = cloud_ensure_omg(ctx, c))) return rc;
  std::vector<float4> nrm(n), omg(3 * (size_t)n);
  std::vector<float> eig;
  if (p4) CK(ctx, cudaMemcpyAsync(p4, c->pts, 16 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaMemcpyAsync(nrm.data(), c->nrm, 16 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaMemcpyAsync(omg.data(), c->omg, 48 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  if (ev3 || U9) {
    eig.resize(kStatsWords * (size_t)n);
    CK(ctx, cudaMemcpyAsync(eig.data(), c->eig, 4 * kStatsWords * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; i++) {
    if (p4) p4[4 * i + 3] = 1.0f;  // the device keeps a "has a normal" flag in w
    if (n4) { n4[4 * i] = nrm[i].x; n4[4 * i + 1] = nrm[i].y; n4[4 * i + 2] = nrm[i].z; n4[4 * i + 3] = 0.0f; }
    if (curv) curv[i] = nrm[i].w;
    const float *o = reinterpret_cast<const float *>(&omg[3 * (size_t)i]);
    // (Op00 Op01 Op02 Op11)(Op12 Op22 On00 On01)(On02 On11 On12 On22)
    if (op9) {
      float *d = op9 + 9 * (size_t)i;
      d[0] = o[0]; d[1] = o[1]; d[2] = o[2]; d[3] = o[1]; d[4] = o[3]; d[5] = o[4]; d[6] = o[2]; d[7] = o[4]; d[8] = o[5];
    }
    if (on9) {
      float *d = on9 + 9 * (size_t)i;
      d[0] = o[6]; d[1] = o[7]; d[2] = o[8]; d[3] = o[7]; d[4] = o[9]; d[5] = o[10]; d[6] = o[8]; d[7] = o[10]; d[8] = o[11];
    }
    if (ev3) for (int k = 0; k < 3; k++) ev3[3 * (size_t)i + k] = eig[kStatsWords * (size_t)i + k];
    if (U9) for (int k = 0; k < 9; k++) U9[9 * (size_t)i + k] = eig[kStatsWords * (size_t)i + 3 + k];
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_download_stats(nicp_cloud *c, float *eigval3, float *eigvec9, float *mean3, int *n_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c) return NICP_EINVAL;
  nicp_ctx *ctx = c->ctx;
  int n = 0;
  int rc = nicp_cloud_size(c, &n);
  if (rc) return rc;
  if (n == 0) return NICP_OK;
  if (!c->eig_valid) return fail(ctx, NICP_ESTATE, "cloud was built without keep_stats");
  std::vector<float> e(kStatsWords * (size_t)n);
  CK(ctx, cudaMemcpyAsync(e.data(), c->eig, 4 * kStatsWords * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; i++) {
    const float *r = &e[kStatsWords * (size_t)i];
    if (eigval3) for (int k = 0; k < 3; k++) eigval3[3 * (size_t)i + k] = r[k];
    if (eigvec9) for (int k = 0; k < 9; k++) eigvec9[9 * (size_t)i + k] = r[3 + k];
    if (mean3) for (int k = 0; k < 3; k++) mean3[3 * (size_t)i + k] = r[12 + k];
    if (n_out) n_out[i] = (int)r[15];
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_download_gaussians(nicp_cloud *c, float *mean3, float *cov9) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c) return NICP_EINVAL;
  nicp_ctx *ctx = c->ctx;
  int n = 0;
  int rc = nicp_cloud_size(c, &n);
  if (rc) return rc;
  if (n == 0) return NICP_OK;
  if (!c->gauss_valid) return fail(ctx, NICP_ESTATE, "cloud was built without keep_gaussians");
  std::vector<float4> g(3 * (size_t)n);
  CK(ctx, cudaMemcpyAsync(g.data(), c->gauss, 48 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; i++) {
    const float *o = reinterpret_cast<const float *>(&g[3 * (size_t)i]);
    if (mean3) for (int k = 0; k < 3; k++) mean3[3 * (size_t)i + k] = o[k];
    if (cov9) for (int k = 0; k < 9; k++) cov9[9 * (size_t)i + k] = o[3 + k];
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_upload(nicp_cloud *c, int n, const float *p4, const float *n4, const float *curv,
                                 const float *op9, const float *on9) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c || n < 0 || (n > 0 && (!p4 || !n4 || !curv))) return NICP_EINVAL;
  nicp_ctx *ctx = c->ctx;
  int rc = cloud_reserve(c, n, c->rows, c->cols, false);
  if (rc) return rc;
  c->eig_valid = c->gauss_valid = false;
  c->omega_structured = false;
  c->omg_valid = true;
  std::vector<float4> pts(n), nrm(n), omg(3 * (size_t)n);
  int counts[2] = {n, 0};
  for (int i = 0; i < n; i++) {
    bool has_normal = n4[4 * i] != 0.0f || n4[4 * i + 1] != 0.0f || n4[4 * i + 2] != 0.0f;
    counts[1] += has_normal;
    pts[i] = make_float4(p4[4 * i], p4[4 * i + 1], p4[4 * i + 2], has_normal ? 1.0f : kNoNormalW);
    nrm[i] = make_float4(n4[4 * i], n4[4 * i + 1], n4[4 * i + 2], curv[i]);
    float o[12] = {0};
    if (op9) { const float *s = op9 + 9 * (size_t)i; o[0] = s[0]; o[1] = s[1]; o[2] = s[2]; o[3] = s[4]; o[4] = s[5]; o[5] = s[8]; }
    if (on9) { const float *s = on9 + 9 * (size_t)i; o[6] = s[0]; o[7] = s[1]; o[8] = s[2]; o[9] = s[4]; o[10] = s[5]; o[11] = s[8]; }
    std::memcpy(&omg[3 * (size_t)i], o, sizeof(o));
  }
  if (n > 0) {
    CK(ctx, cudaMemcpyAsync(c->pts, pts.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(c->nrm, nrm.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(c->omg, omg.data(), 48 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
  }
  CK(ctx, cudaMemcpyAsync(c->count, counts, sizeof(counts), cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_transform(nicp_cloud *c, const float T16[16]) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(c ? c->ctx : nullptr);
  if (!c || !T16) return NICP_EINVAL;
  nicp_ctx *ctx = c->ctx;
  if (!c->mem) return NICP_OK;
  HM4 m = HM4::from(T16);
  bool ident = true;
  HM4 I = HM4::identity();
  for (int i = 0; i < 16; i++) ident = ident && (m.a[i] == I.a[i]);
  if (ident) return NICP_OK;  // cloud.cpp:194
  char *pin;
  int rc = pin_up(ctx, 64, &pin);
  if (rc) return rc;
  rows12(m, (float *)pin);
  Layout L;
  size_t o = L.take(48);
  if ((rc = ensure_ws(ctx, L.off))) return rc;
  CK(ctx, cudaMemcpyAsync(ctx->ws + o, pin, 48, cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, ctx->stream));
  launch_cloud_transform(c->pts, c->nrm, c->omg_valid ? c->omg : nullptr, c->eig_valid ? c->eig : nullptr,
                         c->gauss_valid ? c->gauss : nullptr,
                         c->count, c->capacity, (const float *)(ctx->ws + o), ctx->stream, &ctx->prof);
  CK(ctx, cudaGetLastError());
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ cloud build
namespace {
struct FrameIn {
  const void *depth;
  bool u16;
  bool on_device;
  size_t pitch;
  int rows, cols;
  const float *transform;  // projector transform for the unprojection (null = identity)
};
}  // namespace

// Times k_stats on a chunk (its moments complete) with every launch shape
// and returns the fastest.  The kernel writes the same outputs under every
// shape; only its count of points with a normal accumulates, so that count
// is zeroed before each run (and before the real run that follows).
static int tune_stats(nicp_ctx *ctx, int precision, bool lean, const FrameDev *dfr, int nf, int max_pixels,
                      int *best) {
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  CK(ctx, cudaEventCreate(&e0));
  CK(ctx, cudaEventCreate(&e1));
  const bool prof = ctx->prof.enabled;
  ctx->prof.enabled = false;
  float best_ms = 0;
  *best = 0;
  int rc = NICP_OK;
  for (int rep = 0; rep < 2 && rc == NICP_OK; rep++)  // the first pass also loads the kernels
    for (int shape = 0; shape < kStatsShapes; shape++) {
      launch_reset_normal_counts(dfr, nf, s);
      cudaEventRecord(e0, s);
      launch_stats(precision, dfr, nf, max_pixels, shape, lean, s, &ctx->prof);
      cudaEventRecord(e1, s);
      float ms = 0;
      cudaError_t e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        rc = fail(ctx, NICP_ECUDA, std::string("stats autotune: ") + cudaGetErrorString(e));
        break;
      }
      if (rep == 1 && (shape == 0 || ms < best_ms)) {
        best_ms = ms;
        *best = shape;
      }
    }
  launch_reset_normal_counts(dfr, nf, s);
  ctx->prof.enabled = prof;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Builds clouds for frames [0, n) in chunks that bound the integral-image
// scratch.  The descriptors of every chunk are filled first and uploaded in
// one copy.  Frames that need staging (host frames, or device frames that
// are not packed and 16-byte aligned) are then copied into one staging
// region on the copy stream, chunk by chunk, each chunk followed by an
// event; a chunk's kernels wait for its own event only, so the copies of
// later chunks overlap the kernels of earlier ones.  (An upload on the
// compute stream issued after the staging copies would queue behind them in
// the copy engine and hold up every chunk.)  With host frames, chunks hold at
// most kStreamChunkFrames frames (the first kStreamFirstChunkFrames), so
// that the first kernels start early.
static int build_frames(nicp_ctx *ctx, int n, const FrameIn *fin, const nicp_camera *cams, const nicp_cloud_params *prm,
                        nicp_cloud *const *clouds, bool unproject_only) {
  cudaStream_t s = ctx->stream;
  const size_t msz = moment_bytes(prm->moments_precision);
  const size_t kChunkMoments = (size_t)3 << 30;  // bytes of integral image per chunk
  // host frames are built in chunks sized to whole waves of the band sweep
  // (one CTA per 16-row band and frame): the first chunk one wave, so that
  // the kernels start after a few frames' copies, the others the number of
  // waves closest to 32 frames (640x480 at 4 sweep CTAs per SM: 19, then 39)
  const int prec = std::min(std::max(prm->moments_precision, 0), 2);
  if (!ctx->sweep_ctas_per_sm[prec]) ctx->sweep_ctas_per_sm[prec] = moment_sweep_ctas_per_sm(prm->moments_precision);
  const long long wave = (long long)ctx->sweep_ctas_per_sm[prec] * ctx->sm_count;
  auto stream_chunk = [&](int i0, bool first) {
    const int bands = std::max(1, (fin[i0].rows + moment_band_rows() - 1) / moment_band_rows());
    const long long k = first ? 1 : std::max(1LL, (32LL * bands + wave / 2) / wave);
    return (int)std::max(1LL, std::min(65535LL, k * wave / bands));
  };
  int rc;
  for (int i = 0; i < n; i++) {
    if (!fin[i].depth || fin[i].rows <= 0 || fin[i].cols <= 0 || !clouds[i] || !valid_camera(&cams[i]))
      return fail(ctx, NICP_EINVAL, "bad frame " + std::to_string(i));
    if ((long long)fin[i].rows * fin[i].cols > (1ll << 30)) return fail(ctx, NICP_EINVAL, "frame too large");
    if (fin[i].pitch && fin[i].pitch < (size_t)fin[i].cols * (fin[i].u16 ? 2 : 4))
      return fail(ctx, NICP_EINVAL, "row pitch of frame " + std::to_string(i) + " is below its row width");
    if ((rc = cloud_reserve(clouds[i], fin[i].rows * fin[i].cols, fin[i].rows, fin[i].cols, prm->keep_stats != 0,
                            prm->keep_gaussians != 0)))
      return rc;
  }
  if (n <= 0) return NICP_OK;
  // staging needs and chunks
  std::vector<char> staged(n, 0);
  bool any_host = false, any_staged = false;
  for (int i = 0; i < n; i++) {
    const FrameIn &f = fin[i];
    const size_t esz = f.u16 ? 2 : 4;
    const bool packed = f.pitch == 0 || f.pitch == f.cols * esz;
    const bool aligned = ((uintptr_t)f.depth & 15) == 0;
    staged[i] = (!f.on_device || !packed || !aligned) ? 1 : 0;
    any_host |= !f.on_device;
    any_staged |= staged[i] != 0;
  }
  std::vector<std::pair<int, int>> chunks;
  for (int i0 = 0; i0 < n;) {
    // with host frames the first chunk is short, so the kernels start after
    // a few frames' copies
    // (frames per launch are the grids' y dimension: at most 65535)
    const int max_frames = std::min(65535, !any_host ? n : stream_chunk(i0, i0 == 0));
    int i1 = i0;
    size_t mom = 0;
    while (i1 < n && i1 - i0 < max_frames) {
      size_t m = (size_t)fin[i1].rows * fin[i1].cols * 10 * msz;
      if (i1 > i0 && mom + m > kChunkMoments) break;
      mom += m;
      i1++;
    }
    chunks.push_back({i0, i1});
    i0 = i1;
  }
  // one layout for the call: staging region, descriptors, then the scratch
  // of the largest chunk (reused chunk after chunk, in stream order)
  const int nb_rows = moment_band_rows();
  Layout L;
  std::vector<size_t> o_stage(n, 0);
  for (int i = 0; i < n; i++)
    if (staged[i]) o_stage[i] = L.take((size_t)fin[i].rows * fin[i].cols * (fin[i].u16 ? 2 : 4)) + 1;  // +1: "staged"
  // descriptors of every frame, then per chunk the frame of each CTA of the
  // 1-D build grids: unprojection tiles, 16-row bands, band-carry CTAs
  std::vector<size_t> tab_off(chunks.size() + 1, 0);
  std::vector<int> tab_tiles(chunks.size(), 0), tab_bands(chunks.size(), 0);
  for (size_t ci = 0; ci < chunks.size(); ci++) {
    size_t t = 0, b = 0, k = 0;
    for (int i = chunks[ci].first; i < chunks[ci].second; i++) {
      const size_t P = (size_t)fin[i].rows * fin[i].cols;
      t += (P + kUnprojTilePixels - 1) / kUnprojTilePixels;
      b += (fin[i].rows + nb_rows - 1) / nb_rows;
      k += (10 * (size_t)fin[i].cols + 127) / 128;
    }
    tab_tiles[ci] = (int)t;
    tab_bands[ci] = (int)b;
    tab_off[ci + 1] = tab_off[ci] + t + b + k;
  }
  const size_t frames_bytes = sizeof(FrameDev) * n + 4 * tab_off[chunks.size()];
  const size_t o_frames_all = L.take(frames_bytes);
  const size_t scratch0 = L.off;
  size_t scratch_max = scratch0;
  for (auto &c : chunks) {
    Layout C;
    C.off = scratch0;
    const bool rowpath = moments_row_path(c.second - c.first);
    for (int i = c.first; i < c.second; i++) {
      const size_t P = (size_t)fin[i].rows * fin[i].cols;
      C.take(4 * ((P + kUnprojTilePixels - 1) / kUnprojTilePixels));
      if (!unproject_only) {
        C.take(P * 10 * msz);
        C.take((size_t)((fin[i].rows + nb_rows - 1) / nb_rows) * 10 * fin[i].cols * msz);
        if (rowpath) C.take(P * 10 * moment_acc_bytes(prm->moments_precision));
      }
    }
    scratch_max = std::max(scratch_max, C.off);
  }
  if ((rc = ensure_ws(ctx, scratch_max))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, frames_bytes, &pin))) return rc;
  int *tab_all = reinterpret_cast<int *>(pin + sizeof(FrameDev) * n);
  struct Grid { int tiles, bands, carryctas, max_bands, max_pixels; };
  std::vector<Grid> grids(chunks.size());
  for (size_t ci = 0; ci < chunks.size(); ci++) {
    const int i0 = chunks[ci].first, nf = chunks[ci].second - i0;
    Layout C;
    C.off = scratch0;
    std::vector<size_t> o_tiles(nf), o_mom(nf), o_band(nf), o_rowpre(nf, 0);
    const bool rowpath = moments_row_path(nf);
    for (int k = 0; k < nf; k++) {
      const FrameIn &f = fin[i0 + k];
      size_t P = (size_t)f.rows * f.cols;
      o_tiles[k] = C.take(4 * ((P + kUnprojTilePixels - 1) / kUnprojTilePixels));
      o_mom[k] = unproject_only ? 0 : C.take(P * 10 * msz);
      o_band[k] = unproject_only ? 0 : C.take((size_t)((f.rows + nb_rows - 1) / nb_rows) * 10 * f.cols * msz);
      if (!unproject_only && rowpath) o_rowpre[k] = C.take(P * 10 * moment_acc_bytes(prm->moments_precision));
    }
    FrameDev *fd = reinterpret_cast<FrameDev *>(pin) + i0;
    int *tab_t = tab_all + tab_off[ci], *tab_b = tab_t + tab_tiles[ci], *tab_k = tab_b + tab_bands[ci];
    int tiles = 0, bands = 0, carryctas = 0, max_bands = 0, max_pixels = 0;
    for (int k = 0; k < nf; k++) {
      const FrameIn &f = fin[i0 + k];
      const nicp_camera &cam = cams[i0 + k];
      nicp_cloud *cl = clouds[i0 + k];
      size_t P = (size_t)f.rows * f.cols;
      const void *src = o_stage[i0 + k] ? (const void *)(ctx->ws + (o_stage[i0 + k] - 1)) : f.depth;
      FrameDev &d = fd[k];
      std::memset(&d, 0, sizeof(d));
      d.depth_u16 = f.u16 ? (const uint16_t *)src : nullptr;
      d.depth_f32 = f.u16 ? nullptr : (const float *)src;
      d.rows = f.rows;
      d.cols = f.cols;
      d.tile_base = tiles;
      d.band_base = bands;
      d.col_base = carryctas;
      for (int q = 0, m = (int)((P + kUnprojTilePixels - 1) / kUnprojTilePixels); q < m; q++) tab_t[tiles + q] = k;
      for (int q = 0, m = (f.rows + nb_rows - 1) / nb_rows; q < m; q++) tab_b[bands + q] = k;
      for (int q = 0, m = (10 * f.cols + 127) / 128; q < m; q++) tab_k[carryctas + q] = k;
      tiles += (int)((P + kUnprojTilePixels - 1) / kUnprojTilePixels);
      bands += (f.rows + nb_rows - 1) / nb_rows;
      max_bands = std::max(max_bands, (f.rows + nb_rows - 1) / nb_rows);
      max_pixels = std::max(max_pixels, (int)P);
      carryctas += (10 * f.cols + 127) / 128;
      d.depth_scale = prm->depth_scale;
      d.min_d = cam.min_distance;
      d.max_d = cam.max_distance;
      HM4 KRt, iKRt;
      projector_matrices(cam, HM4::from(f.transform), KRt, iKRt);
      rows12(iKRt, d.iKRt);
      cam_K(cam, d.K);
      d.world_radius = prm->world_radius;
      d.min_radius = prm->min_image_radius;
      d.max_radius = prm->max_image_radius;
      d.min_points = prm->min_points;
      d.curv_thr = prm->curvature_threshold;
      for (int q = 0; q < 3; q++) {
        d.pim_flat[q] = prm->pim_flat[q]; d.pim_nonflat[q] = prm->pim_nonflat[q];
        d.nim_flat[q] = prm->nim_flat[q]; d.nim_nonflat[q] = prm->nim_nonflat[q];
      }
      d.pim_thr = prm->pim_curvature_threshold;
      d.nim_thr = prm->nim_curvature_threshold;
      d.keep_stats = prm->keep_stats && cl->has_eig;
      cl->eig_valid = d.keep_stats != 0;
      {
        float K[9];
        cam_K(cam, K);
        hm_inv3(K, d.iK);
        d.fB = cam.baseline * K[0];
        d.alpha = cam.alpha;
      }
      d.gauss = (prm->keep_gaussians && cl->has_gauss) ? cl->gauss : nullptr;
      cl->gauss_valid = d.gauss != nullptr;
      cl->omega_structured = prm->pim_flat[1] == prm->pim_flat[2] && prm->pim_nonflat[1] == prm->pim_nonflat[2] &&
                             prm->nim_flat[1] == prm->nim_flat[2] && prm->nim_nonflat[1] == prm->nim_nonflat[2];
      // the stats kernel's lean form (below) leaves Omega implicit; an
      // unprojection-only build writes no normals or matrices at all
      cl->omg_valid = unproject_only || !(!prm->keep_stats && cl->omega_structured);
      {
        const float od[8] = {prm->pim_flat[0], prm->pim_flat[1], prm->pim_nonflat[0], prm->pim_nonflat[1],
                             prm->nim_flat[0], prm->nim_flat[1], prm->nim_nonflat[0], prm->nim_nonflat[1]};
        std::memcpy(cl->omd, od, sizeof(od));
      }
      d.index = cl->index;
      d.pts = cl->pts;
      d.nrm = cl->nrm;
      d.omg = cl->omg;
      d.eig = cl->eig;
      d.count = cl->count;
      d.tile_counts = (int *)(ctx->ws + o_tiles[k]);
      d.moments = unproject_only ? nullptr : (void *)(ctx->ws + o_mom[k]);
      d.band_tot = unproject_only ? nullptr : (void *)(ctx->ws + o_band[k]);
      d.rowpre = o_rowpre[k] ? (void *)(ctx->ws + o_rowpre[k]) : nullptr;
    }
    grids[ci] = {tiles, bands, carryctas, max_bands, max_pixels};
  }
  FrameDev *dfr_all = (FrameDev *)(ctx->ws + o_frames_all);
  CK(ctx, cudaMemcpyAsync(dfr_all, pin, frames_bytes, cudaMemcpyHostToDevice, s));
  ctx->h2d_bytes += frames_bytes;
  const int *dtab_all = reinterpret_cast<const int *>(ctx->ws + o_frames_all + sizeof(FrameDev) * n);
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  if (any_staged) {
    if (!ctx->copy_stream) CK(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if (!ctx->copy_start) CK(ctx, cudaEventCreateWithFlags(&ctx->copy_start, cudaEventDisableTiming));
    while (ctx->copy_ev.size() < chunks.size()) {
      cudaEvent_t e;
      CK(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ctx->copy_ev.push_back(e);
    }
    // the staging region may still be read by earlier work on the compute stream
    CK(ctx, cudaEventRecord(ctx->copy_start, s));
    CK(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_start, 0));
    for (size_t c = 0; c < chunks.size(); c++) {
      for (int i = chunks[c].first; i < chunks[c].second; i++) {
        if (!staged[i]) continue;
        const FrameIn &f = fin[i];
        const size_t esz = f.u16 ? 2 : 4;
        const size_t pitch = f.pitch ? f.pitch : f.cols * esz;
        const cudaMemcpyKind kind = f.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        cudaError_t e;
        if (pitch == f.cols * esz)  // packed rows: one linear copy
          e = cudaMemcpyAsync(ctx->ws + (o_stage[i] - 1), f.depth, pitch * f.rows, kind, ctx->copy_stream);
        else
          e = cudaMemcpy2DAsync(ctx->ws + (o_stage[i] - 1), f.cols * esz, f.depth, pitch, f.cols * esz, f.rows, kind,
                                ctx->copy_stream);
        if (e != cudaSuccess) {
          cudaStreamSynchronize(ctx->copy_stream);  // copies already queued may read the caller's frames
          return fail(ctx, NICP_ECUDA, std::string("depth staging copy: ") + cudaGetErrorString(e));
        }
        if (!f.on_device) ctx->h2d_bytes += (unsigned long long)f.cols * esz * f.rows;
      }
      cudaError_t e = cudaEventRecord(ctx->copy_ev[c], ctx->copy_stream);
      if (e != cudaSuccess) {
        cudaStreamSynchronize(ctx->copy_stream);
        return fail(ctx, NICP_ECUDA, std::string("staging event: ") + cudaGetErrorString(e));
      }
    }
  }
  // From here on an error return first waits for the staging copies: they
  // may read the caller's host frames, which the caller may free on error.
  auto fail_staged = [&](cudaError_t e, const char *what) {
    if (any_staged) cudaStreamSynchronize(ctx->copy_stream);
    return fail(ctx, NICP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  for (size_t ci = 0; ci < chunks.size(); ci++) {
    const int i0 = chunks[ci].first, nf = chunks[ci].second - i0;
    const Grid &g = grids[ci];
    cudaError_t e;
    if (any_staged && (e = cudaStreamWaitEvent(s, ctx->copy_ev[ci], 0)) != cudaSuccess)
      return fail_staged(e, "cudaStreamWaitEvent");
    const FrameDev *dfr = dfr_all + i0;
    const int *ft = dtab_all + tab_off[ci], *fb = ft + tab_tiles[ci], *fk = fb + tab_bands[ci];
    launch_unproject(dfr, nf, g.tiles, ft, s, &ctx->prof);
    if (!unproject_only) {
      launch_moments(prm->moments_precision, dfr, nf, g.bands, g.carryctas, g.max_bands, fb, fk, s, &ctx->prof);
      // only the smallest eigenpair is needed unless Stats are kept or an
      // information matrix has distinct second and third diagonal entries
      const bool lean = !prm->keep_stats && prm->pim_flat[1] == prm->pim_flat[2] &&
                        prm->pim_nonflat[1] == prm->pim_nonflat[2] && prm->nim_flat[1] == prm->nim_flat[2] &&
                        prm->nim_nonflat[1] == prm->nim_nonflat[2];
      int shape = 0;
      if (ctx->autotune) {
        // the chunk's frame sizes and the moment precision select the shape
        std::map<std::pair<int, int>, int> hist;
        for (int i = i0; i < i0 + nf; i++) hist[{fin[i].rows, fin[i].cols}]++;
        std::string key = std::to_string(prm->moments_precision) + ":";
        for (auto &h : hist)
          key += std::to_string(h.first.first) + "x" + std::to_string(h.first.second) + "*" +
                 std::to_string(h.second) + " ";
        auto it = ctx->stats_tuned.find(key);
        if (it == ctx->stats_tuned.end()) {
          int best = 0, rc = tune_stats(ctx, prm->moments_precision, lean, dfr, nf, g.max_pixels, &best);
          if (rc) {
            if (any_staged) cudaStreamSynchronize(ctx->copy_stream);
            return rc;
          }
          it = ctx->stats_tuned.emplace(key, best).first;
        }
        shape = it->second;
      }
      ctx->stats_shape = shape;
      launch_stats(prm->moments_precision, dfr, nf, g.max_pixels, shape, lean, s, &ctx->prof);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail_staged(e, "build launch");
  }
  return NICP_OK;
}

static int build_one(nicp_ctx *ctx, const void *depth, bool u16, int rows, int cols, size_t pitch, int on_device,
                     const nicp_camera *cam, const nicp_cloud_params *prm, const float *offset, nicp_cloud *out,
                     int32_t *index_out) {
  if (!ctx || !out || !prm) return NICP_EINVAL;
  if (out->ctx != ctx) return fail(ctx, NICP_EINVAL, "cloud belongs to another context");
  FrameIn f{depth, u16, on_device != 0, pitch, rows, cols, nullptr};
  int rc = build_frames(ctx, 1, &f, cam, prm, &out, false);
  if (rc) return rc;
  if (offset && (rc = nicp_cloud_transform(out, offset))) return rc;
  if (index_out) {
    CK(ctx, cudaMemcpyAsync(index_out, out->index, 4 * (size_t)rows * cols, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return NICP_OK;
}

extern "C" int nicp_cloud_from_depth_u16(nicp_ctx *ctx, const uint16_t *depth, int rows, int cols, size_t pitch,
                                         int on_device, const nicp_camera *cam, const nicp_cloud_params *prm,
                                         const float *offset, nicp_cloud *out, int32_t *index_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  return build_one(ctx, depth, true, rows, cols, pitch, on_device, cam, prm, offset, out, index_out);
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_from_depth_f32(nicp_ctx *ctx, const float *depth, int rows, int cols, size_t pitch,
                                         int on_device, const nicp_camera *cam, const nicp_cloud_params *prm,
                                         const float *offset, nicp_cloud *out, int32_t *index_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  return build_one(ctx, depth, false, rows, cols, pitch, on_device, cam, prm, offset, out, index_out);
  NICP_ABI_CATCH
}

extern "C" int nicp_build_batch(nicp_ctx *ctx, int n, const uint16_t *const *depth, const int *rows, const int *cols,
                                int on_device, const nicp_camera *cams, const nicp_cloud_params *prm,
                                nicp_cloud *const *out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || n < 0 || (n > 0 && (!depth || !rows || !cols || !cams || !prm || !out))) return NICP_EINVAL;
  std::vector<FrameIn> f(n);
  for (int i = 0; i < n; i++) {
    if (out[i] && out[i]->ctx != ctx) return fail(ctx, NICP_EINVAL, "cloud belongs to another context");
    f[i] = FrameIn{depth[i], true, on_device != 0, 0, rows[i], cols[i], nullptr};
  }
  return build_frames(ctx, n, f.data(), cams, prm, out, false);
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ projector API
extern "C" int nicp_projector_matrices(const nicp_camera *cam, const float T16[16], float KRt16[16], float iKRt16[16]) {
  NICP_ABI_TRY
  if (!cam || !KRt16 || !iKRt16) return NICP_EINVAL;
  HM4 K, iK;
  projector_matrices(*cam, HM4::from(T16), K, iK);
  std::memcpy(KRt16, K.a, sizeof(K.a));
  std::memcpy(iKRt16, iK.a, sizeof(iK.a));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_unproject(nicp_ctx *ctx, const float *depth, int rows, int cols, const nicp_camera *cam,
                              const float T16[16], float *points4_out, int32_t *index_out, int *n) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !depth || !cam || !n) return NICP_EINVAL;
  int rc;
  if (!ctx->scratch_cloud && (rc = nicp_cloud_create(ctx, &ctx->scratch_cloud))) return rc;
  nicp_cloud_params prm;
  nicp_default_cloud_params(&prm);
  FrameIn f{depth, false, false, 0, rows, cols, T16};
  nicp_cloud *c = ctx->scratch_cloud;
  if ((rc = build_frames(ctx, 1, &f, cam, &prm, &c, true))) return rc;
  if ((rc = nicp_cloud_size(c, n))) return rc;
  if (points4_out && *n) {
    CK(ctx, cudaMemcpyAsync(points4_out, c->pts, 16 * (size_t)*n, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (index_out) CK(ctx, cudaMemcpyAsync(index_out, c->index, 4 * (size_t)rows * cols, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_project_intervals(nicp_ctx *ctx, const float *depth, int rows, int cols, const nicp_camera *cam,
                                      float world_radius, int32_t *radius_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !depth || !cam || !radius_out || rows <= 0 || cols <= 0) return NICP_EINVAL;
  size_t P = (size_t)rows * cols;
  Layout L;
  size_t o_d = L.take(4 * P), o_k = L.take(36), o_o = L.take(4 * P);
  int rc;
  if ((rc = ensure_ws(ctx, L.off))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, 36, &pin))) return rc;
  cam_K(*cam, (float *)pin);
  CK(ctx, cudaMemcpyAsync(ctx->ws + o_k, pin, 36, cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, ctx->stream));
  CK(ctx, cudaMemcpyAsync(ctx->ws + o_d, depth, 4 * P, cudaMemcpyHostToDevice, ctx->stream));
  launch_intervals((const float *)(ctx->ws + o_d), (int)P, (const float *)(ctx->ws + o_k), cam->min_distance,
                   cam->max_distance, world_radius, (int32_t *)(ctx->ws + o_o), ctx->stream, &ctx->prof);
  CK(ctx, cudaGetLastError());
  CK(ctx, cudaMemcpyAsync(radius_out, ctx->ws + o_o, 4 * P, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ pair workspace
namespace {
struct PairPlan {
  int n = 0;
  size_t o_extra = 0;
  bool keep_ref = false, list_mode = false;
  bool structured = false;  // every current cloud has structured Omegas (k_corr_lin<true>)
  int total_tiles = 0, max_pt_tiles = 0;  // max_pt_tiles: 1024-point tiles of the largest projected cloud
  int max_tiles = 0;                      // pixel tiles of the largest pair image
  size_t o_pairs = 0, o_states = 0, o_krt = 0, o_guess = 0, o_roff = 0, o_zbuf = 0, zbuf_bytes = 0;
  size_t o_tile_pair = 0;  // int per pixel tile: its pair
  std::vector<size_t> o_cur, o_ref, o_part, o_list, o_ltc, o_np;
  std::vector<int> P, tiles;
};
}  // namespace

// Lays out per-pair buffers; cams[i] gives the projection image of pair i.
static int plan_pairs(nicp_ctx *ctx, int n, const nicp_camera *cams, const nicp_cloud *const *refs, bool keep_ref,
                      bool list_mode, PairPlan &pl, size_t extra_bytes = 0) {
  pl.n = n;
  pl.keep_ref = keep_ref;
  pl.list_mode = list_mode;
  Layout L;
  pl.o_pairs = L.take(sizeof(PairDev) * n);
  pl.o_states = L.take(sizeof(PairState) * n);
  pl.o_krt = L.take(48 * (size_t)n);
  pl.o_guess = L.take(128 * (size_t)n);
  pl.o_roff = L.take(128 * (size_t)n);
  size_t ztot = 0;
  pl.P.resize(n);
  pl.tiles.resize(n);
  for (int i = 0; i < n; i++) {
    if (!valid_camera(&cams[i])) return fail(ctx, NICP_EINVAL, "bad camera for pair " + std::to_string(i));
    size_t P = (size_t)cam_rows(cams[i]) * cam_cols(cams[i]);
    if (P > (1u << 30)) return fail(ctx, NICP_EINVAL, "projection image too large");
    pl.P[i] = (int)P;
    pl.tiles[i] = (int)((P + kCorrTilePixels - 1) / kCorrTilePixels);
    pl.max_tiles = std::max(pl.max_tiles, pl.tiles[i]);
    ztot += align_up(8 * P, 256);
  }
  pl.o_zbuf = L.take(ztot);
  pl.zbuf_bytes = ztot;
  pl.o_cur.resize(n); pl.o_ref.resize(n); pl.o_part.resize(n);
  pl.o_list.resize(n); pl.o_ltc.resize(n); pl.o_np.resize(n);
  pl.total_tiles = 0;
  pl.max_pt_tiles = 0;
  for (int i = 0; i < n; i++) {
    size_t P = pl.P[i];
    pl.o_cur[i] = L.take(4 * P);
    pl.o_ref[i] = (keep_ref || list_mode) ? L.take(4 * P) : 0;
    pl.o_part[i] = L.take(8 * kPartialWords * (size_t)pl.tiles[i]);
    pl.o_list[i] = list_mode ? L.take(8 * P) : 0;
    pl.o_ltc[i] = list_mode ? L.take(4 * (size_t)pl.tiles[i]) : 0;
    pl.o_np[i] = L.take(4);
    pl.total_tiles += pl.tiles[i];
    int cap = std::max(refs[i] ? refs[i]->capacity : 0, 1);
    pl.max_pt_tiles = std::max(pl.max_pt_tiles, (cap + kPointsPerCta - 1) / kPointsPerCta);
  }
  pl.o_tile_pair = L.take(4 * (size_t)std::max(pl.total_tiles, 1));
  pl.o_extra = L.take(std::max<size_t>(extra_bytes, 1));
  return ensure_ws(ctx, L.off);
}

// Fills the PairDev descriptors in host memory.
static void fill_pairs(nicp_ctx *ctx, const PairPlan &pl, const nicp_camera *cams, const nicp_cloud *const *refs,
                       const nicp_cloud *const *curs, PairDev *pd) {
  char *ws = ctx->ws;
  int tb = 0;
  size_t zoff = pl.o_zbuf;
  for (int i = 0; i < pl.n; i++) {
    PairDev &d = pd[i];
    std::memset(&d, 0, sizeof(d));
    const nicp_cloud *r = refs[i], *c = curs[i];
    d.ref_pts = r ? r->pts : nullptr;
    d.ref_nrm = r ? r->nrm : nullptr;
    d.ref_count = r ? r->count : nullptr;
    d.cur_pts = c ? c->pts : nullptr;
    d.cur_nrm = c ? c->nrm : nullptr;
    d.cur_omg = c ? c->omg : nullptr;
    d.cur_count = c ? c->count : nullptr;
    d.cur_structured = (c && c->omega_structured) ? 1 : 0;
    if (c) std::memcpy(d.cur_omd, c->omd, sizeof(d.cur_omd));
    d.rows = cam_rows(cams[i]);
    d.cols = cam_cols(cams[i]);
    d.tile_base = tb;
    d.ref_capacity = std::max(r ? r->capacity : 0, 1);
    tb += pl.tiles[i];
    d.min_d = cams[i].min_distance;
    d.max_d = cams[i].max_distance;
    cam_K(cams[i], d.K);
    d.cur_index = (int32_t *)(ws + pl.o_cur[i]);
    d.ref_index = pl.o_ref[i] ? (int32_t *)(ws + pl.o_ref[i]) : nullptr;
    d.zbuf = (unsigned long long *)(ws + zoff);
    zoff += align_up(8 * (size_t)pl.P[i], 256);
    d.partials = (double *)(ws + pl.o_part[i]);
    d.pairs = pl.o_list[i] ? (int32_t *)(ws + pl.o_list[i]) : nullptr;
    d.list_tile_counts = pl.o_ltc[i] ? (int *)(ws + pl.o_ltc[i]) : nullptr;
    d.num_pairs = (int *)(ws + pl.o_np[i]);
    d.state = (PairState *)(ws + pl.o_states) + i;
  }
}

// ------------------------------------------------------------------ correspondences / linearizer API
extern "C" int nicp_correspond(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const int32_t *ref_index,
                               const int32_t *cur_index, int rows, int cols, const float T16[16],
                               const nicp_corr_params *prm, int32_t *pairs_out, int *num_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !ref || !cur || !ref_index || !cur_index || rows <= 0 || cols <= 0 || !T16 || !prm || !num_out)
    return NICP_EINVAL;
  if (prm->row_search_region < 0 || prm->col_search_region < 0 || prm->row_search_region > 16 ||
      prm->col_search_region > 16)
    return fail(ctx, NICP_EINVAL, "search regions must lie in [0, 16]");
  nicp_camera cam;
  nicp_default_camera(&cam);
  cam.rows = rows;
  cam.cols = cols;
  PairPlan pl;
  int rc;
  if ((rc = plan_pairs(ctx, 1, &cam, &ref, false, true, pl))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, sizeof(PairDev) + 48, &pin))) return rc;
  PairDev *pd = (PairDev *)pin;
  fill_pairs(ctx, pl, &cam, &ref, &cur, pd);
  float *T12 = (float *)(pin + sizeof(PairDev));
  rows12(HM4::from(T16), T12);
  cudaStream_t s = ctx->stream;
  size_t P = (size_t)rows * cols;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_pairs, pin, sizeof(PairDev), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_krt, T12, 48, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_ref[0], ref_index, 4 * P, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_cur[0], cur_index, 4 * P, cudaMemcpyHostToDevice, s));
  launch_corr_list((const PairDev *)(ctx->ws + pl.o_pairs), 1, pl.total_tiles, corr_params(*prm), 0,
                   (const float *)(ctx->ws + pl.o_krt), s, &ctx->prof);
  CK(ctx, cudaGetLastError());
  CK(ctx, cudaMemcpyAsync(num_out, ctx->ws + pl.o_np[0], 4, cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  if (pairs_out && *num_out > 0) {
    CK(ctx, cudaMemcpyAsync(pairs_out, ctx->ws + pl.o_list[0], 8 * (size_t)*num_out, cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaStreamSynchronize(s));
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_linearize(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const int32_t *pairs,
                              int num_pairs, const float T16[16], const nicp_lin_params *prm, int parity_threads,
                              double H36[36], double b6[6], double *error, int *inliers) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !ref || !cur || (num_pairs > 0 && !pairs) || num_pairs < 0 || !T16 || !prm) return NICP_EINVAL;
  // list slots are tiled like pixels: a one-row image of num_pairs pixels
  nicp_camera cam;
  nicp_default_camera(&cam);
  cam.rows = 1;
  cam.cols = std::max(num_pairs, 1);
  PairPlan pl;
  int rc;
  if ((rc = plan_pairs(ctx, 1, &cam, &ref, false, true, pl))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, sizeof(PairDev) + 48 + 4, &pin))) return rc;
  if ((rc = cloud_ensure_omg(ctx, cur))) return rc;  // the list linearizer reads the matrices
  PairDev *pd = (PairDev *)pin;
  fill_pairs(ctx, pl, &cam, &ref, &cur, pd);
  float *T12 = (float *)(pin + sizeof(PairDev));
  rows12(HM4::from(T16), T12);
  int *np = (int *)(pin + sizeof(PairDev) + 48);
  *np = num_pairs;
  cudaStream_t s = ctx->stream;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_pairs, pin, sizeof(PairDev), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_krt, T12, 48, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_np[0], np, 4, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  if (num_pairs > 0)
    CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_list[0], pairs, 8 * (size_t)num_pairs, cudaMemcpyHostToDevice, s));
  const PairDev *dpd = (const PairDev *)(ctx->ws + pl.o_pairs);
  launch_lin_list(dpd, 1, pl.total_tiles, lin_params(*prm), std::max(1, parity_threads), 0,
                  (const float *)(ctx->ws + pl.o_krt), s, &ctx->prof);
  launch_solve(dpd, 1, 0.0f, 2 | (prm->cross_block_f32 ? kSolveCrossF32 : 0), 0.0, 1, s, &ctx->prof);
  CK(ctx, cudaGetLastError());
  char *pd_host;
  if ((rc = pin_down(ctx, sizeof(PairState), &pd_host))) return rc;
  CK(ctx, cudaMemcpyAsync(pd_host, ctx->ws + pl.o_states, sizeof(PairState), cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  const PairState *st = (const PairState *)pd_host;
  if (H36) std::memcpy(H36, st->H, sizeof(st->H));
  if (b6) std::memcpy(b6, st->b, sizeof(st->b));
  if (error) *error = st->error;
  if (inliers) *inliers = st->inliers;
  return NICP_OK;
  NICP_ABI_CATCH
}

// Scratch-free linearizer (see nicp_gpu.h): unpacks the cloud handles and
// enqueues k_lin_noalloc; no allocation and no error text on this path.
extern "C" int nicp_linearize_noalloc(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur,
                                      const int32_t *pairs_dev, int num_pairs, const float T16[16],
                                      const nicp_lin_params *prm, int parity_threads, double *out_dev) {
  NICP_ABI_TRY
  if (!ctx || !ref || !cur || !T16 || !prm || !out_dev || num_pairs < 0 || (num_pairs > 0 && !pairs_dev))
    return NICP_EINVAL;
  if (num_pairs > NICP_LINEARIZE_NOALLOC_MAX_PAIRS) return NICP_EINVAL;
  if (!ref->mem || !cur->mem) return NICP_EINVAL;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return NICP_ECUDA;
  if (device != ctx->device) return NICP_ESTATE;
  if (!cur->omg_valid) {  // an implicit Omega is written out first (no allocation)
    launch_materialize_omg(cur->pts, cur->nrm, cur->omg, cur->count, cur->capacity, cur->omd, ctx->stream);
    if (cudaGetLastError() != cudaSuccess) return NICP_ECUDA;
    cur->omg_valid = true;
  }
  NoAllocLinArgs a;
  a.ref_pts = ref->pts;
  a.ref_nrm = ref->nrm;
  a.ref_count = ref->count;
  a.cur_pts = cur->pts;
  a.cur_nrm = cur->nrm;
  a.cur_omg = cur->omg;
  a.cur_count = cur->count;
  a.pairs = pairs_dev;
  a.num_pairs = num_pairs;
  a.parity_threads = std::max(1, parity_threads);
  rows12(HM4::from(T16), a.T);
  a.lp = lin_params(*prm);
  return lin_noalloc(a, out_dev, ctx->stream);
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ projection API
extern "C" int nicp_project(nicp_ctx *ctx, const nicp_cloud *cloud, const nicp_camera *cam, const float T16[16],
                            int32_t *index_out, float *depth_out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !cloud || !cam || !valid_camera(cam)) return NICP_EINVAL;
  PairPlan pl;
  int rc;
  size_t P = (size_t)cam_rows(*cam) * cam_cols(*cam);
  if ((rc = plan_pairs(ctx, 1, cam, &cloud, false, false, pl, 4 * P))) return rc;
  size_t o_depth = pl.o_extra;
  char *pin;
  if ((rc = pin_up(ctx, sizeof(PairDev) + 48, &pin))) return rc;
  const nicp_cloud *cur = cloud;
  fill_pairs(ctx, pl, cam, &cloud, &cur, (PairDev *)pin);
  HM4 KRt, iKRt;
  projector_matrices(*cam, HM4::from(T16), KRt, iKRt);
  float *k12 = (float *)(pin + sizeof(PairDev));
  rows12(KRt, k12);
  cudaStream_t s = ctx->stream;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_pairs, pin, sizeof(PairDev), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_krt, k12, 48, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  CK(ctx, cudaMemsetAsync(ctx->ws + pl.o_zbuf, 0xff, pl.zbuf_bytes, s));
  const PairDev *dpd = (const PairDev *)(ctx->ws + pl.o_pairs);
  launch_zbuffer(dpd, 1, pl.max_pt_tiles, 0, (const float *)(ctx->ws + pl.o_krt), kZbufDefaultPPT, s, &ctx->prof);
  launch_resolve(dpd, 1, pl.max_tiles, 0, (float *)(ctx->ws + o_depth), 0, s, &ctx->prof);
  CK(ctx, cudaGetLastError());
  if (index_out) CK(ctx, cudaMemcpyAsync(index_out, ctx->ws + pl.o_cur[0], 4 * P, cudaMemcpyDeviceToHost, s));
  if (depth_out) CK(ctx, cudaMemcpyAsync(depth_out, ctx->ws + o_depth, 4 * P, cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ multi-resolution input
extern "C" int nicp_depth_scale(nicp_ctx *ctx, const void *depth, int is_u16, int rows, int cols, size_t pitch_bytes,
                                int on_device, float depth_scale, int step, float max_depth_cov, float *out,
                                int out_on_device) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !depth || !out || rows <= 0 || cols <= 0 || step < 1) return NICP_EINVAL;
  const size_t elem = is_u16 ? 2 : 4;
  if (pitch_bytes == 0) pitch_bytes = elem * (size_t)cols;
  if (pitch_bytes < elem * (size_t)cols || pitch_bytes % elem) return fail(ctx, NICP_EINVAL, "bad row pitch");
  const int orows = rows / step, ocols = cols / step;
  const size_t in_bytes = pitch_bytes * (size_t)rows, out_bytes = 4 * (size_t)orows * ocols;
  if (orows == 0 || ocols == 0) return NICP_OK;
  Layout L;
  size_t o_in = L.take(on_device ? 1 : in_bytes), o_out = L.take(out_on_device ? 1 : out_bytes);
  int rc;
  if ((rc = ensure_ws(ctx, L.off))) return rc;
  cudaStream_t s = ctx->stream;
  const void *src = depth;
  if (!on_device) {
    char *pin;
    if ((rc = pin_up(ctx, in_bytes, &pin))) return rc;
    std::memcpy(pin, depth, in_bytes);
    CK(ctx, cudaMemcpyAsync(ctx->ws + o_in, pin, in_bytes, cudaMemcpyHostToDevice, s));
    CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
    ctx->h2d_bytes += in_bytes;
    src = ctx->ws + o_in;
  }
  float *dst = out_on_device ? out : (float *)(ctx->ws + o_out);
  launch_depth_scale(is_u16 ? (const uint16_t *)src : nullptr, is_u16 ? nullptr : (const float *)src,
                     pitch_bytes / elem, rows, cols, depth_scale, step, max_depth_cov, dst, s);
  CK(ctx, cudaGetLastError());
  if (!out_on_device) {
    char *pin;
    if ((rc = pin_down(ctx, out_bytes, &pin))) return rc;
    CK(ctx, cudaMemcpyAsync(pin, dst, out_bytes, cudaMemcpyDeviceToHost, s));
    CK(ctx, cudaStreamSynchronize(s));
    std::memcpy(out, pin, out_bytes);
    ctx->d2h_bytes += out_bytes;
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ nearest-neighbour association
static int cloud_counts2(nicp_cloud *c, int out[2]);

namespace {
// Workspace of one NN alignment: the grid over the current cloud, the match
// / flag / position arrays over the reference points, the pair list, FP64
// partials, the pair descriptor and state.
struct NNPlan {
  int nr = 0, nc = 0, tiles = 0;
  NNGrid grid{};
  size_t o_keys, o_skeys, o_idx, o_sidx, o_feat, o_sfeat, o_cstart, o_cend, o_temp, temp_bytes;
  size_t o_match, o_flag, o_pos, o_pairs, o_np, o_part, o_pd, o_st, o_guess, o_roff;
};

// Bounding box of the current cloud (host), then the grid: cell h =
// cbrt(volume / points) (about one cell per point of a surface patch; at
// least 1 mm), at most 2^24 cells.
int nn_plan(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, float radius, NNPlan &pl) {
  int rc;
  int cr[2], cc[2];
  if ((rc = cloud_counts2(const_cast<nicp_cloud *>(ref), cr)) || (rc = cloud_counts2(const_cast<nicp_cloud *>(cur), cc)))
    return rc;
  pl.nr = cr[0];
  pl.nc = cc[0];
  std::vector<float4> pts(std::max(pl.nc, 1));
  if (pl.nc > 0) {
    CK(ctx, cudaMemcpyAsync(pts.data(), cur->pts, 16 * (size_t)pl.nc, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
  }
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int j = 0; j < pl.nc; j++) {
    const float v[3] = {pts[j].x, pts[j].y, pts[j].z};
    for (int a = 0; a < 3; a++) {
      if (j == 0 || v[a] < lo[a]) lo[a] = v[a];
      if (j == 0 || v[a] > hi[a]) hi[a] = v[a];
    }
  }
  double ext[3], vol = 1.0;
  for (int a = 0; a < 3; a++) {
    ext[a] = std::max(1e-3, (double)hi[a] - lo[a]);
    vol *= ext[a];
  }
  double h = std::max(1e-3, std::cbrt(vol / std::max(pl.nc, 1)));
  for (;;) {
    double cells = 1.0;
    for (int a = 0; a < 3; a++) cells *= std::floor(ext[a] / h) + 1;
    if (cells <= (double)(1 << 24)) break;
    h *= 1.25;
  }
  NNGrid &g = pl.grid;
  g.h = (float)h;
  g.inv_h = (float)(1.0 / h);
  for (int a = 0; a < 3; a++) {
    g.origin[a] = lo[a];
    g.dim[a] = (int)std::floor(ext[a] / h) + 1;
  }
  g.max_shell = (int)std::ceil(radius / h) + 1;
  const size_t ncells = (size_t)g.dim[0] * g.dim[1] * g.dim[2];
  const size_t NC = std::max(pl.nc, 1), NR = std::max(pl.nr, 1);
  pl.tiles = (int)((NR + kCorrTilePixels - 1) / kCorrTilePixels);
  pl.temp_bytes = std::max(nn_temp_bytes((int)NC), nn_temp_bytes((int)NR));
  Layout L;
  pl.o_keys = L.take(4 * NC); pl.o_skeys = L.take(4 * NC); pl.o_idx = L.take(4 * NC); pl.o_sidx = L.take(4 * NC);
  pl.o_feat = L.take(24 * NC); pl.o_sfeat = L.take(24 * NC);
  pl.o_cstart = L.take(4 * ncells); pl.o_cend = L.take(4 * ncells);
  pl.o_temp = L.take(pl.temp_bytes);
  pl.o_match = L.take(4 * NR); pl.o_flag = L.take(4 * NR); pl.o_pos = L.take(4 * NR);
  pl.o_pairs = L.take(8 * NR); pl.o_np = L.take(4);
  pl.o_part = L.take(8 * kPartialWords * (size_t)pl.tiles);
  pl.o_pd = L.take(sizeof(PairDev)); pl.o_st = L.take(sizeof(PairState));
  pl.o_guess = L.take(128); pl.o_roff = L.take(128);
  return ensure_ws(ctx, L.off);
}

int nn_build(nicp_ctx *ctx, const NNPlan &pl, const nicp_cloud *cur, float nscale) {
  char *ws = ctx->ws;
  NNBuild b{};
  b.nc = pl.nc;
  b.cur_pts = cur->pts;
  b.cur_nrm = cur->nrm;
  b.nscale = nscale;
  b.grid = pl.grid;
  const size_t ncells = (size_t)pl.grid.dim[0] * pl.grid.dim[1] * pl.grid.dim[2];
  b.key_bits = 1;
  while (b.key_bits < 32 && ((size_t)1 << b.key_bits) < ncells) b.key_bits++;
  b.keys = (unsigned *)(ws + pl.o_keys); b.skeys = (unsigned *)(ws + pl.o_skeys);
  b.idx = (unsigned *)(ws + pl.o_idx); b.sidx = (unsigned *)(ws + pl.o_sidx);
  b.feat6 = (float *)(ws + pl.o_feat); b.sfeat6 = (float *)(ws + pl.o_sfeat);
  b.cstart = (int *)(ws + pl.o_cstart); b.cend = (int *)(ws + pl.o_cend);
  b.temp = ws + pl.o_temp;
  b.temp_bytes = pl.temp_bytes;
  if (launch_nn_build(b, ctx->stream)) return fail(ctx, NICP_ECUDA, "nearest-neighbour index build failed");
  return NICP_OK;
}

NNQuery nn_query(nicp_ctx *ctx, const NNPlan &pl, const nicp_cloud *ref, const nicp_cloud *cur, float nscale,
                 const nicp_corr_params &cp, const float *Tg, const PairState *state) {
  char *ws = ctx->ws;
  NNQuery q{};
  q.nr = pl.nr;
  q.ref_pts = ref->pts; q.ref_nrm = ref->nrm;
  q.cur_pts = cur->pts; q.cur_nrm = cur->nrm;
  q.Tg = Tg;
  q.state = state;
  q.nscale = nscale;
  q.sq = cp.inlier_distance_threshold * cp.inlier_distance_threshold;
  q.cos_thr = cp.inlier_normal_angular_threshold;
  q.demoted = cp.demoted_to_gicp;
  q.grid = pl.grid;
  q.cstart = (const int *)(ws + pl.o_cstart); q.cend = (const int *)(ws + pl.o_cend);
  q.sfeat6 = (const float *)(ws + pl.o_sfeat); q.sidx = (const unsigned *)(ws + pl.o_sidx);
  q.match = (int *)(ws + pl.o_match);
  return q;
}
}  // namespace

extern "C" int nicp_correspond_nn(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const float T16[16],
                                  float normal_scaling, const nicp_corr_params *corr, int32_t *pairs_out,
                                  int *num_pairs) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !ref || !cur || !T16 || !corr || !num_pairs) return NICP_EINVAL;
  NNPlan pl;
  int rc = nn_plan(ctx, ref, cur, corr->inlier_distance_threshold, pl);
  if (rc) return rc;
  *num_pairs = 0;
  if (pl.nr == 0 || pl.nc == 0) return NICP_OK;
  if ((rc = nn_build(ctx, pl, cur, normal_scaling))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, 48, &pin))) return rc;
  rows12(HM4::from(T16), (float *)pin);
  cudaStream_t s = ctx->stream;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_guess, pin, 48, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  NNQuery q = nn_query(ctx, pl, ref, cur, normal_scaling, *corr, (const float *)(ctx->ws + pl.o_guess), nullptr);
  if (launch_nn_correspond(q, (int *)(ctx->ws + pl.o_flag), (int *)(ctx->ws + pl.o_pos), ctx->ws + pl.o_temp,
                           pl.temp_bytes, (int32_t *)(ctx->ws + pl.o_pairs), (int *)(ctx->ws + pl.o_np), s))
    return fail(ctx, NICP_ECUDA, "nearest-neighbour query failed");
  int K = 0;
  CK(ctx, cudaMemcpyAsync(&K, ctx->ws + pl.o_np, 4, cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  if (pairs_out && K > 0)
    CK(ctx, cudaMemcpy(pairs_out, ctx->ws + pl.o_pairs, 8 * (size_t)K, cudaMemcpyDeviceToHost));
  *num_pairs = K;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_align_nn(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const float guess16[16],
                             float normal_scaling, const nicp_corr_params *corr, const nicp_lin_params *lin,
                             const nicp_align_params *prm, nicp_align_result *out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !ref || !cur || !corr || !lin || !prm || !out) return NICP_EINVAL;
  if (prm->outer_iterations < 0 || prm->inner_iterations < 1 || prm->outer_iterations > 1000 ||
      prm->inner_iterations > 100)
    return fail(ctx, NICP_EINVAL, "iteration counts out of range");
  if (!ref->mem || !cur->mem || ref->ctx != ctx || cur->ctx != ctx)
    return fail(ctx, NICP_EINVAL, "both clouds must be built on this context");
  NNPlan pl;
  int rc = nn_plan(ctx, ref, cur, corr->inlier_distance_threshold, pl);
  if (rc) return rc;
  if ((rc = nn_build(ctx, pl, cur, normal_scaling))) return rc;
  char *ws = ctx->ws;
  cudaStream_t s = ctx->stream;
  // the pair descriptor: the pair list plays the pixel image of the list
  // kernels (1 x nr), one FP64 partial per 1024 list entries
  char *pin;
  if ((rc = pin_up(ctx, sizeof(PairDev) + 256, &pin))) return rc;
  PairDev &d = *(PairDev *)pin;
  std::memset(&d, 0, sizeof(d));
  d.ref_pts = ref->pts; d.ref_nrm = ref->nrm; d.ref_count = ref->count;
  if ((rc = cloud_ensure_omg(ctx, cur))) return rc;
  d.cur_pts = cur->pts; d.cur_nrm = cur->nrm; d.cur_omg = cur->omg; d.cur_count = cur->count;
  d.rows = 1;
  d.cols = std::max(pl.nr, 1);
  d.tile_base = 0;
  d.ref_capacity = std::max(pl.nr, 1);
  d.K[0] = d.K[4] = d.K[8] = 1.0f;
  d.partials = (double *)(ws + pl.o_part);
  d.pairs = (int32_t *)(ws + pl.o_pairs);
  d.num_pairs = (int *)(ws + pl.o_np);
  d.state = (PairState *)(ws + pl.o_st);
  double *gs = (double *)(pin + sizeof(PairDev));
  HM4 G = HM4::from(guess16);
  for (int k = 0; k < 16; k++) gs[k] = G.a[k];
  double *ro = gs + 16;
  for (int k = 0; k < 16; k++) ro[k] = (k % 5 == 0) ? 1.0 : 0.0;
  CK(ctx, cudaMemcpyAsync(ws + pl.o_pd, pin, sizeof(PairDev), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ws + pl.o_guess, gs, 256, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  const PairDev *dpd = (const PairDev *)(ws + pl.o_pd);
  LinParams lp = lin_params(*lin);
  const int xb = lin->cross_block_f32 ? kSolveCrossF32 : 0;
  launch_init_pairs(dpd, 1, (const double *)(ws + pl.o_guess), (const double *)(ws + pl.o_guess + 128), nullptr, 0,
                    s, &ctx->prof);
  NNQuery q = nn_query(ctx, pl, ref, cur, normal_scaling, *corr, nullptr, (const PairState *)(ws + pl.o_st));
  for (int i = 0; i < prm->outer_iterations; i++) {
    // correspondences with the state's T^-1 (alignernn.cpp:40-45)
    if (launch_nn_correspond(q, (int *)(ws + pl.o_flag), (int *)(ws + pl.o_pos), ws + pl.o_temp, pl.temp_bytes,
                             d.pairs, d.num_pairs, s))
      return fail(ctx, NICP_ECUDA, "nearest-neighbour query failed");
    for (int k = 0; k < prm->inner_iterations; k++) {
      launch_lin_list(dpd, 1, pl.tiles, lp, 1, 1, nullptr, s, &ctx->prof);
      launch_solve(dpd, 1, prm->lambda, ((k == prm->inner_iterations - 1) ? 1 : 0) | xb, prm->early_exit_eps, 0, s,
                   &ctx->prof);
    }
  }
  if (prm->compute_statistics) {
    launch_lin_list(dpd, 1, pl.tiles, lp, 1, 2, nullptr, s, &ctx->prof);
    launch_solve(dpd, 1, 0.0f, 4 | xb, 0.0, 1, s, &ctx->prof);
  }
  CK(ctx, cudaGetLastError());
  PairState st;
  CK(ctx, cudaMemcpyAsync(&st, ws + pl.o_st, sizeof(PairState), cudaMemcpyDeviceToHost, s));
  CK(ctx, cudaStreamSynchronize(s));
  std::memcpy(out->T, st.T, sizeof(out->T));
  out->error = st.error;
  out->inliers = st.inliers;
  out->num_correspondences = st.num_corr;
  out->outer_iterations_run = st.iterations;
  out->status = st.status;
  out->translational_ratio = out->rotational_ratio = 0;
  out->solution_valid = -1;
  std::memset(out->omega, 0, sizeof(out->omega));
  std::memset(out->mean, 0, sizeof(out->mean));
  if (prm->compute_statistics) {
    solution_statistics(st.Hstat, st.T, &out->translational_ratio, &out->rotational_ratio, out->omega, out->mean);
    out->solution_valid = !(out->rotational_ratio > prm->rotational_min_eigen_ratio ||
                            out->translational_ratio > prm->translational_min_eigen_ratio);
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ scene
// Grows a cloud's allocation to `capacity` points keeping its first n
// points (all arrays) and its counts.
static int cloud_grow(nicp_cloud *c, int capacity, int n) {
  nicp_ctx *ctx = c->ctx;
  Layout L;
  size_t o_pts = L.take(16 * (size_t)capacity), o_nrm = L.take(16 * (size_t)capacity);
  size_t o_omg = L.take(48 * (size_t)capacity);
  size_t o_eig = c->has_eig ? L.take(4 * kStatsWords * (size_t)capacity) : 0;
  size_t o_gauss = c->has_gauss ? L.take(48 * (size_t)capacity) : 0;
  size_t o_cnt = L.take(2 * sizeof(int));
  size_t P = std::max<size_t>((size_t)c->rows * c->cols, 1);
  size_t o_idx = L.take(4 * P);
  char *mem = nullptr;
  if (cudaMalloc(&mem, L.off) != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, NICP_ENOMEM, "cloud allocation failed");
  }
  cudaStream_t s = ctx->stream;
  CK(ctx, cudaMemcpyAsync(mem + o_pts, c->pts, 16 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(mem + o_nrm, c->nrm, 16 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(mem + o_omg, c->omg, 48 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  if (c->has_eig) CK(ctx, cudaMemcpyAsync(mem + o_eig, c->eig, 4 * kStatsWords * (size_t)n, cudaMemcpyDeviceToDevice, s));
  if (c->has_gauss) CK(ctx, cudaMemcpyAsync(mem + o_gauss, c->gauss, 48 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(mem + o_cnt, c->count, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaStreamSynchronize(s));
  cudaFree(c->mem);
  ctx->cloud_bytes += L.off - c->bytes;
  c->mem = mem;
  c->bytes = L.off;
  c->capacity = capacity;
  c->pts = (float4 *)(mem + o_pts);
  c->nrm = (float4 *)(mem + o_nrm);
  c->omg = (float4 *)(mem + o_omg);
  c->eig = c->has_eig ? (float *)(mem + o_eig) : nullptr;
  c->gauss = c->has_gauss ? (float4 *)(mem + o_gauss) : nullptr;
  c->count = (int *)(mem + o_cnt);
  c->index = (int32_t *)(mem + o_idx);
  return NICP_OK;
}

static int cloud_counts2(nicp_cloud *c, int out[2]) {
  out[0] = out[1] = 0;
  if (!c->mem) return NICP_OK;
  nicp_ctx *ctx = c->ctx;
  char *pin;
  int rc = pin_down(ctx, 2 * sizeof(int), &pin);
  if (rc) return rc;
  CK(ctx, cudaMemcpyAsync(pin, c->count, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, pin, 2 * sizeof(int));
  return NICP_OK;
}

extern "C" int nicp_cloud_add(nicp_cloud *dst, nicp_cloud *src, const float T16[16]) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(dst ? dst->ctx : nullptr);
  if (!dst || !src || dst == src || dst->ctx != src->ctx) return NICP_EINVAL;
  nicp_ctx *ctx = dst->ctx;
  int rc = T16 ? nicp_cloud_transform(src, T16) : NICP_OK;  // Cloud::add moves the added cloud itself
  if (rc) return rc;
  int cd[2], cs[2];
  if ((rc = cloud_counts2(dst, cd)) || (rc = cloud_counts2(src, cs))) return rc;
  const int nd = cd[0], ns = cs[0];
  if (ns == 0) return NICP_OK;
  const bool empty = nd == 0;
  const bool eig = src->eig_valid && (empty || dst->eig_valid);
  const bool gauss = src->gauss_valid && (empty || dst->gauss_valid);
  const bool structured = src->omega_structured &&
                          (empty || (dst->omega_structured && std::memcmp(dst->omd, src->omd, sizeof(src->omd)) == 0));
  if (empty) {
    if ((rc = cloud_reserve(dst, ns, src->rows, src->cols, eig, gauss))) return rc;
  } else if (dst->capacity < nd + ns || (eig && !dst->has_eig) || (gauss && !dst->has_gauss)) {
    dst->has_eig = dst->has_eig && eig;
    dst->has_gauss = dst->has_gauss && gauss;
    int cap = std::max(nd + ns, dst->capacity + dst->capacity / 2);
    if ((rc = cloud_grow(dst, cap, nd))) return rc;
  }
  cudaStream_t s = ctx->stream;
  // the result keeps an implicit Omega when both parts have one (and the same
  // parameters); otherwise both parts' matrices are written out first
  const bool implicit = structured && !src->omg_valid && (empty || !dst->omg_valid);
  if (!implicit) {
    if ((rc = cloud_ensure_omg(ctx, src))) return rc;
    if (!empty && (rc = cloud_ensure_omg(ctx, dst))) return rc;
  }
  CK(ctx, cudaMemcpyAsync(dst->pts + nd, src->pts, 16 * (size_t)ns, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(dst->nrm + nd, src->nrm, 16 * (size_t)ns, cudaMemcpyDeviceToDevice, s));
  if (!implicit)
    CK(ctx, cudaMemcpyAsync(dst->omg + 3 * (size_t)nd, src->omg, 48 * (size_t)ns, cudaMemcpyDeviceToDevice, s));
  if (eig && dst->eig)
    CK(ctx, cudaMemcpyAsync(dst->eig + kStatsWords * (size_t)nd, src->eig, 4 * kStatsWords * (size_t)ns,
                            cudaMemcpyDeviceToDevice, s));
  if (gauss && dst->gauss)
    CK(ctx, cudaMemcpyAsync(dst->gauss + 3 * (size_t)nd, src->gauss, 48 * (size_t)ns, cudaMemcpyDeviceToDevice, s));
  char *pin;
  if ((rc = pin_up(ctx, 2 * sizeof(int), &pin))) return rc;
  int *cnt = (int *)pin;
  cnt[0] = nd + ns;
  cnt[1] = cd[1] + cs[1];
  CK(ctx, cudaMemcpyAsync(dst->count, cnt, 2 * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaStreamSynchronize(s));
  dst->eig_valid = eig && dst->eig;
  dst->gauss_valid = gauss && dst->gauss;
  dst->omega_structured = structured;
  dst->omg_valid = !implicit;
  if (empty) std::memcpy(dst->omd, src->omd, sizeof(src->omd));
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_merge(nicp_ctx *ctx, nicp_cloud *cloud, const nicp_camera *cam, const float T16[16],
                          float distance_threshold, float max_point_depth, int *removed) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  if (!ctx || !cloud || !cam || !valid_camera(cam) || cloud->ctx != ctx) return NICP_EINVAL;
  if (removed) *removed = 0;
  int cnt[2];
  int rc = cloud_counts2(cloud, cnt);
  if (rc) return rc;
  const int n = cnt[0];
  if (n == 0) return NICP_OK;
  if (!cloud->gauss_valid)
    return fail(ctx, NICP_ESTATE, "merge needs the cloud's Gaussians: build it with keep_gaussians");
  const size_t P = (size_t)cam_rows(*cam) * cam_cols(*cam);
  const size_t N = (size_t)n;
  Layout E;  // inside the plan's extra region
  size_t o_depth = E.take(4 * P);
  size_t o_int[7];
  for (int k = 0; k < 7; k++) o_int[k] = E.take(4 * N);
  size_t scan_bytes = merge_scan_temp_bytes(n);
  size_t o_scan = E.take(scan_bytes);
  size_t o_pts = E.take(16 * N), o_nrm = E.take(16 * N), o_omg = E.take(48 * N);
  size_t o_eig = E.take(cloud->eig_valid ? 4 * kStatsWords * N : 16), o_gauss = E.take(48 * N), o_cnt = E.take(8);
  PairPlan pl;
  const nicp_cloud *cc = cloud;
  if ((rc = plan_pairs(ctx, 1, cam, &cc, false, false, pl, E.off))) return rc;
  char *pin;
  if ((rc = pin_up(ctx, sizeof(PairDev) + 48, &pin))) return rc;
  fill_pairs(ctx, pl, cam, &cc, &cc, (PairDev *)pin);
  HM4 KRt, iKRt;
  projector_matrices(*cam, HM4::from(T16), KRt, iKRt);
  float *k12 = (float *)(pin + sizeof(PairDev));
  rows12(KRt, k12);
  cudaStream_t s = ctx->stream;
  char *ex = ctx->ws + pl.o_extra;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_pairs, pin, sizeof(PairDev), cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_krt, k12, 48, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  CK(ctx, cudaMemsetAsync(ctx->ws + pl.o_zbuf, 0xff, pl.zbuf_bytes, s));
  const PairDev *dpd = (const PairDev *)(ctx->ws + pl.o_pairs);
  // the serial z-buffer of PinholePointProjector::project, all points kept
  launch_zbuffer(dpd, 1, pl.max_pt_tiles, 0, (const float *)(ctx->ws + pl.o_krt), kZbufDefaultPPT, s, &ctx->prof);
  launch_resolve(dpd, 1, pl.max_tiles, 0, (float *)(ex + o_depth), 0, s, &ctx->prof);
  MergeArgs a{};
  a.n = n;
  a.count = cloud->count;
  a.pts = cloud->pts;
  a.nrm = cloud->nrm;
  a.omg = cloud->omg;
  a.eig = cloud->eig_valid ? cloud->eig : nullptr;
  a.gauss = cloud->gauss;
  a.KRt12 = (const float *)(ctx->ws + pl.o_krt);
  a.rows = cam_rows(*cam);
  a.cols = cam_cols(*cam);
  a.min_d = cam->min_distance;
  a.max_d = cam->max_distance;
  a.max_depth = max_point_depth;
  a.dthr = distance_threshold;
  a.index = (const int32_t *)(ctx->ws + pl.o_cur[0]);
  a.depth = (const float *)(ex + o_depth);
  int *ints[7];
  for (int k = 0; k < 7; k++) ints[k] = (int *)(ex + o_int[k]);
  a.tgt = ints[0]; a.cnt = ints[1]; a.off = ints[2]; a.fill = ints[3]; a.list = ints[4]; a.keep = ints[5];
  a.pos = ints[6];
  a.scan_temp = ex + o_scan;
  a.scan_temp_bytes = scan_bytes;
  a.o_pts = (float4 *)(ex + o_pts);
  a.o_nrm = (float4 *)(ex + o_nrm);
  a.o_omg = (float4 *)(ex + o_omg);
  a.o_eig = cloud->eig_valid ? (float *)(ex + o_eig) : nullptr;
  a.o_gauss = (float4 *)(ex + o_gauss);
  a.out_count = (int *)(ex + o_cnt);
  if (launch_merge(a, s)) {
    cudaError_t e = cudaGetLastError();
    return fail(ctx, NICP_ECUDA, std::string("merge: ") + cudaGetErrorString(e));
  }
  // the compacted cloud back in place
  CK(ctx, cudaMemcpyAsync(cloud->pts, a.o_pts, 16 * N, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(cloud->nrm, a.o_nrm, 16 * N, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(cloud->omg, a.o_omg, 48 * N, cudaMemcpyDeviceToDevice, s));
  if (a.o_eig) CK(ctx, cudaMemcpyAsync(cloud->eig, a.o_eig, 4 * kStatsWords * N, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(cloud->gauss, a.o_gauss, 48 * N, cudaMemcpyDeviceToDevice, s));
  CK(ctx, cudaMemcpyAsync(cloud->count, a.out_count, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s));
  int after[2];
  if ((rc = cloud_counts2(cloud, after))) return rc;
  if (removed) *removed = n - after[0];
  return NICP_OK;
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ aligner
namespace {
struct AlignCall {
  int n;
  const nicp_cloud *const *refs;
  const nicp_cloud *const *curs;
  const nicp_camera *cams;
  const float *guesses;      // n*16 or null
  const float *ref_offsets;  // n*16 or null
  const float *cur_offsets;  // n*16 or null
  const nicp_corr_params *corr;
  const nicp_lin_params *lin;
  const nicp_align_params *prm;
  bool graph;
  bool foreign_clouds = false;  // clouds of another context on the same device (the server's workers)
};
}  // namespace

// Enqueues the whole Gauss-Newton loop for the planned pairs.
static void enqueue_loop(nicp_ctx *ctx, const PairPlan &pl, const AlignCall &a) {
  cudaStream_t s = ctx->stream;
  const PairDev *dpd = (const PairDev *)(ctx->ws + pl.o_pairs);
  CorrParams cp = corr_params(*a.corr);
  LinParams lp = lin_params(*a.lin);
  const nicp_align_params &p = *a.prm;
  int outer = p.outer_iterations, inner = p.inner_iterations;
  bool stats = p.compute_statistics != 0;
  const int xb = a.lin->cross_block_f32 ? kSolveCrossF32 : 0;
  cudaMemsetAsync(ctx->ws + pl.o_zbuf, 0xff, pl.zbuf_bytes, s);
  int *tile_pair = (int *)(ctx->ws + pl.o_tile_pair);
  launch_init_pairs(dpd, pl.n, (const double *)(ctx->ws + pl.o_guess), (const double *)(ctx->ws + pl.o_roff),
                    tile_pair, pl.max_tiles, s, &ctx->prof);
  // current cloud, seen from its sensor offset, projected once (alignerprojective.cpp:36-39)
  const nicp_ctx::Launch &L = ctx->launch;
  launch_zbuffer(dpd, pl.n, pl.max_pt_tiles, 0, (const float *)(ctx->ws + pl.o_krt), L.zb_ppt, s, &ctx->prof);
  // outside list (parity) mode, current pixels whose point has no normal are
  // dropped from the index image: the gates would reject them anyway
  launch_resolve(dpd, pl.n, pl.max_tiles, 0, nullptr, (pl.list_mode || cp.demoted) ? 0 : 1, s, &ctx->prof);
  for (int i = 0; i < outer; i++) {
    launch_zbuffer(dpd, pl.n, pl.max_pt_tiles, 1, nullptr, L.zb_ppt, s, &ctx->prof);
    if (pl.list_mode) {
      launch_resolve(dpd, pl.n, pl.max_tiles, 1, nullptr, 0, s, &ctx->prof);
      launch_corr_list(dpd, pl.n, pl.total_tiles, cp, 1, nullptr, s, &ctx->prof);
      for (int k = 0; k < inner; k++) {
        launch_lin_list(dpd, pl.n, pl.total_tiles, lp, std::max(1, a.corr->parity_threads), 1, nullptr, s, &ctx->prof);
        launch_solve(dpd, pl.n, p.lambda, ((k == inner - 1) ? 1 : 0) | xb, p.early_exit_eps, 0, s, &ctx->prof);
      }
    } else {
      for (int k = 0; k < inner; k++) {
        int flags = (k == 0) ? (1 | 2 | (pl.keep_ref ? 4 : 0)) : 0;
        launch_corr_lin(dpd, pl.n, pl.total_tiles, cp, lp, flags, pl.structured, L.corr_ctas, tile_pair, s,
                        &ctx->prof);
        launch_solve(dpd, pl.n, p.lambda, ((k == inner - 1) ? 1 : 0) | xb, p.early_exit_eps, 0, s, &ctx->prof);
      }
    }
  }
  if (stats) {
    // Aligner::_computeStatistics: one more linearization at the final pose
    // with the last correspondences (aligner.cpp:90-95)
    if (pl.list_mode)
      launch_lin_list(dpd, pl.n, pl.total_tiles, lp, std::max(1, a.corr->parity_threads), 2, nullptr, s, &ctx->prof);
    else
      launch_corr_lin(dpd, pl.n, pl.total_tiles, cp, lp, 8, pl.structured, L.corr_ctas, tile_pair, s, &ctx->prof);
    launch_solve(dpd, pl.n, 0.0f, 4 | xb, 0.0, 1, s, &ctx->prof);
  }
}

static std::string graph_key(nicp_ctx *ctx, const PairPlan &pl, const AlignCall &a) {
  std::string k;
  auto put = [&](const void *p, size_t n) { k.append((const char *)p, n); };
  put(&ctx->ws, sizeof(ctx->ws));
  put(&pl.n, sizeof(int));
  put(&pl.keep_ref, 1);
  put(&pl.list_mode, 1);
  put(&pl.structured, 1);
  put(&pl.total_tiles, sizeof(int));
  put(&pl.max_pt_tiles, sizeof(int));
  put(&pl.max_tiles, sizeof(int));
  put(&pl.zbuf_bytes, sizeof(size_t));
  put(a.corr, sizeof(*a.corr));
  put(a.lin, sizeof(*a.lin));
  put(a.prm, sizeof(*a.prm));
  bool pe = ctx->prof.enabled;
  put(&pe, 1);
  put(&ctx->launch, sizeof(ctx->launch));
  return k;
}

// The resolution mix of a batch: sorted (rows, cols, count) plus the loop
// shape; the autotuner keeps one choice per key.
static std::string tune_key(const PairPlan &pl, const AlignCall &a) {
  std::map<std::pair<int, int>, int> hist;
  for (int i = 0; i < a.n; i++) hist[{cam_rows(a.cams[i]), cam_cols(a.cams[i])}]++;
  std::string k;
  for (auto &h : hist) k += std::to_string(h.first.first) + "x" + std::to_string(h.first.second) + ":" +
                           std::to_string(h.second) + " ";
  k += "o" + std::to_string(a.prm->outer_iterations) + "i" + std::to_string(a.prm->inner_iterations) +
       (pl.structured ? "s" : "g") + (a.prm->compute_statistics ? "t" : "");
  return k;
}

// Z-buffer points per thread unless the autotuner picked: once the
// projection grid spans about two waves of its 128-thread CTAs (16 per SM),
// more independent loads and atomics per thread pay (the 199-pair 640x480
// sequence: 8 points per thread, 3 % faster than 4); below that (one or a
// few pairs) more threads do.
static int default_zb_ppt(const nicp_ctx *ctx, const PairPlan &pl) {
  const long long ctas = (long long)pl.max_pt_tiles * pl.n;
  return ctas >= 16ll * ctx->sm_count ? kZbufWidePPT : kZbufDefaultPPT;
}

// Times the loop with each candidate launch shape (direct launches, CUDA
// events on the context stream) and keeps the fastest: z-buffer points per
// thread first, then the fused kernel's CTAs per SM.  The loop re-initialises
// every pair from its guess, so trials leave no trace in the results.
static int autotune_loop(nicp_ctx *ctx, const PairPlan &pl, const AlignCall &a, nicp_ctx::Launch *best) {
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  CK(ctx, cudaEventCreate(&e0));
  CK(ctx, cudaEventCreate(&e1));
  bool prof = ctx->prof.enabled;
  ctx->prof.enabled = false;
  std::vector<float> times;
  auto trial = [&](const nicp_ctx::Launch &c, float *ms) -> int {
    ctx->launch = c;
    CK(ctx, cudaEventRecord(e0, s));
    enqueue_loop(ctx, pl, a);
    CK(ctx, cudaEventRecord(e1, s));
    CK(ctx, cudaEventSynchronize(e1));
    CK(ctx, cudaEventElapsedTime(ms, e0, e1));
    times.push_back(*ms);
    return NICP_OK;
  };
  const nicp_ctx::Launch cur = ctx->launch;  // the default shape for this call
  float ms = 0, best_ms = 0;
  int rc = trial(cur, &ms);  // warm-up (module load, caches)
  if (!rc) rc = trial(cur, &best_ms);
  *best = cur;
  const int ppts[] = {1, 2, 4, 8};  // the default is among them: skipped
  for (int i = 0; i < 4 && !rc; i++) {
    if (ppts[i] == cur.zb_ppt) continue;
    nicp_ctx::Launch c = *best;
    c.zb_ppt = ppts[i];
    if (!(rc = trial(c, &ms)) && ms < best_ms) { best_ms = ms; *best = c; }
  }
  const int ctas[] = {2, 3};  // fused kernel CTAs (128 threads) per SM
  for (int i = 0; i < 2 && !rc; i++) {
    nicp_ctx::Launch c = *best;
    c.corr_ctas = ctas[i];
    if (!(rc = trial(c, &ms)) && ms < best_ms) { best_ms = ms; *best = c; }
  }
  ctx->prof.enabled = prof;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->tune_ms[tune_key(pl, a)] = times;
  return rc;
}

static int align_impl(nicp_ctx *ctx, const AlignCall &a, nicp_align_result *out) {
  if (!ctx || a.n < 0 || !a.cams || !a.corr || !a.lin || !a.prm || (a.n > 0 && (!a.refs || !a.curs || !out)))
    return NICP_EINVAL;
  if (a.n == 0) return NICP_OK;
  const nicp_align_params &p = *a.prm;
  if (p.outer_iterations < 0 || p.inner_iterations < 1 || p.outer_iterations > 1000 || p.inner_iterations > 100)
    return fail(ctx, NICP_EINVAL, "iteration counts out of range");
  for (int i = 0; i < a.n; i++) {
    if (!a.refs[i] || !a.curs[i] || !a.refs[i]->mem || !a.curs[i]->mem)
      return fail(ctx, NICP_EINVAL, "pair " + std::to_string(i) + " has an empty cloud");
    if (!a.foreign_clouds && (a.refs[i]->ctx != ctx || a.curs[i]->ctx != ctx))
      return fail(ctx, NICP_EINVAL, "cloud of another context");
  }
  if (a.corr->row_search_region < 0 || a.corr->col_search_region < 0 || a.corr->row_search_region > 16 ||
      a.corr->col_search_region > 16)
    return fail(ctx, NICP_EINVAL, "search regions must lie in [0, 16]");
  // windowed correspondences and the reference's partition drops run on
  // the correspondence-list kernels
  bool list_mode = a.corr->parity_threads > 1 || a.corr->row_search_region > 0 || a.corr->col_search_region > 0;
  bool keep_ref = p.inner_iterations > 1 || p.compute_statistics;
  // point tiles cover the larger of the two clouds: the current cloud is
  // projected once with the same grid as the reference cloud
  std::vector<const nicp_cloud *> big(a.n);
  for (int j = 0; j < a.n; j++) big[j] = (a.curs[j]->capacity > a.refs[j]->capacity) ? a.curs[j] : a.refs[j];
  PairPlan pl;
  int rc;
  if ((rc = plan_pairs(ctx, a.n, a.cams, big.data(), keep_ref, list_mode, pl))) return rc;
  pl.structured = !list_mode;
  for (int i = 0; i < a.n && pl.structured; i++) pl.structured = a.curs[i] && a.curs[i]->omega_structured;
  // the list linearizer reads the current clouds' matrices (the fused kernel
  // rebuilds a structured cloud's Omega itself)
  for (int i = 0; i < a.n && list_mode; i++)
    if ((rc = cloud_ensure_omg(ctx, a.curs[i]))) return rc;
  size_t up = sizeof(PairDev) * a.n + 48 * (size_t)a.n + 256 * (size_t)a.n;
  char *pin;
  if ((rc = pin_up(ctx, up, &pin))) return rc;
  PairDev *pd = (PairDev *)pin;
  fill_pairs(ctx, pl, a.cams, big.data(), a.curs, pd);
  for (int i = 0; i < a.n; i++) {
    pd[i].ref_pts = a.refs[i]->pts;
    pd[i].ref_nrm = a.refs[i]->nrm;
    pd[i].ref_count = a.refs[i]->count;
  }
  float *krt = (float *)(pin + sizeof(PairDev) * a.n);
  double *gs = (double *)(pin + sizeof(PairDev) * a.n + 48 * (size_t)a.n);
  double *ro = gs + 16 * (size_t)a.n;
  for (int i = 0; i < a.n; i++) {
    HM4 KRt, iKRt;
    projector_matrices(a.cams[i], HM4::from(a.cur_offsets ? a.cur_offsets + 16 * i : nullptr), KRt, iKRt);
    rows12(KRt, krt + 12 * i);
    HM4 G = HM4::from(a.guesses ? a.guesses + 16 * i : nullptr);
    HM4 R = HM4::from(a.ref_offsets ? a.ref_offsets + 16 * i : nullptr);
    for (int k = 0; k < 16; k++) {
      gs[16 * i + k] = G.a[k];
      ro[16 * i + k] = R.a[k];
    }
  }
  cudaStream_t s = ctx->stream;
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_pairs, pd, sizeof(PairDev) * a.n, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_krt, krt, 48 * (size_t)a.n, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_guess, gs, 128 * (size_t)a.n, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaMemcpyAsync(ctx->ws + pl.o_roff, ro, 128 * (size_t)a.n, cudaMemcpyHostToDevice, s));
  CK(ctx, cudaEventRecord(ctx->pin_up_ev, s));
  ctx->h2d_bytes += (sizeof(PairDev) + 48 + 256) * (unsigned long long)a.n;
  ctx->launch = nicp_ctx::Launch();
  ctx->launch.zb_ppt = default_zb_ppt(ctx, pl);
  if (ctx->autotune && !list_mode) {
    std::string tk = tune_key(pl, a);
    auto it = ctx->tuned.find(tk);
    if (it == ctx->tuned.end()) {
      nicp_ctx::Launch best;
      if ((rc = autotune_loop(ctx, pl, a, &best))) return rc;
      it = ctx->tuned.emplace(tk, best).first;
    }
    ctx->launch = it->second;
  }
  // Events recorded while a stream is captured are capture-internal and
  // cannot be timed after a replay, so a profiled call launches the same
  // kernels directly.
  if (a.graph && !ctx->prof.enabled) {
    std::string key = graph_key(ctx, pl, a);
    GraphEntry *ge = nullptr;
    for (auto &g : ctx->graphs)
      if (g.key == key) ge = &g;
    if (!ge) {
      GraphEntry g;
      g.key = key;
      size_t rec0 = ctx->prof.recs.size();
      unsigned long long l0 = ctx->prof.launches;
      cudaGraph_t graph;
      CK(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      ctx->prof.capturing = true;
      enqueue_loop(ctx, pl, a);
      ctx->prof.capturing = false;
      cudaError_t e = cudaStreamEndCapture(s, &graph);
      if (e != cudaSuccess) return fail(ctx, NICP_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(ctx, NICP_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      g.kernels = ctx->prof.launches - l0;
      ctx->prof.launches = l0;
      g.recs.assign(ctx->prof.recs.begin() + rec0, ctx->prof.recs.end());
      ctx->prof.recs.resize(rec0);
      if (ctx->graphs.size() >= 16) {
        cudaGraphExecDestroy(ctx->graphs.front().exec);
        ctx->graphs.erase(ctx->graphs.begin());
      }
      ctx->graphs.push_back(g);
      ge = &ctx->graphs.back();
    }
    CK(ctx, cudaGraphLaunch(ge->exec, s));
    ctx->prof.launches += ge->kernels;
    if (ctx->prof.enabled) ctx->prof.recs.insert(ctx->prof.recs.end(), ge->recs.begin(), ge->recs.end());
  } else {
    enqueue_loop(ctx, pl, a);
  }
  CK(ctx, cudaGetLastError());
  char *res;
  if ((rc = pin_down(ctx, sizeof(PairState) * a.n, &res))) return rc;
  CK(ctx, cudaMemcpyAsync(res, ctx->ws + pl.o_states, sizeof(PairState) * a.n, cudaMemcpyDeviceToHost, s));
  ctx->d2h_bytes += sizeof(PairState) * (unsigned long long)a.n;
  CK(ctx, cudaStreamSynchronize(s));
  const PairState *st = (const PairState *)res;
  for (int i = 0; i < a.n; i++) {
    nicp_align_result &r = out[i];
    std::memcpy(r.T, st[i].T, sizeof(r.T));
    r.error = st[i].error;
    r.inliers = st[i].inliers;
    r.num_correspondences = st[i].num_corr;
    r.outer_iterations_run = st[i].iterations;
    r.status = st[i].status;
    r.translational_ratio = r.rotational_ratio = 0;
    r.solution_valid = -1;
    std::memset(r.omega, 0, sizeof(r.omega));
    std::memset(r.mean, 0, sizeof(r.mean));
    if (p.compute_statistics) {
      solution_statistics(st[i].Hstat, st[i].T, &r.translational_ratio, &r.rotational_ratio, r.omega, r.mean);
      r.solution_valid = !(r.rotational_ratio > p.rotational_min_eigen_ratio ||
                           r.translational_ratio > p.translational_min_eigen_ratio);
    }
  }
  return NICP_OK;
}

extern "C" int nicp_align(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const nicp_camera *cam,
                          const float guess16[16], const float ref_offset16[16], const float cur_offset16[16],
                          const nicp_corr_params *corr, const nicp_lin_params *lin, const nicp_align_params *prm,
                          nicp_align_result *out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  // replayed from a cached CUDA graph like a batch: the pair descriptors are
  // uploaded per call, so one graph serves every pair of the same shape
  AlignCall a{1, &ref, &cur, cam, guess16, ref_offset16, cur_offset16, corr, lin, prm, true};
  return align_impl(ctx, a, out);
  NICP_ABI_CATCH
}

extern "C" int nicp_align_batch(nicp_ctx *ctx, int n, const nicp_cloud *const *refs, const nicp_cloud *const *curs,
                                const nicp_camera *cams, const float *guesses, const nicp_corr_params *corr,
                                const nicp_lin_params *lin, const nicp_align_params *prm, nicp_align_result *out) {
  NICP_ABI_TRY
  NICP_ON_DEVICE(ctx);
  AlignCall a{n, refs, curs, cams, guesses, nullptr, nullptr, corr, lin, prm, true};
  return align_impl(ctx, a, out);
  NICP_ABI_CATCH
}

// ------------------------------------------------------------------ internal hooks of the server
namespace nicp {
namespace internal {

// Makes the context's device current on the calling thread: a thread that
// did not create the context starts on device 0.
int ctx_make_current(nicp_ctx *ctx) {
  if (!ctx) return NICP_EINVAL;
  return cudaSetDevice(ctx->device) == cudaSuccess ? NICP_OK : NICP_ECUDA;
}

// Batch build into clouds that may belong to another context of this device.
int build_batch(nicp_ctx *ctx, int n, const uint16_t *const *depth, const int *rows, const int *cols,
                const nicp_camera *cams, const nicp_cloud_params *prm, nicp_cloud *const *out) {
  if (!ctx || n < 0) return NICP_EINVAL;
  NICP_ON_DEVICE(ctx);
  std::vector<FrameIn> f(n);
  for (int i = 0; i < n; i++) f[i] = FrameIn{depth[i], true, false, 0, rows[i], cols[i], nullptr};
  return build_frames(ctx, n, f.data(), cams, prm, out, false);
}

// Batch align with direct launches (batch shapes vary from call to call).
int align_batch(nicp_ctx *ctx, int n, const nicp_cloud *const *refs, const nicp_cloud *const *curs,
                const nicp_camera *cams, const float *guesses, const nicp_corr_params *corr,
                const nicp_lin_params *lin, const nicp_align_params *prm, nicp_align_result *out) {
  NICP_ON_DEVICE(ctx);
  AlignCall a{n, refs, curs, cams, guesses, nullptr, nullptr, corr, lin, prm, false, true};
  return align_impl(ctx, a, out);
}

// Counts of points with a normal of n clouds, with one synchronisation.
int cloud_normal_counts(nicp_ctx *ctx, int n, const nicp_cloud *const *c, int *out) {
  NICP_ON_DEVICE(ctx);
  char *pin;
  int rc = pin_down(ctx, sizeof(int) * (size_t)std::max(n, 1), &pin);
  if (rc) return rc;
  for (int i = 0; i < n; i++) {
    if (!c[i]->mem) { reinterpret_cast<int *>(pin)[i] = 0; continue; }
    CK(ctx, cudaMemcpyAsync(pin + sizeof(int) * i, c[i]->count + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, pin, sizeof(int) * (size_t)n);
  return NICP_OK;
}

size_t cloud_bytes(const nicp_cloud *c) { return c ? c->bytes : 0; }

// Host copies of a cloud (for the .nicp writer): points (w reported as 1),
// normals + curvature, and the kStatsWords-word Stats records when kept.
int cloud_host_arrays(nicp_cloud *c, std::vector<float> &pts4, std::vector<float> &nrm4, std::vector<float> &stats,
                      bool &has_stats) {
  int n = 0;
  int rc = nicp_cloud_size(c, &n);
  if (rc) return rc;
  nicp_ctx *ctx = c->ctx;
  NICP_ON_DEVICE(ctx);
  pts4.resize(4 * (size_t)n);
  nrm4.resize(4 * (size_t)n);
  has_stats = c->eig_valid;
  stats.assign(has_stats ? kStatsWords * (size_t)n : 0, 0.0f);
  if (n == 0) return NICP_OK;
  CK(ctx, cudaMemcpyAsync(pts4.data(), c->pts, 16 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaMemcpyAsync(nrm4.data(), c->nrm, 16 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  if (has_stats)
    CK(ctx, cudaMemcpyAsync(stats.data(), c->eig, 4 * kStatsWords * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; i++) pts4[4 * (size_t)i + 3] = 1.0f;
  return NICP_OK;
}

// Fills a cloud from host arrays (the .nicp reader): points with their w
// codes, normals + curvature, information matrices (12 floats per point, the
// omg layout), Stats records; `normals` points have a normal.
int cloud_set_host_arrays(nicp_cloud *c, int n, const float *pts4, const float *nrm4, const float *omg12,
                          const float *stats, int normals, bool structured, const float omd[8]) {
  nicp_ctx *ctx = c->ctx;
  NICP_ON_DEVICE(ctx);
  int rc = cloud_reserve(c, n, c->rows, c->cols, true, false);
  if (rc) return rc;
  if (n > 0) {
    CK(ctx, cudaMemcpyAsync(c->pts, pts4, 16 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(c->nrm, nrm4, 16 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(c->omg, omg12, 48 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(c->eig, stats, 4 * kStatsWords * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
  }
  int counts[2] = {n, normals};
  CK(ctx, cudaMemcpyAsync(c->count, counts, sizeof(counts), cudaMemcpyHostToDevice, ctx->stream));
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  c->eig_valid = true;
  c->gauss_valid = false;
  c->omega_structured = structured;
  c->omg_valid = true;
  std::memcpy(c->omd, omd, sizeof(c->omd));
  return NICP_OK;
}

}  // namespace internal
}  // namespace nicp
