// capi.cu -- the extern "C" boundary of libsdfgpu.so (declared in include/sdfgpu.h).
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "common.cuh"

namespace sdfgpu {

static thread_local std::string g_create_error;

int upload_directions(sdfgpu_ctx* ctx, const double* dirs);

int fail(sdfgpu_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  else g_create_error = msg;
  return code;
}

int scratch(sdfgpu_ctx* ctx, const char* name, size_t bytes, void** out) {
  DevBuf& b = ctx->ns.empty() ? ctx->bufs[name] : ctx->bufs[ctx->ns + name];
  if (b.cap < bytes) {
    if (b.p) {
      cudaError_t e = cudaFree(b.p);
      b.p = nullptr;
      b.cap = 0;
      if (e != cudaSuccess) return fail(ctx, SDFGPU_ERR_CUDA, std::string("cudaFree: ") + cudaGetErrorString(e));
    }
    size_t want = bytes + bytes / 8;  // headroom for slowly growing sizes
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
      b.p = nullptr;
      cudaGetLastError();
      return fail(ctx, SDFGPU_ERR_OUT_OF_MEMORY,
                  std::string("device allocation of ") + std::to_string(want) + " bytes for '" + name + "' failed: " +
                      cudaGetErrorString(e));
    }
    b.cap = want;
  }
  *out = b.p;
  return 0;
}

// ---- host arithmetic shared with the reference's Julia semantics ----------------------------
namespace {

double norm3_host(double x, double y, double z) {  // generic_norm2 for length 3
  const double ax = std::fabs(x), ay = std::fabs(y), az = std::fabs(z);
  double m;
  if (std::isnan(ax) || std::isnan(ay) || std::isnan(az)) m = std::numeric_limits<double>::quiet_NaN();
  else m = std::max(ax, std::max(ay, az));
  if (m == 0.0 || std::isinf(m)) return m;
  if (std::isfinite(3.0 * m * m) && (m * m) != 0.0) {
    double s = x * x;
    s = s + y * y;
    s = s + z * z;
    return std::sqrt(s);
  }
  double s = (ax / m) * (ax / m);
  s = s + (ay / m) * (ay / m);
  s = s + (az / m) * (az / m);
  return m * std::sqrt(s);
}

// generate_ray_directions_prioritized (RaycastingSignDetection.jl:162-227).
void host_directions(double D[36][3]) {
  const double axes[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
  const double face[12][3] = {{1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1}, {1, 0, -1},
                              {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
  const double body[8][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {1, -1, -1},
                             {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
  int r = 0;
  auto put = [&](const double* v) {  // normalize: multiply by inv(norm)
    const double inv = 1.0 / norm3_host(v[0], v[1], v[2]);
    D[r][0] = v[0] * inv;
    D[r][1] = v[1] * inv;
    D[r][2] = v[2] * inv;
    ++r;
  };
  for (auto& v : axes) put(v);
  for (auto& v : face) put(v);
  for (auto& v : body) put(v);
  const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
  const double two_pi = 2.0 * 3.14159265358979323846;
  for (int i = 1; i <= 10; ++i) {
    const double theta = two_pi * std::fmod((double)i * phi, 1.0);
    const double z = 1.0 - 2.0 * ((double)i / 10.0);
    const double rr = std::sqrt(1.0 - z * z);
    D[r][0] = rr * std::cos(theta);
    D[r][1] = rr * std::sin(theta);
    D[r][2] = z;
    ++r;
  }
}

int grid_core(const double xmin[3], const double xmax[3], int64_t n_max, int64_t margin, double origin[3],
              double amax[3], int64_t N[3], double* h, int64_t* ngp) {
  if (n_max <= 0 || margin < 0) return SDFGPU_ERR_INVALID_ARGUMENT;
  double ext = xmax[0] - xmin[0];
  for (int a = 1; a < 3; ++a) ext = std::max(ext, xmax[a] - xmin[a]);
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(xmin[a]) || !std::isfinite(xmax[a])) return SDFGPU_ERR_INVALID_ARGUMENT;
  if (!(ext > 0.0)) return SDFGPU_ERR_INVALID_ARGUMENT;
  const double cs = ext / (double)n_max;  // maximum(AABB_max .- AABB_min) ./ N_max
  int64_t prod = 1;
  for (int a = 0; a < 3; ++a) {
    const double lo = xmin[a] - (double)margin * cs;
    const double hi = xmax[a] + (double)margin * cs;
    const double q = std::ceil((hi - lo) / cs);
    if (!std::isfinite(q) || q < 0 || q > 4.0e9) return SDFGPU_ERR_INVALID_ARGUMENT;
    N[a] = (int64_t)q;
    origin[a] = lo;
    amax[a] = lo + (double)N[a] * cs;  // AABB_min + N .* cell_size
    prod *= (N[a] + 1);
  }
  *h = cs;
  *ngp = prod;
  return 0;
}

}  // namespace

int make_grid(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], GridP& g, int64_t k0,
              int64_t k1) {
  if (!origin || !N) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "origin and N must not be NULL");
  if (!(h > 0.0) || !std::isfinite(h)) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "cell size must be finite and > 0");
  for (int a = 0; a < 3; ++a) {
    if (N[a] < 0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "N must be >= 0");
    if (!std::isfinite(origin[a])) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "origin must be finite");
  }
  if (k1 < 0) {
    k0 = 0;
    k1 = N[2];
  }
  if (k0 < 0 || k1 < k0 || k1 > N[2])
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "z layers must satisfy 0 <= k0 <= k1 <= N[2]");
  const int64_t nloc[3] = {N[0], N[1], k1 - k0};
  double ngp = 1.0;
  for (int a = 0; a < 3; ++a) ngp *= (double)(nloc[a] + 1);
  if (ngp > 2147483647.0)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "grid has more than 2^31-1 nodes (split it into z slabs)");
  const MeshDev& M = ctx->mesh;
  g.k0 = k0;
  for (int a = 0; a < 3; ++a) {
    g.o[a] = origin[a];
    g.N[a] = nloc[a];
    g.n[a] = nloc[a] + 1;
    g.center[a] = M.center[a];
    g.t[a] = ctx->tile[a];
    g.nt[a] = cdiv(g.n[a], g.t[a]);
  }
  g.h = h;
  g.ngp = g.n[0] * g.n[1] * g.n[2];
  g.ntiles = g.nt[0] * g.nt[1] * g.nt[2];
  double E = M.E;
  for (int a = 0; a < 3; ++a) {
    const double lo = origin[a], hi = origin[a] + h * (double)N[a];
    E = std::max(E, std::max(std::fabs(lo - M.center[a]), std::fabs(hi - M.center[a])));
  }
  g.E = E;
  return 0;
}

// ---- call scaffolding shared by the entry points here and in batch.cu -------------------------

int begin_call(sdfgpu_ctx* ctx) {
  if (!ctx) return SDFGPU_ERR_INVALID_ARGUMENT;
  ctx->err.clear();
  SDF_CUDA(ctx, cudaSetDevice(ctx->device));
  return 0;
}

int need_mesh(sdfgpu_ctx* ctx) {
  if (!ctx->has_mesh) return fail(ctx, SDFGPU_ERR_NO_MESH, "no mesh: call sdfgpu_set_mesh first");
  return 0;
}

int reset_counters(sdfgpu_ctx* ctx) {
  SDF_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, sizeof(int64_t) * C_NUM, ctx->stream));
  std::memset(ctx->h_counters, 0, sizeof(ctx->h_counters));
  return 0;
}

int finish_counters(sdfgpu_ctx* ctx, const GridP& g) {
  int64_t tile_pairs = ctx->h_counters[C_TILE_PAIRS];
  SDF_CUDA(ctx, cudaMemcpyAsync(ctx->h_counters, ctx->d_counters, sizeof(int64_t) * C_NUM, cudaMemcpyDeviceToHost,
                                ctx->stream));
  SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->h_counters[C_TILE_PAIRS] = tile_pairs;
  sdfgpu_stats& s = ctx->stats;
  const int64_t* c = ctx->h_counters;
  s.ngp = g.ngp;
  s.nel = ctx->mesh.nel;
  s.tile_pairs = c[C_TILE_PAIRS];
  s.candidate_nodes = c[C_CAND_NODES];
  s.fp64_evals = c[C_FP64];
  s.knn_fallback_nodes = c[C_KNN];
  s.band_nodes = c[C_BAND];
  s.row_hits = c[C_ROW_HITS];
  s.undecided_nodes = c[C_LIST_UNDECIDED];
  s.extra_rays = c[C_EXTRA_RAYS];
  s.winding_nodes = c[C_WINDING];
  s.winding_ambiguous = c[C_WIND_AMBIG];
  s.unbounded_fallbacks = c[C_UNB_FALLBACK];
  s.rho_max = ctx->mesh.rho_max;
  s.certified_nodes = c[C_CERTIFIED];
  s.bvh_visits = c[C_VISITS];
  s.sign_band_reruns = c[C_SIGN_BAND];
  s.radius_loss = ctx->radius.loss;
  if (c[C_ERR_STACK]) return fail(ctx, SDFGPU_ERR_CAPACITY, "BVH traversal stack overflow");
  if (c[C_ERR_CAPACITY])
    return fail(ctx, SDFGPU_ERR_CAPACITY, "a per-node hit or candidate buffer overflowed (" + std::to_string(c[C_ERR_CAPACITY]) + " nodes)");
  return 0;
}

int check_sign_args(sdfgpu_ctx* ctx, int min_rays, int max_rays, double conf) {
  if (min_rays < 1 || min_rays > 36) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "min_rays must be in 1..36");
  if (max_rays < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "max_rays must be >= 1");
  if (!std::isfinite(conf)) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "confidence_threshold must be finite");
  return 0;
}

int check_mode(sdfgpu_ctx* ctx, int mode, int learned) {
  if (mode < SDFGPU_MODE_REF_RULE || mode > SDFGPU_MODE_LEARNED)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "unknown distance mode");
  if (mode == SDFGPU_MODE_LEARNED && !ctx->radius.trained)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "SDFGPU_MODE_LEARNED: no radius network (sdfgpu_train_radius)");
  if (learned && mode != SDFGPU_MODE_UNBOUNDED)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "use_learned_radius needs SDFGPU_MODE_UNBOUNDED");
  if (learned && !ctx->radius.trained)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "use_learned_radius: no radius network (sdfgpu_train_radius)");
  return 0;
}

// Runs the requested stages into device buffers.
int run_all(sdfgpu_ctx* ctx, const GridP& g, bool want_dist, bool want_sign, int mode, int learned, int min_rays,
            int max_rays, double conf, int use_winding, double* d_dist, double* d_xp, double* d_sign, double* d_conf,
            double* d_sdf, DistPlan* defer) {
  if (mode == SDFGPU_MODE_LEARNED) {  // the unbounded search with the learned radius
    mode = SDFGPU_MODE_UNBOUNDED;
    learned = 1;
  }
  SDF_TRY(reset_counters(ctx));
  ctx->launches = 0;
  for (int i = 0; i < T_NUM; ++i) SDF_MARK(ctx, i);
  // The sign stage runs on its own stream, forked after the counters are cleared: its row counting
  // is enqueued first, the distance stage next (its one host wait covers the row count too), and
  // the rest of the sign stage while the distance fold runs.  The join precedes the combine.
  cudaStream_t ss = ctx->sign_stream;
  SignPlan P;
  bool forked = false;
  // Every exit, failures included, leaves the context stream ordered after the sign stream and
  // the LBVH build, so nothing of this call is still running behind the next one.
  auto join = [&]() {
    if (forked && cudaEventRecord(ctx->ev_join, ss) == cudaSuccess) cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
    forked = false;
    cudaStreamWaitEvent(ctx->stream, ctx->ev_obb, 0);
  };
  auto stages = [&]() -> int {
    if (want_sign) {
      SDF_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
      SDF_CUDA(ctx, cudaStreamWaitEvent(ss, ctx->ev_fork, 0));
      forked = true;
      SDF_MARK_ON(ctx, T_SIGN0, ss);
      SDF_TRY(sign_begin(ctx, g, P));
    }
    if (want_dist) {
      if (defer)  // a batch runs the fold later, together with other meshes'
        SDF_TRY(dist_prepare(ctx, g, mode, d_dist, d_xp, *defer, learned));
      else
        SDF_TRY(run_distances(ctx, g, mode, learned, d_dist, d_xp));
    }
    SDF_MARK(ctx, T_DIST1);
    if (want_sign) {
      for (int i = T_ROWS; i <= T_PARITY; ++i) SDF_MARK_ON(ctx, i, ss);
      // Rays past the 36th are never cast, so every max_rays >= 44 gives the same votes as 44.
      const int max_eff = max_rays > 44 ? 44 : max_rays;
      SDF_TRY(sign_finish(ctx, g, P, min_rays, max_eff, conf, use_winding, d_sign, d_conf));
      SDF_MARK_ON(ctx, T_SIGN1, ss);
    }
    join();
    if (want_dist && want_sign && d_sdf && !defer) SDF_TRY(run_combine(ctx, g, d_dist, d_sign, d_sdf));
    return 0;
  };
  const int rc = stages();
  if (rc != 0) {
    join();
    return rc;
  }
  SDF_TRY(finish_counters(ctx, g));
  auto span = [&](int a, int b, double* out) -> int {
    float ms = 0.f;
    SDF_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->tev[a], ctx->tev[b]));
    *out = ms > 0.f ? ms : 0.0;
    return 0;
  };
  sdfgpu_stats& s = ctx->stats;
  SDF_TRY(span(T_DIST0, T_DIST1, &s.ms_distance));
  SDF_TRY(span(T_SIGN0, T_SIGN1, &s.ms_sign));
  SDF_TRY(span(T_DIST0, T_TILES, &s.ms_tiles));
  SDF_TRY(span(T_TILES, T_FOLD, &s.ms_fold));
  SDF_TRY(span(T_SIGN0, T_ROWS, &s.ms_rows));
  SDF_TRY(span(T_ROWS, T_PARITY, &s.ms_parity));
  SDF_TRY(span(T_PARITY, T_SIGN1, &s.ms_vote));
  if (!want_dist) s.ms_distance = s.ms_tiles = s.ms_fold = 0.0;
  if (!want_sign) s.ms_sign = s.ms_rows = s.ms_parity = s.ms_vote = 0.0;
  s.launches = ctx->launches;
  return 0;
}

// The fused distance x sign over z layers k0..k1 of the grid (k1 < 0: every layer), device outputs.
int sdf_device_impl(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int64_t k0, int64_t k1,
                    int mode, int min_rays, int max_rays, double conf, int use_winding, double* d_sdf, double* d_dist,
                    double* d_sign, double* d_conf) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  SDF_TRY(check_mode(ctx, mode, 0));
  SDF_TRY(check_sign_args(ctx, min_rays, max_rays, conf));
  if (!d_sdf) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "d_sdf must not be NULL");
  GridP g;
  SDF_TRY(make_grid(ctx, origin, h, N, g, k0, k1));
  if (!d_dist) SDF_TRY(scratch_t(ctx, "out_dist", (size_t)g.ngp, &d_dist));
  if (!d_sign) SDF_TRY(scratch_t(ctx, "out_sign", (size_t)g.ngp, &d_sign));
  if (!d_conf) SDF_TRY(scratch_t(ctx, "out_conf", (size_t)g.ngp, &d_conf));
  return run_all(ctx, g, true, true, mode, 0, min_rays, max_rays, conf, use_winding, d_dist, nullptr, d_sign, d_conf,
                 d_sdf);
}

// Same, results copied to host buffers.
int sdf_host_impl(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int64_t k0, int64_t k1,
                  int mode, int min_rays, int max_rays, double conf, int use_winding, double* sdf_out,
                  double* dist_out, double* sign_out, double* conf_out) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  if (!sdf_out) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "sdf_out must not be NULL");
  GridP g;
  SDF_TRY(make_grid(ctx, origin, h, N, g, k0, k1));
  double *d_sdf, *d_dist, *d_sign, *d_conf;
  SDF_TRY(scratch_t(ctx, "out_sdf", (size_t)g.ngp, &d_sdf));
  SDF_TRY(scratch_t(ctx, "out_dist", (size_t)g.ngp, &d_dist));
  SDF_TRY(scratch_t(ctx, "out_sign", (size_t)g.ngp, &d_sign));
  SDF_TRY(scratch_t(ctx, "out_conf", (size_t)g.ngp, &d_conf));
  SDF_TRY(sdf_device_impl(ctx, origin, h, N, k0, k1, mode, min_rays, max_rays, conf, use_winding, d_sdf, d_dist,
                          d_sign, d_conf));
  cudaStream_t st = ctx->stream;
  const size_t bytes = sizeof(double) * g.ngp;
  SDF_CUDA(ctx, cudaMemcpyAsync(sdf_out, d_sdf, bytes, cudaMemcpyDeviceToHost, st));
  if (dist_out) SDF_CUDA(ctx, cudaMemcpyAsync(dist_out, d_dist, bytes, cudaMemcpyDeviceToHost, st));
  if (sign_out) SDF_CUDA(ctx, cudaMemcpyAsync(sign_out, d_sign, bytes, cudaMemcpyDeviceToHost, st));
  if (conf_out) SDF_CUDA(ctx, cudaMemcpyAsync(conf_out, d_conf, bytes, cudaMemcpyDeviceToHost, st));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));
  return SDFGPU_OK;
}

// A context on device opts->device.  stage_priority: run the sign stage and the LBVH build on
// high-priority streams (what sdfgpu_create does); the worker contexts of a batch share the GPU with
// each other and use equal priorities (see batch.cu).
int create_context(const sdfgpu_opts* opts, sdfgpu_ctx** out, bool stage_priority) {
  if (!out) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "out must not be NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(nullptr, SDFGPU_ERR_NO_DEVICE,
                std::string("no CUDA device available: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
  }
  const int dev = opts ? opts->device : 0;
  if (dev < 0 || dev >= ndev) return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess)
    return fail(nullptr, SDFGPU_ERR_CUDA, "cudaGetDeviceProperties failed");
  if (prop.major < 10)
    return fail(nullptr, SDFGPU_ERR_NO_DEVICE, std::string("libsdfgpu is built for sm_100a; device is ") + prop.name);
  sdfgpu_ctx* ctx = new sdfgpu_ctx();
  ctx->device = dev;
  if (opts)
    for (int a = 0; a < 3; ++a)
      if (opts->tile[a] > 0) ctx->tile[a] = opts->tile[a];
  const int tn = ctx->tile[0] * ctx->tile[1] * ctx->tile[2];
  if (tn > 256 || tn < 32 || tn % 32 != 0) {
    delete ctx;
    return fail(nullptr, SDFGPU_ERR_INVALID_ARGUMENT, "a tile must hold 32, 64, ..., 256 nodes");
  }
  auto bail = [&](const char* what, cudaError_t err) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(err);
    sdfgpu_destroy(ctx);
    return fail(nullptr, SDFGPU_ERR_CUDA, m);
  };
  if ((e = cudaSetDevice(dev)) != cudaSuccess) return bail("cudaSetDevice", e);
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail("cudaStreamCreate", e);
  // The sign stage and the LBVH build run beside the distance fold, whose launch queues thousands of
  // CTAs: at the same priority their kernels would wait until the last fold CTA is dispatched.  At
  // the highest priority the scheduler hands them SMs as fold CTAs retire, so they finish inside the
  // fold instead of after it.  Not for batch workers: with several contexts sharing the GPU, one
  // worker's high-priority sign stage would hold back another's tile lists, which its host thread
  // waits for, and the workers would overlap less.
  int prio_least = 0, prio_greatest = 0;
  if ((e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest)) != cudaSuccess)
    return bail("cudaDeviceGetStreamPriorityRange", e);
  const int stage_prio = stage_priority ? prio_greatest : prio_least;
  if ((e = cudaStreamCreateWithPriority(&ctx->sign_stream, cudaStreamNonBlocking, stage_prio)) != cudaSuccess)
    return bail("cudaStreamCreate", e);
  if ((e = cudaStreamCreateWithPriority(&ctx->bvh_stream, cudaStreamNonBlocking, stage_prio)) != cudaSuccess)
    return bail("cudaStreamCreate", e);
  for (cudaEvent_t* ev : {&ctx->ev_fork, &ctx->ev_join, &ctx->ev_rows, &ctx->ev_mesh, &ctx->ev_bvh, &ctx->ev_obb})
    if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return bail("cudaEventCreate", e);
  if ((e = cudaHostAlloc((void**)&ctx->h_scalars, sizeof(int64_t) * S_NUM, cudaHostAllocDefault)) != cudaSuccess)
    return bail("cudaHostAlloc", e);
  for (auto& ev : ctx->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail("cudaEventCreate", e);
  for (auto& ev : ctx->tev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bail("cudaEventCreate", e);
  if ((e = cudaMalloc(&ctx->d_counters, sizeof(int64_t) * C_NUM)) != cudaSuccess) return bail("cudaMalloc", e);
  double D[36][3];
  host_directions(D);
  if (upload_directions(ctx, &D[0][0]) != 0) {
    std::string m = ctx->err;
    sdfgpu_destroy(ctx);
    return fail(nullptr, SDFGPU_ERR_CUDA, m);
  }
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return bail("cudaStreamSynchronize", e);
  *out = ctx;
  return SDFGPU_OK;
}

}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" {

int sdfgpu_abi_version(void) { return SDFGPU_ABI_VERSION; }

const char* sdfgpu_last_error(const sdfgpu_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int sdfgpu_create(const sdfgpu_opts* opts, sdfgpu_ctx** out) { return create_context(opts, out, true); }

int sdfgpu_destroy(sdfgpu_ctx* ctx) {
  if (!ctx) return SDFGPU_OK;
  for (sdfgpu_ctx* w : ctx->workers) sdfgpu_destroy(w);
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->sign_stream) cudaStreamSynchronize(ctx->sign_stream);
  if (ctx->bvh_stream) cudaStreamSynchronize(ctx->bvh_stream);
  for (auto& kv : ctx->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  for (auto& ev : ctx->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : ctx->tev)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {ctx->ev_fork, ctx->ev_join, ctx->ev_rows, ctx->ev_mesh, ctx->ev_bvh, ctx->ev_obb})
    if (ev) cudaEventDestroy(ev);
  if (ctx->bvh_stream) cudaStreamDestroy(ctx->bvh_stream);
  if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
  if (ctx->sign_stream) cudaStreamDestroy(ctx->sign_stream);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SDFGPU_OK;
}

int sdfgpu_grid_setup(const double xmin[3], const double xmax[3], int64_t n_max, int64_t margin, double origin[3],
                      double aabb_max[3], int64_t N[3], double* cell_size, int64_t* ngp) {
  if (!xmin || !xmax || !origin || !aabb_max || !N || !cell_size || !ngp) return SDFGPU_ERR_INVALID_ARGUMENT;
  return grid_core(xmin, xmax, n_max, margin, origin, aabb_max, N, cell_size, ngp);
}

int sdfgpu_grid_from_cell_size(const double* X, int64_t nnp, double B, double origin[3], double aabb_max[3],
                               int64_t N[3], double* cell_size, int64_t* ngp) {
  if (!X || nnp <= 0 || !(B > 0.0) || !std::isfinite(B)) return SDFGPU_ERR_INVALID_ARGUMENT;
  double xmin[3] = {X[0], X[1], X[2]}, xmax[3] = {X[0], X[1], X[2]};
  for (int64_t v = 1; v < nnp; ++v)
    for (int a = 0; a < 3; ++a) {
      xmin[a] = std::min(xmin[a], X[3 * v + a]);
      xmax[a] = std::max(xmax[a], X[3 * v + a]);
    }
  double ext = xmax[0] - xmin[0];
  for (int a = 1; a < 3; ++a) ext = std::max(ext, xmax[a] - xmin[a]);
  const double q = std::floor(ext / B);  // N_new = floor(Int, maximum(X_max .- X_min) / B)
  if (!std::isfinite(q) || q < 1 || q > 4.0e9) return SDFGPU_ERR_INVALID_ARGUMENT;
  return grid_core(xmin, xmax, (int64_t)q, 3, origin, aabb_max, N, cell_size, ngp);
}

int sdfgpu_set_mesh(sdfgpu_ctx* ctx, const double* X, int64_t nnp, const int64_t* IEN, int64_t nel) {
  SDF_TRY(begin_call(ctx));
  return mesh_upload_and_build(ctx, X, nnp, IEN, nel, false);
}

int sdfgpu_set_mesh_device(sdfgpu_ctx* ctx, const double* d_X, int64_t nnp, const int64_t* d_IEN, int64_t nel) {
  SDF_TRY(begin_call(ctx));
  return mesh_upload_and_build(ctx, d_X, nnp, d_IEN, nel, true);
}

int sdfgpu_distances(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], double* dist_out,
                     double* xp_out, int32_t mode, int32_t use_learned_radius) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  SDF_TRY(check_mode(ctx, mode, use_learned_radius));
  if (!dist_out) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "dist_out must not be NULL");
  GridP g;
  SDF_TRY(make_grid(ctx, origin, h, N, g));
  double *d_dist, *d_xp = nullptr;
  SDF_TRY(scratch_t(ctx, "out_dist", (size_t)g.ngp, &d_dist));
  if (xp_out) SDF_TRY(scratch_t(ctx, "out_xp", (size_t)g.ngp * 3, &d_xp));
  SDF_TRY(run_all(ctx, g, true, false, mode, use_learned_radius, 0, 0, 0.0, 0, d_dist, d_xp, nullptr, nullptr, nullptr));
  SDF_CUDA(ctx, cudaMemcpyAsync(dist_out, d_dist, sizeof(double) * g.ngp, cudaMemcpyDeviceToHost, ctx->stream));
  if (xp_out)
    SDF_CUDA(ctx, cudaMemcpyAsync(xp_out, d_xp, sizeof(double) * 3 * g.ngp, cudaMemcpyDeviceToHost, ctx->stream));
  SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SDFGPU_OK;
}

int sdfgpu_signs(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t min_rays,
                 int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, double* sign_out,
                 double* conf_out) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  SDF_TRY(check_sign_args(ctx, min_rays, max_rays, confidence_threshold));
  if (!sign_out) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "sign_out must not be NULL");
  GridP g;
  SDF_TRY(make_grid(ctx, origin, h, N, g));
  double *d_sign, *d_conf;
  SDF_TRY(scratch_t(ctx, "out_sign", (size_t)g.ngp, &d_sign));
  SDF_TRY(scratch_t(ctx, "out_conf", (size_t)g.ngp, &d_conf));
  SDF_TRY(run_all(ctx, g, false, true, 0, 0, min_rays, max_rays, confidence_threshold, use_winding_fallback, nullptr,
                  nullptr, d_sign, d_conf, nullptr));
  SDF_CUDA(ctx, cudaMemcpyAsync(sign_out, d_sign, sizeof(double) * g.ngp, cudaMemcpyDeviceToHost, ctx->stream));
  if (conf_out)
    SDF_CUDA(ctx, cudaMemcpyAsync(conf_out, d_conf, sizeof(double) * g.ngp, cudaMemcpyDeviceToHost, ctx->stream));
  SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SDFGPU_OK;
}

int sdfgpu_sdf_device(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t mode,
                      int32_t min_rays, int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback,
                      double* d_sdf, double* d_dist, double* d_sign, double* d_conf) {
  return sdf_device_impl(ctx, origin, h, N, 0, -1, mode, min_rays, max_rays, confidence_threshold,
                         use_winding_fallback, d_sdf, d_dist, d_sign, d_conf);
}

int sdfgpu_sdf(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t mode, int32_t min_rays,
               int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, double* sdf_out,
               double* dist_out, double* sign_out, double* conf_out) {
  return sdf_host_impl(ctx, origin, h, N, 0, -1, mode, min_rays, max_rays, confidence_threshold, use_winding_fallback,
                       sdf_out, dist_out, sign_out, conf_out);
}

int sdfgpu_sdf_slab(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int64_t k0, int64_t k1,
                    int32_t mode, int32_t min_rays, int32_t max_rays, double confidence_threshold,
                    int32_t use_winding_fallback, double* sdf_out, double* dist_out, double* sign_out,
                    double* conf_out) {
  if (k1 < 0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "z layers must satisfy 0 <= k0 <= k1 <= N[2]");
  return sdf_host_impl(ctx, origin, h, N, k0, k1, mode, min_rays, max_rays, confidence_threshold,
                       use_winding_fallback, sdf_out, dist_out, sign_out, conf_out);
}

int sdfgpu_sdf_slab_device(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int64_t k0,
                           int64_t k1, int32_t mode, int32_t min_rays, int32_t max_rays, double confidence_threshold,
                           int32_t use_winding_fallback, double* d_sdf, double* d_dist, double* d_sign,
                           double* d_conf) {
  if (k1 < 0) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "z layers must satisfy 0 <= k0 <= k1 <= N[2]");
  return sdf_device_impl(ctx, origin, h, N, k0, k1, mode, min_rays, max_rays, confidence_threshold,
                         use_winding_fallback, d_sdf, d_dist, d_sign, d_conf);
}

int sdfgpu_train_radius(sdfgpu_ctx* ctx, int32_t coarse_n, int32_t steps, int32_t batch, float lr, uint64_t seed,
                        float* final_loss) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  if (coarse_n < 9 || coarse_n > 1024 || steps < 0 || batch < 32 || !(lr > 0.f))
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "train_radius: need 9 <= coarse_n <= 1024, steps >= 0, batch >= 32, lr > 0");
  SDF_TRY(reset_counters(ctx));
  ctx->launches = 0;
  RadiusNorm& R = ctx->radius;
  R.train_coarse = coarse_n;
  R.train_steps = steps;
  R.train_batch = batch;
  R.train_lr = lr;
  R.train_seed = seed;
  SDF_MARK(ctx, T_DIST0);
  SDF_TRY(train_radius(ctx, coarse_n, steps, batch, lr, seed, final_loss));
  SDF_MARK(ctx, T_DIST1);
  SDF_CUDA(ctx, cudaEventSynchronize(ctx->tev[T_DIST1]));
  float ms = 0.f;
  SDF_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->tev[T_DIST0], ctx->tev[T_DIST1]));
  ctx->stats.ms_train = ms;
  ctx->stats.train_launches = ctx->launches;
  ctx->stats.radius_loss = ctx->radius.loss;
  return SDFGPU_OK;
}

int sdfgpu_radius_param_count(void) { return kParams; }

int sdfgpu_radius_params(sdfgpu_ctx* ctx, float* params, double norm[4]) {
  SDF_TRY(begin_call(ctx));
  if (!params || !norm) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "NULL argument");
  return get_radius_params(ctx, params, norm);
}

int sdfgpu_set_radius_params(sdfgpu_ctx* ctx, const float* params, const double norm[4]) {
  SDF_TRY(begin_call(ctx));
  if (!params || !norm || !(norm[3] > 0.0)) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "bad params or norm");
  return set_radius_params(ctx, params, norm);
}

int sdfgpu_set_radius_margin(sdfgpu_ctx* ctx, float alpha, float beta) {
  SDF_TRY(begin_call(ctx));
  if (!((alpha >= 0.f && alpha <= 10.f) || std::isinf(alpha) && alpha > 0.f) || !(beta >= 0.f && beta <= 100.f))
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT,
                "radius margin: need 0 <= alpha <= 10 (or +inf: no bound) and 0 <= beta <= 100");
  ctx->radius.alpha = alpha;
  ctx->radius.beta = beta;
  return SDFGPU_OK;
}

int sdfgpu_set_brick(sdfgpu_ctx* ctx, const int32_t brick[3]) {
  SDF_TRY(begin_call(ctx));
  if (!brick || brick[0] < 1 || brick[1] < 1 || brick[2] < 1 || brick[0] * brick[1] * brick[2] != 32)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "brick: three positive extents whose product is 32");
  for (int a = 0; a < 3; ++a) ctx->brick[a] = brick[a];
  return SDFGPU_OK;
}

int sdfgpu_radius_eval(sdfgpu_ctx* ctx, const float* xn, int64_t B, float* dhat) {
  SDF_TRY(begin_call(ctx));
  if (!xn || !dhat || B < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "bad arguments");
  float *dx, *dy;
  SDF_TRY(scratch_t(ctx, "reval_x", (size_t)B * 3, &dx));
  SDF_TRY(scratch_t(ctx, "reval_y", (size_t)B, &dy));
  SDF_CUDA(ctx, cudaMemcpyAsync(dx, xn, sizeof(float) * 3 * B, cudaMemcpyHostToDevice, ctx->stream));
  SDF_TRY(run_radius(ctx, nullptr, dx, B, -1.f, 0.f, dy));
  SDF_CUDA(ctx, cudaMemcpyAsync(dhat, dy, sizeof(float) * B, cudaMemcpyDeviceToHost, ctx->stream));
  SDF_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SDFGPU_OK;
}

int sdfgpu_mlp_train_eval(sdfgpu_ctx* ctx, const float* params, const float* xn, const float* target, int64_t B,
                          float* dhat, float* loss, float* grad) {
  SDF_TRY(begin_call(ctx));
  if (!params || !xn || B < 1) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "bad arguments");
  if ((loss || grad) && !target) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "loss and gradient need targets");
  return mlp_eval_host(ctx, params, xn, target, B, dhat, loss, grad);
}

int sdfgpu_get_stream(sdfgpu_ctx* ctx, void** stream) {
  if (!ctx || !stream) return SDFGPU_ERR_INVALID_ARGUMENT;
  *stream = (void*)ctx->stream;
  return SDFGPU_OK;
}

int sdfgpu_get_stats(const sdfgpu_ctx* ctx, sdfgpu_stats* out) {
  if (!ctx || !out) return SDFGPU_ERR_INVALID_ARGUMENT;
  *out = ctx->stats;
  return SDFGPU_OK;
}

}  // extern "C"
