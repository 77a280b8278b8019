// batch.cu -- many meshes per call (sdfgpu_sdf_batch) and the tile autotuner (sdfgpu_autotune).
//
// A batch is a queue of (mesh, grid) items drained by worker contexts, one host thread and one
// CUDA stream each, largest first (longest-processing-time order).  The per-mesh pipeline has
// host-sized stages (the (tile, triangle) pair count, the axis-row hit count, the undecided-node
// count), so one mesh alone leaves the GPU idle while its host thread waits; several workers fill
// those gaps with the kernels of other meshes.
//
// Reference-rule and h-bounded batches run in three phases:
//   1. the workers prepare every item -- mesh records and LBVH, the distance tile lists, the whole
//      sign stage -- each item in its own buffers (scratch names in a per-worker slot namespace, so
//      repeated batches reuse them);
//   2. the folds of all items run in ONE persistent kernel (k_tile_fold_multi: CTAs stride over the
//      (item, tile) work list of the whole batch, one tile volume for all, autotuned on the largest
//      item), followed by every item's 3-nearest-vertex fallback and combine -- the whole sequence
//      captured in one CUDA graph and launched once;
//   3. the fields are copied to the callers' buffers.
// Unbounded and learned-radius batches (SDFGPU_MODE_UNBOUNDED / _LEARNED) take the same phases:
// phase 1 stops the distance stage at the search's arguments (and, learned, trains each mesh's
// radius network on a coarse grid of at most half the mesh grid's nodes per axis and predicts the
// radius of every warp brick); phase 2's persistent launch is the multi-mesh search
// (k_unbounded_multi: warps take (item, brick) work items from one queue; with the radius, a second
// launch reruns the bricks the first did not certify).  In the per-item form a worker trains and
// searches each mesh in turn.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>

#include "common.cuh"

namespace sdfgpu {
namespace {

constexpr int32_t kTiles[][3] = {{4, 4, 4}, {8, 4, 2}, {4, 4, 2}, {8, 4, 4}, {4, 4, 8}, {8, 8, 4}};
// Warp bricks (nodes of one warp) of the unbounded search.
constexpr int32_t kBricks[][3] = {{4, 2, 4}, {4, 4, 2}, {2, 4, 4}, {8, 4, 1}, {4, 8, 1}, {32, 1, 1}};
constexpr int kMaxStreams = 64;

uint32_t pack_tile(const int32_t t[3]) { return (uint32_t)(t[0] | (t[1] << 8) | (t[2] << 16)); }
void unpack_tile(uint32_t p, int32_t t[3]) {
  t[0] = (int32_t)(p & 0xff);
  t[1] = (int32_t)((p >> 8) & 0xff);
  t[2] = (int32_t)((p >> 16) & 0xff);
}

int64_t item_ngp(const sdfgpu_batch_item& it) { return (it.N[0] + 1) * (it.N[1] + 1) * (it.N[2] + 1); }

double item_work(const sdfgpu_batch_item& it) {
  return (double)item_ngp(it) * std::log2(std::max(2.0, (double)it.nel));
}

// Size class of an item for the autotuner: floor(log4 ngp), floor(log4 nel).
int64_t size_class(const sdfgpu_batch_item& it) {
  auto lg4 = [](double v) { return (int64_t)std::floor(std::log2(std::max(1.0, v)) / 2.0); };
  return lg4((double)item_ngp(it)) * 64 + lg4((double)it.nel);
}

void add_stats(sdfgpu_stats& a, const sdfgpu_stats& b) {
  a.ngp += b.ngp;
  a.nel += b.nel;
  a.tile_pairs += b.tile_pairs;
  a.active_tiles += b.active_tiles;
  a.candidate_nodes += b.candidate_nodes;
  a.fp64_evals += b.fp64_evals;
  a.knn_fallback_nodes += b.knn_fallback_nodes;
  a.band_nodes += b.band_nodes;
  a.row_hits += b.row_hits;
  a.undecided_nodes += b.undecided_nodes;
  a.extra_rays += b.extra_rays;
  a.winding_nodes += b.winding_nodes;
  a.winding_ambiguous += b.winding_ambiguous;
  a.rho_max = std::max(a.rho_max, b.rho_max);
  a.ms_distance += b.ms_distance;
  a.ms_sign += b.ms_sign;
  a.ms_mesh += b.ms_mesh;
  a.launches += b.launches;
  a.mesh_launches += b.mesh_launches;
  a.ms_tiles += b.ms_tiles;
  a.ms_fold += b.ms_fold;
  a.ms_rows += b.ms_rows;
  a.ms_parity += b.ms_parity;
  a.ms_vote += b.ms_vote;
  a.certified_nodes += b.certified_nodes;
  a.unbounded_fallbacks += b.unbounded_fallbacks;
  a.bvh_visits += b.bvh_visits;
  a.ms_train += b.ms_train;
  a.train_launches += b.train_launches;
  a.sign_band_reruns += b.sign_band_reruns;
}

struct BatchJob {
  sdfgpu_ctx* parent;
  sdfgpu_batch_item* items;
  std::vector<int64_t> order;
  int mode, min_rays, max_rays, use_winding, autotune;
  double conf;
  RadiusNorm train;  // SDFGPU_MODE_LEARNED: the training options every mesh gets
  std::atomic<int64_t> next{0};
  std::atomic<bool> stop{false};
  std::mutex mu;  // guards rc, err, stats and parent->tuned
  int rc = 0;
  std::string err;
  sdfgpu_stats stats = {};
};

}  // namespace

// Times the distance stage of the current mesh on grid (origin, h, N) with every tile of kTiles, or,
// in the unbounded mode (which has no tiles), with every warp brick of kBricks.
int autotune_tile(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int mode, int32_t best[3],
                  double* best_ms) {
  const bool bricks = mode == SDFGPU_MODE_UNBOUNDED || mode == SDFGPU_MODE_LEARNED;
  const bool learned = mode == SDFGPU_MODE_LEARNED;  // the learned search itself (the network is trained)
  int32_t* shape = bricks ? ctx->brick : ctx->tile;
  const int32_t(*table)[3] = bricks ? kBricks : kTiles;
  const int count = bricks ? (int)(sizeof(kBricks) / sizeof(kBricks[0])) : (int)(sizeof(kTiles) / sizeof(kTiles[0]));
  const int32_t keep[3] = {shape[0], shape[1], shape[2]};
  double best_t = 1e300;
  int best_i = -1;
  double* d_dist = nullptr;
  for (int c = 0; c < count; ++c) {
    for (int a = 0; a < 3; ++a) shape[a] = table[c][a];
    GridP g;
    int rc = make_grid(ctx, origin, h, N, g);
    if (rc == 0) rc = scratch_t(ctx, "out_dist", (size_t)g.ngp, &d_dist);
    double t_min = 1e300;
    for (int rep = 0; rep < 2 && rc == 0; ++rep) {
      rc = reset_counters(ctx);
      if (rc == 0 && cudaEventRecord(ctx->ev[0], ctx->stream) != cudaSuccess) rc = SDFGPU_ERR_CUDA;
      if (rc == 0)
        rc = run_distances(ctx, g, learned ? SDFGPU_MODE_UNBOUNDED : mode, learned ? 1 : 0, d_dist, nullptr);
      if (rc == 0 && cudaEventRecord(ctx->ev[1], ctx->stream) != cudaSuccess) rc = SDFGPU_ERR_CUDA;
      if (rc == 0) rc = finish_counters(ctx, g);
      float ms = 0.f;
      if (rc == 0 && cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]) != cudaSuccess) rc = SDFGPU_ERR_CUDA;
      if (rc == 0) t_min = std::min(t_min, (double)ms);
    }
    if (rc != 0) {
      for (int a = 0; a < 3; ++a) shape[a] = keep[a];
      if (ctx->err.empty()) ctx->err = "autotune: CUDA event failure";
      return rc;
    }
    if (t_min < best_t) {
      best_t = t_min;
      best_i = c;
    }
  }
  for (int a = 0; a < 3; ++a) shape[a] = best[a] = table[best_i][a];
  if (best_ms) *best_ms = best_t;
  return 0;
}

namespace {

int pick_tile(BatchJob& J, sdfgpu_ctx* w, const sdfgpu_batch_item& it) {
  // per mode: the unbounded mode tunes warp bricks, the others tiles
  const int64_t key = size_class(it) * 4 + J.mode;
  {
    std::lock_guard<std::mutex> lk(J.mu);
    auto f = J.parent->tuned.find(key);
    if (f != J.parent->tuned.end()) {
      unpack_tile(f->second, (J.mode == SDFGPU_MODE_UNBOUNDED || J.mode == SDFGPU_MODE_LEARNED) ? w->brick : w->tile);
      return 0;
    }
  }
  int32_t t[3];
  SDF_TRY(autotune_tile(w, it.origin, it.h, it.N, J.mode, t, nullptr));
  std::lock_guard<std::mutex> lk(J.mu);
  J.parent->tuned.emplace(key, pack_tile(t));  // a concurrent tuning of the same class may have won
  return 0;
}

// An item's radius network (SDFGPU_MODE_LEARNED), on a coarse grid of its own: at most half the
// nodes of the item's grid per axis, the batch context's other training options and search margin.
int train_item(BatchJob& J, sdfgpu_ctx* w, const sdfgpu_batch_item& it, sdfgpu_stats& ms) {
  const int64_t K = std::max(it.N[0], std::max(it.N[1], it.N[2])) + 1;
  const int coarse = (int)std::max<int64_t>(16, std::min<int64_t>(J.train.train_coarse, K / 2));
  const int rc = sdfgpu_train_radius(w, coarse, J.train.train_steps, J.train.train_batch, J.train.train_lr,
                                     J.train.train_seed, nullptr);
  ms.ms_train = w->stats.ms_train;
  ms.train_launches = w->stats.train_launches;
  w->radius.alpha = J.train.alpha;  // the batch context's search margin
  w->radius.beta = J.train.beta;
  return rc;
}

void worker_main(BatchJob& J, sdfgpu_ctx* w) {
  const int64_t n = (int64_t)J.order.size();
  w->ns.clear();
  for (;;) {
    if (J.stop.load()) return;
    const int64_t k = J.next.fetch_add(1);
    if (k >= n) return;
    const int64_t i = J.order[k];
    sdfgpu_batch_item& it = J.items[i];
    int rc = sdfgpu_set_mesh(w, it.X, it.nnp, it.IEN, it.nel);
    sdfgpu_stats ms = w->stats;
    if (rc == 0 && J.mode == SDFGPU_MODE_LEARNED) rc = train_item(J, w, it, ms);
    if (rc == 0 && J.autotune) rc = pick_tile(J, w, it);
    if (rc == 0)
      rc = sdfgpu_sdf(w, it.origin, it.h, it.N, J.mode, J.min_rays, J.max_rays, J.conf, J.use_winding, it.sdf, it.dist,
                      it.sign, it.conf);
    std::lock_guard<std::mutex> lk(J.mu);
    if (rc != 0) {
      if (J.rc == 0) {
        J.rc = rc;
        J.err = "batch item " + std::to_string(i) + ": " + w->err;
      }
      J.stop.store(true);
      return;
    }
    sdfgpu_stats s = w->stats;
    s.ms_mesh = ms.ms_mesh;
    s.mesh_launches = ms.mesh_launches;
    s.ms_train = ms.ms_train;
    s.train_launches = ms.train_launches;
    add_stats(J.stats, s);
  }
}

// One prepared item of a persistent batch.
struct Prepared {
  DistPlan plan;
  double *d_dist = nullptr, *d_sign = nullptr, *d_conf = nullptr, *d_sdf = nullptr;
  int64_t ngp = 0;
};

// Phase 1 of a reference-rule / h-bounded batch: everything but the fold, fallback and combine,
// for the items assigned to this worker (`mine`, a fixed longest-processing-time assignment, so a
// repeated batch puts every item in the same worker slot and its buffers are reused as they are).
void worker_prepare(BatchJob& J, sdfgpu_ctx* w, const std::vector<int64_t>& mine, std::vector<Prepared>& prep) {
  int slot = 0;
  for (const int64_t i : mine) {
    if (J.stop.load()) return;
    sdfgpu_batch_item& it = J.items[i];
    Prepared& P = prep[(size_t)i];
    w->ns = "s" + std::to_string(slot++) + ":";
    int rc = sdfgpu_set_mesh(w, it.X, it.nnp, it.IEN, it.nel);
    sdfgpu_stats ms = w->stats;
    if (rc == 0 && J.mode == SDFGPU_MODE_LEARNED) rc = train_item(J, w, it, ms);
    if (rc == 0 && J.autotune) rc = pick_tile(J, w, it);
    GridP g;
    if (rc == 0) rc = make_grid(w, it.origin, it.h, it.N, g);
    if (rc == 0) rc = scratch_t(w, "out_dist", (size_t)g.ngp, &P.d_dist);
    if (rc == 0) rc = scratch_t(w, "out_sign", (size_t)g.ngp, &P.d_sign);
    if (rc == 0) rc = scratch_t(w, "out_conf", (size_t)g.ngp, &P.d_conf);
    if (rc == 0) rc = scratch_t(w, "out_sdf", (size_t)g.ngp, &P.d_sdf);
    if (rc == 0)
      rc = run_all(w, g, true, true, J.mode, 0, J.min_rays, J.max_rays, J.conf, J.use_winding, P.d_dist, nullptr,
                   P.d_sign, P.d_conf, P.d_sdf, &P.plan);
    P.ngp = g.ngp;
    std::lock_guard<std::mutex> lk(J.mu);
    if (rc != 0) {
      if (J.rc == 0) {
        J.rc = rc;
        J.err = "batch item " + std::to_string(i) + ": " + w->err;
      }
      J.stop.store(true);
      return;
    }
    sdfgpu_stats s = w->stats;
    s.ms_mesh = ms.ms_mesh;
    s.mesh_launches = ms.mesh_launches;
    s.ms_train = ms.ms_train;
    s.train_launches = ms.train_launches;
    add_stats(J.stats, s);
  }
}

// Phases 2 and 3 on ctx's stream: one graph with the persistent fold of every item, then each
// item's fallback and combine; then the copies to the callers' buffers.
int run_persistent(sdfgpu_ctx* ctx, BatchJob& J, std::vector<Prepared>& prep, int nw, int threads) {
  cudaStream_t st = ctx->stream;
  for (int k = 0; k < nw; ++k) {  // everything the workers enqueued is done
    sdfgpu_ctx* w = ctx->workers[k];
    SDF_CUDA(ctx, cudaStreamSynchronize(w->stream));
    SDF_CUDA(ctx, cudaStreamSynchronize(w->sign_stream));
    SDF_CUDA(ctx, cudaStreamSynchronize(w->bvh_stream));
  }
  const int64_t count = (int64_t)prep.size();
  // unbounded / learned items: one search over every (item, brick) work item (plan.unb); the others
  // one fold over every (item, tile)
  const bool unb = prep[0].plan.unbounded;
  bool radius = unb;
  for (const Prepared& P : prep) radius = radius && P.plan.unb_radius;
  const size_t sz = unb ? unb_args_size() : fold_args_size();
  std::vector<unsigned char> args(sz * (size_t)count);
  std::vector<int64_t> off((size_t)count + 1);
  int64_t total = 0;
  for (int64_t i = 0; i < count; ++i) {
    off[(size_t)i] = total;
    total += unb ? prep[i].plan.nbricks : prep[i].plan.ntiles;
  }
  off[(size_t)count] = total;
  int64_t* redo = nullptr;
  unsigned long long* heads = nullptr;
  if (unb) {
    SDF_TRY(scratch_t(ctx, "batch_redo", (size_t)total, &redo));
    SDF_TRY(scratch_t(ctx, "batch_heads", 3, &heads));
  }
  for (int64_t i = 0; i < count; ++i) {
    if (unb) {
      plan_set_redo(prep[i].plan, redo, heads + 2, off[(size_t)i]);
      std::memcpy(args.data() + sz * (size_t)i, prep[i].plan.unb, sz);
    } else {
      plan_set_counters(prep[i].plan, ctx->d_counters);
      std::memcpy(args.data() + sz * (size_t)i, prep[i].plan.fold, sz);
    }
  }
  void* d_args;
  int64_t* d_off;
  SDF_TRY(scratch(ctx, "batch_args", args.size(), &d_args));
  SDF_TRY(scratch_t(ctx, "batch_off", (size_t)count + 1, &d_off));
  SDF_TRY(reset_counters(ctx));
  SDF_CUDA(ctx, cudaMemcpyAsync(d_args, args.data(), args.size(), cudaMemcpyHostToDevice, st));
  SDF_CUDA(ctx, cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * (count + 1), cudaMemcpyHostToDevice, st));
  int64_t grid = 1;
  if (unb) SDF_TRY(unb_multi_grid(ctx, total, &grid));
  else SDF_TRY(dist_fold_multi_grid(ctx, threads, total, &grid));
  SDF_CUDA(ctx, cudaStreamSynchronize(st));  // the argument arrays are in place before the capture

  // the items' fallbacks and combines after the fold, on the (idle) worker streams side by side
  std::vector<cudaEvent_t> evs((size_t)nw + 1, nullptr);
  for (auto& e : evs)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      for (auto& x : evs)
        if (x) cudaEventDestroy(x);
      return fail(ctx, SDFGPU_ERR_CUDA, "batch: cudaEventCreate failed");
    }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  SDF_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = unb ? unb_multi(ctx, d_args, d_off, (int)count, radius, redo, heads, grid, st)
               : dist_fold_multi(ctx, d_args, d_off, (int)count, total, threads, grid, st);
  if (rc == 0 && cudaEventRecord(evs[(size_t)nw], st) != cudaSuccess) rc = fail(ctx, SDFGPU_ERR_CUDA, "batch fork");
  for (int k = 0; k < nw && rc == 0; ++k)
    if (cudaStreamWaitEvent(ctx->workers[k]->stream, evs[(size_t)nw], 0) != cudaSuccess)
      rc = fail(ctx, SDFGPU_ERR_CUDA, "batch fork");
  for (int64_t i = 0; i < count && rc == 0; ++i) {
    const Prepared& P = prep[(size_t)i];
    cudaStream_t si = ctx->workers[i % nw]->stream;
    if (P.plan.knn) rc = dist_knn(ctx, P.plan, si, false);
    if (rc == 0) rc = launch_combine(ctx, P.ngp, P.d_dist, P.d_sign, P.d_sdf, si);
  }
  for (int k = 0; k < nw; ++k)  // join every forked stream, also after a failure, to end the capture
    if (cudaEventRecord(evs[(size_t)k], ctx->workers[k]->stream) == cudaSuccess)
      cudaStreamWaitEvent(st, evs[(size_t)k], 0);
  const cudaError_t ce = cudaStreamEndCapture(st, &graph);  // always leave capture mode
  for (auto& e : evs) cudaEventDestroy(e);
  if (rc == 0 && ce != cudaSuccess) rc = fail(ctx, SDFGPU_ERR_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(ce));
  if (rc == 0) {
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) rc = fail(ctx, SDFGPU_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
  float ms = 0.f;
  if (rc == 0 && (cudaEventRecord(ctx->ev[0], st) != cudaSuccess || cudaGraphLaunch(exec, st) != cudaSuccess ||
                  cudaEventRecord(ctx->ev[1], st) != cudaSuccess))
    rc = fail(ctx, SDFGPU_ERR_CUDA, "batch graph launch failed");
  for (int64_t i = 0; i < count && rc == 0; ++i) {
    const sdfgpu_batch_item& it = J.items[i];
    const Prepared& P = prep[(size_t)i];
    const size_t bytes = sizeof(double) * (size_t)P.ngp;
    cudaError_t e = cudaMemcpyAsync(it.sdf, P.d_sdf, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && it.dist) e = cudaMemcpyAsync(it.dist, P.d_dist, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && it.sign) e = cudaMemcpyAsync(it.sign, P.d_sign, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && it.conf) e = cudaMemcpyAsync(it.conf, P.d_conf, bytes, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = fail(ctx, SDFGPU_ERR_CUDA, std::string("batch copy: ") + cudaGetErrorString(e));
  }
  int64_t c[C_NUM] = {};
  if (rc == 0) {
    cudaError_t e = cudaMemcpyAsync(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    if (e != cudaSuccess) rc = fail(ctx, SDFGPU_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (rc != 0) return rc;
  if (c[C_ERR_STACK]) return fail(ctx, SDFGPU_ERR_CAPACITY, "BVH traversal stack overflow");
  if (c[C_ERR_CAPACITY]) return fail(ctx, SDFGPU_ERR_CAPACITY, "a per-node candidate buffer overflowed");
  J.stats.fp64_evals += c[C_FP64];
  J.stats.candidate_nodes += c[C_CAND_NODES];
  J.stats.knn_fallback_nodes += c[C_KNN];
  J.stats.certified_nodes += c[C_CERTIFIED];
  J.stats.unbounded_fallbacks += c[C_UNB_FALLBACK];
  J.stats.bvh_visits += c[C_VISITS];
  J.stats.ms_fold += ms;
  J.stats.ms_distance += ms;
  J.stats.launches += 1 + count;
  return 0;
}

}  // namespace
}  // namespace sdfgpu

using namespace sdfgpu;

extern "C" {

int sdfgpu_autotune(sdfgpu_ctx* ctx, const double origin[3], double h, const int64_t N[3], int32_t mode,
                    int32_t tile_out[3], double* ms_out) {
  SDF_TRY(begin_call(ctx));
  SDF_TRY(need_mesh(ctx));
  SDF_TRY(check_mode(ctx, mode, 0));
  int32_t t[3];
  double ms = 0.0;
  SDF_TRY(autotune_tile(ctx, origin, h, N, mode, t, &ms));
  if (tile_out)
    for (int a = 0; a < 3; ++a) tile_out[a] = t[a];
  if (ms_out) *ms_out = ms;
  return SDFGPU_OK;
}

int sdfgpu_sdf_batch(sdfgpu_ctx* ctx, sdfgpu_batch_item* items, int64_t count, int32_t mode, int32_t min_rays,
                     int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, int32_t streams,
                     int32_t autotune) {
  return sdfgpu_sdf_batch_ex(ctx, items, count, mode, min_rays, max_rays, confidence_threshold, use_winding_fallback,
                             streams, autotune, 0);
}

int sdfgpu_sdf_batch_ex(sdfgpu_ctx* ctx, sdfgpu_batch_item* items, int64_t count, int32_t mode, int32_t min_rays,
                        int32_t max_rays, double confidence_threshold, int32_t use_winding_fallback, int32_t streams,
                        int32_t autotune, int32_t persistent) {
  SDF_TRY(begin_call(ctx));
  if (count < 0 || (count > 0 && !items)) return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "items must hold count entries");
  if (streams < 0 || streams > kMaxStreams)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "streams must be in 0.." + std::to_string(kMaxStreams));
  if (mode < SDFGPU_MODE_REF_RULE || mode > SDFGPU_MODE_LEARNED)
    return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "unknown distance mode");
  if (mode != SDFGPU_MODE_LEARNED) SDF_TRY(check_mode(ctx, mode, 0));  // a learned batch trains every mesh itself
  SDF_TRY(check_sign_args(ctx, min_rays, max_rays, confidence_threshold));
  for (int64_t i = 0; i < count; ++i) {
    const sdfgpu_batch_item& it = items[i];
    if (!it.X || !it.IEN || !it.sdf || it.nnp < 1 || it.nel < 1)
      return fail(ctx, SDFGPU_ERR_INVALID_ARGUMENT, "batch item " + std::to_string(i) + ": needs X, IEN, sdf and a non-empty mesh");
  }
  ctx->stats = sdfgpu_stats{};
  if (count == 0) return SDFGPU_OK;
  const int nw = (int)std::min<int64_t>(streams == 0 ? 8 : streams, count);
  while ((int)ctx->workers.size() < nw) {
    sdfgpu_opts o = {};
    o.device = ctx->device;
    for (int a = 0; a < 3; ++a) o.tile[a] = ctx->tile[a];
    sdfgpu_ctx* w = nullptr;
    if (create_context(&o, &w, false) != SDFGPU_OK)
      return fail(ctx, SDFGPU_ERR_CUDA, std::string("batch worker: ") + sdfgpu_last_error(nullptr));
    ctx->workers.push_back(w);
  }
  BatchJob J;
  J.parent = ctx;
  J.items = items;
  J.mode = mode;
  J.min_rays = min_rays;
  J.max_rays = max_rays;
  J.conf = confidence_threshold;
  J.use_winding = use_winding_fallback;
  J.autotune = autotune;
  J.train = ctx->radius;
  J.order.resize((size_t)count);
  std::iota(J.order.begin(), J.order.end(), (int64_t)0);
  std::stable_sort(J.order.begin(), J.order.end(),
                   [&](int64_t a, int64_t b) { return item_work(items[a]) > item_work(items[b]); });
  for (int k = 0; k < nw; ++k)
    if (!autotune)
      for (int a = 0; a < 3; ++a) {
        ctx->workers[k]->tile[a] = ctx->tile[a];
        ctx->workers[k]->brick[a] = ctx->brick[a];
      }
  std::vector<std::thread> threads;
  threads.reserve(nw);
  if (!persistent) {  // per-item pipelines
    for (int k = 0; k < nw; ++k) threads.emplace_back(worker_main, std::ref(J), ctx->workers[k]);
    for (auto& t : threads) t.join();
    ctx->stats = J.stats;
    if (J.rc != 0) return fail(ctx, J.rc, J.err);
    return SDFGPU_OK;
  }
  // Fixed longest-processing-time assignment of the items to the workers.
  std::vector<std::vector<int64_t>> mine((size_t)nw);
  {
    std::vector<double> load((size_t)nw, 0.0);
    for (const int64_t i : J.order) {
      const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
      mine[k].push_back(i);
      load[k] += item_work(items[i]);
    }
  }
  std::vector<Prepared> prep((size_t)count);
  for (int k = 0; k < nw; ++k)
    threads.emplace_back(worker_prepare, std::ref(J), ctx->workers[k], std::cref(mine[(size_t)k]), std::ref(prep));
  for (auto& t : threads) t.join();
  if (J.rc != 0) {
    ctx->stats = J.stats;
    return fail(ctx, J.rc, J.err);
  }
  int tvol = 32;  // the persistent fold's CTA holds the largest tile of the batch
  for (const Prepared& P : prep) tvol = std::max(tvol, P.plan.threads);
  const int rc = run_persistent(ctx, J, prep, nw, tvol);
  ctx->stats = J.stats;
  return rc;
}

}  // extern "C"
