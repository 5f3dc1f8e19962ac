// fr_batch.cu -- many reconstructions in one persistent insertion launch, and
// the tile/schedule autotuner.
//
// A batch holds independent FourierReconstructor states (uneven N, modes and
// symmetries: even/odd half maps, heterogeneity classes).  Each insert call
// runs every job's prologue on the batch stream, then ONE persistent insertion
// launch (k_column) whose work list interleaves all jobs' (tile, slice block)
// items, heaviest first, then the small face-tap kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <tuple>
#include <vector>

#include "fr_handle.h"

using namespace fr;

namespace fr {

// ------------------------------------------------------------------ tuning
// Choices per (N, mode, nsym): >= 0 gather with that tile, -2 scatter.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, int> g_tuned;
constexpr int kTunedScatter = -2;
// Particles per job per round of a batched insertion (bounds the scratch).
constexpr int kBatchChunk = 4096;

int tuned_tile(int N, int mode, int nsym) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(std::make_tuple(N, mode, nsym));
  return it == g_tuned.end() ? -1 : it->second;
}

int default_tile(int mode, int N, int nsym, int np) {
  (void)nsym; (void)np; (void)N; (void)mode;
  // unless the autotuner measured otherwise: the pixel-major kernel for the
  // narrow windows, the barrier-free column kernel for gauss_5
  return mode == FR_MODE_GAUSS5 ? kColumn3Tile : kPixelTile;
}

}  // namespace fr

// ------------------------------------------------------------------ batch
namespace fr {
// Device copies of a batched launch's job table and work list.
struct BatchScratch {
  DevBuf d_jobs, d_work, d_counter;
  PinnedRing ring;
  cudaEvent_t done = nullptr;     // after the last launch that read this scratch
  cudaStream_t last = nullptr;
  ~BatchScratch() {
    if (done) { cudaEventSynchronize(done); cudaEventDestroy(done); }
    ring.release();
  }
};
}  // namespace fr

struct fr_batch {
  std::vector<fr_recon *> jobs;
  cudaStream_t own = nullptr, stream = nullptr;
  int tile = -1;
  fr::BatchScratch *bs = nullptr;
  std::mutex mu;
};

extern "C" {

int fr_batch_create(const fr_params *jobs, int njobs, fr_batch **out) {
  if (!jobs || !out) return fail(FR_ENULL, "null argument");
  if (njobs <= 0) return fail(FR_EINVAL_PARAM, "a batch needs at least one job");
  *out = nullptr;
  fr_batch *b = new fr_batch();
  if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return fail(FR_ECUDA, "cudaStreamCreate failed");
  }
  b->stream = b->own;
  for (int j = 0; j < njobs; j++) {
    fr_recon *r = nullptr;
    int rc = fr_create(&jobs[j], &r);
    if (rc == FR_OK) rc = fr_set_stream(r, b->stream);
    if (rc == FR_OK) rc = fr_setup(r);
    if (rc != FR_OK) {
      if (r) fr_destroy(r);
      for (fr_recon *q : b->jobs) fr_destroy(q);
      cudaStreamDestroy(b->own);
      delete b;
      return rc;
    }
    b->jobs.push_back(r);
  }
  *out = b;
  return FR_OK;
}

int fr_batch_destroy(fr_batch *b) {
  if (!b) return FR_OK;
  cudaStreamSynchronize(b->stream);
  delete b->bs;
  for (fr_recon *r : b->jobs) fr_destroy(r);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return FR_OK;
}

int fr_batch_set_stream(fr_batch *b, void *stream) {
  if (!b) return fail(FR_ENULL, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  b->stream = stream ? (cudaStream_t)stream : b->own;
  for (fr_recon *r : b->jobs) fr_set_stream(r, b->stream);
  return FR_OK;
}

}  // extern "C"

namespace fr {

// One caller at a time per handle: lock them in address order.
static int lock_handles(const std::vector<fr_recon *> &jobs,
                        std::vector<std::unique_lock<std::mutex>> &locks) {
  std::vector<fr_recon *> order(jobs);
  std::sort(order.begin(), order.end());
  if (std::adjacent_find(order.begin(), order.end()) != order.end())
    return fail(FR_EINVAL_PARAM, "a handle appears twice");
  for (fr_recon *r : order) locks.emplace_back(r->mu);
  return FR_OK;
}

// One round of a batched insertion: every participating job's InsertJob,
// its schedule, and per schedule the ordered work list of one launch.
struct RoundGroup {
  int tile = 0, max_mode = FR_MODE_NEAREST, maxN = 0;
  size_t off = 0, nwork = 0;   // byte offset and item count in the work buffer
};
struct RoundPlan {
  std::vector<InsertJob> hj;
  std::vector<int> owner, jt;
  std::vector<RoundGroup> groups;
  std::vector<unsigned char> work;   // every group's items, 16-byte aligned
};

static bool is_column(int tile) { return is_column_tile(tile); }

// Each job's schedule: the caller's pin, else the autotuner's measurement for
// its (N, mode, nsym), else the barrier-free column kernel.  Jobs that share
// a schedule share one persistent launch per round.
static int job_tile(const fr_recon *r, int tile_pref) {
  if (tile_pref != -1) return effective_tile(tile_pref, r->mode);
  const int t = tuned_tile(r->N, r->mode, r->nsym);
  return effective_tile(t != -1 ? t : default_tile(r->mode, r->N, r->nsym, 0), r->mode);
}

// Adds job r's InsertJob (its chunk's slices, rotations and weights in its
// scratch) to the plan, with the tile list of its schedule.
static void plan_add(RoundPlan &P, fr_recon *r, int owner, int np, int tile_pref) {
  InsertJob J = make_job(r, r->s_slices.as<float2>(), r->s_t3d.as<float>(), meta_view(r->d_meta, np).w,
                         np);
  const int tile = job_tile(r, tile_pref);
  if (tile != kTunedScatter && r->tiles_tile != tile) {
    if (is_column(tile))
      column_tiles(r->N, r->mode, r->p.corners, r->tiles, r->tx, r->ty, r->tz, &r->tile_dist);
    else gather_tiles(r->N, r->mode, tile, r->p.corners, r->tiles, r->tx, r->ty, r->tz);
    r->tiles_tile = tile;
    r->work_np = -1;
  }
  J.tiles_x = r->tx;
  J.tiles_y = r->ty;
  J.tiles_z = r->tz;
  P.hj.push_back(J);
  P.owner.push_back(owner);
  P.jt.push_back(tile);
}

// Builds each schedule group's work list.  Column items run slice-bucket-major
// (slice_bucket per job, so the CTAs in flight share a bucket's slices in L2)
// and within a bucket by estimated cost, heaviest first: the slices meeting a
// tile fall off with its distance from the origin (tiles are sorted by
// distance), times the slices in the item's block.
static void plan_groups(const std::vector<fr_recon *> &jobs, RoundPlan &P) {
  std::vector<int> tiles_used(P.jt);
  std::sort(tiles_used.begin(), tiles_used.end());
  tiles_used.erase(std::unique(tiles_used.begin(), tiles_used.end()), tiles_used.end());
  for (const int tile : tiles_used) {
    RoundGroup g;
    g.tile = tile;
    if (tile == kTunedScatter) { P.groups.push_back(g); continue; }
    const bool column = is_column(tile);
    std::vector<std::pair<double, int4>> items;
    for (size_t k = 0; k < P.hj.size(); k++) {
      if (P.jt[k] != tile) continue;
      const fr_recon *r = jobs[P.owner[k]];
      g.maxN = std::max(g.maxN, r->N);
      if (r->mode == FR_MODE_GAUSS5) g.max_mode = FR_MODE_GAUSS5;
      else if (g.max_mode != FR_MODE_GAUSS5 && r->mode != FR_MODE_NEAREST) g.max_mode = r->mode;
      const int nsl = P.hj[k].np * P.hj[k].nsym;
      const double nt = (double)r->tiles.size();
      const int bucket = slice_bucket(r->N, r->nsym);
      for (size_t t = 0; t < r->tiles.size(); t++) {
        const double frac = (double)t / std::max(1.0, nt);
        const double fall = 1.0 / (1.0 + 8.0 * std::cbrt(frac) * r->N / 16.0);
        if (column) {
          const int blk = column_block(r->tile_dist[t]);
          for (int s0 = 0; s0 < nsl; s0 += blk) {
            const int len = std::min(blk, nsl - s0);
            // bucket first (costs are below 1e4), then heaviest first
            items.push_back({1e12 * (s0 / bucket) - len * fall,
                             make_int4((int)k, r->tiles[t], s0, s0 + len)});
          }
        } else {
          items.push_back({-nsl * fall, make_int4((int)k, r->tiles[t], 0, 0)});
        }
      }
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const std::pair<double, int4> &a, const std::pair<double, int4> &c) {
                       return a.first < c.first;
                     });
    g.off = (P.work.size() + 15) & ~(size_t)15;
    g.nwork = items.size();
    const size_t isz = column ? sizeof(int4) : sizeof(int2);
    P.work.resize(g.off + isz * items.size());
    for (size_t i = 0; i < items.size(); i++) {
      if (column) memcpy(&P.work[g.off + i * isz], &items[i].second, isz);
      else {
        const int2 w2 = make_int2(items[i].second.x, items[i].second.y);
        memcpy(&P.work[g.off + i * isz], &w2, isz);
      }
    }
    P.groups.push_back(g);
  }
}

// Job table and work lists to the device (host sources are pageable
// vectors: the copies have taken them when cudaMemcpyAsync returns).
static int plan_upload(const RoundPlan &P, BatchScratch &bs, cudaStream_t st) {
  TRY(bs.d_jobs.ensure(sizeof(InsertJob) * std::max<size_t>(1, P.hj.size())));
  TRY(bs.d_counter.ensure(sizeof(int)));
  TRY(bs.d_work.ensure(std::max<size_t>(16, P.work.size())));
  TRY(bs.ring.upload(bs.d_jobs.p, P.hj.data(), sizeof(InsertJob) * P.hj.size(), st));
  if (!P.work.empty()) TRY(bs.ring.upload(bs.d_work.p, P.work.data(), P.work.size(), st));
  return FR_OK;
}

// Device work of the round: per schedule group one persistent launch (or the
// scatter), then the face taps.  Kernels and memsets only.
static int plan_launch(const RoundPlan &P, BatchScratch &bs, cudaStream_t st) {
  const InsertJob *d_jobs = bs.d_jobs.as<InsertJob>();
  for (const RoundGroup &g : P.groups) {
    if (g.tile == kTunedScatter) {
      for (size_t k = 0; k < P.hj.size(); k++)
        if (P.jt[k] == g.tile) TRY(run_scatter(P.hj[k], false, st));
      continue;
    }
    const void *w = (const unsigned char *)bs.d_work.p + g.off;
    if (g.tile == kPixelTile)
      CU(launch_pixel(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, bs.d_counter.as<int>(),
                      g.maxN, st));
    else if (g.tile == kColumn3Tile)
      CU(launch_column3(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, bs.d_counter.as<int>(),
                        g.maxN, st));
    else if (g.tile == kColumnTile)
      CU(launch_column(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, bs.d_counter.as<int>(),
                       g.max_mode, st));
    else
      CU(launch_gather(d_jobs, P.hj.data(), (int)P.hj.size(), (const int2 *)w, (int)g.nwork,
                       g.tile, bs.d_counter.as<int>(), g.max_mode, st));
    for (size_t k = 0; k < P.hj.size(); k++)
      if (P.jt[k] == g.tile) TRY(run_scatter(P.hj[k], true, st));
  }
  return FR_OK;
}

// Inserts, for every job, counts[j] particles through the caller pipeline;
// all jobs' insertion work goes through one persistent launch per schedule
// per round.  Every job runs on `st` for the duration of the call.
static int batch_insert(std::vector<fr_recon *> &jobs, BatchScratch &bs, int tile_pref,
                        cudaStream_t st, const float *const *imgs, const int *boxes,
                        const int *counts, const fr_particle *const *meta) {
  const int nj = (int)jobs.size();
  struct StreamSwap {
    std::vector<fr_recon *> &j;
    std::vector<cudaStream_t> saved;
    StreamSwap(std::vector<fr_recon *> &jj, cudaStream_t s) : j(jj) {
      for (fr_recon *r : j) { saved.push_back(r->stream); r->stream = s; }
    }
    ~StreamSwap() { for (size_t i = 0; i < j.size(); i++) j[i]->stream = saved[i]; }
  } swap(jobs, st);
  bool host_src = false;
  for (int j = 0; j < nj; j++) {
    TRY(check_state(jobs[j]));
    if (counts[j] < 0 || (counts[j] > 0 && (boxes[j] <= 0 || !imgs[j] || !meta[j])))
      return fail(FR_EINVAL_PARAM, "job %d: bad particle count, box or buffers", j);
    if (counts[j] > 0 && !is_device_ptr(imgs[j])) host_src = true;
  }
  // Work goes to `st` after each handle's and the scratch's earlier work on
  // other streams; the call returns once everything is enqueued.
  if (!bs.done) CU(cudaEventCreateWithFlags(&bs.done, cudaEventDisableTiming));
  if (bs.last && bs.last != st) CU(cudaStreamWaitEvent(st, bs.done, 0));
  for (int j = 0; j < nj; j++) TRY(stream_enter(jobs[j], st));
  // Rounds of at most `chunk` particles per job, so scratch stays bounded.
  const int chunk = kBatchChunk;
  int rounds = 0;
  for (int j = 0; j < nj; j++) rounds = std::max(rounds, (counts[j] + chunk - 1) / chunk);
  for (int rd = 0; rd < rounds; rd++) {
    RoundPlan P;
    for (int j = 0; j < nj; j++) {
      fr_recon *r = jobs[j];
      const int p0 = rd * chunk;
      const int c = std::max(0, std::min(chunk, counts[j] - p0));
      if (c == 0) continue;
      const int box = boxes[j];
      const void *d_raw = nullptr;
      TRY(to_device(imgs[j] + (size_t)p0 * box * box, sizeof(float) * (size_t)c * box * box,
                    r->s_in, st, &d_raw));
      TRY(prologue_chunk(r, (const float *)d_raw, c, box, meta[j] + p0));
      plan_add(P, r, j, c, tile_pref);
    }
    if (P.hj.empty()) continue;
    plan_groups(jobs, P);
    TRY(plan_upload(P, bs, st));
    TRY(plan_launch(P, bs, st));
  }
  CU(cudaEventRecord(bs.done, st));
  bs.last = st;
  for (int j = 0; j < nj; j++) TRY(stream_leave(jobs[j], st));
  if (host_src) CU(cudaStreamSynchronize(st));   // host images may be pinned: read them before returning
  return FR_OK;
}

}  // namespace fr

extern "C" {

int fr_batch_insert_particles(fr_batch *b, const float *const *imgs, const int *boxes,
                              const int *counts, const fr_particle *const *meta) {
  if (!b || !imgs || !boxes || !counts || !meta) return fail(FR_ENULL, "null argument");
  std::lock_guard<std::mutex> lk(b->mu);
  if (!b->bs) b->bs = new BatchScratch();
  return batch_insert(b->jobs, *b->bs, b->tile, b->stream, imgs, boxes, counts, meta);
}

int fr_insert_particles_multi(fr_recon *const *handles, int nh, const float *const *imgs,
                              const int *boxes, const int *counts,
                              const fr_particle *const *meta, void *stream) {
  if (!handles || nh <= 0 || !imgs || !boxes || !counts || !meta)
    return fail(FR_ENULL, "null argument");
  std::vector<fr_recon *> jobs(handles, handles + nh);
  for (fr_recon *r : jobs)
    if (!r) return fail(FR_ENULL, "null reconstructor handle");
  std::vector<std::unique_lock<std::mutex>> locks;
  TRY(lock_handles(jobs, locks));
  static thread_local BatchScratch bs;
  cudaStream_t st = stream ? (cudaStream_t)stream : jobs[0]->stream;
  return batch_insert(jobs, bs, -1, st, imgs, boxes, counts, meta);
}

// ------------------------------------------------------------------ graphs
// A batched insertion round of fixed shapes captured once as a CUDA graph.
// The graph owns the images' device slots and every job's chunk scratch (so
// later calls on the same handles cannot move them); a replay writes the
// particles' metadata into pinned staging, copies it and the images in, and
// launches the graph.
}  // extern "C"

namespace fr {
struct JobBufs {
  DevBuf img, slices, mean, spec, t3d, img2, meta;
  void swap_with(fr_recon *r) {
    std::swap(img, r->s_img);
    std::swap(slices, r->s_slices);
    std::swap(mean, r->s_mean);
    std::swap(spec, r->s_spec);
    std::swap(t3d, r->s_t3d);
    std::swap(img2, r->s_img2);
    std::swap(meta, r->s_meta);
  }
  void release() {
    for (DevBuf *b : {&img, &slices, &mean, &spec, &t3d, &img2, &meta}) b->release();
  }
};
}  // namespace fr

struct fr_graph {
  std::vector<fr_recon *> jobs;
  cudaStream_t st = nullptr;
  std::vector<int> boxes, counts, ctf;
  std::vector<fr::DevBuf> slots;
  std::vector<fr::JobBufs> bufs;
  std::vector<size_t> meta_off;
  size_t meta_bytes = 0;
  unsigned char *pinned[2] = {nullptr, nullptr};
  cudaEvent_t staged[2] = {nullptr, nullptr};
  bool staged_used[2] = {false, false};
  int next = 0;
  long long kernels = 0;          // this library's kernels per replay
  fr::BatchScratch bs;
  fr::RoundPlan plan;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::mutex mu;
};

namespace fr {

static void graph_free(fr_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto &s : g->slots) s.release();
  for (auto &jb : g->bufs) jb.release();
  g->bs.d_jobs.release();
  g->bs.d_work.release();
  g->bs.d_counter.release();
  for (int k = 0; k < 2; k++) {
    if (g->pinned[k]) cudaFreeHost(g->pinned[k]);
    if (g->staged[k]) cudaEventDestroy(g->staged[k]);
  }
  delete g;
}

static int graph_create(const std::vector<fr_recon *> &jobs, cudaStream_t st, int tile_pref,
                        const int *boxes, const int *counts, const int *ctf, fr_graph **out) {
  const int nj = (int)jobs.size();
  int total = 0;
  for (int j = 0; j < nj; j++) {
    TRY(check_state(jobs[j]));
    if (counts[j] < 0 || counts[j] > kBatchChunk || (counts[j] > 0 && boxes[j] <= 0))
      return fail(FR_EINVAL_PARAM, "job %d: count must be in [0, %d] with a positive box", j,
                  kBatchChunk);
    total += counts[j];
  }
  if (total == 0) return fail(FR_EINVAL_PARAM, "a graph needs at least one particle");
  fr_graph *g = new fr_graph();
  g->jobs = jobs;
  g->st = st;
  g->boxes.assign(boxes, boxes + nj);
  g->counts.assign(counts, counts + nj);
  g->ctf.assign(nj, 0);
  for (int j = 0; ctf && j < nj; j++) g->ctf[j] = ctf[j] ? 1 : 0;
  g->slots.resize(nj);
  g->bufs.resize(nj);
  g->meta_off.assign(nj, 0);
  for (int j = 0; j < nj; j++) {
    g->meta_off[j] = g->meta_bytes;
    g->meta_bytes += (prologue_meta_bytes(counts[j]) + 15) & ~(size_t)15;
  }
  std::vector<cudaStream_t> saved;
  for (fr_recon *r : jobs) { saved.push_back(r->stream); r->stream = st; }
  // Sizing pass on the graph-owned scratch (swapped into the handles): a
  // prologue of weight-0 particles allocates every buffer and FFT plan the
  // capture uses, so the captured work allocates nothing.
  for (int j = 0; j < nj; j++) g->bufs[j].swap_with(jobs[j]);
  int rc = FR_OK;
  for (int j = 0; j < nj && rc == FR_OK; j++) rc = stream_enter(jobs[j], st);
  std::vector<unsigned char> blk(std::max<size_t>(16, g->meta_bytes));
  for (int j = 0; j < nj && rc == FR_OK; j++) {
    fr_recon *r = jobs[j];
    const int n = counts[j];
    if (n == 0) continue;
    const size_t bytes = sizeof(float) * (size_t)n * boxes[j] * boxes[j];
    if ((rc = g->slots[j].ensure(bytes)) != FR_OK) break;
    if (cudaMemsetAsync(g->slots[j].p, 0, bytes, st) != cudaSuccess) {
      rc = fail(FR_ECUDA, "memset failed");
      break;
    }
    std::vector<fr_particle> parts(n);
    for (fr_particle &m : parts) {
      memset(&m, 0, sizeof m);
      m.rot[0] = m.rot[4] = m.rot[8] = 1.0f;
      m.defocus = g->ctf[j] ? 1.5f : 0.0f;
      m.voltage = 300.0f;
      m.cs = 2.7f;
      m.apix = 1.0f;
      m.ampcont = 10.0f;
    }
    prologue_meta(r->N, n, parts.data(), blk.data() + g->meta_off[j]);
    if ((rc = prologue_upload(r, n, blk.data() + g->meta_off[j], st)) != FR_OK) break;
    if ((rc = prologue_device(r, g->slots[j].as<float>(), n, boxes[j], g->ctf[j])) != FR_OK) break;
    plan_add(g->plan, r, j, n, tile_pref);
  }
  if (rc == FR_OK) {
    plan_groups(jobs, g->plan);
    rc = plan_upload(g->plan, g->bs, st);
  }
  if (rc == FR_OK && cudaStreamSynchronize(st) != cudaSuccess)
    rc = fail(FR_ECUDA, "sizing pass failed: %s", cudaGetErrorString(cudaGetLastError()));
  // Capture: the device halves of the prologues and the round's launches.
  if (rc == FR_OK) {
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
      rc = fail(FR_ECUDA, "cudaStreamBeginCapture failed");
    } else {
      const long long noted = launches_noted();
      for (int j = 0; j < nj && rc == FR_OK; j++)
        if (counts[j] > 0) {
          jobs[j]->d_meta = jobs[j]->s_meta.as<unsigned char>();   // the graph's block
          rc = prologue_device(jobs[j], g->slots[j].as<float>(), counts[j], boxes[j], g->ctf[j]);
        }
      if (rc == FR_OK) rc = plan_launch(g->plan, g->bs, st);
      const cudaError_t e = cudaStreamEndCapture(st, &g->graph);
      if (rc == FR_OK && e != cudaSuccess)
        rc = fail(FR_ECUDA, "stream capture failed: %s", cudaGetErrorString(e));
      g->kernels = launches_noted() - noted;
    }
  }
  if (rc == FR_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
    rc = fail(FR_ECUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(cudaGetLastError()));
  for (int j = 0; j < nj; j++) g->bufs[j].swap_with(jobs[j]);
  for (int k = 0; k < 2 && rc == FR_OK; k++) {
    if (cudaHostAlloc((void **)&g->pinned[k], std::max<size_t>(16, g->meta_bytes),
                      cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->staged[k], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(FR_ENOMEM, "pinned staging allocation failed");
  }
  for (int j = 0; j < nj; j++) {
    stream_leave(jobs[j], st);
    jobs[j]->stream = saved[j];
  }
  if (rc != FR_OK) {
    cudaGetLastError();
    graph_free(g);
    return rc;
  }
  *out = g;
  return FR_OK;
}

}  // namespace fr

extern "C" {

int fr_graph_create(fr_recon *const *handles, int nh, const int *boxes, const int *counts,
                    const int *ctf, void *stream, fr_graph **out) {
  if (!handles || nh <= 0 || !boxes || !counts || !out) return fail(FR_ENULL, "null argument");
  *out = nullptr;
  std::vector<fr_recon *> jobs(handles, handles + nh);
  for (fr_recon *r : jobs)
    if (!r) return fail(FR_ENULL, "null reconstructor handle");
  std::vector<std::unique_lock<std::mutex>> locks;
  TRY(lock_handles(jobs, locks));
  cudaStream_t st = stream ? (cudaStream_t)stream : jobs[0]->stream;
  return graph_create(jobs, st, -1, boxes, counts, ctf, out);
}

int fr_batch_graph_create(fr_batch *b, const int *boxes, const int *counts, const int *ctf,
                          fr_graph **out) {
  if (!b || !boxes || !counts || !out) return fail(FR_ENULL, "null argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lk(b->mu);
  std::vector<std::unique_lock<std::mutex>> locks;
  TRY(lock_handles(b->jobs, locks));
  return graph_create(b->jobs, b->stream, b->tile, boxes, counts, ctf, out);
}

int fr_graph_slot(fr_graph *g, int job, float **d_images) {
  if (!g || !d_images) return fail(FR_ENULL, "null argument");
  if (job < 0 || job >= (int)g->slots.size()) return fail(FR_EINVAL_PARAM, "job %d out of range", job);
  *d_images = g->slots[job].as<float>();
  return FR_OK;
}

int fr_graph_launch(fr_graph *g, const float *const *imgs, const fr_particle *const *meta) {
  if (!g || !meta) return fail(FR_ENULL, "null argument");
  std::lock_guard<std::mutex> glk(g->mu);
  std::vector<std::unique_lock<std::mutex>> locks;
  TRY(lock_handles(g->jobs, locks));
  for (fr_recon *r : g->jobs) TRY(check_state(r));
  cudaStream_t st = g->st;
  const int nj = (int)g->counts.size();
  const int k = g->next;
  // this staging block was last read by the copies two replays ago
  if (g->staged_used[k]) CU(cudaEventSynchronize(g->staged[k]));
  for (int j = 0; j < nj; j++) {
    const int n = g->counts[j];
    if (n == 0) continue;
    if (!meta[j]) return fail(FR_ENULL, "job %d: null metadata", j);
    if (imgs && !imgs[j]) return fail(FR_ENULL, "job %d: null images", j);
    const bool any = prologue_meta(g->jobs[j]->N, n, meta[j], g->pinned[k] + g->meta_off[j]);
    if ((int)any != g->ctf[j])
      return fail(FR_EINVAL_PARAM, "job %d: the graph was captured %s a CTF phase flip", j,
                  g->ctf[j] ? "with" : "without");
  }
  g->next ^= 1;
  for (fr_recon *r : g->jobs) TRY(stream_enter(r, st));
  bool host_src = false;
  for (int j = 0; j < nj; j++) {
    const int n = g->counts[j];
    if (n == 0) continue;
    CU(cudaMemcpyAsync(g->bufs[j].meta.p, g->pinned[k] + g->meta_off[j], prologue_meta_bytes(n),
                       cudaMemcpyHostToDevice, st));
  }
  CU(cudaEventRecord(g->staged[k], st));
  g->staged_used[k] = true;
  for (int j = 0; imgs && j < nj; j++) {
    const int n = g->counts[j];
    if (n == 0 || imgs[j] == g->slots[j].as<float>()) continue;
    const size_t bytes = sizeof(float) * (size_t)n * g->boxes[j] * g->boxes[j];
    host_src |= !is_device_ptr(imgs[j]);
    CU(cudaMemcpyAsync(g->slots[j].p, imgs[j], bytes, cudaMemcpyDefault, st));
  }
  CU(cudaGraphLaunch(g->exec, st));
  note_launch((int)g->kernels);
  for (fr_recon *r : g->jobs) TRY(stream_leave(r, st));
  if (host_src) CU(cudaStreamSynchronize(st));   // host images may be pinned: read them first
  return FR_OK;
}

int fr_graph_destroy(fr_graph *g) {
  if (!g) return FR_OK;
  {
    std::lock_guard<std::mutex> lk(g->mu);
    cudaStreamSynchronize(g->st);
  }
  graph_free(g);
  return FR_OK;
}

int fr_batch_finish(fr_batch *b, int job, int doift, float *out, float *normout) {
  if (!b) return fail(FR_ENULL, "null batch");
  if (job < 0 || job >= (int)b->jobs.size()) return fail(FR_EINVAL_PARAM, "job %d out of range", job);
  return fr_finish(b->jobs[job], doift, out, normout);
}

int fr_batch_get_accumulators(fr_batch *b, int job, float *data, float *norm) {
  if (!b) return fail(FR_ENULL, "null batch");
  if (job < 0 || job >= (int)b->jobs.size()) return fail(FR_EINVAL_PARAM, "job %d out of range", job);
  return fr_get_accumulators(b->jobs[job], data, norm);
}

int fr_set_tile(int N, int mode, int nsym, int tile) {
  if (tile != kTunedScatter && (tile < -1 || tile > kPixelTile))
    return fail(FR_EINVAL_PARAM, "tile %d out of range", tile);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (tile == -1) g_tuned.erase(std::make_tuple(N, mode, nsym));
  else g_tuned[std::make_tuple(N, mode, nsym)] = tile;
  return FR_OK;
}

// Measures the gather schedule with every tile shape, and the scatter
// schedule, on random slices of size N through random orientations; records
// the fastest for (N, mode, nsym).  tile_out: chosen tile (-2 = scatter);
// ms_out[kPixelTile+2]: per-candidate milliseconds (register tiles 0-3,
// staged column 4, barrier-free column 5, pixel-major 6 (gauss_5: -1), then
// scatter).
int fr_autotune(int N, int mode, int nsym, int nparticles, int *tile_out, float *ms_out) {
  if (nparticles <= 0) return fail(FR_EINVAL_PARAM, "nparticles must be positive");
  fr_params p;
  memset(&p, 0, sizeof p);
  p.nx = p.ny = p.nz = N;
  p.mode = mode;
  snprintf(p.sym, sizeof p.sym, "c%d", std::max(1, nsym));
  fr_recon *r = nullptr;
  TRY(fr_create(&p, &r));
  int rc = fr_setup(r);
  std::vector<float> sl(slice_floats(N) * (size_t)nparticles), rot(9 * (size_t)nparticles),
      w(nparticles, 1.0f);
  std::mt19937 rng(1234);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (auto &v : sl) v = nd(rng);
  for (int i = 0; i < nparticles; i++) {
    float q[4], n2 = 0;
    for (float &c : q) { c = nd(rng); n2 += c * c; }
    const float s = 1.0f / std::sqrt(n2);
    for (float &c : q) c *= s;
    const double e0 = q[0], e1 = q[1], e2 = q[2], e3 = q[3];
    float *m = &rot[9 * i];
    m[0] = (float)(e0 * e0 + e1 * e1 - e2 * e2 - e3 * e3);
    m[1] = (float)(2.0 * (e1 * e2 + e0 * e3));
    m[2] = (float)(2.0 * (e1 * e3 - e0 * e2));
    m[3] = (float)(2.0 * (e2 * e1 - e0 * e3));
    m[4] = (float)(e0 * e0 - e1 * e1 + e2 * e2 - e3 * e3);
    m[5] = (float)(2.0 * (e2 * e3 + e0 * e1));
    m[6] = (float)(2.0 * (e3 * e1 + e0 * e2));
    m[7] = (float)(2.0 * (e3 * e2 - e0 * e1));
    m[8] = (float)(e0 * e0 - e1 * e1 - e2 * e2 + e3 * e3);
  }
  float best = 1e30f;
  int best_tile = kTunedScatter;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // inputs staged on the device so the timing covers the insertion only
  DevBuf ds, dr, dw;
  if (rc == FR_OK) rc = ds.ensure(sizeof(float) * sl.size());
  if (rc == FR_OK) rc = dr.ensure(sizeof(float) * rot.size());
  if (rc == FR_OK) rc = dw.ensure(sizeof(float) * w.size());
  if (rc == FR_OK &&
      (cudaMemcpy(ds.p, sl.data(), sizeof(float) * sl.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(dr.p, rot.data(), sizeof(float) * rot.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(dw.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice) != cudaSuccess))
    rc = fail(FR_ECUDA, "autotune: staging failed");
  int measured = 0;
  for (int cand = 0; cand <= kPixelTile + 1 && rc == FR_OK; cand++) {
    const bool scatter = cand == kPixelTile + 1;
    if (!scatter && effective_tile(cand, mode) != cand) {   // no pixel-major gauss_5
      if (ms_out) ms_out[cand] = -1.0f;
      continue;
    }
    r->tile = scatter ? -1 : cand;
    const int sched = scatter ? FR_SCHED_SCATTER : FR_SCHED_GATHER;
    // one warm-up call, then one timed call; a schedule that cannot run this
    // shape (a launch error) is skipped with ms = -1
    float ms = -1.0f;
    int crc = fr_insert_slices(r, ds.as<float>(), nparticles, dr.as<float>(), dw.as<float>(),
                               nullptr, 0, nullptr, sched);
    if (crc == FR_OK) {
      cudaEventRecord(e0, r->stream);
      crc = fr_insert_slices(r, ds.as<float>(), nparticles, dr.as<float>(), dw.as<float>(),
                             nullptr, 0, nullptr, sched);
      cudaEventRecord(e1, r->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) crc = FR_ECUDA;
      if (crc == FR_OK) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (crc != FR_OK) {
      cudaGetLastError();
      ms = -1.0f;
    } else {
      measured++;
    }
    if (ms_out) ms_out[cand] = ms;
    if (ms >= 0 && ms < best) { best = ms; best_tile = scatter ? kTunedScatter : cand; }
  }
  if (rc == FR_OK && measured == 0) rc = fail(FR_ECUDA, "autotune: no schedule ran");
  ds.release();
  dr.release();
  dw.release();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fr_destroy(r);
  if (rc != FR_OK) return rc;
  fr_set_tile(N, mode, nsym, best_tile);
  if (tile_out) *tile_out = best_tile;
  return FR_OK;
}

}  // extern "C"
