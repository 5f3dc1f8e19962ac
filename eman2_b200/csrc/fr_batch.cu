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

int tuned_tile(int N, int mode, int nsym) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(std::make_tuple(N, mode, nsym));
  return it == g_tuned.end() ? -1 : it->second;
}

int default_tile(int mode, int N, int nsym, int np) {
  (void)nsym; (void)np; (void)N; (void)mode;
  return kColumn3Tile;   // the barrier-free column kernel unless the autotuner measured otherwise
}

}  // namespace fr

// ------------------------------------------------------------------ batch
namespace fr {
// Device copies of a batched launch's job table and work list.
struct BatchScratch {
  DevBuf d_jobs, d_work, d_counter;
  cudaEvent_t done = nullptr;     // after the last launch that read this scratch
  cudaStream_t last = nullptr;
  ~BatchScratch() {
    if (done) { cudaEventSynchronize(done); cudaEventDestroy(done); }
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

// Inserts, for every job, counts[j] particles through the caller pipeline;
// all jobs' insertion work goes through one persistent launch per round.
// Every job runs on `st` for the duration of the call.
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
  const int chunk = 4096;
  int rounds = 0;
  for (int j = 0; j < nj; j++) rounds = std::max(rounds, (counts[j] + chunk - 1) / chunk);
  // Each job's schedule: the caller's pin, else the autotuner's measurement
  // for its (N, mode, nsym), else the barrier-free column kernel.  Jobs that
  // share a schedule share one persistent launch per round.
  auto job_tile = [&](const fr_recon *r) {
    if (tile_pref != -1) return tile_pref;
    const int t = tuned_tile(r->N, r->mode, r->nsym);
    return t != -1 ? t : default_tile(r->mode, r->N, r->nsym, 0);
  };
  for (int rd = 0; rd < rounds; rd++) {
    std::vector<InsertJob> hj;
    std::vector<int> owner, jt;
    for (int j = 0; j < nj; j++) {
      fr_recon *r = jobs[j];
      const int p0 = rd * chunk;
      const int c = std::max(0, std::min(chunk, counts[j] - p0));
      if (c == 0) continue;
      const int box = boxes[j];
      const float *src = imgs[j] + (size_t)p0 * box * box;
      const void *d_raw = nullptr;
      TRY(to_device(src, sizeof(float) * (size_t)c * box * box, r->s_in, st, &d_raw));
      TRY(prologue_chunk(r, (const float *)d_raw, c, box, meta[j] + p0));
      InsertJob J = make_job(r, r->s_slices.as<float2>(), r->s_t3d.as<float>(), r->s_w.as<float>(), c);
      const int tile = job_tile(r);
      if (tile != kTunedScatter && r->tiles_tile != tile) {
        if (tile == kColumnTile || tile == kColumn3Tile)
          column_tiles(r->N, r->mode, r->p.corners, r->tiles, r->tx, r->ty, r->tz, &r->tile_dist);
        else gather_tiles(r->N, r->mode, tile, r->p.corners, r->tiles, r->tx, r->ty, r->tz);
        r->tiles_tile = tile;
        r->work_np = -1;
      }
      J.tiles_x = r->tx;
      J.tiles_y = r->ty;
      J.tiles_z = r->tz;
      hj.push_back(J);
      owner.push_back(j);
      jt.push_back(tile);
    }
    if (hj.empty()) continue;
    TRY(bs.d_jobs.ensure(sizeof(InsertJob) * hj.size()));
    TRY(bs.d_counter.ensure(sizeof(int)));
    CU(cudaMemcpyAsync(bs.d_jobs.p, hj.data(), sizeof(InsertJob) * hj.size(),
                       cudaMemcpyHostToDevice, st));
    std::vector<int> tiles_used(jt);
    std::sort(tiles_used.begin(), tiles_used.end());
    tiles_used.erase(std::unique(tiles_used.begin(), tiles_used.end()), tiles_used.end());
    for (const int tile : tiles_used) {
      if (tile == kTunedScatter) {
        for (size_t k = 0; k < hj.size(); k++)
          if (jt[k] == tile) TRY(run_scatter(hj[k], false, st));
        continue;
      }
      const bool column = tile == kColumnTile || tile == kColumn3Tile;
      int max_mode = FR_MODE_NEAREST, maxN = 0;
      // Order the group's work items slice-bucket-major (slice_bucket per
      // job, so the CTAs in flight share a bucket's slices in
      // L2), and within a bucket by estimated cost, heaviest first: the slices
      // meeting a tile fall off with its distance from the origin (tiles are
      // sorted by distance), times the slices in the item's block.
      std::vector<std::pair<double, int4>> items;
      std::vector<int> bucket_of;
      for (size_t k = 0; k < hj.size(); k++) {
        if (jt[k] != tile) continue;
        fr_recon *r = jobs[owner[k]];
        maxN = std::max(maxN, r->N);
        if (r->mode == FR_MODE_GAUSS5) max_mode = FR_MODE_GAUSS5;
        else if (max_mode != FR_MODE_GAUSS5 && r->mode != FR_MODE_NEAREST) max_mode = r->mode;
        const int nsl = hj[k].np * hj[k].nsym;
        const double nt = (double)r->tiles.size();
        for (size_t t = 0; t < r->tiles.size(); t++) {
          const double frac = (double)t / std::max(1.0, nt);
          const double fall = 1.0 / (1.0 + 8.0 * std::cbrt(frac) * r->N / 16.0);
          if (column) {
            const int blk = column_block(r->tile_dist[t]);
            for (int s0 = 0; s0 < nsl; s0 += blk) {
              const int len = std::min(blk, nsl - s0);
              items.push_back({-len * fall, make_int4((int)k, r->tiles[t], s0, s0 + len)});
            bucket_of.push_back(s0 / slice_bucket(r->N, r->nsym));
            }
          } else {
            items.push_back({-nsl * fall, make_int4((int)k, r->tiles[t], 0, 0)});
            bucket_of.push_back(0);
          }
        }
      }
      // bucket first (costs are below 1e4), then heaviest first
      for (size_t i = 0; i < items.size(); i++) items[i].first += 1e12 * bucket_of[i];
      std::stable_sort(items.begin(), items.end(),
                       [](const std::pair<double, int4> &a, const std::pair<double, int4> &c) {
                         return a.first < c.first;
                       });
      if (column) {
        std::vector<int4> work(items.size());
        for (size_t i = 0; i < items.size(); i++) work[i] = items[i].second;
        TRY(bs.d_work.ensure(sizeof(int4) * std::max<size_t>(1, work.size())));
        CU(cudaMemcpyAsync(bs.d_work.p, work.data(), sizeof(int4) * work.size(),
                           cudaMemcpyHostToDevice, st));
        if (tile == kColumn3Tile)
          CU(launch_column3(bs.d_jobs.as<InsertJob>(), bs.d_work.as<int4>(), (int)work.size(),
                            kColumnBlock, bs.d_counter.as<int>(), maxN, st));
        else
          CU(launch_column(bs.d_jobs.as<InsertJob>(), bs.d_work.as<int4>(), (int)work.size(),
                           kColumnBlock, bs.d_counter.as<int>(), max_mode, st));
      } else {
        std::vector<int2> work(items.size());
        for (size_t i = 0; i < items.size(); i++) work[i] = make_int2(items[i].second.x, items[i].second.y);
        TRY(bs.d_work.ensure(sizeof(int2) * std::max<size_t>(1, work.size())));
        CU(cudaMemcpyAsync(bs.d_work.p, work.data(), sizeof(int2) * work.size(),
                           cudaMemcpyHostToDevice, st));
        CU(launch_gather(bs.d_jobs.as<InsertJob>(), hj.data(), (int)hj.size(), bs.d_work.as<int2>(),
                         (int)work.size(), tile, bs.d_counter.as<int>(), max_mode, st));
      }
      for (size_t k = 0; k < hj.size(); k++)
        if (jt[k] == tile) TRY(run_scatter(hj[k], true, st));
    }
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
  // One caller at a time per handle: lock them in address order.
  std::vector<fr_recon *> order(jobs);
  std::sort(order.begin(), order.end());
  order.erase(std::unique(order.begin(), order.end()), order.end());
  if (order.size() != jobs.size()) return fail(FR_EINVAL_PARAM, "a handle appears twice");
  std::vector<std::unique_lock<std::mutex>> locks;
  for (fr_recon *r : order) locks.emplace_back(r->mu);
  static thread_local BatchScratch bs;
  cudaStream_t st = stream ? (cudaStream_t)stream : jobs[0]->stream;
  return batch_insert(jobs, bs, -1, st, imgs, boxes, counts, meta);
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
  if (tile != kTunedScatter && (tile < -1 || tile > kColumn3Tile))
    return fail(FR_EINVAL_PARAM, "tile %d out of range", tile);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (tile == -1) g_tuned.erase(std::make_tuple(N, mode, nsym));
  else g_tuned[std::make_tuple(N, mode, nsym)] = tile;
  return FR_OK;
}

// Measures the gather schedule with every tile shape, and the scatter
// schedule, on random slices of size N through random orientations; records
// the fastest for (N, mode, nsym).  tile_out: chosen tile (-2 = scatter);
// ms_out[kColumn3Tile+2]: per-candidate milliseconds (register tiles 0-3,
// staged column 4, barrier-free column 5, then scatter).
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
  for (int cand = 0; cand <= kColumn3Tile + 1 && rc == FR_OK; cand++) {
    const bool scatter = cand == kColumn3Tile + 1;
    r->tile = scatter ? -1 : cand;
    const int sched = scatter ? FR_SCHED_SCATTER : FR_SCHED_GATHER;
    // one warm-up call, then one timed call
    rc = fr_insert_slices(r, sl.data(), nparticles, rot.data(), w.data(), nullptr, 0, nullptr, sched);
    if (rc != FR_OK) break;
    // stage inputs on the device so the timing covers the insertion only
    float ms = 0;
    {
      DevBuf ds, dr, dw;
      if ((rc = ds.ensure(sizeof(float) * sl.size())) != FR_OK) break;
      if ((rc = dr.ensure(sizeof(float) * rot.size())) != FR_OK) break;
      if ((rc = dw.ensure(sizeof(float) * w.size())) != FR_OK) break;
      cudaMemcpy(ds.p, sl.data(), sizeof(float) * sl.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(dr.p, rot.data(), sizeof(float) * rot.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(dw.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice);
      cudaEventRecord(e0, r->stream);
      rc = fr_insert_slices(r, ds.as<float>(), nparticles, dr.as<float>(), dw.as<float>(), nullptr,
                            0, nullptr, sched);
      cudaEventRecord(e1, r->stream);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      ds.release();
      dr.release();
      dw.release();
    }
    if (ms_out) ms_out[cand] = ms;
    if (ms < best) { best = ms; best_tile = scatter ? kTunedScatter : cand; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  fr_destroy(r);
  if (rc != FR_OK) return rc;
  fr_set_tile(N, mode, nsym, best_tile);
  if (tile_out) *tile_out = best_tile;
  return FR_OK;
}

}  // extern "C"
