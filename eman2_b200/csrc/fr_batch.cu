// fr_batch.cu -- many reconstructions in one persistent insertion launch, and
// the tile/schedule autotuner.
//
// A batch holds independent FourierReconstructor states (uneven N, modes and
// symmetries: even/odd half maps, heterogeneity classes).  Each insert call
// runs one prologue per group of jobs of equal (N, box) on the batch
// stream, then per schedule ONE persistent insertion launch whose work list
// interleaves all its jobs' (tile, slice block) items, heaviest first, and one
// launch of their face taps (or one scatter launch over all its jobs' slices).
#include <algorithm>
#include <climits>
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
// Scratch of one prologue group (see ProGroup), with the group's own FFT
// plans: the scratch, not a member handle, owns them, so a batched call
// leaves no plans behind on the handles it served and a captured graph's
// transforms use plans and a work area that only the graph holds.
struct ProBufs {
  DevBuf img, slices, spec, t3d, img2;
  std::unique_ptr<PlanCache> plans;
  ProScratch view() { return {&img, &slices, &spec, &t3d, &img2}; }
  PlanCache &fft() {
    if (!plans) plans.reset(new PlanCache());
    return *plans;
  }
  void release() {
    for (DevBuf *b : {&img, &slices, &spec, &t3d, &img2}) b->release();
    plans.reset();
  }
};

// Device copies of a batched launch's job table and work list, the round's
// metadata block and the prologue groups' scratch.
struct BatchScratch {
  DevBuf d_jobs, d_work, d_counter, d_meta;
  std::vector<ProBufs> gbufs;
  PinnedRing ring;
  cudaEvent_t done = nullptr;     // after the last launch that read this scratch
  cudaStream_t last = nullptr;
  void release() {
    if (done) { cudaEventSynchronize(done); cudaEventDestroy(done); done = nullptr; }
    for (DevBuf *b : {&d_jobs, &d_work, &d_counter, &d_meta}) b->release();
    for (ProBufs &g : gbufs) g.release();
    gbufs.clear();
    ring.release();
  }
  ~BatchScratch() { release(); }
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
  // (job, slice) units of the group's scatter, or of its face taps after a
  // gather launch: offset in the work buffer, count, largest pixel (rim) count
  size_t units_off = 0, nunits = 0;
  int max_px = 0;
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

// Adds job r's InsertJob (its chunk's np slices, composed rotations and
// weights) to the plan, with the tile list of its schedule.
static void plan_add(RoundPlan &P, fr_recon *r, int owner, int np, int tile_pref,
                     const float2 *slices, const float *t3d, const float *pw) {
  InsertJob J = make_job(r, slices, t3d, pw, np);
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

// Appends the (job, slice) units of group g's jobs to the work buffer: every
// slice for a scatter group, every slice of a job with rim pixels for the
// face taps that follow a gather launch.
static void plan_units(RoundPlan &P, RoundGroup &g, bool edge) {
  std::vector<int2> u;
  int mx = 0;
  for (size_t k = 0; k < P.hj.size(); k++) {
    if (P.jt[k] != g.tile) continue;
    const InsertJob &J = P.hj[k];
    const int px = edge ? J.nrim : J.N * (J.N / 2 + 1);
    if (px == 0) continue;
    mx = std::max(mx, px);
    for (int s = 0; s < J.np * J.nsym; s++) u.push_back(make_int2((int)k, s));
  }
  g.units_off = (P.work.size() + 15) & ~(size_t)15;
  g.nunits = u.size();
  g.max_px = mx;
  P.work.resize(g.units_off + sizeof(int2) * u.size());
  if (!u.empty()) memcpy(&P.work[g.units_off], u.data(), sizeof(int2) * u.size());
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
    if (tile == kTunedScatter) {
      plan_units(P, g, false);
      P.groups.push_back(g);
      continue;
    }
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
    plan_units(P, g, true);
    P.groups.push_back(g);
  }
}

// Job table and work lists to the device (host sources are pageable
// vectors: the copies have taken them when cudaMemcpyAsync returns).
static int plan_upload(const RoundPlan &P, BatchScratch &bs, cudaStream_t st) {
  TRY(bs.d_jobs.ensure(sizeof(InsertJob) * std::max<size_t>(1, P.hj.size())));
  TRY(bs.d_counter.ensure(sizeof(int) * std::max<size_t>(1, P.groups.size())));
  TRY(bs.d_work.ensure(std::max<size_t>(16, P.work.size())));
  TRY(bs.ring.upload(bs.d_jobs.p, P.hj.data(), sizeof(InsertJob) * P.hj.size(), st));
  if (!P.work.empty()) TRY(bs.ring.upload(bs.d_work.p, P.work.data(), P.work.size(), st));
  return FR_OK;
}

// Device work of schedule group gi: one persistent launch (or the scatter
// over all its jobs), then the face taps.  Kernels only; each group has its
// own work counter, so groups (which insert into different jobs) may run
// concurrently.
static int plan_launch_group(const RoundPlan &P, BatchScratch &bs, size_t gi, cudaStream_t st) {
  const InsertJob *d_jobs = bs.d_jobs.as<InsertJob>();
  const RoundGroup &g = P.groups[gi];
  int *counter = bs.d_counter.as<int>() + gi;
  const int2 *units = (const int2 *)((const unsigned char *)bs.d_work.p + g.units_off);
  if (g.tile == kTunedScatter) {
    CU(launch_scatter_multi(d_jobs, units, (int)g.nunits, g.max_px, false, st));
    return FR_OK;
  }
  const void *w = (const unsigned char *)bs.d_work.p + g.off;
  if (g.tile == kPixelTile)
    CU(launch_pixel(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, counter, g.maxN, st));
  else if (g.tile == kColumn3Tile)
    CU(launch_column3(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, counter, g.maxN, st));
  else if (g.tile == kColumnTile)
    CU(launch_column(d_jobs, (const int4 *)w, (int)g.nwork, kColumnBlock, counter, g.max_mode, st));
  else
    CU(launch_gather(d_jobs, P.hj.data(), (int)P.hj.size(), (const int2 *)w, (int)g.nwork, g.tile,
                     counter, g.max_mode, st));
  CU(launch_scatter_multi(d_jobs, units, (int)g.nunits, g.max_px, true, st));
  return FR_OK;
}

// The round's schedule groups one after another on st.
static int plan_launch(const RoundPlan &P, BatchScratch &bs, cudaStream_t st) {
  for (size_t gi = 0; gi < P.groups.size(); gi++) TRY(plan_launch_group(P, bs, gi, st));
  return FR_OK;
}

// ------------------------------------------------------------ prologue groups
// Jobs of a round that share (N, box) run ONE prologue over their
// concatenated particles, so each prologue stage is one launch (or one
// batched FFT) per group rather than per job.  A group's metadata block is
// the prologue_meta layout for all its particles, then a table of their raw
// image addresses (the jobs' images need not be contiguous), then each
// particle's symmetry operators and first slice (jobs of one group may have
// different symmetries).
struct ProGroup {
  int N = 0, box = 0, n = 0;
  long nslices = 0;                     // symmetry copies of all its particles
  bool ctf = false;                     // the group runs the CTF round trip
  fr_recon *lead = nullptr;             // its symmetry table serves the group
  std::vector<int> jobs, first, count;  // job indices, first particle and count of each
  std::vector<long> slice0;             // each job's first slice in the group
  size_t meta_off = 0;                  // the group's block in the round's block
};

static size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }
static size_t group_tab_off(int n) { return align16(prologue_meta_bytes(n)); }
static size_t group_psym_off(int n) { return group_tab_off(n) + sizeof(float *) * (size_t)n; }
static size_t group_meta_bytes(int n) { return group_psym_off(n) + sizeof(PartSym) * (size_t)n; }

// Groups the jobs with counts[j] > 0 (in job order); returns the bytes of
// the round's metadata block, or kGroupsTooLarge when a group would hold more
// than INT_MAX particles or slices (its slice indices are ints on the device).
constexpr size_t kGroupsTooLarge = ~(size_t)0;
static size_t make_groups(const std::vector<fr_recon *> &jobs, const int *counts,
                          const int *boxes, std::vector<ProGroup> &G) {
  G.clear();
  for (int j = 0; j < (int)jobs.size(); j++) {
    if (counts[j] <= 0) continue;
    fr_recon *r = jobs[j];
    ProGroup *g = nullptr;
    for (ProGroup &q : G)
      if (q.N == r->N && q.box == boxes[j]) {
        g = &q;
        break;
      }
    if (!g) {
      G.emplace_back();
      g = &G.back();
      g->N = r->N;
      g->box = boxes[j];
      g->lead = r;
    }
    g->jobs.push_back(j);
    g->first.push_back(g->n);
    g->count.push_back(counts[j]);
    g->slice0.push_back(g->nslices);
    g->n += counts[j];
    g->nslices += (long)counts[j] * r->nsym;
    if (g->nslices > INT_MAX || g->n > INT_MAX - kBatchChunk) return kGroupsTooLarge;
  }
  size_t off = 0;
  for (ProGroup &g : G) {
    g.meta_off = off;
    off += align16(group_meta_bytes(g.n));
  }
  return off;
}

// Writes group g's block at blk: each job's particle metadata meta[j],
// particle i of job j's raw image address src[j] + i * box^2, and its
// symmetry operators (the job's) and first slice.  Returns whether any
// particle carries a CTF.
static bool group_meta(const std::vector<fr_recon *> &jobs, const ProGroup &g,
                       const fr_particle *const *meta, const float *const *src,
                       unsigned char *blk) {
  bool any = false;
  const float **tab = reinterpret_cast<const float **>(blk + group_tab_off(g.n));
  PartSym *ps = reinterpret_cast<PartSym *>(blk + group_psym_off(g.n));
  const size_t img = (size_t)g.box * g.box;
  for (size_t k = 0; k < g.jobs.size(); k++) {
    const int j = g.jobs[k];
    const fr_recon *r = jobs[j];
    any |= prologue_meta_range(g.N, g.n, g.first[k], g.count[k], meta[j], blk);
    for (int i = 0; i < g.count[k]; i++) {
      tab[g.first[k] + i] = src[j] + (size_t)i * img;
      PartSym &q = ps[g.first[k] + i];
      q.sym = r->d_sym.as<float>();
      q.nsym = r->nsym;
      q.slice0 = (int)(g.slice0[k] + (long)i * r->nsym);
    }
  }
  return any;
}

// The device half of group g's prologue (block at d_blk, scratch b) on st;
// with P, its jobs' InsertJobs (their parts of the group's slices, rotations
// and weights) join the plan.
static int group_run(const std::vector<fr_recon *> &jobs, const ProGroup &g, ProBufs &b,
                     const unsigned char *d_blk, RoundPlan *P, int tile_pref, cudaStream_t st,
                     bool exact_fft = false) {
  const float *const *tab = reinterpret_cast<const float *const *>(d_blk + group_tab_off(g.n));
  const PartSym *ps = reinterpret_cast<const PartSym *>(d_blk + group_psym_off(g.n));
  TRY(prologue_run(b.fft(), b.view(), d_blk, nullptr, tab, g.n, g.box, g.N,
                   g.lead->d_sym.as<float>(), g.lead->nsym, g.ctf, st, exact_fft, ps, g.nslices));
  if (!P) return FR_OK;
  const MetaView mv = meta_view(d_blk, g.n);
  const size_t sl = (size_t)g.N * (g.N / 2 + 1);
  for (size_t k = 0; k < g.jobs.size(); k++) {
    const int j = g.jobs[k], f = g.first[k];
    plan_add(*P, jobs[j], j, g.count[k], tile_pref, b.slices.as<float2>() + (size_t)f * sl,
             b.t3d.as<float>() + (size_t)g.slice0[k] * 9, mv.w + f);
  }
  return FR_OK;
}

// Inserts, for every job, counts[j] particles through the caller pipeline:
// per round one prologue per group of jobs of equal (N, box), and
// all jobs' insertion work in one persistent launch per schedule.  Every
// job runs on `st` for the duration of the call.
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
    TRY(require_cubic(jobs[j], "a batched insertion"));
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
    std::vector<int> c(nj, 0);
    std::vector<const float *> src(nj, nullptr);
    std::vector<const fr_particle *> m(nj, nullptr);
    const int p0 = rd * chunk;
    for (int j = 0; j < nj; j++) {
      c[j] = std::max(0, std::min(chunk, counts[j] - p0));
      if (c[j] == 0) continue;
      const int box = boxes[j];
      const void *d_raw = nullptr;
      TRY(to_device(imgs[j] + (size_t)p0 * box * box, sizeof(float) * (size_t)c[j] * box * box,
                    jobs[j]->s_in, st, &d_raw));
      src[j] = (const float *)d_raw;
      m[j] = meta[j] + p0;
    }
    std::vector<ProGroup> G;
    const size_t bytes = make_groups(jobs, c.data(), boxes, G);
    if (bytes == kGroupsTooLarge)
      return fail(FR_EINVAL_PARAM, "a round's jobs of one (N, box) exceed INT_MAX slices; "
                  "split the call");
    if (G.empty()) continue;
    int slot;
    unsigned char *blk;
    TRY(bs.ring.acquire(bytes, &slot, &blk));
    for (ProGroup &g : G) g.ctf = group_meta(jobs, g, m.data(), src.data(), blk + g.meta_off);
    TRY(bs.d_meta.ensure(bytes));
    CU(cudaMemcpyAsync(bs.d_meta.p, blk, bytes, cudaMemcpyHostToDevice, st));
    TRY(bs.ring.done(slot, st));
    if (bs.gbufs.size() < G.size()) bs.gbufs.resize(G.size());
    RoundPlan P;
    for (size_t gi = 0; gi < G.size(); gi++)
      TRY(group_run(jobs, G[gi], bs.gbufs[gi], bs.d_meta.as<unsigned char>() + G[gi].meta_off, &P,
                    tile_pref, st));
    plan_groups(jobs, P);
    TRY(plan_upload(P, bs, st));
    TRY(plan_launch(P, bs, st));
  }
  CU(cudaEventRecord(bs.done, st));
  bs.last = st;
  TRY(stream_leave_all(jobs, st));
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
  // this thread's scratch on the current device (its buffers and events
  // belong to one device)
  int dev = 0;
  CU(cudaGetDevice(&dev));
  static thread_local std::map<int, BatchScratch> scratch;
  BatchScratch &bs = scratch[dev];
  cudaStream_t st = stream ? (cudaStream_t)stream : jobs[0]->stream;
  return batch_insert(jobs, bs, -1, st, imgs, boxes, counts, meta);
}

// ------------------------------------------------------------------ graphs
// A batched insertion round of fixed shapes captured once as a CUDA graph.
// The graph owns the device slots for host images and every prologue
// group's scratch (so later calls on the same handles cannot move them); a
// replay writes the particles' metadata and image addresses into pinned
// staging, copies that one block (and any host images) in, and launches the
// graph.  Device images are read in place.
}  // extern "C"

struct fr_graph {
  std::vector<fr_recon *> jobs;
  cudaStream_t st = nullptr;
  std::vector<int> boxes, counts;
  std::vector<fr::DevBuf> slots;        // device images of host sources (and the caller's own)
  std::vector<fr::ProGroup> groups;     // prologue groups, fixed at capture
  std::vector<fr::ProBufs> gbufs;
  fr::DevBuf d_meta;                    // the round's metadata block
  size_t meta_bytes = 0;
  unsigned char *pinned[2] = {nullptr, nullptr};
  cudaEvent_t staged[2] = {nullptr, nullptr};
  bool staged_used[2] = {false, false};
  int next = 0;
  // The groups' prologues are captured as parallel branches on side streams.
  static constexpr int kSide = 8;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr, join[kSide] = {};
  long long kernels = 0;          // this library's kernels per replay
  fr::BatchScratch bs;
  fr::RoundPlan plan;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t meta_node = nullptr;   // the metadata upload, the graph's first node
  std::shared_ptr<fr::SharedEvent> after; // recorded after each replay, held by the handles
  std::mutex mu;
};

namespace fr {

static void graph_free(fr_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto &s : g->slots) s.release();
  for (auto &b : g->gbufs) b.release();
  g->d_meta.release();
  g->bs.release();
  for (int k = 0; k < 2; k++) {
    if (g->pinned[k]) cudaFreeHost(g->pinned[k]);
    if (g->staged[k]) cudaEventDestroy(g->staged[k]);
  }
  for (int k = 0; k < fr_graph::kSide; k++) {
    if (g->side[k]) cudaStreamDestroy(g->side[k]);
    if (g->join[k]) cudaEventDestroy(g->join[k]);
  }
  if (g->fork) cudaEventDestroy(g->fork);
  delete g;
}

// The graph's device work: the metadata upload (its source, one of the two
// pinned staging blocks, is set per replay), the groups' prologues (parallel
// branches when there are several), then the round's insertion launches (one
// branch per schedule group).
static int graph_device_work(fr_graph *g, cudaStream_t st) {
  CU(cudaMemcpyAsync(g->d_meta.p, g->pinned[0], g->meta_bytes, cudaMemcpyHostToDevice, st));
  const int ng = (int)g->groups.size();
  const int nside = std::min(ng, (int)fr_graph::kSide);
  if (ng > 1) {
    CU(cudaEventRecord(g->fork, st));
    for (int k = 0; k < nside; k++) CU(cudaStreamWaitEvent(g->side[k], g->fork, 0));
  }
  for (int gi = 0; gi < ng; gi++) {
    cudaStream_t s = ng > 1 ? g->side[gi % fr_graph::kSide] : st;
    TRY(group_run(g->jobs, g->groups[gi], g->gbufs[gi],
                  g->d_meta.as<unsigned char>() + g->groups[gi].meta_off, nullptr, -1, s, true));
  }
  if (ng > 1)
    for (int k = 0; k < nside; k++) {
      CU(cudaEventRecord(g->join[k], g->side[k]));
      CU(cudaStreamWaitEvent(st, g->join[k], 0));
    }
  // the schedule groups (disjoint jobs) as parallel branches too
  const int nsched = (int)g->plan.groups.size();
  if (nsched <= 1) return plan_launch(g->plan, g->bs, st);
  const int nside2 = std::min(nsched, (int)fr_graph::kSide);
  CU(cudaEventRecord(g->fork, st));
  for (int k = 0; k < nside2; k++) CU(cudaStreamWaitEvent(g->side[k], g->fork, 0));
  for (int gi = 0; gi < nsched; gi++)
    TRY(plan_launch_group(g->plan, g->bs, gi, g->side[gi % fr_graph::kSide]));
  for (int k = 0; k < nside2; k++) {
    CU(cudaEventRecord(g->join[k], g->side[k]));
    CU(cudaStreamWaitEvent(st, g->join[k], 0));
  }
  return FR_OK;
}

// The captured metadata upload: the memcpy node that writes d_meta.
static int find_meta_node(fr_graph *g) {
  size_t nn = 0;
  CU(cudaGraphGetNodes(g->graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  CU(cudaGraphGetNodes(g->graph, nodes.data(), &nn));
  for (cudaGraphNode_t n : nodes) {
    cudaGraphNodeType t;
    CU(cudaGraphNodeGetType(n, &t));
    if (t != cudaGraphNodeTypeMemcpy) continue;
    cudaMemcpy3DParms p;
    CU(cudaGraphMemcpyNodeGetParams(n, &p));
    if (p.dstPtr.ptr == g->d_meta.p) {
      g->meta_node = n;
      return FR_OK;
    }
  }
  return fail(FR_ECUDA, "captured graph has no metadata upload node");
}

static int graph_create(const std::vector<fr_recon *> &jobs, cudaStream_t st, int tile_pref,
                        const int *boxes, const int *counts, const int *ctf, fr_graph **out) {
  const int nj = (int)jobs.size();
  int total = 0;
  for (int j = 0; j < nj; j++) {
    TRY(check_state(jobs[j]));
    TRY(require_cubic(jobs[j], "a batched insertion graph"));
    if (counts[j] < 0 || counts[j] > kBatchChunk || (counts[j] > 0 && boxes[j] <= 0))
      return fail(FR_EINVAL_PARAM, "job %d: count must be in [0, %d] with a positive box", j,
                  kBatchChunk);
    if (total > INT_MAX - counts[j])
      return fail(FR_EINVAL_PARAM, "a graph holds at most INT_MAX particles");
    total += counts[j];
  }
  if (total == 0) return fail(FR_EINVAL_PARAM, "a graph needs at least one particle");
  std::vector<ProGroup> groups;
  const size_t meta_bytes = make_groups(jobs, counts, boxes, groups);
  if (meta_bytes == kGroupsTooLarge)
    return fail(FR_EINVAL_PARAM, "the graph's jobs of one (N, box) exceed INT_MAX slices");
  fr_graph *g = new fr_graph();
  g->jobs = jobs;
  g->st = st;
  g->boxes.assign(boxes, boxes + nj);
  g->counts.assign(counts, counts + nj);
  g->slots.resize(nj);
  g->meta_bytes = meta_bytes;
  g->groups = std::move(groups);
  g->gbufs.resize(g->groups.size());
  // a group runs the CTF round trip when any of its jobs was captured with one
  for (ProGroup &q : g->groups)
    for (int j : q.jobs) q.ctf = q.ctf || (ctf && ctf[j]);
  int rc = FR_OK;
  for (int k = 0; k < 2 && rc == FR_OK; k++)
    if (cudaHostAlloc((void **)&g->pinned[k], std::max<size_t>(16, g->meta_bytes),
                      cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->staged[k], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(FR_ENOMEM, "pinned staging allocation failed");
  for (int k = 0; k < fr_graph::kSide && rc == FR_OK; k++)
    if (cudaStreamCreateWithFlags(&g->side[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&g->join[k], cudaEventDisableTiming) != cudaSuccess)
      rc = fail(FR_ECUDA, "stream creation failed");
  if (rc == FR_OK && cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming) != cudaSuccess)
    rc = fail(FR_ECUDA, "cudaEventCreate failed");
  if (rc == FR_OK) rc = g->d_meta.ensure(std::max<size_t>(16, g->meta_bytes));
  for (int j = 0; j < nj && rc == FR_OK; j++) rc = stream_enter(jobs[j], st);
  // Sizing pass: a prologue of weight-0 particles read from the zeroed slots
  // allocates every buffer and FFT plan the capture uses, so the captured
  // work allocates nothing.
  std::vector<std::vector<fr_particle>> zero(nj);
  std::vector<const fr_particle *> zmeta(nj, nullptr);
  std::vector<const float *> src(nj, nullptr);
  for (int j = 0; j < nj && rc == FR_OK; j++) {
    const int n = counts[j];
    if (n == 0) continue;
    const size_t bytes = sizeof(float) * (size_t)n * boxes[j] * boxes[j];
    if ((rc = g->slots[j].ensure(bytes)) != FR_OK) break;
    if (cudaMemsetAsync(g->slots[j].p, 0, bytes, st) != cudaSuccess) {
      rc = fail(FR_ECUDA, "memset failed");
      break;
    }
    src[j] = g->slots[j].as<float>();
    zero[j].resize(n);
    for (fr_particle &m : zero[j]) {
      memset(&m, 0, sizeof m);
      m.rot[0] = m.rot[4] = m.rot[8] = 1.0f;
      m.defocus = (ctf && ctf[j]) ? 1.5f : 0.0f;
      m.voltage = 300.0f;
      m.cs = 2.7f;
      m.apix = 1.0f;
      m.ampcont = 10.0f;
    }
    zmeta[j] = zero[j].data();
  }
  if (rc == FR_OK) {
    std::vector<unsigned char> blk(std::max<size_t>(16, g->meta_bytes));
    for (const ProGroup &q : g->groups)
      group_meta(jobs, q, zmeta.data(), src.data(), blk.data() + q.meta_off);
    if (cudaMemcpyAsync(g->d_meta.p, blk.data(), g->meta_bytes, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      rc = fail(FR_ECUDA, "metadata upload failed");
    if (rc == FR_OK && cudaStreamSynchronize(st) != cudaSuccess)   // blk is pageable
      rc = fail(FR_ECUDA, "metadata upload failed");
  }
  for (size_t gi = 0; gi < g->groups.size() && rc == FR_OK; gi++)
    rc = group_run(jobs, g->groups[gi], g->gbufs[gi],
                   g->d_meta.as<unsigned char>() + g->groups[gi].meta_off, &g->plan, tile_pref, st,
                   true);
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
      rc = graph_device_work(g, st);
      const cudaError_t e = cudaStreamEndCapture(st, &g->graph);
      if (rc == FR_OK && e != cudaSuccess)
        rc = fail(FR_ECUDA, "stream capture failed: %s", cudaGetErrorString(e));
      g->kernels = launches_noted() - noted;
    }
  }
  if (rc == FR_OK) rc = find_meta_node(g);
  if (rc == FR_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
    rc = fail(FR_ECUDA, "cudaGraphInstantiate failed: %s", cudaGetErrorString(cudaGetLastError()));
  stream_leave_all(jobs, st);
  if (rc != FR_OK) {
    cudaGetLastError();
    cudaStreamSynchronize(st);
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
  // particle sources: device images in place, host images through the slots
  std::vector<const float *> src(nj, nullptr);
  bool host_src = false;
  for (int j = 0; j < nj; j++) {
    if (g->counts[j] == 0) continue;
    if (!meta[j]) return fail(FR_ENULL, "job %d: null metadata", j);
    if (imgs && !imgs[j]) return fail(FR_ENULL, "job %d: null images", j);
    const bool in_place = imgs && is_device_ptr(imgs[j]);
    src[j] = in_place ? imgs[j] : g->slots[j].as<float>();
    host_src |= imgs && !in_place;
  }
  const int k = g->next;
  // this staging block was last read by the replay before the previous one
  if (g->staged_used[k]) CU(cudaEventSynchronize(g->staged[k]));
  for (const ProGroup &q : g->groups) {
    const bool any = group_meta(g->jobs, q, meta, src.data(), g->pinned[k] + q.meta_off);
    if (any && !q.ctf)
      return fail(FR_EINVAL_PARAM,
                  "jobs of box %d (N %d) carry a CTF but were captured without the phase flip",
                  q.box, q.N);
  }
  g->next ^= 1;
  for (fr_recon *r : g->jobs) TRY(stream_enter(r, st));
  for (int j = 0; host_src && j < nj; j++) {
    const int n = g->counts[j];
    if (n == 0 || is_device_ptr(imgs[j])) continue;
    const size_t bytes = sizeof(float) * (size_t)n * g->boxes[j] * g->boxes[j];
    CU(cudaMemcpyAsync(g->slots[j].p, imgs[j], bytes, cudaMemcpyHostToDevice, st));
  }
  // the graph's first node uploads this replay's block
  CU(cudaGraphExecMemcpyNodeSetParams1D(g->exec, g->meta_node, g->d_meta.p, g->pinned[k],
                                        g->meta_bytes, cudaMemcpyHostToDevice));
  CU(cudaGraphLaunch(g->exec, st));
  CU(cudaEventRecord(g->staged[k], st));
  g->staged_used[k] = true;
  note_launch((int)g->kernels);
  TRY(stream_leave_all(g->jobs, st, &g->after));
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
