// fr_handle.h -- the reconstruction handle and host helpers shared by the
// C-ABI translation units (fr_api.cu, fr_batch.cu).  Not part of the C ABI.
#pragma once
#include <cufft.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eman2_b200.h"
#include "fr_internal.h"

namespace fr {

int fail(int code, const char *fmt, ...);

#define CU(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return ::fr::fail(e_ == cudaErrorMemoryAllocation ? FR_ENOMEM : FR_ECUDA,        \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define CUFFT(call)                                                                   \
  do {                                                                                \
    cufftResult r_ = (call);                                                          \
    if (r_ != CUFFT_SUCCESS)                                                          \
      return ::fr::fail(r_ == CUFFT_ALLOC_FAILED ? FR_ENOMEM : FR_ECUDA, "%s: cufft error %d", \
                        #call, (int)r_);                                              \
  } while (0)

#define TRY(call)                 \
  do {                            \
    int rc_ = (call);             \
    if (rc_ != FR_OK) return rc_; \
  } while (0)

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return FR_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(FR_ENOMEM, "device allocation of %zu bytes failed", bytes);
    }
    cap = bytes;
    return FR_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};


// Pinned host staging for per-call uploads (metadata blocks, job tables,
// work lists).  A pageable source would make cudaMemcpyAsync wait for the
// stream to drain; from pinned memory the upload is queued and the host runs
// ahead.  Slots are used in turn; a slot is rewritten only after the upload
// that read it has completed.
struct PinnedRing {
  static constexpr int kSlots = 4;
  unsigned char *buf[kSlots] = {};
  size_t cap[kSlots] = {};
  cudaEvent_t ev[kSlots] = {};
  bool pending[kSlots] = {};
  int next = 0;
  // A pinned block of `bytes` for the caller to fill; *slot names it for done().
  int acquire(size_t bytes, int *slot, unsigned char **out) {
    const int k = next;
    next = (next + 1) % kSlots;
    if (pending[k]) {
      if (cudaEventSynchronize(ev[k]) != cudaSuccess) return fail(FR_ECUDA, "staging wait failed");
      pending[k] = false;
    } else if (!ev[k] && cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
      return fail(FR_ECUDA, "cudaEventCreate failed");
    }
    if (cap[k] < bytes) {
      if (buf[k]) cudaFreeHost(buf[k]);
      buf[k] = nullptr;
      cap[k] = 0;
      if (cudaHostAlloc((void **)&buf[k], bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return fail(FR_ENOMEM, "pinned host allocation of %zu bytes failed", bytes);
      }
      cap[k] = bytes;
    }
    *slot = k;
    *out = buf[k];
    return FR_OK;
  }
  // Marks the end of the uploads that read `slot` (queued on st).
  int done(int slot, cudaStream_t st) {
    if (cudaEventRecord(ev[slot], st) != cudaSuccess) return fail(FR_ECUDA, "cudaEventRecord failed");
    pending[slot] = true;
    return FR_OK;
  }
  // One upload of a host block through the ring.
  int upload(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return FR_OK;
    int k;
    unsigned char *p;
    int rc = acquire(bytes, &k, &p);
    if (rc != FR_OK) return rc;
    memcpy(p, src, bytes);
    if (cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return fail(FR_ECUDA, "upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    return done(k, st);
  }
  void release() {
    for (int k = 0; k < kSlots; k++) {
      if (pending[k]) cudaEventSynchronize(ev[k]);
      if (buf[k]) cudaFreeHost(buf[k]);
      if (ev[k]) cudaEventDestroy(ev[k]);
      buf[k] = nullptr;
      ev[k] = nullptr;
      cap[k] = 0;
      pending[k] = false;
    }
  }
};

// An event marking the end of a handle's last work.  A call over many
// handles on one stream records ONE event and shares it among them; a handle
// that leaves alone on another stream gets a fresh event of its own.
struct SharedEvent {
  cudaEvent_t ev = nullptr;
  ~SharedEvent() {
    if (ev) cudaEventDestroy(ev);
  }
};

bool is_device_ptr(const void *p);
int to_device(const void *src, size_t bytes, DevBuf &stage, cudaStream_t st, const void **out);
int from_device(void *dst, const void *dsrc, size_t bytes, cudaStream_t st);

// ------------------------------------------------------------- cuFFT plans
// Plans made with cuFFT's own work-area allocation turned off: every plan of
// one cache runs in stream order on one stream at a time, so they share ONE
// work area, sized to the largest plan, instead of holding one each (a cache
// of power-of-two batches up to 1024 would otherwise keep twice the largest
// transform's work area per direction).
struct PlanCache {
  std::map<std::pair<int, int>, cufftHandle> r2c, c2r;   // key (N, batch)
  std::map<cufftHandle, size_t> need;                   // each plan's work-area bytes
  cufftHandle c2r3 = 0, r2c3 = 0;
  int c2r3_N = 0, r2c3_N = 0, c2r3_NZ = 0;
  DevBuf work;
  PlanCache() = default;
  PlanCache(const PlanCache &) = delete;
  PlanCache &operator=(const PlanCache &) = delete;
  ~PlanCache() { release(); }
  void release() {
    for (auto &kv : r2c) cufftDestroy(kv.second);
    for (auto &kv : c2r) cufftDestroy(kv.second);
    if (c2r3) cufftDestroy(c2r3);
    if (r2c3) cufftDestroy(r2c3);
    r2c.clear();
    c2r.clear();
    need.clear();
    c2r3 = r2c3 = 0;
    c2r3_N = r2c3_N = c2r3_NZ = 0;
    work.release();
  }
  // Drops one plan (a 3-D plan replaced by another size).
  void drop(cufftHandle &h) {
    if (!h) return;
    need.erase(h);
    cufftDestroy(h);
    h = 0;
  }
  // A fresh handle with the work area left to this cache.
  static int fresh(cufftHandle *h) {
    CUFFT(cufftCreate(h));
    const cufftResult r = cufftSetAutoAllocation(*h, 0);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(*h);
      return fail(FR_ECUDA, "cufftSetAutoAllocation: cufft error %d", (int)r);
    }
    return FR_OK;
  }
  // Points h at the shared work area (grown to h's need) and at stream st.
  int bind(cufftHandle h, cudaStream_t st) {
    const size_t bytes = need[h];
    if (bytes > work.cap) {
      // a larger area replaces the old one; queued transforms that use the
      // old one end first (the free waits for the device)
      TRY(work.ensure(bytes));
    }
    if (bytes) CUFFT(cufftSetWorkArea(h, work.p));
    CUFFT(cufftSetStream(h, st));
    return FR_OK;
  }
  int make3d(cufftHandle *h, int nz, int ny, int nx, cufftType type) {
    TRY(fresh(h));
    size_t ws = 0;
    const cufftResult r = cufftMakePlan3d(*h, nz, ny, nx, type, &ws);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(*h);
      *h = 0;
      return fail(r == CUFFT_ALLOC_FAILED ? FR_ENOMEM : FR_ECUDA,
                  "cufftMakePlan3d(%d, %d, %d): cufft error %d", nz, ny, nx, (int)r);
    }
    need[*h] = ws;
    return FR_OK;
  }
  int get3d_r2c(int N, cudaStream_t st, cufftHandle *out) {
    if (!r2c3 || r2c3_N != N) {
      drop(r2c3);
      TRY(make3d(&r2c3, N, N, N, CUFFT_R2C));
      r2c3_N = N;
    }
    TRY(bind(r2c3, st));
    *out = r2c3;
    return FR_OK;
  }
  int get3d(int N, cudaStream_t st, cufftHandle *out, int NZ = 0) {
    if (!NZ) NZ = N;
    if (!c2r3 || c2r3_N != N || c2r3_NZ != NZ) {
      drop(c2r3);
      TRY(make3d(&c2r3, NZ, N, N, CUFFT_C2R));
      c2r3_N = N;
      c2r3_NZ = NZ;
    }
    TRY(bind(c2r3, st));
    *out = c2r3;
    return FR_OK;
  }
  int get2d(bool forward, int N, int batch, cudaStream_t st, cufftHandle *out) {
    auto &m = forward ? r2c : c2r;
    auto key = std::make_pair(N, batch);
    auto it = m.find(key);
    if (it == m.end()) {
      cufftHandle h;
      TRY(fresh(&h));
      int n[2] = {N, N};
      const int dist_r = N * N, dist_c = N * (N / 2 + 1);
      size_t ws = 0;
      const cufftResult r =
          forward ? cufftMakePlanMany(h, 2, n, nullptr, 1, dist_r, nullptr, 1, dist_c, CUFFT_R2C,
                                      batch, &ws)
                  : cufftMakePlanMany(h, 2, n, nullptr, 1, dist_c, nullptr, 1, dist_r, CUFFT_C2R,
                                      batch, &ws);
      if (r != CUFFT_SUCCESS) {
        cufftDestroy(h);
        return fail(r == CUFFT_ALLOC_FAILED ? FR_ENOMEM : FR_ECUDA,
                    "cufftMakePlanMany(%s, N %d, batch %d): cufft error %d",
                    forward ? "R2C" : "C2R", N, batch, (int)r);
      }
      need[h] = ws;
      it = m.emplace(key, h).first;
    }
    TRY(bind(it->second, st));
    *out = it->second;
    return FR_OK;
  }
  // n batched 2-D transforms of size N (contiguous, unpadded) run as a
  // binary decomposition into power-of-two batches (at most 1024), so the
  // plans are shared by every chunk length instead of one plan per length.
  // exact: one plan of batch n (a captured graph's fixed shapes: one launch
  // sequence instead of one per power of two).
  int exec2d(bool forward, int N, int n, const void *in, void *out, cudaStream_t st,
             bool exact = false) {
    const size_t img = (size_t)N * N, spec = (size_t)N * (N / 2 + 1);
    int done = 0;
    while (done < n) {
      int b = 1;
      if (exact) b = n;
      else while (2 * b <= n - done && 2 * b <= 1024) b *= 2;
      cufftHandle h;
      int rc = get2d(forward, N, b, st, &h);
      if (rc != FR_OK) return rc;
      if (forward)
        CUFFT(cufftExecR2C(h, (cufftReal *)in + done * img, (cufftComplex *)out + done * spec));
      else
        CUFFT(cufftExecC2R(h, (cufftComplex *)in + done * spec, (cufftReal *)out + done * img));
      done += b;
    }
    return FR_OK;
  }
};


size_t vol_floats(int N);
size_t norm_floats(int N);
size_t slice_floats(int N);

// Tile choice for the gather schedule (fr_batch.cu): measured choice when the
// autotuner has one for (N, mode, nsym), else a size-based default.
int tuned_tile(int N, int mode, int nsym);
int default_tile(int mode, int N, int nsym, int np);

}  // namespace fr

// ------------------------------------------------------------------ handle
struct fr_recon {
  fr_params p;
  int N = 0;
  int NZ = 0;                 // the volume's z size (N for the cubic volume)
  int mode = FR_MODE_GAUSS2;
  int nsym = 1;
  std::vector<float> syms;
  int state = 0;              // 0 created, 1 accumulating, 2 finished
  cudaStream_t own = nullptr, stream = nullptr;
  fr::Geom *geom = nullptr;
  fr::Geom *wgeom = nullptr;  // the Wiener reconstructor's pixel disk (looked up on first use)
  fr::DevBuf ref;             // the iterative reconstructor's reference volume [N][N][N+2]
  bool has_ref = false;
  float wfilt = 0.0f;         // 1: Wiener normalisation, data / (weight + 1)
  fr::DevBuf vol_data, vol_norm, d_sym;
  // scratch
  fr::DevBuf s_in, s_slices, s_rot, s_w, s_t3d, s_img, s_img2, s_spec, s_ctf, s_txy, s_out,
      s_ssnr, s_jobs, s_work, s_counter;
  fr::PlanCache plans;
  int tile = -1;              // gather tile shape (-1: tuned default)
  std::vector<int> tiles;
  std::vector<float> tile_dist;   // nearest-cell distance of each tile (column kernel)
  int tiles_tile = -1, tx = 0, ty = 0, tz = 0;
  int work_np = -1, nwork = 0;   // cached work list signature (slices) and size
  // Insertion calls return once their work is enqueued.  `done` is recorded
  // after the handle's last enqueued work on stream `last`; a call on another
  // stream first makes that stream wait for it.
  std::shared_ptr<fr::SharedEvent> done;
  cudaStream_t last = nullptr;
  // Host particle chunks go through two device staging buffers filled on a
  // copy stream: the upload of one chunk overlaps the work on the one before.
  cudaStream_t copy_st = nullptr;
  fr::DevBuf s_stage[2];
  cudaEvent_t staged[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
  bool consumed_set[2] = {false, false};
  int stage_next = 0;
  // pinned staging of the per-call uploads: chunk metadata, job and work lists
  fr::PinnedRing ring_meta, ring_small;
  // The current chunk's metadata block on the device (prologue_meta layout):
  // s_meta for device inputs, or the tail of the chunk's staging buffer.
  fr::DevBuf s_meta;
  const unsigned char *d_meta = nullptr;
  // Device copies of the last two insertion jobs, reused while unchanged.
  fr::InsertJob job_cache[2];
  bool job_valid[2] = {false, false};
  int job_next = 0;
  std::mutex mu;
};


namespace fr {
int check_state(fr_recon *r);
// Floats of the handle's complex and weight volumes: [NZ][N][N+2], [NZ][N][N/2+1].
inline size_t rvol_floats(const fr_recon *r) { return (size_t)r->NZ * r->N * (r->N + 2); }
inline size_t rnorm_floats(const fr_recon *r) { return (size_t)r->NZ * r->N * (r->N / 2 + 1); }
// Paths built for the cubic volume only: FR_EUNSUPPORTED otherwise.
int require_cubic(const fr_recon *r, const char *what);
// Orders work enqueued on st after the handle's earlier work on other streams.
int stream_enter(fr_recon *r, cudaStream_t st);
// Marks the end of the handle's work enqueued so far on st.
int stream_leave(fr_recon *r, cudaStream_t st);
// The same for many handles whose work went to st: one event for all.
// reuse: a caller that always leaves on the same stream may keep the event
// and have it recorded again (handles that still hold it from an earlier call
// then wait for a later point of that stream, which includes their work).
int stream_leave_all(const std::vector<fr_recon *> &rs, cudaStream_t st,
                     std::shared_ptr<SharedEvent> *reuse = nullptr);
InsertJob make_job(fr_recon *r, const float2 *slices, const float *t3d, const float *pw, int np);
int run_scatter(const InsertJob &j0, bool edge_only, cudaStream_t st);
int insert_device(fr_recon *r, const float2 *d_slices, const float *d_t3d, const float *d_pw, int np,
                  int schedule, const float *d_ssnr, int nssnr);
int check_device_error(fr_recon *r);
int alloc_volume(fr_recon *r);
// Prologue of one chunk of device particles into r's scratch: s_slices,
// s_t3d and s_w hold the chunk's slices, composed rotations and weights.
int prologue_chunk(fr_recon *r, const float *d_raw, int n, int box, const fr_particle *meta);
// Its halves: metadata block on the host, upload, device work only.
size_t prologue_meta_bytes(int n);
bool prologue_meta(int N, int n, const fr_particle *meta, unsigned char *blk);
// Entries [first, first + count) of the block of n particles.
bool prologue_meta_range(int N, int n, int first, int count, const fr_particle *meta,
                         unsigned char *blk);
int prologue_upload(fr_recon *r, int n, const unsigned char *blk, cudaStream_t st);
// The arrays of a metadata block of n particles (prologue_meta's layout).
struct MetaView {
  const void *ctf;
  const float *txy, *w, *rot;
};
MetaView meta_view(const unsigned char *d_meta, int n);
// Scratch of one prologue run: padded images, slices, spectra (and the r2c
// input), composed rotations, the CTF round trip's images.
struct ProScratch {
  DevBuf *img, *slices, *spec, *t3d, *img2;
};
// The device half of a prologue over n particles of size box into slices of
// size N: metadata block (prologue_meta layout) at d_meta, raw images at
// d_raw (contiguous) or through d_src (a device table of per-particle
// pointers).  Kernels and FFTs only once the scratch and plans exist.
int prologue_run(PlanCache &plans, const ProScratch &b, const unsigned char *d_meta,
                 const float *d_raw, const float *const *d_src, int n, int box, int N,
                 const float *d_sym, int nsym, bool any_ctf, cudaStream_t st,
                 bool exact_fft = false, const PartSym *d_psym = nullptr, long nslices = -1);
int prologue_device(fr_recon *r, const float *d_raw, int n, int box, bool any_ctf);
int particles_chunk(fr_recon *r, const float *d_raw, int n, int box, const fr_particle *meta,
                    int schedule);
}  // namespace fr
