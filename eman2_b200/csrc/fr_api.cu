// fr_api.cu -- the C ABI (include/eman2_b200.h): reconstruction handles,
// parameter checks, device memory, cuFFT plans and the dispatch of the
// prologue / insertion / agreement / finish kernels.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/eman2_b200.h"
#include "fr_handle.h"

namespace fr {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// --------------------------------------------------------------- accounting
static std::atomic<long long> g_launches{0}, g_ins_launches{0}, g_slices{0}, g_gather_launches{0};
static std::atomic<int> g_profile{0};
static std::mutex g_stat_mu;
static double g_insert_ms = 0.0, g_gather_ms = 0.0;

void note_launch(int n) { g_launches += n; }
long long launches_noted() { return g_launches.load(); }

// ----------------------------------------------------------- device consts
static std::mutex g_mu;
static std::map<int, Consts> g_consts;
static std::map<std::pair<int, int>, Geom *> g_geoms[64];

// Table index of Util::fast_exp(-r*h) for a float r >= 0, evaluated with the
// reference's rounding points (f = -r*h in float; (int)(-f*50.0+0.5) in
// double); -1 when f < -19.98 (the exp() branch).
static int exp_index(float r, float h) {
  volatile float rv = r, hv = h;
  const float f = -(rv * hv);
  if ((double)f > 0 || (double)f < -19.98) return -1;
  return (int)(-(double)f * 50.0 + 0.5);
}

// Smallest float r >= 0 with pred(r) true, for pred monotone in r.
template <class P> static float min_float_where(P pred, float hi) {
  uint32_t lo_b = 0, hi_b;
  memcpy(&hi_b, &hi, 4);
  while (lo_b < hi_b) {
    const uint32_t mid = lo_b + (hi_b - lo_b) / 2;
    float m;
    memcpy(&m, &mid, 4);
    if (pred(m)) hi_b = mid;
    else lo_b = mid + 1;
  }
  float out;
  memcpy(&out, &lo_b, 4);
  return out;
}

// Builds the step table of fast_exp(-r*h) over r in [0, rmax).
static void build_steps(float h, float K, float rmax, const float *tab, ExpSteps &out) {
  const float rout = min_float_where([&](float r) { return exp_index(r, h) < 0 && r > 0; }, 1e4f);
  const float rend = std::min(rmax, rout);
  const int nb = (int)std::ceil(rend * K) + 1;
  std::vector<float4> bins(nb);
  for (int b = 0; b < nb; b++) {
    const float r0 = (float)b / K, r1 = (float)(b + 1) / K;
    int g0 = exp_index(r0, h);
    float4 e;
    if (g0 < 0) {   // the whole bin is past the table: entries unused
      e = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      float thr = INFINITY;
      if (g0 + 1 <= 999) {
        const float t = min_float_where([&](float r) { int g = exp_index(r, h); return g < 0 || g >= g0 + 1; }, 1e4f);
        if (t < r1) thr = t;
      }
      const int g1 = std::min(g0 + 1, 999);
      e = make_float4(thr, tab[g0], tab[g1], 0.f);
    }
    bins[b] = e;
    // at most one threshold per bin (thresholds are 1/(50h) apart in r)
    if (g0 >= 0) {
      const float below_r1 = std::nextafter(r1, 0.0f);
      const int g1 = exp_index(below_r1, h);
      if (g1 >= 0 && g1 > g0 + 1)
        fprintf(stderr, "eman2_b200: exp step table bin %d holds two thresholds\n", b);
    }
  }
  out.K = K;
  out.rout = rout;
  out.nbins = nb;
  cudaMalloc(&out.d_bins, sizeof(float4) * nb);
  cudaMemcpy(out.d_bins, bins.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice);
}

Consts &consts() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_consts.find(dev);
  if (it != g_consts.end()) return it->second;
  Consts c;
  // Util::fast_exp table (libEM/util.cpp:793): (float)exp(-i/50.0).
  float tab[1000];
  for (int i = 0; i < 1000; i++) tab[i] = (float)std::exp(-i / 50.0);
  cudaMalloc(&c.d_exp, sizeof tab);
  cudaMemcpy(c.d_exp, tab, sizeof tab, cudaMemcpyHostToDevice);
  cudaMalloc(&c.d_err, sizeof(int));
  cudaMemset(c.d_err, 0, sizeof(int));
  // h = 1.0f / EMConsts::I2G and 1.0f / EMConsts::I5G (libEM/emobject.cpp:53-56,
  // libEM/reconstructor_tools.cpp:152,344).
  volatile float i2g = (float)(4.0 / (M_PI * M_PI));
  volatile float i5g = (float)(10.4 / (M_PI * M_PI));
  c.h2 = 1.0f / i2g;
  c.h5 = 1.0f / i5g;
  build_steps(c.h2, 256.0f, 3.01f, tab, c.steps2);   // gauss_2 taps: |d| <= 1 per axis, r <= 3
  build_steps(c.h5, 64.0f, 40.0f, tab, c.steps5);
  return g_consts[dev] = c;
}

// Pixel selection of do_insert_slice_work (libEM/reconstructor.cpp:1178-1181):
// keep (x,y) when Util::hypot_fast_int(x,y) = round(hypot(x,y)) <= N/2,
// i.e. (int)(hypotf(x,y) + 0.5f) <= N/2; corners keeps every pixel.
static int hypot_fast_int(int x, int y) {
  const float h = (float)std::sqrt((double)x * x + (double)y * y);
  return (int)(h + 0.5f);
}

Geom *get_geom(int N, int corners) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mu);
  auto key = std::make_pair(N, corners);
  auto &m = g_geoms[dev & 63];
  auto it = m.find(key);
  if (it != m.end()) return it->second;
  Geom *g = new Geom();
  g->N = N;
  g->corners = corners;
  const int n2 = N / 2;
  g->xmax.assign(N, -1);
  std::vector<int> rim;
  int npix = 0;
  for (int y = -n2; y < n2; y++) {
    int xm = -1;
    for (int x = 0; x <= n2; x++) {
      if (corners == 3) {
        // FourierIterReconstructor: r > iny/2+3 skipped (libEM/reconstructor.cpp:544-545)
        if (hypot_fast_int(x, y) > n2 + 3) continue;
      } else if (corners == 2) {
        // WienerFourierReconstructor: rn = (float)hypot(x/(inx-2), y/iny) < .5
        // (libEM/reconstructor.cpp:1703-1707)
        const float rx = (float)x / (float)N, ry = (float)y / (float)N;
        if ((float)std::hypot((double)rx, (double)ry) >= 0.5f) continue;
      } else {
        const int r = hypot_fast_int(x, y);
        if (!corners && r > n2) continue;   // (r > iny/2 && abs(inx-iny) < 3): square input
      }
      xm = x;                              // kept pixels form a prefix of the row
      npix++;
      // Pixels that can reach a cube face (|i|, |j| or |k| = N/2): their
      // points satisfy some |p_a| >= N/2 - 3.5, hence |p| >= N/2 - 3.5.
      if (std::sqrt((double)x * x + (double)y * y) >= n2 - 3.6) rim.push_back(x | ((y + n2) << 16));
    }
    g->xmax[y + n2] = xm;
  }
  g->npix = npix;
  std::vector<float> rtab(N + 2);
  for (int i = -n2; i <= n2 + 1; i++) rtab[i + n2] = (float)i / (float)N;
  cudaMalloc(&g->d_xmax, sizeof(int) * N);
  cudaMemcpy(g->d_xmax, g->xmax.data(), sizeof(int) * N, cudaMemcpyHostToDevice);
  cudaMalloc(&g->d_rtab, sizeof(float) * (N + 2));
  cudaMemcpy(g->d_rtab, rtab.data(), sizeof(float) * (N + 2), cudaMemcpyHostToDevice);
  g->nrim = (int)rim.size();
  cudaMalloc(&g->d_rim, sizeof(int) * std::max<size_t>(1, rim.size()));
  if (!rim.empty())
    cudaMemcpy(g->d_rim, rim.data(), sizeof(int) * rim.size(), cudaMemcpyHostToDevice);
  m[key] = g;
  return g;
}

// ---------------------------------------------------------------- symmetry
// Transform::set_rotation "eman" branch (libEM/transform.cpp:654-666).
void eman_matrix(double az, double alt, double phi, float *m) {
  const double d2r = 3.141592653589793238462643383279502884197169399 / 180.0;
  const double azp = az * d2r, altp = alt * d2r, phip = phi * d2r;
  m[0] = (float)(cos(phip) * cos(azp) - cos(altp) * sin(azp) * sin(phip));
  m[1] = (float)(cos(phip) * sin(azp) + cos(altp) * cos(azp) * sin(phip));
  m[2] = (float)(sin(altp) * sin(phip));
  m[3] = (float)(-sin(phip) * cos(azp) - cos(altp) * sin(azp) * cos(phip));
  m[4] = (float)(-sin(phip) * sin(azp) + cos(altp) * cos(azp) * cos(phip));
  m[5] = (float)(sin(altp) * cos(phip));
  m[6] = (float)(sin(altp) * sin(azp));
  m[7] = (float)(-sin(altp) * cos(azp));
  m[8] = (float)cos(altp);
}

// The platonic groups' operators as EMAN Euler triples (az, alt, phi), in the
// reference's order: TetrahedralSym::get_sym (libEM/symmetry.cpp:2007-2027),
// OctahedralSym::get_sym (:1950-1973), IcosahedralSym::get_sym (:1822-1868,
// with its +90 / -90 azimuth alignment).  Each group is a few levels of
// altitude, each with a ring of azimuths and a ring of in-plane angles.
static int platonic_ops(const std::string &name, std::vector<float> &out) {
  const double rad2deg = 180.0 / 3.141592653589793238462643383279502884197169399;
  std::vector<float> e;   // (az, alt, phi) triples
  if (name == "tet") {
    const float l1 = (float)(rad2deg * acos((double)(-1.0f / 3.0f)));
    for (int k = 0; k < 3; k++) e.insert(e.end(), {0.0f, 0.0f, 120.0f * k});
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < 3; k++) e.insert(e.end(), {120.0f * a, l1, 60.0f + 120.0f * k});
  } else if (name == "oct") {
    for (int k = 0; k < 4; k++) e.insert(e.end(), {0.0f, 0.0f, 90.0f * k});
    for (int a = 0; a < 4; a++)
      for (int k = 0; k < 4; k++) e.insert(e.end(), {90.0f * a, 90.0f, 90.0f * k});
    for (int k = 0; k < 4; k++) e.insert(e.end(), {0.0f, 180.0f, 90.0f * k});
  } else if (name == "icos" || name == "icos5") {
    const float l1 = (float)(rad2deg * atan((double)2.0f));
    const float l2 = 180.0f - l1;
    // in-plane ring of a pentagon centred on a level: 0, 288, 216, 144, 72
    // (or those plus 36: 36, 324, 252, 180, 108)
    auto ring = [](int k, float base) {
      float v = base - 72.0f * k;
      return v < 0 ? v + 360.0f : v;
    };
    for (int k = 0; k < 5; k++) e.insert(e.end(), {0.0f, 0.0f, ring(k, 0.0f)});
    for (int a = 0; a < 5; a++)
      for (int k = 0; k < 5; k++) e.insert(e.end(), {72.0f * a, l1, ring(k, 36.0f)});
    for (int a = 0; a < 5; a++)
      for (int k = 0; k < 5; k++) e.insert(e.end(), {36.0f + 72.0f * a, l2, ring(k, 0.0f)});
    for (int k = 0; k < 5; k++) e.insert(e.end(), {0.0f, 180.0f, ring(k, 0.0f)});
    for (size_t i = 0; i < e.size(); i += 3) {   // get_az_alignment_offset() == 234
      e[i] = e[i] + 90.0f;
      e[i + 2] = e[i + 2] - 90.0f;
    }
  } else {
    return -1;
  }
  out.clear();
  float m[9];
  for (size_t i = 0; i < e.size(); i += 3) {
    eman_matrix((double)e[i], (double)e[i + 1], (double)e[i + 2], m);
    out.insert(out.end(), m, m + 9);
  }
  return (int)(e.size() / 3);
}

// Symmetry3D::get_symmetries (libEM/symmetry.cpp:1240-1246) for the cyclic
// (CSym::get_sym, :1407-1417), dihedral (DSym::get_sym, :1452-1470) and
// platonic groups (tet, oct, icos / icos5); the name parse follows
// Factory<Symmetry3D>::get (:76-130): "c" -> c1.  Orders are parsed with a
// range check: at most kMaxSymOps operators (c1000, d500), so a malformed
// or huge order is refused before any operator is built.
int sym_ops(const std::string &sym_in, std::vector<float> &out) {
  std::string sym;
  for (char ch : sym_in) sym.push_back((char)tolower((unsigned char)ch));
  if (sym.empty()) return -1;
  if (sym == "tet" || sym == "oct" || sym == "icos" || sym == "icos5")
    return platonic_ops(sym, out);
  const char kind = sym[0];
  if (kind != 'c' && kind != 'd') return -1;
  long nsym = 1;
  if (sym.size() > 1) {
    if (sym.size() > 8) return -1;
    for (size_t i = 1; i < sym.size(); i++)
      if (sym[i] < '0' || sym[i] > '9') return -1;
    char *end = nullptr;
    nsym = strtol(sym.c_str() + 1, &end, 10);
    if (!end || *end) return -1;
  }
  if (nsym <= 0 || (kind == 'c' ? nsym : 2 * nsym) > kMaxSymOps) return -1;
  out.clear();
  float m[9];
  if (kind == 'c') {
    for (int n = 0; n < nsym; n++) {
      const float az = (float)(n % nsym) * 360.0f / (float)nsym;
      eman_matrix((double)az, 0.0, 0.0, m);
      out.insert(out.end(), m, m + 9);
    }
    return nsym;
  }
  const int ns = 2 * nsym;
  for (int n = 0; n < ns; n++) {
    float az, alt;
    if (n >= ns / 2) { az = (float)((n % ns) - ns / 2) * 360.0f / (float)(ns / 2); alt = 180.0f; }
    else { az = (float)(n % ns) * 360.0f / (float)(ns / 2); alt = 0.0f; }
    eman_matrix((double)az, (double)alt, 0.0, m);
    out.insert(out.end(), m, m + 9);
  }
  return ns;
}

// ------------------------------------------------------------ device memory
bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device view of a caller buffer: device pointers pass through; host buffers
// are copied into `stage` on `st`.
int to_device(const void *src, size_t bytes, DevBuf &stage, cudaStream_t st,
                     const void **out) {
  if (is_device_ptr(src)) { *out = src; return FR_OK; }
  TRY(stage.ensure(bytes));
  CU(cudaMemcpyAsync(stage.p, src, bytes, cudaMemcpyHostToDevice, st));
  *out = stage.p;
  return FR_OK;
}

int from_device(void *dst, const void *dsrc, size_t bytes, cudaStream_t st) {
  if (is_device_ptr(dst)) {
    CU(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToDevice, st));
    CU(cudaStreamSynchronize(st));
  } else {
    CU(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
  }
  return FR_OK;
}

}  // namespace fr

using namespace fr;

namespace fr {

size_t vol_floats(int N) { return (size_t)N * N * (N + 2); }
size_t norm_floats(int N) { return (size_t)N * N * (N / 2 + 1); }
size_t slice_floats(int N) { return (size_t)N * (N + 2); }


int require_cubic(const fr_recon *r, const char *what) {
  if (r->NZ != r->N)
    return fail(FR_EUNSUPPORTED, "%s needs a cubic volume (this one is %d x %d x %d)", what, r->N,
                r->N, r->NZ);
  return FR_OK;
}

int check_state(fr_recon *r) {
  if (!r) return fail(FR_ENULL, "null reconstructor handle");
  if (r->state != 1)
    return fail(FR_ESTATE, r->state == 0 ? "setup() has not been called"
                                         : "finish() was called; call setup() again");
  return FR_OK;
}

int stream_enter(fr_recon *r, cudaStream_t st) {
  if (r->last && r->last != st) CU(cudaStreamWaitEvent(st, r->done->ev, 0));
  return FR_OK;
}

static int new_event(std::shared_ptr<SharedEvent> &out) {
  auto e = std::make_shared<SharedEvent>();
  CU(cudaEventCreateWithFlags(&e->ev, cudaEventDisableTiming));
  out = std::move(e);
  return FR_OK;
}

int stream_leave(fr_recon *r, cudaStream_t st) {
  // a shared event still marks the other handles' point: take a fresh one
  if (!r->done || r->done.use_count() > 1) TRY(new_event(r->done));
  CU(cudaEventRecord(r->done->ev, st));
  r->last = st;
  return FR_OK;
}

int stream_leave_all(const std::vector<fr_recon *> &rs, cudaStream_t st,
                     std::shared_ptr<SharedEvent> *reuse) {
  std::shared_ptr<SharedEvent> e;
  if (reuse && *reuse) e = *reuse;
  else TRY(new_event(e));
  if (reuse) *reuse = e;
  CU(cudaEventRecord(e->ev, st));
  for (fr_recon *r : rs) {
    r->done = e;
    r->last = st;
  }
  return FR_OK;
}

// Builds the job view for the insertion kernels.
InsertJob make_job(fr_recon *r, const float2 *slices, const float *t3d, const float *pw,
                          int np) {
  InsertJob j;
  memset(&j, 0, sizeof j);   // padding too: jobs are compared bytewise for reuse
  j.data = r->vol_data.as<float>();
  j.norm = r->vol_norm.as<float>();
  j.slices = slices;
  j.t3d = t3d;
  j.pw = pw;
  j.xmax = r->geom->d_xmax;
  j.rtab = r->geom->d_rtab;
  j.rim = r->geom->d_rim;
  j.nrim = r->geom->nrim;
  j.ref = r->has_ref ? r->ref.as<float>() : nullptr;
  j.wsnr = nullptr;
  j.wundo = nullptr;
  j.nwsnr = 0;
  j.ssnr = nullptr;
  j.nssnr = 0;
  j.sscale = 1.0f;
  j.N = r->N;
  j.mode = r->mode;
  j.nsym = r->nsym;
  j.np = np;
  j.tiles_x = j.tiles_y = j.tiles_z = 0;
  j.nz = r->NZ != r->N ? r->NZ : 0;
  return j;
}

// Scatter (and edge) launches split so grid.y stays within 65535 slices.
int run_scatter(const InsertJob &j0, bool edge_only, cudaStream_t st) {
  const int per = std::max(1, 65535 / j0.nsym);
  for (int p0 = 0; p0 < j0.np; p0 += per) {
    InsertJob j = j0;
    j.np = std::min(per, j0.np - p0);
    j.slices = j0.slices + (size_t)p0 * j0.N * (j0.N / 2 + 1);
    j.t3d = j0.t3d + (size_t)p0 * j0.nsym * 9;
    j.pw = j0.pw + p0;
    if (j0.ssnr) j.ssnr = j0.ssnr + (size_t)p0 * j0.nssnr;
    if (j0.wsnr) j.wsnr = j0.wsnr + (size_t)p0 * j0.nwsnr;
    if (j0.wundo) j.wundo = j0.wundo + p0;
    CU(edge_only ? launch_edge(j, st) : launch_scatter(j, st));
  }
  return FR_OK;
}

// Inserts np device slices (t3d already composed, weights per particle).
int insert_device(fr_recon *r, const float2 *d_slices, const float *d_t3d, const float *d_pw,
                         int np, int schedule, const float *d_ssnr, int nssnr) {
  if (np == 0) return FR_OK;
  cudaStream_t st = r->stream;
  InsertJob j = make_job(r, d_slices, d_t3d, d_pw, np);
  if (d_ssnr) {
    j.ssnr = d_ssnr;
    j.nssnr = nssnr;
    j.sscale = (float)(2.0 * (nssnr - 1) / (float)r->N);
  }
  const int tuned = tuned_tile(r->N, r->mode, r->nsym);
  // the iterative inserter and non-cubic volumes: scatter only
  int sched = (r->mode == FR_MODE_ITER || r->NZ != r->N) ? FR_SCHED_SCATTER : schedule;
  if (sched == FR_SCHED_AUTO) {
    // Few slices: the per-tile culling and the volume read/write of the gather
    // pass are not amortised, so atomics win; a measured choice overrides.
    const long slices = (long)np * r->nsym;
    if (slices < 64) sched = FR_SCHED_SCATTER;
    else if (tuned == -2) sched = FR_SCHED_SCATTER;
    else if (tuned >= 0) sched = FR_SCHED_GATHER;
    else sched = (slices >= 256 && r->mode != FR_MODE_NEAREST) ? FR_SCHED_GATHER : FR_SCHED_SCATTER;
  }
  const bool prof = g_profile.load() != 0;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  if (prof)
    for (auto &e : ev) CU(cudaEventCreate(&e));
  g_ins_launches++;
  g_slices += (long long)np * r->nsym;
  if (sched == FR_SCHED_SCATTER || d_ssnr) {
    if (prof) CU(cudaEventRecord(ev[0], st));
    TRY(run_scatter(j, false, st));
    if (prof) {
      CU(cudaEventRecord(ev[2], st));
      CU(cudaEventSynchronize(ev[2]));
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[0], ev[2]);
      std::lock_guard<std::mutex> lk(g_stat_mu);
      g_insert_ms += ms;
      for (auto &e : ev) cudaEventDestroy(e);
    }
    return FR_OK;
  }
  int tile = r->tile >= 0 ? r->tile : (tuned >= 0 ? tuned : default_tile(r->mode, r->N, r->nsym, np));
  tile = effective_tile(tile, r->mode);
  if (r->tiles_tile != tile) {
    if (is_column_tile(tile))
      column_tiles(r->N, r->mode, r->p.corners, r->tiles, r->tx, r->ty, r->tz, &r->tile_dist);
    else gather_tiles(r->N, r->mode, tile, r->p.corners, r->tiles, r->tx, r->ty, r->tz);
    r->tiles_tile = tile;
    r->work_np = -1;
  }
  j.tiles_x = r->tx;
  j.tiles_y = r->ty;
  j.tiles_z = r->tz;
  const int nsl = np * r->nsym;
  int nwork = 0;
  const bool column = is_column_tile(tile);
  if (column) {
    // work items (job 0, tile, first slice of the block)
    if (r->work_np != nsl) {
      // Slice-bucket-major order: every item of a bucket (slice_bucket;
      // all block sizes divide it) before the next bucket, tiles nearest the
      // origin (heaviest) first within a bucket.  The CTAs in flight then
      // read one bucket's slices, mostly from L2, instead of each tile
      // streaming every slice from HBM.
      const int bucket = slice_bucket(r->N, r->nsym);
      std::vector<int4> work;
      for (int b0 = 0; b0 < nsl; b0 += bucket)
        for (size_t ti = 0; ti < r->tiles.size(); ti++) {
          const int blk = column_block(r->tile_dist[ti]);
          const int b1 = std::min(nsl, b0 + bucket);
          for (int s0 = b0; s0 < b1; s0 += blk)
            work.push_back(make_int4(0, r->tiles[ti], s0, std::min(b1, s0 + blk)));
        }
      TRY(r->s_work.ensure(sizeof(int4) * std::max<size_t>(1, work.size())));
      TRY(r->ring_small.upload(r->s_work.p, work.data(), sizeof(int4) * work.size(), st));
      r->work_np = nsl;
      r->nwork = (int)work.size();
    }
    nwork = r->nwork;
  } else if (r->work_np != -2) {
    std::vector<int2> work(r->tiles.size());
    for (size_t i = 0; i < work.size(); i++) work[i] = make_int2(0, r->tiles[i]);
    TRY(r->s_work.ensure(sizeof(int2) * std::max<size_t>(1, work.size())));
    TRY(r->ring_small.upload(r->s_work.p, work.data(), sizeof(int2) * work.size(), st));
    r->work_np = -2;
  }
  // the job in device memory: one of the last two uploaded when unchanged (an
  // upload queued behind a large copy would hold the stream up)
  const void *jobs_before = r->s_jobs.p;
  TRY(r->s_jobs.ensure(2 * sizeof(InsertJob)));
  if (r->s_jobs.p != jobs_before) r->job_valid[0] = r->job_valid[1] = false;
  TRY(r->s_counter.ensure(sizeof(int)));
  int jslot = -1;
  for (int q = 0; q < 2; q++)
    if (r->job_valid[q] && memcmp(&r->job_cache[q], &j, sizeof j) == 0) jslot = q;
  if (jslot < 0) {
    jslot = r->job_next;
    r->job_next ^= 1;
    TRY(r->ring_small.upload(r->s_jobs.as<InsertJob>() + jslot, &j, sizeof(InsertJob), st));
    r->job_cache[jslot] = j;
    r->job_valid[jslot] = true;
  }
  const InsertJob *d_job = r->s_jobs.as<InsertJob>() + jslot;
  if (prof) CU(cudaEventRecord(ev[0], st));
  if (tile == kPixelTile)
    CU(launch_pixel(d_job, r->s_work.as<int4>(), nwork, kColumnBlock,
                    r->s_counter.as<int>(), r->N, st));
  else if (tile == kColumn3Tile)
    CU(launch_column3(d_job, r->s_work.as<int4>(), nwork, kColumnBlock,
                      r->s_counter.as<int>(), r->N, st));
  else if (tile == kColumnTile)
    CU(launch_column(d_job, r->s_work.as<int4>(), nwork, kColumnBlock,
                     r->s_counter.as<int>(), r->mode, st));
  else
    CU(launch_gather(d_job, &j, 1, r->s_work.as<int2>(), (int)r->tiles.size(),
                     tile, r->s_counter.as<int>(), r->mode, st));
  if (prof) CU(cudaEventRecord(ev[1], st));
  TRY(run_scatter(j, true, st));
  g_gather_launches++;
  if (prof) {
    CU(cudaEventRecord(ev[2], st));
    CU(cudaEventSynchronize(ev[2]));
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[0], ev[2]);
    std::lock_guard<std::mutex> lk(g_stat_mu);
    g_gather_ms += a;
    g_insert_ms += b;
    for (auto &e : ev) cudaEventDestroy(e);
  }
  // Host-side sources above (work list, job struct) are pageable: the copies
  // have taken them by the time cudaMemcpyAsync returns.  Later calls reuse
  // the scratch in stream order (stream_enter for another stream).
  return FR_OK;
}

int check_device_error(fr_recon *r) {
  int h = 0;
  CU(cudaStreamSynchronize(r->stream));
  CU(cudaMemcpy(&h, consts().d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(consts().d_err, 0, sizeof(int));
    return fail(FR_EDEVICE, "insertion kernel reported inconsistency code %d", h);
  }
  return FR_OK;
}

int alloc_volume(fr_recon *r) {
  TRY(r->vol_data.ensure(rvol_floats(r) * sizeof(float)));
  TRY(r->vol_norm.ensure(rnorm_floats(r) * sizeof(float)));
  TRY(r->d_sym.ensure(sizeof(float) * r->syms.size()));
  CU(cudaMemcpyAsync(r->d_sym.p, r->syms.data(), sizeof(float) * r->syms.size(),
                     cudaMemcpyHostToDevice, r->stream));
  return FR_OK;
}

// The caller pipeline of programs/e2spa_make3d.py:300-345 for one chunk of
// particles already on the device, in two halves: the host half turns the
// particles' metadata into one block of device-ready arrays, the device half
// is kernels and FFTs only (so it can be captured in a CUDA graph).

size_t prologue_meta_bytes(int n) {
  return ctf_dev_size() * (size_t)n + sizeof(float) * 12 * (size_t)n;
}

// Writes [CTF constants: ctf_dev_size()*n][txy: 2n][w: n][rot: 9n] into blk;
// returns whether any particle carries a CTF.
bool prologue_meta(int N, int n, const fr_particle *meta, unsigned char *blk) {
  return prologue_meta_range(N, n, 0, n, meta, blk);
}

bool prologue_meta_range(int N, int n, int first, int count, const fr_particle *meta,
                         unsigned char *blk) {
  const size_t cs = ctf_dev_size();
  float *txy = reinterpret_cast<float *>(blk + cs * n);
  float *w = txy + 2 * (size_t)n;
  float *rot = w + n;
  bool any_ctf = false;
  for (int i = first; i < first + count; i++) {
    const fr_particle &m = meta[i - first];
    ctf_constants(m.defocus, m.dfdiff, m.dfang, m.voltage, m.cs, m.apix, m.ampcont, N,
                  blk + cs * i);
    if (std::fabs(m.defocus) > 1e-4f) any_ctf = true;
    // ts = inverse of the translation-only part of xform.projection; the
    // bilinear xform then applies ts^-1, i.e. +(tx, ty) (programs/e2spa_make3d.py:339-342).
    txy[2 * i] = m.tx;
    txy[2 * i + 1] = m.ty;
    w[i] = m.weight > 0 ? m.weight : 0.0f;   // wt <= 0: skipped (programs/e2spa_make3d.py:304)
    memcpy(&rot[9 * (size_t)i], m.rot, sizeof(float) * 9);
  }
  return any_ctf;
}

MetaView meta_view(const unsigned char *d_meta, int n) {
  MetaView v;
  v.ctf = d_meta;
  v.txy = reinterpret_cast<const float *>(d_meta + ctf_dev_size() * (size_t)n);
  v.w = v.txy + 2 * (size_t)n;
  v.rot = v.w + n;
  return v;
}

// Copies a metadata block to the handle's device block (s_meta).
int prologue_upload(fr_recon *r, int n, const unsigned char *blk, cudaStream_t st) {
  const size_t bytes = prologue_meta_bytes(n);
  TRY(r->s_meta.ensure(bytes));
  CU(cudaMemcpyAsync(r->s_meta.p, blk, bytes, cudaMemcpyHostToDevice, st));
  r->d_meta = r->s_meta.as<unsigned char>();
  return FR_OK;
}

int prologue_run(PlanCache &plans, const ProScratch &b, const unsigned char *d_meta,
                 const float *d_raw, const float *const *d_src, int n, int box, int N,
                 const float *d_sym, int nsym, bool any_ctf, cudaStream_t st, bool exact_fft,
                 const PartSym *d_psym, long nslices) {
  const size_t img = (size_t)N * N, spec = (size_t)N * (N / 2 + 1);
  const MetaView mv = meta_view(d_meta, n);
  TRY(b.img->ensure(sizeof(float) * img * n));
  TRY(b.slices->ensure(sizeof(float) * slice_floats(N) * n));
  TRY(b.spec->ensure(std::max(sizeof(cufftComplex) * spec, sizeof(float) * img) * n));
  TRY(b.t3d->ensure(sizeof(float) * 9 * (size_t)(nslices >= 0 ? nslices : (long)n * nsym)));
  if (any_ctf) TRY(b.img2->ensure(sizeof(float) * img * n));
  CU(launch_pad_compose(d_raw, d_src, n, box, N, b.img->as<float>(), mv.rot, d_sym, nsym,
                        b.t3d->as<float>(), st, d_psym));
  const float *img_on = nullptr;
  if (any_ctf) {
    TRY(plans.exec2d(true, N, n, b.img->p, b.spec->p, st, exact_fft));
    CU(launch_ctf_flip_dev(b.spec->as<cufftComplex>(), mv.ctf, n, N, st));
    TRY(plans.exec2d(false, N, n, b.spec->p, b.img2->p, st, exact_fft));
    img_on = b.img2->as<float>();
  }
  // edge mean (in the shift kernel); preprocess_slice: shift, phase origin
  // to corner, x sqrt((N+2)/N), r2c.  spec is the real staging for the r2c
  // input.
  volatile float inv = 1.0f / (float)N;
  const float scale = sqrtf(inv * (float)(N + 2));
  CU(launch_shift_corner(b.img->as<float>(), img_on, any_ctf ? mv.ctf : nullptr, nullptr, mv.txy,
                         2, n, N, scale, b.spec->as<float>(), st, true));
  TRY(plans.exec2d(true, N, n, b.spec->p, b.slices->p, st, exact_fft));
  return FR_OK;
}

int prologue_device(fr_recon *r, const float *d_raw, int n, int box, bool any_ctf) {
  const ProScratch b{&r->s_img, &r->s_slices, &r->s_spec, &r->s_t3d, &r->s_img2};
  return prologue_run(r->plans, b, r->d_meta, d_raw, nullptr, n, box, r->N, r->d_sym.as<float>(),
                      r->nsym, any_ctf, r->stream);
}

int prologue_chunk(fr_recon *r, const float *d_raw, int n, int box, const fr_particle *meta) {
  int k;
  unsigned char *blk;
  TRY(r->ring_meta.acquire(prologue_meta_bytes(n), &k, &blk));
  const bool any_ctf = prologue_meta(r->N, n, meta, blk);
  TRY(prologue_upload(r, n, blk, r->stream));
  TRY(r->ring_meta.done(k, r->stream));
  return prologue_device(r, d_raw, n, box, any_ctf);
}

int particles_chunk(fr_recon *r, const float *d_raw, int n, int box, const fr_particle *meta,
                    int schedule) {
  TRY(prologue_chunk(r, d_raw, n, box, meta));
  return insert_device(r, r->s_slices.as<float2>(), r->s_t3d.as<float>(), meta_view(r->d_meta, n).w, n,
                       schedule, nullptr, 0);
}

}  // namespace fr

// ================================================================== C ABI
extern "C" {

const char *fr_last_error(void) { return g_err.c_str(); }

int fr_profile(int on) {
  g_profile = on ? 1 : 0;
  return FR_OK;
}

int fr_stats_get(fr_stats *out) {
  if (!out) return fail(FR_ENULL, "null argument");
  out->kernel_launches = g_launches.load();
  out->insert_launches = g_ins_launches.load();
  out->slices_inserted = g_slices.load();
  out->gather_launches = g_gather_launches.load();
  std::lock_guard<std::mutex> lk(g_stat_mu);
  out->insert_ms = g_insert_ms;
  out->gather_ms = g_gather_ms;
  return FR_OK;
}

int fr_stats_reset(void) {
  g_launches = 0;
  g_ins_launches = 0;
  g_slices = 0;
  g_gather_launches = 0;
  std::lock_guard<std::mutex> lk(g_stat_mu);
  g_insert_ms = g_gather_ms = 0.0;
  return FR_OK;
}
const char *fr_version(void) { return "eman2_b200 0.1 (sm_100a)"; }

size_t fr_footprint_bytes(int N) {
  return (vol_floats(N) + norm_floats(N)) * sizeof(float);
}

int fr_sym_ops(const char *sym, float *out, int cap) {
  if (!sym) return -1;
  std::vector<float> v;
  const int n = sym_ops(sym, v);
  if (n < 0) return -1;
  if (out) {
    if (cap < n) return -1;
    memcpy(out, v.data(), sizeof(float) * 9 * n);
  }
  return n;
}

int fr_create(const fr_params *p, fr_recon **out) {
  if (!p || !out) return fail(FR_ENULL, "null argument");
  *out = nullptr;
  if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0)
    return fail(FR_EINVAL_PARAM, "size must be three positive integers");
  // square slices into an nx x nx x nz volume (e.g. programs/e2tomogram.py:2024,
  // size=[pad,pad,zthick]); a z size other than nx takes the scatter path
  if (p->nx != p->ny)
    return fail(FR_EUNSUPPORTED, "size %d %d %d: x and y must be equal (square slices)", p->nx,
                p->ny, p->nz);
  if (p->nx % 2 || p->nz % 2)
    return fail(FR_EUNSUPPORTED, "odd sizes (fftodd volumes) are not supported (size %d %d %d)",
                p->nx, p->ny, p->nz);
  if (p->nx < 4 || p->nx > 4094 || p->nz < 4 || p->nz > 4094)
    return fail(FR_EUNSUPPORTED, "size %d %d %d outside [4, 4094]", p->nx, p->ny, p->nz);
  if (p->nz != p->nx && p->mode == FR_MODE_ITER)
    return fail(FR_EUNSUPPORTED, "the iterative reconstructor needs a cubic volume");
  if (p->mode != FR_MODE_NEAREST && p->mode != FR_MODE_GAUSS2 && p->mode != FR_MODE_GAUSS5 &&
      p->mode != FR_MODE_TRILINEAR && p->mode != FR_MODE_ITER)
    return fail(FR_EUNSUPPORTED, "inserter mode %d is not built", p->mode);
  std::vector<float> ops;
  const int ns = sym_ops(p->sym, ops);
  if (ns < 0) return fail(FR_EUNSUPPORTED, "symmetry '%s' is not supported (c<n>, d<n> up to 1000 operators, tet, oct, icos)", p->sym);
  fr_recon *r = new fr_recon();
  r->p = *p;
  r->N = p->nx;
  r->NZ = p->nz;
  r->mode = p->mode;
  r->nsym = ns;
  r->syms = ops;
  if (cudaStreamCreateWithFlags(&r->own, cudaStreamNonBlocking) != cudaSuccess) {
    delete r;
    return fail(FR_ECUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  r->stream = r->own;
  if (new_event(r->done) != FR_OK) {
    cudaStreamDestroy(r->own);
    delete r;
    return fail(FR_ECUDA, "cudaEventCreate failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  consts();
  r->geom = get_geom(r->N, p->mode == FR_MODE_ITER ? 3 : p->corners);
  *out = r;
  return FR_OK;
}

int fr_destroy(fr_recon *r) {
  if (!r) return FR_OK;
  {
    std::lock_guard<std::mutex> lk(r->mu);
    if (r->last) cudaEventSynchronize(r->done->ev);
    if (r->stream) cudaStreamSynchronize(r->stream);
    DevBuf *bufs[] = {&r->vol_data, &r->vol_norm, &r->d_sym, &r->s_in, &r->s_slices, &r->s_rot,
                      &r->s_meta, &r->ref,
                      &r->s_w, &r->s_t3d, &r->s_img, &r->s_img2, &r->s_spec, &r->s_ctf,
                      &r->s_txy, &r->s_out, &r->s_ssnr, &r->s_jobs, &r->s_work,
                      &r->s_counter};
    for (DevBuf *b : bufs) b->release();
    for (int k = 0; k < 2; k++) {
      r->s_stage[k].release();
      if (r->staged[k]) cudaEventDestroy(r->staged[k]);
      if (r->consumed[k]) cudaEventDestroy(r->consumed[k]);
    }
    r->ring_meta.release();
    r->ring_small.release();
    if (r->copy_st) {
      cudaStreamSynchronize(r->copy_st);
      cudaStreamDestroy(r->copy_st);
    }
    r->done.reset();
    if (r->own) cudaStreamDestroy(r->own);
  }
  delete r;
  return FR_OK;
}

int fr_set_stream(fr_recon *r, void *stream) {
  if (!r) return fail(FR_ENULL, "null handle");
  std::lock_guard<std::mutex> lk(r->mu);
  r->stream = stream ? (cudaStream_t)stream : r->own;
  return FR_OK;
}

int fr_get_stream(const fr_recon *r, void **stream) {
  if (!r || !stream) return fail(FR_ENULL, "null argument");
  *stream = (void *)r->stream;
  return FR_OK;
}

int fr_get_size(const fr_recon *r, int *N) {
  if (!r || !N) return fail(FR_ENULL, "null argument");
  *N = r->N;
  return FR_OK;
}

int fr_setup(fr_recon *r) {
  if (!r) return fail(FR_ENULL, "null handle");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  TRY(alloc_volume(r));
  CU(cudaMemsetAsync(r->vol_data.p, 0, rvol_floats(r) * sizeof(float), r->stream));
  CU(cudaMemsetAsync(r->vol_norm.p, 0, rnorm_floats(r) * sizeof(float), r->stream));
  CU(cudaStreamSynchronize(r->stream));
  r->has_ref = false;   // FourierIterReconstructor::setup drops the reference volume
  if (r->p.verbose) {
    printf("3D Fourier dimensions are %d %d %d\n", r->N + 2, r->N, r->N);
    printf("You will require approximately %1.3g GB of memory to reconstruct this volume\n",
           ((float)(r->N + 2) * r->N * r->N * sizeof(float) * 1.5) / 1000000000.0);
  }
  r->state = 1;
  return FR_OK;
}

int fr_setup_seed(fr_recon *r, const float *seed, float seed_weight) {
  if (!r) return fail(FR_ENULL, "null handle");
  TRY(require_cubic(r, "setup_seed"));
  if (!seed) return fail(FR_ENULL, "null seed volume");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  TRY(alloc_volume(r));
  const void *d = nullptr;
  TRY(to_device(seed, vol_floats(r->N) * sizeof(float), r->s_in, r->stream, &d));
  CU(launch_seed((const float *)d, seed_weight, r->N, r->vol_data.as<float>(),
                 r->vol_norm.as<float>(), r->stream));
  CU(cudaStreamSynchronize(r->stream));
  r->state = 1;
  return FR_OK;
}

int fr_setup_seedandweights(fr_recon *r, const float *seed, const float *weights) {
  if (!r) return fail(FR_ENULL, "null handle");
  TRY(require_cubic(r, "setup_seedandweights"));
  if (!seed || !weights) return fail(FR_ENULL, "null seed or weight volume");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  TRY(alloc_volume(r));
  const cudaMemcpyKind k1 = is_device_ptr(seed) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind k2 = is_device_ptr(weights) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CU(cudaMemcpyAsync(r->vol_data.p, seed, vol_floats(r->N) * sizeof(float), k1, r->stream));
  CU(cudaMemcpyAsync(r->vol_norm.p, weights, norm_floats(r->N) * sizeof(float), k2, r->stream));
  CU(cudaStreamSynchronize(r->stream));
  r->state = 1;
  return FR_OK;
}

int fr_clear(fr_recon *r) {
  TRY(check_state(r));
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  CU(cudaMemsetAsync(r->vol_data.p, 0, rvol_floats(r) * sizeof(float), r->stream));
  CU(cudaMemsetAsync(r->vol_norm.p, 0, rnorm_floats(r) * sizeof(float), r->stream));
  CU(cudaStreamSynchronize(r->stream));
  return FR_OK;
}

// preprocess_slice for n device images into n device slices (scratch owned by r).
static int preprocess_device(fr_recon *r, const float *d_imgs, int n, const float *d_txy,
                             int txy_stride, float *d_out_slices) {
  const int N = r->N;
  cudaStream_t st = r->stream;
  TRY(r->s_img2.ensure(sizeof(float) * (size_t)n * N * N));
  // sqrt(1.0f/ysize * xsize) with ysize = N, xsize = N+2 (libEM/reconstructor.cpp:1054)
  volatile float inv = 1.0f / (float)N;
  const float scale = sqrtf(inv * (float)(N + 2));
  CU(launch_shift_corner(d_imgs, nullptr, nullptr, nullptr, d_txy, txy_stride, n, N, scale,
                         r->s_img2.as<float>(), st));
  TRY(r->plans.exec2d(true, N, n, r->s_img2.p, d_out_slices, st));
  return FR_OK;
}

int fr_preprocess_slices(fr_recon *r, const float *imgs, int n, const float *inv_txy,
                         float *out_slices) {
  if (!r) return fail(FR_ENULL, "null handle");
  if (n < 0) return fail(FR_EINVAL_PARAM, "negative count");
  if (n == 0) return FR_OK;
  if (!imgs || !out_slices) return fail(FR_ENULL, "null image or output");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  const void *d_in = nullptr, *d_t = nullptr;
  TRY(to_device(imgs, sizeof(float) * (size_t)n * N * N, r->s_in, r->stream, &d_in));
  if (inv_txy) TRY(to_device(inv_txy, sizeof(float) * 2 * n, r->s_txy, r->stream, &d_t));
  const bool dev_out = is_device_ptr(out_slices);
  float *d_out = out_slices;
  if (!dev_out) {
    TRY(r->s_out.ensure(sizeof(float) * slice_floats(N) * n));
    d_out = r->s_out.as<float>();
  }
  TRY(preprocess_device(r, (const float *)d_in, n, (const float *)d_t, 2, d_out));
  if (!dev_out) TRY(from_device(out_slices, d_out, sizeof(float) * slice_floats(N) * n, r->stream));
  else CU(cudaStreamSynchronize(r->stream));
  return FR_OK;
}

int fr_insert_slices(fr_recon *r, const float *slices, int n, const float *rot, const float *weights,
                     const float *ssnr, int nssnr, int *status_out, int schedule) {
  TRY(check_state(r));
  if (n < 0) return fail(FR_EINVAL_PARAM, "negative count");
  if (n == 0) return FR_OK;
  if (!slices || !rot || !weights) return fail(FR_ENULL, "EMData pointer (input image) is NULL");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  // insert_slice (libEM/reconstructor.cpp:1080-1090): usessnr turns the weight
  // into the SSNR flag (-1) when class_ssnr is present, else into 0; a zero
  // weight returns -1 without inserting.
  std::vector<float> w(n);
  const bool wdev = is_device_ptr(weights);
  if (wdev) CU(cudaMemcpy(w.data(), weights, sizeof(float) * n, cudaMemcpyDeviceToHost));
  else memcpy(w.data(), weights, sizeof(float) * n);
  const bool have_ssnr = ssnr && nssnr > 0;
  if (r->p.usessnr) {
    for (int i = 0; i < n; i++) w[i] = have_ssnr ? -1.0f : 0.0f;
  }
  // A negative weight selects the SSNR path (libEM/reconstructor.cpp:1158-1162),
  // which reads the slice's class_ssnr attribute; without it the reference
  // throws NotExistingObjectException (libEM/emdata_metadata.cpp:1142).
  bool any_neg = false;
  for (int i = 0; i < n; i++) any_neg |= w[i] < 0.0f;
  if (r->mode == FR_MODE_ITER) any_neg = false;   // its insert_slice takes any weight as is
  if (any_neg && !have_ssnr)
    return fail(FR_ENOTEXIST, "The requested key does not exist: class_ssnr (a negative weight "
                "selects the SSNR insertion path)");
  for (int i = 0; i < n; i++)
    if (status_out) status_out[i] = (w[i] == 0.0f) ? -1 : 0;
  const bool use_ssnr = any_neg;
  const void *d_sl = nullptr, *d_rot = nullptr, *d_ss = nullptr;
  TRY(to_device(slices, sizeof(float) * slice_floats(N) * n, r->s_in, st, &d_sl));
  TRY(to_device(rot, sizeof(float) * 9 * n, r->s_rot, st, &d_rot));
  if (use_ssnr)
    TRY(to_device(ssnr, sizeof(float) * (size_t)nssnr * n, r->s_ssnr, st, &d_ss));
  TRY(r->s_w.ensure(sizeof(float) * n));
  TRY(r->ring_small.upload(r->s_w.p, w.data(), sizeof(float) * n, st));
  TRY(r->s_t3d.ensure(sizeof(float) * 9 * (size_t)n * r->nsym));
  CU(launch_compose((const float *)d_rot, r->d_sym.as<float>(), n, r->nsym, r->s_t3d.as<float>(),
                    st));
  TRY(insert_device(r, (const float2 *)d_sl, r->s_t3d.as<float>(), r->s_w.as<float>(), n, schedule,
                    (const float *)d_ss, nssnr));
  TRY(stream_leave(r, st));
  // Host sources may be pinned, read by DMA after the call returns: finish
  // those reads before handing the buffers back to the caller.
  if (d_sl != slices || d_rot != rot || (use_ssnr && d_ss != ssnr)) CU(cudaStreamSynchronize(st));
  return FR_OK;
}

int fr_set_reference(fr_recon *r, const float *vol, int is_complex) {
  TRY(check_state(r));
  TRY(require_cubic(r, "the iterative reconstructor"));
  if (!vol) return fail(FR_ENULL, "null reference volume");
  if (r->mode != FR_MODE_ITER)
    return fail(FR_EINVAL_PARAM, "a reference volume belongs to the iterative reconstructor");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  TRY(r->ref.ensure(vol_floats(N) * sizeof(float)));
  if (is_complex) {
    const cudaMemcpyKind k = is_device_ptr(vol) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CU(cudaMemcpyAsync(r->ref.p, vol, vol_floats(N) * sizeof(float), k, st));
  } else {
    // seed->do_fft() after xform.phaseorigin.tocorner (libEM/reconstructor.cpp:481-488)
    const size_t n3 = (size_t)N * N * N;
    const void *d = nullptr;
    TRY(to_device(vol, n3 * sizeof(float), r->s_in, st, &d));
    TRY(r->s_out.ensure(n3 * sizeof(float)));
    CU(launch_tocorner3(static_cast<const float *>(d), N, r->s_out.as<float>(), st));
    cufftHandle plan;
    TRY(r->plans.get3d_r2c(N, st, &plan));
    CUFFT(cufftExecR2C(plan, r->s_out.as<cufftReal>(), r->ref.as<cufftComplex>()));
  }
  CU(cudaStreamSynchronize(st));
  r->has_ref = true;
  r->job_valid[0] = r->job_valid[1] = false;
  return FR_OK;
}

int fr_set_wiener(fr_recon *r, int on) {
  if (!r) return fail(FR_ENULL, "null handle");
  std::lock_guard<std::mutex> lk(r->mu);
  r->wfilt = on ? 1.0f : 0.0f;
  return FR_OK;
}

int fr_insert_slices_wiener(fr_recon *r, const float *slices, int n, const float *rot,
                            const float *weights, const float *snr, int nsnr, const int *undo,
                            int *status_out) {
  TRY(check_state(r));
  TRY(require_cubic(r, "wiener_fourier insertion"));
  if (n < 0) return fail(FR_EINVAL_PARAM, "negative count");
  if (n == 0) return FR_OK;
  if (!slices || !rot || !weights) return fail(FR_ENULL, "EMData pointer (input image) is NULL");
  if (!snr || nsnr < 1)
    return fail(FR_ENOTEXIST, "The requested key does not exist: ctf_snr_total (No SNR "
                "information present in class-average. Must use the ctf.auto or ctfw.auto averager.)");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  if (!r->wgeom) r->wgeom = get_geom(N, 2);
  // WienerFourierReconstructor::insert_slice (libEM/reconstructor.cpp:1643-1677)
  // inserts every slice (a zero weight still enters through the SNR weights);
  // the sign of the weight selects subtraction.
  std::vector<float> w(n);
  if (is_device_ptr(weights)) CU(cudaMemcpy(w.data(), weights, sizeof(float) * n, cudaMemcpyDeviceToHost));
  else memcpy(w.data(), weights, sizeof(float) * n);
  for (int i = 0; i < n; i++) {
    w[i] = w[i] < 0.0f ? -1.0f : 1.0f;
    if (status_out) status_out[i] = 0;
  }
  const void *d_sl = nullptr, *d_rot = nullptr, *d_snr = nullptr, *d_undo = nullptr;
  TRY(to_device(slices, sizeof(float) * slice_floats(N) * n, r->s_in, st, &d_sl));
  TRY(to_device(rot, sizeof(float) * 9 * n, r->s_rot, st, &d_rot));
  TRY(to_device(snr, sizeof(float) * (size_t)nsnr * n, r->s_ssnr, st, &d_snr));
  if (undo) TRY(to_device(undo, sizeof(int) * n, r->s_txy, st, &d_undo));
  TRY(r->s_w.ensure(sizeof(float) * n));
  TRY(r->ring_small.upload(r->s_w.p, w.data(), sizeof(float) * n, st));
  TRY(r->s_t3d.ensure(sizeof(float) * 9 * (size_t)n * r->nsym));
  CU(launch_compose((const float *)d_rot, r->d_sym.as<float>(), n, r->nsym, r->s_t3d.as<float>(),
                    st));
  InsertJob j = make_job(r, (const float2 *)d_sl, r->s_t3d.as<float>(), r->s_w.as<float>(), n);
  j.xmax = r->wgeom->d_xmax;
  j.wsnr = (const float *)d_snr;
  j.nwsnr = nsnr;
  j.wundo = (const int *)d_undo;
  g_ins_launches++;
  g_slices += (long long)n * r->nsym;
  TRY(run_scatter(j, false, st));
  TRY(stream_leave(r, st));
  if (d_sl != slices || d_rot != rot || d_snr != snr || (undo && d_undo != undo))
    CU(cudaStreamSynchronize(st));
  return FR_OK;
}

int fr_insert_particles(fr_recon *r, const float *imgs, int n, int box, const fr_particle *meta,
                        int schedule) {
  TRY(check_state(r));
  if (n < 0 || box <= 0) return fail(FR_EINVAL_PARAM, "bad particle count or box");
  if (n == 0) return FR_OK;
  if (!imgs || !meta) return fail(FR_ENULL, "EMData pointer (input image) is NULL");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  // Chunk so the per-chunk scratch (about 5 N^2 floats per particle) stays near 8 GiB.
  const size_t per = (size_t)N * N * 4 * 5 + (size_t)box * box * 4;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(8192, (8ull << 30) / per));
  const bool dev = is_device_ptr(imgs);
  if (!dev && !r->copy_st) {
    CU(cudaStreamCreateWithFlags(&r->copy_st, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
      CU(cudaEventCreateWithFlags(&r->staged[k], cudaEventDisableTiming));
      CU(cudaEventCreateWithFlags(&r->consumed[k], cudaEventDisableTiming));
    }
  }
  int last = -1;
  for (int p0 = 0; p0 < n; p0 += chunk) {
    const int c = std::min(chunk, n - p0);
    const float *src = imgs + (size_t)p0 * box * box;
    if (dev) {
      TRY(particles_chunk(r, src, c, box, meta + p0, schedule));
      continue;
    }
    // Host images: the chunk's images and its metadata block go, on the copy
    // stream, into the staging buffer the chunk before last used, once the
    // work that read it is done.  Nothing is uploaded on the compute stream,
    // where it would queue behind this copy on the copy engine.
    const int k = r->stage_next;
    r->stage_next ^= 1;
    const size_t ibytes = sizeof(float) * (size_t)c * box * box;
    const size_t moff = (ibytes + 255) & ~(size_t)255;
    const size_t bytes = moff + prologue_meta_bytes(c);
    if (r->s_stage[k].cap < bytes) {
      if (r->consumed_set[k]) CU(cudaEventSynchronize(r->consumed[k]));
      TRY(r->s_stage[k].ensure(bytes));
    }
    int slot;
    unsigned char *blk;
    TRY(r->ring_meta.acquire(prologue_meta_bytes(c), &slot, &blk));
    const bool any_ctf = prologue_meta(r->N, c, meta + p0, blk);
    if (r->consumed_set[k]) CU(cudaStreamWaitEvent(r->copy_st, r->consumed[k], 0));
    unsigned char *stage = r->s_stage[k].as<unsigned char>();
    CU(cudaMemcpyAsync(stage + moff, blk, prologue_meta_bytes(c), cudaMemcpyHostToDevice, r->copy_st));
    TRY(r->ring_meta.done(slot, r->copy_st));
    CU(cudaMemcpyAsync(stage, src, ibytes, cudaMemcpyHostToDevice, r->copy_st));
    CU(cudaEventRecord(r->staged[k], r->copy_st));
    CU(cudaStreamWaitEvent(r->stream, r->staged[k], 0));
    last = k;
    r->d_meta = stage + moff;
    TRY(prologue_device(r, (const float *)stage, c, box, any_ctf));
    TRY(insert_device(r, r->s_slices.as<float2>(), r->s_t3d.as<float>(), meta_view(r->d_meta, c).w,
                      c, schedule, nullptr, 0));
    CU(cudaEventRecord(r->consumed[k], r->stream));
    r->consumed_set[k] = true;
  }
  TRY(stream_leave(r, r->stream));
  // host images may be pinned: return once they are read, not once inserted
  if (last >= 0) CU(cudaEventSynchronize(r->staged[last]));
  return FR_OK;
}

int fr_determine_slice_agreement(fr_recon *r, const float *slices, int n, const float *rot,
                                 const float *weights, float apix, int sub, float *out) {
  TRY(check_state(r));
  TRY(require_cubic(r, "determine_slice_agreement"));
  if (n < 0) return fail(FR_EINVAL_PARAM, "negative count");
  if (n == 0) return FR_OK;
  if (!slices || !rot || !weights || !out) return fail(FR_ENULL, "EMData pointer (input image) is NULL");
  if (sub)
    return fail(FR_ENOTEXIST,
                "class_ssnr: sub=True inserts the slice through the SSNR path, which needs the "
                "class_ssnr attribute (NotExistingObjectException in the reference)");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  const void *d_sl = nullptr, *d_rot = nullptr, *d_w = nullptr;
  TRY(to_device(slices, sizeof(float) * slice_floats(N) * n, r->s_in, st, &d_sl));
  TRY(to_device(rot, sizeof(float) * 9 * n, r->s_rot, st, &d_rot));
  TRY(to_device(weights, sizeof(float) * n, r->s_w, st, &d_w));
  TRY(r->s_t3d.ensure(sizeof(float) * 9 * (size_t)n * r->nsym));
  CU(launch_compose((const float *)d_rot, r->d_sym.as<float>(), n, r->nsym, r->s_t3d.as<float>(), st));
  const bool dev_out = is_device_ptr(out);
  float *d_out = out;
  if (!dev_out) {
    TRY(r->s_out.ensure(sizeof(float) * 5 * n));
    d_out = r->s_out.as<float>();
  }
  CU(launch_agree_rt(r->vol_data.as<float>(), r->vol_norm.as<float>(), N, (const float *)d_sl,
                     r->s_t3d.as<float>(), n, r->nsym, (const float *)d_w, apix, r->geom->d_rtab,
                     d_out, st));
  if (!dev_out) TRY(from_device(out, d_out, sizeof(float) * 5 * n, st));
  else CU(cudaStreamSynchronize(st));
  return FR_OK;
}

int fr_projection_xf(fr_recon *r, const float *xf, int ret_fourier, float *out) {
  TRY(check_state(r));
  TRY(require_cubic(r, "projection"));
  if (!xf || !out) return fail(FR_ENULL, "null argument");
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  // the rotation block (the reference drops scale, mirror and translation
  // for the slice itself) and the translation the result is shifted by
  float h[12];
  if (is_device_ptr(xf)) CU(cudaMemcpy(h, xf, sizeof h, cudaMemcpyDeviceToHost));
  else memcpy(h, xf, sizeof h);
  const float rot[9] = {h[0], h[1], h[2], h[4], h[5], h[6], h[8], h[9], h[10]};
  TRY(r->s_rot.ensure(sizeof rot));
  CU(cudaMemcpyAsync(r->s_rot.p, rot, sizeof rot, cudaMemcpyHostToDevice, st));
  TRY(r->s_out.ensure(sizeof(float) * (slice_floats(N) + (size_t)N * N)));
  float *spec = r->s_out.as<float>();
  CU(cudaMemsetAsync(spec, 0, sizeof(float) * slice_floats(N), st));
  CU(launch_projection_rt(r->vol_data.as<float>(), r->vol_norm.as<float>(), N, r->s_rot.as<float>(),
                          r->geom->d_rtab, spec, st));
  CU(launch_proj_shift(spec, N, h[3], h[7], ret_fourier ? 0 : 1, ret_fourier ? 0 : 1, st));
  if (ret_fourier) {
    TRY(from_device(out, spec, sizeof(float) * slice_floats(N), st));
    return FR_OK;
  }
  // do_ift (libEM/emdata_transform.cpp:330-375): inverse real FFT, then each
  // value times 1.0f / (N*N)
  float *real = spec + slice_floats(N);
  TRY(r->plans.exec2d(false, N, 1, spec, real, st));
  const float scale = 1.0f / (float)(N * N);
  CU(launch_scale(real, (size_t)N * N, scale, real, st));
  TRY(from_device(out, real, sizeof(float) * (size_t)N * N, st));
  return FR_OK;
}

int fr_projection(fr_recon *r, const float *rot, float *out_slice) {
  if (!rot || !out_slice) return fail(FR_ENULL, "null argument");
  float h[9];
  if (is_device_ptr(rot)) CU(cudaMemcpy(h, rot, sizeof h, cudaMemcpyDeviceToHost));
  else memcpy(h, rot, sizeof h);
  const float xf[12] = {h[0], h[1], h[2], 0.f, h[3], h[4], h[5], 0.f, h[6], h[7], h[8], 0.f};
  return fr_projection_xf(r, xf, 1, out_slice);
}

int fr_get_accumulators(fr_recon *r, float *data, float *norm) {
  TRY(check_state(r));
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  TRY(check_device_error(r));
  if (data) TRY(from_device(data, r->vol_data.p, rvol_floats(r) * sizeof(float), r->stream));
  if (norm) TRY(from_device(norm, r->vol_norm.p, rnorm_floats(r) * sizeof(float), r->stream));
  return FR_OK;
}

int fr_finish(fr_recon *r, int doift, float *out, float *normout) {
  TRY(check_state(r));
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  const int N = r->N;
  cudaStream_t st = r->stream;
  TRY(check_device_error(r));
  const int NZ = r->NZ, nz = NZ != N ? NZ : 0;
  CU(launch_normalize(r->vol_data.as<float>(), r->vol_norm.as<float>(), N, r->p.sqrtnorm, st,
                      r->wfilt, nz));
  if (normout) TRY(from_device(normout, r->vol_norm.p, rnorm_floats(r) * sizeof(float), st));
  if (doift) {
    cufftHandle plan;
    TRY(r->plans.get3d(N, st, &plan, NZ));
    CUFFT(cufftExecC2R(plan, r->vol_data.as<cufftComplex>(), r->vol_data.as<cufftReal>()));
    // do_ift scale 1.0f / (nx*ny*nz) (libEM/emdata_transform.cpp:411-412)
    const size_t nreal = (size_t)N * N * NZ;
    const float scale = 1.0f / (float)nreal;
    if (out) {
      if (is_device_ptr(out)) {
        CU(launch_depad_center(r->vol_data.as<float>(), N, scale, out, st, nz));
        CU(cudaStreamSynchronize(st));
      } else {
        TRY(r->s_out.ensure(sizeof(float) * nreal));
        CU(launch_depad_center(r->vol_data.as<float>(), N, scale, r->s_out.as<float>(), st, nz));
        TRY(from_device(out, r->s_out.p, sizeof(float) * nreal, st));
      }
    }
  } else if (out) {
    TRY(from_device(out, r->vol_data.p, rvol_floats(r) * sizeof(float), st));
  }
  CU(cudaStreamSynchronize(st));
  r->state = 2;
  return FR_OK;
}

// Page-locked host memory (cudaHostAlloc / cudaHostRegister): the copy
// engine reads and writes it without a staging copy, so copies into it are
// asynchronous.
static bool is_pinned_host(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int fr_finish_async(fr_recon *r, int doift, float *out, float *normout, void *stream) {
  TRY(check_state(r));
  for (const void *b : {(const void *)out, (const void *)normout})
    if (b && !is_device_ptr(b) && !is_pinned_host(b))
      return fail(FR_EINVAL_PARAM, "fr_finish_async writes device or page-locked host memory only");
  std::lock_guard<std::mutex> lk(r->mu);
  cudaStream_t st = stream ? (cudaStream_t)stream : r->stream;
  TRY(stream_enter(r, st));
  const int N = r->N, NZ = r->NZ, nz = NZ != N ? NZ : 0;
  CU(launch_normalize(r->vol_data.as<float>(), r->vol_norm.as<float>(), N, r->p.sqrtnorm, st,
                      r->wfilt, nz));
  if (normout)
    CU(cudaMemcpyAsync(normout, r->vol_norm.p, rnorm_floats(r) * sizeof(float), cudaMemcpyDefault,
                       st));
  if (doift) {
    cufftHandle plan;
    TRY(r->plans.get3d(N, st, &plan, NZ));
    CUFFT(cufftExecC2R(plan, r->vol_data.as<cufftComplex>(), r->vol_data.as<cufftReal>()));
    const size_t nreal = (size_t)N * N * NZ;
    const float scale = 1.0f / (float)nreal;
    if (out) {
      if (is_device_ptr(out)) {
        CU(launch_depad_center(r->vol_data.as<float>(), N, scale, out, st, nz));
      } else {
        TRY(r->s_out.ensure(sizeof(float) * nreal));
        CU(launch_depad_center(r->vol_data.as<float>(), N, scale, r->s_out.as<float>(), st, nz));
        CU(cudaMemcpyAsync(out, r->s_out.p, sizeof(float) * nreal, cudaMemcpyDeviceToHost, st));
      }
    }
  } else if (out) {
    CU(cudaMemcpyAsync(out, r->vol_data.p, rvol_floats(r) * sizeof(float), cudaMemcpyDefault, st));
  }
  TRY(stream_leave(r, st));
  r->state = 2;
  return FR_OK;
}

int fr_finish_corrected(fr_recon *r, float gauss_width, int outx, int outy, int outz, float *out,
                        float *normout) {
  TRY(check_state(r));
  TRY(require_cubic(r, "finish_corrected"));
  if (!out) return fail(FR_ENULL, "null output");
  const int N = r->N;
  if (outx <= 0 || outy <= 0 || outz <= 0 || outx > N || outy > N || outz > N)
    return fail(FR_EINVAL_PARAM, "clip size %d %d %d outside (0, %d]", outx, outy, outz, N);
  std::lock_guard<std::mutex> lk(r->mu);
  TRY(stream_enter(r, r->stream));
  cudaStream_t st = r->stream;
  TRY(check_device_error(r));
  CU(launch_normalize(r->vol_data.as<float>(), r->vol_norm.as<float>(), N, r->p.sqrtnorm, st,
                      r->wfilt));
  if (normout) TRY(from_device(normout, r->vol_norm.p, norm_floats(N) * sizeof(float), st));
  cufftHandle plan;
  TRY(r->plans.get3d(N, st, &plan));
  CUFFT(cufftExecC2R(plan, r->vol_data.as<cufftComplex>(), r->vol_data.as<cufftReal>()));
  const float scale = 1.0f / (float)((size_t)N * N * N);
  const size_t bytes = sizeof(float) * (size_t)outx * outy * outz;
  if (is_device_ptr(out)) {
    CU(launch_finish_out(r->vol_data.as<float>(), N, scale, gauss_width, outx, outy, outz, out, st));
  } else {
    TRY(r->s_out.ensure(bytes));
    CU(launch_finish_out(r->vol_data.as<float>(), N, scale, gauss_width, outx, outy, outz,
                         r->s_out.as<float>(), st));
    TRY(from_device(out, r->s_out.p, bytes, st));
  }
  CU(cudaStreamSynchronize(st));
  r->state = 2;
  return FR_OK;
}

int fr_kernel_fix(float *vol, int nx, int ny, int nz, float gauss_width, void *stream) {
  if (!vol) return fail(FR_ENULL, "null volume");
  if (nx <= 0 || ny <= 0 || nz <= 0) return fail(FR_EDIM, "bad volume size %d %d %d", nx, ny, nz);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = sizeof(float) * (size_t)nx * ny * nz;
  if (is_device_ptr(vol)) {
    CU(launch_kernel_fix(vol, nx, ny, nz, gauss_width, st));
    CU(cudaStreamSynchronize(st));
    return FR_OK;
  }
  DevBuf d;
  TRY(d.ensure(bytes));
  int rc = FR_OK;
  if (cudaMemcpyAsync(d.p, vol, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      launch_kernel_fix(d.as<float>(), nx, ny, nz, gauss_width, st) != cudaSuccess ||
      cudaMemcpyAsync(vol, d.p, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    rc = fail(FR_ECUDA, "kernel fix failed: %s", cudaGetErrorString(cudaGetLastError()));
  d.release();
  return rc;
}

}  // extern "C"
