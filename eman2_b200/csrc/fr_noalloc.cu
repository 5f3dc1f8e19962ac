// fr_noalloc.cu -- insertion that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a process that reserves
// all of its HBM up front for its own pool allocator (a long-running
// reconstruction server, a framework that budgets every byte of the device),
// or code on a latency-critical path where cudaMalloc/cudaFree can stall or
// implicitly synchronise the device.  fr_insert_slices_noalloc serves them:
// the caller owns every input and output buffer, and the little scratch the
// insertion needs (the exp table, the pixel-row and coordinate tables, the
// symmetry operators and the composed per-slice rotations) lives in one
// file-scope __device__ array that is part of the library image.
//
// The array's device address is looked up once per device, with that device
// current, on the first call made on it.  Every call shares the array and
// overwrites the parts it uses, so calls that overlap on the GPU (on
// different streams, or from different host threads) race; serialise them.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fr_handle.h"

namespace fr {
namespace noalloc {

constexpr int kMaxN = 1024;           // largest padded size
constexpr int kMaxOps = 240;          // largest symmetry group (d120)
constexpr int kMaxSlices = 16384;     // particles x symmetry copies per call
constexpr size_t kExpOff = 0;                              // 1000 floats
constexpr size_t kRtabOff = 1024;                          // N+2 floats
constexpr size_t kXmaxOff = kRtabOff + kMaxN + 8;          // N ints
constexpr size_t kSymOff = kXmaxOff + kMaxN;               // nsym*9 floats
constexpr size_t kT3dOff = kSymOff + 9 * kMaxOps;          // slices*9 floats
constexpr size_t kFloats = kT3dOff + 9 * (size_t)kMaxSlices;

// The scratch: 152,696 floats (596 KiB) on every device that loads the
// library, held until exit.
static __device__ __align__(256) float g_scratch[kFloats];

static std::mutex g_mu;
static std::vector<float *> g_ptr;    // device address of g_scratch, per device

// Whether p is device memory of device dev, or managed memory (which every
// device reaches).  The kernels and the scratch are on the current device; a
// buffer of another device would be read and written across devices.
static bool on_device(const void *p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// Set-up once per device (the device is current): the symbol's address and
// the exp table, which never changes.  The upload waits for the stream, so
// this first call on a device must not be captured into a graph: it is
// refused with FR_EINVAL_PARAM on a capturing stream instead of breaking the
// caller's capture.
static int scratch_for_current_device(cudaStream_t st, int dev, float **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_ptr.size() <= dev) g_ptr.resize(dev + 1, nullptr);
  if (!g_ptr[dev]) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CU(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return fail(FR_EINVAL_PARAM, "the first allocation-free call on device %d sets up its "
                  "scratch and cannot be captured; make one call before capturing", dev);
    float *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_scratch);
    if (e != cudaSuccess || !p)
      return fail(FR_ECUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev,
                  cudaGetErrorString(e));
    // Util::fast_exp table (libEM/util.cpp:793)
    float tab[1000];
    for (int i = 0; i < 1000; i++) tab[i] = (float)std::exp(-i / 50.0);
    CU(cudaMemcpyAsync(p + kExpOff, tab, sizeof tab, cudaMemcpyHostToDevice, st));
    CU(cudaStreamSynchronize(st));
    g_ptr[dev] = p;
  }
  *out = g_ptr[dev];
  return FR_OK;
}

}  // namespace noalloc
}  // namespace fr

using namespace fr;

extern "C" int fr_insert_slices_noalloc(const float *d_slices, int n, int N, int mode,
                                        const char *sym, const float *d_rot,
                                        const float *d_weights, float *d_data, float *d_norm,
                                        void *stream) {
  using namespace fr::noalloc;
  if (!d_slices || !d_rot || !d_weights || !d_data || !d_norm || !sym)
    return fail(FR_ENULL, "null argument");
  if (n < 0) return fail(FR_EINVAL_PARAM, "negative slice count");
  if (N < 4 || N % 2 || N > kMaxN)
    return fail(FR_EINVAL_PARAM, "size %d: the allocation-free insertion takes even sizes up to %d",
                N, kMaxN);
  if (mode != FR_MODE_NEAREST && mode != FR_MODE_GAUSS2 && mode != FR_MODE_GAUSS5 &&
      mode != FR_MODE_TRILINEAR)
    return fail(FR_EUNSUPPORTED, "inserter mode %d is not built", mode);
  std::vector<float> ops;
  const int nsym = sym_ops(sym, ops);
  if (nsym < 0) return fail(FR_EUNSUPPORTED, "symmetry '%s' is not supported (c<n>, d<n> up to 1000 operators, tet, oct, icos)", sym);
  if (nsym > kMaxOps)
    return fail(FR_EINVAL_PARAM, "symmetry '%s' has %d operators; the allocation-free insertion "
                "takes at most %d", sym, nsym, kMaxOps);
  if ((long)n * nsym > kMaxSlices)
    return fail(FR_EINVAL_PARAM, "%d slices x %d symmetry copies = %ld exceeds the allocation-free "
                "limit of %d per call; split the batch", n, nsym, (long)n * nsym, kMaxSlices);
  int dev = 0;
  CU(cudaGetDevice(&dev));
  const void *ptrs[] = {d_slices, d_rot, d_weights, d_data, d_norm};
  for (const void *q : ptrs)
    if (!on_device(q, dev))
      return fail(FR_EINVAL_PARAM, "all buffers must be device memory of the current device (%d)",
                  dev);
  cudaStream_t st = (cudaStream_t)stream;
  float *scr = nullptr;
  TRY(scratch_for_current_device(st, dev, &scr));
  if (n == 0) return FR_OK;
  // Per-size tables, formed on the host exactly as get_geom() forms them.
  const int n2 = N / 2;
  std::vector<float> rtab(N + 2);
  for (int i = -n2; i <= n2 + 1; i++) rtab[i + n2] = (float)i / (float)N;
  std::vector<int> xmax(N, -1);
  for (int y = -n2; y < n2; y++) {
    int xm = -1;
    for (int x = 0; x <= n2; x++) {
      const float hyp = (float)std::sqrt((double)x * x + (double)y * y);
      if ((int)(hyp + 0.5f) <= n2) xm = x;
    }
    xmax[y + n2] = xm;
  }
  CU(cudaMemcpyAsync(scr + kRtabOff, rtab.data(), sizeof(float) * rtab.size(),
                     cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(scr + kXmaxOff, xmax.data(), sizeof(int) * xmax.size(),
                     cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(scr + kSymOff, ops.data(), sizeof(float) * ops.size(),
                     cudaMemcpyHostToDevice, st));
  CU(launch_compose(d_rot, scr + kSymOff, n, nsym, scr + kT3dOff, st));
  InsertJob j;
  memset(&j, 0, sizeof j);
  j.data = d_data;
  j.norm = d_norm;
  j.slices = reinterpret_cast<const float2 *>(d_slices);
  j.t3d = scr + kT3dOff;
  j.pw = d_weights;
  j.xmax = reinterpret_cast<const int *>(scr + kXmaxOff);
  j.rtab = scr + kRtabOff;
  j.N = N;
  j.mode = mode;
  j.nsym = nsym;
  j.np = n;
  j.sscale = 1.0f;
  // 1.0f / EMConsts::I2G and 1.0f / EMConsts::I5G (libEM/emobject.cpp:53-56)
  volatile float i2g = (float)(4.0 / (M_PI * M_PI));
  volatile float i5g = (float)(10.4 / (M_PI * M_PI));
  const float h = mode == FR_MODE_GAUSS5 ? 1.0f / i5g : 1.0f / i2g;
  CU(launch_scatter_tables(j, scr + kExpOff, h, st));
  return FR_OK;
}
