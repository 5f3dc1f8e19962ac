// fr_insert.cu -- slice insertion into the (complex, weight) volume.
//
// Reference: FourierReconstructor::do_insert_slice_work
// (libEM/reconstructor.cpp:1122-1210) driving the pixel inserters
// (libEM/reconstructor_tools.cpp:113-189, 315-376) and
// EMData::add_complex_at_fast (libEM/emdata_core.h:368-410).
//
// Three kernels:
//  * k_scatter  -- one thread per (slice, pixel); every tap is added with FP32
//                  atomics exactly as add_complex_at_fast places it.  Used for
//                  single slices and small batches.
//  * k_gather   -- a persistent kernel over voxel tiles.  A tile owns its
//                  cells; for each slice whose plane passes the tile it stages
//                  the slice's pixel patch in shared memory and every voxel
//                  collects the taps that land on it, in registers.  No
//                  atomics; the volume is read and written once per launch.
//                  Covers every cell with |x|,|y|,|z| < N/2.
//  * k_edge     -- the taps on the cube faces (|i|, |j| or |k| = N/2) of rim
//                  pixels, with atomics.  Those taps write only face cells,
//                  which the gather kernel never touches, and vice versa.
#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>

#include "fr_device.cuh"
#include "fr_internal.h"

namespace fr {

const TileShape kTiles[kNumTiles] = {{8, 8, 8}, {16, 8, 8}, {8, 8, 4}, {16, 16, 4}};

// ---------------------------------------------------------------- compose
// t3d[p*nsym+q] = arg[p] * sym[q] (libEM/transform.cpp:1384-1395), float.
__global__ void k_compose(const float *__restrict__ arg, const float *__restrict__ sym, int np,
                          int nsym, float *__restrict__ t3d) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= np * nsym * 9) return;
  const int e = idx % 9, s = idx / 9, p = s / nsym, q = s % nsym;
  const int i = e / 3, j = e % 3;
  const float *a = arg + 9 * p;
  const float *b = sym + 9 * q;
  float v = __fmul_rn(a[3 * i + 0], b[j]);
  v = __fadd_rn(v, __fmul_rn(a[3 * i + 1], b[3 + j]));
  v = __fadd_rn(v, __fmul_rn(a[3 * i + 2], b[6 + j]));
  t3d[idx] = v;
}

cudaError_t launch_compose(const float *d_arg, const float *d_sym, int np, int nsym, float *d_t3d,
                           cudaStream_t st) {
  const int n = np * nsym * 9;
  if (n == 0) return cudaSuccess;
  note_launch();
  k_compose<<<(n + 255) / 256, 256, 0, st>>>(d_arg, d_sym, np, nsym, d_t3d);
  return cudaGetLastError();
}

// ------------------------------------------------------------- scatter path
// One pixel's full insert_pixel with atomics.  Window selection and reject
// rules follow libEM/reconstructor_tools.cpp:113-126 (nearest),
// :128-166 (gauss_2), :191-230 (trilinear), :315-376 (gauss_5).
// face_only: process only taps with a coordinate at +-N/2 (edge kernel).
// NZ: the volume's z size (its window clamps and placement; N when cubic).
template <int MODE>
__device__ __forceinline__ void insert_pixel_atomic(float *__restrict__ data, float *__restrict__ norm,
                                                    int N, int NZ, float xx, float yy, float zz,
                                                    float re, float im, float w, float h,
                                                    const float *__restrict__ table, bool face_only) {
  const int n2 = N >> 1, nz2 = NZ >> 1;
  if (MODE == MODE_NEAREST) {
    const int x0 = (int)floorf(__fadd_rn(xx, 0.5f));
    const int y0 = (int)floorf(__fadd_rn(yy, 0.5f));
    const int z0 = (int)floorf(__fadd_rn(zz, 0.5f));
    if (face_only && abs(x0) != n2 && abs(y0) != n2 && abs(z0) != nz2) return;
    add_tap_atomic(data, norm, N, NZ, x0, y0, z0, __fmul_rn(re, w), __fmul_rn(im, w), w);
  } else if (MODE == MODE_GAUSS2 || MODE == MODE_TRILINEAR) {
    const int x0 = (int)floorf(xx), y0 = (int)floorf(yy), z0 = (int)floorf(zz);
    if (x0 < -n2 - 1 || y0 < -n2 - 1 || z0 < -nz2 - 1 || x0 > n2 || y0 > n2 || z0 > nz2) return;
    for (int k = z0; k <= z0 + 1; k++)
      for (int j = y0; j <= y0 + 1; j++)
        for (int i = x0; i <= x0 + 1; i++) {
          if (face_only && abs(i) != n2 && abs(j) != n2 && abs(k) != nz2) continue;
          float vre, vim, vw;
          tap_value<MODE>(i, j, k, xx, yy, zz, re, im, w, h, table, vre, vim, vw);
          add_tap_atomic(data, norm, N, NZ, i, j, k, vre, vim, vw);
        }
  } else {  // MODE_GAUSS5
    int x0 = floor_minus_2p5(xx), y0 = floor_minus_2p5(yy), z0 = floor_minus_2p5(zz);
    if (x0 < -n2 - 4 || y0 < -n2 - 4 || z0 < -nz2 - 4 || x0 > n2 + 3 || y0 > n2 + 3 ||
        z0 > nz2 + 3)
      return;
    int x1 = x0 + 5, y1 = y0 + 5, z1 = z0 + 5;
    x0 = max(x0, -n2); x1 = min(x1, n2);
    y0 = max(y0, -n2); y1 = min(y1, n2);
    z0 = max(z0, -nz2); z1 = min(z1, nz2);
    for (int k = z0; k <= z1; k++)
      for (int j = y0; j <= y1; j++)
        for (int i = x0; i <= x1; i++) {
          if (face_only && abs(i) != n2 && abs(j) != n2 && abs(k) != nz2) continue;
          float vre, vim, vw;
          tap_value<MODE>(i, j, k, xx, yy, zz, re, im, w, h, table, vre, vim, vw);
          add_tap_atomic(data, norm, N, NZ, i, j, k, vre, vim, vw);
        }
  }
}

// EMData::get_complex_at(x, y, z) of a complex volume [N][N][N+2]
// (libEM/emdata_core.cpp:134-144): 0 outside, the conjugate for x < 0.
__device__ __forceinline__ float2 volume_at(const float *__restrict__ v, int N, int x, int y, int z) {
  if (abs(x) >= (N + 2) / 2 || abs(y) > N / 2 || abs(z) > N / 2) return make_float2(0.f, 0.f);
  const size_t nxf = (size_t)N + 2, nxy = nxf * (size_t)N;
  if (x < 0) {
    const size_t idx = (size_t)(-x * 2) + (size_t)(y <= 0 ? -y : N - y) * nxf +
                       (size_t)(z <= 0 ? -z : N - z) * nxy;
    return make_float2(__ldg(&v[idx]), -__ldg(&v[idx + 1]));
  }
  const size_t idx = (size_t)x * 2 + (size_t)(y < 0 ? N + y : y) * nxf + (size_t)(z < 0 ? N + z : z) * nxy;
  return make_float2(__ldg(&v[idx]), __ldg(&v[idx + 1]));
}

// FourierIterReconstructor::insert_slice's per-pixel insertion
// (libEM/reconstructor.cpp:555-640): the gauss_5 window (floor(xx-2.5), the
// same reject rule) clamped with nx2 = nx/2-2 = N/2-1 along x; without a
// reference volume a Gaussian of width h = 1/(|p|^2/4000 + .15) (at least
// 0.1) and the pixel's value; with one, h = 1/2, cells past radius N/2
// skipped, and the value dt + ref(i,j,k) - ref(p) (ref(p) trilinear).
__device__ __forceinline__ void insert_pixel_iter(const InsertJob &J, float xx, float yy, float zz,
                                                  float re, float im, float w,
                                                  const float *__restrict__ table) {
  const int N = J.N, n2 = N >> 1;
  const int nx2 = n2 - 1, ny2 = n2, nz2 = n2;
  int x0 = floor_minus_2p5(xx), y0 = floor_minus_2p5(yy), z0 = floor_minus_2p5(zz);
  if (x0 < -nx2 - 4 || y0 < -ny2 - 4 || z0 < -nz2 - 4 || x0 > nx2 + 3 || y0 > ny2 + 3 || z0 > nz2 + 3)
    return;
  int x1 = x0 + 5, y1 = y0 + 5, z1 = z0 + 5;
  x0 = max(x0, -nx2); x1 = min(x1, nx2);
  y0 = max(y0, -ny2); y1 = min(y1, ny2);
  z0 = max(z0, -nz2); z1 = min(z1, nz2);
  float h;
  float2 nodt = make_float2(0.f, 0.f);
  if (J.ref) {
    // Util::trilinear_interpolate_complex (libEM/util.h:645-654) of the 8
    // cells around p, in its order of products and sums
    const float fx = floorf(xx), fy = floorf(yy), fz = floorf(zz);
    const float t = __fsub_rn(xx, fx), u = __fsub_rn(yy, fy), v = __fsub_rn(zz, fz);
    const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    const float t1 = __fsub_rn(1.0f, t), u1 = __fsub_rn(1.0f, u), v1 = __fsub_rn(1.0f, v);
    const float c[8] = {__fmul_rn(__fmul_rn(t1, u1), v1), __fmul_rn(__fmul_rn(t, u1), v1),
                        __fmul_rn(__fmul_rn(t1, u), v1),  __fmul_rn(__fmul_rn(t, u), v1),
                        __fmul_rn(__fmul_rn(t1, u1), v),  __fmul_rn(__fmul_rn(t, u1), v),
                        __fmul_rn(__fmul_rn(t1, u), v),   __fmul_rn(__fmul_rn(t, u), v)};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float2 pq = volume_at(J.ref, N, ix + (q & 1), iy + ((q >> 1) & 1), iz + (q >> 2));
      nodt.x = q ? __fadd_rn(nodt.x, __fmul_rn(c[q], pq.x)) : __fmul_rn(c[q], pq.x);
      nodt.y = q ? __fadd_rn(nodt.y, __fmul_rn(c[q], pq.y)) : __fmul_rn(c[q], pq.y);
    }
    h = 0.5f;
  } else {
    const float hs = __fadd_rn(__fadd_rn(__fmul_rn(xx, xx), __fmul_rn(yy, yy)), __fmul_rn(zz, zz));
    float hf = (float)(1.0 / ((double)__fdiv_rn(hs, 4000.0f) + 0.15));
    if ((double)hf < 0.1) hf = (float)0.1;
    h = hf;
  }
  const int ny2sq = N * N / 4;
  for (int k = z0; k <= z1; k++)
    for (int j = y0; j <= y1; j++)
      for (int i = x0; i <= x1; i++) {
        if (J.ref && i * i + j * j + k * k > ny2sq) continue;
        const float r = dist2(i, j, k, xx, yy, zz);
        const float gg = fast_exp(__fmul_rn(-r, h), table);
        float vre, vim;
        if (J.ref) {
          const float2 nt = volume_at(J.ref, N, i, j, k);
          const float ure = __fsub_rn(__fadd_rn(re, nt.x), nodt.x);
          const float uim = __fsub_rn(__fadd_rn(im, nt.y), nodt.y);
          vre = __fmul_rn(__fmul_rn(ure, gg), w);
          vim = __fmul_rn(__fmul_rn(uim, gg), w);
        } else {
          vre = __fmul_rn(__fmul_rn(re, gg), w);
          vim = __fmul_rn(__fmul_rn(im, gg), w);
        }
        add_tap_atomic(J.data, J.norm, N, N, i, j, k, vre, vim, __fmul_rn(gg, w));
      }
}

// Per-pixel weight: the particle weight, or with usessnr the slice's
// class_ssnr table at the pixel radius, max(0, ssnr[int(r*sscale)])
// (libEM/reconstructor.cpp:1170-1184).
// WienerFourierReconstructor::do_insert_slice_work (libEM/reconstructor.cpp:1679-1731):
// the weight at the pixel's radius, rn = |(x,y)|/N scaled by 2*len, linearly
// interpolated in the slice's ctf_snr_total (or its last entry, times the
// sign of the insert weight, past the end); the value is scaled by
// (weight+1)/weight when the slice was Wiener filtered.  Returns
// weight*sign, the weight insert_pixel gets.
__device__ __forceinline__ float wiener_weight(const InsertJob &J, int p, int x, int y, float w,
                                               float &vscale) {
  const float sub = w < 0.0f ? -1.0f : 1.0f;
  const float rx = __fdiv_rn((float)x, (float)J.N);
  const float ry = __fdiv_rn((float)y, (float)J.N);
  float rn = (float)hypot((double)rx, (double)ry);
  rn = __fmul_rn(rn, __fmul_rn((float)J.nwsnr, 2.0f));
  const int rni = (int)floorf(rn);
  const float *snr = J.wsnr + (size_t)p * J.nwsnr;
  float weight;
  if ((unsigned)rni >= (unsigned)(J.nwsnr - 1)) {
    weight = __fmul_rn(snr[J.nwsnr - 1], sub);
  } else {
    const float t = __fsub_rn(rn, (float)rni);   // Util::linear_interpolate (libEM/util.h:518-521)
    weight = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, t), snr[rni]), __fmul_rn(t, snr[rni + 1]));
  }
  vscale = (J.wundo && J.wundo[p]) ? __fdiv_rn(__fadd_rn(weight, 1.0f), weight) : 1.0f;
  return __fmul_rn(weight, sub);
}

__device__ __forceinline__ float pixel_weight(const InsertJob &J, int p, int x, int y, float w) {
  if (!J.ssnr) return w;
  const int r = (int)__fadd_rn((float)sqrt((double)(x * x + y * y)), 0.5f);
  const int k = min((int)__fmul_rn((float)r, J.sscale), J.nssnr - 1);
  const float sv = J.ssnr[(size_t)p * J.nssnr + k];
  return sv > 0.0f ? sv : 0.0f;
}

// Resets a persistent launch's work counter.  A kernel rather than a memset:
// on the copy engine a memset would queue behind uploads of other streams.
__global__ void k_zero_int(int *p) { *p = 0; }

cudaError_t set_max_smem(const void *func, size_t smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  std::lock_guard<std::mutex> lk(mu);
  size_t &have = done[std::make_pair(func, dev)];
  if (have >= smem) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) have = smem;
  return e;
}

cudaError_t zero_counter(int *d_counter, cudaStream_t st) {
  note_launch();
  k_zero_int<<<1, 1, 0, st>>>(d_counter);
  return cudaGetLastError();
}

// One pixel of slice s (particle*nsym+sym) of job J, scattered with atomics.
// pix indexes the N*(N/2+1) pixel grid.
template <int MODE>
__device__ __forceinline__ void scatter_pixel(const InsertJob &J, int s, int pix,
                                              const float *__restrict__ table, float h) {
  const int N = J.N, n2 = N >> 1, w2 = n2 + 1;
  const int p = s / J.nsym;
  const float w = J.pw[p];
  if (w == 0.0f) return;
  if (pix >= N * w2) return;
  const int x = pix % w2, y = pix / w2 - n2;
  if (x > __ldg(&J.xmax[y + n2])) return;
  float M[6];
#pragma unroll
  for (int i = 0; i < 6; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
  const int NZ = J.nz ? J.nz : N;
  float xx, yy, zz;
  pixel_coords_z(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, (float)N, (float)NZ, xx, yy,
                 zz);
  float2 v = slice_value(J.slices + (size_t)p * N * w2, N, x, y);
  float pw;
  if (J.wsnr) {
    float vs;
    pw = wiener_weight(J, p, x, y, w, vs);
    if (vs != 1.0f) { v.x = __fmul_rn(v.x, vs); v.y = __fmul_rn(v.y, vs); }
  } else {
    pw = pixel_weight(J, p, x, y, w);
  }
  insert_pixel_atomic<MODE>(J.data, J.norm, N, NZ, xx, yy, zz, v.x, v.y, pw, h, table, false);
}

// The iterative reconstructor's insertion of one pixel of its disk.
__device__ __forceinline__ void scatter_pixel_iter(const InsertJob &J, int s, int pix,
                                                   const float *__restrict__ table) {
  const int N = J.N, n2 = N >> 1, w2 = n2 + 1;
  const int p = s / J.nsym;
  const float w = J.pw[p];
  if (w == 0.0f) return;
  if (pix >= N * w2) return;
  const int x = pix % w2, y = pix / w2 - n2;
  if (x > __ldg(&J.xmax[y + n2])) return;
  float M[6];
#pragma unroll
  for (int i = 0; i < 6; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
  float xx, yy, zz;
  pixel_coords(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, (float)N, xx, yy, zz);
  const float2 v = slice_value(J.slices + (size_t)p * N * w2, N, x, y);
  insert_pixel_iter(J, xx, yy, zz, v.x, v.y, w, table);
}

// Face taps of rim pixel r (index into J.rim) of slice s.
template <int MODE>
__device__ __forceinline__ void edge_pixel(const InsertJob &J, int s, int r,
                                           const float *__restrict__ table, float h) {
  const int N = J.N, n2 = N >> 1, w2 = n2 + 1;
  const int p = s / J.nsym;
  const float w = J.pw[p];
  if (w == 0.0f) return;
  if (r >= J.nrim) return;
  const int code = __ldg(&J.rim[r]);
  const int x = code & 0xFFFF, y = (code >> 16) - n2;
  float M[6];
#pragma unroll
  for (int i = 0; i < 6; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
  float xx, yy, zz;
  pixel_coords(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, (float)N, xx, yy, zz);
  const float2 v = slice_value(J.slices + (size_t)p * N * w2, N, x, y);
  insert_pixel_atomic<MODE>(J.data, J.norm, N, N, xx, yy, zz, v.x, v.y, pixel_weight(J, p, x, y, w),
                            h, table, true);
}

// grid.x covers the N*(N/2+1) pixel grid, grid.y = slice (particle*nsym+sym).
template <int MODE>
__global__ void __launch_bounds__(256) k_scatter(InsertJob J, const float *__restrict__ table,
                                                 float h) {
  scatter_pixel<MODE>(J, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x, table, h);
}

__global__ void __launch_bounds__(256) k_scatter_iter(InsertJob J, const float *__restrict__ table) {
  scatter_pixel_iter(J, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x, table);
}

// Face taps of rim pixels: grid.x covers the rim list, grid.y = slice.
template <int MODE>
__global__ void __launch_bounds__(128) k_edge(InsertJob J, const float *__restrict__ table,
                                              float h) {
  edge_pixel<MODE>(J, blockIdx.y, blockIdx.x * blockDim.x + threadIdx.x, table, h);
}

// Several jobs' scatter (or face taps) in one launch: grid.x = unit
// (job, slice); the grid.y blocks of a unit stride over its job's pixel grid
// (or rim list).  A slice of weight 0 costs one check per block.
__global__ void __launch_bounds__(256) k_scatter_multi(const InsertJob *__restrict__ jobs,
                                                       const int2 *__restrict__ units,
                                                       const float *__restrict__ table, float h2,
                                                       float h5, int edge) {
  const int2 u = units[blockIdx.x];
  const InsertJob &J = jobs[u.x];
  if (J.pw[u.y / J.nsym] == 0.0f) return;
  const int mode = J.mode;
  const int npx = edge ? J.nrim : J.N * (J.N / 2 + 1);
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < npx; i += gridDim.y * blockDim.x) {
    if (edge) {
      switch (mode) {
        case MODE_NEAREST: edge_pixel<MODE_NEAREST>(J, u.y, i, table, h2); break;
        case MODE_GAUSS2: edge_pixel<MODE_GAUSS2>(J, u.y, i, table, h2); break;
        case MODE_GAUSS5: edge_pixel<MODE_GAUSS5>(J, u.y, i, table, h5); break;
        case MODE_TRILINEAR: edge_pixel<MODE_TRILINEAR>(J, u.y, i, table, h2); break;
        default: break;
      }
      continue;
    }
    switch (mode) {
      case MODE_NEAREST: scatter_pixel<MODE_NEAREST>(J, u.y, i, table, h2); break;
      case MODE_GAUSS2: scatter_pixel<MODE_GAUSS2>(J, u.y, i, table, h2); break;
      case MODE_GAUSS5: scatter_pixel<MODE_GAUSS5>(J, u.y, i, table, h5); break;
      case MODE_TRILINEAR: scatter_pixel<MODE_TRILINEAR>(J, u.y, i, table, h2); break;
      case MODE_ITER: scatter_pixel_iter(J, u.y, i, table); break;
      default: break;
    }
  }
}

static float mode_h(int mode) {
  const Consts &c = consts();
  return mode == MODE_GAUSS5 ? c.h5 : c.h2;
}

cudaError_t launch_scatter(const InsertJob &j, cudaStream_t st) {
  const int nsl = j.np * j.nsym;
  if (nsl == 0) return cudaSuccess;
  const int npx = j.N * (j.N / 2 + 1);
  dim3 grid((npx + 255) / 256, nsl);
  const float *tab = consts().d_exp;
  const float h = mode_h(j.mode);
  note_launch();
  if (j.mode == MODE_ITER) {
    k_scatter_iter<<<grid, 256, 0, st>>>(j, tab);
    return cudaGetLastError();
  }
  switch (j.mode) {
    case MODE_NEAREST: k_scatter<MODE_NEAREST><<<grid, 256, 0, st>>>(j, tab, h); break;
    case MODE_GAUSS2: k_scatter<MODE_GAUSS2><<<grid, 256, 0, st>>>(j, tab, h); break;
    case MODE_GAUSS5: k_scatter<MODE_GAUSS5><<<grid, 256, 0, st>>>(j, tab, h); break;
    case MODE_TRILINEAR: k_scatter<MODE_TRILINEAR><<<grid, 256, 0, st>>>(j, tab, h); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// The scatter launch with caller-supplied exp table and Gaussian factor
// (no use of the lazily allocated per-device constants).
cudaError_t launch_scatter_tables(const InsertJob &j, const float *table, float h,
                                  cudaStream_t st) {
  const int nsl = j.np * j.nsym;
  if (nsl == 0) return cudaSuccess;
  const int npx = j.N * (j.N / 2 + 1);
  dim3 grid((npx + 255) / 256, nsl);
  note_launch();
  switch (j.mode) {
    case MODE_NEAREST: k_scatter<MODE_NEAREST><<<grid, 256, 0, st>>>(j, table, h); break;
    case MODE_GAUSS2: k_scatter<MODE_GAUSS2><<<grid, 256, 0, st>>>(j, table, h); break;
    case MODE_GAUSS5: k_scatter<MODE_GAUSS5><<<grid, 256, 0, st>>>(j, table, h); break;
    case MODE_TRILINEAR: k_scatter<MODE_TRILINEAR><<<grid, 256, 0, st>>>(j, table, h); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_edge(const InsertJob &j, cudaStream_t st) {
  const int nsl = j.np * j.nsym;
  if (nsl == 0 || j.nrim == 0) return cudaSuccess;
  dim3 grid((j.nrim + 127) / 128, nsl);
  const float *tab = consts().d_exp;
  const float h = mode_h(j.mode);
  note_launch();
  switch (j.mode) {
    case MODE_NEAREST: k_edge<MODE_NEAREST><<<grid, 128, 0, st>>>(j, tab, h); break;
    case MODE_GAUSS2: k_edge<MODE_GAUSS2><<<grid, 128, 0, st>>>(j, tab, h); break;
    case MODE_GAUSS5: k_edge<MODE_GAUSS5><<<grid, 128, 0, st>>>(j, tab, h); break;
    case MODE_TRILINEAR: k_edge<MODE_TRILINEAR><<<grid, 128, 0, st>>>(j, tab, h); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_scatter_multi(const InsertJob *d_jobs, const int2 *d_units, int nunits,
                                 int max_px, bool edge_only, cudaStream_t st) {
  if (nunits == 0 || max_px == 0) return cudaSuccess;
  const Consts &c = consts();
  // blocks per unit: enough for ~4 waves of resident blocks in all, each
  // striding over its job's pixels (one pixel per thread at most)
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long want = (4L * sms * 8 + nunits - 1) / nunits;
  const int per = (int)std::max(1L, std::min<long>(want, (max_px + 255) / 256));
  dim3 grid(nunits, per);
  note_launch();
  k_scatter_multi<<<grid, 256, 0, st>>>(d_jobs, d_units, c.d_exp, c.h2, c.h5, edge_only ? 1 : 0);
  return cudaGetLastError();
}

// -------------------------------------------------------------- gather path

// Extent of the pixel-point box around a target tap t: a pixel at p reaches
// t iff t - lo <= p < t + hi per axis (window rules of each inserter).
template <int MODE> struct Reach;
template <> struct Reach<MODE_GAUSS5> { static constexpr float lo = 2.5f, hi = 3.5f; };
template <> struct Reach<MODE_GAUSS2> { static constexpr float lo = 1.0f, hi = 1.0f; };
template <> struct Reach<MODE_TRILINEAR> { static constexpr float lo = 1.0f, hi = 1.0f; };
template <> struct Reach<MODE_NEAREST> { static constexpr float lo = 0.5f, hi = 0.5f; };

// Exact window membership of tap coordinate t for a pixel coordinate p.
template <int MODE> __device__ __forceinline__ bool in_window(int t, float p) {
  const float tf = (float)t;
  if (MODE == MODE_GAUSS5) return __fadd_rn(tf, -2.5f) <= p && p < __fadd_rn(tf, 3.5f);
  if (MODE == MODE_NEAREST) {
    const float s = __fadd_rn(p, 0.5f);
    return tf <= s && s < __fadd_rn(tf, 1.0f);
  }
  return __fadd_rn(tf, -1.0f) <= p && p < __fadd_rn(tf, 1.0f);
}

constexpr float kDel = 0.02f;     // slack on the approximate plane geometry
constexpr float kPlaneTol = 0.05f;

// Range of dot(m, q) over the box q in [lo, hi] (per axis).
__device__ __forceinline__ void box_dot(const float *m, const float *lo, const float *hi, float &mn,
                                        float &mx) {
  mn = 0.f; mx = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float u = m[a] * lo[a], v = m[a] * hi[a];
    mn += fminf(u, v);
    mx += fmaxf(u, v);
  }
}

template <int MODE, int TX, int TY, int TZ>
__device__ __forceinline__ void gather_tile(const InsertJob &J, int bx, int by, int bz,
                                            const float *s_exp, float h, int *s_hits,
                                            int *s_wcount, float4 *s_pt, float2 *s_pv, int side,
                                            int *err) {
  constexpr int NV = TX * TY * TZ;
  constexpr int VPT = (NV + 255) / 256;
  const float RLO = Reach<MODE>::lo, RHI = Reach<MODE>::hi;
  const int N = J.N, n2 = N >> 1, w2 = n2 + 1;
  const float Nf = (float)N;
  const int ex = min(bx + TX - 1, n2 - 1), ey = min(by + TY - 1, n2 - 1), ez = min(bz + TZ - 1, n2 - 1);

  int vx[VPT], vy[VPT], vz[VPT];
  bool valid[VPT];
  double ar[VPT], ai[VPT], aw[VPT];
  int touch = 0;
#pragma unroll
  for (int v = 0; v < VPT; v++) {
    const int lin = threadIdx.x + v * 256;
    vx[v] = bx + lin % TX;
    vy[v] = by + (lin / TX) % TY;
    vz[v] = bz + lin / (TX * TY);
    valid[v] = lin < NV && vx[v] <= ex && vy[v] <= ey && vz[v] <= ez;
    ar[v] = ai[v] = aw[v] = 0.0;
  }

  const int total = J.np * J.nsym;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < total; base += 256) {
    // ---- cull: does slice s's plane pass within reach of this tile?
    const int s = base + threadIdx.x;
    bool hit = false;
    if (s < total && __ldg(&J.pw[s / J.nsym]) != 0.0f) {
      const float n[3] = {__ldg(&J.t3d[9 * s + 6]), __ldg(&J.t3d[9 * s + 7]),
                          __ldg(&J.t3d[9 * s + 8])};
      // Direct taps reach the tile from [b - RLO, e + RHI], conjugate taps
      // (mirrored) from [b - RHI, e + RLO]; the plane passes through the
      // origin, so one test against the union box covers both passes.
      const float RC = fmaxf(RLO, RHI) + kDel;
      const float lo[3] = {bx - RC, by - RC, bz - RC};
      const float hi[3] = {ex + RC, ey + RC, ez + RC};
      float mn, mx;
      box_dot(n, lo, hi, mn, mx);
      hit = mn <= kPlaneTol && mx >= -kPlaneTol;
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_wcount[warp] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int c = s_wcount[i];
      off += (i < warp) ? c : 0;
      tot += c;
    }
    if (hit) s_hits[off + __popc(b & ((1u << lane) - 1u))] = s;
    __syncthreads();

    for (int hI = 0; hI < tot; hI++) {
      const int s2 = s_hits[hI];
      const int p = s2 / J.nsym;
      float M[9];
#pragma unroll
      for (int i = 0; i < 9; i++) M[i] = __ldg(&J.t3d[9 * s2 + i]);
      const float *m0 = M, *m1 = M + 3, *nrm = M + 6;
      const float w = __ldg(&J.pw[p]);
      const float2 *sl = J.slices + (size_t)p * N * w2;
      float inv0[3];
#pragma unroll
      for (int a = 0; a < 3; a++) inv0[a] = fabsf(m0[a]) > 1e-4f ? 1.0f / m0[a] : 0.0f;

#pragma unroll 1
      for (int pass = 0; pass < 2; pass++) {
        const int sg = pass ? -1 : 1;
        float lo[3], hi[3];
        if (!pass) {
          lo[0] = bx; lo[1] = by; lo[2] = bz; hi[0] = ex; hi[1] = ey; hi[2] = ez;
        } else {
          lo[0] = -ex; lo[1] = -ey; lo[2] = -ez; hi[0] = -bx; hi[1] = -by; hi[2] = -bz;
        }
#pragma unroll
        for (int a = 0; a < 3; a++) { lo[a] -= RLO + kDel; hi[a] += RHI + kDel; }
        float xl, xh, yl, yh;
        box_dot(m0, lo, hi, xl, xh);
        box_dot(m1, lo, hi, yl, yh);
        const int px0 = max(0, (int)floorf(xl) - 1), px1 = min(n2, (int)ceilf(xh) + 1);
        const int py0 = max(-n2, (int)floorf(yl) - 1), py1 = min(n2 - 1, (int)ceilf(yh) + 1);
        if (px0 > px1 || py0 > py1) continue;
        int PW = px1 - px0 + 1, PH = py1 - py0 + 1;
        if (PW > side || PH > side) {
          // Cannot happen for an orthonormal block; record and stay in bounds.
          if (threadIdx.x == 0) atomicOr(err, 2);
          PW = min(PW, side);
          PH = min(PH, side);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < PW * PH; i += 256) {
          const int x = px0 + i % PW, y = py0 + i / PW;
          float4 pt;
          float2 pv;
          if (x > __ldg(&J.xmax[y + n2])) {
            pt = make_float4(1e30f, 1e30f, 1e30f, 0.f);
            pv = make_float2(0.f, 0.f);
          } else {
            pixel_coords(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, Nf, pt.x, pt.y, pt.z);
            pt.w = w;
            pv = slice_value(sl, N, x, y);
          }
          s_pt[i] = pt;
          s_pv[i] = pv;
        }
        __syncthreads();

#pragma unroll
        for (int v = 0; v < VPT; v++) {
          if (!valid[v]) continue;
          const bool origin = vx[v] == 0 && vy[v] == 0 && vz[v] == 0;
          if (pass && origin) continue;  // the origin tap adds no conjugate
          const int t[3] = {sg * vx[v], sg * vy[v], sg * vz[v]};
          const float tlo[3] = {t[0] - RLO - kDel, t[1] - RLO - kDel, t[2] - RLO - kDel};
          const float thi[3] = {t[0] + RHI + kDel, t[1] + RHI + kDel, t[2] + RHI + kDel};
          float dmn, dmx;
          box_dot(nrm, tlo, thi, dmn, dmx);
          if (dmn > kPlaneTol || dmx < -kPlaneTol) continue;
          float ryl, ryh;
          box_dot(m1, tlo, thi, ryl, ryh);
          const int r0 = max(py0, (int)ceilf(ryl)), r1 = min(py0 + PH - 1, (int)floorf(ryh));
          float pre = 0.f, pim = 0.f, pwt = 0.f;
          int cnt = 0;
          for (int y = r0; y <= r1; y++) {
            float xlo = (float)px0, xhi = (float)(px0 + PW - 1);
#pragma unroll
            for (int a = 0; a < 3; a++) {
              const float c = m1[a] * (float)y;
              const float L = tlo[a] - c, U = thi[a] - c;
              if (inv0[a] > 0.f) { xlo = fmaxf(xlo, L * inv0[a]); xhi = fminf(xhi, U * inv0[a]); }
              else if (inv0[a] < 0.f) { xlo = fmaxf(xlo, U * inv0[a]); xhi = fminf(xhi, L * inv0[a]); }
              else {
                const float slack = 1e-4f * (float)(n2 + 1);
                if (L > slack || U < -slack) xhi = -1.f;
              }
            }
            const int c0 = max(px0, (int)ceilf(xlo));
            const int c1 = min(px0 + PW - 1, (int)floorf(xhi));
            const int rowoff = (y - py0) * PW - px0;
            for (int x = c0; x <= c1; x++) {
              const float4 pt = s_pt[rowoff + x];
              if (!(in_window<MODE>(t[0], pt.x) && in_window<MODE>(t[1], pt.y) &&
                    in_window<MODE>(t[2], pt.z)))
                continue;
              const float2 pv = s_pv[rowoff + x];
              float vre, vim, vw;
              tap_value<MODE>(t[0], t[1], t[2], pt.x, pt.y, pt.z, pv.x, pv.y, pt.w, h, s_exp, vre,
                              vim, vw);
              pre += vre;
              pim += vim;
              pwt += vw;
              cnt++;
            }
          }
          if (!cnt) continue;
          if (origin) {
            ar[v] += pre;          // real part only; the imaginary part is set to 0
            aw[v] += pwt;
            touch = 1;
          } else if (pass) {
            ar[v] += pre;          // conjugate add (re, -im)
            ai[v] -= pim;
            if (vx[v] != 0) aw[v] += pwt;   // x=0 conjugates carry no weight
          } else {
            ar[v] += pre;
            ai[v] += pim;
            aw[v] += pwt;
          }
        }
      }
    }
    __syncthreads();
  }

  // ---- write back: the tile owns these cells for the whole launch.
  const size_t nxf = (size_t)N + 2;
#pragma unroll
  for (int v = 0; v < VPT; v++) {
    if (!valid[v]) continue;
    if (ar[v] == 0.0 && ai[v] == 0.0 && aw[v] == 0.0 && !(touch && vx[v] == 0 && vy[v] == 0 && vz[v] == 0))
      continue;
    const size_t row = (size_t)(vy[v] < 0 ? N + vy[v] : vy[v]);
    const size_t slab = (size_t)(vz[v] < 0 ? N + vz[v] : vz[v]);
    const size_t di = (size_t)vx[v] * 2 + row * nxf + slab * nxf * (size_t)N;
    const size_t ni = (size_t)vx[v] + row * (size_t)w2 + slab * (size_t)w2 * (size_t)N;
    float2 d = *reinterpret_cast<float2 *>(&J.data[di]);
    d.x = __fadd_rn(d.x, (float)ar[v]);
    if (touch && vx[v] == 0 && vy[v] == 0 && vz[v] == 0) d.y = 0.0f;
    else d.y = __fadd_rn(d.y, (float)ai[v]);
    *reinterpret_cast<float2 *>(&J.data[di]) = d;
    J.norm[ni] = __fadd_rn(J.norm[ni], (float)aw[v]);
  }
}

template <int TX, int TY, int TZ>
__global__ void __launch_bounds__(256) k_gather(const InsertJob *__restrict__ jobs,
                                                const int2 *__restrict__ work, int nwork,
                                                int *counter, const float *__restrict__ exp_g,
                                                float h2, float h5, int side, int max_mode,
                                                int *err) {
  __shared__ float s_exp[1000];
  __shared__ int s_hits[256];
  __shared__ int s_wcount[8];
  __shared__ int s_work;
  extern __shared__ float4 s_dyn[];
  float4 *s_pt = s_dyn;
  float2 *s_pv = reinterpret_cast<float2 *>(s_dyn + side * side);
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) s_exp[i] = exp_g[i];
  (void)max_mode;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_work = atomicAdd(counter, 1);
    __syncthreads();
    const int wi = s_work;
    if (wi >= nwork) break;
    const int2 wk = work[wi];
    const InsertJob J = jobs[wk.x];
    const int n2 = J.N >> 1;
    const int tix = wk.y % J.tiles_x, tiy = (wk.y / J.tiles_x) % J.tiles_y,
              tiz = wk.y / (J.tiles_x * J.tiles_y);
    const int bx = tix * TX, by = -n2 + 1 + tiy * TY, bz = -n2 + 1 + tiz * TZ;
    switch (J.mode) {
      case MODE_GAUSS2:
        gather_tile<MODE_GAUSS2, TX, TY, TZ>(J, bx, by, bz, s_exp, h2, s_hits, s_wcount, s_pt, s_pv, side, err);
        break;
      case MODE_GAUSS5:
        gather_tile<MODE_GAUSS5, TX, TY, TZ>(J, bx, by, bz, s_exp, h5, s_hits, s_wcount, s_pt, s_pv, side, err);
        break;
      case MODE_NEAREST:
        gather_tile<MODE_NEAREST, TX, TY, TZ>(J, bx, by, bz, s_exp, h2, s_hits, s_wcount, s_pt, s_pv, side, err);
        break;
      case MODE_TRILINEAR:
        gather_tile<MODE_TRILINEAR, TX, TY, TZ>(J, bx, by, bz, s_exp, h2, s_hits, s_wcount, s_pt, s_pv, side, err);
        break;
      default:
        if (threadIdx.x == 0) atomicOr(err, 4);
    }
  }
}

static float reach_sum(int mode) {
  switch (mode) {
    case MODE_GAUSS5: return 6.0f;
    case MODE_NEAREST: return 1.0f;
    default: return 2.0f;
  }
}

// Patch side bound: the pixel-space extent of the tile box grown by the
// window reach, projected on a unit in-plane axis, plus rounding margins.
static int patch_side(int tile, int max_mode) {
  const TileShape &t = kTiles[tile];
  const float r = reach_sum(max_mode) + 2 * kDel;
  const float ex = t.tx - 1 + r, ey = t.ty - 1 + r, ez = t.tz - 1 + r;
  return (int)std::ceil(std::sqrt(ex * ex + ey * ey + ez * ez)) + 5;
}

void gather_tiles(int N, int mode, int tile, int corners, std::vector<int> &out, int &tx, int &ty,
                  int &tz) {
  const TileShape &T = kTiles[tile];
  const int n2 = N / 2;
  tx = (n2 + T.tx - 1) / T.tx;
  ty = (N - 1 + T.ty - 1) / T.ty;
  tz = (N - 1 + T.tz - 1) / T.tz;
  // Kept pixels satisfy round(hypot(x,y)) <= N/2, so their points lie within
  // N/2 + 0.5 of the origin (to float rounding); corners mode keeps the whole
  // square (radius N/2 * sqrt 2).  A tile farther than that plus the window
  // reach (per axis, hence x sqrt 3) receives nothing.
  const double reach = reach_sum(mode) * 0.5 + 0.5;
  const double rpix = corners ? n2 * 1.41422 + 1.0 : n2 + 0.5 + 0.01;
  const double rmax = rpix + reach * 1.7321 + 0.1;
  std::vector<std::pair<double, int>> order;
  for (int iz = 0; iz < tz; iz++)
    for (int iy = 0; iy < ty; iy++)
      for (int ix = 0; ix < tx; ix++) {
        const int bx = ix * T.tx, by = -n2 + 1 + iy * T.ty, bz = -n2 + 1 + iz * T.tz;
        const int ex = std::min(bx + T.tx - 1, n2 - 1), ey = std::min(by + T.ty - 1, n2 - 1),
                  ez = std::min(bz + T.tz - 1, n2 - 1);
        auto dmin = [](int a, int b) {
          return (a <= 0 && b >= 0) ? 0.0 : (double)std::min(std::abs(a), std::abs(b));
        };
        const double dx = dmin(bx, ex), dy = dmin(by, ey), dz = dmin(bz, ez);
        const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (d <= rmax) order.push_back({d, ix + tx * (iy + ty * iz)});
      }
  // Nearest tiles first: they meet the most slices, so they start first.
  std::stable_sort(order.begin(), order.end());
  out.clear();
  for (auto &o : order) out.push_back(o.second);
}

template <int TX, int TY, int TZ>
static cudaError_t launch_gather_t(const InsertJob *d_jobs, int nwork, const int2 *d_work,
                                   int *d_counter, int side, int max_mode, cudaStream_t st) {
  const Consts &c = consts();
  const size_t smem = (size_t)side * side * (sizeof(float4) + sizeof(float2));
  cudaError_t ea = set_max_smem((const void *)k_gather<TX, TY, TZ>, smem);
  if (ea != cudaSuccess) return ea;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather<TX, TY, TZ>, 256, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(nwork, sms * per_sm));
  note_launch();
  k_gather<TX, TY, TZ><<<grid, 256, smem, st>>>(d_jobs, d_work, nwork, d_counter, c.d_exp, c.h2,
                                                c.h5, side, max_mode, c.d_err);
  return cudaGetLastError();
}

cudaError_t launch_gather(const InsertJob *d_jobs, const InsertJob *h_jobs, int njobs,
                          const int2 *d_work, int nwork, int tile, int *d_counter, int max_mode,
                          cudaStream_t st) {
  (void)h_jobs; (void)njobs;
  if (nwork == 0) return cudaSuccess;
  cudaError_t e = zero_counter(d_counter, st);
  if (e != cudaSuccess) return e;
  const int side = patch_side(tile, max_mode);
  switch (tile) {
    case 0: return launch_gather_t<8, 8, 8>(d_jobs, nwork, d_work, d_counter, side, max_mode, st);
    case 1: return launch_gather_t<16, 8, 8>(d_jobs, nwork, d_work, d_counter, side, max_mode, st);
    case 2: return launch_gather_t<8, 8, 4>(d_jobs, nwork, d_work, d_counter, side, max_mode, st);
    case 3: return launch_gather_t<16, 16, 4>(d_jobs, nwork, d_work, d_counter, side, max_mode, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace fr
