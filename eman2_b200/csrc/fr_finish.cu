// fr_finish.cu -- normalisation, finish(), seeding, slice agreement and
// projection kernels.
#include <cmath>

#include "fr_device.cuh"
#include "fr_internal.h"

namespace fr {

// ------------------------------------------------------------ normalize_threed
// ReconstructorVolumeData::normalize_threed (libEM/reconstructor.cpp:315-390),
// full-volume case.  Stage 1: weights of conjugate pairs in the x=0 and
// x=N/2 planes are summed into both cells; five special cells are doubled.
// The pairs are disjoint from one another and from the special cells, so one
// thread per (z, y) pair does them all.
// NZ: the volume's z size (N when cubic).
__global__ void k_norm_pairs(float *__restrict__ norm, int N, int NZ) {
  const long nnx = N / 2 + 1, nnxy = (long)N * nnx;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ny2 = N / 2 + 1;
  if (i < NZ * ny2) {
    const int z = i / ny2 - NZ / 2, y = i % ny2;
    if (z <= 0 && (y == 0 || y == N / 2)) return;
    long idx1 = (long)(y == 0 ? 0 : N - y) * nnx + (long)(z <= 0 ? -z : NZ - z) * nnxy;
    long idx2 = (long)y * nnx + (long)(z < 0 ? NZ + z : z) * nnxy;
    if (idx1 == idx2) return;
    float s = __fadd_rn(norm[idx1], norm[idx2]);
    norm[idx1] = s;
    norm[idx2] = s;
    idx1 += nnx - 1;
    idx2 += nnx - 1;
    s = __fadd_rn(norm[idx1], norm[idx2]);
    norm[idx1] = s;
    norm[idx2] = s;
  } else if (i < NZ * ny2 + 5) {
    const int c = i - NZ * ny2;
    const long h = N / 2, hz = NZ / 2;
    long idx;
    switch (c) {
      case 0: idx = 0 + 0 * nnx + hz * nnxy; break;
      case 1: idx = 0 + h * nnx + 0 * nnxy; break;
      case 2: idx = 0 + h * nnx + hz * nnxy; break;
      case 3: idx = (nnx - 1) + 0 * nnx + hz * nnxy; break;
      default: idx = (nnx - 1) + h * nnx + 0 * nnxy; break;
    }
    norm[idx] = __fmul_rn(norm[idx], 2.0f);
  }
}

// Stage 2: data /= norm (or sqrt(norm)); zero where the weight is 0.
// wfilt: 1 for the Wiener reconstructor (normalize_threed(sqrtnorm, true),
// libEM/reconstructor.cpp:376-390): data / (d + 1), still 0 where d == 0.
__global__ void k_divide(float2 *__restrict__ data, const float *__restrict__ norm, long n,
                         int sqrtnorm, float wfilt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float d = norm[i];
  if (sqrtnorm) d = __fsqrt_rn(d);
  float2 v = data[i];
  if (d == 0.0f) { v.x = 0.f; v.y = 0.f; }
  else {
    const float dd = __fadd_rn(d, wfilt);
    v.x = __fdiv_rn(v.x, dd);
    v.y = __fdiv_rn(v.y, dd);
  }
  data[i] = v;
}

cudaError_t launch_normalize(float *d_data, float *d_norm, int N, int sqrtnorm, cudaStream_t st,
                             float wfilt, int nz) {
  const int NZ = nz ? nz : N;
  const int np = NZ * (N / 2 + 1) + 5;
  note_launch();
  k_norm_pairs<<<(np + 255) / 256, 256, 0, st>>>(d_norm, N, NZ);
  const long n = (long)NZ * N * (N / 2 + 1);
  note_launch();
  k_divide<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(reinterpret_cast<float2 *>(d_data), d_norm,
                                                         n, sqrtnorm, wfilt);
  return cudaGetLastError();
}

// do_ift scale x 1/N^3, depad (drop the two x padding floats) and phase origin
// to centre (libEM/reconstructor.cpp:1593-1597) in one pass.
__global__ void k_depad_center(const float *__restrict__ in, int N, int NZ, float scale,
                               float *__restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n3 = (long)N * N * NZ;
  if (i >= n3) return;
  const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / ((long)N * N));
  const int h = N / 2;
  const int sx = (x + h) % N, sy = (y + h) % N, sz = (z + NZ / 2) % NZ;
  out[i] = __fmul_rn(in[((long)sz * N + sy) * (N + 2) + sx], scale);
}

cudaError_t launch_depad_center(const float *d_real_padded, int N, float scale, float *d_out,
                                cudaStream_t st, int nz) {
  const int NZ = nz ? nz : N;
  const long n3 = (long)N * N * NZ;
  note_launch();
  k_depad_center<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d_real_padded, N, NZ, scale, d_out);
  return cudaGetLastError();
}

// math.gausskernelfix: MaskGaussInvProcessor (libEM/processor.h:4131-4176)
// run by CoordinateProcessor::process_inplace (libEM/processor.cpp:2439-2473)
// divides each voxel by exp(-dist * gauss_width / (ny*ny)), dist the squared
// distance (float, as CircularMaskProcessor::process_pixel forms it,
// libEM/processor.h:3785-3789) to (floor(nx/2), floor(ny/2), floor(nz/2)).
// The quotient is taken in double and rounded once.
__device__ __forceinline__ float kernel_fix(float v, int x, int y, int z, float xc, float yc,
                                            float zc, float sv) {
  const float dx = __fsub_rn((float)x, xc), dy = __fsub_rn((float)y, yc),
              dz = __fsub_rn((float)z, zc);
  const float dist = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  const float f = __fmul_rn(-dist, sv);
  return (float)((double)v / exp((double)f));
}

__global__ void k_kernel_fix(float *__restrict__ vol, int nx, int ny, int nz, float sv) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)nx * ny * nz) return;
  const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long)nx * ny));
  vol[i] = kernel_fix(vol[i], x, y, z, floorf(nx / 2.0f), floorf(ny / 2.0f), floorf(nz / 2.0f), sv);
}

cudaError_t launch_kernel_fix(float *d_vol, int nx, int ny, int nz, float gauss_width,
                              cudaStream_t st) {
  const long n = (long)nx * ny * nz;
  if (n == 0) return cudaSuccess;
  const float sv = gauss_width / (float)(ny * ny);   // gauss_width / (ny * ny), float
  note_launch();
  k_kernel_fix<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_vol, nx, ny, nz, sv);
  return cudaGetLastError();
}

// The end of e2make3dpar's reconstruction (programs/e2make3dpar.py:421-431)
// fused into finish's last pass: depad + phase origin to centre + 1/N^3
// (as k_depad_center), the radial kernel correction when sv > 0, and the
// clip to the centred (onx, ony, onz) region starting at (x0, y0, z0).
__global__ void k_finish_out(const float *__restrict__ in, int N, float scale, float sv, int x0,
                             int y0, int z0, int onx, int ony, int onz, float *__restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)onx * ony * onz) return;
  const int x = x0 + (int)(i % onx), y = y0 + (int)((i / onx) % ony),
            z = z0 + (int)(i / ((long)onx * ony));
  const int h = N / 2;
  const int sx = (x + h) % N, sy = (y + h) % N, sz = (z + h) % N;
  float v = __fmul_rn(in[((long)sz * N + sy) * (N + 2) + sx], scale);
  if (sv > 0.0f) {
    const float c = floorf(N / 2.0f);
    v = kernel_fix(v, x, y, z, c, c, c, sv);
  }
  out[i] = v;
}

cudaError_t launch_finish_out(const float *d_real_padded, int N, float scale, float gauss_width,
                              int onx, int ony, int onz, float *d_out, cudaStream_t st) {
  const long n = (long)onx * ony * onz;
  if (n == 0) return cudaSuccess;
  const float sv = gauss_width > 0.0f ? gauss_width / (float)(N * N) : 0.0f;
  // Region((nx-outx)/2, ...) with Python floor division
  const int x0 = (N - onx) / 2, y0 = (N - ony) / 2, z0 = (N - onz) / 2;
  note_launch();
  k_finish_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_real_padded, N, scale, sv, x0, y0,
                                                           z0, onx, ony, onz, d_out);
  return cudaGetLastError();
}

// xform.phaseorigin.tocorner of a real N^3 volume (even N): a circular shift
// by N/2 along each axis.
__global__ void k_tocorner3(const float *__restrict__ in, int N, float *__restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n3 = (long)N * N * N;
  if (i >= n3) return;
  const int x = (int)(i % N), y = (int)((i / N) % N), z = (int)(i / ((long)N * N));
  const int h = N / 2;
  out[i] = in[((long)((z + h) % N) * N + (y + h) % N) * N + (x + h) % N];
}

cudaError_t launch_tocorner3(const float *d_in, int N, float *d_out, cudaStream_t st) {
  const long n3 = (long)N * N * N;
  note_launch();
  k_tocorner3<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(d_in, N, d_out);
  return cudaGetLastError();
}

// FourierReconstructor::setup_seed (libEM/reconstructor.cpp:865-895):
// data = seed * w (mult skips f == 1), norm = w, with the x=0 and x=N/2
// planes at w/2 and four cells restored to w.
__global__ void k_seed(const float *__restrict__ seed, float w, int N, float *__restrict__ data,
                       float *__restrict__ norm) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nn = (long)N * N * (N / 2 + 1);
  if (i >= nn) return;
  const int nnx = N / 2 + 1;
  const int x = (int)(i % nnx), y = (int)((i / nnx) % N), z = (int)(i / ((long)nnx * N));
  float2 v = reinterpret_cast<const float2 *>(seed)[i];
  if (w != 1.0f) { v.x = __fmul_rn(v.x, w); v.y = __fmul_rn(v.y, w); }
  reinterpret_cast<float2 *>(data)[i] = v;
  float nv = w;
  if (x == 0 || x == nnx - 1) {
    nv = (float)(w / 2.0);
    if ((y == N / 2 && z == 0) || (y == 0 && z == N / 2)) nv = w;
  }
  norm[i] = nv;
}

cudaError_t launch_seed(const float *d_seed, float w, int N, float *d_data, float *d_norm,
                        cudaStream_t st) {
  const long nn = (long)N * N * (N / 2 + 1);
  note_launch();
  k_seed<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(d_seed, w, N, d_data, d_norm);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- agreement
// FourierReconstructor::do_compare_slice_work (libEM/reconstructor.cpp:1259-1381)
// with pixel_at (:1448-1462).  One block per slice; all symmetry copies;
// FP64 block reductions.  The reference loops one column past Nyquist and
// reads the slice buffer directly (so the x=0, y<0 entries are the stored
// ones, not conjugates); the read past the last row's end returns 0 here.
__device__ __forceinline__ int ref_round(float x) {
  if (x < 0) return (int)__fsub_rn(x, 0.5f);
  return (int)__fadd_rn(x, 0.5f);
}

__global__ void __launch_bounds__(256) k_agree(const float *__restrict__ rdata,
                                               const float *__restrict__ norm, int N,
                                               const float *__restrict__ slices,
                                               const float *__restrict__ t3d, int nsym,
                                               const float *__restrict__ wts, float apix,
                                               const float *__restrict__ rtab,
                                               float *__restrict__ out) {
  __shared__ double s_red[8][8];
  const int p = blockIdx.x;
  const int n2 = N / 2, nxf = N + 2;
  const long slen = (long)N * nxf;
  const float *sl = slices + (size_t)p * slen;
  const float iny = (float)N, inx = (float)nxf;
  float rmax = (float)(iny * apix / 12.0);
  if (rmax > iny / 2.0 - 1.0) rmax = (float)(iny / 2.0 - 1.0);
  if (rmax < 5.0) rmax = 5.0f;
  const long nxy = (long)nxf * N;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // dotlow dlpow dlpow2 dot vweight power power2 nval
  const int xw = n2 + 2;                       // x = 0 .. N/2+1
  const int npx = xw * N;
  for (int s = 0; s < nsym; s++) {
    float M[6];
#pragma unroll
    for (int k = 0; k < 6; k++) M[k] = t3d[((size_t)p * nsym + s) * 9 + k];
    for (int i = threadIdx.x; i < npx; i += blockDim.x) {
      const int x = i % xw, y = i / xw - n2;
      if (x == 0 && y == 0) continue;
      const float rx = __fdiv_rn((float)x, __fsub_rn(inx, 2.0f));
      const float ry = __ldg(&rtab[y + n2]);
      float xx = __fadd_rn(__fmul_rn(rx, M[0]), __fmul_rn(ry, M[3]));
      float yy = __fadd_rn(__fmul_rn(rx, M[1]), __fmul_rn(ry, M[4]));
      float zz = __fadd_rn(__fmul_rn(rx, M[2]), __fmul_rn(ry, M[5]));
      if (fabsf(xx) > 0.5f || fabsf(yy) >= 0.5f || fabsf(zz) >= 0.5f) continue;
      xx = __fmul_rn(xx, (float)N);
      yy = __fmul_rn(yy, (float)N);
      zz = __fmul_rn(zz, (float)N);
      const long idx = (long)__fadd_rn((float)(x * 2), __fmul_rn(inx, (float)(y < 0 ? N + y : y)));
      const float d2r = idx < slen ? sl[idx] : 0.0f;
      const float d2i = idx + 1 < slen ? sl[idx + 1] : 0.0f;
      const int x0 = ref_round(xx), y0 = ref_round(yy), z0 = ref_round(zz);
      float vre = 0.f, vim = 0.f;
      long cidx;
      if (x0 < 0) cidx = (long)(-x0) * 2 + (long)(y0 <= 0 ? -y0 : N - y0) * nxf + (long)(z0 <= 0 ? -z0 : N - z0) * nxy;
      else cidx = (long)x0 * 2 + (long)(y0 < 0 ? N + y0 : y0) * nxf + (long)(z0 < 0 ? N + z0 : z0) * nxy;
      if (!(abs(x0) >= nxf / 2 || abs(y0) > N / 2 || abs(z0) > N / 2)) {
        vre = rdata[cidx];
        vim = x0 < 0 ? -rdata[cidx + 1] : rdata[cidx + 1];
      }
      const float nv = norm[cidx / 2];
      if (nv == 0.0f) continue;
      const float dt0 = __fdiv_rn(vre, nv), dt1 = __fdiv_rn(vim, nv);
      const float r = (float)sqrt((double)(x * x + y * y));
      const float pdot = __fmul_rn(__fadd_rn(__fmul_rn(dt0, d2r), __fmul_rn(dt1, d2i)), nv);
      const float pv = __fmul_rn(__fadd_rn(__fmul_rn(dt0, dt0), __fmul_rn(dt1, dt1)), nv);
      const float pi2 = __fmul_rn(__fadd_rn(__fmul_rn(d2r, d2r), __fmul_rn(d2i, d2i)), nv);
      if (r > 3 && r < rmax) { acc[0] += pdot; acc[1] += pv; acc[2] += pi2; }
      acc[3] += pdot;
      acc[4] += nv;
      acc[5] += pv;
      acc[6] += pi2;
      acc[7] += 1.0;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    double v = acc[k];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[8];
    for (int k = 0; k < 8; k++) {
      t[k] = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t[k] += s_red[k][w];
    }
    double dotlow = t[0], dlpow = t[1], dlpow2 = t[2], dot = t[3], vweight = t[4];
    const double power = t[5], power2 = t[6];
    const int nval = (int)t[7];
    dot /= sqrt(power * power2);
    if (dlpow * dlpow2 > 0) dotlow /= sqrt(dlpow * dlpow2);
    const float weight = wts[p];
    float *o = out + 5 * p;
    o[0] = (float)(power2 <= 0 ? 1.0 : sqrt(power / power2));
    o[1] = (float)dot;
    o[2] = (float)dotlow;
    const float rw = weight <= 0 ? 1.0f : 1.0f / weight;
    o[3] = (float)(dot * rw / ((rw - 1.0) * dot + 1.0));
    o[4] = (float)(vweight / (float)nval);
  }
}

cudaError_t launch_agree_rt(const float *d_data, const float *d_norm, int N, const float *d_slices,
                            const float *d_t3d, int np, int nsym, const float *d_w, float apix,
                            const float *d_rtab, float *d_out, cudaStream_t st) {
  if (np == 0) return cudaSuccess;
  note_launch();
  k_agree<<<np, 256, 0, st>>>(d_data, d_norm, N, d_slices, d_t3d, nsym, d_w, apix, d_rtab, d_out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- projection
// FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1432),
// Fourier-space part: nearest-voxel value/weight for each slice pixel.
// pixel_at divides by the weight; cells with weight < 0.005 stay 0; x=0 and
// x=N/2 columns are halved except at y=0 and y=-N/2.
// Value of pixel (x, y) of FourierReconstructor::projection
// (libEM/reconstructor.cpp:1407-1431): the slice coordinate rotated
// (transpose multiply), the nearest voxel's value over its weight
// (pixel_at, :1448-1462); false where the reference skips the pixel.
__device__ __forceinline__ bool proj_pixel(const float *__restrict__ rdata,
                                           const float *__restrict__ norm, int N,
                                           const float *__restrict__ rot,
                                           const float *__restrict__ rtab, int x, int y,
                                           float &d0, float &d1) {
  const int n2 = N / 2, nxf = N + 2;
  const long nxy = (long)nxf * N;
  const float rx = __fdiv_rn((float)x, (float)(nxf - 2));
  const float ry = __ldg(&rtab[y + n2]);
  float xx = __fadd_rn(__fmul_rn(rx, rot[0]), __fmul_rn(ry, rot[3]));
  float yy = __fadd_rn(__fmul_rn(rx, rot[1]), __fmul_rn(ry, rot[4]));
  float zz = __fadd_rn(__fmul_rn(rx, rot[2]), __fmul_rn(ry, rot[5]));
  if (fabsf(xx) > 0.5f || fabsf(yy) >= 0.5f || fabsf(zz) >= 0.5f) return false;
  xx = __fmul_rn(xx, (float)N);
  yy = __fmul_rn(yy, (float)N);
  zz = __fmul_rn(zz, (float)N);
  const int x0 = ref_round(xx), y0 = ref_round(yy), z0 = ref_round(zz);
  long cidx;
  if (x0 < 0) cidx = (long)(-x0) * 2 + (long)(y0 <= 0 ? -y0 : N - y0) * nxf + (long)(z0 <= 0 ? -z0 : N - z0) * nxy;
  else cidx = (long)x0 * 2 + (long)(y0 < 0 ? N + y0 : y0) * nxf + (long)(z0 < 0 ? N + z0 : z0) * nxy;
  float vre = 0.f, vim = 0.f;
  if (!(abs(x0) >= nxf / 2 || abs(y0) > N / 2 || abs(z0) > N / 2)) {
    vre = rdata[cidx];
    vim = x0 < 0 ? -rdata[cidx + 1] : rdata[cidx + 1];
  }
  const float nv = norm[cidx / 2];
  if (nv < 0.005f) return false;
  d0 = __fdiv_rn(vre, nv);
  d1 = __fdiv_rn(vim, nv);
  // the x == nx/2 branch of the reference's halving is the column past
  // Nyquist, which set_complex_at drops
  if (x == 0 && y != 0 && y != -n2) { d0 = d0 / 2; d1 = d1 / 2; }
  return true;
}

// The projection's complex slice, written as the 2-D EMData::set_complex_at
// writes it (libEM/emdata_core.cpp:171-206): columns x = 0 and x = N/2 are
// kept Hermitian, a pixel at y > 0 setting rows y and N-y (its conjugate),
// the one at -y only when the pixel at y was skipped (it comes first in the
// reference's loop); rows 0 and N/2 of those columns keep the real part.
// out[N][N+2] zeroed beforehand.  Grid: (N/2+1) x N pixels.
__global__ void k_projection(const float *__restrict__ rdata, const float *__restrict__ norm, int N,
                             const float *__restrict__ rot, const float *__restrict__ rtab,
                             float *__restrict__ out) {
  const int n2 = N / 2, nxf = N + 2, xw = n2 + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= xw * N) return;
  const int x = i % xw, y = i / xw - n2;
  float d0, d1;
  if (x == 0 || x == n2) {
    if (y == 0 || y == -n2) {
      if (proj_pixel(rdata, norm, N, rot, rtab, x, y, d0, d1)) {
        const long o = (long)(y == 0 ? 0 : n2) * nxf + 2 * x;
        out[o] = d0;
        out[o + 1] = 0.0f;
      }
      return;
    }
    if (y < 0) return;
    const long op = (long)y * nxf + 2 * x, om = (long)(N - y) * nxf + 2 * x;
    if (proj_pixel(rdata, norm, N, rot, rtab, x, y, d0, d1)) {
      out[op] = d0; out[op + 1] = d1;
      out[om] = d0; out[om + 1] = -d1;
    } else if (proj_pixel(rdata, norm, N, rot, rtab, x, -y, d0, d1)) {
      out[om] = d0; out[om + 1] = d1;
      out[op] = d0; out[op + 1] = -d1;
    }
    return;
  }
  if (proj_pixel(rdata, norm, N, rot, rtab, x, y, d0, d1)) {
    const long o = (long)(y < 0 ? N + y : y) * nxf + 2 * x;
    out[o] = d0;
    out[o + 1] = d1;
  }
}

// The projection's translation (libEM/reconstructor.cpp:1435-1437): the
// xform processor's 2-D complex branch for a rotation-free transform
// (libEM/processor.cpp:11082-11178) copies each value and rotates it by the
// phase -2*pi*(ky*ty + kx*tx)/N (ky of row r: r - N for r > N/2).  The
// reference forms the phase in long double and rounds it to float, and
// takes cos/sin and the products in double; here the phase is formed in
// double.  checker: the phase origin to the centre (center_origin_fft,
// libEM/sparx/emdata_sparx.cpp:8420-8462: -1 where x + row is odd);
// c2r_prep: the imaginary parts of the four self-conjugate values set to 0
// (the part of them an inverse real FFT ignores).
__global__ void k_proj_shift(float *__restrict__ out, int N, float tx, float ty, int checker,
                             int c2r_prep) {
  const int n2 = N / 2, nxf = N + 2, xw = n2 + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= xw * N) return;
  const int x = i % xw, row = i / xw;
  const int ky = row >= n2 + 1 ? row - N : row;
  const double pi = 3.141592653589793238462643383279502884197169399;
  const float phase_y = (float)((((-2.0 * pi) * ky) * (double)ty) / N);
  const float phase = (float)((double)phase_y - (((2.0 * pi) * x) * (double)tx) / N);
  const double c = cos((double)phase), s = sin((double)phase);
  const long o = (long)row * nxf + 2 * x;
  const double re = out[o], im = out[o + 1];
  float a = (float)(re * c - im * s), b = (float)(re * s + im * c);
  if (checker && ((x + row) & 1)) { a = -a; b = -b; }
  if (c2r_prep && (x == 0 || x == n2) && (row == 0 || row == n2)) b = 0.0f;
  out[o] = a;
  out[o + 1] = b;
}

__global__ void k_scale(const float *__restrict__ in, size_t n, float scale, float *__restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i] * scale;
}

cudaError_t launch_projection_rt(const float *d_data, const float *d_norm, int N, const float *d_rot,
                                 const float *d_rtab, float *d_out, cudaStream_t st) {
  const int n = (N / 2 + 1) * N;
  note_launch();
  k_projection<<<(n + 255) / 256, 256, 0, st>>>(d_data, d_norm, N, d_rot, d_rtab, d_out);
  return cudaGetLastError();
}

cudaError_t launch_proj_shift(float *d_out, int N, float tx, float ty, int checker, int c2r_prep,
                              cudaStream_t st) {
  const int n = (N / 2 + 1) * N;
  note_launch();
  k_proj_shift<<<(n + 255) / 256, 256, 0, st>>>(d_out, N, tx, ty, checker, c2r_prep);
  return cudaGetLastError();
}

cudaError_t launch_scale(const float *d_in, size_t n, float scale, float *d_out, cudaStream_t st) {
  note_launch();
  const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
  k_scale<<<grid, 256, 0, st>>>(d_in, n, scale, d_out);
  return cudaGetLastError();
}

}  // namespace fr
