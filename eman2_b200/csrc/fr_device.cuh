// fr_device.cuh -- device-side arithmetic shared by the insertion, agreement
// and finish kernels.  Every rounding point of the reference's FP32 path is
// reproduced with explicit round-to-nearest intrinsics, so no FMA contraction
// or reassociation can move a window boundary or an exp-table index.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fr {

enum { MODE_NEAREST = 1, MODE_GAUSS2 = 2, MODE_GAUSS5 = 5, MODE_TRILINEAR = 6, MODE_ITER = 7 };

// Util::fast_exp (libEM/util.cpp:788-800): table of exp(-i/50) indexed by
// (int)(-f*50.0 + 0.5) in double arithmetic; exp() outside [-19.98, 0].
// The index is formed exactly in single precision: 50*y = p + e exactly
// (p rounded product, e its FMA residual), so floor(50*y + 0.5) is
// floor(p) + [frac(p) + e >= 0.5], with frac(p) exact by Sterbenz.
// The comparison f < -19.98f selects the same floats as the double
// comparison f < -19.98 (the float nearest 19.98 lies below it).
__device__ __forceinline__ float fast_exp(float f, const float *__restrict__ table) {
  if (f > 0.0f || f < -19.98f) return expf(f);
  const float y = -f;
  const float p = __fmul_rn(y, 50.0f);
  const float e = __fmaf_rn(y, 50.0f, -p);
  const float q = floorf(p);
  const float fr = __fsub_rn(p, q);
  // q is integral and < 2^23: adding 2^23 leaves it in the low mantissa bits.
  int g = __float_as_int(__fadd_rn(q, 8388608.0f)) - 0x4B000000;
  g += (fr > 0.5f || (fr == 0.5f && e >= 0.0f)) ? 1 : 0;
  return table[g];
}

// floor(xx - 2.5) evaluated exactly (the reference subtracts in double,
// libEM/reconstructor_tools.cpp:317).  With j = floor(xx), xx - j is exact
// in float (Sterbenz for |xx| >= 1; for j = -1 it may round, but never to
// the other side of 0.5, which is representable), and
// floor(xx - 2.5) = j - 3 + [xx - j >= 0.5].  Checked against the double
// expression for every float of magnitude <= 256.
__device__ __forceinline__ int floor_minus_2p5(float xx) {
  const float j = floorf(xx);
  return (int)j - 3 + (__fsub_rn(xx, j) >= 0.5f ? 1 : 0);
}

// (rx, ry, 0) * t3d, transpose multiply (libEM/transform.h:547-553), then
// scaled by the volume size (libEM/reconstructor.cpp:1193-1196).
// M is the row-major 3x3 rotation block; only rows 0 and 1 enter.
__device__ __forceinline__ void pixel_coords(float rx, float ry, const float *M, float Nf,
                                             float &xx, float &yy, float &zz) {
  xx = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[0]), __fmul_rn(ry, M[3])), Nf);
  yy = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[1]), __fmul_rn(ry, M[4])), Nf);
  zz = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[2]), __fmul_rn(ry, M[5])), Nf);
}
// The same into a volume of z size NZf (x and y: Nf).
__device__ __forceinline__ void pixel_coords_z(float rx, float ry, const float *M, float Nf,
                                               float NZf, float &xx, float &yy, float &zz) {
  xx = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[0]), __fmul_rn(ry, M[3])), Nf);
  yy = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[1]), __fmul_rn(ry, M[4])), Nf);
  zz = __fmul_rn(__fadd_rn(__fmul_rn(rx, M[2]), __fmul_rn(ry, M[5])), NZf);
}

// Util::hypot3sq (libEM/util.h:816-819) of (i-xx, j-yy, k-zz).
__device__ __forceinline__ float dist2(int i, int j, int k, float xx, float yy, float zz) {
  const float dx = __fsub_rn((float)i, xx);
  const float dy = __fsub_rn((float)j, yy);
  const float dz = __fsub_rn((float)k, zz);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Tap arithmetic of the three inserters for tap (i,j,k) of a pixel at
// (xx,yy,zz) with value (re,im) and weight w.  Writes the complex value
// added and the weight added (libEM/reconstructor_tools.cpp:113-189,315-376).
template <int MODE>
__device__ __forceinline__ void tap_value(int i, int j, int k, float xx, float yy, float zz,
                                          float re, float im, float w, float h,
                                          const float *__restrict__ table, float &vre,
                                          float &vim, float &vw) {
  if (MODE == MODE_NEAREST) {
    vre = __fmul_rn(re, w);
    vim = __fmul_rn(im, w);
    vw = w;
  } else if (MODE == MODE_GAUSS2) {
    const float r = dist2(i, j, k, xx, yy, zz);
    const float gg = __fmul_rn(fast_exp(__fmul_rn(-r, h), table), w);
    vre = __fmul_rn(re, gg);
    vim = __fmul_rn(im, gg);
    vw = gg;
  } else if (MODE == MODE_GAUSS5) {
    const float r = dist2(i, j, k, xx, yy, zz);
    const float gg = fast_exp(__fmul_rn(-r, h), table);
    vre = __fmul_rn(__fmul_rn(re, gg), w);
    vim = __fmul_rn(__fmul_rn(im, gg), w);
    vw = __fmul_rn(gg, w);
  } else {  // MODE_TRILINEAR (libEM/reconstructor_tools.cpp:191-230): double products
    double a = (1.0 - fabs((double)__fsub_rn((float)i, xx))) *
               (1.0 - fabs((double)__fsub_rn((float)j, yy)));
    a = a * (1.0 - fabs((double)__fsub_rn((float)k, zz)));
    const float gg = (float)(a * (double)w);
    vre = __fmul_rn(re, gg);
    vim = __fmul_rn(im, gg);
    vw = gg;
  }
}

// EMData::add_complex_at_fast (libEM/emdata_core.h:368-410) plus the weight
// add at the returned index, with FP32 atomics.  data: [N][N][N+2] floats,
// norm: [N][N][N/2+1].  The two "imaginary := 0" cells are written with a
// plain store: no other tap ever adds to their imaginary parts.
// NZ: the volume's z size (N for the cubic volume; [NZ][N][N+2] otherwise).
__device__ __forceinline__ void add_tap_atomic(float *__restrict__ data, float *__restrict__ norm,
                                               int N, int NZ, int x, int y, int z, float re,
                                               float im, float wt) {
  const int h = N >> 1;
  if (abs(x) > h || abs(y) > h || abs(z) > (NZ >> 1)) return;
  const size_t nxf = (size_t)N + 2;
  const size_t nxy = nxf * (size_t)N;
  const size_t rc = (size_t)(y <= 0 ? -y : N - y) * nxf + (size_t)(z <= 0 ? -z : NZ - z) * nxy;
  if (x == 0) {
    if (y == 0 && z == 0) {
      atomicAdd(&data[0], re);
      data[1] = 0.0f;
      atomicAdd(&norm[0], wt);
      return;
    }
    atomicAdd(reinterpret_cast<float2 *>(&data[rc]), make_float2(re, -im));
  }
  if (abs(x) == h) {
    if (y == 0 && z == 0) {
      atomicAdd(&data[nxf - 2], re);
      data[nxf - 1] = 0.0f;
      atomicAdd(&norm[(nxf - 2) >> 1], wt);
      return;
    }
    atomicAdd(reinterpret_cast<float2 *>(&data[nxf - 2 + rc]), make_float2(re, -im));
  }
  if (x < 0) {
    const size_t idx = (size_t)(-x * 2) + rc;
    atomicAdd(reinterpret_cast<float2 *>(&data[idx]), make_float2(re, -im));
    atomicAdd(&norm[idx >> 1], wt);
    return;
  }
  const size_t idx = (size_t)x * 2 + (size_t)(y < 0 ? N + y : y) * nxf +
                     (size_t)(z < 0 ? NZ + z : z) * nxy;
  atomicAdd(reinterpret_cast<float2 *>(&data[idx]), make_float2(re, im));
  atomicAdd(&norm[idx >> 1], wt);
}

// EMData::get_complex_at(x,y) of a 2-D slice (libEM/emdata_core.cpp:126-132)
// for x in [0,N/2], y in [-N/2,N/2): row |y| conjugated when x == 0, y < 0.
__device__ __forceinline__ float2 slice_value(const float2 *__restrict__ s, int N, int x, int y) {
  const int w = (N >> 1) + 1;
  if (x == 0 && y < 0) {
    const float2 v = __ldg(&s[(size_t)(-y) * w]);
    return make_float2(v.x, -v.y);
  }
  return __ldg(&s[(size_t)(y < 0 ? N + y : y) * w + x]);
}

// The same read with the load cached in L2 only (ld.global.cg): for values
// staged once into shared memory, so they do not evict L1-resident tables.
__device__ __forceinline__ float2 slice_value_cg(const float2 *__restrict__ s, int N, int x, int y) {
  const int w = (N >> 1) + 1;
  if (x == 0 && y < 0) {
    const float2 v = __ldcg(&s[(size_t)(-y) * w]);
    return make_float2(v.x, -v.y);
  }
  return __ldcg(&s[(size_t)(y < 0 ? N + y : y) * w + x]);
}

}  // namespace fr
