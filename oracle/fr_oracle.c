/*
 * fr_oracle.c -- CPU restatement of EMAN2's direct Fourier inversion
 * (FourierReconstructor, Reconstructors.get("fourier")).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the GPU product
 * (eman2_b200/) never links, loads or calls it.  Only tests/, the smoke check
 * in __graft_entry__.py and the cpu_baseline / --impl reference legs of
 * bench.py use it, always as the checker or the timed CPU baseline.
 *
 * Parity status: the reference's own tests hold no golden vectors for this
 * path (rt/pyem/test_reconstructor.py:94-115 asserts nothing; the only
 * asserting test, :48-90, is disabled).  This restatement is pinned against
 * the reference's own inserter and Hermitian-add source compiled from where it
 * lies (oracle/build_ref.sh -> oracle/_ref/), see tests/test_oracle_ref.py.
 *
 * One source, three builds:
 *   OR_REAL=float  -> the FP32-faithful oracle: the same operation order and
 *                     rounding points as the reference source, evaluated with
 *                     strict IEEE single precision (no contraction, no
 *                     reassociation, divisions as written).
 *   OR_REAL=float, OR_ACC=double
 *                  -> FP32 tap arithmetic (identical tap selection, exp-table
 *                     indices and products) summed in double: isolates the
 *                     FP32 summation-order noise of any schedule.
 *   OR_REAL=double -> the FP64 oracle: the same algorithm (table exp, the same
 *                     Hermitian bookkeeping) with double coordinates, weights
 *                     and accumulators.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * eman2 source tree).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#ifndef OR_REAL
#define OR_REAL float
#endif
typedef OR_REAL real;
#ifndef OR_ACC
#define OR_ACC OR_REAL
#endif
typedef OR_ACC acc_t;   /* volume accumulators */
#define IS_F32 (sizeof(real) == sizeof(float))

#define OR_EXPORT __attribute__((visibility("default")))

/* EMConsts (libEM/emobject.cpp:53-59). */
static const double OR_PI = 3.141592653589793238462643383279502884197169399;
#define OR_DEG2RAD (OR_PI / 180.0)
static float or_I2G(void) { return (float)(4.0 / (M_PI * M_PI)); }
static float or_I5G(void) { return (float)(10.4 / (M_PI * M_PI)); }

enum { MODE_NEAREST = 1, MODE_GAUSS2 = 2, MODE_GAUSS5 = 5, MODE_TRILINEAR = 6 };

/* ------------------------------------------------------------------ util */

/* Util::fast_exp (libEM/util.cpp:788-800): 1000-entry table of exp(-i/50),
 * nearest entry by (int)(-f*50.0+0.5) (double arithmetic); exp() outside
 * [-19.98, 0].  The FP32 build keeps the float table and std::exp(float). */
static real g_exp_table[1000];
static int g_exp_init = 0;
static void or_init_tables(void) {
  if (g_exp_init) return;
  for (int i = 0; i < 1000; i++) g_exp_table[i] = (real)exp(-i / 50.0);
  g_exp_init = 1;
}
static inline real or_fast_exp(real f) {
  if ((double)f > 0 || (double)f < -19.98) return IS_F32 ? (real)expf((float)f) : (real)exp((double)f);
  int g = (int)(-(double)f * 50.0 + 0.5);
  return g_exp_table[g];
}

/* Util::hypot_fast_int (libEM/util.cpp:764-786): (short)Util::round(hypot(x,y))
 * with std::hypot(float,float); Util::round (libEM/util.h:465-470). */
static inline int or_hypot_fast_int(int x, int y) {
  float h = hypotf((float)abs(x), (float)abs(y));
  return (int)(h + 0.5f);
}
/* Util::hypot_fast (libEM/util.cpp:742-762): float hypot table. */
static inline float or_hypot_fast(int x, int y) { return hypotf((float)abs(x), (float)abs(y)); }

/* Util::round (libEM/util.h:465-470). */
static inline int or_round(real x) {
  if (x < 0) return (int)(x - (real)0.5);
  return (int)(x + (real)0.5);
}

/* ------------------------------------------------------------ transforms */

/* Transform::set_rotation, "eman" branch (libEM/transform.cpp:654-666).
 * Output m[9] row-major 3x3 (the Transform's upper-left block). */
OR_EXPORT void or_eman_matrix(double az, double alt, double phi, float *m) {
  double azp = az * OR_DEG2RAD, altp = alt * OR_DEG2RAD, phip = phi * OR_DEG2RAD;
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

/* Transform::set_rotation, "quaternion" branch (libEM/transform.cpp:667-678). */
OR_EXPORT void or_quaternion_matrix(double e0, double e1, double e2, double e3, float *m) {
  m[0] = (float)(e0 * e0 + e1 * e1 - e2 * e2 - e3 * e3);
  m[1] = (float)(2.0f * (e1 * e2 + e0 * e3));
  m[2] = (float)(2.0f * (e1 * e3 - e0 * e2));
  m[3] = (float)(2.0f * (e2 * e1 - e0 * e3));
  m[4] = (float)(e0 * e0 - e1 * e1 + e2 * e2 - e3 * e3);
  m[5] = (float)(2.0f * (e2 * e3 + e0 * e1));
  m[6] = (float)(2.0f * (e3 * e1 + e0 * e2));
  m[7] = (float)(2.0f * (e3 * e2 - e0 * e1));
  m[8] = (float)(e0 * e0 - e1 * e1 - e2 * e2 + e3 * e3);
}

/* CSym::get_sym (libEM/symmetry.cpp:1407-1417) and DSym::get_sym
 * (libEM/symmetry.cpp:1452-1470), both built through the "eman" Euler
 * branch.  kind 'c' or 'd'.  Writes nops*9 floats; returns nops or -1. */
OR_EXPORT int or_sym_ops(char kind, int nsym, float *out, int cap) {
  if (nsym <= 0) return -1;
  if (kind == 'c') {
    if (cap < nsym) return -1;
    for (int n = 0; n < nsym; n++) {
      float az = (float)(n % nsym) * 360.0f / (float)nsym;
      or_eman_matrix((double)az, 0.0, 0.0, out + 9 * n);
    }
    return nsym;
  }
  if (kind == 'd') {
    int ns = 2 * nsym;
    if (cap < ns) return -1;
    for (int n = 0; n < ns; n++) {
      float az, alt;
      if (n >= ns / 2) { az = (float)((n % ns) - ns / 2) * 360.0f / (float)(ns / 2); alt = 180.0f; }
      else { az = (float)(n % ns) * 360.0f / (float)(ns / 2); alt = 0.0f; }
      or_eman_matrix((double)az, (double)alt, 0.0, out + 9 * n);
    }
    return ns;
  }
  /* Platonic groups, row by row of the reference's Euler tables:
   * 't' TetrahedralSym::get_sym (libEM/symmetry.cpp:2007-2027),
   * 'o' OctahedralSym::get_sym (:1950-1973),
   * 'i' IcosahedralSym::get_sym (:1822-1868; az + 90, phi - 90). */
  if (kind == 't' || kind == 'o' || kind == 'i') {
    const int count = kind == 't' ? 12 : kind == 'o' ? 24 : 60;
    if (cap < count) return -1;
    const float tlvl1 = (float)((180.0 / M_PI) * acos((double)(-1.0f / 3.0f)));
    const float ilvl1 = (float)((180.0 / M_PI) * atan((double)2.0f));
    for (int idx = 0; idx < count; idx++) {
      float az, alt, phi;
      if (kind == 't') {
        if (idx < 3) { az = 0.0f; alt = 0.0f; phi = 120.0f * idx; }
        else { az = 120.0f * ((idx - 3) / 3); alt = tlvl1; phi = 60.0f + 120.0f * ((idx - 3) % 3); }
      } else if (kind == 'o') {
        const int row = idx / 4, col = idx % 4;
        phi = 90.0f * col;
        if (row == 0) { az = 0.0f; alt = 0.0f; }
        else if (row == 5) { az = 0.0f; alt = 180.0f; }
        else { az = 90.0f * (row - 1); alt = 90.0f; }
      } else {
        const int row = idx / 5, col = idx % 5;
        const int p0 = (360 - 72 * col) % 360;           /* 0, 288, 216, 144, 72 */
        const int p36 = (36 - 72 * col + 360) % 360;     /* 36, 324, 252, 180, 108 */
        if (row == 0) { az = 0.0f; alt = 0.0f; phi = (float)p0; }
        else if (row <= 5) { az = 72.0f * (row - 1); alt = ilvl1; phi = (float)p36; }
        else if (row <= 10) { az = 36.0f + 72.0f * (row - 6); alt = 180.0f - ilvl1; phi = (float)p0; }
        else { az = 0.0f; alt = 180.0f; phi = (float)p0; }
        az = az + 90.0f;
        phi = phi - 90.0f;
      }
      or_eman_matrix((double)az, (double)alt, (double)phi, out + 9 * idx);
    }
    return count;
  }
  return -1;
}

/* EMAN::operator*(Transform,Transform) (libEM/transform.cpp:1384-1395),
 * rotation block only (both translations are zero on the insertion path). */
OR_EXPORT void or_compose(const float *a, const float *b, float *out) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      float s = a[3 * i + 0] * b[0 * 3 + j];
      s = s + a[3 * i + 1] * b[1 * 3 + j];
      s = s + a[3 * i + 2] * b[2 * 3 + j];
      out[3 * i + j] = s;
    }
}

/* ------------------------------------------------------------- the volume */

typedef struct {
  acc_t *data;  /* complex volume, [nz][ny][nx] floats, nx = N+2 */
  acc_t *norm;  /* weights, [nz][ny][nx/2] */
  int nx, ny, nz;
  long nxyz;
} or_vol;

/* EMData::add_complex_at_fast (libEM/emdata_core.h:368-410), identical logic
 * to EMData::add_complex_at (libEM/emdata_core.cpp:251-295). */
static inline long or_add_complex_at(or_vol *v, int x, int y, int z, real re, real im) {
  const int nx = v->nx, ny = v->ny, nz = v->nz;
  const long nxy = (long)nx * ny;
  acc_t *rdata = v->data;
  if (abs(x) >= nx / 2 || abs(y) > ny / 2 || abs(z) > nz / 2) return v->nxyz;
  long idx;
  if (x == 0) {
    if (y == 0 && z == 0) { rdata[0] += re; rdata[1] = 0; return 0; }
    idx = (long)(y <= 0 ? -y : ny - y) * nx + (long)(z <= 0 ? -z : nz - z) * nxy;
    rdata[idx] += re; rdata[idx + 1] += -im;
  }
  if (abs(x) == nx / 2 - 1) {
    if (y == 0 && z == 0) { rdata[nx - 2] += re; rdata[nx - 1] = 0; return nx - 2; }
    idx = nx - 2 + (long)(y <= 0 ? -y : ny - y) * nx + (long)(z <= 0 ? -z : nz - z) * nxy;
    rdata[idx] += re; rdata[idx + 1] += -im;
  }
  if (x < 0) {
    idx = (long)(-x * 2) + (long)(y <= 0 ? -y : ny - y) * nx + (long)(z <= 0 ? -z : nz - z) * nxy;
    rdata[idx] += re; rdata[idx + 1] += -im;
    return idx;
  }
  idx = (long)x * 2 + (long)(y < 0 ? ny + y : y) * nx + (long)(z < 0 ? nz + z : z) * nxy;
  rdata[idx] += re; rdata[idx + 1] += im;
  return idx;
}

/* FourierInserter3DMode1::insert_pixel "nearest_neighbor"
 * (libEM/reconstructor_tools.cpp:113-126). */
static void or_insert_nearest(or_vol *v, real xx, real yy, real zz, real dre, real dim, real w) {
  int x0 = (int)floor(xx + (real)0.5), y0 = (int)floor(yy + (real)0.5), z0 = (int)floor(zz + (real)0.5);
  long off = or_add_complex_at(v, x0, y0, z0, dre * w, dim * w);
  if (off != v->nxyz) v->norm[off / 2] += w;
}

/* FourierInserter3DMode2::insert_pixel "gauss_2", full-volume branch
 * (libEM/reconstructor_tools.cpp:128-166). */
static void or_insert_gauss2(or_vol *v, real xx, real yy, real zz, real dre, real dim, real w) {
  const int nx2 = v->nx / 2 - 1, ny2 = v->ny / 2, nz2 = v->nz / 2;
  int x0 = (int)floor(xx), y0 = (int)floor(yy), z0 = (int)floor(zz);
  if (x0 < -nx2 - 1 || y0 < -ny2 - 1 || z0 < -nz2 - 1 || x0 > nx2 || y0 > ny2 || z0 > nz2) return;
  const real h = IS_F32 ? (real)(1.0f / or_I2G()) : (real)(1.0 / (4.0 / (M_PI * M_PI)));
  for (int k = z0; k <= z0 + 1; k++)
    for (int j = y0; j <= y0 + 1; j++)
      for (int i = x0; i <= x0 + 1; i++) {
        real dx = (real)i - xx, dy = (real)j - yy, dz = (real)k - zz;
        real r = dx * dx + dy * dy;
        r = r + dz * dz;
        real gg = or_fast_exp(-r * h) * w;
        long off = or_add_complex_at(v, i, j, k, dre * gg, dim * gg);
        if (off != v->nxyz) v->norm[off / 2] += gg;
      }
}

/* FourierInserter3DMode2l::insert_pixel "trilinear", full-volume branch
 * (libEM/reconstructor_tools.cpp:191-230). */
static void or_insert_trilinear(or_vol *v, real xx, real yy, real zz, real dre, real dim, real w) {
  const int nx2 = v->nx / 2 - 1, ny2 = v->ny / 2, nz2 = v->nz / 2;
  int x0 = (int)floor(xx), y0 = (int)floor(yy), z0 = (int)floor(zz);
  if (x0 < -nx2 - 1 || y0 < -ny2 - 1 || z0 < -nz2 - 1 || x0 > nx2 || y0 > ny2 || z0 > nz2) return;
  for (int k = z0; k <= z0 + 1; k++)
    for (int j = y0; j <= y0 + 1; j++)
      for (int i = x0; i <= x0 + 1; i++) {
        /* (1.0-fabs(i-xx))*(1.0-fabs(j-yy))*(1.0-fabs(k-zz))*weight: the
         * 1.0 literals make this double arithmetic, rounded to float once. */
        double a = (1.0 - fabs((double)((real)i - xx))) * (1.0 - fabs((double)((real)j - yy)));
        a = a * (1.0 - fabs((double)((real)k - zz)));
        real gg = (real)(a * (double)w);
        long off = or_add_complex_at(v, i, j, k, dre * gg, dim * gg);
        if (off != v->nxyz) v->norm[off / 2] += gg;
      }
}

/* FourierInserter3DMode5::insert_pixel "gauss_5", full-volume branch
 * (libEM/reconstructor_tools.cpp:315-376).  Window start by floor(xx-2.5)
 * in double, clamped window, no range check on the weight add. */
static void or_insert_gauss5(or_vol *v, real xx, real yy, real zz, real dre, real dim, real w) {
  const int nx2 = v->nx / 2 - 1, ny2 = v->ny / 2, nz2 = v->nz / 2;
  int x0 = (int)floor((double)xx - 2.5), y0 = (int)floor((double)yy - 2.5), z0 = (int)floor((double)zz - 2.5);
  if (x0 < -nx2 - 4 || y0 < -ny2 - 4 || z0 < -nz2 - 4 || x0 > nx2 + 3 || y0 > ny2 + 3 || z0 > nz2 + 3) return;
  int x1 = x0 + 5, y1 = y0 + 5, z1 = z0 + 5;
  if (x0 < -nx2) x0 = -nx2;
  if (x1 > nx2) x1 = nx2;
  if (y0 < -ny2) y0 = -ny2;
  if (y1 > ny2) y1 = ny2;
  if (z0 < -nz2) z0 = -nz2;
  if (z1 > nz2) z1 = nz2;
  const real h = IS_F32 ? (real)(1.0f / or_I5G()) : (real)(1.0 / (10.4 / (M_PI * M_PI)));
  for (int k = z0; k <= z1; k++)
    for (int j = y0; j <= y1; j++)
      for (int i = x0; i <= x1; i++) {
        real dx = (real)i - xx, dy = (real)j - yy, dz = (real)k - zz;
        real r = dx * dx + dy * dy;
        r = r + dz * dz;
        real gg = or_fast_exp(-r * h);
        real gre = dre * gg, gim = dim * gg;
        long off = or_add_complex_at(v, i, j, k, gre * w, gim * w);
        v->norm[off / 2] += gg * w;
      }
}

/* EMData::get_complex_at(x,y) for a 2-D complex slice
 * (libEM/emdata_core.cpp:126-132); slice is [ny][nx] floats, nx = N+2. */
static inline void or_slice_at(const float *s, int nx, int ny, int x, int y, real *re, real *im) {
  if (abs(x) >= nx / 2 || abs(y) > ny / 2) { *re = 0; *im = 0; return; }
  if (x >= 0 && y >= 0) { *re = s[x * 2 + y * nx]; *im = s[x * 2 + y * nx + 1]; return; }
  if (x > 0 && y < 0) { *re = s[x * 2 + (ny + y) * nx]; *im = s[x * 2 + (ny + y) * nx + 1]; return; }
  if (x < 0 && y > 0) { *re = s[-x * 2 + (ny - y) * nx]; *im = -s[-x * 2 + (ny - y) * nx + 1]; return; }
  *re = s[-x * 2 - y * nx]; *im = -s[-x * 2 - y * nx + 1];
}

/* FourierReconstructor::do_insert_slice_work (libEM/reconstructor.cpp:1122-1210)
 * for one preprocessed slice and its already-composed per-symmetry rotation
 * blocks t3d[nsym*9] (arg*sym, libEM/transform.cpp:1384).
 * vol_data [N][N][N+2], vol_norm [N][N][N/2+1]; slice [N][N+2] (complex).
 * weight < 0 selects the SSNR path (ssnr table of nssnr entries). */
static int or_insert_slice_nz(acc_t *vol_data, acc_t *vol_norm, int N, int NZ, int mode,
                              const float *slice, const float *t3d, int nsym,
                              float weight, int corners, const float *ssnr, int nssnr) {
  or_init_tables();
  or_vol v;
  v.data = vol_data; v.norm = vol_norm;
  v.nx = N + 2; v.ny = N; v.nz = NZ;
  v.nxyz = (long)v.nx * v.ny * v.nz;
  const float inx = (float)(N + 2), iny = (float)N;
  const int nx = N + 2, ny = N, nz = NZ;  /* FourierReconstructor members after setup() */
  float sscale = 1.0f;
  if (weight < 0) {
    if (!ssnr || nssnr < 1) return -1;
    sscale = (float)(2.0 * (nssnr - 1) / iny);
  }
  for (int s = 0; s < nsym; s++) {
    const float *M = t3d + 9 * s;
    for (int y = (int)(-iny / 2); y < iny / 2; y++) {
      for (int x = 0; x < inx / 2; x++) {
        real rweight = weight;
        if (corners) {
          if (weight < 0) {
            int r = or_hypot_fast_int(x, y);
            float sv = ssnr[(int)(r * sscale)];
            rweight = sv > 0.0f ? sv : 0.0f;
          }
        } else {
          int r = or_hypot_fast_int(x, y);
          if (r > iny / 2 && fabsf(inx - iny) < 3) continue;
          if (weight < 0) {
            float sv = ssnr[(int)(r * sscale)];
            rweight = sv > 0.0f ? sv : 0.0f;
          }
        }
        real rx, ry, xx, yy, zz;
        if (IS_F32) {
          rx = (real)((float)x / (inx - 2.0f));
          ry = (real)((float)y / iny);
        } else {
          rx = (real)x / (real)(inx - 2.0f);
          ry = (real)y / (real)iny;
        }
        /* Vec3f(rx,ry,0) * t3d, transpose multiply (libEM/transform.h:547-553) */
        xx = rx * (real)M[0] + ry * (real)M[3];
        yy = rx * (real)M[1] + ry * (real)M[4];
        zz = rx * (real)M[2] + ry * (real)M[5];
        xx = xx * (real)(nx - 2);
        yy = yy * (real)ny;
        zz = zz * (real)nz;
        real dre, dim;
        or_slice_at(slice, nx, ny, x, y, &dre, &dim);
        switch (mode) {
          case MODE_NEAREST: or_insert_nearest(&v, xx, yy, zz, dre, dim, rweight); break;
          case MODE_GAUSS2: or_insert_gauss2(&v, xx, yy, zz, dre, dim, rweight); break;
          case MODE_GAUSS5: or_insert_gauss5(&v, xx, yy, zz, dre, dim, rweight); break;
          case MODE_TRILINEAR: or_insert_trilinear(&v, xx, yy, zz, dre, dim, rweight); break;
          default: return -2;
        }
      }
    }
  }
  return 0;
}

OR_EXPORT int or_insert_slice(acc_t *vol_data, acc_t *vol_norm, int N, int mode,
                              const float *slice, const float *t3d, int nsym,
                              float weight, int corners, const float *ssnr, int nssnr) {
  return or_insert_slice_nz(vol_data, vol_norm, N, N, mode, slice, t3d, nsym, weight, corners,
                            ssnr, nssnr);
}

/* The pixel stream of do_insert_slice_work (libEM/reconstructor.cpp:1122-1210)
 * for one slice of weight > 0 and its composed rotations t3d[nsym*9]: for
 * every symmetry copy and every pixel inside the radius, (xx, yy, zz, re, im,
 * weight) as that loop hands them to FourierPixelInserter3D::insert_pixel, six
 * floats each, into px (room for cap pixels).  Returns the pixel count, or -1
 * when px is too small.  Lets the reference's own inserter (oracle/_ref)
 * consume exactly the pixels the restatement inserts. */
OR_EXPORT long or_slice_pixels(int N, const float *slice, const float *t3d, int nsym, float weight,
                               float *px, long cap) {
  const float inx = (float)(N + 2), iny = (float)N;
  const int nx = N + 2, ny = N, nz = N;
  long n = 0;
  for (int s = 0; s < nsym; s++) {
    const float *M = t3d + 9 * s;
    for (int y = (int)(-iny / 2); y < iny / 2; y++) {
      for (int x = 0; x < inx / 2; x++) {
        int r = or_hypot_fast_int(x, y);
        if (r > iny / 2 && fabsf(inx - iny) < 3) continue;
        if (n >= cap) return -1;
        const float rx = (float)x / (inx - 2.0f), ry = (float)y / iny;
        float xx = rx * M[0] + ry * M[3];
        float yy = rx * M[1] + ry * M[4];
        float zz = rx * M[2] + ry * M[5];
        xx = xx * (float)(nx - 2);
        yy = yy * (float)ny;
        zz = zz * (float)nz;
        real dre, dim;
        or_slice_at(slice, nx, ny, x, y, &dre, &dim);
        float *q = px + 6 * n++;
        q[0] = xx; q[1] = yy; q[2] = zz; q[3] = (float)dre; q[4] = (float)dim; q[5] = weight;
      }
    }
  }
  return n;
}

/* The same into a volume of size [NZ][N][N+2] (square N x N slices; the z
 * coordinate scaled by NZ, libEM/reconstructor.cpp:1193-1196). */
OR_EXPORT int or_insert_batch_nz(acc_t *vol_data, acc_t *vol_norm, int N, int NZ, int mode,
                                 const float *slices, int n, const float *arg, const float *sym,
                                 int nsym, const float *weights) {
  float *t3d = (float *)malloc(sizeof(float) * 9 * nsym);
  if (!t3d) return -3;
  const long sl = (long)N * (N + 2);
  for (int p = 0; p < n; p++) {
    if (weights[p] == 0) continue;
    for (int s = 0; s < nsym; s++) or_compose(arg + 9 * p, sym + 9 * s, t3d + 9 * s);
    int rc = or_insert_slice_nz(vol_data, vol_norm, N, NZ, mode, slices + sl * p, t3d, nsym,
                                weights[p], 0, NULL, 0);
    if (rc) { free(t3d); return rc; }
  }
  free(t3d);
  return 0;
}

/* WienerFourierReconstructor::do_insert_slice_work (libEM/reconstructor.cpp:1679-1731)
 * for one slice: pixels with rn = |(x/(inx-2), y/iny)| < .5, weight = the
 * slice's ctf_snr_total (snr[nsnr]) linearly interpolated at rn*2*nsnr (its
 * last entry times the insert weight's sign past the end), the value scaled
 * by (w+1)/w for a Wiener-filtered slice, inserted with weight*sign. */
OR_EXPORT int or_insert_slice_wiener(acc_t *vol_data, acc_t *vol_norm, int N, int mode,
                                     const float *slice, const float *t3d, int nsym,
                                     float inweight, const float *snr, int nsnr, int undo) {
  or_init_tables();
  or_vol v;
  v.data = vol_data; v.norm = vol_norm;
  v.nx = N + 2; v.ny = N; v.nz = N;
  v.nxyz = (long)v.nx * v.ny * v.nz;
  const float inx = (float)(N + 2), iny = (float)N;
  const int nx = N + 2, ny = N, nz = N;
  if (!snr || nsnr < 1) return -1;
  const float sub = inweight < 0 ? -1.0f : 1.0f;
  for (int s = 0; s < nsym; s++) {
    const float *M = t3d + 9 * s;
    for (int y = (int)(-iny / 2); y < iny / 2; y++) {
      for (int x = 0; x <= inx / 2; x++) {
        const float rx = (float)x / (inx - 2.0f);
        const float ry = (float)y / iny;
        float rn = (float)hypot(rx, ry);
        if (rn >= .5) continue;
        rn *= nsnr * 2.0f;
        const int rni = (int)floor(rn);
        float weight;
        if ((unsigned int)rni >= (unsigned int)(nsnr - 1)) weight = snr[nsnr - 1] * sub;
        else {
          rn -= rni;
          weight = (1 - rn) * snr[rni] + rn * snr[rni + 1];
        }
        real xx = (real)rx * (real)M[0] + (real)ry * (real)M[3];
        real yy = (real)rx * (real)M[1] + (real)ry * (real)M[4];
        real zz = (real)rx * (real)M[2] + (real)ry * (real)M[5];
        xx = xx * (real)(nx - 2);
        yy = yy * (real)ny;
        zz = zz * (real)nz;
        real dre, dim;
        or_slice_at(slice, nx, ny, x, y, &dre, &dim);
        if (undo) {
          const float f = (weight + 1.0f) / weight;
          dre = (real)((float)dre * f);
          dim = (real)((float)dim * f);
        }
        const real w = (real)(weight * sub);
        switch (mode) {
          case MODE_NEAREST: or_insert_nearest(&v, xx, yy, zz, dre, dim, w); break;
          case MODE_GAUSS2: or_insert_gauss2(&v, xx, yy, zz, dre, dim, w); break;
          case MODE_GAUSS5: or_insert_gauss5(&v, xx, yy, zz, dre, dim, w); break;
          case MODE_TRILINEAR: or_insert_trilinear(&v, xx, yy, zz, dre, dim, w); break;
          default: return -2;
        }
      }
    }
  }
  return 0;
}

/* EMData::get_complex_at(x,y,z) of a complex volume [N][N][N+2]
 * (libEM/emdata_core.cpp:134-144). */
static void or_volume_at(const float *v, int N, int x, int y, int z, float *re, float *im) {
  const int nx = N + 2, ny = N, nz = N;
  const long nxy = (long)nx * ny;
  if (abs(x) >= nx / 2 || abs(y) > ny / 2 || abs(z) > nz / 2) { *re = 0; *im = 0; return; }
  if (x < 0) {
    long idx = (long)(-x * 2) + (long)(y <= 0 ? -y : ny - y) * nx + (long)(z <= 0 ? -z : nz - z) * nxy;
    *re = v[idx]; *im = -v[idx + 1];
    return;
  }
  long idx = (long)x * 2 + (long)(y < 0 ? ny + y : y) * nx + (long)(z < 0 ? nz + z : z) * nxy;
  *re = v[idx]; *im = v[idx + 1];
}

/* FourierIterReconstructor::insert_slice (libEM/reconstructor.cpp:522-648)
 * for one slice with composed blocks t3d[nsym*9]; ref: the reference
 * volume [N][N][N+2] or NULL.  Single precision as the reference computes. */
OR_EXPORT int or_insert_slice_iter(acc_t *vol_data, acc_t *vol_norm, int N, const float *slice,
                                   const float *t3d, int nsym, float weight, const float *ref) {
  or_init_tables();
  or_vol v;
  v.data = vol_data; v.norm = vol_norm;
  v.nx = N + 2; v.ny = N; v.nz = N;
  v.nxyz = (long)v.nx * v.ny * v.nz;
  const float inx = (float)(N + 2), iny = (float)N;
  const int nx = N + 2, ny = N, nz = N;
  const int nx2 = nx / 2 - 2, ny2 = ny / 2, nz2 = nz / 2;
  const long ny2sq = (long)ny * ny / 4;
  for (int s = 0; s < nsym; s++) {
    const float *M = t3d + 9 * s;
    for (int y = (int)(-iny / 2); y < iny / 2; y++) {
      for (int x = 0; x < inx / 2; x++) {
        const float rx = (float)x / (inx - 2.0f);
        const float ry = (float)y / iny;
        const int r = or_hypot_fast_int(x, y);
        if (r > iny / 2 + 3 && fabsf(inx - iny) < 3) continue;
        float xx = rx * M[0] + ry * M[3];
        float yy = rx * M[1] + ry * M[4];
        float zz = rx * M[2] + ry * M[5];
        xx = xx * (float)(nx - 2);
        yy = yy * (float)ny;
        zz = zz * (float)nz;
        int x0 = (int)floor(xx - 2.5), y0 = (int)floor(yy - 2.5), z0 = (int)floor(zz - 2.5);
        real dre, dim;
        or_slice_at(slice, nx, ny, x, y, &dre, &dim);
        if (x0 < -nx2 - 4 || y0 < -ny2 - 4 || z0 < -nz2 - 4 || x0 > nx2 + 3 || y0 > ny2 + 3 || z0 > nz2 + 3)
          continue;
        int x1 = x0 + 5, y1 = y0 + 5, z1 = z0 + 5;
        if (x0 < -nx2) x0 = -nx2;
        if (x1 > nx2) x1 = nx2;
        if (y0 < -ny2) y0 = -ny2;
        if (y1 > ny2) y1 = ny2;
        if (z0 < -nz2) z0 = -nz2;
        if (z1 > nz2) z1 = nz2;
        if (ref) {
          const float xx0 = floorf(xx), yy0 = floorf(yy), zz0 = floorf(zz);
          const float t = xx - xx0, u = yy - yy0, w3 = zz - zz0;
          float pr[8], pi[8];
          for (int q = 0; q < 8; q++)
            or_volume_at(ref, N, (int)xx0 + (q & 1), (int)yy0 + ((q >> 1) & 1), (int)zz0 + (q >> 2),
                         &pr[q], &pi[q]);
          const float c[8] = {(1 - t) * (1 - u) * (1 - w3), t * (1 - u) * (1 - w3),
                              (1 - t) * u * (1 - w3),       t * u * (1 - w3),
                              (1 - t) * (1 - u) * w3,       t * (1 - u) * w3,
                              (1 - t) * u * w3,             t * u * w3};
          float nre = c[0] * pr[0], nim = c[0] * pi[0];
          for (int q = 1; q < 8; q++) { nre = nre + c[q] * pr[q]; nim = nim + c[q] * pi[q]; }
          const float h = 1.0f / 2.0f;
          for (int k = z0; k <= z1; k++)
            for (int j = y0; j <= y1; j++)
              for (int i = x0; i <= x1; i++) {
                if ((long)i * i + j * j + k * k > ny2sq) continue;
                float tre, tim;
                or_volume_at(ref, N, i, j, k, &tre, &tim);
                const float ure = ((float)dre + tre) - nre, uim = ((float)dim + tim) - nim;
                const float dx = (float)i - xx, dy = (float)j - yy, dz = (float)k - zz;
                const float rl = (dx * dx + dy * dy) + dz * dz;
                const float gg = (float)or_fast_exp((real)(-rl * h));
                long off = or_add_complex_at(&v, i, j, k, (real)((ure * gg) * weight),
                                             (real)((uim * gg) * weight));
                if (off != v.nxyz) v.norm[off / 2] += (real)(gg * weight);
              }
        } else {
          const float hs = (xx * xx + yy * yy) + zz * zz;
          float h = (float)(1.0f / ((hs / 4000) + .15));
          h = h < 0.1 ? (float)0.1 : h;
          for (int k = z0; k <= z1; k++)
            for (int j = y0; j <= y1; j++)
              for (int i = x0; i <= x1; i++) {
                const float dx = (float)i - xx, dy = (float)j - yy, dz = (float)k - zz;
                const float rl = (dx * dx + dy * dy) + dz * dz;
                const float gg = (float)or_fast_exp((real)(-rl * h));
                long off = or_add_complex_at(&v, i, j, k, (real)(((float)dre * gg) * weight),
                                             (real)(((float)dim * gg) * weight));
                if (off != v.nxyz) v.norm[off / 2] += (real)(gg * weight);
              }
        }
      }
    }
  }
  return 0;
}

/* Convenience for tests: insert n slices with per-slice orientation blocks
 * arg[n*9] composed with the symmetry operators sym[nsym*9]. */
OR_EXPORT int or_insert_batch(acc_t *vol_data, acc_t *vol_norm, int N, int mode,
                              const float *slices, int n, const float *arg,
                              const float *sym, int nsym, const float *weights, int corners) {
  float *t3d = (float *)malloc(sizeof(float) * 9 * nsym);
  if (!t3d) return -3;
  const long sl = (long)N * (N + 2);
  for (int p = 0; p < n; p++) {
    if (weights[p] == 0) continue;   /* insert_slice returns -1 (libEM/reconstructor.cpp:1090) */
    for (int s = 0; s < nsym; s++) or_compose(arg + 9 * p, sym + 9 * s, t3d + 9 * s);
    int rc = or_insert_slice(vol_data, vol_norm, N, mode, slices + sl * p, t3d, nsym, weights[p], corners, NULL, 0);
    if (rc) { free(t3d); return rc; }
  }
  free(t3d);
  return 0;
}

/* ReconstructorVolumeData::normalize_threed (libEM/reconstructor.cpp:315-390),
 * full-volume case; wiener adds 1 to each nonzero denominator (:376-390). */
OR_EXPORT void or_normalize_nz(acc_t *rdata, acc_t *norm, int N, int NZ, int sqrtnorm,
                               int wiener) {
  const int nx = N + 2, ny = N, nz = NZ;
  const long nnx = nx / 2, nnxy = (long)ny * nnx;
  for (int z = -nz / 2; z < nz / 2; z++) {
    for (int y = 0; y <= ny / 2; y++) {
      if (z <= 0 && (y == 0 || y == ny / 2)) continue;
      long idx1 = (long)(y == 0 ? 0 : ny - y) * nnx + (long)(z <= 0 ? -z : nz - z) * nnxy;
      long idx2 = (long)y * nnx + (long)(z < 0 ? nz + z : z) * nnxy;
      if (idx1 == idx2) continue;
      acc_t snorm = norm[idx1] + norm[idx2];
      norm[idx1] = norm[idx2] = snorm;
      idx1 += nnx - 1;
      idx2 += nnx - 1;
      snorm = norm[idx1] + norm[idx2];
      norm[idx1] = norm[idx2] = snorm;
    }
  }
  norm[0 + 0 * nnx + (nz / 2) * nnxy] *= 2;
  norm[0 + (ny / 2) * nnx + 0 * nnxy] *= 2;
  norm[0 + (ny / 2) * nnx + (nz / 2) * nnxy] *= 2;
  norm[nx / 2 - 1 + 0 * nnx + (nz / 2) * nnxy] *= 2;
  norm[nx / 2 - 1 + (ny / 2) * nnx + 0 * nnxy] *= 2;
  const long total = (long)nx * ny * nz;
  for (long i = 0; i < total; i += 2) {
    acc_t d = norm[i / 2];
    if (sqrtnorm) d = (sizeof(acc_t) == sizeof(float)) ? (acc_t)sqrtf((float)d) : (acc_t)sqrt((double)d);
    if (d == 0) { rdata[i] = 0; rdata[i + 1] = 0; }
    else {
      const acc_t dd = d + (acc_t)(wiener ? 1.0f : 0.0f);
      rdata[i] /= dd;
      rdata[i + 1] /= dd;
    }
  }
}

OR_EXPORT void or_normalize_w(acc_t *rdata, acc_t *norm, int N, int sqrtnorm, int wiener) {
  or_normalize_nz(rdata, norm, N, N, sqrtnorm, wiener);
}

OR_EXPORT void or_normalize(acc_t *rdata, acc_t *norm, int N, int sqrtnorm) {
  or_normalize_w(rdata, norm, N, sqrtnorm, 0);
}

/* FourierReconstructor::pixel_at (libEM/reconstructor.cpp:1448-1462) with
 * EMData::get_complex_at(x,y,z) (libEM/emdata_core.cpp:134-145) and
 * get_complex_index_fast (libEM/emdata_core.h:302-308). */
static inline void or_pixel_at(const acc_t *rdata, const acc_t *norm, int N, real xx, real yy, real zz, real *dt) {
  const int nx = N + 2, ny = N, nz = N;
  const long nxy = (long)nx * ny;
  int x0 = or_round(xx), y0 = or_round(yy), z0 = or_round(zz);
  real vre, vim;
  if (abs(x0) >= nx / 2 || abs(y0) > ny / 2 || abs(z0) > nz / 2) { vre = 0; vim = 0; }
  else if (x0 < 0) {
    long idx = (long)(-x0 * 2) + (long)(y0 <= 0 ? -y0 : ny - y0) * nx + (long)(z0 <= 0 ? -z0 : nz - z0) * nxy;
    vre = rdata[idx]; vim = -rdata[idx + 1];
  } else {
    long idx = (long)x0 * 2 + (long)(y0 < 0 ? ny + y0 : y0) * nx + (long)(z0 < 0 ? nz + z0 : z0) * nxy;
    vre = rdata[idx]; vim = rdata[idx + 1];
  }
  long cidx;
  if (x0 < 0) cidx = (long)x0 * -2 + (long)(y0 <= 0 ? -y0 : ny - y0) * nx + (long)(z0 <= 0 ? -z0 : nz - z0) * nxy;
  else cidx = (long)x0 * 2 + (long)(y0 < 0 ? ny + y0 : y0) * nx + (long)(z0 < 0 ? nz + z0 : z0) * nxy;
  real nv = norm[cidx / 2];
  dt[0] = vre / nv;
  dt[1] = vim / nv;
  dt[2] = nv;
}

/* FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1445),
 * Fourier-space part, into out[N][N+2] (zeroed here): each pixel x in
 * [0, N/2+1], y in [-N/2, N/2) rotated (transpose multiply, float), the
 * nearest voxel's value over its weight, skipped where the weight is below
 * 0.005, the x = 0 column halved off rows 0 and -N/2, written with the 2-D
 * EMData::set_complex_at (libEM/emdata_core.cpp:171-206); then the
 * translation (tx, ty) applied by the xform processor's 2-D complex branch
 * (libEM/processor.cpp:11082-11178, a rotation-free transform: each value
 * copied and rotated by its phase, the phase formed in long double --
 * the processor's pi, libEM/sparx/emconstants.h:38 -- and rounded to
 * float, cos/sin and the products in double). */
static void or_set_complex_2d(float *d, int nx, int ny, int x, int y, float re, float im) {
  if (abs(x) >= nx / 2 || abs(y) > ny / 2) return;
  if (x == 0 || x == nx / 2 - 1) {
    const int c = x == 0 ? 0 : nx - 2;
    if (y == 0) { d[c] = re; d[c + 1] = 0; }
    else if (y == ny / 2 || y == -ny / 2) { d[ny / 2 * nx + c] = re; d[ny / 2 * nx + c + 1] = 0; }
    else if (y > 0) {
      d[y * nx + c] = d[(ny - y) * nx + c] = re;
      d[y * nx + c + 1] = im;
      d[(ny - y) * nx + c + 1] = -im;
    } else {
      d[(ny + y) * nx + c] = d[-y * nx + c] = re;
      d[(ny + y) * nx + c + 1] = im;
      d[-y * nx + c + 1] = -im;
    }
    return;
  }
  if (y >= 0) { d[x * 2 + y * nx] = re; d[x * 2 + y * nx + 1] = im; }
  else { d[x * 2 + (ny + y) * nx] = re; d[x * 2 + (ny + y) * nx + 1] = im; }
}

OR_EXPORT void or_projection(const acc_t *rdata, const acc_t *norm, int N, const float *rot,
                             float tx, float ty, float *out) {
  const int nx = N + 2, ny = N, nz = N;
  memset(out, 0, sizeof(float) * (size_t)nx * ny);
  for (int y = -ny / 2; y < ny / 2; y++) {
    for (int x = 0; x <= nx / 2; x++) {
      const float rx = (float)x / (nx - 2);
      const float ry = (float)y / ny;
      float xx = rx * rot[0] + ry * rot[3];
      float yy = rx * rot[1] + ry * rot[4];
      float zz = rx * rot[2] + ry * rot[5];
      if (fabsf(xx) > 0.5f || fabsf(yy) >= 0.5f || fabsf(zz) >= 0.5f) continue;
      xx = xx * (nx - 2);
      yy = yy * ny;
      zz = zz * nz;
      real dt[3];
      or_pixel_at(rdata, norm, N, xx, yy, zz, dt);
      if (dt[2] < 0.005) continue;
      float d0 = (float)dt[0], d1 = (float)dt[1];
      if ((x == 0 || x == nx / 2) && (y != 0 && y != -ny / 2)) { d0 /= 2; d1 /= 2; }
      or_set_complex_2d(out, nx, ny, x, y, d0, d1);
    }
  }
  const long double pi = 3.141592653589793238462643383279502884197L;
  for (int kyN = 0; kyN < ny; kyN++) {
    const int kyNew = kyN >= nx / 2 ? kyN - ny : kyN;
    const float phaseY = (float)(-2 * pi * kyNew * ty / ny);
    for (int kx = 0; kx < nx / 2; kx++) {
      const float phase = (float)(phaseY - 2 * pi * kx * tx / ny);
      const float r = out[2 * kx + nx * kyN], i = out[2 * kx + 1 + nx * kyN];
      out[2 * kx + nx * kyN] = (float)((double)r * cos((double)phase) - (double)i * sin((double)phase));
      out[2 * kx + 1 + nx * kyN] = (float)((double)r * sin((double)phase) + (double)i * cos((double)phase));
    }
  }
}

/* FourierReconstructor::do_compare_slice_work (libEM/reconstructor.cpp:1259-1381),
 * CPU branch.  out[0..4] = reconstruct_norm, reconstruct_absqual,
 * reconstruct_absqual_lowres, reconstruct_qual, reconstruct_weight.
 * The loop reads one column past Nyquist (x = N/2+1), i.e. the first element
 * of the next row; on the last row that is past the end of the slice buffer
 * in the reference, and reads 0 here. */
OR_EXPORT void or_compare_slice(const acc_t *rdata, const acc_t *norm, int N, const float *slice,
                                const float *t3d, int nsym, float weight, float apix, float *out) {
  const int nx = N + 2, ny = N, nz = N;
  const float inx = (float)(N + 2), iny = (float)N;
  const long slice_len = (long)(N + 2) * N;
  float rmax = (float)(iny * apix / 12.0);
  if (rmax > iny / 2.0 - 1.0) rmax = (float)(iny / 2.0 - 1.0);
  if (rmax < 5.0) rmax = 5.0f;
  double dotlow = 0, dlpow = 0, dlpow2 = 0, dot = 0, vweight = 0, power = 0, power2 = 0;
  int nval = 0;
  for (int s = 0; s < nsym; s++) {
    const float *M = t3d + 9 * s;
    for (int y = (int)(-iny / 2); y < iny / 2; y++) {
      for (int x = 0; x <= inx / 2; x++) {
        if (x == 0 && y == 0) continue;
        real rx, ry;
        if (IS_F32) { rx = (real)((float)x / (inx - 2)); ry = (real)((float)y / iny); }
        else { rx = (real)x / (real)(inx - 2); ry = (real)y / (real)iny; }
        real xx = rx * (real)M[0] + ry * (real)M[3];
        real yy = rx * (real)M[1] + ry * (real)M[4];
        real zz = rx * (real)M[2] + ry * (real)M[5];
        if (fabs((double)xx) > 0.5 || fabs((double)yy) >= 0.5 || fabs((double)zz) >= 0.5) continue;
        xx = xx * (real)(nx - 2);
        yy = yy * (real)ny;
        zz = zz * (real)nz;
        long idx = (long)(x * 2 + inx * (y < 0 ? iny + y : y));
        real d2r = idx < slice_len ? (real)slice[idx] : 0;
        real d2i = idx + 1 < slice_len ? (real)slice[idx + 1] : 0;
        real dt[3];
        or_pixel_at(rdata, norm, N, xx, yy, zz, dt);
        if (dt[2] == 0) continue;
        float r = or_hypot_fast(x, y);
        real pdot = (dt[0] * d2r + dt[1] * d2i) * dt[2];
        real pv = (dt[0] * dt[0] + dt[1] * dt[1]) * dt[2];
        real pi2 = (d2r * d2r + d2i * d2i) * dt[2];
        if (r > 3 && r < rmax) { dotlow += pdot; dlpow += pv; dlpow2 += pi2; }
        vweight += dt[2];
        dot += pdot;
        power += pv;
        power2 += pi2;
        nval++;
      }
    }
  }
  dot /= sqrt(power * power2);
  if (dlpow * dlpow2 > 0) dotlow /= sqrt(dlpow * dlpow2);
  out[0] = (float)(power2 <= 0 ? 1.0 : sqrt(power / power2));
  out[1] = (float)dot;
  out[2] = (float)dotlow;
  float rw = weight <= 0 ? 1.0f : 1.0f / weight;
  out[3] = (float)(dot * rw / ((rw - 1.0) * dot + 1.0));
  out[4] = (float)(vweight / (float)nval);
}

/* ----------------------------------------------------------- prologue */

/* EMData::get_edge_mean, 2-D branch (libEM/emdata_metadata.cpp:713-735). */
OR_EXPORT float or_edge_mean(const float *d, int nx, int ny) {
  double edge_sum = 0;
  long nxy = (long)nx * ny;
  for (long i = 0, j = (long)(ny - 1) * nx; i < nx; ++i, ++j) edge_sum += d[i] + d[j];
  for (long i = 0, j = nx - 1; i < nxy; i += nx, j += nx) edge_sum += d[i] + d[j];
  return (float)edge_sum / (nx * 2 + ny * 2);
}

/* CTF_SIGN image of EMAN2Ctf::compute_2d_complex (libEM/ctf.cpp:964-1000,
 * 1076-1090), lambda (libEM/ctf.h:290-294), df (libEM/ctf.h:300-303),
 * get_phase (libEM/ctf.cpp:671-675).  Writes sign[N][N/2+1] (+1/-1). */
OR_EXPORT void or_ctf_sign(float *sign, int N, float defocus, float dfdiff, float dfang,
                           float voltage, float cs, float apix, float ampcont) {
  const int nx = N + 2, ny = N;
  float ds = 1.0f / (apix * ny);
  float lam = 12.2639f / sqrtf(voltage * 1000.0f + 0.97845f * voltage * voltage);
  float g1 = (float)(M_PI / 2.0 * cs * 1.0e7 * powf(lam, 3.0f));
  float g2 = (float)(M_PI * lam * 10000.0);
  float phase;
  if (ampcont > -100.0 && ampcont <= 100.0) phase = (float)asin(ampcont / 100.0);
  else if (ampcont > 100.0) phase = (float)(M_PI - asin(2.0f - ampcont / 100.0));
  else phase = (float)(-M_PI - asin(-2.0 - ampcont / 100.0));
  float acac = (float)(M_PI / 2.0 - phase);
  for (int y = -ny / 2; y < ny / 2; y++) {
    int y2 = (y + ny) % ny;
    for (int x = 0; x < nx / 2; x++) {
      float s = or_hypot_fast(x, y) * ds;
      float gam;
      if (dfdiff == 0) gam = -g1 * s * s * s * s + g2 * defocus * s * s;
      else {
        float ang = atan2f((float)y, (float)x);
        float df = (float)(defocus + dfdiff / 2.0f * cos(2.0f * ang - 2.0f * M_PI / 180.0f * dfang));
        gam = -g1 * s * s * s * s + g2 * df * s * s;
      }
      float v = cosf(gam - acac);
      sign[y2 * (nx / 2) + x] = v < 0 ? -1.0f : 1.0f;
    }
  }
}

/* TransformProcessor::transform, 2-D real branch (libEM/processor.cpp:11025-11080)
 * for a translation-only transform whose inverse translates by (tx,ty):
 * soln = inv*coord = (1*x + 0*y + tx, 0*x + 1*y + ty), then + (nx/2, ny/2);
 * bilinear interpolation (libEM/util.h:543-547). */
OR_EXPORT void or_translate_bilinear(const float *src, float *dst, int nx, int ny, float tx, float ty) {
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      float cx = (float)(i - nx / 2), cy = (float)(j - ny / 2);
      float sx = 1.0f * cx + 0.0f * cy;
      sx = sx + tx;
      float sy = 0.0f * cx + 1.0f * cy;
      sy = sy + ty;
      float x2 = sx + (float)(nx / 2);
      float y2 = sy + (float)(ny / 2);
      if (x2 < 0 || x2 >= nx || y2 < 0 || y2 >= ny) { dst[i + j * nx] = 0; continue; }
      int ii = (int)x2, jj = (int)y2;
      int k0 = ii + jj * nx, k1 = k0 + 1, k2 = k0 + nx, k3 = k0 + nx + 1;
      if (ii == nx - 1) { k1--; k3--; }
      if (jj == ny - 1) { k2 -= nx; k3 -= nx; }
      float t = x2 - ii, u = y2 - jj;
      float p1 = src[k0], p2 = src[k1], p3 = src[k2], p4 = src[k3];
      float a = (1 - t) * (1 - u) * p1;
      a = a + t * (1 - u) * p2;
      a = a + (1 - t) * u * p3;
      a = a + t * u * p4;
      dst[i + j * nx] = a;
    }
  }
}

/* math.gausskernelfix (MaskGaussInvProcessor, libEM/processor.h:4131-4176,
 * through CoordinateProcessor::process_inplace, libEM/processor.cpp:2439-2473):
 * centre (floor(nx/2), floor(ny/2), floor(nz/2)), slice_value =
 * gauss_width / (ny*ny) in float, dist the float squared distance formed as
 * CircularMaskProcessor::process_pixel does (libEM/processor.h:3785-3789),
 * and the voxel divided by exp(-dist*slice_value) in double. */
OR_EXPORT void or_kernel_fix(float *vol, int nx, int ny, int nz, float gauss_width) {
  const float xc = floorf(nx / 2.0f), yc = floorf(ny / 2.0f), zc = floorf(nz / 2.0f);
  const float sv = gauss_width / (float)(ny * ny);
  size_t i = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++, i++) {
        const float dx = (float)x - xc, dy = (float)y - yc, dz = (float)z - zc;
        const float dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
        const float dist = (dxx + dyy) + dzz;
        const float f = -dist * sv;
        vol[i] = (float)((double)vol[i] / exp((double)f));
      }
}

OR_EXPORT int or_real_size(void) { return (int)sizeof(real); }
OR_EXPORT int or_acc_size(void) { return (int)sizeof(acc_t); }
OR_EXPORT float or_fast_exp_value(float f) { or_init_tables(); return (float)or_fast_exp((real)f); }
OR_EXPORT int or_hypot_int(int x, int y) { return or_hypot_fast_int(x, y); }

#ifdef _OPENMP
#include <omp.h>
/* Timed CPU baseline: the same restatement over many particles with one
 * private (complex, weight) accumulator pair per thread, merged at the end by
 * plain addition of the un-normalised accumulators, as the reference's own
 * parallel make3d merges per-task volumes (programs/e2spa_make3d.py:175-188).
 * The reference's shared-volume threading races on the += and is not used. */
OR_EXPORT int or_insert_batch_omp(acc_t *vol_data, acc_t *vol_norm, int N, int mode,
                                  const float *slices, int n, const float *arg,
                                  const float *sym, int nsym, const float *weights, int nthreads) {
  if (nthreads < 1) nthreads = omp_get_max_threads();
  const long vd = (long)N * N * (N + 2), vn = (long)N * N * (N / 2 + 1);
  const long sl = (long)N * (N + 2);
  int rc_all = 0;
  or_init_tables();
#pragma omp parallel num_threads(nthreads)
  {
    int tid = omp_get_thread_num(), nt = omp_get_num_threads();
    acc_t *pd = (tid == 0) ? vol_data : (acc_t *)calloc(vd, sizeof(acc_t));
    acc_t *pn = (tid == 0) ? vol_norm : (acc_t *)calloc(vn, sizeof(acc_t));
    float *t3d = (float *)malloc(sizeof(float) * 9 * nsym);
    if (!pd || !pn || !t3d) {
#pragma omp atomic write
      rc_all = -3;
    } else {
      for (int p = tid; p < n; p += nt) {
        if (weights[p] == 0) continue;
        for (int s = 0; s < nsym; s++) or_compose(arg + 9 * p, sym + 9 * s, t3d + 9 * s);
        or_insert_slice(pd, pn, N, mode, slices + sl * p, t3d, nsym, weights[p], 0, NULL, 0);
      }
    }
#pragma omp barrier
    if (tid != 0 && pd && pn) {
#pragma omp critical
      {
        for (long i = 0; i < vd; i++) vol_data[i] += pd[i];
        for (long i = 0; i < vn; i++) vol_norm[i] += pn[i];
      }
    }
    if (tid != 0) { free(pd); free(pn); }
    free(t3d);
  }
  return rc_all;
}
#endif

/* Per-pixel entry with the same contract as the reference inserter driver in
 * ref_driver.cpp: n calls of insert_pixel with px[n*6] =
 * (xx, yy, zz, re, im, weight).  Used only to pin this restatement. */
OR_EXPORT int or_insert_pixels(int mode, acc_t *data, acc_t *norm, int N, const float *px, long n) {
  or_init_tables();
  or_vol v;
  v.data = data; v.norm = norm;
  v.nx = N + 2; v.ny = N; v.nz = N;
  v.nxyz = (long)v.nx * v.ny * v.nz;
  for (long i = 0; i < n; i++) {
    const float *p = px + 6 * i;
    switch (mode) {
      case MODE_NEAREST: or_insert_nearest(&v, p[0], p[1], p[2], p[3], p[4], p[5]); break;
      case MODE_GAUSS2: or_insert_gauss2(&v, p[0], p[1], p[2], p[3], p[4], p[5]); break;
      case MODE_GAUSS5: or_insert_gauss5(&v, p[0], p[1], p[2], p[3], p[4], p[5]); break;
      case MODE_TRILINEAR: or_insert_trilinear(&v, p[0], p[1], p[2], p[3], p[4], p[5]); break;
      default: return -2;
    }
  }
  return 0;
}
