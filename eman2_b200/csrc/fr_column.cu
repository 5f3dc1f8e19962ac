// fr_column.cu -- the column-owner insertion kernel (gather schedule, v2).
//
// Work item = (job, 16^3 voxel tile, block of slices).  For each slice of the
// block whose plane passes the tile, the slice's pixel patch is staged in
// shared memory; then each of the 256 threads owns one voxel column of the
// tile along the axis a on which the slice's plane normal is largest, walks
// the pixels whose window covers its column (b, c), and adds each pixel's taps
// along a to the tile accumulators in shared memory.  A voxel is touched by
// one thread per slice, so the accumulation needs no atomics; the tile's
// partial sums go to the volume once per work item.  The tap arithmetic is
// the reference's (fr_device.cuh): window starts, exp-table indices and
// Hermitian placement are bit-exact; only the summation order differs.
//
// Reference: do_insert_slice_work (libEM/reconstructor.cpp:1122-1210),
// insert_pixel (libEM/reconstructor_tools.cpp:113-189, 315-376),
// add_complex_at_fast (libEM/emdata_core.h:368-410).
#include <algorithm>
#include <cmath>

#include "fr_device.cuh"
#include "fr_internal.h"

namespace fr {

namespace col {

constexpr int T = 16;          // tile edge
constexpr int NT = 256;        // threads: one per column
constexpr int NV = T * T * T;  // voxels per tile
constexpr int PIXCAP = 1024;   // staged pixels per patch chunk (rows are chunked to fit)
constexpr int STEPCAP = 1360;  // step-table entries held in shared memory
constexpr float kDel = 0.02f;  // slack on the approximate plane geometry
constexpr float kPlaneTol = 0.05f;

template <int MODE> struct Win;
template <> struct Win<MODE_GAUSS5> { static constexpr float lo = 2.5f, hi = 3.5f; static constexpr int K = 6; };
template <> struct Win<MODE_GAUSS2> { static constexpr float lo = 1.0f, hi = 1.0f; static constexpr int K = 2; };
template <> struct Win<MODE_TRILINEAR> { static constexpr float lo = 1.0f, hi = 1.0f; static constexpr int K = 2; };
template <> struct Win<MODE_NEAREST> { static constexpr float lo = 0.5f, hi = 0.5f; static constexpr int K = 1; };

// Exact window membership of tap coordinate t for pixel coordinate p.
template <int MODE> __device__ __forceinline__ bool in_win(int t, float p) {
  const float tf = (float)t;
  if (MODE == MODE_GAUSS5) return __fadd_rn(tf, -2.5f) <= p && p < __fadd_rn(tf, 3.5f);
  if (MODE == MODE_NEAREST) {
    const float s = __fadd_rn(p, 0.5f);
    return tf <= s && s < __fadd_rn(tf, 1.0f);
  }
  return __fadd_rn(tf, -1.0f) <= p && p < __fadd_rn(tf, 1.0f);
}

// First tap coordinate of a pixel's window along one axis (exact).
template <int MODE> __device__ __forceinline__ int win_start(float p) {
  if (MODE == MODE_GAUSS5) return floor_minus_2p5(p);
  if (MODE == MODE_NEAREST) return (int)floorf(__fadd_rn(p, 0.5f));
  return (int)floorf(p);
}

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

__device__ __forceinline__ float comp(const float4 &v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// fast_exp(-r*h) through the exact step table (see ExpSteps): one exact bin
// (K is a power of two, so r*K is exact), one compare.  Past the table the
// reference calls exp(f) with f = -r*h in float.
__device__ __forceinline__ float step_exp(float r, float h, const ExpSteps &st,
                                          const float4 *__restrict__ bins) {
  if (r >= st.rout) return expf(__fmul_rn(-r, h));
  const int b = (int)floorf(__fmul_rn(r, st.K));
  const float4 e = bins[b];
  return r >= e.x ? e.z : e.y;
}

struct Smem {
  float4 *acc;      // [NV] (re, im, w, origin-touched)
  float4 *steps;    // [STEPCAP] fast_exp step table of the current mode
  float4 *pt;       // [PIXCAP] (xx, yy, zz, re)
  float *pim;       // [PIXCAP] im
  int *hits;        // [block]
  int *wcount;      // [8]
  int *steps_mode;  // mode whose table is loaded
};

// One pass (direct or conjugate targets) of one slice for the thread's column.
// A: column axis (compile time); sg: +1 direct, -1 conjugate.
template <int MODE, int A>
__device__ __forceinline__ void column_pass(const Smem &S, const float *m0, const float *m1, int sg,
                                            const int *base, const int *ext, int px0, int py0,
                                            int PW, int PH, float w, float h,
                                            const ExpSteps &steps) {
  constexpr int B = (A == 0) ? 1 : 0;
  constexpr int C = (A == 2) ? 1 : 2;
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  constexpr int K = Win<MODE>::K;
  const int lb = threadIdx.x & 15, lc = threadIdx.x >> 4;
  // voxel column (v_b, v_c); inactive past the clipped tile edge
  const int vb = base[B] + lb, vc = base[C] + lc;
  if (vb > ext[B] || vc > ext[C]) return;
  const int tb = sg * vb, tc = sg * vc;
  const int ta_lo = sg > 0 ? base[A] : -ext[A];
  const int ta_hi = sg > 0 ? ext[A] : -base[A];
  // constraint boxes on the pixel point p (approximate geometry, padded)
  float lo[3], hi[3];
  // a pixel's window covers t_a iff t_a - RLO <= p_a < t_a + RHI
  lo[A] = ta_lo - RLO - kDel; hi[A] = ta_hi + RHI + kDel;
  lo[B] = tb - RLO - kDel;    hi[B] = tb + RHI + kDel;
  lo[C] = tc - RLO - kDel;    hi[C] = tc + RHI + kDel;
  // rows: y over the (b, c) parallelogram, p ~ x*m0 + y*m1
  const float det = m0[B] * m1[C] - m0[C] * m1[B];
  if (fabsf(det) < 0.5f) return;   // |n_a| >= 1/sqrt(3) by the choice of a
  const float idet = 1.0f / det;
  float ymin = 1e30f, ymax = -1e30f;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float pb = (i & 1) ? hi[B] : lo[B], pc = (i & 2) ? hi[C] : lo[C];
    const float y = (m0[B] * pc - m0[C] * pb) * idet;
    ymin = fminf(ymin, y);
    ymax = fmaxf(ymax, y);
  }
  const int r0 = max(py0, (int)ceilf(ymin)), r1 = min(py0 + PH - 1, (int)floorf(ymax));
  float inv0[3];
#pragma unroll
  for (int a = 0; a < 3; a++) inv0[a] = fabsf(m0[a]) > 1e-4f ? 1.0f / m0[a] : 0.0f;
  // accumulator addressing: voxel v = sg * t, local l = v - base
  const int la_off = (sg > 0 ? -base[A] : -base[A]);
  const int str[3] = {1, T, T * T};
  const int col_addr = (vb - base[B]) * str[B] + (vc - base[C]) * str[C];
  const bool xzero_col = (A != 0) && (((B == 0) ? vb : vc) == 0);   // column in the x=0 plane
  for (int y = r0; y <= r1; y++) {
    float xlo = (float)px0, xhi = (float)(px0 + PW - 1);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float c = m1[a] * (float)y;
      const float L = lo[a] - c, U = hi[a] - c;
      if (inv0[a] > 0.f) { xlo = fmaxf(xlo, L * inv0[a]); xhi = fminf(xhi, U * inv0[a]); }
      else if (inv0[a] < 0.f) { xlo = fmaxf(xlo, U * inv0[a]); xhi = fminf(xhi, L * inv0[a]); }
      else if (L > 0.05f || U < -0.05f) xhi = -1e30f;
    }
    const int c0 = max(px0, (int)ceilf(xlo)), c1 = min(px0 + PW - 1, (int)floorf(xhi));
    const int rowoff = (y - py0) * PW - px0;
    for (int x = c0; x <= c1; x++) {
      const float4 pt = S.pt[rowoff + x];
      const float pa = comp(pt, A), pb = comp(pt, B), pc = comp(pt, C);
      if (!(in_win<MODE>(tb, pb) && in_win<MODE>(tc, pc))) continue;
      const int a0 = win_start<MODE>(pa);
      if (a0 + K - 1 < ta_lo || a0 > ta_hi) continue;
      const float pim = S.pim[rowoff + x];
      const float re = pt.w;
      // fixed parts of the distance, kept in the reference's order
      // ((dx^2 + dy^2) + dz^2) (libEM/util.h:816-819)
      float f0 = 0.f, f1 = 0.f;
      if (MODE == MODE_GAUSS2 || MODE == MODE_GAUSS5) {
        if (A == 0) {
          const float dy = __fsub_rn((float)tb, pt.y), dz = __fsub_rn((float)tc, pt.z);
          f0 = __fmul_rn(dy, dy);
          f1 = __fmul_rn(dz, dz);
        } else if (A == 1) {
          const float dx = __fsub_rn((float)tb, pt.x), dz = __fsub_rn((float)tc, pt.z);
          f0 = __fmul_rn(dx, dx);
          f1 = __fmul_rn(dz, dz);
        } else {
          const float dx = __fsub_rn((float)tb, pt.x), dy = __fsub_rn((float)tc, pt.y);
          f0 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        }
      }
#pragma unroll
      for (int kk = 0; kk < K; kk++) {
        const int k = a0 + kk;
        if (k < ta_lo || k > ta_hi) continue;
        float vre, vim, vw;
        if (MODE == MODE_GAUSS2 || MODE == MODE_GAUSS5) {
          const float d = __fsub_rn((float)k, pa);
          const float d2 = __fmul_rn(d, d);
          float r;
          if (A == 0) r = __fadd_rn(__fadd_rn(d2, f0), f1);
          else if (A == 1) r = __fadd_rn(__fadd_rn(f0, d2), f1);
          else r = __fadd_rn(f0, d2);
          if (MODE == MODE_GAUSS2) {
            const float gg = __fmul_rn(step_exp(r, h, steps, S.steps), w);
            vre = __fmul_rn(re, gg);
            vim = __fmul_rn(pim, gg);
            vw = gg;
          } else {
            const float gg = step_exp(r, h, steps, S.steps);
            vre = __fmul_rn(__fmul_rn(re, gg), w);
            vim = __fmul_rn(__fmul_rn(pim, gg), w);
            vw = __fmul_rn(gg, w);
          }
        } else {
          int t[3];
          t[A] = k; t[B] = tb; t[C] = tc;
          tap_value<MODE>(t[0], t[1], t[2], pt.x, pt.y, pt.z, re, pim, w, h, nullptr, vre, vim, vw);
        }
        const int la = sg * k + la_off;
        float4 *cell = &S.acc[col_addr + la * str[A]];
        float4 v = *cell;
        const bool origin = (k == 0 && tb == 0 && tc == 0);
        if (sg > 0) {
          // direct add; the origin keeps only its real part and is marked
          v.x += vre;
          if (origin) v.w = 1.0f;
          else v.y += vim;
          v.z += vw;
        } else {
          if (origin) continue;   // the origin adds no conjugate
          v.x += vre;
          v.y -= vim;
          const bool xzero = (A == 0) ? (k == 0) : xzero_col;
          if (!xzero) v.z += vw;   // x=0 conjugates carry no weight
        }
        *cell = v;
      }
    }
  }
}

template <int MODE>
__device__ void tile_item(const InsertJob &J, int tile, int s0, int s1, const Smem &S, int side,
                          float h, const ExpSteps &steps, int *err) {
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  const int N = J.N, n2 = N >> 1, w2 = n2 + 1;
  const float Nf = (float)N;
  const int tix = tile % J.tiles_x, tiy = (tile / J.tiles_x) % J.tiles_y,
            tiz = tile / (J.tiles_x * J.tiles_y);
  const int base[3] = {tix * T, -n2 + 1 + tiy * T, -n2 + 1 + tiz * T};
  const int ext[3] = {min(base[0] + T - 1, n2 - 1), min(base[1] + T - 1, n2 - 1),
                      min(base[2] + T - 1, n2 - 1)};
  // ---- cull the block's slices against the tile box (grown by the reach)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int nhit = 0;
  for (int r = s0; r < s1; r += NT) {
    const int s = r + threadIdx.x;
    bool hit = false;
    if (s < s1 && __ldg(&J.pw[s / J.nsym]) != 0.0f) {
      const float n[3] = {__ldg(&J.t3d[9 * s + 6]), __ldg(&J.t3d[9 * s + 7]), __ldg(&J.t3d[9 * s + 8])};
      // A pixel's direct taps reach the tile from [base - RLO, ext + RHI];
      // its conjugate taps (mirrored) from [base - RHI, ext + RLO].  The
      // plane passes through the origin, so one test against the union box
      // covers both passes (gauss_5's window is asymmetric: 2.5 / 3.5).
      constexpr float RC = (RLO > RHI ? RLO : RHI) + kDel;
      const float lo[3] = {base[0] - RC, base[1] - RC, base[2] - RC};
      const float hi[3] = {ext[0] + RC, ext[1] + RC, ext[2] + RC};
      float mn, mx;
      box_dot(n, lo, hi, mn, mx);
      hit = mn <= kPlaneTol && mx >= -kPlaneTol;
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) S.wcount[warp] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < NT / 32; i++) {
      const int c = S.wcount[i];
      off += (i < warp) ? c : 0;
      tot += c;
    }
    if (hit) S.hits[nhit + off + __popc(b & ((1u << lane) - 1u))] = s;
    nhit += tot;
    __syncthreads();
  }
  if (nhit == 0) return;
  // ---- this mode's exp step table into shared memory (if not there yet)
  if ((MODE == MODE_GAUSS2 || MODE == MODE_GAUSS5) && *S.steps_mode != MODE) {
    const int nb = min(steps.nbins, STEPCAP);
    for (int i = threadIdx.x; i < nb; i += NT) S.steps[i] = __ldg(&steps.d_bins[i]);
    if (threadIdx.x == 0 && steps.nbins > STEPCAP) atomicOr(err, 8);
  }
  // ---- zero the tile accumulators
  for (int i = threadIdx.x; i < NV; i += NT) S.acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  if (threadIdx.x == 0) *S.steps_mode = MODE;
  for (int hI = 0; hI < nhit; hI++) {
    const int s = S.hits[hI];
    const int p = s / J.nsym;
    float M[9];
#pragma unroll
    for (int i = 0; i < 9; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
    const float *m0 = M, *m1 = M + 3, *nrm = M + 6;
    const float w = __ldg(&J.pw[p]);
    const float2 *sl = J.slices + (size_t)p * N * w2;
    const float an0 = fabsf(nrm[0]), an1 = fabsf(nrm[1]), an2 = fabsf(nrm[2]);
    const int A = (an0 >= an1 && an0 >= an2) ? 0 : (an1 >= an2 ? 1 : 2);
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {
      const int sg = pass ? -1 : 1;
      float lo[3], hi[3];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        lo[a] = (pass ? -ext[a] : base[a]) - RLO - kDel;
        hi[a] = (pass ? -base[a] : ext[a]) + RHI + kDel;
      }
      float xl, xh, yl, yh;
      box_dot(m0, lo, hi, xl, xh);
      box_dot(m1, lo, hi, yl, yh);
      const int px0 = max(0, (int)floorf(xl) - 1), px1 = min(n2, (int)ceilf(xh) + 1);
      const int py0 = max(-n2, (int)floorf(yl) - 1), py1 = min(n2 - 1, (int)ceilf(yh) + 1);
      if (px0 > px1 || py0 > py1) continue;
      const int PW = px1 - px0 + 1;
      if (PW > side) {   // cannot happen for an orthonormal block; stay in bounds
        if (threadIdx.x == 0) atomicOr(err, 2);
        continue;
      }
      const int rows_per = PIXCAP / PW;
      // patches larger than the staging buffer go through in row chunks: the
      // column work of one pixel row does not depend on any other row
      for (int ry0 = py0; ry0 <= py1; ry0 += rows_per) {
        const int PH = min(rows_per, py1 - ry0 + 1);
        __syncthreads();
        for (int i = threadIdx.x; i < PW * PH; i += NT) {
          const int x = px0 + i % PW, y = ry0 + i / PW;
          float4 pt;
          float pim = 0.f;
          if (x > __ldg(&J.xmax[y + n2])) {
            pt = make_float4(1e30f, 1e30f, 1e30f, 0.f);
          } else {
            pixel_coords(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, Nf, pt.x, pt.y, pt.z);
            const float2 v = slice_value_cg(sl, N, x, y);
            pt.w = v.x;
            pim = v.y;
          }
          S.pt[i] = pt;
          S.pim[i] = pim;
        }
        __syncthreads();
        switch (A) {
          case 0: column_pass<MODE, 0>(S, m0, m1, sg, base, ext, px0, ry0, PW, PH, w, h, steps); break;
          case 1: column_pass<MODE, 1>(S, m0, m1, sg, base, ext, px0, ry0, PW, PH, w, h, steps); break;
          default: column_pass<MODE, 2>(S, m0, m1, sg, base, ext, px0, ry0, PW, PH, w, h, steps); break;
        }
      }
    }
  }
  __syncthreads();
  // ---- flush the tile's partial sums into the volume
  const size_t nxf = (size_t)N + 2;
  for (int i = threadIdx.x; i < NV; i += NT) {
    const float4 v = S.acc[i];
    if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
    const int vx = base[0] + (i & 15), vy = base[1] + ((i >> 4) & 15), vz = base[2] + (i >> 8);
    if (vx > ext[0] || vy > ext[1] || vz > ext[2]) continue;
    const size_t row = (size_t)(vy < 0 ? N + vy : vy);
    const size_t slab = (size_t)(vz < 0 ? N + vz : vz);
    const size_t di = (size_t)vx * 2 + row * nxf + slab * nxf * (size_t)N;
    const size_t ni = (size_t)vx + row * (size_t)w2 + slab * (size_t)w2 * (size_t)N;
    if (v.w != 0.f) {               // the origin: real part only, imaginary part := 0
      atomicAdd(&J.data[di], v.x);
      J.data[di + 1] = 0.0f;
    } else {
      atomicAdd(reinterpret_cast<float2 *>(&J.data[di]), make_float2(v.x, v.y));
    }
    if (v.z != 0.f) atomicAdd(&J.norm[ni], v.z);
  }
  __syncthreads();
}

// ------------------------------------------------------------------ v3
// Barrier-free variant: no patch staging.  Hits are grouped by the column
// axis A; within a group every thread walks all slices for its own column,
// computing each candidate pixel's coordinates itself (the same exact
// operations), so threads never wait for one another until A changes.
// Three CTAs of 256 threads per SM (24 warps; the kernel is bound by
// latency, so warps count most): shared memory is the 64 KB accumulator
// tile plus compact tables (16-bit slice offsets and row limits; the
// fast_exp table serves gauss_2 too, with the same exact index), ~74 KB.
struct Smem3 {
  float4 *acc;      // [NV]
  float4 *steps;    // (not used by this kernel)
  float *exp;       // [1000] fast_exp table
  float *rtab;      // [N+2]
  short *xmax;      // [N]
  unsigned short *hits;  // [block] slice - s0, grouped by axis
  unsigned short *tmp;   // [block] (slice - s0) | group << 14
  int *wcount;      // [3 * NT/32]
  int *gcount;      // [3]
  int *state;       // [0] steps mode loaded, [1] job geometry loaded (N)
};
constexpr int STEP2CAP = 800;   // gauss_2 step table entries (K = 256 over r <= 3.01: 772)

// Tile-local coordinates (x, y, z) of cell i in layout L: L = A holds the
// tile A-major, (a, b, c) at a*T*T + c*T + b with b < c the other two axes;
// layout 2 is the volume's own [z][y][x] order.
__device__ __forceinline__ void tile_cell(int L, int i, int *l) {
  const int a = i >> 8, c = (i >> 4) & 15, b = i & 15;
  if (L == 0) { l[0] = a; l[1] = b; l[2] = c; }
  else if (L == 1) { l[0] = b; l[1] = a; l[2] = c; }
  else { l[0] = b; l[1] = c; l[2] = a; }
}
__device__ __forceinline__ int tile_index(int L, const int *l) {
  if (L == 0) return (l[0] << 8) | (l[2] << 4) | l[1];
  if (L == 1) return (l[1] << 8) | (l[2] << 4) | l[0];
  return (l[2] << 8) | (l[1] << 4) | l[0];
}
// Moves the tile's accumulators from layout `from` to layout `to` (all
// threads; barriers inside).  Layouts 0 -> 1 swap the x and y digits of the
// cell index, 1 -> 2 the y and z digits: each an involution, done as pair
// swaps with no scratch; 0 -> 2 is both.
__device__ __forceinline__ void swap_digits(float4 *acc, int hi_shift, int lo_shift) {
  // cells (.., u at hi_shift, .., v at lo_shift, ..) <-> (.., v, .., u, ..), u < v
  for (int i = threadIdx.x; i < NV; i += blockDim.x) {
    const int u = (i >> hi_shift) & 15, v = (i >> lo_shift) & 15;
    if (u < v) {
      const int j = i + ((v - u) << hi_shift) - ((v - u) << lo_shift);
      const float4 a = acc[i];
      acc[i] = acc[j];
      acc[j] = a;
    }
  }
}
__device__ __noinline__ void relayout(float4 *acc, int from, int to) {
  __syncthreads();
  if (from == 0) {          // L0 = x:8, z:4, y:0  ->  L1 = y:8, z:4, x:0
    swap_digits(acc, 8, 0);
    __syncthreads();
    from = 1;
  }
  if (from == 1 && to == 2) {   // L1 = y:8, z:4, x:0  ->  L2 = z:8, y:4, x:0
    swap_digits(acc, 8, 4);
    __syncthreads();
  }
}

template <int MODE, int A>
__device__ __forceinline__ void column_work(const Smem3 &S, const float *M, int sg, const int *base,
                                            const int *ext, int N, const float2 *__restrict__ sl,
                                            float w, float h, const ExpSteps &steps) {
  constexpr int B = (A == 0) ? 1 : 0;
  constexpr int C = (A == 2) ? 1 : 2;
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  constexpr int K = Win<MODE>::K;
  const int n2 = N >> 1;
  const float Nf = (float)N;
  const float *m0 = M, *m1 = M + 3, *nrm = M + 6;
  // A warp's 32 columns are an 8 x 4 patch of the tile's (b, c) face: the
  // band of columns a slice's plane reaches in a tile cuts compact patches
  // less often than 16 x 2 strips, so fewer lanes idle (a model of every
  // tile a slice meets: 65 % of a warp's tap slots used against 57 %).
  const int wl = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int lb = (wl & 7) + ((wp & 1) << 3), lc = (wl >> 3) + ((wp >> 1) << 2);
  const int vb = base[B] + lb, vc = base[C] + lc;
  if (vb > ext[B] || vc > ext[C]) return;
  const int tb = sg * vb, tc = sg * vc;
  const int ta_lo = sg > 0 ? base[A] : -ext[A];
  const int ta_hi = sg > 0 ? ext[A] : -base[A];
  float lo[3], hi[3];
  lo[A] = ta_lo - RLO - kDel; hi[A] = ta_hi + RHI + kDel;
  lo[B] = tb - RLO - kDel;    hi[B] = tb + RHI + kDel;
  lo[C] = tc - RLO - kDel;    hi[C] = tc + RHI + kDel;
  // quick reject: heights of the plane over the column's (b, c) window
  {
    const float ia = 1.0f / nrm[A];
    float pmin = 1e30f, pmax = -1e30f;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float pb = (i & 1) ? hi[B] : lo[B], pc = (i & 2) ? hi[C] : lo[C];
      const float pa = -(nrm[B] * pb + nrm[C] * pc) * ia;
      pmin = fminf(pmin, pa);
      pmax = fmaxf(pmax, pa);
    }
    if (pmax < lo[A] - 0.05f || pmin > hi[A] + 0.05f) return;
  }
  const float det = m0[B] * m1[C] - m0[C] * m1[B];
  const float idet = 1.0f / det;
  float ymin = 1e30f, ymax = -1e30f;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float pb = (i & 1) ? hi[B] : lo[B], pc = (i & 2) ? hi[C] : lo[C];
    const float y = (m0[B] * pc - m0[C] * pb) * idet;
    ymin = fminf(ymin, y);
    ymax = fmaxf(ymax, y);
  }
  const int r0 = max(-n2, (int)ceilf(ymin)), r1 = min(n2 - 1, (int)floorf(ymax));
  float inv0[3];
#pragma unroll
  for (int a = 0; a < 3; a++) inv0[a] = fabsf(m0[a]) > 1e-4f ? 1.0f / m0[a] : 0.0f;
  // The tile is held A-major while group A runs: cell (a, b, c) of the tile
  // at a*T*T + c*T + b, so a thread's column is c*T + b + a*T*T; each quarter
  // warp holds 8 consecutive b of one c, so a warp's float4 accesses take the
  // minimum 4 shared wavefronts whatever taps its lanes add.
  const int col_addr = lc * T + lb;
  const bool xzero_col = (A != 0) && (vb == 0);
  for (int y = r0; y <= r1; y++) {
    const int xm = S.xmax[y + n2];
    float xlo = 0.f, xhi = (float)xm;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float c = m1[a] * (float)y;
      const float L = lo[a] - c, U = hi[a] - c;
      if (inv0[a] > 0.f) { xlo = fmaxf(xlo, L * inv0[a]); xhi = fminf(xhi, U * inv0[a]); }
      else if (inv0[a] < 0.f) { xlo = fmaxf(xlo, U * inv0[a]); xhi = fminf(xhi, L * inv0[a]); }
      else if (L > 0.05f || U < -0.05f) xhi = -1e30f;
    }
    const int c0 = max(0, (int)ceilf(xlo)), c1 = min(xm, (int)floorf(xhi));
    if (c0 > c1) continue;
    const float ry = S.rtab[y + n2];
    // the row's slice values; pixel (0, y < 0) reads (0, -y) conjugated
    const int w2s = (N >> 1) + 1;
    const float2 *rowp = sl + (size_t)(y < 0 ? N + y : y) * w2s;
    const float2 *mirp = sl + (size_t)(y < 0 ? -y : 0) * w2s;
    for (int x = c0; x <= c1; x++) {
      float xx, yy, zz;
      pixel_coords(S.rtab[x + n2], ry, M, Nf, xx, yy, zz);
      const float pa = A == 0 ? xx : (A == 1 ? yy : zz);
      const float pb = B == 0 ? xx : yy;
      const float pc = C == 1 ? yy : zz;
      if (!(in_win<MODE>(tb, pb) && in_win<MODE>(tc, pc))) continue;
      const int a0 = win_start<MODE>(pa);
      const int k0 = max(a0, ta_lo), k1 = min(a0 + K - 1, ta_hi);
      if (k0 > k1) continue;
      const bool herm = (x == 0) && (y < 0);
      float2 v = __ldg(herm ? mirp : rowp + x);
      if (herm) v.y = -v.y;
      float f0 = 0.f, f1 = 0.f;
      if (MODE == MODE_GAUSS2 || MODE == MODE_GAUSS5) {
        if (A == 0) {
          const float dy = __fsub_rn((float)tb, yy), dz = __fsub_rn((float)tc, zz);
          f0 = __fmul_rn(dy, dy); f1 = __fmul_rn(dz, dz);
        } else if (A == 1) {
          const float dx = __fsub_rn((float)tb, xx), dz = __fsub_rn((float)tc, zz);
          f0 = __fmul_rn(dx, dx); f1 = __fmul_rn(dz, dz);
        } else {
          const float dx = __fsub_rn((float)tb, xx), dy = __fsub_rn((float)tc, yy);
          f0 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
        }
      }
      // the window's taps along A inside the tile (the rest belong to the
      // neighbouring tile's work item): a predicated straight line for the
      // 2-tap windows, a loop for gauss_5's 6 (its unrolled form is slower)
      auto tap = [&](int k, float kf) {
        float vre, vim, vw;
        if (MODE == MODE_GAUSS2 || MODE == MODE_GAUSS5) {
          const float d = __fsub_rn(kf, pa);
          const float d2 = __fmul_rn(d, d);
          float r;
          if (A == 0) r = __fadd_rn(__fadd_rn(d2, f0), f1);
          else if (A == 1) r = __fadd_rn(__fadd_rn(f0, d2), f1);
          else r = __fadd_rn(f0, d2);
          if (MODE == MODE_GAUSS2) {
            // r >= 0 and h > 0, so f <= 0: fast_exp's f > 0 branch never runs
            const float f = __fmul_rn(-r, h);
            float g = S.exp[min(__double2int_rz(__fma_rn((double)(-f), 50.0, 0.5)), 999)];
            if (f < -19.98f) g = expf(f);
            const float gg = __fmul_rn(g, w);
            vre = __fmul_rn(v.x, gg);
            vim = __fmul_rn(v.y, gg);
            vw = gg;
          } else {
            // Util::fast_exp(f): the table index (int)(-f*50.0+0.5) is formed
            // in double as the reference forms it; -f*50 + 0.5 is exact in
            // double (a float times 50 plus 0.5 needs at most 31 bits), so
            // one DFMA and a truncating conversion give the reference's index.
            // The entry is read for every tap (index clamped to the table) and
            // replaced by exp(f) past it, so the common path has no branch;
            // f <= 0 always (r >= 0, h > 0).
            const float f = __fmul_rn(-r, h);
            float gg = S.exp[min(__double2int_rz(__fma_rn((double)(-f), 50.0, 0.5)), 999)];
            if (f < -19.98f) gg = expf(f);
            vre = __fmul_rn(__fmul_rn(v.x, gg), w);
            vim = __fmul_rn(__fmul_rn(v.y, gg), w);
            vw = __fmul_rn(gg, w);
          }
        } else {
          int t[3];
          t[A] = k; t[B] = tb; t[C] = tc;
          tap_value<MODE>(t[0], t[1], t[2], xx, yy, zz, v.x, v.y, w, h, nullptr, vre, vim, vw);
        }
        const int la = sg * k - base[A];
        float4 *cell = &S.acc[col_addr + la * (T * T)];
        float4 u = *cell;
        const bool origin = (k == 0 && tb == 0 && tc == 0);
        if (sg > 0) {
          u.x += vre;
          if (origin) u.w = 1.0f;
          else u.y += vim;
          u.z += vw;
        } else {
          if (origin) return;
          u.x += vre;
          u.y -= vim;
          const bool xzero = (A == 0) ? (k == 0) : xzero_col;
          if (!xzero) u.z += vw;
        }
        *cell = u;
      };
      if (K <= 2) {
#pragma unroll
        for (int j = 0; j < K; j++) {
          const int k = a0 + j;
          if (k >= k0 && k <= k1) tap(k, (float)k);
        }
      } else {
        float kf = (float)k0;   // exact: |k| < 2^24
        for (int k = k0; k <= k1; k++, kf += 1.0f) tap(k, kf);
      }
    }
  }
}

template <int MODE, int A>
__device__ __forceinline__ void group_work(const InsertJob &J, const Smem3 &S, int g0, int g1,
                                           const int *base, const int *ext, float h,
                                           const ExpSteps &steps, int s0) {
  const int N = J.N, w2 = (N >> 1) + 1;
  for (int hI = g0; hI < g1; hI++) {
    const int s = s0 + S.hits[hI];
    const int p = s / J.nsym;
    float M[9];
#pragma unroll
    for (int i = 0; i < 9; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
    const float w = __ldg(&J.pw[p]);
    const float2 *sl = J.slices + (size_t)p * N * w2;
    column_work<MODE, A>(S, M, 1, base, ext, N, sl, w, h, steps);
    column_work<MODE, A>(S, M, -1, base, ext, N, sl, w, h, steps);
  }
}

template <int MODE>
__device__ void tile_item3(const InsertJob &J, int tile, int s0, int s1, const Smem3 &S, float h,
                           const ExpSteps &steps, int *err) {
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  const int N = J.N, n2 = N >> 1;
  const int tix = tile % J.tiles_x, tiy = (tile / J.tiles_x) % J.tiles_y,
            tiz = tile / (J.tiles_x * J.tiles_y);
  const int base[3] = {tix * T, -n2 + 1 + tiy * T, -n2 + 1 + tiz * T};
  const int ext[3] = {min(base[0] + T - 1, n2 - 1), min(base[1] + T - 1, n2 - 1),
                      min(base[2] + T - 1, n2 - 1)};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = NT / 32;
  // ---- cull, and count the hits of each axis group
  int nhit = 0;
  for (int r = s0; r < s1; r += NT) {
    const int s = r + threadIdx.x;
    int grp = -1;
    if (s < s1 && __ldg(&J.pw[s / J.nsym]) != 0.0f) {
      const float n[3] = {__ldg(&J.t3d[9 * s + 6]), __ldg(&J.t3d[9 * s + 7]), __ldg(&J.t3d[9 * s + 8])};
      // A pixel's direct taps reach the tile from [base - RLO, ext + RHI];
      // its conjugate taps (mirrored) from [base - RHI, ext + RLO].  The
      // plane passes through the origin, so one test against the union box
      // covers both passes (gauss_5's window is asymmetric: 2.5 / 3.5).
      constexpr float RC = (RLO > RHI ? RLO : RHI) + kDel;
      const float lo[3] = {base[0] - RC, base[1] - RC, base[2] - RC};
      const float hi[3] = {ext[0] + RC, ext[1] + RC, ext[2] + RC};
      float mn, mx;
      box_dot(n, lo, hi, mn, mx);
      if (mn <= kPlaneTol && mx >= -kPlaneTol) {
        const float a0 = fabsf(n[0]), a1 = fabsf(n[1]), a2 = fabsf(n[2]);
        grp = (a0 >= a1 && a0 >= a2) ? 0 : (a1 >= a2 ? 1 : 2);
      }
    }
    const unsigned b = __ballot_sync(0xffffffffu, grp >= 0);
    if (lane == 0) S.wcount[warp] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      const int c = S.wcount[i];
      off += (i < warp) ? c : 0;
      tot += c;
    }
    if (grp >= 0) {
      const int at = nhit + off + __popc(b & ((1u << lane) - 1u));
      S.tmp[at] = (unsigned short)((s - s0) | (grp << 14));
    }
    nhit += tot;
    __syncthreads();
  }
  if (nhit == 0) return;
  // ---- stable partition of the hits by axis group
  if (threadIdx.x < 3) S.gcount[threadIdx.x] = 0;
  __syncthreads();
  int gstart[4];
  {
    int base_g = 0;
    for (int g = 0; g < 3; g++) {
      gstart[g] = base_g;
      for (int r = 0; r < nhit; r += NT) {
        const int i = r + threadIdx.x;
        const bool in = i < nhit && (S.tmp[i] >> 14) == g;
        const unsigned b = __ballot_sync(0xffffffffu, in);
        if (lane == 0) S.wcount[warp] = __popc(b);
        __syncthreads();
        int off = 0, tot = 0;
#pragma unroll
        for (int q = 0; q < NW; q++) {
          const int c = S.wcount[q];
          off += (q < warp) ? c : 0;
          tot += c;
        }
        if (in) S.hits[base_g + off + __popc(b & ((1u << lane) - 1u))] = S.tmp[i] & 0x3FFF;
        base_g += tot;
        __syncthreads();
      }
    }
    gstart[3] = base_g;
  }
  // ---- per-job tables and this mode's exp table
  if (*(S.state + 1) != J.N) {
    for (int i = threadIdx.x; i < N + 2; i += NT) S.rtab[i] = __ldg(&J.rtab[i]);
    for (int i = threadIdx.x; i < N; i += NT) S.xmax[i] = (short)__ldg(&J.xmax[i]);
  }
  for (int i = threadIdx.x; i < NV; i += NT) S.acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (MODE == MODE_GAUSS2) *S.state = MODE;
    *(S.state + 1) = J.N;
  }
  // ---- the three axis groups; ownership of a voxel changes only between
  // them, and so does the tile's layout (A-major for group A)
  int layout = -1;   // -1: nothing added yet, any layout holds the zeros
  if (gstart[1] > gstart[0]) {
    group_work<MODE, 0>(J, S, gstart[0], gstart[1], base, ext, h, steps, s0);
    layout = 0;
  }
  __syncthreads();
  if (gstart[2] > gstart[1]) {
    if (layout == 0) relayout(S.acc, 0, 1);
    group_work<MODE, 1>(J, S, gstart[1], gstart[2], base, ext, h, steps, s0);
    layout = 1;
  }
  __syncthreads();
  if (gstart[3] > gstart[2]) {
    if (layout == 0 || layout == 1) relayout(S.acc, layout, 2);
    group_work<MODE, 2>(J, S, gstart[2], gstart[3], base, ext, h, steps, s0);
    layout = 2;
  }
  __syncthreads();
  // ---- flush
  const size_t nxf = (size_t)N + 2;
  const int w2 = n2 + 1;
  for (int i = threadIdx.x; i < NV; i += NT) {
    const float4 v = S.acc[i];
    if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
    int l3[3];
    tile_cell(layout, i, l3);
    const int vx = base[0] + l3[0], vy = base[1] + l3[1], vz = base[2] + l3[2];
    if (vx > ext[0] || vy > ext[1] || vz > ext[2]) continue;
    const size_t row = (size_t)(vy < 0 ? N + vy : vy);
    const size_t slab = (size_t)(vz < 0 ? N + vz : vz);
    const size_t di = (size_t)vx * 2 + row * nxf + slab * nxf * (size_t)N;
    const size_t ni = (size_t)vx + row * (size_t)w2 + slab * (size_t)w2 * (size_t)N;
    if (v.w != 0.f) {
      atomicAdd(&J.data[di], v.x);
      J.data[di + 1] = 0.0f;
    } else {
      atomicAdd(reinterpret_cast<float2 *>(&J.data[di]), make_float2(v.x, v.y));
    }
    if (v.z != 0.f) atomicAdd(&J.norm[ni], v.z);
  }
  __syncthreads();
}


// ------------------------------------------------------------------ v4
// Pixel-major variant for the windows one or two taps wide (nearest,
// gauss_2, trilinear), where walking columns spends most of its
// instructions finding candidate pixels for two taps.  Each warp takes
// whole hit slices and, for each, bounds the slice's pixels whose window can
// meet the tile (or its mirror): rows from the projection of the tile box on
// the slice's y axis, x ranges per row, a warp prefix sum.  Its lanes then run
// over those pixels with the reference's exact coordinate and tap arithmetic
// and add every tap that lands in the tile to the shared-memory
// accumulators with shared atomics.  No block barriers between slices.
constexpr int PROWS = 32;   // rows per row batch of a pass

struct Smem4 {
  float *are, *aim, *awt;     // accumulators, one array per component [NV]
  int *origin;                // the volume's origin cell got a direct tap (its imag is 0)
  float *rexp;                // gauss_2's fast_exp entries, kRexpCopies interleaved copies
  float *rtab;
  int *xmax;
  int *hits;
  int *tmp;
  int *wcount;
  int *next;                   // next (slice, pass) unit of the work item
  unsigned long long *state;   // [0] exp copies loaded (mode), [1] xmax table loaded (address)
};

// gauss_2 taps have r <= 3, so fast_exp(-r*h) only reads entries 0..370 of
// the 1000-entry table.  Eight interleaved copies, entry g of copy c at
// 8g + c, with lane l reading copy l & 7: the four lanes that share a copy
// meet in one bank only when their entries differ by a multiple of 4, so a
// warp's lookup takes ~2 shared wavefronts instead of the ~4.5 a 16-byte
// step-table entry took.
constexpr int kRexpEntries = 376;
constexpr int kRexpCopies = 8;

// Util::fast_exp(f) for f in [-19.98, 0] read from the interleaved copies.
// The index (int)(-f*50.0+0.5) is formed in double as the reference forms it:
// -f*50 + 0.5 is exact in double, so one DFMA and a truncating conversion give
// it (1 % faster here than an exact FP32 construction of the same index).
__device__ __forceinline__ float rexp_lookup(float f, const float *rexp) {
  const int g = __double2int_rz(__fma_rn((double)(-f), 50.0, 0.5));
  return rexp[g * kRexpCopies + (threadIdx.x & (kRexpCopies - 1))];
}

// Slot of local cell (lx, ly, lz) in the component arrays.  Each pair of rows
// (ly >> 1, lz) fills 32 consecutive words, one per bank; within it the
// position lx + 16 (ly & 1) is XORed with a 5-bit hash of (ly >> 1, lz), so
// the cells a warp's pixels hit (a patch of the slice plane, in any
// orientation) spread over the banks.  Multipliers 5 and 9 came from a
// search over odd pairs on simulated warps of random orientations: 2.9
// wavefronts per atomic against 3.6 for an XOR of lx with (ly >> 1) + lz.
__device__ __forceinline__ int cell_slot(int lx, int ly, int lz) {
  return ((lz * T + ly) >> 1) * 32 + ((lx + 16 * (ly & 1)) ^ (((ly >> 1) * 5 + lz * 9) & 31));
}

// Adds one tap's contribution to cell (i,j,k) of the window under the
// placement rules of add_complex_at_fast (libEM/emdata_core.h:368-410):
// pass sg = +1 takes the direct cells (i >= 0), pass sg = -1 the conjugate
// cells (-i,-j,-k) of taps with i <= 0; the x = 0 plane's conjugate copy
// carries no weight and the origin keeps only its real part.
__device__ __forceinline__ void tile_tap(const Smem4 &S, int sg, int i, int j, int k,
                                         const int *base, const int *ext, float vre, float vim,
                                         float vw) {
  int ti = i, tj = j, tk = k;
  if (sg < 0) { ti = -i; tj = -j; tk = -k; }
  if (ti < base[0] || ti > ext[0] || tj < base[1] || tj > ext[1] || tk < base[2] || tk > ext[2])
    return;
  const bool origin = (i == 0 && j == 0 && k == 0);
  const int c = cell_slot(ti - base[0], tj - base[1], tk - base[2]);
  if (sg > 0) {
    atomicAdd(&S.are[c], vre);
    if (origin) *S.origin = 1;
    else atomicAdd(&S.aim[c], vim);
    atomicAdd(&S.awt[c], vw);
  } else {
    if (origin) return;
    atomicAdd(&S.are[c], vre);
    atomicAdd(&S.aim[c], -vim);
    if (i != 0) atomicAdd(&S.awt[c], vw);
  }
}

template <int MODE>
__device__ __forceinline__ void pixel_pass(const InsertJob &J, const Smem4 &S, const float *M,
                                           int sg, const int *base, const int *ext,
                                           const float2 *__restrict__ sl, float w, float h) {
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  const int N = J.N, n2 = N >> 1;
  const float Nf = (float)N;
  const int lane = threadIdx.x & 31;
  float lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    lo[a] = (sg > 0 ? base[a] : -ext[a]) - RLO - kDel;
    hi[a] = (sg > 0 ? ext[a] : -base[a]) + RHI + kDel;
  }
  // mapped point of pixel (x, y) ~ x*u + y*v with u, v the first two rows of
  // M (orthonormal), so y ~ p.v: rows from the box's extent along v
  const float *u = M, *v = M + 3;
  float ymn, ymx;
  box_dot(v, lo, hi, ymn, ymx);
  const int r0 = max(-n2, (int)ceilf(ymn - 0.05f)), r1 = min(n2 - 1, (int)floorf(ymx + 0.05f));
  for (int rb = r0; rb <= r1; rb += PROWS) {
    // ---- this row batch's x ranges and prefix offsets
    const int y = rb + lane;
    int c0 = 0, cnt = 0;
    if (y <= r1) {
      float xlo = 0.0f, xhi = (float)S.xmax[y + n2];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        if (fabsf(u[a]) > 0.05f) {
          const float c = v[a] * (float)y;
          const float L = (lo[a] - c) / u[a], U = (hi[a] - c) / u[a];
          xlo = fmaxf(xlo, fminf(L, U) - 0.05f);
          xhi = fminf(xhi, fmaxf(L, U) + 0.05f);
        }
      }
      c0 = max(0, (int)ceilf(xlo));
      const int c1 = min(S.xmax[y + n2], (int)floorf(xhi));
      cnt = max(0, c1 - c0 + 1);
    }
    // ---- the batch's nonempty rows, compacted: lane j holds the j-th one
    // (its row in the batch, first pixel column, pixel count, first pixel)
    const unsigned full = 0xffffffffu;
    const unsigned ne = __ballot_sync(full, cnt > 0);
    const int nrows = __popc(ne);
    int src;
    {
      int lo = 0, hi = 31;   // position of the (lane+1)-th set bit of ne
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__popc(ne & ((2u << mid) - 1u)) >= lane + 1) hi = mid;
        else lo = mid + 1;
      }
      src = lo;
    }
    const int rc0 = __shfl_sync(full, c0, src);
    int rcnt = __shfl_sync(full, cnt, src);
    if (lane >= nrows) rcnt = 0;
    int incl = rcnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(full, incl, 31);
    const int rstart = incl - rcnt;
    // ---- the pixels of the batch, one per lane.  The row of pixel wb+lane:
    // the row holding pixel wb, plus the rows starting in (wb, wb+lane], read
    // from a mask of the row starts inside the window (registers only).
    for (int wb = 0; wb < total; wb += 32) {
      const bool real = lane < nrows;
      const unsigned le = __ballot_sync(full, real && rstart <= wb);
      const int kb = 31 - __clz(le);
      const unsigned bit = (real && rstart > wb && rstart < wb + 32) ? (1u << (rstart - wb)) : 0u;
      const unsigned starts = __reduce_or_sync(full, bit);
      const int kr = kb + __popc(starts & ((2u << lane) - 1u));
      const int kx0 = __shfl_sync(full, rc0, kr), ks = __shfl_sync(full, rstart, kr),
                krow = __shfl_sync(full, src, kr);
      const int idx = wb + lane;
      if (idx >= total) continue;
      const int x = kx0 + (idx - ks);
      const int py = rb + krow;
      float xx, yy, zz;
      pixel_coords(S.rtab[x + n2], S.rtab[py + n2], M, Nf, xx, yy, zz);
      const float2 val = slice_value(sl, N, x, py);
      if (MODE == MODE_NEAREST) {
        // FourierInserter3DMode1 (libEM/reconstructor_tools.cpp:113-126)
        const int i = (int)floorf(__fadd_rn(xx, 0.5f)), j = (int)floorf(__fadd_rn(yy, 0.5f)),
                  k = (int)floorf(__fadd_rn(zz, 0.5f));
        tile_tap(S, sg, i, j, k, base, ext, __fmul_rn(val.x, w), __fmul_rn(val.y, w), w);
      } else {
        const int x0 = (int)floorf(xx), y0 = (int)floorf(yy), z0 = (int)floorf(zz);
        float dxx[2], dyy[2], dzz[2];
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const float dx = __fsub_rn((float)(x0 + q), xx), dy = __fsub_rn((float)(y0 + q), yy),
                      dz = __fsub_rn((float)(z0 + q), zz);
          dxx[q] = __fmul_rn(dx, dx);
          dyy[q] = __fmul_rn(dy, dy);
          dzz[q] = __fmul_rn(dz, dz);
        }
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
          for (int b = 0; b < 2; b++)
#pragma unroll
            for (int a = 0; a < 2; a++) {
              float vre, vim, vw;
              if (MODE == MODE_GAUSS2) {
                const float r = __fadd_rn(__fadd_rn(dxx[a], dyy[b]), dzz[c]);
                const float gg = __fmul_rn(rexp_lookup(__fmul_rn(-r, h), S.rexp), w);
                vre = __fmul_rn(val.x, gg);
                vim = __fmul_rn(val.y, gg);
                vw = gg;
              } else {
                tap_value<MODE>(x0 + a, y0 + b, z0 + c, xx, yy, zz, val.x, val.y, w, h, nullptr,
                                vre, vim, vw);
              }
              tile_tap(S, sg, x0 + a, y0 + b, z0 + c, base, ext, vre, vim, vw);
            }
      }
    }
    __syncwarp();
  }
}

template <int MODE>
__device__ void tile_item4(const InsertJob &J, int tile, int s0, int s1, const Smem4 &S, float h,
                           const float *__restrict__ exp_g) {
  constexpr float RLO = Win<MODE>::lo, RHI = Win<MODE>::hi;
  const int N = J.N, n2 = N >> 1;
  const int tix = tile % J.tiles_x, tiy = (tile / J.tiles_x) % J.tiles_y,
            tiz = tile / (J.tiles_x * J.tiles_y);
  const int base[3] = {tix * T, -n2 + 1 + tiy * T, -n2 + 1 + tiz * T};
  const int ext[3] = {min(base[0] + T - 1, n2 - 1), min(base[1] + T - 1, n2 - 1),
                      min(base[2] + T - 1, n2 - 1)};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = NT / 32;
  // ---- cull: slices whose plane passes the tile (and so its mirror)
  int nhit = 0;
  for (int r = s0; r < s1; r += NT) {
    const int s = r + threadIdx.x;
    bool hit = false;
    if (s < s1 && __ldg(&J.pw[s / J.nsym]) != 0.0f) {
      const float n[3] = {__ldg(&J.t3d[9 * s + 6]), __ldg(&J.t3d[9 * s + 7]), __ldg(&J.t3d[9 * s + 8])};
      // A pixel's direct taps reach the tile from [base - RLO, ext + RHI];
      // its conjugate taps (mirrored) from [base - RHI, ext + RLO].  The
      // plane passes through the origin, so one test against the union box
      // covers both passes (gauss_5's window is asymmetric: 2.5 / 3.5).
      constexpr float RC = (RLO > RHI ? RLO : RHI) + kDel;
      const float lo[3] = {base[0] - RC, base[1] - RC, base[2] - RC};
      const float hi[3] = {ext[0] + RC, ext[1] + RC, ext[2] + RC};
      float mn, mx;
      box_dot(n, lo, hi, mn, mx);
      hit = mn <= kPlaneTol && mx >= -kPlaneTol;
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) S.wcount[warp] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      const int c = S.wcount[i];
      off += (i < warp) ? c : 0;
      tot += c;
    }
    if (hit) S.hits[nhit + off + __popc(b & ((1u << lane) - 1u))] = s;
    nhit += tot;
    __syncthreads();
  }
  if (nhit == 0) return;
  // ---- per-job tables and this mode's step table
  if (S.state[1] != (unsigned long long)J.xmax) {
    for (int i = threadIdx.x; i < N + 2; i += NT) S.rtab[i] = __ldg(&J.rtab[i]);
    for (int i = threadIdx.x; i < N; i += NT) S.xmax[i] = __ldg(&J.xmax[i]);
  }
  if (MODE == MODE_GAUSS2 && S.state[0] != (unsigned long long)MODE)
    for (int i = threadIdx.x; i < kRexpEntries * kRexpCopies; i += NT)
      S.rexp[i] = __ldg(&exp_g[i / kRexpCopies]);
  for (int i = threadIdx.x; i < NV; i += NT) {
    S.are[i] = 0.f;
    S.aim[i] = 0.f;
    S.awt[i] = 0.f;
  }
  if (threadIdx.x == 0) {
    *S.next = 0;
    *S.origin = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (MODE == MODE_GAUSS2) S.state[0] = (unsigned long long)MODE;
    S.state[1] = (unsigned long long)J.xmax;
  }
  // ---- warps take (slice, pass) units as they come free
  const int w2 = n2 + 1;
  while (true) {
    int u = 0;
    if (lane == 0) u = atomicAdd(S.next, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= 2 * nhit) break;
    const int s = S.hits[u >> 1];
    const int p = s / J.nsym;
    float M[9];
#pragma unroll
    for (int i = 0; i < 9; i++) M[i] = __ldg(&J.t3d[9 * s + i]);
    const float w = __ldg(&J.pw[p]);
    const float2 *sl = J.slices + (size_t)p * N * w2;
    pixel_pass<MODE>(J, S, M, (u & 1) ? -1 : 1, base, ext, sl, w, h);
  }
  __syncthreads();
  // ---- flush (as tile_item3)
  const size_t nxf = (size_t)N + 2;
  for (int i = threadIdx.x; i < NV; i += NT) {
    const int lz = i >> 8, ly = (i >> 4) & 15, lx = i & 15;
    const int c = cell_slot(lx, ly, lz);
    const int vx = base[0] + lx, vy = base[1] + ly, vz = base[2] + lz;
    const bool org = vx == 0 && vy == 0 && vz == 0 && *S.origin;
    const float4 v = make_float4(S.are[c], S.aim[c], S.awt[c], org ? 1.0f : 0.0f);
    if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
    if (vx > ext[0] || vy > ext[1] || vz > ext[2]) continue;
    const size_t row = (size_t)(vy < 0 ? N + vy : vy);
    const size_t slab = (size_t)(vz < 0 ? N + vz : vz);
    const size_t di = (size_t)vx * 2 + row * nxf + slab * nxf * (size_t)N;
    const size_t ni = (size_t)vx + row * (size_t)w2 + slab * (size_t)w2 * (size_t)N;
    if (v.w != 0.f) {
      atomicAdd(&J.data[di], v.x);
      J.data[di + 1] = 0.0f;
    } else {
      atomicAdd(reinterpret_cast<float2 *>(&J.data[di]), make_float2(v.x, v.y));
    }
    if (v.z != 0.f) atomicAdd(&J.norm[ni], v.z);
  }
  __syncthreads();
}
}  // namespace col

// work[i] = (job, tile, first slice, end slice); blocks are at most `block`.
__global__ void __launch_bounds__(col::NT, 2)
    k_column(const InsertJob *__restrict__ jobs, const int4 *__restrict__ work, int nwork, int block,
             int *counter, const float *__restrict__ exp_g, float h2, float h5, ExpSteps st2,
             ExpSteps st5, int side, int *err) {
  extern __shared__ float4 s_dyn[];
  __shared__ int s_work;
  __shared__ int s_wcount[col::NT / 32];
  __shared__ int s_steps_mode;
  col::Smem S;
  S.acc = s_dyn;
  S.steps = s_dyn + col::NV;
  S.pt = S.steps + col::STEPCAP;
  S.pim = reinterpret_cast<float *>(S.pt + col::PIXCAP);
  S.hits = reinterpret_cast<int *>(S.pim + col::PIXCAP);
  S.wcount = s_wcount;
  S.steps_mode = &s_steps_mode;
  if (threadIdx.x == 0) s_steps_mode = -1;
  (void)exp_g;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_work = atomicAdd(counter, 1);
    __syncthreads();
    const int wi = s_work;
    if (wi >= nwork) break;
    const int4 wk = work[wi];
    const InsertJob J = jobs[wk.x];
    const int s0 = wk.z, s1 = min(min(wk.w, wk.z + block), J.np * J.nsym);
    switch (J.mode) {
      case MODE_GAUSS2: col::tile_item<MODE_GAUSS2>(J, wk.y, s0, s1, S, side, h2, st2, err); break;
      case MODE_GAUSS5: col::tile_item<MODE_GAUSS5>(J, wk.y, s0, s1, S, side, h5, st5, err); break;
      case MODE_NEAREST: col::tile_item<MODE_NEAREST>(J, wk.y, s0, s1, S, side, h2, st2, err); break;
      case MODE_TRILINEAR: col::tile_item<MODE_TRILINEAR>(J, wk.y, s0, s1, S, side, h2, st2, err); break;
      default:
        if (threadIdx.x == 0) atomicOr(err, 4);
    }
  }
}

__global__ void __launch_bounds__(col::NT, 3)
    k_column3(const InsertJob *__restrict__ jobs, const int4 *__restrict__ work, int nwork,
              int block, int *counter, const float *__restrict__ exp_g, float h2, float h5,
              ExpSteps st2, ExpSteps st5, int maxN, int *err) {
  extern __shared__ float4 s_dyn[];
  __shared__ int s_work;
  __shared__ int s_wcount[col::NT / 32];
  __shared__ int s_gcount[3];
  __shared__ int s_state[2];
  col::Smem3 S;
  S.acc = s_dyn;
  S.steps = nullptr;
  S.exp = reinterpret_cast<float *>(s_dyn + col::NV);
  S.rtab = S.exp + 1000;
  S.xmax = reinterpret_cast<short *>(S.rtab + maxN + 2);
  S.hits = reinterpret_cast<unsigned short *>(S.xmax + maxN + 2);
  S.tmp = S.hits + block;
  S.wcount = s_wcount;
  S.gcount = s_gcount;
  S.state = s_state;
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) S.exp[i] = exp_g[i];
  if (threadIdx.x == 0) { s_state[0] = -1; s_state[1] = -1; }
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_work = atomicAdd(counter, 1);
    __syncthreads();
    const int wi = s_work;
    if (wi >= nwork) break;
    const int4 wk = work[wi];
    const InsertJob J = jobs[wk.x];
    const int s0 = wk.z, s1 = min(min(wk.w, wk.z + block), J.np * J.nsym);
    switch (J.mode) {
      case MODE_GAUSS2: col::tile_item3<MODE_GAUSS2>(J, wk.y, s0, s1, S, h2, st2, err); break;
      case MODE_GAUSS5: col::tile_item3<MODE_GAUSS5>(J, wk.y, s0, s1, S, h5, st5, err); break;
      case MODE_NEAREST: col::tile_item3<MODE_NEAREST>(J, wk.y, s0, s1, S, h2, st2, err); break;
      case MODE_TRILINEAR: col::tile_item3<MODE_TRILINEAR>(J, wk.y, s0, s1, S, h2, st2, err); break;
      default:
        if (threadIdx.x == 0) atomicOr(err, 4);
    }
  }
}

cudaError_t launch_column3(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                           int *d_counter, int maxN, cudaStream_t st) {
  if (nwork == 0) return cudaSuccess;
  const Consts &c = consts();
  const size_t smem = sizeof(float4) * col::NV + sizeof(float) * 1000 +
                      sizeof(float) * (maxN + 2) + sizeof(short) * (maxN + 2) +
                      2 * sizeof(unsigned short) * block;
  cudaError_t ea = set_max_smem((const void *)k_column3, smem);
  if (ea != cudaSuccess) return ea;
  cudaError_t e = zero_counter(d_counter, st);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_column3, col::NT, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(nwork, sms * per_sm));
  note_launch();
  k_column3<<<grid, col::NT, smem, st>>>(d_jobs, d_work, nwork, block, d_counter, c.d_exp, c.h2,
                                         c.h5, c.steps2, c.steps5, maxN, c.d_err);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(col::NT, 3)
    k_pixel(const InsertJob *__restrict__ jobs, const int4 *__restrict__ work, int nwork,
            int block, int *counter, float h2, const float *__restrict__ exp_g, int maxN,
            int *err) {
  extern __shared__ float4 s_dyn[];
  __shared__ int s_work;
  __shared__ int s_wcount[col::NT / 32];
  __shared__ unsigned long long s_state[2];
  __shared__ int s_next, s_origin;
  col::Smem4 S;
  S.are = reinterpret_cast<float *>(s_dyn);
  S.aim = S.are + col::NV;
  S.awt = S.aim + col::NV;
  S.origin = &s_origin;
  S.rexp = S.awt + col::NV;
  S.rtab = S.rexp + col::kRexpEntries * col::kRexpCopies;
  S.xmax = reinterpret_cast<int *>(S.rtab + maxN + 2);
  S.hits = S.xmax + maxN;
  S.wcount = s_wcount;
  S.next = &s_next;
  S.state = s_state;
  if (threadIdx.x == 0) { s_state[0] = ~0ull; s_state[1] = 0ull; }
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_work = atomicAdd(counter, 1);
    __syncthreads();
    const int wi = s_work;
    if (wi >= nwork) break;
    const int4 wk = work[wi];
    const InsertJob J = jobs[wk.x];
    const int s0 = wk.z, s1 = min(min(wk.w, wk.z + block), J.np * J.nsym);
    switch (J.mode) {
      case MODE_GAUSS2: col::tile_item4<MODE_GAUSS2>(J, wk.y, s0, s1, S, h2, exp_g); break;
      case MODE_NEAREST: col::tile_item4<MODE_NEAREST>(J, wk.y, s0, s1, S, h2, exp_g); break;
      case MODE_TRILINEAR: col::tile_item4<MODE_TRILINEAR>(J, wk.y, s0, s1, S, h2, exp_g); break;
      default:
        if (threadIdx.x == 0) atomicOr(err, 4);   // gauss_5 takes the column kernel
    }
  }
}

cudaError_t launch_pixel(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                         int *d_counter, int maxN, cudaStream_t st) {
  if (nwork == 0) return cudaSuccess;
  const Consts &c = consts();
  const size_t smem = sizeof(float) * 3 * col::NV +
                      sizeof(float) * col::kRexpEntries * col::kRexpCopies +
                      sizeof(float) * (maxN + 2) + sizeof(int) * maxN + sizeof(int) * block;
  cudaError_t ea = set_max_smem((const void *)k_pixel, smem);
  if (ea != cudaSuccess) return ea;
  cudaError_t e = zero_counter(d_counter, st);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pixel, col::NT, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(nwork, sms * per_sm));
  note_launch();
  k_pixel<<<grid, col::NT, smem, st>>>(d_jobs, d_work, nwork, block, d_counter, c.h2, c.d_exp,
                                       maxN, c.d_err);
  return cudaGetLastError();
}

int column_side(int max_mode) {
  const float r = (max_mode == MODE_GAUSS5 ? 6.0f : max_mode == MODE_NEAREST ? 1.0f : 2.0f) +
                  2 * col::kDel;
  const float e = col::T - 1 + r;
  return (int)std::ceil(std::sqrt(3.0f) * e) + 5;
}

size_t column_smem(int side, int block) {
  (void)side;
  return sizeof(float4) * (col::NV + col::STEPCAP + col::PIXCAP) + sizeof(float) * col::PIXCAP +
         sizeof(int) * block;
}

cudaError_t launch_column(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                          int *d_counter, int max_mode, cudaStream_t st) {
  if (nwork == 0) return cudaSuccess;
  const Consts &c = consts();
  const int side = column_side(max_mode);
  const size_t smem = column_smem(side, block);
  cudaError_t ea = set_max_smem((const void *)k_column, smem);
  if (ea != cudaSuccess) return ea;
  cudaError_t e = zero_counter(d_counter, st);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_column, col::NT, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(nwork, sms * per_sm));
  note_launch();
  k_column<<<grid, col::NT, smem, st>>>(d_jobs, d_work, nwork, block, d_counter, c.d_exp, c.h2, c.h5,
                                        c.steps2, c.steps5, side, c.d_err);
  return cudaGetLastError();
}

// Column-kernel tiles of a job (16^3 over the interior cells) that can
// receive taps, nearest to the origin first.
void column_tiles(int N, int mode, int corners, std::vector<int> &out, int &tx, int &ty, int &tz,
                  std::vector<float> *dist) {
  const int n2 = N / 2, T = col::T;
  tx = (n2 + T - 1) / T;
  ty = (N - 1 + T - 1) / T;
  tz = (N - 1 + T - 1) / T;
  const double reach = (mode == MODE_GAUSS5 ? 3.5 : mode == MODE_NEAREST ? 0.5 : 1.0);
  const double rpix = corners ? n2 * 1.41422 + 1.0 : n2 + 0.5 + 0.01;
  const double rmax = rpix + reach * 1.7321 + 0.1;
  std::vector<std::pair<double, int>> order;
  for (int iz = 0; iz < tz; iz++)
    for (int iy = 0; iy < ty; iy++)
      for (int ix = 0; ix < tx; ix++) {
        const int b[3] = {ix * T, -n2 + 1 + iy * T, -n2 + 1 + iz * T};
        double d2 = 0;
        for (int a = 0; a < 3; a++) {
          const int e = std::min(b[a] + T - 1, n2 - 1);
          const double d = (b[a] <= 0 && e >= 0) ? 0.0 : (double)std::min(std::abs(b[a]), std::abs(e));
          d2 += d * d;
        }
        const double d = std::sqrt(d2);
        if (d <= rmax) order.push_back({d, ix + tx * (iy + ty * iz)});
      }
  std::stable_sort(order.begin(), order.end());
  out.clear();
  if (dist) dist->clear();
  for (auto &o : order) {
    out.push_back(o.second);
    if (dist) dist->push_back((float)o.first);
  }
}

}  // namespace fr
