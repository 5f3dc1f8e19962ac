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

struct Smem {
  float4 *acc;      // [NV] (re, im, w, origin-touched)
  float4 *pt;       // [side^2] (xx, yy, zz, re)
  float *pim;       // [side^2] im
  int *hits;        // [block]
  float *exp;       // [1000]
  int *wcount;      // [8]
};

// One pass (direct or conjugate targets) of one slice for the thread's column.
// A: column axis (compile time); sg: +1 direct, -1 conjugate.
template <int MODE, int A>
__device__ __forceinline__ void column_pass(const Smem &S, const float *m0, const float *m1, int sg,
                                            const int *base, const int *ext, int px0, int py0,
                                            int PW, int PH, float w, float h) {
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
      const int k0 = max(a0, ta_lo), k1 = min(a0 + K - 1, ta_hi);
      if (k0 > k1) continue;
      const float pim = S.pim[rowoff + x];
      for (int k = k0; k <= k1; k++) {
        int t[3];
        t[A] = k; t[B] = tb; t[C] = tc;
        float vre, vim, vw;
        tap_value<MODE>(t[0], t[1], t[2], pt.x, pt.y, pt.z, pt.w, pim, w, h, S.exp, vre, vim, vw);
        const int la = sg * k + la_off;
        float4 *cell = &S.acc[col_addr + la * str[A]];
        float4 v = *cell;
        if (sg > 0) {
          // direct add; the origin keeps only its real part and is marked
          const bool origin = (t[0] == 0 && t[1] == 0 && t[2] == 0);
          v.x += vre;
          if (origin) v.w = 1.0f;
          else v.y += vim;
          v.z += vw;
        } else {
          if (t[0] == 0 && t[1] == 0 && t[2] == 0) continue;   // the origin adds no conjugate
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
                          float h, int *err) {
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
      const float lo[3] = {base[0] - RLO - kDel, base[1] - RLO - kDel, base[2] - RLO - kDel};
      const float hi[3] = {ext[0] + RHI + kDel, ext[1] + RHI + kDel, ext[2] + RHI + kDel};
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
  // ---- zero the tile accumulators
  for (int i = threadIdx.x; i < NV; i += NT) S.acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
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
      int PW = px1 - px0 + 1, PH = py1 - py0 + 1;
      if (PW > side || PH > side) {
        if (threadIdx.x == 0) atomicOr(err, 2);
        PW = min(PW, side);
        PH = min(PH, side);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < PW * PH; i += NT) {
        const int x = px0 + i % PW, y = py0 + i / PW;
        float4 pt;
        float pim = 0.f;
        if (x > __ldg(&J.xmax[y + n2])) {
          pt = make_float4(1e30f, 1e30f, 1e30f, 0.f);
        } else {
          pixel_coords(__ldg(&J.rtab[x + n2]), __ldg(&J.rtab[y + n2]), M, Nf, pt.x, pt.y, pt.z);
          const float2 v = slice_value(sl, N, x, y);
          pt.w = v.x;
          pim = v.y;
        }
        S.pt[i] = pt;
        S.pim[i] = pim;
      }
      __syncthreads();
      switch (A) {
        case 0: column_pass<MODE, 0>(S, m0, m1, sg, base, ext, px0, py0, PW, PH, w, h); break;
        case 1: column_pass<MODE, 1>(S, m0, m1, sg, base, ext, px0, py0, PW, PH, w, h); break;
        default: column_pass<MODE, 2>(S, m0, m1, sg, base, ext, px0, py0, PW, PH, w, h); break;
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

}  // namespace col

// work[i] = (job, tile, first slice, end slice); blocks are at most `block`.
__global__ void __launch_bounds__(col::NT, 2)
    k_column(const InsertJob *__restrict__ jobs, const int4 *__restrict__ work, int nwork, int block,
             int *counter, const float *__restrict__ exp_g, float h2, float h5, int side, int *err) {
  extern __shared__ float4 s_dyn[];
  __shared__ int s_work;
  __shared__ int s_wcount[col::NT / 32];
  col::Smem S;
  S.acc = s_dyn;
  S.pt = s_dyn + col::NV;
  S.pim = reinterpret_cast<float *>(S.pt + side * side);
  S.hits = reinterpret_cast<int *>(S.pim + side * side);
  S.exp = reinterpret_cast<float *>(S.hits + block);
  S.wcount = s_wcount;
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) S.exp[i] = exp_g[i];
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
      case MODE_GAUSS2: col::tile_item<MODE_GAUSS2>(J, wk.y, s0, s1, S, side, h2, err); break;
      case MODE_GAUSS5: col::tile_item<MODE_GAUSS5>(J, wk.y, s0, s1, S, side, h5, err); break;
      case MODE_NEAREST: col::tile_item<MODE_NEAREST>(J, wk.y, s0, s1, S, side, h2, err); break;
      case MODE_TRILINEAR: col::tile_item<MODE_TRILINEAR>(J, wk.y, s0, s1, S, side, h2, err); break;
      default:
        if (threadIdx.x == 0) atomicOr(err, 4);
    }
  }
}

int column_side(int max_mode) {
  const float r = (max_mode == MODE_GAUSS5 ? 6.0f : max_mode == MODE_NEAREST ? 1.0f : 2.0f) +
                  2 * col::kDel;
  const float e = col::T - 1 + r;
  return (int)std::ceil(std::sqrt(3.0f) * e) + 5;
}

size_t column_smem(int side, int block) {
  return sizeof(float4) * (col::NV + (size_t)side * side) + sizeof(float) * side * side +
         sizeof(int) * block + sizeof(float) * 1000;
}

cudaError_t launch_column(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                          int *d_counter, int max_mode, cudaStream_t st) {
  if (nwork == 0) return cudaSuccess;
  const Consts &c = consts();
  const int side = column_side(max_mode);
  const size_t smem = column_smem(side, block);
  static size_t configured = 0;
  if (configured < smem) {
    cudaFuncSetAttribute(k_column, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    configured = smem;
  }
  cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_column, col::NT, smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = std::max(1, std::min(nwork, sms * per_sm));
  note_launch();
  k_column<<<grid, col::NT, smem, st>>>(d_jobs, d_work, nwork, block, d_counter, c.d_exp, c.h2, c.h5,
                                        side, c.d_err);
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
