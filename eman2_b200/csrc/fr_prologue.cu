// fr_prologue.cu -- per-particle preparation before insertion.
//
// The reference caller (programs/e2spa_make3d.py:300-342) does, per particle:
//   img -= img.get_edge_mean()              (libEM/emdata_metadata.cpp:713-735)
//   img.clip_inplace(Region(...,pad,pad))   zero fill (libEM/emdata.cpp:350)
//   FFT, x CTF_SIGN, IFT                    (libEM/ctf.cpp:1076-1090)
//   img -= img.get_edge_mean()
//   recon.preprocess_slice(img, ts)         (libEM/reconstructor.cpp:1022-1061):
//     bilinear xform (libEM/processor.cpp:11025-11080), phase origin to corner,
//     r2c FFT, x sqrt((N+2)/N)
// Here the FFTs are batched cuFFT plans and everything between them is one
// kernel per stage over all particles of a chunk.
#include <algorithm>
#include <cmath>

#include "fr_device.cuh"
#include "fr_internal.h"

namespace fr {

// Block reduction of a double across 256 threads.
__device__ __forceinline__ double block_sum(double v, double *s_red) {
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += s_red[i];
    s_red[0] = t;
  }
  __syncthreads();
  const double r = s_red[0];
  __syncthreads();
  return r;
}

// EMData::get_edge_mean, 2-D branch: sums of (top+bottom) and (left+right)
// pairs, each pair added in float, accumulated in double; then
// (float)sum / (2nx + 2ny) in float.  Values are v*scale as stored after a
// do_ift (scale = 1/N^2) or v (scale = 1).
__device__ float edge_mean_dev(const float *img, int nx, int ny, float scale, double *s_red) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    const float a = __fmul_rn(img[i], scale), b = __fmul_rn(img[(size_t)(ny - 1) * nx + i], scale);
    acc += (double)__fadd_rn(a, b);
  }
  for (int r = threadIdx.x; r < ny; r += blockDim.x) {
    const float a = __fmul_rn(img[(size_t)r * nx], scale), b = __fmul_rn(img[(size_t)r * nx + nx - 1], scale);
    acc += (double)__fadd_rn(a, b);
  }
  const double s = block_sum(acc, s_red);
  return __fdiv_rn((float)s, (float)(nx * 2 + ny * 2));
}

// Edge-mean subtract and zero-padded clip of box x box raw particles to N x N.
// Particle p's raw image is raw[p] (contiguous images), or src[p] when a
// per-particle table is given (the particles of several jobs in one launch).
// grid.x = particle; the grid.y blocks of a particle share its pixels (each
// forms the same edge mean).  With rot, block (p, 0) also composes the
// particle's symmetry copies, t3d[p*nsym+q] = rot[p] * sym[q] (with psym:
// the particle's own operators, from its first slice on)
// (libEM/transform.cpp:1384-1395), in float with the products and sums
// rounded in that order.
__global__ void __launch_bounds__(256) k_pad(const float *__restrict__ raw,
                                             const float *const *__restrict__ src_tab, int box,
                                             int N, float *__restrict__ out,
                                             const float *__restrict__ rot,
                                             const float *__restrict__ sym, int nsym,
                                             float *__restrict__ t3d,
                                             const PartSym *__restrict__ psym) {
  __shared__ double s_red[8];
  const int p = blockIdx.x;
  if (rot && blockIdx.y == 0) {
    const float *sy = sym;
    int ns = nsym;
    size_t s0 = (size_t)p * nsym;
    if (psym) {
      const PartSym ps = psym[p];
      sy = ps.sym;
      ns = ps.nsym;
      s0 = (size_t)ps.slice0;
    }
    for (int t = threadIdx.x; t < ns * 9; t += blockDim.x) {
      const int q = t / 9, e = t % 9, i = e / 3, j = e % 3;
      const float *a = rot + 9 * (size_t)p;
      const float *b = sy + 9 * q;
      float v = __fmul_rn(a[3 * i + 0], b[j]);
      v = __fadd_rn(v, __fmul_rn(a[3 * i + 1], b[3 + j]));
      v = __fadd_rn(v, __fmul_rn(a[3 * i + 2], b[6 + j]));
      t3d[(s0 + q) * 9 + e] = v;
    }
  }
  const float *src = src_tab ? src_tab[p] : raw + (size_t)p * box * box;
  const float mean = edge_mean_dev(src, box, box, 1.0f, s_red);
  // Region origin (box - N) // 2 (Python floor division).
  const int o = (box - N) >= 0 ? (box - N) / 2 : -((N - box + 1) / 2);
  float *dst = out + (size_t)p * N * N;
  // (row, column) of i carried along the stride instead of divided out
  const int stride = gridDim.y * blockDim.x, dy = stride / N, dx = stride % N;
  int i = blockIdx.y * blockDim.x + threadIdx.x;
  int y = i / N, x = i % N;
  for (; i < N * N; i += stride) {
    const int sy = y + o, sx = x + o;
    float v = 0.0f;
    if (sy >= 0 && sy < box && sx >= 0 && sx < box) v = __fsub_rn(src[(size_t)sy * box + sx], mean);
    dst[i] = v;
    x += dx;
    y += dy;
    if (x >= N) { x -= N; y++; }
  }
}

cudaError_t launch_pad_compose(const float *d_raw, const float *const *d_src, int n, int box, int N,
                               float *d_img, const float *d_rot, const float *d_sym, int nsym,
                               float *d_t3d, cudaStream_t st, const PartSym *d_psym) {
  if (n == 0) return cudaSuccess;
  // few particles: several blocks each, so the launch still fills the device
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int parts = std::max(1, std::min(16, (16 * sms + n - 1) / n));
  note_launch();
  k_pad<<<dim3(n, parts), 256, 0, st>>>(d_raw, d_src, box, N, d_img, d_rot, d_sym, nsym, d_t3d,
                                        d_psym);
  return cudaGetLastError();
}

// Util::hypot_fast value: std::hypot(float,float) of small integers, which
// glibc evaluates as a double square root rounded once to float.
__device__ __forceinline__ float hypot_int(int x, int y) {
  return (float)sqrt((double)(x * x + y * y));
}

// x CTF_SIGN(defocus) on r2c spectra (n, N, N/2+1).  The per-particle
// constants (g1, g2, acac, ds) are formed on the host exactly as
// EMAN2Ctf::compute_2d_complex forms them; the sign of cos(gam - acac) is
// taken from a double cosine of the float argument, which is the sign the
// correctly rounded float cosine returns.
struct CtfDev { float g1, g2, acac, ds, defocus, dfdiff, dfang, on; };

// Blocks of 256 threads per particle for a launch over n particles of npx
// elements each: about `waves` blocks per SM in all, at most one element
// per thread.  Few particles get many blocks each; many get one.
static int blocks_per_particle(int n, int npx, int waves) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long want = ((long)waves * sms + n - 1) / n;
  return (int)std::max(1L, std::min<long>(want, (npx + 255) / 256));
}

// One spectrum element i = r*(N/2+1) + x of a particle: x CTF_SIGN at its
// frequency.
__device__ __forceinline__ void flip_one(cufftComplex *__restrict__ spec, const CtfDev &k, int N,
                                         int i, int r, int x) {
  const int y = r < N / 2 ? r : r - N;
  const float s = __fmul_rn(hypot_int(x, y), k.ds);
  float gam;
  const float t1 = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(-k.g1, s), s), s), s);
  if (k.dfdiff == 0.0f) {
    gam = __fadd_rn(t1, __fmul_rn(__fmul_rn(__fmul_rn(k.g2, k.defocus), s), s));
  } else {
    const float ang = atan2f((float)y, (float)x);
    const double a2 = (double)__fmul_rn(2.0f, ang) - 2.0 * 3.14159265358979323846 / 180.0f * (double)k.dfang;
    const float df = (float)((double)k.defocus + (double)(k.dfdiff / 2.0f) * cos(a2));
    gam = __fadd_rn(t1, __fmul_rn(__fmul_rn(__fmul_rn(k.g2, df), s), s));
  }
  const double v = cos((double)__fsub_rn(gam, k.acac));
  const float sg = v < 0.0 ? -1.0f : 1.0f;
  cufftComplex z = spec[i];
  z.x = __fmul_rn(z.x, sg);
  z.y = __fmul_rn(z.y, sg);
  spec[i] = z;
}

// grid.y = particle; the grid.x blocks of a particle stride over its
// N*(N/2+1) spectrum.
__global__ void k_ctf_flip(cufftComplex *__restrict__ spec, const CtfDev *__restrict__ c, int N) {
  const int w = N / 2 + 1;
  const int p = blockIdx.y;
  const CtfDev k = c[p];
  if (k.on == 0.0f) return;
  // (row, column) of i carried along the stride instead of divided out
  const int stride = gridDim.x * blockDim.x, dr = stride / w, dx = stride % w;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int r = i / w, x = i % w;
  for (; i < N * w; i += stride) {
    flip_one(spec + (size_t)p * N * w, k, N, i, r, x);
    x += dx;
    r += dr;
    if (x >= w) { x -= w; r++; }
  }
}

cudaError_t launch_ctf_flip_dev(cufftComplex *d_spec, const void *d_ctf, int n, int N,
                                cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const int w = N / 2 + 1;
  dim3 grid(blocks_per_particle(n, N * w, 8), n);
  note_launch();
  k_ctf_flip<<<grid, 256, 0, st>>>(d_spec, reinterpret_cast<const CtfDev *>(d_ctf), N);
  return cudaGetLastError();
}

// Host-side CTF constants, mirroring EMAN2Ctf::compute_2d_complex
// (libEM/ctf.cpp:985-992), EMAN2Ctf::lambda (libEM/ctf.h:290-294) and
// EMAN2Ctf::get_phase (libEM/ctf.cpp:671-675).
void ctf_constants(float defocus, float dfdiff, float dfang, float voltage, float cs, float apix,
                   float ampcont, int N, void *out) {
  CtfDev &k = *reinterpret_cast<CtfDev *>(out);
  volatile float lam = 12.2639f / sqrtf(voltage * 1000.0f + 0.97845f * voltage * voltage);
  k.ds = 1.0f / (apix * N);
  k.g1 = (float)(M_PI / 2.0 * cs * 1.0e7 * powf(lam, 3.0f));
  k.g2 = (float)(M_PI * lam * 10000.0);
  float phase;
  if (ampcont > -100.0 && ampcont <= 100.0) phase = (float)asin(ampcont / 100.0);
  else if (ampcont > 100.0) phase = (float)(M_PI - asin(2.0f - ampcont / 100.0));
  else phase = (float)(-M_PI - asin(-2.0 - ampcont / 100.0));
  k.acac = (float)(M_PI / 2.0 - phase);
  k.defocus = defocus;
  k.dfdiff = dfdiff;
  k.dfang = dfang;
  k.on = fabsf(defocus) > 1e-4f ? 1.0f : 0.0f;
}
size_t ctf_dev_size() { return sizeof(CtfDev); }

// Per-particle image source after the optional CTF round trip: particles
// whose phase flip ran read the c2r output (img_on, scaled by 1/N^2 as do_ift
// scales it); the others read the padded image unchanged (img_off, scale 1).
struct SrcSel {
  const float *img_off, *img_on;
  const CtfDev *ctf;   // may be null: every particle reads img_off
  float inv_n2;
  __device__ __forceinline__ const float *img(int p, size_t stride) const {
    return ((ctf && ctf[p].on != 0.0f) ? img_on : img_off) + (size_t)p * stride;
  }
  __device__ __forceinline__ float scale(int p) const {
    return (ctf && ctf[p].on != 0.0f) ? inv_n2 : 1.0f;
  }
};


// src(k) = (v_k * scale_in) - mean: the image after do_ift's scaling and the
// second edge-mean subtraction.
__device__ __forceinline__ float src_at(const float *img, size_t k, float scale_in, float mean) {
  return __fsub_rn(__fmul_rn(img[k], scale_in), mean);
}

// Bilinear translation (TransformProcessor::transform, 2-D real branch) by the
// inverse translation (tx, ty), then phase origin to corner, then x scale_out
// (the sqrt((N+2)/N) factor, applied before the r2c instead of after it).
// txy == nullptr or |t| < 1e-6 (Transform::is_identity) copies.
// fuse_mean: each block forms its particle's edge mean itself (the same
// partition and summation order in every block, so the same value) instead
// of reading mean[p].  grid.y = particle; the grid.x blocks of a particle
// stride over its N*N pixels, so the edge-mean reduction is paid once per
// block, not once per 256 pixels.
__global__ void __launch_bounds__(256) k_shift_corner(SrcSel sel, const float *__restrict__ mean,
                                                      const float *__restrict__ txy,
                                                      int txy_stride, int N, float scale_out,
                                                      float *__restrict__ out, int fuse_mean) {
  __shared__ double s_red[8];
  const int p = blockIdx.y;
  const float *src = sel.img(p, (size_t)N * N);
  const float scale_in = sel.scale(p);
  const float m = fuse_mean ? edge_mean_dev(src, N, N, scale_in, s_red) : (mean ? mean[p] : 0.0f);
  float tx = 0.f, ty = 0.f;
  if (txy) { tx = txy[(size_t)p * txy_stride]; ty = txy[(size_t)p * txy_stride + 1]; }
  const bool copy = fabsf(tx) < 1e-6f && fabsf(ty) < 1e-6f;
  const int h = N / 2;
  // (row, column) of i carried along the stride instead of divided out
  const int stride = gridDim.x * blockDim.x, dyo = stride / N, dxo = stride % N;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int yo = i / N, xo = i % N;
  for (; i < N * N; i += stride, xo += dxo, yo += dyo) {
    if (xo >= N) { xo -= N; yo++; }
    // phase origin to corner (even N): out[y][x] = in[(y+N/2)%N][(x+N/2)%N]
    const int j = (yo + h) % N, ii = (xo + h) % N;
    float v;
    if (copy) {
      v = src_at(src, (size_t)j * N + ii, scale_in, m);
    } else {
      const float cx = (float)(ii - h), cy = (float)(j - h);
      const float sx = __fadd_rn(__fadd_rn(__fmul_rn(1.0f, cx), __fmul_rn(0.0f, cy)), tx);
      const float sy = __fadd_rn(__fadd_rn(__fmul_rn(0.0f, cx), __fmul_rn(1.0f, cy)), ty);
      const float x2 = __fadd_rn(sx, (float)h), y2 = __fadd_rn(sy, (float)h);
      if (x2 < 0 || x2 >= N || y2 < 0 || y2 >= N) {
        v = 0.0f;
      } else {
        const int ix = (int)x2, jy = (int)y2;
        int k0 = ix + jy * N, k1 = k0 + 1, k2 = k0 + N, k3 = k0 + N + 1;
        if (ix == N - 1) { k1--; k3--; }
        if (jy == N - 1) { k2 -= N; k3 -= N; }
        const float t = __fsub_rn(x2, (float)ix), u = __fsub_rn(y2, (float)jy);
        const float p1 = src_at(src, k0, scale_in, m), p2 = src_at(src, k1, scale_in, m);
        const float p3 = src_at(src, k2, scale_in, m), p4 = src_at(src, k3, scale_in, m);
        const float omt = __fsub_rn(1.0f, t), omu = __fsub_rn(1.0f, u);
        float a = __fmul_rn(__fmul_rn(omt, omu), p1);
        a = __fadd_rn(a, __fmul_rn(__fmul_rn(t, omu), p2));
        a = __fadd_rn(a, __fmul_rn(__fmul_rn(omt, u), p3));
        a = __fadd_rn(a, __fmul_rn(__fmul_rn(t, u), p4));
        v = a;
      }
    }
    out[(size_t)p * N * N + i] = __fmul_rn(v, scale_out);
  }
}

cudaError_t launch_shift_corner(const float *d_img_off, const float *d_img_on, const void *d_ctf,
                                const float *d_mean, const float *d_txy, int txy_stride, int n,
                                int N, float scale_out, float *d_out, cudaStream_t st,
                                bool fuse_mean) {
  if (n == 0) return cudaSuccess;
  SrcSel sel{d_img_off, d_img_on, reinterpret_cast<const CtfDev *>(d_ctf),
             1.0f / ((float)N * (float)N)};
  // with the edge mean formed per block, about two blocks per SM in all
  dim3 grid(blocks_per_particle(n, N * N, fuse_mean ? 2 : 8), n);
  note_launch();
  k_shift_corner<<<grid, 256, 0, st>>>(sel, d_mean, d_txy, txy_stride, N, scale_out, d_out,
                                       fuse_mean ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace fr
