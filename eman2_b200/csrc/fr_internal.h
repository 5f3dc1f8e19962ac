// fr_internal.h -- host/device structures and launcher declarations shared by
// the library's translation units.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace fr {

// Per-size geometry tables, built on the host with the reference's own
// scalar arithmetic and kept on the device.
struct Geom {
  int N = 0;
  int corners = 0;           // 1: no radius cut; 2: the Wiener reconstructor's rn < 0.5 disk;
                             // 3: the iterative reconstructor's r <= N/2 + 3 disk
  int *d_xmax = nullptr;     // [N]: largest x kept in row y (index y+N/2), -1 none
  float *d_rtab = nullptr;   // [N+2]: (float)i/(float)N for i in [-N/2, N/2+1]
  int *d_rim = nullptr;      // rim pixels (x | (y+N/2)<<16) that can reach the cube faces
  int nrim = 0;
  int npix = 0;              // kept pixels per slice
  std::vector<int> xmax;     // host copy
};

// Gather tile shapes (the autotuner picks one of these by index).
struct TileShape { int tx, ty, tz; };
constexpr int kNumTiles = 4;
extern const TileShape kTiles[kNumTiles];

// One reconstruction's view for the insertion kernels.
struct InsertJob {
  float *data;               // [N][N][N+2]
  float *norm;               // [N][N][N/2+1]
  const float2 *slices;      // [np][N][N/2+1]
  const float *t3d;          // [np*nsym][9]
  const float *pw;           // [np] weight per particle
  const int *xmax;
  const float *rtab;
  const int *rim;
  int nrim;
  const float *wsnr;         // optional [np][nwsnr] ctf_snr_total curves (wiener_fourier)
  const int *wundo;          // optional [np]: the slice is Wiener filtered, undo it
  int nwsnr;
  const float *ref;          // FourierIterReconstructor's reference volume [N][N][N+2] or null
  const float *ssnr;         // optional [np][nssnr] class_ssnr tables (usessnr)
  int nssnr;
  float sscale;              // 2*(nssnr-1)/N (libEM/reconstructor.cpp:1162)
  int N, mode, nsym, np;
  int tiles_x, tiles_y, tiles_z;
  int nz;                    // the volume's z size when it differs from N (scatter only); 0: N
};

// Launch accounting (fr_api.cu).
void note_launch(int n = 1);
cudaError_t zero_counter(int *d_counter, cudaStream_t st);
// Raises kernel func's dynamic shared-memory limit on the current device to
// at least smem bytes (the attribute is per device; set once per size).
cudaError_t set_max_smem(const void *func, size_t smem);
long long launches_noted();

// fast_exp(-r*h) as a function of r: the table index is monotone in r, so
// it is a step function with thresholds R_k.  Bins of width 1/K (K a power
// of two, so floor(r*K) is exact) hold at most one threshold each; an entry
// is (threshold, weight below it, weight from it on, unused).  r >= rout
// leaves the table (the reference's exp() branch).
struct ExpSteps {
  float4 *d_bins = nullptr;
  int nbins = 0;
  float K = 0, rout = 0;
};

struct Consts {
  float *d_exp = nullptr;    // Util::fast_exp table [1000]
  float h2 = 0, h5 = 0;      // 1/I2G, 1/I5G as the reference forms them
  int *d_err = nullptr;      // device error word
  ExpSteps steps2, steps5;   // gauss_2 and gauss_5 step tables
};
Consts &consts();            // lazily initialised on the current device

// Builds (or fetches) the geometry for size N.
Geom *get_geom(int N, int corners);

// Launchers (fr_insert.cu).  All enqueue on `st`.
cudaError_t launch_compose(const float *d_arg, const float *d_sym, int np, int nsym, float *d_t3d,
                           cudaStream_t st);
cudaError_t launch_scatter(const InsertJob &j, cudaStream_t st);
cudaError_t launch_gather(const InsertJob *d_jobs, const InsertJob *h_jobs, int njobs,
                          const int2 *d_work, int nwork, int tile, int *d_counter, int max_mode,
                          cudaStream_t st);
cudaError_t launch_edge(const InsertJob &j, cudaStream_t st);
cudaError_t launch_scatter_tables(const InsertJob &j, const float *table, float h,
                                  cudaStream_t st);
// Scatter (edge_only: face taps of the rim pixels) of several jobs in one
// launch: units[u] = (job index in d_jobs, slice), max_px = the largest pixel
// (or rim) count of those jobs.
cudaError_t launch_scatter_multi(const InsertJob *d_jobs, const int2 *d_units, int nunits,
                                 int max_px, bool edge_only, cudaStream_t st);
// Column-owner kernel (fr_column.cu): 16^3 tiles, work items (job, tile,
// first slice, end slice) over slice blocks of at most kColumnBlock.
constexpr int kColumnTile = kNumTiles;   // tile id selecting the column kernel
constexpr int kColumnBlock = 1024;       // largest slice block (shared-memory hit list)
// Slices per bucket of the column kernels' work order: the CTAs in flight
// work through one bucket at a time.  Sized so a bucket holds about 176 MB of
// distinct slice data (the nsym copies of a particle share its slice): at
// N = 384, d7 (4096 slices) the measured DRAM traffic of a 2048-particle
// launch is 4.6 GB against 12.8 GB for 1024-slice buckets and 26.8 GB for
// tile-major order.  A power of two, at least the largest block.
inline int slice_bucket(int N, int nsym) {
  const double slice_bytes = 8.0 * (N / 2 + 1) * N;
  const double want = 176e6 / slice_bytes * nsym;
  int b = kColumnBlock;
  while (2.0 * b <= want && b < (1 << 20)) b *= 2;
  return b;
}
// Slices per work item for a tile whose nearest cell is `dist` voxels from the
// origin: every slice meets the centre tiles, so their FP32 chains in shared
// memory are kept short; far tiles meet few slices and take long blocks.
inline int column_block(double dist) {
  return dist < 16 ? 64 : dist < 32 ? 128 : dist < 64 ? 256 : kColumnBlock;
}
cudaError_t launch_column(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                          int *d_counter, int max_mode, cudaStream_t st);
void column_tiles(int N, int mode, int corners, std::vector<int> &out, int &tx, int &ty, int &tz,
                  std::vector<float> *dist = nullptr);
// The barrier-free column kernel (no patch staging; hits grouped by axis).
constexpr int kColumn3Tile = kNumTiles + 1;
// The pixel-major kernel for windows one or two taps wide (nearest,
// gauss_2, trilinear); gauss_5 jobs given this id take k_column3.
constexpr int kPixelTile = kNumTiles + 2;
cudaError_t launch_pixel(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                         int *d_counter, int maxN, cudaStream_t st);
// The kernel a job of this mode runs for a requested tile id.
inline int effective_tile(int tile, int mode) {
  return (tile == kPixelTile && mode == 5 /* gauss_5 */) ? kColumn3Tile : tile;
}
inline bool is_column_tile(int tile) {
  return tile == kColumnTile || tile == kColumn3Tile || tile == kPixelTile;
}
cudaError_t launch_column3(const InsertJob *d_jobs, const int4 *d_work, int nwork, int block,
                           int *d_counter, int maxN, cudaStream_t st);
// Ordered work list (tile ids of a job that can receive interior taps).
void gather_tiles(int N, int mode, int tile, int corners, std::vector<int> &out, int &tx, int &ty,
                  int &tz);

// Prologue (fr_prologue.cu).
// Symmetry composition per particle, for a launch over the particles of
// several jobs: the particle's job's operators, their count and the
// particle's first slice in the launch's rotation blocks.
struct PartSym {
  const float *sym;
  int nsym, slice0;
};
// Edge-mean subtraction and zero-pad clip of n raw images of size box to N
// (from d_raw, or particle p from d_src[p] when a device pointer table is
// given) and, in the same launch, the rotation composition launch_compose does.
cudaError_t launch_pad_compose(const float *d_raw, const float *const *d_src, int n, int box, int N,
                               float *d_img, const float *d_rot, const float *d_sym, int nsym,
                               float *d_t3d, cudaStream_t st, const PartSym *d_psym = nullptr);
void ctf_constants(float defocus, float dfdiff, float dfang, float voltage, float cs, float apix,
                   float ampcont, int N, void *out);
size_t ctf_dev_size();
cudaError_t launch_ctf_flip_dev(cufftComplex *d_spec, const void *d_ctf, int n, int N,
                                cudaStream_t st);
// Shift, phase origin to corner and scale of n images of size N.  fuse_mean:
// each block forms its particle's edge mean from the selected image (the
// same value in every block) instead of reading d_mean.
cudaError_t launch_shift_corner(const float *d_img_off, const float *d_img_on, const void *d_ctf,
                                const float *d_mean, const float *d_txy, int txy_stride, int n,
                                int N, float scale_out, float *d_out, cudaStream_t st,
                                bool fuse_mean = false);

// Finish / agreement (fr_finish.cu).
// nz: the volume's z size (0: N, the cubic volume).
cudaError_t launch_normalize(float *d_data, float *d_norm, int N, int sqrtnorm, cudaStream_t st,
                             float wfilt = 0.0f, int nz = 0);
cudaError_t launch_depad_center(const float *d_real_padded, int N, float scale, float *d_out,
                                cudaStream_t st, int nz = 0);
cudaError_t launch_tocorner3(const float *d_in, int N, float *d_out, cudaStream_t st);
cudaError_t launch_kernel_fix(float *d_vol, int nx, int ny, int nz, float gauss_width,
                              cudaStream_t st);
cudaError_t launch_finish_out(const float *d_real_padded, int N, float scale, float gauss_width,
                              int onx, int ony, int onz, float *d_out, cudaStream_t st);
cudaError_t launch_seed(const float *d_seed, float w, int N, float *d_data, float *d_norm,
                        cudaStream_t st);
cudaError_t launch_agree_rt(const float *d_data, const float *d_norm, int N, const float *d_slices,
                            const float *d_t3d, int np, int nsym, const float *d_w, float apix,
                            const float *d_rtab, float *d_out, cudaStream_t st);
cudaError_t launch_projection_rt(const float *d_data, const float *d_norm, int N,
                                 const float *d_rot, const float *d_rtab, float *d_out,
                                 cudaStream_t st);
cudaError_t launch_proj_shift(float *d_out, int N, float tx, float ty, int checker, int c2r_prep,
                              cudaStream_t st);
cudaError_t launch_scale(const float *d_in, size_t n, float scale, float *d_out, cudaStream_t st);

// Host-side symmetry (Symmetry3D::get_symmetries for c<n>, d<n>, tet, oct,
// icos): the operator count, or -1 for an unknown name or an order beyond
// kMaxSymOps operators.
constexpr int kMaxSymOps = 1000;
int sym_ops(const std::string &sym, std::vector<float> &out);
void eman_matrix(double az, double alt, double phi, float *m);

}  // namespace fr
