/*
 * eman2_b200.h -- C ABI of the B200 direct Fourier inversion library
 * (libeman2_b200.so).  Plain pointers and sizes; no C++ or torch types.
 *
 * The library replaces EMAN2's FourierReconstructor behind
 * Reconstructors.get("fourier", {...}) (libEM/reconstructor.h:388-565,
 * libEM/reconstructor.cpp:686-1641) and its Python binding
 * (libpyEM/libpyReconstructor2.cpp:50-86,192-226).  Every entry point names
 * the reference interface it stands in for.
 *
 * Volumes use the reference's layout:
 *   complex volume : float[N][N][N+2]   (z, y, x-interleaved re/im, x = 0..N/2)
 *   weight volume  : float[N][N][N/2+1]
 *   slice          : float[N][N+2]      (r2c spectrum of an N x N image)
 * Pointers may be host or device memory; the library detects which.
 * All functions return FR_OK (0) or an FR_E* status; fr_last_error() gives
 * the message of the calling thread's last failure.
 */
#ifndef EMAN2_B200_H
#define EMAN2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FR_API __attribute__((visibility("default")))

/* Status codes; the Python layer raises the reference's exception class of
 * the same meaning (libEM/exception.h). */
enum {
  FR_OK = 0,
  FR_EINVAL_PARAM = 1,   /* InvalidParameterException (libEM/emobject.h:931-938) */
  FR_EDIM = 2,           /* ImageDimensionException (libEM/reconstructor.cpp:767,861) */
  FR_ENULL = 3,          /* NullPointerException (libEM/reconstructor.cpp:1067) */
  FR_ESTATE = 4,         /* used before setup() or after finish() */
  FR_ECUDA = 5,          /* CUDA / cuFFT runtime failure */
  FR_ENOMEM = 6,         /* device allocation failed */
  FR_EUNSUPPORTED = 7,   /* parameter value outside the built scope */
  FR_ENOTEXIST = 8,      /* NotExistingObjectException (libEM/emdata_metadata.cpp:1142) */
  FR_EDEVICE = 9         /* a kernel reported an internal consistency error */
};

/* Inserter modes (FourierPixelInserter3D factory names,
 * libEM/reconstructor_tools.cpp:42-53). */
enum {
  FR_MODE_NEAREST = 1,   /* "nearest_neighbor" */
  FR_MODE_GAUSS2 = 2,    /* "gauss_2" (default) */
  FR_MODE_GAUSS5 = 5,    /* "gauss_5" */
  FR_MODE_TRILINEAR = 6, /* "trilinear" */
  FR_MODE_ITER = 7       /* FourierIterReconstructor ("fourier_iter") insertion */
};

/* Insertion schedules. */
enum {
  FR_SCHED_AUTO = 0,     /* pick by batch size and mode */
  FR_SCHED_SCATTER = 1,  /* one thread per slice pixel, FP32 atomics */
  FR_SCHED_GATHER = 2    /* voxel tiles own their cells; no atomics */
};

/* FourierReconstructor parameters (libEM/reconstructor.h:501-516). */
typedef struct {
  int nx, ny, nz;        /* "size": padded real-space volume, even sizes with nx == ny
                            (square slices); nz != nx takes the scatter insertion and
                            has no batched forms, agreement, projection or seeds */
  int mode;              /* FR_MODE_* */
  char sym[16];          /* "c<n>", "d<n>", "tet", "oct", "icos" */
  int corners;           /* "corners" */
  int sqrtnorm;          /* "sqrtnorm" */
  int usessnr;           /* "usessnr" */
  int verbose;           /* "verbose" */
} fr_params;

/* Per-particle metadata for the batched caller pipeline
 * (programs/e2spa_make3d.py:300-345). */
typedef struct {
  float rot[9];          /* xform.projection rotation block, row-major */
  float tx, ty;          /* xform.projection translation */
  float weight;          /* insertion weight (<= 0: particle skipped) */
  float defocus;         /* um; |defocus| <= 1e-4 disables the phase flip */
  float dfdiff, dfang;   /* astigmatism */
  float voltage, cs;     /* kV, mm */
  float apix;            /* A/pixel */
  float ampcont;         /* amplitude contrast, percent */
} fr_particle;

typedef struct fr_recon fr_recon;

/* Factory<Reconstructor>::get("fourier", params) + set_params
 * (libpyEM/libpyReconstructor2.cpp:221-226, libEM/emobject.h:916-938). */
FR_API int fr_create(const fr_params *p, fr_recon **out);

/* ~FourierReconstructor (libEM/reconstructor.h:400). */
FR_API int fr_destroy(fr_recon *r);

/* Binds the handle to an existing CUDA stream (cudaStream_t); 0 restores the
 * handle's own stream.  Insertion calls (fr_insert_slices,
 * fr_insert_particles and the batched forms) return once their work is
 * enqueued on that stream, after copying any host inputs; device inputs must
 * stay valid until the stream reaches that point.  A call on another stream
 * first waits for the handle's earlier work.  Calls that return results
 * (agreement, accumulators, finish) synchronise. */
FR_API int fr_set_stream(fr_recon *r, void *stream);

/* The stream the handle's work goes to (cudaStream_t), for callers that
 * order their own work against it.  No counterpart in the reference. */
FR_API int fr_get_stream(const fr_recon *r, void **stream);

/* FourierReconstructor::setup (libEM/reconstructor.cpp:730-818). */
FR_API int fr_setup(fr_recon *r);

/* FourierReconstructor::setup_seed (libEM/reconstructor.cpp:820-902):
 * data = seed * seed_weight, weights = seed_weight (halved on the x=0 and
 * x=Nyquist planes, four cells kept whole). seed: float[N][N][N+2]. */
FR_API int fr_setup_seed(fr_recon *r, const float *seed, float seed_weight);

/* FourierReconstructor::setup_seedandweights (libEM/reconstructor.cpp:904-996). */
FR_API int fr_setup_seedandweights(fr_recon *r, const float *seed, const float *weights);

/* FourierReconstructor::clear (libEM/reconstructor.cpp:999-1020). */
FR_API int fr_clear(fr_recon *r);

/* FourierReconstructor::preprocess_slice (libEM/reconstructor.cpp:1022-1061)
 * for n real N x N images and translation-only transforms whose inverse
 * translates by inv_txy[2*i], inv_txy[2*i+1] (the reference applies the
 * inverse of the transform it is given, libEM/processor.cpp:11029).
 * Writes n slices float[N][N+2]. */
FR_API int fr_preprocess_slices(fr_recon *r, const float *imgs, int n, const float *inv_txy,
                                float *out_slices);

/* FourierReconstructor::insert_slice (libEM/reconstructor.cpp:1064-1119) for
 * n preprocessed slices float[N][N+2] with rotation blocks rot[9*n] and
 * weights[n].  status_out[i] (optional) receives insert_slice's return
 * value (0, or -1 when the weight is 0).  ssnr (optional, nssnr entries per
 * slice) carries class_ssnr for usessnr=1. */
FR_API int fr_insert_slices(fr_recon *r, const float *slices, int n, const float *rot,
                            const float *weights, const float *ssnr, int nssnr,
                            int *status_out, int schedule);

/* The reference caller's per-particle loop (programs/e2spa_make3d.py:300-345):
 * edge-mean subtract, clip to N, CTF phase flip, edge-mean subtract,
 * preprocess_slice with the inverted translation, insert_slice.  imgs:
 * float[n][box][box]. */
FR_API int fr_insert_particles(fr_recon *r, const float *imgs, int n, int box,
                               const fr_particle *meta, int schedule);

/* FourierReconstructor::determine_slice_agreement (libEM/reconstructor.cpp:1212-1257)
 * for n preprocessed slices.  out[5*i..] = reconstruct_norm, _absqual,
 * _absqual_lowres, _qual, _weight.  apix: the slices' apix_x.  sub=1 needs
 * usessnr with class_ssnr (as in the reference). */
FR_API int fr_determine_slice_agreement(fr_recon *r, const float *slices, int n,
                                        const float *rot, const float *weights, float apix,
                                        int sub, float *out);

/* FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1445) of
 * the current accumulators.  xf: the Transform as its 3x4 matrix (float[12],
 * row-major: rotation block and the translation column xf[3], xf[7],
 * xf[11]); the slice uses the rotation only and is then shifted by the
 * translation (the xform processor, :1435-1437).  ret_fourier=1: out =
 * float[N][N+2] complex slice; ret_fourier=0: phase origin to the centre and
 * the inverse FFT, out = float[N][N] real image. */
FR_API int fr_projection_xf(fr_recon *r, const float *xf, int ret_fourier, float *out);
/* The same for a rotation block rot[9] with no translation, ret_fourier=1:
 * out = float[N][N+2]. */
FR_API int fr_projection(fr_recon *r, const float *rot, float *out_slice);

/* FourierReconstructor::finish (libEM/reconstructor.cpp:1552-1641).
 * doift=1: out = float[N][N][N] real map (inverse FFT, depad, phase origin
 * to centre); doift=0: out = normalised float[N][N][N+2] complex volume.
 * normout (optional) = float[N][N][N/2+1] weights (the "normout" param).
 * The handle needs fr_setup() again afterwards (ownership passes out). */
FR_API int fr_finish(fr_recon *r, int doift, float *out, float *normout);

/* fr_finish without waiting (no counterpart in the reference, whose finish
 * returns the map): the same work is enqueued on `stream` (NULL: the
 * handle's stream) after the handle's earlier work, with out and normout
 * device memory or page-locked host memory (FR_EINVAL_PARAM otherwise), and
 * the call returns once it is enqueued.  The results are complete when the
 * stream reaches this point (an event recorded after the call).  A server
 * retiring a job this way keeps inserting other jobs meanwhile.  Device-side
 * inconsistency codes of earlier insertions are reported by the handle's
 * next synchronous call instead. */
FR_API int fr_finish_async(fr_recon *r, int doift, float *out, float *normout, void *stream);

/* finish(True) followed by what e2make3dpar does with the map
 * (programs/e2make3dpar.py:421-431): the radial kernel correction
 * math.gausskernelfix with gauss_width (MaskGaussInvProcessor,
 * libEM/processor.h:4131-4176; <= 0 skips it) and the clip to the centred
 * outx x outy x outz region (clip_inplace(Region((N-outx)/2, ...))), fused
 * into the pass that writes the real map.  out: float[outz][outy][outx]. */
FR_API int fr_finish_corrected(fr_recon *r, float gauss_width, int outx, int outy, int outz,
                               float *out, float *normout);

/* The processor math.gausskernelfix on a real volume float[nz][ny][nx], host
 * or device, in place (EMData::process_inplace("math.gausskernelfix",
 * {"gauss_width": w}), libEM/processor.h:4131-4176,
 * libEM/processor.cpp:2439-2473).  stream: NULL for the default stream. */
FR_API int fr_kernel_fix(float *vol, int nx, int ny, int nz, float gauss_width, void *stream);

/* Un-normalised accumulators (finish(False) + normout before normalisation);
 * the form the reference's parallel make3d merges (programs/e2spa_make3d.py:175-188).
 * Either pointer may be NULL. */
FR_API int fr_get_accumulators(fr_recon *r, float *data, float *norm);

/* Sizes and state. */
FR_API int fr_get_size(const fr_recon *r, int *N);
FR_API size_t fr_footprint_bytes(int N);

/* Symmetry operators of a symmetry name (Symmetry3D::get_symmetries,
 * libEM/symmetry.cpp:1240-1246) as rotation blocks; returns the count or -1. */
FR_API int fr_sym_ops(const char *sym, float *out, int cap);

/* Launch accounting and insertion-kernel timing.  With profiling on, CUDA
 * events bracket every insertion launch (gather + face taps, or scatter) on
 * the stream it runs on.  No counterpart in the reference (it has no timers
 * on this path). */
typedef struct {
  long long kernel_launches;     /* kernels this library launched (cuFFT's not counted) */
  long long insert_launches;     /* insertion passes (one gather or scatter pass each) */
  long long slices_inserted;     /* particle-slices x symmetry copies inserted */
  double insert_ms;              /* summed event time of the insertion passes */
  double gather_ms;              /* summed event time of the gather kernel alone */
  long long gather_launches;
} fr_stats;
FR_API int fr_profile(int on);
FR_API int fr_stats_get(fr_stats *out);
FR_API int fr_stats_reset(void);

/* Insertion that allocates no device memory, for callers that cannot let a
 * library call cudaMalloc: processes that reserve all of their HBM for their
 * own pool allocator, or paths where an allocation's stall or implicit device
 * synchronisation is not acceptable.  No counterpart in the reference.
 * The caller passes device buffers: n preprocessed slices float[N][N+2],
 * rotation blocks rot[9*n], weights[n], and the accumulators it owns,
 * data float[N][N][N+2] and norm float[N][N][N/2+1], to which the slices'
 * taps are added (atomic scatter, same arithmetic as fr_insert_slices).
 * Scratch (tables, symmetry operators, composed rotations) lives in a static
 * __device__ array of 596 KiB (152,696 floats) inside the library, held by
 * every GPU that loads it until exit.  Limits: even N <= 1024, at most 240 symmetry operators and
 * n * nsym <= 16384 per call; larger requests fail with FR_EINVAL_PARAM.
 * Every buffer must be device memory of the current device (or managed
 * memory); others fail with FR_EINVAL_PARAM.
 * The first call on a device looks up the array's address (with that device
 * current) and uploads the exp table: make that first call before any stream
 * capture (a first call on a capturing stream fails with FR_EINVAL_PARAM).
 * All calls share the array: calls that overlap on the GPU race. */
FR_API int fr_insert_slices_noalloc(const float *d_slices, int n, int N, int mode,
                                    const char *sym, const float *d_rot,
                                    const float *d_weights, float *d_data, float *d_norm,
                                    void *stream);

/* FourierIterReconstructor ("fourier_iter", libEM/reconstructor.cpp:430-682):
 * a handle created with mode FR_MODE_ITER inserts with that class's
 * inserter (gauss_5 window clamped to |x| <= N/2-1, the r <= N/2+3 pixel
 * disk; width 1/(|p|^2/4000+.15) without a reference volume, else width
 * 1/2 and the update dt + ref(i,j,k) - ref(p)); fr_set_reference sets the
 * reference from a seed (setup_seed, :481-488): a complex volume as is, or a
 * real N^3 map after phase origin to corner and an r2c FFT.  fr_setup drops
 * it. */
FR_API int fr_set_reference(fr_recon *r, const float *vol, int is_complex);

/* WienerFourierReconstructor ("wiener_fourier", libEM/reconstructor.cpp:1643-1731,
 * 1921-1947).  fr_set_wiener(r, 1) makes finish divide by (weight + 1)
 * (normalize_threed(sqrtnorm, true), libEM/reconstructor.cpp:376-390).
 * fr_insert_slices_wiener inserts n preprocessed slices whose per-pixel
 * weight is their ctf_snr_total curve (snr[n][nsnr]) interpolated at the
 * pixel radius, inside the rn < 0.5 disk; weights[i] < 0 subtracts;
 * undo[i] != 0 (ctf_wiener_filtered) scales the values by (w+1)/w.
 * Without a curve: FR_ENOTEXIST, as the reference's
 * NotExistingObjectException. */
FR_API int fr_set_wiener(fr_recon *r, int on);
FR_API int fr_insert_slices_wiener(fr_recon *r, const float *slices, int n, const float *rot,
                                   const float *weights, const float *snr, int nsnr,
                                   const int *undo, int *status_out);

/* Last error message of the calling thread. */
FR_API const char *fr_last_error(void);

/* Library version string. */
FR_API const char *fr_version(void);

/* ---------------------------------------------------------------- batched
 * Many independent reconstructions (uneven N, mode, symmetry) inserted by one
 * persistent launch per chunk.  No counterpart in the reference beyond
 * running several FourierReconstructors (even/odd half maps,
 * programs/e2gmm.py:115-139). */
typedef struct fr_batch fr_batch;

/* Creates a batch of njobs reconstructions (each set up as fr_setup). */
FR_API int fr_batch_create(const fr_params *jobs, int njobs, fr_batch **out);
FR_API int fr_batch_destroy(fr_batch *b);
FR_API int fr_batch_set_stream(fr_batch *b, void *stream);

/* Inserts, for every job j, counts[j] particles whose images start at
 * imgs[j] (float[counts[j]][box_j][box_j]) with metadata meta[j].  All jobs'
 * particles go through one prologue pass per box size and one persistent
 * insertion launch. */
FR_API int fr_batch_insert_particles(fr_batch *b, const float *const *imgs, const int *boxes,
                                     const int *counts, const fr_particle *const *meta);

/* The same batched insertion over independent, already set-up handles (each
 * keeps its resident volume): imgs[j], boxes[j], counts[j], meta[j] go to
 * handles[j].  One persistent insertion launch per round of chunks; runs on
 * `stream` (NULL: the first handle's stream).  The serving loop's tick. */
FR_API int fr_insert_particles_multi(fr_recon *const *handles, int nh, const float *const *imgs,
                                     const int *boxes, const int *counts,
                                     const fr_particle *const *meta, void *stream);

/* A batched insertion round of fixed shapes (counts[j] <= 4096 particles of
 * box boxes[j] for handle j; 0 leaves a job out), captured once as a CUDA
 * graph on `stream` (NULL: the first handle's): the prologue (pad, CTF flip
 * pair where ctf[j] is set, edge mean, shift, r2c, rotation composition), run
 * once per group of jobs of equal (N, box) over their particles,
 * the groups as parallel branches; then the insertion launches (per schedule
 * one persistent launch or one scatter over all its jobs) and the face taps.
 * The graph owns the device image slots and the prologue scratch; the
 * handles must outlive it.  No counterpart in the reference. */
typedef struct fr_graph fr_graph;
FR_API int fr_graph_create(fr_recon *const *handles, int nh, const int *boxes, const int *counts,
                           const int *ctf, void *stream, fr_graph **out);
/* The same over a batch's jobs, on the batch stream. */
FR_API int fr_batch_graph_create(fr_batch *b, const int *boxes, const int *counts, const int *ctf,
                                 fr_graph **out);
/* Device slot of job j's images (float[counts[j]][box][box]): a caller may
 * write the particles there and pass imgs = NULL to fr_graph_launch. */
FR_API int fr_graph_slot(fr_graph *g, int job, float **d_images);
/* One replay on the batch stream: meta[j] (counts[j] particles each) and the
 * particles' image addresses are staged through pinned memory and uploaded
 * as one block; device imgs[j] are read in place (unchanged until the replay
 * has run on the stream), host imgs[j] are copied into the slots, NULL reads
 * the slots as filled; then the graph is launched.  Returns once enqueued
 * (after reading host images).  Particles with a CTF need their group to have
 * been captured with the phase flip (ctf[j] set for one of its jobs;
 * FR_EINVAL_PARAM otherwise); particles without one are accepted either way. */
FR_API int fr_graph_launch(fr_graph *g, const float *const *imgs, const fr_particle *const *meta);
FR_API int fr_graph_destroy(fr_graph *g);

/* Finishes job j like fr_finish. */
FR_API int fr_batch_finish(fr_batch *b, int job, int doift, float *out, float *normout);
FR_API int fr_batch_get_accumulators(fr_batch *b, int job, float *data, float *norm);

/* Schedule selection for the insertion, measured on the device with
 * nparticles random slices and cached per (N, mode, nsym): candidates are the
 * register-tile gather shapes 0-3, the staged column kernel (4), the
 * barrier-free column kernel (5), the pixel-major kernel for windows one or
 * two taps wide (6; not for gauss_5) and the atomic scatter (tile_out = -2).
 * ms_out, if not NULL, receives 8 timings in that order (-1: not run).  fr_set_tile pins a
 * choice (-1 clears it).  No counterpart in the reference. */
FR_API int fr_autotune(int N, int mode, int nsym, int nparticles, int *tile_out,
                       float *ms_out);
FR_API int fr_set_tile(int N, int mode, int nsym, int tile);

/* Decodes n raw image values of MRC mode `mode` (0 unsigned bytes, 17 signed
 * bytes, 101 packed 4-bit, 1 int16, 6 uint16, 12 float16, 2 float32; swap:
 * the file's byte order is not the host's) from device bytes into float32,
 * as MrcIO::read_data converts them (libEM/io/mrcio.cpp:1040-1140), so stacks
 * cross PCIe in their stored width.  Asynchronous on `stream`. */
FR_API int fr_decode_images(const void *d_src, int mode, int swap, long long n, float *d_dst,
                            void *stream);

/* Measured roofs of the scattered accumulation, in taps/s (a tap adds a
 * complex value and a weight to one voxel): conflict-free float4
 * read-modify-write in shared memory (the column kernel's update), FP32
 * atomicAdd to random shared-memory words, and FP32 red.global.add to an
 * L2-resident buffer (the scatter schedule's update).  Runs three short
 * microbenchmarks on the current device.  No counterpart in the reference. */
FR_API int fr_update_peaks(double *smem_rmw_taps, double *smem_atom_taps, double *l2_red_taps);

#ifdef __cplusplus
}
#endif
#endif /* EMAN2_B200_H */
