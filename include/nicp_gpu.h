/*
 * nicp_gpu.h -- C ABI of the B200-native NICP registration path.
 *
 * One shared library (libnicp_b200.so, sm_100a) implements the yorsh87/nicp
 * depth -> cloud -> projective-ICP path with hand-written CUDA kernels.  The
 * reference's C++ plugin classes map onto these entry points (the header
 * include/nicp_b200/nicp.hpp re-exposes them under the reference's class
 * names):
 *
 *   reference (file:line inside yorsh87/nicp)            entry point here
 *   -------------------------------------------------------------------------
 *   DepthImageConverterIntegralImage::compute             nicp_cloud_from_depth_u16
 *     (nicp/nicp/depthimageconverterintegralimage.cpp:18-64)  nicp_cloud_from_depth_f32
 *     + DepthImage_convert_16UC1_to_32FC1 (imageutils.cpp:85-99)
 *   PinholePointProjector::unProject                      nicp_unproject
 *     (nicp/nicp/pinholepointprojector.cpp:68-91)
 *   PinholePointProjector::projectIntervals               nicp_project_intervals
 *     (nicp/nicp/pinholepointprojector.cpp:136-148)
 *   PinholePointProjector::project                        nicp_project
 *     (nicp/nicp/pinholepointprojector.cpp:33-66)
 *   PinholePointProjector::_updateMatrices                nicp_projector_matrices
 *     (nicp/nicp/pinholepointprojector.cpp:16-31)
 *   CorrespondenceFinderProjective::compute               nicp_correspond
 *     (nicp/nicp/correspondencefinderprojective.cpp:16-115)
 *   Linearizer::update                                    nicp_linearize
 *     (nicp/nicp/linearizer.cpp:21-134)
 *   AlignerProjective::align (+ Aligner::_computeStatistics)   nicp_align
 *     (nicp/nicp/alignerprojective.cpp:21-136, aligner.cpp:82-135)
 *   Cloud accessors / transformInPlace                    nicp_cloud_download / _upload /
 *     (nicp/nicp/cloud.h:20-193, cloud.cpp:191-204)         nicp_cloud_transform
 *   (no counterpart: many pairs in one device-side loop)  nicp_build_batch / nicp_align_batch
 *
 * Conventions
 *   - Every function returns an int status (NICP_OK on success); the text of
 *     the last failure on a context is nicp_ctx_last_error().  No C++
 *     exception crosses this boundary: a host allocation failure inside a
 *     call returns NICP_ENOMEM (any other exception NICP_ESTATE).
 *   - Matrices are row-major.  Transforms are 4x4 isometries; row 3 is
 *     forced to (0 0 0 1) as the reference does.
 *   - Host buffers are caller-owned; device buffers (clouds, scratch) are
 *     owned by the library.  Calls on one context are ordered on its CUDA
 *     stream; functions that return data in host memory synchronize it.
 *   - Cloud builds from host depth (nicp_cloud_from_depth_*, nicp_build_batch
 *     with on_device 0) return before the frames are copied when nothing is
 *     returned in host memory: keep pinned host frames valid until the
 *     context's stream has passed the call (pageable frames are copied
 *     before the call returns).  The copies run on a second, library-owned
 *     stream that is ordered after earlier work on the context's stream and
 *     before the build kernels that read them.
 *   - There is no CPU fallback: creating a context fails on a host without
 *     an sm_100 GPU.
 *   - A context is not thread-safe: use one per host thread.  Every call
 *     that takes a context (or a cloud of one) runs on the context's device
 *     whatever device the calling thread has current, and leaves the
 *     thread's current device as it found it (nicp_ctx_create and
 *     nicp_ctx_destroy included), so one thread may drive contexts on
 *     several GPUs.  The one exception is nicp_linearize_noalloc, which
 *     switches nothing and refuses a call whose context's device is not
 *     current (NICP_ESTATE).
 *   - A cloud is not thread-safe either: calls that read a cloud may write
 *     out its implicit information matrices (see nicp_cloud_download), so
 *     two threads must not use one cloud at the same time.
 *   - The library's per-device state (kernel attributes set once per
 *     device, the allocation-free linearizer's array address) does not
 *     survive cudaDeviceReset: destroy every context and server first, and
 *     do not use the library on a device after resetting it.
 */
#ifndef NICP_GPU_H
#define NICP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NICP_API_VERSION 2

enum {
  NICP_OK = 0,
  NICP_EINVAL = 1,   /* bad argument (null, size, range)                 */
  NICP_ENOMEM = 2,   /* device or host allocation failed                 */
  NICP_EBUDGET = 3,  /* request exceeds the configured HBM budget        */
  NICP_ETIMEOUT = 4, /* a bounded device-side wait ran out               */
  NICP_ECUDA = 5,    /* CUDA runtime error (text in nicp_ctx_last_error) */
  NICP_ESTATE = 6    /* call not valid in the object's current state     */
};

typedef struct nicp_ctx nicp_ctx;
typedef struct nicp_cloud nicp_cloud;

/* PinholePointProjector state (pinholepointprojector.cpp:5-31,150-155;
 * pointprojector.cpp:6-15,106-112; defaults from those constructors).  The
 * effective camera matrix is (fx, fy, cx, cy) with its first two rows times
 * `scaling`; the projection image is (rows, cols) times `scaling`. */
typedef struct {
  float fx, fy, cx, cy;
  float scaling;
  int rows, cols;
  float min_distance, max_distance;
  float baseline, alpha;
} nicp_camera;

enum { NICP_MOMENTS_F64 = 0, NICP_MOMENTS_F32 = 1, NICP_MOMENTS_TWOFLOAT = 2 };

/* StatsCalculatorIntegralImage (statscalculatorintegralimage.cpp:12-18) and
 * Point/NormalInformationMatrixCalculator (informationmatrixcalculator.h:
 * 22-29,115-119,150-155) settings, plus the depth scale of the u16 input. */
typedef struct {
  float depth_scale;
  float world_radius;
  int min_image_radius, max_image_radius, min_points;
  float curvature_threshold;
  float pim_flat[3], pim_nonflat[3];
  float pim_curvature_threshold;
  float nim_flat[3], nim_nonflat[3];
  float nim_curvature_threshold;
  int moments_precision; /* NICP_MOMENTS_*; F64 is the default */
  int keep_stats;        /* also store eigenvalues/eigenvectors per point */
  /* also store the per-point sensor-noise Gaussian3f (mean + covariance) of
   * PinholePointProjector::unProject(points, gaussians, ...)
   * (pinholepointprojector.cpp:93-134).  The reference always computes it;
   * only the Merger consumes it, so here it is opt-in (0 = off). */
  int keep_gaussians;
} nicp_cloud_params;

/* CorrespondenceFinder(Projective) (correspondencefinder.cpp:9-18). */
typedef struct {
  float inlier_distance_threshold;
  float inlier_normal_angular_threshold; /* cosine, default cosf(M_PI/6) */
  float flat_curvature_threshold;
  float inlier_curvature_ratio_threshold;
  int demoted_to_gicp;
  /* Emulates the reference's OpenMP partition with this many threads:
   * the last rows % T image rows and the last K % T correspondences are
   * skipped exactly as the reference skips them.  1 (default) = no drops. */
  int parity_threads;
  /* CorrespondenceFinderProjective::setRowSearchRegion / setColSearchRegion
   * (correspondencefinderprojective.h:146-150).  0 0 (default): the pixel's
   * own current point (_computeSingle); otherwise every reference pixel
   * takes the best current point of the (2 rows + 1) x (2 cols + 1) window
   * around it (_computeMulti, correspondencefinderprojective.cpp:119-257);
   * the aligner then runs its list path.  At most 16 each. */
  int row_search_region, col_search_region;
} nicp_corr_params;

/* Linearizer (linearizer.cpp:9-19). */
typedef struct {
  float inlier_max_chi2;
  int robust_kernel;
  int z_scaling;
  float scale;
  int demoted_to_gicp;
  /* Precision study: sum the per-tile FP64 partials in FP32 instead of FP64
   * (the reference sums its per-thread float partials in float,
   * linearizer.cpp:119-127).  0 (default) = FP64. */
  int cross_block_f32;
} nicp_lin_params;

/* Aligner (aligner.cpp:21-41) plus the device-loop controls. */
typedef struct {
  int outer_iterations, inner_iterations;
  float lambda;
  int min_inliers;
  float translational_min_eigen_ratio, rotational_min_eigen_ratio;
  int compute_statistics; /* run Aligner::_computeStatistics after the loop */
  /* Stop a pair once the pose change of an outer iteration is below this
   * (max-abs over translation and quaternion-vector parts).  0 = never,
   * which is the reference's behaviour. */
  double early_exit_eps;
} nicp_align_params;

typedef struct {
  double T[16];          /* current -> reference */
  float error;           /* Linearizer::error() of the last inner iteration */
  int inliers;           /* Linearizer::inliers() of the last inner iteration */
  int num_correspondences;
  int outer_iterations_run;
  double translational_ratio, rotational_ratio;
  int solution_valid;    /* -1 when statistics were not computed */
  int status;            /* NICP_OK or a per-pair error */
  /* Aligner::omega() (aligner.h:325, filled at aligner.cpp:108-134): the
   * 6x6 information matrix of the solution in (t, quaternion-vector)
   * coordinates, row-major, symmetrised; Aligner::_mean: the mean of the
   * unscented reconstruction.  Zero when statistics were not computed or
   * the system was singular. */
  double omega[36];
  double mean[6];
} nicp_align_result;

void nicp_default_camera(nicp_camera *c);
void nicp_default_cloud_params(nicp_cloud_params *p);
void nicp_default_corr_params(nicp_corr_params *p);
void nicp_default_lin_params(nicp_lin_params *p);
void nicp_default_align_params(nicp_align_params *p);

/* ------------------------------------------------------------ context */
/* stream: a cudaStream_t to run on, or NULL for a stream the context owns. */
int nicp_ctx_create(int device, void *stream, nicp_ctx **out);
int nicp_ctx_destroy(nicp_ctx *ctx);
const char *nicp_ctx_last_error(const nicp_ctx *ctx);
int nicp_ctx_synchronize(nicp_ctx *ctx);
void *nicp_ctx_stream(nicp_ctx *ctx);
/* Bytes of device memory currently held by the context and its clouds. */
size_t nicp_ctx_device_bytes(const nicp_ctx *ctx);

/* Per-kernel timing with CUDA events on the context stream.  When enabled,
 * every launch of the kernels below is bracketed by events; reading
 * synchronizes and resets the counters. */
enum {
  NICP_K_UNPROJECT = 0, NICP_K_MOMENTS_BANDS, NICP_K_MOMENTS_SWEEP, NICP_K_STATS,
  NICP_K_ZBUFFER, NICP_K_RESOLVE, NICP_K_CORR_LIN, NICP_K_CORR_LIST, NICP_K_LIN_LIST,
  NICP_K_SOLVE, NICP_K_TRANSFORM, NICP_K_COUNT
};
int nicp_ctx_set_profiling(nicp_ctx *ctx, int enable);

/* Autotuner (no reference counterpart).  When enabled, the first alignment
 * call with a new resolution mix (the multiset of pair image sizes, with the
 * iteration counts) times the Gauss-Newton loop with each candidate launch
 * shape -- z-buffer points per thread 1/2/4/8, fused correspondence +
 * linearizer CTAs per SM 2/3/as many as fit -- and keeps the fastest for
 * that mix; the first build of a new frame-size mix likewise times the
 * stats kernel (normals, curvature, information matrices) at 256 x 3,
 * 128 x 6, 64 x 12 and 256 x 2 (threads per CTA x CTAs per SM) and keeps
 * the fastest.  Results do not depend on the launch shapes (bitwise).  The
 * trials run on the context stream before the call's own work and
 * synchronize it once. */
int nicp_ctx_set_autotune(nicp_ctx *ctx, int enable);
/* Launch shape used by the last alignment call (corr_ctas_per_sm 0 = as many
 * as fit), the number of resolution mixes tuned so far, and the stats
 * kernel's shape in the last build.  Any pointer may be NULL. */
int nicp_ctx_launch_shape(const nicp_ctx *ctx, int *zbuffer_points_per_thread, int *corr_ctas_per_sm,
                          int *tuned_mixes, int *stats_threads, int *stats_ctas_per_sm);
/* Kernels this context has launched so far (graph replays included). */
unsigned long long nicp_ctx_kernel_launches(const nicp_ctx *ctx);
/* Host->device and device->host bytes the context has copied so far. */
int nicp_ctx_transfer_bytes(const nicp_ctx *ctx, unsigned long long *h2d, unsigned long long *d2h);
int nicp_ctx_read_profile(nicp_ctx *ctx, int kernel, double *total_ms, int *launches);
const char *nicp_kernel_name(int kernel);

/* --------------------------------------------------------------- clouds */
int nicp_cloud_create(nicp_ctx *ctx, nicp_cloud **out);
int nicp_cloud_destroy(nicp_cloud *c);
/* Number of points (synchronizes). */
int nicp_cloud_size(nicp_cloud *c, int *n);
/* Number of points with a normal, counted by the build (no reference
 * counterpart; the serving loop's keyframe test uses it; synchronizes). */
int nicp_cloud_normal_count(nicp_cloud *c, int *n);

/* Cloud::gaussians() (cloud.h:107; filled by unProject,
 * pinholepointprojector.cpp:93-134, moved by Gaussian3fVector::
 * transformInPlace, gaussian3.h:66-73): per point the mean (3 floats) and
 * the 3x3 covariance (9 floats, row-major).  Either pointer may be null.
 * NICP_ESTATE when the cloud was not built with keep_gaussians. */
int nicp_cloud_download_gaussians(nicp_cloud *cloud, float *mean3, float *cov9);

/* The Stats of each point (stats.h:13-116; kept with keep_stats): eigenvalues
 * (n*3, ascending), eigenvectors (n*9, row-major, columns are the vectors),
 * the window mean (n*3) and the window's point count (n; 0 where the stats
 * calculator did not reach the pixel).  Any pointer may be NULL. */
int nicp_cloud_download_stats(nicp_cloud *cloud, float *eigval3, float *eigvec9, float *mean3, int *n);

/* Any output may be NULL.  points4/normals4: n*4 floats (w = 1 / 0);
 * curvature: n; omega_p9/omega_n9: n*9 (3x3 blocks); eigval3: n*3;
 * eigvec9: n*9 (columns are eigenvectors; needs keep_stats).
 * A cloud built with information matrices of the form U diag(d0, d1, d1) U^T
 * and without keep_stats holds them implicitly (d1 I + (d0 - d1) n n^T from
 * its float normal, evaluated in double and rounded once); the first call
 * that needs them -- this download, the list-mode linearizer, an add of
 * clouds with different forms -- writes them out on the context's stream. */
int nicp_cloud_download(nicp_cloud *c, float *points4, float *normals4, float *curvature,
                        float *omega_p9, float *omega_n9, float *eigval3, float *eigvec9);
int nicp_cloud_upload(nicp_cloud *c, int n, const float *points4, const float *normals4,
                      const float *curvature, const float *omega_p9, const float *omega_n9);
/* Cloud::transformInPlace (cloud.cpp:191-204). */
int nicp_cloud_transform(nicp_cloud *c, const float T16[16]);

/* CorrespondenceFinderNN::compute (correspondencefindernn.cpp:44-97): for
 * each reference point moved by T16 (the aligner passes _T.inverse()), the
 * nearest current point in (p, normal_scaling * n) within the squared
 * inlier distance, then the reference's gates (normals present, point
 * distance, normal angle).  Exact nearest neighbour (ties: lowest index)
 * where the reference asks FLANN for an approximate one.  pairs_out: 2*K
 * int32 (reference, current) in reference-index order (may be NULL);
 * capacity = number of reference points. */
int nicp_correspond_nn(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const float T16[16],
                       float normal_scaling, const nicp_corr_params *corr, int32_t *pairs_out, int *num_pairs);
/* AlignerNN::align (alignernn.cpp:21-118): the Gauss-Newton loop of
 * nicp_align with nearest-neighbour correspondences (no projection, so no
 * camera), recomputed once per outer iteration.  guess16 may be NULL. */
int nicp_align_nn(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const float guess16[16],
                  float normal_scaling, const nicp_corr_params *corr, const nicp_lin_params *lin,
                  const nicp_align_params *prm, nicp_align_result *out);

/* Cloud::save (cloud.cpp:20-25,100-150): writes every step-th point in the
 * reference's .nicp format -- header "NICPCLOUD <n/step> <binary>", t2v(T16)
 * (NULL = identity), then per point text "POINTWITHSTATS x y z nx ny nz
 * <Stats 4x4 row by row>" or binary Point (16 B), Normal (16 B) and the raw
 * 96-byte Stats (4x4 column-major, int n, 3 eigenvalues, bool
 * curvatureComputed at byte 80, float curvature at byte 84; padding zeroed).
 * Stats come from keep_stats; a cloud built without them is written with
 * zeroed Stats, as the reference writes a cloud with no stats. */
int nicp_cloud_save(nicp_cloud *cloud, const char *filename, const float T16[16], int step, int binary);
/* Cloud::load (cloud.cpp:13-18,42-98): reads a .nicp file (text or binary)
 * into the cloud and its pose v2t(x) into T16_out (may be NULL).  The file
 * holds points, normals and Stats only; the information matrices are
 * recomputed from them with prm's calculators (NULL = defaults), as
 * Point/NormalInformationMatrixCalculator::compute would.  *num_points: the
 * points read.  NICP_EINVAL for a bad header or a short file. */
int nicp_cloud_load(nicp_cloud *cloud, const char *filename, const nicp_cloud_params *prm, float T16_out[16],
                    int *num_points);
/* One line of the trajectory file of nicp_simple_aligner.cpp:175-181:
 * "timestamp tx ty tz qx qy qz qw\n" (normalised quaternion of the rotation,
 * numbers as iostream prints floats).  NICP_EINVAL if `capacity` is short. */
int nicp_trajectory_line(const char *timestamp, const float T16[16], char *out, size_t capacity);

/* DepthImage_scale (imageutils.cpp:6-37; used with
 * DepthImage_convert_16UC1_to_32FC1, imageutils.cpp:85-99, and
 * PinholePointProjector::scale, pinholepointprojector.cpp:150-155, for
 * coarse input): out[(rows/step) x (cols/step)] float metres, each pixel the
 * mean of its step x step block's positive depths, 0 when the block has none
 * or their variance exceeds max_depth_cov (reference default 0.01).  `depth`
 * is u16 (times depth_scale) when is_u16, else float metres; row pitch in
 * bytes (0 = packed); input and output each in host or device memory.  Feed
 * the result to nicp_cloud_from_depth_f32 with a camera whose `scaling` is
 * 1/step. */
int nicp_depth_scale(nicp_ctx *ctx, const void *depth, int is_u16, int rows, int cols, size_t pitch_bytes,
                     int on_device, float depth_scale, int step, float max_depth_cov, float *out, int out_on_device);

/* Cloud::add (cloud.cpp:163-189): `src` is first transformed in place by T16
 * (NULL = identity), as the reference does, then its points are appended to
 * `dst` (grown as needed).  Stats, Gaussians and the structured-Omega flag
 * survive only when both clouds carry them.  Both clouds belong to one
 * context. */
int nicp_cloud_add(nicp_cloud *dst, nicp_cloud *src, const float T16[16]);

/* Merger::merge (merger.cpp:15-109; defaults merger.cpp:5-13: distance
 * threshold 0.1, max point depth 10).  The cloud is projected by the camera
 * moved by T16 (z-buffer: smallest depth, then lowest index); each point that
 * lands on another point's pixel within `distance_threshold` in depth adds
 * its Gaussian's information to that point's and is removed; a point that
 * won its own pixel takes its (fused) Gaussian's mean as position.  Needs a
 * cloud with Gaussians (keep_gaussians).  *removed: points removed (may be
 * NULL). */
int nicp_merge(nicp_ctx *ctx, nicp_cloud *cloud, const nicp_camera *cam, const float T16[16],
               float distance_threshold, float max_point_depth, int *removed);

/* DepthImageConverterIntegralImage::compute.  depth: rows x cols u16 with
 * row pitch `pitch_bytes` (0 = packed; otherwise at least cols * 2, else
 * NICP_EINVAL), in host memory or, when
 * depth_on_device != 0, in device memory.  sensor_offset may be NULL
 * (identity).  index_out: optional host rows*cols int32 index image. */
int nicp_cloud_from_depth_u16(nicp_ctx *ctx, const uint16_t *depth, int rows, int cols,
                              size_t pitch_bytes, int depth_on_device, const nicp_camera *cam,
                              const nicp_cloud_params *prm, const float *sensor_offset,
                              nicp_cloud *out, int32_t *index_out);
/* Same from a float depth image in metres (DepthImage). */
int nicp_cloud_from_depth_f32(nicp_ctx *ctx, const float *depth, int rows, int cols,
                              size_t pitch_bytes, int depth_on_device, const nicp_camera *cam,
                              const nicp_cloud_params *prm, const float *sensor_offset,
                              nicp_cloud *out, int32_t *index_out);

/* ------------------------------------------------------------ projector */
/* KRt and iKRt for projector transform T (both 4x4 row-major floats). */
int nicp_projector_matrices(const nicp_camera *cam, const float T16[16], float KRt16[16],
                            float iKRt16[16]);
/* PinholePointProjector::unProject from a float depth image (host).
 * points4_out: rows*cols*4 floats capacity; returns the count in *n. */
int nicp_unproject(nicp_ctx *ctx, const float *depth, int rows, int cols, const nicp_camera *cam,
                   const float T16[16], float *points4_out, int32_t *index_out, int *n);
/* PinholePointProjector::projectIntervals: radius image (both Vec2i
 * components are equal; -1 outside the depth range). */
int nicp_project_intervals(nicp_ctx *ctx, const float *depth, int rows, int cols,
                           const nicp_camera *cam, float world_radius, int32_t *radius_out);
/* PinholePointProjector::project: z-buffer of the cloud seen from T into
 * the (scaled) rows x cols image.  Host outputs; either may be NULL. */
int nicp_project(nicp_ctx *ctx, const nicp_cloud *cloud, const nicp_camera *cam,
                 const float T16[16], int32_t *index_out, float *depth_out);

/* ------------------------------------------------- correspondences, H, b */
/* CorrespondenceFinderProjective::compute with the given index images (host,
 * rows x cols) and T (the aligner passes _T.inverse()).  pairs_out: host,
 * capacity 2*rows*cols int32 (reference index, current index), row-major
 * order.  *num_out = numCorrespondences(). */
int nicp_correspond(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur,
                    const int32_t *ref_index, const int32_t *cur_index, int rows, int cols,
                    const float T16[16], const nicp_corr_params *prm, int32_t *pairs_out,
                    int *num_out);
/* Linearizer::update over a host correspondence list.  H36 is the full 6x6
 * (H(3:6,0:3) = Htr^T, as the reference assembles it); the sums are
 * accumulated in FP64.  parity_threads: the reference's K % T drop (1 = none). */
int nicp_linearize(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur,
                   const int32_t *pairs, int num_pairs, const float T16[16],
                   const nicp_lin_params *prm, int parity_threads, double H36[36], double b6[6],
                   double *error, int *inliers);

/* The linearizer without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: a real-time loop
 * (an odometry thread with a frame deadline) that cannot afford the
 * device-wide synchronisation and unbounded latency of an allocation, or a
 * host framework that owns all device memory and forbids libraries from
 * taking more.  Same result as nicp_linearize, but:
 *   - pairs_dev (2 * num_pairs int32) and out_dev (44 doubles: H 6x6
 *     row-major, b[6], error, inliers) are caller-owned DEVICE buffers;
 *   - the per-tile partial sums live in a fixed array inside the library's
 *     device image (256 KB; every GPU that loads the library holds it until
 *     the process exits), which limits num_pairs to
 *     NICP_LINEARIZE_NOALLOC_MAX_PAIRS -- larger lists return NICP_EINVAL;
 *   - the call is asynchronous on the context's stream; read out_dev after
 *     synchronising that stream;
 *   - every call shares that array, so calls whose kernels overlap on the
 *     GPU (two streams, two host threads on one device) race; serialise them;
 *   - the first call on a device looks the array's address up (once per
 *     device, with the context's device current); make that first call
 *     before any stream capture.
 * Returns NICP_EINVAL for null arguments or a list beyond the limit,
 * NICP_ESTATE when the context's device is not current, NICP_ECUDA when a
 * launch or the address lookup fails; it writes no error text. */
#define NICP_LINEARIZE_NOALLOC_MAX_PAIRS 1048576
int nicp_linearize_noalloc(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur,
                           const int32_t *pairs_dev, int num_pairs, const float T16[16],
                           const nicp_lin_params *prm, int parity_threads, double *out_dev);

/* -------------------------------------------------------------- aligner */
/* AlignerProjective::align for one pair (one call, one pair).  guess,
 * ref_offset, cur_offset may be NULL (identity).  The Gauss-Newton loop is
 * captured as a CUDA graph on the first call of a shape (image size,
 * iteration counts, parameters) and replayed by later calls; the call
 * synchronizes the context's stream to return its result. */
int nicp_align(nicp_ctx *ctx, const nicp_cloud *ref, const nicp_cloud *cur, const nicp_camera *cam,
               const float guess16[16], const float ref_offset16[16], const float cur_offset16[16],
               const nicp_corr_params *corr, const nicp_lin_params *lin,
               const nicp_align_params *prm, nicp_align_result *out);

/* ------------------------------------------------------------- batching */
/* Builds n clouds in one pass of launches.  depth[i]: packed rows[i] x
 * cols[i] u16 frames (host, or device when depth_on_device != 0). */
int nicp_build_batch(nicp_ctx *ctx, int n, const uint16_t *const *depth, const int *rows,
                     const int *cols, int depth_on_device, const nicp_camera *cams,
                     const nicp_cloud_params *prm, nicp_cloud *const *out);
/* Aligns n independent pairs in one device-side Gauss-Newton loop (all
 * outer x inner iterations captured as one CUDA graph, 6x6 solves on the
 * device, per-pair early exit).  guesses: n*16 floats or NULL.  Results are
 * independent of batch composition: every pair's sums use a fixed tile
 * order. */
int nicp_align_batch(nicp_ctx *ctx, int n, const nicp_cloud *const *refs,
                     const nicp_cloud *const *curs, const nicp_camera *cams, const float *guesses,
                     const nicp_corr_params *corr, const nicp_lin_params *lin,
                     const nicp_align_params *prm, nicp_align_result *out);

/* -------------------------------------------------------------- serving */
/* A request loop (no counterpart in the reference; the closest caller is the
 * frame-to-frame odometry of nicp_simple_aligner.cpp:129-184): every camera
 * stream keeps its keyframe cloud resident on the device; each submitted
 * frame is built into a cloud and aligned against its stream's keyframe.
 * Requests are admitted while the device memory they need fits the budget,
 * and batched as they arrive: whenever one of `workers` batch slots frees,
 * it takes the oldest admissible pending requests, up to max_batch and its
 * share (1/workers) of the active streams (at most one request in flight
 * per stream, so a stream's frames stay in order).  Batches of different workers
 * run on different CUDA streams and overlap on the device.  A stream's
 * keyframe is replaced by the current frame when inliers fall below
 * keyframe_min_inlier_ratio x the keyframe's points (points with a normal);
 * the first frame of a stream becomes its keyframe (result T = identity).
 * Each alignment starts from a constant-velocity prediction against the
 * same keyframe: last * prev^-1 * last over the stream's last two estimates
 * (the last estimate after one, the identity right after a replacement). */
typedef struct nicp_server nicp_server;

typedef struct {
  size_t hbm_budget_bytes;        /* device memory for in-flight work and keyframes */
  int max_batch;                  /* requests per batch */
  int workers;                    /* batches in flight */
  float keyframe_min_inlier_ratio;
  nicp_cloud_params cloud;
  nicp_corr_params corr;
  nicp_lin_params lin;
  nicp_align_params align;        /* compute_statistics is ignored */
} nicp_server_params;

typedef struct {
  uint64_t request_id;
  int stream_id;
  int status;             /* NICP_OK, or NICP_EBUDGET when the request can never fit */
  double T[16];           /* current frame -> its stream's keyframe */
  float error;
  int inliers;
  int keyframe_points;
  int keyframe_replaced;  /* the frame became the stream's keyframe */
  int batch_size;         /* requests in the batch that carried it */
  double latency_ms;      /* submit -> result available */
  double queue_ms;        /* submit -> batch start */
} nicp_server_result;

void nicp_default_server_params(nicp_server_params *p);
int nicp_server_create(int device, const nicp_server_params *prm, nicp_server **out);
/* Copies the u16 frame; returns immediately. */
int nicp_server_submit(nicp_server *s, int stream_id, uint64_t request_id, const uint16_t *depth, int rows,
                       int cols, const nicp_camera *cam);
/* Up to max finished results; waits up to wait_ms for the first one. */
int nicp_server_poll(nicp_server *s, nicp_server_result *out, int max, int *n, int wait_ms);
/* pending = submitted but not finished; device_bytes = held by the server. */
int nicp_server_status(nicp_server *s, int *pending, size_t *device_bytes);
int nicp_server_destroy(nicp_server *s);

#ifdef __cplusplus
}
#endif
#endif
