/*
 * nicp_oracle.h -- C API of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a plain C++17 + OpenMP restatement of the yorsh87/nicp
 * depth -> cloud -> projective-ICP path.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it; the product (nicp_b200) never
 * links, imports or calls it.
 *
 * Parity status: UNPINNED.  The reference ships no tests, golden vectors or
 * fixtures for this path, and it cannot be compiled here (its required
 * dependencies Eigen3 >= 3.2, OpenCV >= 3.2 and FLANN are absent), so the
 * restatement is checked only against analytic known-answer tests and its
 * own committed fixtures.
 *
 * Two modes share one templated implementation:
 *   ORC_REF32 (0): float arithmetic in the reference's operation order
 *                  (no FMA, reciprocal-multiplies, double promotions where
 *                  the reference has them, OpenMP partition drops).
 *   ORC_F64   (1): the same algorithm in double with no drops: the FP64
 *                  oracle every GPU result is measured against.
 */
#ifndef NICP_ORACLE_H
#define NICP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_REF32 = 0, ORC_F64 = 1 };

/* PinholePointProjector state (pinholepointprojector.cpp:5-31,150-155,
 * pointprojector.cpp:6-15,106-112).  K is the "original" camera matrix;
 * the effective one has its first two rows multiplied by `scaling`. */
typedef struct {
  float fx, fy, cx, cy;
  float scaling;
  int rows, cols;            /* original image size (setImageSize) */
  float min_distance, max_distance;
  float baseline, alpha;
} orc_camera;

/* StatsCalculatorIntegralImage + Point/NormalInformationMatrixCalculator
 * (statscalculatorintegralimage.cpp:12-18, informationmatrixcalculator.h). */
typedef struct {
  float depth_scale;
  float world_radius;
  int min_image_radius, max_image_radius, min_points;
  float curvature_threshold;
  float pim_flat[3], pim_nonflat[3];
  float pim_curvature_threshold;
  float nim_flat[3], nim_nonflat[3];
  float nim_curvature_threshold;
} orc_cloud_params;

/* CorrespondenceFinder(+Projective), Linearizer and Aligner setters
 * (correspondencefinder.cpp:9-18, linearizer.cpp:9-19, aligner.cpp:21-41). */
typedef struct {
  float inlier_distance_threshold;
  float inlier_normal_angular_threshold;   /* a cosine */
  float flat_curvature_threshold;
  float inlier_curvature_ratio_threshold;
  int corr_demoted_to_gicp;
  float inlier_max_chi2;
  int robust_kernel;
  int z_scaling;
  float lin_scale;
  int lin_demoted_to_gicp;
  int outer_iterations, inner_iterations;
  float lambda;
  float translational_min_eigen_ratio, rotational_min_eigen_ratio;
  int threads;               /* emulated omp_get_max_threads() */
  double early_exit_eps;     /* stop once an outer iteration moves the pose by less
                                (max |t2v(T T_start^-1)|); 0 = the reference's fixed count */
  int row_search_region, col_search_region;  /* CorrespondenceFinderProjective search window
                                                (correspondencefinderprojective.h:146-150); 0 0 = single */
} orc_align_params;

typedef struct orc_cloud orc_cloud;

/* imageutils.cpp:85-99 (u16 -> float metres). */
void orc_convert_u16(const uint16_t *src, int rows, int cols, float scale, float *dst);

/* DepthImageConverterIntegralImage::compute on a u16 depth image (the
 * app-level conversion fused in).  sensor_offset: 16 doubles row-major or
 * NULL for identity.  index_out (rows*cols int32) may be NULL. */
orc_cloud *orc_cloud_build_u16(int mode, const uint16_t *depth, int rows, int cols,
                               const orc_camera *cam, const orc_cloud_params *prm,
                               const double *sensor_offset, int32_t *index_out);

/* The same from a float depth image in metres (DepthImage). */
orc_cloud *orc_cloud_build_f32(int mode, const float *depth, int rows, int cols, const orc_camera *cam,
                               const orc_cloud_params *prm, const double *offset, int32_t *index_out);

/* A cloud assembled from arrays (for feeding the oracle the GPU's own
 * cloud).  points4/normals4: n*4; omega_p9/omega_n9: n*9 (3x3 row-major). */
orc_cloud *orc_cloud_from_arrays(int mode, int n, const double *points4, const double *normals4,
                                 const double *curvature, const double *omega_p9,
                                 const double *omega_n9);
void orc_cloud_free(orc_cloud *c);
int orc_cloud_size(const orc_cloud *c);
/* DepthImage_scale (imageutils.cpp:6-37), float; dst: (rows/step) x (cols/step). */
void orc_depth_scale(const float *src, int rows, int cols, int step, float max_cov, float *dst);
/* Cloud::transformInPlace (cloud.cpp:191-204, gaussian3.h:66-73). */
void orc_cloud_transform(orc_cloud *c, const double *T16);
/* Cloud::add (cloud.cpp:163-189): transforms src in place, appends it to dst
 * (both of the same mode). */
void orc_cloud_add(orc_cloud *dst, orc_cloud *src, const double *T16);
/* Merger::merge (merger.cpp:15-109) with the projector of `cam` moved by T16;
 * returns the number of points removed. */
int orc_merge(int mode, orc_cloud *c, const orc_camera *cam, const double *T16, double distance_threshold,
              double max_point_depth);
/* field: 0 points(4n) 1 normals(4n) 2 curvature(n) 3 omega_p(9n) 4 omega_n(9n)
 *        5 eigenvalues(3n) 6 eigenvectors(9n, row-major 3x3, columns = vectors)
 *        7 stats_n(n) 8 gaussian covariance (9n) 9 gaussian mean (3n) */
int orc_cloud_get(const orc_cloud *c, int field, double *out);

/* PinholePointProjector::_updateMatrices outputs for transform T. */
void orc_projector_matrices(int mode, const orc_camera *cam, const double *T16,
                            double *KRt16, double *iKRt16);

/* PinholePointProjector::project (pinholepointprojector.cpp:33-66). */
void orc_project(int mode, const orc_cloud *c, const orc_camera *cam, const double *T16,
                 int32_t *index_out, double *depth_out);

/* CorrespondenceFinderProjective::_computeSingle.  Returns K; pairs_out
 * holds 2*K int32 (reference index, current index) in output order. */
int orc_correspond(int mode, const orc_cloud *ref, const orc_cloud *cur,
                   const int32_t *ref_index, const int32_t *cur_index, int rows, int cols,
                   const double *T16, const orc_align_params *prm, int32_t *pairs_out);

/* Linearizer::update over a correspondence list. H36 row-major (full). */
void orc_linearize(int mode, const orc_cloud *ref, const orc_cloud *cur,
                   const int32_t *pairs, int num_pairs, const double *T16,
                   const orc_align_params *prm, double *H36, double *b6,
                   double *error, int *inliers);

/* AlignerProjective::align (+ _computeStatistics when stats_out != NULL:
 * stats_out = {translationalRatio, rotationalRatio, solutionValid}). */
typedef struct {
  double T[16];
  double error;
  int inliers;
  int num_correspondences;   /* of the last outer iteration */
  double translational_ratio, rotational_ratio;
  int solution_valid;
  int outer_iterations_run;
  double omega[36];          /* Aligner::omega() (aligner.cpp:124-126), row-major */
  double mean[6];            /* Aligner::_mean: the reconstructed Gaussian's mean */
} orc_align_result;

/* CorrespondenceFinderNN::compute (correspondencefindernn.cpp:44-97) with an
 * exact nearest neighbour in (p, normal_scaling * n); pairs: 2*K int32 in
 * reference-index order; returns K. */
int orc_correspond_nn(int mode, const orc_cloud *ref, const orc_cloud *cur, const double *T16, double normal_scaling,
                      const orc_align_params *prm, int32_t *pairs);
/* AlignerNN::align (alignernn.cpp:21-118). */
void orc_align_nn(int mode, const orc_cloud *ref, const orc_cloud *cur, const double *guess, double normal_scaling,
                  const orc_align_params *prm, int stats, orc_align_result *out);

void orc_align(int mode, const orc_cloud *ref, const orc_cloud *cur, const orc_camera *cam,
               const double *guess16, const double *ref_offset16, const double *cur_offset16,
               const orc_align_params *prm, int compute_statistics, orc_align_result *out);

/* Building blocks, exposed for known-answer tests. */
void orc_eig3(int mode, const double *A6, double *lambda3, double *U9);
void orc_ldlt_solve(int mode, const double *A36, const double *b6, double *x6);
void orc_v2t(int mode, const double *x6, double *T16);
void orc_t2v(int mode, const double *T16, double *x6);
void orc_iso_inverse(int mode, const double *T16, double *out16);

/* Integral-image region query (pointintegralimage.cpp:53-66) of a cloud's
 * moments over a rows x cols index image, for box-sum KATs.  out10 =
 * {n, Sx, Sy, Sz, Sxx, Sxy, Sxz, Syy, Syz, Szz}. */
void orc_integral_region(int mode, const orc_cloud *c, const int32_t *index, int rows, int cols,
                         int xmin, int xmax, int ymin, int ymax, double *out10);

#ifdef __cplusplus
}
#endif
#endif
