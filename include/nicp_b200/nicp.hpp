// nicp.hpp -- the reference's C++ plugin classes over the C ABI of nicp_gpu.h.
//
// Header-only: a C++ caller of yorsh87/nicp switches to the B200 path by
// including this header instead of nicp/*.h and linking libnicp_b200.so.
// Class names, setters, getters, defaults and the wiring of
// nicp_simple_aligner.cpp:213-268 are kept:
//
//   nicp::PinholePointProjector proj;  proj.setCameraMatrix(K);
//   nicp::StatsCalculatorIntegralImage stats;
//   nicp::PointInformationMatrixCalculator pim;  nicp::NormalInformationMatrixCalculator nim;
//   nicp::DepthImageConverterIntegralImage conv(&proj, &stats, &pim, &nim);
//   nicp::Cloud ref, cur;  conv.compute(ref, depth0);  conv.compute(cur, depth1);
//   nicp::CorrespondenceFinderProjective cf;  nicp::Linearizer lin;
//   nicp::AlignerProjective aligner(&proj, &lin, &cf);
//   aligner.setReferenceCloud(&ref);  aligner.setCurrentCloud(&cur);  aligner.align();
//
// Differences, by design: Eigen and OpenCV types are replaced by the small
// value types below (Isometry3f, Matrix3f, images as (rows, cols, data));
// clouds live on the device; errors throw nicp::Error (the reference only
// asserts, which compiles out in release builds).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../nicp_gpu.h"

namespace nicp {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// Row-major 4x4 isometry (row 3 = 0 0 0 1), the role of Eigen::Isometry3f.
struct Isometry3f {
  float m[16];
  Isometry3f() { setIdentity(); }
  static Isometry3f Identity() { return Isometry3f(); }
  void setIdentity() {
    for (int i = 0; i < 16; i++) m[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  }
  float &operator()(int r, int c) { return m[r * 4 + c]; }
  float operator()(int r, int c) const { return m[r * 4 + c]; }
  const float *data() const { return m; }
  static Isometry3f fromArray(const float a[16]) {
    Isometry3f r;
    for (int i = 0; i < 16; i++) r.m[i] = a[i];
    return r;
  }
  Isometry3f operator*(const Isometry3f &o) const {
    Isometry3f r;
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        float s = 0;
        for (int k = 0; k < 4; k++) s += (*this)(i, k) * o(k, j);
        r(i, j) = s;
      }
    return r;
  }
  Isometry3f inverse() const {
    Isometry3f r;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) r(i, j) = (*this)(j, i);
    for (int i = 0; i < 3; i++) r(i, 3) = -(r(i, 0) * m[3] + r(i, 1) * m[7] + r(i, 2) * m[11]);
    return r;
  }
};

struct Matrix3f {
  float m[9];
  float &operator()(int r, int c) { return m[r * 3 + c]; }
  float operator()(int r, int c) const { return m[r * 3 + c]; }
};

inline void check(nicp_ctx *ctx, int rc) {
  if (rc != NICP_OK) throw Error(rc, ctx ? nicp_ctx_last_error(ctx) : "nicp call failed");
}

// One device + stream + workspace.  default_context() mirrors the reference's
// implicit single-threaded use; pass an explicit Context per host thread.
class Context {
 public:
  explicit Context(int device = 0, void *stream = nullptr) {
    int rc = nicp_ctx_create(device, stream, &h_);
    if (rc != NICP_OK) throw Error(rc, "nicp: cannot create a context (an sm_100 GPU is required)");
  }
  ~Context() {
    if (h_) nicp_ctx_destroy(h_);
  }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  nicp_ctx *handle() const { return h_; }
  void synchronize() { check(h_, nicp_ctx_synchronize(h_)); }

 private:
  nicp_ctx *h_ = nullptr;
};

inline Context &default_context() {
  static Context ctx(0);
  return ctx;
}

// cloud.h:20-193: device-resident points, normals, curvature, Omegas.
class Cloud {
 public:
  explicit Cloud(Context &ctx = default_context()) : ctx_(&ctx) { check(ctx.handle(), nicp_cloud_create(ctx.handle(), &h_)); }
  ~Cloud() {
    if (h_) nicp_cloud_destroy(h_);
  }
  Cloud(const Cloud &) = delete;
  Cloud &operator=(const Cloud &) = delete;
  nicp_cloud *handle() const { return h_; }
  Context &context() const { return *ctx_; }
  size_t size() const {
    int n = 0;
    check(ctx_->handle(), nicp_cloud_size(h_, &n));
    return (size_t)n;
  }
  // points(): n x 4 floats (w = 1); normals(): n x 4 (w = 0)
  std::vector<float> points() const { return field(0); }
  std::vector<float> normals() const { return field(1); }
  std::vector<float> curvature() const { return field(2); }
  // gaussians() (cloud.h:107): means n x 3 and covariances n x 9 (row-major);
  // needs a converter with setKeepGaussians(true)
  void gaussians(std::vector<float> &means, std::vector<float> &covariances) const {
    size_t n = size();
    means.resize(3 * n);
    covariances.resize(9 * n);
    check(ctx_->handle(), nicp_cloud_download_gaussians(h_, means.data(), covariances.data()));
  }
  void transformInPlace(const Isometry3f &T) { check(ctx_->handle(), nicp_cloud_transform(h_, T.data())); }
  // save(filename, T, step, binary) / load(T, filename) (cloud.cpp:13-150): the .nicp format.
  bool save(const char *filename, const Isometry3f &T = Isometry3f::Identity(), int step = 1,
            bool binary = true) const {
    return nicp_cloud_save(h_, filename, T.data(), step, binary ? 1 : 0) == NICP_OK;
  }
  bool load(Isometry3f &T, const char *filename) {
    float t[16];
    if (nicp_cloud_load(h_, filename, nullptr, t, nullptr) != NICP_OK) return false;
    T = Isometry3f::fromArray(t);
    return true;
  }
  // add(cloud, T) (cloud.cpp:163-189): `cloud` is transformed in place, then appended.
  void add(Cloud &cloud, const Isometry3f &T = Isometry3f::Identity()) {
    check(ctx_->handle(), nicp_cloud_add(h_, cloud.h_, T.data()));
  }

 private:
  std::vector<float> field(int which) const {
    size_t n = size();
    std::vector<float> out(which == 2 ? n : 4 * n);
    float *p[3] = {nullptr, nullptr, nullptr};
    p[which] = out.data();
    check(ctx_->handle(), nicp_cloud_download(h_, p[0], p[1], p[2], nullptr, nullptr, nullptr, nullptr));
    return out;
  }
  Context *ctx_;
  nicp_cloud *h_ = nullptr;
};

// pinholepointprojector.{h,cpp} + pointprojector.{h,cpp}.
class PinholePointProjector {
 public:
  explicit PinholePointProjector(Context &ctx = default_context()) : ctx_(&ctx) { nicp_default_camera(&cam_); }
  void setCameraMatrix(const Matrix3f &K) {
    cam_.fx = K(0, 0); cam_.fy = K(1, 1); cam_.cx = K(0, 2); cam_.cy = K(1, 2);
  }
  Matrix3f cameraMatrix() const {
    Matrix3f K = {{cam_.fx * cam_.scaling, 0, cam_.cx * cam_.scaling, 0, cam_.fy * cam_.scaling,
                   cam_.cy * cam_.scaling, 0, 0, 1}};
    return K;
  }
  void setTransform(const Isometry3f &T) { T_ = T; }
  const Isometry3f &transform() const { return T_; }
  void setMinDistance(float v) { cam_.min_distance = v; }
  float minDistance() const { return cam_.min_distance; }
  void setMaxDistance(float v) { cam_.max_distance = v; }
  float maxDistance() const { return cam_.max_distance; }
  void setBaseline(float v) { cam_.baseline = v; }
  float baseline() const { return cam_.baseline; }
  void setAlpha(float v) { cam_.alpha = v; }
  float alpha() const { return cam_.alpha; }
  // Unlike the reference, the (scaled) image size is usable right after
  // setImageSize(); scale() rescales it (pointprojector.cpp:106-112).
  void setImageSize(int rows, int cols) { cam_.rows = rows; cam_.cols = cols; }
  void scale(float s) { cam_.scaling = s; }
  float scalingFactor() const { return cam_.scaling; }
  int imageRows() const { return (int)((float)cam_.rows * cam_.scaling); }
  int imageCols() const { return (int)((float)cam_.cols * cam_.scaling); }
  const nicp_camera &camera() const { return cam_; }
  Context &context() const { return *ctx_; }

  // project(indexImage, depthImage, points): host images of imageRows() x imageCols().
  void project(std::vector<int32_t> &indexImage, std::vector<float> &depthImage, const Cloud &cloud) const {
    size_t P = (size_t)imageRows() * imageCols();
    indexImage.resize(P);
    depthImage.resize(P);
    check(ctx_->handle(), nicp_project(ctx_->handle(), cloud.handle(), &cam_, T_.data(), indexImage.data(),
                                       depthImage.data()));
  }
  // unProject(points, indexImage, depthImage) for a rows x cols float image.
  void unProject(std::vector<float> &points4, std::vector<int32_t> &indexImage, const float *depth, int rows,
                 int cols) const {
    nicp_camera c = cam_;
    c.rows = rows;
    c.cols = cols;
    points4.resize((size_t)rows * cols * 4);
    indexImage.resize((size_t)rows * cols);
    int n = 0;
    check(ctx_->handle(), nicp_unproject(ctx_->handle(), depth, rows, cols, &c, T_.data(), points4.data(),
                                         indexImage.data(), &n));
    points4.resize((size_t)n * 4);
  }
  void projectIntervals(std::vector<int32_t> &radius, const float *depth, int rows, int cols, float worldRadius) const {
    nicp_camera c = cam_;
    c.rows = rows;
    c.cols = cols;
    radius.resize((size_t)rows * cols);
    check(ctx_->handle(), nicp_project_intervals(ctx_->handle(), depth, rows, cols, &c, worldRadius, radius.data()));
  }

 private:
  Context *ctx_;
  nicp_camera cam_;
  Isometry3f T_;
};

class StatsCalculatorIntegralImage {
 public:
  StatsCalculatorIntegralImage() { nicp_default_cloud_params(&p_); }
  void setWorldRadius(float v) { p_.world_radius = v; }
  float worldRadius() const { return p_.world_radius; }
  void setMaxImageRadius(int v) { p_.max_image_radius = v; }
  int maxImageRadius() const { return p_.max_image_radius; }
  void setMinImageRadius(int v) { p_.min_image_radius = v; }
  int minImageRadius() const { return p_.min_image_radius; }
  void setMinPoints(int v) { p_.min_points = v; }
  int minPoints() const { return p_.min_points; }
  void setCurvatureThreshold(float v) { p_.curvature_threshold = v; }
  float curvatureThreshold() const { return p_.curvature_threshold; }
  void setMomentsPrecision(int v) { p_.moments_precision = v; }
  const nicp_cloud_params &params() const { return p_; }

 private:
  nicp_cloud_params p_;
};

class InformationMatrixCalculator {
 public:
  // The reference's InformationMatrix is a 4x4 with only the diagonal 3x3
  // block used (informationmatrix.h:13-84); the diagonal is what is set.
  void setFlatInformationMatrix(float d0, float d1, float d2) { flat_[0] = d0; flat_[1] = d1; flat_[2] = d2; }
  void setNonFlatInformationMatrix(float d0, float d1, float d2) { nonflat_[0] = d0; nonflat_[1] = d1; nonflat_[2] = d2; }
  void setCurvatureThreshold(float v) { thr_ = v; }
  float curvatureThreshold() const { return thr_; }
  const float *flat() const { return flat_; }
  const float *nonflat() const { return nonflat_; }

 protected:
  float flat_[3], nonflat_[3], thr_ = 0.02f;
};

class PointInformationMatrixCalculator : public InformationMatrixCalculator {
 public:
  PointInformationMatrixCalculator() {  // informationmatrixcalculator.h:115-119
    setFlatInformationMatrix(1000.0f, 0.001f, 0.001f);
    setNonFlatInformationMatrix(1.0f, 0.1f, 0.1f);
  }
};

class NormalInformationMatrixCalculator : public InformationMatrixCalculator {
 public:
  NormalInformationMatrixCalculator() {  // informationmatrixcalculator.h:150-155
    setFlatInformationMatrix(1000.0f, 0.001f, 0.001f);
    setNonFlatInformationMatrix(0.1f, 1.0f, 1.0f);
  }
};

// depthimageconverterintegralimage.{h,cpp}.
class DepthImageConverterIntegralImage {
 public:
  DepthImageConverterIntegralImage(PinholePointProjector *projector, StatsCalculatorIntegralImage *stats,
                                   PointInformationMatrixCalculator *pim, NormalInformationMatrixCalculator *nim)
      : proj_(projector), stats_(stats), pim_(pim), nim_(nim) {}
  void setDepthScale(float s) { depth_scale_ = s; }
  // Also fill Cloud::gaussians() (the reference always does; opt-in here).
  void setKeepGaussians(bool v) { keep_gaussians_ = v; }
  // compute(cloud, depthImage, sensorOffset): u16 depth in depthScale units.
  void compute(Cloud &cloud, const uint16_t *depth, int rows, int cols,
               const Isometry3f &sensorOffset = Isometry3f::Identity()) {
    nicp_cloud_params p = params();
    proj_->setImageSize(rows, cols);
    proj_->setTransform(Isometry3f::Identity());  // depthimageconverterintegralimage.cpp:42
    nicp_camera c = proj_->camera();
    check(cloud.context().handle(), nicp_cloud_from_depth_u16(cloud.context().handle(), depth, rows, cols, 0, 0, &c,
                                                              &p, sensorOffset.data(), cloud.handle(), nullptr));
  }
  // compute(cloud, depthImage) for a float depth image in metres (DepthImage).
  void compute(Cloud &cloud, const float *depth, int rows, int cols,
               const Isometry3f &sensorOffset = Isometry3f::Identity()) {
    nicp_cloud_params p = params();
    proj_->setImageSize(rows, cols);
    proj_->setTransform(Isometry3f::Identity());  // depthimageconverterintegralimage.cpp:42
    nicp_camera c = proj_->camera();
    check(cloud.context().handle(), nicp_cloud_from_depth_f32(cloud.context().handle(), depth, rows, cols, 0, 0, &c,
                                                              &p, sensorOffset.data(), cloud.handle(), nullptr));
  }
  PinholePointProjector *projector() { return proj_; }
  StatsCalculatorIntegralImage *statsCalculator() { return stats_; }

 private:
  nicp_cloud_params params() const {
    nicp_cloud_params p = stats_->params();
    p.depth_scale = depth_scale_;
    std::memcpy(p.pim_flat, pim_->flat(), sizeof(p.pim_flat));
    std::memcpy(p.pim_nonflat, pim_->nonflat(), sizeof(p.pim_nonflat));
    p.pim_curvature_threshold = pim_->curvatureThreshold();
    std::memcpy(p.nim_flat, nim_->flat(), sizeof(p.nim_flat));
    std::memcpy(p.nim_nonflat, nim_->nonflat(), sizeof(p.nim_nonflat));
    p.nim_curvature_threshold = nim_->curvatureThreshold();
    p.keep_gaussians = keep_gaussians_ ? 1 : 0;
    return p;
  }
  PinholePointProjector *proj_;
  StatsCalculatorIntegralImage *stats_;
  PointInformationMatrixCalculator *pim_;
  NormalInformationMatrixCalculator *nim_;
  float depth_scale_ = 0.001f;
  bool keep_gaussians_ = false;
};

// merger.{h,cpp}: fuses points of a cloud that land on one pixel of a view;
// the cloud needs Gaussians (DepthImageConverterIntegralImage::setKeepGaussians).
class Merger {
 public:
  explicit Merger(Context &ctx = default_context()) : ctx_(&ctx) {}
  float distanceThreshold() const { return distance_threshold_; }
  void setDistanceThreshold(float v) { distance_threshold_ = v; }
  float normalThreshold() const { return normal_threshold_; }  // kept; merge() does not use it (merger.cpp:61-63)
  void setNormalThreshold(float v) { normal_threshold_ = v; }
  float maxPointDepth() const { return max_point_depth_; }
  void setMaxPointDepth(float v) { max_point_depth_ = v; }
  DepthImageConverterIntegralImage *depthImageConverter() const { return converter_; }
  void setDepthImageConverter(DepthImageConverterIntegralImage *c) { converter_ = c; }
  void setImageSize(int r, int c) { rows_ = r; cols_ = c; }
  int removed() const { return removed_; }
  void merge(Cloud *cloud, const Isometry3f &transform = Isometry3f::Identity());

 private:
  Context *ctx_;
  float distance_threshold_ = 0.1f;
  float normal_threshold_ = std::cos(10.0f * 3.14159265358979f / 180.0f);
  float max_point_depth_ = 10.0f;
  DepthImageConverterIntegralImage *converter_ = nullptr;
  int rows_ = 0, cols_ = 0, removed_ = 0;
};

inline void Merger::merge(Cloud *cloud, const Isometry3f &transform) {
  if (!converter_ || !converter_->projector() || rows_ <= 0 || cols_ <= 0)
    throw Error(NICP_ESTATE, "Merger: set the converter and the image size first");
  nicp_camera cam = converter_->projector()->camera();
  cam.rows = rows_;
  cam.cols = cols_;
  check(ctx_->handle(),
        nicp_merge(ctx_->handle(), cloud->handle(), &cam, transform.data(), distance_threshold_, max_point_depth_,
                   &removed_));
}

// correspondencefinder{,projective}.{h,cpp}.
class CorrespondenceFinderProjective {
 public:
  struct Correspondence {
    int referenceIndex, currentIndex;
  };
  explicit CorrespondenceFinderProjective(Context &ctx = default_context()) : ctx_(&ctx) {
    nicp_default_corr_params(&p_);
  }
  void setInlierDistanceThreshold(float v) { p_.inlier_distance_threshold = v; }
  float inlierDistanceThreshold() const { return p_.inlier_distance_threshold; }
  void setInlierNormalAngularThreshold(float v) { p_.inlier_normal_angular_threshold = v; }
  float inlierNormalAngularThreshold() const { return p_.inlier_normal_angular_threshold; }
  void setFlatCurvatureThreshold(float v) { p_.flat_curvature_threshold = v; }
  float flatCurvatureThreshold() const { return p_.flat_curvature_threshold; }
  void setInlierCurvatureRatioThreshold(float v) { p_.inlier_curvature_ratio_threshold = v; }
  float inlierCurvatureRatioThreshold() const { return p_.inlier_curvature_ratio_threshold; }
  void setDemotedToGICP(bool v) { p_.demoted_to_gicp = v; }
  void setParityThreads(int t) { p_.parity_threads = t; }
  // correspondencefinderprojective.h:146-150 (0 0: the pixel itself)
  void setRowSearchRegion(int r) { p_.row_search_region = r; }
  void setColSearchRegion(int c) { p_.col_search_region = c; }
  int rowSearchRegion() const { return p_.row_search_region; }
  int colSearchRegion() const { return p_.col_search_region; }
  void setImageSize(int rows, int cols) { rows_ = rows; cols_ = cols; }
  std::vector<int32_t> &referenceIndexImage() { return ref_index_; }
  std::vector<int32_t> &currentIndexImage() { return cur_index_; }
  const std::vector<Correspondence> &correspondences() const { return corr_; }
  int numCorrespondences() const { return (int)corr_.size(); }
  const nicp_corr_params &params() const { return p_; }

  void compute(const Cloud &referenceScene, const Cloud &currentScene, const Isometry3f &T) {
    std::vector<int32_t> pairs(2 * (size_t)rows_ * cols_);
    int k = 0;
    check(ctx_->handle(), nicp_correspond(ctx_->handle(), referenceScene.handle(), currentScene.handle(),
                                          ref_index_.data(), cur_index_.data(), rows_, cols_, T.data(), &p_,
                                          pairs.data(), &k));
    corr_.resize(k);
    for (int i = 0; i < k; i++) corr_[i] = Correspondence{pairs[2 * i], pairs[2 * i + 1]};
  }

 private:
  Context *ctx_;
  nicp_corr_params p_;
  int rows_ = 0, cols_ = 0;
  std::vector<int32_t> ref_index_, cur_index_;
  std::vector<Correspondence> corr_;
};

class AlignerProjective;

// linearizer.{h,cpp}; update() accumulates in FP64.
class Linearizer {
 public:
  explicit Linearizer(Context &ctx = default_context()) : ctx_(&ctx) { nicp_default_lin_params(&p_); }
  void setAligner(AlignerProjective *a) { aligner_ = a; }
  AlignerProjective *aligner() const { return aligner_; }
  void setT(const Isometry3f &T) { T_ = T; }
  const Isometry3f &T() const { return T_; }
  void setInlierMaxChi2(float v) { p_.inlier_max_chi2 = v; }
  float inlierMaxChi2() const { return p_.inlier_max_chi2; }
  void setRobustKernel(bool v) { p_.robust_kernel = v; }
  bool robustKernel() const { return p_.robust_kernel != 0; }
  void setZScaling(bool v) { p_.z_scaling = v; }
  void setScale(float v) { p_.scale = v; }
  void setDemotedToGeneralizedICP(bool v) { p_.demoted_to_gicp = v; }
  const double *H() const { return H_; }
  const double *b() const { return b_; }
  float error() const { return (float)error_; }
  int inliers() const { return inliers_; }
  const nicp_lin_params &params() const { return p_; }
  inline void update();
  void linearize() { update(); }
  void setResult(float e, int i) { error_ = e; inliers_ = i; }

 private:
  Context *ctx_;
  AlignerProjective *aligner_ = nullptr;
  nicp_lin_params p_;
  Isometry3f T_;
  double H_[36] = {0}, b_[6] = {0}, error_ = 0;
  int inliers_ = 0;
};

// aligner.{h,cpp} + alignerprojective.{h,cpp}: the Gauss-Newton loop runs on
// the device with one host synchronisation per align().
class AlignerProjective {
 public:
  AlignerProjective(PinholePointProjector *projector, Linearizer *linearizer, CorrespondenceFinderProjective *cf)
      : proj_(projector), cf_(cf) {
    nicp_default_align_params(&p_);
    setLinearizer(linearizer);
  }
  void setProjector(PinholePointProjector *p) { proj_ = p; }
  PinholePointProjector *projector() { return proj_; }
  void setLinearizer(Linearizer *l) {
    lin_ = l;
    if (l) l->setAligner(this);  // aligner.h:212-216
  }
  Linearizer *linearizer() { return lin_; }
  void setCorrespondenceFinder(CorrespondenceFinderProjective *cf) { cf_ = cf; }
  CorrespondenceFinderProjective *correspondenceFinder() { return cf_; }
  void setReferenceCloud(Cloud *c) { ref_ = c; }
  const Cloud *referenceCloud() const { return ref_; }
  void setCurrentCloud(Cloud *c) { cur_ = c; }
  const Cloud *currentCloud() const { return cur_; }
  void setOuterIterations(int v) { p_.outer_iterations = v; }
  int outerIterations() const { return p_.outer_iterations; }
  void setInnerIterations(int v) { p_.inner_iterations = v; }
  int innerIterations() const { return p_.inner_iterations; }
  void setInitialGuess(const Isometry3f &T) { guess_ = T; }
  const Isometry3f &initialGuess() const { return guess_; }
  void setSensorOffset(const Isometry3f &T) { ref_off_ = cur_off_ = T; }
  void setReferenceSensorOffset(const Isometry3f &T) { ref_off_ = T; }
  void setCurrentSensorOffset(const Isometry3f &T) { cur_off_ = T; }
  void setLambda(float v) { p_.lambda = v; }
  float lambda() const { return p_.lambda; }
  void setMinInliers(int v) { p_.min_inliers = v; }
  int minInliers() const { return p_.min_inliers; }
  void setTranslationalMinEigenRatio(float v) { p_.translational_min_eigen_ratio = v; }
  void setRotationalMinEigenRatio(float v) { p_.rotational_min_eigen_ratio = v; }
  void setComputeStatistics(bool v) { p_.compute_statistics = v; }
  void setEarlyExitEps(double v) { p_.early_exit_eps = v; }
  void setDebug(bool v) { debug_ = v; }

  void align() {
    if (!proj_ || !lin_ || !cf_ || !ref_ || !cur_) throw Error(NICP_ESTATE, "AlignerProjective: missing components");
    nicp_camera c = proj_->camera();
    nicp_corr_params cp = cf_->params();
    nicp_lin_params lp = lin_->params();
    Context &ctx = ref_->context();
    check(ctx.handle(), nicp_align(ctx.handle(), ref_->handle(), cur_->handle(), &c, guess_.data(), ref_off_.data(),
                                   cur_off_.data(), &cp, &lp, &p_, &res_));
    for (int i = 0; i < 16; i++) T_.m[i] = (float)res_.T[i];
    lin_->setResult(res_.error, res_.inliers);
  }
  const Isometry3f &T() const { return T_; }
  const double *Td() const { return res_.T; }  // the FP64 pose kept on the device
  float error() const { return res_.error; }
  int inliers() const { return res_.inliers; }
  bool solutionValid() const { return res_.solution_valid == 1; }
  float translationalEigenRatio() const { return (float)res_.translational_ratio; }
  float rotationalEigenRatio() const { return (float)res_.rotational_ratio; }
  // Aligner::omega() (aligner.h:325): 6x6 row-major, (t, quaternion-vector)
  const double *omega() const { return res_.omega; }
  const double *mean() const { return res_.mean; }
  const nicp_align_result &result() const { return res_; }

 private:
  PinholePointProjector *proj_;
  Linearizer *lin_ = nullptr;
  CorrespondenceFinderProjective *cf_;
  Cloud *ref_ = nullptr, *cur_ = nullptr;
  nicp_align_params p_;
  Isometry3f guess_, ref_off_, cur_off_, T_;
  nicp_align_result res_ = {};
  bool debug_ = false;
};

inline void Linearizer::update() {
  if (!aligner_) throw Error(NICP_ESTATE, "Linearizer: missing aligner");
  CorrespondenceFinderProjective *cf = aligner_->correspondenceFinder();
  const auto &c = cf->correspondences();
  std::vector<int32_t> pairs(2 * c.size());
  for (size_t i = 0; i < c.size(); i++) {
    pairs[2 * i] = c[i].referenceIndex;
    pairs[2 * i + 1] = c[i].currentIndex;
  }
  check(ctx_->handle(), nicp_linearize(ctx_->handle(), aligner_->referenceCloud()->handle(),
                                       aligner_->currentCloud()->handle(), pairs.data(), (int)c.size(), T_.data(), &p_,
                                       cf->params().parity_threads, H_, b_, &error_, &inliers_));
}

}  // namespace nicp
