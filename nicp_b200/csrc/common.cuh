// common.cuh -- device-side data layout and arithmetic shared by the NICP kernels.
//
// Data layout in HBM (one cloud):
//   pts[V]   float4 (x, y, z, 1)                          16 B / point
//   nrm[V]   float4 (nx, ny, nz, curvature)               16 B / point
//   omg[3V]  float4 x3: (Op00 Op01 Op02 Op11) (Op12 Op22 On00 On01)
//                       (On02 On11 On12 On22)              48 B / point
//   eig[16V] optional (keep_stats): the reference's Stats -- eigenvalues (3),
//            eigenvectors (9, row-major, columns are vectors), window mean
//            (3), window point count (1).
//   gauss[3V] optional (keep_gaussians): Gaussian3f mean + covariance.
// Images are packed row-major (pitch == cols).
//
// Arithmetic that decides a discrete outcome (which pixel a point lands on,
// which index a z-buffer keeps, whether a correspondence passes a gate) is
// written with __fmul_rn/__fadd_rn so the compiler cannot contract it into
// FMAs: products and sums round exactly as the reference's SSE (no FMA)
// build rounds them, in one fixed order -- sequential over the inner index,
// ((a0*b0 + a1*b1) + a2*b2) + a3*b3.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nicp {

constexpr int kCorrTilePixels = 1024;   // pixels per CTA in the pair-image kernels
constexpr int kCorrThreads = 256;       // 4 pixels per thread
constexpr int kUnprojTilePixels = 4096; // 16 pixels per thread, 256 threads
constexpr int kStatsThreads = 256;
constexpr int kPartialWords = 32;       // doubles per CTA partial (21 H + 6 b + chi2 + inliers + C + K + pad)
constexpr int kSolveCrossF32 = 32;      // k_solve mode bit: FP32 sum of the tile partials
constexpr int kPointsPerCta = 1024;     // z-buffer kernel tile (points per CTA; threads = 1024 / points per thread)
constexpr int kZbufDefaultPPT = 4;      // points per thread for small grids (one or a few clouds)
constexpr int kZbufWidePPT = 8;         // points per thread for grids of two waves or more

// pts[i].w is kNoNormalW for a point without a normal, and 1 + class for a
// point with one, class = (point information matrix non-flat) + 2 (normal
// information matrix non-flat) as the converter chose them (the reference's
// Point has w = 1; downloads report 1).  The z-buffer key carries the
// no-normal bit below the point index, (depth key << 32) | (i << 1) | bit,
// which keeps the packed minimum ordered by (depth, index) exactly, and lets
// the correspondence kernel reject a pixel whose point has no normal without
// gathering it.
constexpr float kNoNormalW = 0.5f;
// Per-point Stats kept with keep_stats: eigenvalues (3), eigenvectors (9,
// row-major, columns are the vectors), window mean (3), window point count
// n (as float) -- the content of the reference's Stats (stats.h:13-116).
constexpr int kStatsWords = 16;
__host__ __device__ __forceinline__ bool point_has_normal(float w) { return w >= 1.0f; }

// ---- per-frame descriptor for the cloud-build kernels
struct FrameDev {
  const uint16_t *depth_u16;  // packed rows*cols, or null when depth_f32 is used
  const float *depth_f32;
  int rows, cols;
  int tile_base;              // first unprojection tile of this frame in the grid
  int band_base;              // first 16-row moment band of this frame in the band grid
  int col_base;               // first band-carry CTA of this frame (128 of its 10 x cols columns each)
  float depth_scale;
  float min_d, max_d;
  float iKRt[12];             // unprojection matrix (rows 0..2 of 4x4)
  float K[9];                 // effective camera matrix
  float world_radius;
  int min_radius, max_radius, min_points;
  float curv_thr;
  float pim_flat[3], pim_nonflat[3], pim_thr;
  float nim_flat[3], nim_nonflat[3], nim_thr;
  int keep_stats;
  float iK[9];                // K^-1 (Gaussian Jacobian)
  float fB, alpha;            // baseline * fx, depth noise coefficient
  // outputs
  int32_t *index;             // rows*cols
  float4 *pts, *nrm, *omg;
  float4 *gauss;              // 3 float4 per point (mean xyz, 9 covariance entries) or null
  float *eig;
  int *count;                 // device: [0] number of points, [1] points with a normal
  // scratch
  int *tile_counts;           // per unprojection tile
  void *moments;              // 10 planes of rows*cols values (double / float / float2)
  void *band_tot;             // per 16-row band: 10 x cols totals, then carries (double / float)
  void *rowpre;               // few-frame builds: 10 planes of row prefixes (double / float), else null
};

// ---- per-pair device state of the Gauss-Newton loop
struct PairState {
  double T[16];        // current estimate, current -> reference
  double invT[16];     // inner-loop variable (alignerprojective.cpp:66-96)
  double Tstart[16];   // T at the start of the outer iteration (early exit)
  double ref_offset[16];
  float KRt[12];       // projects the reference cloud with T * ref_offset
  float Tgate[12];     // float T^-1 used by the correspondence gates
  float Tlin[12];      // float invT used by the linearizer
  float Tgate_used[12]; // gating transform of the last completed outer iteration
  double H[36], b[6];  // last system (before lambda)
  double Hstat[36];    // system of the statistics pass (Aligner::_computeStatistics)
  float error;
  int inliers;
  int num_corr;
  int candidates;
  int iterations;
  int done;
  int status;
  int pad;
};

struct PairDev {
  const float4 *ref_pts, *ref_nrm;
  const int *ref_count;
  const float4 *cur_pts, *cur_nrm, *cur_omg;
  const int *cur_count;
  // The current cloud's information matrices have the converter's structure
  // Omega = d1 I + (d0 - d1) n n^T (n its normal): the fused kernel rebuilds
  // them from the normal and the class code in the point's w instead of
  // gathering them.  cur_omd: (d0, d1) of point-flat, point-non-flat,
  // normal-flat, normal-non-flat.
  int cur_structured;
  float cur_omd[8];
  int rows, cols;       // projection image (scaled)
  int tile_base;        // first pixel tile of this pair in the grid
  int ref_capacity;     // upper bound on reference points
  float min_d, max_d;
  float K[9];
  int32_t *cur_index;   // rows*cols, current cloud projected once
  int32_t *ref_index;   // rows*cols, kept when inner > 1 or statistics are wanted
  unsigned long long *zbuf;  // rows*cols reference z-buffer (all ones when empty)
  double *partials;     // ntiles * kPartialWords
  int32_t *pairs;       // list mode: 2 * rows*cols
  int *list_tile_counts;
  int *num_pairs;       // list mode: device scalar K
  PairState *state;
};

struct CorrParams {
  float sq_thr, cos_thr, flat_thr, min_ratio, max_ratio;
  int demoted;
  int row_limit_threads;  // parity threads T (rows beyond T*(rows/T) skipped)
  int row_search, col_search;  // search window half-sizes (0 0: the pixel itself)
};

struct LinParams {
  float max_chi2;
  int robust;
  int z_scaling;
  float scale;
  int demoted;
};

// ------------------------------------------------------------ float helpers
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsb(float a, float b) { return __fsub_rn(a, b); }

// rows 0..2 of a 4x4 with row 3 = (0 0 0 1), applied to (x, y, z, w)
__device__ __forceinline__ float row4(const float *A, float x, float y, float z, float w) {
  float s = fm(A[0], x);
  s = fa(s, fm(A[1], y));
  s = fa(s, fm(A[2], z));
  s = fa(s, fm(A[3], w));
  return s;
}

__device__ __forceinline__ float3 xform_point(const float *A, float4 p) {
  return make_float3(row4(A, p.x, p.y, p.z, 1.0f), row4(A + 4, p.x, p.y, p.z, 1.0f),
                     row4(A + 8, p.x, p.y, p.z, 1.0f));
}
__device__ __forceinline__ float3 xform_normal(const float *A, float4 n) {
  return make_float3(row4(A, n.x, n.y, n.z, 0.0f), row4(A + 4, n.x, n.y, n.z, 0.0f),
                     row4(A + 8, n.x, n.y, n.z, 0.0f));
}
// ((a0*b0 + a1*b1) + a2*b2) + 0*0 -- the w terms of the reference's 4-vectors are zero
__device__ __forceinline__ float dot3x(float ax, float ay, float az, float bx, float by, float bz) {
  float s = fm(ax, bx);
  s = fa(s, fm(ay, by));
  s = fa(s, fm(az, bz));
  s = fa(s, 0.0f);
  return s;
}

// Monotone 32-bit key of a float (total order as unsigned).
__device__ __forceinline__ uint32_t float_key(float d) {
  uint32_t u = __float_as_uint(d);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// pinholepointprojector.h:253-262 plus the range/image checks of
// pinholepointprojector.cpp:54-58.
__device__ __forceinline__ bool project_pixel(const float *KRt, float4 p, int rows, int cols, float min_d,
                                              float max_d, int &x, int &y, float &d) {
  float ix = row4(KRt, p.x, p.y, p.z, 1.0f);
  float iy = row4(KRt + 4, p.x, p.y, p.z, 1.0f);
  d = row4(KRt + 8, p.x, p.y, p.z, 1.0f);
  if (!(d >= min_d && d <= max_d)) return false;
  float inv = __frcp_rn(d);
  float px = roundf(fm(ix, inv)), py = roundf(fm(iy, inv));
  if (!(fabsf(px) < 1073741824.0f) || !(fabsf(py) < 1073741824.0f)) return false;
  x = (int)px;
  y = (int)py;
  return x >= 0 && x < cols && y >= 0 && y < rows;
}

// pinholepointprojector.h:293-302: (int)max(K*(R,R,0) * (1/d)); -1 outside the range.
__device__ __forceinline__ int interval_radius(const float *K, float d, float min_d, float max_d, float R) {
  if (d < min_d || d > max_d) return -1;
  float p0 = fa(fa(fm(K[0], R), fm(K[1], R)), fm(K[2], 0.0f));
  float p1 = fa(fa(fm(K[3], R), fm(K[4], R)), fm(K[5], 0.0f));
  float inv = __frcp_rn(d);
  float a = fm(p0, inv), b = fm(p1, inv);
  float m = (a < b) ? b : a;
  return (int)m;
}

// imageutils.cpp:85-99 followed by pinholepointprojector.h:275-280.
__device__ __forceinline__ float depth_of(const FrameDev &f, int pix) {
  if (f.depth_u16) {
    uint16_t u = f.depth_u16[pix];
    return u ? fm(f.depth_scale, (float)(int)u) : 0.0f;
  }
  return f.depth_f32[pix];
}
__device__ __forceinline__ bool depth_valid(float d, float min_d, float max_d) {
  return !(d == 0.0f || d < min_d || d > max_d);
}
__device__ __forceinline__ float4 unproject_pixel(const float *iKRt, int c, int r, float d) {
  float qx = fm((float)c, d), qy = fm((float)r, d);
  return make_float4(row4(iKRt, qx, qy, d, 1.0f), row4(iKRt + 4, qx, qy, d, 1.0f),
                     row4(iKRt + 8, qx, qy, d, 1.0f), 1.0f);
}

// ------------------------------------------------------------ FP64 linear algebra
// Same algorithms as the oracle restatement: symmetric 3x3 eigensolver from
// the trigonometric roots of the characteristic cubic (Smith 1961) with
// eigenvectors from cross products / the orthogonal complement (Eberly
// 2014); LDL^T with symmetric diagonal pivoting (Golub & Van Loan 4.2).
template <typename T>
__device__ __forceinline__ void t_cross(const T *a, const T *b, T *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
template <typename T>
__device__ __forceinline__ T t_dot(const T *a, const T *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void d_cross(const double *a, const double *b, double *c) { t_cross(a, b, c); }
__device__ __forceinline__ double d_dot(const double *a, const double *b) { return t_dot(a, b); }

// A unit vector spanning the null space of B - mu I (B symmetric,
// {b00 b01 b02 b11 b12 b22}): the largest cross product of two rows.
__device__ inline void d_null_vector(const double *B, double mu, double *v) {
  double r0[3] = {B[0] - mu, B[1], B[2]};
  double r1[3] = {B[1], B[3] - mu, B[4]};
  double r2[3] = {B[2], B[4], B[5] - mu};
  double c0[3], c1[3], c2[3];
  d_cross(r0, r1, c0);
  d_cross(r0, r2, c1);
  d_cross(r1, r2, c2);
  double d0 = d_dot(c0, c0), d1 = d_dot(c1, c1), d2 = d_dot(c2, c2);
  // select by value (a pointer into the candidates would put them in local memory)
  double b0 = c0[0], b1 = c0[1], b2 = c0[2], db = d0;
  if (d1 > db) { b0 = c1[0]; b1 = c1[1]; b2 = c1[2]; db = d1; }
  if (d2 > db) { b0 = c2[0]; b1 = c2[1]; b2 = c2[2]; db = d2; }
  if (!(db > 0.0)) { v[0] = 1; v[1] = 0; v[2] = 0; return; }
  const double inv = rsqrt(db);
  v[0] = b0 * inv; v[1] = b1 * inv; v[2] = b2 * inv;
}

// The eigenvector of eigenvalue mu within the plane orthogonal to the unit
// eigenvector e.
__device__ inline void d_plane_vector(const double *B, const double *e, double mu, double *v) {
  double u[3];
  if (fabs(e[0]) > fabs(e[1])) {
    const double il = rsqrt(e[0] * e[0] + e[2] * e[2]);
    u[0] = -e[2] * il; u[1] = 0; u[2] = e[0] * il;
  } else {
    const double il = rsqrt(e[1] * e[1] + e[2] * e[2]);
    u[0] = 0; u[1] = e[2] * il; u[2] = -e[1] * il;
  }
  double w[3];
  d_cross(e, u, w);
  double Bu[3] = {B[0] * u[0] + B[1] * u[1] + B[2] * u[2], B[1] * u[0] + B[3] * u[1] + B[4] * u[2],
                  B[2] * u[0] + B[4] * u[1] + B[5] * u[2]};
  double Bw[3] = {B[0] * w[0] + B[1] * w[1] + B[2] * w[2], B[1] * w[0] + B[3] * w[1] + B[4] * w[2],
                  B[2] * w[0] + B[4] * w[1] + B[5] * w[2]};
  double m00 = d_dot(u, Bu) - mu, m01 = d_dot(u, Bw), m11 = d_dot(w, Bw) - mu;
  double n0 = m00 * m00 + m01 * m01, n1 = m01 * m01 + m11 * m11;
  double a, b;
  if (n0 >= n1) {
    if (n0 > 0.0) { const double il = rsqrt(n0); a = -m01 * il; b = m00 * il; }
    else { a = 1; b = 0; }
  } else {
    const double il = rsqrt(n1); a = -m11 * il; b = m01 * il;
  }
  v[0] = a * u[0] + b * w[0];
  v[1] = a * u[1] + b * w[1];
  v[2] = a * u[2] + b * w[2];
}

// A = {a00 a01 a02 a11 a12 a22}; lam ascending; U row-major, column k <-> lam[k].
// With B = A / max|a|, m = tr(B) / 3 and p = sqrt(|B - m I|_F^2 / 6), the
// eigenvalues are m + 2 p cos(phi + 2 pi k / 3), phi = acos(det((B - m I) / p) / 2) / 3;
// the largest (k = 0) and the smallest (k = 1) come from one sincos:
// cos(phi + 2 pi / 3) = -cos(phi) / 2 - sin(phi) sqrt(3) / 2.
// The eigenvalues of a symmetric 3x3 A (lower triangle 00 10 11 20 21 22 as
// 00 01 02 11 12 22): returns true with lam and U filled for the degenerate
// cases (A = 0, or A a multiple of the identity); otherwise false with B =
// A / amax and its ascending eigenvalues l0 <= l1 <= l2 (of B).
__device__ inline bool d_eig3_values(const double *A, double *B, double &amax, double &l0, double &l1, double &l2,
                                     double *lam, double *U) {
  amax = fabs(A[0]);
  for (int i = 1; i < 6; i++) amax = fmax(amax, fabs(A[i]));
  if (!(amax > 0.0)) {
    lam[0] = lam[1] = lam[2] = 0;
    for (int i = 0; i < 9; i++) U[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return true;
  }
  const double is = 1.0 / amax;
  for (int i = 0; i < 6; i++) B[i] = A[i] * is;
  const double third = 1.0 / 3.0;
  const double m = (B[0] + B[3] + B[5]) * third;
  const double b00 = B[0] - m, b11 = B[3] - m, b22 = B[5] - m;
  const double off = B[1] * B[1] + B[2] * B[2] + B[4] * B[4];
  const double p2 = b00 * b00 + b11 * b11 + b22 * b22 + 2.0 * off;
  if (!(p2 > 0.0)) {
    lam[0] = lam[1] = lam[2] = m * amax;
    for (int i = 0; i < 9; i++) U[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return true;
  }
  const double p26 = p2 * (1.0 / 6.0);
  const double ip = rsqrt(p26), p = p26 * ip;
  const double c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = B[1] * ip, c02 = B[2] * ip, c12 = B[4] * ip;
  const double det = c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02);
  const double q = fmin(1.0, fmax(-1.0, 0.5 * det));
  const double phi = acos(q) * third;
  double sphi, cphi;
  sincos(phi, &sphi, &cphi);
  const double half_sqrt3 = 0.86602540378443864676;
  l2 = m + 2.0 * p * cphi;
  l0 = m - p * cphi - 2.0 * half_sqrt3 * p * sphi;
  l1 = 3.0 * m - l0 - l2;
  double t;
  if (l1 < l0) { t = l1; l1 = l0; l0 = t; }
  if (l2 < l1) { t = l2; l2 = l1; l1 = t; }
  if (l1 < l0) { t = l1; l1 = l0; l0 = t; }
  return false;
}

// The orthonormal eigenvectors of B for its eigenvalues l0 <= l1 <= l2: the
// best separated end eigenvalue's vector from a null vector, the middle one
// in the plane orthogonal to it, the third by a cross product.
__device__ inline void d_eig3_vectors(const double *B, double l0, double l1, double l2, double *v0, double *v1,
                                      double *v2) {
  if (l1 - l0 >= l2 - l1) {
    d_null_vector(B, l0, v0);
    d_plane_vector(B, v0, l1, v1);
    d_cross(v0, v1, v2);
  } else {
    d_null_vector(B, l2, v2);
    d_plane_vector(B, v2, l1, v1);
    d_cross(v1, v2, v0);
  }
}

__device__ inline void d_eig3(const double *A, double *lam, double *U) {
  double B[6], amax, l0, l1, l2;
  if (d_eig3_values(A, B, amax, l0, l1, l2, lam, U)) return;
  double v0[3], v1[3], v2[3];
  d_eig3_vectors(B, l0, l1, l2, v0, v1, v2);
  lam[0] = l0 * amax; lam[1] = l1 * amax; lam[2] = l2 * amax;
  for (int r = 0; r < 3; r++) { U[r * 3 + 0] = v0[r]; U[r * 3 + 1] = v1[r]; U[r * 3 + 2] = v2[r]; }
}

// Solve A x = b for a symmetric 6x6 A given by its lower triangle: LDL^T
// with symmetric diagonal pivoting.  Every index is a compile-time constant
// (the pivot's row and column swaps are predicated per candidate), so the
// factor stays in registers.
__device__ __forceinline__ void d_ldlt_solve6(const double *A, const double *b, double *x) {
  double M[6][6];
  int perm[6];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    perm[i] = i;
#pragma unroll
    for (int j = 0; j < 6; j++) M[i][j] = (i >= j) ? A[i * 6 + j] : A[j * 6 + i];
  }
  double d[6];
#pragma unroll
  for (int k = 0; k < 6; k++) {
    int piv = k;
    double best = fabs(M[k][k]);
#pragma unroll
    for (int i = k + 1; i < 6; i++)
      if (fabs(M[i][i]) > best) { best = fabs(M[i][i]); piv = i; }
#pragma unroll
    for (int i = k + 1; i < 6; i++) {
      const bool sw = piv == i;
#pragma unroll
      for (int j = 0; j < 6; j++) {
        const double a = M[k][j], c = M[i][j];
        M[k][j] = sw ? c : a;
        M[i][j] = sw ? a : c;
      }
#pragma unroll
      for (int r = 0; r < 6; r++) {
        const double a = M[r][k], c = M[r][i];
        M[r][k] = sw ? c : a;
        M[r][i] = sw ? a : c;
      }
      const int a = perm[k], c = perm[i];
      perm[k] = sw ? c : a;
      perm[i] = sw ? a : c;
    }
    d[k] = M[k][k];
    double col[6];
#pragma unroll
    for (int i = k + 1; i < 6; i++) col[i] = M[i][k];
#pragma unroll
    for (int i = k + 1; i < 6; i++) M[i][k] = col[i] / d[k];
#pragma unroll
    for (int i = k + 1; i < 6; i++)
#pragma unroll
      for (int j = k + 1; j <= i; j++) {
        M[i][j] = M[i][j] - M[i][k] * col[j];
        M[j][i] = M[i][j];
      }
  }
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    y[i] = b[0];
#pragma unroll
    for (int j = 1; j < 6; j++) y[i] = perm[i] == j ? b[j] : y[i];
  }
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) y[i] = y[i] - M[i][j] * y[j];
#pragma unroll
  for (int i = 0; i < 6; i++) y[i] = y[i] / d[i];
#pragma unroll
  for (int i = 5; i >= 0; i--)
#pragma unroll
    for (int j = i + 1; j < 6; j++) y[i] = y[i] - M[j][i] * y[j];
#pragma unroll
  for (int j = 0; j < 6; j++) {  // x[perm[i]] = y[i]
    double v = y[0];
#pragma unroll
    for (int i = 1; i < 6; i++) v = perm[i] == j ? y[i] : v;
    x[j] = v;
  }
}

// bm_se3.h:10-52 in FP64.
__device__ inline void d_v2t(const double *x, double *T) {
  double qx = x[3], qy = x[4], qz = x[5];
  double qw = sqrt(fmax(0.0, 1.0 - (qx * qx + qy * qy + qz * qz)));
  T[0] = qw * qw + qx * qx - qy * qy - qz * qz;
  T[1] = 2 * (qx * qy - qw * qz);
  T[2] = 2 * (qx * qz + qw * qy);
  T[4] = 2 * (qx * qy + qz * qw);
  T[5] = qw * qw - qx * qx + qy * qy - qz * qz;
  T[6] = 2 * (qy * qz - qx * qw);
  T[8] = 2 * (qx * qz - qy * qw);
  T[9] = 2 * (qy * qz + qx * qw);
  T[10] = qw * qw - qx * qx - qy * qy + qz * qz;
  T[3] = x[0]; T[7] = x[1]; T[11] = x[2];
  T[12] = 0; T[13] = 0; T[14] = 0; T[15] = 1;
}

// Shepperd's method, normalised, vector part with w >= 0.
__device__ inline void d_t2v(const double *T, double *x) {
  double R[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) R[i][j] = T[i * 4 + j];
  double qx, qy, qz, qw;
  double tr = R[0][0] + R[1][1] + R[2][2];
  if (tr > 0) {
    double s = sqrt(tr + 1.0);
    qw = 0.5 * s;
    s = 0.5 / s;
    qx = (R[2][1] - R[1][2]) * s;
    qy = (R[0][2] - R[2][0]) * s;
    qz = (R[1][0] - R[0][1]) * s;
  } else {
    // the largest diagonal entry i picks the component computed first, with
    // (j, k) = (i + 1, i + 2) mod 3 -- written out per i, so that every
    // index is a compile-time constant
    int i = 0;
    if (R[1][1] > R[0][0]) i = 1;
    if (R[2][2] > (i == 1 ? R[1][1] : R[0][0])) i = 2;
    if (i == 0) {
      double s = sqrt(R[0][0] - R[1][1] - R[2][2] + 1.0);
      qx = 0.5 * s;
      s = 0.5 / s;
      qw = (R[2][1] - R[1][2]) * s;
      qy = (R[1][0] + R[0][1]) * s;
      qz = (R[2][0] + R[0][2]) * s;
    } else if (i == 1) {
      double s = sqrt(R[1][1] - R[2][2] - R[0][0] + 1.0);
      qy = 0.5 * s;
      s = 0.5 / s;
      qw = (R[0][2] - R[2][0]) * s;
      qz = (R[2][1] + R[1][2]) * s;
      qx = (R[0][1] + R[1][0]) * s;
    } else {
      double s = sqrt(R[2][2] - R[0][0] - R[1][1] + 1.0);
      qz = 0.5 * s;
      s = 0.5 / s;
      qw = (R[1][0] - R[0][1]) * s;
      qx = (R[0][2] + R[2][0]) * s;
      qy = (R[1][2] + R[2][1]) * s;
    }
  }
  double n = sqrt(qx * qx + qy * qy + qz * qz + qw * qw);
  qx /= n; qy /= n; qz /= n; qw /= n;
  if (qw < 0) { qx = -qx; qy = -qy; qz = -qz; }
  x[0] = T[3]; x[1] = T[7]; x[2] = T[11];
  x[3] = qx; x[4] = qy; x[5] = qz;
}

__device__ inline void d_mm4(const double *A, const double *B, double *C) {
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
      C[i * 4 + j] = A[i * 4 + 0] * B[0 * 4 + j] + A[i * 4 + 1] * B[1 * 4 + j] + A[i * 4 + 2] * B[2 * 4 + j] +
                     A[i * 4 + 3] * B[3 * 4 + j];
}

__device__ inline void d_iso_inverse(const double *T, double *R) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) R[i * 4 + j] = T[j * 4 + i];
#pragma unroll
  for (int i = 0; i < 3; i++)
    R[i * 4 + 3] = -(R[i * 4 + 0] * T[3] + R[i * 4 + 1] * T[7] + R[i * 4 + 2] * T[11]);
  R[12] = 0; R[13] = 0; R[14] = 0; R[15] = 1;
}

}  // namespace nicp
