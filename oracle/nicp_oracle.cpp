// nicp_oracle.cpp -- CPU oracle for the NICP registration path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++17 + OpenMP,
// the algorithm of yorsh87/nicp's depth -> cloud -> projective ICP path so
// that the CUDA product can be checked against it.  The product never links
// or calls it.
//
// Parity status: UNPINNED.  The reference has no tests or golden vectors and
// cannot be built here (Eigen3 / OpenCV / FLANN are absent), so this
// restatement is validated only by analytic known-answer tests.
//
// Semantics follow the reference file by file (citations are paths inside
// the reference project).  The third-party arithmetic the reference takes from
// Eigen is re-derived from published mathematics, not from Eigen:
//   * symmetric 3x3 eigensolver: trigonometric roots of the characteristic
//     cubic (O. K. Smith, CACM 4(4), 1961) and eigenvectors by the
//     cross-product / orthogonal-complement construction described in
//     D. Eberly, "A Robust Eigensolver for 3x3 Symmetric Matrices" (2014);
//   * 6x6 LDL^T with symmetric diagonal pivoting (Golub & Van Loan,
//     Matrix Computations, sec. 4.2);
//   * rotation -> quaternion by Shepperd's method (J. Guidance & Control,
//     1978);
//   * 3x3 inverse by adjugate times the reciprocal determinant.
// Fixed-size products use one explicit order everywhere: sequential
// accumulation over the inner index, ((a0*b0 + a1*b1) + a2*b2) + a3*b3, with
// no fused multiply-add (built with -ffp-contract=off).  "REF32" is bit-exact
// with respect to this restatement; last-ulp agreement with a real
// Eigen/SSE build of the reference is not claimed.
#include "nicp_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

template <class S> struct V4 {
  S v[4];
  S &operator[](int i) { return v[i]; }
  const S &operator[](int i) const { return v[i]; }
};

template <class S> struct M4 {
  S a[16];
  S &operator()(int r, int c) { return a[r * 4 + c]; }
  const S &operator()(int r, int c) const { return a[r * 4 + c]; }
  static M4 zero() { M4 m; for (int i = 0; i < 16; i++) m.a[i] = S(0); return m; }
  static M4 identity() { M4 m = zero(); for (int i = 0; i < 4; i++) m(i, i) = S(1); return m; }
};

template <class S> static inline V4<S> mv(const M4<S> &A, const V4<S> &x) {
  V4<S> r;
  for (int i = 0; i < 4; i++) {
    S s = A(i, 0) * x[0];
    s = s + A(i, 1) * x[1];
    s = s + A(i, 2) * x[2];
    s = s + A(i, 3) * x[3];
    r[i] = s;
  }
  return r;
}

template <class S> static inline M4<S> mm(const M4<S> &A, const M4<S> &B) {
  M4<S> C;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      S s = A(i, 0) * B(0, j);
      s = s + A(i, 1) * B(1, j);
      s = s + A(i, 2) * B(2, j);
      s = s + A(i, 3) * B(3, j);
      C(i, j) = s;
    }
  return C;
}

template <class S> static inline M4<S> transpose(const M4<S> &A) {
  M4<S> T;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T(i, j) = A(j, i);
  return T;
}

template <class S> static inline S dot4(const V4<S> &a, const V4<S> &b) {
  S s = a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  s = s + a[3] * b[3];
  return s;
}

// Eigen::Isometry3f::inverse(): [R^T, -R^T t; 0 0 0 1].
template <class S> static M4<S> iso_inverse(const M4<S> &T) {
  M4<S> r = M4<S>::identity();
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r(i, j) = T(j, i);
  for (int i = 0; i < 3; i++) {
    S s = r(i, 0) * T(0, 3);
    s = s + r(i, 1) * T(1, 3);
    s = s + r(i, 2) * T(2, 3);
    r(i, 3) = -s;
  }
  return r;
}

template <class S> static inline void set_row3(M4<S> &T) {
  T(3, 0) = S(0); T(3, 1) = S(0); T(3, 2) = S(0); T(3, 3) = S(1);
}

// 3x3 inverse: adjugate times reciprocal determinant (row-major in/out).
template <class S> static void inv3(const S m[9], S out[9]) {
  S c00 = m[4] * m[8] - m[5] * m[7];
  S c01 = m[5] * m[6] - m[3] * m[8];
  S c02 = m[3] * m[7] - m[4] * m[6];
  S det = m[0] * c00;
  det = det + m[1] * c01;
  det = det + m[2] * c02;
  S id = S(1) / det;
  out[0] = c00 * id;
  out[3] = c01 * id;
  out[6] = c02 * id;
  out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// ----------------------------------------------------------------- se(3)
// bm_se3.h:10-66.
template <class S> static void quat2mat(S qx, S qy, S qz, S R[9]) {
  S n2 = qx * qx;
  n2 = n2 + qy * qy;
  n2 = n2 + qz * qz;
  S qw = std::sqrt(S(1) - n2);
  R[0] = qw * qw + qx * qx - qy * qy - qz * qz;
  R[1] = S(2) * (qx * qy - qw * qz);
  R[2] = S(2) * (qx * qz + qw * qy);
  R[3] = S(2) * (qx * qy + qz * qw);
  R[4] = qw * qw - qx * qx + qy * qy - qz * qz;
  R[5] = S(2) * (qy * qz - qx * qw);
  R[6] = S(2) * (qx * qz - qy * qw);
  R[7] = S(2) * (qy * qz + qx * qw);
  R[8] = qw * qw - qx * qx - qy * qy + qz * qz;
}

// Shepperd's method, then normalise and return the vector part with w >= 0.
template <class S> static void mat2quat(const M4<S> &T, S q[3]) {
  S R[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[i][j] = T(i, j);
  S x, y, z, w;
  S tr = R[0][0] + R[1][1];
  tr = tr + R[2][2];
  if (tr > S(0)) {
    S s = std::sqrt(tr + S(1));
    w = S(0.5) * s;
    s = S(0.5) / s;
    x = (R[2][1] - R[1][2]) * s;
    y = (R[0][2] - R[2][0]) * s;
    z = (R[1][0] - R[0][1]) * s;
  } else {
    int i = 0;
    if (R[1][1] > R[0][0]) i = 1;
    if (R[2][2] > R[i][i]) i = 2;
    int j = (i + 1) % 3, k = (j + 1) % 3;
    S s = std::sqrt(R[i][i] - R[j][j] - R[k][k] + S(1));
    S qv[3];
    qv[i] = S(0.5) * s;
    s = S(0.5) / s;
    w = (R[k][j] - R[j][k]) * s;
    qv[j] = (R[j][i] + R[i][j]) * s;
    qv[k] = (R[k][i] + R[i][k]) * s;
    x = qv[0]; y = qv[1]; z = qv[2];
  }
  S n2 = x * x;
  n2 = n2 + y * y;
  n2 = n2 + z * z;
  n2 = n2 + w * w;
  if (n2 > S(0)) {
    S n = std::sqrt(n2);
    x = x / n; y = y / n; z = z / n; w = w / n;
  }
  if (w < S(0)) { x = -x; y = -y; z = -z; }
  q[0] = x; q[1] = y; q[2] = z;
}

template <class S> static M4<S> v2t(const S x[6]) {
  M4<S> T = M4<S>::identity();
  S R[9];
  quat2mat(x[3], x[4], x[5], R);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) T(i, j) = R[i * 3 + j];
  T(0, 3) = x[0]; T(1, 3) = x[1]; T(2, 3) = x[2];
  return T;
}

template <class S> static void t2v(const M4<S> &T, S x[6]) {
  x[0] = T(0, 3); x[1] = T(1, 3); x[2] = T(2, 3);
  mat2quat(T, x + 3);
}

// ------------------------------------------------------- 3x3 eigensolver
// A = {a00, a01, a02, a11, a12, a22}.  lambda ascending; U row-major with
// column k the unit eigenvector of lambda[k].
template <class S> static inline void cross3(const S a[3], const S b[3], S c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
template <class S> static inline S dot3(const S a[3], const S b[3]) {
  S s = a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}

// Unit vector spanning the null space of (B - mu I) for a simple eigenvalue mu.
template <class S> static void null_vector(const S B[6], S mu, S v[3]) {
  S r0[3] = {B[0] - mu, B[1], B[2]};
  S r1[3] = {B[1], B[3] - mu, B[4]};
  S r2[3] = {B[2], B[4], B[5] - mu};
  S c0[3], c1[3], c2[3];
  cross3(r0, r1, c0);
  cross3(r0, r2, c1);
  cross3(r1, r2, c2);
  S d0 = dot3(c0, c0), d1 = dot3(c1, c1), d2 = dot3(c2, c2);
  const S *best = c0;
  S db = d0;
  if (d1 > db) { best = c1; db = d1; }
  if (d2 > db) { best = c2; db = d2; }
  if (!(db > S(0))) { v[0] = S(1); v[1] = S(0); v[2] = S(0); return; }
  S inv = S(1) / std::sqrt(db);
  v[0] = best[0] * inv; v[1] = best[1] * inv; v[2] = best[2] * inv;
}

// Eigenvector of B for mu restricted to the plane orthogonal to unit e.
template <class S> static void plane_vector(const S B[6], const S e[3], S mu, S v[3]) {
  S u[3];
  if (std::fabs(e[0]) > std::fabs(e[1])) {
    S il = S(1) / std::sqrt(e[0] * e[0] + e[2] * e[2]);
    u[0] = -e[2] * il; u[1] = S(0); u[2] = e[0] * il;
  } else {
    S il = S(1) / std::sqrt(e[1] * e[1] + e[2] * e[2]);
    u[0] = S(0); u[1] = e[2] * il; u[2] = -e[1] * il;
  }
  S w[3];
  cross3(e, u, w);
  S Bu[3] = {dot3(B, u), B[1] * u[0] + B[3] * u[1] + B[4] * u[2], B[2] * u[0] + B[4] * u[1] + B[5] * u[2]};
  S Bw[3] = {B[0] * w[0] + B[1] * w[1] + B[2] * w[2], B[1] * w[0] + B[3] * w[1] + B[4] * w[2],
             B[2] * w[0] + B[4] * w[1] + B[5] * w[2]};
  S m00 = dot3(u, Bu) - mu, m01 = dot3(u, Bw), m11 = dot3(w, Bw) - mu;
  S n0 = m00 * m00 + m01 * m01, n1 = m01 * m01 + m11 * m11;
  S a, b;
  if (n0 >= n1) {
    if (n0 > S(0)) { S il = S(1) / std::sqrt(n0); a = -m01 * il; b = m00 * il; }
    else { a = S(1); b = S(0); }
  } else {
    S il = S(1) / std::sqrt(n1); a = -m11 * il; b = m01 * il;
  }
  v[0] = a * u[0] + b * w[0];
  v[1] = a * u[1] + b * w[1];
  v[2] = a * u[2] + b * w[2];
}

template <class S> static void eig3(const S A[6], S lam[3], S U[9]) {
  S amax = std::fabs(A[0]);
  for (int i = 1; i < 6; i++) amax = std::max(amax, (S)std::fabs(A[i]));
  if (!(amax > S(0))) {
    lam[0] = lam[1] = lam[2] = S(0);
    for (int i = 0; i < 9; i++) U[i] = (i % 4 == 0) ? S(1) : S(0);
    return;
  }
  S is = S(1) / amax;
  S B[6];
  for (int i = 0; i < 6; i++) B[i] = A[i] * is;
  S m = (B[0] + B[3] + B[5]) / S(3);
  S b00 = B[0] - m, b11 = B[3] - m, b22 = B[5] - m;
  S off = B[1] * B[1] + B[2] * B[2] + B[4] * B[4];
  S p2 = b00 * b00 + b11 * b11 + b22 * b22 + S(2) * off;
  if (!(p2 > S(0))) {
    lam[0] = lam[1] = lam[2] = m * amax;
    for (int i = 0; i < 9; i++) U[i] = (i % 4 == 0) ? S(1) : S(0);
    return;
  }
  S p = std::sqrt(p2 / S(6));
  S ip = S(1) / p;
  S c00 = b00 * ip, c11 = b11 * ip, c22 = b22 * ip, c01 = B[1] * ip, c02 = B[2] * ip, c12 = B[4] * ip;
  S det = c00 * (c11 * c22 - c12 * c12) - c01 * (c01 * c22 - c12 * c02) + c02 * (c01 * c12 - c11 * c02);
  S q = det / S(2);
  if (q < S(-1)) q = S(-1);
  if (q > S(1)) q = S(1);
  S phi = std::acos(q) / S(3);
  const S tpi3 = S(2.0943951023931954923);  // 2*pi/3
  S l2 = m + S(2) * p * std::cos(phi);
  S l0 = m + S(2) * p * std::cos(phi + tpi3);
  S l1 = S(3) * m - l0 - l2;
  // guard the ordering against rounding
  if (l1 < l0) std::swap(l1, l0);
  if (l2 < l1) std::swap(l2, l1);
  if (l1 < l0) std::swap(l1, l0);
  S v0[3], v1[3], v2[3];
  if (l1 - l0 >= l2 - l1) {
    null_vector(B, l0, v0);
    plane_vector(B, v0, l1, v1);
    cross3(v0, v1, v2);
  } else {
    null_vector(B, l2, v2);
    plane_vector(B, v2, l1, v1);
    cross3(v1, v2, v0);
  }
  lam[0] = l0 * amax; lam[1] = l1 * amax; lam[2] = l2 * amax;
  for (int r = 0; r < 3; r++) { U[r * 3 + 0] = v0[r]; U[r * 3 + 1] = v1[r]; U[r * 3 + 2] = v2[r]; }
}

// ------------------------------------------------------ LDL^T, 6x6 solve
// Symmetric diagonal pivoting; reads the lower triangle of A (row-major).
template <class S> static void ldlt_solve(const S A[36], const S b[6], S x[6]) {
  S M[6][6];
  int perm[6];
  for (int i = 0; i < 6; i++) {
    perm[i] = i;
    for (int j = 0; j < 6; j++) M[i][j] = (i >= j) ? A[i * 6 + j] : A[j * 6 + i];
  }
  S d[6];
  for (int k = 0; k < 6; k++) {
    int piv = k;
    S best = std::fabs(M[k][k]);
    for (int i = k + 1; i < 6; i++)
      if (std::fabs(M[i][i]) > best) { best = std::fabs(M[i][i]); piv = i; }
    if (piv != k) {
      for (int j = 0; j < 6; j++) std::swap(M[k][j], M[piv][j]);
      for (int i = 0; i < 6; i++) std::swap(M[i][k], M[i][piv]);
      std::swap(perm[k], perm[piv]);
    }
    d[k] = M[k][k];
    S col[6];
    for (int i = k + 1; i < 6; i++) col[i] = M[i][k];
    for (int i = k + 1; i < 6; i++) M[i][k] = col[i] / d[k];
    for (int i = k + 1; i < 6; i++)
      for (int j = k + 1; j <= i; j++) {
        M[i][j] = M[i][j] - M[i][k] * col[j];
        M[j][i] = M[i][j];
      }
  }
  S y[6];
  for (int i = 0; i < 6; i++) y[i] = b[perm[i]];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < i; j++) y[i] = y[i] - M[i][j] * y[j];
  for (int i = 0; i < 6; i++) y[i] = y[i] / d[i];
  for (int i = 5; i >= 0; i--)
    for (int j = i + 1; j < 6; j++) y[i] = y[i] - M[j][i] * y[j];
  for (int i = 0; i < 6; i++) x[perm[i]] = y[i];
}

// ------------------------------------------------------------- data model
template <class S> struct Cloud {
  int n = 0;
  std::vector<V4<S>> points, normals;
  std::vector<S> curvature;        // Stats::curvature()
  std::vector<S> eigval, eigvec;   // Stats eigenvalues (3) / eigenvectors (9)
  std::vector<S> omega_p, omega_n; // 3x3 blocks of the InformationMatrix
  std::vector<S> gauss_cov;        // Gaussian3f covariance (9)
  std::vector<S> gauss_mean;       // Gaussian3f mean (3)
  std::vector<int> stats_n;
  void resize(int k) {
    n = k;
    points.resize(k); normals.resize(k); curvature.assign(k, S(0));
    eigval.assign(3 * k, S(0)); eigvec.assign(9 * k, S(0));
    omega_p.assign(9 * k, S(0)); omega_n.assign(9 * k, S(0));
    gauss_cov.assign(9 * k, S(0)); gauss_mean.assign(3 * k, S(0)); stats_n.assign(k, 0);
  }
};

template <class S> struct Projector {
  S K[9];      // effective camera matrix (_cameraMatrix)
  S iK[9];
  M4<S> KRt, iKRt;
  int rows, cols;
  S min_d, max_d, baseline, alpha;
};

// pinholepointprojector.cpp:16-31 with pointprojector.cpp:106-112 and
// pinholepointprojector.cpp:150-155 (scale()).
template <class S> static Projector<S> make_projector(const orc_camera &c, const M4<S> &transform) {
  Projector<S> P;
  S K0[9] = {S(c.fx), S(0), S(c.cx), S(0), S(c.fy), S(c.cy), S(0), S(0), S(1)};
  S sc = S(c.scaling);
  for (int i = 0; i < 9; i++) P.K[i] = (i < 6) ? K0[i] * sc : K0[i];
  P.rows = (int)((float)c.rows * c.scaling);
  P.cols = (int)((float)c.cols * c.scaling);
  P.min_d = S(c.min_distance);
  P.max_d = S(c.max_distance);
  P.baseline = S(c.baseline);
  P.alpha = S(c.alpha);
  M4<S> t = iso_inverse(transform);
  set_row3(t);
  inv3(P.K, P.iK);
  P.KRt = M4<S>::identity();
  P.iKRt = M4<S>::identity();
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) {
      S s = P.K[i * 3 + 0] * t(0, j);
      s = s + P.K[i * 3 + 1] * t(1, j);
      s = s + P.K[i * 3 + 2] * t(2, j);
      P.KRt(i, j) = s;
      S u = transform(i, 0) * P.iK[0 * 3 + j];
      u = u + transform(i, 1) * P.iK[1 * 3 + j];
      u = u + transform(i, 2) * P.iK[2 * 3 + j];
      P.iKRt(i, j) = u;
    }
    S s = P.K[i * 3 + 0] * t(0, 3);
    s = s + P.K[i * 3 + 1] * t(1, 3);
    s = s + P.K[i * 3 + 2] * t(2, 3);
    P.KRt(i, 3) = s;
    P.iKRt(i, 3) = transform(i, 3);
  }
  return P;
}

// pinholepointprojector.h:253-262.
template <class S> static inline bool project_point(const Projector<S> &P, const V4<S> &p, int &x, int &y, S &d) {
  V4<S> ip = mv(P.KRt, p);
  d = ip[2];
  if (d < P.min_d || d > P.max_d) return false;
  S inv = S(1) / d;
  S px = ip[0] * inv, py = ip[1] * inv;
  px = std::round(px);
  py = std::round(py);
  if (!(std::fabs(px) < S(1 << 30)) || !(std::fabs(py) < S(1 << 30))) return false;
  x = (int)px;
  y = (int)py;
  return true;
}

// pinholepointprojector.h:293-302 (the integer truncation is cv::Vec2i's).
template <class S> static inline int interval_radius(const Projector<S> &P, S d, S world_radius) {
  if (d < P.min_d || d > P.max_d) return -1;
  S p[3];
  for (int i = 0; i < 3; i++) {
    S s = P.K[i * 3 + 0] * world_radius;
    s = s + P.K[i * 3 + 1] * world_radius;
    s = s + P.K[i * 3 + 2] * S(0);
    p[i] = s;
  }
  S inv = S(1) / d;
  S a = p[0] * inv, b = p[1] * inv;
  S m = (a < b) ? b : a;
  return (int)m;
}

// Stats::curvature() (stats.h:93-98): float sum, double +1e-9 and divide.
template <class S> static inline S curvature_of(const S l[3]);
template <> inline float curvature_of<float>(const float l[3]) {
  float s = l[0] + l[1];
  s = s + l[2];
  return (float)((double)l[0] / ((double)s + 1e-9));
}
template <> inline double curvature_of<double>(const double l[3]) {
  double s = l[0] + l[1];
  s = s + l[2];
  return l[0] / (s + 1e-9);
}

// Omega = (U * D) * U^T over the 3x3 block (informationmatrixcalculator.cpp:9-57).
template <class S> static void omega_of(const S U[9], const S D[3], S out[9]) {
  S UD[9];
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) UD[i * 3 + k] = U[i * 3 + k] * D[k];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      S s = UD[i * 3 + 0] * U[j * 3 + 0];
      s = s + UD[i * 3 + 1] * U[j * 3 + 1];
      s = s + UD[i * 3 + 2] * U[j * 3 + 2];
      out[i * 3 + j] = s;
    }
}

// The integral image of the 10 unique point moments, stored image
// row-major (pointintegralimage.cpp:7-44; the reference's PointAccumulator
// holds Sum(p) and Sum(p p^T) with w = 1, i.e. exactly these 10 values).
template <class S> struct Integral {
  int rows = 0, cols = 0;
  std::vector<S> m;  // rows*cols*10
  S *at(int x, int y) { return &m[((size_t)y * cols + x) * 10]; }
  void compute(const int32_t *index, int rows_, int cols_, const std::vector<V4<S>> &pts) {
    rows = rows_; cols = cols_;
    m.assign((size_t)rows * cols * 10, S(0));
    for (int y = 0; y < rows; y++)
      for (int x = 0; x < cols; x++) {
        int idx = index[(size_t)y * cols + x];
        if (idx < 0) continue;
        const V4<S> &p = pts[idx];
        S *a = at(x, y);
        a[0] = S(0) + S(1);
        a[1] = S(0) + p[0]; a[2] = S(0) + p[1]; a[3] = S(0) + p[2];
        a[4] = S(0) + p[0] * p[0]; a[5] = S(0) + p[0] * p[1]; a[6] = S(0) + p[0] * p[2];
        a[7] = S(0) + p[1] * p[1]; a[8] = S(0) + p[1] * p[2]; a[9] = S(0) + p[2] * p[2];
      }
    // prefix along image x, then along image y
#pragma omp parallel for
    for (int y = 0; y < rows; y++)
      for (int x = 1; x < cols; x++) {
        S *a = at(x, y), *b = at(x - 1, y);
        for (int k = 0; k < 10; k++) a[k] = a[k] + b[k];
      }
    for (int y = 1; y < rows; y++) {
#pragma omp parallel for
      for (int x = 0; x < cols; x++) {
        S *a = at(x, y), *b = at(x, y - 1);
        for (int k = 0; k < 10; k++) a[k] = a[k] + b[k];
      }
    }
  }
  // pointintegralimage.cpp:53-66: each bound decremented by one then clamped.
  void region(int xmin, int xmax, int ymin, int ymax, S out[10]) {
    auto cl = [](int v, int lo, int hi) { v = (v < lo) ? lo : v; v = (v > hi) ? hi : v; return v; };
    xmin = cl(xmin - 1, 0, cols - 1);
    xmax = cl(xmax - 1, 0, cols - 1);
    ymin = cl(ymin - 1, 0, rows - 1);
    ymax = cl(ymax - 1, 0, rows - 1);
    S *A = at(xmax, ymax), *B = at(xmin, ymin), *C = at(xmin, ymax), *D = at(xmax, ymin);
    for (int k = 0; k < 10; k++) {
      S s = A[k] + B[k];
      s = s - C[k];
      s = s - D[k];
      out[k] = s;
    }
  }
};

// imageutils.cpp:85-99: dest = scale * src for non-zero pixels, computed in
// float: the converter's input is the float DepthImage this conversion writes
// (cv::Mat_<float>), so both modes start from the same float depths and F64
// promotes them exactly.  (Converting in double instead moves the FP64 pose by
// as much as a one-ulp perturbation of the float depths does; that is a
// different input, not a more precise evaluation of this one.)
template <class S> static inline S cast_depth(float scale, uint16_t u) {
  if (!u) return S(0);
  return S(scale * (float)u);
}

// Cloud::transformInPlace (cloud.cpp:191-204), with the Gaussians moved as
// Gaussian3fVector::transformInPlace does (gaussian3.h:66-73).  Row 3 of m is
// forced to (0 0 0 1); the identity leaves the cloud untouched.
template <class S> static void transform_in_place(Cloud<S> &c, M4<S> m) {
  Cloud<S> *cl = &c;
  const int count = c.n;
  set_row3(m);
  bool ident = true;
  M4<S> I4 = M4<S>::identity();
  for (int i = 0; i < 16; i++) ident = ident && (m.a[i] == I4.a[i]);
  if (ident) return;
  M4<S> Tr = m;
  for (int i = 0; i < 4; i++) { Tr(3, i) = S(0); Tr(i, 3) = S(0); }
  M4<S> Trt = transpose(Tr);
  for (int i = 0; i < count; i++) {
    cl->points[i] = mv(m, cl->points[i]);
    cl->points[i][3] = S(1);
    cl->normals[i] = mv(m, cl->normals[i]);
    cl->normals[i][3] = S(0);
    M4<S> U = M4<S>::zero();
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) U(a, b) = cl->eigvec[9 * i + a * 3 + b];
    M4<S> RU = mm(m, U);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) cl->eigvec[9 * i + a * 3 + b] = RU(a, b);
    // Gaussian3fVector::transformInPlace (gaussian3.h:66-73):
    // mean' = R mean + t, covariance' = (R C) R^T
    {
      S *gm = &cl->gauss_mean[3 * (size_t)i], *gc = &cl->gauss_cov[9 * (size_t)i];
      S mo[3], RC[9];
      for (int a = 0; a < 3; a++) {
        S v = m(a, 0) * gm[0];
        v = v + m(a, 1) * gm[1];
        v = v + m(a, 2) * gm[2];
        mo[a] = v + m(a, 3);
      }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          S v = m(a, 0) * gc[0 * 3 + b];
          v = v + m(a, 1) * gc[1 * 3 + b];
          RC[a * 3 + b] = v + m(a, 2) * gc[2 * 3 + b];
        }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          S v = RC[a * 3 + 0] * m(b, 0);
          v = v + RC[a * 3 + 1] * m(b, 1);
          gc[a * 3 + b] = v + RC[a * 3 + 2] * m(b, 2);
        }
      for (int k = 0; k < 3; k++) gm[k] = mo[k];
    }
    for (int which = 0; which < 2; which++) {
      S *om = which ? &cl->omega_n[9 * i] : &cl->omega_p[9 * i];
      M4<S> O = M4<S>::zero();
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) O(a, b) = om[a * 3 + b];
      M4<S> R = mm(mm(Tr, O), Trt);
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) om[a * 3 + b] = R(a, b);
    }
  }
}

// DepthImageConverterIntegralImage::compute (depthimageconverterintegralimage.cpp:18-64).
template <class S>
static Cloud<S> *build_cloud(const uint16_t *depth, int rows, int cols, const orc_camera &cam,
                             const orc_cloud_params &prm, const double *offset, int32_t *index_out,
                             const float *depth_f32 = nullptr) {
  Projector<S> P = make_projector<S>(cam, M4<S>::identity());
  size_t NP = (size_t)rows * cols;
  std::vector<S> d(NP);
  for (size_t i = 0; i < NP; i++) d[i] = depth_f32 ? S(depth_f32[i]) : cast_depth<S>(prm.depth_scale, depth[i]);
  std::vector<int32_t> index(NP);
  auto *cl = new Cloud<S>();
  // unProject with Gaussians (pinholepointprojector.cpp:93-134)
  int count = 0;
  std::vector<V4<S>> pts;
  pts.reserve(NP);
  std::vector<S> gcov;
  gcov.reserve(NP * 9);
  S fB = P.baseline * P.K[0];
  for (int r = 0; r < rows; r++)
    for (int c = 0; c < cols; c++) {
      S z = d[(size_t)r * cols + c];
      if (z == S(0) || z < P.min_d || z > P.max_d) { index[(size_t)r * cols + c] = -1; continue; }
      V4<S> q = {{S(c) * z, S(r) * z, z, S(1)}};
      V4<S> p = mv(P.iKRt, q);
      p[3] = S(1);
      pts.push_back(p);
      S zv = (P.alpha * z * z) / (fB + z * P.alpha);
      S J[9] = {z, S(0), S(c), S(0), z, S(r), S(0), S(0), S(1)};
      S IJ[9];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          S s = P.iK[i * 3 + 0] * J[0 * 3 + j];
          s = s + P.iK[i * 3 + 1] * J[1 * 3 + j];
          s = s + P.iK[i * 3 + 2] * J[2 * 3 + j];
          IJ[i * 3 + j] = s;
        }
      S Dg[3] = {S(3), S(3), zv};
      S G[9];
      omega_of(IJ, Dg, G);
      for (int k = 0; k < 9; k++) gcov.push_back(G[k]);
      index[(size_t)r * cols + c] = count++;
    }
  cl->resize(count);
  cl->points = pts;
  cl->gauss_cov = gcov;
  cl->gauss_mean.resize(3 * (size_t)count);
  for (int i = 0; i < count; i++)
    for (int k = 0; k < 3; k++) cl->gauss_mean[3 * (size_t)i + k] = pts[i][k];
  // default Stats: identity eigenvectors, zero eigenvalues, curvature 0
  for (int i = 0; i < count; i++) {
    cl->normals[i] = V4<S>{{S(0), S(0), S(0), S(0)}};
    S *U = &cl->eigvec[9 * i];
    U[0] = U[4] = U[8] = S(1);
  }
  // StatsCalculatorIntegralImage::compute (statscalculatorintegralimage.cpp:20-82)
  if (count > 0) {
    Integral<S> I;
    I.compute(index.data(), rows, cols, cl->points);
    S wr = S(prm.world_radius);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < rows; r++)
      for (int c = 0; c < cols; c++) {
        int idx = index[(size_t)r * cols + c];
        int rad = interval_radius(P, d[(size_t)r * cols + c], wr);
        if (idx < 0 || rad < 0) continue;
        if (rad < prm.min_image_radius) continue;
        if (rad > prm.max_image_radius) rad = prm.max_image_radius;
        S acc[10];
        I.region(c - rad, c + rad, r - rad, r + rad, acc);
        int n = (int)acc[0];
        if (n < prm.min_points) continue;
        // PointAccumulator::covariance (pointaccumulator.h:66-86)
        S dn = S(1) / acc[0];
        S mu[3] = {acc[1] * dn, acc[2] * dn, acc[3] * dn};
        S C[6] = {acc[4] * dn - mu[0] * mu[0], acc[5] * dn - mu[0] * mu[1], acc[6] * dn - mu[0] * mu[2],
                  acc[7] * dn - mu[1] * mu[1], acc[8] * dn - mu[1] * mu[2], acc[9] * dn - mu[2] * mu[2]};
        S lam[3], U[9];
        eig3(C, lam, U);
        if (lam[0] < S(0)) lam[0] = S(0);
        for (int k = 0; k < 3; k++) cl->eigval[3 * idx + k] = lam[k];
        for (int k = 0; k < 9; k++) cl->eigvec[9 * idx + k] = U[k];
        cl->stats_n[idx] = n;
        S kappa = curvature_of(lam);
        cl->curvature[idx] = kappa;
        V4<S> nrm = {{U[0], U[3], U[6], S(0)}};
        if (kappa < S(prm.curvature_threshold)) {
          if (dot4(nrm, cl->points[idx]) > S(0)) { nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2]; }
        } else {
          nrm = V4<S>{{S(0), S(0), S(0), S(0)}};
        }
        cl->normals[idx] = nrm;
      }
  }
  // Point/NormalInformationMatrixCalculator::compute
#pragma omp parallel for schedule(static)
  for (int i = 0; i < count; i++) {
    if (!(dot4(cl->normals[i], cl->normals[i]) > S(0))) continue;
    const S *U = &cl->eigvec[9 * i];
    S kappa = cl->curvature[i];
    S Dp[3], Dn[3];
    for (int k = 0; k < 3; k++) {
      Dp[k] = S(kappa < S(prm.pim_curvature_threshold) ? prm.pim_flat[k] : prm.pim_nonflat[k]);
      Dn[k] = S(kappa < S(prm.nim_curvature_threshold) ? prm.nim_flat[k] : prm.nim_nonflat[k]);
    }
    omega_of(U, Dp, &cl->omega_p[9 * i]);
    omega_of(U, Dn, &cl->omega_n[9 * i]);
  }
  // Cloud::transformInPlace(sensorOffset) (cloud.cpp:191-204)
  if (offset) {
    M4<S> m;
    for (int i = 0; i < 16; i++) m.a[i] = S(offset[i]);
    transform_in_place(*cl, m);
  }
  if (index_out) std::memcpy(index_out, index.data(), NP * sizeof(int32_t));
  return cl;
}

// PinholePointProjector::project (pinholepointprojector.cpp:33-66): serial
// z-buffer, the smallest depth wins and ties keep the lowest index.
template <class S>
static void project(const Cloud<S> &c, const Projector<S> &P, int32_t *index, S *depth) {
  size_t NP = (size_t)P.rows * P.cols;
  for (size_t i = 0; i < NP; i++) { index[i] = -1; depth[i] = std::numeric_limits<S>::max(); }
  for (int i = 0; i < c.n; i++) {
    int x, y;
    S d;
    if (!project_point(P, c.points[i], x, y, d) || d < P.min_d || d > P.max_d || x < 0 || x >= P.cols ||
        y < 0 || y >= P.rows)
      continue;
    S &od = depth[(size_t)y * P.cols + x];
    if (!od || od > d) {
      od = d;
      index[(size_t)y * P.cols + x] = i;
    }
  }
}

template <class S> static M4<S> load_T(const double *T16) {
  M4<S> T;
  for (int i = 0; i < 16; i++) T.a[i] = S(T16[i]);
  return T;
}

template <class S> static inline S curv_ratio(S kr, S kc);
template <> inline float curv_ratio<float>(float kr, float kc) {
  return (float)(((double)kr + 1e-5) / ((double)kc + 1e-5));
}
template <> inline double curv_ratio<double>(double kr, double kc) { return (kr + 1e-5) / (kc + 1e-5); }

// CorrespondenceFinderProjective::_computeSingle (correspondencefinderprojective.cpp:23-115).
// With `threads` = T, rows [T*(rows/T), rows) are never visited (the
// reference's partition); the output is row-major over the visited rows.
template <class S>
static int correspond_multi(const Cloud<S> &ref, const Cloud<S> &cur, const int32_t *ri, const int32_t *ci,
                            int rows, int cols, M4<S> T, const orc_align_params &prm, int32_t *pairs,
                            bool f64mode);

template <class S>
static int correspond(const Cloud<S> &ref, const Cloud<S> &cur, const int32_t *ri, const int32_t *ci,
                      int rows, int cols, M4<S> T, const orc_align_params &prm, int32_t *pairs,
                      bool f64mode) {
  if (prm.row_search_region != 0 || prm.col_search_region != 0)  // compute(), :16-21
    return correspond_multi(ref, cur, ri, ci, rows, cols, T, prm, pairs, f64mode);
  set_row3(T);
  S thr = S(prm.inlier_distance_threshold);
  S sq = thr * thr;
  S minr = S(1) / S(prm.inlier_curvature_ratio_threshold);
  S maxr = S(prm.inlier_curvature_ratio_threshold);
  S cosT = S(prm.inlier_normal_angular_threshold);
  S flat = S(prm.flat_curvature_threshold);
  int nth = (f64mode || prm.threads < 1) ? 1 : prm.threads;
  int rpt = rows / nth;
  std::vector<std::vector<int32_t>> local(nth);
#pragma omp parallel for num_threads(nth) schedule(static, 1)
  for (int t = 0; t < nth; t++) {
    std::vector<int32_t> &out = local[t];
    out.reserve((size_t)rpt * cols * 2);
    for (int r = t * rpt; r < (t + 1) * rpt; r++)
      for (int c = 0; c < cols; c++) {
        int a = ri[(size_t)r * cols + c], b = ci[(size_t)r * cols + c];
        if (a < 0 || b < 0) continue;
        const V4<S> &cn = cur.normals[b];
        const V4<S> &rn0 = ref.normals[a];
        const V4<S> &cp = cur.points[b];
        const V4<S> &rp0 = ref.points[a];
        if (!prm.corr_demoted_to_gicp && (dot4(cn, cn) == S(0) || dot4(rn0, rn0) == S(0))) continue;
        V4<S> rp = mv(T, rp0);
        rp[3] = S(1);
        V4<S> rn = mv(T, rn0);
        rn[3] = S(0);
        V4<S> dv = {{cp[0] - rp[0], cp[1] - rp[1], cp[2] - rp[2], cp[3] - rp[3]}};
        if (dot4(dv, dv) > sq) continue;
        if (!prm.corr_demoted_to_gicp) {
          if (dot4(cn, rn) < cosT) continue;
          S kr = ref.curvature[a], kc = cur.curvature[b];
          if (kr < flat) kr = flat;
          if (kc < flat) kc = flat;
          S ratio = curv_ratio<S>(kr, kc);
          if (ratio < minr || ratio > maxr) continue;
        }
        out.push_back(a);
        out.push_back(b);
      }
  }
  int k = 0;
  for (int t = 0; t < nth; t++)
    for (size_t i = 0; i < local[t].size(); i += 2) {
      pairs[2 * k] = local[t][i];
      pairs[2 * k + 1] = local[t][i + 1];
      k++;
    }
  return k;
}

// CorrespondenceFinderProjective::_computeMulti
// (correspondencefinderprojective.cpp:119-257), used by compute() when a
// search region is set (:16-21): every reference pixel looks for the best
// current pixel in the (2 rsr + 1) x (2 csr + 1) window around it (clamped
// to the image), scanned row-major; gates in the order normal present,
// normal angle, distance, curvature ratio; a later candidate replaces the
// kept one only if it is both strictly closer and strictly better aligned.
// Row partition and thread-order assembly as _computeSingle (rows % T
// dropped).
template <class S>
static int correspond_multi(const Cloud<S> &ref, const Cloud<S> &cur, const int32_t *ri, const int32_t *ci,
                            int rows, int cols, M4<S> T, const orc_align_params &prm, int32_t *pairs,
                            bool f64mode) {
  set_row3(T);
  S thr = S(prm.inlier_distance_threshold);
  S sq = thr * thr;
  S minr = S(1) / S(prm.inlier_curvature_ratio_threshold);
  S maxr = S(prm.inlier_curvature_ratio_threshold);
  S cosT = S(prm.inlier_normal_angular_threshold);
  S flat = S(prm.flat_curvature_threshold);
  const int R = prm.row_search_region, Cc = prm.col_search_region;
  int nth = (f64mode || prm.threads < 1) ? 1 : prm.threads;
  int rpt = rows / nth;
  std::vector<std::vector<int32_t>> local(nth);
#pragma omp parallel for num_threads(nth) schedule(static, 1)
  for (int t = 0; t < nth; t++) {
    std::vector<int32_t> &out = local[t];
    for (int r = t * rpt; r < (t + 1) * rpt; r++) {
      const int rmin = std::max(r - R, 0), rmax = std::min(r + R + 1, rows);
      for (int c = 0; c < cols; c++) {
        const int a = ri[(size_t)r * cols + c];
        if (a < 0) continue;
        const V4<S> &rn0 = ref.normals[a];
        if (dot4(rn0, rn0) == S(0)) continue;
        V4<S> rp = mv(T, ref.points[a]);
        rp[3] = S(1);
        V4<S> rn = mv(T, rn0);
        rn[3] = S(0);
        S kr = ref.curvature[a];
        if (kr < flat) kr = flat;
        const int cmin = std::max(c - Cc, 0), cmax = std::min(c + Cc + 1, cols);
        int best = -1;
        S bestN = S(0), bestD = S(1e20);
        for (int r2 = rmin; r2 < rmax; r2++)
          for (int c2 = cmin; c2 < cmax; c2++) {
            const int b = ci[(size_t)r2 * cols + c2];
            if (b < 0) continue;
            const V4<S> &cn = cur.normals[b];
            if (dot4(cn, cn) == S(0)) continue;
            const V4<S> &cp = cur.points[b];
            const S nd = dot4(cn, rn);
            if (nd < cosT) continue;
            V4<S> dv = {{cp[0] - rp[0], cp[1] - rp[1], cp[2] - rp[2], cp[3] - rp[3]}};
            const S d = dot4(dv, dv);
            if (d > sq) continue;
            S kc = cur.curvature[b];
            if (kc < flat) kc = flat;
            const S ratio = curv_ratio<S>(kr, kc);
            if (ratio < minr || ratio > maxr) continue;
            if (best == -1 || (d < bestD && nd > bestN)) {
              best = b;
              bestN = nd;
              bestD = d;
            }
          }
        if (best > -1) {
          out.push_back(a);
          out.push_back(best);
        }
      }
    }
  }
  int k = 0;
  for (int t = 0; t < nth; t++)
    for (size_t i = 0; i < local[t].size(); i += 2) {
      pairs[2 * k] = local[t][i];
      pairs[2 * k + 1] = local[t][i + 1];
      k++;
    }
  return k;
}

template <class S> static inline M4<S> skew4(const V4<S> &v) {
  M4<S> s = M4<S>::zero();
  S tx = S(2) * v[0], ty = S(2) * v[1], tz = S(2) * v[2];
  s(0, 1) = tz;  s(1, 0) = -tz;
  s(0, 2) = -ty; s(2, 0) = ty;
  s(1, 2) = tx;  s(2, 1) = -tx;
  return s;
}

template <class S> static inline M4<S> om4(const S *o9) {
  M4<S> O = M4<S>::zero();
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) O(a, b) = o9[a * 3 + b];
  return O;
}

// Linearizer::update (linearizer.cpp:21-134).
template <class S>
static void linearize(const Cloud<S> &ref, const Cloud<S> &cur, const int32_t *pairs, int K, M4<S> T,
                      const orc_align_params &prm, bool f64mode, double H36[36], double b6[6],
                      double *error_out, int *inliers_out) {
  set_row3(T);
  int nth = (f64mode || prm.threads < 1) ? 1 : prm.threads;
  int ipt = K / nth;
  M4<S> HttT = M4<S>::zero(), HtrT = M4<S>::zero(), HrrT = M4<S>::zero();
  V4<S> btT = {{S(0), S(0), S(0), S(0)}}, brT = btT;
  S errT = S(0);
  int inlT = 0;
  S maxc = S(prm.inlier_max_chi2);
  S scale = S(prm.lin_scale);
  struct Part { M4<S> Htt, Htr, Hrr; V4<S> bt, br; S err; int inl; };
  std::vector<Part> parts(nth);
#pragma omp parallel for num_threads(nth) schedule(static, 1)
  for (int t = 0; t < nth; t++) {
    int imin = ipt * t, imax = imin + ipt;
    if (imax > K) imax = K;
    M4<S> Htt = M4<S>::zero(), Htr = M4<S>::zero(), Hrr = M4<S>::zero();
    V4<S> bt = {{S(0), S(0), S(0), S(0)}}, br = bt;
    S err = S(0);
    int inl = 0;
    for (int i = imin; i < imax; i++) {
      int a = pairs[2 * i], b = pairs[2 * i + 1];
      V4<S> rp = mv(T, ref.points[a]);
      rp[3] = S(1);
      V4<S> rn = mv(T, ref.normals[a]);
      rn[3] = S(0);
      const V4<S> &cp = cur.points[b];
      const V4<S> &cn = cur.normals[b];
      M4<S> Op = om4(&cur.omega_p[9 * b]);
      M4<S> On = om4(&cur.omega_n[9 * b]);
      for (int k = 0; k < 16; k++) On.a[k] = scale * On.a[k];
      if (prm.z_scaling) {
        S f = S(1) / std::fabs(cp[2]);
        for (int k = 0; k < 16; k++) { Op.a[k] = Op.a[k] * f; On.a[k] = On.a[k] * f; }
      }
      if (prm.lin_demoted_to_gicp) On = M4<S>::zero();
      V4<S> pe = {{rp[0] - cp[0], rp[1] - cp[1], rp[2] - cp[2], rp[3] - cp[3]}};
      V4<S> ne = {{rn[0] - cn[0], rn[1] - cn[1], rn[2] - cn[2], rn[3] - cn[3]}};
      V4<S> ep = mv(Op, pe), en = mv(On, ne);
      S le = dot4(pe, ep) + dot4(ne, en);
      S ks = S(1);
      if (le > maxc) {
        if (prm.robust_kernel) ks = maxc / le;
        else continue;
      }
      inl++;
      err = err + ks * le;
      M4<S> Sp = skew4(rp), Sn = skew4(rn);
      M4<S> Spt = transpose(Sp), Snt = transpose(Sn);
      M4<S> OpSp = mm(Op, Sp);
      M4<S> A = mm(mm(Spt, Op), Sp), B = mm(mm(Snt, On), Sn);
      V4<S> u = mv(Spt, ep), w = mv(Snt, en);
      for (int k = 0; k < 16; k++) {
        Htt.a[k] = Htt.a[k] + Op.a[k] * ks;
        Htr.a[k] = Htr.a[k] + OpSp.a[k] * ks;
        Hrr.a[k] = Hrr.a[k] + (A.a[k] + B.a[k]) * ks;
      }
      for (int k = 0; k < 4; k++) {
        bt[k] = bt[k] + ks * ep[k];
        br[k] = br[k] + ks * (u[k] + w[k]);
      }
    }
    parts[t] = Part{Htt, Htr, Hrr, bt, br, err, inl};
  }
  // thread-order reduction of the per-thread float partials (linearizer.cpp:111-127)
  for (int t = 0; t < nth; t++) {
    const Part &p = parts[t];
    for (int k = 0; k < 16; k++) {
      HttT.a[k] = HttT.a[k] + p.Htt.a[k];
      HtrT.a[k] = HtrT.a[k] + p.Htr.a[k];
      HrrT.a[k] = HrrT.a[k] + p.Hrr.a[k];
    }
    for (int k = 0; k < 4; k++) { btT[k] = btT[k] + p.bt[k]; brT[k] = brT[k] + p.br[k]; }
    errT = errT + p.err;
    inlT += p.inl;
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      H36[i * 6 + j] = (double)HttT(i, j);
      H36[i * 6 + 3 + j] = (double)HtrT(i, j);
      H36[(3 + i) * 6 + 3 + j] = (double)HrrT(i, j);
      H36[(3 + i) * 6 + j] = (double)HtrT(j, i);
    }
  for (int i = 0; i < 3; i++) { b6[i] = (double)btT[i]; b6[3 + i] = (double)brT[i]; }
  *error_out = (double)errT;
  *inliers_out = inlT;
}

// ----------------------------------------------- solution statistics (FP64)
// Aligner::_computeStatistics (aligner.cpp:82-135) with unscented.h:23-65.
static void jacobi_eig(int n, double *A, double *V, double *w) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) V[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) off += A[i * n + j] * A[i * n + j];
    if (off < 1e-300) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        double apq = A[p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < n; k++) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; i++) w[i] = A[i * n + i];
}

static bool inverse6(const double *A, double *out) {
  double M[6][12];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 12; j++) M[i][j] = (j < 6) ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; c++) {
    int p = c;
    for (int r = c + 1; r < 6; r++)
      if (std::fabs(M[r][c]) > std::fabs(M[p][c])) p = r;
    if (M[p][c] == 0) return false;
    if (p != c)
      for (int j = 0; j < 12; j++) std::swap(M[p][j], M[c][j]);
    double iv = 1 / M[c][c];
    for (int j = 0; j < 12; j++) M[c][j] *= iv;
    for (int r = 0; r < 6; r++)
      if (r != c) {
        double f = M[r][c];
        for (int j = 0; j < 12; j++) M[r][j] -= f * M[c][j];
      }
  }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) out[i * 6 + j] = M[i][j + 6];
  return true;
}

static void solution_statistics(const double H36[36], const M4<double> &T, double *tr, double *rr,
                                double *omega36, double *mean6) {
  *tr = std::numeric_limits<double>::max();
  *rr = std::numeric_limits<double>::max();
  for (int i = 0; i < 36; i++) omega36[i] = 0;
  for (int i = 0; i < 6; i++) mean6[i] = 0;
  double A[36], V[36], w[6];
  for (int i = 0; i < 36; i++) A[i] = H36[i];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < i; j++) A[i * 6 + j] = A[j * 6 + i] = 0.5 * (H36[i * 6 + j] + H36[j * 6 + i]);
  jacobi_eig(6, A, V, w);
  double smax = 0;
  for (int i = 0; i < 6; i++) smax = std::max(smax, std::fabs(w[i]));
  double thr = smax * 6 * (double)FLT_EPSILON;
  double Sig[36] = {0};
  for (int k = 0; k < 6; k++) {
    if (!(std::fabs(w[k]) > thr)) continue;
    double iv = 1.0 / w[k];
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) Sig[i * 6 + j] += V[i * 6 + k] * iv * V[j * 6 + k];
  }
  const int dim = 6, np = 13;
  const double alpha = 1e-3, beta = 2.0, lambda = alpha * alpha * dim;
  const double wi = 1.0 / (2.0 * (dim + lambda));
  double L[36] = {0};
  double C[36];
  for (int i = 0; i < 36; i++) C[i] = Sig[i] * (dim + lambda);
  for (int j = 0; j < 6; j++) {
    double s = C[j * 6 + j];
    for (int k = 0; k < j; k++) s -= L[j * 6 + k] * L[j * 6 + k];
    if (!(s > 0)) return;
    L[j * 6 + j] = std::sqrt(s);
    for (int i = j + 1; i < 6; i++) {
      double t = C[i * 6 + j];
      for (int k = 0; k < j; k++) t -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = t / L[j * 6 + j];
    }
  }
  double samp[np][6], wmean[np], wcov[np];
  for (int k = 0; k < 6; k++) samp[0][k] = 0;
  wmean[0] = lambda / (dim + lambda);
  wcov[0] = lambda / (dim + lambda) + (1.0 - alpha * alpha + beta);
  for (int i = 0; i < 6; i++)
    for (int s = 0; s < 2; s++) {
      int k = 1 + 2 * i + s;
      for (int r = 0; r < 6; r++) samp[k][r] = (s ? -1.0 : 1.0) * L[r * 6 + i];
      wmean[k] = wcov[k] = wi;
    }
  for (int k = 0; k < np; k++) {
    M4<double> X = iso_inverse(v2t(samp[k]));
    M4<double> Y = mm(T, X);
    t2v(Y, samp[k]);
  }
  double mean[6] = {0}, cov[36] = {0};
  for (int k = 0; k < np; k++)
    for (int r = 0; r < 6; r++) mean[r] += wmean[k] * samp[k][r];
  for (int k = 0; k < np; k++)
    for (int r = 0; r < 6; r++)
      for (int c = 0; c < 6; c++) cov[r * 6 + c] += wcov[k] * (samp[k][r] - mean[r]) * (samp[k][c] - mean[c]);
  for (int i = 0; i < 6; i++) mean6[i] = mean[i];
  double Om[36];
  if (!inverse6(cov, Om)) return;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) A[i * 6 + j] = 0.5 * (Om[i * 6 + j] + Om[j * 6 + i]);
  for (int i = 0; i < 36; i++) omega36[i] = A[i];
  for (int blk = 0; blk < 2; blk++) {
    double B6[6] = {A[(3 * blk) * 6 + 3 * blk], A[(3 * blk) * 6 + 3 * blk + 1], A[(3 * blk) * 6 + 3 * blk + 2],
                    A[(3 * blk + 1) * 6 + 3 * blk + 1], A[(3 * blk + 1) * 6 + 3 * blk + 2],
                    A[(3 * blk + 2) * 6 + 3 * blk + 2]};
    double lam[3], U[9];
    eig3(B6, lam, U);
    double s0 = std::max(std::fabs(lam[0]), std::max(std::fabs(lam[1]), std::fabs(lam[2])));
    double s2 = std::min(std::fabs(lam[0]), std::min(std::fabs(lam[1]), std::fabs(lam[2])));
    double ratio = s0 / s2;
    if (blk == 0) *tr = ratio; else *rr = ratio;
  }
}

// AlignerProjective::align (alignerprojective.cpp:21-136).
template <class S>
static void align(const Cloud<S> &ref, const Cloud<S> &cur, const orc_camera &cam, const double *guess,
                  const double *roff, const double *coff, const orc_align_params &prm, bool f64mode,
                  int stats, orc_align_result *out) {
  M4<S> I4 = M4<S>::identity();
  M4<S> G = guess ? load_T<S>(guess) : I4;
  M4<S> RO = roff ? load_T<S>(roff) : I4;
  M4<S> CO = coff ? load_T<S>(coff) : I4;
  Projector<S> Pc = make_projector<S>(cam, CO);
  size_t NP = (size_t)Pc.rows * Pc.cols;
  std::vector<int32_t> ci(NP), ri(NP), pairs(2 * NP);
  std::vector<S> cd(NP), rd(NP);
  project(cur, Pc, ci.data(), cd.data());
  M4<S> T = G;
  double H[36], b[6], err = 0;
  int inl = 0, K = 0, run = 0;
  for (int i = 0; i < prm.outer_iterations; i++) {
    set_row3(T);
    const M4<S> Tstart = T;
    Projector<S> Pr = make_projector<S>(cam, mm(T, RO));
    project(ref, Pr, ri.data(), rd.data());
    K = correspond(ref, cur, ri.data(), ci.data(), Pr.rows, Pr.cols, iso_inverse(T), prm, pairs.data(), f64mode);
    M4<S> invT = iso_inverse(T);
    for (int k = 0; k < prm.inner_iterations; k++) {
      set_row3(invT);
      linearize(ref, cur, pairs.data(), K, invT, prm, f64mode, H, b, &err, &inl);
      S Hs[36], bs[6], dx[6];
      for (int q = 0; q < 36; q++) Hs[q] = S(H[q]);
      for (int q = 0; q < 6; q++) { Hs[q * 6 + q] = Hs[q * 6 + q] + S(prm.lambda); bs[q] = -S(b[q]); }
      ldlt_solve(Hs, bs, dx);
      invT = mm(v2t(dx), invT);
    }
    T = iso_inverse(invT);
    S x[6];
    t2v(T, x);
    T = v2t(x);
    set_row3(T);
    run++;
    if (prm.early_exit_eps > 0) {  // new (the reference always runs every iteration)
      S dv[6];
      t2v(mm(T, iso_inverse(Tstart)), dv);
      double m = 0;
      for (int k = 0; k < 6; k++) m = std::max(m, std::fabs((double)dv[k]));
      if (m < prm.early_exit_eps) break;
    }
  }
  for (int i = 0; i < 16; i++) out->T[i] = (double)T.a[i];
  out->error = err;
  out->inliers = inl;
  out->num_correspondences = K;
  out->outer_iterations_run = run;
  out->translational_ratio = out->rotational_ratio = 0;
  out->solution_valid = 0;
  for (int i = 0; i < 36; i++) out->omega[i] = 0;
  for (int i = 0; i < 6; i++) out->mean[i] = 0;
  if (stats) {
    M4<S> invT = iso_inverse(T);
    set_row3(invT);
    double Hs[36], bs[6], e2;
    int i2;
    linearize(ref, cur, pairs.data(), K, invT, prm, f64mode, Hs, bs, &e2, &i2);
    M4<double> Td;
    for (int i = 0; i < 16; i++) Td.a[i] = (double)T.a[i];
    solution_statistics(Hs, Td, &out->translational_ratio, &out->rotational_ratio, out->omega, out->mean);
    out->solution_valid = !(out->rotational_ratio > prm.rotational_min_eigen_ratio ||
                            out->translational_ratio > prm.translational_min_eigen_ratio);
  }
}

// CorrespondenceFinderNN::compute (correspondencefindernn.cpp:44-97) with
// an exact nearest neighbour where the reference asks FLANN's randomized
// kd-tree (approximate, 16 checks) for the nearest current point within
// the squared radius in the 6-D space (p, s n): here every current point is
// tested, the smallest squared distance wins and ties keep the lowest index.
// Distances sum the six squared differences in coordinate order.  T is the
// transform applied to the reference (the aligner passes _T.inverse()).
template <class S>
static int correspond_nn(const Cloud<S> &ref, const Cloud<S> &cur, M4<S> T, S nscale,
                         const orc_align_params &prm, int32_t *pairs) {
  set_row3(T);
  const S thr = S(prm.inlier_distance_threshold);
  const S sq = thr * thr;
  const S cosT = S(prm.inlier_normal_angular_threshold);
  const int nr = ref.n, nc = cur.n;
  std::vector<S> cf(6 * (size_t)nc);
  for (int j = 0; j < nc; j++) {  // _model2linear(dest, src, nscale)
    for (int a = 0; a < 3; a++) cf[6 * (size_t)j + a] = cur.points[j][a];
    for (int a = 0; a < 3; a++) cf[6 * (size_t)j + 3 + a] = nscale * cur.normals[j][a];
  }
  M4<S> sR = M4<S>::zero();  // T.linear() * nscale
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) sR(a, b) = T(a, b) * nscale;
  std::vector<int32_t> match(nr, -1);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < nr; i++) {
    V4<S> p = mv(T, ref.points[i]);
    V4<S> n0 = ref.normals[i];
    n0[3] = S(0);
    V4<S> sn = mv(sR, n0);
    const S q[6] = {p[0], p[1], p[2], sn[0], sn[1], sn[2]};
    int best = -1;
    S bd = S(0);
    for (int j = 0; j < nc; j++) {
      const S *c = &cf[6 * (size_t)j];
      S d = S(0);
      for (int a = 0; a < 6; a++) {
        S e = q[a] - c[a];
        d = d + e * e;
      }
      if (d < sq && (best < 0 || d < bd)) { best = j; bd = d; }
    }
    if (best < 0) continue;
    // the gates (correspondencefindernn.cpp:80-93)
    M4<S> R = T;
    for (int a = 0; a < 3; a++) R(a, 3) = S(0);
    V4<S> rn = mv(R, n0);
    V4<S> rp = p;
    const V4<S> &cn = cur.normals[best], &cp = cur.points[best];
    S rn2 = rn[0] * rn[0]; rn2 = rn2 + rn[1] * rn[1]; rn2 = rn2 + rn[2] * rn[2];
    S cn2 = cn[0] * cn[0]; cn2 = cn2 + cn[1] * cn[1]; cn2 = cn2 + cn[2] * cn[2];
    if (!prm.corr_demoted_to_gicp && (rn2 == S(0) || cn2 == S(0))) continue;
    S dx = rp[0] - cp[0], dy = rp[1] - cp[1], dz = rp[2] - cp[2];
    S dd = dx * dx; dd = dd + dy * dy; dd = dd + dz * dz;
    if (dd > sq) continue;
    if (std::isnan(cn[0]) || std::isnan(cn[1]) || std::isnan(cn[2]) || std::isnan(rn[0]) || std::isnan(rn[1]) ||
        std::isnan(rn[2]))
      continue;
    S dot = rn[0] * cn[0]; dot = dot + rn[1] * cn[1]; dot = dot + rn[2] * cn[2];
    if (!prm.corr_demoted_to_gicp && dot < cosT) continue;
    match[i] = best;
  }
  int K = 0;
  for (int i = 0; i < nr; i++)
    if (match[i] >= 0) {
      pairs[2 * K] = i;
      pairs[2 * K + 1] = match[i];
      K++;
    }
  return K;
}

// AlignerNN::align (alignernn.cpp:21-118): AlignerProjective's loop with
// nearest-neighbour correspondences (no projection).
template <class S>
static void align_nn(const Cloud<S> &ref, const Cloud<S> &cur, const double *guess, S nscale,
                     const orc_align_params &prm, bool f64mode, int stats, orc_align_result *out) {
  M4<S> T = guess ? load_T<S>(guess) : M4<S>::identity();
  std::vector<int32_t> pairs(2 * (size_t)std::max(ref.n, 1));
  double H[36], b[6], err = 0;
  int inl = 0, K = 0, run = 0;
  for (int i = 0; i < prm.outer_iterations; i++) {
    set_row3(T);
    const M4<S> Tstart = T;
    K = correspond_nn(ref, cur, iso_inverse(T), nscale, prm, pairs.data());
    M4<S> invT = iso_inverse(T);
    for (int k = 0; k < prm.inner_iterations; k++) {
      set_row3(invT);
      linearize(ref, cur, pairs.data(), K, invT, prm, f64mode, H, b, &err, &inl);
      S Hs[36], bs[6], dx[6];
      for (int q = 0; q < 36; q++) Hs[q] = S(H[q]);
      for (int q = 0; q < 6; q++) { Hs[q * 6 + q] = Hs[q * 6 + q] + S(prm.lambda); bs[q] = -S(b[q]); }
      ldlt_solve(Hs, bs, dx);
      invT = mm(v2t(dx), invT);
    }
    T = iso_inverse(invT);
    S x[6];
    t2v(T, x);
    T = v2t(x);
    set_row3(T);
    run++;
    if (prm.early_exit_eps > 0) {  // new (the reference always runs every iteration)
      S dv[6];
      t2v(mm(T, iso_inverse(Tstart)), dv);
      double m = 0;
      for (int k = 0; k < 6; k++) m = std::max(m, std::fabs((double)dv[k]));
      if (m < prm.early_exit_eps) break;
    }
  }
  for (int i = 0; i < 16; i++) out->T[i] = (double)T.a[i];
  out->error = err;
  out->inliers = inl;
  out->num_correspondences = K;
  out->outer_iterations_run = run;
  out->translational_ratio = out->rotational_ratio = 0;
  out->solution_valid = 0;
  for (int i = 0; i < 36; i++) out->omega[i] = 0;
  for (int i = 0; i < 6; i++) out->mean[i] = 0;
  if (stats) {
    M4<S> invT = iso_inverse(T);
    set_row3(invT);
    double Hs[36], bs[6], e2;
    int i2;
    linearize(ref, cur, pairs.data(), K, invT, prm, f64mode, Hs, bs, &e2, &i2);
    M4<double> Td;
    for (int i = 0; i < 16; i++) Td.a[i] = (double)T.a[i];
    solution_statistics(Hs, Td, &out->translational_ratio, &out->rotational_ratio, out->omega, out->mean);
    out->solution_valid = !(out->rotational_ratio > prm.rotational_min_eigen_ratio ||
                            out->translational_ratio > prm.translational_min_eigen_ratio);
  }
}

}  // namespace orc

using namespace orc;

struct orc_cloud {
  int mode;
  Cloud<float> *f;
  Cloud<double> *d;
};

template <class S> static Cloud<S> *get(const orc_cloud *c);
template <> Cloud<float> *get<float>(const orc_cloud *c) { return c->f; }
template <> Cloud<double> *get<double>(const orc_cloud *c) { return c->d; }

// Definitions below take C linkage from their declarations in nicp_oracle.h.

void orc_convert_u16(const uint16_t *src, int rows, int cols, float scale, float *dst) {
  for (size_t i = 0; i < (size_t)rows * cols; i++) dst[i] = cast_depth<float>(scale, src[i]);
}

// DepthImage_scale (imageutils.cpp:6-37): each output pixel is the mean of
// the step x step block's positive depths (zeros add nothing to the sums but
// are not counted), or 0 when the block has none or its variance
// acc2/np - mu^2 exceeds max_cov.  Float, in the reference's loop order.
void orc_depth_scale(const float *src, int rows, int cols, int step, float max_cov, float *dst) {
  const int R = rows / step, Cn = cols / step;
  for (int r = 0; r < R; r++)
    for (int c = 0; c < Cn; c++) {
      float acc = 0, acc2 = 0;
      int np = 0;
      const int sr = r * step, sc = c * step;
      for (int i = 0; i < step; i++)
        for (int j = 0; j < step; j++)
          if (sr + i < rows && sc + j < cols) {
            const float f = src[(size_t)(sr + i) * cols + sc + j];
            acc += f;
            acc2 += f * f;
            np += f > 0;
          }
      float out = 0;
      if (np) {
        float mu = acc / np;
        float sigma = acc2 / np - mu * mu;
        if (!(sigma > max_cov)) out = mu;
      }
      dst[(size_t)r * Cn + c] = out;
    }
}

orc_cloud *orc_cloud_build_f32(int mode, const float *depth, int rows, int cols, const orc_camera *cam,
                               const orc_cloud_params *prm, const double *offset, int32_t *index_out) {
  auto *c = new orc_cloud{mode, nullptr, nullptr};
  if (mode == ORC_F64) c->d = build_cloud<double>(nullptr, rows, cols, *cam, *prm, offset, index_out, depth);
  else c->f = build_cloud<float>(nullptr, rows, cols, *cam, *prm, offset, index_out, depth);
  return c;
}

orc_cloud *orc_cloud_build_u16(int mode, const uint16_t *depth, int rows, int cols, const orc_camera *cam,
                               const orc_cloud_params *prm, const double *offset, int32_t *index_out) {
  auto *c = new orc_cloud{mode, nullptr, nullptr};
  if (mode == ORC_F64) c->d = build_cloud<double>(depth, rows, cols, *cam, *prm, offset, index_out);
  else c->f = build_cloud<float>(depth, rows, cols, *cam, *prm, offset, index_out);
  return c;
}

template <class S>
static Cloud<S> *from_arrays(int n, const double *p4, const double *n4, const double *k, const double *op,
                             const double *on) {
  auto *c = new Cloud<S>();
  c->resize(n);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < 4; j++) {
      c->points[i][j] = S(p4[4 * i + j]);
      c->normals[i][j] = S(n4[4 * i + j]);
    }
    c->curvature[i] = S(k[i]);
    for (int j = 0; j < 9; j++) {
      c->omega_p[9 * i + j] = op ? S(op[9 * i + j]) : S(0);
      c->omega_n[9 * i + j] = on ? S(on[9 * i + j]) : S(0);
    }
  }
  return c;
}

orc_cloud *orc_cloud_from_arrays(int mode, int n, const double *p4, const double *n4, const double *k,
                                 const double *op, const double *on) {
  auto *c = new orc_cloud{mode, nullptr, nullptr};
  if (mode == ORC_F64) c->d = from_arrays<double>(n, p4, n4, k, op, on);
  else c->f = from_arrays<float>(n, p4, n4, k, op, on);
  return c;
}

void orc_cloud_free(orc_cloud *c) {
  if (!c) return;
  delete c->f;
  delete c->d;
  delete c;
}

int orc_cloud_size(const orc_cloud *c) { return c->mode == ORC_F64 ? c->d->n : c->f->n; }

// Cloud::add (cloud.cpp:163-189): `src` is transformed in place by T, then
// appended to `dst`.
template <class S> static void cloud_add(Cloud<S> &dst, Cloud<S> &src, const M4<S> &T) {
  transform_in_place(src, T);
  Cloud<S> out = dst;
  const int a = dst.n, b = src.n;
  out.n = a + b;
  auto cat = [](std::vector<S> &x, const std::vector<S> &y) { x.insert(x.end(), y.begin(), y.end()); };
  out.points.insert(out.points.end(), src.points.begin(), src.points.end());
  out.normals.insert(out.normals.end(), src.normals.begin(), src.normals.end());
  cat(out.curvature, src.curvature);
  cat(out.eigval, src.eigval);
  cat(out.eigvec, src.eigvec);
  cat(out.omega_p, src.omega_p);
  cat(out.omega_n, src.omega_n);
  cat(out.gauss_cov, src.gauss_cov);
  cat(out.gauss_mean, src.gauss_mean);
  out.stats_n.insert(out.stats_n.end(), src.stats_n.begin(), src.stats_n.end());
  dst = out;
}

// Gaussian<float,3>::_updateInfo (gaussian.h): information matrix = C^-1,
// information vector = (C^-1) mean; products in the order written.
template <class S> static void gaussian_info(const S C[9], const S mean[3], S Om[9], S eta[3]) {
  inv3(C, Om);
  for (int a = 0; a < 3; a++) {
    S v = Om[a * 3 + 0] * mean[0];
    v = v + Om[a * 3 + 1] * mean[1];
    eta[a] = v + Om[a * 3 + 2] * mean[2];
  }
}

// Merger::merge (merger.cpp:15-109).  Project the cloud with `T` (serial
// z-buffer, as PinholePointProjector::project); then, point by point in
// index order: a point that wins its own pixel is kept ("collapsed" onto
// itself); a point whose depth is within `dthr` of the pixel's winner adds
// its information (Gaussian3f::addInformation) to the winner and is
// removed.  Survivors that won their pixel take the mean of their (fused)
// Gaussian as their position; the cloud is compacted in index order.
// Returns the number of removed points.
template <class S> static int merge(Cloud<S> &c, const orc_camera &cam, const M4<S> &T, S dthr, S maxd) {
  Projector<S> P = make_projector<S>(cam, T);
  const size_t NP = (size_t)P.rows * P.cols;
  std::vector<int32_t> index(NP);
  std::vector<S> depth(NP);
  project(c, P, index.data(), depth.data());
  const int n = c.n;
  std::vector<int> collapsed(n, -1);
  std::vector<char> info(n, 0);
  std::vector<S> Om(9 * (size_t)n), eta(3 * (size_t)n);
  auto update_info = [&](int i) {
    if (info[i]) return;
    gaussian_info(&c.gauss_cov[9 * (size_t)i], &c.gauss_mean[3 * (size_t)i], &Om[9 * (size_t)i], &eta[3 * (size_t)i]);
    info[i] = 1;
  };
  for (int i = 0; i < n; i++) {
    int x = -1, y = -1;
    S d = S(0);
    if (!project_point(P, c.points[i], x, y, d)) continue;  // x, y stay -1 in the reference
    if (d < S(0) || d > maxd || y < 0 || y >= P.rows || x < 0 || x >= P.cols) continue;
    const size_t pix = (size_t)y * P.cols + x;
    const int target = index[pix];
    if (target < 0) continue;
    if (target == i) {
      collapsed[i] = i;
    } else if (std::fabs(d - depth[pix]) < dthr) {
      update_info(target);
      S Oi[9], ei[3];
      gaussian_info(&c.gauss_cov[9 * (size_t)i], &c.gauss_mean[3 * (size_t)i], Oi, ei);
      for (int k = 0; k < 9; k++) Om[9 * (size_t)target + k] = Om[9 * (size_t)target + k] + Oi[k];
      for (int k = 0; k < 3; k++) eta[3 * (size_t)target + k] = eta[3 * (size_t)target + k] + ei[k];
      collapsed[i] = target;
    }
  }
  // Gaussian3f::_updateMoments for the fused ones: C = Om^-1, mean = C eta
  for (int i = 0; i < n; i++) {
    if (!info[i]) continue;
    S Cn[9], mn[3];
    inv3(&Om[9 * (size_t)i], Cn);
    for (int a = 0; a < 3; a++) {
      S v = Cn[a * 3 + 0] * eta[3 * (size_t)i + 0];
      v = v + Cn[a * 3 + 1] * eta[3 * (size_t)i + 1];
      mn[a] = v + Cn[a * 3 + 2] * eta[3 * (size_t)i + 2];
    }
    for (int k = 0; k < 9; k++) c.gauss_cov[9 * (size_t)i + k] = Cn[k];
    for (int k = 0; k < 3; k++) c.gauss_mean[3 * (size_t)i + k] = mn[k];
  }
  int k = 0, removed = 0;
  for (int i = 0; i < n; i++) {
    if (collapsed[i] == i)
      for (int a = 0; a < 3; a++) c.points[i][a] = c.gauss_mean[3 * (size_t)i + a];
    if (collapsed[i] < 0 || collapsed[i] == i) {
      c.points[k] = c.points[i];
      c.normals[k] = c.normals[i];
      c.curvature[k] = c.curvature[i];
      c.stats_n[k] = c.stats_n[i];
      for (int a = 0; a < 3; a++) c.eigval[3 * (size_t)k + a] = c.eigval[3 * (size_t)i + a];
      for (int a = 0; a < 9; a++) {
        c.eigvec[9 * (size_t)k + a] = c.eigvec[9 * (size_t)i + a];
        c.omega_p[9 * (size_t)k + a] = c.omega_p[9 * (size_t)i + a];
        c.omega_n[9 * (size_t)k + a] = c.omega_n[9 * (size_t)i + a];
        c.gauss_cov[9 * (size_t)k + a] = c.gauss_cov[9 * (size_t)i + a];
      }
      for (int a = 0; a < 3; a++) c.gauss_mean[3 * (size_t)k + a] = c.gauss_mean[3 * (size_t)i + a];
      k++;
    } else {
      removed++;
    }
  }
  c.points.resize(k); c.normals.resize(k); c.curvature.resize(k); c.stats_n.resize(k);
  c.eigval.resize(3 * (size_t)k); c.eigvec.resize(9 * (size_t)k);
  c.omega_p.resize(9 * (size_t)k); c.omega_n.resize(9 * (size_t)k);
  c.gauss_cov.resize(9 * (size_t)k); c.gauss_mean.resize(3 * (size_t)k);
  c.n = k;
  return removed;
}

void orc_cloud_transform(orc_cloud *c, const double *T16) {
  if (c->mode == ORC_F64) transform_in_place(*c->d, load_T<double>(T16));
  else transform_in_place(*c->f, load_T<float>(T16));
}

void orc_cloud_add(orc_cloud *dst, orc_cloud *src, const double *T16) {
  if (dst->mode == ORC_F64) cloud_add(*dst->d, *src->d, load_T<double>(T16));
  else cloud_add(*dst->f, *src->f, load_T<float>(T16));
}

int orc_merge(int mode, orc_cloud *c, const orc_camera *cam, const double *T16, double distance_threshold,
              double max_point_depth) {
  if (mode == ORC_F64)
    return merge(*c->d, *cam, load_T<double>(T16), distance_threshold, max_point_depth);
  return merge(*c->f, *cam, load_T<float>(T16), (float)distance_threshold, (float)max_point_depth);
}

template <class S> static int cloud_get(const Cloud<S> &c, int field, double *out) {
  int n = c.n;
  switch (field) {
    case 0: for (int i = 0; i < n; i++) for (int j = 0; j < 4; j++) out[4 * i + j] = c.points[i][j]; return 4 * n;
    case 1: for (int i = 0; i < n; i++) for (int j = 0; j < 4; j++) out[4 * i + j] = c.normals[i][j]; return 4 * n;
    case 2: for (int i = 0; i < n; i++) out[i] = c.curvature[i]; return n;
    case 3: for (int i = 0; i < 9 * n; i++) out[i] = c.omega_p[i]; return 9 * n;
    case 4: for (int i = 0; i < 9 * n; i++) out[i] = c.omega_n[i]; return 9 * n;
    case 5: for (int i = 0; i < 3 * n; i++) out[i] = c.eigval[i]; return 3 * n;
    case 6: for (int i = 0; i < 9 * n; i++) out[i] = c.eigvec[i]; return 9 * n;
    case 7: for (int i = 0; i < n; i++) out[i] = c.stats_n[i]; return n;
    case 8: for (int i = 0; i < 9 * n && i < (int)c.gauss_cov.size(); i++) out[i] = c.gauss_cov[i]; return 9 * n;
    case 9: for (int i = 0; i < 3 * n && i < (int)c.gauss_mean.size(); i++) out[i] = c.gauss_mean[i]; return 3 * n;
  }
  return -1;
}

int orc_cloud_get(const orc_cloud *c, int field, double *out) {
  return c->mode == ORC_F64 ? cloud_get(*c->d, field, out) : cloud_get(*c->f, field, out);
}

template <class S> static void proj_mats(const orc_camera *cam, const double *T16, double *KRt, double *iKRt) {
  Projector<S> P = make_projector<S>(*cam, T16 ? load_T<S>(T16) : M4<S>::identity());
  for (int i = 0; i < 16; i++) { KRt[i] = P.KRt.a[i]; iKRt[i] = P.iKRt.a[i]; }
}

void orc_projector_matrices(int mode, const orc_camera *cam, const double *T16, double *KRt16, double *iKRt16) {
  if (mode == ORC_F64) proj_mats<double>(cam, T16, KRt16, iKRt16);
  else proj_mats<float>(cam, T16, KRt16, iKRt16);
}

template <class S>
static void project_api(const orc_cloud *c, const orc_camera *cam, const double *T16, int32_t *index, double *depth) {
  Projector<S> P = make_projector<S>(*cam, T16 ? load_T<S>(T16) : M4<S>::identity());
  size_t NP = (size_t)P.rows * P.cols;
  std::vector<S> d(NP);
  project(*get<S>(c), P, index, d.data());
  if (depth)
    for (size_t i = 0; i < NP; i++) depth[i] = (double)d[i];
}

void orc_project(int mode, const orc_cloud *c, const orc_camera *cam, const double *T16, int32_t *index_out,
                 double *depth_out) {
  if (mode == ORC_F64) project_api<double>(c, cam, T16, index_out, depth_out);
  else project_api<float>(c, cam, T16, index_out, depth_out);
}

int orc_correspond(int mode, const orc_cloud *ref, const orc_cloud *cur, const int32_t *ri, const int32_t *ci,
                   int rows, int cols, const double *T16, const orc_align_params *prm, int32_t *pairs) {
  if (mode == ORC_F64)
    return correspond(*ref->d, *cur->d, ri, ci, rows, cols, load_T<double>(T16), *prm, pairs, true);
  return correspond(*ref->f, *cur->f, ri, ci, rows, cols, load_T<float>(T16), *prm, pairs, false);
}

void orc_linearize(int mode, const orc_cloud *ref, const orc_cloud *cur, const int32_t *pairs, int K,
                   const double *T16, const orc_align_params *prm, double *H36, double *b6, double *error,
                   int *inliers) {
  if (mode == ORC_F64)
    linearize(*ref->d, *cur->d, pairs, K, load_T<double>(T16), *prm, true, H36, b6, error, inliers);
  else
    linearize(*ref->f, *cur->f, pairs, K, load_T<float>(T16), *prm, false, H36, b6, error, inliers);
}

void orc_align(int mode, const orc_cloud *ref, const orc_cloud *cur, const orc_camera *cam, const double *guess,
               const double *roff, const double *coff, const orc_align_params *prm, int stats,
               orc_align_result *out) {
  if (mode == ORC_F64) align(*ref->d, *cur->d, *cam, guess, roff, coff, *prm, true, stats, out);
  else align(*ref->f, *cur->f, *cam, guess, roff, coff, *prm, false, stats, out);
}

int orc_correspond_nn(int mode, const orc_cloud *ref, const orc_cloud *cur, const double *T16, double normal_scaling,
                      const orc_align_params *prm, int32_t *pairs) {
  if (mode == ORC_F64) return correspond_nn(*ref->d, *cur->d, load_T<double>(T16), normal_scaling, *prm, pairs);
  return correspond_nn(*ref->f, *cur->f, load_T<float>(T16), (float)normal_scaling, *prm, pairs);
}

void orc_align_nn(int mode, const orc_cloud *ref, const orc_cloud *cur, const double *guess, double normal_scaling,
                  const orc_align_params *prm, int stats, orc_align_result *out) {
  if (mode == ORC_F64) align_nn(*ref->d, *cur->d, guess, normal_scaling, *prm, true, stats, out);
  else align_nn(*ref->f, *cur->f, guess, (float)normal_scaling, *prm, false, stats, out);
}

template <class S> static void eig_api(const double *A6, double *l3, double *U9) {
  S A[6], l[3], U[9];
  for (int i = 0; i < 6; i++) A[i] = S(A6[i]);
  eig3(A, l, U);
  for (int i = 0; i < 3; i++) l3[i] = l[i];
  for (int i = 0; i < 9; i++) U9[i] = U[i];
}
void orc_eig3(int mode, const double *A6, double *l3, double *U9) {
  if (mode == ORC_F64) eig_api<double>(A6, l3, U9);
  else eig_api<float>(A6, l3, U9);
}

template <class S> static void ldlt_api(const double *A36, const double *b6, double *x6) {
  S A[36], b[6], x[6];
  for (int i = 0; i < 36; i++) A[i] = S(A36[i]);
  for (int i = 0; i < 6; i++) b[i] = S(b6[i]);
  ldlt_solve(A, b, x);
  for (int i = 0; i < 6; i++) x6[i] = x[i];
}
void orc_ldlt_solve(int mode, const double *A36, const double *b6, double *x6) {
  if (mode == ORC_F64) ldlt_api<double>(A36, b6, x6);
  else ldlt_api<float>(A36, b6, x6);
}

template <class S> static void v2t_api(const double *x6, double *T16) {
  S x[6];
  for (int i = 0; i < 6; i++) x[i] = S(x6[i]);
  M4<S> T = v2t(x);
  for (int i = 0; i < 16; i++) T16[i] = T.a[i];
}
void orc_v2t(int mode, const double *x6, double *T16) {
  if (mode == ORC_F64) v2t_api<double>(x6, T16);
  else v2t_api<float>(x6, T16);
}

template <class S> static void t2v_api(const double *T16, double *x6) {
  S x[6];
  t2v(load_T<S>(T16), x);
  for (int i = 0; i < 6; i++) x6[i] = x[i];
}
void orc_t2v(int mode, const double *T16, double *x6) {
  if (mode == ORC_F64) t2v_api<double>(T16, x6);
  else t2v_api<float>(T16, x6);
}

template <class S> static void inv_api(const double *T16, double *o16) {
  M4<S> r = iso_inverse(load_T<S>(T16));
  for (int i = 0; i < 16; i++) o16[i] = r.a[i];
}
void orc_iso_inverse(int mode, const double *T16, double *o16) {
  if (mode == ORC_F64) inv_api<double>(T16, o16);
  else inv_api<float>(T16, o16);
}

template <class S>
static void region_api(const orc_cloud *c, const int32_t *index, int rows, int cols, int xmin, int xmax, int ymin,
                       int ymax, double *out10) {
  Integral<S> I;
  I.compute(index, rows, cols, get<S>(c)->points);
  S o[10];
  I.region(xmin, xmax, ymin, ymax, o);
  for (int k = 0; k < 10; k++) out10[k] = o[k];
}
void orc_integral_region(int mode, const orc_cloud *c, const int32_t *index, int rows, int cols, int xmin, int xmax,
                         int ymin, int ymax, double *out10) {
  if (mode == ORC_F64) region_api<double>(c, index, rows, cols, xmin, xmax, ymin, ymax, out10);
  else region_api<float>(c, index, rows, cols, xmin, xmax, ymin, ymax, out10);
}

