// stats_host.cpp -- Aligner::_computeStatistics (aligner.cpp:82-135, unscented.h:23-65)
// in FP64 on the host, from the 6x6 system of one extra linearization at the
// final pose.  Steps: pseudo-inverse of H through a symmetric (Jacobi)
// eigendecomposition (singular values below 6 * FLT_EPSILON * max are
// dropped), unscented sampling (alpha 1e-3, beta 2, 13 sigma points through a
// Cholesky factor of Sigma * (6 + lambda)), each sample remapped through
// t2v(T * v2t(s)^-1), Gaussian reconstruction, inverse, symmetrisation, and
// the max/min singular-value ratio of the translational and rotational 3x3
// blocks.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>

namespace nicp {

namespace {

void jacobi_sym(int n, double *A, double *V, double *w) {
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

bool inverse6(const double *A, double *out) {
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

void v2t(const double *x, double *T) {
  double qx = x[3], qy = x[4], qz = x[5];
  double qw = std::sqrt(std::max(0.0, 1.0 - (qx * qx + qy * qy + qz * qz)));
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

void t2v(const double *T, double *x) {
  double R[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[i][j] = T[i * 4 + j];
  double q[4];  // x y z w
  double tr = R[0][0] + R[1][1] + R[2][2];
  if (tr > 0) {
    double s = std::sqrt(tr + 1.0);
    q[3] = 0.5 * s;
    s = 0.5 / s;
    q[0] = (R[2][1] - R[1][2]) * s;
    q[1] = (R[0][2] - R[2][0]) * s;
    q[2] = (R[1][0] - R[0][1]) * s;
  } else {
    int i = 0;
    if (R[1][1] > R[0][0]) i = 1;
    if (R[2][2] > R[i][i]) i = 2;
    int j = (i + 1) % 3, k = (j + 1) % 3;
    double s = std::sqrt(R[i][i] - R[j][j] - R[k][k] + 1.0);
    q[i] = 0.5 * s;
    s = 0.5 / s;
    q[3] = (R[k][j] - R[j][k]) * s;
    q[j] = (R[j][i] + R[i][j]) * s;
    q[k] = (R[k][i] + R[i][k]) * s;
  }
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (double &v : q) v /= n;
  if (q[3] < 0) { q[0] = -q[0]; q[1] = -q[1]; q[2] = -q[2]; }
  x[0] = T[3]; x[1] = T[7]; x[2] = T[11];
  x[3] = q[0]; x[4] = q[1]; x[5] = q[2];
}

void mm4(const double *A, const double *B, double *C) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double s = 0;
      for (int k = 0; k < 4; k++) s += A[i * 4 + k] * B[k * 4 + j];
      C[i * 4 + j] = s;
    }
}

void iso_inverse(const double *T, double *R) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[i * 4 + j] = T[j * 4 + i];
  for (int i = 0; i < 3; i++) R[i * 4 + 3] = -(R[i * 4 + 0] * T[3] + R[i * 4 + 1] * T[7] + R[i * 4 + 2] * T[11]);
  R[12] = 0; R[13] = 0; R[14] = 0; R[15] = 1;
}

double block_ratio(const double *A6x6, int o) {
  double B[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) B[i * 3 + j] = A6x6[(o + i) * 6 + o + j];
  double V[9], w[3];
  jacobi_sym(3, B, V, w);
  double smax = 0, smin = std::numeric_limits<double>::max();
  for (double x : w) { smax = std::max(smax, std::fabs(x)); smin = std::min(smin, std::fabs(x)); }
  return smax / smin;
}

}  // namespace

void solution_statistics(const double H36[36], const double T16[16], double *tr, double *rr, double omega36[36],
                         double mean6[6]) {
  *tr = std::numeric_limits<double>::max();
  *rr = std::numeric_limits<double>::max();
  for (int i = 0; i < 36; i++) omega36[i] = 0;
  for (int i = 0; i < 6; i++) mean6[i] = 0;
  double A[36], V[36], w[6];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) A[i * 6 + j] = 0.5 * (H36[i * 6 + j] + H36[j * 6 + i]);
  jacobi_sym(6, A, V, w);
  double smax = 0;
  for (double x : w) smax = std::max(smax, std::fabs(x));
  double thr = smax * 6 * (double)FLT_EPSILON;
  double Sig[36] = {0};
  for (int k = 0; k < 6; k++) {
    if (!(std::fabs(w[k]) > thr)) continue;
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) Sig[i * 6 + j] += V[i * 6 + k] * V[j * 6 + k] / w[k];
  }
  const int dim = 6, np = 2 * dim + 1;
  const double alpha = 1e-3, beta = 2.0, lambda = alpha * alpha * dim;
  const double wi = 1.0 / (2.0 * (dim + lambda));
  double L[36] = {0};
  for (int j = 0; j < 6; j++) {
    double s = Sig[j * 6 + j] * (dim + lambda);
    for (int k = 0; k < j; k++) s -= L[j * 6 + k] * L[j * 6 + k];
    if (!(s > 0)) return;
    L[j * 6 + j] = std::sqrt(s);
    for (int i = j + 1; i < 6; i++) {
      double t = Sig[i * 6 + j] * (dim + lambda);
      for (int k = 0; k < j; k++) t -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = t / L[j * 6 + j];
    }
  }
  double samp[np][6], wm[np], wc[np];
  for (int k = 0; k < 6; k++) samp[0][k] = 0;
  wm[0] = lambda / (dim + lambda);
  wc[0] = lambda / (dim + lambda) + (1.0 - alpha * alpha + beta);
  for (int i = 0; i < 6; i++)
    for (int s = 0; s < 2; s++) {
      int k = 1 + 2 * i + s;
      for (int r = 0; r < 6; r++) samp[k][r] = (s ? -1.0 : 1.0) * L[r * 6 + i];
      wm[k] = wc[k] = wi;
    }
  for (int k = 0; k < np; k++) {
    double X[16], Xi[16], Y[16];
    v2t(samp[k], X);
    iso_inverse(X, Xi);
    mm4(T16, Xi, Y);
    t2v(Y, samp[k]);
  }
  double mean[6] = {0}, cov[36] = {0};
  for (int k = 0; k < np; k++)
    for (int r = 0; r < 6; r++) mean[r] += wm[k] * samp[k][r];
  for (int k = 0; k < np; k++)
    for (int r = 0; r < 6; r++)
      for (int c = 0; c < 6; c++) cov[r * 6 + c] += wc[k] * (samp[k][r] - mean[r]) * (samp[k][c] - mean[c]);
  for (int i = 0; i < 6; i++) mean6[i] = mean[i];
  double Om[36];
  if (!inverse6(cov, Om)) return;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) A[i * 6 + j] = 0.5 * (Om[i * 6 + j] + Om[j * 6 + i]);
  for (int i = 0; i < 36; i++) omega36[i] = A[i];
  *tr = block_ratio(A, 0);
  *rr = block_ratio(A, 3);
}

}  // namespace nicp
