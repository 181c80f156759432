// cloud_io.cpp -- the reference's on-disk formats for clouds and trajectories.
//
//   .nicp cloud (Cloud::save / Cloud::load, cloud.cpp:13-150)
//     line 1: "NICPCLOUD <points / step> <binary 0|1>"
//     line 2: t2v(T) -- tx ty tz qx qy qz, space separated, trailing space
//     then per written point (every step-th point, i = 0, step, 2 step, ...):
//       text:   "POINTWITHSTATS x y z nx ny nz s00 s01 s02 s03 s10 ... s33 "
//               (the Stats 4x4 row by row)
//       binary: Point (4 floats, w = 1), Normal (4 floats, w = 0), then the
//               raw Stats object, 96 bytes: the 4x4 column-major (64), int n
//               (64), eigenvalues (68..79), bool curvatureComputed (80), float
//               curvature (84); bytes 81-83 and 88-95 are alignment padding
//               (the reference's Eigen-aligned layout), written as zeros.
//     Numbers in text are printed as an iostream prints a float (%g, 6
//     significant digits).  As in the reference, the header counts
//     points / step (integer division) while the loop writes every step-th
//     point; the reader reads the header's count.
//   trajectory line (nicp_simple_aligner.cpp:175-181): "timestamp tx ty tz qx
//     qy qz qw" with the normalised quaternion of the rotation (no sign fix).
//
// The Stats stored here (keep_stats) are the reference's content: for a
// pixel the stats calculator reached, [[U, mean], [0 0 0 1]], n, eigenvalues,
// curvature computed; otherwise the default Stats (identity, n = 0, zero
// eigenvalues, curvature 1 not computed), moved by any transform the cloud
// went through.  A cloud built without keep_stats is written with zeroed
// Stats, as the reference writes a cloud whose stats vector is empty.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "abi_guard.hpp"
#include "nicp_gpu.h"

namespace nicp {
namespace internal {
int cloud_host_arrays(nicp_cloud *c, std::vector<float> &pts4, std::vector<float> &nrm4, std::vector<float> &stats,
                      bool &has_stats);
int cloud_set_host_arrays(nicp_cloud *c, int n, const float *pts4, const float *nrm4, const float *omg12,
                          const float *stats, int normals, bool structured, const float omd[8]);
}  // namespace internal
}  // namespace nicp

namespace {

constexpr int kStatsWords = 16;  // eigenvalues 3, eigenvectors 9 (row-major), mean 3, n 1
constexpr size_t kStatsBytes = 96;

// Quaternion (x, y, z, w) of a rotation matrix by Shepperd's method (branch on
// the trace, else on the largest diagonal entry), then normalised.
void quat_of(const double R[3][3], double q[4]) {
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
  double nq = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (int a = 0; a < 4; a++) q[a] /= nq;
}

void rot_of(const float T16[16], double R[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) R[i][j] = T16[i * 4 + j];
}

// t2v (bm_se3.h:45-52): translation and the quaternion's vector part, w >= 0.
void t2v(const float T16[16], double x[6]) {
  double R[3][3], q[4];
  rot_of(T16, R);
  quat_of(R, q);
  if (q[3] < 0)
    for (int a = 0; a < 4; a++) q[a] = -q[a];
  x[0] = T16[3]; x[1] = T16[7]; x[2] = T16[11];
  x[3] = q[0]; x[4] = q[1]; x[5] = q[2];
}

// v2t (bm_se3.h:10-43): w = sqrt(1 - |q|^2).
void v2t(const double x[6], float T16[16]) {
  double qx = x[3], qy = x[4], qz = x[5];
  double qw = std::sqrt(std::max(0.0, 1.0 - (qx * qx + qy * qy + qz * qz)));
  double R[9] = {qw * qw + qx * qx - qy * qy - qz * qz, 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy),
                 2 * (qx * qy + qz * qw), qw * qw - qx * qx + qy * qy - qz * qz, 2 * (qy * qz - qx * qw),
                 2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), qw * qw - qx * qx - qy * qy + qz * qz};
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) T16[i * 4 + j] = (float)R[i * 3 + j];
    T16[i * 4 + 3] = (float)x[i];
  }
  T16[12] = T16[13] = T16[14] = 0.0f;
  T16[15] = 1.0f;
}

std::string g(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%g", v);
  return b;
}

// The Stats of point i as the reference holds it.
struct StatsRec {
  float M[16];  // row-major 4x4
  int n;
  float ev[3];
  bool computed;
  float curvature;
};

StatsRec stats_of(const float *rec, float curvature) {
  StatsRec s{};
  std::memset(s.M, 0, sizeof(s.M));
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) s.M[r * 4 + c] = rec[3 + r * 3 + c];
    s.M[r * 4 + 3] = rec[12 + r];
  }
  s.M[15] = 1.0f;
  s.n = (int)rec[15];
  for (int k = 0; k < 3; k++) s.ev[k] = rec[k];
  s.computed = s.n > 0;
  s.curvature = s.computed ? curvature : 1.0f;
  return s;
}

StatsRec zero_stats() {  // `Stats zero; zero.setZero();` (cloud.cpp:142-143)
  StatsRec s{};
  std::memset(s.M, 0, sizeof(s.M));
  s.n = 0;
  s.ev[0] = s.ev[1] = s.ev[2] = 0.0f;
  s.computed = false;
  s.curvature = 1.0f;
  return s;
}

void pack_stats(const StatsRec &s, unsigned char out[kStatsBytes]) {
  std::memset(out, 0, kStatsBytes);
  float colmajor[16];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) colmajor[c * 4 + r] = s.M[r * 4 + c];
  std::memcpy(out, colmajor, 64);
  std::memcpy(out + 64, &s.n, 4);
  std::memcpy(out + 68, s.ev, 12);
  out[80] = s.computed ? 1 : 0;
  std::memcpy(out + 84, &s.curvature, 4);
}

StatsRec unpack_stats(const unsigned char in[kStatsBytes]) {
  StatsRec s{};
  float colmajor[16];
  std::memcpy(colmajor, in, 64);
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) s.M[r * 4 + c] = colmajor[c * 4 + r];
  std::memcpy(&s.n, in + 64, 4);
  std::memcpy(s.ev, in + 68, 12);
  s.computed = in[80] != 0;
  std::memcpy(&s.curvature, in + 84, 4);
  return s;
}

// Stats::curvature (stats.h:93-98): the cached value, or the formula with
// its float sum and double promotion.
float curvature_of(const StatsRec &s) {
  if (s.computed) return s.curvature;
  float sum = s.ev[0] + s.ev[1];
  sum = sum + s.ev[2];
  return (float)((double)s.ev[0] / ((double)sum + 1e-9));
}

}  // namespace

extern "C" int nicp_cloud_save(nicp_cloud *cloud, const char *filename, const float T16[16], int step, int binary) {
  NICP_ABI_TRY
  if (!cloud || !filename || step < 1) return NICP_EINVAL;
  std::vector<float> pts, nrm, st;
  bool has_stats = false;
  int rc = nicp::internal::cloud_host_arrays(cloud, pts, nrm, st, has_stats);
  if (rc) return rc;
  const size_t n = pts.size() / 4;
  std::ofstream os(filename, std::ios::binary);
  if (!os) return NICP_EINVAL;
  float I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  double x[6];
  t2v(T16 ? T16 : I, x);
  os << "NICPCLOUD " << n / step << " " << (binary ? 1 : 0) << "\n";
  for (int k = 0; k < 6; k++) os << g((float)x[k]) << " ";
  os << "\n";
  for (size_t i = 0; i < n; i += step) {
    const float *p = &pts[4 * i], *q = &nrm[4 * i];
    StatsRec s = has_stats ? stats_of(&st[kStatsWords * i], q[3]) : zero_stats();
    if (!binary) {
      os << "POINTWITHSTATS ";
      for (int k = 0; k < 3; k++) os << g(p[k]) << " ";
      for (int k = 0; k < 3; k++) os << g(q[k]) << " ";
      for (int k = 0; k < 16; k++) os << g(s.M[k]) << " ";
      os << "\n";
    } else {
      float P[4] = {p[0], p[1], p[2], 1.0f}, N[4] = {q[0], q[1], q[2], 0.0f};
      unsigned char raw[kStatsBytes];
      pack_stats(s, raw);
      os.write((const char *)P, 16);
      os.write((const char *)N, 16);
      os.write((const char *)raw, kStatsBytes);
    }
  }
  return os.good() ? NICP_OK : NICP_EINVAL;
  NICP_ABI_CATCH
}

extern "C" int nicp_cloud_load(nicp_cloud *cloud, const char *filename, const nicp_cloud_params *prm,
                               float T16_out[16], int *num_points) {
  NICP_ABI_TRY
  if (!cloud || !filename) return NICP_EINVAL;
  std::ifstream is(filename, std::ios::binary);
  if (!is) return NICP_EINVAL;
  std::string line;
  std::getline(is, line);
  std::istringstream hs(line);
  std::string tag;
  long long count = 0;
  int binary = 0;
  hs >> tag >> count >> binary;
  if (tag != "NICPCLOUD" || !hs || count < 0 || count > (1ll << 30)) return NICP_EINVAL;
  std::getline(is, line);
  std::istringstream ts(line);
  double x[6] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 6; k++) ts >> x[k];
  if (T16_out) v2t(x, T16_out);
  nicp_cloud_params def;
  nicp_default_cloud_params(&def);
  const nicp_cloud_params &P = prm ? *prm : def;
  const size_t n = (size_t)count;
  // The arrays grow with the records actually read: the header's count
  // bounds the loop but does not size an allocation (a damaged or hostile
  // header could claim 2^30 points).
  std::vector<float> pts, nrm, omg, st;
  try {
    const size_t r = std::min<size_t>(n, (size_t)1 << 16);
    pts.reserve(4 * r);
    nrm.reserve(4 * r);
    omg.reserve(12 * r);
    st.reserve(kStatsWords * r);
  } catch (const std::bad_alloc &) {
    return NICP_ENOMEM;
  }
  int normals = 0;
  size_t k = 0;
  while (k < n && is.good()) {
    float p[4] = {0, 0, 0, 1}, q[4] = {0, 0, 0, 0};
    StatsRec s;
    if (!binary) {
      if (!std::getline(is, line)) break;
      std::istringstream ls(line);
      std::string w;
      ls >> w;
      if (w != "POINTWITHSTATS") continue;
      for (int a = 0; a < 3; a++) ls >> p[a];
      for (int a = 0; a < 3; a++) ls >> q[a];
      s = zero_stats();
      for (int a = 0; a < 16; a++) ls >> s.M[a];
    } else {
      unsigned char raw[kStatsBytes];
      is.read((char *)p, 16);
      is.read((char *)q, 16);
      is.read((char *)raw, kStatsBytes);
      if (!is) break;
      s = unpack_stats(raw);
    }
    try {
      pts.resize(4 * (k + 1));
      nrm.resize(4 * (k + 1));
      omg.resize(12 * (k + 1));
      st.resize(kStatsWords * (k + 1));
    } catch (const std::bad_alloc &) {
      return NICP_ENOMEM;
    }
    // the device record: eigenvalues, eigenvectors, mean, n
    float *rec = &st[kStatsWords * k];
    for (int a = 0; a < 3; a++) rec[a] = s.ev[a];
    for (int r = 0; r < 3; r++) {
      for (int c = 0; c < 3; c++) rec[3 + r * 3 + c] = s.M[r * 4 + c];
      rec[12 + r] = s.M[r * 4 + 3];
    }
    rec[15] = (float)s.n;
    const float kappa = curvature_of(s);
    const bool has = q[0] != 0.0f || q[1] != 0.0f || q[2] != 0.0f;
    // Point/NormalInformationMatrixCalculator::compute (informationmatrixcalculator.cpp:9-57)
    float om[12] = {0};
    int cls = 0;
    if (has) {
      const bool pflat = kappa < P.pim_curvature_threshold, nflat = kappa < P.nim_curvature_threshold;
      cls = (pflat ? 0 : 1) + (nflat ? 0 : 2);
      const float *Dp = pflat ? P.pim_flat : P.pim_nonflat, *Dn = nflat ? P.nim_flat : P.nim_nonflat;
      const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
      for (int e = 0; e < 6; e++) {
        // U D U^T: ((U_i0 D0) U_j0 + (U_i1 D1) U_j1) + (U_i2 D2) U_j2
        float sp = 0.0f, sn = 0.0f;
        for (int c = 0; c < 3; c++) {
          sp = sp + (s.M[ii[e] * 4 + c] * Dp[c]) * s.M[jj[e] * 4 + c];
          sn = sn + (s.M[ii[e] * 4 + c] * Dn[c]) * s.M[jj[e] * 4 + c];
        }
        om[e] = sp;
        om[6 + e] = sn;
      }
      normals++;
    }
    pts[4 * k] = p[0]; pts[4 * k + 1] = p[1]; pts[4 * k + 2] = p[2];
    pts[4 * k + 3] = has ? 1.0f + (float)cls : 0.5f;
    nrm[4 * k] = q[0]; nrm[4 * k + 1] = q[1]; nrm[4 * k + 2] = q[2]; nrm[4 * k + 3] = kappa;
    std::memcpy(&omg[12 * k], om, sizeof(om));
    k++;
  }
  const bool structured = P.pim_flat[1] == P.pim_flat[2] && P.pim_nonflat[1] == P.pim_nonflat[2] &&
                          P.nim_flat[1] == P.nim_flat[2] && P.nim_nonflat[1] == P.nim_nonflat[2];
  const float omd[8] = {P.pim_flat[0], P.pim_flat[1], P.pim_nonflat[0], P.pim_nonflat[1],
                        P.nim_flat[0], P.nim_flat[1], P.nim_nonflat[0], P.nim_nonflat[1]};
  int rc = nicp::internal::cloud_set_host_arrays(cloud, (int)k, pts.data(), nrm.data(), omg.data(), st.data(),
                                                 normals, structured, omd);
  if (rc) return rc;
  if (num_points) *num_points = (int)k;
  return k == n ? NICP_OK : NICP_EINVAL;
  NICP_ABI_CATCH
}

extern "C" int nicp_trajectory_line(const char *timestamp, const float T16[16], char *out, size_t capacity) {
  NICP_ABI_TRY
  if (!timestamp || !T16 || !out) return NICP_EINVAL;
  double R[3][3], q[4];
  rot_of(T16, R);
  quat_of(R, q);
  float qf[4];
  for (int a = 0; a < 4; a++) qf[a] = (float)q[a];
  std::string s = std::string(timestamp) + " " + g(T16[3]) + " " + g(T16[7]) + " " + g(T16[11]) + " " + g(qf[0]) +
                  " " + g(qf[1]) + " " + g(qf[2]) + " " + g(qf[3]) + "\n";
  if (s.size() + 1 > capacity) return NICP_EINVAL;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return NICP_OK;
  NICP_ABI_CATCH
}
