// k_merge.cu -- Merger::merge (merger.cpp:15-109) on the device.
//
//   k_merge_classify   per point: project with the merger's transform (the
//                      same exact-order projection as k_zbuffer), compare
//                      with the pixel's z-buffer winner: "self" (the point
//                      won its own pixel), "fused into the winner" (depth
//                      within the threshold) or untouched; counts the
//                      contributions per winner
//   k_merge_scatter    lists every winner's contributors (unordered)
//   k_merge_fuse       per winner: sorts its contributors by index and adds
//                      their information in that order (the reference's
//                      serial loop order), then returns to moments
//                      (Gaussian3f::addInformation / _updateMoments)
//   k_merge_compact    keeps untouched and self points in index order; a
//                      self point takes its Gaussian's mean as position
//
// All floating-point steps are single-rounded in the order written (no FMA
// contraction), like the oracle's REF32 restatement.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.hpp"

namespace nicp {

// Gaussian3f of point i: (mean, 9 covariance entries), see write_gaussian.
__device__ __forceinline__ void load_gaussian(const float4 *g, float m[3], float C[9]) {
  float4 a = g[0], b = g[1], c = g[2];
  m[0] = a.x; m[1] = a.y; m[2] = a.z;
  C[0] = a.w; C[1] = b.x; C[2] = b.y; C[3] = b.z; C[4] = b.w; C[5] = c.x; C[6] = c.y; C[7] = c.z; C[8] = c.w;
}

// 3x3 inverse by cofactors times the reciprocal determinant.
__device__ __forceinline__ void inv3_rn(const float m[9], float out[9]) {
  float c00 = fsb(fm(m[4], m[8]), fm(m[5], m[7]));
  float c01 = fsb(fm(m[5], m[6]), fm(m[3], m[8]));
  float c02 = fsb(fm(m[3], m[7]), fm(m[4], m[6]));
  float det = fm(m[0], c00);
  det = fa(det, fm(m[1], c01));
  det = fa(det, fm(m[2], c02));
  float id = __frcp_rn(det);
  out[0] = fm(c00, id);
  out[3] = fm(c01, id);
  out[6] = fm(c02, id);
  out[1] = fm(fsb(fm(m[2], m[7]), fm(m[1], m[8])), id);
  out[4] = fm(fsb(fm(m[0], m[8]), fm(m[2], m[6])), id);
  out[7] = fm(fsb(fm(m[1], m[6]), fm(m[0], m[7])), id);
  out[2] = fm(fsb(fm(m[1], m[5]), fm(m[2], m[4])), id);
  out[5] = fm(fsb(fm(m[2], m[3]), fm(m[0], m[5])), id);
  out[8] = fm(fsb(fm(m[0], m[4]), fm(m[1], m[3])), id);
}

__device__ __forceinline__ void mat3_vec(const float A[9], const float v[3], float out[3]) {
#pragma unroll
  for (int a = 0; a < 3; a++) out[a] = fa(fa(fm(A[a * 3 + 0], v[0]), fm(A[a * 3 + 1], v[1])), fm(A[a * 3 + 2], v[2]));
}

// Information form (Gaussian::_updateInfo): Om = C^-1, eta = Om mean.
__device__ __forceinline__ void gaussian_info(const float4 *g, float Om[9], float eta[3]) {
  float m[3], C[9];
  load_gaussian(g, m, C);
  inv3_rn(C, Om);
  mat3_vec(Om, m, eta);
}

// tgt[i]: i (self), the winner it fuses into, or -1 (untouched).
__global__ void k_merge_classify(const float4 *__restrict__ pts, const int *__restrict__ count,
                                 const float *__restrict__ KRt12, int rows, int cols, float min_d, float max_d,
                                 float max_depth, float dthr, const int32_t *__restrict__ index,
                                 const float *__restrict__ depth, int *__restrict__ tgt, int *__restrict__ cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *count) return;
  tgt[i] = -1;
  float K[12];
#pragma unroll
  for (int k = 0; k < 12; k++) K[k] = KRt12[k];
  int x, y;
  float d;
  if (!project_pixel(K, pts[i], rows, cols, min_d, max_d, x, y, d)) return;
  if (d < 0.0f || d > max_depth) return;
  const size_t pix = (size_t)y * cols + x;
  const int target = index[pix];
  if (target < 0) return;
  if (target == i) {
    tgt[i] = i;
  } else if (fabsf(fsb(d, depth[pix])) < dthr) {
    tgt[i] = target;
    atomicAdd(cnt + target, 1);
  }
}

__global__ void k_merge_scatter(const int *__restrict__ tgt, const int *__restrict__ count,
                                const int *__restrict__ off, int *__restrict__ fill, int *__restrict__ list) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *count) return;
  int t = tgt[i];
  if (t < 0 || t == i) return;
  list[off[t] + atomicAdd(fill + t, 1)] = i;
}

// One thread per winner with contributors.  The contributor list is sorted
// by index (insertion sort: lists hold the points that landed on one pixel),
// so the float sums follow the reference's loop order exactly.
__global__ void k_merge_fuse(const int *__restrict__ count, const int *__restrict__ cnt, const int *__restrict__ off,
                             int *__restrict__ list, float4 *__restrict__ gauss) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *count) return;
  const int m = cnt[t];
  if (m == 0) return;
  int *L = list + off[t];
  for (int a = 1; a < m; a++) {
    int v = L[a], b = a - 1;
    while (b >= 0 && L[b] > v) {
      L[b + 1] = L[b];
      b--;
    }
    L[b + 1] = v;
  }
  float Om[9], eta[3];
  gaussian_info(gauss + 3 * (size_t)t, Om, eta);
  for (int a = 0; a < m; a++) {
    float Oi[9], ei[3];
    gaussian_info(gauss + 3 * (size_t)L[a], Oi, ei);
#pragma unroll
    for (int k = 0; k < 9; k++) Om[k] = fa(Om[k], Oi[k]);
#pragma unroll
    for (int k = 0; k < 3; k++) eta[k] = fa(eta[k], ei[k]);
  }
  // Gaussian::_updateMoments: C = Om^-1, mean = C eta
  float C[9], mn[3];
  inv3_rn(Om, C);
  mat3_vec(C, eta, mn);
  float4 *g = gauss + 3 * (size_t)t;
  g[0] = make_float4(mn[0], mn[1], mn[2], C[0]);
  g[1] = make_float4(C[1], C[2], C[3], C[4]);
  g[2] = make_float4(C[5], C[6], C[7], C[8]);
}

__global__ void k_merge_keep(const int *__restrict__ tgt, const int *__restrict__ count, int *__restrict__ keep) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *count) return;
  int t = tgt[i];
  keep[i] = (t < 0 || t == i) ? 1 : 0;
}

// Survivors to their compacted positions in the staging arrays; new counts
// (points, points with a normal) in out_count.
__global__ void k_merge_compact(const int *__restrict__ tgt, const int *__restrict__ count,
                                const int *__restrict__ pos, const float4 *__restrict__ pts,
                                const float4 *__restrict__ nrm, const float4 *__restrict__ omg,
                                const float *__restrict__ eig, const float4 *__restrict__ gauss, float4 *o_pts,
                                float4 *o_nrm, float4 *o_omg, float *o_eig, float4 *o_gauss, int *out_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *count;
  bool has = false;
  if (i < n) {
    const int t = tgt[i];
    if (t < 0 || t == i) {
      const int j = pos[i];
      float4 p = pts[i];
      if (t == i) {  // merger.cpp:77-79: a self point takes its Gaussian's mean
        float4 g0 = gauss[3 * (size_t)i];
        p.x = g0.x; p.y = g0.y; p.z = g0.z;
      }
      o_pts[j] = p;
      float4 nn = nrm[i];
      o_nrm[j] = nn;
      has = point_has_normal(p.w);
#pragma unroll
      for (int k = 0; k < 3; k++) o_omg[3 * (size_t)j + k] = omg[3 * (size_t)i + k];
      if (eig)
        for (int k = 0; k < kStatsWords; k++) o_eig[kStatsWords * (size_t)j + k] = eig[kStatsWords * (size_t)i + k];
      if (gauss)
#pragma unroll
        for (int k = 0; k < 3; k++) o_gauss[3 * (size_t)j + k] = gauss[3 * (size_t)i + k];
      if (i == n - 1) out_count[0] = j + 1;
    } else if (i == n - 1) {
      out_count[0] = pos[i];
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(out_count + 1, __popc(m));
}

size_t merge_scan_temp_bytes(int n) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const int *)nullptr, (int *)nullptr, n);
  return bytes;
}

int launch_merge(const MergeArgs &a, cudaStream_t s) {
  const int n = a.n;
  if (n <= 0) return 0;
  const int B = 256, G = (n + B - 1) / B;
  cudaMemsetAsync(a.cnt, 0, sizeof(int) * (size_t)n, s);
  cudaMemsetAsync(a.fill, 0, sizeof(int) * (size_t)n, s);
  cudaMemsetAsync(a.out_count, 0, 2 * sizeof(int), s);
  k_merge_classify<<<G, B, 0, s>>>(a.pts, a.count, a.KRt12, a.rows, a.cols, a.min_d, a.max_d, a.max_depth, a.dthr,
                                   a.index, a.depth, a.tgt, a.cnt);
  size_t tb = a.scan_temp_bytes;
  if (cub::DeviceScan::ExclusiveSum(a.scan_temp, tb, a.cnt, a.off, n, s) != cudaSuccess) return 1;
  k_merge_scatter<<<G, B, 0, s>>>(a.tgt, a.count, a.off, a.fill, a.list);
  k_merge_fuse<<<G, B, 0, s>>>(a.count, a.cnt, a.off, a.list, a.gauss);
  k_merge_keep<<<G, B, 0, s>>>(a.tgt, a.count, a.keep);
  tb = a.scan_temp_bytes;
  if (cub::DeviceScan::ExclusiveSum(a.scan_temp, tb, a.keep, a.pos, n, s) != cudaSuccess) return 1;
  k_merge_compact<<<G, B, 0, s>>>(a.tgt, a.count, a.pos, a.pts, a.nrm, a.omg, a.eig, a.gauss, a.o_pts, a.o_nrm,
                                  a.o_omg, a.o_eig, a.o_gauss, a.out_count);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace nicp
