// k_nn.cu -- nearest-neighbour data association (CorrespondenceFinderNN,
// correspondencefindernn.cpp:44-97) on the device.
//
// The reference asks FLANN's randomized kd-tree (approximate, 16 checks) for
// the nearest current point within the squared radius in the 6-D space
// (p, s n).  Here the search is exact: the current cloud is bucketed in a
// uniform grid over xyz (cell h), sorted by cell; a query scans Chebyshev
// shells of cells around its own cell and stops once the shell's lower
// bound on the xyz distance -- a lower bound of the 6-D distance -- exceeds
// the best squared distance found (or the radius).  Ties keep the lowest
// current index, as the oracle's exhaustive scan does.
//
//   k_nn_keys      per current point: cell id, 6-D feature
//   (CUB radix sort of (cell id, point index))
//   k_nn_ranges    first / one-past-last sorted position of every cell
//   k_nn_gather    features in sorted order (a cell's points contiguous)
//   k_nn_query     per reference point: transform, shell search, the
//                  reference's gates; match[i] = current index or -1
//   k_nn_flag / k_nn_write  ordered compaction into (ref, cur) pairs
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.hpp"

namespace nicp {

__device__ __forceinline__ int cell_coord(float v, float origin, float inv_h) {
  return (int)floorf((v - origin) * inv_h);
}

__global__ void k_nn_keys(const float4 *__restrict__ pts, const float4 *__restrict__ nrm, int n, float nscale,
                          NNGrid g, unsigned *__restrict__ keys, unsigned *__restrict__ idx,
                          float *__restrict__ feat6) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  float4 p = pts[j], q = nrm[j];
  int cx = min(max(cell_coord(p.x, g.origin[0], g.inv_h), 0), g.dim[0] - 1);
  int cy = min(max(cell_coord(p.y, g.origin[1], g.inv_h), 0), g.dim[1] - 1);
  int cz = min(max(cell_coord(p.z, g.origin[2], g.inv_h), 0), g.dim[2] - 1);
  keys[j] = (unsigned)((cz * g.dim[1] + cy) * g.dim[0] + cx);
  idx[j] = (unsigned)j;
  float *f = feat6 + 6 * (size_t)j;
  f[0] = p.x; f[1] = p.y; f[2] = p.z;
  // _model2linear: the normal scaled by nscale (correspondencefindernn.cpp:13-27)
  f[3] = fm(nscale, q.x); f[4] = fm(nscale, q.y); f[5] = fm(nscale, q.z);
}

__global__ void k_nn_ranges(const unsigned *__restrict__ skeys, int n, int *__restrict__ cstart,
                            int *__restrict__ cend) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned c = skeys[k];
  if (k == 0 || skeys[k - 1] != c) cstart[c] = k;
  if (k == n - 1 || skeys[k + 1] != c) cend[c] = k + 1;
}

__global__ void k_nn_gather(const unsigned *__restrict__ sidx, int n, const float *__restrict__ feat6,
                            float *__restrict__ sfeat6) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float *a = feat6 + 6 * (size_t)sidx[k];
  float *b = sfeat6 + 6 * (size_t)k;
#pragma unroll
  for (int t = 0; t < 6; t++) b[t] = a[t];
}

// One reference point per thread.  Tg: rows 0..2 of the transform applied to
// the reference (the aligner's _T.inverse()).
__global__ void k_nn_query(NNQuery a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nr) return;
  a.match[i] = -1;
  float Tg[12];
#pragma unroll
  for (int k = 0; k < 12; k++) Tg[k] = a.Tg ? a.Tg[k] : a.state->Tgate[k];
  const float4 p0 = a.ref_pts[i], n0 = a.ref_nrm[i];
  const float3 p = xform_point(Tg, p0);
  // sR = T.linear() * nscale, then sR * n
  float sR[12];
#pragma unroll
  for (int r = 0; r < 3; r++) {
#pragma unroll
    for (int c = 0; c < 3; c++) sR[r * 4 + c] = fm(Tg[r * 4 + c], a.nscale);
    sR[r * 4 + 3] = 0.0f;
  }
  const float3 sn = xform_normal(sR, n0);
  const float q[6] = {p.x, p.y, p.z, sn.x, sn.y, sn.z};
  const NNGrid &g = a.grid;
  const int qx = cell_coord(p.x, g.origin[0], g.inv_h), qy = cell_coord(p.y, g.origin[1], g.inv_h),
            qz = cell_coord(p.z, g.origin[2], g.inv_h);
  // shells beyond the grid hold no cells
  int kcover = 0;
  kcover = max(kcover, max(qx, g.dim[0] - 1 - qx));
  kcover = max(kcover, max(qy, g.dim[1] - 1 - qy));
  kcover = max(kcover, max(qz, g.dim[2] - 1 - qz));
  const int kmax = min(g.max_shell, kcover);
  int best = -1;
  float bd = 0.0f;
  for (int k = 0; k <= kmax; k++) {
    // every point of shell k is at least (k - 1) h away in xyz
    if (k >= 2) {
      const float lb = (float)(k - 1) * g.h;
      const float lb2 = lb * lb;
      if (lb2 > a.sq * 1.0001f) break;
      if (best >= 0 && lb2 > bd * 1.0001f) break;
    }
    for (int dz = -k; dz <= k; dz++) {
      const int cz = qz + dz;
      if (cz < 0 || cz >= g.dim[2]) continue;
      for (int dy = -k; dy <= k; dy++) {
        const int cy = qy + dy;
        if (cy < 0 || cy >= g.dim[1]) continue;
        const bool face = (dz == -k || dz == k || dy == -k || dy == k);
        for (int dx = -k; dx <= k; dx += (face ? 1 : 2 * k)) {
          const int cx = qx + dx;
          if (cx >= 0 && cx < g.dim[0]) {
            const int cell = (cz * g.dim[1] + cy) * g.dim[0] + cx;
            const int s0 = a.cstart[cell], s1 = a.cend[cell];
            for (int s = s0; s < s1; s++) {
              const float *c = a.sfeat6 + 6 * (size_t)s;
              float d = 0.0f;
#pragma unroll
              for (int t = 0; t < 6; t++) {
                const float e = fsb(q[t], c[t]);
                d = fa(d, fm(e, e));
              }
              if (d < a.sq) {
                const int j = (int)a.sidx[s];
                if (best < 0 || d < bd || (d == bd && j < best)) {
                  best = j;
                  bd = d;
                }
              }
            }
          }
          if (k == 0) break;
        }
      }
    }
  }
  if (best < 0) return;
  // the gates (correspondencefindernn.cpp:80-93)
  const float3 rn = xform_normal(Tg, n0);
  const float4 cn = a.cur_nrm[best], cp = a.cur_pts[best];
  const float rn2 = dot3x(rn.x, rn.y, rn.z, rn.x, rn.y, rn.z), cn2 = dot3x(cn.x, cn.y, cn.z, cn.x, cn.y, cn.z);
  if (!a.demoted && (rn2 == 0.0f || cn2 == 0.0f)) return;
  const float dx = fsb(p.x, cp.x), dy = fsb(p.y, cp.y), dz = fsb(p.z, cp.z);
  if (dot3x(dx, dy, dz, dx, dy, dz) > a.sq) return;
  if (isnan(cn.x) || isnan(cn.y) || isnan(cn.z) || isnan(rn.x) || isnan(rn.y) || isnan(rn.z)) return;
  if (!a.demoted && dot3x(rn.x, rn.y, rn.z, cn.x, cn.y, cn.z) < a.cos_thr) return;
  a.match[i] = best;
}

__global__ void k_nn_flag(const int *__restrict__ match, int n, int *__restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = match[i] >= 0 ? 1 : 0;
}

__global__ void k_nn_write(const int *__restrict__ match, const int *__restrict__ pos, int n,
                           int32_t *__restrict__ pairs, int *__restrict__ num_pairs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = match[i];
  if (m >= 0) {
    pairs[2 * (size_t)pos[i]] = i;
    pairs[2 * (size_t)pos[i] + 1] = m;
  }
  if (i == n - 1) *num_pairs = pos[i] + (m >= 0 ? 1 : 0);
}

size_t nn_temp_bytes(int n) {
  size_t a = 0, b = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, a, (const unsigned *)nullptr, (unsigned *)nullptr,
                                  (const unsigned *)nullptr, (unsigned *)nullptr, n);
  cub::DeviceScan::ExclusiveSum(nullptr, b, (const int *)nullptr, (int *)nullptr, n);
  return a > b ? a : b;
}

int launch_nn_build(const NNBuild &b, cudaStream_t s) {
  const int n = b.nc;
  if (n <= 0) return 0;
  const int B = 256, G = (n + B - 1) / B;
  k_nn_keys<<<G, B, 0, s>>>(b.cur_pts, b.cur_nrm, n, b.nscale, b.grid, b.keys, b.idx, b.feat6);
  size_t tb = b.temp_bytes;
  if (cub::DeviceRadixSort::SortPairs(b.temp, tb, b.keys, b.skeys, b.idx, b.sidx, n, 0, b.key_bits, s) !=
      cudaSuccess)
    return 1;
  const size_t ncells = (size_t)b.grid.dim[0] * b.grid.dim[1] * b.grid.dim[2];
  cudaMemsetAsync(b.cstart, 0, 4 * ncells, s);
  cudaMemsetAsync(b.cend, 0, 4 * ncells, s);
  k_nn_ranges<<<G, B, 0, s>>>(b.skeys, n, b.cstart, b.cend);
  k_nn_gather<<<G, B, 0, s>>>(b.sidx, n, b.feat6, b.sfeat6);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int launch_nn_correspond(const NNQuery &q, int *flag, int *pos, void *temp, size_t temp_bytes, int32_t *pairs,
                         int *num_pairs, cudaStream_t s) {
  const int n = q.nr;
  if (n <= 0) {
    cudaMemsetAsync(num_pairs, 0, sizeof(int), s);
    return 0;
  }
  const int B = 128, G = (n + B - 1) / B;
  k_nn_query<<<G, B, 0, s>>>(q);
  k_nn_flag<<<(n + 255) / 256, 256, 0, s>>>(q.match, n, flag);
  size_t tb = temp_bytes;
  if (cub::DeviceScan::ExclusiveSum(temp, tb, flag, pos, n, s) != cudaSuccess) return 1;
  k_nn_write<<<(n + 255) / 256, 256, 0, s>>>(q.match, pos, n, pairs, num_pairs);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace nicp
