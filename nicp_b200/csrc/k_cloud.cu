// k_cloud.cu -- depth image -> cloud kernels (DepthImageConverterIntegralImage::compute).
//
//   k_unproject_count / k_unproject_write
//       u16 (or f32) depth -> index image + points, with the reference's
//       row-major point numbering (pinholepointprojector.cpp:93-134).  Each
//       CTA owns a 4096-pixel tile; 16 pixels per thread are read with two
//       128-bit loads.  The first pass counts valid pixels per tile, the second
//       re-reads the tile (from L2), sums the counts of the preceding tiles of
//       its frame and writes indices and points at their final positions.
//   k_moments_band_totals / k_moments_band_carry / k_moments_band_sweep
//       integral image of the 10 unique point moments (n, Sx, Sy, Sz, Sxx,
//       Sxy, Sxz, Syy, Syz, Szz) -- pointintegralimage.cpp:7-44 -- as 10
//       planes, over bands of 16 image rows: band column totals, their
//       prefix over the bands, then one sweep per band that writes every
//       value once.
//   k_stats
//       one thread per pixel: interval radius, 4-corner box query, FP64 3x3
//       covariance and eigensolve, curvature, oriented normal, and both
//       information matrices (statscalculatorintegralimage.cpp:20-82,
//       informationmatrixcalculator.cpp:9-57).
//   k_cloud_transform
//       Cloud::transformInPlace (cloud.cpp:191-204).
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "kernels.hpp"

namespace nicp {

// ------------------------------------------------------------ unprojection
// Loads the depth of 16 consecutive pixels starting at pix0; pixels at or
// beyond P read as 0 (invalid).
__device__ __forceinline__ void load16(const FrameDev &f, int pix0, int P, float d[16]) {
  if (f.depth_u16) {
    if (pix0 + 16 <= P && ((reinterpret_cast<uintptr_t>(f.depth_u16 + pix0) & 15) == 0)) {
      const uint4 *src = reinterpret_cast<const uint4 *>(f.depth_u16 + pix0);
      uint4 a = __ldg(src), b = __ldg(src + 1);
      uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int k = 0; k < 8; k++) {
        uint32_t lo = w[k] & 0xffffu, hi = w[k] >> 16;
        d[2 * k] = lo ? fm(f.depth_scale, (float)(int)lo) : 0.0f;
        d[2 * k + 1] = hi ? fm(f.depth_scale, (float)(int)hi) : 0.0f;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; k++) {
        int p = pix0 + k;
        uint16_t u = (p < P) ? f.depth_u16[p] : 0;
        d[k] = u ? fm(f.depth_scale, (float)(int)u) : 0.0f;
      }
    }
  } else {
    if (pix0 + 16 <= P && ((reinterpret_cast<uintptr_t>(f.depth_f32 + pix0) & 15) == 0)) {
      const float4 *src = reinterpret_cast<const float4 *>(f.depth_f32 + pix0);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float4 v = __ldg(src + k);
        d[4 * k] = v.x; d[4 * k + 1] = v.y; d[4 * k + 2] = v.z; d[4 * k + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; k++) {
        int p = pix0 + k;
        d[k] = (p < P) ? f.depth_f32[p] : 0.0f;
      }
    }
  }
}

__device__ __forceinline__ int block_sum_int(int v, int *smem) {
  // 256 threads
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  int t = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += smem[i];
  return t;
}

// frame_of[blockIdx.x]: the frame of the CTA (a table filled on the host
// with the frame descriptors; no search per CTA).
__global__ void __launch_bounds__(256) k_unproject_count(const FrameDev *__restrict__ frames,
                                                         const int *__restrict__ frame_of) {
  __shared__ int red[32];
  int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  int tile = blockIdx.x - f.tile_base;
  int P = f.rows * f.cols;
  int pix0 = tile * kUnprojTilePixels + threadIdx.x * 16;
  float d[16];
  load16(f, pix0, P, d);
  int cnt = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) cnt += depth_valid(d[k], f.min_d, f.max_d) ? 1 : 0;
  int tot = block_sum_int(cnt, red);
  if (threadIdx.x == 0) f.tile_counts[tile] = tot;
  if (tile == 0 && threadIdx.x == 0) f.count[1] = 0;  // points with a normal, counted by k_stats
}

// Gaussian3f of an unprojected pixel (pinholepointprojector.cpp:93-134):
// zVariation = (alpha z z) / (fB + z alpha), J = K^-1 [[z,0,c],[0,z,r],[0,0,1]],
// covariance = J diag(3, 3, zVariation) J^T, every product and sum in the
// order written, single rounding each.  All nine entries are kept: entry
// (i, j) is sum_k (J_ik D_k) J_jk, which differs from (j, i) in the last bit,
// as in the reference's product.  Stored as (mean, c00), (c01, c02, c10,
// c11), (c12, c20, c21, c22).
__device__ __forceinline__ void write_gaussian(const FrameDev &f, float4 *g, float4 pt, int c, int r, float z) {
  float zv = __fdiv_rn(fm(fm(f.alpha, z), z), fa(f.fB, fm(z, f.alpha)));
  const float J[9] = {z, 0.0f, (float)c, 0.0f, z, (float)r, 0.0f, 0.0f, 1.0f};
  float IJ[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      IJ[i * 3 + j] = fa(fa(fm(f.iK[i * 3 + 0], J[0 * 3 + j]), fm(f.iK[i * 3 + 1], J[1 * 3 + j])),
                         fm(f.iK[i * 3 + 2], J[2 * 3 + j]));
  const float D[3] = {3.0f, 3.0f, zv};
  float UD[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) UD[i * 3 + k] = fm(IJ[i * 3 + k], D[k]);
  float C[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C[i * 3 + j] = fa(fa(fm(UD[i * 3 + 0], IJ[j * 3 + 0]), fm(UD[i * 3 + 1], IJ[j * 3 + 1])),
                        fm(UD[i * 3 + 2], IJ[j * 3 + 2]));
  g[0] = make_float4(pt.x, pt.y, pt.z, C[0]);
  g[1] = make_float4(C[1], C[2], C[3], C[4]);
  g[2] = make_float4(C[5], C[6], C[7], C[8]);
}

// Thread t handles pixels t, t + 256, ... of its tile (kUnprojTilePixels /
// 256 rounds), so that depth loads, index stores and -- after the
// compaction -- point stores of a warp are consecutive.  The numbering is
// row-major: within the tile, pixel order is (round, warp, lane) order.
constexpr int kUnprojRounds = kUnprojTilePixels / 256;

__global__ void __launch_bounds__(256) k_unproject_write(const FrameDev *__restrict__ frames,
                                                         const int *__restrict__ frame_of) {
  __shared__ int red[32];
  __shared__ int rcnt[kUnprojRounds * 8];  // valid pixels per (round, warp), then their exclusive prefix
  __shared__ int wtot[4];
  int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  const int tile = blockIdx.x - f.tile_base;
  const int P = f.rows * f.cols;
  const int ntiles = (P + kUnprojTilePixels - 1) / kUnprojTilePixels;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  // points numbered before this tile
  int before = 0;
  for (int q = t; q < tile; q += blockDim.x) before += f.tile_counts[q];
  before = block_sum_int(before, red);
  const int base = tile * kUnprojTilePixels + t;
  // The tile's depths come in with 128-bit loads (thread t: bytes 16 t,
  // 16 (t + 256), ... of the tile) into shared memory, from where thread t
  // takes pixels t, t + 256, ...; unaligned or partial tiles load per pixel.
  __shared__ __align__(16) unsigned char sdepth[kUnprojTilePixels * 4];
  const int tile0 = tile * kUnprojTilePixels;
  const int n_in = min(kUnprojTilePixels, P - tile0);
  float d[kUnprojRounds];
  if (f.depth_u16) {
    const uint16_t *src = f.depth_u16 + tile0;
    uint16_t *dst = reinterpret_cast<uint16_t *>(sdepth);
    if (n_in == kUnprojTilePixels && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
      const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
      uint4 v[kUnprojTilePixels / 8 / 256];
#pragma unroll
      for (int k = 0; k < kUnprojTilePixels / 8 / 256; k++) v[k] = __ldg(s4 + t + 256 * k);
#pragma unroll
      for (int k = 0; k < kUnprojTilePixels / 8 / 256; k++) reinterpret_cast<uint4 *>(dst)[t + 256 * k] = v[k];
    } else {
#pragma unroll
      for (int k = 0; k < kUnprojRounds; k++) {
        const int q = t + 256 * k;
        dst[q] = q < n_in ? src[q] : (uint16_t)0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kUnprojRounds; k++) {
      const uint16_t u = dst[t + 256 * k];
      d[k] = u ? fm(f.depth_scale, (float)(int)u) : 0.0f;
    }
  } else {
    const float *src = f.depth_f32 + tile0;
    float *dst = reinterpret_cast<float *>(sdepth);
    if (n_in == kUnprojTilePixels && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
      const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
      uint4 v[kUnprojTilePixels / 4 / 256];
#pragma unroll
      for (int k = 0; k < kUnprojTilePixels / 4 / 256; k++) v[k] = __ldg(s4 + t + 256 * k);
#pragma unroll
      for (int k = 0; k < kUnprojTilePixels / 4 / 256; k++) reinterpret_cast<uint4 *>(dst)[t + 256 * k] = v[k];
    } else {
#pragma unroll
      for (int k = 0; k < kUnprojRounds; k++) {
        const int q = t + 256 * k;
        dst[q] = q < n_in ? src[q] : 0.0f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kUnprojRounds; k++) d[k] = dst[t + 256 * k];
  }
  unsigned mask = 0;
#pragma unroll
  for (int k = 0; k < kUnprojRounds; k++) {
    const int p = base + k * 256;
    const bool valid = p < P && depth_valid(d[k], f.min_d, f.max_d);
    mask |= (valid ? 1u : 0u) << k;
    const unsigned bal = __ballot_sync(0xffffffffu, valid);
    if (lane == 0) rcnt[k * 8 + wid] = __popc(bal);
  }
  __syncthreads();
  // exclusive prefix of the kUnprojRounds x 8 counts in (round, warp) order
  if (t < kUnprojRounds * 8) {
    const int v = rcnt[t];
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) wtot[wid] = inc;
    __syncwarp();
    asm volatile("bar.sync 1, %0;" ::"r"(kUnprojRounds * 8));  // the first kUnprojRounds * 8 threads
    int off = 0;
    for (int w = 0; w < wid; w++) off += wtot[w];
    rcnt[t] = off + inc - v;
    if (t == kUnprojRounds * 8 - 1 && tile == ntiles - 1) *f.count = before + off + inc;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < kUnprojRounds; k++) {
    const int p = base + k * 256;
    const bool valid = (mask >> k) & 1u;
    const unsigned bal = __ballot_sync(0xffffffffu, valid);
    int out = -1;
    if (valid) {
      const int idx = before + rcnt[k * 8 + wid] + __popc(bal & lt);
      const int r = p / f.cols, c = p - r * f.cols;
      const float4 pt = unproject_pixel(f.iKRt, c, r, d[k]);
      f.pts[idx] = pt;
      if (f.gauss) write_gaussian(f, f.gauss + 3 * (size_t)idx, pt, c, r, d[k]);
      out = idx;
    }
    if (p < P) f.index[p] = out;
  }
}

// ------------------------------------------------------------ moments
// Storage policies for the integral image.  The ten moment planes are kept
// as five interleaved plane pairs: pair k holds planes 2k and 2k + 1 of
// pixel i side by side (element 2 (k P + i) + (m & 1)), so that the stats
// kernel reads a corner's ten sums with five paired loads and the sweep
// writes them with five paired stores.
struct MomF64 {
  typedef double T;
  __device__ static double val(double v) { return v; }
  __device__ static void store(void *base, size_t P, int m, size_t i, double v) {
    static_cast<double *>(base)[2 * ((size_t)(m >> 1) * P + i) + (m & 1)] = v;
  }
  __device__ static void store2(void *base, size_t P, int k, size_t i, double a, double b) {
    static_cast<double2 *>(base)[(size_t)k * P + i] = make_double2(a, b);
  }
  __device__ static void load2(const void *base, size_t P, int k, size_t i, double &a, double &b) {
    const double2 v = static_cast<const double2 *>(base)[(size_t)k * P + i];
    a = v.x;
    b = v.y;
  }
};
struct MomF32 {
  typedef float T;
  __device__ static double val(float v) { return (double)v; }
  __device__ static void store(void *base, size_t P, int m, size_t i, double v) {
    static_cast<float *>(base)[2 * ((size_t)(m >> 1) * P + i) + (m & 1)] = (float)v;
  }
  __device__ static void store2(void *base, size_t P, int k, size_t i, double a, double b) {
    static_cast<float2 *>(base)[(size_t)k * P + i] = make_float2((float)a, (float)b);
  }
  __device__ static void load2(const void *base, size_t P, int k, size_t i, double &a, double &b) {
    const float2 v = static_cast<const float2 *>(base)[(size_t)k * P + i];
    a = (double)v.x;
    b = (double)v.y;
  }
};
// Two-float: an unevaluated sum hi + lo of two floats (about 48 significant
// bits); values travel as double inside the kernels and are split on store.
struct MomTwoFloat {
  typedef float2 T;
  __device__ static double val(float2 v) { return (double)v.x + (double)v.y; }
  __device__ static float2 split(double v) {
    const float hi = (float)v;
    return make_float2(hi, (float)(v - (double)hi));
  }
  __device__ static void store(void *base, size_t P, int m, size_t i, double v) {
    static_cast<float2 *>(base)[2 * ((size_t)(m >> 1) * P + i) + (m & 1)] = split(v);
  }
  __device__ static void store2(void *base, size_t P, int k, size_t i, double a, double b) {
    const float2 x = split(a), y = split(b);
    static_cast<float4 *>(base)[(size_t)k * P + i] = make_float4(x.x, x.y, y.x, y.y);
  }
  __device__ static void load2(const void *base, size_t P, int k, size_t i, double &a, double &b) {
    const float4 v = static_cast<const float4 *>(base)[(size_t)k * P + i];
    a = (double)v.x + (double)v.y;
    b = (double)v.z + (double)v.w;
  }
};

// The arithmetic type the moments are accumulated in for each storage.
template <class M> struct MomAcc { typedef double T; };
template <> struct MomAcc<MomF32> { typedef float T; };

__device__ __forceinline__ void point_moments(float4 p, bool valid, double m[10]) {
  double x = p.x, y = p.y, z = p.z;
  double v = valid ? 1.0 : 0.0;
  m[0] = v;
  m[1] = v * x; m[2] = v * y; m[3] = v * z;
  m[4] = v * x * x; m[5] = v * x * y; m[6] = v * x * z;
  m[7] = v * y * y; m[8] = v * y * z; m[9] = v * z * z;
}
__device__ __forceinline__ void point_moments(float4 p, bool valid, float m[10]) {
  float x = p.x, y = p.y, z = p.z;
  float v = valid ? 1.0f : 0.0f;
  m[0] = v;
  m[1] = v * x; m[2] = v * y; m[3] = v * z;
  m[4] = v * fm(x, x); m[5] = v * fm(x, y); m[6] = v * fm(x, z);
  m[7] = v * fm(y, y); m[8] = v * fm(y, z); m[9] = v * fm(z, z);
}

constexpr int kRowThreads = 128;
constexpr int kRowPix = 5;  // 128 x 5 = 640: one chunk per 640-pixel row

// One chunk of one image row (kRowThreads x kRowPix pixels from x0):
// inclusive prefix along x of the 10 moments, starting from carry[] (the
// chunks to its left), which is advanced by the chunk total.  Each thread
// keeps the points of its kRowPix pixels (depths d[]); the moments are
// formed twice (for the thread total, then per pixel for emit) to keep
// register use low.  emit(k, c, acc) receives pixel c = x0 + t kRowPix + k
// with its 10 prefix values.  [kM0, kM0 + kNM) selects the moments the call
// scans (the band sweep runs two calls of five, which halves the registers
// the pixels' moments hold and fits 4 CTAs per SM; every moment's additions
// are the same either way).  Contains two __syncthreads.
template <class M, int kM0 = 0, int kNM = 10, class Emit>
__device__ __forceinline__ void row_chunk_scan(const FrameDev &f, int r, int x0, const float d[kRowPix],
                                               typename MomAcc<M>::T carry[10],
                                               typename MomAcc<M>::T (*wtot)[10], Emit &&emit) {
  typedef typename MomAcc<M>::T A;
  const int cols = f.cols;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c0 = x0 + threadIdx.x * kRowPix;
  float4 pt[kRowPix];
  unsigned vmask = 0;
  A acc[10];
#pragma unroll
  for (int m = kM0; m < kM0 + kNM; m++) acc[m] = A(0);
#pragma unroll
  for (int k = 0; k < kRowPix; k++) {
    const int c = c0 + k;
    const bool valid = c < cols && depth_valid(d[k], f.min_d, f.max_d);
    pt[k] = valid ? unproject_pixel(f.iKRt, c, r, d[k]) : make_float4(0, 0, 0, 0);
    vmask |= (valid ? 1u : 0u) << k;
    A mk[10];
    point_moments(pt[k], valid, mk);
#pragma unroll
    for (int m = kM0; m < kM0 + kNM; m++) acc[m] = acc[m] + mk[m];
  }
  // warp inclusive scan of the thread totals; acc becomes the exclusive offset
#pragma unroll
  for (int m = kM0; m < kM0 + kNM; m++) {
    A inc = acc[m];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      A y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc = inc + y;
    }
    if (lane == 31) wtot[wid][m] = inc;
    acc[m] = inc - acc[m];
  }
  __syncthreads();
#pragma unroll
  for (int m = kM0; m < kM0 + kNM; m++) {
    A off = carry[m] + acc[m], tot = A(0);
    for (int w = 0; w < kRowThreads / 32; w++) {
      A t = wtot[w][m];
      if (w < wid) off = off + t;
      tot = tot + t;
    }
    acc[m] = off;
    carry[m] = carry[m] + tot;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kRowPix; k++) {
    A mk[10];
    point_moments(pt[k], (vmask >> k) & 1u, mk);
#pragma unroll
    for (int m = kM0; m < kM0 + kNM; m++) acc[m] = acc[m] + mk[m];
    emit(k, c0 + k, acc);
  }
}

// Raw depth words (u16 value or float bits), loaded ahead of use; the
// conversion happens where the depth is consumed, so that a prefetch does
// not wait for its own load.
__device__ __forceinline__ unsigned depth_raw(const FrameDev &f, int pix) {
  return f.depth_u16 ? (unsigned)f.depth_u16[pix] : __float_as_uint(f.depth_f32[pix]);
}
__device__ __forceinline__ float depth_from_raw(const FrameDev &f, unsigned w) {
  if (f.depth_u16) return w ? fm(f.depth_scale, (float)(int)w) : 0.0f;
  return __uint_as_float(w);
}
__device__ __forceinline__ void load_row_raw(const FrameDev &f, int r, int c0, unsigned w[kRowPix]) {
#pragma unroll
  for (int k = 0; k < kRowPix; k++) w[k] = c0 + k < f.cols ? depth_raw(f, r * f.cols + c0 + k) : 0u;
}

// ---- integral image in three passes over bands of kBandRows image rows.
// With R(r, c) the prefix along x of row r, the integral image is
// I(r, c) = carry_b(c) + the sum of R(r', c) over the rows r' <= r of r's
// band b, where carry_b(c) = the sum over the bands above of their column
// totals.
//   k_moments_band_totals  per band: column sums of the raw moments over the
//                          band's rows, then their prefix along x (= the
//                          sum of the band's row prefixes)
//   k_moments_band_carry   per (plane, column): exclusive prefix of the
//                          band totals over the bands, in place
//   k_moments_band_sweep   per band: row prefixes (row_chunk_scan) added
//                          down the band onto carry_b; every integral value
//                          is written once, from shared memory, coalesced
constexpr int kBandRows = 16;
constexpr int kChunkPix = kRowThreads * kRowPix;

template <class M>
constexpr int band_smem_bytes() { return 10 * kChunkPix * (int)sizeof(typename MomAcc<M>::T); }

template <class M>
__global__ void __launch_bounds__(kRowThreads) k_moments_band_totals(const FrameDev *__restrict__ frames,
                                                                     const int *__restrict__ frame_of) {
  typedef typename MomAcc<M>::T A;
  extern __shared__ __align__(16) unsigned char band_raw[];
  A *cs = reinterpret_cast<A *>(band_raw);  // [10][kChunkPix]
  __shared__ A wtot[kRowThreads / 32][10];
  const int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  const int b = blockIdx.x - f.band_base;
  const int cols = f.cols;
  const int r0 = b * kBandRows, nr = min(f.rows - r0, kBandRows);
  A *tot = static_cast<A *>(f.band_tot) + (size_t)b * 10 * cols;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  A carry[10];
#pragma unroll
  for (int m = 0; m < 10; m++) carry[m] = A(0);
  for (int x0 = 0; x0 < cols; x0 += kChunkPix) {
    const int n = min(kChunkPix, cols - x0);
    // column sums over the band (thread t: columns x0 + t + kRowThreads j)
#pragma unroll 1
    for (int j = 0; j < kRowPix; j++) {
      const int q = j * kRowThreads + t;
      A acc[10];
#pragma unroll
      for (int m = 0; m < 10; m++) acc[m] = A(0);
      if (q < n) {
        const int c = x0 + q;
        unsigned w[kBandRows];
#pragma unroll
        for (int i = 0; i < kBandRows; i++) w[i] = i < nr ? depth_raw(f, (r0 + i) * cols + c) : 0u;
#pragma unroll
        for (int i = 0; i < kBandRows; i++) {
          const float d = depth_from_raw(f, w[i]);
          const bool valid = i < nr && depth_valid(d, f.min_d, f.max_d);
          const float4 p = valid ? unproject_pixel(f.iKRt, c, r0 + i, d) : make_float4(0, 0, 0, 0);
          A mk[10];
          point_moments(p, valid, mk);
#pragma unroll
          for (int m = 0; m < 10; m++) acc[m] = acc[m] + mk[m];
        }
      }
#pragma unroll
      for (int m = 0; m < 10; m++) cs[m * kChunkPix + q] = acc[m];
    }
    __syncthreads();
    // inclusive prefix along x of the column sums, in place (thread t:
    // entries t kRowPix .. t kRowPix + kRowPix - 1)
    A loc[10];
#pragma unroll
    for (int m = 0; m < 10; m++) {
      A sum = A(0);
#pragma unroll
      for (int k = 0; k < kRowPix; k++) sum = sum + cs[m * kChunkPix + t * kRowPix + k];
      A inc = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        A y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = inc + y;
      }
      if (lane == 31) wtot[wid][m] = inc;
      loc[m] = inc - sum;
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 10; m++) {
      A off = carry[m] + loc[m], all = A(0);
      for (int w = 0; w < kRowThreads / 32; w++) {
        const A v = wtot[w][m];
        if (w < wid) off = off + v;
        all = all + v;
      }
      carry[m] = carry[m] + all;
#pragma unroll
      for (int k = 0; k < kRowPix; k++) {
        off = off + cs[m * kChunkPix + t * kRowPix + k];
        cs[m * kChunkPix + t * kRowPix + k] = off;
      }
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 10; m++)
#pragma unroll
      for (int j = 0; j < kRowPix; j++) {
        const int q = j * kRowThreads + t;
        if (q < n) tot[(size_t)m * cols + x0 + q] = cs[m * kChunkPix + q];
      }
    __syncthreads();  // the copy-out has read cs before the next chunk overwrites it
  }
}

// One thread per (plane, column) of a frame: band totals -> band carries.
template <class M>
__global__ void __launch_bounds__(128) k_moments_band_carry(const FrameDev *__restrict__ frames,
                                                            const int *__restrict__ frame_of) {
  typedef typename MomAcc<M>::T A;
  constexpr int kAhead = 8;
  const int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  const int q = (blockIdx.x - f.col_base) * 128 + threadIdx.x;
  const size_t stride = (size_t)10 * f.cols;
  if (q >= (int)stride) return;
  const int nb = (f.rows + kBandRows - 1) / kBandRows;
  A *tot = static_cast<A *>(f.band_tot) + q;
  A acc = A(0);
  for (int b0 = 0; b0 < nb; b0 += kAhead) {
    A v[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; k++) v[k] = b0 + k < nb ? tot[(size_t)(b0 + k) * stride] : A(0);
#pragma unroll
    for (int k = 0; k < kAhead; k++)
      if (b0 + k < nb) {
        tot[(size_t)(b0 + k) * stride] = acc;
        acc = acc + v[k];
      }
  }
}

// Grid (band, frame): the frame is blockIdx.y, no search over the frame
// descriptors; CTAs past a smaller frame's last band return at once.
template <class M>
__global__ void __launch_bounds__(kRowThreads, 4) k_moments_band_sweep(const FrameDev *__restrict__ frames, int nframes) {
  typedef typename MomAcc<M>::T A;
  extern __shared__ __align__(16) unsigned char band_raw[];
  A *state = reinterpret_cast<A *>(band_raw);  // [10][kChunkPix]: I(r, c) of the current row
  __shared__ A wtot[kRowThreads / 32][10];
  __shared__ A rowc[kBandRows][10];  // row carries across chunks (frames wider than a chunk)
  const FrameDev &f = frames[blockIdx.y];
  const int b = blockIdx.x;
  const int cols = f.cols;
  const size_t P = (size_t)f.rows * cols;
  if (b * kBandRows >= f.rows) return;
  const int r0 = b * kBandRows, r1 = min(f.rows, r0 + kBandRows);
  const A *carry_b = static_cast<const A *>(f.band_tot) + (size_t)b * 10 * cols;
  const int t = threadIdx.x;
  for (int x0 = 0; x0 < cols; x0 += kChunkPix) {
    const int n = min(kChunkPix, cols - x0);
    const int c0 = x0 + t * kRowPix;
    // the band's carry row; made visible to the owners of the columns by the
    // first barrier inside the first scan
#pragma unroll
    for (int m = 0; m < 10; m++)
#pragma unroll
      for (int j = 0; j < kRowPix; j++) {
        const int q = j * kRowThreads + t;
        state[m * kChunkPix + q] = q < n ? carry_b[(size_t)m * cols + x0 + q] : A(0);
      }
    unsigned wn[kRowPix];
    load_row_raw(f, r0, c0, wn);
    for (int r = r0; r < r1; r++) {
      float d[kRowPix];
#pragma unroll
      for (int k = 0; k < kRowPix; k++) d[k] = depth_from_raw(f, wn[k]);
      if (r + 1 < r1) load_row_raw(f, r + 1, c0, wn);
      A carry[10];
#pragma unroll
      for (int m = 0; m < 10; m++) carry[m] = x0 ? rowc[r - r0][m] : A(0);
      // every thread has finished the previous row's copy-out once it has
      // passed the first barrier inside the scan
      row_chunk_scan<M, 0, 5>(f, r, x0, d, carry, wtot, [&](int, int c, const A *acc) {
        if (c < cols) {
#pragma unroll
          for (int m = 0; m < 5; m++)
            state[m * kChunkPix + (c - x0)] = state[m * kChunkPix + (c - x0)] + acc[m];
        }
      });
      row_chunk_scan<M, 5, 5>(f, r, x0, d, carry, wtot, [&](int, int c, const A *acc) {
        if (c < cols) {
#pragma unroll
          for (int m = 5; m < 10; m++)
            state[m * kChunkPix + (c - x0)] = state[m * kChunkPix + (c - x0)] + acc[m];
        }
      });
      if (t == 0 && x0 + kChunkPix < cols) {
#pragma unroll
        for (int m = 0; m < 10; m++) rowc[r - r0][m] = carry[m];
      }
      __syncthreads();
      const size_t row0 = (size_t)r * cols + x0;
#pragma unroll
      for (int k = 0; k < 5; k++)
#pragma unroll
        for (int j = 0; j < kRowPix; j++) {
          const int q = j * kRowThreads + t;
          if (q < n)
            M::store2(f.moments, P, k, row0 + q, (double)state[2 * k * kChunkPix + q],
                      (double)state[(2 * k + 1) * kChunkPix + q]);
        }
    }
    __syncthreads();  // the last copy-out has read the state before the next chunk's carry row
  }
}

// ------------------------------------------------------------ stats + omegas
// Grid (pixel tile, frame): the frame is blockIdx.y, no search over the frame
// descriptors.
// One thread per pixel: the CTA size and the CTAs per SM the compiler
// budgets registers for are launch shapes only (the autotuner picks one per
// frame-size mix); every pixel's result is the same under all of them.
// kLean: Stats are not kept and the information matrices have the
// converter's form U diag(d0, d1, d1) U^T (decided on the host for the launch).
template <class M, int kThreads, int kMinCtas, bool kLean>
__global__ void __launch_bounds__(kThreads, kMinCtas) k_stats(const FrameDev *__restrict__ frames, int nframes) {
  const FrameDev &f = frames[blockIdx.y];
  int pix = blockIdx.x * kThreads + threadIdx.x;
  int rows = f.rows, cols = f.cols;
  int P = rows * cols;
  if (pix >= P) return;
  // index and depth loaded together (the depth is not needed when the index is negative)
  const int idx = f.index[pix];
  const float d = depth_of(f, pix);
  if (idx < 0) return;
  int r = pix / cols, c = pix - r * cols;
  float4 nout = make_float4(0.f, 0.f, 0.f, 0.f);
  float om[12];
#pragma unroll
  for (int k = 0; k < 12; k++) om[k] = 0.f;
  double lam[3] = {0, 0, 0};
  double U[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  bool reached = false;
  int omega_class = 0;
  double mean[3] = {0.0, 0.0, 0.0};
  int nwin = 0;
  int rad = interval_radius(f.K, d, f.min_d, f.max_d, f.world_radius);
  if (rad >= 0 && rad >= f.min_radius) {
    if (rad > f.max_radius) rad = f.max_radius;
    // pointintegralimage.cpp:53-66
    int xm = min(max(c - rad - 1, 0), cols - 1), xM = min(max(c + rad - 1, 0), cols - 1);
    int ym = min(max(r - rad - 1, 0), rows - 1), yM = min(max(r + rad - 1, 0), rows - 1);
    size_t iA = (size_t)yM * cols + xM, iB = (size_t)ym * cols + xm;
    size_t iC = (size_t)yM * cols + xm, iD = (size_t)ym * cols + xM;
    double S[10];
    // the four corners of each plane pair: 20 paired loads
#pragma unroll
    for (int k = 0; k < 5; k++) {
      double a0, a1, b0, b1, c0, c1, d0, d1;
      M::load2(f.moments, P, k, iA, a0, a1);
      M::load2(f.moments, P, k, iB, b0, b1);
      M::load2(f.moments, P, k, iC, c0, c1);
      M::load2(f.moments, P, k, iD, d0, d1);
      double s0 = a0 + b0, s1 = a1 + b1;
      s0 = s0 - c0;
      s1 = s1 - c1;
      S[2 * k] = s0 - d0;
      S[2 * k + 1] = s1 - d1;
    }
    int n = (int)S[0];
    if (n >= f.min_points) {
      double dn = 1.0 / S[0];
      double mu0 = S[1] * dn, mu1 = S[2] * dn, mu2 = S[3] * dn;
      mean[0] = mu0; mean[1] = mu1; mean[2] = mu2;
      nwin = n;
      double C[6] = {S[4] * dn - mu0 * mu0, S[5] * dn - mu0 * mu1, S[6] * dn - mu0 * mu2,
                     S[7] * dn - mu1 * mu1, S[8] * dn - mu1 * mu2, S[9] * dn - mu2 * mu2};
      // FP64 solve.  (An FP32 trigonometric solve refined in FP64 was
      // measured: no faster, and its refinement could settle on the wrong
      // root when the two smallest eigenvalues are close.)  Without kept
      // Stats and with information matrices of the converter's form
      // U diag(d0, d1, d1) U^T, only the smallest eigenpair matters: the
      // eigenvalues come first, and the normal's eigenvector is computed only
      // for a flat pixel, from its null vector when the smallest eigenvalue is
      // the better separated one -- the same arithmetic as the full solve, so
      // the normal is bitwise the full solve's.
      constexpr bool lean = kLean;
      double B[6], amax = 1.0, l0 = 0, l1 = 0, l2 = 0;
      bool degenerate = true;
      if (lean) {
        degenerate = d_eig3_values(C, B, amax, l0, l1, l2, lam, U);
        if (!degenerate) { lam[0] = l0 * amax; lam[1] = l1 * amax; lam[2] = l2 * amax; }
      } else {
        d_eig3(C, lam, U);
      }
      if (lam[0] < 0) lam[0] = 0;
      reached = true;
      double kappa = lam[0] / (((lam[0] + lam[1]) + lam[2]) + 1e-9);
      nout.w = (float)kappa;
      if (kappa < (double)f.curv_thr) {
        double u0[3] = {U[0], U[3], U[6]};
        if (lean && !degenerate) {
          if (l1 - l0 >= l2 - l1) {
            d_null_vector(B, l0, u0);
          } else {
            double v1[3], v2[3];
            d_eig3_vectors(B, l0, l1, l2, u0, v1, v2);
          }
        }
        float4 p = unproject_pixel(f.iKRt, c, r, d);
        double nx = u0[0], ny = u0[1], nz = u0[2];
        if (nx * p.x + ny * p.y + nz * p.z > 0) { nx = -nx; ny = -ny; nz = -nz; }
        nout.x = (float)nx; nout.y = (float)ny; nout.z = (float)nz;
        // information matrices: Omega = U diag(D) U^T
        double Dp[3], Dn[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          Dp[k] = (kappa < (double)f.pim_thr) ? f.pim_flat[k] : f.pim_nonflat[k];
          Dn[k] = (kappa < (double)f.nim_thr) ? f.nim_flat[k] : f.nim_nonflat[k];
        }
        omega_class = (kappa < (double)f.pim_thr ? 0 : 1) + (kappa < (double)f.nim_thr ? 0 : 2);
        const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
        if (lean) {
          // U diag(d0, d1, d1) U^T = d1 I + (d0 - d1) u0 u0^T
#pragma unroll
          for (int e = 0; e < 6; e++) {
            const int i = ii[e], j = jj[e];
            const double uu = u0[i] * u0[j];
            om[e] = (float)((i == j ? Dp[1] : 0.0) + (Dp[0] - Dp[1]) * uu);
            om[6 + e] = (float)((i == j ? Dn[1] : 0.0) + (Dn[0] - Dn[1]) * uu);
          }
        } else {
#pragma unroll
          for (int e = 0; e < 6; e++) {
            int i = ii[e], j = jj[e];
            double sp = 0, sn = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
              double uu = U[i * 3 + k] * U[j * 3 + k];
              sp += Dp[k] * uu;
              sn += Dn[k] * uu;
            }
            om[e] = (float)sp;
            om[6 + e] = (float)sn;
          }
        }
      }
    }
  }
  f.nrm[idx] = nout;
  {
    // count the points that got a normal (one atomic per warp)
    const bool has = nout.x != 0.0f || nout.y != 0.0f || nout.z != 0.0f;
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, has);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(act) - 1) && m) atomicAdd(f.count + 1, __popc(m));
  }
  // the point's w carries "has a normal" and the information-matrix class
  // (see kNoNormalW)
  reinterpret_cast<float *>(f.pts + idx)[3] =
      (nout.x != 0.0f || nout.y != 0.0f || nout.z != 0.0f) ? 1.0f + (float)omega_class : kNoNormalW;
  // With the converter's structure the information matrices stay implicit:
  // d1 I + (d0 - d1) n n^T from the normal, the class code in the point's w
  // and the cloud's (d0, d1) per class (the fused kernel uses them so, and
  // k_materialize_omg writes them out for a reader that needs the matrices).
  if (!kLean) {
    float4 *o = f.omg + 3 * (size_t)idx;
    o[0] = make_float4(om[0], om[1], om[2], om[3]);
    o[1] = make_float4(om[4], om[5], om[6], om[7]);
    o[2] = make_float4(om[8], om[9], om[10], om[11]);
  }
  if (f.keep_stats) {
    float *e = f.eig + kStatsWords * (size_t)idx;
    if (!reached) { lam[0] = lam[1] = lam[2] = 0; }
    e[0] = (float)lam[0]; e[1] = (float)lam[1]; e[2] = (float)lam[2];
#pragma unroll
    for (int k = 0; k < 9; k++) e[3 + k] = (float)U[k];
    e[12] = (float)mean[0]; e[13] = (float)mean[1]; e[14] = (float)mean[2];
    e[15] = (float)nwin;
  }
}

// ------------------------------------------------------------ transform
__global__ void k_cloud_transform(float4 *pts, float4 *nrm, float4 *omg, float *eig, float4 *gauss, const int *count,
                                  int capacity, const float *__restrict__ m12) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= capacity || i >= *count) return;
  float A[12];
#pragma unroll
  for (int k = 0; k < 12; k++) A[k] = m12[k];
  float4 p0 = pts[i];
  float3 p = xform_point(A, p0);
  pts[i] = make_float4(p.x, p.y, p.z, p0.w);
  float4 n0 = nrm[i];
  float3 n = xform_normal(A, n0);
  nrm[i] = make_float4(n.x, n.y, n.z, n0.w);
  // Omega' = (R Omega) R^T over the 3x3 block (an implicit Omega -- omg
  // null -- follows the rotated normal by itself)
  float R[9] = {A[0], A[1], A[2], A[4], A[5], A[6], A[8], A[9], A[10]};
  if (omg) {
    float4 o0 = omg[3 * i], o1 = omg[3 * i + 1], o2 = omg[3 * i + 2];
    float Op[9] = {o0.x, o0.y, o0.z, o0.y, o0.w, o1.x, o0.z, o1.x, o1.y};
    float On[9] = {o1.z, o1.w, o2.x, o1.w, o2.y, o2.z, o2.x, o2.z, o2.w};
    float res[2][6];
    for (int w = 0; w < 2; w++) {
      const float *O = w ? On : Op;
      float RO[9];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          RO[a * 3 + b] = fa(fa(fm(R[a * 3 + 0], O[0 * 3 + b]), fm(R[a * 3 + 1], O[1 * 3 + b])), fm(R[a * 3 + 2], O[2 * 3 + b]));
      const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
      for (int e = 0; e < 6; e++) {
        int a = ii[e], b = jj[e];
        res[w][e] = fa(fa(fm(RO[a * 3 + 0], R[b * 3 + 0]), fm(RO[a * 3 + 1], R[b * 3 + 1])), fm(RO[a * 3 + 2], R[b * 3 + 2]));
      }
    }
    omg[3 * i] = make_float4(res[0][0], res[0][1], res[0][2], res[0][3]);
    omg[3 * i + 1] = make_float4(res[0][4], res[0][5], res[1][0], res[1][1]);
    omg[3 * i + 2] = make_float4(res[1][2], res[1][3], res[1][4], res[1][5]);
  }
  if (gauss) {
    // Gaussian3fVector::transformInPlace (gaussian3.h:66-73): mean' = R mean + t,
    // covariance' = (R C) R^T
    float4 g0 = gauss[3 * i], g1 = gauss[3 * i + 1], g2 = gauss[3 * i + 2];
    float C[9] = {g0.w, g1.x, g1.y, g1.z, g1.w, g2.x, g2.y, g2.z, g2.w};
    float m[3] = {g0.x, g0.y, g0.z}, mo[3];
    for (int a = 0; a < 3; a++)
      mo[a] = fa(fa(fa(fm(R[a * 3 + 0], m[0]), fm(R[a * 3 + 1], m[1])), fm(R[a * 3 + 2], m[2])), A[a * 4 + 3]);
    float RC[9], Co[9];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        RC[a * 3 + b] = fa(fa(fm(R[a * 3 + 0], C[0 * 3 + b]), fm(R[a * 3 + 1], C[1 * 3 + b])), fm(R[a * 3 + 2], C[2 * 3 + b]));
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        Co[a * 3 + b] =
            fa(fa(fm(RC[a * 3 + 0], R[b * 3 + 0]), fm(RC[a * 3 + 1], R[b * 3 + 1])), fm(RC[a * 3 + 2], R[b * 3 + 2]));
    gauss[3 * i] = make_float4(mo[0], mo[1], mo[2], Co[0]);
    gauss[3 * i + 1] = make_float4(Co[1], Co[2], Co[3], Co[4]);
    gauss[3 * i + 2] = make_float4(Co[5], Co[6], Co[7], Co[8]);
  }
  if (eig) {
    // StatsVector::transformInPlace (stats.h): the 4x4 Stats times m --
    // eigenvectors rotated, the mean column (w = 1: the window mean of a
    // reached point, or the identity's (0 0 0 1) of a default Stats) moved
    // like a point
    float *e = eig + kStatsWords * (size_t)i;
    float U[9];
    for (int k = 0; k < 9; k++) U[k] = e[3 + k];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        e[3 + a * 3 + b] = fa(fa(fm(R[a * 3 + 0], U[0 * 3 + b]), fm(R[a * 3 + 1], U[1 * 3 + b])), fm(R[a * 3 + 2], U[2 * 3 + b]));
    float mo[3];
    for (int a = 0; a < 3; a++) mo[a] = row4(A + 4 * a, e[12], e[13], e[14], 1.0f);
    e[12] = mo[0]; e[13] = mo[1]; e[14] = mo[2];
  }
}

// PinholePointProjector::projectIntervals (pinholepointprojector.cpp:136-148).
__global__ void k_intervals(const float *__restrict__ depth, int P, const float *__restrict__ K9, float min_d, float max_d,
                            float R, int32_t *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  float K[9];
#pragma unroll
  for (int k = 0; k < 9; k++) K[k] = K9[k];
  out[i] = interval_radius(K, depth[i], min_d, max_d, R);
}

// ------------------------------------------------------------ launchers
void launch_intervals(const float *d_depth, int P, const float *d_K9, float min_d, float max_d, float R, int32_t *d_out,
                      cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_STATS, s);
  if (P > 0) k_intervals<<<(P + 255) / 256, 256, 0, s>>>(d_depth, P, d_K9, min_d, max_d, R, d_out);
  prof->end(NICP_K_STATS, s);
}

// DepthImage_scale (imageutils.cpp:6-37), with the u16 -> float conversion
// of DepthImage_convert_16UC1_to_32FC1 (imageutils.cpp:85-99) fused in front
// when the input is u16.  One thread per output pixel; sums and the variance
// test in the reference's order, single-rounded.
__global__ void k_depth_scale(const uint16_t *__restrict__ u16, const float *__restrict__ f32, size_t pitch_elems,
                              int rows, int cols, float depth_scale, int step, float max_cov, float *__restrict__ out,
                              int out_rows, int out_cols) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= out_rows * out_cols) return;
  const int r = idx / out_cols, c = idx - r * out_cols;
  const int sr = r * step, sc = c * step;
  float acc = 0.0f, acc2 = 0.0f;
  int np = 0;
  for (int i = 0; i < step; i++)
    for (int j = 0; j < step; j++) {
      if (sr + i >= rows || sc + j >= cols) continue;
      const size_t at = (size_t)(sr + i) * pitch_elems + sc + j;
      float f;
      if (u16) {
        const uint16_t u = u16[at];
        f = u ? fm(depth_scale, (float)(int)u) : 0.0f;
      } else {
        f = f32[at];
      }
      acc = fa(acc, f);
      acc2 = fa(acc2, fm(f, f));
      np += f > 0.0f;
    }
  float v = 0.0f;
  if (np) {
    const float mu = __fdiv_rn(acc, (float)np);
    const float sigma = fsb(__fdiv_rn(acc2, (float)np), fm(mu, mu));
    if (!(sigma > max_cov)) v = mu;
  }
  out[idx] = v;
}

void launch_depth_scale(const uint16_t *u16, const float *f32, size_t pitch_elems, int rows, int cols,
                        float depth_scale, int step, float max_cov, float *out, cudaStream_t s) {
  const int orows = rows / step, ocols = cols / step, n = orows * ocols;
  if (n > 0)
    k_depth_scale<<<(n + 255) / 256, 256, 0, s>>>(u16, f32, pitch_elems, rows, cols, depth_scale, step, max_cov, out,
                                                  orows, ocols);
}

void launch_unproject(const FrameDev *d_frames, int nframes, int total_tiles, const int *frame_of_tile, cudaStream_t s,
                      Profiler *prof) {
  (void)nframes;
  prof->begin(NICP_K_UNPROJECT, s);
  k_unproject_count<<<total_tiles, 256, 0, s>>>(d_frames, frame_of_tile);
  k_unproject_write<<<total_tiles, 256, 0, s>>>(d_frames, frame_of_tile);
  prof->end(NICP_K_UNPROJECT, s, 2);
}

// ---- few-frame path (no more than kRowPathFrames frames per launch).  The
// sweep walks a band's 16 rows in sequence, which on a single frame leaves
// the GPU nearly idle.  Here the row prefixes R of every row are computed in
// parallel (one CTA per image row, row_chunk_scan) into `rowpre`, then one
// thread per (band, plane, column) adds them down the band onto the band's
// carry: the sweep's additions in the sweep's order, so the planes are
// bitwise those of the sweep and results do not depend on how frames are
// batched.
constexpr int kRowPathFrames = 2;

template <class M>
__global__ void __launch_bounds__(kRowThreads) k_moments_rowpre(const FrameDev *__restrict__ frames,
                                                                const int *__restrict__ frame_of) {
  typedef typename MomAcc<M>::T A;
  __shared__ A wtot[kRowThreads / 32][10];
  const int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  const int r = ((int)blockIdx.x - f.band_base) * kBandRows + (int)blockIdx.y;
  if (r >= f.rows) return;  // the whole CTA
  const int cols = f.cols;
  const size_t P = (size_t)f.rows * cols;
  A *Rp = static_cast<A *>(f.rowpre) + (size_t)r * cols;
  A carry[10];
#pragma unroll
  for (int m = 0; m < 10; m++) carry[m] = A(0);
  for (int x0 = 0; x0 < cols; x0 += kChunkPix) {
    unsigned w[kRowPix];
    load_row_raw(f, r, x0 + threadIdx.x * kRowPix, w);
    float d[kRowPix];
#pragma unroll
    for (int k = 0; k < kRowPix; k++) d[k] = depth_from_raw(f, w[k]);
    row_chunk_scan<M>(f, r, x0, d, carry, wtot, [&](int, int c, const A *acc) {
      if (c < cols) {
#pragma unroll
        for (int m = 0; m < 10; m++) Rp[m * P + c] = acc[m];
      }
    });
  }
}

template <class M>
__global__ void __launch_bounds__(128) k_moments_colsum(const FrameDev *__restrict__ frames,
                                                        const int *__restrict__ frame_of) {
  typedef typename MomAcc<M>::T A;
  const int fi = frame_of[blockIdx.x];
  const FrameDev &f = frames[fi];
  const int cols = f.cols;
  const int q = ((int)blockIdx.x - f.col_base) * 128 + (int)threadIdx.x;  // plane * cols + column
  const int b = blockIdx.y, r0 = b * kBandRows;
  if (q >= 10 * cols || r0 >= f.rows) return;
  const int r1 = min(f.rows, r0 + kBandRows);
  const int m = q / cols, c = q - m * cols;
  const size_t P = (size_t)f.rows * cols;
  A s = static_cast<const A *>(f.band_tot)[(size_t)b * 10 * cols + q];
  const A *Rp = static_cast<const A *>(f.rowpre) + m * P + c;
  A v[kBandRows];
#pragma unroll
  for (int k = 0; k < kBandRows; k++) v[k] = r0 + k < r1 ? Rp[(size_t)(r0 + k) * cols] : A(0);
#pragma unroll
  for (int k = 0; k < kBandRows; k++) {
    if (r0 + k < r1) {
      s = s + v[k];
      M::store(f.moments, P, m, (size_t)(r0 + k) * cols + c, (double)s);
    }
  }
}

bool moments_row_path(int nframes) { return nframes <= kRowPathFrames; }

// The dynamic shared-memory opt-in of a kernel holds for the device that was
// current when it was set: it is set once per device and instantiation
// (std::call_once, so that host threads building at the same time wait for
// it rather than race).
template <class M>
static void configure_bands() {
  constexpr int kMaxDevices = 64;
  static std::once_flag once[kMaxDevices];
  int dev = 0;
  cudaGetDevice(&dev);
  auto set = [] {
    cudaFuncSetAttribute(k_moments_band_totals<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, band_smem_bytes<M>());
    cudaFuncSetAttribute(k_moments_band_sweep<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, band_smem_bytes<M>());
  };
  if (dev >= 0 && dev < kMaxDevices)
    std::call_once(once[dev], set);
  else
    set();
}

template <class M>
static void launch_bands(const FrameDev *d_frames, int nframes, int total_bands, int total_carry_ctas, int max_bands,
                         const int *frame_of_band, const int *frame_of_carry, cudaStream_t s, Profiler *prof) {
  configure_bands<M>();
  prof->begin(NICP_K_MOMENTS_BANDS, s);
  k_moments_band_totals<M><<<total_bands, kRowThreads, band_smem_bytes<M>(), s>>>(d_frames, frame_of_band);
  k_moments_band_carry<M><<<total_carry_ctas, 128, 0, s>>>(d_frames, frame_of_carry);
  prof->end(NICP_K_MOMENTS_BANDS, s, 2);
  prof->begin(NICP_K_MOMENTS_SWEEP, s);
  if (moments_row_path(nframes) && max_bands <= 65535) {  // (grid y of the column sums)
    k_moments_rowpre<M><<<dim3(total_bands, kBandRows), kRowThreads, 0, s>>>(d_frames, frame_of_band);
    k_moments_colsum<M><<<dim3(total_carry_ctas, max_bands), 128, 0, s>>>(d_frames, frame_of_carry);
    prof->end(NICP_K_MOMENTS_SWEEP, s, 2);
  } else {
    k_moments_band_sweep<M><<<dim3(max_bands, nframes), kRowThreads, band_smem_bytes<M>(), s>>>(d_frames, nframes);
    prof->end(NICP_K_MOMENTS_SWEEP, s);
  }
}

int moment_band_rows() { return kBandRows; }
size_t moment_acc_bytes(int precision) { return precision == NICP_MOMENTS_F32 ? 4 : 8; }

void launch_moments(int precision, const FrameDev *d_frames, int nframes, int total_bands, int total_carry_ctas,
                    int max_bands, const int *frame_of_band, const int *frame_of_carry, cudaStream_t s,
                    Profiler *prof) {
  if (precision == NICP_MOMENTS_F32)
    launch_bands<MomF32>(d_frames, nframes, total_bands, total_carry_ctas, max_bands, frame_of_band, frame_of_carry, s,
                         prof);
  else if (precision == NICP_MOMENTS_TWOFLOAT)
    launch_bands<MomTwoFloat>(d_frames, nframes, total_bands, total_carry_ctas, max_bands, frame_of_band,
                              frame_of_carry, s, prof);
  else
    launch_bands<MomF64>(d_frames, nframes, total_bands, total_carry_ctas, max_bands, frame_of_band, frame_of_carry, s,
                         prof);
}

template <class M>
static int sweep_occupancy() {
  configure_bands<M>();
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_moments_band_sweep<M>, kRowThreads, band_smem_bytes<M>()) !=
      cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  return n > 0 ? n : 1;
}

int moment_sweep_ctas_per_sm(int precision) {
  if (precision == NICP_MOMENTS_F32) return sweep_occupancy<MomF32>();
  if (precision == NICP_MOMENTS_TWOFLOAT) return sweep_occupancy<MomTwoFloat>();
  return sweep_occupancy<MomF64>();
}

// Stats launch shapes: (threads per CTA, CTAs per SM of the register budget).
#ifdef NICP_STATS_WIDE_DEFAULT
static const int kStatsShape[kStatsShapes][2] = {{256, 2}, {128, 6}, {64, 12}, {256, 3}};
#else
static const int kStatsShape[kStatsShapes][2] = {{256, 3}, {128, 6}, {64, 12}, {256, 2}};
#endif

int stats_shape_threads(int shape) { return kStatsShape[shape][0]; }
int stats_shape_min_ctas(int shape) { return kStatsShape[shape][1]; }

template <class M, bool kLean>
static void stats_launch(int shape, dim3 g, const FrameDev *d_frames, int nframes, cudaStream_t s) {
  const int threads = kStatsShape[shape][0], ctas = kStatsShape[shape][1];
  if (threads == 128) k_stats<M, 128, 6, kLean><<<g, 128, 0, s>>>(d_frames, nframes);
  else if (threads == 64) k_stats<M, 64, 12, kLean><<<g, 64, 0, s>>>(d_frames, nframes);
  else if (ctas == 2) k_stats<M, 256, 2, kLean><<<g, 256, 0, s>>>(d_frames, nframes);
  else k_stats<M, 256, 3, kLean><<<g, 256, 0, s>>>(d_frames, nframes);
}

template <class M>
static void stats_launch(int shape, bool lean, dim3 g, const FrameDev *d_frames, int nframes, cudaStream_t s) {
  if (lean) stats_launch<M, true>(shape, g, d_frames, nframes, s);
  else stats_launch<M, false>(shape, g, d_frames, nframes, s);
}

void launch_stats(int precision, const FrameDev *d_frames, int nframes, int max_pixels, int shape, bool lean,
                  cudaStream_t s, Profiler *prof) {
  if (shape < 0 || shape >= kStatsShapes) shape = 0;
  prof->begin(NICP_K_STATS, s);
  const int threads = kStatsShape[shape][0];
  const dim3 g((max_pixels + threads - 1) / threads, nframes);
  if (precision == NICP_MOMENTS_F32) stats_launch<MomF32>(shape, lean, g, d_frames, nframes, s);
  else if (precision == NICP_MOMENTS_TWOFLOAT) stats_launch<MomTwoFloat>(shape, lean, g, d_frames, nframes, s);
  else stats_launch<MomF64>(shape, lean, g, d_frames, nframes, s);
  prof->end(NICP_K_STATS, s);
}

// Zeroes the frames' counts of points with a normal (k_stats adds to them),
// so that the stats kernel can run again with another launch shape.
__global__ void k_reset_normal_counts(const FrameDev *__restrict__ frames, int nframes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nframes) frames[i].count[1] = 0;
}

void launch_reset_normal_counts(const FrameDev *d_frames, int nframes, cudaStream_t s) {
  if (nframes > 0) k_reset_normal_counts<<<(nframes + 127) / 128, 128, 0, s>>>(d_frames, nframes);
}

// The information matrices of a cloud whose Omega is implicit (built with
// the converter's structure): per point with a normal n and class code c in
// its w, Omega = d1 I + (d0 - d1) n n^T with (d0, d1) of c's flat / non-flat
// point and normal calculators (omd: point flat, point non-flat, normal flat,
// normal non-flat), evaluated in double and rounded once; zero for a point
// without a normal (as the stats kernel leaves it).
__global__ void k_materialize_omg(const float4 *__restrict__ pts, const float4 *__restrict__ nrm, float4 *omg,
                                  const int *__restrict__ count, int capacity, OmegaParams op) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= capacity || i >= *count) return;
  float om[12];
#pragma unroll
  for (int k = 0; k < 12; k++) om[k] = 0.0f;
  const float w = pts[i].w;
  if (point_has_normal(w)) {
    const int cls = (int)w - 1;
    const float *dp = op.omd + 2 * (cls & 1), *dn = op.omd + 4 + 2 * ((cls >> 1) & 1);
    const float4 n = nrm[i];
    const double u[3] = {(double)n.x, (double)n.y, (double)n.z};
    const int ii[6] = {0, 0, 0, 1, 1, 2}, jj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int e = 0; e < 6; e++) {
      const int a = ii[e], b = jj[e];
      const double uu = u[a] * u[b];
      om[e] = (float)((a == b ? (double)dp[1] : 0.0) + ((double)dp[0] - (double)dp[1]) * uu);
      om[6 + e] = (float)((a == b ? (double)dn[1] : 0.0) + ((double)dn[0] - (double)dn[1]) * uu);
    }
  }
  float4 *o = omg + 3 * (size_t)i;
  o[0] = make_float4(om[0], om[1], om[2], om[3]);
  o[1] = make_float4(om[4], om[5], om[6], om[7]);
  o[2] = make_float4(om[8], om[9], om[10], om[11]);
}

void launch_materialize_omg(const float4 *pts, const float4 *nrm, float4 *omg, const int *count, int capacity,
                            const float omd[8], cudaStream_t s) {
  OmegaParams op;
  for (int k = 0; k < 8; k++) op.omd[k] = omd[k];
  const int blocks = (capacity + 255) / 256;
  if (blocks > 0) k_materialize_omg<<<blocks, 256, 0, s>>>(pts, nrm, omg, count, capacity, op);
}

void launch_cloud_transform(float4 *pts, float4 *nrm, float4 *omg, float *eig, float4 *gauss, const int *count,
                            int capacity, const float *d_m12, cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_TRANSFORM, s);
  int blocks = (capacity + 255) / 256;
  if (blocks > 0) k_cloud_transform<<<blocks, 256, 0, s>>>(pts, nrm, omg, eig, gauss, count, capacity, d_m12);
  prof->end(NICP_K_TRANSFORM, s);
}

size_t moment_bytes(int precision) {
  if (precision == NICP_MOMENTS_F32) return 4;
  return 8;  // double or two-float
}

}  // namespace nicp
