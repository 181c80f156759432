// k_align.cu -- projective ICP kernels (AlignerProjective::align and its parts).
//
//   k_zbuffer    PinholePointProjector::project (pinholepointprojector.cpp:33-66):
//                one thread per point, 64-bit atomicMin of (depth key << 32 | index)
//                into a per-pair z-buffer.  The serial reference keeps the first
//                point with the strictly smallest depth, i.e. the minimum of
//                (depth, index) -- exactly what the packed minimum keeps.
//   k_resolve    z-buffer -> index image (+ depth image), resetting the z-buffer.
//   k_corr_lin   fused CorrespondenceFinderProjective::_computeSingle
//                (correspondencefinderprojective.cpp:23-115) and Linearizer::update
//                (linearizer.cpp:21-134): per pixel, gate the pair, and if accepted
//                add its 21 H + 6 b + chi2 + inlier terms.  Per-thread sums in FP32
//                over 4 pixels, then FP64: warp butterfly reduce-scatter, shared
//                memory, one partial per CTA tile (fixed tile -> partial mapping).
//   k_corr_count / k_corr_write
//                the same gates with ordered compaction into the reference's
//                row-major correspondence list (parity / list mode).
//   k_lin_list   Linearizer::update over a correspondence list (with the
//                reference's K % T drop when T > 1).
//   k_solve      per pair: fixed-order FP64 sum of the tile partials, H + lambda I,
//                6x6 LDL^T, pose update and renormalisation (alignerprojective.cpp:
//                72-100), early exit, and the float matrices of the next iteration.
#include <cuda_runtime.h>

#include <type_traits>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"

namespace nicp {

// The pair whose pixel tiles hold tile `key` (largest i with tile_base <= key).
__device__ __forceinline__ int find_pair(const PairDev *pairs, int n, int key) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    int b = pairs[mid].tile_base;
    if (b <= key) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------ z-buffer
// mode 0: project the current cloud with pair.KRt_cur-equivalent `explicit_KRt`
// (one matrix for all pairs, host-computed); mode 1: the reference cloud with
// the pair state's KRt.
// A CTA covers kPointsPerCta points with kPointsPerCta / PPT threads, PPT
// independent points per thread (their loads and atomics overlap); the
// result does not depend on PPT (atomicMin is order-free).  Grid: (point
// tile, pair) -- the pair comes from blockIdx.y, with no search, so a CTA's
// first loads are its pose and its points.
template <int PPT>
__global__ void __launch_bounds__(kPointsPerCta / PPT)
    k_zbuffer(const PairDev *__restrict__ pairs, int npairs, int mode, const float *__restrict__ explicit_KRt,
              int pair0) {
  constexpr int kThreads = kPointsPerCta / PPT;
  const int pi = pair0 + (int)blockIdx.y;
  if (pi >= npairs) return;
  const PairDev &pd = pairs[pi];
  const PairState *st = pd.state;
  if (mode == 1 && st->done) return;
  const int i0 = blockIdx.x * kPointsPerCta + threadIdx.x;
  const float4 *pts = mode ? pd.ref_pts : pd.cur_pts;
  const int n = mode ? *pd.ref_count : *pd.cur_count;
  if (i0 >= n) return;
  float K[12];
  const float *src = mode ? st->KRt : explicit_KRt + 12 * pi;
#pragma unroll
  for (int k = 0; k < 12; k++) K[k] = src[k];
  float4 p[PPT];
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    int i = i0 + k * kThreads;
    p[k] = (i < n) ? pts[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
#pragma unroll
  for (int k = 0; k < PPT; k++) {
    int i = i0 + k * kThreads;
    int x, y;
    float d;
    if (i >= n || !project_pixel(K, p[k], pd.rows, pd.cols, pd.min_d, pd.max_d, x, y, d)) continue;
    unsigned long long key =
        ((unsigned long long)float_key(d) << 32) | ((unsigned)i << 1) | (point_has_normal(p[k].w) ? 0u : 1u);
    atomicMin(pd.zbuf + (size_t)y * pd.cols + x, key);
  }
}

// Decodes a z-buffer word: the point index, or -1 when empty -- or, with
// drop_no_normal, when the point has no normal (such a pixel can never pass
// the correspondence gates unless they are demoted to GICP).
__device__ __forceinline__ int zbuf_index(unsigned long long z, bool drop_no_normal) {
  if (z == ~0ull) return -1;
  unsigned lo = (unsigned)(z & 0xffffffffull);
  if (drop_no_normal && (lo & 1u)) return -1;
  return (int)(lo >> 1);
}

// z-buffer -> int index image (and optional depth image, FLT_MAX where empty);
// the z-buffer is left all ones for its next use.  Thread t handles pixels
// t, t + 256, ... of its tile: every warp access is one contiguous run.
// Grid (pixel tile, pair): the pair is pair0 + blockIdx.y, no search.
__global__ void k_resolve(const PairDev *__restrict__ pairs, int npairs, int to_ref, float *depth_out,
                          int drop_no_normal, int pair0) {
  const int pi = pair0 + (int)blockIdx.y;
  if (pi >= npairs) return;
  const PairDev &pd = pairs[pi];
  const int P = pd.rows * pd.cols;
  const int pix0 = blockIdx.x * kCorrTilePixels + threadIdx.x;
  int32_t *dst = to_ref ? pd.ref_index : pd.cur_index;
  unsigned long long z[kCorrTilePixels / kCorrThreads];
#pragma unroll
  for (int k = 0; k < kCorrTilePixels / kCorrThreads; k++) {
    const int p = pix0 + k * kCorrThreads;
    z[k] = p < P ? pd.zbuf[p] : ~0ull;
  }
#pragma unroll
  for (int k = 0; k < kCorrTilePixels / kCorrThreads; k++) {
    const int p = pix0 + k * kCorrThreads;
    if (p < P) {
      pd.zbuf[p] = ~0ull;
      dst[p] = zbuf_index(z[k], drop_no_normal != 0);
      if (depth_out) depth_out[p] = (z[k] == ~0ull) ? 3.402823466e+38f : key_float((uint32_t)(z[k] >> 32));
    }
  }
}

// ------------------------------------------------------------ gates + terms
struct Acc {
  // 0..5 Htt lower (00 10 11 20 21 22), 6..14 Htr row-major, 15..20 Hrr lower,
  // 21..23 bt, 24..26 br, 27 chi2, 28 inliers, 29 candidates, 30 accepted.
  // The rotational Jacobian block is skew(2 p) (linearizer.cpp:59-100); the
  // per-pixel terms use skew(p), so Htr and br hold half and Hrr a quarter of
  // their values, and the reductions scale the FP64 tile sums by 2 and 4
  // (exact: powers of two).  The three counts (28 inliers, 29 candidates,
  // 30 accepted) share one integer, 10 bits each (a thread adds at most 8
  // pixels or 4 list entries to a tile partial).
  float v[28];
  unsigned cnt;
  static constexpr unsigned kInlier = 1u, kCandidate = 1u << 10, kAccepted = 1u << 20;
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int k = 0; k < 28; k++) v[k] = 0.0f;
    cnt = 0u;
  }
  // element k of the partial (0..30) as a float
  __device__ __forceinline__ float get(int k) const {
    return k < 28 ? v[k] : (float)((cnt >> (10 * (k - 28))) & 1023u);
  }
};
// Power-of-two factor of each Acc element (see Acc).
__device__ __forceinline__ double acc_scale(int k) {
  return (k >= 15 && k <= 20) ? 4.0 : ((k >= 6 && k <= 14) || (k >= 24 && k <= 26)) ? 2.0 : 1.0;
}

// The gate's arithmetic: dot3x and xform_normal without the reference's
// zero w terms ("+ 0 * 0" of the 4-vector dot products, "+ A3 * 0" of the
// normal transform), which change at most the sign of a zero -- no
// comparison of the gates can tell, so the decisions stay bitwise the
// reference's -- and xform_point with its "+ A3 * 1" written as "+ A3".
__device__ __forceinline__ float dot3g(float ax, float ay, float az, float bx, float by, float bz) {
  float s = fm(ax, bx);
  s = fa(s, fm(ay, by));
  return fa(s, fm(az, bz));
}
// The reference's "normal.squaredNorm() == 0" (correspondencefinderprojective.cpp:69,
// the normal's w is 0): a sum of non-negative float squares is zero exactly
// when every square rounds to zero, and x * x rounds to zero (round to
// nearest even, subnormals kept) exactly when |x| <= 2^-75, since 2^-150 is
// the tie between 0 and the smallest subnormal 2^-149.  A NaN component
// makes the squared norm NaN, not zero, and every comparison below false.
// Three compares instead of three products and two sums.
__device__ __forceinline__ bool normal_is_zero(float x, float y, float z) {
  constexpr float t = 0x1p-75f;
  return fabsf(x) <= t && fabsf(y) <= t && fabsf(z) <= t;
}
__device__ __forceinline__ float rowg(const float *A, float x, float y, float z) {
  float s = fm(A[0], x);
  s = fa(s, fm(A[1], y));
  return fa(s, fm(A[2], z));
}
// rowg with its first two products in one packed multiply (sm_100 FMUL2;
// each half is rounded as __fmul_rn rounds it, so the sum is bitwise rowg's):
// ((A0 x + A1 y) + A2 z).  A is read element by element (it may be a
// thread's register array as well as a shared row).
__device__ __forceinline__ float rowg2(const float *A, float2 xy, float z) {
  const float2 m = __fmul2_rn(make_float2(A[0], A[1]), xy);
  return fa(fa(m.x, m.y), fm(A[2], z));
}
__device__ __forceinline__ float3 xform_point_g2(const float *A, float4 p) {
  const float2 xy = make_float2(p.x, p.y);
  return make_float3(fa(rowg2(A, xy, p.z), A[3]), fa(rowg2(A + 4, xy, p.z), A[7]), fa(rowg2(A + 8, xy, p.z), A[11]));
}
__device__ __forceinline__ float3 xform_normal_g2(const float *A, float4 n) {
  const float2 xy = make_float2(n.x, n.y);
  return make_float3(rowg2(A, xy, n.z), rowg2(A + 4, xy, n.z), rowg2(A + 8, xy, n.z));
}
__device__ __forceinline__ float3 xform_normal_g(const float *A, float4 n) {
  return make_float3(rowg(A, n.x, n.y, n.z), rowg(A + 4, n.x, n.y, n.z), rowg(A + 8, n.x, n.y, n.z));
}
// row4 with w = 1: "+ A3 * 1" adds A3 exactly
__device__ __forceinline__ float3 xform_point_g(const float *A, float4 p) {
  return make_float3(fa(rowg(A, p.x, p.y, p.z), A[3]), fa(rowg(A + 4, p.x, p.y, p.z), A[7]),
                     fa(rowg(A + 8, p.x, p.y, p.z), A[11]));
}

// correspondencefinderprojective.cpp:59-101.  T12: rows 0..2 of the gating
// transform (the aligner passes _T.inverse()).
// The transformed reference point and normal are returned in rp / rn (rn
// only when the normal gates run, i.e. not demoted).
__device__ __forceinline__ bool gate_t(const CorrParams &cp, const float *T12, float4 rp0, float4 rn0, float4 cpt,
                                       float4 cn, float3 &rp, float3 &rn) {
  if (!cp.demoted) {
    if (normal_is_zero(cn.x, cn.y, cn.z)) return false;
    if (normal_is_zero(rn0.x, rn0.y, rn0.z)) return false;
  }
  rp = xform_point_g2(T12, rp0);
  float dx = fsb(cpt.x, rp.x), dy = fsb(cpt.y, rp.y), dz = fsb(cpt.z, rp.z);
  if (dot3g(dx, dy, dz, dx, dy, dz) > cp.sq_thr) return false;
  if (!cp.demoted) {
    rn = xform_normal_g2(T12, rn0);
    if (dot3g(cn.x, cn.y, cn.z, rn.x, rn.y, rn.z) < cp.cos_thr) return false;
    float kr = rn0.w, kc = cn.w;
    if (kr < cp.flat_thr) kr = cp.flat_thr;
    if (kc < cp.flat_thr) kc = cp.flat_thr;
    // equal curvatures (in particular both below the flat threshold) give a
    // ratio of exactly 1: skip the division
    float ratio =
        (kr == kc) ? 1.0f : __double2float_rn(__ddiv_rn(__dadd_rn((double)kr, 1e-5), __dadd_rn((double)kc, 1e-5)));
    if (ratio < cp.min_ratio || ratio > cp.max_ratio) return false;
  }
  return true;
}

__device__ __forceinline__ bool gate(const CorrParams &cp, const float *T12, float4 rp0, float4 rn0, float4 cpt,
                                     float4 cn) {
  float3 rp, rn;
  return gate_t(cp, T12, rp0, rn0, cpt, cn, rp, rn);
}

// linearizer.cpp:59-100 for one correspondence, FP32.
__device__ __forceinline__ void lin_terms(const LinParams &lp, const float *T12, float4 rp0, float4 rn0, float4 cpt,
                                         float4 cn, float4 o0, float4 o1, float4 o2, Acc &acc) {
  float3 rp = xform_point_g(T12, rp0);
  float3 rn = xform_normal_g(T12, rn0);
  // symmetric 3x3 as (00 01 02 11 12 22)
  float Op[6] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y};
  float On[6] = {o1.z, o1.w, o2.x, o2.y, o2.z, o2.w};
#pragma unroll
  for (int k = 0; k < 6; k++) On[k] = lp.scale * On[k];
  if (lp.z_scaling) {
    float f = 1.0f / fabsf(cpt.z);
#pragma unroll
    for (int k = 0; k < 6; k++) { Op[k] *= f; On[k] *= f; }
  }
  if (lp.demoted) {
#pragma unroll
    for (int k = 0; k < 6; k++) On[k] = 0.0f;
  }
  float pe[3] = {rp.x - cpt.x, rp.y - cpt.y, rp.z - cpt.z};
  float ne[3] = {rn.x - cn.x, rn.y - cn.y, rn.z - cn.z};
  float ep[3] = {Op[0] * pe[0] + Op[1] * pe[1] + Op[2] * pe[2], Op[1] * pe[0] + Op[3] * pe[1] + Op[4] * pe[2],
                 Op[2] * pe[0] + Op[4] * pe[1] + Op[5] * pe[2]};
  float en[3] = {On[0] * ne[0] + On[1] * ne[1] + On[2] * ne[2], On[1] * ne[0] + On[3] * ne[1] + On[4] * ne[2],
                 On[2] * ne[0] + On[4] * ne[1] + On[5] * ne[2]};
  float le = (pe[0] * ep[0] + pe[1] * ep[1] + pe[2] * ep[2]) + (ne[0] * en[0] + ne[1] * en[1] + ne[2] * en[2]);
  float ks = 1.0f;
  if (le > lp.max_chi2) {
    if (lp.robust) ks = lp.max_chi2 / le;
    else return;
  }
  acc.v[27] += ks * le;
  acc.cnt += Acc::kInlier;
  // skew(v) = [[0, c, -b], [-c, 0, a], [b, -a, 0]], (a, b, c) = v (the
  // Jacobian's factor 2 is applied to the tile sums, see Acc)
  float a = rp.x, b = rp.y, c = rp.z;
  float an = rn.x, bn = rn.y, cn2 = rn.z;
  // Htt += Op * ks
  acc.v[0] += Op[0] * ks; acc.v[1] += Op[1] * ks; acc.v[2] += Op[3] * ks;
  acc.v[3] += Op[2] * ks; acc.v[4] += Op[4] * ks; acc.v[5] += Op[5] * ks;
  // Htr += (Op Sp) ks: (Op S)_i0 = -c Op_i1 + b Op_i2; _i1 = c Op_i0 - a Op_i2; _i2 = -b Op_i0 + a Op_i1
  const float Om[3][3] = {{Op[0], Op[1], Op[2]}, {Op[1], Op[3], Op[4]}, {Op[2], Op[4], Op[5]}};
#pragma unroll
  for (int i = 0; i < 3; i++) {
    acc.v[6 + i * 3 + 0] += (-c * Om[i][1] + b * Om[i][2]) * ks;
    acc.v[6 + i * 3 + 1] += (c * Om[i][0] - a * Om[i][2]) * ks;
    acc.v[6 + i * 3 + 2] += (-b * Om[i][0] + a * Om[i][1]) * ks;
  }
  // Hrr += (S^T O S) for the point and the normal terms
  const float Nm[3][3] = {{On[0], On[1], On[2]}, {On[1], On[3], On[4]}, {On[2], On[4], On[5]}};
  float Ap[3][3], An[3][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    Ap[0][j] = -c * Om[1][j] + b * Om[2][j];
    Ap[1][j] = c * Om[0][j] - a * Om[2][j];
    Ap[2][j] = -b * Om[0][j] + a * Om[1][j];
    An[0][j] = -cn2 * Nm[1][j] + bn * Nm[2][j];
    An[1][j] = cn2 * Nm[0][j] - an * Nm[2][j];
    An[2][j] = -bn * Nm[0][j] + an * Nm[1][j];
  }
  float R[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    R[i][0] = (-c * Ap[i][1] + b * Ap[i][2]) + (-cn2 * An[i][1] + bn * An[i][2]);
    R[i][1] = (c * Ap[i][0] - a * Ap[i][2]) + (cn2 * An[i][0] - an * An[i][2]);
    R[i][2] = (-b * Ap[i][0] + a * Ap[i][1]) + (-bn * An[i][0] + an * An[i][1]);
  }
  acc.v[15] += R[0][0] * ks; acc.v[16] += R[1][0] * ks; acc.v[17] += R[1][1] * ks;
  acc.v[18] += R[2][0] * ks; acc.v[19] += R[2][1] * ks; acc.v[20] += R[2][2] * ks;
  // bt += ks ep; br += ks (Sp^T ep + Sn^T en), S^T e = v x e
  acc.v[21] += ks * ep[0]; acc.v[22] += ks * ep[1]; acc.v[23] += ks * ep[2];
  float u0 = b * ep[2] - c * ep[1], u1 = c * ep[0] - a * ep[2], u2 = a * ep[1] - b * ep[0];
  float w0 = bn * en[2] - cn2 * en[1], w1 = cn2 * en[0] - an * en[2], w2 = an * en[1] - bn * en[0];
  acc.v[24] += ks * (u0 + w0); acc.v[25] += ks * (u1 + w1); acc.v[26] += ks * (u2 + w2);
}

// lin_terms for a current point whose information matrices have the
// converter's structure Omega = d1 I + (d0 - d1) u u^T, u its normal (the
// smallest-eigenvalue eigenvector; Omega = U diag(d0, d1, d1) U^T,
// informationmatrixcalculator.cpp:9-57).  With S = skew(v) (S x = x cross v,
// v the moved point; the Jacobian's factor 2 is applied to the tile sums, see
// Acc) and w = S^T u:  Omega e = a e + b (u.e) u,  Omega S = a S + b u w^T,
// S^T Omega S = a (|v|^2 I - v v^T) + b w w^T.  The class code in the
// point's w selects (d0, d1); omd holds them for the four classes.
// rp, rn: the reference point and normal already moved by the linearizer's
// transform.  Every accumulator update is one fused chain of FMAs; the
// robust kernel's weight ks (linearizer.cpp:83-89) is folded into the
// weights and residual terms only for the pixels beyond the chi2 bound.
__device__ __forceinline__ void lin_terms_structured_xf(const LinParams &lp, const float *omd, float3 rp, float3 rn,
                                                       float4 cpt, float4 cn, Acc &acc) {
  float alp = 0.0f, bep = 0.0f, aln = 0.0f, ben = 0.0f;
  if (point_has_normal(cpt.w)) {
    const int cls = (int)cpt.w - 1;
    const float *dp = omd + 2 * (cls & 1), *dn = omd + 4 + 2 * ((cls >> 1) & 1);
    alp = dp[1];
    bep = dp[0] - dp[1];
    aln = lp.scale * dn[1];
    ben = lp.scale * dn[0] - aln;
  }
  if (lp.z_scaling) {
    float f = 1.0f / fabsf(cpt.z);
    alp *= f; bep *= f; aln *= f; ben *= f;
  }
  if (lp.demoted) { aln = 0.0f; ben = 0.0f; }
  const float ux = cn.x, uy = cn.y, uz = cn.z;
  float pe0 = rp.x - cpt.x, pe1 = rp.y - cpt.y, pe2 = rp.z - cpt.z;
  float ne0 = rn.x - cn.x, ne1 = rn.y - cn.y, ne2 = rn.z - cn.z;
  const float bu = bep * fmaf(uz, pe2, fmaf(uy, pe1, ux * pe0));
  const float bv = ben * fmaf(uz, ne2, fmaf(uy, ne1, ux * ne0));
  float ep0 = fmaf(bu, ux, alp * pe0), ep1 = fmaf(bu, uy, alp * pe1), ep2 = fmaf(bu, uz, alp * pe2);
  float en0 = fmaf(bv, ux, aln * ne0), en1 = fmaf(bv, uy, aln * ne1), en2 = fmaf(bv, uz, aln * ne2);
  float le = fmaf(ne2, en2, fmaf(ne1, en1, fmaf(ne0, en0, fmaf(pe2, ep2, fmaf(pe1, ep1, pe0 * ep0)))));
  if (le > lp.max_chi2) {
    if (!lp.robust) return;
    const float ks = lp.max_chi2 / le;
    le *= ks;
    alp *= ks; bep *= ks; aln *= ks; ben *= ks;
    ep0 *= ks; ep1 *= ks; ep2 *= ks;
    en0 *= ks; en1 *= ks; en2 *= ks;
  }
  acc.v[27] += le;
  acc.cnt += Acc::kInlier;
  const float a = rp.x, b = rp.y, c = rp.z;
  const float an = rn.x, bn = rn.y, cn2 = rn.z;
  // Htt += Omega_p
  const float t0 = bep * ux, t1 = bep * uy, t2 = bep * uz;
  acc.v[0] = fmaf(t0, ux, acc.v[0] + alp);
  acc.v[1] = fmaf(t0, uy, acc.v[1]);
  acc.v[2] = fmaf(t1, uy, acc.v[2] + alp);
  acc.v[3] = fmaf(t0, uz, acc.v[3]);
  acc.v[4] = fmaf(t1, uz, acc.v[4]);
  acc.v[5] = fmaf(t2, uz, acc.v[5] + alp);
  // Htr += Omega_p S = alp S + bep u wp^T, S = [[0, c, -b], [-c, 0, a], [b, -a, 0]]
  const float wp0 = fmaf(b, uz, -c * uy), wp1 = fmaf(c, ux, -a * uz), wp2 = fmaf(a, uy, -b * ux);
  const float wn0 = fmaf(bn, uz, -cn2 * uy), wn1 = fmaf(cn2, ux, -an * uz), wn2 = fmaf(an, uy, -bn * ux);
  acc.v[6] = fmaf(t0, wp0, acc.v[6]);
  acc.v[7] = fmaf(t0, wp1, fmaf(alp, c, acc.v[7]));
  acc.v[8] = fmaf(t0, wp2, fmaf(-alp, b, acc.v[8]));
  acc.v[9] = fmaf(t1, wp0, fmaf(-alp, c, acc.v[9]));
  acc.v[10] = fmaf(t1, wp1, acc.v[10]);
  acc.v[11] = fmaf(t1, wp2, fmaf(alp, a, acc.v[11]));
  acc.v[12] = fmaf(t2, wp0, fmaf(alp, b, acc.v[12]));
  acc.v[13] = fmaf(t2, wp1, fmaf(-alp, a, acc.v[13]));
  acc.v[14] = fmaf(t2, wp2, acc.v[14]);
  // Hrr += S^T Omega_p S + Sn^T Omega_n Sn
  //      = alp (|v|^2 I - v v^T) + aln (|vn|^2 I - vn vn^T) + bep wp wp^T + ben wn wn^T
  const float qa = alp * a, qb = alp * b, qc = alp * c;
  const float qan = aln * an, qbn = aln * bn, qcn = aln * cn2;
  const float pw0 = bep * wp0, pw1 = bep * wp1, pw2 = bep * wp2;
  const float nw0 = ben * wn0, nw1 = ben * wn1, nw2 = ben * wn2;
  acc.v[15] = fmaf(nw0, wn0, fmaf(pw0, wp0, fmaf(qcn, cn2, fmaf(qbn, bn, fmaf(qc, c, fmaf(qb, b, acc.v[15]))))));
  acc.v[16] = fmaf(nw1, wn0, fmaf(pw1, wp0, fmaf(-qbn, an, fmaf(-qb, a, acc.v[16]))));
  acc.v[17] = fmaf(nw1, wn1, fmaf(pw1, wp1, fmaf(qcn, cn2, fmaf(qan, an, fmaf(qc, c, fmaf(qa, a, acc.v[17]))))));
  acc.v[18] = fmaf(nw2, wn0, fmaf(pw2, wp0, fmaf(-qcn, an, fmaf(-qc, a, acc.v[18]))));
  acc.v[19] = fmaf(nw2, wn1, fmaf(pw2, wp1, fmaf(-qcn, bn, fmaf(-qc, b, acc.v[19]))));
  acc.v[20] = fmaf(nw2, wn2, fmaf(pw2, wp2, fmaf(qbn, bn, fmaf(qan, an, fmaf(qb, b, fmaf(qa, a, acc.v[20]))))));
  // bt += ep; br += Sp^T ep + Sn^T en (S^T e = v x e)
  acc.v[21] += ep0; acc.v[22] += ep1; acc.v[23] += ep2;
  acc.v[24] = fmaf(bn, en2, fmaf(-cn2, en1, fmaf(b, ep2, fmaf(-c, ep1, acc.v[24]))));
  acc.v[25] = fmaf(cn2, en0, fmaf(-an, en2, fmaf(c, ep0, fmaf(-a, ep2, acc.v[25]))));
  acc.v[26] = fmaf(an, en1, fmaf(-bn, en0, fmaf(a, ep1, fmaf(-b, ep0, acc.v[26]))));
}

__device__ __forceinline__ void lin_terms_structured(const LinParams &lp, const float *T12, const float *omd,
                                                    float4 rp0, float4 rn0, float4 cpt, float4 cn, Acc &acc) {
  lin_terms_structured_xf(lp, omd, xform_point_g(T12, rp0), xform_normal_g(T12, rn0), cpt, cn, acc);
}

// Reduces every thread's Acc to one FP64 partial of the CTA (fixed order).
// (A pairwise FP32 tree inside the warp measured 3 % faster but moved an
// ill-conditioned pose -- a frame against a subscene rendered from a merged
// scene -- from 1e-5 to 2e-5 rad of the FP64 oracle: the warp sums stay FP64.)
template <int kThreads>
__device__ __forceinline__ void block_reduce_store(const Acc &acc, double *out) {
  __shared__ double wsum[kThreads / 32][32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double v[32];
#pragma unroll
  for (int k = 0; k < 31; k++) v[k] = (double)acc.get(k);
  v[31] = 0.0;
  // butterfly reduce-scatter: lane L ends with the warp total of element L
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    bool upper = (lane & off) != 0;
#pragma unroll
    for (int j = 0; j < off; j++) {
      double send = upper ? v[j] : v[j + off];
      double keep = upper ? v[j + off] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  wsum[wid][lane] = v[0];
  __syncthreads();
  if (wid == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++) s += wsum[w][lane];
    out[lane] = s * acc_scale(lane);
  }
}

// ---- fused correspondence + linearizer: persistent, cp.async-pipelined.
// A pair image is cut into tiles of kCorrTilePixels; every tile yields one
// FP64 partial, so results do not depend on the grid or the batch.  A CTA
// walks its tiles (blockIdx.x, +gridDim.x, ...) in sub-tiles of 256 pixels
// (kFusedPX per thread, at slots t and t + kFusedThreads, so that every
// access of one slot row is coalesced; the per-sub-tile bookkeeping and the
// per-tile reduction are shared by a thread's pixels).  For each pixel the
// thread reads the two indices, then
// stages the 7 gathered float4 (reference point and normal, current point
// and normal, 3 x Omega) into its own shared-memory slot with cp.async;
// kCorrStages sub-tiles are in flight while the oldest one is gated and
// linearized.  Each thread reads back only what it copied itself, so the
// gathered data needs no barrier.
constexpr int kFusedThreads = 128;
constexpr int kFusedPX = 2;
constexpr int kSubPix = kFusedThreads * kFusedPX;        // pixels per sub-tile
constexpr int kSubsPerTile = kCorrTilePixels / kSubPix;  // 4
constexpr int kCorrStages = 3;  // general Omega: gather, gate + Omega gather, linearize
// The only data threads share are a tile's constants (transforms, Omega
// parameters, pair, skip flags) and the per-tile reduction.  The constants
// live in a ring of kConstSlots tiles and the CTA meets at a barrier once per
// tile, in the iteration that writes the next tile's constants: tile U's are
// written before the barrier of iteration 4U - 1 (4U - 2 with three stages)
// and read in iterations up to 4U + 3, and their slot is rewritten for tile
// U + kConstSlots only after the barrier of iteration 4U + 4 kConstSlots - 5
// (- 6), which every thread reaches after its iteration 4U + 3 when
// kConstSlots >= 3.  The reduction's own barrier orders its shared sums.
constexpr int kConstSlots = 4;
#ifndef NICP_CORR_S_STAGES
#define NICP_CORR_S_STAGES 2      // structured Omega: gather, gate + linearize
#endif

// Structure-of-arrays stage: thread t owns slots t + k kFusedThreads of
// every array, so a warp's accesses to one field are consecutive 16-byte
// words (no bank conflicts).
struct GatherStageS {  // structured Omega: rebuilt from the current normal
  float4 rp[kSubPix], rn[kSubPix], cp[kSubPix], cn[kSubPix];
  int valid[kSubPix];
};
struct GatherStageG : GatherStageS {  // general Omega: gathered for accepted pixels
  float4 o0[kSubPix], o1[kSubPix], o2[kSubPix];
  int ci[kSubPix];
};
#ifndef NICP_CORR_S_CTAS
#define NICP_CORR_S_CTAS 5
#endif
template <bool kStructured>
using GatherStage = typename std::conditional<kStructured, GatherStageS, GatherStageG>::type;

// block_reduce_store for the fused kernel, with the warp's step done
// through shared memory instead of a shuffle butterfly: the warp's 32 x 31
// partial sums are written to the warp's own slots of the stage it has just
// consumed (rp, rn, cp, cn at slots 32w.. and 128 + 32w..: eight runs of
// four 32-float rows), and lane L < 31 then sums row L -- the 32 lanes'
// partials of element L -- in FP64, in a fixed order (each lane starts its
// row at another 16-byte column, so that the eight lanes of a quarter-warp
// read eight different bank groups).  The warps' totals are added in FP64
// as in block_reduce_store.  The barrier inside also orders the row reads
// before the next gathers into these slots.
template <int kThreads, class StageT>
__device__ __forceinline__ void block_reduce_store_staged(const Acc &acc, double *out, StageT &g) {
  __shared__ double wsum[kThreads / 32][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float *base = reinterpret_cast<float *>(&g.rp[0]);
  auto row_of = [&](int k) {  // element k: run k / 4, row k % 4 of the warp's region
    const int run = k >> 2;
    return base + 4 * ((run >> 1) * kSubPix + (run & 1) * kFusedThreads + 32 * wid) + 32 * (k & 3);
  };
  __syncwarp();  // every lane of the warp is done with its slots of this stage
#pragma unroll
  for (int k = 0; k < 31; k++) row_of(k)[lane] = acc.get(k);
  __syncwarp();
  double v = 0.0;
  if (lane < 31) {
    const float4 *r4 = reinterpret_cast<const float4 *>(row_of(lane));
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 x = r4[(q + lane) & 7];
      v += (double)x.x;
      v += (double)x.y;
      v += (double)x.z;
      v += (double)x.w;
    }
  }
  wsum[wid][lane] = v;
  __syncthreads();
  if (wid == 0) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++) s += wsum[w][lane];
    out[lane] = s * acc_scale(lane);
  }
}
template <bool kStructured>
__host__ __device__ constexpr int corr_stages() { return kStructured ? NICP_CORR_S_STAGES : kCorrStages; }
template <bool kStructured>
constexpr int corr_smem() { return corr_stages<kStructured>() * (int)sizeof(GatherStage<kStructured>); }

// 16-byte gather into shared memory through L2 only (.cg): a gathered point
// or normal is read about once per pass, so caching it in L1 only displaces
// the index and descriptor lines the pipeline does reuse (0.97 against 1.02
// ms per launch with .ca).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// flags: bit0 read the reference index from the z-buffer (else ref_index),
// bit1 reset the z-buffer after reading, bit2 keep the resolved reference
// index image, bit3 statistics pass (gate with Tgate_used; ignores `done`).
// kStructured: every pair's current cloud has structured information
// matrices (no Omega gathers, smaller stages).
template <bool kStructured>
__global__ void __launch_bounds__(kFusedThreads, kStructured ? NICP_CORR_S_CTAS : 3)
    k_corr_lin(const PairDev *__restrict__ pairs, int npairs, const int *__restrict__ tile_pair, int total_tiles,
               CorrParams cp, LinParams lp, int flags) {
  extern __shared__ __align__(16) unsigned char corr_smem_raw[];
  using Stage = GatherStage<kStructured>;
  Stage *stages = reinterpret_cast<Stage *>(corr_smem_raw);
  const int t = threadIdx.x;
  // per-tile constants for the two tiles the pipeline can span:
  // [0..11] gating T, [12..23] linearizer T, [24..31] the current cloud's
  // Omega parameters, then pair index, skip flag and structured-Omega flag
  __shared__ float sT[kConstSlots][32];
  __shared__ int sPair[kConstSlots], sSkip[kConstSlots], sStruct[kConstSlots], sSame[kConstSlots];
  const bool stats_pass = flags & 8;
  if ((int)blockIdx.x >= total_tiles) return;
  const int ntiles = (total_tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int nsub = ntiles * kSubsPerTile;
  const bool drop_no_normal = !cp.demoted;
  auto tile_of = [&](int j) { return (int)blockIdx.x + (j / kSubsPerTile) * (int)gridDim.x; };
  auto stage_of = [&](int j) -> Stage & { return stages[j % corr_stages<kStructured>()]; };

  // Tile -> pair lookups, cached per pipeline stage (a stage's tile changes
  // once every kSubsPerTile sub-tiles).
  int lt_tile = -1, lt_pi = 0, gt_tile = -1, gt_pi = 0, gt_ctile = -1, gt_rc = 0, gt_cc = 0;
  bool lt_skip = false, gt_skip = false;
  auto lookup = [&](int tile, int &ctile, int &cpi, bool &cskip) {
    if (tile != ctile) {
      ctile = tile;
      cpi = tile_pair[tile];  // filled once per alignment by k_tile_pairs
      cskip = !stats_pass && pairs[cpi].state->done;
    }
  };

  // Phase I (one iteration ahead, plain loads into registers): the two index
  // words of the thread's pixels of sub-tile j.
  unsigned long long zI[kFusedPX];
  int cI[kFusedPX];
  auto load_indices = [&](int j) {
#pragma unroll
    for (int k = 0; k < kFusedPX; k++) {
      zI[k] = ~0ull;
      cI[k] = -1;
    }
    if (j >= nsub) return;
    int tile = tile_of(j);
    lookup(tile, lt_tile, lt_pi, lt_skip);
    if (lt_skip) return;
    const PairDev &pd = pairs[lt_pi];
    const int P = pd.rows * pd.cols;
    const int p0 = (tile - pd.tile_base) * kCorrTilePixels + (j % kSubsPerTile) * kSubPix + t;
#pragma unroll
    for (int k = 0; k < kFusedPX; k++) {
      const int p = p0 + k * kFusedThreads;
      if (p < P) {
        if (flags & 1) zI[k] = pd.zbuf[p];
        else cI[k] = pd.ref_index[p];  // stashed in cI until phase G1 reads the current index
        if (flags & 1) cI[k] = pd.cur_index[p];
        else zI[k] = (unsigned long long)(unsigned)pd.cur_index[p];
      }
    }
  };

  // Phase G1 (two sub-tiles ahead): decode the indices, reset the z-buffer,
  // gather points and normals of both clouds.
  auto issue_g1 = [&](int j) {
    Stage &g = stage_of(j);
    int ci[kFusedPX], valid[kFusedPX];
#pragma unroll
    for (int k = 0; k < kFusedPX; k++) {
      ci[k] = -1;
      valid[k] = 0;
    }
    if (j < nsub) {
      int tile = tile_of(j);
      lookup(tile, gt_tile, gt_pi, gt_skip);
      const PairDev &pd = pairs[gt_pi];
      if (!gt_skip) {
        if (gt_ctile != tile) {  // point counts, read once per tile
          gt_ctile = tile;
          gt_rc = *pd.ref_count;
          gt_cc = *pd.cur_count;
        }
        const int P = pd.rows * pd.cols;
        const int p0 = (tile - pd.tile_base) * kCorrTilePixels + (j % kSubsPerTile) * kSubPix + t;
#pragma unroll
        for (int k = 0; k < kFusedPX; k++) {
          const int p = p0 + k * kFusedThreads, sl = t + k * kFusedThreads;
          if (p < P) {
            int ri;
            if (flags & 1) {
              // an empty word (all ones) decodes to -1 with drop_no_normal
              // and to 2^31 - 1 without, which the bounds test below rejects
              const unsigned lo = (unsigned)zI[k];
              ri = (drop_no_normal && (lo & 1u)) ? -1 : (int)(lo >> 1);
              ci[k] = cI[k];
              // evict-first: the word is read again only by the next
              // projection, long after it would have left L2, where it
              // would displace the gathered clouds
              if (flags & 2) __stcs(pd.zbuf + p, ~0ull);
              if (flags & 4) pd.ref_index[p] = ri;
            } else {
              ri = cI[k];
              ci[k] = (int)(unsigned)zI[k];
            }
            valid[k] = (unsigned)ri < (unsigned)gt_rc && (unsigned)ci[k] < (unsigned)gt_cc;
            if (valid[k] && cp.row_limit_threads > 1)
              valid[k] = p / pd.cols < (pd.rows / cp.row_limit_threads) * cp.row_limit_threads;
            if (valid[k]) {
              cp_async16(&g.rp[sl], pd.ref_pts + ri);
              cp_async16(&g.rn[sl], pd.ref_nrm + ri);
              cp_async16(&g.cp[sl], pd.cur_pts + ci[k]);
              cp_async16(&g.cn[sl], pd.cur_nrm + ci[k]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kFusedPX; k++) {
      if constexpr (!kStructured) g.ci[t + k * kFusedThreads] = ci[k];
      g.valid[t + k * kFusedThreads] = valid[k];
    }
    cp_async_commit();
  };

  // Per-tile constants, written when the tile's first sub-tile enters G1.
  auto tile_constants = [&](int j) {
    if (j >= nsub || j % kSubsPerTile) return;
    int e = (j / kSubsPerTile) % kConstSlots;
    lookup(tile_of(j), gt_tile, gt_pi, gt_skip);
    const int pi = gt_pi;
    const PairState *st = pairs[pi].state;
    if (threadIdx.x < 24)
      sT[e][threadIdx.x] = threadIdx.x < 12 ? (stats_pass ? st->Tgate_used : st->Tgate)[threadIdx.x]
                                            : st->Tlin[threadIdx.x - 12];
    else if (threadIdx.x < 32)
      sT[e][threadIdx.x] = pairs[pi].cur_omd[threadIdx.x - 24];
    if (threadIdx.x == 0) {
      sPair[e] = pi;
      sSkip[e] = st->done && !stats_pass;
      sStruct[e] = pairs[pi].cur_structured;
      // gating and linearizer transforms equal (first inner iteration): the
      // linearizer reuses the gate's transformed point and normal
      const float *tg = stats_pass ? st->Tgate_used : st->Tgate;
      int same = 1;
      for (int k = 0; k < 12; k++) same &= (tg[k] == st->Tlin[k]);
      sSame[e] = same;
    }
  };

  // Gate (one sub-tile ahead), then gather Omega only for accepted pairs.
  auto gate_g2 = [&](int j) {
    if (j < nsub) {
      Stage &g = stage_of(j);
      int e = (j / kSubsPerTile) % kConstSlots;
      if constexpr (kStructured) {
        // structured: nothing to gather after the gate; it runs with the
        // linearizer in the main step
        (void)g;
        (void)e;
      } else {
#pragma unroll
        for (int k = 0; k < kFusedPX; k++) {
          const int sl = t + k * kFusedThreads;
          int acc_ok = 0;
          if (g.valid[sl] && !sSkip[e]) {
            acc_ok = gate(cp, sT[e], g.rp[sl], g.rn[sl], g.cp[sl], g.cn[sl]) ? 2 : 1;
            if (acc_ok == 2 && !sStruct[e]) {
              const float4 *o = pairs[sPair[e]].cur_omg + 3 * (size_t)g.ci[sl];
              cp_async16(&g.o0[sl], o);
              cp_async16(&g.o1[sl], o + 1);
              cp_async16(&g.o2[sl], o + 2);
            }
          }
          g.valid[sl] = acc_ok;  // 0 none, 1 candidate rejected, 2 accepted
        }
      }
    }
    cp_async_commit();
  };

  Acc acc;
  acc.zero();
  // Linearizes sub-tile j (its gather -- and, for general Omega, its gate --
  // complete); at a tile's last sub-tile the CTA stores the tile's partial.
  auto consume = [&](int j) {
    const int e = (j / kSubsPerTile) % kConstSlots;
    const int sub = j % kSubsPerTile;
    if (sub == 0) {
      acc.zero();
    }
    if (!sSkip[e]) {
      const Stage &g = stage_of(j);
#pragma unroll
      for (int k = 0; k < kFusedPX; k++) {
        const int sl = t + k * kFusedThreads;
        const int v = g.valid[sl];
        if constexpr (kStructured) {
          if (v) {
            acc.cnt += Acc::kCandidate;
            const float4 rp0 = g.rp[sl], rn0 = g.rn[sl], cpt = g.cp[sl], cn = g.cn[sl];
            float3 rp, rn;
            if (gate_t(cp, sT[e], rp0, rn0, cpt, cn, rp, rn)) {
              acc.cnt += Acc::kAccepted;
              if (sSame[e] && !cp.demoted)
                lin_terms_structured_xf(lp, sT[e] + 24, rp, rn, cpt, cn, acc);
              else
                lin_terms_structured(lp, sT[e] + 12, sT[e] + 24, rp0, rn0, cpt, cn, acc);
            }
          }
        } else {
          if (v) acc.cnt += Acc::kCandidate;
          if (v == 2) {
            acc.cnt += Acc::kAccepted;
            if (sStruct[e])
              lin_terms_structured(lp, sT[e] + 12, sT[e] + 24, g.rp[sl], g.rn[sl], g.cp[sl], g.cn[sl], acc);
            else
              lin_terms(lp, sT[e] + 12, g.rp[sl], g.rn[sl], g.cp[sl], g.cn[sl], g.o0[sl], g.o1[sl], g.o2[sl],
                        acc);
          }
        }
      }
      if (sub == kSubsPerTile - 1) {
        const PairDev &pd = pairs[sPair[e]];
        block_reduce_store_staged<kFusedThreads>(acc, pd.partials + (size_t)(tile_of(j) - pd.tile_base) * kPartialWords,
                                                 stage_of(j));
      }
    }
  };
  if constexpr (corr_stages<kStructured>() == 2) {
    // two stages: sub-tile j+1 is gathered while j is gated and linearized
    load_indices(0);
    tile_constants(0);
    issue_g1(0);
    load_indices(1);
    __syncthreads();          // tile 0's constants visible
    for (int j = 0; j < nsub; j++) {
      tile_constants(j + 1);
      issue_g1(j + 1);        // uses the indices loaded in the previous iteration
      load_indices(j + 2);
      if ((j + 1) % kSubsPerTile == 0) __syncthreads();  // the next tile's constants visible
      cp_async_wait<1>();     // G1(j) complete (G1(j+1) may be in flight)
      consume(j);
    }
  } else {
    // prologue: sub-tile 0 through G1 and the gate, sub-tile 1 through G1
    load_indices(0);
    tile_constants(0);
    issue_g1(0);
    load_indices(1);
    tile_constants(1);
    issue_g1(1);
    load_indices(2);
    __syncthreads();
    cp_async_wait<1>();
    gate_g2(0);
    for (int j = 0; j < nsub; j++) {
      tile_constants(j + 2);
      issue_g1(j + 2);          // uses the indices loaded in the previous iteration
      load_indices(j + 3);
      if ((j + 2) % kSubsPerTile == 0) __syncthreads();  // the constants of j + 2's tile visible
      cp_async_wait<2>();       // G1(j+1) complete (groups after it: G2(j), G1(j+2))
      gate_g2(j + 1);
      cp_async_wait<2>();       // G2(j) complete (groups after it: G1(j+2), G2(j+1))
      consume(j);
    }
  }
  cp_async_wait<0>();
}

// ------------------------------------------------------------ list mode
// CorrespondenceFinderProjective::_computeMulti for reference pixel p
// (correspondencefinderprojective.cpp:150-240): the best current point of
// the window of rows [r - R, r + R] x cols [c - C, c + C] (clamped), scanned
// row-major with the reference's gate order and its replacement rule
// (strictly closer AND strictly better aligned); -1 when none passes.
__device__ int multi_best(const PairDev &pd, const CorrParams &cp, const float *Tg, int p, int ri, int ncur) {
  const float4 rn0 = pd.ref_nrm[ri];
  if (normal_is_zero(rn0.x, rn0.y, rn0.z)) return -1;
  const float3 rp = xform_point_g(Tg, pd.ref_pts[ri]);
  const float3 rn = xform_normal_g(Tg, rn0);
  float kr = rn0.w;
  if (kr < cp.flat_thr) kr = cp.flat_thr;
  const int r = p / pd.cols, c = p - r * pd.cols;
  const int r0 = max(r - cp.row_search, 0), r1 = min(r + cp.row_search + 1, pd.rows);
  const int c0 = max(c - cp.col_search, 0), c1 = min(c + cp.col_search + 1, pd.cols);
  int best = -1;
  float bestN = 0.0f, bestD = 1e20f;
  for (int r2 = r0; r2 < r1; r2++)
    for (int c2 = c0; c2 < c1; c2++) {
      const int ci = pd.cur_index[r2 * pd.cols + c2];
      if (ci < 0 || ci >= ncur) continue;
      const float4 cn = pd.cur_nrm[ci];
      if (normal_is_zero(cn.x, cn.y, cn.z)) continue;
      const float nd = dot3g(cn.x, cn.y, cn.z, rn.x, rn.y, rn.z);
      if (nd < cp.cos_thr) continue;
      const float4 cpt = pd.cur_pts[ci];
      const float dx = fsb(cpt.x, rp.x), dy = fsb(cpt.y, rp.y), dz = fsb(cpt.z, rp.z);
      const float d = dot3g(dx, dy, dz, dx, dy, dz);
      if (d > cp.sq_thr) continue;
      float kc = cn.w;
      if (kc < cp.flat_thr) kc = cp.flat_thr;
      const float ratio = __double2float_rn(__ddiv_rn(__dadd_rn((double)kr, 1e-5), __dadd_rn((double)kc, 1e-5)));
      if (ratio < cp.min_ratio || ratio > cp.max_ratio) continue;
      if (best == -1 || (d < bestD && nd > bestN)) {
        best = ci;
        bestN = nd;
        bestD = d;
      }
    }
  return best;
}

// Gate decisions of four consecutive pixels (bit k: pixel pix0 + k has a
// correspondence) and the current point each one takes.
__device__ __forceinline__ unsigned list_mask(const PairDev &pd, const CorrParams &cp, const float *Tg, int pix0,
                                              int P, int rmax, int *cur_of) {
  unsigned m = 0;
  const int nref = *pd.ref_count, ncur = *pd.cur_count;
  const bool multi = cp.row_search > 0 || cp.col_search > 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    cur_of[k] = -1;
    int p = pix0 + k;
    if (p >= P) break;
    int ri = pd.ref_index[p];
    if (ri < 0 || ri >= nref || p / pd.cols >= rmax) continue;
    if (multi) {
      cur_of[k] = multi_best(pd, cp, Tg, p, ri, ncur);
      if (cur_of[k] >= 0) m |= 1u << k;
      continue;
    }
    int ci = pd.cur_index[p];
    if (ci < 0 || ci >= ncur) continue;
    cur_of[k] = ci;
    if (gate(cp, Tg, pd.ref_pts[ri], pd.ref_nrm[ri], pd.cur_pts[ci], pd.cur_nrm[ci])) m |= 1u << k;
  }
  return m;
}

__global__ void __launch_bounds__(kCorrThreads) k_corr_count(const PairDev *__restrict__ pairs, int npairs, CorrParams cp,
                                                             int use_state_T, const float *__restrict__ explicit_T) {
  __shared__ int red[32];
  int pi = find_pair(pairs, npairs, blockIdx.x);
  const PairDev &pd = pairs[pi];
  if (use_state_T && pd.state->done) return;
  int tile = blockIdx.x - pd.tile_base;
  int P = pd.rows * pd.cols;
  int rmax = pd.rows;
  if (cp.row_limit_threads > 1) rmax = (pd.rows / cp.row_limit_threads) * cp.row_limit_threads;
  float Tg[12];
  const float *src = use_state_T ? pd.state->Tgate : explicit_T + 12 * pi;
#pragma unroll
  for (int k = 0; k < 12; k++) Tg[k] = src[k];
  int cur_of[4];
  unsigned m = list_mask(pd, cp, Tg, tile * kCorrTilePixels + threadIdx.x * 4, P, rmax, cur_of);
  int v = __popc(m);
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < kCorrThreads / 32; i++) t += red[i];
    pd.list_tile_counts[tile] = t;
  }
}

__global__ void __launch_bounds__(kCorrThreads) k_corr_write(const PairDev *__restrict__ pairs, int npairs, CorrParams cp,
                                                             int use_state_T, const float *__restrict__ explicit_T) {
  __shared__ int red[32];
  __shared__ int wsum[kCorrThreads / 32];
  int pi = find_pair(pairs, npairs, blockIdx.x);
  const PairDev &pd = pairs[pi];
  if (use_state_T && pd.state->done) return;
  int tile = blockIdx.x - pd.tile_base;
  int P = pd.rows * pd.cols;
  int ntiles = (P + kCorrTilePixels - 1) / kCorrTilePixels;
  int rmax = pd.rows;
  if (cp.row_limit_threads > 1) rmax = (pd.rows / cp.row_limit_threads) * cp.row_limit_threads;
  float Tg[12];
  const float *src = use_state_T ? pd.state->Tgate : explicit_T + 12 * pi;
#pragma unroll
  for (int k = 0; k < 12; k++) Tg[k] = src[k];
  int before = 0;
  for (int t = threadIdx.x; t < tile; t += blockDim.x) before += pd.list_tile_counts[t];
  for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = before;
  __syncthreads();
  before = 0;
  for (int i = 0; i < kCorrThreads / 32; i++) before += red[i];
  int pix0 = tile * kCorrTilePixels + threadIdx.x * 4;
  int cur_of[4];
  unsigned m = list_mask(pd, cp, Tg, pix0, P, rmax, cur_of);
  int cnt = __popc(m);
  int inc = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  int woff = 0, btot = 0;
  for (int i = 0; i < kCorrThreads / 32; i++) {
    if (i < wid) woff += wsum[i];
    btot += wsum[i];
  }
  int o = before + woff + inc - cnt;
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (m & (1u << k)) {
      int p = pix0 + k;
      pd.pairs[2 * o] = pd.ref_index[p];
      pd.pairs[2 * o + 1] = cur_of[k];
      o++;
    }
  if (tile == ntiles - 1 && threadIdx.x == 0) *pd.num_pairs = before + btot;
}

// Linearizer::update over pd.pairs[0, K - K % T).  Tiles cover list slots.
// use_state_T: 0 explicit T, 1 the pair state's Tlin (skipping converged
// pairs), 2 the state's Tlin for every pair (statistics pass).
__global__ void __launch_bounds__(kCorrThreads) k_lin_list(const PairDev *__restrict__ pairs, int npairs, LinParams lp,
                                                           int parity_threads, int use_state_T,
                                                           const float *__restrict__ explicit_T) {
  int pi = find_pair(pairs, npairs, blockIdx.x);
  const PairDev &pd = pairs[pi];
  if (use_state_T == 1 && pd.state->done) return;
  int tile = blockIdx.x - pd.tile_base;
  int K = *pd.num_pairs;
  if (parity_threads > 1) K = (K / parity_threads) * parity_threads;
  float Tl[12];
  const float *src = use_state_T ? pd.state->Tlin : explicit_T + 12 * pi;
#pragma unroll
  for (int k = 0; k < 12; k++) Tl[k] = src[k];
  const int nref = *pd.ref_count, ncur = *pd.cur_count;
  Acc acc;
  acc.zero();
  int i0 = tile * kCorrTilePixels + threadIdx.x * 4;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int i = i0 + k;
    if (i >= K) break;
    int ri = pd.pairs[2 * i], ci = pd.pairs[2 * i + 1];
    if (ri < 0 || ci < 0 || ri >= nref || ci >= ncur) continue;
    acc.cnt += Acc::kCandidate;
    acc.cnt += Acc::kAccepted;
    const float4 *o = pd.cur_omg + 3 * (size_t)ci;
    lin_terms(lp, Tl, pd.ref_pts[ri], pd.ref_nrm[ri], pd.cur_pts[ci], pd.cur_nrm[ci], o[0], o[1], o[2], acc);
  }
  block_reduce_store<kCorrThreads>(acc, pd.partials + (size_t)tile * kPartialWords);
}

// ------------------------------------------------------------ solve
__device__ inline void float12_of(const double *T, float *o) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 4; j++) o[i * 4 + j] = (float)T[i * 4 + j];
}

// KRt of the projector placed at X (pinholepointprojector.cpp:16-31), in FP64.
__device__ inline void krt_of(const float *K, const double *X, float *o) {
  double t[16];
  d_iso_inverse(X, t);
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++)
      o[i * 4 + j] = (float)((double)K[i * 3 + 0] * t[0 * 4 + j] + (double)K[i * 3 + 1] * t[1 * 4 + j] +
                             (double)K[i * 3 + 2] * t[2 * 4 + j]);
    o[i * 4 + 3] = (float)((double)K[i * 3 + 0] * t[3] + (double)K[i * 3 + 1] * t[7] + (double)K[i * 3 + 2] * t[11]);
  }
}

// Prepares the matrices of an outer iteration from st->T.
__device__ inline void begin_outer(const PairDev &pd, PairState *st) {
  for (int k = 0; k < 16; k++) st->Tstart[k] = st->T[k];
  double X[16];
  d_mm4(st->T, st->ref_offset, X);
  krt_of(pd.K, X, st->KRt);
  d_iso_inverse(st->T, st->invT);
  float12_of(st->invT, st->Tgate);
  float12_of(st->invT, st->Tlin);
}

__global__ void k_init_pairs(const PairDev *__restrict__ pairs, int npairs, const double *__restrict__ guesses,
                             const double *__restrict__ ref_offsets) {
  int pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= npairs) return;
  const PairDev &pd = pairs[pi];
  PairState *st = pd.state;
  for (int k = 0; k < 16; k++) {
    st->T[k] = guesses[16 * pi + k];
    st->ref_offset[k] = ref_offsets[16 * pi + k];
  }
  st->T[12] = 0; st->T[13] = 0; st->T[14] = 0; st->T[15] = 1;
  st->error = 0; st->inliers = 0; st->num_corr = 0; st->candidates = 0;
  st->iterations = 0; st->done = 0; st->status = 0;
  for (int k = 0; k < 36; k++) st->H[k] = 0;
  for (int k = 0; k < 6; k++) st->b[k] = 0;
  begin_outer(pd, st);
  for (int k = 0; k < 12; k++) st->Tgate_used[k] = st->Tgate[k];
}

// mode: bit0 last inner iteration of the outer loop, bit1 reduce only (no
// pose update: Linearizer results of a list pass), bit2 statistics pass
// (reduce into Hstat only), kSolveCrossF32 sum the tile partials in FP32.
__global__ void __launch_bounds__(128) k_solve(const PairDev *__restrict__ pairs, int npairs, float lambda, int mode,
                                              double early_eps, int ignore_done) {
  __shared__ double part[4][32];
  __shared__ double tot[32];
  const PairDev &pd = pairs[blockIdx.x];
  PairState *st = pd.state;
  if (st->done && !ignore_done) return;
  int P = pd.rows * pd.cols;
  int nt = (P + kCorrTilePixels - 1) / kCorrTilePixels;
  int e = threadIdx.x & 31, g = threadIdx.x >> 5;
  if (mode & kSolveCrossF32) {
    // precision study: the same fixed order, in FP32
    float s = 0.0f;
    for (int t = g; t < nt; t += 4) s += (float)pd.partials[(size_t)t * kPartialWords + e];
    part[g][e] = (double)s;
    __syncthreads();
    if (threadIdx.x < 32)
      tot[e] = (double)((((float)part[0][e] + (float)part[1][e]) + (float)part[2][e]) + (float)part[3][e]);
  } else {
    // the fixed order t = g, g + 4, ..., with eight loads in flight
    double s = 0.0;
    int t = g;
    for (; t + 28 < nt; t += 32) {
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = pd.partials[(size_t)(t + 4 * q) * kPartialWords + e];
#pragma unroll
      for (int q = 0; q < 8; q++) s += v[q];
    }
    for (; t < nt; t += 4) s += pd.partials[(size_t)t * kPartialWords + e];
    part[g][e] = s;
    __syncthreads();
    if (threadIdx.x < 32) tot[e] = ((part[0][e] + part[1][e]) + part[2][e]) + part[3][e];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  // (every index below is a compile-time constant: H, b and A stay in registers)
  constexpr int li[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};
  double H[36], b[6];
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int i = li[q][0], j = li[q][1];
    H[i * 6 + j] = H[j * 6 + i] = tot[q];
    H[(3 + i) * 6 + 3 + j] = H[(3 + j) * 6 + 3 + i] = tot[15 + q];
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      H[i * 6 + 3 + j] = tot[6 + i * 3 + j];
      H[(3 + j) * 6 + i] = tot[6 + i * 3 + j];
    }
#pragma unroll
  for (int i = 0; i < 3; i++) { b[i] = tot[21 + i]; b[3 + i] = tot[24 + i]; }
  if (mode & 4) {
#pragma unroll
    for (int k = 0; k < 36; k++) st->Hstat[k] = H[k];
    return;
  }
#pragma unroll
  for (int k = 0; k < 36; k++) st->H[k] = H[k];
#pragma unroll
  for (int k = 0; k < 6; k++) st->b[k] = b[k];
  st->error = (float)tot[27];
  st->inliers = (int)tot[28];
  st->candidates = (int)tot[29];
  st->num_corr = (int)tot[30];
  if (mode & 2) return;
  // H += lambda I; dx = H^-1 (-b); invT = v2t(dx) invT  (alignerprojective.cpp:72-95)
  double A[36], nb[6], dx[6];
#pragma unroll
  for (int k = 0; k < 36; k++) A[k] = H[k];
#pragma unroll
  for (int i = 0; i < 6; i++) { A[i * 6 + i] += (double)lambda; nb[i] = -b[i]; }
  d_ldlt_solve6(A, nb, dx);
  double dT[16], nT[16];
  d_v2t(dx, dT);
  d_mm4(dT, st->invT, nT);
  for (int k = 0; k < 16; k++) st->invT[k] = nT[k];
  st->invT[12] = 0; st->invT[13] = 0; st->invT[14] = 0; st->invT[15] = 1;
  float12_of(st->invT, st->Tlin);
  if (!(mode & 1)) return;
  // T = invT^-1, renormalised through t2v/v2t (alignerprojective.cpp:98-100)
  double T[16], x[6];
  d_iso_inverse(st->invT, T);
  d_t2v(T, x);
  d_v2t(x, st->T);
  st->iterations += 1;
  for (int k = 0; k < 12; k++) st->Tgate_used[k] = st->Tgate[k];
  if (early_eps > 0) {
    double Si[16], D[16], dv[6];
    d_iso_inverse(st->Tstart, Si);
    d_mm4(st->T, Si, D);
    d_t2v(D, dv);
    double m = 0;
    for (int k = 0; k < 6; k++) m = fmax(m, fabs(dv[k]));
    if (m < early_eps) st->done = 1;
  }
  begin_outer(pd, st);
}

// ------------------------------------------------------------ launchers
void launch_zbuffer(const PairDev *d_pairs, int npairs, int max_pt_tiles, int mode, const float *explicit_KRt,
                    int ppt, cudaStream_t s, Profiler *prof) {
  if (max_pt_tiles <= 0 || npairs <= 0) return;
  prof->begin(NICP_K_ZBUFFER, s);
  const int kMaxGridY = 65535;
  for (int p0 = 0; p0 < npairs; p0 += kMaxGridY) {
    const dim3 g(max_pt_tiles, std::min(kMaxGridY, npairs - p0));
    switch (ppt) {
      case 1: k_zbuffer<1><<<g, kPointsPerCta, 0, s>>>(d_pairs, npairs, mode, explicit_KRt, p0); break;
      case 2: k_zbuffer<2><<<g, kPointsPerCta / 2, 0, s>>>(d_pairs, npairs, mode, explicit_KRt, p0); break;
      case 8: k_zbuffer<8><<<g, kPointsPerCta / 8, 0, s>>>(d_pairs, npairs, mode, explicit_KRt, p0); break;
      default: k_zbuffer<4><<<g, kPointsPerCta / 4, 0, s>>>(d_pairs, npairs, mode, explicit_KRt, p0); break;
    }
  }
  prof->end(NICP_K_ZBUFFER, s);
}

void launch_resolve(const PairDev *d_pairs, int npairs, int max_tiles, int to_ref, float *depth_out,
                    int drop_no_normal, cudaStream_t s, Profiler *prof) {
  if (max_tiles <= 0 || npairs <= 0) return;
  prof->begin(NICP_K_RESOLVE, s);
  const int kMaxGridY = 65535;
  for (int p0 = 0; p0 < npairs; p0 += kMaxGridY)
    k_resolve<<<dim3(max_tiles, std::min(kMaxGridY, npairs - p0)), kCorrThreads, 0, s>>>(d_pairs, npairs, to_ref,
                                                                                        depth_out, drop_no_normal, p0);
  prof->end(NICP_K_RESOLVE, s);
}

// Persistent grid: as many CTAs as fit on the device at once, never more
// than there are tiles.
// The shared-memory opt-in holds for the device that was current when it was
// set, and the occupancy is that device's: both are taken once per device
// (std::call_once: host threads on other contexts wait rather than race).
template <bool kStructured>
static int corr_lin_grid(int total_tiles, int ctas_per_sm) {
  struct Occupancy {
    int sm_count = 1, per_sm_max = 1;
  };
  constexpr int kMaxDevices = 64;
  static Occupancy occ[kMaxDevices];
  static std::once_flag once[kMaxDevices];
  auto query = [](int dev, Occupancy *o) {
    cudaFuncSetAttribute(k_corr_lin<kStructured>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         corr_smem<kStructured>());
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_corr_lin<kStructured>, kFusedThreads,
                                                  corr_smem<kStructured>());
    o->per_sm_max = std::max(1, per_sm);
    o->sm_count = std::max(1, sms);
  };
  int dev = 0;
  cudaGetDevice(&dev);
  Occupancy local;
  const Occupancy *o = &local;
  if (dev >= 0 && dev < kMaxDevices) {
    std::call_once(once[dev], query, dev, &occ[dev]);
    o = &occ[dev];
  } else {
    query(dev, &local);
  }
  const int resident = o->sm_count * o->per_sm_max;
  const int grid = (ctas_per_sm > 0 && ctas_per_sm < o->per_sm_max) ? o->sm_count * ctas_per_sm : resident;
  return std::min(total_tiles, grid);
}

void launch_corr_lin(const PairDev *d_pairs, int npairs, int total_tiles, const CorrParams &cp, const LinParams &lp,
                     int flags, bool structured, int ctas_per_sm, const int *tile_pair, cudaStream_t s,
                     Profiler *prof) {
  if (total_tiles <= 0) return;
  prof->begin(NICP_K_CORR_LIN, s);
  if (structured) {
    int grid = corr_lin_grid<true>(total_tiles, ctas_per_sm);
    k_corr_lin<true><<<grid, kFusedThreads, corr_smem<true>(), s>>>(d_pairs, npairs, tile_pair, total_tiles, cp,
                                                                    lp, flags);
  } else {
    int grid = corr_lin_grid<false>(total_tiles, ctas_per_sm);
    k_corr_lin<false><<<grid, kFusedThreads, corr_smem<false>(), s>>>(d_pairs, npairs, tile_pair, total_tiles,
                                                                      cp, lp, flags);
  }
  prof->end(NICP_K_CORR_LIN, s);
}

void launch_corr_list(const PairDev *d_pairs, int npairs, int total_tiles, const CorrParams &cp, int use_state_T,
                      const float *explicit_T, cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_CORR_LIST, s);
  k_corr_count<<<total_tiles, kCorrThreads, 0, s>>>(d_pairs, npairs, cp, use_state_T, explicit_T);
  k_corr_write<<<total_tiles, kCorrThreads, 0, s>>>(d_pairs, npairs, cp, use_state_T, explicit_T);
  prof->end(NICP_K_CORR_LIST, s, 2);
}

void launch_lin_list(const PairDev *d_pairs, int npairs, int total_tiles, const LinParams &lp, int parity_threads,
                     int use_state_T, const float *explicit_T, cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_LIN_LIST, s);
  k_lin_list<<<total_tiles, kCorrThreads, 0, s>>>(d_pairs, npairs, lp, parity_threads, use_state_T, explicit_T);
  prof->end(NICP_K_LIN_LIST, s);
}

// tile_pair[tile] = the pair whose pixel image holds the tile (grid: tiles
// of a pair, pair), so that the persistent fused kernel finds a tile's pair
// with one load instead of a search.
__global__ void k_tile_pairs(const PairDev *__restrict__ pairs, int npairs, int *__restrict__ tile_pair, int pair0) {
  const int pi = pair0 + (int)blockIdx.y;
  if (pi >= npairs) return;
  const PairDev &pd = pairs[pi];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ntiles = (pd.rows * pd.cols + kCorrTilePixels - 1) / kCorrTilePixels;
  if (t < ntiles) tile_pair[pd.tile_base + t] = pi;
}

void launch_init_pairs(const PairDev *d_pairs, int npairs, const double *d_guesses, const double *d_ref_offsets,
                       int *tile_pair, int max_tiles, cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_SOLVE, s);
  k_init_pairs<<<(npairs + 63) / 64, 64, 0, s>>>(d_pairs, npairs, d_guesses, d_ref_offsets);
  const int kMaxGridY = 65535;
  if (tile_pair && max_tiles > 0)
    for (int p0 = 0; p0 < npairs; p0 += kMaxGridY)
      k_tile_pairs<<<dim3((max_tiles + 255) / 256, std::min(kMaxGridY, npairs - p0)), 256, 0, s>>>(d_pairs, npairs,
                                                                                                  tile_pair, p0);
  prof->end(NICP_K_SOLVE, s, tile_pair && max_tiles > 0 ? 2 : 1);
}

void launch_solve(const PairDev *d_pairs, int npairs, float lambda, int mode, double early_eps, int ignore_done,
                  cudaStream_t s, Profiler *prof) {
  prof->begin(NICP_K_SOLVE, s);
  k_solve<<<npairs, 128, 0, s>>>(d_pairs, npairs, lambda, mode, early_eps, ignore_done);
  prof->end(NICP_K_SOLVE, s);
}

// ------------------------------------------------------------ scratch-free linearizer
// The linearizer of nicp_linearize, for callers that must not allocate
// device memory: the per-tile FP64 partials go to this fixed array instead
// of the context workspace.  The array is part of the library's device
// image, so it exists on every GPU that loads the library, from the first
// load until the process exits.  Every call uses the same array: calls whose
// kernels overlap on the GPU (different streams, or different host threads
// on one device) race on it.  Nothing in it needs clearing -- each call
// writes every partial it later reads.
constexpr int kNoAllocMaxTiles = NICP_LINEARIZE_NOALLOC_MAX_PAIRS / kCorrTilePixels;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxTiles * kPartialWords];

__global__ void __launch_bounds__(kCorrThreads) k_lin_noalloc(NoAllocLinArgs a, double *__restrict__ partials) {
  const int tile = blockIdx.x;
  if (tile >= kNoAllocMaxTiles) return;  // the host refuses longer lists; never write past the array
  int K = a.num_pairs;
  if (a.parity_threads > 1) K = (K / a.parity_threads) * a.parity_threads;
  const int nref = *a.ref_count, ncur = *a.cur_count;
  Acc acc;
  acc.zero();
  const int i0 = tile * kCorrTilePixels + threadIdx.x * 4;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int i = i0 + k;
    if (i >= K) break;
    const int ri = a.pairs[2 * i], ci = a.pairs[2 * i + 1];
    if (ri < 0 || ci < 0 || ri >= nref || ci >= ncur) continue;
    acc.cnt += Acc::kCandidate;
    acc.cnt += Acc::kAccepted;
    const float4 *o = a.cur_omg + 3 * (size_t)ci;
    lin_terms(a.lp, a.T, a.ref_pts[ri], a.ref_nrm[ri], a.cur_pts[ci], a.cur_nrm[ci], o[0], o[1], o[2], acc);
  }
  block_reduce_store<kCorrThreads>(acc, partials + (size_t)tile * kPartialWords);
}

// Sums the tile partials in the same fixed order as k_solve and writes
// H (36, row-major), b (6), error, inliers to out.
__global__ void __launch_bounds__(128) k_lin_noalloc_sum(int ntiles, const double *__restrict__ partials,
                                                         double *__restrict__ out) {
  __shared__ double part[4][32];
  __shared__ double tot[32];
  const int e = threadIdx.x & 31, g = threadIdx.x >> 5;
  double s = 0.0;
  const int nt = min(ntiles, kNoAllocMaxTiles);
  for (int t = g; t < nt; t += 4) s += partials[(size_t)t * kPartialWords + e];
  part[g][e] = s;
  __syncthreads();
  if (threadIdx.x < 32) tot[e] = ((part[0][e] + part[1][e]) + part[2][e]) + part[3][e];
  __syncthreads();
  if (threadIdx.x != 0) return;
  const int li[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};
  for (int q = 0; q < 6; q++) {
    const int i = li[q][0], j = li[q][1];
    out[i * 6 + j] = out[j * 6 + i] = tot[q];
    out[(3 + i) * 6 + 3 + j] = out[(3 + j) * 6 + 3 + i] = tot[15 + q];
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) out[i * 6 + 3 + j] = out[(3 + j) * 6 + i] = tot[6 + i * 3 + j];
  for (int i = 0; i < 3; i++) {
    out[36 + i] = tot[21 + i];
    out[39 + i] = tot[24 + i];
  }
  out[42] = (double)(float)tot[27];  // Linearizer::error() is a float
  out[43] = (double)(int)tot[28];
}

// Device address of g_noalloc_partials, looked up once per device with that
// device current (host code must not use the symbol itself as an address).
static double *noalloc_partials_on(int device, cudaError_t *err) {
  constexpr int kMaxDevices = 64;
  static double *addr[kMaxDevices] = {};
  static std::mutex m;
  *err = cudaSuccess;
  if (device < 0 || device >= kMaxDevices) {
    *err = cudaErrorInvalidDevice;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(m);
  if (!addr[device]) {
    double *p = nullptr;
    *err = cudaGetSymbolAddress((void **)&p, g_noalloc_partials);
    if (*err != cudaSuccess) return nullptr;
    addr[device] = p;
  }
  return addr[device];
}

int lin_noalloc(const NoAllocLinArgs &args, double *out_dev, cudaStream_t s) {
  if (args.num_pairs < 0 || args.num_pairs > NICP_LINEARIZE_NOALLOC_MAX_PAIRS) return NICP_EINVAL;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return NICP_ECUDA;
  cudaError_t err;
  double *partials = noalloc_partials_on(device, &err);
  if (!partials) return NICP_ECUDA;
  const int ntiles = std::max(1, (args.num_pairs + kCorrTilePixels - 1) / kCorrTilePixels);
  k_lin_noalloc<<<ntiles, kCorrThreads, 0, s>>>(args, partials);
  k_lin_noalloc_sum<<<1, 128, 0, s>>>(ntiles, partials, out_dev);
  return cudaGetLastError() == cudaSuccess ? NICP_OK : NICP_ECUDA;
}

}  // namespace nicp
