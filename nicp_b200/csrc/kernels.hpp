// kernels.hpp -- host-side launchers of the NICP kernels and the event profiler.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "nicp_gpu.h"

namespace nicp {

// Brackets kernel launches with CUDA events on the launching stream.  Events
// recorded during stream capture become graph nodes and are re-recorded on
// every replay of that graph.
struct Profiler {
  struct Rec {
    int kernel;
    int nkernels;
    cudaEvent_t a, b;
  };
  bool enabled = false;
  bool capturing = false;            // events taken now belong to a graph
  std::vector<cudaEvent_t> pool;     // reusable events of direct launches
  std::vector<cudaEvent_t> owned;    // events baked into captured graphs
  size_t next = 0;
  std::vector<Rec> recs;
  cudaEvent_t open[NICP_K_COUNT] = {};
  int open_kernels[NICP_K_COUNT] = {};
  unsigned long long launches = 0;  // kernels launched through the launchers

  cudaEvent_t take() {
    if (capturing) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      owned.push_back(e);
      return e;
    }
    if (next == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[next++];
  }
  void begin(int k, cudaStream_t s) {
    if (!enabled) return;
    open[k] = take();
    cudaEventRecord(open[k], s);
  }
  void end(int k, cudaStream_t s, int nk = 1) {
    launches += nk;
    if (!enabled) return;
    cudaEvent_t b = take();
    cudaEventRecord(b, s);
    recs.push_back(Rec{k, nk, open[k], b});
  }
  ~Profiler() {
    for (auto e : pool) cudaEventDestroy(e);
    for (auto e : owned) cudaEventDestroy(e);
  }
};

// frame_of_*: the frame of each CTA of the 1-D build grids (unprojection
// tiles, 16-row bands, band-carry CTAs), filled on the host.
void launch_unproject(const FrameDev *d_frames, int nframes, int total_tiles, const int *frame_of_tile, cudaStream_t s,
                      Profiler *prof);
void launch_depth_scale(const uint16_t *u16, const float *f32, size_t pitch_elems, int rows, int cols,
                        float depth_scale, int step, float max_cov, float *out, cudaStream_t s);
// Integral image over 16-row bands (moment_band_rows()): total_bands band
// CTAs, total_carry_ctas = sum over frames of ceil(10 cols / 128).
int moment_band_rows();
// Few-frame launches (moments_row_path) compute every row prefix in parallel
// into FrameDev::rowpre (10 planes of moment_acc_bytes per pixel) instead of
// sweeping the bands; the planes are bitwise the same.
bool moments_row_path(int nframes);
size_t moment_acc_bytes(int precision);
// Resident band-sweep CTAs per SM (one per 16-row band and frame): frame
// chunks of whole waves of them leave no half-empty last wave.
int moment_sweep_ctas_per_sm(int precision);
void launch_moments(int precision, const FrameDev *d_frames, int nframes, int total_bands, int total_carry_ctas,
                    int max_bands, const int *frame_of_band, const int *frame_of_carry, cudaStream_t s,
                    Profiler *prof);
// (pixel tile, frame) grid over max_pixels, the largest frame of the launch;
// nframes <= 65535.  shape: one of kStatsShapes (CTA size, CTAs per SM).
constexpr int kStatsShapes = 4;  // k_stats launch shapes the autotuner chooses from (0: default)
int stats_shape_threads(int shape);
int stats_shape_min_ctas(int shape);
// lean: no Stats kept and information matrices U diag(d0, d1, d1) U^T (only
// the smallest eigenpair is computed).
void launch_stats(int precision, const FrameDev *d_frames, int nframes, int max_pixels, int shape, bool lean,
                  cudaStream_t s, Profiler *prof);
void launch_reset_normal_counts(const FrameDev *d_frames, int nframes, cudaStream_t s);
struct OmegaParams {
  float omd[8];  // (d0, d1) of point flat, point non-flat, normal flat, normal non-flat
};
// Writes the information matrices of a cloud whose Omega is implicit.
void launch_materialize_omg(const float4 *pts, const float4 *nrm, float4 *omg, const int *count, int capacity,
                            const float omd[8], cudaStream_t s);
// omg may be null: an implicit Omega follows the rotated normal by itself.
void launch_cloud_transform(float4 *pts, float4 *nrm, float4 *omg, float *eig, float4 *gauss, const int *count,
                            int capacity, const float *d_m12, cudaStream_t s, Profiler *prof);
size_t moment_bytes(int precision);
void launch_intervals(const float *d_depth, int P, const float *d_K9, float min_d, float max_d, float R, int32_t *d_out,
                      cudaStream_t s, Profiler *prof);

// Host-side Aligner::_computeStatistics (FP64): translational / rotational
// eigen-ratios of the solution information matrix, the matrix itself
// (Aligner::omega(), row-major 6x6) and the reconstructed mean.
void solution_statistics(const double H36[36], const double T16[16], double *translational_ratio,
                         double *rotational_ratio, double omega36[36], double mean6[6]);

// Grid (max_pt_tiles, npairs): max_pt_tiles = the largest number of
// 1024-point tiles of any pair's projected cloud.
void launch_zbuffer(const PairDev *d_pairs, int npairs, int max_pt_tiles, int mode, const float *explicit_KRt,
                    int ppt, cudaStream_t s, Profiler *prof);
// Grid (max_tiles, npairs): max_tiles = the largest number of 1024-pixel
// tiles of any pair's image.
void launch_resolve(const PairDev *d_pairs, int npairs, int max_tiles, int to_ref, float *depth_out,
                    int drop_no_normal, cudaStream_t s, Profiler *prof);
void launch_corr_lin(const PairDev *d_pairs, int npairs, int total_tiles, const CorrParams &cp, const LinParams &lp,
                     int flags, bool structured, int ctas_per_sm, const int *tile_pair, cudaStream_t s,
                     Profiler *prof);
void launch_corr_list(const PairDev *d_pairs, int npairs, int total_tiles, const CorrParams &cp, int use_state_T,
                      const float *explicit_T, cudaStream_t s, Profiler *prof);
void launch_lin_list(const PairDev *d_pairs, int npairs, int total_tiles, const LinParams &lp, int parity_threads,
                     int use_state_T, const float *explicit_T, cudaStream_t s, Profiler *prof);
// Initialises the pair states and, when tile_pair is given, the tile -> pair
// table of the fused kernel (total pixel tiles entries).
void launch_init_pairs(const PairDev *d_pairs, int npairs, const double *d_guesses, const double *d_ref_offsets,
                       int *tile_pair, int max_tiles, cudaStream_t s, Profiler *prof);
void launch_solve(const PairDev *d_pairs, int npairs, float lambda, int mode, double early_eps, int ignore_done,
                  cudaStream_t s, Profiler *prof);

// Inputs of the scratch-free linearizer, passed by value to the kernel.
struct NoAllocLinArgs {
  const float4 *ref_pts, *ref_nrm;
  const int *ref_count;
  const float4 *cur_pts, *cur_nrm, *cur_omg;
  const int *cur_count;
  const int32_t *pairs;  // device, 2 * num_pairs
  int num_pairs;
  int parity_threads;
  float T[12];
  LinParams lp;
};
// Enqueues the scratch-free linearizer on s; allocates nothing.
int lin_noalloc(const NoAllocLinArgs &args, double *out_dev, cudaStream_t s);

// Merger::merge on the device (k_merge.cu).  n points (host copy of *count);
// every per-point array below holds n ints; the o_* staging arrays receive the
// compacted cloud, out_count its counts (points, points with a normal).
struct MergeArgs {
  int n;
  const int *count;
  const float4 *pts, *nrm, *omg;
  const float *eig;       // or null
  float4 *gauss;          // fused in place
  const float *KRt12;     // device, the projector's KRt for the merge transform
  int rows, cols;
  float min_d, max_d, max_depth, dthr;
  const int32_t *index;   // z-buffer winners, rows*cols
  const float *depth;     // their depths
  int *tgt, *cnt, *off, *fill, *list, *keep, *pos;
  void *scan_temp;
  size_t scan_temp_bytes;
  float4 *o_pts, *o_nrm, *o_omg;
  float *o_eig;
  float4 *o_gauss;
  int *out_count;
};
// Uniform grid over the current cloud's xyz (k_nn.cu).
struct NNGrid {
  float origin[3];
  float h, inv_h;
  int dim[3];
  int max_shell;  // shells needed to cover the radius
};
struct NNBuild {
  int nc;
  const float4 *cur_pts, *cur_nrm;
  float nscale;
  NNGrid grid;
  int key_bits;
  unsigned *keys, *skeys, *idx, *sidx;
  float *feat6, *sfeat6;
  int *cstart, *cend;
  void *temp;
  size_t temp_bytes;
};
struct NNQuery {
  int nr;
  const float4 *ref_pts, *ref_nrm;
  const float4 *cur_pts, *cur_nrm;
  const float *Tg;          // rows 0..2 of the transform, or null: the pair state's Tgate
  const PairState *state;
  float nscale, sq, cos_thr;
  int demoted;
  NNGrid grid;
  const int *cstart, *cend;
  const float *sfeat6;
  const unsigned *sidx;
  int *match;
};
size_t nn_temp_bytes(int n);
int launch_nn_build(const NNBuild &b, cudaStream_t s);
int launch_nn_correspond(const NNQuery &q, int *flag, int *pos, void *temp, size_t temp_bytes, int32_t *pairs,
                         int *num_pairs, cudaStream_t s);

size_t merge_scan_temp_bytes(int n);
int launch_merge(const MergeArgs &a, cudaStream_t s);

}  // namespace nicp
