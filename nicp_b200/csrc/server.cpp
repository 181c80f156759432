// server.cpp -- continuous-batching request loop over the NICP path
// (nicp_server_* in include/nicp_gpu.h).
//
// Threads: the caller submits frames (copied to host memory) and polls
// results; `workers` threads each own a context (device + CUDA stream +
// workspace) and repeatedly take a batch of admissible requests, build their
// clouds in one pass of launches, align them against their streams'
// keyframes in one device loop, and publish the results.  Admission:
//   - at most one request per camera stream in flight, so every stream's
//     frames are processed in submission order against the keyframe its
//     previous frame left;
//   - the device memory of resident keyframes plus in-flight requests
//     (cloud + build scratch + alignment workspace, estimated per pixel)
//     stays within hbm_budget_bytes; a request that could never fit is
//     answered with NICP_EBUDGET.
// Clouds are recycled per resolution, so the steady state allocates nothing.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "abi_guard.hpp"
#include "nicp_gpu.h"

namespace nicp {
namespace internal {
int build_batch(nicp_ctx *ctx, int n, const uint16_t *const *depth, const int *rows, const int *cols,
                const nicp_camera *cams, const nicp_cloud_params *prm, nicp_cloud *const *out);
int align_batch(nicp_ctx *ctx, int n, const nicp_cloud *const *refs, const nicp_cloud *const *curs,
                const nicp_camera *cams, const float *guesses, const nicp_corr_params *corr,
                const nicp_lin_params *lin, const nicp_align_params *prm, nicp_align_result *out);
int cloud_normal_counts(nicp_ctx *ctx, int n, const nicp_cloud *const *c, int *out);
size_t cloud_bytes(const nicp_cloud *c);
int ctx_make_current(nicp_ctx *ctx);
}  // namespace internal
}  // namespace nicp

namespace {

using Clock = std::chrono::steady_clock;

// Bytes per pixel a request holds while in flight: its cloud (points,
// normals, information matrices: 80 B/pt, index image 4 B/px), the FP64
// integral image of the build (80 B/px) and the alignment workspace
// (z-buffer 8, index images 4 + 4, partials ~0.25 B/px).
constexpr size_t kInflightBytesPerPixel = 84 + 80 + 17;
constexpr size_t kKeyframeBytesPerPixel = 84;

struct Request {
  uint64_t id;
  int stream;
  int rows, cols;
  nicp_camera cam;
  std::vector<uint16_t> depth;
  Clock::time_point submitted;
  size_t bytes() const { return kInflightBytesPerPixel * (size_t)rows * cols; }
};

struct StreamState {
  nicp_cloud *keyframe = nullptr;
  int key_rows = 0, key_cols = 0;
  nicp_camera key_cam{};
  int key_points = 0;  // keyframe points with a normal
  // the last two estimates against the keyframe (frame -> keyframe) and
  // how many there are since the keyframe was set (at most 2 kept)
  double last[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  double prev[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  int estimates = 0;
  // Initial guess of the next frame: a constant-velocity prediction,
  // last * prev^-1 * last (the motion between the last two frames applied
  // once more), with one estimate the last one, with none the identity.
  void guess(float *g) const {
    double G[16];
    if (estimates >= 2) {
      double pi[16], m[16];
      iso_inverse(prev, pi);
      mm4(last, pi, m);
      mm4(m, last, G);
    } else {
      for (int k = 0; k < 16; k++) G[k] = estimates ? last[k] : (k % 5 == 0 ? 1.0 : 0.0);
    }
    for (int k = 0; k < 16; k++) g[k] = (float)G[k];
    g[12] = g[13] = g[14] = 0.0f;
    g[15] = 1.0f;
  }
  void push(const double *T) {
    std::memcpy(prev, last, sizeof(last));
    std::memcpy(last, T, sizeof(last));
    estimates = std::min(estimates + 1, 2);
  }
  void reset() { estimates = 0; }
  static void mm4(const double *A, const double *B, double *C) {
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++) {
        double s = 0;
        for (int k = 0; k < 4; k++) s += A[i * 4 + k] * B[k * 4 + j];
        C[i * 4 + j] = s;
      }
  }
  static void iso_inverse(const double *T, double *R) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) R[i * 4 + j] = T[j * 4 + i];
    for (int i = 0; i < 3; i++) R[i * 4 + 3] = -(R[i * 4 + 0] * T[3] + R[i * 4 + 1] * T[7] + R[i * 4 + 2] * T[11]);
    R[12] = R[13] = R[14] = 0;
    R[15] = 1;
  }
  bool busy = false;
};

}  // namespace

struct nicp_server {
  nicp_server_params prm;
  int device = 0;
  std::vector<nicp_ctx *> ctxs;
  std::vector<std::thread> threads;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::unordered_map<int, std::deque<Request>> queues;  // pending requests per stream, in order
  int npending = 0;
  std::deque<nicp_server_result> done;
  std::unordered_map<int, StreamState> streams;
  // Free clouds by (worker, pixel count).  A cloud belongs to the context of
  // the worker that created it: only that worker builds into it (its
  // allocation and counters are ordered on that worker's stream); any worker
  // may read it as a keyframe once its build has completed.
  std::map<std::pair<int, size_t>, std::vector<nicp_cloud *>> pool;
  std::unordered_map<const nicp_cloud *, int> owner;
  std::vector<nicp_cloud *> all_clouds;
  size_t inflight_bytes = 0, keyframe_bytes = 0;
  int inflight_requests = 0;
  bool stop = false;

  nicp_cloud *take_cloud(int w, size_t pixels) {
    auto it = pool.find({w, pixels});
    if (it != pool.end() && !it->second.empty()) {
      nicp_cloud *c = it->second.back();
      it->second.pop_back();
      return c;
    }
    nicp_cloud *c = nullptr;
    if (nicp_cloud_create(ctxs[w], &c) != NICP_OK) return nullptr;
    all_clouds.push_back(c);
    owner[c] = w;
    return c;
  }
  void give_cloud(size_t pixels, nicp_cloud *c) { pool[{owner[c], pixels}].push_back(c); }

  void worker(int w);
};

void nicp_server::worker(int w) {
  nicp_ctx *ctx = ctxs[w];
  // the contexts were created on the submitting thread; every library call
  // below makes the context's device current for itself (a device that cannot
  // be made current fails each request's calls with NICP_ECUDA), so this only
  // sets the thread's default for anything else it does
  nicp::internal::ctx_make_current(ctx);
  for (;;) {
    std::vector<Request> batch;
    std::vector<nicp_cloud *> cur_clouds;
    {
      std::unique_lock<std::mutex> lk(m);
      cv_work.wait(lk, [&] { return stop || npending > 0; });
      if (stop) return;
      // Candidates: the oldest pending request of every stream with none in
      // flight, admitted oldest first while the batch and budget allow.
      size_t budget = prm.hbm_budget_bytes;
      std::vector<std::pair<Clock::time_point, int>> heads;
      for (auto &kv : queues)
        if (!kv.second.empty() && !streams[kv.first].busy) heads.push_back({kv.second.front().submitted, kv.first});
      std::sort(heads.begin(), heads.end());
      // Share the active streams between the workers, so that under load
      // every worker has a batch going (host and device work of the batches
      // overlap) instead of one worker taking every stream.
      int active = 0;
      for (auto &kv : streams) active += kv.second.busy;
      active += (int)heads.size();
      int cap = std::min(prm.max_batch, std::max(1, (active + prm.workers - 1) / prm.workers));
      for (auto &h : heads) {
        if ((int)batch.size() >= cap) break;
        std::deque<Request> &q = queues[h.second];
        Request &rq = q.front();
        size_t need = rq.bytes() + kKeyframeBytesPerPixel * (size_t)rq.rows * rq.cols;
        if (need > budget) {
          // can never fit: answer now
          nicp_server_result r{};
          r.request_id = rq.id;
          r.stream_id = rq.stream;
          r.status = NICP_EBUDGET;
          r.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - rq.submitted).count();
          done.push_back(r);
          q.pop_front();
          npending--;
          cv_done.notify_all();
          continue;
        }
        if (inflight_bytes + keyframe_bytes + rq.bytes() > budget) continue;
        streams[rq.stream].busy = true;
        inflight_bytes += rq.bytes();
        inflight_requests++;
        batch.push_back(std::move(rq));
        q.pop_front();
        npending--;
      }
      if (batch.empty()) {
        // nothing admissible now (busy streams or memory): wait for a batch to finish
        cv_work.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
      for (auto &r : batch) cur_clouds.push_back(take_cloud(w, (size_t)r.rows * r.cols));
    }
    Clock::time_point start = Clock::now();
    int n = (int)batch.size();
    std::vector<const uint16_t *> dptr(n);
    std::vector<int> rows(n), cols(n);
    std::vector<nicp_camera> cams(n);
    for (int i = 0; i < n; i++) {
      dptr[i] = batch[i].depth.data();
      rows[i] = batch[i].rows;
      cols[i] = batch[i].cols;
      cams[i] = batch[i].cam;
    }
    int rc = NICP_OK;
    for (auto *c : cur_clouds)
      if (!c) rc = NICP_ENOMEM;
    if (rc == NICP_OK)
      rc = nicp::internal::build_batch(ctx, n, dptr.data(), rows.data(), cols.data(), cams.data(), &prm.cloud,
                                       cur_clouds.data());
    // pairs: requests whose stream has a keyframe of the same resolution
    std::vector<int> pair_of(n, -1);
    std::vector<const nicp_cloud *> refs, curs;
    std::vector<nicp_camera> pcams;
    std::vector<float> guesses;
    {
      std::lock_guard<std::mutex> lk(m);
      for (int i = 0; i < n; i++) {
        StreamState &ss = streams[batch[i].stream];
        if (ss.keyframe && ss.key_rows == rows[i] && ss.key_cols == cols[i]) {
          pair_of[i] = (int)refs.size();
          refs.push_back(ss.keyframe);
          curs.push_back(cur_clouds[i]);
          pcams.push_back(cams[i]);
          float g[16];
          ss.guess(g);
          guesses.insert(guesses.end(), g, g + 16);
        }
      }
    }
    std::vector<nicp_align_result> res(refs.size());
    std::vector<int> cur_counts(n, 0);
    if (rc == NICP_OK && !refs.empty()) {
      nicp_align_params ap = prm.align;
      ap.compute_statistics = 0;
      rc = nicp::internal::align_batch(ctx, (int)refs.size(), refs.data(), curs.data(), pcams.data(),
                                       guesses.data(), &prm.corr, &prm.lin, &ap, res.data());
    }
    if (rc == NICP_OK) rc = nicp::internal::cloud_normal_counts(ctx, n, cur_clouds.data(), cur_counts.data());
    if (rc == NICP_OK) rc = nicp_ctx_synchronize(ctx);
    Clock::time_point end = Clock::now();
    {
      std::lock_guard<std::mutex> lk(m);
      for (int i = 0; i < n; i++) {
        Request &rq = batch[i];
        StreamState &ss = streams[rq.stream];
        nicp_server_result r{};
        r.request_id = rq.id;
        r.stream_id = rq.stream;
        r.status = rc;
        r.batch_size = n;
        for (int k = 0; k < 16; k++) r.T[k] = (k % 5 == 0) ? 1.0 : 0.0;
        bool replace = true;
        if (rc == NICP_OK && pair_of[i] >= 0) {
          const nicp_align_result &a = res[pair_of[i]];
          std::memcpy(r.T, a.T, sizeof(r.T));
          r.error = a.error;
          r.inliers = a.inliers;
          r.keyframe_points = ss.key_points;
          replace = (double)a.inliers < (double)prm.keyframe_min_inlier_ratio * ss.key_points;
          ss.push(a.T);  // the next frame's guess builds on this estimate
        }
        size_t px = (size_t)rq.rows * rq.cols;
        if (rc == NICP_OK && replace) {
          if (ss.keyframe) {
            keyframe_bytes -= kKeyframeBytesPerPixel * (size_t)ss.key_rows * ss.key_cols;
            give_cloud((size_t)ss.key_rows * ss.key_cols, ss.keyframe);
          }
          ss.keyframe = cur_clouds[i];
          ss.key_rows = rq.rows;
          ss.key_cols = rq.cols;
          ss.key_cam = rq.cam;
          ss.key_points = cur_counts[i];
          ss.reset();
          keyframe_bytes += kKeyframeBytesPerPixel * px;
          r.keyframe_replaced = 1;
        } else if (cur_clouds[i]) {
          give_cloud(px, cur_clouds[i]);
        }
        ss.busy = false;
        inflight_bytes -= rq.bytes();
        inflight_requests--;
        r.queue_ms = std::chrono::duration<double, std::milli>(start - rq.submitted).count();
        r.latency_ms = std::chrono::duration<double, std::milli>(end - rq.submitted).count();
        done.push_back(r);
      }
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

extern "C" void nicp_default_server_params(nicp_server_params *p) {
  p->hbm_budget_bytes = (size_t)60 << 30;
  p->max_batch = 64;
  p->workers = 2;
  p->keyframe_min_inlier_ratio = 0.4f;
  nicp_default_cloud_params(&p->cloud);
  nicp_default_corr_params(&p->corr);
  nicp_default_lin_params(&p->lin);
  nicp_default_align_params(&p->align);
  p->align.compute_statistics = 0;
}

extern "C" int nicp_server_create(int device, const nicp_server_params *prm, nicp_server **out) {
  NICP_ABI_TRY
  if (!prm || !out || prm->workers < 1 || prm->workers > 16 || prm->max_batch < 1) return NICP_EINVAL;
  *out = nullptr;
  auto *s = new nicp_server();
  s->prm = *prm;
  s->device = device;
  for (int w = 0; w < prm->workers; w++) {
    nicp_ctx *ctx = nullptr;
    int rc = nicp_ctx_create(device, nullptr, &ctx);
    if (rc != NICP_OK) {
      for (auto *c : s->ctxs) nicp_ctx_destroy(c);
      delete s;
      return rc;
    }
    s->ctxs.push_back(ctx);
  }
  for (int w = 0; w < prm->workers; w++) s->threads.emplace_back([s, w] { s->worker(w); });
  *out = s;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_server_submit(nicp_server *s, int stream_id, uint64_t request_id, const uint16_t *depth, int rows,
                                  int cols, const nicp_camera *cam) {
  NICP_ABI_TRY
  if (!s || !depth || rows <= 0 || cols <= 0 || !cam) return NICP_EINVAL;
  Request r;
  r.submitted = Clock::now();  // latency counts the copy of the frame below
  r.id = request_id;
  r.stream = stream_id;
  r.rows = rows;
  r.cols = cols;
  r.cam = *cam;
  r.cam.rows = rows;
  r.cam.cols = cols;
  r.depth.assign(depth, depth + (size_t)rows * cols);
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->queues[stream_id].push_back(std::move(r));
    s->npending++;
  }
  s->cv_work.notify_one();
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_server_poll(nicp_server *s, nicp_server_result *out, int max, int *n, int wait_ms) {
  NICP_ABI_TRY
  if (!s || !out || !n || max < 0) return NICP_EINVAL;
  std::unique_lock<std::mutex> lk(s->m);
  if (s->done.empty() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  int k = 0;
  while (k < max && !s->done.empty()) {
    out[k++] = s->done.front();
    s->done.pop_front();
  }
  *n = k;
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_server_status(nicp_server *s, int *pending, size_t *device_bytes) {
  NICP_ABI_TRY
  if (!s) return NICP_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  if (pending) *pending = s->npending + s->inflight_requests;
  if (device_bytes) {
    size_t b = 0;
    for (auto *c : s->ctxs) b += nicp_ctx_device_bytes(c);
    *device_bytes = b;
  }
  return NICP_OK;
  NICP_ABI_CATCH
}

extern "C" int nicp_server_destroy(nicp_server *s) {
  NICP_ABI_TRY
  if (!s) return NICP_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->threads) t.join();
  for (auto *c : s->all_clouds) nicp_cloud_destroy(c);
  for (auto *c : s->ctxs) nicp_ctx_destroy(c);
  delete s;
  return NICP_OK;
  NICP_ABI_CATCH
}
