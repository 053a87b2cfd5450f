// Scenes of several rigid bodies and the native continuous-batching server over them: the C-ABI counterparts of the
// reference's Scene (bodies with surfaces and poses, src/warpSPHBoundaries/scene/scene.py:1230-1300), of the fused
// wall aggregate over all its bodies (scene/fused.py:506-547, through scene/provider.py:89-110) and of a request loop
// that keeps scenes resident and batches queries from many simulations (serve.BoundaryServer's scheduling, in C++).
//
// Server scheduling (one host thread drives submit / poll; the server is not thread-safe):
//  * a request is split into work items: one item when it has at most max_batch_rows rows (packable), else chunks of
//    max_batch_rows rows evaluated in place on the caller's arrays;
//  * poll() retires finished batches (their completion events), then fills every free stream slot: the oldest queued
//    item and, when it is packable, every later packable item of the same (scene, kernel, precision, grad) while the
//    rows fit max_batch_rows -- one launch family over the concatenated rows (copies into and out of the slot's
//    persistent buffers);
//  * rows are independent (each row's pairs are summed in a fixed order), so a request's result is bit-identical alone
//    and in any batch;
//  * admission by device memory: a slot's persistent buffers grow on demand only while the server's total stays under
//    hbm_budget; a batch waits for a slot that fits;
//  * a request's inputs are read after the caller's stream reaches the point of submission (an event), and its
//    completion is the batch's end event; latency = completion observed by poll - submission.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace {

using wsb::Surface;

struct SceneBody {
  double pose[4] = {0.0, 0.0, 1.0, 0.0};   // cx, cy, cos, sin
  std::vector<const wsb_surface*> surfaces;
  double obb[4] = {0.0, 0.0, 0.0, 0.0};
  int unbounded = 0;
};

constexpr int kOutputs = 5;                        // lam, G, Cov, m1, m2
constexpr int kOutWidth[kOutputs] = {1, 2, 4, 2, 4};
constexpr int kRowDoubles = 13;                    // sum of kOutWidth

using Clock = std::chrono::steady_clock;

}  // namespace

struct wsb_scene {
  int device = 0;
  std::vector<SceneBody> bodies;
  double* d_pose = nullptr;      // [capacity * 4] device copy of the poses
  int capacity = 0;
};

struct ServeRequest {
  int64_t id = 0;
  const wsb_scene* scene = nullptr;
  int kernel = 0, precision = 0, grad = 0;
  const double* pos = nullptr;
  const double* sup = nullptr;
  int64_t n = 0;
  double* out[kOutputs] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* d_pos = nullptr;
  cudaEvent_t ready = nullptr;   // the caller's stream at submission
  int pending = 0;               // work items not yet completed
  bool done = false;
  Clock::time_point arrival, finished;
};

struct ServeItem {
  int64_t req = 0;
  int64_t r0 = 0, r1 = 0;        // rows [r0, r1) of the request
  bool packable = true;
};

struct ServeSlot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<ServeItem> items;
  int64_t cap = 0;               // rows of the persistent buffers
  int B = 0;                     // bodies the output buffers hold
  double* pos = nullptr;         // [cap * 2]
  double* sup = nullptr;         // [cap]
  double* ones = nullptr;        // [cap]
  double* dpos = nullptr;        // [cap * 2]
  double* out = nullptr;         // [B * cap * 13]: per output a [B, cap, width] block
  size_t buf_bytes = 0;
  void* ws = nullptr;
  size_t ws_bytes = 0;
};

struct wsb_server {
  int device = 0;
  int64_t max_rows = 0;
  size_t budget = 0, reserved = 0;
  std::vector<ServeSlot> slots;
  std::deque<ServeItem> queue;
  std::unordered_map<int64_t, ServeRequest> reqs;
  int64_t next_id = 1;
  std::vector<double> latency_ms;   // completed requests, in completion order
};

namespace wsb {

static void scene_bbox(SceneBody& b) {
  double lo_x = INFINITY, lo_y = INFINITY, hi_x = -INFINITY, hi_y = -INFINITY;
  int unb = 0;
  for (const wsb_surface* s_ : b.surfaces) {
    const Surface* s = reinterpret_cast<const Surface*>(s_);
    lo_x = std::min(lo_x, s->bbox[0]);
    lo_y = std::min(lo_y, s->bbox[1]);
    hi_x = std::max(hi_x, s->bbox[2]);
    hi_y = std::max(hi_y, s->bbox[3]);
    unb |= s->background != 0;
  }
  b.obb[0] = lo_x;
  b.obb[1] = lo_y;
  b.obb[2] = hi_x;
  b.obb[3] = hi_y;
  b.unbounded = unb;
}

static size_t scene_ws_bytes(const wsb_scene* sc, int64_t n) {
  size_t need = 0;
  for (const SceneBody& b : sc->bodies)
    for (const wsb_surface* s : b.surfaces)
      need = std::max(need, wsb_aggregate_workspace_size(s, n) + wsb_aggregate_staging_size(s, n));
  return need;
}

// every body's outputs of n rows: per group g and output k the array out_k[g] + b * ld * width_k (row stride ld)
static int scene_aggregate(const wsb_scene* sc, int n_groups, const int32_t* kernels, int precision, const double* pos,
                           const double* sup, const int32_t* allowed, int64_t n, int64_t ld, double* const* outs[5],
                           void* ws, size_t ws_bytes, cudaStream_t st) {
  std::vector<double*> ptr[kOutputs];
  for (int k = 0; k < kOutputs; ++k) ptr[k].resize(n_groups);
  for (size_t b = 0; b < sc->bodies.size(); ++b) {
    const SceneBody& body = sc->bodies[b];
    for (int k = 0; k < kOutputs; ++k)
      for (int g = 0; g < n_groups; ++g)
        ptr[k][g] = outs[k] && outs[k][g] ? outs[k][g] + (int64_t)b * ld * kOutWidth[k] : nullptr;
    if (body.surfaces.empty()) {                       // a body without surfaces: zeros
      for (int k = 0; k < kOutputs; ++k)
        for (int g = 0; g < n_groups; ++g)
          if (ptr[k][g]) WSB_CUDA(cudaMemsetAsync(ptr[k][g], 0, sizeof(double) * n * kOutWidth[k], st));
      continue;
    }
    for (size_t ri = 0; ri < body.surfaces.size(); ++ri) {
      const int mode = WSB_OUT_ALL | (ri == 0 ? WSB_OUT_ASSIGN : 0);     // the first surface assigns, the rest add
      const int rc = wsb_aggregate_groups(body.surfaces[ri], n_groups, kernels, precision, pos, sup, allowed, n,
                                          sc->d_pose + 4 * b, body.obb, body.unbounded, mode, ptr[0].data(),
                                          ptr[1].data(), ptr[2].data(), ptr[3].data(), ptr[4].data(), ws, ws_bytes, st);
      if (rc) return rc;
    }
  }
  return WSB_OK;
}

// d sum(lam) / dx of n rows summed over every body and surface, ADDED into d_pos (ones: n device ones)
static int scene_backward(const wsb_scene* sc, int kernel, const double* pos, const double* sup, int64_t n,
                          const double* ones, double* d_pos, void* ws, size_t ws_bytes, cudaStream_t st) {
  for (size_t b = 0; b < sc->bodies.size(); ++b) {
    const SceneBody& body = sc->bodies[b];
    for (const wsb_surface* s : body.surfaces) {
      const int rc = wsb_aggregate_backward(s, kernel, pos, sup, nullptr, n, sc->d_pose + 4 * b, body.obb,
                                            body.unbounded, ones, nullptr, nullptr, d_pos, nullptr, ws, ws_bytes, st);
      if (rc) return rc;
    }
  }
  return WSB_OK;
}

static size_t slot_buffer_bytes(int64_t cap, int B) {
  return sizeof(double) * (size_t)cap * (2 + 1 + 1 + 2 + (size_t)B * kRowDoubles);
}

static void slot_free(ServeSlot& s) {
  cudaFree(s.pos);
  cudaFree(s.ws);
  s.pos = s.sup = s.ones = s.dpos = s.out = nullptr;
  s.ws = nullptr;
  s.buf_bytes = s.ws_bytes = 0;
  s.cap = 0;
  s.B = 0;
}

// grow a slot's persistent buffers for B bodies x cap rows and a workspace of ws bytes, within the server's budget;
// returns 1 when the slot is ready, 0 when the budget has no room (the batch waits), < 0 on an error
static int slot_fit(wsb_server* srv, ServeSlot& s, int B, size_t ws) {
  const int64_t cap = srv->max_rows;
  const bool grow_buf = s.cap < cap || s.B < B;
  const bool grow_ws = s.ws_bytes < ws;
  if (!grow_buf && !grow_ws) return 1;
  const size_t nb = grow_buf ? slot_buffer_bytes(cap, std::max(B, s.B)) : s.buf_bytes;
  const size_t nw = grow_ws ? ws : s.ws_bytes;
  const size_t after = srv->reserved - s.buf_bytes - s.ws_bytes + nb + nw;
  if (after > srv->budget) return 0;
  if (grow_buf) {
    WSB_CUDA(cudaStreamSynchronize(s.stream));
    srv->reserved -= s.buf_bytes;
    cudaFree(s.pos);
    s.pos = nullptr;
    s.buf_bytes = 0;
    void* p = nullptr;
    WSB_CUDA(cudaMalloc(&p, nb));
    const int Bn = std::max(B, s.B);
    s.pos = static_cast<double*>(p);
    s.sup = s.pos + 2 * cap;
    s.ones = s.sup + cap;
    s.dpos = s.ones + cap;
    s.out = s.dpos + 2 * cap;
    s.cap = cap;
    s.B = Bn;
    s.buf_bytes = nb;
    srv->reserved += nb;
    std::vector<double> one((size_t)cap, 1.0);
    WSB_CUDA(cudaMemcpy(s.ones, one.data(), sizeof(double) * cap, cudaMemcpyHostToDevice));
  }
  if (grow_ws) {
    WSB_CUDA(cudaStreamSynchronize(s.stream));
    srv->reserved -= s.ws_bytes;
    cudaFree(s.ws);
    s.ws = nullptr;
    s.ws_bytes = 0;
    WSB_CUDA(cudaMalloc(&s.ws, nw));
    s.ws_bytes = nw;
    srv->reserved += nw;
  }
  return 1;
}

// launch one batch of work items (all of one (scene, kernel, precision, grad); packable ones copied through the slot's
// buffers, an in-place chunk straight on the request's arrays) on slot s
static int slot_launch(wsb_server* srv, ServeSlot& s, const std::vector<ServeItem>& items) {
  const ServeRequest& first = srv->reqs[items[0].req];
  const wsb_scene* sc = first.scene;
  const int B = (int)sc->bodies.size();
  const int32_t kern = first.kernel;
  cudaStream_t st = s.stream;
  for (const ServeItem& it : items) WSB_CUDA(cudaStreamWaitEvent(st, srv->reqs[it.req].ready, 0));
  if (!items[0].packable) {                          // a chunk of a large request, in place
    const ServeItem& it = items[0];
    const ServeRequest& r = first;
    const int64_t m = it.r1 - it.r0;
    double* const* o[kOutputs];
    double* p[kOutputs];
    for (int k = 0; k < kOutputs; ++k) {
      p[k] = r.out[k] ? r.out[k] + it.r0 * kOutWidth[k] : nullptr;
      o[k] = &p[k];
    }
    int rc = scene_aggregate(sc, 1, &kern, r.precision, r.pos + 2 * it.r0, r.sup + it.r0, nullptr, m, r.n, o, s.ws,
                             s.ws_bytes, st);
    if (rc) return rc;
    if (r.grad) {
      WSB_CUDA(cudaMemsetAsync(r.d_pos + 2 * it.r0, 0, sizeof(double) * 2 * m, st));
      rc = scene_backward(sc, kern, r.pos + 2 * it.r0, r.sup + it.r0, m, s.ones, r.d_pos + 2 * it.r0, s.ws, s.ws_bytes,
                          st);
      if (rc) return rc;
    }
  } else {
    int64_t rows = 0;
    for (const ServeItem& it : items) {
      const ServeRequest& r = srv->reqs[it.req];
      WSB_CUDA(cudaMemcpyAsync(s.pos + 2 * rows, r.pos, sizeof(double) * 2 * r.n, cudaMemcpyDeviceToDevice, st));
      WSB_CUDA(cudaMemcpyAsync(s.sup + rows, r.sup, sizeof(double) * r.n, cudaMemcpyDeviceToDevice, st));
      rows += r.n;
    }
    double* base[kOutputs];
    double* const* o[kOutputs];
    size_t off = 0;
    for (int k = 0; k < kOutputs; ++k) {
      base[k] = s.out + off;
      o[k] = &base[k];
      off += (size_t)B * s.cap * kOutWidth[k];
    }
    int rc = scene_aggregate(sc, 1, &kern, first.precision, s.pos, s.sup, nullptr, rows, s.cap, o, s.ws, s.ws_bytes, st);
    if (rc) return rc;
    if (first.grad) {
      WSB_CUDA(cudaMemsetAsync(s.dpos, 0, sizeof(double) * 2 * rows, st));
      rc = scene_backward(sc, kern, s.pos, s.sup, rows, s.ones, s.dpos, s.ws, s.ws_bytes, st);
      if (rc) return rc;
    }
    int64_t at = 0;
    for (const ServeItem& it : items) {
      const ServeRequest& r = srv->reqs[it.req];
      for (int k = 0; k < kOutputs; ++k) {
        if (!r.out[k]) continue;
        const int w = kOutWidth[k];
        // the request's [B, n, w] block from rows [at, at + n) of the slot's [B, cap, w] block
        WSB_CUDA(cudaMemcpy2DAsync(r.out[k], sizeof(double) * r.n * w, base[k] + at * w, sizeof(double) * s.cap * w,
                                   sizeof(double) * r.n * w, B, cudaMemcpyDeviceToDevice, st));
      }
      if (r.grad)
        WSB_CUDA(cudaMemcpyAsync(r.d_pos, s.dpos + 2 * at, sizeof(double) * 2 * r.n, cudaMemcpyDeviceToDevice, st));
      at += r.n;
    }
  }
  WSB_CUDA(cudaEventRecord(s.done, st));
  s.items = items;
  s.busy = true;
  return WSB_OK;
}

static bool same_key(const ServeRequest& a, const ServeRequest& b) {
  return a.scene == b.scene && a.kernel == b.kernel && a.precision == b.precision && a.grad == b.grad;
}

static int fill_slots(wsb_server* srv, bool* launched);

static int server_step(wsb_server* srv) {
  // retire finished batches
  for (ServeSlot& s : srv->slots) {
    if (!s.busy) continue;
    const cudaError_t q = cudaEventQuery(s.done);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return cuda_fail(q, "wsb_serve_poll: batch");
    const Clock::time_point now = Clock::now();
    for (const ServeItem& it : s.items) {
      ServeRequest& r = srv->reqs[it.req];
      if (--r.pending == 0) {
        r.done = true;
        r.finished = now;
        srv->latency_ms.push_back(std::chrono::duration<double, std::milli>(now - r.arrival).count());
      }
    }
    s.items.clear();
    s.busy = false;
  }
  bool launched = false;
  int rc = fill_slots(srv, &launched);
  if (rc) return rc;
  bool busy = false;
  for (const ServeSlot& s : srv->slots) busy = busy || s.busy;
  if (!busy && !srv->queue.empty()) {
    // nothing runs and the head fits in no slot next to the others' buffers: the idle slots give their memory back
    for (ServeSlot& s : srv->slots) {
      srv->reserved -= s.buf_bytes + s.ws_bytes;
      slot_free(s);
    }
    rc = fill_slots(srv, &launched);
    if (rc) return rc;
    if (!launched) return fail(WSB_ERR_SIZE, "wsb_serve: a batch does not fit the server's budget");
  }
  return WSB_OK;
}

static int fill_slots(wsb_server* srv, bool* launched) {
  for (ServeSlot& s : srv->slots) {
    if (s.busy || srv->queue.empty()) continue;
    const ServeItem head = srv->queue.front();
    const ServeRequest& hr = srv->reqs[head.req];
    const int B = (int)hr.scene->bodies.size();
    const int fit = slot_fit(srv, s, B, scene_ws_bytes(hr.scene, srv->max_rows));
    if (fit < 0) return fit;
    if (fit == 0) continue;                          // no room under the budget in this slot now
    std::vector<ServeItem> batch{head};
    srv->queue.pop_front();
    if (head.packable) {
      int64_t rows = head.r1 - head.r0;
      for (auto it = srv->queue.begin(); it != srv->queue.end();) {
        const ServeRequest& r = srv->reqs[it->req];
        if (it->packable && same_key(r, hr) && rows + (it->r1 - it->r0) <= srv->max_rows) {
          rows += it->r1 - it->r0;
          batch.push_back(*it);
          it = srv->queue.erase(it);
        } else {
          ++it;
        }
      }
    }
    const int rc = slot_launch(srv, s, batch);
    if (rc) return rc;
    *launched = true;
  }
  return WSB_OK;
}

}  // namespace wsb

using namespace wsb;

// ------------------------------------------------------------------------------------------------ scenes
extern "C" int wsb_scene_create(int device, wsb_scene** out) {
  if (!out) return fail(WSB_ERR_ARG, "wsb_scene_create: NULL out");
  *out = nullptr;
  int count = 0;
  WSB_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(WSB_ERR_ARG, "wsb_scene_create: no device " + std::to_string(device));
  wsb_scene* sc = new wsb_scene();
  sc->device = device;
  *out = sc;
  return WSB_OK;
}

extern "C" int wsb_scene_destroy(wsb_scene* sc) {
  if (!sc) return WSB_OK;
  if (sc->d_pose) {
    cudaSetDevice(sc->device);
    cudaFree(sc->d_pose);
  }
  delete sc;
  return WSB_OK;
}

extern "C" int wsb_scene_add_body(wsb_scene* sc, const double* pose, int* body) {
  if (!sc || !pose) return fail(WSB_ERR_ARG, "wsb_scene_add_body: NULL argument");
  for (int k = 0; k < 4; ++k)
    if (!std::isfinite(pose[k])) return fail(WSB_ERR_ARG, "wsb_scene_add_body: non-finite pose");
  WSB_CUDA(cudaSetDevice(sc->device));
  const int B = (int)sc->bodies.size();
  if (B + 1 > sc->capacity) {
    const int cap = std::max(4, 2 * sc->capacity);
    double* p = nullptr;
    WSB_CUDA(cudaMalloc(&p, sizeof(double) * 4 * cap));
    if (sc->d_pose) {
      WSB_CUDA(cudaMemcpy(p, sc->d_pose, sizeof(double) * 4 * B, cudaMemcpyDeviceToDevice));
      cudaFree(sc->d_pose);
    }
    sc->d_pose = p;
    sc->capacity = cap;
  }
  SceneBody b;
  for (int k = 0; k < 4; ++k) b.pose[k] = pose[k];
  sc->bodies.push_back(b);
  WSB_CUDA(cudaMemcpy(sc->d_pose + 4 * B, pose, sizeof(double) * 4, cudaMemcpyHostToDevice));
  if (body) *body = B;
  return WSB_OK;
}

extern "C" int wsb_scene_add_surface(wsb_scene* sc, int body, const wsb_surface* s_) {
  if (!sc || !s_) return fail(WSB_ERR_ARG, "wsb_scene_add_surface: NULL argument");
  if (body < 0 || body >= (int)sc->bodies.size()) return fail(WSB_ERR_ARG, "wsb_scene_add_surface: no such body");
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (s->device != sc->device) return fail(WSB_ERR_ARG, "wsb_scene_add_surface: the surface lives on another device");
  sc->bodies[body].surfaces.push_back(s_);
  scene_bbox(sc->bodies[body]);
  return WSB_OK;
}

extern "C" int wsb_scene_set_pose(wsb_scene* sc, int body, const double* pose, void* stream) {
  if (!sc || !pose) return fail(WSB_ERR_ARG, "wsb_scene_set_pose: NULL argument");
  if (body < 0 || body >= (int)sc->bodies.size()) return fail(WSB_ERR_ARG, "wsb_scene_set_pose: no such body");
  for (int k = 0; k < 4; ++k)
    if (!std::isfinite(pose[k])) return fail(WSB_ERR_ARG, "wsb_scene_set_pose: non-finite pose");
  WSB_CUDA(cudaSetDevice(sc->device));
  for (int k = 0; k < 4; ++k) sc->bodies[body].pose[k] = pose[k];
  WSB_CUDA(cudaMemcpyAsync(sc->d_pose + 4 * body, pose, sizeof(double) * 4, cudaMemcpyHostToDevice,
                           (cudaStream_t)stream));
  WSB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));      // the host array may go away after the call
  return WSB_OK;
}

extern "C" int wsb_scene_info(const wsb_scene* sc, int* n_bodies, int* n_surfaces) {
  if (!sc) return fail(WSB_ERR_ARG, "wsb_scene_info: NULL scene");
  if (n_bodies) *n_bodies = (int)sc->bodies.size();
  if (n_surfaces) {
    int m = 0;
    for (const SceneBody& b : sc->bodies) m += (int)b.surfaces.size();
    *n_surfaces = m;
  }
  return WSB_OK;
}

extern "C" size_t wsb_scene_workspace_size(const wsb_scene* sc, int64_t n) {
  if (!sc || n < 0) return 0;
  return scene_ws_bytes(sc, n);
}

extern "C" int wsb_scene_aggregate(const wsb_scene* sc, int n_groups, const int32_t* kernels, int precision,
                                   const double* pos, const double* sup, const int32_t* allowed, int64_t n, int64_t ld,
                                   double* const* lam, double* const* G, double* const* cov, double* const* m1,
                                   double* const* m2, void* workspace, size_t workspace_bytes, void* stream) {
  if (!sc) return fail(WSB_ERR_ARG, "wsb_scene_aggregate: NULL scene");
  if (n_groups < 1 || n_groups > WSB_MAX_GROUPS || !kernels)
    return fail(WSB_ERR_ARG, "wsb_scene_aggregate: 1 to " + std::to_string(WSB_MAX_GROUPS) + " kernel groups expected");
  if (n < 0 || ld < n) return fail(WSB_ERR_ARG, "wsb_scene_aggregate: need 0 <= n <= ld");
  if (n == 0) return WSB_OK;
  if (!pos || !sup) return fail(WSB_ERR_ARG, "wsb_scene_aggregate: NULL array");
  if (workspace_bytes < scene_ws_bytes(sc, n) || !workspace)
    return fail(WSB_ERR_SIZE, "wsb_scene_aggregate: workspace of " + std::to_string(workspace_bytes) + " bytes, need " +
                                  std::to_string(scene_ws_bytes(sc, n)));
  WSB_CUDA(cudaSetDevice(sc->device));
  double* const* outs[kOutputs] = {lam, G, cov, m1, m2};
  return scene_aggregate(sc, n_groups, kernels, precision, pos, sup, allowed, n, ld, outs, workspace, workspace_bytes,
                         (cudaStream_t)stream);
}

// ------------------------------------------------------------------------------------------------ server
extern "C" int wsb_server_create(int device, int n_streams, int64_t max_batch_rows, size_t hbm_budget,
                                 wsb_server** out) {
  if (!out) return fail(WSB_ERR_ARG, "wsb_server_create: NULL out");
  *out = nullptr;
  if (n_streams < 1 || n_streams > 64) return fail(WSB_ERR_ARG, "wsb_server_create: 1 to 64 streams");
  if (max_batch_rows < 1 || max_batch_rows > (int64_t)INT32_MAX)
    return fail(WSB_ERR_ARG, "wsb_server_create: max_batch_rows out of range");
  int count = 0;
  WSB_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(WSB_ERR_ARG, "wsb_server_create: no device " + std::to_string(device));
  WSB_CUDA(cudaSetDevice(device));
  wsb_server* srv = new wsb_server();
  srv->device = device;
  srv->max_rows = max_batch_rows;
  srv->budget = hbm_budget;
  srv->slots.resize(n_streams);
  for (ServeSlot& s : srv->slots) {
    cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      wsb_server_destroy(srv);
      return cuda_fail(e, "wsb_server_create");
    }
  }
  *out = srv;
  return WSB_OK;
}

extern "C" int wsb_server_destroy(wsb_server* srv) {
  if (!srv) return WSB_OK;
  cudaSetDevice(srv->device);
  for (ServeSlot& s : srv->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    slot_free(s);
    if (s.done) cudaEventDestroy(s.done);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  for (auto& kv : srv->reqs)
    if (kv.second.ready) cudaEventDestroy(kv.second.ready);
  delete srv;
  return WSB_OK;
}

extern "C" int wsb_serve_submit(wsb_server* srv, const wsb_scene* sc, int kernel, int precision, int grad,
                                const double* pos, const double* sup, int64_t n, double* lam, double* G, double* cov,
                                double* m1, double* m2, double* d_pos, void* stream, int64_t* request_id) {
  if (!srv || !sc || !request_id) return fail(WSB_ERR_ARG, "wsb_serve_submit: NULL argument");
  *request_id = 0;
  if (sc->device != srv->device) return fail(WSB_ERR_ARG, "wsb_serve_submit: the scene lives on another device");
  if (kernel < 0 || kernel >= kNumKernels) return fail(WSB_ERR_UNSUPPORTED, "wsb_serve_submit: unknown kernel id");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_serve_submit: unknown precision mode");
  if (n < 1 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_serve_submit: row count out of range");
  if (!pos || !sup) return fail(WSB_ERR_ARG, "wsb_serve_submit: NULL positions or supports");
  if (grad && !d_pos) return fail(WSB_ERR_ARG, "wsb_serve_submit: grad needs d_pos");
  const int B = (int)sc->bodies.size();
  const size_t need = slot_buffer_bytes(srv->max_rows, B) + scene_ws_bytes(sc, srv->max_rows);
  if (need > srv->budget)
    return fail(WSB_ERR_SIZE, "wsb_serve_submit: one batch slot for this scene needs " + std::to_string(need) +
                                  " bytes, the server's budget is " + std::to_string(srv->budget));
  WSB_CUDA(cudaSetDevice(srv->device));
  ServeRequest r;
  r.id = srv->next_id++;
  r.scene = sc;
  r.kernel = kernel;
  r.precision = precision;
  r.grad = grad != 0;
  r.pos = pos;
  r.sup = sup;
  r.n = n;
  double* o[kOutputs] = {lam, G, cov, m1, m2};
  for (int k = 0; k < kOutputs; ++k) r.out[k] = o[k];
  r.d_pos = d_pos;
  WSB_CUDA(cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming));
  WSB_CUDA(cudaEventRecord(r.ready, (cudaStream_t)stream));
  r.arrival = Clock::now();
  if (n <= srv->max_rows) {
    srv->queue.push_back(ServeItem{r.id, 0, n, true});
    r.pending = 1;
  } else {
    for (int64_t r0 = 0; r0 < n; r0 += srv->max_rows) {
      srv->queue.push_back(ServeItem{r.id, r0, std::min(n, r0 + srv->max_rows), false});
      ++r.pending;
    }
  }
  srv->reqs[r.id] = r;
  *request_id = r.id;
  return server_step(srv);
}

extern "C" int wsb_serve_poll(wsb_server* srv, int64_t request_id, int* done) {
  if (!srv) return fail(WSB_ERR_ARG, "wsb_serve_poll: NULL server");
  WSB_CUDA(cudaSetDevice(srv->device));
  const int rc = server_step(srv);
  if (rc) return rc;
  if (done) {
    *done = 0;
    if (request_id > 0) {
      auto it = srv->reqs.find(request_id);
      if (it == srv->reqs.end()) return fail(WSB_ERR_ARG, "wsb_serve_poll: unknown request " + std::to_string(request_id));
      *done = it->second.done ? 1 : 0;
    } else {
      bool idle = srv->queue.empty();
      for (const ServeSlot& s : srv->slots) idle = idle && !s.busy;
      *done = idle ? 1 : 0;
    }
  }
  return WSB_OK;
}

extern "C" int wsb_serve_wait(wsb_server* srv, int64_t request_id) {
  if (!srv) return fail(WSB_ERR_ARG, "wsb_serve_wait: NULL server");
  for (;;) {
    int done = 0;
    const int rc = wsb_serve_poll(srv, request_id, &done);
    if (rc) return rc;
    if (done) return WSB_OK;
    bool any = false;
    for (ServeSlot& s : srv->slots)
      if (s.busy) {
        WSB_CUDA(cudaEventSynchronize(s.done));
        any = true;
        break;
      }
    if (!any && srv->queue.empty() && request_id > 0)
      return fail(WSB_ERR_ARG, "wsb_serve_wait: request " + std::to_string(request_id) + " is neither queued nor running");
  }
}

extern "C" int wsb_serve_release(wsb_server* srv, int64_t request_id) {
  if (!srv) return fail(WSB_ERR_ARG, "wsb_serve_release: NULL server");
  auto it = srv->reqs.find(request_id);
  if (it == srv->reqs.end()) return fail(WSB_ERR_ARG, "wsb_serve_release: unknown request");
  if (!it->second.done) return fail(WSB_ERR_ARG, "wsb_serve_release: the request has not completed");
  cudaEventDestroy(it->second.ready);
  srv->reqs.erase(it);
  return WSB_OK;
}

extern "C" int wsb_server_stats(const wsb_server* srv, int64_t* completed, double* p50_ms, double* p99_ms,
                                size_t* reserved_bytes) {
  if (!srv) return fail(WSB_ERR_ARG, "wsb_server_stats: NULL server");
  std::vector<double> v = srv->latency_ms;
  if (completed) *completed = (int64_t)v.size();
  auto pct = [&](double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t k = std::min(v.size() - 1, (size_t)std::ceil(q * (double)v.size()) - (q > 0 ? 1 : 0));
    return v[k];
  };
  if (p50_ms) *p50_ms = pct(0.50);
  if (p99_ms) *p99_ms = pct(0.99);
  if (reserved_bytes) *reserved_bytes = srv->reserved;
  return WSB_OK;
}
