// Serving loop: a resident Hash DAG editing a stream of requests with
// continuous batching.
//
// Requests (each a list of sphere / box primitives) are queued in arrival
// order.  A worker thread coalesces every queued request into one batch (up
// to max_batch_prims primitives / max_batch_requests requests), copies it
// from pinned host memory and launches the batched edit on the server's
// stream (one CUDA graph per upload slot, captured at creation, which reads
// the batch size from device memory, so a batch is two copies and one
// launch; batches within the small-edit threshold replay a second graph that
// holds the edit as one cooperative kernel); the copies run on a second stream and overlap the previous edit); up to max_inflight batches are in flight, so requests that arrive
// while the GPU works on one batch are admitted into the next as soon as a
// slot frees, and their upload overlaps the running edit.  A completion
// thread waits for each batch's event, stamps every request of the batch with
// the commit time and the root the batch published.  Batches apply in arrival
// order, so the DAG always equals sequential application of the committed
// requests in arrival order.
//
// Admission by the memory a request needs: edits are copy-on-write, so every
// batch adds nodes to the tables (superseded ones stay until a compaction).
// Each request carries an estimate, per level, of the nodes its primitives
// can create there (the cells their surfaces cross, see estimate_need), and a
// request joins a batch only while the tables' use (exact, from the header of
// the last completed batch) plus the estimates of the batches in flight, of
// the batch so far and of the request stay within compact_at_fill of every
// table's room (index, pool, leaf set).  When not even the first queued
// request fits, the worker waits for the in-flight batches and compacts the
// DAG.  A batch that still runs out of room (status VX_ERR_CAPACITY) is
// recovered: the in-flight batches are drained, their requests requeued in
// order, the DAG compacted and the batch size halved until it fits (a single
// request that cannot fit is reported with its status).
#include "common.cuh"
#include "dag_internal.cuh"
#include "profile.cuh"
#include "tuning.cuh"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

namespace {

uint64_t now_ns() {
  return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(
                                   std::chrono::steady_clock::now().time_since_epoch())
                                   .count());
}

// Estimated new nodes per level (index depth = leaves).
using Need = std::array<double, 16>;

// Upper estimate of the nodes the primitives can create at each level: a
// level-l node is rebuilt only where a primitive cuts its cell partially, and
// those cells lie in the shell of thickness side * sqrt(3) around a sphere's
// surface, or in a box's bounding cells minus its interior ones; each level
// is also capped by the primitive's bounding cells and the level's cell
// count.
Need estimate_need(const vx_primitive *p, size_t n, uint32_t depth) {
  Need need{};
  for (size_t i = 0; i < n; ++i) {
    const uint32_t shape = vx_prim_shape(&p[i]);
    double ext[3];
    for (int a = 0; a < 3; ++a)
      ext[a] = shape == VX_SHAPE_AABB ? double(p[i].r[a])
                                      : 2.0 * double(shape == VX_SHAPE_SPHERE ? p[i].r[0] : p[i].r[a]) + 1.0;
    for (uint32_t l = 1; l <= depth; ++l) {
      const double side = double(4u << (depth - std::min(l, depth)));
      double bbox = 1.0, inner = 1.0;
      for (int a = 0; a < 3; ++a) {
        bbox *= ext[a] / side + 2.0;
        inner *= std::max(0.0, ext[a] / side - 2.0);
      }
      double cells = bbox - inner;
      if (shape == VX_SHAPE_SPHERE) {
        const double r = p[i].r[0], w = side * 1.7320508075688772;
        const double shell = 4.18879020478639 * (std::pow(r + w, 3) - std::pow(std::max(0.0, r - w), 3)) /
                             (side * side * side);
        cells = std::min(bbox, shell);
      }
      need[l] += std::min(cells, std::ldexp(1.0, static_cast<int>(std::min(3 * l, 60u))));
    }
  }
  need[0] = 1.0;
  return need;
}

struct Request {
  uint64_t id;
  uint64_t arrival_ns;
  std::vector<vx_primitive> prims;
  Need need{};
};

struct Batch {
  std::vector<Request> reqs;
  uint32_t nprims = 0;
  int slot = -1;
  cudaEvent_t done = nullptr;
  Need need{};
};

} // namespace

struct vx_server {
  vx_dag *dag = nullptr;
  vx_serve_config cfg{};
  cudaStream_t stream = nullptr;
  int device = 0;
  // two upload slots: pinned host buffer, device buffer, header copy
  vx_primitive *h_buf[2] = {nullptr, nullptr};
  vx_primitive *d_buf[2] = {nullptr, nullptr};
  // per slot: a graph of the batched edit reading its batch size from d_count
  uint32_t *h_count = nullptr; // pinned, one word per slot
  uint32_t *d_count = nullptr; // one word per slot
  vx_graph *graph[2] = {nullptr, nullptr};
  // per slot: the same edit for batches of at most small_cap primitives,
  // captured as the single cooperative kernel of small edits
  vx_graph *graph_small[2] = {nullptr, nullptr};
  uint32_t small_cap = 0;
  // uploads run on their own stream, so a batch's copy overlaps the edit
  // of the batch before it; the edit waits on the slot's upload event
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t uploaded[2] = {nullptr, nullptr};
  unsigned char *h_hdr[2] = {nullptr, nullptr};
  bool slot_busy[2] = {false, false};
  std::vector<unsigned char> last_hdr; // header copy of the last completed batch
  bool have_hdr = false;
  uint32_t depth = 0;

  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request> queue;
  std::deque<Batch> inflight;
  std::vector<vx_serve_completion> done;
  bool stop = false;
  bool recovering = false;
  bool compacted_for_head = false; // the head request got its compaction
  uint32_t batch_cap = 0; // current primitive cap (halved on failures)
  uint32_t hard_cap = 0;  // capacity of the upload buffers
  bool worker_done = false;
  uint64_t submitted = 0, completed = 0;
  vx_serve_stats stats{};
  std::thread worker, completer;
  vx_status fatal = VX_OK;
};

namespace {

// Compact the DAG on the server stream (worker or completion thread; nothing
// in flight), then take a fresh copy of its header for admission.
vx_status compact(vx_server *s) {
  const uint64_t t0 = now_ns();
  vx_status st = vx_dag_status(s->dag, s->stream); // clears a sticky error
  (void)st;
  st = vx_dag_compact(s->dag, s->stream);
  std::vector<unsigned char> hdr(vx::dag::header_bytes());
  const vx_status hs = vx::dag::read_header(s->dag, hdr.data(), s->stream);
  std::lock_guard<std::mutex> lock(s->mu);
  s->stats.compactions += 1;
  s->stats.compact_ms += (now_ns() - t0) * 1e-6;
  s->have_hdr = hs == VX_OK;
  if (s->have_hdr) s->last_hdr.swap(hdr);
  return st;
}

// Whether a batch of estimated need `add` fits in the tables' room on top of
// their use in the last header and the batches in flight (caller holds mu).
bool fits(const vx_server *s, const Need &add) {
  if (!s->have_hdr) return true;
  const vx::dag::TableRoom r = vx::dag::table_room(s->dag, s->last_hdr.data());
  const double f = s->cfg.compact_at_fill;
  for (uint32_t l = 0; l <= r.depth; ++l) {
    double inflight = 0.0;
    for (const Batch &b : s->inflight) inflight += b.need[l];
    const double level_cells = std::ldexp(1.0, static_cast<int>(std::min(3 * l, 60u)));
    const double add_l = std::min(add[l] + inflight, level_cells * (1.0 + s->inflight.size()));
    if (double(r.nodes[l]) + add_l > f * double(r.node_cap[l])) return false;
    if (r.word_cap[l] != 0) {
      // words per new item: the level's average so far, plus one
      const double wpi = (r.nodes[l] ? double(r.words[l]) / double(r.nodes[l]) : 9.0) + 1.0;
      if (double(r.words[l]) + add_l * wpi > f * double(r.word_cap[l])) return false;
    }
  }
  return true;
}

void worker_loop(vx_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    Batch b;
    bool need_compact = false;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv.wait(lock, [&] {
        return (s->stop && s->queue.empty()) ||
               (!s->queue.empty() && !s->recovering &&
                s->inflight.size() < s->cfg.max_inflight &&
                (!s->slot_busy[0] || !s->slot_busy[1]));
      });
      if (s->queue.empty()) { // stop requested and nothing left
        s->worker_done = true;
        break;
      }
      if (!fits(s, s->queue.front().need) && !s->compacted_for_head) {
        // Not even the next request fits: wait for the in-flight batches,
        // then compact (once per head request; if it still does not fit it
        // runs alone and the overflow recovery takes over).
        s->cv.wait(lock, [&] { return s->inflight.empty(); });
        need_compact = true;
        s->compacted_for_head = true;
      } else {
        // Coalesce queued requests in arrival order while they fit.
        while (!s->queue.empty()) {
          Request &r = s->queue.front();
          const uint32_t n = static_cast<uint32_t>(r.prims.size());
          if (!b.reqs.empty()) {
            if (b.nprims + n > s->batch_cap || b.reqs.size() >= s->cfg.max_batch_requests)
              break;
            Need sum = b.need;
            for (uint32_t l = 0; l < 16; ++l) sum[l] += r.need[l];
            if (!fits(s, sum)) break;
          }
          b.nprims += n;
          for (uint32_t l = 0; l < 16; ++l) b.need[l] += r.need[l];
          b.reqs.push_back(std::move(r));
          s->queue.pop_front();
        }
        s->compacted_for_head = false;
        b.slot = s->slot_busy[0] ? 1 : 0;
        s->slot_busy[b.slot] = true;
      }
    }
    if (need_compact) {
      const vx_status st = compact(s);
      if (st != VX_OK) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->fatal = st;
      }
      s->cv.notify_all();
      continue;
    }
    // Upload (pinned -> device) and launch; everything is stream-ordered.
    if (b.nprims > s->hard_cap) {
      // one request larger than the upload buffer: report it as rejected
      std::lock_guard<std::mutex> lock(s->mu);
      for (const Request &r : b.reqs)
        s->done.push_back(vx_serve_completion{r.id, r.arrival_ns, now_ns(),
                                              static_cast<uint32_t>(VX_ERR_CAPACITY), 0});
      s->completed += b.reqs.size();
      s->slot_busy[b.slot] = false;
      s->cv.notify_all();
      continue;
    }
    uint32_t off = 0;
    for (const Request &r : b.reqs) {
      std::memcpy(s->h_buf[b.slot] + off, r.prims.data(), r.prims.size() * sizeof(vx_primitive));
      off += static_cast<uint32_t>(r.prims.size());
    }
    cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming);
    // The slot is not reused before this batch completes, so its buffers
    // (pinned and device) are stable until the copies and the edit ran.
    cudaMemcpyAsync(s->d_buf[b.slot], s->h_buf[b.slot], b.nprims * sizeof(vx_primitive),
                    cudaMemcpyHostToDevice, s->copy_stream);
    s->h_count[b.slot] = b.nprims;
    cudaMemcpyAsync(s->d_count + b.slot, s->h_count + b.slot, sizeof(uint32_t),
                    cudaMemcpyHostToDevice, s->copy_stream);
    cudaEventRecord(s->uploaded[b.slot], s->copy_stream);
    cudaStreamWaitEvent(s->stream, s->uploaded[b.slot], 0);
    if (s->graph_small[b.slot] != nullptr && b.nprims <= s->small_cap) {
      vx_graph_launch(s->graph_small[b.slot], s->stream);
    } else if (s->graph[b.slot] != nullptr) {
      vx_graph_launch(s->graph[b.slot], s->stream);
    } else if (b.nprims) {
      vx_dag_apply_primitives(s->dag, s->d_buf[b.slot], b.nprims, s->stream);
    }
    cudaMemcpyAsync(s->h_hdr[b.slot], vx::dag::device_header(s->dag), vx::dag::header_bytes(),
                    cudaMemcpyDeviceToHost, s->stream);
    cudaEventRecord(b.done, s->stream);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->stats.batches += 1;
      s->stats.prims += b.nprims;
      s->inflight.push_back(std::move(b));
    }
    s->cv.notify_all();
  }
}

void completer_loop(vx_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    cudaEvent_t ev;
    int slot;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv.wait(lock, [&] { return !s->inflight.empty() || s->worker_done; });
      if (s->inflight.empty()) break;
      ev = s->inflight.front().done;
      slot = s->inflight.front().slot;
    }
    cudaEventSynchronize(ev);
    const uint64_t t = now_ns();
    const unsigned char *hh = s->h_hdr[slot];
    const uint32_t status = vx::dag::header_status(hh);
    const uint32_t root = vx::dag::header_root(hh);
    std::unique_lock<std::mutex> lock(s->mu);
    if (status == vx::kDevOk) {
      Batch b = std::move(s->inflight.front());
      s->inflight.pop_front();
      for (const Request &r : b.reqs)
        s->done.push_back(vx_serve_completion{r.id, r.arrival_ns, t, 0u, root});
      s->completed += b.reqs.size();
      s->stats.requests += b.reqs.size();
      s->slot_busy[b.slot] = false;
      s->last_hdr.assign(hh, hh + vx::dag::header_bytes());
      s->have_hdr = true;
      s->batch_cap = s->cfg.max_batch_prims;
      cudaEventDestroy(b.done);
      lock.unlock();
      s->cv.notify_all();
      continue;
    }
    // Failure: every later in-flight batch was skipped by the sticky device
    // status.  Drain, requeue all of them in order, compact, shrink batches.
    s->recovering = true;
    lock.unlock();
    cudaStreamSynchronize(s->stream);
    lock.lock();
    std::deque<Request> again;
    const bool single = s->inflight.front().reqs.size() == 1;
    Batch failed = std::move(s->inflight.front());
    s->inflight.pop_front();
    if (single) {
      // cannot shrink further: report it
      for (const Request &r : failed.reqs)
        s->done.push_back(vx_serve_completion{r.id, r.arrival_ns, t,
                                              static_cast<uint32_t>(vx::status_from_device(status)), 0});
      s->completed += failed.reqs.size();
    } else {
      for (Request &r : failed.reqs) again.push_back(std::move(r));
      s->batch_cap = std::max<uint32_t>(1u, failed.nprims / 2);
    }
    s->slot_busy[failed.slot] = false;
    cudaEventDestroy(failed.done);
    while (!s->inflight.empty()) {
      Batch b = std::move(s->inflight.front());
      s->inflight.pop_front();
      for (Request &r : b.reqs) again.push_back(std::move(r));
      s->slot_busy[b.slot] = false;
      cudaEventDestroy(b.done);
    }
    while (!again.empty()) {
      s->queue.push_front(std::move(again.back()));
      again.pop_back();
    }
    lock.unlock();
    const vx_status cst = compact(s);
    lock.lock();
    if (cst != VX_OK) s->fatal = cst;
    s->recovering = false;
    s->stats.recoveries += 1;
    lock.unlock();
    s->cv.notify_all();
  }
}

} // namespace

extern "C" {

uint64_t vx_serve_now_ns(void) { return now_ns(); }

vx_status vx_serve_create(vx_dag *dag, const vx_serve_config *cfg, vx_server **out) {
  if (dag == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  auto *s = new (std::nothrow) vx_server;
  if (s == nullptr) return VX_ERR_MEMORY_ALLOCATION;
  s->dag = dag;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.max_batch_prims == 0) s->cfg.max_batch_prims = 1u << 16;
  if (s->cfg.max_batch_requests == 0) s->cfg.max_batch_requests = 0xffffffffu;
  if (s->cfg.compact_at_fill <= 0.0) s->cfg.compact_at_fill = 0.9;
  if (s->cfg.max_inflight == 0 || s->cfg.max_inflight > 2) s->cfg.max_inflight = 2;
  // the upload buffers also hold a single request larger than the batch cap
  s->hard_cap = std::max<uint32_t>(s->cfg.max_batch_prims, 1u << 16);
  s->batch_cap = s->cfg.max_batch_prims;
  cudaGetDevice(&s->device);
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k)
    e = cudaEventCreateWithFlags(&s->uploaded[k], cudaEventDisableTiming);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
    e = cudaMallocHost(&s->h_buf[k], s->hard_cap * sizeof(vx_primitive));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_buf[k], s->hard_cap * sizeof(vx_primitive));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_hdr[k], vx::dag::header_bytes());
  }
  if (e == cudaSuccess) e = cudaMallocHost(&s->h_count, 2 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&s->d_count, 2 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    vx_serve_destroy(s);
    return vx::from_cuda(e);
  }
  // A compaction before the first request: its kernels are loaded now (the
  // first launch of a kernel loads its code, a cost no request should wait
  // for), and the tables start without garbage.  An arena too small for it
  // changes nothing and is reported by the first compaction under load.
  {
    const vx_status cs = vx_dag_compact(dag, s->stream);
    if (cs != VX_OK && cs != VX_ERR_CAPACITY) {
      vx_serve_destroy(s);
      return cs;
    }
  }
  // the tables' current use, for admission
  s->last_hdr.resize(vx::dag::header_bytes());
  const vx_status hs = vx::dag::read_header(dag, s->last_hdr.data(), s->stream);
  if (hs != VX_OK) {
    vx_serve_destroy(s);
    return hs;
  }
  s->have_hdr = true;
  s->depth = vx::dag::table_room(dag, s->last_hdr.data()).depth;
  if (s->cfg.launch_mode == 0) {
    s->small_cap = std::min<uint32_t>(
        s->hard_cap, static_cast<uint32_t>(vx::tune::get(vx::tune::kEditSmallMaxPrims)));
    for (int k = 0; k < 2; ++k) {
      vx_status st = vx::dag::graph_primitives_grid(
          dag, s->d_buf[k], s->d_count + k, s->hard_cap,
          static_cast<uint32_t>(vx::tune::get(vx::tune::kServeBlocksPerSm)), &s->graph[k]);
      if (st == VX_OK && s->small_cap > 0)
        st = vx::dag::graph_primitives_grid(dag, s->d_buf[k], s->d_count + k, s->small_cap, 0,
                                            &s->graph_small[k]);
      if (st != VX_OK) {
        vx_serve_destroy(s);
        return st;
      }
    }
  }
  s->worker = std::thread(worker_loop, s);
  s->completer = std::thread(completer_loop, s);
  *out = s;
  return VX_OK;
}

vx_status vx_serve_submit(vx_server *s, uint64_t request_id, const vx_primitive *host_prims,
                          uint32_t count, uint64_t arrival_ns) {
  if (s == nullptr || (host_prims == nullptr && count != 0)) return VX_ERR_INVALID_VALUE;
  Request r;
  r.id = request_id;
  r.arrival_ns = arrival_ns;
  r.prims.assign(host_prims, host_prims + count);
  r.need = estimate_need(host_prims, count, s->depth);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return VX_ERR_INVALID_VALUE;
    s->queue.push_back(std::move(r));
    s->submitted += 1;
  }
  s->cv.notify_all();
  return VX_OK;
}

vx_status vx_serve_poll(vx_server *s, vx_serve_completion *out, uint32_t capacity,
                        uint32_t *n_out) {
  if (s == nullptr || n_out == nullptr || (out == nullptr && capacity != 0))
    return VX_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(s->mu);
  const uint32_t n = static_cast<uint32_t>(std::min<size_t>(capacity, s->done.size()));
  std::copy(s->done.begin(), s->done.begin() + n, out);
  s->done.erase(s->done.begin(), s->done.begin() + n);
  *n_out = n;
  return s->fatal;
}

vx_status vx_serve_drain(vx_server *s) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  std::unique_lock<std::mutex> lock(s->mu);
  s->cv.wait(lock, [&] { return s->completed == s->submitted || s->fatal != VX_OK; });
  return s->fatal;
}

vx_status vx_serve_get_stats(vx_server *s, vx_serve_stats *out) {
  if (s == nullptr || out == nullptr) return VX_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(s->mu);
  *out = s->stats;
  return VX_OK;
}

vx_status vx_serve_destroy(vx_server *s) {
  if (s == nullptr) return VX_ERR_INVALID_VALUE;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->worker_done = true;
  }
  s->cv.notify_all();
  if (s->completer.joinable()) s->completer.join();
  if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (int k = 0; k < 2; ++k) {
    if (s->graph[k]) vx_graph_destroy(s->graph[k]);
    if (s->graph_small[k]) vx_graph_destroy(s->graph_small[k]);
    if (s->h_buf[k]) cudaFreeHost(s->h_buf[k]);
    if (s->d_buf[k]) cudaFree(s->d_buf[k]);
    if (s->h_hdr[k]) cudaFreeHost(s->h_hdr[k]);
  }
  if (s->h_count) cudaFreeHost(s->h_count);
  if (s->d_count) cudaFree(s->d_count);
  for (int k = 0; k < 2; ++k)
    if (s->uploaded[k]) cudaEventDestroy(s->uploaded[k]);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return VX_OK;
}

// Seeded served-request stream of a benchmark mix into host memory (the
// generator of vx_workload.h).  Call with NULL arrays to get the counts.
vx_status vx_generate_requests(const vx_edit_mix *mix, uint64_t seed, double rate,
                               double seconds, double zipf_s, uint32_t max_size,
                               uint64_t max_requests, uint64_t *host_arrival_ns,
                               uint32_t *host_sizes, uint64_t max_prims,
                               vx_primitive *host_prims, uint64_t *host_requests,
                               uint64_t *host_total_prims) {
  if (mix == nullptr || rate <= 0.0 || seconds < 0.0 || max_size == 0 ||
      host_requests == nullptr || host_total_prims == nullptr)
    return VX_ERR_INVALID_VALUE;
  *host_requests = vx_generate_requests_host(mix, seed, rate, seconds, zipf_s, max_size,
                                             max_requests, host_arrival_ns, host_sizes,
                                             max_prims, host_prims, host_total_prims);
  return VX_OK;
}

} // extern "C"
