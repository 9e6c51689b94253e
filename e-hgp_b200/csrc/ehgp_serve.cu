// Serving engine: many point clouds of uneven sizes on one GPU, continuous batching.
//
// The reference plans this as its Python front end's `fit` and a request loop
// (morsehgp3d/docs/GPU_G4_ARCHITECTURE.md:117-136 memory plan at 80 % of the device,
// :269-294 API); it has no batching or serving code.  Here:
//  * a server owns W workers; each worker owns one context (its own CUDA stream and
//    device buffers) and one host thread, and runs one request at a time through the
//    whole chain: canonical cloud + LBVH, Boruvka EMST, pair and triple/quad supports,
//    direct hierarchy of orders 1..K with vertical maps;
//  * submit copies the request's points and queues it; a worker takes the oldest queued
//    request as soon as it is idle and the request fits the memory budget, so requests
//    that arrive while others run are admitted as workers and memory free up, and their
//    device work and host passes overlap with the others' (continuous batching);
//  * admission by memory: every running request reserves an estimate of the device bytes
//    its cloud needs (bytes per point, seeded conservatively and raised to the largest
//    per-point footprint a worker's context has reached); a request is admitted when the
//    reservations stay within hbm_fraction of the device's memory;
//  * a request's LBVH, supports and event state stay on the device while it runs; when it
//    completes, its result (forest nodes with the supports of their levels, child arena,
//    forest batches, final roots, vertical maps, EMST edges) is copied to host memory the
//    request owns, and the worker moves on.
// Results are those of running the same cloud alone: each request runs on a context of its
// own with no state shared with the others.
#include "ehgp_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  int state = EHGP_REQ_QUEUED;
  int status = EHGP_OK;
  std::string error;
  uint64_t n = 0;
  uint32_t K = 10;
  bool f32 = false;
  std::vector<double> xyz64;
  std::vector<float> xyz32;
  uint64_t reserved = 0;
  uint32_t worker = 0;
  Clock::time_point t_submit, t_start, t_end;
  double device_ms = 0;
  // result
  ehgp_hier_counts counts{};
  std::vector<ehgp_forest_node> nodes;
  std::vector<uint32_t> children;
  std::vector<ehgp_forest_batch> batches;
  std::vector<ehgp_forest_root> roots;
  std::vector<ehgp_vertical_assignment> vertical;
  std::vector<uint32_t> node_support;  // 5 words per node
  std::vector<uint32_t> emst_u, emst_v;
};

struct Worker {
  ehgp_ctx* ctx = nullptr;
  std::thread thread;
  uint64_t max_n_seen = 0;
};

}  // namespace

struct ehgp_server {
  int device = 0;
  ehgp_server_limits limits{};
  uint64_t budget = 0;              // bytes the running requests may reserve
  double bytes_per_point = 0;       // admission estimate (raised by measurement)
  uint64_t reserved = 0;            // reservations of the running requests
  std::vector<Worker> workers;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  uint64_t next_id = 1;
  uint64_t admitted = 0, completed = 0, waits_for_memory = 0;
};

namespace {

uint64_t estimate(const ehgp_server& s, uint64_t n) { return (uint64_t)(s.bytes_per_point * (double)n) + (64ull << 20); }

// The whole chain for one request on the worker's context; fills the request's result.
int run_request(ehgp_ctx* ctx, Request& r) {
  if (ehgp_step_begin(ctx) != EHGP_OK) return EHGP_ERR_CUDA;
  ehgp_lbvh_out none{};
  int st = r.f32 ? ehgp_lbvh_build_f32(ctx, r.xyz32.data(), r.n, &none) : ehgp_lbvh_build(ctx, r.xyz64.data(), r.n, &none);
  if (st != EHGP_OK) return st;
  if (r.n >= 2) {
    r.emst_u.resize(r.n - 1);
    r.emst_v.resize(r.n - 1);
    ehgp_emst_out eo{};
    eo.u = r.emst_u.data();
    eo.v = r.emst_v.data();
    if ((st = ehgp_emst(ctx, &eo)) != EHGP_OK) return st;
  }
  st = ehgp_hierarchy(ctx, r.K, &r.counts);
  double ms = 0;
  ehgp_step_end(ctx, &ms);
  r.device_ms = ms;
  if (st != EHGP_OK) return st;
  const ehgp_hier_counts& c = r.counts;
  r.nodes.resize(c.nodes);
  r.children.resize(c.children);
  r.batches.resize(c.journal_batches);
  r.roots.resize(c.final_roots);
  r.vertical.resize(c.vertical_assignments);
  ehgp_hier_out out{};
  out.nodes = r.nodes.data();
  out.children = r.children.data();
  out.batches = r.batches.data();
  out.roots = r.roots.data();
  out.vertical = r.vertical.data();
  if ((st = ehgp_hier_copy(ctx, &out)) != EHGP_OK) return st;
  std::vector<uint32_t> lev(c.nodes);
  for (uint64_t i = 0; i < c.nodes; ++i) lev[i] = r.nodes[i].level_event;
  r.node_support.resize(5 * c.nodes);
  return ehgp_event_supports(ctx, lev.data(), c.nodes, r.node_support.data());
}

void worker_loop(ehgp_server* s, uint32_t w) {
  Worker& me = s->workers[w];
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      for (;;) {
        if (s->stop) return;
        if (!s->queue.empty()) {
          Request* head = s->reqs.at(s->queue.front()).get();
          const uint64_t need = estimate(*s, head->n);
          if (s->reserved + need <= s->budget || s->reserved == 0) {  // FIFO; a lone request always runs
            s->queue.pop_front();
            head->reserved = need;
            s->reserved += need;
            head->state = EHGP_REQ_RUNNING;
            head->worker = w;
            head->t_start = Clock::now();
            ++s->admitted;
            r = head;
            break;
          }
          ++s->waits_for_memory;
        }
        s->cv_work.wait(lock);
      }
    }
    const int st = run_request(me.ctx, *r);
    const uint64_t held = ehgp_ctx_device_bytes(me.ctx);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      me.max_n_seen = std::max(me.max_n_seen, r->n);
      if (st == EHGP_OK && r->n >= 1024)  // the context's footprint per point of the largest cloud it holds
        s->bytes_per_point = std::max(s->bytes_per_point, (double)held / (double)me.max_n_seen);
      r->status = st;
      if (st != EHGP_OK) r->error = ehgp_last_error(me.ctx);
      r->state = st == EHGP_OK ? EHGP_REQ_DONE : EHGP_REQ_FAILED;
      r->t_end = Clock::now();
      s->reserved -= r->reserved;
      r->reserved = 0;
      r->xyz64.clear();
      r->xyz64.shrink_to_fit();
      r->xyz32.clear();
      r->xyz32.shrink_to_fit();
      ++s->completed;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

Request* find(ehgp_server* s, ehgp_request_id id) {
  auto it = s->reqs.find(id);
  return it == s->reqs.end() ? nullptr : it->second.get();
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

extern "C" {

int ehgp_server_create(int device, const ehgp_server_limits* limits, ehgp_server** out) {
  if (!limits || !out || limits->workers == 0 || limits->workers > 64 || limits->max_points == 0 ||
      !(limits->hbm_fraction > 0.0 && limits->hbm_fraction <= 1.0))
    return EHGP_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return EHGP_ERR_CUDA;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return EHGP_ERR_CUDA;
  std::unique_ptr<ehgp_server> s(new ehgp_server());
  s->device = device;
  s->limits = *limits;
  s->budget = (uint64_t)(limits->hbm_fraction * (double)total_b);
  // before any measurement: about 120 KB per point covers the 50,653-point lattice's
  // supports and hierarchy with room
  s->bytes_per_point = 120.0 * 1024.0;
  const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
  for (uint32_t w = 0; w < limits->workers; ++w) {
    ehgp_limits cl{limits->max_points, limits->hbm_fraction};
    Worker wk;
    const int st = ehgp_ctx_create(device, &cl, &wk.ctx);
    if (st != EHGP_OK) {
      for (auto& x : s->workers) ehgp_ctx_destroy(x.ctx);
      return st;
    }
    // the host passes of the workers share the CPUs
    ehgp_hier_schedule(wk.ctx, 0, 0, std::max(12u, hw / limits->workers));
    s->workers.push_back(std::move(wk));
  }
  for (uint32_t w = 0; w < limits->workers; ++w) s->workers[w].thread = std::thread(worker_loop, s.get(), w);
  *out = s.release();
  return EHGP_OK;
}

int ehgp_server_destroy(ehgp_server* s) {
  if (!s) return EHGP_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers)
    if (w.thread.joinable()) w.thread.join();
  for (auto& w : s->workers) ehgp_ctx_destroy(w.ctx);
  delete s;
  return EHGP_OK;
}

int ehgp_cloud_submit(ehgp_server* s, const ehgp_cloud_desc* d, ehgp_request_id* id) {
  if (!s || !d || !id || !d->xyz || d->n == 0 || d->K == 0 || d->K > 10 || d->dtype > 1)
    return EHGP_ERR_INVALID_ARGUMENT;
  if (d->n > s->limits.max_points) return EHGP_ERR_CAPACITY;
  std::unique_ptr<Request> r(new Request());
  r->n = d->n;
  r->K = d->K;
  r->f32 = d->dtype == EHGP_DTYPE_F32;
  if (r->f32) r->xyz32.assign((const float*)d->xyz, (const float*)d->xyz + 3 * d->n);
  else r->xyz64.assign((const double*)d->xyz, (const double*)d->xyz + 3 * d->n);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (estimate(*s, d->n) > s->budget) return EHGP_ERR_OUT_OF_MEMORY;
    r->id = s->next_id++;
    *id = r->id;
    s->queue.push_back(r->id);
    s->reqs.emplace(r->id, std::move(r));
  }
  s->cv_work.notify_one();
  return EHGP_OK;
}

int ehgp_poll(ehgp_server* s, ehgp_request_id id, int32_t* state) {
  if (!s || !state) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  Request* r = find(s, id);
  if (!r) return EHGP_ERR_INVALID_ARGUMENT;
  *state = r->state;
  return EHGP_OK;
}

int ehgp_wait(ehgp_server* s, ehgp_request_id id, uint64_t timeout_ns, int32_t* status) {
  if (!s) return EHGP_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mu);
  Request* r = find(s, id);
  if (!r) return EHGP_ERR_INVALID_ARGUMENT;
  const auto done = [&] { return r->state == EHGP_REQ_DONE || r->state == EHGP_REQ_FAILED; };
  if (!s->cv_done.wait_for(lock, std::chrono::nanoseconds(timeout_ns), done)) return EHGP_ERR_TIMEOUT;
  if (status) *status = r->status;
  return EHGP_OK;
}

int ehgp_request_info(ehgp_server* s, ehgp_request_id id, ehgp_request_stats* info) {
  if (!s || !info) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  Request* r = find(s, id);
  if (!r) return EHGP_ERR_INVALID_ARGUMENT;
  *info = ehgp_request_stats{};
  info->state = r->state;
  info->status = r->status;
  info->points = r->n;
  info->K = r->K;
  info->worker = r->worker;
  const bool started = r->state != EHGP_REQ_QUEUED, ended = r->state == EHGP_REQ_DONE || r->state == EHGP_REQ_FAILED;
  info->queued_ms = started ? ms_between(r->t_submit, r->t_start) : ms_between(r->t_submit, Clock::now());
  info->service_ms = ended ? ms_between(r->t_start, r->t_end) : 0.0;
  info->latency_ms = ended ? ms_between(r->t_submit, r->t_end) : 0.0;
  info->device_ms = r->device_ms;
  info->counts = r->counts;
  return EHGP_OK;
}

const char* ehgp_request_error(ehgp_server* s, ehgp_request_id id) {
  if (!s) return "";
  std::lock_guard<std::mutex> lock(s->mu);
  Request* r = find(s, id);
  return r ? r->error.c_str() : "";
}

int ehgp_result_copy(ehgp_server* s, ehgp_request_id id, const ehgp_served_out* out) {
  if (!s || !out) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  Request* r = find(s, id);
  if (!r) return EHGP_ERR_INVALID_ARGUMENT;
  if (r->state != EHGP_REQ_DONE) return EHGP_ERR_NOT_BUILT;
  auto put = [](auto* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  put(out->nodes, r->nodes);
  put(out->children, r->children);
  put(out->batches, r->batches);
  put(out->roots, r->roots);
  put(out->vertical, r->vertical);
  put(out->node_supports, r->node_support);
  put(out->emst_u, r->emst_u);
  put(out->emst_v, r->emst_v);
  return EHGP_OK;
}

int ehgp_result_release(ehgp_server* s, ehgp_request_id id) {
  if (!s) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return EHGP_ERR_INVALID_ARGUMENT;
  if (it->second->state != EHGP_REQ_DONE && it->second->state != EHGP_REQ_FAILED) return EHGP_ERR_NOT_BUILT;
  s->reqs.erase(it);
  return EHGP_OK;
}

int ehgp_server_info(ehgp_server* s, uint64_t* info, uint32_t count) {
  if (!s || !info) return EHGP_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  uint64_t held = 0, running = 0;
  for (const auto& w : s->workers) held += ehgp_ctx_device_bytes(w.ctx);
  for (const auto& kv : s->reqs) running += kv.second->state == EHGP_REQ_RUNNING;
  const uint64_t v[8] = {s->budget, s->reserved, held, (uint64_t)s->bytes_per_point, s->queue.size(), running,
                         s->completed, s->waits_for_memory};
  for (uint32_t i = 0; i < count && i < 8; ++i) info[i] = v[i];
  return EHGP_OK;
}

}  // extern "C"
