// server.cu -- request loop: MCE jobs on different graphs admitted by
// estimated HBM footprint, run concurrently on the device.
//
// No reference counterpart.  Continuous batching: a request queued while others
// run is admitted as soon as a worker slot and enough of the memory budget are
// free; each worker owns a CUDA stream and a scratch context, so the GPU
// preprocessing and the enumeration of admitted requests overlap on the
// device.  Each request's grid is capped so concurrent requests share the SMs.
// Admission takes the oldest queued request that fits (a large request does
// not block smaller ones behind it; it is admitted when the budget frees up).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  std::vector<uint32_t> u, v;
  uint64_t est_bytes = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  uint32_t share = 1;  // requests running on the device when this one was admitted (itself included)
  mce_status status = MCE_OK;
  std::unique_ptr<mce_result> result;
  Clock::time_point t_submit, t_done;
  double dev_start_ms = -1, dev_end_ms = -1;  // device clock, from the server's base event
};

}  // namespace

struct mce_server {
  mce_server_options opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
  std::vector<std::thread> workers;
  uint64_t budget = 0, in_use = 0, next_id = 1;
  uint32_t running = 0;
  bool stop = false;
  int sms = 148;
  // recorded (and completed) at creation: request spans are measured from it
  // on the device's own clock
  cudaEvent_t base = nullptr;
};

namespace mce {
namespace {

constexpr uint32_t kServeBlocksPerSm = 4;  // the enumeration kernel's residency

uint64_t estimate_bytes(const Request &r) {
  uint32_t maxlab = 0;
  for (size_t i = 0; i < r.u.size(); i++) maxlab = std::max(maxlab, std::max(r.u[i], r.v[i]));
  // pairs on device and the sort buffers (~12 words per pair), the label map,
  // the CSR and root arrays, plus the enumeration scratch of a capped grid
  return 96ULL * r.u.size() + 8ULL * ((uint64_t)maxlab + 1) + (256ULL << 20);
}

void run_request(mce_server *s, Request *r, cudaStream_t st, Scratch *scr) {
  DeviceGraph g;
  mce_status rc = MCE_OK;
  const uint64_t np = r->u.size();
  const size_t bytes = std::max<uint64_t>(np, 1) * 4;
  auto t0 = Clock::now();
  // the request's device span: from before its upload to after its results
  // are read back, on the worker's stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess) rc = MCE_ERR_CUDA;
  if (ev0) cudaEventRecord(ev0, st);
  // the request's pairs go to the worker's kept scratch (grown on demand and
  // reused by later requests), so a request of a size seen before allocates
  // nothing here
  uint32_t *ud = (uint32_t *)scr->get(7, 2 * bytes, &rc);
  uint32_t *vd = ud ? ud + bytes / 4 : nullptr;
  if (rc == MCE_OK && np &&
      (cudaMemcpyAsync(ud, r->u.data(), np * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
       cudaMemcpyAsync(vd, r->v.data(), np * 4, cudaMemcpyHostToDevice, st) != cudaSuccess))
    rc = MCE_ERR_CUDA;
  if (rc == MCE_OK) rc = build_from_pairs(ud, vd, np, MCE_ORDER_DEGENERACY, 1ULL << 34, st, &g);
  auto t1 = Clock::now();
  std::unique_ptr<mce_result> res(new mce_result());
  std::memset(res.get(), 0, sizeof(mce_result));
  if (rc == MCE_OK) {
    const size_t res_bytes = sizeof(SlotResult) + MCE_HIST_LEN * sizeof(unsigned long long);
    char *dres = (char *)scr->get(0, res_bytes, &rc);
    if (dres && cudaMemsetAsync(dres, 0, res_bytes, st) != cudaSuccess) rc = MCE_ERR_CUDA;
    if (rc == MCE_OK) {
      EnumConfig cfg;
      // A request admitted onto an idle device gets the whole GPU; one admitted
      // beside k others gets 1/(k+1) of it (at least one block per SM), so
      // concurrent persistent grids fit on the SMs side by side.
      const uint32_t full = (uint32_t)s->sms * kServeBlocksPerSm;
      cfg.max_blocks = std::max<uint32_t>(full / std::max<uint32_t>(r->share, 1), (uint32_t)s->sms);
      EnumStats stats;
      rc = enumerate(g, cfg, scr, st, (SlotResult *)dres, (unsigned long long *)(dres + sizeof(SlotResult)), &stats);
      if (rc == MCE_OK) {
        SlotResult hs;
        if (cudaMemcpyAsync(&hs, dres, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(res->hist, dres + sizeof(SlotResult), MCE_HIST_LEN * 8, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
          rc = MCE_ERR_CUDA;
        res->count = hs.count;
        res->checksum = hs.checksum;
        res->max_size = hs.max_size;
        res->roots = stats.roots;
        res->heavy_roots = stats.heavy_roots;
        res->phase_ms[MCE_PHASE_ENUMERATE] = stats.ms_enum;
      }
    }
  }
  res->num_vertices = g.n;
  res->num_edges = g.m;
  res->max_degree = g.max_degree;
  res->degeneracy = g.degeneracy;
  res->phase_ms[MCE_PHASE_PREPROCESS] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  free_graph(&g);
  float span0 = -1, span1 = -1;
  if (ev1) {
    cudaEventRecord(ev1, st);
    if (cudaEventSynchronize(ev1) != cudaSuccess || cudaEventElapsedTime(&span0, s->base, ev0) != cudaSuccess ||
        cudaEventElapsedTime(&span1, s->base, ev1) != cudaSuccess)
      span0 = span1 = -1;
  }
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  cudaStreamSynchronize(st);
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(s->mu);
  r->dev_start_ms = span0;
  r->dev_end_ms = span1;
  r->status = rc;
  r->result = std::move(res);
  r->t_done = Clock::now();
  r->result->phase_ms[MCE_PHASE_TOTAL] = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  r->state = 2;
  r->u.clear();
  r->u.shrink_to_fit();
  r->v.clear();
  r->v.shrink_to_fit();
}

void worker_main(mce_server *s) {
  cudaSetDevice(s->opt.device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  Scratch scr;
  scr.device = s->opt.device;
  for (;;) {
    Request *r = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stop) break;
        // oldest queued request whose footprint fits the free budget; an
        // oversize request runs alone once the device is otherwise idle
        for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
          Request *q = *it;
          if (s->in_use + q->est_bytes <= s->budget || s->running == 0) {
            r = q;
            s->queue.erase(it);
            break;
          }
        }
        if (r) break;
        s->cv_work.wait(lk);
      }
      if (!r) break;
      r->state = 1;
      s->in_use += r->est_bytes;
      s->running++;
      r->share = s->running;
    }
    run_request(s, r, st, &scr);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= r->est_bytes;
      s->running--;
    }
    // The worker keeps its scratch for the next request: freeing device memory
    // would synchronise the whole device and stall the other requests.
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  scr.release();
  cudaStreamDestroy(st);
}

}  // namespace
}  // namespace mce

extern "C" {

mce_status mce_server_create(const mce_server_options *opt, mce_server **out) {
  if (!out) return MCE_ERR_INVALID_ARG;
  *out = nullptr;
  mce_server_options o{};
  if (opt) o = *opt;
  if (o.max_inflight == 0) o.max_inflight = 8;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return MCE_ERR_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= count) return MCE_ERR_INVALID_ARG;
  MCE_CUDA_TRY(cudaSetDevice(o.device));
  mce::keep_pool_memory(o.device);
  size_t freeb = 0, totalb = 0;
  MCE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
  mce_server *s = new (std::nothrow) mce_server();
  if (!s) return MCE_ERR_OUT_OF_MEMORY;
  s->opt = o;
  s->budget = o.memory_budget ? o.memory_budget : (uint64_t)(freeb * 0.6);
  if (cudaEventCreate(&s->base) != cudaSuccess || cudaEventRecord(s->base, 0) != cudaSuccess ||
      cudaEventSynchronize(s->base) != cudaSuccess) {
    if (s->base) cudaEventDestroy(s->base);
    delete s;
    return MCE_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, o.device);
  for (uint32_t i = 0; i < o.max_inflight; i++) s->workers.emplace_back(mce::worker_main, s);
  *out = s;
  return MCE_OK;
}

mce_status mce_server_submit(mce_server *s, const uint32_t *u, const uint32_t *v, uint64_t n_pairs,
                             uint64_t *request_id) {
  if (!s || !request_id || (n_pairs && (!u || !v))) return MCE_ERR_INVALID_ARG;
  std::unique_ptr<Request> r(new (std::nothrow) Request());
  if (!r) return MCE_ERR_OUT_OF_MEMORY;
  r->u.assign(u, u + n_pairs);
  r->v.assign(v, v + n_pairs);
  r->est_bytes = mce::estimate_bytes(*r);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return MCE_ERR_BUSY;
    r->id = s->next_id++;
    *request_id = r->id;
    s->queue.push_back(r.get());
    s->all[r->id] = std::move(r);
  }
  s->cv_work.notify_one();
  return MCE_OK;
}

mce_status mce_server_poll(mce_server *s, uint64_t request_id, int *done, mce_result *out, double *latency_ms) {
  if (!s || !done) return MCE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(request_id);
  if (it == s->all.end()) return MCE_ERR_NOT_FOUND;
  Request *r = it->second.get();
  *done = r->state == 2;
  if (!*done) return MCE_OK;
  if (out && r->result) *out = *r->result;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  return r->status;
}

mce_status mce_server_request_span(mce_server *s, uint64_t request_id, double *device_start_ms,
                                   double *device_end_ms) {
  if (!s || !device_start_ms || !device_end_ms) return MCE_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(request_id);
  if (it == s->all.end()) return MCE_ERR_NOT_FOUND;
  const Request *r = it->second.get();
  if (r->state != 2) return MCE_ERR_BUSY;
  *device_start_ms = r->dev_start_ms;
  *device_end_ms = r->dev_end_ms;
  return r->dev_start_ms < 0 ? MCE_ERR_CUDA : MCE_OK;
}

mce_status mce_server_drain(mce_server *s) {
  if (!s) return MCE_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&]() { return s->queue.empty() && s->running == 0; });
  return MCE_OK;
}

void mce_server_free(mce_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto &t : s->workers) t.join();
  if (s->base) {
    cudaSetDevice(s->opt.device);
    cudaEventDestroy(s->base);
  }
  delete s;
}

}  // extern "C"
