// server.cu -- request loop: MCE jobs on different graphs, admitted by
// estimated HBM footprint and enumerated in shared launches.
//
// No reference counterpart.  Continuous batching: two dispatcher threads, each
// with its own CUDA stream and scratch, repeatedly take every queued request
// that fits the memory budget (oldest first), build them on the GPU as one
// disjoint-union graph with a result slot per request, and enumerate them in
// one persistent launch, where the warps share all requests' work.  Requests
// that arrive meanwhile join the next admission; while one dispatcher's batch
// enumerates, the other uploads and builds the next, so builds overlap
// enumeration on the device.  A single queued request runs alone with the
// whole GPU.  Results equal the request solved alone (the maximal cliques of a
// disjoint union are those of its parts).
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
  uint64_t label_span = 0;  // largest label + 1 (0 without pairs)
  int state = 0;            // 0 queued, 1 running, 2 done
  mce_status status = MCE_OK;
  std::unique_ptr<mce_result> result;
  Clock::time_point t_submit, t_done;
  double dev_start_ms = -1, dev_end_ms = -1;  // device clock, from the server's base event
};

constexpr int kDispatchers = 2;
constexpr uint32_t kDefaultInflight = 256;

}  // namespace

struct mce_server {
  mce_server_options opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
  std::vector<std::thread> workers;
  uint64_t budget = 0, in_use = 0, next_id = 1;
  uint32_t running = 0;  // requests in admitted batches
  bool stop = false;
  // recorded (and completed) at creation: request spans are measured from it
  // on the device's own clock
  cudaEvent_t base = nullptr;
};

namespace mce {
namespace {

// pairs on the device and the build's sort buffers (~12 words a pair), the
// label map, the CSR and roots, the per-request result slot, plus a share of
// the enumeration's scratch
uint64_t estimate_bytes(const Request &r) {
  return 96ULL * r.u.size() + 8ULL * r.label_span + (MCE_HIST_LEN + 8) * 8ULL + (64ULL << 20);
}

// Oldest queued requests that fit the free budget, the device's request cap
// and the union's 31-bit label space; a request too large for the budget
// runs alone once nothing else is admitted.  Caller holds s->mu.
std::vector<Request *> take_batch(mce_server *s) {
  std::vector<Request *> batch;
  uint64_t bytes = 0, span = 0;
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    Request *q = *it;
    const bool first = batch.empty();
    const bool fits = s->in_use + bytes + q->est_bytes <= s->budget &&
                      s->running + batch.size() < s->opt.max_inflight && span + q->label_span < (1ULL << 31);
    if (fits || (first && s->running == 0)) {
      batch.push_back(q);
      bytes += q->est_bytes;
      span += q->label_span;
      it = s->queue.erase(it);
      if (!fits) break;  // an oversize request goes alone
    } else if (first) {
      ++it;  // the oldest does not fit now: a later, smaller one may
    } else {
      break;
    }
  }
  return batch;
}

void finish(mce_server *s, std::vector<Request *> &batch, mce_status rc, float span0, float span1) {
  std::lock_guard<std::mutex> lk(s->mu);
  const auto now = Clock::now();
  for (Request *r : batch) {
    r->status = rc;
    r->dev_start_ms = span0;
    r->dev_end_ms = span1;
    r->t_done = now;
    if (!r->result) r->result.reset(new mce_result());
    r->result->phase_ms[MCE_PHASE_TOTAL] = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
    r->state = 2;
    r->u.clear();
    r->u.shrink_to_fit();
    r->v.clear();
    r->v.shrink_to_fit();
  }
}

void run_batch(mce_server *s, std::vector<Request *> &batch, cudaStream_t st, Scratch *scr) {
  const uint32_t k = (uint32_t)batch.size();
  mce_status rc = MCE_OK;
  // the batch's device span: from before its upload to after its results are
  // read back, on this dispatcher's stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess) rc = MCE_ERR_CUDA;
  if (ev0) cudaEventRecord(ev0, st);
  std::vector<uint64_t> poff(k + 1, 0);
  for (uint32_t i = 0; i < k; i++) poff[i + 1] = poff[i] + batch[i]->u.size();
  const uint64_t np = poff[k];
  const size_t bytes = std::max<uint64_t>(np, 1) * 4;
  // pairs go to the dispatcher's kept scratch (grown stream-ordered, reused)
  uint32_t *ud = rc == MCE_OK ? (uint32_t *)scr->get(7, 2 * bytes, &rc) : nullptr;
  uint32_t *vd = ud ? ud + bytes / 4 : nullptr;
  for (uint32_t i = 0; rc == MCE_OK && i < k; i++) {
    const uint64_t n = batch[i]->u.size();
    if (n && (cudaMemcpyAsync(ud + poff[i], batch[i]->u.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
              cudaMemcpyAsync(vd + poff[i], batch[i]->v.data(), n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess))
      rc = MCE_ERR_CUDA;
  }
  DeviceGraph g;
  UnionCounts uc;
  const auto t0 = Clock::now();
  if (rc == MCE_OK) {
    if (k == 1) {
      rc = build_from_pairs(ud, vd, np, MCE_ORDER_DEGENERACY, 1ULL << 34, st, &g);
      uc.nv = {g.n};
      uc.ne = {g.m};
      uc.max_degree = {g.max_degree};
      uc.degeneracy = {g.degeneracy};
    } else {
      rc = build_union(ud, vd, poff.data(), k, MCE_ORDER_DEGENERACY, 1ULL << 34, st, &g, &uc);
    }
  }
  const double build_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  const size_t slot_bytes = sizeof(SlotResult) * k, hist_bytes = sizeof(unsigned long long) * MCE_HIST_LEN * k;
  char *dres = rc == MCE_OK ? (char *)scr->get(0, slot_bytes + hist_bytes, &rc) : nullptr;
  if (dres && cudaMemsetAsync(dres, 0, slot_bytes + hist_bytes, st) != cudaSuccess) rc = MCE_ERR_CUDA;
  EnumStats stats;
  std::vector<SlotResult> hs(k);
  std::vector<uint64_t> hh((size_t)k * MCE_HIST_LEN);
  if (rc == MCE_OK) {
    EnumConfig cfg;
    cfg.n_slots = k;
    cfg.hist_len = MCE_HIST_LEN;
    rc = enumerate(g, cfg, scr, st, (SlotResult *)dres, (unsigned long long *)(dres + slot_bytes), &stats);
    if (rc == MCE_OK &&
        (cudaMemcpyAsync(hs.data(), dres, slot_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
         cudaMemcpyAsync(hh.data(), dres + slot_bytes, hist_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess))
      rc = MCE_ERR_CUDA;
  }
  if (g.off) free_graph(&g);
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
  for (uint32_t i = 0; i < k; i++) {
    std::unique_ptr<mce_result> res(new mce_result());
    std::memset(res.get(), 0, sizeof(mce_result));
    if (rc == MCE_OK) {
      res->count = hs[i].count;
      res->checksum = hs[i].checksum;
      res->max_size = hs[i].max_size;
      std::memcpy(res->hist, hh.data() + (size_t)i * MCE_HIST_LEN, MCE_HIST_LEN * 8);
      res->num_vertices = uc.nv[i];
      res->num_edges = uc.ne[i];
      res->roots = uc.ne[i];
      res->max_degree = uc.max_degree[i];
      res->degeneracy = uc.degeneracy[i];
      res->phase_ms[MCE_PHASE_PREPROCESS] = build_ms;
      res->phase_ms[MCE_PHASE_ENUMERATE] = stats.ms_enum;
      res->launches = stats.launches;
      res->blocks_per_sm = stats.blocks_per_sm;
    }
    batch[i]->result = std::move(res);
  }
  finish(s, batch, rc, span0, span1);
}

void worker_main(mce_server *s) {
  cudaSetDevice(s->opt.device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  Scratch scr;
  scr.device = s->opt.device;
  scr.ordered = st;  // growing a dispatcher's buffers must not stall the other's work
  for (;;) {
    std::vector<Request *> batch;
    uint64_t bytes = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stop) break;
        batch = take_batch(s);
        if (!batch.empty()) break;
        s->cv_work.wait(lk);
      }
      if (batch.empty()) break;
      for (Request *r : batch) {
        r->state = 1;
        bytes += r->est_bytes;
      }
      s->in_use += bytes;
      s->running += (uint32_t)batch.size();
    }
    run_batch(s, batch, st, &scr);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= bytes;
      s->running -= (uint32_t)batch.size();
    }
    // The dispatcher keeps its scratch for the next batch: freeing device
    // memory would synchronise the whole device.
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  scr.release();
  scr.ordered = nullptr;  // the stream goes away next; the destructor must not touch it
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
  if (o.max_inflight == 0) o.max_inflight = kDefaultInflight;
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
  const int nd = (int)std::min<uint32_t>(kDispatchers, o.max_inflight);
  for (int i = 0; i < nd; i++) s->workers.emplace_back(mce::worker_main, s);
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
  uint32_t maxlab = 0;
  for (uint64_t i = 0; i < n_pairs; i++) maxlab = std::max(maxlab, std::max(u[i], v[i]));
  r->label_span = n_pairs ? (uint64_t)maxlab + 1 : 0;
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
