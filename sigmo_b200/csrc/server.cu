// Serving loop: a resident molecule database answering query requests with
// continuous batching.
//
// The reference runs one query batch against one data batch per process
// (library/src/sigmo.cpp:98-160).  Here the data graphs, their adjacency rows
// and their signatures for iterations 1..R stay in device memory for the
// life of the server; requests (query batches of any size) are queued, and
// each of `max_inflight` workers (one host thread and one CUDA stream each)
// repeatedly takes the queued requests in arrival order, up to
// `max_batch_queries` query graphs, builds their plane program, admits the
// batch once its projected device footprint fits the memory budget next to
// the batches already on the device, and runs the batched form on its
// stream.  Batches of different workers overlap on the device; requests
// that arrive meanwhile wait for the next free worker.
//
// A request's results do not depend on the requests it was batched with:
// every stage of the batched form is per (query graph, data graph) pair,
// except the reference's literal join of the data graphs that start below
// vertex 256, which carries DFS state from one pair to the next
// (isomorphism.hpp:309) and therefore runs once per request
// (BatchedRun::query_ranges).
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Per-query totals over the GMCR slots of a batch: matched pairs (count > 0)
// and the sum of counts.  Shared-memory histograms per block, one global
// atomic per (block, query).
__global__ void k_query_totals(const uint32_t* __restrict__ indices, const uint64_t* __restrict__ counts, uint64_t total,
                               uint32_t QG, unsigned long long* __restrict__ matched, unsigned long long* __restrict__ sum) {
  extern __shared__ unsigned long long hist[];  // [2][QG]
  for (uint32_t i = threadIdx.x; i < 2 * QG; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < total;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t c = counts[s];
    if (c) {
      const uint32_t q = indices[s];
      atomicAdd(&hist[q], 1ull);
      atomicAdd(&hist[QG + q], static_cast<unsigned long long>(c));
    }
  }
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < QG; q += blockDim.x) {
    if (hist[q]) atomicAdd(&matched[q], hist[q]);
    if (hist[QG + q]) atomicAdd(&sum[q], hist[QG + q]);
  }
}

__global__ void k_pair_flags(const uint64_t* __restrict__ counts, uint64_t total, uint32_t* __restrict__ flag) {
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < total;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    flag[s] = counts[s] != 0 ? 1u : 0u;
}

// Matched pairs in GMCR slot order (data graph, then query graph).
__global__ void k_pair_scatter(const uint32_t* __restrict__ indices, const uint32_t* __restrict__ pair_graph,
                               const uint64_t* __restrict__ counts, const uint32_t* __restrict__ pos, uint64_t total,
                               uint32_t* __restrict__ out_q, uint32_t* __restrict__ out_g, uint64_t* __restrict__ out_c) {
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < total;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint64_t c = counts[s];
    if (c) {
      const uint32_t p = pos[s];
      out_q[p] = indices[s];
      out_g[p] = pair_graph[s];
      out_c[p] = c;
    }
  }
}

struct Request {
  uint64_t ticket = 0;
  uint32_t flags = 0;
  std::vector<uint32_t> goff, roff, col;
  std::vector<uint8_t> nl, el;
  uint32_t num_queries = 0;
  uint64_t query_nodes = 0;
  Clock::time_point t_submit, t_start, t_done;
  bool done = false;
  int status = SIGMO_OK;
  std::string error;
  sigmo_request_result res{};
  std::vector<uint64_t> q_matched, q_total;
  std::vector<uint32_t> pair_q, pair_g;
  std::vector<uint64_t> pair_c;
};

struct Worker {
  sigmo_queue_t q = nullptr;
  sigmo_gmcr_t m = nullptr;
  std::thread th;
};

}  // namespace

struct Server {
  int device = 0;
  sigmo_options opts{};
  sigmo_server_options so{};
  sigmo_queue_t q0 = nullptr;
  sigmo_graph_t data = nullptr;
  uint64_t* dsig = nullptr;
  ResidentPlanes rp;  // every threshold plane of the database
  uint64_t resident_bytes = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_mem;
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_ticket = 1, next_batch = 1;
  uint64_t mem_in_use = 0, mem_peak = 0;
  uint32_t batches_in_flight = 0, max_batches_in_flight = 0;  // admitted batches
  bool stopping = false;
  std::vector<Worker> workers;
  sigmo_server_stats stats{};

  void worker_loop(Worker* w);
  void run_batch(Worker* w, std::vector<Request*>& batch);
};

namespace {

// Device footprint of a batch once its plane program is known: planes (none
// when the database's planes are resident), the
// non-empty matrix, the GMCR arrays for every (query, data graph) pair, the
// join's per-chunk level masks and the result arrays.
uint64_t projected_bytes(const Graph* query, const Graph* data, bool resident) {
  const PlaneProgram& pp = query->pp;
  const uint64_t G = data->num_graphs, GW = (G + 31) / 32, QG = query->num_graphs;
  const uint64_t pairs = QG * G;
  const uint64_t planes = resident ? 0 : 8ull * GW * 32 * pp.K * data->adj_words;
  const uint64_t ne = 4ull * pp.C * GW + 4ull * QG * GW;
  const uint64_t gmcr = 4ull * (G + 1) + pairs * (4 + 4 + 8);
  // level masks + setup records per chunk of slots (two chunk buffers, one per
  // stream, once the pairs exceed one chunk), and the overflow list
  const uint64_t chunk = std::min<uint64_t>(pairs, 8ull << 20);
  const uint64_t join = (pairs > chunk ? 2 : 1) * chunk * (8ull * 16 + 16) + 4ull * pairs;
  const uint64_t results = pairs * (4 + 4 + 4 + 8);
  return planes + ne + gmcr + join + results + (16ull << 20);
}

}  // namespace

void Server::worker_loop(Worker* w) {
  cudaSetDevice(device);
  for (;;) {
    std::vector<Request*> batch;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stopping || !pending.empty(); });
      if (pending.empty()) return;  // stopping
      if (so.batch_window_us) {
        // wait (bounded) for the batch to fill once a request is queued
        const auto deadline = pending.front()->t_submit + std::chrono::microseconds(so.batch_window_us);
        cv_work.wait_until(lk, deadline, [&] {
          uint64_t nq = 0;
          for (Request* r : pending) nq += r->num_queries;
          return stopping || nq >= so.max_batch_queries;
        });
        if (pending.empty()) continue;
      }
      uint64_t nq = 0;
      while (!pending.empty()) {
        Request* r = pending.front();
        if (!batch.empty() && nq + r->num_queries > so.max_batch_queries) break;
        batch.push_back(r);
        nq += r->num_queries;
        pending.pop_front();
      }
    }
    run_batch(w, batch);
  }
}

void Server::run_batch(Worker* w, std::vector<Request*>& batch) {
  Queue* q = w->q;
  const auto t_start = Clock::now();
  for (Request* r : batch) r->t_start = t_start;
  // the batch's query graphs, concatenated in request order
  uint64_t QG = 0, Qn = 0, Qe = 0;
  for (Request* r : batch) {
    QG += r->num_queries;
    Qn += r->query_nodes;
    Qe += r->col.size();
  }
  std::vector<uint32_t> goff{0}, roff{0}, col, ranges{0};
  std::vector<uint8_t> nl, el;
  goff.reserve(QG + 1);
  roff.reserve(Qn + 1);
  col.reserve(Qe);
  nl.reserve(Qn);
  el.reserve(Qe);
  for (Request* r : batch) {
    const uint32_t vbase = static_cast<uint32_t>(nl.size()), ebase = static_cast<uint32_t>(col.size());
    for (uint32_t i = 1; i < r->goff.size(); ++i) goff.push_back(vbase + r->goff[i]);
    for (uint32_t i = 1; i < r->roff.size(); ++i) roff.push_back(ebase + r->roff[i]);
    for (uint32_t c : r->col) col.push_back(vbase + c);
    nl.insert(nl.end(), r->nl.begin(), r->nl.end());
    el.insert(el.end(), r->el.begin(), r->el.end());
    ranges.push_back(static_cast<uint32_t>(goff.size() - 1));
  }
  sigmo_host_graphs hq{};
  hq.num_graphs = static_cast<uint32_t>(QG);
  hq.total_nodes = Qn;
  hq.total_edges = Qe;
  hq.graph_offsets = goff.data();
  hq.row_offsets = roff.data();
  hq.column_indices = col.data();
  hq.node_labels = nl.data();
  hq.edge_labels = el.data();

  int rc = SIGMO_OK;
  std::string err;
  uint64_t reserved = 0, batch_id = 0;
  sigmo_graph_t qg = nullptr;
  sigmo_match_result mr{};
  uint64_t gathered = 0;  // resident plane bytes the admission gathered
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float dev_ms = 0;
  std::vector<unsigned long long> h_matched(QG), h_sum(QG);
  std::vector<uint32_t> h_pq, h_pg;
  std::vector<uint64_t> h_pc;
  const bool want_pairs = std::any_of(batch.begin(), batch.end(), [](Request* r) { return r->flags & SIGMO_REQUEST_PAIRS; });
  auto note = [&](int code) {
    if (code && !rc) {
      rc = code;
      err = get_error_message();
    }
  };
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "event creation failed"));
  if (!rc && cudaEventRecord(e0, q->stream) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "event record failed"));
  if (!rc) note(sigmo_graph_create(w->q, &hq, &qg));
  if (!rc && qg->max_nodes > kMaxQueryNodes)
    note(fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (largest: %u)", kMaxQueryNodes, qg->max_nodes));
  if (!rc) note(build_plane_program(q, qg, so.iterations));
  // admission by the batch's projected device footprint
  if (!rc) {
    const uint64_t need = projected_bytes(qg, data, rp.planes != nullptr);
    std::unique_lock<std::mutex> lk(mu);
    if (need > so.memory_budget) {
      note(fail(SIGMO_ERR_OOM, "batch of %llu query graphs needs %llu bytes, above the serving memory budget (%llu bytes)",
                (unsigned long long)QG, (unsigned long long)need, (unsigned long long)so.memory_budget));
    } else {
      cv_mem.wait(lk, [&] { return mem_in_use + need <= so.memory_budget; });
      mem_in_use += need;
      mem_peak = std::max(mem_peak, mem_in_use);
      reserved = need;
      batch_id = next_batch++;
      ++batches_in_flight;
      max_batches_in_flight = std::max(max_batches_in_flight, batches_in_flight);
    }
  }
  if (!rc) {
    BatchedRun run;
    run.dsig = dsig;
    run.resident = rp.planes ? &rp : nullptr;
    run.query_ranges = ranges.data();
    run.nranges = static_cast<uint32_t>(batch.size());
    note(match_batched(q, qg, data, so.iterations, so.find_first, false, nullptr, w->m, &mr, run));
    if (!rc && rp.planes)
      gathered = 8ull * ((data->num_graphs + 31ull) / 32ull) * 32ull * qg->pp.K * data->adj_words;
  }
  // per-query totals (and the matched pairs when a request asked for them)
  if (!rc && QG) {
    void* buf = nullptr;
    const uint64_t total = w->m->total;
    note(tmp_alloc(q, &buf, 16ull * QG + 256));
    auto* d_matched = static_cast<unsigned long long*>(buf);
    auto* d_sum = d_matched + QG;
    if (!rc && cudaMemsetAsync(buf, 0, 16ull * QG, q->stream) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "memset failed"));
    if (!rc && total) {
      const size_t smem = 16ull * QG;
      if (smem <= 48u * 1024u) {
        k_query_totals<<<grid_for(total, 256, 148u * 4u), 256, smem, q->stream>>>(w->m->indices, w->m->counts, total,
                                                                                 static_cast<uint32_t>(QG), d_matched, d_sum);
        note(check_launch(q, "k_query_totals"));
      } else {
        note(fail(SIGMO_ERR_DOMAIN, "a serving batch holds at most %u query graphs", 48u * 1024u / 16u));
      }
    }
    if (!rc && cudaMemcpyAsync(h_matched.data(), d_matched, 8ull * QG, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess)
      note(fail(SIGMO_ERR_CUDA, "D2H failed"));
    if (!rc && cudaMemcpyAsync(h_sum.data(), d_sum, 8ull * QG, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess)
      note(fail(SIGMO_ERR_CUDA, "D2H failed"));
    if (!rc && want_pairs && total > 0x7FFFFFFFull)
      note(fail(SIGMO_ERR_DOMAIN, "matched-pair lists are limited to 2^31 admitted pairs per batch"));
    if (!rc && want_pairs && total) {
      void* pbuf = nullptr;
      size_t temp = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, temp, static_cast<const uint32_t*>(nullptr), static_cast<uint32_t*>(nullptr),
                                    static_cast<int>(std::min<uint64_t>(total, 0x7FFFFFFF)), q->stream);
      const uint64_t b_flag = (4 * total + 255) & ~255ull;
      note(tmp_alloc(q, &pbuf, 2 * b_flag + temp + 256));
      if (!rc) {
        auto* flag = static_cast<uint32_t*>(pbuf);
        auto* pos = reinterpret_cast<uint32_t*>(static_cast<char*>(pbuf) + b_flag);
        void* tmp = static_cast<char*>(pbuf) + 2 * b_flag;
        k_pair_flags<<<grid_for(total, 256, 148u * 16u), 256, 0, q->stream>>>(w->m->counts, total, flag);
        note(check_launch(q, "k_pair_flags"));
        if (!rc && cub::DeviceScan::ExclusiveSum(tmp, temp, flag, pos, static_cast<int>(total), q->stream) != cudaSuccess)
          note(fail(SIGMO_ERR_CUDA, "pair scan failed"));
        uint32_t last[2] = {0, 0};
        if (!rc && cudaMemcpyAsync(&last[0], pos + total - 1, 4, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess)
          note(fail(SIGMO_ERR_CUDA, "D2H failed"));
        if (!rc && cudaMemcpyAsync(&last[1], flag + total - 1, 4, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess)
          note(fail(SIGMO_ERR_CUDA, "D2H failed"));
        if (!rc && cudaStreamSynchronize(q->stream) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "synchronisation failed"));
        const uint64_t np = static_cast<uint64_t>(last[0]) + last[1];
        void* obuf = nullptr;
        if (!rc) note(tmp_alloc(q, &obuf, 16ull * np + 256));
        if (!rc) {
          auto* oq = static_cast<uint32_t*>(obuf);
          auto* og = oq + np;
          auto* oc = reinterpret_cast<uint64_t*>(static_cast<char*>(obuf) + ((8 * np + 255) & ~255ull));
          k_pair_scatter<<<grid_for(total, 256, 148u * 16u), 256, 0, q->stream>>>(w->m->indices, w->m->pair_graph, w->m->counts,
                                                                                  pos, total, oq, og, oc);
          note(check_launch(q, "k_pair_scatter"));
          h_pq.resize(np);
          h_pg.resize(np);
          h_pc.resize(np);
          if (!rc && np) {
            if (cudaMemcpyAsync(h_pq.data(), oq, 4 * np, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
                cudaMemcpyAsync(h_pg.data(), og, 4 * np, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
                cudaMemcpyAsync(h_pc.data(), oc, 8 * np, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess)
              note(fail(SIGMO_ERR_CUDA, "D2H failed"));
          }
          dev_free(q, obuf);
        }
        dev_free(q, pbuf);
      }
    }
    dev_free(q, buf);
  }
  if (!rc && cudaEventRecord(e1, q->stream) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "event record failed"));
  if (cudaStreamSynchronize(q->stream) != cudaSuccess) note(fail(SIGMO_ERR_CUDA, "synchronisation failed"));
  if (!rc) cudaEventElapsedTime(&dev_ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (qg) sigmo_graph_destroy(qg);
  const auto t_done = Clock::now();
  // The matched pairs split into per-request lists in one pass over the
  // batch's pairs, before the server lock is taken (requests cover contiguous
  // query ranges of the batch, in order).
  std::vector<std::vector<uint32_t>> req_pq(batch.size()), req_pg(batch.size());
  std::vector<std::vector<uint64_t>> req_pc(batch.size());
  if (!rc && !h_pq.empty()) {
    std::vector<int32_t> owner(QG, -1);
    std::vector<uint32_t> first_query(batch.size());
    uint32_t qb = 0;
    for (size_t i = 0; i < batch.size(); ++i) {
      first_query[i] = qb;
      if (batch[i]->flags & SIGMO_REQUEST_PAIRS)
        for (uint32_t k = 0; k < batch[i]->num_queries; ++k) owner[qb + k] = static_cast<int32_t>(i);
      qb += batch[i]->num_queries;
    }
    for (size_t p = 0; p < h_pq.size(); ++p) {
      const int32_t i = h_pq[p] < QG ? owner[h_pq[p]] : -1;
      if (i < 0) continue;
      req_pq[i].push_back(h_pq[p] - first_query[i]);
      req_pg[i].push_back(h_pg[p]);
      req_pc[i].push_back(h_pc[p]);
    }
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    if (reserved) {
      mem_in_use -= reserved;
      --batches_in_flight;
    }
    uint32_t qb = 0;
    for (size_t i = 0; i < batch.size(); ++i) {
      Request* r = batch[i];
      const uint32_t qe = qb + r->num_queries;
      r->t_done = t_done;
      r->status = rc;
      r->error = err;
      sigmo_request_result& o = r->res;
      o.status = rc;
      o.num_queries = r->num_queries;
      o.batch_id = batch_id;
      o.batch_queries = static_cast<uint32_t>(QG);
      o.batch_requests = static_cast<uint32_t>(batch.size());
      o.ms_queue = ms_between(r->t_submit, r->t_start);
      o.ms_device = dev_ms;
      o.ms_latency = ms_between(r->t_submit, t_done);
      o.ms_filter = mr.ms_signatures + mr.ms_filter;
      o.ms_mapping = mr.ms_mapping;
      o.ms_join = mr.ms_join;
      o.gathered_plane_bytes = gathered;
      o.projected_bytes = reserved;
      o.pairs = static_cast<uint64_t>(r->num_queries) * data->num_graphs;
      if (!rc) {
        r->q_matched.assign(h_matched.begin() + qb, h_matched.begin() + qe);
        r->q_total.assign(h_sum.begin() + qb, h_sum.begin() + qe);
        for (uint32_t k = 0; k < r->num_queries; ++k) {
          o.matched_pairs += r->q_matched[k];
          o.total_matches += r->q_total[k];
        }
        if (r->flags & SIGMO_REQUEST_PAIRS) {
          r->pair_q = std::move(req_pq[i]);
          r->pair_g = std::move(req_pg[i]);
          r->pair_c = std::move(req_pc[i]);
        }
      }
      r->done = true;
      qb = qe;
      ++stats.requests_completed;
      if (rc) ++stats.requests_failed;
      stats.queries_completed += r->num_queries;
    }
    if (!rc) {
      ++stats.batches;
      stats.pairs += QG * data->num_graphs;
      stats.admitted_pairs += mr.admitted_pairs;
      stats.device_ms += dev_ms;
    }
    stats.peak_reserved_bytes = mem_peak;
    stats.max_batches_in_flight = max_batches_in_flight;
  }
  cv_mem.notify_all();
  cv_done.notify_all();
}

}  // namespace sigmo_b200

using namespace sigmo_b200;

struct sigmo_server_s : sigmo_b200::Server {};

namespace {

int copy_request(const sigmo_host_graphs* h, Request* r) {
  if (!h || !h->graph_offsets || !h->row_offsets || (h->total_edges && !h->column_indices) || (h->total_nodes && !h->node_labels))
    return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: null arrays");
  if (h->num_graphs == 0) return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: empty request");
  if (h->graph_offsets[0] != 0 || h->graph_offsets[h->num_graphs] != h->total_nodes || h->row_offsets[h->total_nodes] != h->total_edges)
    return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: offsets disagree with totals");
  for (uint32_t g = 0; g < h->num_graphs; ++g) {
    const uint32_t n = h->graph_offsets[g + 1] - h->graph_offsets[g];
    if (h->graph_offsets[g + 1] < h->graph_offsets[g]) return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: decreasing offsets");
    if (n > kMaxQueryNodes)
      return fail(SIGMO_ERR_DOMAIN, "query graphs of up to %u vertices are supported (graph %u has %u)", kMaxQueryNodes, g, n);
  }
  for (uint64_t e = 0; e < h->total_edges; ++e)
    if (h->column_indices[e] >= h->total_nodes) return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: neighbour id out of range");
  r->goff.assign(h->graph_offsets, h->graph_offsets + h->num_graphs + 1);
  r->roff.assign(h->row_offsets, h->row_offsets + h->total_nodes + 1);
  r->col.assign(h->column_indices, h->column_indices + h->total_edges);
  r->nl.assign(h->node_labels, h->node_labels + h->total_nodes);
  if (h->edge_labels) r->el.assign(h->edge_labels, h->edge_labels + h->total_edges);
  else r->el.assign(h->total_edges, 0);
  r->num_queries = h->num_graphs;
  r->query_nodes = h->total_nodes;
  return SIGMO_OK;
}

Request* find(sigmo_server_t s, uint64_t ticket) {
  auto it = s->reqs.find(ticket);
  return it == s->reqs.end() ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

void sigmo_server_default_options(sigmo_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->iterations = 6;
  o->find_first = 1;
  o->max_inflight = 2;
  o->max_batch_queries = 64;
  o->memory_budget = 0;
  o->batch_window_us = 0;
}

int sigmo_server_create(int device, const sigmo_host_graphs* database, const sigmo_options* opts, const sigmo_server_options* so,
                        sigmo_server_t* out) {
  if (!database || !out) return fail(SIGMO_ERR_INVALID, "sigmo_server_create: null argument");
  *out = nullptr;
  sigmo_server_options o;
  sigmo_server_default_options(&o);
  if (so) o = *so;
  if (o.max_inflight == 0 || o.max_inflight > 16) return fail(SIGMO_ERR_INVALID, "max_inflight must be in 1..16");
  if (o.max_batch_queries == 0) return fail(SIGMO_ERR_INVALID, "max_batch_queries must be positive");
  if (o.iterations > 64) return fail(SIGMO_ERR_INVALID, "iterations must be <= 64");
  if (opts && opts->profile == SIGMO_PROFILE_REF_X86)
    return fail(SIGMO_ERR_DOMAIN, "the serving loop runs the REF_PTX and EXACT profiles");
  std::unique_ptr<sigmo_server_s> s(new (std::nothrow) sigmo_server_s());
  if (!s) return fail(SIGMO_ERR_OOM, "host allocation failed");
  s->device = device;
  s->so = o;
  SIGMO_TRY(sigmo_queue_create(device, opts, &s->q0));
  s->opts = s->q0->opts;
  auto cleanup = [&](int rc) {
    if (s->rp.planes) dev_free(s->q0, s->rp.planes);
    if (s->dsig) dev_free(s->q0, s->dsig);
    if (s->data) sigmo_graph_destroy(s->data);
    cudaStreamSynchronize(s->q0->stream);
    sigmo_queue_destroy(s->q0);
    return rc;
  };
  int rc = sigmo_graph_create(s->q0, database, &s->data);
  if (rc) return cleanup(rc);
  if (s->data->max_nodes > 64u * kMaxAdjWords)
    return cleanup(fail(SIGMO_ERR_DOMAIN, "the serving loop supports data graphs of up to %u vertices (largest: %u)",
                        64u * kMaxAdjWords, s->data->max_nodes));
  const uint64_t N = s->data->total_nodes;
  rc = dev_alloc(s->q0, reinterpret_cast<void**>(&s->dsig), 8ull * (o.iterations ? o.iterations : 1) * (N ? N : 1));
  if (!rc && o.iterations) rc = launch_sig_all(s->q0, s->data, o.iterations, s->dsig);
  if (!rc && cudaStreamSynchronize(s->q0->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "database upload failed");
  // the planes of every threshold that occurs in the database, built once:
  // a batch then gathers its planes instead of evaluating signatures
  if (!rc && o.iterations) {
    rc = build_resident_planes(s->q0, s->data, s->dsig, o.iterations, &s->rp);
    if (rc == SIGMO_ERR_DOMAIN) {  // too many distinct thresholds for one tile: build planes per batch
      if (s->rp.planes) dev_free(s->q0, s->rp.planes);
      s->rp = ResidentPlanes{};
      rc = SIGMO_OK;
    }
  }
  if (rc) return cleanup(rc);
  s->resident_bytes = 4ull * (s->data->num_graphs + 1) + 4ull * (N + 1) + 5ull * s->data->total_edges + N +
                      4ull * N + 8ull * N * s->data->adj_words + 8ull * o.iterations * N +
                      8ull * ((s->data->num_graphs + 31) / 32) * 32 * s->rp.rows * s->data->adj_words;
  if (o.memory_budget == 0) {
    size_t freeb = 0, totalb = 0;
    if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) return cleanup(fail(SIGMO_ERR_CUDA, "cudaMemGetInfo failed"));
    s->so.memory_budget = freeb / 2;
  }
  // Warm the pool of per-call temporaries: one allocation of a quarter of the
  // budget, freed at once.  The pool keeps the memory (its release threshold
  // is unlimited), so the batches' stream-ordered temporaries are carved from
  // it instead of mapping new memory while requests wait.
  {
    void* warm = nullptr;
    const uint64_t want = std::min<uint64_t>(s->so.memory_budget / 4, 32ull << 30);
    if (want && tmp_alloc(s->q0, &warm, want) == SIGMO_OK) {
      dev_free(s->q0, warm);
      cudaStreamSynchronize(s->q0->stream);
    }
    cudaGetLastError();
  }
  s->workers.resize(o.max_inflight);
  for (auto& w : s->workers) {
    rc = sigmo_queue_create(device, &s->opts, &w.q);
    if (!rc) rc = sigmo_queue_set_join_budget(w.q, o.join_step_budget);
    if (!rc) rc = sigmo_gmcr_create(w.q, &w.m);
    if (rc) break;
  }
  if (rc) {
    for (auto& w : s->workers) {
      if (w.m) sigmo_gmcr_destroy(w.m);
      if (w.q) sigmo_queue_destroy(w.q);
    }
    return cleanup(rc);
  }
  sigmo_server_s* raw = s.get();
  for (auto& w : s->workers) w.th = std::thread([raw, &w] { raw->worker_loop(&w); });
  *out = s.release();
  return SIGMO_OK;
}

int sigmo_server_submit(sigmo_server_t s, const sigmo_host_graphs* queries, uint32_t flags, uint64_t* ticket) {
  if (!s || !queries || !ticket) return fail(SIGMO_ERR_INVALID, "sigmo_server_submit: null argument");
  std::unique_ptr<Request> r(new (std::nothrow) Request());
  if (!r) return fail(SIGMO_ERR_OOM, "host allocation failed");
  SIGMO_TRY(copy_request(queries, r.get()));
  r->flags = flags;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return fail(SIGMO_ERR_INVALID, "the server is shutting down");
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->pending.push_back(r.get());
    s->reqs.emplace(r->ticket, std::move(r));
    ++s->stats.requests_submitted;
  }
  s->cv_work.notify_one();
  return SIGMO_OK;
}

int sigmo_server_wait(sigmo_server_t s, uint64_t ticket, int64_t timeout_ms, sigmo_request_result* out) {
  if (!s || !out) return fail(SIGMO_ERR_INVALID, "sigmo_server_wait: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  Request* r = find(s, ticket);
  if (!r) return fail(SIGMO_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
    return fail(SIGMO_ERR_TIMEOUT, "request %llu not finished within %lld ms", (unsigned long long)ticket, (long long)timeout_ms);
  *out = r->res;
  if (r->status) return fail(r->status, "%s", r->error.c_str());
  return SIGMO_OK;
}

int sigmo_server_query_totals(sigmo_server_t s, uint64_t ticket, uint64_t* matched, uint64_t* total, uint32_t n) {
  if (!s) return fail(SIGMO_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request* r = find(s, ticket);
  if (!r) return fail(SIGMO_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  if (!r->done) return fail(SIGMO_ERR_INVALID, "request %llu is not finished", (unsigned long long)ticket);
  if (r->status) return fail(r->status, "%s", r->error.c_str());
  if (n != r->num_queries) return fail(SIGMO_ERR_INVALID, "request has %u query graphs, not %u", r->num_queries, n);
  if (matched) std::copy(r->q_matched.begin(), r->q_matched.end(), matched);
  if (total) std::copy(r->q_total.begin(), r->q_total.end(), total);
  return SIGMO_OK;
}

int sigmo_server_pairs(sigmo_server_t s, uint64_t ticket, uint32_t* query, uint32_t* molecule, uint64_t* count,
                       uint64_t capacity, uint64_t* n) {
  if (!s || !n) return fail(SIGMO_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  Request* r = find(s, ticket);
  if (!r) return fail(SIGMO_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  if (!r->done) return fail(SIGMO_ERR_INVALID, "request %llu is not finished", (unsigned long long)ticket);
  if (r->status) return fail(r->status, "%s", r->error.c_str());
  if (!(r->flags & SIGMO_REQUEST_PAIRS)) return fail(SIGMO_ERR_INVALID, "request %llu did not ask for pairs", (unsigned long long)ticket);
  *n = r->pair_q.size();
  const uint64_t k = std::min<uint64_t>(capacity, r->pair_q.size());
  if (query) std::copy(r->pair_q.begin(), r->pair_q.begin() + k, query);
  if (molecule) std::copy(r->pair_g.begin(), r->pair_g.begin() + k, molecule);
  if (count) std::copy(r->pair_c.begin(), r->pair_c.begin() + k, count);
  return SIGMO_OK;
}

int sigmo_server_release(sigmo_server_t s, uint64_t ticket) {
  if (!s) return fail(SIGMO_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  Request* r = find(s, ticket);
  if (!r) return fail(SIGMO_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  if (!r->done) return fail(SIGMO_ERR_INVALID, "request %llu is not finished", (unsigned long long)ticket);
  s->reqs.erase(ticket);
  return SIGMO_OK;
}

int sigmo_server_get_stats(sigmo_server_t s, sigmo_server_stats* out) {
  if (!s || !out) return fail(SIGMO_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->resident_bytes = s->resident_bytes;
  out->memory_budget = s->so.memory_budget;
  out->pending_requests = s->pending.size();
  return SIGMO_OK;
}

int sigmo_server_destroy(sigmo_server_t s) {
  if (!s) return SIGMO_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers)
    if (w.th.joinable()) w.th.join();  // workers finish the queued requests first
  for (auto& w : s->workers) {
    if (w.m) sigmo_gmcr_destroy(w.m);
    if (w.q) {
      cudaStreamSynchronize(w.q->stream);
      sigmo_queue_destroy(w.q);
    }
  }
  if (s->rp.planes) dev_free(s->q0, s->rp.planes);
  if (s->dsig) dev_free(s->q0, s->dsig);
  if (s->data) sigmo_graph_destroy(s->data);
  cudaStreamSynchronize(s->q0->stream);
  sigmo_queue_destroy(s->q0);
  delete s;
  return SIGMO_OK;
}

}  // extern "C"
