// C-ABI entry points of sigmo_b200 (declared in include/sigmo_b200.h).  Each
// public stage brackets its launches with CUDA events on the queue's stream so
// sigmo_queue_last_stage_ms reports its device time, like the reference's
// BatchedEvent::getProfilingInfo (library/include/utils.hpp:149-157).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>
#include <new>

#include "internal.hpp"

namespace sigmo_b200 {

int normalize_tuning(sigmo_tuning* t) {
  const sigmo_tuning d = Queue{}.tune;
  if (!t->join_blocks_per_sm) t->join_blocks_per_sm = d.join_blocks_per_sm;
  if (!t->join_chunk) t->join_chunk = d.join_chunk;
  if (!t->overflow_blocks) t->overflow_blocks = d.overflow_blocks;
  if (!t->mask_chunk_slots) t->mask_chunk_slots = d.mask_chunk_slots;
  if (!t->overflow_split) t->overflow_split = d.overflow_split;
  if (!t->join_pool) t->join_pool = d.join_pool;
  if (t->join_blocks_per_sm > 4) return fail(SIGMO_ERR_INVALID, "join_blocks_per_sm must be 1..4");
  if (t->join_chunk > 64) return fail(SIGMO_ERR_INVALID, "join_chunk must be 1..64");
  if (t->overflow_blocks > 65535) return fail(SIGMO_ERR_INVALID, "overflow_blocks must be <= 65535");
  if (t->overflow_serial > 1) return fail(SIGMO_ERR_INVALID, "overflow_serial must be 0 or 1");
  if (t->mask_chunk_slots > 64) return fail(SIGMO_ERR_INVALID, "mask_chunk_slots must be 1..64");
  if (t->overflow_split > 64) return fail(SIGMO_ERR_INVALID, "overflow_split must be 1..64");
  if (t->join_kernel > 2) return fail(SIGMO_ERR_INVALID, "join_kernel must be 0, 1 or 2");
  if (t->join_pool > 16) return fail(SIGMO_ERR_INVALID, "join_pool must be 1..16");
  return SIGMO_OK;
}

int allow_max_dynamic_smem(const void* kernel, int device) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& d : done)
    if (d.first == kernel && d.second == device) return SIGMO_OK;
  int optin = 0;
  SIGMO_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  cudaFuncAttributes fa{};
  SIGMO_CUDA_TRY(cudaFuncGetAttributes(&fa, kernel));
  SIGMO_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      optin - static_cast<int>(fa.sharedSizeBytes)));
  done.emplace_back(kernel, device);
  return SIGMO_OK;
}

int check_launch(Queue* q, const char* what) {
  q->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SIGMO_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return SIGMO_OK;
}

int stage_begin(Queue* q) {
  SIGMO_CUDA_TRY(cudaEventRecord(q->ev_start, q->stream));
  return SIGMO_OK;
}
int stage_end(Queue* q) {
  SIGMO_CUDA_TRY(cudaEventRecord(q->ev_end, q->stream));
  q->stage_recorded = true;
  return SIGMO_OK;
}

int dev_alloc(Queue* q, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 1;
  cudaError_t e = cudaMallocAsync(p, bytes, q->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? SIGMO_ERR_OOM : SIGMO_ERR_CUDA, "device allocation of %zu bytes failed: %s",
                bytes, cudaGetErrorString(e));
  }
  return SIGMO_OK;
}
void dev_free(Queue* q, void* p) {
  if (p) cudaFreeAsync(p, q->stream);
}

namespace {
// One pool per device for per-call temporaries; its release threshold is
// unlimited, so freed blocks stay mapped for the next call.
int tmp_pool(int device, cudaMemPool_t* out) {
  static std::mutex mu;
  static std::vector<std::pair<int, cudaMemPool_t>> pools;
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& d : pools)
    if (d.first == device) {
      *out = d.second;
      return SIGMO_OK;
    }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  SIGMO_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
  uint64_t threshold = UINT64_MAX;
  SIGMO_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  pools.emplace_back(device, pool);
  *out = pool;
  return SIGMO_OK;
}
}  // namespace

int tmp_alloc(Queue* q, void** p, size_t bytes) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SIGMO_CUDA_TRY(cudaStreamIsCapturing(q->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return dev_alloc(q, p, bytes);
  *p = nullptr;
  cudaMemPool_t pool = nullptr;
  SIGMO_TRY(tmp_pool(q->device, &pool));
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, q->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(e == cudaErrorMemoryAllocation ? SIGMO_ERR_OOM : SIGMO_ERR_CUDA, "device allocation of %zu bytes failed: %s",
                bytes, cudaGetErrorString(e));
  }
  return SIGMO_OK;
}
int queue_scratch(Queue* q, size_t bytes, void** p) {
  if (bytes > q->scratch_bytes) {
    dev_free(q, q->scratch);
    q->scratch = nullptr;
    q->scratch_bytes = 0;
    size_t want = std::max<size_t>(bytes, 1 << 20);
    SIGMO_TRY(dev_alloc(q, &q->scratch, want));
    q->scratch_bytes = want;
  }
  *p = q->scratch;
  return SIGMO_OK;
}

int join_status_reset(Queue* q) {
  SIGMO_CUDA_TRY(cudaMemsetAsync(q->d_status, 0, sizeof(unsigned int), q->stream));
  return SIGMO_OK;
}
int join_status_fetch(Queue* q) {
  SIGMO_CUDA_TRY(cudaMemcpyAsync(static_cast<char*>(q->pinned) + kPinnedStatusOffset, q->d_status, sizeof(unsigned int),
                                 cudaMemcpyDeviceToHost, q->stream));
  return SIGMO_OK;
}
int join_status_result(Queue* q) {
  const unsigned st = *reinterpret_cast<const unsigned*>(static_cast<const char*>(q->pinned) + kPinnedStatusOffset);
  if (st & kJoinStatusBudget)
    return fail(SIGMO_ERR_TIMEOUT, "a join lane used up the step budget of %llu DFS levels; the counts are incomplete",
                static_cast<unsigned long long>(q->join_budget));
  return SIGMO_OK;
}

namespace {

int set_device(Queue* q) {
  SIGMO_CUDA_TRY(cudaSetDevice(q->device));
  return SIGMO_OK;
}

}  // namespace

int finish_graph(Graph* g) {
  static std::atomic<uint64_t> next_stamp{1};
  g->stamp = next_stamp++;
  // max graph size and low-offset count from the host copy of graph_offsets
  uint32_t mx = 0, low = 0;
  for (uint32_t i = 0; i < g->num_graphs; ++i) {
    mx = std::max(mx, g->host_graph_offsets[i + 1] - g->host_graph_offsets[i]);
    if (g->host_graph_offsets[i] < kLowOffsetLimit) low = i + 1;
  }
  g->max_nodes = mx;
  g->low_offset_graphs = low;
  SIGMO_TRY(launch_graph_derive(g));
  // lets work on another stream wait for this graph alone
  if (!g->ready) SIGMO_CUDA_TRY(cudaEventCreateWithFlags(&g->ready, cudaEventDisableTiming));
  SIGMO_CUDA_TRY(cudaEventRecord(g->ready, g->q->stream));
  return SIGMO_OK;
}

}  // namespace sigmo_b200

namespace sigmo_b200 {
namespace {

void queue_free(Queue* q) {
  cudaSetDevice(q->device);
  if (q->stream) {
    dev_free(q, q->scratch);
    cudaStreamSynchronize(q->stream);
    cudaStreamDestroy(q->stream);
  }
  if (q->side) {
    cudaStreamSynchronize(q->side);
    cudaStreamDestroy(q->side);
  }
  if (q->aux) {
    cudaStreamSynchronize(q->aux);
    cudaStreamDestroy(q->aux);
  }
  if (q->ev_fork) cudaEventDestroy(q->ev_fork);
  if (q->ev_join) cudaEventDestroy(q->ev_join);
  if (q->ev_aux_fork) cudaEventDestroy(q->ev_aux_fork);
  if (q->ev_aux_join) cudaEventDestroy(q->ev_aux_join);
  for (cudaEvent_t e : q->ev_masks)
    if (e) cudaEventDestroy(e);
  if (q->ev_start) cudaEventDestroy(q->ev_start);
  if (q->ev_end) cudaEventDestroy(q->ev_end);
  if (q->pinned) cudaFreeHost(q->pinned);
  if (q->d_status) cudaFree(q->d_status);
  delete static_cast<sigmo_queue_t>(q);
}

}  // namespace

Queue* queue_retain(Queue* q) {
  q->refs.fetch_add(1, std::memory_order_relaxed);
  return q;
}

void queue_release(Queue* q) {
  if (q->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) queue_free(q);
}

}  // namespace sigmo_b200

using namespace sigmo_b200;

extern "C" {

void sigmo_default_options(sigmo_options* o) {
  if (!o) return;
  o->profile = SIGMO_PROFILE_REF_PTX;
  o->join_work_group_size = 128;
  o->filter_work_group_size = 512;
}

int sigmo_queue_create(int device, const sigmo_options* opts, sigmo_queue_t* out) {
  if (!out) return fail(SIGMO_ERR_INVALID, "sigmo_queue_create: null output");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SIGMO_ERR_NO_DEVICE, "no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  }
  if (device < 0 || device >= n) return fail(SIGMO_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, n);
  sigmo_options o;
  sigmo_default_options(&o);
  if (opts) o = *opts;
  if (o.profile != SIGMO_PROFILE_REF_PTX && o.profile != SIGMO_PROFILE_EXACT && o.profile != SIGMO_PROFILE_REF_X86)
    return fail(SIGMO_ERR_INVALID, "unknown semantics profile %d", o.profile);
  if (o.join_work_group_size == 0) o.join_work_group_size = 128;
  if (o.join_work_group_size > 1024 || (o.join_work_group_size & 31u))
    return fail(SIGMO_ERR_INVALID, "join work-group size %u must be a multiple of 32 <= 1024", o.join_work_group_size);
  sigmo_queue_t q = new (std::nothrow) sigmo_queue_s();
  if (!q) return fail(SIGMO_ERR_OOM, "host allocation failed");
  q->device = device;
  q->opts = o;
  cudaError_t st = cudaSetDevice(device);
  if (st == cudaSuccess) st = cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
  if (st == cudaSuccess) st = cudaEventCreate(&q->ev_start);
  if (st == cudaSuccess) st = cudaEventCreate(&q->ev_end);
  if (st == cudaSuccess) st = cudaMallocHost(&q->pinned, 4096);
  if (st == cudaSuccess) st = cudaMalloc(reinterpret_cast<void**>(&q->d_status), 256);
  if (st == cudaSuccess) st = cudaMemset(q->d_status, 0, 256);
  if (st == cudaSuccess) st = cudaStreamCreateWithFlags(&q->side, cudaStreamNonBlocking);
  if (st == cudaSuccess) st = cudaEventCreateWithFlags(&q->ev_fork, cudaEventDisableTiming);
  if (st == cudaSuccess) st = cudaEventCreateWithFlags(&q->ev_join, cudaEventDisableTiming);
  if (st == cudaSuccess) st = cudaStreamCreateWithFlags(&q->aux, cudaStreamNonBlocking);
  if (st == cudaSuccess) st = cudaEventCreateWithFlags(&q->ev_aux_fork, cudaEventDisableTiming);
  if (st == cudaSuccess) st = cudaEventCreateWithFlags(&q->ev_aux_join, cudaEventDisableTiming);
  for (int i = 0; i < 2 && st == cudaSuccess; ++i) st = cudaEventCreateWithFlags(&q->ev_masks[i], cudaEventDisableTiming);
  if (st == cudaSuccess) {
    // Keep freed stream-ordered allocations cached in the device's default pool
    // (per-call scratch is then reused instead of being remapped every call).
    cudaMemPool_t pool;
    st = cudaDeviceGetDefaultMemPool(&pool, device);
    uint64_t threshold = UINT64_MAX;
    if (st == cudaSuccess) st = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  if (st != cudaSuccess) {
    int rc = fail(SIGMO_ERR_CUDA, "queue creation failed: %s", cudaGetErrorString(st));
    sigmo_queue_destroy(q);
    return rc;
  }
  *out = q;
  return SIGMO_OK;
}

int sigmo_queue_destroy(sigmo_queue_t q) {
  if (!q) return SIGMO_OK;
  queue_release(q);
  return SIGMO_OK;
}

int sigmo_queue_wait(sigmo_queue_t q) {
  if (!q) return fail(SIGMO_ERR_INVALID, "null queue");
  SIGMO_CUDA_TRY(cudaStreamSynchronize(q->stream));
  return SIGMO_OK;
}

int sigmo_queue_stream(sigmo_queue_t q, void** stream) {
  if (!q || !stream) return fail(SIGMO_ERR_INVALID, "null argument");
  *stream = static_cast<void*>(q->stream);
  return SIGMO_OK;
}

int sigmo_queue_last_stage_ms(sigmo_queue_t q, double* ms) {
  if (!q || !ms) return fail(SIGMO_ERR_INVALID, "null argument");
  if (!q->stage_recorded) {
    *ms = 0.0;
    return SIGMO_OK;
  }
  SIGMO_CUDA_TRY(cudaEventSynchronize(q->ev_end));
  float f = 0.f;
  SIGMO_CUDA_TRY(cudaEventElapsedTime(&f, q->ev_start, q->ev_end));
  *ms = f;
  return SIGMO_OK;
}

int sigmo_queue_device_info(sigmo_queue_t q, uint64_t* global_mem, char* name, size_t name_len) {
  if (!q) return fail(SIGMO_ERR_INVALID, "null queue");
  cudaDeviceProp p;
  SIGMO_CUDA_TRY(cudaGetDeviceProperties(&p, q->device));
  if (global_mem) *global_mem = p.totalGlobalMem;
  if (name && name_len) {
    std::strncpy(name, p.name, name_len - 1);
    name[name_len - 1] = 0;
  }
  return SIGMO_OK;
}

int sigmo_queue_set_tuning(sigmo_queue_t q, const sigmo_tuning* t) {
  if (!q || !t) return fail(SIGMO_ERR_INVALID, "null argument");
  sigmo_tuning n = *t;
  SIGMO_TRY(normalize_tuning(&n));
  q->tune = n;
  return SIGMO_OK;
}

int sigmo_queue_get_tuning(sigmo_queue_t q, sigmo_tuning* t) {
  if (!q || !t) return fail(SIGMO_ERR_INVALID, "null argument");
  *t = q->tune;
  return SIGMO_OK;
}

int sigmo_queue_set_join_budget(sigmo_queue_t q, uint64_t steps) {
  if (!q) return fail(SIGMO_ERR_INVALID, "null queue");
  q->join_budget = steps;
  return SIGMO_OK;
}

int sigmo_queue_get_join_budget(sigmo_queue_t q, uint64_t* steps) {
  if (!q || !steps) return fail(SIGMO_ERR_INVALID, "null argument");
  *steps = q->join_budget;
  return SIGMO_OK;
}

int sigmo_queue_launch_count(sigmo_queue_t q, uint64_t* launches) {
  if (!q || !launches) return fail(SIGMO_ERR_INVALID, "null argument");
  *launches = q->launches;
  return SIGMO_OK;
}

// ---- graphs ----------------------------------------------------------------
int sigmo_graph_create(sigmo_queue_t q, const sigmo_host_graphs* h, sigmo_graph_t* out) {
  if (!q || !h || !out) return fail(SIGMO_ERR_INVALID, "sigmo_graph_create: null argument");
  *out = nullptr;
  SIGMO_TRY(set_device(q));
  if (!h->graph_offsets || !h->row_offsets || (h->total_edges && !h->column_indices) || (h->total_nodes && !h->node_labels))
    return fail(SIGMO_ERR_INVALID, "sigmo_graph_create: null arrays");
  if (h->graph_offsets[h->num_graphs] != h->total_nodes || h->row_offsets[h->total_nodes] != h->total_edges)
    return fail(SIGMO_ERR_INVALID, "sigmo_graph_create: offsets disagree with totals");
  sigmo_graph_t g = new (std::nothrow) sigmo_graph_s();
  if (!g) return fail(SIGMO_ERR_OOM, "host allocation failed");
  g->q = queue_retain(q);
  g->num_graphs = h->num_graphs;
  g->total_nodes = h->total_nodes;
  g->total_edges = h->total_edges;
  g->host_graph_offsets.assign(h->graph_offsets, h->graph_offsets + h->num_graphs + 1);
  int rc = SIGMO_OK;
  auto cp = [&](void** dst, const void* src, size_t bytes) {
    if (rc) return;
    rc = dev_alloc(q, dst, bytes);
    if (rc) return;
    if (bytes) {
      cudaError_t e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, q->stream);
      if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "H2D copy failed: %s", cudaGetErrorString(e));
    }
  };
  cp(reinterpret_cast<void**>(&g->graph_offsets), h->graph_offsets, sizeof(uint32_t) * (h->num_graphs + 1ull));
  cp(reinterpret_cast<void**>(&g->row_offsets), h->row_offsets, sizeof(uint32_t) * (h->total_nodes + 1ull));
  cp(reinterpret_cast<void**>(&g->column_indices), h->column_indices, sizeof(uint32_t) * h->total_edges);
  cp(reinterpret_cast<void**>(&g->node_labels), h->node_labels, h->total_nodes);
  cp(reinterpret_cast<void**>(&g->edge_labels), h->edge_labels, h->total_edges);
  if (!rc) rc = finish_graph(g);
  if (rc) {
    sigmo_graph_destroy(g);
    return rc;
  }
  *out = g;
  return SIGMO_OK;
}

int sigmo_graph_create_device(sigmo_queue_t q, uint32_t num_graphs, uint64_t total_nodes, uint64_t total_edges,
                              const uint32_t* d_graph_offsets, const uint32_t* d_row_offsets,
                              const uint32_t* d_column_indices, const uint8_t* d_node_labels, const uint8_t* d_edge_labels,
                              sigmo_graph_t* out) {
  if (!q || !out || !d_graph_offsets || !d_row_offsets) return fail(SIGMO_ERR_INVALID, "sigmo_graph_create_device: null argument");
  *out = nullptr;
  SIGMO_TRY(set_device(q));
  sigmo_graph_t g = new (std::nothrow) sigmo_graph_s();
  if (!g) return fail(SIGMO_ERR_OOM, "host allocation failed");
  g->q = queue_retain(q);
  g->owned = false;
  g->num_graphs = num_graphs;
  g->total_nodes = total_nodes;
  g->total_edges = total_edges;
  g->graph_offsets = const_cast<uint32_t*>(d_graph_offsets);
  g->row_offsets = const_cast<uint32_t*>(d_row_offsets);
  g->column_indices = const_cast<uint32_t*>(d_column_indices);
  g->node_labels = const_cast<uint8_t*>(d_node_labels);
  g->edge_labels = const_cast<uint8_t*>(d_edge_labels);
  g->host_graph_offsets.resize(num_graphs + 1ull);
  cudaError_t e = cudaMemcpyAsync(g->host_graph_offsets.data(), d_graph_offsets, sizeof(uint32_t) * (num_graphs + 1ull),
                                  cudaMemcpyDeviceToHost, q->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
  int rc = e == cudaSuccess ? SIGMO_OK : fail(SIGMO_ERR_CUDA, "reading graph offsets failed: %s", cudaGetErrorString(e));
  if (!rc && g->host_graph_offsets[num_graphs] != total_nodes)
    rc = fail(SIGMO_ERR_INVALID, "graph_offsets[num_graphs] (%u) != total_nodes (%llu)", g->host_graph_offsets[num_graphs],
              (unsigned long long)total_nodes);
  if (!rc) rc = finish_graph(g);
  if (rc) {
    sigmo_graph_destroy(g);
    return rc;
  }
  *out = g;
  return SIGMO_OK;
}

int sigmo_graph_set_vertex_base(sigmo_graph_t g, uint32_t base) {
  if (!g) return fail(SIGMO_ERR_INVALID, "null graph");
  if (base != 0 && base < kLowOffsetLimit)
    return fail(SIGMO_ERR_DOMAIN, "a shard must start at global vertex 0 or at %u or above (got %u)", kLowOffsetLimit, base);
  if (static_cast<uint64_t>(base) + g->total_nodes > 0xFFFFFFFFull)
    return fail(SIGMO_ERR_DOMAIN, "base + vertices exceeds 2^32");
  g->vertex_base = base;
  uint32_t low = 0;
  for (uint32_t i = 0; i < g->num_graphs; ++i)
    if (static_cast<uint64_t>(g->host_graph_offsets[i]) + base < kLowOffsetLimit) low = i + 1;
  g->low_offset_graphs = low;
  return SIGMO_OK;
}

int sigmo_graph_destroy(sigmo_graph_t g) {
  if (!g) return SIGMO_OK;
  Queue* q = g->q;
  cudaSetDevice(q->device);
  if (g->owned) {
    dev_free(q, g->graph_offsets);
    dev_free(q, g->row_offsets);
    dev_free(q, g->column_indices);
    dev_free(q, g->node_labels);
    dev_free(q, g->edge_labels);
  }
  dev_free(q, g->node_graph);
  dev_free(q, g->adj);
  dev_free(q, g->sym);
  dev_free(q, g->qorder);
  dev_free(q, g->qsel);
  dev_free(q, g->qsel_id);
  release_plane_program(g);
  if (g->ready) cudaEventDestroy(g->ready);
  delete g;
  queue_release(q);
  return SIGMO_OK;
}

int sigmo_graph_info(sigmo_graph_t g, uint32_t* num_graphs, uint64_t* total_nodes, uint64_t* total_edges,
                     uint32_t* max_graph_nodes) {
  if (!g) return fail(SIGMO_ERR_INVALID, "null graph");
  if (num_graphs) *num_graphs = g->num_graphs;
  if (total_nodes) *total_nodes = g->total_nodes;
  if (total_edges) *total_edges = g->total_edges;
  if (max_graph_nodes) *max_graph_nodes = g->max_nodes;
  return SIGMO_OK;
}

int sigmo_graph_alloc_size(sigmo_graph_t g, uint64_t* bytes) {
  if (!g || !bytes) return fail(SIGMO_ERR_INVALID, "null argument");
  // getDeviceCSRGraphAllocSize (graph.hpp:324-328)
  *bytes = g->total_nodes * 1 + (g->num_graphs + 1ull) * 4 + (g->total_nodes + 1) * 4 + g->total_edges * 4 + g->total_edges * 1;
  return SIGMO_OK;
}

// ---- candidates --------------------------------------------------------------
int sigmo_candidates_create(sigmo_queue_t q, uint64_t source_nodes, uint64_t target_nodes, sigmo_candidates_t* out) {
  if (!q || !out) return fail(SIGMO_ERR_INVALID, "sigmo_candidates_create: null argument");
  *out = nullptr;
  SIGMO_TRY(set_device(q));
  sigmo_candidates_t c = new (std::nothrow) sigmo_candidates_s();
  if (!c) return fail(SIGMO_ERR_OOM, "host allocation failed");
  c->q = queue_retain(q);
  c->rows = source_nodes;
  c->targets = target_nodes;
  c->W = (target_nodes + 31) / 32;
  c->Wp = (c->W + 31) / 32 * 32;
  const uint64_t bytes = c->rows * c->Wp * 4;
  int rc = dev_alloc(q, reinterpret_cast<void**>(&c->bits), bytes);
  if (!rc && bytes) {
    cudaError_t e = cudaMemsetAsync(c->bits, 0, bytes, q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "zero fill failed: %s", cudaGetErrorString(e));
  }
  if (rc) {
    sigmo_candidates_destroy(c);
    return rc;
  }
  c->known_zero = true;
  *out = c;
  return SIGMO_OK;
}

int sigmo_candidates_destroy(sigmo_candidates_t c) {
  if (!c) return SIGMO_OK;
  cudaSetDevice(c->q->device);
  Queue* q = c->q;
  dev_free(q, c->bits);
  delete c;
  queue_release(q);
  return SIGMO_OK;
}

int sigmo_candidates_words_per_row(sigmo_candidates_t c, uint64_t* words) {
  if (!c || !words) return fail(SIGMO_ERR_INVALID, "null argument");
  *words = c->W;
  return SIGMO_OK;
}

int sigmo_candidates_alloc_size(sigmo_candidates_t c, uint64_t* bytes) {
  if (!c || !bytes) return fail(SIGMO_ERR_INVALID, "null argument");
  *bytes = c->rows * c->W * 4;
  return SIGMO_OK;
}

int sigmo_candidates_download(sigmo_candidates_t c, uint64_t row0, uint64_t rows, uint32_t* host) {
  if (!c || (!host && rows)) return fail(SIGMO_ERR_INVALID, "null argument");
  if (row0 + rows > c->rows) return fail(SIGMO_ERR_INVALID, "rows [%llu, %llu) outside %llu", (unsigned long long)row0,
                                         (unsigned long long)(row0 + rows), (unsigned long long)c->rows);
  SIGMO_TRY(set_device(c->q));
  if (rows && c->W) {
    SIGMO_CUDA_TRY(cudaMemcpy2DAsync(host, c->W * 4, c->bits + row0 * c->Wp, c->Wp * 4, c->W * 4, rows,
                                     cudaMemcpyDeviceToHost, c->q->stream));
  }
  SIGMO_CUDA_TRY(cudaStreamSynchronize(c->q->stream));
  return SIGMO_OK;
}

int sigmo_candidates_row_counts(sigmo_candidates_t c, uint32_t* host_counts) {
  if (!c || (!host_counts && c->rows)) return fail(SIGMO_ERR_INVALID, "null argument");
  SIGMO_TRY(set_device(c->q));
  if (!c->rows) return SIGMO_OK;
  void* d = nullptr;
  SIGMO_TRY(dev_alloc(c->q, &d, c->rows * 4));
  int rc = launch_row_counts(c->q, c, static_cast<uint32_t*>(d));
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(host_counts, d, c->rows * 4, cudaMemcpyDeviceToHost, c->q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "row counts read-back failed: %s", cudaGetErrorString(e));
  }
  dev_free(c->q, d);
  return rc;
}

int sigmo_candidates_digest(sigmo_candidates_t c, uint64_t* digest) {
  if (!c || !digest) return fail(SIGMO_ERR_INVALID, "null argument");
  SIGMO_TRY(set_device(c->q));
  void* d = nullptr;
  SIGMO_TRY(dev_alloc(c->q, &d, 8));
  int rc = launch_digest(c->q, c, static_cast<uint64_t*>(d));
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(c->q->pinned, d, 8, cudaMemcpyDeviceToHost, c->q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "digest read-back failed: %s", cudaGetErrorString(e));
    else *digest = *static_cast<uint64_t*>(c->q->pinned);
  }
  dev_free(c->q, d);
  return rc;
}

// ---- signatures --------------------------------------------------------------
int sigmo_signature_create(sigmo_queue_t q, uint64_t data_nodes, uint64_t query_nodes, sigmo_signature_t* out) {
  if (!q || !out) return fail(SIGMO_ERR_INVALID, "sigmo_signature_create: null argument");
  *out = nullptr;
  SIGMO_TRY(set_device(q));
  sigmo_signature_t s = new (std::nothrow) sigmo_signature_s();
  if (!s) return fail(SIGMO_ERR_OOM, "host allocation failed");
  s->q = queue_retain(q);
  s->data_nodes = data_nodes;
  s->query_nodes = query_nodes;
  s->reach_words = q->opts.profile == kProfileExact ? kMaxAdjWords : 1u;
  int rc = dev_alloc(q, reinterpret_cast<void**>(&s->data_sig), 8 * data_nodes);
  if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&s->query_sig), 8 * query_nodes);
  if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&s->data_reach), 8ull * s->reach_words * data_nodes);
  if (!rc) rc = dev_alloc(q, reinterpret_cast<void**>(&s->query_reach), 8ull * s->reach_words * query_nodes);
  if (!rc) {
    cudaError_t e = cudaSuccess;
    if (data_nodes) e = cudaMemsetAsync(s->data_sig, 0, 8 * data_nodes, q->stream);
    if (e == cudaSuccess && query_nodes) e = cudaMemsetAsync(s->query_sig, 0, 8 * query_nodes, q->stream);
    if (e == cudaSuccess && data_nodes) e = cudaMemsetAsync(s->data_reach, 0, 8ull * s->reach_words * data_nodes, q->stream);
    if (e == cudaSuccess && query_nodes) e = cudaMemsetAsync(s->query_reach, 0, 8ull * s->reach_words * query_nodes, q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "signature zero fill failed: %s", cudaGetErrorString(e));
  }
  if (rc) {
    sigmo_signature_destroy(s);
    return rc;
  }
  *out = s;
  return SIGMO_OK;
}

int sigmo_signature_destroy(sigmo_signature_t s) {
  if (!s) return SIGMO_OK;
  cudaSetDevice(s->q->device);
  dev_free(s->q, s->data_sig);
  dev_free(s->q, s->query_sig);
  dev_free(s->q, s->data_reach);
  dev_free(s->q, s->query_reach);
  dev_free(s->q, s->data_planes);
  Queue* q = s->q;
  delete s;
  queue_release(q);
  return SIGMO_OK;
}

int sigmo_signature_generate(sigmo_signature_t s, sigmo_graph_t g, int scope) {
  if (!s || !g) return fail(SIGMO_ERR_INVALID, "null argument");
  const bool data = scope == SIGMO_SCOPE_DATA;
  if (g->total_nodes != (data ? s->data_nodes : s->query_nodes))
    return fail(SIGMO_ERR_INVALID, "graph has %llu vertices, signature holds %llu", (unsigned long long)g->total_nodes,
                (unsigned long long)(data ? s->data_nodes : s->query_nodes));
  Queue* q = s->q;
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  SIGMO_TRY(launch_sig_generate(q, g, data ? s->data_sig : s->query_sig));
  if (data) s->planes_valid = false;
  return stage_end(q);
}

int sigmo_signature_refine(sigmo_signature_t s, sigmo_graph_t g, int scope, uint32_t view_size) {
  if (!s || !g) return fail(SIGMO_ERR_INVALID, "null argument");
  const bool data = scope == SIGMO_SCOPE_DATA;
  if (g->total_nodes != (data ? s->data_nodes : s->query_nodes))
    return fail(SIGMO_ERR_INVALID, "graph has %llu vertices, signature holds %llu", (unsigned long long)g->total_nodes,
                (unsigned long long)(data ? s->data_nodes : s->query_nodes));
  Queue* q = s->q;
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  SIGMO_TRY(launch_sig_refine(q, g, view_size, data ? s->data_sig : s->query_sig, data ? s->data_reach : s->query_reach,
                              s->reach_words));
  if (data) s->planes_valid = false;
  return stage_end(q);
}

int sigmo_signature_download(sigmo_signature_t s, int scope, uint64_t* host, uint64_t count) {
  if (!s || (!host && count)) return fail(SIGMO_ERR_INVALID, "null argument");
  const bool data = scope == SIGMO_SCOPE_DATA;
  if (count > (data ? s->data_nodes : s->query_nodes)) return fail(SIGMO_ERR_INVALID, "count exceeds the signature size");
  SIGMO_TRY(set_device(s->q));
  if (count)
    SIGMO_CUDA_TRY(cudaMemcpyAsync(host, data ? s->data_sig : s->query_sig, 8 * count, cudaMemcpyDeviceToHost, s->q->stream));
  SIGMO_CUDA_TRY(cudaStreamSynchronize(s->q->stream));
  return SIGMO_OK;
}

int sigmo_signature_alloc_size(sigmo_signature_t s, int scope, uint64_t* bytes) {
  if (!s || !bytes) return fail(SIGMO_ERR_INVALID, "null argument");
  // getData/QuerySignatureAllocationSize (signature.hpp:181-198): signatures +
  // a 16-byte Bitset<uint64_t> per vertex.
  const uint64_t n = scope == SIGMO_SCOPE_DATA ? s->data_nodes : s->query_nodes;
  *bytes = n * 8 + n * 16;
  return SIGMO_OK;
}

// ---- filter / refine -----------------------------------------------------------
static int check_fgraph(sigmo_graph_t query, sigmo_graph_t data, sigmo_signature_t s, sigmo_candidates_t c) {
  if (!query || !data || !s || !c) return fail(SIGMO_ERR_INVALID, "null argument");
  if (c->rows != query->total_nodes || c->targets != data->total_nodes)
    return fail(SIGMO_ERR_INVALID, "candidates are %llu x %llu, graphs are %llu x %llu", (unsigned long long)c->rows,
                (unsigned long long)c->targets, (unsigned long long)query->total_nodes, (unsigned long long)data->total_nodes);
  if (s->query_nodes != query->total_nodes || s->data_nodes != data->total_nodes)
    return fail(SIGMO_ERR_INVALID, "signature sizes do not match the graphs");
  return SIGMO_OK;
}

int sigmo_filter_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_signature_t s,
                            sigmo_candidates_t c) {
  if (!q) return fail(SIGMO_ERR_INVALID, "null queue");
  SIGMO_TRY(check_fgraph(query, data, s, c));
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  SIGMO_TRY(launch_filter(q, query, data, c));
  return stage_end(q);
}

int sigmo_refine_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_signature_t s,
                            sigmo_candidates_t c) {
  if (!q) return fail(SIGMO_ERR_INVALID, "null queue");
  SIGMO_TRY(check_fgraph(query, data, s, c));
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  if (!s->data_planes || s->planes_Wp != c->Wp) {
    dev_free(q, s->data_planes);
    s->data_planes = nullptr;
    SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&s->data_planes), 16ull * 16 * c->Wp));
    s->planes_Wp = c->Wp;
    s->planes_valid = false;
  }
  if (!s->planes_valid) {
    SIGMO_TRY(launch_sig_planes(q, s->data_sig, s->data_nodes, c->Wp, s->data_planes));
    s->planes_valid = true;
  }
  SIGMO_TRY(launch_refine(q, s->query_sig, s->data_planes, c));
  return stage_end(q);
}

// ---- GMCR ---------------------------------------------------------------------
int sigmo_gmcr_create(sigmo_queue_t q, sigmo_gmcr_t* out) {
  if (!q || !out) return fail(SIGMO_ERR_INVALID, "null argument");
  sigmo_gmcr_t m = new (std::nothrow) sigmo_gmcr_s();
  if (!m) return fail(SIGMO_ERR_OOM, "host allocation failed");
  m->q = queue_retain(q);
  *out = m;
  return SIGMO_OK;
}

int sigmo_gmcr_destroy(sigmo_gmcr_t m) {
  if (!m) return SIGMO_OK;
  cudaSetDevice(m->q->device);
  if (m->graph) cudaGraphExecDestroy(m->graph);
  dev_free(m->q, m->offsets);
  dev_free(m->q, m->indices);
  dev_free(m->q, m->pair_graph);
  dev_free(m->q, m->counts);
  Queue* q = m->q;
  delete m;
  queue_release(q);
  return SIGMO_OK;
}

int sigmo_gmcr_generate(sigmo_gmcr_t m, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c) {
  if (!m || !query || !data || !c) return fail(SIGMO_ERR_INVALID, "null argument");
  if (m->graph) {  // the captured batch refers to the arrays this call may replace
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
    for (auto& k : m->graph_key) k = 0;
  }
  if (c->rows != query->total_nodes || c->targets != data->total_nodes)
    return fail(SIGMO_ERR_INVALID, "candidate bitset does not match the graphs");
  Queue* q = m->q;
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  SIGMO_TRY(launch_gmcr(q, query, data, c, m, true, 0));
  return stage_end(q);
}

int sigmo_gmcr_total(sigmo_gmcr_t m, uint64_t* total) {
  if (!m || !total) return fail(SIGMO_ERR_INVALID, "null argument");
  *total = m->total;
  return SIGMO_OK;
}

int sigmo_gmcr_download(sigmo_gmcr_t m, uint32_t* offsets, uint64_t offsets_len, uint32_t* indices, uint64_t indices_len) {
  if (!m) return fail(SIGMO_ERR_INVALID, "null gmcr");
  SIGMO_TRY(set_device(m->q));
  if (offsets) {
    if (offsets_len < m->num_data_graphs + 1ull) return fail(SIGMO_ERR_INVALID, "offsets buffer too small");
    SIGMO_CUDA_TRY(cudaMemcpyAsync(offsets, m->offsets, 4ull * (m->num_data_graphs + 1), cudaMemcpyDeviceToHost, m->q->stream));
  }
  if (indices && m->total) {
    if (indices_len < m->total) return fail(SIGMO_ERR_INVALID, "indices buffer too small");
    SIGMO_CUDA_TRY(cudaMemcpyAsync(indices, m->indices, 4ull * m->total, cudaMemcpyDeviceToHost, m->q->stream));
  }
  SIGMO_CUDA_TRY(cudaStreamSynchronize(m->q->stream));
  return SIGMO_OK;
}

// ---- join ---------------------------------------------------------------------
int sigmo_join_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c, sigmo_gmcr_t m,
                          uint64_t* num_matches, int find_first, uint64_t* per_pair) {
  if (!q || !query || !data || !c || !m || !num_matches) return fail(SIGMO_ERR_INVALID, "null argument");
  if (m->num_data_graphs != data->num_graphs || !m->offsets) return fail(SIGMO_ERR_INVALID, "GMCR was not generated for this data graph");
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  uint64_t* d_total = nullptr;
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&d_total), 8));
  SIGMO_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, q->stream));
  int rc = join_status_reset(q);
  if (!rc) rc = launch_join_literal(q, query, data, c, m, find_first, 0, data->num_graphs, d_total, 0, 0xFFFFFFFFu);
  if (!rc) rc = stage_end(q);
  if (!rc) rc = join_status_fetch(q);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(q->pinned, d_total, 8, cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess && per_pair && m->total) e = cudaMemcpyAsync(per_pair, m->counts, 8 * m->total, cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "join read-back failed: %s", cudaGetErrorString(e));
    else rc = join_status_result(q);
    if (!rc) {
      *num_matches += *static_cast<uint64_t*>(q->pinned);
      m->counts_valid = true;
    }
  }
  dev_free(q, d_total);
  return rc;
}

// joinWildcardCandidates (isomorphism.hpp:435-560): bond-label-aware join,
// off the driver path (sigmo.cpp never calls it).
int sigmo_join_wildcard_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c, sigmo_gmcr_t m,
                          uint64_t* num_matches, int find_first, uint64_t* per_pair) {
  if (q && q->opts.profile == kProfileX86)
    return fail(SIGMO_ERR_DOMAIN, "joinWildcardCandidates runs under the REF_PTX and EXACT profiles");
  if (!q || !query || !data || !c || !m || !num_matches) return fail(SIGMO_ERR_INVALID, "null argument");
  if (m->num_data_graphs != data->num_graphs || !m->offsets) return fail(SIGMO_ERR_INVALID, "GMCR was not generated for this data graph");
  SIGMO_TRY(set_device(q));
  SIGMO_TRY(stage_begin(q));
  uint64_t* d_total = nullptr;
  SIGMO_TRY(dev_alloc(q, reinterpret_cast<void**>(&d_total), 8));
  SIGMO_CUDA_TRY(cudaMemsetAsync(d_total, 0, 8, q->stream));
  int rc = launch_join_wildcard(q, query, data, c, m, find_first, d_total);
  if (!rc) rc = stage_end(q);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(q->pinned, d_total, 8, cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess && per_pair && m->total) e = cudaMemcpyAsync(per_pair, m->counts, 8 * m->total, cudaMemcpyDeviceToHost, q->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "join read-back failed: %s", cudaGetErrorString(e));
    else {
      *num_matches += *static_cast<uint64_t*>(q->pinned);
      m->counts_valid = true;
    }
  }
  dev_free(q, d_total);
  return rc;
}

int sigmo_match_download_counts(sigmo_gmcr_t m, uint64_t* per_pair, uint64_t len) {
  if (!m || (!per_pair && m->total)) return fail(SIGMO_ERR_INVALID, "null argument");
  if (!m->counts_valid) return fail(SIGMO_ERR_INVALID, "no join has run on this GMCR");
  if (len < m->total) return fail(SIGMO_ERR_INVALID, "buffer of %llu < %llu slots", (unsigned long long)len, (unsigned long long)m->total);
  SIGMO_TRY(set_device(m->q));
  if (m->total) SIGMO_CUDA_TRY(cudaMemcpyAsync(per_pair, m->counts, 8 * m->total, cudaMemcpyDeviceToHost, m->q->stream));
  SIGMO_CUDA_TRY(cudaStreamSynchronize(m->q->stream));
  return SIGMO_OK;
}

}  // extern "C"
