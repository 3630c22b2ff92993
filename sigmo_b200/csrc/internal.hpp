// Handle types and launch plumbing of the sigmo_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <vector>

#include "common.hpp"
#include "device.cuh"

namespace sigmo_b200 {

struct ResidentPlanes;

#define SIGMO_CUDA_TRY(expr)                                                                       \
  do {                                                                                             \
    cudaError_t _e = (expr);                                                                       \
    if (_e != cudaSuccess)                                                                         \
      return ::sigmo_b200::fail(_e == cudaErrorMemoryAllocation ? SIGMO_ERR_OOM : SIGMO_ERR_CUDA, \
                                "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, \
                                __LINE__);                                                         \
  } while (0)

#define SIGMO_TRY(expr)      \
  do {                       \
    int _rc = (expr);        \
    if (_rc != SIGMO_OK) return _rc; \
  } while (0)

struct Queue {
  int device = 0;
  cudaStream_t stream = nullptr;
  sigmo_options opts{};
  sigmo_tuning tune{4, 4, 148 * 8, 0, 8, 16, 2, 2};
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
  bool stage_recorded = false;
  uint64_t launches = 0;
  // Scratch reused by stages (grown on demand, freed with the queue).
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  void* pinned = nullptr;  // small pinned host buffer for scalar read-backs
  cudaStream_t side = nullptr;  // second stream for work that overlaps the main one
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // third stream: the join's odd chunks (level masks of one chunk overlap the
  // join of the previous one), with its fork/join events and the events after
  // each stream's last level-mask pass
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_aux_fork = nullptr, ev_aux_join = nullptr, ev_masks[2] = {nullptr, nullptr};
  // Join step budget (0: none) and the device status word the join kernels
  // raise when a lane runs out of it (kJoinStatusBudget).
  uint64_t join_budget = 0;
  unsigned int* d_status = nullptr;
  // References: the caller's handle plus one per graph, candidate bitset,
  // signature and GMCR created on the queue.  sigmo_queue_destroy drops the
  // caller's; the queue (its streams, which those objects free their memory
  // on) is released with the last reference, whatever the order of the
  // destroy calls.
  std::atomic<int> refs{1};
};
Queue* queue_retain(Queue* q);
void queue_release(Queue* q);

// What a join kernel gets of the queue's step budget: the most DFS levels one
// lane (one warp for the frontier join) may leave in a launch, 0 for no limit,
// and the status word it sets when the budget runs out; the lane then stops,
// and lanes that see the word take no further work.
struct JoinLimit {
  uint64_t budget;
  unsigned int* status;
};
constexpr unsigned kJoinStatusBudget = 1u;
inline JoinLimit join_limit(const Queue* q) { return JoinLimit{q->join_budget, q->d_status}; }
// Byte offset in the queue's pinned buffer where the status word is read back.
constexpr size_t kPinnedStatusOffset = 64;
// Clears the status word on the queue's stream (before the join kernels).
int join_status_reset(Queue* q);
// Queues the read-back of the status word into the pinned buffer (before the
// host synchronises), and after the synchronisation turns a raised word into
// SIGMO_ERR_TIMEOUT.
int join_status_fetch(Queue* q);
int join_status_result(Queue* q);

// A contiguous range of query graphs whose planes fit one k_planes_admit
// tile in shared memory (a batch too large for one tile is admitted group by
// group).  Device arrays are in group-local plane ids; row_of maps a local
// plane to its row in the batch's plane array.
struct PlaneGroup {
  uint32_t q0 = 0, q1 = 0;
  uint32_t K = 0, C = 0, nlab = 0;
  uint32_t* spec = nullptr;      // [K]
  uint32_t* r_begin = nullptr;   // [R + 1]
  uint32_t* row_of = nullptr;    // [K] plane row in the batch
  uint16_t* prog = nullptr;      // the group's class programs, local plane ids
  uint32_t* qc_off = nullptr;    // [q1 - q0 + 1]
  uint32_t* qc = nullptr;        // per entry in evaluation order, its local program range (begin, end)
  size_t n_qc = 0, n_prog = 0;
};

// Per-query-batch plane program of the batched form (kernels_planes.cu).
struct PlaneProgram {
  bool valid = false;
  uint32_t R = 0;
  int profile = 0;
  uint32_t K = 0;                 // planes per data graph
  uint32_t C = 0;                 // classes of identical query vertices
  uint32_t* spec = nullptr;       // [K] plane definitions
  uint32_t* prog_off = nullptr;   // [C + 1]
  uint16_t* prog = nullptr;       // plane indices of each class's program
  uint32_t* cls = nullptr;        // [query vertices] class of each vertex
  uint32_t nlab = 0;              // label planes (spec[0 .. nlab))
  uint32_t* r_begin = nullptr;    // [R + 1] first threshold plane of each iteration
  uint32_t max_len = 0;           // longest program
  // host copies (class evaluation order)
  std::vector<uint32_t> h_spec, h_prog_off, h_cls, h_qgoff;
  std::vector<uint16_t> h_prog;
  // per query graph, its distinct classes in evaluation order for one data
  // graph's label frequencies (rebuilt when the data graph changes)
  uint32_t* qc_off = nullptr;     // [query graphs + 1]
  uint32_t* qc = nullptr;         // per entry, its class's program range in prog: (begin, end) u32 pairs
  size_t h_qc_n = 0;              // entries of qc
  std::vector<PlaneGroup> groups; // empty: the whole batch fits one tile
  const void* qc_for = nullptr;   // the data graph the order was built for
  uint64_t qc_stamp = 0;
  uint64_t* qsig_all = nullptr;   // [R][query vertices] signatures, iterations 1..R
};

struct Graph {
  Queue* q = nullptr;
  bool owned = true;
  uint32_t num_graphs = 0;
  uint64_t total_nodes = 0, total_edges = 0;
  uint32_t* graph_offsets = nullptr;
  uint32_t* row_offsets = nullptr;
  uint32_t* column_indices = nullptr;
  uint8_t* node_labels = nullptr;
  uint8_t* edge_labels = nullptr;
  // Derived on the device at creation:
  uint32_t max_nodes = 0;          // largest graph
  uint32_t adj_words = 1;          // u64 words per local adjacency row (<= 4)
  uint32_t* node_graph = nullptr;  // [total_nodes] graph id of each vertex
  uint64_t* adj = nullptr;         // [total_nodes * adj_words] local neighbour sets
  uint8_t* sym = nullptr;          // [num_graphs] 1 if the adjacency is mirrored
  uint32_t low_offset_graphs = 0;  // graphs whose first vertex is < 256
  uint32_t vertex_base = 0;        // global id of vertex 0 when the batch is a shard of a larger one
  // Query-side matching orders (built on first use by the batched join):
  uint8_t* qorder = nullptr;       // [total_nodes] local id placed at level k
  uint64_t* qsel = nullptr;        // [total_nodes] adjacency to earlier levels
  uint64_t* qsel_id = nullptr;     // [total_nodes] same, identity order
  std::vector<uint32_t> host_graph_offsets;  // host copy (sizes, dispatch)
  std::vector<uint64_t> label_hist;          // vertices per label (filled on first use, 256 entries)
  uint64_t stamp = 0;                        // unique per graph object (cache keys)
  cudaEvent_t ready = nullptr;               // recorded after the creation work on the queue's stream
  PlaneProgram pp;                 // when this graph is the query side of a batched match
};

struct Candidates {
  Queue* q = nullptr;
  uint64_t rows = 0;     // source_nodes (query vertices)
  uint64_t targets = 0;  // target_nodes (data vertices)
  uint64_t W = 0;        // reference words per row: ceil(targets / 32)
  uint64_t Wp = 0;       // device row stride in words (W rounded up to 32)
  uint32_t* bits = nullptr;
  bool known_zero = true;  // no bit set since the last zero fill
};

struct Signature {
  Queue* q = nullptr;
  uint64_t data_nodes = 0, query_nodes = 0;
  uint64_t* data_sig = nullptr;
  uint64_t* query_sig = nullptr;
  uint64_t* data_reach = nullptr;
  uint64_t* query_reach = nullptr;
  uint32_t reach_words = 1;  // 1 (REF_PTX) or 4 (EXACT)
  uint32_t* data_planes = nullptr;  // bit-sliced data signatures [16][Wp] x uint4 (k_sig_planes)
  uint64_t planes_Wp = 0;
  bool planes_valid = false;
};

struct Gmcr {
  Queue* q = nullptr;
  uint32_t num_data_graphs = 0;
  uint32_t* offsets = nullptr;  // [num_data_graphs + 1]
  uint32_t* indices = nullptr;  // [capacity]
  uint32_t* pair_graph = nullptr;  // data graph of each slot [capacity]
  uint64_t* counts = nullptr;   // per-slot match counts of the last join
  uint64_t total = 0;
  uint64_t capacity = 0;
  bool counts_valid = false;
  // CUDA graph of the last batched match run in graph mode, and what it was built for
  cudaGraphExec_t graph = nullptr;
  uint64_t graph_key[7] = {0, 0, 0, 0, 0, 0, 0};  // inputs, mode, profile, tuning, join budget
  uint64_t graph_launches = 0;  // kernels in the captured batch
};

// Stage timing: every public stage brackets its launches with these.
int stage_begin(Queue* q);
int stage_end(Queue* q);

// Stream-ordered device allocation on the queue's stream.
int dev_alloc(Queue* q, void** p, size_t bytes);
void dev_free(Queue* q, void* p);
// Per-call temporaries (freed before the call returns): stream-ordered, from
// a pool of their own per device that keeps its memory, so a call's buffers
// are carved from blocks the previous calls freed even when the caller
// creates and destroys graphs between calls (graph arrays come from the
// device's default pool).  Inside a stream capture they come from the
// default pool as graph memory nodes.  Free with dev_free.
int tmp_alloc(Queue* q, void** p, size_t bytes);
// Queue-owned scratch of at least `bytes` (contents undefined).
int queue_scratch(Queue* q, size_t bytes, void** p);

inline unsigned grid_for(uint64_t work, unsigned block, unsigned cap = 0x7FFFFFFFu) {
  uint64_t g = (work + block - 1) / block;
  if (g == 0) g = 1;
  return static_cast<unsigned>(g < cap ? g : cap);
}

int check_launch(Queue* q, const char* what);

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum
// once per (kernel, device).  Kernels launched with different dynamic sizes
// from several host threads (the serving workers) must not lower it for one
// another, so the limit is only ever set to the maximum.
int allow_max_dynamic_smem(const void* kernel, int device);

// ---- kernel launchers (defined in the .cu files) --------------------------
int launch_graph_derive(Graph* g);
// Sizes, low-offset count and the derived arrays of a new device graph whose
// host_graph_offsets and device arrays are set.
int finish_graph(Graph* g);
int launch_query_order(Graph* g);
int launch_sig_generate(Queue* q, const Graph* g, uint64_t* sig);
int launch_sig_refine(Queue* q, const Graph* g, uint32_t view, uint64_t* sig, uint64_t* reach, uint32_t reach_words);
int launch_sig_all(Queue* q, const Graph* g, uint32_t R, uint64_t* sig_all /* [R][N] */);
int launch_sig_planes(Queue* q, const uint64_t* sig, uint64_t n, uint64_t Wp, uint32_t* planes);
int launch_filter(Queue* q, const Graph* query, const Graph* data, Candidates* c);
int launch_refine(Queue* q, const uint64_t* qsig, const uint32_t* planes, Candidates* c);
int launch_fused_filter(Queue* q, const Graph* query, const Graph* data, uint32_t R, const uint64_t* qsig_all,
                        const uint32_t* planes_all, Candidates* c);
int launch_gmcr(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, bool sync_total,
                uint64_t capacity_hint);
// Query graphs [q_begin, q_end) of each segment only (the full range: 0, ~0u).
int launch_join_literal(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                        uint32_t graph_begin, uint32_t graph_end, uint64_t* d_total, uint32_t q_begin, uint32_t q_end);
int launch_join_fast(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                     uint64_t* d_total);
int launch_join_wildcard(Queue* q, const Graph* query, const Graph* data, const Candidates* c, Gmcr* m, int find_first,
                         uint64_t* d_total);
// planes: [graph / 32][planes_rows][AW][32]; prog: the class programs as
// row indices into it (pp.prog for the per-batch planes).
// reserve: persistent join CTA slots left free for a kernel running beside it
int launch_join_fast_planes(Queue* q, const Graph* query, const Graph* data, const PlaneProgram& pp, const uint64_t* planes,
                            uint32_t planes_rows, const uint16_t* prog, Gmcr* m, int find_first, uint64_t* d_total,
                            uint32_t reserve = 0);
int launch_gmcr_from_ne(Queue* q, const Graph* query, const Graph* data, const uint32_t* NE, const uint32_t* cls, Gmcr* m,
                        bool sync_total, uint64_t capacity_hint);
int launch_planes_admit(Queue* q, const Graph* query, const Graph* data, const uint64_t* sig_all, uint32_t R,
                        const PlaneProgram& pp, uint64_t* planes, uint32_t* admit, uint32_t* counts);
// One group of a batch: its planes go to their rows of the batch's planes
// (K_total rows per tile), its admission words to its query graphs' rows, and
// its per-graph admitted counts are added to counts.
int launch_planes_admit_group(Queue* q, const Graph* query, const Graph* data, const uint64_t* sig_all, uint32_t R,
                              const PlaneGroup& grp, uint32_t K_total, uint64_t* planes, uint32_t* admit, uint32_t* counts);
// Shared memory of one k_planes_admit tile budgeted for a query group's planes.
constexpr size_t kGroupSmemBudget = 96u * 1024u;
// The same admission with the tile's planes gathered from resident planes
// (row_map[k] = resident row of the batch's plane k).
int launch_planes_admit_resident(Queue* q, const Graph* query, const Graph* data, const ResidentPlanes& rp,
                                 const PlaneProgram& pp, const uint32_t* row_map, uint32_t* admit, uint32_t* counts);
size_t planes_admit_smem(uint32_t K, uint32_t AW);
// GMCR from admission words admit[query graph][data graph / 32] and the
// admitted count of every data graph (scan, total, sorted fill).
int launch_gmcr_from_admit(Queue* q, const Graph* query, const Graph* data, const uint32_t* admit, const uint32_t* counts,
                           Gmcr* m, bool sync_total, uint64_t capacity_hint);
// Vertices per label of a graph batch (host copy, computed once).
int ensure_label_hist(Queue* q, Graph* g);
int launch_fused_filter_raw(Queue* q, const uint8_t* qlab, const uint64_t* qsig_all, uint64_t Qn, const uint8_t* dlab,
                            uint64_t N, const uint32_t* planes_all, uint64_t Wstride, uint32_t R, uint32_t* bits);
int launch_row_counts(Queue* q, const Candidates* c, uint32_t* d_counts);
int build_plane_program(Queue* q, Graph* query, uint32_t R);
// Fills zero fields of a tuning with the defaults and checks the ranges.
int normalize_tuning(sigmo_tuning* t);

// Options of the batched form beyond the C entry point (the serving loop):
// data signatures already resident ([R][N], iterations 1..R), and the query
// graph ranges of the requests batched together (nranges + 1 boundaries) so
// the literal join of the low-offset graphs runs per request.
// Planes of every threshold that occurs in a resident database (the serving
// loop): rows [tile][rows][AW][32] u64; row `zero_row` is all zeros (a
// threshold above every vertex's count, or a label that never occurs).
struct ResidentPlanes {
  uint64_t* planes = nullptr;
  uint32_t rows = 0;
  uint32_t zero_row = 0;
  uint32_t R = 0;
  std::vector<uint32_t> label_row;  // [256]
  std::vector<uint32_t> base_row;   // [R][16]: row of (r, l, c = 1)
  std::vector<uint8_t> cmax;        // [R][16]: largest count of label l at distance r+1 in any molecule
};
int build_resident_planes(Queue* q, Graph* data, const uint64_t* sig_all, uint32_t R, ResidentPlanes* out);

struct BatchedRun {
  bool capture = false;  // the work is being captured into a CUDA graph: no host synchronisation
  const ResidentPlanes* resident = nullptr;
  const uint64_t* dsig = nullptr;
  const uint32_t* query_ranges = nullptr;
  uint32_t nranges = 0;
};
int match_batched(Queue* q, Graph* query, Graph* data, uint32_t R, int find_first, bool materialize, Candidates* c, Gmcr* m,
                  sigmo_match_result* out, const BatchedRun& run, bool graph = false);
void release_plane_program(Graph* g);
int launch_digest(Queue* q, const Candidates* c, uint64_t* d_digest);

}  // namespace sigmo_b200

// The opaque handle types of the C ABI are the internal structs.
struct sigmo_queue_s : sigmo_b200::Queue {};
struct sigmo_graph_s : sigmo_b200::Graph {};
struct sigmo_candidates_s : sigmo_b200::Candidates {};
struct sigmo_signature_s : sigmo_b200::Signature {};
struct sigmo_gmcr_s : sigmo_b200::Gmcr {};
