/*
 * sigmo_b200 — C ABI of the B200-native SIGMo hot path.
 *
 * The reference (SIGMo, a header-only C++20/SYCL library) exposes no FFI; its
 * boundary is the C++ API that library/src/sigmo.cpp calls.  Every entry point
 * below replaces one of those calls (file:line cited beside it).  Handles are
 * opaque; every function returns a status (SIGMO_OK == 0) and leaves a
 * thread-local message for sigmo_last_error().  No torch types appear here.
 *
 * Semantics profiles.  The reference's hot path contains shift counts that
 * reach the register width and a bitset indexed through uint8_t; its results
 * on the NVIDIA PTX target it was written for are the parity contract:
 *   SIGMO_PROFILE_REF_PTX  (default) shift count >= width yields 0
 *   SIGMO_PROFILE_EXACT    exact sets, correct range masks, injective DFS
 *   SIGMO_PROFILE_REF_X86  shift count taken modulo the width (what the
 *                          reference computes when built for an x86-64 host);
 *                          stage-per-launch calls only
 */
#ifndef SIGMO_B200_H
#define SIGMO_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SIGMO_API __attribute__((visibility("default")))
#else
#define SIGMO_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  SIGMO_OK = 0,
  SIGMO_ERR_INVALID = 1,     /* bad argument / handle / size mismatch        */
  SIGMO_ERR_CUDA = 2,        /* a CUDA runtime call failed                   */
  SIGMO_ERR_OOM = 3,         /* device or host allocation failed             */
  SIGMO_ERR_DOMAIN = 4,      /* input outside the supported domain           */
  SIGMO_ERR_FORMAT = 5,      /* malformed graph text ("Invalid graph format") */
  SIGMO_ERR_NO_DEVICE = 6,   /* no CUDA device / device index out of range    */
  SIGMO_ERR_TIMEOUT = 7      /* a bounded device-side wait ran out            */
};

enum { SIGMO_PROFILE_REF_PTX = 0, SIGMO_PROFILE_REF_X86 = 1, SIGMO_PROFILE_EXACT = 2 };

/* SignatureScope (library/include/signature.hpp:18) */
enum { SIGMO_SCOPE_DATA = 0, SIGMO_SCOPE_QUERY = 1 };

/* Message of the last failing call on this thread ("" if none). */
SIGMO_API const char* sigmo_last_error(void);
/* Library version string. */
SIGMO_API const char* sigmo_version(void);

/* ---- host graphs: io + batching --------------------------------------- */
/* Batched CSR with global vertex ids — the arrays createDeviceCSRGraph builds
 * on the host (library/include/graph.hpp:255-294).  Memory owned by the
 * library when produced by sigmo_parse_graphs / sigmo_generate_*; free with
 * sigmo_host_graphs_free. */
typedef struct sigmo_host_graphs {
  uint32_t num_graphs;
  uint64_t total_nodes;
  uint64_t total_edges;      /* directed CSR entries (2 x undirected edges) */
  uint32_t* graph_offsets;   /* [num_graphs + 1]  first global vertex of g  */
  uint32_t* row_offsets;     /* [total_nodes + 1] global CSR row pointers   */
  uint32_t* column_indices;  /* [total_edges]     global neighbour ids      */
  uint8_t* node_labels;      /* [total_nodes]                               */
  uint8_t* edge_labels;      /* [total_edges]                               */
} sigmo_host_graphs;

/* io::loadCSRGraphsFromLines + createDeviceCSRGraph's host concatenation
 * (library/include/io.hpp:46-55, graph.hpp:154-247, 255-294): one graph per
 * line in the "n#N l#L (id label)xN e#E (u v [label])xE" format; empty lines
 * are skipped.  SIGMO_ERR_FORMAT on a malformed line. */
SIGMO_API int sigmo_parse_graphs(const char* text, size_t len, sigmo_host_graphs* out);
/* Concatenation of already-batched sets (graph order kept; ids re-based). */
SIGMO_API int sigmo_host_graphs_concat(const sigmo_host_graphs* a, const sigmo_host_graphs* b, sigmo_host_graphs* out);
/* Graphs [first, first+count) of a batch as a new batch (ids re-based to 0). */
SIGMO_API int sigmo_host_graphs_slice(const sigmo_host_graphs* in, uint32_t first, uint32_t count, sigmo_host_graphs* out);
/* Write a batch back in the text format (buffer sized by a first call with
 * buf == NULL; *len receives the byte count). */
SIGMO_API int sigmo_format_graphs(const sigmo_host_graphs* in, char* buf, size_t* len);
SIGMO_API void sigmo_host_graphs_free(sigmo_host_graphs* g);
/* Binary batches (no reference counterpart; the reference reads text only):
 * the five arrays as they are, behind a header, so a database loads without
 * parsing.  Loading checks sizes and offsets (SIGMO_ERR_FORMAT otherwise). */
SIGMO_API int sigmo_graphs_save(const sigmo_host_graphs* in, const char* path);
SIGMO_API int sigmo_graphs_load(const char* path, sigmo_host_graphs* out);

/* ---- seeded synthetic inputs (stand-ins for the missing ZINC / SMARTS sets) */
/* kind: 0 = drug-like molecules (sizes uniform in [min_atoms, max_atoms]),
 *       1 = heavy-tailed lognormal sizes (median `median`, clipped to
 *           [min_atoms, max_atoms]) with 5% macrocycles / fused ring systems,
 *       2 = ring-rich molecules (2-6 fused aromatic 6-cycles, carbon chains
 *           up to 20 atoms).
 * Vertex labels use the reference's encoding (scripts/smile2graph.py:13:
 * N=0 Cl=1 *=2 Br=3 I=4 P=5 H=6 O=7 C=8 S=9 F=10); bond labels single=1
 * double=2 triple=3 aromatic=4 (scripts/smile2graph.py:14). */
SIGMO_API int sigmo_generate_molecules(int kind, uint32_t count, uint32_t min_atoms, uint32_t max_atoms, double median,
                             uint64_t seed, sigmo_host_graphs* out);
/* Queries: connected induced subgraphs of freshly seeded molecules (kind as
 * above), sizes in [min_atoms, max_atoms]; skew_lo/skew_hi > 0 skews 70% of
 * the sizes into [skew_lo, skew_hi].  kind 3 = highly automorphic patterns
 * (6-cycles, fused bi/tri-cycles, carbon chains, branched carbon stars). */
SIGMO_API int sigmo_generate_queries(int kind, uint32_t count, uint32_t min_atoms, uint32_t max_atoms, uint32_t skew_lo,
                           uint32_t skew_hi, uint64_t seed, sigmo_host_graphs* out);

/* ---- queue: replaces sycl::queue + device::DeviceOptions ---------------- */
typedef struct sigmo_queue_s* sigmo_queue_t;

typedef struct sigmo_options {
  int profile;                    /* SIGMO_PROFILE_*                          */
  uint32_t join_work_group_size;  /* DeviceOptions, device.hpp:17-21 (128)   */
  uint32_t filter_work_group_size;/* (512) accepted for API parity           */
} sigmo_options;

SIGMO_API void sigmo_default_options(sigmo_options* o);

/* Launch shape of the batched join (no reference counterpart; the
 * reference's only knob is the join work-group size above).  Zero fields take
 * the defaults (overflow_serial and join_kernel: 0 is a value).  sigmo_autotune
 * searches these on a caller's own workload. */
typedef struct sigmo_tuning {
  uint32_t join_blocks_per_sm;   /* persistent join CTAs per SM, 1..4 (4; join_kernel 0 and 1
                                    keep at most 3 resident)                                    */
  uint32_t join_chunk;           /* GMCR slots a lane takes per work grab, 1..64 (4; join_kernel
                                    0 and 1)                                                    */
  uint32_t overflow_blocks;      /* CTAs of the join for queries over 16 vertices (1184)        */
  uint32_t overflow_serial;      /* 0 (default): run those beside the main join; 1: after it       */
  uint32_t mask_chunk_slots;     /* GMCR slots per level-mask pass, in 2^20 units, 1..64 (8)     */
  uint32_t overflow_split;       /* work items per pair of those queries, each taking every
                                    split-th root candidate, 1..64 (16)                          */
  uint32_t join_kernel;          /* 2 (default): per-lane DFS with 9 B of shared state per level
                                    and CTA-local slot regions; 0: per-lane DFS with 17 B per
                                    level and one work cursor; 1: warp-cooperative frontier join
                                    (32 candidate tries per round, one per lane)                 */
  uint32_t join_pool;            /* join_kernel 2: sixteenths of the slots in the pool shared by
                                    all CTAs after their own regions, 1..16 (2)                  */
} sigmo_tuning;
/* sycl::queue{gpu_selector_v, enable_profiling} (library/src/sigmo.cpp:19). */
SIGMO_API int sigmo_queue_create(int device, const sigmo_options* opts, sigmo_queue_t* out);
SIGMO_API int sigmo_queue_destroy(sigmo_queue_t q);
/* queue.wait_and_throw() (sigmo.cpp:103 and after every stage). */
SIGMO_API int sigmo_queue_wait(sigmo_queue_t q);
/* The queue's cudaStream_t (as void*), for callers that order work with it. */
SIGMO_API int sigmo_queue_stream(sigmo_queue_t q, void** stream);
/* The join launch shape used by this queue (defaults until set). */
SIGMO_API int sigmo_queue_set_tuning(sigmo_queue_t q, const sigmo_tuning* t);
SIGMO_API int sigmo_queue_get_tuning(sigmo_queue_t q, sigmo_tuning* t);
/* Step budget of the join kernels (no reference counterpart: the reference's
 * DFS, isomorphism.hpp:330-371, runs until it is done).  steps = the most DFS
 * levels one lane may leave (backtrack from) in one launch, counted per
 * thread of the per-lane joins and per warp of the warp-cooperative one; 0
 * (default) = no limit.  A lane that uses its budget up stops, raises a status
 * word, and lanes that see the word take no further pairs; the call then
 * returns SIGMO_ERR_TIMEOUT and its counts are incomplete.  For callers that
 * must bound the device time of a request (a serving loop that fails one
 * pathological batch instead of holding the GPU). */
SIGMO_API int sigmo_queue_set_join_budget(sigmo_queue_t q, uint64_t steps);
SIGMO_API int sigmo_queue_get_join_budget(sigmo_queue_t q, uint64_t* steps);
/* BatchedEvent::getProfilingInfo (library/include/utils.hpp:149-157): device
 * time of the last stage launched on the queue, after it has completed. */
SIGMO_API int sigmo_queue_last_stage_ms(sigmo_queue_t q, double* ms);
/* Device memory: global_mem_size (sigmo.cpp:20) and name (sigmo.cpp:21). */
SIGMO_API int sigmo_queue_device_info(sigmo_queue_t q, uint64_t* global_mem, char* name, size_t name_len);
/* Kernels launched by this library on this queue since creation. */
SIGMO_API int sigmo_queue_launch_count(sigmo_queue_t q, uint64_t* launches);

/* ---- device batched CSR graph (DeviceBatchedCSRGraph, graph.hpp:62-112) -- */
typedef struct sigmo_graph_s* sigmo_graph_t;

/* createDeviceCSRGraph (graph.hpp:255-314): copies the batch to the device. */
SIGMO_API int sigmo_graph_create(sigmo_queue_t q, const sigmo_host_graphs* host, sigmo_graph_t* out);
/* Same, but the five arrays are already device-resident (no copy; the caller
 * keeps ownership and must keep them alive). */
SIGMO_API int sigmo_graph_create_device(sigmo_queue_t q, uint32_t num_graphs, uint64_t total_nodes, uint64_t total_edges,
                              const uint32_t* d_graph_offsets, const uint32_t* d_row_offsets,
                              const uint32_t* d_column_indices, const uint8_t* d_node_labels,
                              const uint8_t* d_edge_labels, sigmo_graph_t* out);
/* createDeviceCSRGraph with the batching done on the device (the reference
 * concatenates on the host, graph.hpp:254-314, "TODO offload on GPU"): the
 * graphs' own CSR arrays back to back with local ids — node_counts[g],
 * edge_counts[g] (directed entries), each graph's n_g + 1 row pointers from 0
 * (sum n_g + num_graphs entries), local neighbour ids, node and edge labels
 * (edge_labels may be NULL: all 0).  Host arrays, copied as they are; offsets
 * are scanned and ids rebased on the device.  SIGMO_ERR_INVALID if a local id
 * or row pointer is outside its graph. */
SIGMO_API int sigmo_graph_create_from_local(sigmo_queue_t q, uint32_t num_graphs, const uint32_t* node_counts,
                                            const uint32_t* edge_counts, const uint32_t* row_offsets_local,
                                            const uint32_t* columns_local, const uint8_t* node_labels,
                                            const uint8_t* edge_labels, sigmo_graph_t* out);
/* Marks a data batch as a shard of a larger one whose vertex 0 has global id
 * `base` (no reference counterpart; the reference's MPI ranks restart ids at
 * 0, sigmo_mpi.cpp:114,126).  REF_PTX results depend on global ids (the
 * range-mask rule at 32-vertex words, the live `visited` bitset below vertex
 * 256), so a shard keeps the semantics of the unsharded batch.  base must be
 * 0 or >= 256 (the graphs starting below vertex 256 stay in the first shard);
 * sigmo_match_batched then gives the shard's part of the unsharded GMCR and
 * counts.  Used by the batched form's planes route only. */
SIGMO_API int sigmo_graph_set_vertex_base(sigmo_graph_t g, uint32_t base);
/* destroyDeviceCSRGraph (graph.hpp:316-322). */
SIGMO_API int sigmo_graph_destroy(sigmo_graph_t g);
SIGMO_API int sigmo_graph_info(sigmo_graph_t g, uint32_t* num_graphs, uint64_t* total_nodes, uint64_t* total_edges,
                     uint32_t* max_graph_nodes);
/* getDeviceGraphAllocSize (graph.hpp:324-328, 423-432). */
SIGMO_API int sigmo_graph_alloc_size(sigmo_graph_t g, uint64_t* bytes);

/* ---- candidate bitsets (candidates::Candidates, candidates.hpp:14-204) ---- */
typedef struct sigmo_candidates_s* sigmo_candidates_t;

/* Candidates(queue, source_nodes, target_nodes): zero-filled bit matrix
 * (candidates.hpp:165-179).  Rows are padded on the device to a multiple of
 * 32 words (128 B); the host view is the reference's dense [source][W]. */
SIGMO_API int sigmo_candidates_create(sigmo_queue_t q, uint64_t source_nodes, uint64_t target_nodes, sigmo_candidates_t* out);
SIGMO_API int sigmo_candidates_destroy(sigmo_candidates_t c);
/* Words per row in the reference layout: ceil(target_nodes / 32). */
SIGMO_API int sigmo_candidates_words_per_row(sigmo_candidates_t c, uint64_t* words);
/* getAllocationSize (candidates.hpp:196): bytes of the reference layout. */
SIGMO_API int sigmo_candidates_alloc_size(sigmo_candidates_t c, uint64_t* bytes);
/* getHostCandidates (candidates.hpp:185-190): rows [row0, row0+rows) into
 * host memory, dense [rows][W] uint32. */
SIGMO_API int sigmo_candidates_download(sigmo_candidates_t c, uint64_t row0, uint64_t rows, uint32_t* host);
/* Per-row candidate counts (getCandidatesCount(source), candidates.hpp:77-81)
 * computed on the device; host array of source_nodes entries. */
SIGMO_API int sigmo_candidates_row_counts(sigmo_candidates_t c, uint32_t* host_counts);
/* XOR/rotate digest of every row (order-sensitive), for checks at sizes whose
 * bitset does not fit in host memory. */
SIGMO_API int sigmo_candidates_digest(sigmo_candidates_t c, uint64_t* digest);

/* ---- signatures (signature::Signature<PowerGraph,4>, signature.hpp:20-391) */
typedef struct sigmo_signature_s* sigmo_signature_t;

/* Signature(queue, data_nodes, query_nodes): zeroed signatures and reachables
 * (signature.hpp:157-168; the reference leaves reachables unzeroed). */
SIGMO_API int sigmo_signature_create(sigmo_queue_t q, uint64_t data_nodes, uint64_t query_nodes, sigmo_signature_t* out);
SIGMO_API int sigmo_signature_destroy(sigmo_signature_t s);
/* generate{Data,Query}Signatures -> generateCSRSignatures (signature.hpp:57-69,125-152). */
SIGMO_API int sigmo_signature_generate(sigmo_signature_t s, sigmo_graph_t g, int scope);
/* refine{Data,Query}Signatures(g, view_size) -> refineCSRSignatures<PowerGraph>
 * (signature.hpp:62-74,336-390). */
SIGMO_API int sigmo_signature_refine(sigmo_signature_t s, sigmo_graph_t g, int scope, uint32_t view_size);
/* Copy the current signatures of a scope to host (uint64 per vertex). */
SIGMO_API int sigmo_signature_download(sigmo_signature_t s, int scope, uint64_t* host, uint64_t count);
/* getData/QuerySignatureAllocationSize (signature.hpp:181-198). */
SIGMO_API int sigmo_signature_alloc_size(sigmo_signature_t s, int scope, uint64_t* bytes);

/* ---- filter / refine (isomorphism::filter, isomorphism.hpp:22-127) -------- */
/* filterCandidates<Query> (isomorphism.hpp:22-62). */
SIGMO_API int sigmo_filter_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_signature_t s,
                            sigmo_candidates_t c);
/* refineCandidates<Query> (isomorphism.hpp:64-127), race-free. */
SIGMO_API int sigmo_refine_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_signature_t s,
                            sigmo_candidates_t c);

/* ---- GMCR mapping (isomorphism::mapping::GMCR, gmcr.hpp:16-131) ---------- */
typedef struct sigmo_gmcr_s* sigmo_gmcr_t;

SIGMO_API int sigmo_gmcr_create(sigmo_queue_t q, sigmo_gmcr_t* out);          /* GMCR(queue) gmcr.hpp:26 */
SIGMO_API int sigmo_gmcr_destroy(sigmo_gmcr_t m);
/* generateGMCR (gmcr.hpp:33-128).  Query ids within a data graph's segment
 * are ascending; queries with <= 1 vertex are never admitted. */
SIGMO_API int sigmo_gmcr_generate(sigmo_gmcr_t m, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c);
/* total_query_indices (gmcr.hpp:81-82). */
SIGMO_API int sigmo_gmcr_total(sigmo_gmcr_t m, uint64_t* total);
/* data_graph_offsets [num_data_graphs+1] and query_graph_indices [total]. */
SIGMO_API int sigmo_gmcr_download(sigmo_gmcr_t m, uint32_t* offsets, uint64_t offsets_len, uint32_t* indices,
                        uint64_t indices_len);

/* GMCR into caller-owned device buffers, with no device allocation at all.
 * This entry point has no counterpart in the reference.  It is for callers
 * that cannot allocate device memory while it runs: code working inside a
 * fixed device-memory arena owned by another allocator, real-time services
 * that forbid cudaMalloc/cudaFree on their request path after start-up, and
 * callers that cannot afford the implicit synchronisation an allocation may
 * bring.  Results equal sigmo_gmcr_generate's: d_offsets receives
 * data_graph_offsets [num_data_graphs + 1], d_indices the first *total
 * query_graph_indices (capacity = d_indices length in entries), *total the
 * number of admitted pairs (also returned with SIGMO_ERR_INVALID when it
 * exceeds capacity).  Intermediates live in one 32 MiB device array that is
 * part of the library (every GPU that loads it holds the array until exit):
 * batches needing more (query vertices x ceil(data graphs / 32) x 4 bytes plus
 * query graphs x the same, plus 4 bytes per data graph, plus the device scan's
 * temporary storage, each piece rounded up to 256 bytes) are rejected with
 * SIGMO_ERR_DOMAIN.  The first call on a device resolves the array's device
 * address; make that first call before any stream capture.  Every call shares
 * the array, so calls whose work overlaps on the GPU (several queues or
 * threads at once) race; the array keeps the last call's contents.  Every
 * call, not only the first, waits on its queue once (cudaStreamSynchronize,
 * to read the admitted total back to the host); its last kernel may still be
 * running on return — wait on the queue before reading d_indices. */
SIGMO_API int sigmo_gmcr_generate_noalloc(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c,
                                          uint32_t* d_offsets, uint32_t* d_indices, uint64_t capacity, uint64_t* total);

/* ---- join (isomorphism::join::joinCandidates, isomorphism.hpp:270-381) ---- */
/* Adds the number of matches to *num_matches (host, caller-zeroed, like the
 * reference's USM counter, sigmo.cpp:145-146).  find_first: at most one match
 * per (query, data graph) pair.  per_pair (nullable, host) receives the count
 * of every GMCR slot (total_query_indices entries). */
SIGMO_API int sigmo_join_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c,
                          sigmo_gmcr_t m, uint64_t* num_matches, int find_first, uint64_t* per_pair);
/* joinWildcardCandidates (isomorphism.hpp:435-560, with defineMatchingOrder
 * :383-408 and isValidMapping :410-433): the reference's opt-in join that
 * roots each pair's DFS at the query vertex with the most candidates, splits
 * the root's candidates over the 32 lanes of a sub-group and also requires
 * equal bond (edge) labels on query edges.  The driver (sigmo.cpp) never calls
 * it.  find_first ends each lane's DFS at its first match, so the count is
 * then the number of root candidates that extend to a match.  per_pair: the
 * count of every GMCR slot (nullable). */
SIGMO_API int sigmo_join_wildcard_candidates(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, sigmo_candidates_t c,
                                             sigmo_gmcr_t m, uint64_t* num_matches, int find_first, uint64_t* per_pair);

/* ---- batched form: whole pipeline in one call ----------------------------
 * Signatures for iterations 1..R in one BFS, per-data-graph candidate planes
 * (one u64 vertex mask per distinct query label and per distinct (iteration,
 * label, count) threshold), GMCR from the AND-programs of identical-vertex
 * classes, and the persistent work-stealing join — the same GMCR and counts
 * as the stage-per-launch calls (sigmo.cpp:98-160) with one host
 * synchronisation.  The final candidate bitset is not written unless
 * SIGMO_MATCH_MATERIALIZE_BITSET is given (then `c` receives it); `c` may be
 * NULL otherwise.  GMCR and per-pair counts stay on the device in `m`. */
enum { SIGMO_MATCH_MATERIALIZE_BITSET = 1,
       /* Graph mode (no reference counterpart): the first call with these
        * graphs runs normally and then captures the batch's device work into
        * a CUDA graph kept on `m`; later calls with the same query and data
        * graphs, iterations, mode, profile and tuning replay it (one launch,
        * one host synchronisation).  A replay whose admitted total differs
        * from the captured one (the graphs' device arrays were changed) runs
        * and captures again.  Stage times other than ms_total are 0 on a
        * replay. */
       SIGMO_MATCH_CUDA_GRAPH = 2 };

typedef struct sigmo_match_result {
  uint64_t total_matches;     /* sum over admitted pairs                     */
  uint64_t admitted_pairs;    /* total_query_indices of the GMCR             */
  uint64_t pairs;             /* num_query_graphs x num_data_graphs           */
  double ms_signatures;       /* device time per stage (CUDA events)         */
  double ms_filter;
  double ms_mapping;
  double ms_join;
  double ms_total;
} sigmo_match_result;

SIGMO_API int sigmo_match_batched(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, uint32_t iterations,
                        int find_first, uint32_t flags, sigmo_candidates_t c, sigmo_gmcr_t m, sigmo_match_result* out);
/* Autotuner (no reference counterpart): runs sigmo_match_batched on these
 * graphs under candidate join launch shapes (coordinate descent over the
 * sigmo_tuning fields, `reps` timed runs per candidate, median join time),
 * keeps the fastest on the queue and returns it.  Every candidate must give
 * the same total as the default shape, or the call fails. */
SIGMO_API int sigmo_autotune(sigmo_queue_t q, sigmo_graph_t query, sigmo_graph_t data, uint32_t iterations, int find_first,
                             uint32_t reps, sigmo_tuning* best, double* best_ms, double* default_ms);
/* Per-pair counts of the last sigmo_match_batched call on `m` (GMCR slot order). */
SIGMO_API int sigmo_match_download_counts(sigmo_gmcr_t m, uint64_t* per_pair, uint64_t len);

/* ---- serving loop (no reference counterpart) ----------------------------
 * The reference answers one query batch per process run (library/src/
 * sigmo.cpp:98-160).  A server keeps one molecule database resident on the
 * device (CSR, adjacency rows, signatures of iterations 1..R) and answers
 * query requests with continuous batching: each of `max_inflight` workers
 * takes the queued requests in arrival order (up to `max_batch_queries` query
 * graphs), admits the batch once its projected device footprint fits
 * `memory_budget` beside the batches already running, and runs the batched
 * form on its own stream, so batches overlap on the device.  A request's
 * results are those it gets alone: per (query graph, molecule) pair, the
 * count of sigmo_match_batched (find-first: 0/1). */
typedef struct sigmo_server_s* sigmo_server_t;

typedef struct sigmo_server_options {
  uint32_t iterations;         /* refinement iterations R (default 6)                         */
  int32_t find_first;          /* 1 (default): per-pair match flags; 0: embedding counts      */
  uint32_t max_inflight;       /* batches on the device at once, 1..16 (default 2)            */
  uint32_t max_batch_queries;  /* query graphs per batch (default 64); a larger request runs alone */
  uint64_t memory_budget;      /* device bytes the running batches may hold (0: half the free memory
                                  after the database is resident)                              */
  uint32_t batch_window_us;    /* wait up to this long for a batch to fill (default 0)        */
  uint64_t join_step_budget;   /* the workers' join step budget (sigmo_queue_set_join_budget;
                                  0, the default: none); a batch that runs out fails its
                                  requests with SIGMO_ERR_TIMEOUT and the server goes on      */
} sigmo_server_options;

enum { SIGMO_REQUEST_PAIRS = 1 };  /* keep the matched (query, molecule, count) list */

typedef struct sigmo_request_result {
  int32_t status;              /* SIGMO_OK or the request's error                              */
  uint32_t num_queries;
  uint64_t pairs;              /* num_queries x molecules                                      */
  uint64_t matched_pairs;      /* pairs with a non-zero count                                  */
  uint64_t total_matches;      /* sum of the counts (find-first: == matched_pairs)             */
  uint64_t batch_id;           /* the device batch the request ran in                          */
  uint32_t batch_queries;      /* query graphs in that batch (all its requests)               */
  uint32_t batch_requests;
  uint64_t projected_bytes;    /* the batch's admitted device footprint                        */
  double ms_queue;             /* submit -> batch start (host clock)                           */
  double ms_device;            /* the batch's stream time, upload to results (CUDA events)     */
  double ms_latency;           /* submit -> results on the host (host clock)                   */
  double ms_filter;            /* the batch's stages (CUDA events; sigmo_match_result)         */
  double ms_mapping;
  double ms_join;
  uint64_t gathered_plane_bytes; /* resident plane rows the batch's admission read (0 when the
                                    planes were built for the batch); / ms_filter = its
                                    gather bandwidth                                           */
} sigmo_request_result;

typedef struct sigmo_server_stats {
  uint64_t requests_submitted, requests_completed, requests_failed, queries_completed;
  uint64_t batches, pairs, admitted_pairs;
  double device_ms;                 /* sum over batches                                        */
  uint64_t peak_reserved_bytes;     /* largest sum of admitted footprints                      */
  uint32_t max_batches_in_flight;
  uint32_t pending_requests;
  uint64_t resident_bytes;          /* database arrays kept on the device                      */
  uint64_t memory_budget;
} sigmo_server_stats;

SIGMO_API void sigmo_server_default_options(sigmo_server_options* o);
/* Uploads the database (copied; the caller keeps `database`) and starts the
 * workers.  SIGMO_ERR_DOMAIN for molecules of more than 256 atoms. */
SIGMO_API int sigmo_server_create(int device, const sigmo_host_graphs* database, const sigmo_options* opts,
                                  const sigmo_server_options* so, sigmo_server_t* out);
/* Queues a request (the query graphs are copied) and returns at once. */
SIGMO_API int sigmo_server_submit(sigmo_server_t s, const sigmo_host_graphs* queries, uint32_t flags, uint64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit; SIGMO_ERR_TIMEOUT when it
 * runs out).  Returns the request's own status. */
SIGMO_API int sigmo_server_wait(sigmo_server_t s, uint64_t ticket, int64_t timeout_ms, sigmo_request_result* out);
/* Per query graph of a finished request: matched molecules and total count. */
SIGMO_API int sigmo_server_query_totals(sigmo_server_t s, uint64_t ticket, uint64_t* matched, uint64_t* total, uint32_t n);
/* Matched pairs of a request submitted with SIGMO_REQUEST_PAIRS, in molecule
 * then query order (query index within the request); *n receives the count,
 * min(*n, capacity) entries are copied. */
SIGMO_API int sigmo_server_pairs(sigmo_server_t s, uint64_t ticket, uint32_t* query, uint32_t* molecule, uint64_t* count,
                                 uint64_t capacity, uint64_t* n);
/* Forgets a finished request. */
SIGMO_API int sigmo_server_release(sigmo_server_t s, uint64_t ticket);
SIGMO_API int sigmo_server_get_stats(sigmo_server_t s, sigmo_server_stats* out);
/* Finishes the queued requests, stops the workers, frees the database. */
SIGMO_API int sigmo_server_destroy(sigmo_server_t s);

#ifdef __cplusplus
}
#endif

#endif /* SIGMO_B200_H */
