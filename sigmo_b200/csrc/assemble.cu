// Device-side batch assembly (createDeviceCSRGraph, graph.hpp:255-314, whose
// host concatenation is marked "TODO offload on GPU" at graph.hpp:254).
//
// The input is what a caller holds per molecule: each graph's own CSR with
// local ids, placed back to back (node and directed-edge counts per graph,
// each graph's n+1 row pointers starting at 0, local neighbour ids, labels).
// Those arrays are copied as they are; graph offsets and edge bases are two
// device scans, and global row pointers and neighbour ids are rebased on the
// device, with every local id checked against its graph's size.  The result
// is the same batched CSR as sigmo_graph_create on the host-concatenated batch.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <new>
#include <vector>

#include "internal.hpp"

namespace sigmo_b200 {
namespace {

// Global row pointers: local row entry j of graph g (0 <= j <= n_g) sits at
// position graph_offsets[g] + g + j of the back-to-back local arrays; entries
// j < n_g become row_offsets[graph_offsets[g] + j] = edge_base[g] + local.
// The graph of an entry is found by binary search over graph_offsets[g] + g.
__global__ void k_rebase_rows(const uint32_t* __restrict__ goff, const uint64_t* __restrict__ ebase, uint32_t G,
                              const uint32_t* __restrict__ local_rows, uint64_t n_entries, uint32_t* __restrict__ rows,
                              unsigned int* __restrict__ bad) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n_entries;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t lo = 0, hi = G;  // last g with goff[g] + g <= i
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (static_cast<uint64_t>(goff[mid]) + mid <= i) lo = mid;
      else hi = mid;
    }
    const uint32_t g = lo;
    const uint64_t j = i - (static_cast<uint64_t>(goff[g]) + g);
    const uint32_t n = goff[g + 1] - goff[g];
    const uint64_t e = ebase[g + 1] - ebase[g];
    const uint32_t r = local_rows[i];
    if (r > e || (j == 0 && r != 0) || (j == n && r != e)) atomicOr(bad, 1u);
    if (j < n) rows[goff[g] + j] = static_cast<uint32_t>(ebase[g] + r);
  }
}

// Global neighbour ids: entry k of graph g (edge_base[g] <= k < edge_base[g+1])
// gets graph_offsets[g] added; a local id >= n_g is an error.
__global__ void k_rebase_cols(const uint32_t* __restrict__ goff, const uint64_t* __restrict__ ebase, uint32_t G,
                              const uint32_t* __restrict__ local_cols, uint64_t E, uint32_t* __restrict__ cols,
                              unsigned int* __restrict__ bad) {
  for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < E;
       k += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t lo = 0, hi = G;  // last g with ebase[g] <= k
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (ebase[mid] <= k) lo = mid;
      else hi = mid;
    }
    const uint32_t g = lo;
    const uint32_t c = local_cols[k];
    if (c >= goff[g + 1] - goff[g]) atomicOr(bad, 2u);
    cols[k] = goff[g] + c;
  }
}

__global__ void k_widen(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    out[i] = in[i];
}

}  // namespace
}  // namespace sigmo_b200

using namespace sigmo_b200;

extern "C" int sigmo_graph_create_from_local(sigmo_queue_t q, uint32_t num_graphs, const uint32_t* node_counts,
                                             const uint32_t* edge_counts, const uint32_t* row_offsets_local,
                                             const uint32_t* columns_local, const uint8_t* node_labels,
                                             const uint8_t* edge_labels, sigmo_graph_t* out) {
  if (!q || !out || (num_graphs && (!node_counts || !edge_counts || !row_offsets_local)))
    return fail(SIGMO_ERR_INVALID, "sigmo_graph_create_from_local: null argument");
  *out = nullptr;
  SIGMO_CUDA_TRY(cudaSetDevice(q->device));
  // sizes: O(graphs) on the host (the per-element work is on the device)
  uint64_t N = 0, E = 0;
  std::vector<uint32_t> goff(num_graphs + 1ull, 0);
  for (uint32_t g = 0; g < num_graphs; ++g) {
    N += node_counts[g];
    E += edge_counts[g];
    if (N > 0xFFFFFFFFull || E > 0xFFFFFFFFull) return fail(SIGMO_ERR_DOMAIN, "batch exceeds 2^32 vertices or CSR entries");
    goff[g + 1] = static_cast<uint32_t>(N);
  }
  if ((N && !node_labels) || (E && !columns_local)) return fail(SIGMO_ERR_INVALID, "sigmo_graph_create_from_local: null arrays");
  sigmo_graph_t g = new (std::nothrow) sigmo_graph_s();
  if (!g) return fail(SIGMO_ERR_OOM, "host allocation failed");
  g->q = queue_retain(q);
  g->num_graphs = num_graphs;
  g->total_nodes = N;
  g->total_edges = E;
  g->host_graph_offsets = goff;
  const uint64_t n_entries = N + num_graphs;  // every graph's n+1 row pointers
  int rc = SIGMO_OK;
  void* scratch = nullptr;
  auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
  size_t cub_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, static_cast<const uint64_t*>(nullptr), static_cast<uint64_t*>(nullptr),
                                static_cast<int>(num_graphs + 1), q->stream);
  const uint64_t b_rows = al(4 * n_entries), b_cols = al(4 * E), b_counts = al(8ull * (num_graphs + 1)), b_ecnt = al(4ull * num_graphs);
  auto alloc = [&](void** p, uint64_t bytes) {
    if (!rc) rc = dev_alloc(q, p, bytes ? bytes : 4);
  };
  auto h2d = [&](void* dst, const void* src, uint64_t bytes) {
    if (!rc && bytes && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, q->stream) != cudaSuccess)
      rc = fail(SIGMO_ERR_CUDA, "H2D copy failed");
  };
  alloc(reinterpret_cast<void**>(&g->graph_offsets), 4ull * (num_graphs + 1));
  alloc(reinterpret_cast<void**>(&g->row_offsets), 4 * (N + 1));
  alloc(reinterpret_cast<void**>(&g->column_indices), 4 * E);
  alloc(reinterpret_cast<void**>(&g->node_labels), N);
  alloc(reinterpret_cast<void**>(&g->edge_labels), E);
  alloc(&scratch, b_rows + b_cols + 2 * b_counts + b_ecnt + al(cub_bytes) + 256);
  char* p = static_cast<char*>(scratch);
  uint32_t* d_lrows = reinterpret_cast<uint32_t*>(p);
  p += b_rows;
  uint32_t* d_lcols = reinterpret_cast<uint32_t*>(p);
  p += b_cols;
  uint64_t* d_ecnt64 = reinterpret_cast<uint64_t*>(p);
  p += b_counts;
  uint64_t* d_ebase = reinterpret_cast<uint64_t*>(p);
  p += b_counts;
  uint32_t* d_ecnt = reinterpret_cast<uint32_t*>(p);
  p += b_ecnt;
  void* cub_tmp = p;
  p += al(cub_bytes);
  unsigned int* d_bad = reinterpret_cast<unsigned int*>(p);
  h2d(g->graph_offsets, goff.data(), 4ull * (num_graphs + 1));
  h2d(d_lrows, row_offsets_local, 4 * n_entries);
  h2d(d_lcols, columns_local, 4 * E);
  h2d(d_ecnt, edge_counts, 4ull * num_graphs);
  h2d(g->node_labels, node_labels, N);
  if (edge_labels) h2d(g->edge_labels, edge_labels, E);
  else if (!rc && E && cudaMemsetAsync(g->edge_labels, 0, E, q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
  if (!rc && cudaMemsetAsync(d_bad, 0, 4, q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
  if (!rc && cudaMemsetAsync(d_ecnt64, 0, 8ull * (num_graphs + 1), q->stream) != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "memset failed");
  if (!rc && num_graphs) {
    k_widen<<<grid_for(num_graphs, 256, 148u * 8u), 256, 0, q->stream>>>(d_ecnt, num_graphs, d_ecnt64);
    rc = check_launch(q, "k_widen");
  }
  if (!rc) {
    const cudaError_t e = cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, d_ecnt64, d_ebase, static_cast<int>(num_graphs + 1),
                                                       q->stream);
    if (e != cudaSuccess) rc = fail(SIGMO_ERR_CUDA, "edge scan failed: %s", cudaGetErrorString(e));
    q->launches += 2;
  }
  if (!rc && num_graphs) {
    k_rebase_rows<<<grid_for(n_entries, 256, 148u * 16u), 256, 0, q->stream>>>(g->graph_offsets, d_ebase, num_graphs, d_lrows,
                                                                               n_entries, g->row_offsets, d_bad);
    rc = check_launch(q, "k_rebase_rows");
  }
  const uint32_t e32 = static_cast<uint32_t>(E);
  h2d(g->row_offsets + N, &e32, 4);
  if (!rc && E) {
    k_rebase_cols<<<grid_for(E, 256, 148u * 16u), 256, 0, q->stream>>>(g->graph_offsets, d_ebase, num_graphs, d_lcols, E,
                                                                       g->column_indices, d_bad);
    rc = check_launch(q, "k_rebase_cols");
  }
  unsigned int bad = 0;
  if (!rc && (cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
              cudaStreamSynchronize(q->stream) != cudaSuccess))
    rc = fail(SIGMO_ERR_CUDA, "assembly read-back failed");
  if (!rc && bad)
    rc = fail(SIGMO_ERR_INVALID, "sigmo_graph_create_from_local: %s", (bad & 2u) ? "a local neighbour id is outside its graph"
                                                                                 : "a graph's row pointers are inconsistent");
  if (scratch) dev_free(q, scratch);
  if (!rc) rc = finish_graph(g);
  if (rc) {
    sigmo_graph_destroy(g);
    return rc;
  }
  *out = g;
  return SIGMO_OK;
}
