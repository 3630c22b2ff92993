// Shared host-side helpers of the sigmo_b200 library: status/error plumbing.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/sigmo_b200.h"

namespace sigmo_b200 {

// Thread-local message of the last failing call (read by sigmo_last_error).
void set_error_message(const char* msg);
const char* get_error_message();

inline int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  set_error_message(buf);
  return code;
}

// Host-side owned batch helpers (memory from std::malloc; freed by
// sigmo_host_graphs_free).
bool alloc_host_graphs(sigmo_host_graphs* g, uint32_t num_graphs, uint64_t total_nodes, uint64_t total_edges);

}  // namespace sigmo_b200
