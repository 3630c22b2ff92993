// A host-CPU stand-in for the part of SYCL 2020 that SIGMo's hot path uses —
// TEST INFRASTRUCTURE ONLY (it lets oracle/ref_build.py compile the
// reference's own headers with g++ and run them on the host as the checker of
// the oracle; nothing in the product uses it).
//
// Execution model.  A range<D> kernel runs its work-items one after another.
// An nd_range<D> kernel runs one work-group at a time; its work-items are
// cooperative fibers switched round robin: every group_barrier and
// every group / sub-group collective is a yield point, and one pass over the
// fibers moves each work-item to its next yield point, so all members of a
// work-group (or sub-group) meet at each barrier as SYCL requires (x86-64
// only: the switch is a few lines of assembly).  Work-groups
// run in ascending order.  Sub-groups are 32 work-items (the NVIDIA width the
// reference was written for).  Each fiber starts on a zero-filled stack, so
// the private arrays the reference leaves uninitialised start at zero.
//
// USM allocations are host memory with a slack of 1 MiB past the end (the
// reference's refinement kernel reads and writes a few words past the last
// candidate row when the row length is not a multiple of 16 words).
// Events are complete when returned; their profiling times are host clock
// readings around the kernel.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifndef SYCL_EXTERNAL
#define SYCL_EXTERNAL
#endif

namespace sycl {

// ---- index spaces ------------------------------------------------------------
template <int D = 1>
struct range {
  size_t v[D];
  range() { for (auto& x : v) x = 0; }
  range(size_t a) { static_assert(D == 1, "range<1>"); v[0] = a; }
  range(size_t a, size_t b) { static_assert(D == 2, "range<2>"); v[0] = a; v[1] = b; }
  size_t operator[](int d) const { return v[d]; }
  size_t& operator[](int d) { return v[d]; }
  size_t size() const { size_t s = 1; for (auto x : v) s *= x; return s; }
};

template <int D = 1>
struct id {
  size_t v[D];
  id() { for (auto& x : v) x = 0; }
  size_t operator[](int d) const { return v[d]; }
  size_t get(int d) const { return v[d]; }
  template <int E = D, typename = std::enable_if_t<E == 1>>
  operator size_t() const { return v[0]; }
};

template <int D = 1>
struct item {
  id<D> idx;
  range<D> r;
  size_t get_id(int d) const { return idx.v[d]; }
  id<D> get_id() const { return idx; }
  size_t get_range(int d) const { return r.v[d]; }
  size_t get_linear_id() const {
    size_t s = 0;
    for (int d = 0; d < D; ++d) s = s * r.v[d] + idx.v[d];
    return s;
  }
  size_t operator[](int d) const { return idx.v[d]; }
  operator id<D>() const { return idx; }
  template <int E = D, typename = std::enable_if_t<E == 1>>
  operator size_t() const { return idx.v[0]; }
};

template <int D = 1>
struct nd_range {
  range<D> g, l;
  nd_range(range<D> global, range<D> local) : g(global), l(local) {}
  range<D> get_global_range() const { return g; }
  range<D> get_local_range() const { return l; }
};

// ---- fibers: the work-items of one work-group -----------------------------------
// A fiber switch saves the callee-saved registers and the stack pointer of the
// running context and resumes another (x86-64 System V; no signal mask is
// touched, unlike swapcontext, so a switch costs a few nanoseconds).
extern "C" void sigmo_host_fiber_switch(void** save_sp, void* next_sp);
asm(R"(
  .text
  .globl sigmo_host_fiber_switch
  .type sigmo_host_fiber_switch, @function
sigmo_host_fiber_switch:
  pushq %rbp
  pushq %rbx
  pushq %r12
  pushq %r13
  pushq %r14
  pushq %r15
  movq %rsp, (%rdi)
  movq %rsi, %rsp
  popq %r15
  popq %r14
  popq %r13
  popq %r12
  popq %rbx
  popq %rbp
  ret
  .size sigmo_host_fiber_switch, .-sigmo_host_fiber_switch
)");

namespace detail {

constexpr size_t kFiberStack = 128 * 1024;
constexpr size_t kZeroedTop = 32 * 1024;  // the top of each stack is zero-filled per work-item

struct FiberGroup {
  std::vector<void*> sp;  // saved stack pointer of each fiber
  std::vector<uint8_t> done;
  void* main_sp = nullptr;
  size_t current = 0;
  std::function<void(size_t)> body;
  // one value slot per work-item for group collectives
  std::vector<uint64_t> slots;
};

inline FiberGroup*& current_group() {
  static thread_local FiberGroup* g = nullptr;
  return g;
}

[[noreturn]] inline void fiber_entry() {
  FiberGroup* fg = current_group();
  const size_t i = fg->current;
  fg->body(i);
  fg->done[i] = 1;
  sigmo_host_fiber_switch(&fg->sp[i], fg->main_sp);
  __builtin_unreachable();
}

// Yield point: back to the scheduler, which resumes this work-item in the next pass.
inline void yield() {
  FiberGroup* fg = current_group();
  if (!fg) return;  // a range kernel: nothing to wait for
  const size_t i = fg->current;
  sigmo_host_fiber_switch(&fg->sp[i], fg->main_sp);
}

inline void run_group(size_t n, const std::function<void(size_t)>& body) {
  static thread_local std::vector<char*> pool;
  FiberGroup fg;
  fg.sp.resize(n);
  fg.done.assign(n, 0);
  fg.slots.assign(n, 0);
  fg.body = body;
  while (pool.size() < n) {
    char* s = static_cast<char*>(std::malloc(kFiberStack));
    if (!s) throw std::runtime_error("sycl host: fiber stack allocation failed");
    pool.push_back(s);
  }
  for (size_t i = 0; i < n; ++i) {
    char* top = pool[i] + kFiberStack;
    std::memset(top - kZeroedTop, 0, kZeroedTop);
    // initial frame, popped by the first switch into the fiber: six saved
    // registers, then fiber_entry as the return address; the entry then runs
    // with the stack aligned as after a call
    auto* f = reinterpret_cast<void**>(top - 64);
    for (int r = 0; r < 6; ++r) f[r] = nullptr;
    f[6] = reinterpret_cast<void*>(&fiber_entry);
    f[7] = nullptr;
    fg.sp[i] = f;
  }
  FiberGroup* saved = current_group();
  current_group() = &fg;
  for (bool any = true; any;) {
    any = false;
    for (size_t i = 0; i < n; ++i) {
      if (fg.done[i]) continue;
      fg.current = i;
      sigmo_host_fiber_switch(&fg.main_sp, fg.sp[i]);
      any = true;
    }
  }
  current_group() = saved;
}

}  // namespace detail

// ---- groups --------------------------------------------------------------------
template <int D = 1>
struct group {
  size_t gid, ngroups, lid, lsize;
  size_t get_group_linear_id() const { return gid; }
  size_t get_group_linear_range() const { return ngroups; }
  size_t get_local_linear_id() const { return lid; }
  range<D> get_local_range() const { return range<D>(lsize); }
  size_t get_local_linear_range() const { return lsize; }
  bool leader() const { return lid == 0; }
};

struct sub_group {
  size_t sgid, nsg, lane, size;
  size_t get_group_linear_id() const { return sgid; }
  size_t get_group_linear_range() const { return nsg; }
  size_t get_local_linear_id() const { return lane; }
  range<1> get_local_range() const { return range<1>(size); }
  bool leader() const { return lane == 0; }
};

constexpr size_t kSubGroupSize = 32;

template <int D = 1>
struct nd_item {
  size_t gid_, lid_, lsize_, ngroups_;
  size_t get_global_id(int) const { return gid_ * lsize_ + lid_; }
  size_t get_global_linear_id() const { return gid_ * lsize_ + lid_; }
  size_t get_local_id(int) const { return lid_; }
  size_t get_local_linear_id() const { return lid_; }
  size_t get_group_linear_id() const { return gid_; }
  size_t get_group(int) const { return gid_; }
  size_t get_local_range(int) const { return lsize_; }
  size_t get_global_range(int) const { return ngroups_ * lsize_; }
  group<D> get_group() const { return group<D>{gid_, ngroups_, lid_, lsize_}; }
  sub_group get_sub_group() const {
    const size_t nsg = (lsize_ + kSubGroupSize - 1) / kSubGroupSize;
    const size_t sg = lid_ / kSubGroupSize;
    const size_t size = std::min(kSubGroupSize, lsize_ - sg * kSubGroupSize);
    return sub_group{sg, nsg, lid_ % kSubGroupSize, size};
  }
};

template <int D>
inline void group_barrier(const group<D>&) { detail::yield(); }
inline void group_barrier(const sub_group&) { detail::yield(); }

template <typename T = void>
struct plus {
  template <typename A, typename B>
  auto operator()(const A& a, const B& b) const { return a + b; }
};
template <typename T = void>
struct maximum {
  template <typename A, typename B>
  auto operator()(const A& a, const B& b) const { return a > b ? a : b; }
};
template <typename T = void>
struct minimum {
  template <typename A, typename B>
  auto operator()(const A& a, const B& b) const { return a < b ? a : b; }
};

namespace detail {
// Every member writes its value, all meet, each folds the members' values in
// order, all meet again before the slots are reused.
template <typename T, typename Op>
T reduce_members(size_t first, size_t count, size_t me, T x, Op op) {
  FiberGroup* fg = current_group();
  static_assert(sizeof(T) <= sizeof(uint64_t), "collective value wider than 64 bits");
  uint64_t raw = 0;
  std::memcpy(&raw, &x, sizeof(T));
  fg->slots[me] = raw;
  yield();
  T acc{};
  for (size_t i = 0; i < count; ++i) {
    T v;
    std::memcpy(&v, &fg->slots[first + i], sizeof(T));
    acc = i == 0 ? v : static_cast<T>(op(acc, v));
  }
  yield();
  return acc;
}
}  // namespace detail

template <int D, typename T, typename Op>
T reduce_over_group(const group<D>& g, T x, Op op) {
  return detail::reduce_members<T>(0, g.lsize, g.lid, x, op);
}
template <typename T, typename Op>
T reduce_over_group(const sub_group& sg, T x, Op op) {
  const size_t first = sg.sgid * kSubGroupSize;
  return detail::reduce_members<T>(first, sg.size, first + sg.lane, x, op);
}

// ---- atomics (work-items never run at the same time) ------------------------------
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, private_space, generic_space };
}

template <typename T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::generic_space>
struct atomic_ref {
  T& r;
  explicit atomic_ref(T& ref) : r(ref) {}
  T load() const { return r; }
  void store(T v) const { r = v; }
  operator T() const { return r; }
  T operator=(T v) const { return r = v; }
  T fetch_add(T v) const { T o = r; r = static_cast<T>(r + v); return o; }
  T fetch_sub(T v) const { T o = r; r = static_cast<T>(r - v); return o; }
  T fetch_or(T v) const { T o = r; r = static_cast<T>(r | v); return o; }
  T fetch_and(T v) const { T o = r; r = static_cast<T>(r & v); return o; }
  T fetch_max(T v) const { T o = r; r = std::max(r, v); return o; }
  T fetch_min(T v) const { T o = r; r = std::min(r, v); return o; }
  T operator+=(T v) const { return r = static_cast<T>(r + v); }
  T operator-=(T v) const { return r = static_cast<T>(r - v); }
  T operator|=(T v) const { return r = static_cast<T>(r | v); }
  T operator&=(T v) const { return r = static_cast<T>(r & v); }
  T operator++(int) const { return fetch_add(1); }
  T operator++() const { return r = static_cast<T>(r + 1); }
};

// ---- integer and math built-ins ------------------------------------------------------
template <typename T>
inline T popcount(T x) { return static_cast<T>(__builtin_popcountll(static_cast<unsigned long long>(x))); }
template <typename T>
inline T ctz(T x) {
  if (x == 0) return static_cast<T>(sizeof(T) * 8);
  return static_cast<T>(__builtin_ctzll(static_cast<unsigned long long>(x)));
}
template <typename T>
inline T clz(T x) {
  if (x == 0) return static_cast<T>(sizeof(T) * 8);
  return static_cast<T>(__builtin_clzll(static_cast<unsigned long long>(x)) - (64 - sizeof(T) * 8));
}
using std::sqrt;

// ---- device, events, queue ---------------------------------------------------------------
namespace info {
namespace device {
struct name {};
struct global_mem_size {};
struct max_work_group_size {};
}  // namespace device
namespace queue {
struct device {};
}  // namespace queue
namespace event_profiling {
struct command_start {};
struct command_end {};
}  // namespace event_profiling
}  // namespace info

struct device {
  template <typename P>
  auto get_info() const {
    if constexpr (std::is_same_v<P, info::device::name>) return std::string("host CPU (SIGMo SYCL stand-in)");
    else if constexpr (std::is_same_v<P, info::device::global_mem_size>) return static_cast<size_t>(1) << 34;
    else return static_cast<size_t>(1024);
  }
};

struct event {
  uint64_t t0 = 0, t1 = 0;
  void wait() const {}
  void wait_and_throw() const {}
  template <typename P>
  uint64_t get_profiling_info() const {
    if constexpr (std::is_same_v<P, info::event_profiling::command_start>) return t0;
    else return t1;
  }
};

inline uint64_t host_ns() {
  return static_cast<uint64_t>(
      std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count());
}

template <typename T, int D = 1>
struct local_accessor {
  std::shared_ptr<std::vector<T>> mem;
  template <typename H>
  local_accessor(size_t n, H&) : mem(std::make_shared<std::vector<T>>(n)) {}
  T& operator[](size_t i) const { return (*mem)[i]; }
};

namespace detail {
template <int D, typename K>
void run_range(const range<D>& r, const K& k) {
  item<D> it;
  it.r = r;
  if constexpr (D == 1) {
    for (size_t i = 0; i < r.v[0]; ++i) {
      it.idx.v[0] = i;
      k(it);
    }
  } else {
    for (size_t i = 0; i < r.v[0]; ++i)
      for (size_t j = 0; j < r.v[1]; ++j) {
        it.idx.v[0] = i;
        it.idx.v[1] = j;
        k(it);
      }
  }
}

template <typename K>
void run_nd(const nd_range<1>& nr, const K& k) {
  const size_t L = nr.l.v[0];
  if (L == 0 || nr.g.v[0] % L) throw std::runtime_error("sycl host: global range is not a multiple of the local range");
  const size_t G = nr.g.v[0] / L;
  for (size_t g = 0; g < G; ++g)
    run_group(L, [&](size_t lid) { k(nd_item<1>{g, lid, L, G}); });
}
}  // namespace detail

struct handler {
  event ev;
  template <typename Name = void, int D, typename K>
  void parallel_for(range<D> r, const K& k) {
    ev.t0 = host_ns();
    detail::run_range(r, k);
    ev.t1 = host_ns();
  }
  template <typename Name = void, typename K>
  void parallel_for(nd_range<1> r, const K& k) {
    ev.t0 = host_ns();
    detail::run_nd(r, k);
    ev.t1 = host_ns();
  }
  template <typename Name = void, typename K>
  void single_task(const K& k) {
    ev.t0 = host_ns();
    k();
    ev.t1 = host_ns();
  }
  void depends_on(const event&) {}
  void depends_on(const std::vector<event>&) {}
};

namespace property {
namespace queue {
struct enable_profiling {};
struct in_order {};
}  // namespace queue
}  // namespace property
struct property_list {
  template <typename... P>
  property_list(P...) {}
};

struct gpu_selector_t {};
inline constexpr gpu_selector_t gpu_selector_v{};
struct default_selector_t {};
inline constexpr default_selector_t default_selector_v{};

struct queue {
  queue() = default;
  template <typename S>
  explicit queue(const S&) {}
  template <typename S>
  queue(const S&, const property_list&) {}

  template <typename F>
  event submit(F f) {
    handler h;
    f(h);
    return h.ev;
  }
  template <typename Name = void, int D, typename K>
  event parallel_for(range<D> r, const K& k) {
    handler h;
    h.parallel_for<Name>(r, k);
    return h.ev;
  }
  template <typename Name = void, typename K>
  event parallel_for(nd_range<1> r, const K& k) {
    handler h;
    h.parallel_for<Name>(r, k);
    return h.ev;
  }
  template <typename Name = void, typename K>
  event single_task(const K& k) {
    handler h;
    h.single_task<Name>(k);
    return h.ev;
  }
  template <typename T>
  event fill(T* p, const T& v, size_t n) {
    std::fill(p, p + n, v);
    return event{};
  }
  template <typename T, typename V>
  event fill(T* p, const V& v, size_t n) {
    std::fill(p, p + n, static_cast<T>(v));
    return event{};
  }
  event memset(void* p, int v, size_t n) {
    std::memset(p, v, n);
    return event{};
  }
  event memcpy(void* d, const void* s, size_t n) {
    std::memmove(d, s, n);
    return event{};
  }
  template <typename T>
  event copy(const T* src, T* dst, size_t n) {
    std::memmove(dst, src, n * sizeof(T));
    return event{};
  }
  void wait() {}
  void wait_and_throw() {}
  sycl::device get_device() const { return sycl::device{}; }
  template <typename P>
  sycl::device get_info() const { return sycl::device{}; }
};

// ---- unified shared memory -----------------------------------------------------------------
namespace detail {
constexpr size_t kSlack = 1 << 20;
inline void* usm_alloc(size_t bytes) {
  void* p = std::calloc(1, bytes + kSlack);
  if (!p) throw std::runtime_error("sycl host: allocation failed");
  return p;
}
}  // namespace detail
template <typename T>
T* malloc_device(size_t n, const queue&) { return static_cast<T*>(detail::usm_alloc(n * sizeof(T))); }
template <typename T>
T* malloc_host(size_t n, const queue&) { return static_cast<T*>(detail::usm_alloc(n * sizeof(T))); }
template <typename T>
T* malloc_shared(size_t n, const queue&) { return static_cast<T*>(detail::usm_alloc(n * sizeof(T))); }
inline void free(void* p, const queue&) { std::free(p); }

// ---- buffers (used by the reference's query adjacency-matrix path only) ---------------------
template <typename T, int D = 1>
struct buffer {
  std::shared_ptr<std::vector<T>> mem;
  explicit buffer(size_t n) : mem(std::make_shared<std::vector<T>>(n)) {}
  buffer(range<D> r) : mem(std::make_shared<std::vector<T>>(r.size())) {}
};
template <typename T, int D = 1>
struct host_accessor {
  std::shared_ptr<std::vector<T>> mem;
  host_accessor(buffer<T, D>& b) : mem(b.mem) {}
  T& operator[](size_t i) const { return (*mem)[i]; }
};
template <typename T, int D>
host_accessor(buffer<T, D>&) -> host_accessor<T, D>;

}  // namespace sycl
