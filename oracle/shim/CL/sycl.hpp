// Test infrastructure only (oracle build). A host-CPU stand-in for the small
// part of SYCL that the reference's Lyapunov path uses, so that the reference's
// own sources compile unchanged with g++ and run on the host cores.
//
// Semantics follow SYCL 2020 for the pieces used:
//   * nd_range<3>/nd_item<3> with the work decomposed along dimension 2 only
//     (cuda/lyapunov.dp.cpp:342-347 builds range(1,1,bn)*range(1,1,bs));
//   * queue::submit runs the command group synchronously; parallel_for hands
//     work-items to a pool of std::threads (CHAOS_REF_THREADS, default: all
//     hardware threads).  Every work-item runs exactly once, so the reference's
//     per-work-item scratch offsets (index*dim) stay private to one thread;
//   * malloc_device returns zeroed host memory (calloc), which also defines the
//     reference's never-zeroed accumulators (lyapExps, projSum).
#pragma once
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <iostream>
#include <thread>
#include <vector>

#define SYCL_EXTERNAL

namespace sycl {

using std::acos;
using std::fabs;
using std::log;
using std::sqrt;
template <class T> inline T pow(T x, T y) { return std::pow(x, y); }

struct exception : public std::exception {
  const char *what() const noexcept override { return "sycl shim exception"; }
};

template <int D> struct range {
  size_t e[3];
  range(size_t a, size_t b, size_t c) { e[0] = a; e[1] = b; e[2] = c; }
  range operator*(const range &o) const {
    return range(e[0] * o.e[0], e[1] * o.e[1], e[2] * o.e[2]);
  }
};

template <int D> struct nd_range {
  range<D> global, local;
  nd_range(range<D> g, range<D> l) : global(g), local(l) {}
};

template <int D> struct nd_item {
  size_t group, lid, lrange, grange;
  size_t get_group(int) const { return group; }
  size_t get_local_id(int) const { return lid; }
  size_t get_local_range(int) const { return lrange; }
  size_t get_group_range(int) const { return grange; }
};

inline unsigned shim_threads() {
  const char *s = std::getenv("CHAOS_REF_THREADS");
  unsigned n = s ? (unsigned)std::atoi(s) : std::thread::hardware_concurrency();
  return n ? n : 1u;
}

struct handler {
  template <class Kernel> void parallel_for(nd_range<3> r, Kernel k) {
    const size_t lr = r.local.e[2];
    const size_t gr = r.global.e[2] / lr;
    const long total = (long)(gr * lr);
    std::atomic<long> next{0};
    auto worker = [&]() {
      for (;;) {
        long g = next.fetch_add(1);
        if (g >= total) break;
        nd_item<3> it{(size_t)g / lr, (size_t)g % lr, lr, gr};
        k(it);
      }
    };
    unsigned nt = shim_threads();
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
  }
};

struct stream {
  stream(size_t, size_t, handler &) {}
  const stream &operator<<(const char *s) const {
    std::fputs(s, stderr);
    return *this;
  }
};

struct event {
  void wait() {}
};

struct queue {
  event memcpy(void *dst, const void *src, size_t n) {
    std::memcpy(dst, src, n);
    return {};
  }
  template <class CG> event submit(CG cg) {
    handler h;
    cg(h);
    return {};
  }
};

template <class T> T *malloc_device(size_t n, queue &) {
  return static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
}
inline void *malloc_device(size_t bytes, queue &) { return std::calloc(bytes ? bytes : 1, 1); }
inline void free(void *p, queue &) { std::free(p); }

}  // namespace sycl
