// Test infrastructure only (oracle build). Host stand-in for the few dpct
// helpers the reference's Lyapunov path calls: a default queue, device
// selection (a no-op: one host "device"), queues_wait_and_throw (a no-op: the
// shim's submit is synchronous) and global_memory<T,0>, which here just holds
// a host value (the model registrars copy device function pointers out of it).
#pragma once
#include <CL/sycl.hpp>

namespace dpct {

inline sycl::queue &get_default_queue() {
  static sycl::queue q;
  return q;
}

struct device_ext {
  void queues_wait_and_throw() {}
};
inline device_ext &get_current_device() {
  static device_ext d;
  return d;
}

struct dev_mgr {
  static dev_mgr &instance() {
    static dev_mgr m;
    return m;
  }
  void select_device(unsigned) {}
};

template <class T, int Dim> struct global_memory {
  T value;
  explicit global_memory(T v) : value(v) {}
  T *get_ptr() { return &value; }
};

}  // namespace dpct
