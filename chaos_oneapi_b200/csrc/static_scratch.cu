// A mixed-batch entry point that allocates no device memory.
//
// Who needs it: code that must not call cudaMalloc / cudaFree while it runs --
// for example a host application that has handed all device memory to its own
// pool allocator, a real-time loop where an allocation (and the device-wide
// synchronisation that cudaFree implies) would stall other work, or a plugin
// host that does not let its plugins own device memory.  Such a caller cannot
// create a chaos_lyap_handle, because creating one allocates the handle's
// point counters, stream and staging buffers.
//
// What it uses instead: the batch kernel's only scratch is one 64-bit point
// counter per segment.  Here those counters live in a file-scope
// `static __device__` array of kStaticMaxSegments entries, which every GPU
// that loads this library holds from module load until the process exits.
// In host code the array's name only stands in for the device object, so its
// device address is looked up once per device with cudaGetSymbolAddress
// (with that device current) and passed to the kernel.
//
// Limits and rules:
//   * at most kStaticMaxSegments (8) segments per call; more is rejected;
//   * every call uses the same counters: calls on the same device must not
//     overlap on the GPU (issue them on one stream, or synchronise between);
//   * the counters keep the previous call's values; each call zeroes the ones
//     it uses (cudaMemsetAsync on the caller's stream) before its launch;
//   * the first call on a device performs the address lookup above; make that
//     first call before any stream capture begins;
//   * the address is remembered for the life of the process: the entry point
//     does not survive a reset of the device (cudaDeviceReset, or anything
//     else that destroys and recreates its primary context).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/chaos_lyap.h"
#include "kernels.h"

namespace chaos {
// Descriptor validation shared with the handle path (capi.cu).
int validate_desc(const chaos_lyap_desc *d, char *msg, size_t len);
}  // namespace chaos

namespace {

constexpr int kStaticMaxSegments = chaos::kMaxSegments;  // 8 counters, 64 bytes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_batch_counters[kStaticMaxSegments];

std::mutex g_setup_mutex;
unsigned long long *g_counter_ptr[kMaxDevices] = {};

thread_local char g_msg[256];

int failmsg(int code, const char *msg) {
  std::snprintf(g_msg, sizeof g_msg, "%s", msg);
  return code;
}

// Device address of the counters on `device`, which must be current; looked
// up on the first call for that device and remembered.
int counters_for(int device, unsigned long long **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_counter_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_batch_counters);
    if (e != cudaSuccess || !p) {
      std::snprintf(g_msg, sizeof g_msg, "cudaGetSymbolAddress(batch counters): %s",
                    cudaGetErrorString(e));
      return CHAOS_LYAP_ECUDA;
    }
    g_counter_ptr[device] = static_cast<unsigned long long *>(p);
  }
  *out = g_counter_ptr[device];
  return CHAOS_LYAP_OK;
}

}  // namespace

extern "C" const char *chaos_lyap_static_last_error(void) { return g_msg; }

extern "C" int chaos_lyap_run_batch_static(const chaos_lyap_desc *descs,
                                           const chaos_lyap_segment *segs, int nseg,
                                           void *stream) {
  g_msg[0] = 0;
  if (!descs || !segs) return failmsg(CHAOS_LYAP_EINVAL, "descs and segs must not be null");
  if (nseg < 1 || nseg > kStaticMaxSegments)
    return failmsg(CHAOS_LYAP_EINVAL,
                   "chaos_lyap_run_batch_static takes 1..8 segments: its point counters are a "
                   "fixed 8-entry device array");
  chaos::BatchArgs b;
  std::memset(&b, 0, sizeof b);
  b.nseg = nseg;
  const chaos_lyap_desc &d0 = descs[0];
  for (int i = 0; i < nseg; i++) {
    if (descs[i].struct_size != (int32_t)sizeof(chaos_lyap_desc))
      return failmsg(CHAOS_LYAP_EINVAL, "descriptor struct_size mismatch");
    chaos_lyap_desc d = descs[i];
    char name[33];
    std::memcpy(name, d.model, 32);
    name[32] = 0;
    int dim = 0, np = 0;
    const int id = chaos::model_id_of(name, &dim, &np);
    if (id < 0) return failmsg(CHAOS_LYAP_ENOMODEL, "unknown model in a segment descriptor");
    if (d.k == 0) d.k = dim;
    // the handle path's checks first (maps, tolerances, times, h, layout ...)
    const int vrc = chaos::validate_desc(&d, g_msg, sizeof g_msg);
    if (vrc) return vrc;
    const int k = d.k;
    if (d.precision == CHAOS_PREC_COMPAT_FP64)
      return failmsg(CHAOS_LYAP_EUNSUPPORTED, "segments take the adaptive forms (FP64 or FP32)");
    if (dim < 3 || dim > 4 || k != dim)
      return failmsg(CHAOS_LYAP_EUNSUPPORTED, "segments take 3-4 dimensional models, k == dim");
    if (d.precision != d0.precision || d.integrator != d0.integrator || d.device != d0.device)
      return failmsg(CHAOS_LYAP_EINVAL, "segments differ in integrator, precision or device");
    const chaos_lyap_segment &sg = segs[i];
    if (sg.P < 0 || (sg.P > 0 && (!sg.params || !sg.inits || !sg.spectrum)))
      return failmsg(CHAOS_LYAP_EINVAL, "bad segment arrays");
    chaos::AdaptiveArgs &a = b.seg[i];
    const bool soa = d.layout == CHAOS_LAYOUT_COMP_MAJOR;
    a.P = sg.P;
    a.k = k;
    a.gs = d.gs;
    a.rtol = d.rtol;
    a.atol = d.atol;
    a.h0 = d.h;
    a.hmax = d.h_max;
    a.hmin = d.h_min;
    a.t_transient = d.t_transient;
    a.t_align = d.t_align;
    a.t_avg = d.t_avg;
    a.dt_renorm = d.dt_renorm;
    a.max_steps = d.max_steps;
    a.escape = d.escape > 0 ? d.escape : 1e4;
    a.params = soa ? chaos::CView{sg.params, 1, sg.P} : chaos::CView{sg.params, np, 1};
    a.inits = soa ? chaos::CView{sg.inits, 1, sg.P} : chaos::CView{sg.inits, dim, 1};
    a.spectrum = soa ? chaos::View{sg.spectrum, 1, sg.P} : chaos::View{sg.spectrum, k, 1};
    a.t_avg_per_point = sg.t_avg_per_point;
    a.status = sg.status;
    a.steps = sg.steps;
    a.queue_stride = chaos::queue_stride_for(sg.P);
    b.model[i] = id;
  }
  if (d0.device < 0 || d0.device >= kMaxDevices)
    return failmsg(CHAOS_LYAP_EINVAL, "device ordinal out of range");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != d0.device && cudaSetDevice(d0.device) != cudaSuccess)
    return failmsg(CHAOS_LYAP_ECUDA, "cannot select the descriptors' device");
  unsigned long long *counters = nullptr;
  int rc = counters_for(d0.device, &counters);
  if (!rc) {
    b.queues = counters;
    cudaStream_t s = (cudaStream_t)stream;
    const cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned long long) * nseg, s);
    if (e != cudaSuccess) {
      std::snprintf(g_msg, sizeof g_msg, "cudaMemsetAsync(counters): %s", cudaGetErrorString(e));
      rc = CHAOS_LYAP_ECUDA;
    } else {
      const int integ = d0.integrator == CHAOS_INTEG_DOPRI5 ? chaos::kDopri5 : chaos::kDverk65;
      const int prec = d0.precision == CHAOS_PREC_FP32 ? chaos::kFP32 : chaos::kFP64;
      const int block = d0.block > 0 ? d0.block : 128;
      const int lr = chaos::launch_batch(integ, prec, b, block, s);
      if (lr == chaos::kErrUnsupported) {
        rc = failmsg(CHAOS_LYAP_EUNSUPPORTED, "no batch kernel for this combination");
      } else if (lr) {
        std::snprintf(g_msg, sizeof g_msg, "batch launch: %s",
                      cudaGetErrorString((cudaError_t)lr));
        rc = CHAOS_LYAP_ECUDA;
      }
    }
  }
  if (prev >= 0 && prev != d0.device) cudaSetDevice(prev);
  return rc;
}
