// jxb_apply_static: the operator application of jxb_apply, with its brick
// partial sums kept in a fixed, file-scope device array instead of the
// plan's own scratch buffer.
//
// Who this is for: host code that must not allocate device memory at the
// point where it applies the operator -- for example a handler running
// inside a framework that owns all device allocations through its own pool,
// or a latency-critical loop where an allocation (and the implicit device
// synchronisation cudaMalloc/cudaFree can cause) is not acceptable. Such a
// caller still creates the plan beforehand and passes the input and output
// vectors; this entry point itself calls no allocating routine.
//
// The array is JXB_STATIC_SCRATCH_BYTES (16 MiB) of device memory on every
// GPU on which this library is loaded, held until the process exits. Plans
// whose brick scratch is larger are rejected with JXB_ERR_INVALID.
//
// Every call, on every stream, uses the same array. Nothing in it has to
// start at zero (each brick writes its whole footprint before the combine
// pass reads it), but two calls whose work overlaps on the GPU -- on
// different streams, or from different host threads -- race on it and give
// wrong results; order them on one stream or synchronise in between.
//
// The device address of the array is looked up with cudaGetSymbolAddress on
// the first call on each device, with that device current; that first call
// should therefore be made before any stream capture begins. The plan's
// device (the one current when the plan was created) must be current at
// every call; a call made with another device current is refused with
// JXB_ERR_INVALID instead of running the plan's buffers against that
// device's array.
#include <mutex>

#include "jxb_internal.cuh"

#define JXB_STATIC_SCRATCH_BYTES (16u << 20)
#define JXB_STATIC_MAX_DEVICES 64

static __device__ __align__(256) double g_apply_scratch[JXB_STATIC_SCRATCH_BYTES / sizeof(double)];

namespace {
double* g_scratch_addr[JXB_STATIC_MAX_DEVICES] = {};
std::mutex g_scratch_mutex;

// Device address of g_apply_scratch on the current device (looked up once).
int scratch_address(double** out) {
  int dev = 0;
  JXB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= JXB_STATIC_MAX_DEVICES)
    return jxb::fail(JXB_ERR_INVALID, "jxb_apply_static: device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_apply_scratch);
    if (e != cudaSuccess) return jxb::cuda_fail(e, "cudaGetSymbolAddress(g_apply_scratch)");
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return JXB_OK;
}
}  // namespace

extern "C" int jxb_apply_static(jxb_plan* plan, jxb_stream stream, const double* x, double* y, int masked) {
  if (plan && (plan->mp || plan->thb)) return jxb::fail(JXB_ERR_INVALID, "jxb_apply_static: not available on a multipatch or hierarchical plan");
  if (!plan || !x || !y) return jxb::fail(JXB_ERR_INVALID, "jxb_apply_static: null argument");
  const size_t need = plan->scratch_elems * sizeof(double);
  if (need > JXB_STATIC_SCRATCH_BYTES)
    return jxb::fail(JXB_ERR_INVALID,
                     "jxb_apply_static: this plan needs " + std::to_string(need) +
                         " bytes of brick scratch, more than the fixed " +
                         std::to_string((size_t)JXB_STATIC_SCRATCH_BYTES) + "-byte array; use jxb_apply");
  // The address below belongs to the current device; the plan's buffers to
  // the device that was current when it was created. Refuse a mismatch.
  int dev = 0;
  JXB_CUDA(cudaGetDevice(&dev));
  if (dev != plan->device)
    return jxb::fail(JXB_ERR_INVALID, "jxb_apply_static: the plan was created on device " +
                                          std::to_string(plan->device) + " but device " + std::to_string(dev) +
                                          " is current; make the plan's device current first");
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  // A shallow copy of the plan that points its scratch at the static array;
  // every other buffer is the plan's own, so nothing is allocated here.
  jxb_plan view = *plan;
  view.d_scratch = scratch;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  rc = jxb::launch_bricks<double>(&view, s, jxb::MODE_APPLY, x, nullptr, nullptr, masked);
  if (rc) return rc;
  return jxb::launch_combine<double>(&view, s, y, masked, nullptr, nullptr, nullptr);
}
