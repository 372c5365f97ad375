// static_trace.cu -- pt_trace_closest_static: closest hits of host rays
// without any allocation (an added entry point; the reference has none).
//
// Some callers cannot allocate device memory: a host that has handed the
// whole device to its own pool allocator, or code that runs where a
// cudaMalloc would synchronise the device or is forbidden outright.  For
// them, rays and hits travel through one file-scope device array of fixed
// size, kStaticTraceMaxRays rays (2 MiB of rays, 1 MiB of hits), which every
// GPU that loads the library holds until the process exits.
//
// Set-up, once per device (on the first call there, with that device
// current): the array's device address is looked up with
// cudaGetSymbolAddress (the host-side name of a __device__ variable is not a
// device address) and the SM count is read; both are cached.  After that a
// call is: copy the rays in, clear the error word, one launch of the
// warp-scheduled closest-hit loop the wavefront uses, copy the hits and the
// error word out -- all on the per-thread default stream, waited for with a
// stream synchronisation (other streams of the process are not waited on).
// No cudaMalloc, cudaFree or allocating library call is made.
//
// Calls on one device share the array, which keeps the previous call's
// contents (the error word is cleared on every call; hits are written for
// every ray of the call), so calls whose GPU work overlaps would race: a
// mutex serialises the calls made through this library.  The first call on
// a device may load the module: make it before any stream capture on that
// device.  The cached addresses are only valid for the device contexts that
// were current at set-up: resetting a device (cudaDeviceReset) between calls
// is not supported.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <mutex>
#include <string>

#include "device_api.h"
#include "traverse.h"

namespace ptb {

constexpr uint32_t kStaticTraceMaxRays = 1u << 16;
static_assert(kStaticTraceMaxRays == PT_STATIC_TRACE_MAX_RAYS, "limit declared in include/pt_b200.h");
constexpr int kStaticTraceMaxDevices = 64;

struct StaticTraceScratch {
    float4   rays[2 * kStaticTraceMaxRays];   // per ray: origin (w unused), direction (w unused)
    pt_hit   hits[kStaticTraceMaxRays];
    uint32_t err;                             // traversal error bits, cleared before every launch
};

static __device__ __align__(256) StaticTraceScratch g_static_trace;

namespace {

std::mutex g_static_mu;
StaticTraceScratch* g_static_addr[kStaticTraceMaxDevices] = {};
int g_static_sms[kStaticTraceMaxDevices] = {};

__global__ void __launch_bounds__(128) k_trace_closest_static(DeviceScene s, StaticTraceScratch* sc, uint32_t n,
                                                              int watertight) {
    uint32_t err = 0;
    TraceCounters tc{0, 0};
    closest_loop(s, blockIdx.x * blockDim.x + threadIdx.x, n, gridDim.x * blockDim.x, watertight != 0, err, tc,
                 [&](uint32_t i, RayInv& r) {
                     const float4 o = sc->rays[2 * i], d = sc->rays[2 * i + 1];
                     r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
                 },
                 [&](uint32_t i, const ClosestWalk& w) {
                     pt_hit h;
                     h.prim = w.prim;
                     h.t = w.prim >= 0 ? w.best : FLT_MAX;
                     h.u = w.prim >= 0 ? w.bu : 0.0f;
                     h.v = w.prim >= 0 ? w.bv : 0.0f;
                     sc->hits[i] = h;
                 });
    if (err) atomicOr(&sc->err, err);
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string("trace (static scratch): ") + what + ": " + cudaGetErrorString(e));
    return PT_ERR_CUDA;
}

}  // namespace

int trace_closest_static(pt_scene* s, const float* rays, uint32_t n, pt_hit* hits) {
    if (!s->dev.uploaded) { set_error("scene not uploaded"); return PT_ERR_STATE; }
    if (n > kStaticTraceMaxRays) {
        set_error("at most " + std::to_string(kStaticTraceMaxRays) + " rays per call");
        return PT_ERR_INVALID;
    }
    const int dev = s->dev.device;
    if (dev < 0 || dev >= kStaticTraceMaxDevices) { set_error("device ordinal out of range"); return PT_ERR_INVALID; }
    if (n == 0) return PT_OK;
    std::lock_guard<std::mutex> lk(g_static_mu);
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_trace);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        if (!p) { set_error("trace (static scratch): null symbol address"); return PT_ERR_CUDA; }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "SM count");
        g_static_sms[dev] = sms > 0 ? sms : 1;
        g_static_addr[dev] = static_cast<StaticTraceScratch*>(p);
    }
    StaticTraceScratch* sc = g_static_addr[dev];
    const cudaStream_t st = cudaStreamPerThread;
    e = cudaMemcpyAsync(sc->rays, rays, static_cast<size_t>(n) * 2 * sizeof(float4), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "ray upload");
    e = cudaMemsetAsync(&sc->err, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return cuda_fail(e, "clear");
    const DeviceScene v = device_view(s);
    const int wt = (s->host.settings.flags & PT_FLAG_WATERTIGHT) ? 1 : 0;
    // 16 resident blocks of 128 threads per SM; the loop strides over the rays
    const uint32_t max_blocks = static_cast<uint32_t>(g_static_sms[dev]) * 16u;
    const int blocks = static_cast<int>(std::min<uint32_t>((n + 127) / 128, max_blocks));
    k_trace_closest_static<<<blocks, 128, 0, st>>>(v, sc, n, wt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "launch");
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, &sc->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hits, sc->hits, static_cast<size_t>(n) * sizeof(pt_hit), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_fail(e, "download");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "kernel");
    if (err) { set_error("traversal stack overflow"); return PT_ERR_DEVICE; }
    return PT_OK;
}

}  // namespace ptb

extern "C" int pt_trace_closest_static(pt_scene* scene, const float* rays, uint32_t n, pt_hit* hits) {
    if (!scene || (n > 0 && (!rays || !hits))) { ptb::set_error("null argument"); return PT_ERR_INVALID; }
    return ptb::trace_closest_static(scene, rays, n, hits);
}
