// vb_noalloc.cu -- vb_hllc_faces_noalloc: the batched HLLC face fluxes
// without any device allocation.
//
// Who needs it: callers that own all of the GPU's memory themselves -- a
// runtime whose pool allocator must not see foreign cudaMalloc/cudaFree calls
// (cudaFree synchronises the whole device and both calls fragment the pool),
// or a host that reserved the device memory up front.  vb_hllc_faces stages
// its host arrays in a context-owned device buffer that it grows with
// cudaMalloc; this entry point stages them in a fixed array compiled into the
// library instead.
//
// The array is a file-scope __device__ object of VB_NOALLOC_MAX_FACES faces
// (about 7.75 MiB): every GPU that loads the library holds it until the process
// exits.  All calls share it and it keeps the last call's contents; nothing
// here needs it zeroed (each call overwrites every value it reads).  Calls
// whose work overlaps on the GPU (several host threads, or several streams at
// once) race on the array and must be serialised by the caller.
//
// In host code the array's name is only a host-side stand-in, not a device
// address, so the device address is looked up with cudaGetSymbolAddress, with
// the device current, on the first call made on that device.  The address
// belongs to the device's current CUDA context (the module holding the array
// is loaded per context), so it is cached together with that context's
// process-unique id (cuCtxGetId) and looked up again when a call finds a
// different context current: after cudaDeviceReset, or under a caller's own
// context.  That first call on a device (or in a new context) should come
// before any stream capture.
#include <mutex>
#include <string>

#include "../../include/vespa_b200.h"
#include "vb_launch.h"

namespace {

constexpr size_t kFaceBytes = 5 * sizeof(double);
constexpr size_t kStateBytes = (size_t)VB_NOALLOC_MAX_FACES * kFaceBytes;  // one of WL/WR/F
constexpr size_t kAxisBytes = (size_t)VB_NOALLOC_MAX_FACES * sizeof(int32_t);
constexpr size_t kScratchBytes = 3 * kStateBytes + kAxisBytes;

// layout: WL | WR | F | axis
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
// per device: the array's address and the id of the context it belongs to
// (ctx_id 0 = not looked up yet)
struct ScratchSlot {
    void *addr = nullptr;
    unsigned long long ctx_id = 0;
};
ScratchSlot g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry-point
// lookup (the library does not link libcuda directly)
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);

// id of the calling thread's current context; false when none is current
bool current_context_id(unsigned long long *id)
{
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess && a &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess && b) {
            get_current = (PfnCtxGetCurrent)a;
            get_id = (PfnCtxGetId)b;
        }
    });
    if (!get_current || !get_id) return false;
    CUcontext c = nullptr;
    return get_current(&c) == CUDA_SUCCESS && c && get_id(c, id) == CUDA_SUCCESS && *id != 0;
}

int fail(int code, const std::string &msg)
{
    vb::set_last_error(msg.c_str());
    return code;
}

}  // namespace

extern "C" int vb_hllc_faces_noalloc(int64_t nf, const double *WL, const double *WR,
                                     const int32_t *axis, double gamma, double *F, void *stream)
{
    if (nf < 0) return fail(VB_EINVAL, "nf < 0");
    if (nf > VB_NOALLOC_MAX_FACES)
        return fail(VB_EINVAL, "nf = " + std::to_string(nf) +
                                   " exceeds VB_NOALLOC_MAX_FACES = " +
                                   std::to_string(VB_NOALLOC_MAX_FACES) +
                                   "; split the batch or use vb_hllc_faces");
    if (nf == 0) return VB_OK;
    if (!WL || !WR || !axis || !F) return fail(VB_EINVAL, "null buffer");
    if (!(gamma > 1.0)) return fail(VB_EINVAL, "gamma must exceed 1");
    for (int64_t f = 0; f < nf; ++f)
        if (axis[f] < 1 || axis[f] > 3) return fail(VB_EINVAL, "axis entries must be 1, 2 or 3");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(VB_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(VB_ENOTSUP, "device ordinal above 63");
    // once per device and context, with that device current: the array's
    // device address.  With no context current yet on this thread, the lookup
    // itself binds the device's primary context.
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        ScratchSlot &slot = g_scratch[dev];
        unsigned long long ctx_id = 0;
        if (current_context_id(&ctx_id) && slot.addr && slot.ctx_id == ctx_id) {
            base = slot.addr;
        } else {
            e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
            if (e != cudaSuccess || !base)
                return fail(VB_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            if (!current_context_id(&ctx_id))
                return fail(VB_ECUDA, "cuCtxGetCurrent/cuCtxGetId: no current context");
            slot.addr = base;
            slot.ctx_id = ctx_id;
        }
    }

    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *p = (unsigned char *)base;
    double *dWL = (double *)p;
    double *dWR = (double *)(p + kStateBytes);
    double *dF = (double *)(p + 2 * kStateBytes);
    int32_t *dax = (int32_t *)(p + 3 * kStateBytes);
    const size_t bw = (size_t)nf * kFaceBytes, ba = (size_t)nf * sizeof(int32_t);
    if ((e = cudaMemcpyAsync(dWL, WL, bw, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dWR, WR, bw, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dax, axis, ba, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return fail(VB_ECUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    if (vb::launch_hllc_faces(nf, dWL, dWR, dax, gamma, dF, s) < 0)
        return fail(VB_EINVAL, "invalid launch configuration");
    if ((e = cudaGetLastError()) != cudaSuccess)
        return fail(VB_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(F, dF, bw, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(VB_ECUDA, std::string("copy back: ") + cudaGetErrorString(e));
    return VB_OK;
}
