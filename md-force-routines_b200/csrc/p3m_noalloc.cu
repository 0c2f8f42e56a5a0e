// p3m_gf_opt_static: the FP64 optimal influence function for callers that
// cannot allocate device memory.
//
// p3m_gf_opt allocates its output and its per-block partial sums with
// cudaMalloc on every call. Some callers cannot do that: code that owns a
// fixed device-memory budget and hands out every byte itself through its own
// pool or arena (an allocation behind its back can push a full GPU over the
// edge), or long-running services that must not allocate after start-up
// (cudaMalloc can block on the device and fragments memory over time). This
// entry point takes
// the output buffers from the caller and keeps its only scratch -- one FP64
// partial sum per 256-point block -- in the file-scope array below, which
// every GPU that loads the library holds until the process exits
// (kMaxBlocks doubles, 64 KiB).
//
// The array is shared by all calls on a device and keeps the last call's
// contents. Nothing in it needs to start at zero: each call writes every
// slot it later reads. Two calls whose work overlaps on the GPU (on
// different streams, or from different host threads without ordering)
// race on it; callers must order such calls.
#include <cstdio>
#include <mutex>

#include "p3m_kernels.h"

namespace {

constexpr int kMaxMesh = 128;                                         // M <= 128
constexpr int kMaxBlocks = kMaxMesh * kMaxMesh * kMaxMesh / 256;      // 8192 partials
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_gf_scratch[kMaxBlocks];

std::mutex g_setup_mu;
double *g_scratch_addr[kMaxDevices] = {};

// Device address of g_gf_scratch on the current device. (In host code the
// array's name is only a host-side stand-in and must never be passed to a
// kernel.) The address is looked up again on every call made outside stream
// capture -- a cudaDeviceReset, or any teardown of the primary context,
// unloads the module and the array may come back elsewhere -- and the last
// address found is reused while `st` is capturing, when no CUDA call that
// could load a module may run.
cudaError_t scratch_address(int device, cudaStream_t st, double **out)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_gf_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = static_cast<double *>(p);
    } else if (!g_scratch_addr[device]) {
        return cudaErrorStreamCaptureUnsupported;  // first call on this device under capture
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

// A_pm = sum of the per-block partials in block order (the order p3m_gf_opt
// sums them on the host).
__global__ void k_sum_partials(const double *__restrict__ part, int n, double *__restrict__ out)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += part[i];
        *out = s;
    }
}

thread_local char g_msg[256];

int fail_static(int code, const char *msg, const char *detail = nullptr)
{
    snprintf(g_msg, sizeof g_msg, "p3m_gf_opt_static: %s%s%s", msg, detail ? ": " : "",
             detail ? detail : "");
    return code;
}

}  // namespace

extern "C" const char *p3m_gf_opt_static_error(void) { return g_msg; }

extern "C" int p3m_gf_opt_static(double kappa, double alpha, int p, int m_alias, int M,
                                 double box, double *G_k_dev, double *A_pm_dev, void *stream)
{
    g_msg[0] = 0;
    if (!G_k_dev || !A_pm_dev) return fail_static(P3M_EARG, "output pointers must be device memory");
    if (M < 2 || M > kMaxMesh)
        return fail_static(P3M_EARG, "M must be in [2, 128] (the static scratch holds 8192 "
                                     "block partials)");
    if (!(box > 0) || !(alpha > 0) || !(kappa >= 0) || p < 1 || m_alias < 0 || m_alias > 7)
        return fail_static(P3M_EARG, "bad parameter");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_static(P3M_ENODEV, "no current device", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail_static(P3M_ENODEV, "device index out of range");
    int major = 0;
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e != cudaSuccess || major != 10)
        return fail_static(P3M_ENODEV, "library is built for sm_100a (B200)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double *part = nullptr;
    e = scratch_address(dev, st, &part);
    if (e != cudaSuccess) return fail_static(P3M_ECUDA, "scratch address", cudaGetErrorString(e));
    p3m::launch_gf_opt(kappa, alpha, p, m_alias, M, box, G_k_dev, part, st);
    k_sum_partials<<<1, 32, 0, st>>>(part, p3m::gf_opt_blocks(M), A_pm_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_static(P3M_ECUDA, "kernel launch", cudaGetErrorString(e));
    return P3M_OK;
}
