// jw_noalloc.cu -- jw_average_and_symmetrize_noalloc: the correlator
// symmetrisation for callers that cannot allocate device memory.
//
// jw_average_and_symmetrize needs a jw_context, whose creation allocates (a
// stream, twiddle tables and the scratch plane the symmetrisation works
// through).  Some callers cannot do that: a program whose device memory is
// all handed to its own pool allocator (a framework's caching allocator, for
// example) and that must not allocate behind the pool's back, or a
// time-critical loop that cannot afford cudaMalloc/cudaFree, which can
// synchronise the whole device.  This entry point works on a correlator the
// caller already holds in device memory and takes its scratch plane from a
// fixed array compiled into the library instead of allocating one.
//
// The array holds JW_NOALLOC_MAX_N^2 complex doubles (512^2 x 16 B = 4 MiB).
// It lives in every GPU that loads the library, for as long as the process
// runs.  Every call shares it, and it keeps the previous call's contents; each
// call writes the whole part it reads before reading it, so nothing needs
// clearing between calls.  Calls that overlap on the GPU (on different
// streams, or from different host threads) race on the array and must be
// ordered by the caller.
//
// CUDA loads this file's device code lazily (the default module loading of
// CUDA 12): the array is reserved on a device when the first call there
// loads the code.  A caller whose pool allocator takes the device's free
// memory makes one set-up call, jw_average_and_symmetrize_noalloc(NULL, 0,
// NULL), with the device current, before the pool does; it loads the code,
// reserves the array and looks up its address, and launches nothing.
#include <cstdint>
#include <mutex>

#include "jw_internal.h"

#define JW_NOALLOC_MAX_N 512

namespace {

static __device__ __align__(256) double2 g_symmetrize_scratch[JW_NOALLOC_MAX_N * JW_NOALLOC_MAX_N];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
// Per device: the array's device address and the CUDA context it belongs to.
// A context that was destroyed and made again (cudaDeviceReset) loads the
// module anew, possibly at another address, so the address is looked up
// again whenever the current context's id differs from the one recorded.
double2* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

// The unique id of the calling thread's current context (cuCtxGetId, CUDA
// 12.0 and later), through the runtime's driver entry points so that the
// library needs no link against libcuda.  0 when unavailable.
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess && qb == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(a);
            get_id = reinterpret_cast<CtxGetIdFn>(b);
        }
        resolved = true;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// The device address of g_symmetrize_scratch on the current device, looked
// up with that device current (host code cannot use the array's name as a
// device address): once per device and context.
jw_status scratch_for_current_device(double2** out) {
    int dev = -1;
    JW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return JW_EINVAL;
    // 0 when this thread has no current context yet: the lookup below makes
    // the device's primary context current, and its id is recorded after it
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void* p = nullptr;
        JW_CUDA(cudaGetSymbolAddress(&p, g_symmetrize_scratch));
        g_scratch_addr[dev] = static_cast<double2*>(p);
        g_scratch_ctx[dev] = current_context_id();
    }
    *out = g_scratch_addr[dev];
    return JW_OK;
}

// gfield::average_and_symmetrize (field.h:1460-1492) in two phases through
// the scratch plane: tmp = (C + C^T)/2, then C = average of tmp over (+-kx, +-ky).
__global__ void k_noalloc_sym_xy(const double2* __restrict__ c, double2* __restrict__ tmp, int N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)N * N) return;
    const int x = (int)(i / N), y = (int)(i % N);
    const double2 a = c[i], b = c[(long)y * N + x];
    tmp[i] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
}

__global__ void k_noalloc_sym_pm(double2* __restrict__ c, const double2* __restrict__ tmp, int N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)N * N) return;
    const int x = (int)(i / N), y = (int)(i % N);
    const int a = (N - x) % N, b = (N - y) % N;
    const double2 s0 = tmp[(long)x * N + y], s1 = tmp[(long)a * N + y], s2 = tmp[(long)x * N + b],
                  s3 = tmp[(long)a * N + b];
    c[i] = make_double2(0.25 * (((s0.x + s1.x) + s2.x) + s3.x), 0.25 * (((s0.y + s1.y) + s2.y) + s3.y));
}

}  // namespace

JW_EXPORT jw_status jw_average_and_symmetrize_noalloc(double* corr, int N, void* stream) {
    if (!corr && N == 0) {  // set-up only: load the code, reserve the array, look up its address
        double2* tmp = nullptr;
        return scratch_for_current_device(&tmp);
    }
    if (!corr || N < 1) return JW_EINVAL;
    if (reinterpret_cast<uintptr_t>(corr) % alignof(double2) != 0) {
        fprintf(stderr, "libjimwlk: jw_average_and_symmetrize_noalloc: corr must be 16-byte aligned\n");
        return JW_EINVAL;
    }
    if (N > JW_NOALLOC_MAX_N) {
        fprintf(stderr, "libjimwlk: jw_average_and_symmetrize_noalloc: N = %d exceeds the built-in scratch "
                        "(N <= %d); use jw_average_and_symmetrize\n", N, JW_NOALLOC_MAX_N);
        return JW_EINVAL;
    }
    double2* tmp = nullptr;
    jw_status s = scratch_for_current_device(&tmp);
    if (s) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long n2 = (long)N * N;
    const unsigned blocks = (unsigned)((n2 + 255) / 256);
    double2* c = reinterpret_cast<double2*>(corr);
    k_noalloc_sym_xy<<<blocks, 256, 0, st>>>(c, tmp, N);
    k_noalloc_sym_pm<<<blocks, 256, 0, st>>>(c, tmp, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}
