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
#include <mutex>

#include "jw_internal.h"

#define JW_NOALLOC_MAX_N 512

namespace {

static __device__ __align__(256) double2 g_symmetrize_scratch[JW_NOALLOC_MAX_N * JW_NOALLOC_MAX_N];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double2* g_scratch_addr[kMaxDevices] = {};

// The device address of g_symmetrize_scratch on the current device, looked
// up once per device with that device current (host code cannot use the
// array's name as a device address).
jw_status scratch_for_current_device(double2** out) {
    int dev = -1;
    JW_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return JW_EINVAL;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        JW_CUDA(cudaGetSymbolAddress(&p, g_symmetrize_scratch));
        g_scratch_addr[dev] = static_cast<double2*>(p);
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
    if (!corr || N < 1) return JW_EINVAL;
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
