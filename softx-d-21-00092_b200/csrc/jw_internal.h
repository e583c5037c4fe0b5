// jw_internal.h -- host-side internals shared by the libjimwlk translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "../../include/jimwlk.h"
#include "jw_common.cuh"

#define JW_EXPORT extern "C" __attribute__((visibility("default")))


#define JW_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "libjimwlk: %s failed at %s:%d: %s\n", #call, __FILE__, __LINE__, \
                    cudaGetErrorString(e_));                                                  \
            return JW_ECUDA;                                                                  \
        }                                                                                     \
    } while (0)

#define JW_CHECK(cond)                 \
    do {                               \
        if (!(cond)) return JW_EINVAL; \
    } while (0)

namespace jw {

// FP64-accurate twiddle tables exp(+2 pi i m / N), m < N, for one N.
// For an N that is not a power of two in [8, 2048] the FP64 transform runs
// as Bluestein's chirp-z transform over a power-of-two length M >= 2N - 1,
// and the tables are those of the chirp-z form instead (d64 = d32 = null).
struct Twiddles {
    int N = 0;
    double2* d64 = nullptr;
    float2* d32 = nullptr;
    int M = 0;                    // chirp-z length (0: N is a power of two)
    double2* chirp = nullptr;     // w[n] = exp(-i pi n^2 / N), n < N
    double2* bhat = nullptr;      // [2][M]: DFT_M of the wrapped chirp kernel / M, forward then backward
    double2* twM = nullptr;       // exp(+2 pi i m / M), m < M
};
cudaError_t twiddles_create(int N, Twiddles* tw, cudaStream_t s);
void twiddles_destroy(Twiddles* tw);

// Power-of-two N in [8, 2048]: every layer (the engine's fused kernels included).
bool supported_n(int N);
// Any N in [2, 2048]: the call-for-call FP64 layer, whose transform falls back
// to the chirp-z form for N that supported_n rejects.
bool supported_n_fp64(int N);

// Converts a device error-flag word to a status (and clears nothing).
inline jw_status flags_to_status(int flags) {
    if (flags & JW_FLAG_NOCONV) return JW_ENOCONV;
    if (flags & JW_FLAG_NAN) return JW_ENAN;
    if (flags & JW_FLAG_TIMEOUT) return JW_ETIMEOUT;
    return JW_OK;
}

}  // namespace jw

struct jw_context {
    jw_config cfg;
    int device = 0;
    int N = 0;
    cudaStream_t stream = nullptr;
    jw::Twiddles tw;
    int* d_flags = nullptr;       // device error flags
    double2* d_tmp = nullptr;     // one plane of scratch (average_and_symmetrize)
    unsigned long long* d_step = nullptr;  // noise index of jw_evolve_momentum's replayed steps
    std::vector<jw_field*> fields;  // live fields, released by jw_context_destroy
    // position-space evolution (jw_position.cu), allocated on first use
    double2* d_pos_tab = nullptr;   // 2 planes: raw forward DFT of k_x(d), k_y(d)
    int pos_key[3] = {-1, -1, -1};  // (rr, coupling, kernel) of d_pos_tab
    double2* d_pos_scratch = nullptr;  // 18 planes
    std::vector<jw_cholesky*> choleskies;  // live factors, released by jw_context_destroy
    jw_field* pos_work[4] = {};     // xi_x, xi_y, A, B of jw_evolve_position (in `fields`)
    jw_field* mom_work[6] = {};     // xi_x, xi_y, A, B, ux, uy of jw_evolve_momentum (in `fields`)
    jw_field* mv_work = nullptr;    // the charge field of jw_initial_condition (in `fields`)
};

namespace jw {
// Frees what jw_position.cu attached to the context.
void position_release(jw_context* c);
// The position kernel k_x, k_y at distance (dxi, dyi) (positions.h:105-150,
// field.h:2402-2470), host FP64 with the reference's expressions.
void position_kernel_host(int dxi, int dyi, int N, int rr, int coupling, int kernel, double* kx, double* ky);
// S(x, y) = h[x N + y].x (a plane already transformed to position space) ->
// angular bins b = floor(|r| + 1/2) <= N/2 over minimum-image distances and
// Q_s = sqrt(2)/r_s at S(r_s) = exp(-1/2), linear between the bracketing bins
// (0 if none).  Every output pointer may be null.
void dipole_bins(const double2* h, int N, double* S_xy, double* S_bins, double* r_bins, int* counts, int* nbins,
                 double* Qs);
}

struct jw_field {
    jw_context* ctx = nullptr;
    int t = 0;                    // 1 or 9
    double2* d = nullptr;         // t planes of N*N, plane k at d + k*N*N (row-major x, y)
};

// FFT launchers over contiguous planes of N*N complex (rows then columns,
// in place, scaled by `scale` after the column pass).
namespace jw {
template <typename T>
cudaError_t fft2d_planes(C2<T>* planes, int nplanes, int N, int dir, T scale, const Twiddles& tw,
                         cudaStream_t s);
}
