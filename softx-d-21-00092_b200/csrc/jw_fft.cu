// jw_fft.cu -- batched 2-D FFT over contiguous N x N complex planes: a row
// pass (contiguous, several rows per CTA) and a column pass (a tile of C
// adjacent columns per CTA, coalesced row segments), both in place through
// shared memory with the Stockham core of jw_fft.cuh.  This is the transform
// behind jw_execute2D (fftw2D::execute2D, mpi_fftw_class.h:191-315) and the
// engine's measurement.
#include <cmath>

#include "jw_fft.cuh"
#include "jw_internal.h"

namespace jw {

bool supported_n(int N) { return N >= 8 && N <= 2048 && (N & (N - 1)) == 0; }

// The tables are copied on stream s (stream-ordered: a kernel queued on s
// after this call reads the finished tables; a synchronous cudaMemcpy from
// pageable memory may return before its DMA lands, unordered with a
// non-blocking stream).
cudaError_t twiddles_create(int N, Twiddles* tw, cudaStream_t s) {
    std::vector<double2> h64(N);
    std::vector<float2> h32(N);
    for (int m = 0; m < N; ++m) {
        const double a = 2.0 * M_PI * (double)m / (double)N;
        h64[m] = make_double2(std::cos(a), std::sin(a));
        h32[m] = make_float2((float)h64[m].x, (float)h64[m].y);
    }
    tw->N = N;
    cudaError_t e = cudaMalloc(&tw->d64, sizeof(double2) * N);
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&tw->d32, sizeof(float2) * N);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(tw->d64, h64.data(), sizeof(double2) * N, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(tw->d32, h32.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);  // the host tables go out of scope
}

void twiddles_destroy(Twiddles* tw) {
    if (tw->d64) cudaFree(tw->d64);
    if (tw->d32) cudaFree(tw->d32);
    tw->d64 = nullptr;
    tw->d32 = nullptr;
}

template <typename T> __host__ __device__ inline const C2<T>* tw_ptr(const Twiddles& t);
template <> __host__ __device__ inline const double2* tw_ptr<double>(const Twiddles& t) { return t.d64; }
template <> __host__ __device__ inline const float2* tw_ptr<float>(const Twiddles& t) { return t.d32; }

// rows per CTA so that a CTA has about 256 threads
template <int N> constexpr int rows_per_cta() { return (256 / (N / 8)) > 0 ? (256 / (N / 8)) : 1; }
// columns per tile: 128-byte row segments where the tile fits 1024 threads
template <typename T, int N> constexpr int cols_per_cta() {
    constexpr int want = 128 / (int)sizeof(C2<T>);
    constexpr int cap = 8192 / N;
    constexpr int c = want < cap ? want : cap;
    return c < N ? c : N;
}

template <typename T, int N, int ROWS>
__global__ void __launch_bounds__(ROWS * (N / 8)) k_fft_rows(C2<T>* __restrict__ data, int nrows, T sign,
                                                            const C2<T>* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2<T>* sm = reinterpret_cast<C2<T>*>(smem_raw);
    const int tid = threadIdx.x;
    const long row0 = (long)blockIdx.x * ROWS;
    const int nr = (int)min((long)ROWS, (long)nrows - row0);
    C2<T>* g = data + row0 * N;
    for (int i = tid; i < nr * N; i += blockDim.x) sm[pad(i)] = g[i];
    __syncthreads();
    const int r = tid / (N / 8), t = tid % (N / 8);
    fft_smem<T, N>(sm, RowIdx{r * N}, t, r < nr, sign, tw);
    for (int i = tid; i < nr * N; i += blockDim.x) g[i] = sm[pad(i)];
}

template <typename T, int N, int C>
__global__ void __launch_bounds__(C * (N / 8)) k_fft_cols(C2<T>* __restrict__ data, T sign,
                                                         const C2<T>* __restrict__ tw, T scale) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2<T>* sm = reinterpret_cast<C2<T>*>(smem_raw);
    const int tid = threadIdx.x;
    C2<T>* g = data + (size_t)blockIdx.y * N * N + (size_t)blockIdx.x * C;
    for (int i = tid; i < N * C; i += blockDim.x) sm[pad(i)] = g[(size_t)(i / C) * N + (i % C)];
    __syncthreads();
    fft_smem<T, N>(sm, ColIdx<C>{tid % C}, tid / C, true, sign, tw);
    for (int i = tid; i < N * C; i += blockDim.x) g[(size_t)(i / C) * N + (i % C)] = cscale(sm[pad(i)], scale);
}

template <typename T, int N>
static cudaError_t fft2d_n(C2<T>* planes, int nplanes, int dir, T scale, const Twiddles& tw, cudaStream_t s) {
    const T sign = dir ? (T)-1 : (T)1;
    constexpr int ROWS = rows_per_cta<N>();
    constexpr int C = cols_per_cta<T, N>();
    const size_t smr = sizeof(C2<T>) * padded_len(ROWS * N);
    const size_t smc = sizeof(C2<T>) * padded_len(N * C);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_fft_rows<T, N, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
        cudaFuncSetAttribute(k_fft_cols<T, N, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
        configured = true;
    }
    const long nrows = (long)nplanes * N;
    k_fft_rows<T, N, ROWS><<<(unsigned)((nrows + ROWS - 1) / ROWS), ROWS * (N / 8), smr, s>>>(planes, (int)nrows,
                                                                                             sign, tw_ptr<T>(tw));
    k_fft_cols<T, N, C><<<dim3(N / C, nplanes), C * (N / 8), smc, s>>>(planes, sign, tw_ptr<T>(tw), scale);
    return cudaGetLastError();
}

template <typename T>
cudaError_t fft2d_planes(C2<T>* planes, int nplanes, int N, int dir, T scale, const Twiddles& tw, cudaStream_t s) {
    switch (N) {
        case 8: return fft2d_n<T, 8>(planes, nplanes, dir, scale, tw, s);
        case 16: return fft2d_n<T, 16>(planes, nplanes, dir, scale, tw, s);
        case 32: return fft2d_n<T, 32>(planes, nplanes, dir, scale, tw, s);
        case 64: return fft2d_n<T, 64>(planes, nplanes, dir, scale, tw, s);
        case 128: return fft2d_n<T, 128>(planes, nplanes, dir, scale, tw, s);
        case 256: return fft2d_n<T, 256>(planes, nplanes, dir, scale, tw, s);
        case 512: return fft2d_n<T, 512>(planes, nplanes, dir, scale, tw, s);
        case 1024: return fft2d_n<T, 1024>(planes, nplanes, dir, scale, tw, s);
        case 2048: return fft2d_n<T, 2048>(planes, nplanes, dir, scale, tw, s);
        default: return cudaErrorInvalidValue;
    }
}

template cudaError_t fft2d_planes<double>(double2*, int, int, int, double, const Twiddles&, cudaStream_t);
template cudaError_t fft2d_planes<float>(float2*, int, int, int, float, const Twiddles&, cudaStream_t);

}  // namespace jw
