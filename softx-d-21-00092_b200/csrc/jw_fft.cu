// jw_fft.cu -- batched 2-D FFT over contiguous N x N complex planes: a row
// pass (contiguous, several rows per CTA) and a column pass (a tile of C
// adjacent columns per CTA, coalesced row segments), both in place through
// shared memory with the Stockham core of jw_fft.cuh.  This is the transform
// behind jw_execute2D (fftw2D::execute2D, mpi_fftw_class.h:191-315) and the
// engine's measurement.
//
// The reference plans FFTW for any lattice size (mpi_fftw_class.h:165-186,
// Nx = Ny fixed at compile time, config.h:31-32).  For an N that is not a
// power of two the FP64 transform runs as Bluestein's chirp-z transform
// (L. Bluestein, "A linear filtering approach to the computation of the
// discrete Fourier transform", 1970): with w_n = exp(-i pi n^2 / N) and
// n k = (n^2 + k^2 - (k - n)^2) / 2,
//     X_k = w_k sum_n (x_n w_n) conj(w_(k-n))        (forward, sign -1)
// a linear convolution of length 2N - 1, done as a circular one of
// power-of-two length M >= 2N - 1 with the Stockham core: chirp, DFT_M,
// multiply by the tabulated DFT_M of the wrapped kernel, inverse DFT_M,
// chirp.  The backward transform conjugates w.  Each line is one shared-memory
// residency (rows: several per CTA; columns: a tile of adjacent columns), so a
// 2-D transform is still two HBM round trips.
#include <cmath>
#include <complex>
#include <type_traits>

#include "jw_fft.cuh"
#include "jw_internal.h"

namespace jw {

bool supported_n(int N) { return N >= 8 && N <= 2048 && (N & (N - 1)) == 0; }
bool supported_n_fp64(int N) { return N >= 2 && N <= 2048; }

// Smallest power of two M >= max(2N - 1, 8): the chirp-z convolution length.
static int chirp_len(int N) {
    int M = 8;
    while (M < 2 * N - 1) M <<= 1;
    return M;
}

// In-place radix-2 DFT of a power-of-two length on the host (FP64), sign -1
// forward: used once per context to tabulate the chirp-z kernel's spectrum.
static void host_fft_pow2(std::vector<std::complex<double>>& a, int sign) {
    const int n = (int)a.size();
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        for (int k = 0; k < len / 2; ++k) {
            const double ang = 2.0 * M_PI * (double)k / (double)len;
            const std::complex<double> w(std::cos(ang), sign * std::sin(ang));
            for (int s0 = 0; s0 < n; s0 += len) {
                const std::complex<double> u = a[s0 + k], v = a[s0 + k + len / 2] * w;
                a[s0 + k] = u + v;
                a[s0 + k + len / 2] = u - v;
            }
        }
    }
}

// The chirp-z tables of a non-power-of-two N (see the file header).
static cudaError_t chirp_tables_create(int N, Twiddles* tw, cudaStream_t s) {
    const int M = chirp_len(N);
    tw->N = N;
    tw->M = M;
    std::vector<double2> hw(N), htw(M), hb(2 * (size_t)M);
    std::vector<std::complex<double>> w(N);
    for (int n = 0; n < N; ++n) {
        // pi n^2 / N reduced exactly: n^2 mod 2N keeps the argument in [0, 2 pi)
        const long r = ((long)n * n) % (2L * N);
        const double a = M_PI * (double)r / (double)N;
        w[n] = std::complex<double>(std::cos(a), -std::sin(a));
        hw[n] = make_double2(w[n].real(), w[n].imag());
    }
    for (int m = 0; m < M; ++m) {
        const double a = 2.0 * M_PI * (double)m / (double)M;
        htw[m] = make_double2(std::cos(a), std::sin(a));
    }
    for (int dir = 0; dir < 2; ++dir) {
        // forward: b_m = conj(w_|m|); backward: b_m = w_|m|; |m| < N, wrapped mod M
        std::vector<std::complex<double>> b(M, std::complex<double>(0.0, 0.0));
        for (int n = 0; n < N; ++n) {
            const std::complex<double> v = dir == 0 ? std::conj(w[n]) : w[n];
            b[n] = v;
            if (n > 0) b[M - n] = v;
        }
        host_fft_pow2(b, -1);
        for (int m = 0; m < M; ++m) hb[(size_t)dir * M + m] = make_double2(b[m].real() / M, b[m].imag() / M);
    }
    cudaError_t e = cudaMalloc(&tw->chirp, sizeof(double2) * N);
    if (e == cudaSuccess) e = cudaMalloc(&tw->twM, sizeof(double2) * M);
    if (e == cudaSuccess) e = cudaMalloc(&tw->bhat, sizeof(double2) * 2 * (size_t)M);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tw->chirp, hw.data(), sizeof(double2) * N, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tw->twM, htw.data(), sizeof(double2) * M, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(tw->bhat, hb.data(), sizeof(double2) * 2 * (size_t)M, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);  // the host tables go out of scope
}

// The tables are copied on stream s (stream-ordered: a kernel queued on s
// after this call reads the finished tables; a synchronous cudaMemcpy from
// pageable memory may return before its DMA lands, unordered with a
// non-blocking stream).
cudaError_t twiddles_create(int N, Twiddles* tw, cudaStream_t s) {
    if (!supported_n(N)) {
        if (!supported_n_fp64(N)) return cudaErrorInvalidValue;
        return chirp_tables_create(N, tw, s);
    }
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
    if (tw->chirp) cudaFree(tw->chirp);
    if (tw->bhat) cudaFree(tw->bhat);
    if (tw->twM) cudaFree(tw->twM);
    tw->d64 = nullptr;
    tw->d32 = nullptr;
    tw->chirp = tw->bhat = tw->twM = nullptr;
    tw->M = 0;
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

// ---- chirp-z (Bluestein) transform for N that is not a power of two ----

// Chirp factor w_n (forward) or conj(w_n) (backward, sign > 0).
__device__ __forceinline__ double2 chirp_at(const double2* __restrict__ chirp, int n, double sign) {
    double2 w = __ldg(&chirp[n]);
    if (sign > 0.0) w.y = -w.y;
    return w;
}

// Rows: ROWS = 4096 / M rows of length N per CTA, each zero-padded to M
// (M / 8 threads per row).  Thread t of a row holds elements t + m M/8 (m < 8)
// in registers: they load from global memory times the chirp, the forward
// transform starts from and ends in registers (the 16-byte-element core's
// hand-off), the kernel spectrum multiplies in registers, and the inverse
// transform ends in registers that are stored times the chirp.  Shared memory
// carries only the passes in between.
template <int M>
__global__ void __launch_bounds__(512) k_chirp_rows(double2* __restrict__ data, long nrows, int N, double sign,
                                                    const double2* __restrict__ chirp,
                                                    const double2* __restrict__ bhat,
                                                    const double2* __restrict__ twM) {
    constexpr int ROWS = 4096 / M, TPS = M / 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int tid = threadIdx.x, r = tid / TPS, t = tid % TPS;
    const long row = (long)blockIdx.x * ROWS + r;
    const bool active = row < nrows;
    double2* g = data + row * N;
    double2 reg[1][8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int e = t + m * TPS;
        reg[0][m] = active && e < N ? cmul(g[e], chirp_at(chirp, e, sign)) : make_double2(0.0, 0.0);
    }
    const RowIdx16 idx{r * M};
    fft16x<double, M, true, true>(sm, idx, t, active, -1.0, twM, reg);
#pragma unroll
    for (int m = 0; m < 8; ++m) reg[0][m] = cmul(reg[0][m], __ldg(&bhat[t + m * TPS]));
    fft16x<double, M, true, true>(sm, idx, t, active, 1.0, twM, reg);
    if (active) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int e = t + m * TPS;
            if (e < N) g[e] = cmul(reg[0][m], chirp_at(chirp, e, sign));
        }
    }
}

// Columns: a tile of C adjacent columns of one plane (blockIdx.y), each
// zero-padded to M; the last tile of a row may be narrower.  Thread (c, t)
// holds elements t + m M/8 of column c in registers, as in the row kernel.
// Tiles narrower than 8 columns (rows under 128 bytes) are padded by one row
// every 8 rows in shared memory.
template <int M> constexpr int chirp_cols_per_cta() { return M >= 512 ? 4096 / M : 8; }
template <int C>
struct ChirpColIdx {
    int c;
    __device__ __forceinline__ int operator()(int e) const { return e * C + c + (C >= 8 ? 0 : (e >> 3) * C); }
};
template <int M, int C> constexpr int chirp_col_len() { return M * C + (C >= 8 ? 0 : (M / 8) * C); }

template <int M, int C>
__global__ void __launch_bounds__(C * (M / 8)) k_chirp_cols(double2* __restrict__ data, int N, double sign,
                                                            const double2* __restrict__ chirp,
                                                            const double2* __restrict__ bhat,
                                                            const double2* __restrict__ twM, double scale) {
    constexpr int TPS = M / 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int tid = threadIdx.x, cc = tid % C, t = tid / C;
    const int x0 = blockIdx.x * C;
    const bool active = cc < N - x0;
    double2* g = data + (size_t)blockIdx.y * N * N + x0 + cc;
    double2 reg[1][8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int e = t + m * TPS;
        reg[0][m] = active && e < N ? cmul(g[(size_t)e * N], chirp_at(chirp, e, sign)) : make_double2(0.0, 0.0);
    }
    const ChirpColIdx<C> idx{cc};
    fft16x<double, M, true, true>(sm, idx, t, active, -1.0, twM, reg);
#pragma unroll
    for (int m = 0; m < 8; ++m) reg[0][m] = cmul(reg[0][m], __ldg(&bhat[t + m * TPS]));
    fft16x<double, M, true, true>(sm, idx, t, active, 1.0, twM, reg);
    if (active) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int e = t + m * TPS;
            if (e < N) g[(size_t)e * N] = cscale(cmul(reg[0][m], chirp_at(chirp, e, sign)), scale);
        }
    }
}

template <int M>
static cudaError_t chirp2d_m(double2* planes, int nplanes, int dir, double scale, const Twiddles& tw,
                             cudaStream_t s) {
    const int N = tw.N;
    const double sign = dir ? -1.0 : 1.0;
    const double2* bhat = tw.bhat + (dir ? 0 : M);
    constexpr int ROWS = 4096 / M;
    constexpr int C = chirp_cols_per_cta<M>();
    const size_t smr = sizeof(double2) * padded_len16(ROWS * M);
    const size_t smc = sizeof(double2) * chirp_col_len<M, C>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_chirp_rows<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smr);
        cudaFuncSetAttribute(k_chirp_cols<M, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smc);
        configured = true;
    }
    const long nrows = (long)nplanes * N;
    k_chirp_rows<M><<<(unsigned)((nrows + ROWS - 1) / ROWS), ROWS * (M / 8), smr, s>>>(planes, nrows, N, sign,
                                                                                       tw.chirp, bhat, tw.twM);
    k_chirp_cols<M, C><<<dim3((N + C - 1) / C, nplanes), C * (M / 8), smc, s>>>(planes, N, sign, tw.chirp, bhat,
                                                                               tw.twM, scale);
    return cudaGetLastError();
}

static cudaError_t chirp2d_planes(double2* planes, int nplanes, int dir, double scale, const Twiddles& tw,
                                  cudaStream_t s) {
    switch (tw.M) {
        case 8: return chirp2d_m<8>(planes, nplanes, dir, scale, tw, s);
        case 16: return chirp2d_m<16>(planes, nplanes, dir, scale, tw, s);
        case 32: return chirp2d_m<32>(planes, nplanes, dir, scale, tw, s);
        case 64: return chirp2d_m<64>(planes, nplanes, dir, scale, tw, s);
        case 128: return chirp2d_m<128>(planes, nplanes, dir, scale, tw, s);
        case 256: return chirp2d_m<256>(planes, nplanes, dir, scale, tw, s);
        case 512: return chirp2d_m<512>(planes, nplanes, dir, scale, tw, s);
        case 1024: return chirp2d_m<1024>(planes, nplanes, dir, scale, tw, s);
        case 2048: return chirp2d_m<2048>(planes, nplanes, dir, scale, tw, s);
        case 4096: return chirp2d_m<4096>(planes, nplanes, dir, scale, tw, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t fft2d_planes(C2<T>* planes, int nplanes, int N, int dir, T scale, const Twiddles& tw, cudaStream_t s) {
    if constexpr (std::is_same<T, double>::value) {
        if (tw.M != 0) {
            if (tw.N != N) return cudaErrorInvalidValue;
            return chirp2d_planes(planes, nplanes, dir, scale, tw, s);
        }
    }
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
