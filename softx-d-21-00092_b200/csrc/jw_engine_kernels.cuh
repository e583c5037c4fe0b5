// jw_engine_kernels.cuh -- the fused kernels of the batched engine.
//
// One Langevin step (main_optimized.cpp:243-304) of every event in a batch is
// three launches over the events' planes:
//
//  pass 1 (row)    per row x: 16 Philox normals per site (field.h:2116-2243 /
//                  2245-2365), V xi V^dagger (field.h:1892-1933) projected on
//                  the 8 Gell-Mann coefficients, packed as 16 complex sequences
//                     s = 0..3   n_{2s} + i n_{2s+1}       (xi_x)
//                     s = 4..7   m_{2s'} + i m_{2s'+1}     (xi_y)
//                     s = 8..11  bx_{2s'} + i bx_{2s'+1}   (V xi_x V^dagger)
//                     s = 12..15 by_{2s'} + i by_{2s'+1}   (V xi_y V^dagger)
//                  and row-transformed (forward) into P[16][N][N].
//  pass 2 (column) per output plane j and column tile: column transform of the
//                  x- and y-packs, W = K_x Zx + K_y Zy (prepare_A_local,
//                  field.h:1998-2075, with the 1/N^2 of the two unitary
//                  transforms folded into K), inverse column transform into
//                  Q[8][N][N]: j = 0..3 give A, 4..7 give B.
//  pass 3 (row)    inverse row transform of Q's row x, which yields
//                  A_{2s} + i A_{2s+1} (the kernel is Hermitian-symmetric for
//                  the SIN kernel, so both coefficients are real), then per
//                  site the FP64 update V <- exp(+i sqrt(eps) B) V exp(-i sqrt(eps) A)
//                  (update_uf, field.h:1966-1996) through the eigen-route
//                  exponential, optional reunitarisation, and the event's step
//                  counter advances.
//
// Because x_a -> sum_a x_a L_a is linear and the transforms are linear,
// transforming the 8 real coefficients instead of the 9 complex matrix
// entries gives the reference's A and B up to rounding; the 72 plane
// transforms of a reference step become 24 (16 forward, 8 inverse).
//
// The MV initial condition (main_optimized.cpp:178-191) uses the same three
// passes with 4 planes per slice and the Poisson kernel, in FP64.  The dipole
// measurement (main_optimized.cpp:321-334) transforms V's 9 planes in FP64 and
// accumulates |V~|^2 per momentum in the column pass.
#pragma once

#include "jw_fft.cuh"

namespace jw {

struct EventDev {
    double2* V;                 // 9 planes of N*N
    double* acc;                // 4 planes of N*N: sum, sum compensation, err, err compensation
    const double* k64;          // kernel tables: [2][N*N] imag(K_x), imag(K_y), scaled by 1/N^2
    const float* k32;
    const double* kre64;        // real parts of the tables, same layout (a position-space kernel whose
    const float* kre32;         //   DFT has one: LINEAR), or null
    const double* nf64;         // per-site noise factor (NOISE coupling) or null
    const float* nf32;
    unsigned long long seed;
    unsigned long long step;    // next Langevin step index (advanced by pass 2 in mixed precision, pass 3 in FP64)
    double sqrt_eps;            // sqrt(step)
    double mv_sigma;            // g mu / sqrt(ny_slices)
    double mv_mass2;            // (mass * g^2 * mu)^2
    double mv_g;
    int N;
    int reunit;
    int nmeas;
    int pad_;
};

template <int N> constexpr int row_threads() { return (N / 8) > 256 ? (N / 8) : 256; }
// V is staged through shared memory in chunks of at most 512 sites (72 KB)
template <int N> constexpr int v_chunk() { return N < 512 ? N : 512; }
// column tile width: 64-byte row segments, capped so the tile holds <= 64 KB
template <typename T, int N> constexpr int p2_cols() {
    constexpr int want = 64 / (int)sizeof(C2<T>);
    constexpr int cap = 65536 / (N * (int)sizeof(C2<T>));
    constexpr int c = want < cap ? want : (cap > 0 ? cap : 1);
    return c < N ? c : N;
}
template <typename T, int N> constexpr size_t p2_smem() {
    return sizeof(C2<T>) * 2 * padded_len(N * p2_cols<T, N>()) + sizeof(T) * 2 * N * p2_cols<T, N>();
}
template <typename T, int N> constexpr size_t p3_smem() {
    return sizeof(C2<T>) * padded_len(8 * N) + sizeof(double2) * 9 * v_chunk<N>();
}

// ---- asynchronous global -> shared copies (cp.async, sm_80+)
template <int B>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

// V sites [c0, c0 + VC) of row x into smV[k][VC] (16-byte copies)
template <int N>
__device__ __forceinline__ void stage_v(double2* smV, const double2* __restrict__ V, long vol, int x, int c0) {
    constexpr int VC = v_chunk<N>();
    for (int i = threadIdx.x; i < 9 * VC; i += blockDim.x) {
        const int k = i / VC, yy = i - k * VC;
        cp_async<16>(&smV[i], &V[k * vol + (long)x * N + c0 + yy]);
    }
}

// Transform NSEQ contiguous padded sequences in rounds of blockDim/(N/8).
template <typename T, int N, int NSEQ>
__device__ __forceinline__ void fft_rows_smem(C2<T>* sm, T sign, const C2<T>* __restrict__ tw) {
    constexpr int TPS = N / 8;
    const int spr = blockDim.x / TPS;
    const int r = threadIdx.x / TPS;
    for (int s0 = 0; s0 < NSEQ; s0 += spr) {
        const int s = s0 + r;
        fft_smem<T, N>(sm, RowIdx{s * N}, threadIdx.x % TPS, r < spr && s < NSEQ, sign, tw);
    }
}

template <typename T> __device__ __forceinline__ const T* ktab(const EventDev& e);
template <> __device__ __forceinline__ const double* ktab<double>(const EventDev& e) { return e.k64; }
template <> __device__ __forceinline__ const float* ktab<float>(const EventDev& e) { return e.k32; }
template <typename T> __device__ __forceinline__ const T* kretab(const EventDev& e);
template <> __device__ __forceinline__ const double* kretab<double>(const EventDev& e) { return e.kre64; }
template <> __device__ __forceinline__ const float* kretab<float>(const EventDev& e) { return e.kre32; }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// w + re(K_x) X + re(K_y) Y: the real parts of a kernel table (null for the
// momentum kernels and the SIN position kernel, whose tables are imaginary)
template <typename V, typename T>
__device__ __forceinline__ V kmul_re(V w, T rx, T ry, V X, V Y) {
    V r;
    r.x = fma_t(ry, Y.x, fma_t(rx, X.x, w.x));
    r.y = fma_t(ry, Y.y, fma_t(rx, X.y, w.y));
    return r;
}
template <typename T> __device__ __forceinline__ const T* nftab(const EventDev& e);
template <> __device__ __forceinline__ const double* nftab<double>(const EventDev& e) { return e.nf64; }
template <> __device__ __forceinline__ const float* nftab<float>(const EventDev& e) { return e.nf32; }

// ------------------------------------------------------------------ pass 1
// One CTA per row when its 16 sequences and a V chunk fit in shared memory
// (p1_groups == 1): V is staged with cp.async while the CTA draws the noise.
// Otherwise (p1_groups == 2) blockIdx.y = 0 builds sequences 0..7 (the noise)
// and blockIdx.y = 1 sequences 8..15 (V xi V^dagger), each drawing the noise.
template <typename T, int N> constexpr int p1_groups() {
    return (16 * N * (int)sizeof(C2<T>) + 9 * v_chunk<N>() * 16) <= 140 * 1024 ? 1 : 2;
}
template <int N> constexpr int p1_threads() { return N >= 512 ? 512 : 256; }
template <typename T, int N> constexpr size_t p1_smem_bytes() {
    return sizeof(C2<T>) * padded_len(16 / p1_groups<T, N>() * N) + sizeof(double2) * 9 * v_chunk<N>();
}

template <typename T, int N>
__device__ __forceinline__ void p1_noise(const EventDev& e, const T* __restrict__ nf, int x, int y, T z[16]) {
    const long site = (long)x * N + y;
    langevin_normals<T>(e.seed, e.step, (uint32_t)site, z);
    const T f = nf ? nf[site] : (T)1;
#pragma unroll
    for (int k = 0; k < 16; ++k) z[k] *= f;
}

// V xi V^dagger coefficients for xi = sum n_a L_a
template <typename T>
__device__ __forceinline__ void p1_rotate(const C2<T> v[9], const T n[8], T h[8]) {
    C2<T> xi[9], t[9], r[9];
    embed_lambda<T>(n, xi);
    mul3(v, xi, t);
    mul3_adj(t, v, r);
    project_lambda<T>(r, h);
}

template <typename T, int N>
__global__ void __launch_bounds__(p1_threads<N>()) k_step_pass1(const EventDev* __restrict__ ev,
                                                                 const int* __restrict__ slots,
                                                                 C2<T>* __restrict__ P,
                                                                 const C2<T>* __restrict__ tw) {
    using V2 = C2<T>;
    constexpr int VC = v_chunk<N>();
    constexpr int G = p1_groups<T, N>();
    constexpr int NSEQ = 16 / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V2* sm = reinterpret_cast<V2*>(smem_raw);
    double2* smV = reinterpret_cast<double2*>(smem_raw + sizeof(V2) * padded_len(NSEQ * N));
    const int x = blockIdx.x, g = blockIdx.y, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const T* nf = nftab<T>(e);
    const bool want_noise = (G == 1) || g == 0;
    const bool want_rot = (G == 1) || g == 1;
    const int rot_base = (G == 1) ? 8 : 0;  // local sequence index of the first rotated pack
    // one site per thread per chunk: VC <= blockDim.x
    for (int c0 = 0; c0 < N; c0 += VC) {
        if (want_rot) {
            if (c0 > 0) __syncthreads();
            stage_v<N>(smV, e.V, vol, x, c0);
            cp_async_commit();
        }
        const bool have = threadIdx.x < VC;
        const int y = c0 + threadIdx.x;
        T z[16];
        if (have) {
            p1_noise<T, N>(e, nf, x, y, z);
            if (want_noise) {
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    sm[pad(s * N + y)] = mk<T>(z[4 * s], z[4 * s + 2]);            // n_{2s} + i n_{2s+1}
                    sm[pad((4 + s) * N + y)] = mk<T>(z[4 * s + 1], z[4 * s + 3]);  // m_{2s} + i m_{2s+1}
                }
            }
        }
        if (want_rot) {
            cp_async_wait<0>();
            __syncthreads();
            if (have) {
                T n[8], m[8], h[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    n[k] = z[2 * k];
                    m[k] = z[2 * k + 1];
                }
                V2 v[9];
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    const double2 dv = smV[k * VC + threadIdx.x];
                    v[k] = mk<T>((T)dv.x, (T)dv.y);
                }
                p1_rotate<T>(v, n, h);
#pragma unroll
                for (int s = 0; s < 4; ++s) sm[pad((rot_base + s) * N + y)] = mk<T>(h[2 * s], h[2 * s + 1]);
                p1_rotate<T>(v, m, h);
#pragma unroll
                for (int s = 0; s < 4; ++s) sm[pad((rot_base + 4 + s) * N + y)] = mk<T>(h[2 * s], h[2 * s + 1]);
            }
        }
    }
    __syncthreads();
    fft_rows_smem<T, N, NSEQ>(sm, (T)-1, tw);
    V2* out = P + ((long)b * 16 + NSEQ * g) * vol + (long)x * N;
    for (int i = threadIdx.x; i < NSEQ * N; i += blockDim.x) {
        const int s = i / N, y = i - s * N;
        out[s * vol + y] = sm[pad(i)];
    }
}

// ------------------------------------------------------------------ pass 2
template <typename T, int N>
__global__ void __launch_bounds__(p2_cols<T, N>() * (N / 8), p2_cols<T, N>() * (N / 8) <= 512 ? 2 : 1) k_step_pass2(const EventDev* __restrict__ ev,
                                                                           const int* __restrict__ slots,
                                                                           const C2<T>* __restrict__ P,
                                                                           C2<T>* __restrict__ Q,
                                                                           const C2<T>* __restrict__ tw) {
    using V2 = C2<T>;
    constexpr int C = p2_cols<T, N>();
    constexpr int TILE = padded_len(N * C);
    constexpr int TH = C * (N / 8);
    constexpr int PER = (N * C) / TH;  // = 8
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V2* t0 = reinterpret_cast<V2*>(smem_raw);
    V2* t1 = t0 + TILE;
    const int c0 = blockIdx.x * C, j = blockIdx.y, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const int p0 = j < 4 ? j : 8 + (j - 4), p1 = p0 + 4;
    // thread -> (row r0 + q N/8, column cc) of the tile for q < PER
    const int cc = threadIdx.x % C, r0 = threadIdx.x / C;
    constexpr int RSTEP = TH / C;  // = N / 8
    const V2* in0 = P + ((long)b * 16 + p0) * vol + c0 + (long)r0 * N + cc;
    const V2* in1 = P + ((long)b * 16 + p1) * vol + c0 + (long)r0 * N + cc;
    // kernel table tile (imag K_x, imag K_y) beside the data tiles
    T* kxs = reinterpret_cast<T*>(t1 + TILE);
    T* kys = kxs + N * C;
    const T* kt = ktab<T>(e) + c0 + (long)r0 * N + cc;
    const T* kre = kretab<T>(e) ? kretab<T>(e) + c0 + (long)r0 * N + cc : nullptr;
#pragma unroll 1
    for (int q = 0; q < PER; ++q) {
        const int i = threadIdx.x + q * TH;
        const int goff = q * RSTEP * N;
        cp_async<(int)sizeof(V2)>(&t0[pad(i)], in0 + goff);
        cp_async<(int)sizeof(V2)>(&t1[pad(i)], in1 + goff);
        cp_async<(int)sizeof(T)>(&kxs[i], kt + goff);
        cp_async<(int)sizeof(T)>(&kys[i], kt + vol + goff);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const int c = threadIdx.x % C, t = threadIdx.x / C;
    fft_smem<T, N>(t0, ColIdx<C>{c}, t, true, (T)-1, tw);
    fft_smem<T, N>(t1, ColIdx<C>{c}, t, true, (T)-1, tw);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int i = threadIdx.x + q * TH;
        const V2 a = t0[pad(i)], bb = t1[pad(i)];
        const T kx = kxs[i], ky = kys[i];
        // (i kx) a + (i ky) b
        V2 w = mk<T>(-kx * a.y - ky * bb.y, kx * a.x + ky * bb.x);
        if (kre) w = kmul_re(w, __ldg(kre + q * RSTEP * N), __ldg(kre + vol + q * RSTEP * N), a, bb);
        t0[pad(i)] = w;
    }
    __syncthreads();
    fft_smem<T, N>(t0, ColIdx<C>{c}, t, true, (T)1, tw);
    V2* out = Q + ((long)b * 8 + j) * vol + c0 + (long)r0 * N + cc;
#pragma unroll 2
    for (int q = 0; q < PER; ++q) out[q * RSTEP * N] = t0[pad(threadIdx.x + q * TH)];
}

// ------------------------------------------------------------------ pass 3
template <typename T, int N>
__global__ void __launch_bounds__(row_threads<N>(), 2) k_step_pass3(EventDev* __restrict__ ev,
                                                                     const int* __restrict__ slots,
                                                                     const C2<T>* __restrict__ Q,
                                                                     const C2<T>* __restrict__ tw,
                                                                     int* __restrict__ flags) {
    using V2 = C2<T>;
    constexpr int VC = v_chunk<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V2* sm = reinterpret_cast<V2*>(smem_raw);
    double2* smV = reinterpret_cast<double2*>(smem_raw + sizeof(V2) * padded_len(8 * N));
    const int x = blockIdx.x, b = blockIdx.y;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const V2* in = Q + (long)b * 8 * vol + (long)x * N;
    for (int i = threadIdx.x; i < 8 * N; i += blockDim.x)
        cp_async<(int)sizeof(V2)>(&sm[pad(i)], &in[(long)(i / N) * vol + (i % N)]);
    cp_async_commit();
    stage_v<N>(smV, e.V, vol, x, 0);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    fft_rows_smem<T, N, 8>(sm, (T)1, tw);
    const double se = e.sqrt_eps;
    int fl = 0;
    for (int c0 = 0; c0 < N; c0 += VC) {
        if (c0 > 0) {
            __syncthreads();
            stage_v<N>(smV, e.V, vol, x, c0);
            cp_async_commit();
        }
        cp_async_wait<0>();
        __syncthreads();
        for (int y = c0 + threadIdx.x; y < c0 + VC; y += blockDim.x) {
            double a[8], bq[8];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const V2 u = sm[pad(s * N + y)], w = sm[pad((4 + s) * N + y)];
                a[2 * s] = (double)u.x * se;
                a[2 * s + 1] = (double)u.y * se;
                bq[2 * s] = (double)w.x * -se;
                bq[2 * s + 1] = (double)w.y * -se;
            }
            double2 mA[9], mB[9], v[9], tmp[9];
            embed_lambda<double>(a, mA);
            embed_lambda<double>(bq, mB);
            expi_ch(mB, -1.0);  // exp(+i sqrt(eps) B)
            expi_ch(mA, -1.0);  // exp(-i sqrt(eps) A)
#pragma unroll
            for (int k = 0; k < 9; ++k) v[k] = smV[k * VC + (y - c0)];
            mul3(mB, v, tmp);
            mul3(tmp, mA, v);
            if (e.reunit) reunitarize(v);
            const long site = (long)x * N + y;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                if (!isfinite(v[k].x) || !isfinite(v[k].y)) fl |= JW_FLAG_NAN;
                e.V[k * vol + site] = v[k];
            }
        }
    }
    if (fl) atomicOr(flags, fl);
    if (x == 0 && threadIdx.x == 0) e.step += 1;
}

// average_and_symmetrize (field.h:1460-1492) + reduce (field.h:1521-1536) with
// compensated (Neumaier) FP64 accumulation of sum and sum of squares.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double v) {
    const double t = s + v;
    c += (fabs(s) >= fabs(v)) ? (s - t) + v : (v - t) + s;
    s = t;
}

// corr and corrT hold each event's correlator and its transpose
// (corrT[q][p] = corr[p][q]), so that every load below is coalesced.
template <int N>
__device__ __forceinline__ double symmetrized(const double* __restrict__ cb, const double* __restrict__ cbT,
                                              int x, int y) {
    const int a = (N - x) % N, bb = (N - y) % N;
    auto tsym = [&](int p, int q) {
        const long o = (long)p * N + q;
        return 0.5 * (__ldg(cb + o) + __ldg(cbT + o));
    };
    return 0.25 * (((tsym(x, y) + tsym(a, y)) + tsym(x, bb)) + tsym(a, bb));
}

template <int N>
__global__ void k_meas_reduce(EventDev* __restrict__ ev, const int* __restrict__ slots,
                              const double* __restrict__ corr, const double* __restrict__ corrT) {
    const long vol = (long)N * N;
    const int b = blockIdx.y;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    EventDev& e = ev[slots[b]];
    if (i < vol) {
        const int x = (int)(i / N), y = (int)(i % N);
        const double s = symmetrized<N>(corr + (long)b * vol, corrT + (long)b * vol, x, y);
        double* acc = e.acc;
        double s0 = acc[i], s1 = acc[vol + i], e0 = acc[2 * vol + i], e1 = acc[3 * vol + i];
        neumaier_add(s0, s1, s);
        neumaier_add(e0, e1, s * s);
        acc[i] = s0;
        acc[vol + i] = s1;
        acc[2 * vol + i] = e0;
        acc[3 * vol + i] = e1;
    }
    if (i == 0) e.nmeas += 1;
}

// Ensemble measurement: symmetrise the correlators of the nb events of a
// batch and add their sum and sum of squares (over events) into ens[4][N*N]
// (sum, compensation, err, compensation) -- gfield::reduce over stats.
template <int N>
__global__ void k_meas_reduce_ensemble(const double* __restrict__ corr, const double* __restrict__ corrT, int nb,
                                       double* __restrict__ ens) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const int x = (int)(i / N), y = (int)(i % N);
    double s0 = ens[i], s1 = ens[vol + i], e0 = ens[2 * vol + i], e1 = ens[3 * vol + i];
#pragma unroll 4
    for (int b = 0; b < nb; ++b) {
        const double s = symmetrized<N>(corr + (long)b * vol, corrT + (long)b * vol, x, y);
        neumaier_add(s0, s1, s);
        neumaier_add(e0, e1, s * s);
    }
    ens[i] = s0;
    ens[vol + i] = s1;
    ens[2 * vol + i] = e0;
    ens[3 * vol + i] = e1;
}

// The ensemble's compensated sums as the reference's complex fields
// (sum, err), each vol complex doubles with zero imaginary part.
__global__ void k_ens_finalize(const double* __restrict__ ens, long vol, double2* __restrict__ out) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    out[i] = make_double2(ens[i] + ens[vol + i], 0.0);
    out[vol + i] = make_double2(ens[2 * vol + i] + ens[3 * vol + i], 0.0);
}

}  // namespace jw
