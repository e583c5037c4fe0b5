// jw_fft.cuh -- shared-memory FFT core used by every transform in libjimwlk.
//
// Stockham autosort FFT (natural order in and out, no bit reversal) for
// power-of-two lengths 8 <= N <= 2048, radix 8 with a final radix-4 or
// radix-2 pass.  One length-N sequence is processed by N/8 threads that each
// hold 8 complex values per pass: one radix-8 butterfly, two radix-4 or four
// radix-2 butterflies.  A pass loads all values of the CTA's sequences into
// registers, synchronises, and stores them back to the same shared buffer, so
// the transform is in place.  All threads of the CTA must call the routines
// together (they contain __syncthreads); threads without a sequence pass
// active = false.
//
// Pass with radix R after sub-transforms of size Ns (Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors",
// SC'08, Stockham formulation): butterfly b in [0, N/R), k = b mod Ns,
//   v_r = x[b + r N/R] * w^(r k N/(Ns R)),  r < R,   w = exp(sign 2 pi i / N)
//   v   = DFT_R(v)
//   x[(b/Ns) Ns R + k + r Ns] = v_r.
// Twiddles come from a table tw[m] = exp(+2 pi i m / N), m < N, computed in
// FP64 on the host (conjugated for sign = -1).
#pragma once

#include "jw_common.cuh"

namespace jw {

// Padded shared-memory index: one spare slot every 32 elements, which breaks
// the power-of-two strides of the early passes across banks.
__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 5); }

template <typename V, typename T>
__device__ __forceinline__ void bfly2(V& a, V& b) {
    V t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <typename V, typename T>
__device__ __forceinline__ void bfly4(V& a, V& b, V& c, V& d, T sign) {
    V t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = cmul_si(csub(b, d), sign);
    a = cadd(t0, t2);
    c = csub(t0, t2);
    b = cadd(t1, t3);
    d = csub(t1, t3);
}

template <typename V, typename T>
__device__ __forceinline__ void bfly8(V* v, T sign) {
    // even: v0 v2 v4 v6, odd: v1 v3 v5 v7
    bfly4<V, T>(v[0], v[2], v[4], v[6], sign);
    bfly4<V, T>(v[1], v[3], v[5], v[7], sign);
    const T h = (T)0.70710678118654752440;
    // O1 *= (1 + s i)/sqrt2, O2 *= s i, O3 *= (-1 + s i)/sqrt2
    {
        V o = v[3];
        v[3] = mk<T>(h * (o.x - sign * o.y), h * (sign * o.x + o.y));
    }
    v[5] = cmul_si(v[5], sign);
    {
        V o = v[7];
        v[7] = mk<T>(h * (-o.x - sign * o.y), h * (sign * o.x - o.y));
    }
    // X[k] = E[k] + O[k], X[k+4] = E[k] - O[k]; E[k] in v[2k], O[k] in v[2k+1]
    V x0 = cadd(v[0], v[1]), x4 = csub(v[0], v[1]);
    V x1 = cadd(v[2], v[3]), x5 = csub(v[2], v[3]);
    V x2 = cadd(v[4], v[5]), x6 = csub(v[4], v[5]);
    V x3 = cadd(v[6], v[7]), x7 = csub(v[6], v[7]);
    v[0] = x0; v[1] = x1; v[2] = x2; v[3] = x3;
    v[4] = x4; v[5] = x5; v[6] = x6; v[7] = x7;
}

template <typename T, int N, int Ns, int R, typename IdxF>
__device__ __forceinline__ void stockham_pass(C2<T>* __restrict__ sm, const IdxF& idx, int t, bool active, T sign,
                                              const C2<T>* __restrict__ tw) {
    using V = C2<T>;
    constexpr int B = 8 / R;       // butterflies per thread
    constexpr int NB = N / R;      // butterflies per sequence
    constexpr int TPS = N / 8;     // threads per sequence
    constexpr int TWS = N / (Ns * R);
    V v[8];
    if (active) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) v[q * R + r] = sm[idx(b + r * NB)];
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    V w = __ldg(&tw[r * k * TWS]);
                    w.y *= sign;
                    v[q * R + r] = cmul(v[q * R + r], w);
                }
            }
            if constexpr (R == 8) {
                bfly8<V, T>(v, sign);
            } else if constexpr (R == 4) {
                bfly4<V, T>(v[q * 4 + 0], v[q * 4 + 1], v[q * 4 + 2], v[q * 4 + 3], sign);
            } else {
                bfly2<V, T>(v[q * 2 + 0], v[q * 2 + 1]);
            }
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
            const int base = (b / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm[idx(base + r * Ns)] = v[q * R + r];
        }
    }
    __syncthreads();
}

template <typename T, int N, int Ns, typename IdxF>
__device__ __forceinline__ void fft_passes(C2<T>* sm, const IdxF& idx, int t, bool active, T sign,
                                           const C2<T>* __restrict__ tw) {
    if constexpr (Ns < N) {
        constexpr int rem = N / Ns;
        constexpr int R = rem >= 8 ? 8 : rem;
        stockham_pass<T, N, Ns, R>(sm, idx, t, active, sign, tw);
        fft_passes<T, N, Ns * R>(sm, idx, t, active, sign, tw);
    }
}

// Transform the sequence x[e] = sm[idx(e)], e < N, with thread t < N/8 of it.
// sign = -1: forward (X -> K, FFTW_FORWARD); +1: backward.  Unnormalised.
template <typename T, int N, typename IdxF>
__device__ __forceinline__ void fft_smem(C2<T>* sm, const IdxF& idx, int t, bool active, T sign,
                                         const C2<T>* __restrict__ tw) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two N >= 8");
    fft_passes<T, N, 1>(sm, idx, t, active, sign, tw);
}

// Index maps -----------------------------------------------------------------
// contiguous sequence starting at `base` (padded)
struct RowIdx {
    int base;
    __device__ __forceinline__ int operator()(int e) const { return pad(base + e); }
};
// column c of a [N][C] tile (padded flat index)
template <int C>
struct ColIdx {
    int c;
    __device__ __forceinline__ int operator()(int e) const { return pad(e * C + c); }
};

}  // namespace jw

// ============================================================================
// 16-byte-element core: each shared-memory element carries VL complex values
// (VL = 2 for FP32 as float4, VL = 1 for FP64 as double2) that are transformed
// as independent sequences with the same twiddles, so one 128-bit access and
// one twiddle set serve both.  Same Stockham schedule as fft_smem.  Twiddles
// per radix-8 butterfly: w, w^2, w^4 from the table, w^3 = w w^2, w^5 = w^4 w,
// w^6 = w^4 w^2, w^7 = w^4 w^3.
namespace jw {

template <typename T> struct Elem16;
template <> struct Elem16<float> { using E = float4; static constexpr int VL = 2; };
template <> struct Elem16<double> { using E = double2; static constexpr int VL = 1; };

__device__ __forceinline__ void unpack16(const float4& e, float2* v) {
    v[0] = make_float2(e.x, e.y);
    v[1] = make_float2(e.z, e.w);
}
__device__ __forceinline__ float4 pack16(const float2* v) { return make_float4(v[0].x, v[0].y, v[1].x, v[1].y); }
__device__ __forceinline__ void unpack16(const double2& e, double2* v) { v[0] = e; }
__device__ __forceinline__ double2 pack16(const double2* v) { return v[0]; }

// padded row index for 16-byte elements: one spare element every 8
__device__ __forceinline__ int pad16(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int padded_len16(int n) { return n + (n >> 3); }

struct RowIdx16 {
    int base;
    __device__ __forceinline__ int operator()(int e) const { return pad16(base + e); }
};
// column c of a [N][C] tile of 16-byte elements; with C * 16 = 128 bytes a
// quarter warp covers one tile row, so no padding is needed
template <int C>
struct ColIdx16 {
    int c;
    __device__ __forceinline__ int operator()(int e) const { return e * C + c; }
};

// Twiddle sources: the global table (read through the read-only cache) or a
// copy of it in shared memory (TwShared), for kernels that keep one.
template <typename V> struct TwShared {
    const V* p;
};
template <typename V>
__device__ __forceinline__ V tw_get(const V* __restrict__ tw, int m) { return __ldg(&tw[m]); }
template <typename V>
__device__ __forceinline__ V tw_get(const TwShared<V>& tw, int m) { return tw.p[m]; }

template <typename V, typename T, typename TW>
__device__ __forceinline__ V tw_load(const TW& tw, int m, T sign) {
    V w = tw_get(tw, m);
    w.y *= sign;
    return w;
}

__device__ __forceinline__ float2 tw_mul(float2 a, float2 b) {
    return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 tw_mul(double2 a, double2 b) {
    return make_double2(__fma_rn(a.x, b.x, -__dmul_rn(a.y, b.y)), __fma_rn(a.x, b.y, __dmul_rn(a.y, b.x)));
}

// Per-pass twiddle table in shared memory (TwPass): for every pass with
// sub-transform size Ns > 1 and radix R, entry k < Ns holds w^0 .. w^(R-1) of
// that pass's butterfly (w = exp(+2 pi i k TWS / N)), R complex values, so a
// butterfly reads its twiddles with R/2 128-bit loads of one entry and forms
// none of them by multiplication.  w, w^2 and w^4 come from the length-N table
// and w^3, w^5, w^6, w^7 are formed by the same products tw_fill forms at run
// time (conjugation commutes with them exactly), so every twiddle source gives
// bit-identical transforms.  Entries of the pass with size Ns start at value
// tw_pass_voffset<N, Ns, S>(); the table holds tw_pass_values<N, S>() values
// (S: the radix schedule, below).
// Radix schedules.  A transform of N = 8^a r points (r = 1, 2 or 4) takes
// a radix-8 passes and one radix-r pass.  Schedule 0 runs the radix-8 passes
// first and the radix-r pass last (the default of every transform); schedule
// 1 runs the radix-r pass first.  The two round differently, so a schedule is
// a tuning choice that must be recorded with the results.
__host__ __device__ constexpr int lg2c(int n) { return n <= 1 ? 0 : 1 + lg2c(n / 2); }
template <int N, int S>
__host__ __device__ constexpr int fft_radix(int Ns) {
    return (S == 1 && Ns == 1 && lg2c(N) % 3 != 0 && N > 8) ? (1 << (lg2c(N) % 3)) : (N / Ns >= 8 ? 8 : N / Ns);
}
// N has a radix-r pass (r = 2 or 4), so schedule 1 differs from schedule 0
template <int N> constexpr bool fft_has_rem() { return N > 8 && lg2c(N) % 3 != 0; }

template <typename V, int S = 0> struct TwPass {
    const V* p;
};
template <int N, int Ns>
__host__ __device__ constexpr int tw_pass_offset() {
    // sum of the sizes Ns' of the earlier twiddled passes (1 < Ns' < Ns): 8, 64, 512, ...
    int off = 0;
    for (int n = 8; n < Ns && n < N; n *= 8) off += n;
    return off;
}
template <int N>
__host__ __device__ constexpr int tw_pass_entries() {
    int off = 0;
    for (int n = 8; n < N; n *= 8) off += n;
    return off;
}
// Offsets of the compact table of schedule S: the twiddled passes (Ns > 1) in
// order, each with Ns entries of R values.
template <int N, int Ns, int S = 0>
__host__ __device__ constexpr int tw_pass_voffset() {
    int off = 0;
    for (int n = fft_radix<N, S>(1); n < Ns && n < N; n *= fft_radix<N, S>(n)) off += n * fft_radix<N, S>(n);
    return off;
}
template <int N, int S = 0>
__host__ __device__ constexpr int tw_pass_values() {
    int off = 0;
    for (int n = fft_radix<N, S>(1); n < N; n *= fft_radix<N, S>(n)) off += n * fft_radix<N, S>(n);
    return off;
}
template <int N, int S = 0>
__host__ __device__ constexpr int tw_pass_entries_s() {
    int off = 0;
    for (int n = fft_radix<N, S>(1); n < N; n *= fft_radix<N, S>(n)) off += n;
    return off;
}
// Fill a TwPass table (tw_pass_values<N, S>() values) from the length-N table
// tw[m] = exp(+2 pi i m / N); all threads of the CTA call it.
template <typename V, int N, int S = 0>
__device__ __forceinline__ void tw_pass_fill(V* dst, const V* __restrict__ tw) {
    constexpr int E = tw_pass_entries_s<N, S>();
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        int Ns = fft_radix<N, S>(1), base = 0, voff = 0;
        while (e >= base + Ns) {
            base += Ns;
            voff += Ns * fft_radix<N, S>(Ns);
            Ns *= fft_radix<N, S>(Ns);
        }
        const int R = fft_radix<N, S>(Ns);
        const int k = e - base;
        const int TWS = N / (Ns * R);
        V w[8];
        for (int r = 0; r < 8; ++r) w[r] = V{};
        w[0].x = 1.0f;
        w[1] = __ldg(&tw[k * TWS]);
        if (R >= 4) w[2] = __ldg(&tw[2 * k * TWS]);
        if (R == 4) w[3] = tw_mul(w[1], w[2]);
        if (R == 8) {
            w[4] = __ldg(&tw[4 * k * TWS]);
            w[3] = tw_mul(w[1], w[2]);
            w[5] = tw_mul(w[4], w[1]);
            w[6] = tw_mul(w[4], w[2]);
            w[7] = tw_mul(w[4], w[3]);
        }
        // entries before this one: the earlier passes' values (voff), then k entries of R
#pragma unroll
        for (int r = 0; r < 8; ++r)
            if (r < R) dst[voff + k * R + r] = w[r];
    }
}

// The same per-pass table in the layout the row transforms want (TwRows):
// the Ns entries of a pass are stored as 4 blocks of Ns float4 values, block j
// holding (w^2j, w^2j+1) of every butterfly k.  Threads of a row transform read
// consecutive k, so their 128-bit loads are conflict-free; the entry-major
// TwPass layout puts consecutive k 64 bytes apart (a 4-way bank conflict) and
// suits the column transforms, whose quarter-warps share one k.  The values
// are TwPass's, so both give bit-identical transforms.
template <typename V> struct TwRows {
    const V* p;
};
template <typename V, int N>
__device__ __forceinline__ void tw_rows_fill(V* dst, const V* __restrict__ tw) {
    constexpr int E = tw_pass_entries<N>();
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        int Ns = 8, base = 0;
        while (e >= base + Ns) {
            base += Ns;
            Ns *= 8;
        }
        const int rem = N / Ns;
        const int R = rem >= 8 ? 8 : rem;
        const int k = e - base;
        const int TWS = N / (Ns * R);
        V w[8];
        for (int r = 0; r < 8; ++r) w[r] = V{};
        w[0].x = 1.0f;
        w[1] = __ldg(&tw[k * TWS]);
        if (R >= 4) w[2] = __ldg(&tw[2 * k * TWS]);
        if (R == 4) w[3] = tw_mul(w[1], w[2]);
        if (R == 8) {
            w[4] = __ldg(&tw[4 * k * TWS]);
            w[3] = tw_mul(w[1], w[2]);
            w[5] = tw_mul(w[4], w[1]);
            w[6] = tw_mul(w[4], w[2]);
            w[7] = tw_mul(w[4], w[3]);
        }
        for (int j = 0; j < 4; ++j) {
            V* d = dst + 2 * (4 * base + j * Ns + k);
            d[0] = w[2 * j];
            d[1] = w[2 * j + 1];
        }
    }
}

// The twiddles w^1 .. w^(R-1) of butterfly k of pass (Ns, R), conjugated for
// sign = -1.  Products of twiddles use explicit fused multiply-adds, so that
// the per-pass tables (formed from unconjugated values) and this run-time
// derivation (from conjugated ones) agree bit for bit.
template <typename V, typename T, int N, int Ns, int R, typename TW>
__device__ __forceinline__ void tw_fill(const TW& tw, int k, T sign, V (&w)[8]) {
    constexpr int TWS = N / (Ns * R);
    w[1] = tw_load<V>(tw, k * TWS, sign);
    if constexpr (R >= 4) w[2] = tw_load<V>(tw, 2 * k * TWS, sign);
    if constexpr (R == 4) w[3] = tw_mul(w[1], w[2]);
    if constexpr (R == 8) {
        w[4] = tw_load<V>(tw, 4 * k * TWS, sign);
        w[3] = tw_mul(w[1], w[2]);
        w[5] = tw_mul(w[4], w[1]);
        w[6] = tw_mul(w[4], w[2]);
        w[7] = tw_mul(w[4], w[3]);
    }
}
template <typename V, typename T, int N, int Ns, int R, int S>
__device__ __forceinline__ void tw_fill(const TwPass<V, S>& tw, int k, T sign, V (&w)[8]) {
    static_assert(sizeof(V) == 8, "per-pass tables hold complex FP32");
    const float4* e = reinterpret_cast<const float4*>(tw.p + tw_pass_voffset<N, Ns, S>() + k * R);
    const float4 a = e[0];
    w[1] = make_float2(a.z, a.w * sign);
    if constexpr (R >= 4) {
        const float4 b = e[1];
        w[2] = make_float2(b.x, b.y * sign);
        w[3] = make_float2(b.z, b.w * sign);
    }
    if constexpr (R == 8) {
        const float4 c = e[2], d = e[3];
        w[4] = make_float2(c.x, c.y * sign);
        w[5] = make_float2(c.z, c.w * sign);
        w[6] = make_float2(d.x, d.y * sign);
        w[7] = make_float2(d.z, d.w * sign);
    }
}

template <typename V, typename T, int N, int Ns, int R>
__device__ __forceinline__ void tw_fill(const TwRows<V>& tw, int k, T sign, V (&w)[8]) {
    static_assert(sizeof(V) == 8, "per-pass tables hold complex FP32");
    const float4* e = reinterpret_cast<const float4*>(tw.p) + 4 * tw_pass_offset<N, Ns>() + k;
    const float4 a = e[0];
    w[1] = make_float2(a.z, a.w * sign);
    if constexpr (R >= 4) {
        const float4 b = e[Ns];
        w[2] = make_float2(b.x, b.y * sign);
        w[3] = make_float2(b.z, b.w * sign);
    }
    if constexpr (R == 8) {
        const float4 c = e[2 * Ns], d = e[3 * Ns];
        w[4] = make_float2(c.x, c.y * sign);
        w[5] = make_float2(c.z, c.w * sign);
        w[6] = make_float2(d.x, d.y * sign);
        w[7] = make_float2(d.z, d.w * sign);
    }
}

template <typename T, int N, int Ns, int R, typename IdxF, typename TW>
__device__ __forceinline__ void stockham_pass16(typename Elem16<T>::E* __restrict__ sm, const IdxF& idx, int t,
                                                bool active, T sign, const TW& tw) {
    using V = C2<T>;
    using E = typename Elem16<T>::E;
    constexpr int VL = Elem16<T>::VL;
    constexpr int B = 8 / R;
    constexpr int NB = N / R;
    constexpr int TPS = N / 8;
    V v[VL][8];
    if (active) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V u[VL];
                unpack16(sm[idx(b + r * NB)], u);
#pragma unroll
                for (int l = 0; l < VL; ++l) v[l][q * R + r] = u[l];
            }
            if (Ns > 1) {
                V w[8];
                tw_fill<V, T, N, Ns, R>(tw, k, sign, w);
#pragma unroll
                for (int r = 1; r < R; ++r)
#pragma unroll
                    for (int l = 0; l < VL; ++l) v[l][q * R + r] = cmul(v[l][q * R + r], w[r]);
            }
#pragma unroll
            for (int l = 0; l < VL; ++l) {
                if constexpr (R == 8) {
                    bfly8<V, T>(v[l], sign);
                } else if constexpr (R == 4) {
                    bfly4<V, T>(v[l][q * 4 + 0], v[l][q * 4 + 1], v[l][q * 4 + 2], v[l][q * 4 + 3], sign);
                } else {
                    bfly2<V, T>(v[l][q * 2 + 0], v[l][q * 2 + 1]);
                }
            }
        }
    }
    __syncthreads();
    if (active) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
            const int base = (b / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V u[VL];
#pragma unroll
                for (int l = 0; l < VL; ++l) u[l] = v[l][q * R + r];
                sm[idx(base + r * Ns)] = pack16(u);
            }
        }
    }
    __syncthreads();
}

template <typename T, int N, int Ns, typename IdxF, typename TW>
__device__ __forceinline__ void fft16_passes(typename Elem16<T>::E* sm, const IdxF& idx, int t, bool active, T sign,
                                             const TW& tw) {
    if constexpr (Ns < N) {
        constexpr int rem = N / Ns;
        constexpr int R = rem >= 8 ? 8 : rem;
        stockham_pass16<T, N, Ns, R>(sm, idx, t, active, sign, tw);
        fft16_passes<T, N, Ns * R>(sm, idx, t, active, sign, tw);
    }
}

// Synchronisation of the threads that share a transform: the whole CTA
// (SyncCTA), or a named barrier of a group of `count` threads (SyncBar;
// count a multiple of 32, id 1..15, every thread of the group takes part).
struct SyncCTA {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct SyncBar {
    int id, count;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
    }
};

// Register hand-off.  After the last pass thread t holds the elements
// t + m N/8 (m = 0..7) of its sequences, and the first pass reads exactly those
// elements.  So a transform can end in registers (for an elementwise step, a
// reduction or a store) and the next one start from them, without the shared-
// memory round trip.  reg[l][m] is element t + m N/8 of sequence l.
// The general pass loads with idxL and stores with idxS (a transform may read
// its input in one layout and continue in another) and synchronises with sync.
template <typename T, int N, int Ns, int R, bool IN, bool OUT, typename IdxL, typename IdxS, typename TW,
          typename Sync>
__device__ __forceinline__ void stockham_pass16g(typename Elem16<T>::E* __restrict__ sm, const IdxL& idxL,
                                                 const IdxS& idxS, int t, bool active, T sign, const TW& tw,
                                                 C2<T> (&reg)[Elem16<T>::VL][8], const Sync& sync) {
    using V = C2<T>;
    constexpr int VL = Elem16<T>::VL;
    constexpr int B = 8 / R;
    constexpr int NB = N / R;
    constexpr int TPS = N / 8;
    static_assert(!IN || Ns == 1, "register input feeds the first pass");
    static_assert(!OUT || Ns * R == N, "register output comes from the last pass");
    V v[VL][8];
    if (active) {
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (IN) {
#pragma unroll
                    for (int l = 0; l < VL; ++l) v[l][q * R + r] = reg[l][q + r * B];  // element b + r NB
                } else {
                    V u[VL];
                    unpack16(sm[idxL(b + r * NB)], u);
#pragma unroll
                    for (int l = 0; l < VL; ++l) v[l][q * R + r] = u[l];
                }
            }
            if (Ns > 1) {
                V w[8];
                tw_fill<V, T, N, Ns, R>(tw, k, sign, w);
#pragma unroll
                for (int r = 1; r < R; ++r)
#pragma unroll
                    for (int l = 0; l < VL; ++l) v[l][q * R + r] = cmul(v[l][q * R + r], w[r]);
            }
#pragma unroll
            for (int l = 0; l < VL; ++l) {
                if constexpr (R == 8) {
                    bfly8<V, T>(v[l], sign);
                } else if constexpr (R == 4) {
                    bfly4<V, T>(v[l][q * 4 + 0], v[l][q * 4 + 1], v[l][q * 4 + 2], v[l][q * 4 + 3], sign);
                } else {
                    bfly2<V, T>(v[l][q * 2 + 0], v[l][q * 2 + 1]);
                }
            }
        }
    }
    if constexpr (OUT) {
        // output b + r Ns = t + (q + r B) N/8; the caller synchronises before
        // the buffer is written again
        if (active) {
#pragma unroll
            for (int q = 0; q < B; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int l = 0; l < VL; ++l) reg[l][q + r * B] = v[l][q * R + r];
        }
    } else {
        sync();
        if (active) {
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int b = t + q * TPS;
                const int k = b & (Ns - 1);
                const int base = (b / Ns) * Ns * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    V u[VL];
#pragma unroll
                    for (int l = 0; l < VL; ++l) u[l] = v[l][q * R + r];
                    sm[idxS(base + r * Ns)] = pack16(u);
                }
            }
        }
        sync();
    }
}

template <typename T, int N, int Ns, int R, bool IN, bool OUT, typename IdxF, typename TW>
__device__ __forceinline__ void stockham_pass16x(typename Elem16<T>::E* __restrict__ sm, const IdxF& idx, int t,
                                                 bool active, T sign, const TW& tw,
                                                 C2<T> (&reg)[Elem16<T>::VL][8]) {
    stockham_pass16g<T, N, Ns, R, IN, OUT>(sm, idx, idx, t, active, sign, tw, reg, SyncCTA{});
}

template <typename T, int N, int Ns, bool IN, bool OUT, typename IdxL0, typename IdxF, typename TW, typename Sync0,
          typename Sync>
__device__ __forceinline__ void fft16g_passes(typename Elem16<T>::E* sm, const IdxL0& idxL0, const IdxF& idx, int t,
                                              bool active, T sign, const TW& tw, C2<T> (&reg)[Elem16<T>::VL][8],
                                              const Sync0& sync0, const Sync& sync) {
    if constexpr (Ns < N) {
        constexpr int rem = N / Ns;
        constexpr int R = rem >= 8 ? 8 : rem;
        if constexpr (Ns == 1)
            stockham_pass16g<T, N, Ns, R, IN, OUT && Ns * R == N>(sm, idxL0, idx, t, active, sign, tw, reg, sync0);
        else
            stockham_pass16g<T, N, Ns, R, false, OUT && Ns * R == N>(sm, idx, idx, t, active, sign, tw, reg, sync);
        fft16g_passes<T, N, Ns * R, IN, OUT>(sm, idxL0, idx, t, active, sign, tw, reg, sync0, sync);
    }
}

// fft16x with the first pass loading through idxL0 (its input layout) and
// synchronising with sync0, every later access through idx and every later
// pass synchronising with sync.
template <typename T, int N, bool IN, bool OUT, typename IdxL0, typename IdxF, typename TW, typename Sync0,
          typename Sync>
__device__ __forceinline__ void fft16g(typename Elem16<T>::E* sm, const IdxL0& idxL0, const IdxF& idx, int t,
                                       bool active, T sign, const TW& tw, C2<T> (&reg)[Elem16<T>::VL][8],
                                       const Sync0& sync0, const Sync& sync) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two N >= 8");
    fft16g_passes<T, N, 1, IN, OUT>(sm, idxL0, idx, t, active, sign, tw, reg, sync0, sync);
}

template <typename T, int N, int Ns, bool IN, bool OUT, int S, typename IdxF, typename TW>
__device__ __forceinline__ void fft16x_passes(typename Elem16<T>::E* sm, const IdxF& idx, int t, bool active, T sign,
                                              const TW& tw, C2<T> (&reg)[Elem16<T>::VL][8]) {
    if constexpr (Ns < N) {
        constexpr int R = fft_radix<N, S>(Ns);
        stockham_pass16x<T, N, Ns, R, IN && Ns == 1, OUT && Ns * R == N>(sm, idx, t, active, sign, tw, reg);
        fft16x_passes<T, N, Ns * R, IN, OUT, S>(sm, idx, t, active, sign, tw, reg);
    }
}

// fft16 with the first pass reading reg (IN) and/or the last pass writing reg
// (OUT) instead of sm; sm still carries the passes in between.  S is the
// radix schedule (fft_radix).  Whatever the last radix, thread t ends holding
// elements t + m N/8, so the hand-off works for both schedules.
template <typename T, int N, bool IN, bool OUT, int S = 0, typename IdxF, typename TW>
__device__ __forceinline__ void fft16x(typename Elem16<T>::E* sm, const IdxF& idx, int t, bool active, T sign,
                                       const TW& tw, C2<T> (&reg)[Elem16<T>::VL][8]) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two N >= 8");
    fft16x_passes<T, N, 1, IN, OUT, S>(sm, idx, t, active, sign, tw, reg);
}

__device__ __forceinline__ void reg_get(const float4& e, float2 (&reg)[2][8], int m) {
    reg[0][m] = make_float2(e.x, e.y);
    reg[1][m] = make_float2(e.z, e.w);
}
__device__ __forceinline__ float4 reg_put(const float2 (&reg)[2][8], int m) {
    return make_float4(reg[0][m].x, reg[0][m].y, reg[1][m].x, reg[1][m].y);
}
__device__ __forceinline__ void reg_get(const double2& e, double2 (&reg)[1][8], int m) { reg[0][m] = e; }
__device__ __forceinline__ double2 reg_put(const double2 (&reg)[1][8], int m) { return reg[0][m]; }

// Transform the VL sequences held in the elements sm[idx(e)], e < N, with
// thread t < N/8; all threads of the CTA must call it.
template <typename T, int N, typename IdxF, typename TW>
__device__ __forceinline__ void fft16(typename Elem16<T>::E* sm, const IdxF& idx, int t, bool active, T sign,
                                      const TW& tw) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two N >= 8");
    fft16_passes<T, N, 1>(sm, idx, t, active, sign, tw);
}

}  // namespace jw
