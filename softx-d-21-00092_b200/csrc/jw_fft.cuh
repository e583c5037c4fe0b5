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
