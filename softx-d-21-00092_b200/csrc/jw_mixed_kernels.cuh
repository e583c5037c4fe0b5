// jw_mixed_kernels.cuh -- the mixed-precision (FP32 transform) Langevin step
// on "pair planes": each 16-byte element holds two complex FP32 values that
// travel together through the whole step, so every shared-memory access and
// every HBM access moves both at once and one twiddle set serves both.
//
//   pass 1 (row)    P[j]   = (X_j, Y_j)    j = 0..3, X_j = n_{2j} + i n_{2j+1}, Y_j = m_{2j} + i m_{2j+1}
//                   P[4+j] = (BX_j, BY_j)  the same packs of V xi_x V^dagger and V xi_y V^dagger
//                   16 row transforms of length N (8 pair rows), forward.
//   pass 2 (column) per j: column transforms of P[j] and P[4+j], then
//                   W_A = K_x X + K_y Y, W_B = K_x BX + K_y BY (prepare_A_local,
//                   field.h:1998-2075, 1/N^2 folded into K) and the inverse column
//                   transform of (W_A, W_B) into Q[j].
//   pass 3 (row)    inverse row transform of Q[j] = (A_{2j} + i A_{2j+1}, B_{2j} + i B_{2j+1}),
//                   then the FP64 update of V (update_uf, field.h:1966-1996).
//
// HBM per site: pass 1 reads V (144 B) and writes P (128 B); pass 2 reads P
// (128 B) and writes Q (64 B); pass 3 reads Q (64 B) and V and writes V (288 B).
#pragma once

#include <cooperative_groups.h>

#include "jw_async.cuh"
#include "jw_engine_kernels.cuh"

namespace jw {

// Passes 1 and 3 hold whole rows of pair planes in shared memory; each thread
// loads the V of its own sites straight into registers (a warp's loads of one
// plane are contiguous), early enough that the noise or the exponentials of
// the site cover the latency.  From N = 1024 on the 8 pair rows of pass 1
// (147 KB at 1024^2) would leave one CTA per SM, so a cluster of two CTAs
// shares each lattice row through distributed shared memory (mx_pair): rank 0
// holds the noise rows, rank 1 the rotated rows.
template <int N> constexpr bool mx_pair() { return 16 * padded_len16(8 * N) > 113 * 1024; }
template <int N> constexpr int mx_groups() { return mx_pair<N>() ? 2 : 1; }
template <int N> constexpr int mx_p1_threads() { return N >= 2048 ? 512 : 256; }
template <int N> constexpr size_t mx_p1_smem() { return 16 * (size_t)padded_len16(8 / mx_groups<N>() * N); }
template <int N> constexpr int mx_p1_blocks() { return mx_p1_threads<N>() <= 256 && mx_p1_smem<N>() <= 113 * 1024 ? 2 : 1; }
// pass 2 tile width: 4 columns (64-byte rows, padded) while two tiles fit in 80 KB
// (160 KB from N = 1024 on: one CTA of 512 threads, rows of 64 or 32 bytes)
template <int N> constexpr int mx_cols() {
    constexpr int cap = (N >= 1024 ? 65536 : 32768) / (N * 16);
    constexpr int c = cap >= 4 ? 4 : (cap >= 1 ? cap : 1);
    return c < N ? c : N;
}
template <int N> constexpr int mx_p2_threads() { return mx_cols<N>() * (N / 8); }
// column tiles narrower than 128 bytes are padded by one row every 8 rows
template <int C> struct ColIdx16P {
    int c;
    __device__ __forceinline__ int operator()(int e) const {
        return (C >= 8) ? e * C + c : e * C + c + (e >> 3) * C;
    }
};
template <int N> constexpr int mx_tile_len() {
    return mx_cols<N>() >= 8 ? N * mx_cols<N>() : N * mx_cols<N>() + (N / 8) * mx_cols<N>();
}
template <int N> constexpr size_t mx_p2_smem() { return 2 * 16 * (size_t)mx_tile_len<N>(); }
// The step's pass 2 (k_mix_pass2) is built for every column-tile width C in
// {1, 2, 4, 8} that fits (C N/8 <= 1024 threads, two tiles in 227 KB); the
// engine's autotuner picks one per lattice size, mx_s2_cols is the default.
template <int N> constexpr int mx_s2_cols() { return N == 256 ? 8 : mx_cols<N>(); }  // measured best
template <int N, int C> constexpr int mx_s2_threads() { return C * (N / 8); }
template <int N, int C> constexpr int mx_s2_tile_len() { return C >= 8 ? N * C : N * C + (N / 8) * C; }
template <int N, int C> constexpr size_t mx_s2_smem() { return 2 * 16 * (size_t)mx_s2_tile_len<N, C>(); }
template <int N, int C> constexpr int mx_s2_blocks() { return mx_s2_threads<N, C>() <= 256 ? 2 : 1; }
template <int N, int C> constexpr bool mx_s2_valid() {
    return C <= N && mx_s2_threads<N, C>() <= 1024 && mx_s2_smem<N, C>() <= 227 * 1024;
}
// pass 3: mx_p3_threads threads; the 4 inverse-transformed pair rows in shared
// memory.  MEAS: pass 3 also leaves the row-transformed measurement planes of
// the new V (5 FP32 pair planes, as k_meas32_rows writes them) in a fifth row.
template <int N> constexpr int mx_p3_threads() { return row_threads<N>(); }
template <int N> constexpr bool mx_pair();
template <int N, bool MEAS = false> constexpr size_t mx_p3_smem() {
    // the row buffer, then (one-CTA sizes) the old V of one site per thread
    return 16 * (size_t)padded_len16((MEAS ? 5 : 4) * N) + (mx_pair<N>() ? 0 : (size_t)9 * 16 * row_threads<N>());
}
template <int N, bool MEAS = false> constexpr int mx_p3_blocks() {
    return mx_p3_threads<N>() <= 256 && mx_p3_smem<N, MEAS>() <= 113 * 1024 ? 2 : 1;
}
template <int N> constexpr bool mx_p3_meas_fits() { return mx_p3_smem<N, true>() <= 220 * 1024; }

// Gell-Mann coefficients of R = V xi V^dagger, xi = sum_a n_a L_a: only the
// upper triangle and the real diagonal of R are formed (R is Hermitian), and
// t = V xi uses xi's structure (real diagonal d, upper entries c, lower
// entries conj(c)) instead of a general 3 x 3 product.  Passes 1 and 3 + 1
// both rotate; every operation is an explicitly rounded intrinsic, so the two
// kernels give the same bits whatever the compiler would fuse around them.
__device__ __forceinline__ float fm(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ void rotate_herm(const float2 v[9], const float n[8], float h[8]) {
    const float s = __fmul_rn(0.57735026918962573f, n[7]);  // n_7 / sqrt(3)
    const float d0 = __fadd_rn(n[2], s), d1 = __fsub_rn(s, n[2]), d2 = __fmul_rn(-2.0f, s);
    const float2 c01 = make_float2(n[0], n[1]), c02 = make_float2(n[3], n[4]), c12 = make_float2(n[5], n[6]);
    float2 t[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float2 a = v[i * 3 + 0], b = v[i * 3 + 1], c = v[i * 3 + 2];
        // t_i0 = a d0 + b conj(c01) + c conj(c02)
        t[i * 3 + 0] = make_float2(fm(c.y, c02.y, fm(c.x, c02.x, fm(b.y, c01.y, fm(b.x, c01.x, __fmul_rn(a.x, d0))))),
                                   fm(-c.x, c02.y, fm(c.y, c02.x, fm(-b.x, c01.y, fm(b.y, c01.x, __fmul_rn(a.y, d0))))));
        // t_i1 = a c01 + b d1 + c conj(c12)
        t[i * 3 + 1] = make_float2(fm(c.y, c12.y, fm(c.x, c12.x, fm(b.x, d1, fm(-a.y, c01.y, __fmul_rn(a.x, c01.x))))),
                                   fm(-c.x, c12.y, fm(c.y, c12.x, fm(b.y, d1, fm(a.y, c01.x, __fmul_rn(a.x, c01.y))))));
        // t_i2 = a c02 + b c12 + c d2
        t[i * 3 + 2] = make_float2(fm(c.x, d2, fm(-b.y, c12.y, fm(b.x, c12.x, fm(-a.y, c02.y, __fmul_rn(a.x, c02.x))))),
                                   fm(c.y, d2, fm(b.y, c12.x, fm(b.x, c12.y, fm(a.y, c02.x, __fmul_rn(a.x, c02.y))))));
    }
    // R_ij = sum_k t_ik conj(V_jk): real part sum t.x v.x + t.y v.y, imaginary sum t.y v.x - t.x v.y
    auto rij = [&](int i, int j) {
        float re = __fmul_rn(t[i * 3].x, v[j * 3].x), im = __fmul_rn(t[i * 3].y, v[j * 3].x);
        re = fm(t[i * 3].y, v[j * 3].y, re);
        im = fm(-t[i * 3].x, v[j * 3].y, im);
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            re = fm(t[i * 3 + k].x, v[j * 3 + k].x, re);
            re = fm(t[i * 3 + k].y, v[j * 3 + k].y, re);
            im = fm(t[i * 3 + k].y, v[j * 3 + k].x, im);
            im = fm(-t[i * 3 + k].x, v[j * 3 + k].y, im);
        }
        return make_float2(re, im);
    };
    auto rii = [&](int i) {
        float re = __fmul_rn(t[i * 3].x, v[i * 3].x);
        re = fm(t[i * 3].y, v[i * 3].y, re);
#pragma unroll
        for (int k = 1; k < 3; ++k) {
            re = fm(t[i * 3 + k].x, v[i * 3 + k].x, re);
            re = fm(t[i * 3 + k].y, v[i * 3 + k].y, re);
        }
        return re;
    };
    const float2 r01 = rij(0, 1), r02 = rij(0, 2), r12 = rij(1, 2);
    const float r00 = rii(0), r11 = rii(1), r22 = rii(2);
    h[0] = r01.x;
    h[1] = r01.y;
    h[2] = __fmul_rn(0.5f, __fsub_rn(r00, r11));
    h[3] = r02.x;
    h[4] = r02.y;
    h[5] = r12.x;
    h[6] = r12.y;
    h[7] = __fmul_rn(fm(-2.0f, r22, __fadd_rn(r00, r11)), 0.28867513459481287f);  // / (2 sqrt 3)
}

// Transform NP contiguous padded pair rows (16-byte elements) in rounds.
template <int N, int NP, typename TW>
__device__ __forceinline__ void fft16_rows(float4* sm, float sign, const TW& tw) {
    constexpr int TPS = N / 8;
    const int spr = blockDim.x / TPS;
    const int r = threadIdx.x / TPS;
    for (int p0 = 0; p0 < NP; p0 += spr) {
        const int p = p0 + r;
        fft16<float, N>(sm, RowIdx16{p * N}, threadIdx.x % TPS, r < spr && p < NP, sign, tw);
    }
}

// np rows of the padded row buffer, transformed, the last pass storing row p
// straight to out + p stride (no shared-memory round trip for the result)
template <typename T, int N, typename TW>
__device__ __forceinline__ void fft16_rows_store(typename Elem16<T>::E* sm, int np, T sign, const TW& tw,
                                                 typename Elem16<T>::E* __restrict__ out, long stride) {
    constexpr int TPS = N / 8;
    const int spr = blockDim.x / TPS;
    const int r = threadIdx.x / TPS, t = threadIdx.x % TPS;
    for (int p0 = 0; p0 < np; p0 += spr) {
        const int p = p0 + r;
        const bool act = r < spr && p < np;
        C2<T> rv[Elem16<T>::VL][8];
        fft16x<T, N, false, true>(sm, RowIdx16{p * N}, t, act, sign, tw, rv);
        if (act) {
            typename Elem16<T>::E* o = out + (long)p * stride + t;
#pragma unroll
            for (int m = 0; m < 8; ++m) o[(long)m * TPS] = reg_put(rv, m);
        }
    }
}

// One Stockham pass over two rows per thread: rows at sm and sm + off1 (the
// same padded layout), the arithmetic of stockham_pass16g element for
// element, so the transforms are bit-identical to one row per thread.  The
// two rows share butterfly index k, hence one twiddle set per butterfly, and
// a CTA needs half as many rounds (and barriers) for the same rows.
template <int N, int Ns, int R, bool OUT, typename TW>
__device__ __forceinline__ void stockham_pass16_rows2(float4* __restrict__ sm, int off1, int base, int t, float sign,
                                                      const TW& tw, float2 (&reg)[2][2][8]) {
    using V = float2;
    constexpr int B = 8 / R;
    constexpr int NB = N / R;
    constexpr int TPS = N / 8;
    V v[2][2][8];
#pragma unroll
    for (int q = 0; q < B; ++q) {
        const int b = t + q * TPS;
        const int k = b & (Ns - 1);
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int r = 0; r < R; ++r) {
                V u[2];
                unpack16(sm[s * off1 + pad16(base + b + r * NB)], u);
                v[s][0][q * R + r] = u[0];
                v[s][1][q * R + r] = u[1];
            }
        if (Ns > 1) {
            V w[8];
            tw_fill<V, float, N, Ns, R>(tw, k, sign, w);
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int r = 1; r < R; ++r)
#pragma unroll
                    for (int l = 0; l < 2; ++l) v[s][l][q * R + r] = cmul(v[s][l][q * R + r], w[r]);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if constexpr (R == 8) {
                    bfly8<V, float>(v[s][l], sign);
                } else if constexpr (R == 4) {
                    bfly4<V, float>(v[s][l][q * 4 + 0], v[s][l][q * 4 + 1], v[s][l][q * 4 + 2], v[s][l][q * 4 + 3],
                                    sign);
                } else {
                    bfly2<V, float>(v[s][l][q * 2 + 0], v[s][l][q * 2 + 1]);
                }
            }
    }
    if constexpr (OUT) {
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
            for (int q = 0; q < B; ++q)
#pragma unroll
                for (int r = 0; r < R; ++r)
#pragma unroll
                    for (int l = 0; l < 2; ++l) reg[s][l][q + r * B] = v[s][l][q * R + r];
    } else {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const int b = t + q * TPS;
            const int k = b & (Ns - 1);
            const int base2 = (b / Ns) * Ns * R + k;
#pragma unroll
            for (int s = 0; s < 2; ++s)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const V u[2] = {v[s][0][q * R + r], v[s][1][q * R + r]};
                    sm[s * off1 + pad16(base + base2 + r * Ns)] = pack16(u);
                }
        }
        __syncthreads();
    }
}
template <int N, int Ns, typename TW>
__device__ __forceinline__ void fft16_rows2_passes(float4* sm, int off1, int base, int t, float sign, const TW& tw,
                                                   float2 (&reg)[2][2][8]) {
    if constexpr (Ns < N) {
        constexpr int rem = N / Ns;
        constexpr int R = rem >= 8 ? 8 : rem;
        stockham_pass16_rows2<N, Ns, R, Ns * R == N>(sm, off1, base, t, sign, tw, reg);
        fft16_rows2_passes<N, Ns * R>(sm, off1, base, t, sign, tw, reg);
    }
}
// The 2 spr rows of the padded row buffer (spr = blockDim / (N/8), every thread
// active), thread (r, t) transforming rows r and r + spr in one round, the last
// pass storing row p straight to out + p stride.
template <int N, typename TW>
__device__ __forceinline__ void fft16_rows2_store(float4* sm, float sign, const TW& tw, float4* __restrict__ out,
                                                  long stride) {
    constexpr int TPS = N / 8;
    const int spr = blockDim.x / TPS;
    const int r = threadIdx.x / TPS, t = threadIdx.x % TPS;
    const int off1 = padded_len16(spr * N);
    float2 rv[2][2][8];
    fft16_rows2_passes<N, 1>(sm, off1, r * N, t, sign, tw, rv);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        float4* o = out + (long)(r + s * spr) * stride + t;
#pragma unroll
        for (int m = 0; m < 8; ++m) o[(long)m * TPS] = reg_put(rv[s], m);
    }
}

// ------------------------------------------------------------------ pass 1
// One CTA per lattice row: noise and V xi V^dagger for every site into the 8
// pair rows, then their forward row transforms (up to 512^2; larger rows go to
// k_mix_pass1_pair).
template <int N>
__global__ void __launch_bounds__(mx_p1_threads<N>(), mx_p1_blocks<N>()) k_mix_pass1(const EventDev* __restrict__ ev,
                                                                                     const int* __restrict__ slots,
                                                                                     float4* __restrict__ P,
                                                                                     const float2* __restrict__ tw) {
    static_assert(!mx_pair<N>(), "one CTA holds all 8 pair rows");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sm = reinterpret_cast<float4*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const float* nf = e.nf32;
    for (int y = threadIdx.x; y < N; y += blockDim.x) {
        const long site = (long)x * N + y;
        double2 dv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dv[k] = __ldg(&e.V[k * vol + site]);  // in flight during the noise
        float z[16];
        langevin_normals_fast(e.seed, e.step, (uint32_t)site, z);
        if (nf) {  // NOISE coupling: the site-indexed factor (uniform over the event)
            const float f = nf[site];
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] *= f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (X_j, Y_j)
            sm[pad16(j * N + y)] = make_float4(z[4 * j], z[4 * j + 2], z[4 * j + 1], z[4 * j + 3]);
        float n[8], m[8], hx[8], hy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            n[k] = z[2 * k];
            m[k] = z[2 * k + 1];
        }
        float2 v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = make_float2((float)dv[k].x, (float)dv[k].y);
        rotate_herm(v, n, hx);
        rotate_herm(v, m, hy);
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (BX_j, BY_j)
            sm[pad16((4 + j) * N + y)] = make_float4(hx[2 * j], hx[2 * j + 1], hy[2 * j], hy[2 * j + 1]);
    }
    __syncthreads();
    fft16_rows_store<float, N>(sm, 8, -1.0f, tw, P + (long)b * 8 * vol + (long)x * N, vol);
}

// Pass 1 where the 8 pair rows of a lattice row would leave one CTA per SM or
// do not fit one CTA (N >= 1024): a cluster of two CTAs shares the row through
// distributed shared memory.
// Rank 0 holds the 4 noise rows (X_j, Y_j), rank 1 the 4 rotated rows
// (BX_j, BY_j).  Each CTA draws the noise, loads V and rotates for half the
// sites, and stores both pair elements of a site straight into the rows of
// their owner (local or the partner's shared memory).  One cluster barrier
// (release/acquire) orders those stores before each CTA transforms its rows;
// nothing reads the partner's memory after it, so either CTA may finish first.
template <int N>
__global__ void __cluster_dims__(1, 2, 1) __launch_bounds__(mx_p1_threads<N>(), mx_p1_blocks<N>())
    k_mix_pass1_pair(const EventDev* __restrict__ ev, const int* __restrict__ slots, float4* __restrict__ P,
                     const float2* __restrict__ tw) {
    static_assert(mx_pair<N>(), "two CTAs per lattice row");
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sm = reinterpret_cast<float4*>(smem_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();  // = blockIdx.y
    float4* noise_rows = cluster.map_shared_rank(sm, 0);
    float4* rot_rows = cluster.map_shared_rank(sm, 1);
    const int x = blockIdx.x, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const float* nf = e.nf32;
    constexpr int HALF = N / 2;
    for (int y = (int)rank * HALF + threadIdx.x; y < ((int)rank + 1) * HALF; y += blockDim.x) {
        const long site = (long)x * N + y;
        double2 dv[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) dv[k] = __ldg(&e.V[k * vol + site]);  // in flight during the noise
        float z[16];
        langevin_normals_fast(e.seed, e.step, (uint32_t)site, z);
        if (nf) {  // NOISE coupling: the site-indexed factor (uniform over the event)
            const float f = nf[site];
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] *= f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (X_j, Y_j)
            noise_rows[pad16(j * N + y)] = make_float4(z[4 * j], z[4 * j + 2], z[4 * j + 1], z[4 * j + 3]);
        float n[8], m[8], hx[8], hy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            n[k] = z[2 * k];
            m[k] = z[2 * k + 1];
        }
        float2 v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = make_float2((float)dv[k].x, (float)dv[k].y);
        rotate_herm(v, n, hx);
        rotate_herm(v, m, hy);
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (BX_j, BY_j)
            rot_rows[pad16(j * N + y)] = make_float4(hx[2 * j], hx[2 * j + 1], hy[2 * j], hy[2 * j + 1]);
    }
    cluster.sync();
    fft16_rows_store<float, N>(sm, 4, -1.0f, tw, P + ((long)b * 8 + 4 * rank) * vol + (long)x * N, vol);
}

// ------------------------------------------------------------------ pass 2
// Column transforms of planes j (n_x, packed) and 4 + j (n_y), W = (i K_x) X +
// (i K_y) Y per column element, inverse transform of W.  Thread (cc, r0)
// holds rows r0 + m N/8 of column cc between the transforms (fft16x), so the
// plane-j transform starts from global loads, the kernel product and the
// inverse start from registers and the inverse ends in the store.
template <int N, int C, int S = 0>
__global__ void __launch_bounds__(mx_s2_threads<N, C>(), mx_s2_blocks<N, C>()) k_mix_pass2(EventDev* __restrict__ ev,
                                                                   const int* __restrict__ slots,
                                                                   const float4* __restrict__ P,
                                                                   float4* __restrict__ Q,
                                                                   const float2* __restrict__ tw, int advance) {
    constexpr int TH = mx_s2_threads<N, C>();
    constexpr int PER = N * C / TH;  // = 8
    static_assert(PER == 8, "one radix-8 lane per thread and column");
    constexpr int TL = mx_s2_tile_len<N, C>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* ta = reinterpret_cast<float4*>(smem_raw);
    float4* tb = ta + TL;
    const int c0 = blockIdx.x * C, j = blockIdx.y, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    // the step index advances here: pass 1 of this step has read it, and the
    // next step's noise (pass 1, or pass 3 + 1) reads the new value (advance = 0:
    // a timing launch of the autotuner)
    if (advance && blockIdx.x == 0 && j == 0 && threadIdx.x == 0) ev[slots[b]].step += 1;
    const long vol = (long)N * N;
    const int cc = threadIdx.x % C, r0 = threadIdx.x / C;
    constexpr int RSTEP = TH / C;  // = N / 8
    const ColIdx16P<C> cidx{cc};
    const float4* ina = P + ((long)b * 8 + j) * vol + c0 + (long)r0 * N + cc;
    const float4* inb = P + ((long)b * 8 + 4 + j) * vol + c0 + (long)r0 * N + cc;
#pragma unroll 1
    for (int q = 0; q < PER; ++q) cp_async<16>(&tb[cidx(r0 + q * RSTEP)], inb + (long)q * RSTEP * N);
    cp_async_commit();
    float2 ra[2][8];
#pragma unroll
    for (int q = 0; q < PER; ++q) reg_get(__ldg(ina + (long)q * RSTEP * N), ra, q);
    const float* kt = e.k32 + c0 + (long)r0 * N + cc;
    float kx[PER], ky[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        kx[q] = __ldg(kt + (long)q * RSTEP * N);
        ky[q] = __ldg(kt + vol + (long)q * RSTEP * N);
    }
    // (i kx) X + (i ky) Y, X and Y the two halves of a plane element
    fft16x<float, N, true, true, S>(ta, cidx, r0, true, -1.0f, tw, ra);
    float2 w[2][8];
    const float* kr = e.kre32 ? e.kre32 + c0 + (long)r0 * N + cc : nullptr;
#pragma unroll
    for (int q = 0; q < PER; ++q)
        w[0][q] = make_float2(-kx[q] * ra[0][q].y - ky[q] * ra[1][q].y, kx[q] * ra[0][q].x + ky[q] * ra[1][q].x);
    if (kr) {
#pragma unroll
        for (int q = 0; q < PER; ++q)
            w[0][q] = kmul_re(w[0][q], __ldg(kr + (long)q * RSTEP * N), __ldg(kr + vol + (long)q * RSTEP * N), ra[0][q],
                              ra[1][q]);
    }
    cp_async_wait<0>();
    __syncthreads();
    fft16x<float, N, false, true, S>(tb, cidx, r0, true, -1.0f, tw, ra);
#pragma unroll
    for (int q = 0; q < PER; ++q)
        w[1][q] = make_float2(-kx[q] * ra[0][q].y - ky[q] * ra[1][q].y, kx[q] * ra[0][q].x + ky[q] * ra[1][q].x);
    if (kr) {
#pragma unroll
        for (int q = 0; q < PER; ++q)
            w[1][q] = kmul_re(w[1][q], __ldg(kr + (long)q * RSTEP * N), __ldg(kr + vol + (long)q * RSTEP * N), ra[0][q],
                              ra[1][q]);
    }
    // every thread has passed a barrier since its last read of ta
    fft16x<float, N, true, true, S>(ta, cidx, r0, true, 1.0f, tw, w);
    float4* out = Q + ((long)b * 4 + j) * vol + c0 + (long)r0 * N + cc;
#pragma unroll
    for (int q = 0; q < PER; ++q) out[(long)q * RSTEP * N] = reg_put(w, q);
}

// ------------------------------------------------------------------ pass 2, persistent with TMA
// The same column pass as k_mix_pass2 with 8-column tiles (128-byte tile
// rows, no padding needed; one CTA of 512 threads per SM at 512^2), as a
// persistent kernel: each CTA takes a
// contiguous run of the work items (column tile, event, plane pair j), in
// that order.  The tensor memory accelerator moves every tile: loads of P
// (2D boxes {8 float4 elements, up to 256 rows} of P viewed as
// [8 nb N rows][4 N floats]) complete in bytes on one mbarrier per buffer,
// and the result tile of Q leaves shared memory by a bulk tensor store, so
// the threads issue no global loads or stores on the way.  Three tile
// buffers rotate.  Item k finds X (plane j) in xb, Y (plane 4 + j) in yb,
// and the third buffer fb still being read by item k - 1's store.  It
// transforms X into registers, then (once that store has read fb) starts the
// loads of item k + 1's X into fb and Y into xb, transforms Y, runs the
// inverse transform in yb, writes the result tile into yb and stores it.  Item
// k + 1 then finds (X, Y, store) in (fb, xb, yb).  The twiddles sit in shared
// memory (per-pass table) and the kernel-table values of the thread's elements
// stay in registers while the column tile does not change.  The arithmetic is
// k_mix_pass2's, element for element, so Q is bit-identical.  Built for
// 64 <= N <= 1024: 8-column tiles up to 512^2 (64 KB at 512^2), then 64 KB
// tiles of 4 columns at 1024^2.
template <int N, int C> constexpr int mx_t2_threads() { return C * (N / 8); }
template <int N, int C> constexpr size_t mx_t2_tile_bytes() { return (size_t)16 * C * N; }
template <int N, int C, int S = 0> constexpr size_t mx_t2_smem() {
    return 3 * mx_t2_tile_bytes<N, C>() + 1024 + 8 * (size_t)tw_pass_values<N, S>();
}
// tile width of the persistent form: 8 columns up to 512^2, then 4 at 1024^2
// (64 KB tiles, so that three still fit).  Every tile is the dense [N][C] box
// layout of the tensor map (no swizzle).  4-column rows are 64 bytes, so the
// first pass's stores of rows 8 b + r and 8 (b + 1) + r meet in one bank
// (2-way conflict); measured 1.33 ms per 16 x 1024^2 launch against 1.47 ms
// for the best classic width.  At 2048^2 the 2-column form (4-way conflicts)
// measured 2.68 ms against 1.77 ms classic and is not built.
template <int N> constexpr int mx_t2_cols() { return N <= 512 ? 8 : 4096 / N; }
template <int N, int C> constexpr int mx_t2_blocks() {
    return (int)((227 * 1024) / (mx_t2_smem<N, C>() + 1024)) < 1024 / mx_t2_threads<N, C>()
               ? (int)((227 * 1024) / (mx_t2_smem<N, C>() + 1024))
               : 1024 / mx_t2_threads<N, C>();
}
template <int N, int C> constexpr bool mx_t2_valid() {
    return C == mx_t2_cols<N>() && N >= 64 && N <= 1024 && mx_t2_smem<N, C>() <= 227 * 1024;
}

template <int N, int C, int S = 0, bool RE = false>
__global__ void __launch_bounds__(mx_t2_threads<N, C>(), mx_t2_blocks<N, C>()) k_mix_pass2_tma(
    EventDev* __restrict__ ev, const int* __restrict__ slots, const float2* __restrict__ tw, int nb, int advance,
    int* __restrict__ flags, const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap qmap) {
    static_assert(mx_t2_valid<N, C>(), "three C-column tiles per CTA");
    constexpr int PER = 8;
    constexpr int RSTEP = N / 8;
    constexpr int TILES = N / C;
    constexpr int BOX = N < 256 ? N : 256;
    constexpr unsigned TILE_BYTES = (unsigned)mx_t2_tile_bytes<N, C>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[3];
    // the tiles start on a 1024-byte boundary; the offset is added to the
    // shared array itself (not to an integer copy of its address), so that
    // every tile access compiles to a shared-memory instruction rather than a
    // generic one
    const unsigned align_pad = (1024u - (smem_addr(smem_raw) & 1023u)) & 1023u;
    float4* base = reinterpret_cast<float4*>(smem_raw + align_pad);
    float2* tws = reinterpret_cast<float2*>(base + (size_t)3 * N * C);
    const TwPass<float2, S> twsrc{tws};
    const int tid = threadIdx.x;
    const int cc = tid % C, r0 = tid / C;
    const ColIdx16<C> cidx{cc};  // dense [N][C] tile, the TMA box layout
    const long vol = (long)N * N;
    const int items = nb * 4 * TILES;
    // this CTA's run of items [begin, end): item -> (tile, b, j), tile-major
    // (measured faster than a round-robin over tile-fastest items)
    const int per = items / (int)gridDim.x, extra = items % (int)gridDim.x;
    const int begin = (int)blockIdx.x * per + min((int)blockIdx.x, extra);
    const int end = begin + per + ((int)blockIdx.x < extra ? 1 : 0);
    const int stride = 1;
    if (tid == 0) {
        tma_prefetch_map(&pmap);
        tma_prefetch_map(&qmap);
        for (int i = 0; i < 3; ++i) mbar_init(&bar[i], 1);
        mbar_init_fence();
    }
    tw_pass_fill<float2, N, S>(tws, tw);
    __syncthreads();
    auto buf = [&](int bi) { return base + (size_t)bi * N * C; };
    // plane `half` (0: P[j], 1: P[4 + j]) of work item `it` into buffer bi (thread 0)
    auto issue = [&](int it, int half, int bi) {
        const int tile = it / (nb * 4), r = it - tile * nb * 4, j = r & 3, b = r >> 2;
        const int y0 = (b * 8 + (half ? 4 + j : j)) * N;
        mbar_arrive_expect_tx(&bar[bi], TILE_BYTES);
#pragma unroll
        for (int rr = 0; rr < N; rr += BOX) tma_load_2d(buf(bi) + (size_t)rr * C, &pmap, tile * C * 4, y0 + rr, &bar[bi]);
    };
    unsigned parity = 0;     // bit i: the parity buffer i's next completed phase has
    unsigned pending = 0;    // bit i: a load into buffer i is in flight (same value in every thread)
    int xb = 0, yb = 1, fb = 2;
    if (begin < end) {
        if (tid == 0) {
            issue(begin, 0, xb);
            issue(begin, 1, yb);
        }
        pending = (1u << xb) | (1u << yb);
    }
    bool timed_out = false;
    int cur_tile = -1;
    const float* cur_tab = nullptr;
    auto item_tab = [&](int i2) {
        const int t2 = i2 / (nb * 4);
        return ev[slots[(i2 - t2 * nb * 4) >> 2]].k32;
    };
    const float* tab_next = begin < end ? item_tab(begin) : nullptr;
    float kx[PER], ky[PER];
#pragma unroll 1
    for (int it = begin; it < end; it += stride) {
        const bool more = it + stride < end;
        const int tile = it / (nb * 4), rj = it - tile * nb * 4, j = rj & 3, b = rj >> 2;
        const int c0 = tile * C;
        if (advance && tile == 0 && j == 0 && tid == 0) ev[slots[b]].step += 1;
        // kernel-table values of this thread's elements, kept while the tile and
        // the table stay the same (events of one size and coupling share a table;
        // position-space events have their own).  The next item's table pointer
        // is loaded here, an item ahead of its use.
        const float* tab = tab_next;
        if (more) tab_next = item_tab(it + stride);
        if (tile != cur_tile || tab != cur_tab) {
            const float* kt = tab + c0 + (long)r0 * N + cc;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                kx[q] = __ldg(kt + (long)q * RSTEP * N);
                ky[q] = __ldg(kt + vol + (long)q * RSTEP * N);
            }
            cur_tile = tile;
            cur_tab = tab;
        }
        const float* kr0 = RE ? ev[slots[b]].kre32 : nullptr;  // real table parts (RE launches only)
        const float* kr = kr0 ? kr0 + c0 + (long)r0 * N + cc : nullptr;
        float2 ra[2][8], w[2][8];
        timed_out |= !mbar_wait_bounded(&bar[xb], (parity >> xb) & 1u);
        parity ^= 1u << xb;
        pending &= ~(1u << xb);
        fft16x<float, N, false, true, S>(buf(xb), cidx, r0, true, -1.0f, twsrc, ra);
#pragma unroll
        for (int q = 0; q < PER; ++q)
            w[0][q] = make_float2(-kx[q] * ra[0][q].y - ky[q] * ra[1][q].y, kx[q] * ra[0][q].x + ky[q] * ra[1][q].x);
        if (kr) {
#pragma unroll
            for (int q = 0; q < PER; ++q)
                w[0][q] = kmul_re(w[0][q], __ldg(kr + (long)q * RSTEP * N), __ldg(kr + vol + (long)q * RSTEP * N),
                                  ra[0][q], ra[1][q]);
        }
        // every thread is done reading xb; once the previous item's store has
        // read fb, the next item's X goes to fb and its Y to xb (issuing X at
        // the item's start, waiting for that store there, measured slower)
        if (__syncthreads_or(timed_out)) break;
        if (more) {
            if (tid == 0) {
                tma_store_wait_read<0>();
                fence_proxy_async_smem();
                issue(it + stride, 0, fb);
                issue(it + stride, 1, xb);
            }
            pending |= (1u << fb) | (1u << xb);
        }
        timed_out |= !mbar_wait_bounded(&bar[yb], (parity >> yb) & 1u);
        parity ^= 1u << yb;
        pending &= ~(1u << yb);
        fft16x<float, N, false, true, S>(buf(yb), cidx, r0, true, -1.0f, twsrc, ra);
#pragma unroll
        for (int q = 0; q < PER; ++q)
            w[1][q] = make_float2(-kx[q] * ra[0][q].y - ky[q] * ra[1][q].y, kx[q] * ra[0][q].x + ky[q] * ra[1][q].x);
        if (kr) {
#pragma unroll
            for (int q = 0; q < PER; ++q)
                w[1][q] = kmul_re(w[1][q], __ldg(kr + (long)q * RSTEP * N), __ldg(kr + vol + (long)q * RSTEP * N),
                                  ra[0][q], ra[1][q]);
        }
        // the inverse's first pass synchronises before it writes yb
        fft16x<float, N, true, true, S>(buf(yb), cidx, r0, true, 1.0f, twsrc, w);
        // the result tile into yb (dense [N][8] elements, the store box's layout)
        __syncthreads();
        float4* ot = buf(yb);
#pragma unroll
        for (int q = 0; q < PER; ++q) ot[cidx(r0 + q * RSTEP)] = reg_put(w, q);
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            const int y0 = (b * 4 + j) * N;
#pragma unroll
            for (int rr = 0; rr < N; rr += BOX) tma_store_2d(&qmap, c0 * 4, y0 + rr, ot + (size_t)rr * C);
            tma_store_commit();
        }
        const int nx = fb, ny = xb, nf = yb;
        xb = nx;
        yb = ny;
        fb = nf;
    }
    if (tid == 0) tma_store_wait<0>();  // the last stores have completed before the CTA exits
    if (timed_out) {
        if (tid == 0) atomicOr(flags, JW_FLAG_TIMEOUT);
        // loads still in flight land in this CTA's shared memory: wait for them
        // (bounded) before the CTA exits
        for (int i = 0; i < 3; ++i)
            if ((pending >> i) & 1u) mbar_wait_bounded(&bar[i], (parity >> i) & 1u);
    }
}

// ------------------------------------------------------------------ pass 3
// The update of site y: V <- exp(+i sqrt(eps) B) V exp(-i sqrt(eps) A), A and B
// from the inverse row transforms in column y of the row buffer.  The old V is
// loaded first and arrives while exp(+i sqrt(eps) B) is formed; one
// exponential is held at a time.  Reports non-finite entries in fl.
// get_u(j) returns the element of inverse-transformed pair row j at the site.
// get_v(k) returns entry k of the site's old V (by default loaded from e.V).
template <bool CHECK = true, typename GetU, typename GetV>
__device__ __forceinline__ void p3_site_gv(const EventDev& e, GetU get_u, GetV get_v, double se, double2 (&v)[9],
                                           int& fl) {
    double2 v0[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) v0[k] = get_v(k);
    double bq[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float4 u = get_u(j);
        bq[2 * j] = __dmul_rn((double)u.z, -se);
        bq[2 * j + 1] = __dmul_rn((double)u.w, -se);
    }
    // the explicitly rounded forms (xr): passes 3 and 3 + 1 give the same bits
    double2 m[9], tmp[9];
    embed_lambda_x(bq, m);
    xr::expi_ch(m, -1.0);  // exp(+i sqrt(eps) B)
    xr::mul3(m, v0, tmp);
    // A's coefficients are read again here rather than held through the first
    // exponential (fewer live registers there)
    double a[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float4 u = get_u(j);
        a[2 * j] = __dmul_rn((double)u.x, se);
        a[2 * j + 1] = __dmul_rn((double)u.y, se);
    }
    embed_lambda_x(a, m);
    xr::expi_ch(m, -1.0);  // exp(-i sqrt(eps) A)
    xr::mul3(tmp, m, v);
    if (e.reunit) xr::reunitarize(v);
    if constexpr (CHECK) {
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (!isfinite(v[k].x) || !isfinite(v[k].y)) fl |= JW_FLAG_NAN;
    }
}

template <typename GetU>
__device__ __forceinline__ void p3_site_g(const EventDev& e, GetU get_u, long site, long vol, double se,
                                          double2 (&v)[9], int& fl) {
    p3_site_gv(e, get_u, [&](int k) { return e.V[k * vol + site]; }, se, v, fl);
}

template <int N>
__device__ __forceinline__ void p3_site(const EventDev& e, const float4* sm, int y, long site, long vol, double se,
                                        double2 (&v)[9], int& fl) {
    p3_site_g(e, [&](int j) { return sm[pad16(j * N + y)]; }, site, vol, se, v, fl);
}

// The old V of the sites a thread updates in a row pass, copied ahead into
// shared memory with cp.async: slot vs[k * TH + tid] holds entry k of site
// tid + i TH.  start() copies the first site (the caller commits it as the
// last group before the row's transform input is awaited with
// cp_async_wait<1>); take() waits for the current site, reads it and starts
// the copy of the thread's next site into the same slots.  Passes 3 and 3 + 1
// both read V this way, so that their updates compile to the same arithmetic.
template <int N, int TH>
struct VAhead {
    double2* vs;
    const double2* __restrict__ vrow;  // row x of the event's V
    long vol;
    int tid;
    __device__ __forceinline__ void start() const {
        if (tid < N) {
#pragma unroll
            for (int k = 0; k < 9; ++k) cp_async<16>(&vs[k * TH + tid], &vrow[k * vol + tid]);
        }
        cp_async_commit();
    }
    __device__ __forceinline__ void take(int y, double2 (&vold)[9]) const {
        cp_async_wait<0>();
#pragma unroll
        for (int k = 0; k < 9; ++k) vold[k] = vs[k * TH + tid];
        if (y + TH < N) {
#pragma unroll
            for (int k = 0; k < 9; ++k) cp_async<16>(&vs[k * TH + tid], &vrow[k * vol + y + TH]);
            cp_async_commit();
        }
    }
};
// the V slots of the one-CTA row passes (up to 512^2): [9][threads] double2
template <int N> constexpr size_t v_ahead_bytes(int threads) { return mx_pair<N>() ? 0 : (size_t)9 * 16 * threads; }

template <int N, bool MEAS = false>
__global__ void __launch_bounds__(mx_p3_threads<N>(), mx_p3_blocks<N, MEAS>()) k_mix_pass3(EventDev* __restrict__ ev,
                                                                                         const int* __restrict__ slots,
                                                                                         const float4* __restrict__ Q,
                                                                                         const float2* __restrict__ tw,
                                                                                         int* __restrict__ flags,
                                                                                         float4* __restrict__ M) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sm = reinterpret_cast<float4*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.y;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    constexpr int TH = mx_p3_threads<N>();
    constexpr bool AHEAD = !mx_pair<N>();  // one-CTA sizes copy V ahead, like pass 3 + 1
    const float4* in = Q + (long)b * 4 * vol + (long)x * N;
    const VAhead<N, TH> va{reinterpret_cast<double2*>(sm + padded_len16((MEAS ? 5 : 4) * N)), e.V + (long)x * N, vol,
                           (int)threadIdx.x};
    for (int i = threadIdx.x; i < 4 * N; i += blockDim.x)
        cp_async<16>(&sm[pad16(i)], &in[(long)(i / N) * vol + (i % N)]);
    cp_async_commit();
    if constexpr (AHEAD) va.start();
    else cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    fft16_rows<N, 4>(sm, 1.0f, tw);
    const double se = e.sqrt_eps;
    int fl = 0;
    for (int y = threadIdx.x; y < N; y += blockDim.x) {
        const long site = (long)x * N + y;
        double2 v[9];
        if constexpr (AHEAD) {
            double2 vold[9];
            va.take(y, vold);
            p3_site_gv(e, [&](int j) { return sm[pad16(j * N + y)]; }, [&](int k) { return vold[k]; }, se, v, fl);
        } else {
            p3_site<N>(e, sm, y, site, vol, se, v, fl);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) e.V[k * vol + site] = v[k];
        if constexpr (MEAS) {
            // entries 2p, 2p + 1 of the new V as pair element (p, y); this
            // thread alone has read or written column y of the row buffer
#pragma unroll
            for (int p = 0; p < 5; ++p) {
                const double2 hi = p < 4 ? v[2 * p + 1] : make_double2(0.0, 0.0);
                sm[pad16(p * N + y)] = make_float4((float)v[2 * p].x, (float)v[2 * p].y, (float)hi.x, (float)hi.y);
            }
        }
    }
    if (fl) atomicOr(flags, fl);
    if constexpr (MEAS) {
        __syncthreads();
        fft16_rows_store<float, N>(sm, 5, -1.0f, tw, M + (long)b * 5 * vol + (long)x * N, vol);
    }
}

// ------------------------------------------------------------------ pass 3 + next pass 1
// The end of one step and the start of the next for lattice row x, in one
// kernel: the inverse row transforms of Q and the V update (pass 3), then, with
// the new V still in registers, the next step's noise, V xi V^dagger and their
// forward row transforms (pass 1).  This saves the V re-read of pass 1 and lets
// pass 3's memory traffic overlap pass 1's arithmetic.  The new pair rows of
// site y overwrite column y of the inverse transforms, which the same thread
// has just consumed, so the row buffer is pass 1's (8 rows).  Pass 2 has
// advanced the step index, so e.step is the next step's noise index.
template <int N> constexpr int mx_p31_threads() { return mx_p1_threads<N>(); }
// 8 pair rows, then the old V of one site per thread ([9][threads] double2),
// copied ahead with cp.async, then the per-pass twiddle table (TwRows)
template <int N> constexpr size_t mx_p31_tw_offset() { return mx_p1_smem<N>() + v_ahead_bytes<N>(mx_p31_threads<N>()); }
template <int N> constexpr size_t mx_p31_smem() { return mx_p31_tw_offset<N>() + 64 * (size_t)tw_pass_entries<N>(); }
// the cluster form (mx_pair): 2 inverse-transformed Q rows and 4 output rows per CTA
template <int N> constexpr size_t mx_p31p_smem() {
    return 16 * ((size_t)padded_len16(2 * N) + (size_t)padded_len16(4 * N));
}
template <int N> constexpr int mx_p31p_blocks() {
    return mx_p31_threads<N>() <= 256 && mx_p31p_smem<N>() <= 113 * 1024 ? 2 : 1;
}

template <int N>
__global__ void __launch_bounds__(mx_p31_threads<N>(), mx_p1_blocks<N>()) k_mix_pass31(
    EventDev* __restrict__ ev, const int* __restrict__ slots, const float4* __restrict__ Q, float4* __restrict__ P,
    const float2* __restrict__ tw, int* __restrict__ flags) {
    static_assert(!mx_pair<N>(), "one CTA holds all 8 pair rows");
    static_assert(mx_p1_blocks<N>() < 2 || mx_p31_smem<N>() <= 113 * 1024, "two CTAs per SM");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sm = reinterpret_cast<float4*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.y;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    constexpr int TH = mx_p31_threads<N>();
    const int tid = threadIdx.x;
    const float4* in = Q + (long)b * 4 * vol + (long)x * N;
    // the old V of this thread's sites, copied ahead: the first site while the
    // inverse transforms run, the next one while this one is updated
    const VAhead<N, TH> va{reinterpret_cast<double2*>(sm + padded_len16(8 * N)), e.V + (long)x * N, vol, tid};
    for (int i = tid; i < 4 * N; i += TH) cp_async<16>(&sm[pad16(i)], &in[(long)(i / N) * vol + (i % N)]);
    cp_async_commit();
    va.start();
    // the per-pass twiddle table (bit-identical to the run-time derivation
    // from tw), filled while the copies are in flight: the transforms then
    // read their twiddles from shared memory and form none of them
    float2* tws = reinterpret_cast<float2*>(smem_raw + mx_p31_tw_offset<N>());
    tw_rows_fill<float2, N>(tws, tw);
    const TwRows<float2> twsrc{tws};
    cp_async_wait<1>();  // Q has landed (V may still be in flight)
    __syncthreads();
    fft16_rows<N, 4>(sm, 1.0f, twsrc);
    const double se = e.sqrt_eps;
    const float* nf = e.nf32;
    int fl = 0;
    for (int y = tid; y < N; y += TH) {
        const long site = (long)x * N + y;
        float2 v32[9];
        {
            double2 vold[9];
            va.take(y, vold);
            double2 v[9];
            p3_site_gv<false>(e, [&](int j) { return sm[pad16(j * N + y)]; }, [&](int k) { return vold[k]; }, se, v,
                              fl);
            float fin = 0.0f;  // non-finite iff an entry of the new V is (or exceeds the FP32 range)
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                e.V[k * vol + site] = v[k];
                v32[k] = make_float2((float)v[k].x, (float)v[k].y);
                fin += v32[k].x + v32[k].y;
            }
            if (!isfinite(fin)) fl |= JW_FLAG_NAN;
        }
        float z[16];
        langevin_normals_fast(e.seed, e.step, (uint32_t)site, z);
        if (nf) {  // NOISE coupling: the site-indexed factor (uniform over the event)
            const float f = nf[site];
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] *= f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (X_j, Y_j)
            sm[pad16(j * N + y)] = make_float4(z[4 * j], z[4 * j + 2], z[4 * j + 1], z[4 * j + 3]);
        float n[8], m[8], hx[8], hy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            n[k] = z[2 * k];
            m[k] = z[2 * k + 1];
        }
        rotate_herm(v32, n, hx);
        rotate_herm(v32, m, hy);
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (BX_j, BY_j)
            sm[pad16((4 + j) * N + y)] = make_float4(hx[2 * j], hx[2 * j + 1], hy[2 * j], hy[2 * j + 1]);
    }
    if (fl) atomicOr(flags, fl);
    __syncthreads();
    if constexpr (TH == 4 * (N / 8))  // 8 rows, 4 per round: two rows per thread in one round
        fft16_rows2_store<N>(sm, -1.0f, twsrc, P + (long)b * 8 * vol + (long)x * N, vol);
    else
        fft16_rows_store<float, N>(sm, 8, -1.0f, twsrc, P + (long)b * 8 * vol + (long)x * N, vol);
}

// Pass 3 + next pass 1 where a lattice row needs a cluster of two CTAs
// (mx_pair).  Rank r inverse-transforms Q rows 2r, 2r + 1 in its own shared
// memory; after a cluster barrier each CTA updates half the row's sites,
// reading the two other Q rows from its partner, and stores the next step's
// noise pairs into rank 0's output rows and the rotated pairs into rank 1's.
// A second barrier orders those stores before each CTA transforms its 4
// output rows.  Nothing touches the partner's memory after it.
template <int N>
__global__ void __cluster_dims__(1, 2, 1) __launch_bounds__(mx_p31_threads<N>(), mx_p31p_blocks<N>())
    k_mix_pass31_pair(EventDev* __restrict__ ev, const int* __restrict__ slots, const float4* __restrict__ Q,
                      float4* __restrict__ P, const float2* __restrict__ tw, int* __restrict__ flags) {
    static_assert(mx_pair<N>(), "two CTAs per lattice row");
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* qb = reinterpret_cast<float4*>(smem_raw);  // this CTA's 2 Q rows
    float4* ob = qb + padded_len16(2 * N);               // this CTA's 4 output rows
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();  // = blockIdx.y
    const float4* q_lo = cluster.map_shared_rank(qb, 0);  // Q rows 0, 1
    const float4* q_hi = cluster.map_shared_rank(qb, 1);  // Q rows 2, 3
    float4* noise_rows = cluster.map_shared_rank(ob, 0);
    float4* rot_rows = cluster.map_shared_rank(ob, 1);
    const int x = blockIdx.x, b = blockIdx.z;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    constexpr int HALF = N / 2, TH = mx_p31_threads<N>();
    static_assert(TH <= HALF && 9 * TH <= padded_len16(4 * N), "first-site V stage fits the output rows");
    const float4* in = Q + ((long)b * 4 + 2 * rank) * vol + (long)x * N;
    for (int i = threadIdx.x; i < 2 * N; i += blockDim.x)
        cp_async<16>(&qb[pad16(i)], &in[(long)(i / N) * vol + (i % N)]);
    cp_async_commit();
    // the old V of this thread's first site, staged in the output rows (unused
    // until the cluster barrier) while the Q rows transform
    const int y0 = (int)rank * HALF + threadIdx.x;
    double2* vstage = reinterpret_cast<double2*>(ob);
#pragma unroll
    for (int k = 0; k < 9; ++k) cp_async<16>(&vstage[k * TH + threadIdx.x], &e.V[k * vol + (long)x * N + y0]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    fft16_rows<N, 2>(qb, 1.0f, tw);
    cp_async_wait<0>();
    double2 vfirst[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) vfirst[k] = vstage[k * TH + threadIdx.x];
    // the partner writes into this CTA's output rows only after this barrier
    cluster.sync();
    const double se = e.sqrt_eps;
    const float* nf = e.nf32;
    int fl = 0;
    // one site: the update from get_v's old V, then the next step's noise and rotation
    auto site_step = [&](int y, auto get_v) {
        const long site = (long)x * N + y;
        float2 v32[9];
        {
            double2 v[9];
            p3_site_gv(e, [&](int j) { return j < 2 ? q_lo[pad16(j * N + y)] : q_hi[pad16((j - 2) * N + y)]; },
                       get_v, se, v, fl);
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                e.V[k * vol + site] = v[k];
                v32[k] = make_float2((float)v[k].x, (float)v[k].y);
            }
        }
        float z[16];
        langevin_normals_fast(e.seed, e.step, (uint32_t)site, z);
        if (nf) {  // NOISE coupling: the site-indexed factor (uniform over the event)
            const float f = nf[site];
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] *= f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (X_j, Y_j)
            noise_rows[pad16(j * N + y)] = make_float4(z[4 * j], z[4 * j + 2], z[4 * j + 1], z[4 * j + 3]);
        float n[8], m[8], hx[8], hy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            n[k] = z[2 * k];
            m[k] = z[2 * k + 1];
        }
        rotate_herm(v32, n, hx);
        rotate_herm(v32, m, hy);
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (BX_j, BY_j)
            rot_rows[pad16(j * N + y)] = make_float4(hx[2 * j], hx[2 * j + 1], hy[2 * j], hy[2 * j + 1]);
    };
    site_step(y0, [&](int k) { return vfirst[k]; });
#pragma unroll 1
    for (int y = y0 + TH; y < ((int)rank + 1) * HALF; y += TH)
        site_step(y, [&](int k) { return e.V[k * vol + (long)x * N + y]; });
    if (fl) atomicOr(flags, fl);
    cluster.sync();
    if constexpr (mx_p31_threads<N>() == 2 * (N / 8))  // 4 rows, 2 per round: two rows per thread in one round
        fft16_rows2_store<N>(ob, -1.0f, tw, P + ((long)b * 8 + 4 * rank) * vol + (long)x * N, vol);
    else
        fft16_rows_store<float, N>(ob, 4, -1.0f, tw, P + ((long)b * 8 + 4 * rank) * vol + (long)x * N, vol);
}

// Pass 3 + next pass 1 at 2048^2 as a cluster of four CTAs of 256 threads (two
// CTAs per SM, the configuration of the two-CTA form at 1024^2).  Rank r
// inverse-transforms Q row r; after a cluster barrier it updates the sites
// [r N/4, (r + 1) N/4), reading the four Q rows from their owners, and stores
// the next step's pair elements into their owners' rows: pair row p (noise
// rows 0-3, rotated rows 4-7) belongs to rank p / 2 as its local row p % 2.
// A second barrier orders those stores before each CTA transforms its 2
// output rows.  The per-site arithmetic is the two-CTA form's, so lattices are
// bit-identical.
constexpr int kQuadThreads = 256;
template <int N> constexpr size_t mx_p31q_smem() {
    return 16 * ((size_t)padded_len16(N) + (size_t)padded_len16(2 * N));
}
template <int N>
__global__ void __cluster_dims__(1, 4, 1) __launch_bounds__(kQuadThreads, 2)
    k_mix_pass31_quad(EventDev* __restrict__ ev, const int* __restrict__ slots, const float4* __restrict__ Q,
                      float4* __restrict__ P, const float2* __restrict__ tw, int* __restrict__ flags) {
    static_assert(N / 8 == kQuadThreads, "one row transform per CTA round");
    static_assert(mx_p31q_smem<N>() <= 113 * 1024, "two CTAs per SM");
    namespace cg = cooperative_groups;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* qb = reinterpret_cast<float4*>(smem_raw);  // Q row `rank`
    float4* ob = qb + padded_len16(N);                   // pair rows 2 rank, 2 rank + 1
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned rank = cluster.block_rank();  // = blockIdx.y
    const int x = blockIdx.x, b = blockIdx.z;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    constexpr int QUARTER = N / 4, TH = kQuadThreads;
    static_assert(TH <= QUARTER && 9 * TH <= padded_len16(2 * N), "first-site V stage fits the output rows");
    const float4* in = Q + ((long)b * 4 + rank) * vol + (long)x * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) cp_async<16>(&qb[pad16(i)], &in[i]);
    cp_async_commit();
    // the old V of this thread's first site, staged in the output rows (unused
    // until the cluster barrier) while the Q row transforms
    const int y0 = (int)rank * QUARTER + threadIdx.x;
    double2* vstage = reinterpret_cast<double2*>(ob);
#pragma unroll
    for (int k = 0; k < 9; ++k) cp_async<16>(&vstage[k * TH + threadIdx.x], &e.V[k * vol + (long)x * N + y0]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    fft16_rows<N, 1>(qb, 1.0f, tw);
    cp_async_wait<0>();
    double2 vfirst[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) vfirst[k] = vstage[k * TH + threadIdx.x];
    // the other ranks write into this CTA's output rows only after this barrier
    cluster.sync();
    const double se = e.sqrt_eps;
    const float* nf = e.nf32;
    int fl = 0;
    // element y of pair row p (0..7) in its owner's shared memory
    auto orow = [&](int p, int y) -> float4* { return cluster.map_shared_rank(ob, p >> 1) + pad16((p & 1) * N + y); };
    // one site: the update from get_v's old V, then the next step's noise and rotation
    auto site_step = [&](int y, auto get_v) {
        const long site = (long)x * N + y;
        float2 v32[9];
        {
            double2 v[9];
            p3_site_gv(e, [&](int j) { return *(cluster.map_shared_rank(qb, j) + pad16(y)); }, get_v, se, v, fl);
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                e.V[k * vol + site] = v[k];
                v32[k] = make_float2((float)v[k].x, (float)v[k].y);
            }
        }
        float z[16];
        langevin_normals_fast(e.seed, e.step, (uint32_t)site, z);
        if (nf) {  // NOISE coupling: the site-indexed factor (uniform over the event)
            const float f = nf[site];
#pragma unroll
            for (int k = 0; k < 16; ++k) z[k] *= f;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (X_j, Y_j)
            *orow(j, y) = make_float4(z[4 * j], z[4 * j + 2], z[4 * j + 1], z[4 * j + 3]);
        float n[8], m[8], hx[8], hy[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            n[k] = z[2 * k];
            m[k] = z[2 * k + 1];
        }
        rotate_herm(v32, n, hx);
        rotate_herm(v32, m, hy);
#pragma unroll
        for (int j = 0; j < 4; ++j)  // (BX_j, BY_j)
            *orow(4 + j, y) = make_float4(hx[2 * j], hx[2 * j + 1], hy[2 * j], hy[2 * j + 1]);
    };
    site_step(y0, [&](int k) { return vfirst[k]; });
#pragma unroll 1
    for (int y = y0 + TH; y < ((int)rank + 1) * QUARTER; y += TH)
        site_step(y, [&](int k) { return e.V[k * vol + (long)x * N + y]; });
    if (fl) atomicOr(flags, fl);
    cluster.sync();
    fft16_rows2_store<N>(ob, -1.0f, tw, P + ((long)b * 8 + 2 * rank) * vol + (long)x * N, vol);
}

// ------------------------------------------------------------------ measurement (FP64)
// C(k) = sum over the 9 entries of |FFT(V_ij)(k)|^2 / N^6 (lfield::trace,
// field.h:1375-1432, after the unitary forward transform), with the 16-byte
// element core on double2: a row pass writes the 9 row-transformed planes to
// the workspace M, a column pass transforms them and accumulates the trace.

// rows: 4096-element tiles (8 rows at N = 512) of the event's 9N contiguous
// rows, staged with cp.async
template <int N> constexpr int meas_rows16() { return N >= 4096 ? 1 : 4096 / N; }
template <int N> constexpr size_t meas_rows16_smem() { return 16 * (size_t)padded_len16(meas_rows16<N>() * N); }

template <int N>
__global__ void __launch_bounds__(256) k_meas_rows(const EventDev* __restrict__ ev, const int* __restrict__ slots,
                                                   double2* __restrict__ M, const double2* __restrict__ tw) {
    constexpr int RW = meas_rows16<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int b = blockIdx.y;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const long row0 = (long)blockIdx.x * RW;
    const int nr = (int)min((long)RW, 9L * N - row0);
    const double2* in = e.V + row0 * N;
    for (int i = threadIdx.x; i < nr * N; i += blockDim.x) cp_async<16>(&sm[pad16(i)], &in[i]);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    fft16_rows_store<double, N>(sm, nr, -1.0, tw, M + (long)b * 9 * vol + row0 * N, N);
}

// columns: tiles of C columns, the 9 components double-buffered with cp.async
template <int N> constexpr int meas_cols_threads() { return mx_cols<N>() * (N / 8); }
template <int N> constexpr size_t meas_cols_smem() { return 2 * 16 * (size_t)mx_tile_len<N>(); }

template <int N>
__global__ void __launch_bounds__(meas_cols_threads<N>()) k_meas_cols(const int* __restrict__ slots,
                                                                       const double2* __restrict__ M,
                                                                       double* __restrict__ corr,
                                                                       double* __restrict__ corrT,
                                                                       const double2* __restrict__ tw) {
    constexpr int C = mx_cols<N>();
    constexpr int TH = meas_cols_threads<N>();
    constexpr int PER = N * C / TH;  // = 8
    constexpr int RSTEP = TH / C;    // = N / 8
    constexpr int TL = mx_tile_len<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tile[2] = {reinterpret_cast<double2*>(smem_raw), reinterpret_cast<double2*>(smem_raw) + TL};
    const int c0 = blockIdx.x * C, b = blockIdx.y;
    const long vol = (long)N * N;
    const int cc = threadIdx.x % C, r0 = threadIdx.x / C;
    const ColIdx16P<C> cidx{cc};
    auto stage = [&](int comp, double2* t) {
        const double2* in = M + ((long)b * 9 + comp) * vol + c0 + (long)r0 * N + cc;
#pragma unroll
        for (int q = 0; q < PER; ++q) cp_async<16>(&t[cidx(r0 + q * RSTEP)], in + (long)q * RSTEP * N);
        cp_async_commit();
    };
    double acc[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) acc[q] = 0.0;
    stage(0, tile[0]);
#pragma unroll 1
    for (int comp = 0; comp < 9; ++comp) {
        if (comp + 1 < 9) {
            stage(comp + 1, tile[(comp + 1) & 1]);  // the buffer read at comp - 1
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        double2 rv[1][8];
        fft16x<double, N, false, true>(tile[comp & 1], cidx, r0, true, -1.0, tw, rv);
#pragma unroll
        for (int q = 0; q < PER; ++q) acc[q] += rv[0][q].x * rv[0][q].x + rv[0][q].y * rv[0][q].y;
        __syncthreads();
    }
    const double n2 = (double)N * (double)N;
    const double inv = 1.0 / (n2 * n2 * n2);
    double* out = corr + (long)b * vol + c0 + cc;
    double* outT = corrT + (long)b * vol + (long)(c0 + cc) * N + r0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        out[(long)(r0 + q * RSTEP) * N] = acc[q] * inv;
        outT[q * RSTEP] = acc[q] * inv;
    }
    (void)slots;
}

// ---- measurement, mixed precision: the 9 entries of V as 5 FP32 pair planes
// (V_0, V_1), (V_2, V_3), (V_4, V_5), (V_6, V_7), (V_8, 0), transformed like
// the step's pair planes; |.|^2 is summed in FP64.  Workspace: 80 B/site.
template <int N> constexpr int meas32_rows_threads() {
    return (N >= 64 && 5 * (N / 8) <= 1024) ? 5 * (N / 8) : 256;
}
template <int N> constexpr size_t meas32_rows_smem() { return 16 * (size_t)padded_len16(5 * N); }

template <int N>
__global__ void __launch_bounds__(meas32_rows_threads<N>(), N <= 512 ? 2 : 1) k_meas32_rows(const EventDev* __restrict__ ev,
                                                                          const int* __restrict__ slots,
                                                                          float4* __restrict__ M,
                                                                          const float2* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* sm = reinterpret_cast<float4*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.y;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const double2* V = e.V + (long)x * N;
    // the row's 9 N entries in batches of 4 independent loads per thread;
    // entry (k, y) goes to half (k & 1) of pair element (k >> 1, y)
    constexpr int TH = meas32_rows_threads<N>();
    constexpr int B = 4;
    for (int base = 0; base < 9 * N; base += TH * B) {
        double2 v[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int i = base + threadIdx.x + u * TH;
            if (i < 9 * N) v[u] = V[(long)(i / N) * vol + (i % N)];
        }
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int i = base + threadIdx.x + u * TH;
            if (i < 9 * N) {
                const int k = i / N, y = i - k * N;
                reinterpret_cast<float2*>(&sm[pad16((k >> 1) * N + y)])[k & 1] =
                    make_float2((float)v[u].x, (float)v[u].y);
            }
        }
    }
    for (int y = threadIdx.x; y < N; y += TH)
        reinterpret_cast<float2*>(&sm[pad16(4 * N + y)])[1] = make_float2(0.0f, 0.0f);
    __syncthreads();
    fft16_rows_store<float, N>(sm, 5, -1.0f, tw, M + (long)b * 5 * vol + (long)x * N, vol);
}

template <int N>
__global__ void __launch_bounds__(mx_p2_threads<N>(), mx_p2_threads<N>() <= 256 ? 3 : 1) k_meas32_cols(const float4* __restrict__ M,
                                                                    double* __restrict__ corr,
                                                                    double* __restrict__ corrT,
                                                                    const float2* __restrict__ tw) {
    constexpr int C = mx_cols<N>();
    constexpr int TH = mx_p2_threads<N>();
    constexpr int PER = N * C / TH;  // = 8
    constexpr int RSTEP = TH / C;    // = N / 8
    constexpr int TL = mx_tile_len<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* tile[2] = {reinterpret_cast<float4*>(smem_raw), reinterpret_cast<float4*>(smem_raw) + TL};
    const int c0 = blockIdx.x * C, b = blockIdx.y;
    const long vol = (long)N * N;
    const int cc = threadIdx.x % C, r0 = threadIdx.x / C;
    const ColIdx16P<C> cidx{cc};
    auto stage = [&](int p, float4* t) {
        const float4* in = M + ((long)b * 5 + p) * vol + c0 + (long)r0 * N + cc;
#pragma unroll
        for (int q = 0; q < PER; ++q) cp_async<16>(&t[cidx(r0 + q * RSTEP)], in + (long)q * RSTEP * N);
        cp_async_commit();
    };
    double acc[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) acc[q] = 0.0;
    stage(0, tile[0]);
#pragma unroll 1
    for (int p = 0; p < 5; ++p) {
        if (p + 1 < 5) {
            stage(p + 1, tile[(p + 1) & 1]);  // the buffer read at p - 1
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        float2 rv[2][8];
        fft16x<float, N, false, true>(tile[p & 1], cidx, r0, true, -1.0f, tw, rv);
#pragma unroll
        for (int q = 0; q < PER; ++q)
            acc[q] += ((double)rv[0][q].x * rv[0][q].x + (double)rv[0][q].y * rv[0][q].y) +
                      ((double)rv[1][q].x * rv[1][q].x + (double)rv[1][q].y * rv[1][q].y);
        __syncthreads();
    }
    const double n2 = (double)N * (double)N;
    const double inv = 1.0 / (n2 * n2 * n2);
    double* out = corr + (long)b * vol + c0 + cc;
    double* outT = corrT + (long)b * vol + (long)(c0 + cc) * N + r0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        out[(long)(r0 + q * RSTEP) * N] = acc[q] * inv;
        outT[q * RSTEP] = acc[q] * inv;
    }
}

// ---- MV slice (setMVModel / solvePoisson / operator*=, field.h:683-757,
// 867-877, 337-365) in FP64 on the 16-byte-element core: the 8 charge
// coefficients of a site as 4 complex planes (r0 + i r1, ..., r6 + i r7); row
// transform, column transform x Poisson factor x inverse column transform,
// inverse row transform, V <- V exp(+i f).  The Poisson factor
// -g/(-phat2 + m^2) is -g/m^2 at k = 0 (2500 for m a = 0.02): FP32 transforms
// would put its rounding into V, so the slices stay FP64 in both precisions.
template <int N> constexpr int mv16_threads() {
    return 4 * (N / 8) < 64 ? 64 : (4 * (N / 8) > 256 ? 256 : 4 * (N / 8));
}
template <int N> constexpr size_t mv16_row_smem() { return 16 * (size_t)padded_len16(4 * N); }
template <int N> constexpr size_t mv16_col_smem() { return 16 * (size_t)mx_tile_len<N>(); }

// NP rows of the padded row buffer, in rounds of blockDim / (N/8) rows.
template <int N, int NP>
__device__ __forceinline__ void fft16_rows_d(double2* sm, double sign, const double2* __restrict__ tw) {
    constexpr int TPS = N / 8;
    const int spr = blockDim.x / TPS;
    const int r = threadIdx.x / TPS;
    for (int p0 = 0; p0 < NP; p0 += spr) {
        const int pr = p0 + r;
        fft16<double, N>(sm, RowIdx16{pr * N}, threadIdx.x % TPS, r < spr && pr < NP, sign, tw);
    }
}

// NT = float: the 8 normals from the FP32 Box-Muller (mixed precision; relative
// error ~1e-7 against the FP64 stream), the charges and transforms stay FP64.
template <int N, typename NT = double>
__global__ void __launch_bounds__(mv16_threads<N>()) k_mv16_pass1(const EventDev* __restrict__ ev,
                                                                  const int* __restrict__ slots, int slice,
                                                                  double2* __restrict__ P,
                                                                  const double2* __restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.y;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    for (int y = threadIdx.x; y < N; y += blockDim.x) {
        NT zt[8];
        mv_normals<NT>(e.seed, (uint32_t)slice, (uint32_t)((long)x * N + y), zt);
        double z[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) z[k] = (double)zt[k];
#pragma unroll
        for (int s = 0; s < 4; ++s)
            sm[pad16(s * N + y)] = make_double2(z[2 * s] * e.mv_sigma + 0.0, z[2 * s + 1] * e.mv_sigma + 0.0);
    }
    __syncthreads();
    fft16_rows_store<double, N>(sm, 4, -1.0, tw, P + (long)b * 4 * vol + (long)x * N, vol);
}

// column transform, Poisson factor and inverse column transform with the
// register hand-off of fft16x: global loads feed the first pass, the factor
// and the inverse start from registers, the inverse ends in the store
template <int N>
__global__ void __launch_bounds__(mx_p2_threads<N>(), mx_p2_threads<N>() <= 256 ? 2 : 1) k_mv16_pass2(
    const EventDev* __restrict__ ev, const int* __restrict__ slots, double2* __restrict__ P,
    const double2* __restrict__ tw) {
    constexpr int C = mx_cols<N>();
    constexpr int TH = mx_p2_threads<N>();
    constexpr int PER = N * C / TH;  // = 8
    constexpr int RSTEP = TH / C;    // = N / 8
    static_assert(PER == 8, "one radix-8 lane per thread and column");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* t = reinterpret_cast<double2*>(smem_raw);
    const int c0 = blockIdx.x * C, j = blockIdx.y, b = blockIdx.z;
    const EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const int cc = threadIdx.x % C, r0 = threadIdx.x / C;
    const ColIdx16P<C> cidx{cc};
    double2* io = P + ((long)b * 4 + j) * vol + c0 + (long)r0 * N + cc;
    double2 rv[1][8];
#pragma unroll
    for (int q = 0; q < PER; ++q) rv[0][q] = io[(long)q * RSTEP * N];
    fft16x<double, N, true, true>(t, cidx, r0, true, -1.0, tw, rv);
    // -g / (-phat2 + m^2) / N^2 at (kx, ky) = (r0 + q RSTEP, c0 + cc)
    const double inv = 1.0 / ((double)N * (double)N);
#pragma unroll
    for (int q = 0; q < PER; ++q)
        rv[0][q] = cscale(rv[0][q], -1.0 * e.mv_g / (-phat2_d(r0 + q * RSTEP, c0 + cc, N) + e.mv_mass2) * inv);
    // the inverse's first pass synchronises before it writes t
    fft16x<double, N, true, true>(t, cidx, r0, true, 1.0, tw, rv);
#pragma unroll
    for (int q = 0; q < PER; ++q) io[(long)q * RSTEP * N] = rv[0][q];
}

template <int N>
__global__ void __launch_bounds__(mv16_threads<N>()) k_mv16_pass3(EventDev* __restrict__ ev,
                                                                  const int* __restrict__ slots,
                                                                  const double2* __restrict__ P,
                                                                  const double2* __restrict__ tw,
                                                                  int* __restrict__ flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* sm = reinterpret_cast<double2*>(smem_raw);
    const int x = blockIdx.x, b = blockIdx.y;
    EventDev& e = ev[slots[b]];
    const long vol = (long)N * N;
    const double2* in = P + (long)b * 4 * vol + (long)x * N;
    for (int i = threadIdx.x; i < 4 * N; i += blockDim.x)
        cp_async<16>(&sm[pad16(i)], &in[(long)(i / N) * vol + (i % N)]);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    fft16_rows_d<N, 4>(sm, 1.0, tw);
    int fl = 0;
    for (int y = threadIdx.x; y < N; y += blockDim.x) {
        double f[8];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double2 u = sm[pad16(s * N + y)];
            f[2 * s] = u.x;
            f[2 * s + 1] = u.y;
        }
        double2 m[9], v[9], r[9];
        const long site = (long)x * N + y;
#pragma unroll
        for (int k = 0; k < 9; ++k) v[k] = e.V[k * vol + site];  // arrives while exp(+i f) is formed
        embed_lambda<double>(f, m);
        expi_ch(m, 1.0);  // exp(+i f)
        mul3(v, m, r);
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (!isfinite(r[k].x) || !isfinite(r[k].y)) fl |= JW_FLAG_NAN;
            e.V[k * vol + site] = r[k];
        }
    }
    if (fl) atomicOr(flags, fl);
}

}  // namespace jw
