// jw_common.cuh -- device building blocks shared by every kernel of libjimwlk:
// complex arithmetic on float2/double2, the counter-based noise stream, the
// Gell-Mann embedding used by the reference, 3x3 products and the FP64
// Hermitian exponential (eigen route).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Device-side error flags (bit mask in a device int, cleared by the syncs).
#define JW_FLAG_NOCONV 1
#define JW_FLAG_NAN 2
#define JW_FLAG_TIMEOUT 4  // a bounded wait on a barrier or a tile load ran out

namespace jw {

// ------------------------------------------------------------------ complex
template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using C2 = typename cplx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ C2<T> mk(T r, T i) { C2<T> z; z.x = r; z.y = i; return z; }
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) { a.x *= s; a.y *= s; return a; }
template <typename V> __host__ __device__ __forceinline__ auto cabs2(V a) -> decltype(a.x) { return a.x * a.x + a.y * a.y; }
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    V c; c.x = a.x * b.x + a.y * b.y; c.y = a.y * b.x - a.x * b.y; return c;
}
// multiply by (sign * i)
template <typename V, typename S> __host__ __device__ __forceinline__ V cmul_si(V a, S sign) {
    V c; c.x = -sign * a.y; c.y = sign * a.x; return c;
}

// ------------------------------------------------------------------ noise
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the engine's noise
// generator.  Counter layout of the stream (shared with the oracle):
//   Langevin step s, site i, call c in 0..3: {i, lo32(s), 0x4A570000|c, hi32(s)}
//   MV slice l,      site i, call c in 0..1: {i, l,       0x4D560000|c, 0}
//   key = {lo32(seed), hi32(seed)}
// Each call yields 4 words -> 2 Box-Muller pairs -> 4 unit normals; the 16
// Langevin normals of a site are z[4c+j] and enter the reference's draw order
// n_k = z[2k], m_k = z[2k+1] (field.h:2170-2173); the 8 MV normals are z[a].
constexpr uint32_t kTagLangevin = 0x4A570000u;
constexpr uint32_t kTagMV = 0x4D560000u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// Box-Muller in FP64: u = (r + 1/2) 2^-32, z0 = sqrt(-2 ln u0) cos(2 pi u1),
// z1 = sqrt(-2 ln u0) sin(2 pi u1).
__device__ __forceinline__ void box_muller(uint32_t r0, uint32_t r1, double& z0, double& z1) {
    const double u0 = ((double)r0 + 0.5) * 2.3283064365386963e-10;
    const double u1 = ((double)r1 + 0.5) * 2.3283064365386963e-10;
    const double rad = sqrt(-2.0 * log(u0));
    double s, c;
    sincos(6.283185307179586 * u1, &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

// Box-Muller in FP32 for the same words: ln u0 is taken as log(u0) below 1/2
// and as log1p(-(1-u0)) above, with 1-u0 formed from ~r0, so that the result
// carries full single-precision relative accuracy at both ends.
__device__ __forceinline__ void box_muller(uint32_t r0, uint32_t r1, float& z0, float& z1) {
    float lg;
    if (r0 < 0x80000000u) {
        lg = logf(((float)r0 + 0.5f) * 2.3283064365386963e-10f);
    } else {
        lg = log1pf(-(((float)(~r0) + 0.5f) * 2.3283064365386963e-10f));
    }
    const float rad = sqrtf(-2.0f * lg);
    float s, c;
    sincospif(2.0f * (((float)r1 + 0.5f) * 2.3283064365386963e-10f), &s, &c);
    z0 = rad * c;
    z1 = rad * s;
}

// Box-Muller in FP32 with the hardware approximations: ln u0 from __logf
// (absolute error <= 2^-21.4 near 1, relative ~2^-21 elsewhere), the square
// root from sqrt.approx (relative error ~2^-23) and sin/cos of 2 pi u1 - pi
// from __sincosf (absolute error <= 2^-21.4 on [-pi, pi]).  Each normal differs from the FP64 stream by at most ~3e-6
// absolute; used by the mixed-precision engine.
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Every operation is explicitly rounded, so the kernels that draw the noise
// (pass 1 and pass 3 + 1) give the same bits.
__device__ __forceinline__ void box_muller_fast(uint32_t r0, uint32_t r1, float& z0, float& z1) {
    const float u0 = __fmaf_rn(__uint2float_rn(r0), 2.3283064365386963e-10f, 1.1641532182693481e-10f);
    const float u1 = __fmaf_rn(__uint2float_rn(r1), 2.3283064365386963e-10f, 1.1641532182693481e-10f);
    const float rad = sqrt_approx(__fmul_rn(-2.0f, __logf(u0)));
    float s, c;
    __sincosf(__fmaf_rn(6.28318530717958648f, u1, -3.14159265358979324f), &s, &c);
    z0 = __fmul_rn(-rad, c);  // cos(2 pi u1) = -cos(2 pi u1 - pi)
    z1 = __fmul_rn(-rad, s);
}

__device__ __forceinline__ void langevin_normals_fast(uint64_t seed, uint64_t step, uint32_t site, float z[16]) {
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
        uint4 r = philox4x32_10(make_uint4(site, (uint32_t)step, kTagLangevin | c, (uint32_t)(step >> 32)), key);
        box_muller_fast(r.x, r.y, z[4 * c + 0], z[4 * c + 1]);
        box_muller_fast(r.z, r.w, z[4 * c + 2], z[4 * c + 3]);
    }
}

template <typename T>
__device__ __forceinline__ void langevin_normals(uint64_t seed, uint64_t step, uint32_t site, T z[16]) {
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
        uint4 r = philox4x32_10(make_uint4(site, (uint32_t)step, kTagLangevin | c, (uint32_t)(step >> 32)), key);
        box_muller(r.x, r.y, z[4 * c + 0], z[4 * c + 1]);
        box_muller(r.z, r.w, z[4 * c + 2], z[4 * c + 3]);
    }
}

template <typename T>
__device__ __forceinline__ void mv_normals(uint64_t seed, uint32_t slice, uint32_t site, T z[8]) {
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
#pragma unroll
    for (uint32_t c = 0; c < 2; ++c) {
        uint4 r = philox4x32_10(make_uint4(site, slice, kTagMV | c, 0u), key);
        box_muller(r.x, r.y, z[4 * c + 0], z[4 * c + 1]);
        box_muller(r.z, r.w, z[4 * c + 2], z[4 * c + 3]);
    }
}

// ------------------------------------------------------------------ Gell-Mann basis
// The reference embeds 8 real numbers as sum_a n_a L_a with the matrices it
// writes out in generate_gaussian / setMVModel (field.h:2176-2231, 716-746):
//   L0: (0,1)=(1,0)=1          L1: (0,1)=+i, (1,0)=-i     L2: diag(1,-1,0)
//   L3: (0,2)=(2,0)=1          L4: (0,2)=+i, (2,0)=-i     L5: (1,2)=(2,1)=1
//   L6: (1,2)=+i, (2,1)=-i     L7: diag(1,1,-2)/sqrt(3)
// (Gell-Mann lambdas, not lambda/2; L1, L4, L6 are the transposed lambda_2,5,7.)
// tr(L_a L_b) = 2 delta_ab, so the coefficient of a Hermitian traceless H is
// tr(L_a H)/2.
template <typename T, typename V>
__device__ __forceinline__ void embed_lambda(const T n[8], V m[9]) {
    const T inv_s3 = (T)0.57735026918962573;  // 1/sqrt(3)
    const T d8 = n[7] * inv_s3;
    m[0] = mk<T>(n[2] + d8, 0);
    m[1] = mk<T>(n[0], n[1]);
    m[2] = mk<T>(n[3], n[4]);
    m[3] = mk<T>(n[0], -n[1]);
    m[4] = mk<T>(-n[2] + d8, 0);
    m[5] = mk<T>(n[5], n[6]);
    m[6] = mk<T>(n[3], -n[4]);
    m[7] = mk<T>(n[5], -n[6]);
    m[8] = mk<T>((T)-2 * d8, 0);
}

// embed_lambda for FP64 with explicitly rounded arithmetic (the mixed
// engine's update; see namespace xr below)
__device__ __forceinline__ void embed_lambda_x(const double n[8], double2 m[9]) {
    const double d8 = __dmul_rn(n[7], 0.57735026918962573);
    m[0] = make_double2(__dadd_rn(n[2], d8), 0.0);
    m[1] = make_double2(n[0], n[1]);
    m[2] = make_double2(n[3], n[4]);
    m[3] = make_double2(n[0], -n[1]);
    m[4] = make_double2(__dsub_rn(d8, n[2]), 0.0);
    m[5] = make_double2(n[5], n[6]);
    m[6] = make_double2(n[3], -n[4]);
    m[7] = make_double2(n[5], -n[6]);
    m[8] = make_double2(__dmul_rn(-2.0, d8), 0.0);
}

// The reference's exact sequence of accumulations for one site (used by the
// call-for-call FP64 path so that xi matches generate_gaussian bit for bit).
__device__ __forceinline__ void embed_lambda_ref(const double n[8], double2 m[9]) {
    const double s3 = 1.7320508075688772;  // sqrt(3.0)
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = make_double2(0.0, 0.0);
    m[1].x += n[0]; m[3].x += n[0];
    m[1].y += n[1]; m[3].y -= n[1];
    m[0].x += n[2]; m[4].x -= n[2];
    m[2].x += n[3]; m[6].x += n[3];
    m[2].y += n[4]; m[6].y -= n[4];
    m[5].x += n[5]; m[7].x += n[5];
    m[5].y += n[6]; m[7].y -= n[6];
    m[0].x += n[7] / s3; m[4].x += n[7] / s3; m[8].x += -2.0 * n[7] / s3;
}

// Coefficients h_a = tr(L_a H)/2 of a Hermitian H (only the upper triangle
// and the real diagonal are read).
template <typename T, typename V>
__device__ __forceinline__ void project_lambda(const V m[9], T h[8]) {
    const T s3 = (T)1.7320508075688772;
    h[0] = m[1].x;
    h[1] = m[1].y;
    h[2] = (T)0.5 * (m[0].x - m[4].x);
    h[3] = m[2].x;
    h[4] = m[2].y;
    h[5] = m[5].x;
    h[6] = m[5].y;
    h[7] = (m[0].x + m[4].x - (T)2 * m[8].x) / ((T)2 * s3);
}

// ------------------------------------------------------------------ 3x3
template <typename V>
__device__ __forceinline__ void mul3(const V a[9], const V b[9], V c[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            V s = cmul(a[i * 3 + 0], b[0 * 3 + j]);
            s = cadd(s, cmul(a[i * 3 + 1], b[1 * 3 + j]));
            s = cadd(s, cmul(a[i * 3 + 2], b[2 * 3 + j]));
            c[i * 3 + j] = s;
        }
}
// c = a * b^dagger
template <typename V>
__device__ __forceinline__ void mul3_adj(const V a[9], const V b[9], V c[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            V s = cmulc(a[i * 3 + 0], b[j * 3 + 0]);
            s = cadd(s, cmulc(a[i * 3 + 1], b[j * 3 + 1]));
            s = cadd(s, cmulc(a[i * 3 + 2], b[j * 3 + 2]));
            c[i * 3 + j] = s;
        }
}

// ------------------------------------------------------------------ Hermitian eigen / exp (FP64)
// The route su3_matrix::exponentiate takes (su3_matrix.h:173-253, 256-359):
// Cardano eigenvalues, eigenvectors by cross products of the columns of
// A - w I, and the QL fallback (Householder tridiagonalisation + implicit-shift
// QL, at most 30 sweeps) when a cross product is too small.  This is the
// published algorithm of J. Kopp, Int. J. Mod. Phys. C 19 (2008) 523
// (arXiv:physics/0610206), restated here for double2 registers.  Only the
// upper triangle and the real parts of the diagonal are read, except in the
// Householder step, which reads the complex diagonal as the reference does.
//
// Licence notice.  The eigen-solver routines below (eig_cardano,
// tridiag_householder, eig_ql, eigh3) follow, step for step, Kopp's
// zheevh3 library (zheevc3.cpp, zheevq3.cpp, zhetrd3.cpp, zheevh3.cpp in the
// reference's zheevh3-C-1.1 directory), Copyright (C) 2006 Joachim Kopp,
// distributed under the GNU Lesser General Public License version 2.1 or
// later.  The same operation order is kept so that the exponential matches the
// reference's to 1e-13; these routines are therefore a work based on that
// library and are covered by the LGPL 2.1 (or later) terms under which it is
// distributed.
struct Mat3d { double2 a[3][3]; };

__device__ __forceinline__ double d_sqr(double x) { return x * x; }

__device__ __forceinline__ void eig_cardano(const double2 (&A)[3][3], double w[3]) {
    const double2 de = cmul(A[0][1], A[1][2]);
    const double dd = cabs2(A[0][1]), ee = cabs2(A[1][2]), ff = cabs2(A[0][2]);
    const double a = A[0][0].x, b = A[1][1].x, c = A[2][2].x;
    const double m = a + b + c;
    const double c1 = (a * b + a * c + b * c) - (dd + ee + ff);
    const double c0 = c * dd + a * ee + b * ff - a * b * c - 2.0 * (A[0][2].x * de.x + A[0][2].y * de.y);
    const double p = d_sqr(m) - 3.0 * c1;
    const double q = m * (p - 1.5 * c1) - 13.5 * c0;
    const double sqrt_p = sqrt(fabs(p));
    double phi = 27.0 * (0.25 * d_sqr(c1) * (p - c1) + c0 * (q + 6.75 * c0));
    phi = (1.0 / 3.0) * atan2(sqrt(fabs(phi)), q);
    double sn, cs;
    sincos(phi, &sn, &cs);
    const double cc = sqrt_p * cs;
    const double s = 0.57735026918962573 * sqrt_p * sn;
    w[1] = (1.0 / 3.0) * (m - cc);
    w[2] = w[1] + s;
    w[0] = w[1] + cc;
    w[1] -= s;
}

__device__ inline void tridiag_householder(const double2 (&A)[3][3], double2 (&Q)[3][3], double d[3], double e[3]) {
    double2 u[3], q[3], omega, f;
    double K, h, g;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Q[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    h = cabs2(A[0][1]) + cabs2(A[0][2]);
    g = (A[0][1].x > 0) ? -sqrt(h) : sqrt(h);
    e[0] = g;
    f = cscale(A[0][1], g);
    u[1] = make_double2(A[0][1].x - g, -A[0][1].y);
    u[2] = cconj(A[0][2]);
    omega = make_double2(h - f.x, -f.y);
    if (omega.x > 0.0) {
        // omega <- 0.5 (1 + conj(omega)/omega) / Re(omega)
        const double den = cabs2(omega);
        double2 r = cmul(cconj(omega), cconj(omega));  // conj(omega)^2 / |omega|^2 = conj(omega)/omega
        r = cscale(r, 1.0 / den);
        omega = cscale(make_double2(1.0 + r.x, r.y), 0.5 / omega.x);
        K = 0.0;
#pragma unroll
        for (int i = 1; i < 3; ++i) {
            f = cadd(cmul(cconj(A[1][i]), u[1]), cmul(A[i][2], u[2]));
            q[i] = cmul(omega, f);
            K += cmulc(f, u[i]).x;  // Re(conj(u) f)
        }
        K *= 0.5 * cabs2(omega);
#pragma unroll
        for (int i = 1; i < 3; ++i) q[i] = csub(q[i], cscale(u[i], K));
        d[0] = A[0][0].x;
        d[1] = A[1][1].x - 2.0 * cmulc(q[1], u[1]).x;
        d[2] = A[2][2].x - 2.0 * cmulc(q[2], u[2]).x;
#pragma unroll
        for (int j = 1; j < 3; ++j) {
            f = cmul(omega, cconj(u[j]));
#pragma unroll
            for (int i = 1; i < 3; ++i) Q[i][j] = csub(Q[i][j], cmul(f, u[i]));
        }
        f = csub(csub(A[1][2], cmulc(q[1], u[2])), cmulc(u[1], q[2]));
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i) d[i] = A[i][i].x;
        f = A[1][2];
    }
    e[1] = sqrt(cabs2(f));
    if (e[1] != 0.0) {
        f = cscale(cconj(f), 1.0 / e[1]);
#pragma unroll
        for (int i = 1; i < 3; ++i) Q[i][2] = cmul(Q[i][2], f);
    }
}

// Returns 0, or -1 when the QL sweeps did not converge within 30 iterations.
__device__ inline int eig_ql(const double2 (&A)[3][3], double2 (&Q)[3][3], double w[3]) {
    double e[3];
    tridiag_householder(A, Q, w, e);
    for (int l = 0; l < 2; ++l) {
        int nIter = 0;
        for (;;) {
            int m;
            for (m = l; m <= 1; ++m) {
                const double g = fabs(w[m]) + fabs(w[m + 1]);
                if (fabs(e[m]) + g == g) break;
            }
            if (m == l) break;
            if (nIter++ >= 30) return -1;
            double g = (w[l + 1] - w[l]) / (e[l] + e[l]);
            double r = sqrt(d_sqr(g) + 1.0);
            g = (g > 0) ? w[m] - w[l] + e[l] / (g + r) : w[m] - w[l] + e[l] / (g - r);
            double s = 1.0, c = 1.0, p = 0.0;
            for (int i = m - 1; i >= l; --i) {
                const double f = s * e[i];
                const double b = c * e[i];
                if (fabs(f) > fabs(g)) {
                    c = g / f;
                    r = sqrt(d_sqr(c) + 1.0);
                    e[i + 1] = f * r;
                    s = 1.0 / r;
                    c *= s;
                } else {
                    s = f / g;
                    r = sqrt(d_sqr(s) + 1.0);
                    e[i + 1] = g * r;
                    c = 1.0 / r;
                    s *= c;
                }
                g = w[i + 1] - p;
                r = (w[i] - g) * s + 2.0 * c * b;
                p = s * r;
                w[i + 1] = g + p;
                g = c * r - b;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double2 t = Q[k][i + 1];
                    Q[k][i + 1] = cadd(cscale(Q[k][i], s), cscale(t, c));
                    Q[k][i] = csub(cscale(Q[k][i], c), cscale(t, s));
                }
            }
            w[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

// Hybrid solver.  Returns 0 (analytic or converged QL) or -1 (QL failed).
__device__ __forceinline__ int eigh3(const double2 (&A)[3][3], double2 (&Q)[3][3], double w[3]) {
    eig_cardano(A, w);
    double t = fabs(w[0]), u;
    if ((u = fabs(w[1])) > t) t = u;
    if ((u = fabs(w[2])) > t) t = u;
    u = (t < 1.0) ? t : d_sqr(t);
    const double error = 256.0 * 2.220446049250313e-16 * d_sqr(u);
    double2 q01 = csub(cmul(A[0][1], A[1][2]), cscale(A[0][2], A[1][1].x));
    double2 q11 = csub(cmulc(A[0][2], A[0][1]), cscale(A[1][2], A[0][0].x));
    const double q21 = cabs2(A[0][1]);
    double2 v0 = cadd(q01, cscale(A[0][2], w[0]));
    double2 v1 = cadd(q11, cscale(A[1][2], w[0]));
    double v2 = (A[0][0].x - w[0]) * (A[1][1].x - w[0]) - q21;
    double norm = cabs2(v0) + cabs2(v1) + d_sqr(v2);
    if (norm <= error) return eig_ql(A, Q, w);
    norm = sqrt(1.0 / norm);
    Q[0][0] = cscale(v0, norm);
    Q[1][0] = cscale(v1, norm);
    Q[2][0] = make_double2(v2 * norm, 0.0);
    v0 = cadd(q01, cscale(A[0][2], w[1]));
    v1 = cadd(q11, cscale(A[1][2], w[1]));
    v2 = (A[0][0].x - w[1]) * (A[1][1].x - w[1]) - q21;
    norm = cabs2(v0) + cabs2(v1) + d_sqr(v2);
    if (norm <= error) return eig_ql(A, Q, w);
    norm = sqrt(1.0 / norm);
    Q[0][1] = cscale(v0, norm);
    Q[1][1] = cscale(v1, norm);
    Q[2][1] = make_double2(v2 * norm, 0.0);
    Q[0][2] = cconj(csub(cmul(Q[1][0], Q[2][1]), cmul(Q[2][0], Q[1][1])));
    Q[1][2] = cconj(csub(cmul(Q[2][0], Q[0][1]), cmul(Q[0][0], Q[2][1])));
    Q[2][2] = cconj(csub(cmul(Q[0][0], Q[1][1]), cmul(Q[1][0], Q[0][1])));
    return 0;
}

// m <- Q diag(exp(i sign w)) Q^dagger for the Hermitian matrix held in m.
// Returns the eigensolver status.
__device__ __forceinline__ int expi_herm(double2 m[9], double sign) {
    double2 A[3][3], Q[3][3];
    double w[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) A[i][j] = m[i * 3 + j];
    const int status = eigh3(A, Q, w);
    double2 ph[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double s, c;
        sincos(sign * w[k], &s, &c);
        ph[k] = make_double2(c, s);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double2 acc = cmulc(cmul(Q[i][0], ph[0]), Q[j][0]);
            acc = cadd(acc, cmulc(cmul(Q[i][1], ph[1]), Q[j][1]));
            acc = cadd(acc, cmulc(cmul(Q[i][2], ph[2]), Q[j][2]));
            m[i * 3 + j] = acc;
        }
    return status;
}

// exp(i Q) of a traceless Hermitian 3x3 by the Cayley-Hamilton theorem:
// exp(iQ) = f0 + f1 Q + f2 Q^2 with the coefficients of C. Morningstar and
// M. Peardon, Phys. Rev. D 69 (2004) 054501, eqs. (23)-(33):
//   c0 = det Q, c1 = tr(Q^2)/2, c0max = 2 (c1/3)^(3/2), theta = acos(c0/c0max),
//   u = sqrt(c1/3) cos(theta/3), w = sqrt(c1) sin(theta/3), xi0(w) = sin(w)/w,
//   h0 = (u^2 - w^2) e^{2iu} + e^{-iu} [8u^2 cos w + 2iu (3u^2 + w^2) xi0],
//   h1 = 2u e^{2iu} - e^{-iu} [2u cos w - i (3u^2 - w^2) xi0],
//   h2 = e^{2iu} - e^{-iu} [cos w + 3iu xi0],       f_j = h_j / (9u^2 - w^2),
// evaluated for |c0| (f_j(-c0) = (-1)^j conj f_j(c0)) so that 9u^2 - w^2 >= 2 c1.
// For c1 <= 0.05 (|Q| below ~0.3: every Langevin update at the usual step
// sizes) the Taylor series of exp(iQ), reduced with Q^3 = c1 Q + c0, is used
// instead; it needs no transcendental functions.  For c1 <= 2e-3 (typical
// updates) ten terms suffice and are summed as closed-form polynomials in c0
// and c1.
// Only the upper triangle and the real diagonal of m are read.
__device__ __forceinline__ void expi_ch(double2 m[9], double sign) {
    const double a = sign * m[0].x, b = sign * m[4].x, c = sign * m[8].x;
    const double2 d = cscale(m[1], sign), f = cscale(m[2], sign), e = cscale(m[5], sign);
    const double dd = cabs2(d), ee = cabs2(e), ff = cabs2(f);
    // Q^2 (Hermitian): diagonal and upper triangle
    const double q00 = a * a + dd + ff, q11 = dd + b * b + ee, q22 = ff + ee + c * c;
    const double2 q01 = cadd(cscale(d, a + b), cmulc(f, e));           // a d + d b + f conj(e)
    const double2 q02 = cadd(cscale(f, a + c), cmul(d, e));            // a f + d e + f c
    const double2 q12 = cadd(cmul(cconj(d), f), cscale(e, b + c));     // conj(d) f + b e + e c
    const double c1 = 0.5 * (q00 + q11 + q22);
    const double2 def = cmulc(cmul(d, e), f);                          // d e conj(f)
    const double c0 = a * b * c - a * ee - b * ff - c * dd + 2.0 * def.x;
    double2 f0, f1, f2;
    if (c1 <= 2e-3) {
        // The same series truncated after (iQ)^10, with Q^n reduced to
        // f0 + f1 Q + f2 Q^2 in closed form (polynomials in c0 and c1):
        // |Q| <= sqrt(4 c1 / 3) <= 0.052 here, so the first omitted term is
        // below 0.052^11 / 11! < 4e-22.  Evaluated in nested (Horner) form.
        const double x = c0, y = c1, x2 = c0 * c0;
        f0 = make_double2(1.0 + x2 * (-1.0 / 720.0 + y * (1.0 / 20160.0 - y * (1.0 / 1209600.0))),
                          x * (-1.0 / 6.0 + y * (1.0 / 120.0 + y * (-1.0 / 5040.0 + y * (1.0 / 362880.0)))) +
                              x2 * x * (1.0 / 362880.0));
        f1 = make_double2(x * (1.0 / 24.0 + y * (-1.0 / 360.0 + y * (1.0 / 13440.0 - y * (1.0 / 907200.0)))) -
                              x2 * x * (1.0 / 3628800.0),
                          1.0 + y * (-1.0 / 6.0 + y * (1.0 / 120.0 + y * (-1.0 / 5040.0 + y * (1.0 / 362880.0)))) +
                              x2 * (-1.0 / 5040.0 + y * (1.0 / 120960.0)));
        f2 = make_double2(-0.5 + y * (1.0 / 24.0 + y * (-1.0 / 720.0 + y * (1.0 / 40320.0 - y * (1.0 / 3628800.0)))) +
                              x2 * (1.0 / 40320.0 - y * (1.0 / 1209600.0)),
                          x * (1.0 / 120.0 + y * (-1.0 / 2520.0 + y * (1.0 / 120960.0))));
    } else if (c1 <= 0.05) {
        // sum_n (i^n / n!) Q^n with Q^n = a_n + b_n Q + c_n Q^2 and, from
        // Q^3 = c1 Q + c0: (a, b, c)_{n+1} = (c0 c_n, a_n + c1 c_n, b_n).
        // |Q| <= sqrt(2 c1) <= 0.32, so 16 terms leave < 1e-21.
        double an = 1.0, bn = 0.0, cn = 0.0, fac = 1.0;
        double r0 = 0.0, i0 = 0.0, r1 = 0.0, i1 = 0.0, r2 = 0.0, i2 = 0.0;
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            // i^n: n mod 4 = 0 -> +1, 1 -> +i, 2 -> -1, 3 -> -i
            const double sg = (n & 2) ? -fac : fac;
            if (n & 1) { i0 += sg * an; i1 += sg * bn; i2 += sg * cn; }
            else { r0 += sg * an; r1 += sg * bn; r2 += sg * cn; }
            const double a2 = c0 * cn, b2 = an + c1 * cn;
            cn = bn; an = a2; bn = b2;
            fac /= (double)(n + 1);
        }
        f0 = make_double2(r0, i0);
        f1 = make_double2(r1, i1);
        f2 = make_double2(r2, i2);
    } else {
        const bool neg = c0 < 0.0;
        const double c0a = fabs(c0);
        const double s13 = sqrt(c1 / 3.0);
        const double c0max = 2.0 * s13 * s13 * s13;
        const double r = fmin(c0a / c0max, 1.0);
        const double theta = acos(r);
        double st, ct;
        sincos(theta / 3.0, &st, &ct);
        const double u = s13 * ct, w = sqrt(c1) * st;
        const double u2 = u * u, w2 = w * w;
        double su, cu, sw, cw;
        sincos(u, &su, &cu);
        sincos(w, &sw, &cw);
        const double xi0 = (fabs(w) < 0.05) ? 1.0 - w2 / 6.0 * (1.0 - w2 / 20.0 * (1.0 - w2 / 42.0)) : sw / w;
        // e^{2iu} = (cos 2u, sin 2u) from the half angle; e^{-iu} = (cos u, -sin u)
        const double2 e2 = make_double2(1.0 - 2.0 * su * su, 2.0 * su * cu);
        const double2 em = make_double2(cu, -su);
        const double2 h0 = cadd(cscale(e2, u2 - w2), cmul(em, make_double2(8.0 * u2 * cw, 2.0 * u * (3.0 * u2 + w2) * xi0)));
        const double2 h1 = csub(cscale(e2, 2.0 * u), cmul(em, make_double2(2.0 * u * cw, -(3.0 * u2 - w2) * xi0)));
        const double2 h2 = csub(e2, cmul(em, make_double2(cw, 3.0 * u * xi0)));
        const double inv = 1.0 / (9.0 * u2 - w2);
        f0 = cscale(h0, inv);
        f1 = cscale(h1, inv);
        f2 = cscale(h2, inv);
        if (neg) {
            f0 = cconj(f0);
            f1 = make_double2(-f1.x, f1.y);
            f2 = cconj(f2);
        }
    }
    // exp(iQ) = f0 I + f1 Q + f2 Q^2, Q and Q^2 Hermitian
    const double2 Qm[9] = {make_double2(a, 0.0), d, f, cconj(d), make_double2(b, 0.0), e, cconj(f), cconj(e),
                           make_double2(c, 0.0)};
    const double2 Q2[9] = {make_double2(q00, 0.0), q01, q02, cconj(q01), make_double2(q11, 0.0), q12,
                           cconj(q02), cconj(q12), make_double2(q22, 0.0)};
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double2 v = cadd(cmul(f1, Qm[k]), cmul(f2, Q2[k]));
        if (k == 0 || k == 4 || k == 8) v = cadd(v, f0);
        m[k] = v;
    }
}

// Reunitarisation: Gram-Schmidt on rows 0 and 1, row 2 = conj(row0 x row1),
// which is the nearest-in-practice SU(3) projection for a matrix that is
// unitary up to rounding.
__device__ __forceinline__ void reunitarize(double2 m[9]) {
    double n0 = rsqrt(cabs2(m[0]) + cabs2(m[1]) + cabs2(m[2]));
    m[0] = cscale(m[0], n0); m[1] = cscale(m[1], n0); m[2] = cscale(m[2], n0);
    // <r0, r1> = sum conj(r0) r1
    double2 d = cadd(cadd(cmulc(m[3], m[0]), cmulc(m[4], m[1])), cmulc(m[5], m[2]));
    m[3] = csub(m[3], cmul(d, m[0]));
    m[4] = csub(m[4], cmul(d, m[1]));
    m[5] = csub(m[5], cmul(d, m[2]));
    double n1 = rsqrt(cabs2(m[3]) + cabs2(m[4]) + cabs2(m[5]));
    m[3] = cscale(m[3], n1); m[4] = cscale(m[4], n1); m[5] = cscale(m[5], n1);
    m[6] = cconj(csub(cmul(m[1], m[5]), cmul(m[2], m[4])));
    m[7] = cconj(csub(cmul(m[2], m[3]), cmul(m[0], m[5])));
    m[8] = cconj(csub(cmul(m[0], m[4]), cmul(m[1], m[3])));
}

// ------------------------------------------------------------------ explicitly rounded FP64 update
// The mixed-precision engine updates V in two kernels (pass 3, and pass 3
// fused with the next pass 1).  The exponentials, products and
// reunitarisation below spell every operation as a rounded intrinsic, so that
// the compiler cannot fuse them differently in the two kernels: a run of K
// steps gives the same bits however its steps are split into calls.  The
// mathematics is expi_ch / mul3 / reunitarize's.
namespace xr {
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -mul(a.y, b.y)), fma(a.x, b.y, mul(a.y, b.x)));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, mul(a.y, b.y)), fma(a.y, b.x, -mul(a.x, b.y)));
}
// c + a * b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(add(a.x, b.x), add(a.y, b.y)); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(mul(a.x, s), mul(a.y, s)); }
__device__ __forceinline__ double cabs2(double2 a) { return fma(a.x, a.x, mul(a.y, a.y)); }

// c = a b (3 x 3 complex)
__device__ __forceinline__ void mul3(const double2 a[9], const double2 b[9], double2 c[9]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double2 t = cmul(a[i * 3 + 0], b[0 * 3 + j]);
            t = cfma(a[i * 3 + 1], b[1 * 3 + j], t);
            c[i * 3 + j] = cfma(a[i * 3 + 2], b[2 * 3 + j], t);
        }
}

// m <- exp(i sign Q) for the Hermitian Q given by m's upper triangle and real
// diagonal (expi_ch's three branches).
__device__ __forceinline__ void expi_ch(double2 m[9], double sign) {
    const double a = sign * m[0].x, b = sign * m[4].x, c = sign * m[8].x;
    const double2 d = make_double2(sign * m[1].x, sign * m[1].y), f = make_double2(sign * m[2].x, sign * m[2].y),
                  e = make_double2(sign * m[5].x, sign * m[5].y);
    const double dd = cabs2(d), ee = cabs2(e), ff = cabs2(f);
    const double q00 = add(fma(a, a, dd), ff), q11 = add(fma(b, b, dd), ee), q22 = fma(c, c, add(ff, ee));
    const double2 q01 = cadd(cscale(d, add(a, b)), cmulc(f, e));  // a d + d b + f conj(e)
    const double2 q02 = cadd(cscale(f, add(a, c)), cmul(d, e));   // a f + d e + f c
    const double2 q12 = cadd(cmulc(f, d), cscale(e, add(b, c)));   // conj(d) f + b e + e c
    const double c1 = mul(0.5, add(add(q00, q11), q22));
    const double2 de = cmul(d, e);
    const double def = fma(de.x, f.x, mul(de.y, f.y));  // Re(d e conj(f))
    const double c0 = fma(2.0, def, sub(sub(sub(mul(mul(a, b), c), mul(a, ee)), mul(b, ff)), mul(c, dd)));
    double2 f0, f1, f2;
    if (c1 <= 2e-3) {
        const double x = c0, y = c1, x2 = mul(c0, c0);
        f0 = make_double2(
            fma(x2, fma(y, fma(y, -1.0 / 1209600.0, 1.0 / 20160.0), -1.0 / 720.0), 1.0),
            fma(mul(x2, x), 1.0 / 362880.0,
                mul(x, fma(y, fma(y, fma(y, 1.0 / 362880.0, -1.0 / 5040.0), 1.0 / 120.0), -1.0 / 6.0))));
        f1 = make_double2(
            fma(mul(x2, x), -1.0 / 3628800.0,
                mul(x, fma(y, fma(y, fma(y, -1.0 / 907200.0, 1.0 / 13440.0), -1.0 / 360.0), 1.0 / 24.0))),
            fma(x2, fma(y, 1.0 / 120960.0, -1.0 / 5040.0),
                fma(y, fma(y, fma(y, fma(y, 1.0 / 362880.0, -1.0 / 5040.0), 1.0 / 120.0), -1.0 / 6.0), 1.0)));
        f2 = make_double2(
            fma(x2, fma(y, -1.0 / 1209600.0, 1.0 / 40320.0),
                fma(y, fma(y, fma(y, fma(y, -1.0 / 3628800.0, 1.0 / 40320.0), -1.0 / 720.0), 1.0 / 24.0), -0.5)),
            mul(x, fma(y, fma(y, 1.0 / 120960.0, -1.0 / 2520.0), 1.0 / 120.0)));
    } else if (c1 <= 0.05) {
        double an = 1.0, bn = 0.0, cn = 0.0, fac = 1.0;
        double r0 = 0.0, i0 = 0.0, r1 = 0.0, i1 = 0.0, r2 = 0.0, i2 = 0.0;
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const double sg = (n & 2) ? -fac : fac;
            if (n & 1) { i0 = fma(sg, an, i0); i1 = fma(sg, bn, i1); i2 = fma(sg, cn, i2); }
            else { r0 = fma(sg, an, r0); r1 = fma(sg, bn, r1); r2 = fma(sg, cn, r2); }
            const double a2 = mul(c0, cn), b2 = fma(c1, cn, an);
            cn = bn; an = a2; bn = b2;
            fac /= (double)(n + 1);
        }
        f0 = make_double2(r0, i0);
        f1 = make_double2(r1, i1);
        f2 = make_double2(r2, i2);
    } else {
        const bool neg = c0 < 0.0;
        const double c0a = fabs(c0);
        const double s13 = sqrt(c1 / 3.0);
        const double c0max = mul(mul(2.0, s13), mul(s13, s13));
        const double r = fmin(c0a / c0max, 1.0);
        const double theta = acos(r);
        double st, ct;
        sincos(theta / 3.0, &st, &ct);
        const double u = mul(s13, ct), w = mul(sqrt(c1), st);
        const double u2 = mul(u, u), w2 = mul(w, w);
        double su, cu, sw, cw;
        sincos(u, &su, &cu);
        sincos(w, &sw, &cw);
        const double xi0 = (fabs(w) < 0.05)
                               ? sub(1.0, mul(w2 / 6.0, sub(1.0, mul(w2 / 20.0, sub(1.0, w2 / 42.0)))))
                               : sw / w;
        const double2 e2 = make_double2(sub(1.0, mul(2.0, mul(su, su))), mul(2.0, mul(su, cu)));
        const double2 em = make_double2(cu, -su);
        const double2 h0 = cadd(cscale(e2, sub(u2, w2)),
                                cmul(em, make_double2(mul(8.0, mul(u2, cw)), mul(mul(2.0, u), mul(fma(3.0, u2, w2), xi0)))));
        const double2 h1 = cadd(cscale(e2, mul(2.0, u)),
                                cscale(cmul(em, make_double2(mul(mul(2.0, u), cw), -mul(fma(3.0, u2, -w2), xi0))), -1.0));
        const double2 h2 = cadd(e2, cscale(cmul(em, make_double2(cw, mul(mul(3.0, u), xi0))), -1.0));
        const double inv = 1.0 / fma(9.0, u2, -w2);
        f0 = cscale(h0, inv);
        f1 = cscale(h1, inv);
        f2 = cscale(h2, inv);
        if (neg) {
            f0 = make_double2(f0.x, -f0.y);
            f1 = make_double2(-f1.x, f1.y);
            f2 = make_double2(f2.x, -f2.y);
        }
    }
    // exp(iQ) = f0 I + f1 Q + f2 Q^2
    const double2 Qm[9] = {make_double2(a, 0.0), d, f, make_double2(d.x, -d.y), make_double2(b, 0.0), e,
                           make_double2(f.x, -f.y), make_double2(e.x, -e.y), make_double2(c, 0.0)};
    const double2 Q2[9] = {make_double2(q00, 0.0), q01, q02, make_double2(q01.x, -q01.y), make_double2(q11, 0.0),
                           q12, make_double2(q02.x, -q02.y), make_double2(q12.x, -q12.y), make_double2(q22, 0.0)};
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        if (k == 0 || k == 4 || k == 8)
            m[k] = make_double2(fma(f2.x, Q2[k].x, fma(f1.x, Qm[k].x, f0.x)), fma(f2.y, Q2[k].x, fma(f1.y, Qm[k].x, f0.y)));
        else
            m[k] = cfma(f2, Q2[k], cmul(f1, Qm[k]));
    }
}

// Gram-Schmidt on rows 0 and 1, row 2 = conj(row0 x row1) (reunitarize)
__device__ __forceinline__ void reunitarize(double2 m[9]) {
    const double n0 = rsqrt(add(add(cabs2(m[0]), cabs2(m[1])), cabs2(m[2])));
    m[0] = cscale(m[0], n0); m[1] = cscale(m[1], n0); m[2] = cscale(m[2], n0);
    // <r0, r1> = sum conj(r0) r1
    const double2 d = cadd(cadd(cmulc(m[3], m[0]), cmulc(m[4], m[1])), cmulc(m[5], m[2]));
    const double2 md = make_double2(-d.x, -d.y);
    m[3] = cfma(md, m[0], m[3]);
    m[4] = cfma(md, m[1], m[4]);
    m[5] = cfma(md, m[2], m[5]);
    const double n1 = rsqrt(add(add(cabs2(m[3]), cabs2(m[4])), cabs2(m[5])));
    m[3] = cscale(m[3], n1); m[4] = cscale(m[4], n1); m[5] = cscale(m[5], n1);
    auto cross = [](double2 p, double2 q, double2 r, double2 t) {  // conj(p q - r t)
        const double2 u = cfma(make_double2(-r.x, -r.y), t, cmul(p, q));
        return make_double2(u.x, -u.y);
    };
    m[6] = cross(m[1], m[5], m[2], m[4]);
    m[7] = cross(m[2], m[3], m[0], m[5]);
    m[8] = cross(m[0], m[4], m[1], m[3]);
}
}  // namespace xr

// ------------------------------------------------------------------ lattice momenta
// momenta::set (momenta.h:90-124): phat2 = 4 sin^2(pi kx/N) + 4 sin^2(pi ky/N),
// pbar_i = sin(2 pi k_i / N), with the unwrapped index k in 0..N-1.
__device__ __forceinline__ double phat2_d(int kx, int ky, int N) {
    const double sx = sin(3.141592653589793 * kx / (1.0 * N));
    const double sy = sin(3.141592653589793 * ky / (1.0 * N));
    return 4.0 * sx * sx + 4.0 * sy * sy;
}

}  // namespace jw
