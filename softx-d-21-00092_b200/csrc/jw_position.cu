// jw_position.cu -- position-space evolution (main_optimized.cpp:271-304):
// prepare_A_and_B_local for every site as two circular convolutions through
// the transform, the coupling-constant correlation and its complex-symmetric
// Cholesky factor (gmatrix::decompose), the factor applied to the noise
// (gfield::multiplyByCholesky) and reduce_hatta.
//
// prepare_A_and_B_local (field.h:2368-2519) sums, for each output site x,
// k(x - y) xi(y) and k(x - y) V(y) xi(y) V(y)^dagger over all sites y: O(V^2)
// per step.  Both sums are circular convolutions with a real kernel, so with
// K = DFT(k) (raw, computed once per (rr, coupling, kernel)) they are
//   A = U^-1 [K_x U(xi_x) + K_y U(xi_y)],  B = the same with V xi V^dagger,
// U the unitary transform of execute2D: O(V log V) per step.
//
// The Cholesky factor L of the V x V site-site correlation (68.7 GB of
// complex doubles at 256^2) is stored row-major lower, the reference's own
// layout, which column-major BLAS sees as the upper factor U = L^T of
// S = U^T U.  The decomposition is right-looking and blocked (b = 128): a
// one-CTA kernel factors each diagonal block, a warp per row solves the panel
// below it (k_chol_trsm), and the FP64 tensor cores update the trailing lower
// triangle by the complex-symmetric, non-conjugating rank-b product
// (k_chol_syrk).  Applying L streams its lower triangle once per call
// on the FP64 tensor cores (k_chol_apply, mma.sync m8n8k4): each CTA owns 128
// rows and one 4096-column chunk, stages 128 x 16 tiles of L with cp.async,
// and multiplies them with 8, 16 or 24 real right-hand sides.  For the
// Langevin noise the right-hand sides are the 16 unit normals of each site
// (the Gell-Mann embedding is linear and is applied after L), so the kernel
// does 32 FP64 FMAs per 16 B of L: HBM-bound when the tensor pipe runs above
// about 70% of its peak.  Partial products of the chunks are summed in a
// fixed order, so results are deterministic.
#include <algorithm>
#include <cmath>
#include <vector>

#include "jw_internal.h"

using namespace jw;

struct jw_cholesky {
    jw_context* ctx = nullptr;
    long n = 0;                  // N*N
    long np = 0;                 // the factor's order: n padded to the blocking (a multiple of 16 up to 128,
                                 // of 128 above) with an identity block, whose factor is itself
    double2* d_L = nullptr;      // np*np complex, row-major lower, zero above the diagonal
    int2* d_units = nullptr;     // apply work list: (row strip, column chunk)
    int n_units = 0;
    int n_chunks = 0;
    double* d_X = nullptr;       // np x kMaxR real right-hand sides, site-major (rows past n stay zero)
    double2* d_P = nullptr;      // n_chunks x np x kMaxR partial products
    // d_P holds the correlated noise of step `cached_step` (seed `cached_seed`)
    // as the second half of the last two-step apply; any other use of d_P clears it
    mutable bool cached = false;
    mutable uint64_t cached_step = 0, cached_seed = 0;
};

namespace {

constexpr int kThreads = 256;
inline unsigned blocks_for(long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Cholesky apply tiling: 128 rows per CTA, 16 columns per staged tile, three
// stages, 4096 columns per chunk; right-hand sides in multiples of 8 (at most 32:
// the noise of two Langevin steps).
constexpr int kTR = 128, kKT = 16, kTC = 4096, kStages = 3, kMaxR = 32;
template <int NT> constexpr int apply_x_row_bytes() { return NT * 64 + 32; }  // padded: conflict-free B fragments
template <int NT> constexpr int apply_stage_bytes() { return kTR * kKT * 16 + kKT * apply_x_row_bytes<NT>(); }
constexpr int kDiagBlock = 128;

__device__ __forceinline__ void cpa16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

}  // namespace

// ---- position kernel (positions.h:105-150, field.h:2402-2462), host FP64
// with the reference's own expressions so that the tabulated values are the
// reference's bit for bit.
void jw::position_kernel_host(int dxi, int dyi, int N, int rr, int coupling, int kernel, double* kx, double* ky) {
    double dx, dy, rrr;
    if (kernel == JW_SIN_KERNEL) {
        dx = 0.5 * N * std::sin(2.0 * M_PI * dxi / (1.0 * N)) / M_PI;
        dy = 0.5 * N * std::sin(2.0 * M_PI * dyi / (1.0 * N)) / M_PI;
        const double sx = N * std::sin(M_PI * dxi / (1.0 * N)) / M_PI;
        const double sy = N * std::sin(M_PI * dyi / (1.0 * N)) / M_PI;
        rrr = std::pow(sx, 2.0) + std::pow(sy, 2.0);
    } else {
        dx = dxi;
        if (dx >= N / 2) dx = dx - N;
        if (dx < -N / 2) dx = dx + N;
        dy = dyi;
        if (dy >= N / 2) dy = dy - N;
        if (dy < -N / 2) dy = dy + N;
        rrr = 1.0 * (dx * dx + dy * dy);
    }
    double rrrmin = rrr;
    if (coupling == JW_HATTA_COUPLING_CONSTANT) rrrmin = (rrr <= rr) ? rrr : rr;
    const double lambda = std::pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    double sc = 1.0;
    if (coupling == JW_SQRT_COUPLING_CONSTANT || coupling == JW_HATTA_COUPLING_CONSTANT)
        sc = std::sqrt(4.0 * M_PI /
                       ((11.0 - 2.0 * 3.0 / 3.0) *
                        std::log(std::pow(lambda + 1.26 / std::pow(6.0 * 6.0 * rrrmin / N / N, 1.0 / 0.2), 0.2))));
    *kx = 0.0;
    *ky = 0.0;
    if (rrr > 10e-9) {
        *kx = sc * dx / rrr;
        *ky = sc * dy / rrr;
    }
}

namespace {

// out_k = K_x X_k + K_y Y_k for the 9 components (k-space product of the convolution).
__global__ void k_pos_combine(double2* __restrict__ out, const double2* __restrict__ X, const double2* __restrict__ Y,
                              const double2* __restrict__ tab, long vol) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double2 kx = tab[i], ky = tab[vol + i];
#pragma unroll
    for (int k = 0; k < 9; ++k) out[k * vol + i] = cadd(cmul(kx, X[k * vol + i]), cmul(ky, Y[k * vol + i]));
}

// V xi_x V^dagger, V xi_y V^dagger (the B-side integrand, field.h:2479-2497).
__global__ void k_pos_rotate(double2* __restrict__ ox, double2* __restrict__ oy, const double2* __restrict__ V,
                             const double2* __restrict__ xx, const double2* __restrict__ xy, long vol) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    double2 a[9], b[9], t[9], e[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k] = V[k * vol + i];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = xx[k * vol + i];
    mul3(a, b, t);
    mul3_adj(t, a, e);
#pragma unroll
    for (int k = 0; k < 9; ++k) ox[k * vol + i] = e[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = xy[k * vol + i];
    mul3(a, b, t);
    mul3_adj(t, a, e);
#pragma unroll
    for (int k = 0; k < 9; ++k) oy[k * vol + i] = e[k];
}

// ---- gfield::reduce_hatta (field.h:1538-1564)
__global__ void k_reduce_hatta(const double2* __restrict__ c, double2* __restrict__ sum, double2* __restrict__ err,
                               long i) {
    const double2 v = c[i];
    sum[i] = cadd(sum[i], v);
    double2 sq;
    if (v.y == 0.0 && v.x > 0.0) sq = make_double2(v.x * v.x, 0.0);
    else sq = cmul(v, v);
    err[i] = cadd(err[i], sq);
}

// ---- complex square root and division for the diagonal blocks (principal
// branch; Smith's scaled division, CACM 5(8):435, 1962).
__device__ __forceinline__ double2 csqrt_p(double2 z) {
    if (z.x == 0.0 && z.y == 0.0) return make_double2(0.0, z.y);
    const double t = sqrt(0.5 * (hypot(z.x, z.y) + fabs(z.x)));
    if (z.x >= 0.0) return make_double2(t, z.y / (2.0 * t));
    return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}
__device__ __forceinline__ double2 cdiv_smith(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    }
    const double r = b.x / b.y, den = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}

// S(i, j) = corr(|x_i - x_j|, |y_i - y_j|) on and below the diagonal, zero
// above (matrix.h:190-196: non-periodic distances), for i, j < n; the rows
// and columns from n to np are those of the identity, so the factor of the
// padded matrix is the factor of S with an identity block after it.
__global__ void k_chol_fill(double2* __restrict__ M, const double2* __restrict__ corr, int N, long n, long np) {
    const long total = np * np;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long i = idx / np, j = idx - i * np;
        double2 v = make_double2(i == j ? 1.0 : 0.0, 0.0);
        if (i < n && j <= i) {
            const int xi = (int)(i / N), yi = (int)(i % N), xj = (int)(j / N), yj = (int)(j % N);
            v = corr[(long)abs(xi - xj) * N + abs(yi - yj)];
        }
        M[idx] = v;
    }
}

// Unblocked right-looking complex-symmetric Cholesky of one b x b diagonal
// block (row-major lower, leading dimension ld) whose trailing updates from
// the columns to its left are already applied: L_jj = sqrt(a_jj),
// L_ij = a_ij / L_jj, a_il -= L_ij L_lj.  One CTA; the block stays in L2.
__global__ void __launch_bounds__(1024) k_chol_diag(double2* __restrict__ a, long ld, int b) {
    // the block's lower triangle in shared memory, packed by rows: row i
    // starts at i (i + 1) / 2
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* s = reinterpret_cast<double2*>(smem_raw);
    auto at = [](int i, int j) { return i * (i + 1) / 2 + j; };
    for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
        const int i = idx / b, j = idx % b;
        if (j <= i) s[at(i, j)] = a[(long)i * ld + j];
    }
    __syncthreads();
    for (int j = 0; j < b; ++j) {
        if (threadIdx.x == 0) s[at(j, j)] = csqrt_p(s[at(j, j)]);
        __syncthreads();
        const double2 d = s[at(j, j)];
        for (int i = j + 1 + threadIdx.x; i < b; i += blockDim.x) s[at(i, j)] = cdiv_smith(s[at(i, j)], d);
        __syncthreads();
        const int m = b - j - 1;
        for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
            const int i = j + 1 + q / m, l = j + 1 + q % m;
            if (l <= i) s[at(i, l)] = csub(s[at(i, l)], cmul(s[at(i, j)], s[at(l, j)]));
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
        const int i = idx / b, j = idx % b;
        if (j <= i) a[(long)i * ld + j] = s[at(i, j)];
    }
}
constexpr size_t diag_smem_bytes() { return sizeof(double2) * (size_t)kDiagBlock * (kDiagBlock + 1) / 2; }

// One FP64 tensor-core product D(8x8) += A(8x4) B(4x8) (mma.sync m8n8k4):
// lane (g = lane/4, q = lane%4) supplies A[g][q] and B[q][g] and holds
// D[g][2q], D[g][2q+1].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}


// ---- panel solve (the TRSM step of the blocked factorisation): every row a of
// the panel below the diagonal block becomes x with x L_kk^T = a, i.e. for
// j = 0..b-1: x_j = a_j / L_kk[j][j], then a_m -= x_j L_kk[m][j] for m > j
// (right-looking forward substitution).  One warp per panel row, lane l
// holding a_m for m = l + 32 s; the diagonal block's lower triangle sits in
// shared memory packed by columns, so the lanes read column j contiguously.
constexpr int kTrsmThreads = 1024;
__host__ __device__ constexpr int trsm_col_off(int j) { return kDiagBlock * j - j * (j - 1) / 2; }
constexpr size_t trsm_smem_bytes() { return sizeof(double2) * (size_t)trsm_col_off(kDiagBlock); }

__global__ void __launch_bounds__(kTrsmThreads) k_chol_trsm(double2* __restrict__ L, long ld, long k0, long rest) {
    static_assert(kDiagBlock == 128, "four slots of 32 per lane");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* Lc = reinterpret_cast<double2*>(smem_raw);  // column j, rows j..b-1 at trsm_col_off(j) + (m - j)
    const double2* Lkk = L + k0 * ld + k0;
    for (int idx = threadIdx.x; idx < kDiagBlock * kDiagBlock; idx += blockDim.x) {
        const int m = idx / kDiagBlock, jj = idx % kDiagBlock;
        if (jj <= m) Lc[trsm_col_off(jj) + (m - jj)] = Lkk[(long)m * ld + jj];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (long r = (long)blockIdx.x * warps + warp; r < rest; r += (long)gridDim.x * warps) {
        double2* row = L + (k0 + kDiagBlock + r) * ld + k0;
        double2 a[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) a[s] = row[lane + 32 * s];
#pragma unroll
        for (int sj = 0; sj < 4; ++sj) {
#pragma unroll 1
            for (int jl = 0; jl < 32; ++jl) {
                const int j = 32 * sj + jl;
                double2 x = a[sj];
                if (lane == jl) x = cdiv_smith(a[sj], Lc[trsm_col_off(j)]);
                x.x = __shfl_sync(0xffffffffu, x.x, jl);
                x.y = __shfl_sync(0xffffffffu, x.y, jl);
                if (lane == jl) a[sj] = x;
                const double2* col = Lc + trsm_col_off(j) - j;  // col[m] = L_kk[m][j], m >= j
#pragma unroll
                for (int s = sj; s < 4; ++s) {
                    const int m = lane + 32 * s;
                    if (m > j) a[s] = csub(a[s], cmul(x, col[m]));
                }
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) row[lane + 32 * s] = a[s];
    }
}

// ---- trailing update (the SYRK step): S(i, l) -= sum_m P(i, m) P(l, m) for
// the lower triangle of the trailing matrix, P the b = 128 columns of the
// solved panel (complex symmetric: no conjugation), on the FP64 tensor cores.
// One CTA (4 warps) per 64 x 64 tile of the lower triangle, grid-strided; a
// warp owns a 32 x 32 quarter as 4 x 4 complex 8 x 8 blocks, each the four real
// products (re re, -im im, re im, im re) of m8n8k4 fragments that share one
// 16-byte load of the real and imaginary parts.  Stages of 16 complex columns
// of both tiles' panel rows (16 KB each, 16-byte chunks XOR-swizzled by the row
// so that the fragment loads hit every bank once per four lanes) come three
// deep through cp.async.  Diagonal tiles leave their upper part (zero) alone.
constexpr int kSyT = 64, kSyK = 16, kSyStages = 3, kSyThreads = 128;
constexpr size_t kSyStageBytes = 2 * (size_t)kSyT * kSyK * 16;
constexpr size_t syrk_smem_bytes() { return kSyStages * kSyStageBytes; }

__global__ void __launch_bounds__(kSyThreads, 2) k_chol_syrk(double2* __restrict__ L, long ld, long k0, long t0,
                                                             int nt) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int g = lane >> 2, q = lane & 3, wi = w >> 1, wj = w & 1;
    constexpr int chunks = kDiagBlock / kSyK;
    const long ntiles = (long)nt * (nt + 1) / 2;
    // tile index -> (I, J), I >= J, and its first rows / columns
    auto corner = [&](long tile, long& r0, long& c0, bool& diag) {
        long I = (long)((sqrt(8.0 * (double)tile + 1.0) - 1.0) * 0.5);
        while ((I + 1) * (I + 2) / 2 <= tile) ++I;
        while (I * (I + 1) / 2 > tile) --I;
        const long J = tile - I * (I + 1) / 2;
        r0 = t0 + I * kSyT;
        c0 = t0 + J * kSyT;
        diag = I == J;
    };
    // chunk t of the tile at (r0, c0) into the stage buffer of the n-th chunk
    // this CTA stages (chunks are consumed in the order they are staged)
    int staged = 0;
    auto stage = [&](long r0, long c0, int t) {
        unsigned char* sb = smem + (staged++ % kSyStages) * kSyStageBytes;
        const long kb = k0 + (long)t * kSyK;
#pragma unroll
        for (int c = tid; c < 2 * kSyT * kSyK; c += kSyThreads) {
            const int half = c / (kSyT * kSyK), rr = (c % (kSyT * kSyK)) / kSyK, e = c % kSyK;
            const double2* src = L + ((half ? c0 : r0) + rr) * ld + kb + e;
            cpa16(sb + half * (kSyT * kSyK * 16) + rr * (kSyK * 16) + ((e ^ (rr & 7)) << 4), src);
        }
        cpa_commit();
    };
    long tile = blockIdx.x;
    if (tile >= ntiles) return;
    long r0, c0;
    bool diag;
    corner(tile, r0, c0, diag);
    stage(r0, c0, 0);
    stage(r0, c0, 1);
    int consumed = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        // the next tile's first chunks are staged during this tile's last ones
        const long next = tile + gridDim.x;
        long nr0 = 0, nc0 = 0;
        bool ndiag = false;
        if (next < ntiles) corner(next, nr0, nc0, ndiag);
        double acc[4][4][2][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) acc[a][b][c][0] = acc[a][b][c][1] = 0.0;
#pragma unroll 1
        for (int t = 0; t < chunks; ++t) {
            if (t + 2 < chunks) stage(r0, c0, t + 2);
            else if (next < ntiles) stage(nr0, nc0, t + 2 - chunks);
            else cpa_commit();
            cpa_wait<2>();
            __syncthreads();
            const unsigned char* sa = smem + (consumed++ % kSyStages) * kSyStageBytes;
            const unsigned char* sbb = sa + kSyT * kSyK * 16;
#pragma unroll
            for (int ks = 0; ks < kSyK / 4; ++ks) {
                const int e = 4 * ks + q;
                double2 af[4], bf[4];
#pragma unroll
                for (int mi = 0; mi < 4; ++mi) {
                    const int row = 32 * wi + 8 * mi + g;
                    af[mi] = *reinterpret_cast<const double2*>(sa + row * (kSyK * 16) + ((e ^ (row & 7)) << 4));
                }
#pragma unroll
                for (int nj = 0; nj < 4; ++nj) {
                    const int row = 32 * wj + 8 * nj + g;
                    bf[nj] = *reinterpret_cast<const double2*>(sbb + row * (kSyK * 16) + ((e ^ (row & 7)) << 4));
                }
                // the four real products in four sweeps over the 16 blocks, so
                // that products into one accumulator are 32 instructions apart
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int nj = 0; nj < 4; ++nj)
                        dmma(acc[mi][nj][0][0], acc[mi][nj][0][1], af[mi].x, bf[nj].x);  // re re
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int nj = 0; nj < 4; ++nj)
                        dmma(acc[mi][nj][1][0], acc[mi][nj][1][1], af[mi].x, bf[nj].y);  // re im
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int nj = 0; nj < 4; ++nj)
                        dmma(acc[mi][nj][0][0], acc[mi][nj][0][1], af[mi].y, -bf[nj].y);  // - im im
#pragma unroll
                for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                    for (int nj = 0; nj < 4; ++nj)
                        dmma(acc[mi][nj][1][0], acc[mi][nj][1][1], af[mi].y, bf[nj].x);  // im re
            }
            __syncthreads();  // the stage is read by every warp before it is refilled
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int nj = 0; nj < 4; ++nj) {
                const long row = r0 + 32 * wi + 8 * mi + g;
                const long col = c0 + 32 * wj + 8 * nj + 2 * q;
                double2* p = L + row * ld + col;
#pragma unroll
                for (int d = 0; d < 2; ++d)
                    if (!diag || col + d <= row)
                        p[d] = make_double2(p[d].x - acc[mi][nj][0][d], p[d].y - acc[mi][nj][1][d]);
            }
        r0 = nr0;
        c0 = nc0;
        diag = ndiag;
    }
}


// P[chunk][row][c] = sum over the chunk's columns k of L(row, k) X(k, c):
// complex L times RP = 8 NT real right-hand sides on the FP64 tensor cores.
// One CTA (4 warps) per (row strip, chunk) unit, grid-strided.  A stage holds
// 128 rows x 16 complex columns of L (32 KB, each row's 16-byte chunks XOR-
// swizzled by bit 2 on odd rows so that the fragment loads of two rows hit
// disjoint banks) and 16 rows of X (padded rows); three stages in flight with
// cp.async.  Warp w owns complex rows 32w..32w+31 as four groups of eight;
// each group is two m-tiles, the real and the imaginary parts of L, which
// share one 16-byte fragment load and the B fragments, so that each thread
// ends with matching real and imaginary parts of its outputs.
template <int NT>
__global__ void __launch_bounds__(kTR, 2) k_chol_apply(const double2* __restrict__ L, const double* __restrict__ X,
                                                    double2* __restrict__ P, const int2* __restrict__ units,
                                                    int n_units, long n) {
    constexpr int RP = 8 * NT;
    constexpr int XS = apply_x_row_bytes<NT>();
    constexpr int SB = apply_stage_bytes<NT>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int g = lane >> 2, q = lane & 3;
    for (int u = blockIdx.x; u < n_units; u += gridDim.x) {
        const int2 wk = units[u];
        const long row0 = (long)wk.x * kTR;
        const long k0 = (long)wk.y * kTC;
        const long kend = min(k0 + kTC, min(n, row0 + kTR));  // columns past the strip's last row are zero
        const int nt = (int)((kend - k0) / kKT);               // n, kTR and kTC are multiples of kKT
        auto stage = [&](int t) {
            unsigned char* sl = smem + (t % kStages) * SB;
            unsigned char* sx = sl + kTR * kKT * 16;
            const long kb = k0 + (long)t * kKT;
#pragma unroll
            for (int j = 0; j < kKT; ++j) {
                const int c = tid + j * kTR;
                const int r = c / kKT, e = c % kKT;
                if (row0 + r < n) cpa16(sl + r * (kKT * 16) + ((e ^ ((r & 1) << 2)) << 4), L + (row0 + r) * n + kb + e);
            }
            for (int c = tid; c < kKT * RP / 2; c += kTR) {
                const int r = c / (RP / 2), e = c % (RP / 2);
                cpa16(sx + r * XS + e * 16, X + (kb + r) * RP + 2 * e);
            }
        };
        double dr[4][NT][2], di[4][NT][2];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int m = 0; m < NT; ++m) dr[j][m][0] = dr[j][m][1] = di[j][m][0] = di[j][m][1] = 0.0;
        stage(0);
        cpa_commit();
        if (nt > 1) stage(1);
        cpa_commit();
        for (int t = 0; t < nt; ++t) {
            cpa_wait<1>();  // stage t has landed (one later group may be in flight)
            __syncthreads();
            if (t + 2 < nt) stage(t + 2);  // into the buffer computed at t - 1
            cpa_commit();
            const unsigned char* sl = smem + (t % kStages) * SB;
            const unsigned char* sx = sl + kTR * kKT * 16;
#pragma unroll
            for (int ks = 0; ks < kKT / 4; ++ks) {
                const int k = 4 * ks + q;
                double b[NT];
#pragma unroll
                for (int m = 0; m < NT; ++m) b[m] = *reinterpret_cast<const double*>(sx + k * XS + (8 * m + g) * 8);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int a = 32 * w + 8 * j + g;
                    const double2 l = *reinterpret_cast<const double2*>(sl + a * (kKT * 16) + ((k ^ ((a & 1) << 2)) << 4));
#pragma unroll
                    for (int m = 0; m < NT; ++m) {
                        dmma(dr[j][m][0], dr[j][m][1], l.x, b[m]);
                        dmma(di[j][m][0], di[j][m][1], l.y, b[m]);
                    }
                }
            }
        }
        __syncthreads();  // every warp is done with the buffers before the next unit refills them
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const long row = row0 + 32 * w + 8 * j + g;
            if (row < n) {
                double2* p = P + ((long)wk.y * n + row) * RP;
#pragma unroll
                for (int m = 0; m < NT; ++m) {
                    p[8 * m + 2 * q] = make_double2(dr[j][m][0], di[j][m][0]);
                    p[8 * m + 2 * q + 1] = make_double2(dr[j][m][1], di[j][m][1]);
                }
            }
        }
    }
}

// Number of column chunks that hold entries of `row` (those up to the end of its strip).
__device__ __forceinline__ int chunks_of_row(long row, long n) {
    const long last = min(n, (row / kTR + 1) * kTR) - 1;
    return (int)(last / kTC) + 1;
}

// Real right-hand sides of a field, RP per site: X(i, k) = Re xi_k(i),
// X(i, t + k) = Im xi_k(i), zero beyond 2t.
__global__ void k_chol_gather_field(const double2* __restrict__ xi, double* __restrict__ X, long n, int t, int RP) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 2 * t; c < RP; ++c) X[i * RP + c] = 0.0;
    for (int k = 0; k < t; ++k) {
        const double2 v = xi[k * n + i];
        X[i * RP + k] = v.x;
        X[i * RP + t + k] = v.y;
    }
}

// xi_k = Y_k + i Y_{t+k}, Y = sum of the chunk partials in chunk order.
template <int t, int RP>
__global__ void k_chol_finish_field(const double2* __restrict__ P, double2* __restrict__ xi, long n, long np) {
    constexpr int R = 2 * t;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 y[R];
#pragma unroll
    for (int c = 0; c < R; ++c) y[c] = make_double2(0.0, 0.0);
    const int nc = chunks_of_row(i, np);
    for (int ch = 0; ch < nc; ++ch) {
        const double2* p = P + ((long)ch * np + i) * RP;
#pragma unroll
        for (int c = 0; c < R; ++c) y[c] = cadd(y[c], p[c]);
    }
#pragma unroll
    for (int k = 0; k < t; ++k) xi[k * n + i] = make_double2(y[k].x - y[t + k].y, y[k].y + y[t + k].x);
}

// The 16 unit normals of each site in the reference's draw order
// (field.h:2170-2173) for steps step .. step + nsteps - 1, 16 nsteps per site:
// X(i, 16 s + a) = n_a (xi_x), X(i, 16 s + 8 + a) = m_a (xi_y) of step + s.
__global__ void k_chol_noise_X(double* __restrict__ X, long n, uint64_t seed, uint64_t step, int nsteps) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int rp = 16 * nsteps;
    for (int st = 0; st < nsteps; ++st) {
        double z[16];
        langevin_normals<double>(seed, step + (uint64_t)st, (uint32_t)i, z);
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            X[i * rp + 16 * st + a] = z[2 * a];
            X[i * rp + 16 * st + 8 + a] = z[2 * a + 1];
        }
    }
}

// xi_x = sum_a (L n_a) lambda_a, xi_y = sum_a (L m_a) lambda_a: the
// correlated noise L (sum_a n_a lambda_a) of gfield::multiplyByCholesky,
// with the (linear) embedding applied after L.
// P holds rp right-hand sides per site; this step's 16 start at column off.
__global__ void k_chol_finish_noise(const double2* __restrict__ P, double2* __restrict__ xx, double2* __restrict__ xy,
                                    long n, long np, int rp, int off) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 y[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) y[c] = make_double2(0.0, 0.0);
    const int nc = chunks_of_row(i, np);
    for (int ch = 0; ch < nc; ++ch) {
        const double2* p = P + ((long)ch * np + i) * rp + off;
#pragma unroll
        for (int c = 0; c < 16; ++c) y[c] = cadd(y[c], p[c]);
    }
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        double re[8], im[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            re[a] = y[8 * f + a].x;
            im[a] = y[8 * f + a].y;
        }
        double2 mr[9], mi[9];
        embed_lambda_ref(re, mr);
        embed_lambda_ref(im, mi);
        double2* o = f == 0 ? xx : xy;
#pragma unroll
        for (int k = 0; k < 9; ++k) o[k * n + i] = make_double2(mr[k].x - mi[k].y, mr[k].y + mi[k].x);
    }
}

bool same_ctx(const jw_field* a, const jw_field* b) { return a && b && a->ctx == b->ctx; }

jw_status ensure_scratch(jw_context* c) {
    if (c->d_pos_scratch) return JW_OK;
    if (cudaMalloc(&c->d_pos_scratch, sizeof(double2) * 18 * (size_t)c->N * c->N) != cudaSuccess) {
        c->d_pos_scratch = nullptr;
        return JW_ENOMEM;
    }
    return JW_OK;
}

// The raw forward DFT of k_x(d), k_y(d) for (rr, coupling, kernel).
jw_status ensure_table(jw_context* c, int rr, int coupling, int kernel) {
    if (c->d_pos_tab && c->pos_key[0] == rr && c->pos_key[1] == coupling && c->pos_key[2] == kernel) return JW_OK;
    const int N = c->N;
    const long vol = (long)N * N;
    if (!c->d_pos_tab && cudaMalloc(&c->d_pos_tab, sizeof(double2) * 2 * vol) != cudaSuccess) {
        c->d_pos_tab = nullptr;
        return JW_ENOMEM;
    }
    std::vector<double2> h(2 * vol);
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
            double kx, ky;
            position_kernel_host(x, y, N, rr, coupling, kernel, &kx, &ky);
            h[(long)x * N + y] = make_double2(kx, 0.0);
            h[vol + (long)x * N + y] = make_double2(ky, 0.0);
        }
    // the previous table may still be read by work queued on the stream
    JW_CUDA(cudaStreamSynchronize(c->stream));
    c->pos_key[0] = c->pos_key[1] = c->pos_key[2] = -1;
    // on the context's stream: a synchronous cudaMemcpy from pageable memory can
    // return before its DMA lands and is not ordered with the (non-blocking)
    // stream, so the transform below could read a partly copied table
    JW_CUDA(cudaMemcpyAsync(c->d_pos_tab, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice, c->stream));
    JW_CUDA(fft2d_planes<double>(c->d_pos_tab, 2, N, 1, 1.0, c->tw, c->stream));
    c->pos_key[0] = rr;
    c->pos_key[1] = coupling;
    c->pos_key[2] = kernel;
    return JW_OK;
}

bool valid_coupling(int cp) {
    return cp == JW_SQRT_COUPLING_CONSTANT || cp == JW_NOISE_COUPLING_CONSTANT || cp == JW_HATTA_COUPLING_CONSTANT ||
           cp == JW_FIXED_COUPLING_CONSTANT;
}

int apply_grid(const void* fn, int smem, int units) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kTR, smem);
    return std::max(1, std::min(units, sms * std::max(per, 1)));
}

template <int NT>
jw_status launch_apply(const jw_cholesky* L, cudaStream_t s) {
    constexpr int smem = kStages * apply_stage_bytes<NT>();
    JW_CUDA(cudaFuncSetAttribute(k_chol_apply<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int grid = apply_grid((const void*)k_chol_apply<NT>, smem, L->n_units);
    k_chol_apply<NT><<<grid, kTR, smem, s>>>(L->d_L, L->d_X, L->d_P, L->d_units, L->n_units, L->np);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

void cholesky_free(jw_cholesky* L) {
    if (L->d_L) cudaFree(L->d_L);
    if (L->d_units) cudaFree(L->d_units);
    if (L->d_X) cudaFree(L->d_X);
    if (L->d_P) cudaFree(L->d_P);
    delete L;
}

// L applied to the unit normals of nsteps (1 or 2) consecutive Langevin
// steps from `step` in one pass over L (16 nsteps right-hand sides).
jw_status cholesky_noise_apply(jw_context* c, const jw_cholesky* L, uint64_t step, int nsteps) {
    const long n = L->n;
    k_chol_noise_X<<<blocks_for(n), kThreads, 0, c->stream>>>(L->d_X, n, c->cfg.seed, step, nsteps);
    JW_CUDA(cudaGetLastError());
    return nsteps == 2 ? launch_apply<4>(L, c->stream) : launch_apply<2>(L, c->stream);
}

// The correlated noise of step `which` (< nsteps) of the last apply into xi_x, xi_y.
jw_status cholesky_noise_finish(jw_context* c, const jw_cholesky* L, jw_field* xx, jw_field* xy, int nsteps,
                                int which) {
    const long n = L->n;
    k_chol_finish_noise<<<blocks_for(n), kThreads, 0, c->stream>>>(L->d_P, xx->d, xy->d, n, L->np, 16 * nsteps,
                                                                   16 * which);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

}  // namespace

namespace jw {
void position_release(jw_context* c) {
    for (jw_cholesky* L : c->choleskies) cholesky_free(L);
    c->choleskies.clear();
    if (c->d_pos_tab) cudaFree(c->d_pos_tab);
    if (c->d_pos_scratch) cudaFree(c->d_pos_scratch);

    c->d_pos_tab = nullptr;
    c->d_pos_scratch = nullptr;
}
}  // namespace jw

// =================================================================== C ABI

JW_EXPORT jw_status jw_prepare_A_and_B(jw_context* c, jw_field* A, jw_field* B, const jw_field* xi_x,
                                       const jw_field* xi_y, const jw_field* V, int rr, int coupling, int kernel) {
    JW_CHECK(c && same_ctx(A, B) && same_ctx(B, xi_x) && same_ctx(xi_x, xi_y) && same_ctx(xi_y, V) && A->ctx == c);
    JW_CHECK(A->t == 9 && B->t == 9 && xi_x->t == 9 && xi_y->t == 9 && V->t == 9);
    JW_CHECK(A != B && A != xi_x && A != xi_y && A != V && B != xi_x && B != xi_y && B != V);
    JW_CHECK(valid_coupling(coupling) && (kernel == JW_LINEAR_KERNEL || kernel == JW_SIN_KERNEL) && rr >= 0);
    jw_status s = ensure_scratch(c);
    if (!s) s = ensure_table(c, rr, coupling, kernel);
    if (s) return s;
    const int N = c->N;
    const long vol = (long)N * N;
    const double scale = 1.0 / std::sqrt((double)vol);
    double2* S1 = c->d_pos_scratch;
    double2* S2 = c->d_pos_scratch + 9 * vol;
    JW_CUDA(cudaMemcpyAsync(S1, xi_x->d, sizeof(double2) * 9 * vol, cudaMemcpyDeviceToDevice, c->stream));
    JW_CUDA(cudaMemcpyAsync(S2, xi_y->d, sizeof(double2) * 9 * vol, cudaMemcpyDeviceToDevice, c->stream));
    JW_CUDA(fft2d_planes<double>(S1, 18, N, 1, scale, c->tw, c->stream));
    k_pos_combine<<<blocks_for(vol), kThreads, 0, c->stream>>>(A->d, S1, S2, c->d_pos_tab, vol);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(fft2d_planes<double>(A->d, 9, N, 0, scale, c->tw, c->stream));
    k_pos_rotate<<<blocks_for(vol), kThreads, 0, c->stream>>>(S1, S2, V->d, xi_x->d, xi_y->d, vol);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(fft2d_planes<double>(S1, 18, N, 1, scale, c->tw, c->stream));
    k_pos_combine<<<blocks_for(vol), kThreads, 0, c->stream>>>(B->d, S1, S2, c->d_pos_tab, vol);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(fft2d_planes<double>(B->d, 9, N, 0, scale, c->tw, c->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_set_correlations_for_coupling_constant(jw_context* c, jw_field* corr) {
    JW_CHECK(c && corr && corr->ctx == c && corr->t == 1);
    const int N = c->N;
    const long vol = (long)N * N;
    const double w = std::pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    const double f = 4.0 * M_PI / (11.0 - 2.0 * 3.0 / 3.0);
    std::vector<double2> h(vol);
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
            // momenta::set (momenta.h:90-124)
            const double sx = std::sin(M_PI * x / (1.0 * N)), sy = std::sin(M_PI * y / (1.0 * N));
            const double ph2 = 4.0 * std::pow(sx, 2.0) + 4.0 * std::pow(sy, 2.0);
            const double cc = f / std::log(std::pow(w + std::pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2));
            h[(long)x * N + y] = make_double2(cc / std::sqrt((double)(N * N)), 0.0);
        }
    // stream-ordered, like every later use of corr on the context's stream
    JW_CUDA(cudaMemcpyAsync(corr->d, h.data(), sizeof(double2) * vol, cudaMemcpyHostToDevice, c->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_cholesky_decompose(jw_context* c, const jw_field* corr, jw_cholesky** out) {
    JW_CHECK(c && corr && corr->ctx == c && corr->t == 1 && out);
    *out = nullptr;
    const int N = c->N;
    const long n = (long)N * N;
    // the blocked factorisation and the apply tiles take orders that are
    // multiples of the diagonal block (above one block) and of the apply's
    // 16-column stage (up to one block); other orders are padded
    const long np = n <= kDiagBlock ? (n + kKT - 1) / kKT * kKT : (n + kDiagBlock - 1) / kDiagBlock * kDiagBlock;
    const size_t bytesL = sizeof(double2) * (size_t)np * np;
    int n_chunks = (int)((np + kTC - 1) / kTC);
    const size_t bytesX = sizeof(double) * (size_t)np * kMaxR;
    const size_t bytesP = sizeof(double2) * (size_t)n_chunks * np * kMaxR;
    size_t free_b = 0, total_b = 0;
    JW_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytesL + bytesX + bytesP + ((size_t)1 << 30) > free_b) return JW_ENOMEM;
    static bool configured = false;
    if (!configured) {
        JW_CUDA(cudaFuncSetAttribute(k_chol_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem_bytes()));
        JW_CUDA(cudaFuncSetAttribute(k_chol_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem_bytes()));
        JW_CUDA(cudaFuncSetAttribute(k_chol_syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)syrk_smem_bytes()));
        configured = true;
    }
    int dev = 0, sms = 0;
    JW_CUDA(cudaGetDevice(&dev));
    JW_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    jw_cholesky* L = new jw_cholesky();
    L->ctx = c;
    L->n = n;
    L->np = np;
    L->n_chunks = n_chunks;
    if (cudaMalloc(&L->d_L, bytesL) != cudaSuccess || cudaMalloc(&L->d_X, bytesX) != cudaSuccess ||
        cudaMalloc(&L->d_P, bytesP) != cudaSuccess) {
        cholesky_free(L);
        return JW_ENOMEM;
    }
    // apply work list, longest units first
    std::vector<int2> units;
    const long strips = (np + kTR - 1) / kTR;
    for (long s = 0; s < strips; ++s) {
        const long last = std::min(np, (s + 1) * kTR) - 1;
        for (long ch = 0; ch <= last / kTC; ++ch) units.push_back(make_int2((int)s, (int)ch));
    }
    auto work = [&](int2 u) { return std::min((long)(u.y + 1) * kTC, std::min(np, (long)(u.x + 1) * kTR)) - (long)u.y * kTC; };
    std::stable_sort(units.begin(), units.end(), [&](int2 a, int2 b) { return work(a) > work(b); });
    L->n_units = (int)units.size();
    if (cudaMalloc(&L->d_units, sizeof(int2) * units.size()) != cudaSuccess) {
        cholesky_free(L);
        return JW_ENOMEM;
    }
    auto fail = [&](jw_status s) {
        cudaStreamSynchronize(c->stream);
        cholesky_free(L);
        return s;
    };
    if (cudaMemcpyAsync(L->d_units, units.data(), sizeof(int2) * units.size(), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess)
        return fail(JW_ECUDA);
    // the right-hand-side rows past n stay zero: the noise and field kernels write rows < n only
    if (cudaMemsetAsync(L->d_X, 0, bytesX, c->stream) != cudaSuccess) return fail(JW_ECUDA);
    k_chol_fill<<<148 * 16, kThreads, 0, c->stream>>>(L->d_L, corr->d, N, n, np);
    if (cudaGetLastError() != cudaSuccess) return fail(JW_ECUDA);
    // right-looking blocked factorisation, b = 128: factor the diagonal block,
    // solve the panel below it, update the trailing lower triangle
    for (long k0 = 0; k0 < np; k0 += kDiagBlock) {
        const long b = std::min((long)kDiagBlock, np - k0);
        double2* Akk = L->d_L + k0 * np + k0;
        k_chol_diag<<<1, 1024, diag_smem_bytes(), c->stream>>>(Akk, np, (int)b);
        if (cudaGetLastError() != cudaSuccess) return fail(JW_ECUDA);
        const long rest = np - k0 - b;
        if (rest == 0) break;
        const long warps = kTrsmThreads / 32;
        k_chol_trsm<<<(unsigned)std::min((rest + warps - 1) / warps, (long)sms), kTrsmThreads, trsm_smem_bytes(),
                      c->stream>>>(L->d_L, np, k0, rest);
        const int nt = (int)(rest / kSyT);
        const long ntiles = (long)nt * (nt + 1) / 2;
        k_chol_syrk<<<(unsigned)std::min(ntiles, 2L * sms), kSyThreads, syrk_smem_bytes(), c->stream>>>(
            L->d_L, np, k0, k0 + b, nt);
        if (cudaGetLastError() != cudaSuccess) return fail(JW_ECUDA);
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(JW_ECUDA);
    c->choleskies.push_back(L);
    *out = L;
    return JW_OK;
}

JW_EXPORT jw_status jw_cholesky_destroy(jw_cholesky* L) {
    if (!L) return JW_OK;
    jw_context* c = L->ctx;
    cudaStreamSynchronize(c->stream);
    c->choleskies.erase(std::remove(c->choleskies.begin(), c->choleskies.end(), L), c->choleskies.end());
    cholesky_free(L);
    return JW_OK;
}

JW_EXPORT jw_status jw_cholesky_get(const jw_cholesky* L, double* host) {
    JW_CHECK(L && host);
    JW_CUDA(cudaStreamSynchronize(L->ctx->stream));
    // the n x n factor of S: the top-left block of the padded factor
    JW_CUDA(cudaMemcpy2D(host, sizeof(double2) * (size_t)L->n, L->d_L, sizeof(double2) * (size_t)L->np,
                         sizeof(double2) * (size_t)L->n, (size_t)L->n, cudaMemcpyDeviceToHost));
    return JW_OK;
}

JW_EXPORT jw_status jw_multiply_by_cholesky(jw_context* c, jw_field* xi, const jw_cholesky* L) {
    JW_CHECK(c && xi && xi->ctx == c && L && L->ctx == c);
    L->cached = false;  // d_P is about to hold this field's product
    const long n = L->n;
    const int RP = xi->t == 9 ? 24 : 8;
    k_chol_gather_field<<<blocks_for(n), kThreads, 0, c->stream>>>(xi->d, L->d_X, n, xi->t, RP);
    JW_CUDA(cudaGetLastError());
    jw_status s;
    if (xi->t == 9) {
        s = launch_apply<3>(L, c->stream);
        if (s) return s;
        k_chol_finish_field<9, 24><<<blocks_for(n), kThreads, 0, c->stream>>>(L->d_P, xi->d, n, L->np);
    } else {
        s = launch_apply<1>(L, c->stream);
        if (s) return s;
        k_chol_finish_field<1, 8><<<blocks_for(n), kThreads, 0, c->stream>>>(L->d_P, xi->d, n, L->np);
    }
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_reduce_hatta(jw_context* c, const jw_field* corr, jw_field* sum, jw_field* err, int xr,
                                    int yr) {
    JW_CHECK(c && same_ctx(corr, sum) && same_ctx(sum, err) && corr->ctx == c);
    JW_CHECK(corr->t == 1 && sum->t == 1 && err->t == 1 && sum != err && corr != sum && corr != err);
    JW_CHECK(xr >= 0 && xr < c->N && yr >= 0 && yr < c->N);
    k_reduce_hatta<<<1, 1, 0, c->stream>>>(corr->d, sum->d, err->d, (long)xr * c->N + yr);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_evolve_position(jw_context* c, jw_field* V, uint64_t step0, int n, int rr,
                                       const jw_cholesky* L) {
    JW_CHECK(c && V && V->ctx == c && V->t == 9 && n >= 0 && rr >= 0);
    for (jw_field* w : c->pos_work) JW_CHECK(V != w);
    const jw_config& cfg = c->cfg;
    const int coupling = cfg.CouplingChoice;
    JW_CHECK(valid_coupling(coupling));
    const bool correlated = coupling == JW_NOISE_COUPLING_CONSTANT;
    if (correlated) JW_CHECK(L && L->ctx == c);
    // work fields kept in the context: repeated calls allocate nothing
    jw_status s = JW_OK;
    for (int k = 0; k < 4 && !s; ++k)
        if (!c->pos_work[k]) s = jw_field_create(c, 9, &c->pos_work[k]);
    if (s) return s;
    jw_field *xx = c->pos_work[0], *xy = c->pos_work[1], *A = c->pos_work[2], *B = c->pos_work[3];
    // correlated noise: one pass over L serves two steps (32 right-hand sides),
    // halving the factor's HBM traffic per step.  The second step's noise stays
    // in L's partial products for the next step, in this call or the next one
    // (a driver that steps one at a time).  Each column's sum is the one a
    // single step would form, so the noise is the same bit for bit.
    for (int k = 0; k < n && s == JW_OK; ++k) {
        const uint64_t step = step0 + (uint64_t)k;
        if (correlated) {
            int which = 1;
            if (!(L->cached && L->cached_step == step && L->cached_seed == cfg.seed)) {
                s = cholesky_noise_apply(c, L, step, 2);
                which = 0;
            }
            L->cached = which == 0 && !s;
            L->cached_step = step + 1;
            L->cached_seed = cfg.seed;
            if (!s) s = cholesky_noise_finish(c, L, xx, xy, 2, which);
        } else {
            s = jw_generate_gaussian(c, xx, xy, step, 0);
        }
        if (!s) s = jw_prepare_A_and_B(c, A, B, xx, xy, V, rr, coupling, cfg.KernelChoice);
        if (!s) s = jw_update_uf(c, V, B, A, cfg.step);
    }
    return s;
}
