// jw_dropin.cu -- the call-for-call FP64 layer: device fields with the
// reference's semantics and one kernel per reference hot-path function.
//
// Device layout of a field: t planes of N*N double2 (plane k = component k,
// row-major x, y), i.e. structure of arrays, so that each 2-D transform works
// on contiguous planes and each per-site kernel reads every component with
// coalesced 16-byte accesses.  jw_field_set / jw_field_get convert from / to
// the reference's site-major layout (field.h:170-173).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "jw_internal.h"

using namespace jw;

namespace {

constexpr int kThreads = 256;
inline unsigned blocks_for(long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// ---- generate_gaussian (field.h:2116-2243) / _with_noise_coupling_constant (:2245-2365)
// step_ptr, when set, holds the step index instead of `step` (a step captured
// once in a CUDA graph and replayed reads its index there).
__global__ void k_generate_gaussian(double2* __restrict__ xx, double2* __restrict__ xy, int N, uint64_t seed,
                                    uint64_t step, const unsigned long long* __restrict__ step_ptr,
                                    int with_coupling) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    if (step_ptr) step = *step_ptr;
    double z[16];
    langevin_normals<double>(seed, step, (uint32_t)i, z);
    double f = 1.0;
    if (with_coupling) {
        // the coupling factor evaluated at the momentum index equal to the site index (field.h:2273)
        const double tmp = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
        const double tmp2 = 4.0 * 3.141592653589793 / (11.0 - 2.0 * 3.0 / 3.0);
        const double ph2 = phat2_d((int)(i / N), (int)(i % N), N);
        f = sqrt(tmp2 / log(pow(tmp + pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
    }
    double n[8], m[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        n[k] = (z[2 * k] * 1.0 + 0.0) * f;
        m[k] = (z[2 * k + 1] * 1.0 + 0.0) * f;
    }
    double2 a[9], b[9];
    embed_lambda_ref(n, a);
    embed_lambda_ref(m, b);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        xx[k * vol + i] = a[k];
        xy[k * vol + i] = b[k];
    }
}

// ---- setMVModel (field.h:683-757)
__global__ void k_set_mv_model(double2* __restrict__ f, int N, uint64_t seed, int slice, double sigma) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    double z[8], n[8];
    mv_normals<double>(seed, (uint32_t)slice, (uint32_t)i, z);
#pragma unroll
    for (int k = 0; k < 8; ++k) n[k] = z[k] * sigma + 0.0;
    double2 a[9];
    embed_lambda_ref(n, a);
#pragma unroll
    for (int k = 0; k < 9; ++k) f[k * vol + i] = a[k];
}

// ---- solvePoisson (field.h:867-877)
__global__ void k_solve_poisson(double2* __restrict__ f, int N, int t, double mass, double g) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double fac = -1.0 * g / (-phat2_d((int)(i / N), (int)(i % N), N) + mass * mass);
    for (int k = 0; k < t; ++k) f[k * vol + i] = cscale(f[k * vol + i], fac);
}

__device__ __forceinline__ void load9(const double2* __restrict__ p, long vol, long i, double2 m[9]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = p[k * vol + i];
}
__device__ __forceinline__ void store9(double2* __restrict__ p, long vol, long i, const double2 m[9]) {
#pragma unroll
    for (int k = 0; k < 9; ++k) p[k * vol + i] = m[k];
}
__device__ __forceinline__ void flag_status(int* flags, int status, const double2 m[9]) {
    int fl = (status != 0) ? JW_FLAG_NOCONV : 0;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        if (!isfinite(m[k].x) || !isfinite(m[k].y)) fl |= JW_FLAG_NAN;
    if (fl) atomicOr(flags, fl);
}

// ---- operator*= (field.h:337-365)
__global__ void k_mul_exp(double2* __restrict__ V, const double2* __restrict__ f, int N, int* flags) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    double2 a[9], b[9], c[9];
    load9(V, vol, i, a);
    load9(f, vol, i, b);
    const int st = expi_herm(b, 1.0);
    mul3(a, b, c);
    flag_status(flags, st, c);
    store9(V, vol, i, c);
}

// ---- prepare_A_local (field.h:1998-2075)
__global__ void k_prepare_A_local(double2* __restrict__ out, const double2* __restrict__ xx,
                                  const double2* __restrict__ xy, int N, int coupling, int kernel) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double pi = 3.141592653589793;
    const int ix = (int)(i / N), iy = (int)(i % N);
    int xw = ix, yw = iy;
    if (xw >= N / 2) xw -= N;
    if (yw >= N / 2) yw -= N;
    const double px = 2.0 * pi * xw / (1.0 * N), py = 2.0 * pi * yw / (1.0 * N);
    double2 E[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) E[k] = make_double2(0.0, 0.0);
    if (fabs(px * px + py * py) > 10e-9) {
        double cc = 1.0, kx, ky;
        if (kernel == JW_LINEAR_KERNEL) {
            if (coupling == JW_SQRT_COUPLING_CONSTANT)
                cc = 4.0 * pi / ((11.0 - 2.0 * 3.0 / 3.0) *
                                 log(pow(pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2) +
                                             pow(((px * px + py * py) * N * N) / 6.0 / 6.0, 1.0 / 0.2),
                                         0.2)));
            kx = -2.0 * pi * sqrt(cc) * px / (px * px + py * py);
            ky = -2.0 * pi * sqrt(cc) * py / (px * px + py * py);
        } else {
            const double ph2 = phat2_d(ix, iy, N);
            if (coupling == JW_SQRT_COUPLING_CONSTANT)
                cc = 4.0 * pi / ((11.0 - 2.0 * 3.0 / 3.0) *
                                 log(pow(pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2) +
                                             pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
            kx = -2.0 * pi * sqrt(cc) * sin(2.0 * pi * ix / (1.0 * N)) / ph2;
            ky = -2.0 * pi * sqrt(cc) * sin(2.0 * pi * iy / (1.0 * N)) / ph2;
        }
        // (0 + i kx) * xi_x + (0 + i ky) * xi_y
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double2 a = xx[k * vol + i], b = xy[k * vol + i];
            const double2 ca = make_double2(0.0 * a.x - kx * a.y, 0.0 * a.y + kx * a.x);
            const double2 cb = make_double2(0.0 * b.x - ky * b.y, 0.0 * b.y + ky * b.x);
            E[k] = cadd(ca, cb);
        }
    }
    store9(out, vol, i, E);
}

// ---- uxiulocal (field.h:1892-1933)
__global__ void k_uxiulocal(double2* __restrict__ ux, double2* __restrict__ uy, const double2* __restrict__ V,
                            const double2* __restrict__ xx, const double2* __restrict__ xy, int N) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    double2 a[9], b[9], t[9], e[9];
    load9(V, vol, i, a);
    load9(xx, vol, i, b);
    mul3(a, b, t);
    mul3_adj(t, a, e);
    store9(ux, vol, i, e);
    load9(xy, vol, i, b);
    mul3(a, b, t);
    mul3_adj(t, a, e);
    store9(uy, vol, i, e);
}

// ---- update_uf (field.h:1966-1996)
__global__ void k_update_uf(double2* __restrict__ V, const double2* __restrict__ B, const double2* __restrict__ A,
                            int N, double step, int* flags) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double se = sqrt(step);
    double2 v[9], b[9], c[9], t[9];
    load9(B, vol, i, b);
    load9(A, vol, i, c);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        b[k] = cscale(b[k], -se);
        c[k] = cscale(c[k], se);
    }
    int st = expi_herm(b, -1.0);
    st |= expi_herm(c, -1.0);
    load9(V, vol, i, v);
    mul3(b, v, t);
    mul3(t, c, v);
    flag_status(flags, st, v);
    store9(V, vol, i, v);
}

// ---- trace (field.h:1375-1432)
__global__ void k_trace(const double2* __restrict__ Vk, double2* __restrict__ corr, int N) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double v = 1.0 * N * N;
    // C_rr = sum_c a_rc conj(a_rc) is real: its imaginary part a.y a.x - a.x a.y
    // is exactly zero in the reference's arithmetic and is written as 0 here.
    double tr = 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double2 a = Vk[(r * 3 + c) * vol + i];
            const double ax = a.x / v, ay = a.y / v;
            s = s + __dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay));
        }
        tr = tr + s;
    }
    corr[i] = make_double2(tr, 0.0);
}

// ---- average_and_symmetrize (field.h:1460-1492), two phases through a scratch plane
__global__ void k_symmetrize_xy(const double2* __restrict__ c, double2* __restrict__ tmp, int N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)N * N) return;
    const int x = (int)(i / N), y = (int)(i % N);
    const double2 a = c[i], b = c[(long)y * N + x];
    tmp[i] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
}
__global__ void k_symmetrize_pm(double2* __restrict__ c, const double2* __restrict__ tmp, int N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)N * N) return;
    const int x = (int)(i / N), y = (int)(i % N);
    const int a = (N - x) % N, b = (N - y) % N;
    const double2 s0 = tmp[(long)x * N + y], s1 = tmp[(long)a * N + y], s2 = tmp[(long)x * N + b],
                  s3 = tmp[(long)a * N + b];
    c[i] = make_double2(0.25 * (((s0.x + s1.x) + s2.x) + s3.x), 0.25 * (((s0.y + s1.y) + s2.y) + s3.y));
}

// ---- reduce (field.h:1521-1536): err += pow(c, 2.0) (a real square for real positive c)
__global__ void k_reduce(const double2* __restrict__ c, double2* __restrict__ sum, double2* __restrict__ err, int N) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)N * N) return;
    const double2 v = c[i];
    sum[i] = cadd(sum[i], v);
    double2 sq;
    if (v.y == 0.0 && v.x > 0.0) sq = make_double2(v.x * v.x, 0.0);
    else sq = cmul(v, v);
    err[i] = cadd(err[i], sq);
}

// (N^2/3) corr: the dipole's Wiener-Khinchin prefactor, into a scratch plane.
__global__ void k_dipole_scale(const double2* __restrict__ c, double2* __restrict__ out, long vol, double scale) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < vol) out[i] = cscale(c[i], scale);
}

__global__ void k_set_unit(double2* __restrict__ V, int N) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k * vol + i] = make_double2((k == 0 || k == 4 || k == 8) ? 1.0 : 0.0, 0.0);
}

bool same_ctx(const jw_field* a, const jw_field* b) { return a && b && a->ctx == b->ctx; }

}  // namespace

// =================================================================== C ABI

JW_EXPORT const char* jw_status_string(jw_status s) {
    switch (s) {
        case JW_OK: return "ok";
        case JW_EINVAL: return "invalid argument";
        case JW_ENOMEM: return "out of memory";
        case JW_ECUDA: return "CUDA error";
        case JW_ENOCONV: return "eigensolver did not converge";
        case JW_ENAN: return "non-finite value";
        case JW_ETIMEOUT: return "timed out";
        case JW_EUNSUPPORTED: return "unsupported option";
        case JW_ENOTFOUND: return "not found";
        case JW_EBUSY: return "busy";
        default: return "unknown status";
    }
}

JW_EXPORT jw_status jw_context_create(const jw_config* cfg, int device, jw_context** out) {
    JW_CHECK(cfg && out);
    *out = nullptr;
    if (cfg->Nx != cfg->Ny || !supported_n_fp64(cfg->Nx)) return JW_EUNSUPPORTED;
    JW_CUDA(cudaSetDevice(device));
    jw_context* c = new jw_context();
    c->cfg = *cfg;
    c->device = device;
    c->N = cfg->Nx;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        twiddles_create(c->N, &c->tw, c->stream) != cudaSuccess || cudaMalloc(&c->d_flags, sizeof(int)) != cudaSuccess ||
        cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream) != cudaSuccess ||
        cudaMalloc(&c->d_tmp, sizeof(double2) * (size_t)c->N * c->N) != cudaSuccess) {
        jw_context_destroy(c);
        return JW_ENOMEM;
    }
    *out = c;
    return JW_OK;
}

JW_EXPORT jw_status jw_context_destroy(jw_context* c) {
    if (!c) return JW_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (jw_field* f : c->fields) {
        cudaFree(f->d);
        delete f;
    }
    c->fields.clear();
    position_release(c);
    twiddles_destroy(&c->tw);
    if (c->d_flags) cudaFree(c->d_flags);
    if (c->d_tmp) cudaFree(c->d_tmp);
    if (c->d_step) cudaFree(c->d_step);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return JW_OK;
}

JW_EXPORT jw_status jw_context_sync(jw_context* c) {
    JW_CHECK(c);
    JW_CUDA(cudaStreamSynchronize(c->stream));
    int flags = 0;
    JW_CUDA(cudaMemcpy(&flags, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
    // on the stream: a legacy-stream memset is not ordered with later kernels
    if (flags) JW_CUDA(cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream));
    return flags_to_status(flags);
}

JW_EXPORT void* jw_context_stream(jw_context* c) { return c ? (void*)c->stream : nullptr; }

JW_EXPORT jw_status jw_field_create(jw_context* c, int t, jw_field** out) {
    JW_CHECK(c && out && (t == 1 || t == 9));
    *out = nullptr;
    jw_field* f = new jw_field();
    f->ctx = c;
    f->t = t;
    const size_t bytes = sizeof(double2) * (size_t)t * c->N * c->N;
    if (cudaMalloc(&f->d, bytes) != cudaSuccess) {
        delete f;
        return JW_ENOMEM;
    }
    JW_CUDA(cudaMemsetAsync(f->d, 0, bytes, c->stream));
    c->fields.push_back(f);
    *out = f;
    return JW_OK;
}

JW_EXPORT jw_status jw_field_destroy(jw_field* f) {
    if (!f) return JW_OK;
    jw_context* c = f->ctx;
    cudaStreamSynchronize(c->stream);
    cudaFree(f->d);
    c->fields.erase(std::remove(c->fields.begin(), c->fields.end(), f), c->fields.end());
    delete f;
    return JW_OK;
}

JW_EXPORT jw_status jw_field_set(jw_field* f, const double* host) {
    JW_CHECK(f && host);
    const long vol = (long)f->ctx->N * f->ctx->N;
    std::vector<double2> soa((size_t)f->t * vol);
    for (long i = 0; i < vol; ++i)
        for (int k = 0; k < f->t; ++k)
            soa[(size_t)k * vol + i] = make_double2(host[2 * (i * f->t + k)], host[2 * (i * f->t + k) + 1]);
    JW_CUDA(cudaMemcpyAsync(f->d, soa.data(), sizeof(double2) * soa.size(), cudaMemcpyHostToDevice, f->ctx->stream));
    JW_CUDA(cudaStreamSynchronize(f->ctx->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_field_get(const jw_field* f, double* host) {
    JW_CHECK(f && host);
    const long vol = (long)f->ctx->N * f->ctx->N;
    std::vector<double2> soa((size_t)f->t * vol);
    JW_CUDA(cudaMemcpyAsync(soa.data(), f->d, sizeof(double2) * soa.size(), cudaMemcpyDeviceToHost, f->ctx->stream));
    JW_CUDA(cudaStreamSynchronize(f->ctx->stream));
    for (long i = 0; i < vol; ++i)
        for (int k = 0; k < f->t; ++k) {
            host[2 * (i * f->t + k)] = soa[(size_t)k * vol + i].x;
            host[2 * (i * f->t + k) + 1] = soa[(size_t)k * vol + i].y;
        }
    return JW_OK;
}

namespace {
struct FieldFileHeader {
    char magic[8];  // "JWFIELD1"
    int32_t N;
    int32_t t;
};
constexpr char kFieldMagic[8] = {'J', 'W', 'F', 'I', 'E', 'L', 'D', '1'};
}  // namespace

JW_EXPORT jw_status jw_field_save(const jw_field* f, const char* path) {
    JW_CHECK(f && path);
    const long vol = (long)f->ctx->N * f->ctx->N;
    std::vector<double> h(2 * (size_t)f->t * vol);
    jw_status s = jw_field_get(f, h.data());
    if (s) return s;
    FieldFileHeader hd{};
    std::memcpy(hd.magic, kFieldMagic, 8);
    hd.N = f->ctx->N;
    hd.t = f->t;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return JW_EINVAL;
    bool ok = std::fwrite(&hd, sizeof hd, 1, fp) == 1 && std::fwrite(h.data(), sizeof(double), h.size(), fp) == h.size();
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? JW_OK : JW_EINVAL;
}

JW_EXPORT jw_status jw_field_load(jw_field* f, const char* path) {
    JW_CHECK(f && path);
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return JW_EINVAL;
    FieldFileHeader hd{};
    const long vol = (long)f->ctx->N * f->ctx->N;
    std::vector<double> h(2 * (size_t)f->t * vol);
    bool ok = std::fread(&hd, sizeof hd, 1, fp) == 1 && std::memcmp(hd.magic, kFieldMagic, 8) == 0 &&
              hd.N == f->ctx->N && hd.t == f->t && std::fread(h.data(), sizeof(double), h.size(), fp) == h.size();
    std::fclose(fp);
    if (!ok) return JW_EINVAL;
    return jw_field_set(f, h.data());
}

JW_EXPORT jw_status jw_field_copy(jw_field* dst, const jw_field* src) {
    JW_CHECK(same_ctx(dst, src) && dst->t == src->t);
    if (dst == src) return JW_OK;
    JW_CUDA(cudaMemcpyAsync(dst->d, src->d, sizeof(double2) * (size_t)dst->t * dst->ctx->N * dst->ctx->N,
                            cudaMemcpyDeviceToDevice, dst->ctx->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_field_set_unit(jw_field* f) {
    JW_CHECK(f && f->t == 9);
    const int N = f->ctx->N;
    k_set_unit<<<blocks_for((long)N * N), kThreads, 0, f->ctx->stream>>>(f->d, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_field_set_zero(jw_field* f) {
    JW_CHECK(f);
    JW_CUDA(cudaMemsetAsync(f->d, 0, sizeof(double2) * (size_t)f->t * f->ctx->N * f->ctx->N, f->ctx->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_execute2D(jw_context* c, jw_field* f, int dir) {
    JW_CHECK(c && f && f->ctx == c);
    const int N = c->N;
    const double scale = 1.0 / std::sqrt((double)((long)N * N));
    JW_CUDA(fft2d_planes<double>(f->d, f->t, N, dir, scale, c->tw, c->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_generate_gaussian(jw_context* c, jw_field* xx, jw_field* xy, uint64_t step_index,
                                         int with_coupling) {
    JW_CHECK(c && same_ctx(xx, xy) && xx->ctx == c && xx->t == 9 && xy->t == 9 && xx != xy);
    const int N = c->N;
    k_generate_gaussian<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(xx->d, xy->d, N, c->cfg.seed,
                                                                             step_index, nullptr, with_coupling);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

__global__ void k_set_counter(unsigned long long* p, unsigned long long v) { *p = v; }
__global__ void k_advance_counter(unsigned long long* p) { *p += 1; }

JW_EXPORT jw_status jw_set_mv_model(jw_context* c, jw_field* f, int slice, double g, double mu, int ny_slices) {
    JW_CHECK(c && f && f->ctx == c && f->t == 9 && ny_slices > 0 && slice >= 0);
    const int N = c->N;
    const double sigma = g * mu / std::sqrt((double)ny_slices);
    k_set_mv_model<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(f->d, N, c->cfg.seed, slice, sigma);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_solve_poisson(jw_context* c, jw_field* f, double mass, double g) {
    JW_CHECK(c && f && f->ctx == c);
    const int N = c->N;
    k_solve_poisson<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(f->d, N, f->t, mass, g);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_mul_exp(jw_context* c, jw_field* V, const jw_field* f) {
    JW_CHECK(c && same_ctx(V, f) && V->ctx == c && V->t == 9 && f->t == 9 && V != f);
    const int N = c->N;
    k_mul_exp<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(V->d, f->d, N, c->d_flags);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_prepare_A_local(jw_context* c, jw_field* out, const jw_field* xx, const jw_field* xy,
                                       int coupling, int kernel) {
    JW_CHECK(c && same_ctx(out, xx) && same_ctx(xx, xy) && out->ctx == c);
    JW_CHECK(out->t == 9 && xx->t == 9 && xy->t == 9 && out != xx && out != xy);
    JW_CHECK(kernel == JW_LINEAR_KERNEL || kernel == JW_SIN_KERNEL);
    if (coupling != JW_SQRT_COUPLING_CONSTANT && coupling != JW_NOISE_COUPLING_CONSTANT) return JW_EUNSUPPORTED;
    const int N = c->N;
    k_prepare_A_local<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(out->d, xx->d, xy->d, N, coupling,
                                                                           kernel);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_uxiulocal(jw_context* c, jw_field* ux, jw_field* uy, const jw_field* V, const jw_field* xx,
                                 const jw_field* xy) {
    JW_CHECK(c && same_ctx(ux, uy) && same_ctx(uy, V) && same_ctx(V, xx) && same_ctx(xx, xy) && ux->ctx == c);
    JW_CHECK(ux->t == 9 && uy->t == 9 && V->t == 9 && xx->t == 9 && xy->t == 9);
    JW_CHECK(ux != uy && ux != V && ux != xx && ux != xy && uy != V && uy != xx && uy != xy);
    const int N = c->N;
    k_uxiulocal<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(ux->d, uy->d, V->d, xx->d, xy->d, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_update_uf(jw_context* c, jw_field* V, const jw_field* B, const jw_field* A, double step) {
    JW_CHECK(c && same_ctx(V, B) && same_ctx(B, A) && V->ctx == c && V->t == 9 && B->t == 9 && A->t == 9);
    JW_CHECK(V != A && V != B && step >= 0.0);
    const int N = c->N;
    k_update_uf<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(V->d, B->d, A->d, N, step, c->d_flags);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_trace(jw_context* c, const jw_field* Vk, jw_field* corr) {
    JW_CHECK(c && same_ctx(Vk, corr) && Vk->ctx == c && Vk->t == 9 && corr->t == 1);
    const int N = c->N;
    k_trace<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(Vk->d, corr->d, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_average_and_symmetrize(jw_context* c, jw_field* corr) {
    JW_CHECK(c && corr && corr->ctx == c && corr->t == 1);
    const int N = c->N;
    k_symmetrize_xy<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(corr->d, c->d_tmp, N);
    k_symmetrize_pm<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(corr->d, c->d_tmp, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_reduce(jw_context* c, const jw_field* corr, jw_field* sum, jw_field* err) {
    JW_CHECK(c && same_ctx(corr, sum) && same_ctx(sum, err) && corr->ctx == c);
    JW_CHECK(corr->t == 1 && sum->t == 1 && err->t == 1 && sum != err && corr != sum && corr != err);
    const int N = c->N;
    k_reduce<<<blocks_for((long)N * N), kThreads, 0, c->stream>>>(corr->d, sum->d, err->d, N);
    JW_CUDA(cudaGetLastError());
    return JW_OK;
}

JW_EXPORT jw_status jw_dipole(jw_context* c, const jw_field* corr, double* S_xy, double* S_bins, double* r_bins,
                              int* counts, int nbins_cap, int* nbins, double* Qs) {
    JW_CHECK(c && corr && corr->ctx == c && corr->t == 1);
    const int N = c->N;
    const long vol = (long)N * N;
    if (S_bins && nbins_cap < N / 2 + 1) return JW_EINVAL;
    k_dipole_scale<<<blocks_for(vol), kThreads, 0, c->stream>>>(corr->d, c->d_tmp, vol, (double)N * N / 3.0);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(fft2d_planes<double>(c->d_tmp, 1, N, 0, 1.0, c->tw, c->stream));
    std::vector<double2> h(vol);
    JW_CUDA(cudaMemcpyAsync(h.data(), c->d_tmp, sizeof(double2) * vol, cudaMemcpyDeviceToHost, c->stream));
    JW_CUDA(cudaStreamSynchronize(c->stream));
    dipole_bins(h.data(), N, S_xy, S_bins, r_bins, counts, nbins, Qs);
    return JW_OK;
}

JW_EXPORT jw_status jw_initial_condition(jw_context* c, jw_field* V) {
    JW_CHECK(c && V && V->ctx == c && V->t == 9);
    const jw_config& cfg = c->cfg;
    JW_CHECK(cfg.elementaryWilsonLines > 0);
    const double g = 1.0, mu = cfg.mu / c->N;
    JW_CHECK(V != c->mv_work);
    // the charge field is kept in the context: repeated calls allocate nothing
    jw_status s = JW_OK;
    if (!c->mv_work && (s = jw_field_create(c, 9, &c->mv_work))) return s;
    jw_field* f = c->mv_work;
    s = jw_field_set_unit(V);
    for (int i = 0; i < cfg.elementaryWilsonLines && s == JW_OK; ++i) {
        s = jw_set_mv_model(c, f, i, g, mu, cfg.elementaryWilsonLines);
        if (!s) s = jw_execute2D(c, f, 1);
        if (!s) s = jw_solve_poisson(c, f, cfg.mass * std::pow(g, 2.0) * mu, g);
        if (!s) s = jw_execute2D(c, f, 0);
        if (!s) s = jw_mul_exp(c, V, f);
    }
    return s;
}

JW_EXPORT jw_status jw_evolve_momentum(jw_context* c, jw_field* V, uint64_t step0, int n) {
    JW_CHECK(c && V && V->ctx == c && V->t == 9 && n >= 0);
    const jw_config& cfg = c->cfg;
    if (cfg.CouplingChoice == JW_HATTA_COUPLING_CONSTANT) return JW_EUNSUPPORTED;
    for (jw_field* w : c->mom_work) JW_CHECK(V != w);
    // work fields kept in the context: repeated calls allocate nothing
    jw_status s = JW_OK;
    for (int k = 0; k < 6 && !s; ++k)
        if (!c->mom_work[k]) s = jw_field_create(c, 9, &c->mom_work[k]);
    if (s) return s;
    jw_field *xx = c->mom_work[0], *xy = c->mom_work[1], *A = c->mom_work[2], *B = c->mom_work[3],
             *ux = c->mom_work[4], *uy = c->mom_work[5];
    const int with_coupling = cfg.CouplingChoice == JW_NOISE_COUPLING_CONSTANT;
    const int kc = cfg.CouplingChoice == JW_FIXED_COUPLING_CONSTANT ? JW_NOISE_COUPLING_CONSTANT : cfg.CouplingChoice;
    // one step in the reference's call order; from_counter: the noise index is
    // read from (and then advanced in) the context's device counter
    auto step = [&](uint64_t k, bool from_counter) -> jw_status {
        jw_status st = JW_OK;
        if (from_counter) {
            k_generate_gaussian<<<blocks_for((long)c->N * c->N), kThreads, 0, c->stream>>>(
                xx->d, xy->d, c->N, cfg.seed, 0, c->d_step, with_coupling);
            if (cudaGetLastError() != cudaSuccess) st = JW_ECUDA;
        } else {
            st = jw_generate_gaussian(c, xx, xy, step0 + k, with_coupling);
        }
        if (!st) st = jw_execute2D(c, xx, 1);
        if (!st) st = jw_execute2D(c, xy, 1);
        if (!st) st = jw_prepare_A_local(c, A, xx, xy, kc, cfg.KernelChoice);
        if (!st) st = jw_execute2D(c, A, 0);
        if (!st) st = jw_execute2D(c, xx, 0);
        if (!st) st = jw_execute2D(c, xy, 0);
        if (!st) st = jw_uxiulocal(c, ux, uy, V, xx, xy);
        if (!st) st = jw_execute2D(c, ux, 1);
        if (!st) st = jw_execute2D(c, uy, 1);
        if (!st) st = jw_prepare_A_local(c, B, ux, uy, kc, cfg.KernelChoice);
        if (!st) st = jw_execute2D(c, B, 0);
        if (!st) st = jw_update_uf(c, V, B, A, cfg.step);
        if (!st && from_counter) {
            k_advance_counter<<<1, 1, 0, c->stream>>>(c->d_step);
            if (cudaGetLastError() != cudaSuccess) st = JW_ECUDA;
        }
        return st;
    };
    // a short run (or no counter) goes call by call; a longer one runs its
    // first step directly and replays the others from one captured step
    if (n < 4) {
        for (int k = 0; k < n && s == JW_OK; ++k) s = step((uint64_t)k, false);
        return s;
    }
    if (!c->d_step && cudaMalloc(&c->d_step, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        c->d_step = nullptr;
    }
    s = step(0, false);
    if (s || !c->d_step) {
        for (int k = 1; k < n && s == JW_OK; ++k) s = step((uint64_t)k, false);
        return s;
    }
    k_set_counter<<<1, 1, 0, c->stream>>>(c->d_step, step0 + 1);
    JW_CUDA(cudaGetLastError());
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    JW_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const jw_status captured = step(0, true);
    const cudaError_t ended = cudaStreamEndCapture(c->stream, &graph);
    cudaError_t ce = (captured == JW_OK && ended == cudaSuccess) ? cudaGraphInstantiate(&exec, graph, 0)
                                                                  : cudaErrorUnknown;
    for (int k = 1; k < n && ce == cudaSuccess; ++k) ce = cudaGraphLaunch(exec, c->stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (captured != JW_OK) return captured;
    JW_CUDA(ended);
    JW_CUDA(ce);
    return JW_OK;
}

extern "C" jw_status jw_print_host(int N, int measurement, const double* sum, const double* err, double x,
                                   const char* fileroot);

JW_EXPORT jw_status jw_print(jw_context* c, int measurement, const jw_field* sum, const jw_field* err, double x,
                             const char* fileroot) {
    JW_CHECK(c && same_ctx(sum, err) && sum->ctx == c && sum->t == 1 && err->t == 1 && fileroot);
    const long vol = (long)c->N * c->N;
    std::vector<double> hs(2 * vol), he(2 * vol);
    jw_status s = jw_field_get(sum, hs.data());
    if (!s) s = jw_field_get(err, he.data());
    if (!s) s = jw_print_host(c->N, measurement, hs.data(), he.data(), x, fileroot);
    return s;
}
