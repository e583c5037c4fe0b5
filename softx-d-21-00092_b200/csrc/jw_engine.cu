// jw_engine.cu -- the batched engine: resident events grouped by lattice
// size, fused Langevin steps (jw_engine_kernels.cuh) launched per group over
// all requested events at once, CUDA-graph replay of a step, device-side
// dipole accumulation, and the jw_engine_* C ABI.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

#include "jw_engine_kernels.cuh"
#include "jw_mixed_kernels.cuh"
#include "jw_internal.h"

using namespace jw;

namespace {

constexpr int kCouplings = 4;  // indexed by JW_*_COUPLING_CONSTANT

struct Group {
    int N = 0;
    Twiddles tw;
    EventDev* d_ev = nullptr;        // device descriptors, one per slot
    std::vector<int> owner;          // event id per slot, -1 if free
    int* d_slots = nullptr;          // slot lists of the current call
    int slots_cap = 0;
    std::vector<int> h_slots;        // what d_slots holds
    unsigned char* ws = nullptr;     // workspace, ws_events events
    int ws_events = 0;
    double* k64[kCouplings] = {};    // kernel tables per coupling ([2][N*N])
    float* k32[kCouplings] = {};
    double* nf64 = nullptr;          // noise factor (NOISE coupling)
    float* nf32 = nullptr;
    int p2_cols = 0;                 // mixed pass 2 column-tile width (0: the default)
    bool tuned = false;              // the autotuner has run for this size
    int n_re = 0;                    // resident events whose kernel tables have real parts (LINEAR, position)
};

struct Event {
    int id = -1;
    int N = 0;
    int slot = -1;
    jw_event_desc desc{};
    double2* V = nullptr;
    double* acc = nullptr;
    double* k64 = nullptr;   // the event's own kernel tables (position space)
    float* k32 = nullptr;
};

// Per-event table bytes of a position-space event: [4][N*N] in FP64 and FP32
// (imaginary parts of the x and y tables, then their real parts).
size_t position_table_bytes(int N) { return (sizeof(double) + sizeof(float)) * 4 * (size_t)N * N; }

template <typename T> size_t step_ws_bytes(int N) { return sizeof(C2<T>) * 24 * (size_t)N * N; }
size_t meas_ws_bytes(int N) { return (sizeof(double2) * 9 + 2 * sizeof(double)) * (size_t)N * N; }
size_t mv_ws_bytes(int N) { return sizeof(double2) * 4 * (size_t)N * N; }

bool engine_supported(int precision, int N) {
    if (!supported_n(N)) return false;
    if (precision == JW_PRECISION_FP64 && N > 1024) return false;  // pass 3 row of 8 FP64 planes > 128 KB
    return true;
}

// prepare_A_local's kernel (field.h:1998-2075) for the SIN kernel, imaginary
// parts of K_x and K_y divided by N^2 (the two unitary transforms), into
// t64 / t32 ([2][N*N]); computed on the device when a group first needs it.
__global__ void k_kernel_table(double* __restrict__ t64, float* __restrict__ t32, int N, int coupling) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double pi = 3.141592653589793;
    const int ix = (int)(i / N), iy = (int)(i % N);
    int xx = ix, yy = iy;
    if (xx >= N / 2) xx -= N;
    if (yy >= N / 2) yy -= N;
    const double px = 2.0 * pi * xx / (1.0 * N), py = 2.0 * pi * yy / (1.0 * N);
    double kx = 0.0, ky = 0.0;
    if (fabs(px * px + py * py) > 10e-9) {
        const double inv = 1.0 / ((double)N * (double)N);
        const double ph2 = phat2_d(ix, iy, N);
        double cc = 1.0;
        if (coupling == JW_SQRT_COUPLING_CONSTANT)
            cc = 4.0 * pi / ((11.0 - 2.0 * 3.0 / 3.0) *
                             log(pow(pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2) + pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2),
                                     0.2)));
        kx = -2.0 * pi * sqrt(cc) * sin(2.0 * pi * ix / (1.0 * N)) / ph2 * inv;
        ky = -2.0 * pi * sqrt(cc) * sin(2.0 * pi * iy / (1.0 * N)) / ph2 * inv;
    }
    t64[i] = kx;
    t64[vol + i] = ky;
    t32[i] = (float)kx;
    t32[vol + i] = (float)ky;
}

// generate_gaussian_with_noise_coupling_constant's factor at the momentum
// index equal to the site index (field.h:2267-2273).
__global__ void k_noise_factor_table(double* __restrict__ t64, float* __restrict__ t32, int N) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const double tmp = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    const double tmp2 = 4.0 * 3.141592653589793 / (11.0 - 2.0 * 3.0 / 3.0);
    const double ph2 = phat2_d((int)(i / N), (int)(i % N), N);
    const double f = sqrt(tmp2 / log(pow(tmp + pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
    t64[i] = f;
    t32[i] = (float)f;
}


// The position kernel k_i(d) (positions.h:105-150, field.h:2402-2470) on the
// device for all d, as complex planes [2][N*N] (real parts), with the same
// expressions as the host copy in jw_position.cu.
__global__ void k_position_kernel(double2* __restrict__ out, int N, int rr, int coupling, int kernel) {
    const long vol = (long)N * N;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    const int dxi = (int)(i / N), dyi = (int)(i % N);
    const double pi = 3.141592653589793;
    double dx, dy, rrr;
    if (kernel == JW_SIN_KERNEL) {
        dx = 0.5 * N * sin(2.0 * pi * dxi / (1.0 * N)) / pi;
        dy = 0.5 * N * sin(2.0 * pi * dyi / (1.0 * N)) / pi;
        const double sx = N * sin(pi * dxi / (1.0 * N)) / pi, sy = N * sin(pi * dyi / (1.0 * N)) / pi;
        rrr = sx * sx + sy * sy;
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
    const double lambda = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    double sc = 1.0;
    if (coupling == JW_SQRT_COUPLING_CONSTANT || coupling == JW_HATTA_COUPLING_CONSTANT)
        sc = sqrt(4.0 * pi / ((11.0 - 2.0 * 3.0 / 3.0) *
                              log(pow(lambda + 1.26 / pow(6.0 * 6.0 * rrrmin / N / N, 1.0 / 0.2), 0.2))));
    double kx = 0.0, ky = 0.0;
    if (rrr > 10e-9) {
        kx = sc * dx / rrr;
        ky = sc * dy / rrr;
    }
    out[i] = make_double2(kx, 0.0);
    out[vol + i] = make_double2(ky, 0.0);
}

// prepare_A_and_B_local's kernel (field.h:2368-2519) as a multiplier in
// momentum space: the raw DFT of the real position kernel k_i(d)
// (positions.h:105-150); for the SIN kernel k_i is odd in d_i and even in the
// other coordinate, so the DFT is imaginary.  Stored like kernel_table:
// imag(DFT k_i) / N^2.
__global__ void k_position_table(const double2* __restrict__ dft, double* __restrict__ k64, float* __restrict__ k32,
                                 long n2, double inv) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n2) return;
    const double v = dft[i].y * inv, r = dft[i].x * inv;
    k64[i] = v;
    k32[i] = (float)v;
    // real parts after the imaginary ones (read only for kernels that have them)
    k64[n2 + i] = r;
    k32[n2 + i] = (float)r;
}

// One accumulator site of an event: acc[site] and the plane stride.
struct AccSite {
    const double* p;
    long vol;
};
__global__ void k_gather_acc(const AccSite* __restrict__ a, int n, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int q = 0; q < 4; ++q) out[4 * i + q] = a[i].p[q * a[i].vol];
}



// mean symmetrised correlator times N^2/3 as a complex plane (dipole S(r) input)
__global__ void k_dipole_prep(const double* __restrict__ acc, double2* __restrict__ out, long vol, double scale) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
    out[i] = make_double2((acc[i] + acc[vol + i]) * scale, 0.0);
}

__global__ void k_set_unit_planes(double2* V, long vol) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vol) return;
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k * vol + i] = make_double2((k == 0 || k == 4 || k == 8) ? 1.0 : 0.0, 0.0);
}

// reference layout (site-major, 9 interleaved) <-> planes
__global__ void k_aos_to_planes(const double2* __restrict__ aos, double2* __restrict__ V, long vol) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * vol) return;
    const long site = i / 9;
    const int k = (int)(i % 9);
    V[k * vol + site] = aos[i];
}
__global__ void k_planes_to_aos(const double2* __restrict__ V, double2* __restrict__ aos, long vol) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 9 * vol) return;
    const long site = i / 9;
    const int k = (int)(i % 9);
    aos[i] = V[k * vol + site];
}

}  // namespace

struct jw_engine {
    jw_engine_options opt{};
    int device = 0;
    cudaStream_t stream = nullptr;
    int* d_flags = nullptr;
    std::map<int, std::unique_ptr<Group>> groups;  // by N
    std::map<int, Event> events;                   // by id
    int next_id = 1;
    size_t bytes_in_use = 0;
    size_t budget = 0;
    double2* d_stage = nullptr;  // host-layout staging for set/get V
    size_t stage_bytes = 0;
    double2* h_pinned = nullptr;  // pinned host staging
    size_t pinned_bytes = 0;
    std::map<size_t, std::vector<void*>> pool;  // buffers of removed events, by size
    size_t pool_bytes = 0;
};

namespace {

template <typename T> int elem_size() { return (int)sizeof(C2<T>); }

size_t ws_per_event(const jw_engine* e, int N) {
    const size_t s = e->opt.precision == JW_PRECISION_MIXED ? step_ws_bytes<float>(N) : step_ws_bytes<double>(N);
    return std::max(std::max(s, meas_ws_bytes(N)), mv_ws_bytes(N));
}

// Event buffers (V, accumulators, tables) of removed events are kept by size
// for the next event of that size, so that a serving loop does not call
// cudaMalloc and cudaFree (which synchronise the device) per request.  The
// pool holds at most what the budget leaves free and is released when an
// allocation would otherwise fail.
void pool_release(jw_engine* e) {
    if (e->pool_bytes == 0) return;
    cudaStreamSynchronize(e->stream);
    for (auto& kv : e->pool)
        for (void* p : kv.second) cudaFree(p);
    e->pool.clear();
    e->pool_bytes = 0;
}

void* ev_alloc(jw_engine* e, size_t bytes) {
    auto it = e->pool.find(bytes);
    if (it != e->pool.end() && !it->second.empty()) {
        void* p = it->second.back();
        it->second.pop_back();
        e->pool_bytes -= bytes;
        return p;
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) == cudaSuccess) return p;
    cudaGetLastError();  // an allocation failure is not sticky: clear it
    pool_release(e);
    if (cudaMalloc(&p, bytes) == cudaSuccess) return p;
    cudaGetLastError();
    return nullptr;
}

// Stream-ordered reuse: every use of an event buffer is on the engine stream.
void ev_free(jw_engine* e, void* p, size_t bytes) {
    if (!p) return;
    if (e->bytes_in_use + e->pool_bytes + bytes <= e->budget) {
        e->pool[bytes].push_back(p);
        e->pool_bytes += bytes;
    } else {
        cudaFree(p);
    }
}

int chunk_size(const jw_engine* e, int count, int N);

// The workspace of a group grows geometrically (at least doubling), within
// the budget, so that admitting events one by one reallocates it rarely.
jw_status ensure_workspace(jw_engine* e, Group& g, int nev) {
    if (g.ws_events >= nev) return JW_OK;
    const size_t per = ws_per_event(e, g.N);
    const size_t old = per * (size_t)g.ws_events;
    int want = std::max(nev, 2 * g.ws_events);
    want = std::min(want, std::max(nev, chunk_size(e, 1 << 30, g.N)));
    if (e->bytes_in_use - old + per * (size_t)want > e->budget) want = nev;
    const size_t need = per * (size_t)want;
    if (e->bytes_in_use - old + need > e->budget) return JW_ENOMEM;
    JW_CUDA(cudaStreamSynchronize(e->stream));
    if (g.ws) cudaFree(g.ws);
    g.ws = nullptr;
    g.ws_events = 0;
    e->bytes_in_use -= old;
    if (cudaMalloc(&g.ws, need) != cudaSuccess) {
        cudaGetLastError();
        pool_release(e);
        if (cudaMalloc(&g.ws, need) != cudaSuccess) {
            cudaGetLastError();
            g.ws = nullptr;
            return JW_ENOMEM;
        }
    }
    g.ws_events = want;
    e->bytes_in_use += need;
    return JW_OK;
}

jw_status ensure_slots(Group& g, int n) {
    if (g.slots_cap >= n) return JW_OK;
    if (g.d_slots) cudaFree(g.d_slots);
    g.d_slots = nullptr;
    g.h_slots.clear();
    if (cudaMalloc(&g.d_slots, sizeof(int) * n) != cudaSuccess) return JW_ENOMEM;
    g.slots_cap = n;
    return JW_OK;
}

// The momentum-space kernel table of `coupling` (and, for NOISE, the noise
// factor), built on the device the first time an event of the group needs it.
jw_status ensure_tables(jw_engine* e, Group& g, int coupling) {
    const long vol = (long)g.N * g.N;
    const unsigned blocks = (unsigned)((vol + 255) / 256);
    if (!g.k64[coupling]) {
        if (cudaMalloc(&g.k64[coupling], sizeof(double) * 2 * vol) != cudaSuccess ||
            cudaMalloc(&g.k32[coupling], sizeof(float) * 2 * vol) != cudaSuccess) {
            if (g.k64[coupling]) cudaFree(g.k64[coupling]);
            g.k64[coupling] = nullptr;
            g.k32[coupling] = nullptr;
            return JW_ENOMEM;
        }
        k_kernel_table<<<blocks, 256, 0, e->stream>>>(g.k64[coupling], g.k32[coupling], g.N, coupling);
        JW_CUDA(cudaGetLastError());
    }
    if (coupling == JW_NOISE_COUPLING_CONSTANT && !g.nf64) {
        if (cudaMalloc(&g.nf64, sizeof(double) * vol) != cudaSuccess ||
            cudaMalloc(&g.nf32, sizeof(float) * vol) != cudaSuccess) {
            if (g.nf64) cudaFree(g.nf64);
            g.nf64 = nullptr;
            g.nf32 = nullptr;
            return JW_ENOMEM;
        }
        k_noise_factor_table<<<blocks, 256, 0, e->stream>>>(g.nf64, g.nf32, g.N);
        JW_CUDA(cudaGetLastError());
    }
    return JW_OK;
}

jw_status group_get(jw_engine* e, int N, Group** out) {
    auto it = e->groups.find(N);
    if (it != e->groups.end()) {
        *out = it->second.get();
        return JW_OK;
    }
    auto g = std::make_unique<Group>();
    g->N = N;
    JW_CUDA(twiddles_create(N, &g->tw, e->stream));
    *out = g.get();
    e->groups[N] = std::move(g);
    return JW_OK;
}

jw_status grow_slots(Group& g, cudaStream_t s) {
    const int old = (int)g.owner.size();
    const int cap = std::max(4, 2 * old);
    EventDev* d = nullptr;
    if (cudaMalloc(&d, sizeof(EventDev) * cap) != cudaSuccess) return JW_ENOMEM;
    JW_CUDA(cudaMemsetAsync(d, 0, sizeof(EventDev) * cap, s));
    if (g.d_ev) {
        JW_CUDA(cudaMemcpyAsync(d, g.d_ev, sizeof(EventDev) * old, cudaMemcpyDeviceToDevice, s));
        JW_CUDA(cudaStreamSynchronize(s));
        cudaFree(g.d_ev);
    }
    g.d_ev = d;
    g.owner.resize(cap, -1);
    return JW_OK;
}

void group_destroy(Group& g) {
    twiddles_destroy(&g.tw);
    if (g.d_ev) cudaFree(g.d_ev);
    if (g.d_slots) cudaFree(g.d_slots);
    if (g.ws) cudaFree(g.ws);
    for (int c = 0; c < kCouplings; ++c) {
        if (g.k64[c]) cudaFree(g.k64[c]);
        if (g.k32[c]) cudaFree(g.k32[c]);
    }
    if (g.nf64) cudaFree(g.nf64);
    if (g.nf32) cudaFree(g.nf32);
}

// --------------------------------------------------------------- launches
// Kernel kinds of a timed run (jw_engine_step_timed's kernel_ms order).
enum { KIND_P1 = 0, KIND_P2 = 1, KIND_P3 = 2, KIND_P31 = 3, KIND_COUNT = 4 };

// CUDA events around launches, for jw_engine_step_timed.
struct LaunchTimes {
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ev;  // start, end of each timed launch
    std::vector<int> kind;
    void start(int k) {
        cudaEvent_t a = nullptr;
        cudaEventCreate(&a);
        cudaEventRecord(a, stream);
        ev.push_back(a);
        kind.push_back(k);
    }
    void stop() {
        cudaEvent_t b = nullptr;
        cudaEventCreate(&b);
        cudaEventRecord(b, stream);
        ev.push_back(b);
    }
    ~LaunchTimes() {
        for (cudaEvent_t x : ev) cudaEventDestroy(x);
    }
};

// The persistent column pass with tensor-memory-accelerator tile moves
// (k_mix_pass2_tma, mx_t2_cols<N>() columns per tile: 8 up to 512^2, 4 at
// 1024^2) is tuning choice kP2Tma + that width (24 or 20) beside the tile
// widths 1, 2, 4 and 8 of k_mix_pass2; 16 stands for it.
constexpr int kP2Tma = 16;


// cuTensorMapEncodeTiled through the runtime's driver entry points (no link
// against libcuda); null when the driver does not provide it.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// The radix schedule of the column transforms is part of the choice: choice
// c + kRadixFirst (c one of the above) runs the column transforms with the
// radix-2 or radix-4 pass first (fft_radix, schedule 1), for the sizes that
// have one (N = 16, 32, 128, 256, 1024, 2048).  Schedule 1 rounds differently,
// so it is tuned only with jw_engine_options.autotune = 2 and a run's lattices
// depend on the recorded choice (jw_engine_tuning / jw_engine_set_tuning).
constexpr int kRadixFirst = 32;

// f(std::integral_constant<int, C>) for every valid pass-2 tuning choice C.
template <int N, int S, typename F>
void for_each_p2_cols_s(F&& f) {
    constexpr int B = S * kRadixFirst;
    if constexpr (mx_s2_valid<N, 1>()) f(std::integral_constant<int, B + 1>{});
    if constexpr (mx_s2_valid<N, 2>()) f(std::integral_constant<int, B + 2>{});
    if constexpr (mx_s2_valid<N, 4>()) f(std::integral_constant<int, B + 4>{});
    if constexpr (mx_s2_valid<N, 8>()) f(std::integral_constant<int, B + 8>{});
    if constexpr (mx_t2_valid<N, mx_t2_cols<N>()>())
        if (encode_tiled()) f(std::integral_constant<int, B + kP2Tma + mx_t2_cols<N>()>{});
}
template <int N, typename F>
void for_each_p2_cols(F&& f) {
    for_each_p2_cols_s<N, 0>(f);
    if constexpr (fft_has_rem<N>()) for_each_p2_cols_s<N, 1>(f);
}

// Pair planes of a launch group ([planes nb N rows][4 N floats]: P has 8
// planes per event, Q 4) as a 2D tensor with boxes of C float4 elements (C = 8:
// 128 bytes; 4 columns at 1024^2) by min(N, 256) rows, no swizzle (dense
// boxes).  L2 promotion is the box row (128 bytes, or 64 bytes for 4-column
// tiles, which at 128 bytes read 2.1x the algorithmic bytes): with 256-byte
// promotion every row fetched the neighbouring tile's half line too, which the
// column pass reads much later (measured 1.5x the algorithmic DRAM reads).
template <int N, int C>
bool p2_tensor_map(CUtensorMap* map, float4* P, int nb, int planes = 8) {
    const cuuint64_t dims[2] = {(cuuint64_t)4 * N, (cuuint64_t)planes * nb * N};
    const cuuint64_t strides[1] = {(cuuint64_t)4 * N * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)(4 * C), (cuuint32_t)(N < 256 ? N : 256)};
    const cuuint32_t estr[2] = {1, 1};
    return encode_tiled()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, P, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          C >= 8 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_L2_64B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// CTAs of the persistent column pass: every SM filled to its occupancy.
template <int N, int C, int S>
int p2_tma_grid() {
    static int grid = 0;
    if (grid == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mix_pass2_tma<N, C, S>, mx_t2_threads<N, C>(),
                                                      mx_t2_smem<N, C, S>());
        grid = std::max(1, sms * std::max(1, per_sm));
    }
    return grid;
}

// Pass 2 with tuning choice `cols` (0: the default); advance = 0 leaves the
// step index alone (timing launches of the autotuner).
template <int N>
void launch_pass2(jw_engine* e, Group& g, const int* d_slots, int nb, int cols, int advance) {
    const long vol = (long)N * N;
    float4* P = reinterpret_cast<float4*>(g.ws);
    float4* Q = P + (size_t)8 * vol * nb;
    // the default: the persistent TMA form where it is built (measured fastest
    // at 256^2, 512^2 and 1024^2), else the tile width mx_s2_cols
    constexpr int kTma = kP2Tma + mx_t2_cols<N>();
    if (cols == 0) cols = (mx_t2_valid<N, mx_t2_cols<N>()>() && encode_tiled()) ? kTma : mx_s2_cols<N>();
    if (cols == kP2Tma) cols = kTma;
    if (cols == kRadixFirst + kP2Tma) cols = kRadixFirst + kTma;
    for_each_p2_cols<N>([&](auto c) {
        constexpr int CS = decltype(c)::value;
        if (CS != cols) return;
        constexpr int S = CS >= kRadixFirst ? 1 : 0;
        constexpr int C = CS - S * kRadixFirst;
        if constexpr (C > kP2Tma) {
            constexpr int TC = C - kP2Tma;
            CUtensorMap pmap, qmap;
            if (!p2_tensor_map<N, TC>(&pmap, P, nb) || !p2_tensor_map<N, TC>(&qmap, Q, nb, 4)) {
                // no tensor map for these planes: the classic form of the default width
                constexpr int CC = mx_s2_cols<N>();
                k_mix_pass2<N, CC, S><<<dim3(N / CC, 4, nb), mx_s2_threads<N, CC>(), mx_s2_smem<N, CC>(),
                                        e->stream>>>(g.d_ev, d_slots, P, Q, g.tw.d32, advance);
                return;
            }
            const int grid = std::min(p2_tma_grid<N, TC, S>(), nb * 4 * (N / TC));
            // the form that reads real table parts only for groups holding such events
            if (g.n_re > 0)
                k_mix_pass2_tma<N, TC, S, true><<<grid, mx_t2_threads<N, TC>(), mx_t2_smem<N, TC, S>(), e->stream>>>(
                    g.d_ev, d_slots, g.tw.d32, nb, advance, e->d_flags, pmap, qmap);
            else
                k_mix_pass2_tma<N, TC, S><<<grid, mx_t2_threads<N, TC>(), mx_t2_smem<N, TC, S>(), e->stream>>>(
                    g.d_ev, d_slots, g.tw.d32, nb, advance, e->d_flags, pmap, qmap);
        } else {
            k_mix_pass2<N, C, S><<<dim3(N / C, 4, nb), mx_s2_threads<N, C>(), mx_s2_smem<N, C>(), e->stream>>>(
                g.d_ev, d_slots, P, Q, g.tw.d32, advance);
        }
    });
}

template <int N>
void mix_configure() {
    static bool configured = false;
    if (configured) return;
    if constexpr (mx_pair<N>()) {
        cudaFuncSetAttribute(k_mix_pass1_pair<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_p1_smem<N>());
        cudaFuncSetAttribute(k_mix_pass31_pair<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mx_p31p_smem<N>());
        if constexpr (N == 2048)
            cudaFuncSetAttribute(k_mix_pass31_quad<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mx_p31q_smem<N>());
    } else {
        cudaFuncSetAttribute(k_mix_pass1<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_p1_smem<N>());
        cudaFuncSetAttribute(k_mix_pass31<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_p31_smem<N>());
    }
    for_each_p2_cols<N>([](auto c) {
        constexpr int CS = decltype(c)::value;
        constexpr int S = CS >= kRadixFirst ? 1 : 0;
        constexpr int C = CS - S * kRadixFirst;
        if constexpr (C > kP2Tma) {
            cudaFuncSetAttribute(k_mix_pass2_tma<N, C - kP2Tma, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mx_t2_smem<N, C - kP2Tma, S>());
            cudaFuncSetAttribute(k_mix_pass2_tma<N, C - kP2Tma, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mx_t2_smem<N, C - kP2Tma, S>());
        } else
            cudaFuncSetAttribute(k_mix_pass2<N, C, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)mx_s2_smem<N, C>());
    });
    cudaFuncSetAttribute(k_mix_pass3<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_p3_smem<N>());
    if constexpr (mx_p3_meas_fits<N>())
        cudaFuncSetAttribute(k_mix_pass3<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mx_p3_smem<N, true>());
    cudaFuncSetAttribute(k_meas32_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mx_p2_smem<N>());
    configured = true;
}

// One mixed-precision kernel of a launch group.  The workspace holds P (8 pair
// planes per event) and then Q (4 pair planes per event); the measuring pass 3
// writes its 5 row-transformed planes where P was.
template <int N>
void mix_launch(jw_engine* e, Group& g, const int* d_slots, int nb, int kind, bool meas, LaunchTimes* tm) {
    const long vol = (long)N * N;
    float4* P = reinterpret_cast<float4*>(g.ws);
    float4* Q = P + (size_t)8 * vol * nb;
    if (tm) tm->start(kind);
    switch (kind) {
        case KIND_P1:
            if constexpr (mx_pair<N>())
                k_mix_pass1_pair<N><<<dim3(N, 2, nb), mx_p1_threads<N>(), mx_p1_smem<N>(), e->stream>>>(
                    g.d_ev, d_slots, P, g.tw.d32);
            else
                k_mix_pass1<N><<<dim3(N, 1, nb), mx_p1_threads<N>(), mx_p1_smem<N>(), e->stream>>>(
                    g.d_ev, d_slots, P, g.tw.d32);
            break;
        case KIND_P2:
            launch_pass2<N>(e, g, d_slots, nb, g.p2_cols, 1);
            break;
        case KIND_P3:
            if constexpr (mx_p3_meas_fits<N>()) {
                if (meas) {
                    k_mix_pass3<N, true><<<dim3(N, nb), mx_p3_threads<N>(), mx_p3_smem<N, true>(), e->stream>>>(
                        g.d_ev, d_slots, Q, g.tw.d32, e->d_flags, P);
                    break;
                }
            }
            k_mix_pass3<N><<<dim3(N, nb), mx_p3_threads<N>(), mx_p3_smem<N>(), e->stream>>>(g.d_ev, d_slots, Q,
                                                                                            g.tw.d32, e->d_flags,
                                                                                            nullptr);
            break;
        case KIND_P31:
            if constexpr (N == 2048)  // four-CTA clusters, two CTAs per SM
                k_mix_pass31_quad<N><<<dim3(N, 4, nb), kQuadThreads, mx_p31q_smem<N>(), e->stream>>>(
                    g.d_ev, d_slots, Q, P, g.tw.d32, e->d_flags);
            else if constexpr (mx_pair<N>())
                k_mix_pass31_pair<N><<<dim3(N, 2, nb), mx_p31_threads<N>(), mx_p31p_smem<N>(), e->stream>>>(
                    g.d_ev, d_slots, Q, P, g.tw.d32, e->d_flags);
            else
                k_mix_pass31<N><<<dim3(N, nb), mx_p31_threads<N>(), mx_p31_smem<N>(), e->stream>>>(
                    g.d_ev, d_slots, Q, P, g.tw.d32, e->d_flags);
            break;
        default:
            break;
    }
    if (tm) tm->stop();
}

// nsteps >= 1 mixed steps of one launch group: pass 1, then nsteps - 1 times
// (pass 2, pass 3 + next pass 1), then pass 2 and pass 3.  From 1024^2 on,
// passes 1 and 3 + 1 run as two-CTA clusters per lattice row.
// With ens the last pass 3 also row-transforms the new V, and the column pass
// and the ensemble reduction into ens follow (the same result as the steps
// followed by launch_measure_ensemble).  The middle is captured once as a CUDA
// graph and replayed when it repeats and nothing is timed.  Launch groups that
// share the workspace run one after another, each through all its steps.
// The autotuner: every valid pass-2 tile width runs 1 + 3 times on this launch
// group's workspace (the step index frozen; pass 2 only maps P to Q, which the
// run then recomputes), and the fastest by CUDA events is kept for the size.
// With autotune = 2 the radix-first schedules (kRadixFirst) compete too.
template <int N>
cudaError_t tune_mix(jw_engine* e, Group& g, const int* d_slots, int nb) {
    float best = 0.0f;
    int best_cols = 0;
    cudaError_t ce = cudaSuccess;
    for_each_p2_cols<N>([&](auto c) {
        constexpr int C = decltype(c)::value;
        if (ce != cudaSuccess) return;
        if (C >= kRadixFirst && e->opt.autotune < 2) return;  // results must not depend on the choice
        cudaEvent_t a = nullptr, b = nullptr;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        launch_pass2<N>(e, g, d_slots, nb, C, 0);
        cudaEventRecord(a, e->stream);
        for (int r = 0; r < 3; ++r) launch_pass2<N>(e, g, d_slots, nb, C, 0);
        cudaEventRecord(b, e->stream);
        ce = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (ce == cudaSuccess && (best_cols == 0 || ms < best)) {
            best = ms;
            best_cols = C;
        }
    });
    if (ce != cudaSuccess) return ce;
    g.p2_cols = best_cols;
    g.tuned = true;
    return cudaSuccess;
}

template <int N>
cudaError_t launch_mix_run(jw_engine* e, Group& g, const int* d_slots, int nb, int nsteps, double* ens,
                           LaunchTimes* tm) {
    if (nsteps < 1) return cudaErrorInvalidValue;
    if (ens && !mx_p3_meas_fits<N>()) return cudaErrorInvalidValue;
    mix_configure<N>();
    if (e->opt.autotune && !g.tuned) {
        const cudaError_t ce = tune_mix<N>(e, g, d_slots, nb);
        if (ce != cudaSuccess) return ce;
    }
    auto middle = [&]() {
        mix_launch<N>(e, g, d_slots, nb, KIND_P2, false, tm);
        mix_launch<N>(e, g, d_slots, nb, KIND_P31, false, tm);
    };
    mix_launch<N>(e, g, d_slots, nb, KIND_P1, false, tm);
    const int reps = nsteps - 1;
    if (reps >= 3 && !tm) {
        middle();
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) return ce;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if ((ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return ce;
        middle();
        const cudaError_t launched = cudaGetLastError();
        ce = cudaStreamEndCapture(e->stream, &graph);
        if (launched != cudaSuccess || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return launched != cudaSuccess ? launched : ce;
        }
        ce = cudaGraphInstantiate(&exec, graph, 0);
        for (int r = 1; r < reps && ce == cudaSuccess; ++r) ce = cudaGraphLaunch(exec, e->stream);
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return ce;
    } else {
        for (int r = 0; r < reps; ++r) middle();
    }
    mix_launch<N>(e, g, d_slots, nb, KIND_P2, false, tm);
    mix_launch<N>(e, g, d_slots, nb, KIND_P3, ens != nullptr, tm);
    if (ens) {
        const long vol = (long)N * N;
        const float4* M = reinterpret_cast<const float4*>(g.ws);
        double* corr = reinterpret_cast<double*>(g.ws + sizeof(float4) * 5 * (size_t)vol * nb);
        k_meas32_cols<N><<<dim3(N / mx_cols<N>(), nb), mx_p2_threads<N>(), mx_p2_smem<N>(), e->stream>>>(
            M, corr, corr + vol * nb, g.tw.d32);
        k_meas_reduce_ensemble<N><<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(corr, corr + vol * nb, nb,
                                                                                         ens);
    }
    return cudaGetLastError();
}

bool fused_measure_supported(int precision, int N) {
    if (precision != JW_PRECISION_MIXED) return false;
    switch (N) {
        case 8: return mx_p3_meas_fits<8>();
        case 16: return mx_p3_meas_fits<16>();
        case 32: return mx_p3_meas_fits<32>();
        case 64: return mx_p3_meas_fits<64>();
        case 128: return mx_p3_meas_fits<128>();
        case 256: return mx_p3_meas_fits<256>();
        case 512: return mx_p3_meas_fits<512>();
        case 1024: return mx_p3_meas_fits<1024>();
        case 2048: return mx_p3_meas_fits<2048>();
        default: return false;
    }
}

template <typename T, int N>
cudaError_t launch_step(jw_engine* e, Group& g, const int* d_slots, int nb, unsigned char* ws) {
    using V2 = C2<T>;
    const long vol = (long)N * N;
    V2* P = reinterpret_cast<V2*>(ws);
    V2* Q = P + (size_t)16 * vol * nb;
    const V2* tw = (const V2*)(sizeof(T) == 8 ? (const void*)g.tw.d64 : (const void*)g.tw.d32);
    constexpr int RT = row_threads<N>();
    constexpr int C = p2_cols<T, N>();
    const size_t sm1 = p1_smem_bytes<T, N>();
    const size_t sm2 = p2_smem<T, N>();
    const size_t sm3 = p3_smem<T, N>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_step_pass1<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
        cudaFuncSetAttribute(k_step_pass2<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        cudaFuncSetAttribute(k_step_pass3<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3);
        configured = true;
    }
    k_step_pass1<T, N><<<dim3(N, p1_groups<T, N>(), nb), p1_threads<N>(), sm1, e->stream>>>(g.d_ev, d_slots, P, tw);
    k_step_pass2<T, N><<<dim3(N / C, 8, nb), C * (N / 8), sm2, e->stream>>>(g.d_ev, d_slots, P, Q, tw);
    k_step_pass3<T, N><<<dim3(N, nb), RT, sm3, e->stream>>>(g.d_ev, d_slots, Q, tw, e->d_flags);
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_mv_slice(jw_engine* e, Group& g, const int* d_slots, int nb, unsigned char* ws, int slice) {
    double2* P = reinterpret_cast<double2*>(ws);
    const size_t r = mv16_row_smem<N>(), c = mv16_col_smem<N>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mv16_pass1<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r);
        cudaFuncSetAttribute(k_mv16_pass1<N, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r);
        cudaFuncSetAttribute(k_mv16_pass2<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c);
        cudaFuncSetAttribute(k_mv16_pass3<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r);
        configured = true;
    }
    if (e->opt.precision == JW_PRECISION_MIXED)
        k_mv16_pass1<N, float><<<dim3(N, nb), mv16_threads<N>(), r, e->stream>>>(g.d_ev, d_slots, slice, P, g.tw.d64);
    else
        k_mv16_pass1<N><<<dim3(N, nb), mv16_threads<N>(), r, e->stream>>>(g.d_ev, d_slots, slice, P, g.tw.d64);
    k_mv16_pass2<N><<<dim3(N / mx_cols<N>(), 4, nb), mx_p2_threads<N>(), c, e->stream>>>(g.d_ev, d_slots, P,
                                                                                         g.tw.d64);
    k_mv16_pass3<N><<<dim3(N, nb), mv16_threads<N>(), r, e->stream>>>(g.d_ev, d_slots, P, g.tw.d64, e->d_flags);
    return cudaGetLastError();
}

// The correlator planes of a measurement: FP64 transforms for the FP64
// engine, FP32 pair planes (FP64 sums) for the mixed one.  Returns the
// per-event correlators' location in the workspace.
template <int N>
cudaError_t launch_measure_kernels(jw_engine* e, Group& g, const int* d_slots, int nb, unsigned char* ws,
                                   double** corr_out) {
    const long vol = (long)N * N;
    if (e->opt.precision == JW_PRECISION_MIXED) {
        float4* M = reinterpret_cast<float4*>(ws);
        double* corr = reinterpret_cast<double*>(M + (size_t)5 * vol * nb);
        const size_t sm1 = meas32_rows_smem<N>(), sm2 = mx_p2_smem<N>();
        static bool configured = false;
        if (!configured) {
            cudaFuncSetAttribute(k_meas32_rows<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
            cudaFuncSetAttribute(k_meas32_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
            configured = true;
        }
        k_meas32_rows<N><<<dim3(N, nb), meas32_rows_threads<N>(), sm1, e->stream>>>(g.d_ev, d_slots, M, g.tw.d32);
        k_meas32_cols<N><<<dim3(N / mx_cols<N>(), nb), mx_p2_threads<N>(), sm2, e->stream>>>(M, corr, corr + vol * nb,
                                                                                            g.tw.d32);
        *corr_out = corr;
        return cudaGetLastError();
    }
    double2* M = reinterpret_cast<double2*>(ws);
    double* corr = reinterpret_cast<double*>(M + (size_t)9 * vol * nb);
    constexpr int RW = meas_rows16<N>();
    const size_t sm1 = meas_rows16_smem<N>();
    const size_t sm2 = meas_cols_smem<N>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_meas_rows<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
        cudaFuncSetAttribute(k_meas_cols<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        configured = true;
    }
    k_meas_rows<N><<<dim3((unsigned)((9L * N + RW - 1) / RW), nb), 256, sm1, e->stream>>>(g.d_ev, d_slots, M,
                                                                                       g.tw.d64);
    k_meas_cols<N><<<dim3(N / mx_cols<N>(), nb), meas_cols_threads<N>(), sm2, e->stream>>>(d_slots, M, corr,
                                                                                          corr + vol * nb, g.tw.d64);
    *corr_out = corr;
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_measure(jw_engine* e, Group& g, const int* d_slots, int nb, unsigned char* ws) {
    const long vol = (long)N * N;
    double* corr = nullptr;
    cudaError_t err = launch_measure_kernels<N>(e, g, d_slots, nb, ws, &corr);
    if (err != cudaSuccess) return err;
    k_meas_reduce<N><<<dim3((unsigned)((vol + 255) / 256), nb), 256, 0, e->stream>>>(g.d_ev, d_slots, corr,
                                                                                   corr + vol * nb);
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_measure_ensemble(jw_engine* e, Group& g, const int* d_slots, int nb, unsigned char* ws,
                                   double* ens) {
    const long vol = (long)N * N;
    double* corr = nullptr;
    cudaError_t err = launch_measure_kernels<N>(e, g, d_slots, nb, ws, &corr);
    if (err != cudaSuccess) return err;
    k_meas_reduce_ensemble<N><<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(corr, corr + vol * nb, nb, ens);
    return cudaGetLastError();
}

#define JW_DISPATCH_N(N, CALL)                   \
    switch (N) {                                 \
        case 8: { constexpr int NN = 8; return CALL; }       \
        case 16: { constexpr int NN = 16; return CALL; }     \
        case 32: { constexpr int NN = 32; return CALL; }     \
        case 64: { constexpr int NN = 64; return CALL; }     \
        case 128: { constexpr int NN = 128; return CALL; }   \
        case 256: { constexpr int NN = 256; return CALL; }   \
        case 512: { constexpr int NN = 512; return CALL; }   \
        case 1024: { constexpr int NN = 1024; return CALL; } \
        case 2048: { constexpr int NN = 2048; return CALL; } \
        default: return cudaErrorInvalidValue;   \
    }

// One FP64 step (mixed-precision steps go through launch_mix_run).
cudaError_t dispatch_step(jw_engine* e, Group& g, const int* d_slots, int nb) {
    switch (g.N) {
        case 8: return launch_step<double, 8>(e, g, d_slots, nb, g.ws);
        case 16: return launch_step<double, 16>(e, g, d_slots, nb, g.ws);
        case 32: return launch_step<double, 32>(e, g, d_slots, nb, g.ws);
        case 64: return launch_step<double, 64>(e, g, d_slots, nb, g.ws);
        case 128: return launch_step<double, 128>(e, g, d_slots, nb, g.ws);
        case 256: return launch_step<double, 256>(e, g, d_slots, nb, g.ws);
        case 512: return launch_step<double, 512>(e, g, d_slots, nb, g.ws);
        case 1024: return launch_step<double, 1024>(e, g, d_slots, nb, g.ws);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t dispatch_mv(jw_engine* e, Group& g, const int* d_slots, int nb, int slice) {
    JW_DISPATCH_N(g.N, (launch_mv_slice<NN>(e, g, d_slots, nb, g.ws, slice)))
}
cudaError_t dispatch_measure(jw_engine* e, Group& g, const int* d_slots, int nb) {
    JW_DISPATCH_N(g.N, (launch_measure<NN>(e, g, d_slots, nb, g.ws)))
}

cudaError_t dispatch_mix_run(jw_engine* e, Group& g, const int* d_slots, int nb, int nsteps, double* ens,
                             LaunchTimes* tm) {
    JW_DISPATCH_N(g.N, (launch_mix_run<NN>(e, g, d_slots, nb, nsteps, ens, tm)))
}

cudaError_t dispatch_measure_ensemble(jw_engine* e, Group& g, const int* d_slots, int nb, double* ens) {
    JW_DISPATCH_N(g.N, (launch_measure_ensemble<NN>(e, g, d_slots, nb, g.ws, ens)))
}

// One timed FP64 step (the mixed steps are timed through launch_mix_run).
template <int N>
cudaError_t launch_step_timed64(jw_engine* e, Group& g, const int* d_slots, int nb, LaunchTimes* tm) {
    using V2 = double2;
    const long vol = (long)N * N;
    V2* P = reinterpret_cast<V2*>(g.ws);
    V2* Q = P + (size_t)16 * vol * nb;
    const V2* tw = g.tw.d64;
    constexpr int RT = row_threads<N>();
    constexpr int C = p2_cols<double, N>();
    const size_t sm1 = p1_smem_bytes<double, N>();
    const size_t sm2 = p2_smem<double, N>();
    const size_t sm3 = p3_smem<double, N>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_step_pass1<double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
        cudaFuncSetAttribute(k_step_pass2<double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
        cudaFuncSetAttribute(k_step_pass3<double, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm3);
        configured = true;
    }
    tm->start(KIND_P1);
    k_step_pass1<double, N><<<dim3(N, p1_groups<double, N>(), nb), p1_threads<N>(), sm1, e->stream>>>(g.d_ev, d_slots,
                                                                                                    P, tw);
    tm->stop();
    tm->start(KIND_P2);
    k_step_pass2<double, N><<<dim3(N / C, 8, nb), C * (N / 8), sm2, e->stream>>>(g.d_ev, d_slots, P, Q, tw);
    tm->stop();
    tm->start(KIND_P3);
    k_step_pass3<double, N><<<dim3(N, nb), RT, sm3, e->stream>>>(g.d_ev, d_slots, Q, tw, e->d_flags);
    tm->stop();
    return cudaGetLastError();
}

cudaError_t dispatch_step_timed64(jw_engine* e, Group& g, const int* d_slots, int nb, LaunchTimes* tm) {
    switch (g.N) {
        case 8: return launch_step_timed64<8>(e, g, d_slots, nb, tm);
        case 16: return launch_step_timed64<16>(e, g, d_slots, nb, tm);
        case 32: return launch_step_timed64<32>(e, g, d_slots, nb, tm);
        case 64: return launch_step_timed64<64>(e, g, d_slots, nb, tm);
        case 128: return launch_step_timed64<128>(e, g, d_slots, nb, tm);
        case 256: return launch_step_timed64<256>(e, g, d_slots, nb, tm);
        case 512: return launch_step_timed64<512>(e, g, d_slots, nb, tm);
        case 1024: return launch_step_timed64<1024>(e, g, d_slots, nb, tm);
        default: return cudaErrorInvalidValue;
    }
}

// Resolve ids into per-group slot lists.
jw_status collect(jw_engine* e, const int* ids, int n, std::map<int, std::vector<int>>& by_n) {
    if (n < 0 || (n > 0 && !ids)) return JW_EINVAL;
    for (int k = 0; k < n; ++k) {
        auto it = e->events.find(ids[k]);
        if (it == e->events.end()) return JW_ENOTFOUND;
        auto& v = by_n[it->second.N];
        if (std::find(v.begin(), v.end(), it->second.slot) != v.end()) return JW_EINVAL;  // duplicate
        v.push_back(it->second.slot);
    }
    return JW_OK;
}

int chunk_size(const jw_engine* e, int count, int N) {
    int c = count;
    if (e->opt.max_batch > 0) c = std::min(c, e->opt.max_batch);
    if (e->opt.max_batch_sites > 0) {
        const size_t per = std::max<size_t>(1, e->opt.max_batch_sites / ((size_t)N * N));
        c = (int)std::min<size_t>((size_t)c, per);
    }
    return std::max(c, 1);
}

// The device slot list of a call; unchanged lists (the same events stepped
// and measured call after call) are not uploaded again.
jw_status upload_slots(jw_engine* e, Group& g, const std::vector<int>& slots) {
    if (g.d_slots && g.h_slots == slots) return JW_OK;
    jw_status s = ensure_slots(g, (int)slots.size());
    if (s) return s;
    g.h_slots.clear();
    JW_CUDA(cudaMemcpyAsync(g.d_slots, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    g.h_slots = slots;
    return JW_OK;
}

jw_status ensure_stage(jw_engine* e, size_t bytes) {
    if (e->stage_bytes < bytes) {
        if (e->d_stage) cudaFree(e->d_stage);
        e->d_stage = nullptr;
        e->stage_bytes = 0;
        if (cudaMalloc(&e->d_stage, bytes) != cudaSuccess) return JW_ENOMEM;
        e->stage_bytes = bytes;
    }
    if (e->pinned_bytes < bytes) {
        if (e->h_pinned) cudaFreeHost(e->h_pinned);
        e->h_pinned = nullptr;
        e->pinned_bytes = 0;
        if (cudaMallocHost(&e->h_pinned, bytes) != cudaSuccess) return JW_ENOMEM;
        e->pinned_bytes = bytes;
    }
    return JW_OK;
}

// True when both ends of [p, p + bytes) are page-locked host memory
// (cudaMallocHost, cudaHostAlloc, cudaHostRegister).  Only the copy path
// depends on it: cudaMemcpyAsync into pageable memory is correct too.
bool host_pinned(const void* p, size_t bytes) {
    for (const char* q : {static_cast<const char*>(p), static_cast<const char*>(p) + bytes - 1}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

// Two device planes of vol complex doubles (d_out, d_out + vol) to the
// caller's host arrays: straight into page-locked arrays, through the pinned
// stage otherwise.
jw_status copy_out_host(jw_engine* e, const double2* d_out, long vol, double* a, double* b) {
    const size_t bytes = sizeof(double2) * (size_t)vol;
    if (host_pinned(a, bytes) && host_pinned(b, bytes)) {
        JW_CUDA(cudaMemcpyAsync(a, d_out, bytes, cudaMemcpyDeviceToHost, e->stream));
        JW_CUDA(cudaMemcpyAsync(b, d_out + vol, bytes, cudaMemcpyDeviceToHost, e->stream));
        JW_CUDA(cudaStreamSynchronize(e->stream));
        return JW_OK;
    }
    JW_CUDA(cudaMemcpyAsync(e->h_pinned, d_out, 2 * bytes, cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    std::memcpy(a, e->h_pinned, bytes);
    std::memcpy(b, e->h_pinned + vol, bytes);
    return JW_OK;
}

}  // namespace

// =================================================================== C ABI

JW_EXPORT jw_status jw_engine_create(const jw_engine_options* opt, int device, jw_engine** out) {
    JW_CHECK(opt && out);
    *out = nullptr;
    JW_CHECK(opt->precision == JW_PRECISION_FP64 || opt->precision == JW_PRECISION_MIXED);
    JW_CUDA(cudaSetDevice(device));
    auto* e = new jw_engine();
    e->opt = *opt;
    e->device = device;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess ||
        cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&e->d_flags, sizeof(int)) != cudaSuccess ||
        cudaMemsetAsync(e->d_flags, 0, sizeof(int), e->stream) != cudaSuccess) {
        jw_engine_destroy(e);
        return JW_ECUDA;
    }
    e->budget = opt->max_bytes ? opt->max_bytes : (size_t)(0.9 * (double)free_b);
    *out = e;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_destroy(jw_engine* e) {
    if (!e) return JW_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (auto& kv : e->events) {
        cudaFree(kv.second.V);
        cudaFree(kv.second.acc);
        if (kv.second.k64) cudaFree(kv.second.k64);
        if (kv.second.k32) cudaFree(kv.second.k32);
    }
    pool_release(e);
    for (auto& kv : e->groups) group_destroy(*kv.second);
    if (e->d_flags) cudaFree(e->d_flags);
    if (e->d_stage) cudaFree(e->d_stage);
    if (e->h_pinned) cudaFreeHost(e->h_pinned);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_sync(jw_engine* e) {
    JW_CHECK(e);
    JW_CUDA(cudaStreamSynchronize(e->stream));
    int flags = 0;
    JW_CUDA(cudaMemcpy(&flags, e->d_flags, sizeof(int), cudaMemcpyDeviceToHost));
    // on the stream: a legacy-stream memset is not ordered with later kernels
    if (flags) JW_CUDA(cudaMemsetAsync(e->d_flags, 0, sizeof(int), e->stream));
    return flags_to_status(flags);
}

JW_EXPORT void* jw_engine_stream(jw_engine* e) { return e ? (void*)e->stream : nullptr; }

JW_EXPORT size_t jw_engine_event_bytes(const jw_engine* e, const jw_event_desc* d) {
    if (!e || !d || !supported_n(d->N)) return 0;
    const size_t vol = (size_t)d->N * d->N;
    return vol * (sizeof(double2) * 9 + sizeof(double) * 4) + ws_per_event(e, d->N) +
           (d->position_space ? position_table_bytes(d->N) : 0);
}

JW_EXPORT jw_status jw_engine_add_event(jw_engine* e, const jw_event_desc* d, int* event_id) {
    JW_CHECK(e && d && event_id);
    *event_id = -1;
    if (!engine_supported(e->opt.precision, d->N)) return JW_EUNSUPPORTED;
    // the LINEAR kernel in position space only: its momentum-space multiplier
    // is not Hermitian-symmetric at the Nyquist lines (below)
    if (d->kernel != JW_SIN_KERNEL && !(d->position_space && d->kernel == JW_LINEAR_KERNEL)) return JW_EUNSUPPORTED;
    if (d->position_space) {
        if (d->coupling != JW_SQRT_COUPLING_CONSTANT && d->coupling != JW_HATTA_COUPLING_CONSTANT &&
            d->coupling != JW_FIXED_COUPLING_CONSTANT)
            return JW_EUNSUPPORTED;
        JW_CHECK(d->rr >= 0);
    } else if (d->coupling != JW_SQRT_COUPLING_CONSTANT && d->coupling != JW_NOISE_COUPLING_CONSTANT &&
               d->coupling != JW_FIXED_COUPLING_CONSTANT) {
        return JW_EUNSUPPORTED;
    }
    JW_CHECK(d->ny_slices >= 0 && d->step >= 0.0 && std::isfinite(d->mu) && std::isfinite(d->mass) &&
             std::isfinite(d->step));
    const size_t vol = (size_t)d->N * d->N;
    const size_t own = vol * (sizeof(double2) * 9 + sizeof(double) * 4) +
                       (d->position_space ? position_table_bytes(d->N) : 0);
    if (e->bytes_in_use + own + ws_per_event(e, d->N) > e->budget) return JW_ENOMEM;
    Group* g = nullptr;
    jw_status s = group_get(e, d->N, &g);
    if (s) return s;
    if (!d->position_space && (s = ensure_tables(e, *g, d->coupling))) return s;
    int slot = -1;
    for (int k = 0; k < (int)g->owner.size(); ++k)
        if (g->owner[k] < 0) {
            slot = k;
            break;
        }
    if (slot < 0) {
        slot = (int)g->owner.size();
        if ((s = grow_slots(*g, e->stream))) return s;
    }
    Event ev;
    ev.id = e->next_id++;
    ev.N = d->N;
    ev.slot = slot;
    ev.desc = *d;
    const size_t bV = sizeof(double2) * 9 * vol, bA = sizeof(double) * 4 * vol;
    const size_t b64 = sizeof(double) * 4 * vol, b32 = sizeof(float) * 4 * vol, bT = sizeof(double2) * 2 * vol;
    ev.V = static_cast<double2*>(ev_alloc(e, bV));
    ev.acc = static_cast<double*>(ev_alloc(e, bA));
    if (!ev.V || !ev.acc) {
        ev_free(e, ev.V, bV);
        ev_free(e, ev.acc, bA);
        return JW_ENOMEM;
    }
    if (d->position_space) {
        // k_i(d), its DFT in FP64, imag / N^2 into the event's tables
        ev.k64 = static_cast<double*>(ev_alloc(e, b64));
        ev.k32 = static_cast<float*>(ev_alloc(e, b32));
        double2* tmp = static_cast<double2*>(ev_alloc(e, bT));
        if (!ev.k64 || !ev.k32 || !tmp) {
            ev_free(e, ev.V, bV);
            ev_free(e, ev.acc, bA);
            ev_free(e, ev.k64, b64);
            ev_free(e, ev.k32, b32);
            ev_free(e, tmp, bT);
            return JW_ENOMEM;
        }
        k_position_kernel<<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(tmp, d->N, d->rr, d->coupling,
                                                                                d->kernel);
        cudaError_t ce = cudaGetLastError();
        if (ce == cudaSuccess) ce = fft2d_planes<double>(tmp, 2, d->N, 1, 1.0, g->tw, e->stream);
        if (ce == cudaSuccess) {
            k_position_table<<<(unsigned)((2 * vol + 255) / 256), 256, 0, e->stream>>>(
                tmp, ev.k64, ev.k32, (long)(2 * vol), 1.0 / ((double)d->N * d->N));
            ce = cudaGetLastError();
        }
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
        ev_free(e, tmp, bT);
        if (ce != cudaSuccess) {
            ev_free(e, ev.V, bV);
            ev_free(e, ev.acc, bA);
            ev_free(e, ev.k64, b64);
            ev_free(e, ev.k32, b32);
            return JW_ECUDA;
        }
    }
    e->bytes_in_use += own;
    k_set_unit_planes<<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(ev.V, (long)vol);
    JW_CUDA(cudaMemsetAsync(ev.acc, 0, sizeof(double) * 4 * vol, e->stream));
    EventDev h{};
    h.V = ev.V;
    h.acc = ev.acc;
    const int cp = d->coupling;
    h.k64 = d->position_space ? ev.k64 : g->k64[cp];
    h.k32 = d->position_space ? ev.k32 : g->k32[cp];
    // the LINEAR position kernel k_i(d) is not odd at d_i = -N/2, so its DFT has a
    // real part; the SIN kernel's and the momentum kernels' tables are imaginary
    const bool re = d->position_space && d->kernel == JW_LINEAR_KERNEL;
    h.kre64 = re ? ev.k64 + 2 * vol : nullptr;
    h.kre32 = re ? ev.k32 + 2 * vol : nullptr;
    // the site-indexed noise factor belongs to momentum-space NOISE coupling only
    const bool nf = !d->position_space && cp == JW_NOISE_COUPLING_CONSTANT;
    h.nf64 = nf ? g->nf64 : nullptr;
    h.nf32 = nf ? g->nf32 : nullptr;
    h.seed = d->seed;
    h.step = d->step0;
    h.sqrt_eps = std::sqrt(d->step);
    const double gg = 1.0, mu = d->mu / d->N;
    h.mv_sigma = d->ny_slices > 0 ? gg * mu / std::sqrt((double)d->ny_slices) : 0.0;
    const double m = d->mass * std::pow(gg, 2.0) * mu;
    h.mv_mass2 = m * m;
    h.mv_g = gg;
    h.N = d->N;
    h.reunit = e->opt.reunitarize ? 1 : 0;
    h.nmeas = 0;
    JW_CUDA(cudaMemcpyAsync(g->d_ev + slot, &h, sizeof(EventDev), cudaMemcpyHostToDevice, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    g->owner[slot] = ev.id;
    // workspace for every resident event of this size stepping in one launch group
    int resident = 0;
    for (int o : g->owner) resident += o >= 0;
    s = ensure_workspace(e, *g, chunk_size(e, resident, d->N));
    if (s) {
        g->owner[slot] = -1;
        e->bytes_in_use -= own;
        ev_free(e, ev.V, bV);
        ev_free(e, ev.acc, bA);
        ev_free(e, ev.k64, b64);
        ev_free(e, ev.k32, b32);
        return s;
    }
    if (h.kre32) g->n_re += 1;
    e->events[ev.id] = ev;
    *event_id = ev.id;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_remove_event(jw_engine* e, int id) {
    JW_CHECK(e);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    JW_CUDA(cudaStreamSynchronize(e->stream));
    Event& ev = it->second;
    Group& g = *e->groups[ev.N];
    g.owner[ev.slot] = -1;
    if (ev.desc.position_space && ev.desc.kernel == JW_LINEAR_KERNEL) g.n_re -= 1;
    const size_t vol = (size_t)ev.N * ev.N;
    e->bytes_in_use -= vol * (sizeof(double2) * 9 + sizeof(double) * 4) +
                       (ev.desc.position_space ? position_table_bytes(ev.N) : 0);
    ev_free(e, ev.V, sizeof(double2) * 9 * vol);
    ev_free(e, ev.acc, sizeof(double) * 4 * vol);
    ev_free(e, ev.k64, sizeof(double) * 4 * vol);
    ev_free(e, ev.k32, sizeof(float) * 4 * vol);
    e->events.erase(it);
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_set_V(jw_engine* e, int id, const double* host) {
    JW_CHECK(e && host);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const long vol = (long)it->second.N * it->second.N;
    const size_t bytes = sizeof(double2) * 9 * vol;
    jw_status s = ensure_stage(e, bytes);
    if (s) return s;
    std::memcpy(e->h_pinned, host, bytes);
    JW_CUDA(cudaMemcpyAsync(e->d_stage, e->h_pinned, bytes, cudaMemcpyHostToDevice, e->stream));
    k_aos_to_planes<<<(unsigned)((9 * vol + 255) / 256), 256, 0, e->stream>>>(e->d_stage, it->second.V, vol);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(cudaStreamSynchronize(e->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_get_V(jw_engine* e, int id, double* host) {
    JW_CHECK(e && host);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const long vol = (long)it->second.N * it->second.N;
    const size_t bytes = sizeof(double2) * 9 * vol;
    jw_status s = ensure_stage(e, bytes);
    if (s) return s;
    k_planes_to_aos<<<(unsigned)((9 * vol + 255) / 256), 256, 0, e->stream>>>(it->second.V, e->d_stage, vol);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(cudaMemcpyAsync(e->h_pinned, e->d_stage, bytes, cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    std::memcpy(host, e->h_pinned, bytes);
    return JW_OK;
}

// ---- checkpoints: [header][V, reference layout][4 accumulator planes]
namespace {
struct EventFileHeader {
    char magic[8];         // "JWEVENT1"
    jw_event_desc desc;
    uint64_t step;         // next noise index
    int32_t nmeas;
    int32_t reserved;
};
constexpr char kEventMagic[8] = {'J', 'W', 'E', 'V', 'E', 'N', 'T', '1'};
}  // namespace

JW_EXPORT jw_status jw_engine_save_event(jw_engine* e, int id, const char* path) {
    JW_CHECK(e && path);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const Event& ev = it->second;
    const long vol = (long)ev.N * ev.N;
    std::vector<double> V(18 * (size_t)vol), acc(4 * (size_t)vol);
    jw_status s = jw_engine_get_V(e, id, V.data());
    if (s) return s;
    EventDev d{};
    JW_CUDA(cudaMemcpyAsync(acc.data(), ev.acc, sizeof(double) * 4 * vol, cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaMemcpyAsync(&d, e->groups[ev.N]->d_ev + ev.slot, sizeof(EventDev), cudaMemcpyDeviceToHost,
                            e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    EventFileHeader h{};
    std::memcpy(h.magic, kEventMagic, 8);
    h.desc = ev.desc;
    h.step = d.step;
    h.nmeas = d.nmeas;
    FILE* f = std::fopen(path, "wb");
    if (!f) return JW_EINVAL;
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(V.data(), sizeof(double), V.size(), f) == V.size() &&
              std::fwrite(acc.data(), sizeof(double), acc.size(), f) == acc.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? JW_OK : JW_EINVAL;
}

JW_EXPORT jw_status jw_engine_load_event(jw_engine* e, const char* path, int* event_id) {
    JW_CHECK(e && path && event_id);
    *event_id = -1;
    FILE* f = std::fopen(path, "rb");
    if (!f) return JW_EINVAL;
    EventFileHeader h{};
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kEventMagic, 8) != 0 || !supported_n(h.desc.N)) {
        std::fclose(f);
        return JW_EINVAL;
    }
    const long vol = (long)h.desc.N * h.desc.N;
    std::vector<double> V(18 * (size_t)vol), acc(4 * (size_t)vol);
    const bool ok = std::fread(V.data(), sizeof(double), V.size(), f) == V.size() &&
                    std::fread(acc.data(), sizeof(double), acc.size(), f) == acc.size();
    std::fclose(f);
    if (!ok) return JW_EINVAL;
    int id = -1;
    jw_status s = jw_engine_add_event(e, &h.desc, &id);
    if (s) return s;
    s = jw_engine_set_V(e, id, V.data());
    if (s) {
        jw_engine_remove_event(e, id);
        return s;
    }
    const Event& ev = e->events[id];
    EventDev* dev = e->groups[ev.N]->d_ev + ev.slot;
    JW_CUDA(cudaMemcpyAsync(ev.acc, acc.data(), sizeof(double) * 4 * vol, cudaMemcpyHostToDevice, e->stream));
    JW_CUDA(cudaMemcpyAsync(&dev->step, &h.step, sizeof h.step, cudaMemcpyHostToDevice, e->stream));
    JW_CUDA(cudaMemcpyAsync(&dev->nmeas, &h.nmeas, sizeof h.nmeas, cudaMemcpyHostToDevice, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    *event_id = id;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_init_mv(jw_engine* e, const int* ids, int n) {
    JW_CHECK(e);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s) return s;
    for (auto& kv : by_n) {
        Group& g = *e->groups[kv.first];
        // events of one group and one slice count run together
        std::map<int, std::vector<int>> by_ny;
        for (int slot : kv.second) by_ny[e->events[g.owner[slot]].desc.ny_slices].push_back(slot);
        for (auto& nv : by_ny) {
            const std::vector<int>& slots = nv.second;
            const int cs = chunk_size(e, (int)slots.size(), g.N);
            if ((s = ensure_workspace(e, g, cs))) return s;
            if ((s = upload_slots(e, g, slots))) return s;
            for (size_t c0 = 0; c0 < slots.size(); c0 += cs) {
                const int nb = (int)std::min<size_t>(cs, slots.size() - c0);
                for (int slot : std::vector<int>(slots.begin() + c0, slots.begin() + c0 + nb))
                    k_set_unit_planes<<<(unsigned)(((long)g.N * g.N + 255) / 256), 256, 0, e->stream>>>(
                        e->events[g.owner[slot]].V, (long)g.N * g.N);
                for (int sl = 0; sl < nv.first; ++sl) JW_CUDA(dispatch_mv(e, g, g.d_slots + c0, nb, sl));
            }
        }
    }
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_step(jw_engine* e, const int* ids, int n, int nsteps) {
    JW_CHECK(e && nsteps >= 0);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s || nsteps == 0) return s;
    // per group: workspace for one chunk, slot list on the device
    struct Work { Group* g; int nb; int off; };
    std::vector<Work> work;
    for (auto& kv : by_n) {
        Group& g = *e->groups[kv.first];
        const int cs = chunk_size(e, (int)kv.second.size(), kv.first);
        if ((s = ensure_workspace(e, g, cs))) return s;
        if ((s = upload_slots(e, g, kv.second))) return s;
        for (int c0 = 0; c0 < (int)kv.second.size(); c0 += cs)
            work.push_back({&g, std::min(cs, (int)kv.second.size() - c0), c0});
    }
    if (e->opt.precision == JW_PRECISION_MIXED) {
        for (const Work& w : work)
            JW_CUDA(dispatch_mix_run(e, *w.g, w.g->d_slots + w.off, w.nb, nsteps, nullptr, nullptr));
        return JW_OK;
    }
    // FP64: one step of every chunk, captured once as a graph and replayed
    auto record = [&]() -> cudaError_t {
        for (const Work& w : work) {
            cudaError_t ce = dispatch_step(e, *w.g, w.g->d_slots + w.off, w.nb);
            if (ce != cudaSuccess) return ce;
        }
        return cudaSuccess;
    };
    if (nsteps == 1) {
        JW_CUDA(record());
        return JW_OK;
    }
    // groups that share one workspace run chunk after chunk inside the step,
    // which stream order keeps correct within the graph as well
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    JW_CUDA(record());  // first step also sets kernel attributes outside capture
    JW_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = record();
    cudaError_t ce2 = cudaStreamEndCapture(e->stream, &graph);
    if (ce != cudaSuccess || ce2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return JW_ECUDA;
    }
    JW_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    for (int k = 1; k < nsteps; ++k) {
        ce = cudaGraphLaunch(exec, e->stream);
        if (ce != cudaSuccess) break;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    JW_CUDA(ce);
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_measure(jw_engine* e, const int* ids, int n) {
    JW_CHECK(e);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s) return s;
    for (auto& kv : by_n) {
        Group& g = *e->groups[kv.first];
        const int cs = chunk_size(e, (int)kv.second.size(), kv.first);
        if ((s = ensure_workspace(e, g, cs))) return s;
        if ((s = upload_slots(e, g, kv.second))) return s;
        for (int c0 = 0; c0 < (int)kv.second.size(); c0 += cs)
            JW_CUDA(dispatch_measure(e, g, g.d_slots + c0, std::min(cs, (int)kv.second.size() - c0)));
    }
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_get_correlator(jw_engine* e, int id, double* sum, double* err, int* nmeas) {
    JW_CHECK(e);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const Event& ev = it->second;
    const long vol = (long)ev.N * ev.N;
    std::vector<double> h(4 * vol);
    JW_CUDA(cudaMemcpyAsync(h.data(), ev.acc, sizeof(double) * 4 * vol, cudaMemcpyDeviceToHost, e->stream));
    EventDev d{};
    JW_CUDA(cudaMemcpyAsync(&d, e->groups[ev.N]->d_ev + ev.slot, sizeof(EventDev), cudaMemcpyDeviceToHost,
                            e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    for (long i = 0; i < vol; ++i) {
        if (sum) { sum[2 * i] = h[i] + h[vol + i]; sum[2 * i + 1] = 0.0; }
        if (err) { err[2 * i] = h[2 * vol + i] + h[3 * vol + i]; err[2 * i + 1] = 0.0; }
    }
    if (nmeas) *nmeas = d.nmeas;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_reset_correlator(jw_engine* e, int id) {
    JW_CHECK(e);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const Event& ev = it->second;
    JW_CUDA(cudaMemsetAsync(ev.acc, 0, sizeof(double) * 4 * (size_t)ev.N * ev.N, e->stream));
    const int zero = 0;
    JW_CUDA(cudaMemcpyAsync(&e->groups[ev.N]->d_ev[ev.slot].nmeas, &zero, sizeof(int), cudaMemcpyHostToDevice,
                            e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_copy_V(jw_engine* e, int dst, int src) {
    JW_CHECK(e);
    auto a = e->events.find(dst), b = e->events.find(src);
    if (a == e->events.end() || b == e->events.end()) return JW_ENOTFOUND;
    JW_CHECK(a->second.N == b->second.N);
    if (dst == src) return JW_OK;
    JW_CUDA(cudaMemcpyAsync(a->second.V, b->second.V, sizeof(double2) * 9 * (size_t)a->second.N * a->second.N,
                            cudaMemcpyDeviceToDevice, e->stream));
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_reset_correlators(jw_engine* e, const int* ids, int n) {
    JW_CHECK(e && (ids || n == 0) && n >= 0);
    for (int i = 0; i < n; ++i)
        if (e->events.find(ids[i]) == e->events.end()) return JW_ENOTFOUND;
    const int zero = 0;
    for (int i = 0; i < n; ++i) {
        const Event& ev = e->events[ids[i]];
        JW_CUDA(cudaMemsetAsync(ev.acc, 0, sizeof(double) * 4 * (size_t)ev.N * ev.N, e->stream));
        JW_CUDA(cudaMemcpyAsync(&e->groups[ev.N]->d_ev[ev.slot].nmeas, &zero, sizeof(int), cudaMemcpyHostToDevice,
                                e->stream));
    }
    JW_CUDA(cudaStreamSynchronize(e->stream));  // `zero` lives on this frame
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_correlator_at(jw_engine* e, const int* ids, int n, const int* xr, const int* yr,
                                            double* sum, double* err) {
    JW_CHECK(e && ids && xr && yr && n >= 0 && (sum || err));
    for (int i = 0; i < n; ++i) {
        auto it = e->events.find(ids[i]);
        if (it == e->events.end()) return JW_ENOTFOUND;
        JW_CHECK(xr[i] >= 0 && xr[i] < it->second.N && yr[i] >= 0 && yr[i] < it->second.N);
    }
    if (n == 0) return JW_OK;
    // one gather on the device: per event the address of acc[site] and the
    // plane stride go up, four doubles per event (sum, compensation, err,
    // compensation) come back in one copy
    const size_t up = sizeof(AccSite) * n, down = sizeof(double) * 4 * n;
    jw_status st = ensure_stage(e, up + down);
    if (st) return st;
    AccSite* hs = reinterpret_cast<AccSite*>(e->h_pinned);
    for (int i = 0; i < n; ++i) {
        const Event& ev = e->events[ids[i]];
        const long vol = (long)ev.N * ev.N;
        hs[i] = AccSite{ev.acc + (long)xr[i] * ev.N + yr[i], vol};
    }
    unsigned char* ds = reinterpret_cast<unsigned char*>(e->d_stage);
    JW_CUDA(cudaMemcpyAsync(ds, hs, up, cudaMemcpyHostToDevice, e->stream));
    double* dout = reinterpret_cast<double*>(ds + up);
    k_gather_acc<<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(reinterpret_cast<const AccSite*>(ds), n, dout);
    JW_CUDA(cudaGetLastError());
    std::vector<double> h(4 * (size_t)n);
    JW_CUDA(cudaMemcpyAsync(h.data(), dout, down, cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    for (int i = 0; i < n; ++i) {
        if (sum) sum[i] = h[4 * (size_t)i] + h[4 * (size_t)i + 1];
        if (err) err[i] = h[4 * (size_t)i + 2] + h[4 * (size_t)i + 3];
    }
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_event_steps(jw_engine* e, int id, uint64_t* steps) {
    JW_CHECK(e && steps);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    EventDev d{};
    JW_CUDA(cudaMemcpyAsync(&d, e->groups[it->second.N]->d_ev + it->second.slot, sizeof(EventDev),
                            cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    *steps = d.step;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_measure_ensemble(jw_engine* e, const int* ids, int n, double* sum, double* err) {
    JW_CHECK(e && sum && err && n > 0);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s) return s;
    if (by_n.size() != 1) return JW_EINVAL;  // one lattice size per ensemble
    Group& g = *e->groups[by_n.begin()->first];
    const std::vector<int>& slots = by_n.begin()->second;
    const long vol = (long)g.N * g.N;
    const int cs = chunk_size(e, (int)slots.size(), g.N);
    if ((s = ensure_workspace(e, g, cs))) return s;
    if ((s = upload_slots(e, g, slots))) return s;
    if ((s = ensure_stage(e, sizeof(double) * 8 * vol))) return s;
    double* ens = reinterpret_cast<double*>(e->d_stage);
    double2* out = reinterpret_cast<double2*>(ens + 4 * vol);
    JW_CUDA(cudaMemsetAsync(ens, 0, sizeof(double) * 4 * vol, e->stream));
    for (int c0 = 0; c0 < (int)slots.size(); c0 += cs)
        JW_CUDA(dispatch_measure_ensemble(e, g, g.d_slots + c0, std::min(cs, (int)slots.size() - c0), ens));
    k_ens_finalize<<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(ens, vol, out);
    JW_CUDA(cudaGetLastError());
    return copy_out_host(e, out, vol, sum, err);
}

JW_EXPORT jw_status jw_engine_step_measure_ensemble(jw_engine* e, const int* ids, int n, int nsteps, double* sum,
                                                    double* err) {
    JW_CHECK(e && sum && err && n > 0 && nsteps >= 1);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s) return s;
    if (by_n.size() != 1) return JW_EINVAL;  // one lattice size per ensemble
    if (!fused_measure_supported(e->opt.precision, by_n.begin()->first)) {
        if ((s = jw_engine_step(e, ids, n, nsteps))) return s;
        return jw_engine_measure_ensemble(e, ids, n, sum, err);
    }
    Group& g = *e->groups[by_n.begin()->first];
    const std::vector<int>& slots = by_n.begin()->second;
    const long vol = (long)g.N * g.N;
    const int cs = chunk_size(e, (int)slots.size(), g.N);
    if ((s = ensure_workspace(e, g, cs))) return s;
    if ((s = upload_slots(e, g, slots))) return s;
    if ((s = ensure_stage(e, sizeof(double) * 8 * vol))) return s;
    double* ens = reinterpret_cast<double*>(e->d_stage);
    double2* out = reinterpret_cast<double2*>(ens + 4 * vol);
    JW_CUDA(cudaMemsetAsync(ens, 0, sizeof(double) * 4 * vol, e->stream));
    for (int c0 = 0; c0 < (int)slots.size(); c0 += cs)
        JW_CUDA(dispatch_mix_run(e, g, g.d_slots + c0, std::min(cs, (int)slots.size() - c0), nsteps, ens, nullptr));
    k_ens_finalize<<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(ens, vol, out);
    JW_CUDA(cudaGetLastError());
    return copy_out_host(e, out, vol, sum, err);
}

namespace {
template <int N>
bool p2_cols_valid_n(int cols) {
    if (cols == kP2Tma) cols = kP2Tma + mx_t2_cols<N>();
    if (cols == kRadixFirst + kP2Tma) cols = kRadixFirst + kP2Tma + mx_t2_cols<N>();
    bool ok = false;
    for_each_p2_cols<N>([&](auto c) { ok = ok || decltype(c)::value == cols; });
    return ok;
}
bool p2_cols_valid(int N, int cols) {
    switch (N) {
        case 8: return p2_cols_valid_n<8>(cols);
        case 16: return p2_cols_valid_n<16>(cols);
        case 32: return p2_cols_valid_n<32>(cols);
        case 64: return p2_cols_valid_n<64>(cols);
        case 128: return p2_cols_valid_n<128>(cols);
        case 256: return p2_cols_valid_n<256>(cols);
        case 512: return p2_cols_valid_n<512>(cols);
        case 1024: return p2_cols_valid_n<1024>(cols);
        case 2048: return p2_cols_valid_n<2048>(cols);
        default: return false;
    }
}
}  // namespace

JW_EXPORT jw_status jw_engine_set_tuning(jw_engine* e, int N, int p2_cols) {
    JW_CHECK(e);
    auto it = e->groups.find(N);
    if (it == e->groups.end()) return JW_ENOTFOUND;
    if (p2_cols != 0 && !p2_cols_valid(N, p2_cols)) return JW_EINVAL;
    JW_CUDA(cudaStreamSynchronize(e->stream));  // launches already queued keep their width
    it->second->p2_cols = p2_cols;
    it->second->tuned = true;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_tuning(jw_engine* e, int N, int* p2_cols) {
    JW_CHECK(e && p2_cols);
    auto it = e->groups.find(N);
    if (it == e->groups.end()) return JW_ENOTFOUND;
    const Group& g = *it->second;
    *p2_cols = g.tuned ? g.p2_cols : 0;
    return JW_OK;
}

JW_EXPORT jw_status jw_engine_step_timed(jw_engine* e, const int* ids, int n, int nsteps, double* kernel_ms,
                                         int* launches, double* total_ms) {
    JW_CHECK(e && nsteps > 0 && kernel_ms && launches && total_ms);
    std::map<int, std::vector<int>> by_n;
    jw_status s = collect(e, ids, n, by_n);
    if (s) return s;
    if (by_n.size() != 1) return JW_EINVAL;  // timing is reported for one lattice size
    Group& g = *e->groups[by_n.begin()->first];
    const std::vector<int>& slots = by_n.begin()->second;
    const int nb = (int)slots.size();
    const int cs = chunk_size(e, nb, g.N);
    if ((s = ensure_workspace(e, g, cs))) return s;
    if ((s = upload_slots(e, g, slots))) return s;
    const bool mixed = e->opt.precision == JW_PRECISION_MIXED;
    LaunchTimes tm;
    tm.stream = e->stream;
    cudaError_t ce = cudaSuccess;
    for (int c = 0; c * cs < nb && ce == cudaSuccess; ++c) {
        const int nbc = std::min(cs, nb - c * cs);
        if (mixed) {
            ce = dispatch_mix_run(e, g, g.d_slots + c * cs, nbc, nsteps, nullptr, &tm);
        } else {
            for (int k = 0; k < nsteps && ce == cudaSuccess; ++k)
                ce = dispatch_step_timed64(e, g, g.d_slots + c * cs, nbc, &tm);
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    JW_CUDA(ce);
    for (int k = 0; k < KIND_COUNT; ++k) {
        kernel_ms[k] = 0.0;
        launches[k] = 0;
    }
    float a = 0.0f;
    for (size_t i = 0; i < tm.kind.size(); ++i) {
        JW_CUDA(cudaEventElapsedTime(&a, tm.ev[2 * i], tm.ev[2 * i + 1]));
        kernel_ms[tm.kind[i]] += a;
        launches[tm.kind[i]] += 1;
    }
    *total_ms = 0.0;
    if (!tm.ev.empty()) {
        JW_CUDA(cudaEventElapsedTime(&a, tm.ev.front(), tm.ev.back()));
        *total_ms = a;
    }
    return JW_OK;
}

namespace jw {
void dipole_bins(const double2* h, int N, double* S_xy, double* S_bins, double* r_bins, int* counts, int* nbins,
                 double* Qs) {
    const long vol = (long)N * N;
    const int nb = N / 2 + 1;
    if (S_xy)
        for (long i = 0; i < vol; ++i) S_xy[i] = h[i].x;
    std::vector<double> sb(nb, 0.0), rb(nb, 0.0);
    std::vector<int> cb(nb, 0);
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
            const int dx = x > N / 2 ? x - N : x, dy = y > N / 2 ? y - N : y;
            const double r = std::sqrt((double)(dx * dx + dy * dy));
            const int b = (int)std::floor(r + 0.5);
            if (b >= nb) continue;
            sb[b] += h[(long)x * N + y].x;
            rb[b] += r;
            cb[b] += 1;
        }
    for (int b = 0; b < nb; ++b)
        if (cb[b]) {
            sb[b] /= cb[b];
            rb[b] /= cb[b];
        }
    if (S_bins)
        for (int b = 0; b < nb; ++b) {
            S_bins[b] = sb[b];
            if (r_bins) r_bins[b] = rb[b];
            if (counts) counts[b] = cb[b];
        }
    if (nbins) *nbins = nb;
    if (Qs) {
        const double target = std::exp(-0.5);
        double q = 0.0;
        for (int b = 0; b + 1 < nb; ++b)
            if (sb[b] >= target && sb[b + 1] < target) {
                const double t = (sb[b] - target) / (sb[b] - sb[b + 1]);
                const double rs = rb[b] + t * (rb[b + 1] - rb[b]);
                q = rs > 0.0 ? std::sqrt(2.0) / rs : 0.0;
                break;
            }
        *Qs = q;
    }
}
}  // namespace jw

// Dipole in position space from an event's accumulated correlator (the mean
// over its measurements): S(r) = (N^2/3) sum_k C(k) exp(+2 pi i k.r/N) (the
// Wiener-Khinchin form of (1/3N^2) sum_x tr V(x) V^dagger(x+r)), then the
// angular average over bins b = floor(|r| + 1/2), |r| the minimum-image length,
// b <= N/2, and Q_s = sqrt(2)/r_s with S(r_s) = exp(-1/2) interpolated linearly
// between the first pair of bins that brackets it (0 if none).
JW_EXPORT jw_status jw_engine_dipole(jw_engine* e, int id, double* S_xy, double* S_bins, double* r_bins,
                                     int* counts, int nbins_cap, int* nbins, double* Qs) {
    JW_CHECK(e);
    auto it = e->events.find(id);
    if (it == e->events.end()) return JW_ENOTFOUND;
    const Event& ev = it->second;
    const int N = ev.N;
    const long vol = (long)N * N;
    const int nb = N / 2 + 1;
    if (S_bins && nbins_cap < nb) return JW_EINVAL;
    Group& g = *e->groups[N];
    jw_status s = ensure_workspace(e, g, 1);
    if (s) return s;
    EventDev d{};
    JW_CUDA(cudaMemcpyAsync(&d, g.d_ev + ev.slot, sizeof(EventDev), cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    if (d.nmeas <= 0) return JW_EINVAL;
    double2* plane = reinterpret_cast<double2*>(g.ws);
    const double scale = (double)N * (double)N / 3.0 / d.nmeas;
    k_dipole_prep<<<(unsigned)((vol + 255) / 256), 256, 0, e->stream>>>(ev.acc, plane, vol, scale);
    JW_CUDA(cudaGetLastError());
    JW_CUDA(fft2d_planes<double>(plane, 1, N, 0, 1.0, g.tw, e->stream));
    std::vector<double2> h(vol);
    JW_CUDA(cudaMemcpyAsync(h.data(), plane, sizeof(double2) * vol, cudaMemcpyDeviceToHost, e->stream));
    JW_CUDA(cudaStreamSynchronize(e->stream));
    dipole_bins(h.data(), N, S_xy, S_bins, r_bins, counts, nbins, Qs);
    return JW_OK;
}
