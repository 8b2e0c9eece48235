// bmc_capi.cu -- the C ABI declared in include/bmc_b200.h.
//
// Host side of the library: argument checks, a per-device workspace cache, the truncated-Taylor
// tables, event preprocessing, the dispatch over pool count / precision / tangents per launch,
// and the device-side Levenberg-Marquardt loop (every launch asynchronous on the caller's stream,
// no host synchronisation inside a call).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bmc_b200.h"
#include <cub/device/device_radix_sort.cuh>

#include "bmc_lm.cuh"
#include "bmc_joint.cuh"
#include "bmc_adjoint.cuh"
#include "bmc_adjoint_block.cuh"
#include "bmc_design.cuh"

using namespace bmc;

namespace {

thread_local std::string g_err;

bmc_status fail(bmc_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

#define CUDA_TRY(expr)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return fail(BMC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

namespace bmc {
// the same thread-local message for the library's other translation units (bmc_mlp.cu)
bmc_status record_error(bmc_status s, const char* msg) {
    g_err = msg;
    return s;
}
}  // namespace bmc

namespace {

// ------------------------------------------------------------------------------------------------
// truncated-Taylor tables: theta[m] = max t with t^(m+1)/(m+1)! / (1 - t/(m+2)) <= tol, a bound of the
// tail sum_{k>m} t^k/k! of exp (each term at most t/(m+2) times the one before), per sub-step, found by
// bisection
// ------------------------------------------------------------------------------------------------
// f32_eps > 0: the Taylor terms of a degree-m warp whose bound theta[m]^k / k! is at most f32_eps are
// formed in float32 (f32_from[m] = the first such k); f32_eps = 0: none are.
TaylorTable make_table(double tol, int m_max, double dense_theta, double dense_switch, double f32_eps) {
    TaylorTable t{};
    t.m_max = m_max;
    t.theta[0] = 0.0;
    for (int m = 1; m <= kTaylorMMax; ++m) {
        double lo = 0.0, hi = std::min(64.0, (m + 2.0) * (1.0 - 1e-12));
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (lo + hi);
            const double lb = (m + 1) * std::log(mid) - std::lgamma(m + 2.0) - std::log1p(-mid / (m + 2.0));
            if (lb <= std::log(tol)) lo = mid; else hi = mid;
        }
        t.theta[m] = lo;
    }
    double f = 1.0;
    for (int k = 0; k <= kTaylorMMax; ++k) {
        if (k > 0) f *= k;
        t.inv_fact[k] = 1.0 / f;
        t.inv_k[k] = k > 0 ? 1.0 / k : 0.0;
        t.inv_fact_f[k] = float(t.inv_fact[k]);
    }
    for (int m = 0; m <= kTaylorMMax; ++m) {
        int k0 = m + 1;
        if (f32_eps > 0.0) {
            k0 = 2;
            while (k0 <= m && k0 * std::log(t.theta[m]) - std::lgamma(k0 + 1.0) > std::log(f32_eps)) ++k0;
        }
        t.f32_from[m] = k0;
    }
    t.dense_theta = dense_theta;
    int md = 1;
    while (md < kTaylorMMax && t.theta[md] < dense_theta) ++md;
    t.dense_m = md;
    t.dense_switch = dense_switch;
    return t;
}

// The mixed precision's Taylor tolerance and float32 threshold (BMC_MIXED in include/bmc_b200.h); a
// build may set others with -D for a sweep.
#ifndef BMC_MIXED_TOL
#define BMC_MIXED_TOL 1e-8
#endif
#ifndef BMC_MIXED_F32
#define BMC_MIXED_F32 3.0
#endif

__device__ TaylorTable g_tables[3];   // [BMC_F64, BMC_F32, BMC_MIXED], per device

// the three tables, in precision order
void host_tables(TaylorTable* h) {
    h[BMC_F64] = make_table(1e-13, 30, 0.5, 100.0, 1e-6);
    h[BMC_F32] = make_table(std::ldexp(1.0, -24), 16, 0.5, 100.0, 0.0);
    h[BMC_MIXED] = make_table(BMC_MIXED_TOL, 30, 0.5, 100.0, BMC_MIXED_F32);
}

// The host copy of one of the library's device tables: the chain and adjoint kernels take their table by
// value, as a kernel parameter, so that the loads of the Taylor loops with warp-uniform indices come from the
// constant bank. `tt` must point into g_tables (as tables() and noalloc_setup() return).
bmc_status host_table_of(const TaylorTable* tt, TaylorTable* out) {
    static TaylorTable h[3];
    static std::once_flag once;
    std::call_once(once, [] { host_tables(h); });
    // the device address of g_tables, looked up once per device (a call under stream capture then
    // makes no runtime query)
    static std::mutex mu;
    static std::map<int, const TaylorTable*> bases;
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    const TaylorTable* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = bases.find(dev);
        if (it == bases.end()) {
            TaylorTable* b = nullptr;
            CUDA_TRY(cudaGetSymbolAddress((void**)&b, g_tables));
            it = bases.emplace(dev, b).first;
        }
        base = it->second;
    }
    const long long i = tt - base;
    if (i < 0 || i > 2) return fail(BMC_ERR_INVALID, "Taylor table %p is not one of the library's", (const void*)tt);
    *out = h[i];
    return BMC_OK;
}

struct DeviceState {
    bool tables_ready = false;
    TaylorTable* tables = nullptr;   // device address of g_tables, taken once
};
std::mutex g_mu;
std::vector<DeviceState> g_dev;

// Workspaces, one per (device, stream): calls on different streams never share scratch, so they may run
// concurrently from different host threads; calls on one stream are ordered by the stream itself.
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};
std::map<std::pair<int, cudaStream_t>, Workspace> g_ws;

DeviceState& dev_state(int dev) {
    if ((int)g_dev.size() <= dev) g_dev.resize(dev + 1);
    return g_dev[dev];
}

bmc_status tables(int precision, const TaylorTable** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceState& ds = dev_state(dev);
    if (!ds.tables_ready) {
        TaylorTable h[3];
        host_tables(h);
        CUDA_TRY(cudaMemcpyToSymbol(g_tables, h, sizeof(h)));
        CUDA_TRY(cudaGetSymbolAddress((void**)&ds.tables, g_tables));
        ds.tables_ready = true;
    }
    *out = ds.tables + precision;
    return BMC_OK;
}

// The cached workspace of the current device and `st`, grown on demand in stream order: the old buffer
// is released by cudaFreeAsync on the same stream (after the work already queued there that uses it) and
// the new one taken by cudaMallocAsync, so growing never synchronises the device. A call that grows the
// workspace allocates (it is not capturable in a CUDA graph); later calls of the same or a smaller size
// only enqueue kernels.
bmc_status workspace(size_t bytes, cudaStream_t st, void** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    Workspace& w = g_ws[{dev, st}];
    if (w.bytes < bytes) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CUDA_TRY(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone)
            return fail(BMC_ERR_INVALID, "this call needs %zu workspace bytes on a stream that is being captured and "
                        "has %zu: make one call of this size on the same stream before capturing", bytes, w.bytes);
        if (w.ptr) {
            CUDA_TRY(cudaFreeAsync(w.ptr, st));
            w.ptr = nullptr;
            w.bytes = 0;
        }
        const size_t want = bytes + bytes / 4 + (1 << 20);
        CUDA_TRY(cudaMallocAsync(&w.ptr, want, st));
        w.bytes = want;
    }
    *out = w.ptr;
    return BMC_OK;
}

struct Carve {
    char* p;
    size_t used = 0;
    explicit Carve(void* base) : p((char*)base) {}
    template <typename T>
    T* take(size_t n) {
        used = (used + 255) & ~size_t(255);
        T* r = (T*)(p + used);
        used += n * sizeof(T);
        return r;
    }
};
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

bmc_status check_problem(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0) {
    if (!pr || !params || !ev || !m0) return fail(BMC_ERR_INVALID, "null problem, params, events or m0");
    if (pr->n_voxels < 1 || pr->n_offsets < 1 || pr->n_events < 0)
        return fail(BMC_ERR_INVALID, "sizes must be positive (voxels %d, offsets %d, events %d)", pr->n_voxels,
                    pr->n_offsets, pr->n_events);
    if (pr->n_cest < 0 || pr->n_cest > BMC_MAX_CEST)
        return fail(BMC_ERR_UNSUPPORTED, "n_cest %d outside 0..%d", pr->n_cest, BMC_MAX_CEST);
    const int N = 3 * (1 + pr->n_cest) + 1;
    if (pr->mz_loc >= N) return fail(BMC_ERR_INVALID, "mz_loc %d outside the state (size %d)", pr->mz_loc, N);
    if (pr->precision != BMC_F64 && pr->precision != BMC_F32 && pr->precision != BMC_MIXED)
        return fail(BMC_ERR_INVALID, "precision %d is not BMC_F64, BMC_F32 or BMC_MIXED", pr->precision);
    if (pr->n_events > 0 && (!ev->d_type || !ev->d_dt || !ev->d_rf_amp || !ev->d_rf_phase || !ev->d_rf_freq))
        return fail(BMC_ERR_INVALID, "null event field");
    return BMC_OK;
}

bmc_status fill_spread(ChainArgs& a, const bmc_spread* sp) {
    a.n_nodes = 1;
    a.sigma = nullptr;
    a.u[0] = 0.0;
    a.w[0] = 1.0;
    if (!sp) return BMC_OK;
    if (sp->n_nodes < 1 || sp->n_nodes > kMaxNodes || !sp->h_u || !sp->h_w || !sp->d_sigma_hz)
        return fail(BMC_ERR_INVALID, "spread: 1..%d nodes with u, w and sigma required", kMaxNodes);
    a.n_nodes = sp->n_nodes;
    for (int j = 0; j < sp->n_nodes; ++j) {
        a.u[j] = sp->h_u[j];
        a.w[j] = sp->h_w[j];
    }
    a.sigma = sp->d_sigma_hz;
    return BMC_OK;
}

// the repeated block of every row of a table of records (block_scan_kernel), into seg[n_rows]
bmc_status scan_blocks(const EvRec<double>* rec, int n_rows, int n_ev, int stride, int4* seg, cudaStream_t st) {
    if (n_rows <= 0) return BMC_OK;
    block_scan_kernel<double><<<(n_rows + kBlockScanRows - 1) / kBlockScanRows, kBlockScanThreads, 0, st>>>(
        rec, n_rows, n_ev, stride, seg);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

template <typename R>
bmc_status prep_events(const bmc_problem* pr, const bmc_events* ev, EvRec<R>* out, cudaStream_t st) {
    const size_t n = (size_t)pr->n_offsets * pr->n_events;
    if (n == 0) return BMC_OK;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    prep_events_kernel<R><<<blocks, 256, 0, st>>>(pr->n_offsets, pr->n_events, ev->d_type, ev->d_dt, ev->d_rf_amp,
                                                  ev->d_rf_phase, ev->d_rf_freq, out);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}


// ------------------------------------------------------------------------------------------------
// FMA throughput probe: kChains independent fused multiply-add chains per thread, in registers
// ------------------------------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, R seed, R* sink) {
    constexpr int kChains = 8;
    R a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) a[j] = seed + R(threadIdx.x + j);
    const R b = R(0.999999), c = R(1e-7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < kChains; ++j) a[j] = fma(a[j], b, c);
    }
    R s = R(0);
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += a[j];
    if (s == R(-1.2345)) sink[blockIdx.x] = s;      // never true; keeps the loop alive
}

// ------------------------------------------------------------------------------------------------
// launches
// ------------------------------------------------------------------------------------------------
template <int NC, typename R, int NT, bool U, bool COUNT>
bmc_status launch_chain_impl(const ChainArgs& a, const TaylorTable* tt, cudaStream_t st) {
    constexpr int kWarps = ChainLaunch<NC, NT>::kWarps;
    const size_t smem = kWarps * sizeof(DenseSmem<NC, typename DenseReal<R>::type, NT>) +
                        32 * kWarps * sizeof(ChainConst<NC, Dn<R, NT>>);
    // the attribute once per device and instantiation: later calls then only enqueue work (which keeps
    // them capturable in a CUDA graph). Atomic: calls on several devices may come from several threads.
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !((configured.load(std::memory_order_acquire) >> dev) & 1ull)) {
        CUDA_TRY(cudaFuncSetAttribute(chain_kernel<NC, R, NT, U, COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        if (dev < 64) configured.fetch_or(1ull << dev, std::memory_order_acq_rel);
    }
    const long long nch = U ? a.n_chains : (long long)a.n_vox * a.n_off;
    const long long blocks = (nch + kWarps * 32 - 1) / (kWarps * 32);
    if (blocks > 0x7fffffffLL) return fail(BMC_ERR_INVALID, "%lld chains exceed one launch", nch);
    if (blocks == 0) return BMC_OK;
    TaylorTable th;
    if (bmc_status s = host_table_of(tt, &th); s != BMC_OK) return s;
    chain_kernel<NC, R, NT, U, COUNT><<<(unsigned)blocks, kWarps * 32, smem, st>>>(a, th);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

// the counting instantiation only where a.work asks for counts (the uneven plans never do)
template <int NC, typename R, int NT, bool U = false>
bmc_status launch_chain(const ChainArgs& a, const TaylorTable* tt, cudaStream_t st) {
    if constexpr (!U) {
        if (a.work) return launch_chain_impl<NC, R, NT, U, true>(a, tt, st);
    } else {
        if (a.work) return fail(BMC_ERR_UNSUPPORTED, "work counts of an uneven plan");
    }
    return launch_chain_impl<NC, R, NT, U, false>(a, tt, st);
}

// Tangent mode (bmc_set_tangent_mode): BMC_TANGENTS_AUTO takes the adjoint kernel where it applies.
std::atomic<int> g_tangent_mode{BMC_TANGENTS_AUTO};

template <int NC, bool kTan = true>
bmc_status launch_adjoint(const ChainArgs& a, const int* row_ev, int n_tan, const TaylorTable* tt, cudaStream_t st) {
    const size_t smem = kAdjWarps * AdjGroup<NC>::G * sizeof(AdjSlot<NC>);
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !((configured.load(std::memory_order_acquire) >> dev) & 1ull)) {
        CUDA_TRY(cudaFuncSetAttribute(adjoint_kernel<NC, kTan>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        if (dev < 64) configured.fetch_or(1ull << dev, std::memory_order_acq_rel);
    }
    const long long nch = (long long)a.n_vox * a.n_off;
    const long long blocks = (nch + kAdjWarps * 32 - 1) / (kAdjWarps * 32);
    if (blocks > 0x7fffffffLL) return fail(BMC_ERR_INVALID, "%lld chains exceed one launch", nch);
    if (blocks == 0) return BMC_OK;
    TaylorTable th;
    if (bmc_status s = host_table_of(tt, &th); s != BMC_OK) return s;
    adjoint_kernel<NC, kTan><<<(unsigned)blocks, kAdjWarps * 32, smem, st>>>(a, row_ev, n_tan, th);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

template <int NC, bool kTan = true>
bmc_status launch_adjoint_block(const ChainArgs& a, const int4* blk, int n_tan, const TaylorTable* tt, cudaStream_t st) {
    const size_t smem = kAdjBlkWarps * DenseGroup<NC>::G * sizeof(AdjBlkSlot<NC, kTan>);
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !((configured.load(std::memory_order_acquire) >> dev) & 1ull)) {
        CUDA_TRY(cudaFuncSetAttribute(adjoint_block_kernel<NC, kTan>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        if (dev < 64) configured.fetch_or(1ull << dev, std::memory_order_acq_rel);
    }
    const long long blocks = (a.n_chains + kAdjBlkWarps * 32 - 1) / (kAdjBlkWarps * 32);
    if (blocks > 0x7fffffffLL) return fail(BMC_ERR_INVALID, "%lld chains exceed one launch", a.n_chains);
    if (blocks == 0) return BMC_OK;
    TaylorTable th;
    if (bmc_status s = host_table_of(tt, &th); s != BMC_OK) return s;
    adjoint_block_kernel<NC, kTan><<<(unsigned)blocks, kAdjBlkWarps * 32, smem, st>>>(a, blk, n_tan, th);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

// Whether the tangents of a uniform table go through the adjoint kernel: two or more tangents, the
// automatic mode, and every row a single-event row (adjoint_rows_kernel, which also fills row_ev). The
// check reads one flag back, so a stream being captured keeps forward mode.
bmc_status use_adjoint(const EvRec<double>* rec, const bmc_problem* pr, int n_tan, int* row_ev, int* flag,
                       cudaStream_t st, bool* ok) {
    *ok = false;
    if (n_tan < 2 || g_tangent_mode.load(std::memory_order_relaxed) != BMC_TANGENTS_AUTO || pr->mz_loc < 0 ||
        pr->n_events < 1 || pr->n_offsets < 1)
        return BMC_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return BMC_OK;
    CUDA_TRY(cudaMemsetAsync(flag, 1, sizeof(int), st));    // nonzero: every row so far qualifies
    adjoint_rows_kernel<<<(pr->n_offsets + 127) / 128, 128, 0, st>>>(rec, pr->n_offsets, pr->n_events,
                                                                      pr->reset_after_adc, row_ev, flag);
    CUDA_TRY(cudaGetLastError());
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *ok = h != 0;
    return BMC_OK;
}

// Order the chains by estimated cost: `order` and the sort's scratch are carved from `cv`.
template <int NC, typename R>
bmc_status order_chains(ChainArgs& a, Carve& cv, cudaStream_t st) {
    const long long nch = (long long)a.n_vox * a.n_off;
    if (nch < 2 * 128 || a.n_ev == 0) return BMC_OK;
    float* k_in = cv.take<float>(nch);
    float* k_out = cv.take<float>(nch);
    int* i_in = cv.take<int>(nch);
    int* i_out = cv.take<int>(nch);
    size_t tmp = 0;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in, k_out, i_in, i_out, (int)nch, 0, 32, st));
    void* t = cv.take<char>(tmp);
    cost_kernel<NC, R><<<(unsigned)((nch + 127) / 128), 128, 0, st>>>(a, k_in, i_in);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, k_in, k_out, i_in, i_out, (int)nch, 0, 32, st));
    a.order = i_out;
    return BMC_OK;
}

// scratch bytes order_chains carves for n chains
size_t order_bytes(long long nch) {
    size_t tmp = 0;
    float* f = nullptr;
    int* i = nullptr;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, f, f, i, i, (int)std::max<long long>(nch, 1), 0, 32);
    return 4 * align256(sizeof(float) * nch) + align256(tmp) + 1024;
}

// tangents per launch, by pool count (register budget of the dual-number state)
template <int NC>
constexpr int tangents_per_pass() { return NC <= 1 ? 2 : 1; }

template <int NC, bool U = false>
bmc_status run_tangents(ChainArgs a, int P, const TaylorTable* tt, cudaStream_t st) {
    constexpr int TP = tangents_per_pass<NC>();
    for (int t0 = 0; t0 < P; t0 += TP) {
        a.t0 = t0;
        bmc_status s = (P - t0 >= 2 && TP >= 2) ? launch_chain<NC, double, (TP >= 2 ? 2 : 1), U>(a, tt, st)
                                                : launch_chain<NC, double, 1, U>(a, tt, st);
        if (s != BMC_OK) return s;
    }
    return BMC_OK;
}

// An uneven batch: voxels with their own event tables, one pool count. Owns its device buffers
// (preprocessed records of every table, the chain map, the sort scratch); built by bmc_uneven_create.
struct UnevenPlan {
    int dev = 0, n_cest = 0, n_vox = 0, mz = 0, reset = 1, n_tables = 0;
    long long n_chains = 0, n_rec = 0;
    EvRec<double>* rec = nullptr;
    int2* chain_map = nullptr;
    int* vox_table = nullptr;
    long long* tab_base = nullptr;
    int* tab_noff = nullptr;
    int* tab_nev = nullptr;
    int4* seg = nullptr;       // the repeated block of every row of every table
    int* tab_row0 = nullptr;   // first row of each table in seg
    double dense_switch = 0.0; // > 0: the dense path's norm threshold for this plan (bmc_uneven_set_dense_switch)
    int4* adj_blk = nullptr;   // per row: the block the adjoint block kernel takes (adjoint_block_rows_kernel)
    int adj_ok = 0;            // every row of every table qualifies: tangents go through that kernel
    void* scratch = nullptr;   // sort keys and indices, cub scratch, status word
    size_t scratch_bytes = 0;
};

template <int NC>
struct Impl {
    static constexpr int N = Layout<NC>::N;

    // one simulation (or tangent set) of an uneven batch: chains sorted by estimated cost, outputs
    // in canonical chain order (voxel-major, then table row)
    static bmc_status uneven(const UnevenPlan& pl, const double* params, const double* m0, const bmc_spread* sp,
                             const bmc_tangents* tg, const int32_t* active, double* z, double* jz, cudaStream_t st) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(BMC_F64, &tt);
        if (s != BMC_OK) return s;
        ChainArgs a{};
        a.n_vox = pl.n_vox; a.n_off = 1; a.n_ev = 0; a.n_fields = Layout<NC>::NF;
        a.mz = pl.mz; a.reset_after_adc = pl.reset;
        if ((s = fill_spread(a, sp)) != BMC_OK) return s;
        a.params = params; a.m0 = m0; a.out = z; a.jout = jz;
        a.ev = pl.rec;
        a.n_chains = pl.n_chains; a.chain_map = pl.chain_map; a.vox_table = pl.vox_table;
        a.tab_base = pl.tab_base; a.tab_noff = pl.tab_noff; a.tab_nev = pl.tab_nev;
        a.seg = pl.seg; a.tab_row0 = pl.tab_row0; a.active = active; a.dense_switch = pl.dense_switch;
        Carve cv(pl.scratch);
        a.status = cv.take<int>(1);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));
        const long long nch = pl.n_chains;
        if (nch >= 2 * 128) {
            float* k_in = cv.take<float>(nch);
            float* k_out = cv.take<float>(nch);
            int* i_in = cv.take<int>(nch);
            int* i_out = cv.take<int>(nch);
            size_t tmp = 0;
            CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in, k_out, i_in, i_out, (int)nch, 0, 32, st));
            void* t = cv.take<char>(tmp);
            if (cv.used > pl.scratch_bytes) return fail(BMC_ERR_INVALID, "uneven plan: scratch too small");
            cost_kernel<NC, double, true><<<(unsigned)((nch + 127) / 128), 128, 0, st>>>(a, k_in, i_in);
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, k_in, k_out, i_in, i_out, (int)nch, 0, 32, st));
            a.order = i_out;
        }
        // the plan's primal passes: the block kernel's layout without tangents where its rows qualify
        // (forward mode keeps the chain kernel for them too)
        const bool adj = pl.adj_ok && g_tangent_mode.load(std::memory_order_relaxed) == BMC_TANGENTS_AUTO;
        if (!tg) return adj ? launch_adjoint_block<NC, false>(a, pl.adj_blk, 0, tt, st)
                            : launch_chain<NC, double, 0, true>(a, tt, st);
        for (int t = 0; t < tg->n_tangents; ++t) a.field_row[t] = tg->field_row[t];
        a.seed = tg->d_seed;
        a.dm0 = tg->d_dm0;
        if (adj && tg->n_tangents >= 2) return launch_adjoint_block<NC, true>(a, pl.adj_blk, tg->n_tangents, tt, st);
        return run_tangents<NC, true>(a, tg->n_tangents, tt, st);
    }

    static bmc_status simulate(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                               const bmc_spread* sp, double* out, cudaStream_t st, unsigned long long* work = nullptr) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(pr->precision, &tt);
        if (s != BMC_OK) return s;
        const size_t nrec = (size_t)pr->n_offsets * pr->n_events;
        void* ws = nullptr;
        const size_t recb = pr->precision == BMC_F32 ? sizeof(EvRec<float>) : sizeof(EvRec<double>);
        const long long nch = (long long)pr->n_voxels * pr->n_offsets;
        if ((s = workspace(align256(nrec * recb) + 256 + align256(sizeof(int4) * pr->n_offsets) + order_bytes(nch), st,
                           &ws)) != BMC_OK)
            return s;
        Carve cv(ws);
        ChainArgs a{};
        a.n_vox = pr->n_voxels; a.n_off = pr->n_offsets; a.n_ev = pr->n_events; a.n_fields = Layout<NC>::NF;
        a.mz = pr->mz_loc; a.reset_after_adc = pr->reset_after_adc;
        if ((s = fill_spread(a, sp)) != BMC_OK) return s;
        a.params = params; a.m0 = m0; a.out = out; a.work = work;
        a.status = cv.take<int>(1);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));
        if (pr->precision == BMC_F32) {
            EvRec<float>* rec = cv.take<EvRec<float>>(nrec);
            if ((s = prep_events<float>(pr, ev, rec, st)) != BMC_OK) return s;
            a.ev = rec;
            if ((s = order_chains<NC, float>(a, cv, st)) != BMC_OK) return s;
            return launch_chain<NC, float, 0>(a, tt, st);
        }
        EvRec<double>* rec = cv.take<EvRec<double>>(nrec);
        if ((s = prep_events<double>(pr, ev, rec, st)) != BMC_OK) return s;
        a.ev = rec;
        a.seg = cv.take<int4>(pr->n_offsets);
        if ((s = scan_blocks(rec, pr->n_offsets, pr->n_events, pr->n_offsets, const_cast<int4*>(a.seg), st)) != BMC_OK)
            return s;
        if ((s = order_chains<NC, double>(a, cv, st)) != BMC_OK) return s;
        return launch_chain<NC, double, 0>(a, tt, st);
    }

    static bmc_status trajectory(const bmc_problem* pr, const double* params, const bmc_events* ev,
                                 const double* m0, double* traj, cudaStream_t st) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(BMC_F64, &tt);
        if (s != BMC_OK) return s;
        const size_t nrec = (size_t)pr->n_offsets * pr->n_events;
        void* ws = nullptr;
        if ((s = workspace(align256(nrec * sizeof(EvRec<double>)) + 256 + align256(sizeof(double) * pr->n_voxels * pr->n_offsets), st, &ws)) != BMC_OK) return s;
        Carve cv(ws);
        ChainArgs a{};
        a.n_vox = pr->n_voxels; a.n_off = pr->n_offsets; a.n_ev = pr->n_events; a.n_fields = Layout<NC>::NF;
        a.mz = Layout<NC>::izw; a.reset_after_adc = pr->reset_after_adc;
        fill_spread(a, nullptr);
        a.params = params; a.m0 = m0; a.traj = traj;
        a.status = cv.take<int>(1);
        a.out = cv.take<double>((size_t)pr->n_voxels * pr->n_offsets);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));
        EvRec<double>* rec = cv.take<EvRec<double>>(nrec);
        if ((s = prep_events<double>(pr, ev, rec, st)) != BMC_OK) return s;
        a.ev = rec;
        return launch_chain<NC, double, 0>(a, tt, st);
    }

    static bmc_status jvp(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                          const bmc_spread* sp, const bmc_tangents* tg, double* z, double* jz, cudaStream_t st,
                          unsigned long long* work = nullptr) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(BMC_F64, &tt);
        if (s != BMC_OK) return s;
        const size_t nrec = (size_t)pr->n_offsets * pr->n_events;
        void* ws = nullptr;
        const long long nch = (long long)pr->n_voxels * pr->n_offsets;
        if ((s = workspace(align256(nrec * sizeof(EvRec<double>)) + 256 + align256(sizeof(int4) * pr->n_offsets) +
                               align256(sizeof(int) * pr->n_offsets) + 256 + order_bytes(nch), st, &ws)) != BMC_OK)
            return s;
        Carve cv(ws);
        ChainArgs a{};
        a.n_vox = pr->n_voxels; a.n_off = pr->n_offsets; a.n_ev = pr->n_events; a.n_fields = Layout<NC>::NF;
        a.mz = pr->mz_loc; a.reset_after_adc = pr->reset_after_adc;
        if ((s = fill_spread(a, sp)) != BMC_OK) return s;
        a.params = params; a.m0 = m0; a.out = z; a.jout = jz; a.work = work;
        for (int t = 0; t < tg->n_tangents; ++t) a.field_row[t] = tg->field_row[t];
        a.seed = tg->d_seed; a.dm0 = tg->d_dm0;
        a.status = cv.take<int>(1);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));
        EvRec<double>* rec = cv.take<EvRec<double>>(nrec);
        if ((s = prep_events<double>(pr, ev, rec, st)) != BMC_OK) return s;
        a.ev = rec;
        a.seg = cv.take<int4>(pr->n_offsets);
        if ((s = scan_blocks(rec, pr->n_offsets, pr->n_events, pr->n_offsets, const_cast<int4*>(a.seg), st)) != BMC_OK)
            return s;
        int* row_ev = cv.take<int>(pr->n_offsets);
        int* flag = cv.take<int>(1);
        bool adj = false;
        if ((s = use_adjoint(rec, pr, tg->n_tangents, row_ev, flag, st, &adj)) != BMC_OK) return s;
        if ((s = order_chains<NC, double>(a, cv, st)) != BMC_OK) return s;
        if (adj) return launch_adjoint<NC>(a, row_ev, tg->n_tangents, tt, st);
        return run_tangents<NC>(a, tg->n_tangents, tt, st);
    }

    // Z, its tangents and the derivatives of both along one design direction (design_kernel): one launch
    // per tangent, the direction's records prepared beside the table's
    static bmc_status design(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                             const double* params_dir, const bmc_events* ev_dir, const double* m0_dir,
                             const bmc_tangents* tg, double* z, double* jz, double* dz, double* djz, cudaStream_t st) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(BMC_F64, &tt);
        if (s != BMC_OK) return s;
        const size_t nrec = (size_t)pr->n_offsets * pr->n_events;
        const long long nch = (long long)pr->n_voxels * pr->n_offsets;
        const size_t mats = (size_t)nch * (2 * N * N + N);           // Phi, its square, psi per chain
        void* ws = nullptr;
        if ((s = workspace(2 * align256(nrec * sizeof(EvRec<double>)) + 256 + align256(mats * sizeof(Dn<HD, 1>)),
                           st, &ws)) != BMC_OK)
            return s;
        Carve cv(ws);
        ChainArgs a{};
        a.n_vox = pr->n_voxels; a.n_off = pr->n_offsets; a.n_ev = pr->n_events; a.n_fields = Layout<NC>::NF;
        a.mz = pr->mz_loc; a.reset_after_adc = pr->reset_after_adc;
        if ((s = fill_spread(a, nullptr)) != BMC_OK) return s;
        a.params = params; a.params_dir = params_dir; a.m0 = m0; a.out = z; a.jout = jz;
        for (int t = 0; t < tg->n_tangents; ++t) a.field_row[t] = tg->field_row[t];
        a.seed = tg->d_seed;
        a.status = cv.take<int>(1);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));
        EvRec<double>* rec = cv.take<EvRec<double>>(nrec);
        if ((s = prep_events<double>(pr, ev, rec, st)) != BMC_OK) return s;
        a.ev = rec;
        DesignArgs d{};
        if (ev_dir && nrec > 0) {
            EvRec<double>* dr = cv.take<EvRec<double>>(nrec);
            const int blocks = (int)std::min<size_t>((nrec + 255) / 256, 148 * 16);
            prep_dir_kernel<<<blocks, 256, 0, st>>>(pr->n_offsets, pr->n_events, ev->d_rf_phase, ev_dir->d_dt,
                                                   ev_dir->d_rf_amp, ev_dir->d_rf_phase, ev_dir->d_rf_freq, dr);
            CUDA_TRY(cudaGetLastError());
            d.ev_dir = dr;
        }
        d.m0_dir = m0_dir; d.dz = dz; d.djz = djz;
        d.scratch = reinterpret_cast<double*>(cv.take<Dn<HD, 1>>(mats));
        const long long blocks = (nch + 127) / 128;
        if (blocks > 0x7fffffffLL) return fail(BMC_ERR_INVALID, "%lld chains exceed one launch", nch);
        for (int t = 0; t < tg->n_tangents; ++t) {
            a.t0 = t;
            design_kernel<NC, 1><<<(unsigned)blocks, 128, 0, st>>>(a, d, tt);
            CUDA_TRY(cudaGetLastError());
        }
        return BMC_OK;
    }

    static bmc_status lm(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                         const bmc_spread* sp, const bmc_fit_spec* fs, const double* zm, const double* x0,
                         double* x_out, double* cost_traj, double* x_traj, cudaStream_t st) {
        const TaylorTable* tt = nullptr;
        bmc_status s = tables(BMC_F64, &tt);
        if (s != BMC_OK) return s;
        const int nv = pr->n_voxels, no = pr->n_offsets, P = fs->n_params;
        constexpr int NF = Layout<NC>::NF;
        const size_t nrec = (size_t)no * pr->n_events;
        const size_t bytes = align256(nrec * sizeof(EvRec<double>)) + 2 * align256(sizeof(double) * NF * nv) +
                             2 * align256(sizeof(double) * N * nv) + 2 * align256(sizeof(double) * nv) +
                             align256(sizeof(double) * P * nv) + align256(sizeof(double) * P * nv * N) +
                             2 * align256(sizeof(double) * nv * no) + align256(sizeof(double) * P * nv * no) +
                             2 * align256(sizeof(double) * nv * P) + 2 * align256(sizeof(double) * nv) +
                             align256(sizeof(int) * nv) + align256(sizeof(int4) * no) + 4096 +
                             align256(sizeof(int) * no) + 256 + order_bytes((long long)nv * no);
        void* ws = nullptr;
        if ((s = workspace(bytes, st, &ws)) != BMC_OK) return s;
        Carve cv(ws);
        EvRec<double>* rec = cv.take<EvRec<double>>(nrec);
        double* px = cv.take<double>((size_t)NF * nv);
        double* pt = cv.take<double>((size_t)NF * nv);
        double* m0x = cv.take<double>((size_t)N * nv);
        double* m0t = cv.take<double>((size_t)N * nv);
        double* sgx = cv.take<double>(nv);
        double* sgt = cv.take<double>(nv);
        double* seed = cv.take<double>((size_t)P * nv);
        double* dm0 = cv.take<double>((size_t)P * nv * N);
        double* z = cv.take<double>((size_t)nv * no);
        double* zt = cv.take<double>((size_t)nv * no);
        double* J = cv.take<double>((size_t)P * nv * no);
        double* x = cv.take<double>((size_t)nv * P);
        double* xt = cv.take<double>((size_t)nv * P);
        double* lam = cv.take<double>(nv);
        double* cost = cv.take<double>(nv);
        int* need = cv.take<int>(nv);
        int4* seg = cv.take<int4>(no);
        int* status = cv.take<int>(1);
        int* row_ev = cv.take<int>(no);
        int* flag = cv.take<int>(1);
        if ((s = prep_events<double>(pr, ev, rec, st)) != BMC_OK) return s;
        CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), st));
        CUDA_TRY(cudaMemcpyAsync(x, x0, sizeof(double) * nv * P, cudaMemcpyDeviceToDevice, st));
        std::vector<double> hl(nv, fs->lam0);
        std::vector<int> hn(nv, 1);
        CUDA_TRY(cudaMemcpyAsync(lam, hl.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(need, hn.data(), sizeof(int) * nv, cudaMemcpyHostToDevice, st));

        SlotSpec ss{};
        ss.P = P;
        bool has_m = false;
        for (int p = 0; p < P; ++p) {
            ss.field_row[p] = fs->field_row[p]; ss.mode[p] = fs->mode[p]; ss.scale[p] = fs->scale[p];
            ss.lo[p] = fs->lo[p]; ss.hi[p] = fs->hi[p];
            has_m = has_m || fs->field_row[p] == BMC_SLOT_M_START;
        }
        ChainArgs a{};
        a.n_vox = nv; a.n_off = no; a.n_ev = pr->n_events; a.n_fields = NF;
        a.mz = pr->mz_loc; a.reset_after_adc = pr->reset_after_adc;
        if ((s = fill_spread(a, sp)) != BMC_OK) return s;
        const double* sig0 = sp ? sp->d_sigma_hz : nullptr;
        a.ev = rec; a.status = status; a.seg = seg;
        if ((s = scan_blocks(rec, no, pr->n_events, no, seg, st)) != BMC_OK) return s;
        bool adj = false;
        if ((s = use_adjoint(rec, pr, P, row_ev, flag, st, &adj)) != BMC_OK) return s;
        a.params = params; a.m0 = m0;
        if ((s = order_chains<NC, double>(a, cv, st)) != BMC_OK) return s;
        for (int p = 0; p < P; ++p) a.field_row[p] = fs->field_row[p] == BMC_SLOT_M_START ? BMC_SEED_NONE : fs->field_row[p];
        const int vb = (nv + 127) / 128, wb = (nv + 3) / 4;
        for (int it = 0; it < fs->n_iter; ++it) {
            // residual and Jacobian at x, for the voxels whose x moved
            lm_params_kernel<NC><<<vb, 128, 0, st>>>(nv, ss, params, m0, sig0, x, fs->d_free, px, m0x,
                                                      sp ? sgx : nullptr, seed, has_m ? dm0 : nullptr);
            CUDA_TRY(cudaGetLastError());
            ChainArgs aj = a;
            aj.params = px; aj.m0 = m0x; aj.sigma = sp ? sgx : nullptr; aj.seed = seed; aj.dm0 = has_m ? dm0 : nullptr;
            aj.active = need; aj.out = z; aj.jout = J;
            if ((s = adj ? launch_adjoint<NC>(aj, row_ev, P, tt, st) : run_tangents<NC>(aj, P, tt, st)) != BMC_OK)
                return s;
            lm_solve_kernel<<<wb, 128, 0, st>>>(nv, no, fs->n_points_skip, ss, z, zm, J, fs->d_free, x, lam, cost, xt);
            CUDA_TRY(cudaGetLastError());
            // the trial point
            lm_params_kernel<NC><<<vb, 128, 0, st>>>(nv, ss, params, m0, sig0, xt, fs->d_free, pt, m0t,
                                                      sp ? sgt : nullptr, nullptr, nullptr);
            CUDA_TRY(cudaGetLastError());
            ChainArgs at = a;
            at.params = pt; at.m0 = m0t; at.sigma = sp ? sgt : nullptr; at.out = zt;
            // the trial point's Z: with the adjoint tangents, the same dense layout without H
            if ((s = adj ? launch_adjoint<NC, false>(at, row_ev, 0, tt, st) : launch_chain<NC, double, 0>(at, tt, st)) !=
                BMC_OK)
                return s;
            lm_accept_kernel<<<wb, 128, 0, st>>>(nv, no, fs->n_points_skip, P, it, fs->n_iter, zt, zm, cost, xt, x,
                                                 lam, need, cost_traj, x_traj);
            CUDA_TRY(cudaGetLastError());
        }
        CUDA_TRY(cudaMemcpyAsync(x_out, x, sizeof(double) * nv * P, cudaMemcpyDeviceToDevice, st));
        return BMC_OK;
    }
};


}  // namespace

// ------------------------------------------------------------------------------------------------
// exported entry points
// ------------------------------------------------------------------------------------------------
#define BMC_DISPATCH(nc, call)                                   \
    switch (nc) {                                                \
        case 0: return Impl<0>::call;                            \
        case 1: return Impl<1>::call;                            \
        case 2: return Impl<2>::call;                            \
        case 3: return Impl<3>::call;                            \
        case 4: return Impl<4>::call;                            \
        case 5: return Impl<5>::call;                            \
        default: return fail(BMC_ERR_UNSUPPORTED, "n_cest %d", nc); \
    }

extern "C" {

int32_t bmc_abi_version(void) { return BMC_ABI_VERSION; }

const char* bmc_version(void) { return "bmc_b200 0.1.0 (sm_100a)"; }

size_t bmc_last_error(char* buf, size_t n) {
    if (buf && n) {
        const size_t k = std::min(n - 1, g_err.size());
        std::memcpy(buf, g_err.data(), k);
        buf[k] = 0;
    }
    return g_err.size();
}

bmc_status bmc_release(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    cudaError_t first = cudaSuccess;
    for (auto& kv : g_ws) {
        if (!kv.second.ptr) continue;
        cudaSetDevice(kv.first.first);
        const cudaError_t e = cudaFreeAsync(kv.second.ptr, kv.first.second);
        if (first == cudaSuccess) first = e;
    }
    for (auto& kv : g_ws) {
        if (!kv.second.ptr) continue;
        cudaSetDevice(kv.first.first);
        const cudaError_t e = cudaStreamSynchronize(kv.first.second);
        if (first == cudaSuccess) first = e;
    }
    g_ws.clear();
    cudaSetDevice(cur);
    if (first != cudaSuccess) return fail(BMC_ERR_CUDA, "bmc_release: %s", cudaGetErrorString(first));
    return BMC_OK;
}

bmc_status bmc_simulate(const bmc_problem* prob, const double* d_params, const bmc_events* ev, const double* d_m0,
                        const bmc_spread* spread, double* d_out, void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!d_out) return fail(BMC_ERR_INVALID, "null output");
    BMC_DISPATCH(prob->n_cest, simulate(prob, d_params, ev, d_m0, spread, d_out, (cudaStream_t)stream));
}

bmc_status bmc_simulate_counted(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                const double* d_m0, const bmc_spread* spread, double* d_out,
                                unsigned long long* d_work, void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!d_out || !d_work) return fail(BMC_ERR_INVALID, "null output or counters");
    BMC_DISPATCH(prob->n_cest, simulate(prob, d_params, ev, d_m0, spread, d_out, (cudaStream_t)stream, d_work));
}

bmc_status bmc_simulate_trajectory(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                   const double* d_m0, double* d_traj, void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!d_traj) return fail(BMC_ERR_INVALID, "null output");
    BMC_DISPATCH(prob->n_cest, trajectory(prob, d_params, ev, d_m0, d_traj, (cudaStream_t)stream));
}

namespace {
bmc_status check_jvp(const bmc_problem* prob, const double* d_params, const bmc_events* ev, const double* d_m0,
                     const bmc_tangents* tan, const double* d_z, const double* d_jz) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!tan || tan->n_tangents < 1 || tan->n_tangents > BMC_MAX_TANGENTS)
        return fail(BMC_ERR_INVALID, "tangents: 1..%d required", BMC_MAX_TANGENTS);
    if (!tan->d_seed) return fail(BMC_ERR_INVALID, "tangents: null seed array");
    if (prob->mz_loc < 0) return fail(BMC_ERR_INVALID, "bmc_simulate_jvp needs mz_loc >= 0");
    if (prob->precision != BMC_F64) return fail(BMC_ERR_UNSUPPORTED, "tangents are computed in float64 only");
    if (!d_z || !d_jz) return fail(BMC_ERR_INVALID, "null output");
    const int nf = BMC_N_FIELDS(prob->n_cest);
    for (int t = 0; t < tan->n_tangents; ++t)
        if (tan->field_row[t] >= nf || tan->field_row[t] < BMC_SEED_SPREAD_SIGMA)
            return fail(BMC_ERR_INVALID, "tangent %d: field row %d outside -2..%d", t, tan->field_row[t], nf - 1);
    return BMC_OK;
}
}  // namespace

bmc_status bmc_set_tangent_mode(int32_t mode) {
    if (mode != BMC_TANGENTS_AUTO && mode != BMC_TANGENTS_FORWARD)
        return fail(BMC_ERR_INVALID, "tangent mode %d: BMC_TANGENTS_AUTO or BMC_TANGENTS_FORWARD", mode);
    g_tangent_mode.store(mode, std::memory_order_relaxed);
    return BMC_OK;
}

bmc_status bmc_simulate_jvp_counted(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                    const double* d_m0, const bmc_spread* spread, const bmc_tangents* tan,
                                    double* d_z, double* d_jz, unsigned long long* d_work, void* stream) {
    bmc_status s = check_jvp(prob, d_params, ev, d_m0, tan, d_z, d_jz);
    if (s != BMC_OK) return s;
    if (!d_work) return fail(BMC_ERR_INVALID, "null counters");
    BMC_DISPATCH(prob->n_cest, jvp(prob, d_params, ev, d_m0, spread, tan, d_z, d_jz, (cudaStream_t)stream, d_work));
}

bmc_status bmc_simulate_jvp(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                            const double* d_m0, const bmc_spread* spread, const bmc_tangents* tan, double* d_z,
                            double* d_jz, void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!tan || tan->n_tangents < 1 || tan->n_tangents > BMC_MAX_TANGENTS)
        return fail(BMC_ERR_INVALID, "tangents: 1..%d required", BMC_MAX_TANGENTS);
    if (!tan->d_seed) return fail(BMC_ERR_INVALID, "tangents: null seed array");
    if (prob->mz_loc < 0) return fail(BMC_ERR_INVALID, "bmc_simulate_jvp needs mz_loc >= 0");
    if (prob->precision != BMC_F64) return fail(BMC_ERR_UNSUPPORTED, "tangents are computed in float64 only");
    if (!d_z || !d_jz) return fail(BMC_ERR_INVALID, "null output");
    const int nf = BMC_N_FIELDS(prob->n_cest);
    for (int t = 0; t < tan->n_tangents; ++t)
        if (tan->field_row[t] >= nf || tan->field_row[t] < BMC_SEED_SPREAD_SIGMA)
            return fail(BMC_ERR_INVALID, "tangent %d: field row %d outside -2..%d", t, tan->field_row[t], nf - 1);
    BMC_DISPATCH(prob->n_cest, jvp(prob, d_params, ev, d_m0, spread, tan, d_z, d_jz, (cudaStream_t)stream));
}

bmc_status bmc_simulate_design_jvp(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                   const double* d_m0, const double* d_params_dir, const bmc_events* ev_dir,
                                   const double* d_m0_dir, const bmc_tangents* tan, double* d_z, double* d_jz,
                                   double* d_dz, double* d_djz, void* stream) {
    bmc_status s = check_jvp(prob, d_params, ev, d_m0, tan, d_z, d_jz);
    if (s != BMC_OK) return s;
    if (!d_dz || !d_djz) return fail(BMC_ERR_INVALID, "null design-derivative output");
    if (tan->d_dm0) return fail(BMC_ERR_UNSUPPORTED, "bmc_simulate_design_jvp: start-state tangents (d_dm0)");
    for (int t = 0; t < tan->n_tangents; ++t)
        if (tan->field_row[t] < 0)
            return fail(BMC_ERR_UNSUPPORTED, "bmc_simulate_design_jvp: tangent %d seeds the spread (no spread here)", t);
    BMC_DISPATCH(prob->n_cest, design(prob, d_params, ev, d_m0, d_params_dir, ev_dir, d_m0_dir, tan, d_z, d_jz, d_dz,
                                      d_djz, (cudaStream_t)stream));
}

bmc_status bmc_lm_fit(const bmc_problem* prob, const double* d_params, const bmc_events* ev, const double* d_m0,
                      const bmc_spread* spread, const bmc_fit_spec* spec, const double* d_z_meas, const double* d_x0,
                      double* d_x_out, double* d_cost_traj, double* d_x_traj, void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!spec || spec->n_params < 1 || spec->n_params > BMC_MAX_TANGENTS)
        return fail(BMC_ERR_INVALID, "fit spec: 1..%d parameters required", BMC_MAX_TANGENTS);
    if (spec->n_iter < 0) return fail(BMC_ERR_INVALID, "n_iter %d", spec->n_iter);
    if (prob->mz_loc < 0) return fail(BMC_ERR_INVALID, "bmc_lm_fit needs mz_loc >= 0");
    if (spec->n_points_skip < 0 || spec->n_points_skip >= prob->n_offsets)
        return fail(BMC_ERR_INVALID, "n_points_skip %d", spec->n_points_skip);
    if (!d_z_meas || !d_x0 || !d_x_out) return fail(BMC_ERR_INVALID, "null z_meas, x0 or x_out");
    const int nf = BMC_N_FIELDS(prob->n_cest);
    for (int p = 0; p < spec->n_params; ++p) {
        const int fr = spec->field_row[p];
        if (fr >= nf || fr < BMC_SLOT_M_START)
            return fail(BMC_ERR_INVALID, "slot %d: field row %d outside -3..%d", p, fr, nf - 1);
        if (spec->mode[p] < 0 || spec->mode[p] > 2) return fail(BMC_ERR_INVALID, "slot %d: mode %d", p, spec->mode[p]);
        if (fr == BMC_SLOT_SPREAD_SIGMA && !spread)
            return fail(BMC_ERR_INVALID, "slot %d: the spread width needs a spread", p);
    }
    BMC_DISPATCH(prob->n_cest, lm(prob, d_params, ev, d_m0, spread, spec, d_z_meas, d_x0, d_x_out, d_cost_traj,
                                  d_x_traj, (cudaStream_t)stream));
}

bmc_status bmc_normal_blocks(int32_t n_voxels, int32_t n_points, int32_t n_tangents, const double* d_r,
                             const double* d_jz, double* d_H, double* d_g, double* d_c, void* stream) {
    if (n_voxels < 1 || n_points < 1 || n_tangents < 1 || n_tangents > BMC_MAX_TANGENTS)
        return fail(BMC_ERR_INVALID, "normal blocks: bad sizes (%d, %d, %d)", n_voxels, n_points, n_tangents);
    if (!d_r || !d_jz || !d_H || !d_g || !d_c) return fail(BMC_ERR_INVALID, "normal blocks: null pointer");
    normal_blocks_kernel<<<(n_voxels + 3) / 4, 128, 0, (cudaStream_t)stream>>>(n_voxels, n_points, n_tangents, d_r,
                                                                               d_jz, d_H, d_g, d_c);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_uneven_create(int32_t n_cest, int32_t n_voxels, const int32_t* h_voxel_table,
                             const bmc_table_set* tabs, int32_t mz_loc, int32_t reset_after_adc, void** plan,
                             int64_t* n_chains, int64_t* h_chain_start) {
    if (!plan) return fail(BMC_ERR_INVALID, "uneven: null plan pointer");
    *plan = nullptr;
    if (n_cest < 0 || n_cest > BMC_MAX_CEST) return fail(BMC_ERR_UNSUPPORTED, "n_cest %d outside 0..%d", n_cest, BMC_MAX_CEST);
    if (n_voxels < 1 || !h_voxel_table || !tabs || tabs->n_tables < 1 || !tabs->h_n_offsets || !tabs->h_n_events)
        return fail(BMC_ERR_INVALID, "uneven: voxels, their tables and the table sizes are required");
    const int N = 3 * (1 + n_cest) + 1;
    if (mz_loc < 0 || mz_loc >= N) return fail(BMC_ERR_INVALID, "mz_loc %d outside the state (size %d)", mz_loc, N);
    const int nt = tabs->n_tables;
    std::vector<long long> base(nt);
    long long nrec = 0;
    for (int t = 0; t < nt; ++t) {
        if (tabs->h_n_offsets[t] < 1 || tabs->h_n_events[t] < 0)
            return fail(BMC_ERR_INVALID, "uneven: table %d has %d rows and %d events", t, tabs->h_n_offsets[t],
                        tabs->h_n_events[t]);
        base[t] = nrec;
        nrec += (long long)tabs->h_n_offsets[t] * tabs->h_n_events[t];
    }
    if (nrec > 0 && (!tabs->ev.d_type || !tabs->ev.d_dt || !tabs->ev.d_rf_amp || !tabs->ev.d_rf_phase ||
                     !tabs->ev.d_rf_freq))
        return fail(BMC_ERR_INVALID, "uneven: null event field");
    std::vector<int2> cm;
    std::vector<long long> start((size_t)n_voxels + 1);
    for (int v = 0; v < n_voxels; ++v) {
        const int t = h_voxel_table[v];
        if (t < 0 || t >= nt) return fail(BMC_ERR_INVALID, "uneven: voxel %d names table %d of %d", v, t, nt);
        start[v] = (long long)cm.size();
        for (int o = 0; o < tabs->h_n_offsets[t]; ++o) cm.push_back(make_int2(v, o));
    }
    start[n_voxels] = (long long)cm.size();
    const long long nch = (long long)cm.size();
    if (nch > 0x7fffffffLL) return fail(BMC_ERR_INVALID, "uneven: %lld chains exceed one launch", nch);
    UnevenPlan* pl = new UnevenPlan();
    pl->n_cest = n_cest; pl->n_vox = n_voxels; pl->mz = mz_loc; pl->reset = reset_after_adc ? 1 : 0;
    pl->n_tables = nt; pl->n_chains = nch; pl->n_rec = nrec;
    auto undo = [&](bmc_status s) {
        bmc_uneven_destroy(pl);
        return s;
    };
    cudaError_t e = cudaGetDevice(&pl->dev);
    std::vector<int> noff(tabs->h_n_offsets, tabs->h_n_offsets + nt), nev(tabs->h_n_events, tabs->h_n_events + nt);
    std::vector<int> row0(nt);
    long long n_rows = 0;
    for (int t = 0; t < nt; ++t) {
        row0[t] = (int)n_rows;
        n_rows += noff[t];
    }
    pl->scratch_bytes = 256 + order_bytes(nch);
    if (e == cudaSuccess) e = cudaMalloc(&pl->rec, sizeof(EvRec<double>) * std::max<long long>(nrec, 1));
    if (e == cudaSuccess) e = cudaMalloc(&pl->chain_map, sizeof(int2) * std::max<long long>(nch, 1));
    if (e == cudaSuccess) e = cudaMalloc(&pl->vox_table, sizeof(int) * n_voxels);
    if (e == cudaSuccess) e = cudaMalloc(&pl->tab_base, sizeof(long long) * nt);
    if (e == cudaSuccess) e = cudaMalloc(&pl->tab_noff, sizeof(int) * nt);
    if (e == cudaSuccess) e = cudaMalloc(&pl->tab_nev, sizeof(int) * nt);
    if (e == cudaSuccess) e = cudaMalloc(&pl->scratch, pl->scratch_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&pl->seg, sizeof(int4) * std::max<long long>(n_rows, 1));
    if (e == cudaSuccess) e = cudaMalloc(&pl->tab_row0, sizeof(int) * nt);
    if (e == cudaSuccess) e = cudaMalloc(&pl->adj_blk, sizeof(int4) * std::max<long long>(n_rows, 1));
    if (e == cudaSuccess) e = cudaMemcpy(pl->tab_row0, row0.data(), sizeof(int) * nt, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nch) e = cudaMemcpy(pl->chain_map, cm.data(), sizeof(int2) * nch, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->vox_table, h_voxel_table, sizeof(int) * n_voxels, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->tab_base, base.data(), sizeof(long long) * nt, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->tab_noff, noff.data(), sizeof(int) * nt, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pl->tab_nev, nev.data(), sizeof(int) * nt, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return undo(fail(BMC_ERR_CUDA, "uneven plan: %s", cudaGetErrorString(e)));
    // every table's [n_offsets][n_events] arrays, concatenated in table order -> records [n_events][n_offsets]
    for (int t = 0; t < nt; ++t) {
        const size_t n = (size_t)noff[t] * nev[t];
        if (!n) continue;
        const long long b = base[t];
        const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
        prep_events_kernel<double><<<blocks, 256>>>(noff[t], nev[t], tabs->ev.d_type + b, tabs->ev.d_dt + b,
                                                    tabs->ev.d_rf_amp + b, tabs->ev.d_rf_phase + b,
                                                    tabs->ev.d_rf_freq + b, pl->rec + b);
    }
    for (int t = 0; t < nt; ++t) {
        if (e == cudaSuccess && nev[t] > 0)
            block_scan_kernel<double><<<(noff[t] + kBlockScanRows - 1) / kBlockScanRows, kBlockScanThreads>>>(
                pl->rec + base[t], noff[t], nev[t], noff[t], pl->seg + row0[t]);
        else if (e == cudaSuccess)
            e = cudaMemset(pl->seg + row0[t], 0, sizeof(int4) * noff[t]);
    }
    // the rows the adjoint block kernel takes (a flag in the plan's scratch, read back once here)
    int* adj_flag = static_cast<int*>(pl->scratch);
    if (e == cudaSuccess) e = cudaMemset(adj_flag, 1, sizeof(int));
    for (int t = 0; t < nt && e == cudaSuccess; ++t) {
        if (nev[t] > 0 && noff[t] > 0)
            adjoint_block_rows_kernel<<<(noff[t] + 127) / 128, 128>>>(pl->rec + base[t], noff[t], nev[t], noff[t],
                                                                     pl->seg + row0[t], reset_after_adc,
                                                                     pl->adj_blk + row0[t], adj_flag);
        else
            e = cudaMemset(adj_flag, 0, sizeof(int));
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int h_flag = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h_flag, adj_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return undo(fail(BMC_ERR_CUDA, "uneven plan: %s", cudaGetErrorString(e)));
    pl->adj_ok = h_flag != 0;
    if (n_chains) *n_chains = nch;
    if (h_chain_start) std::memcpy(h_chain_start, start.data(), sizeof(long long) * start.size());
    *plan = pl;
    return BMC_OK;
}

bmc_status bmc_uneven_simulate(const void* plan, const double* d_params, const double* d_m0,
                               const bmc_spread* spread, const bmc_tangents* tangents, const int32_t* d_active,
                               double* d_z, double* d_jz, void* stream) {
    if (!plan || !d_params || !d_m0 || !d_z) return fail(BMC_ERR_INVALID, "uneven: null plan, params, m0 or z");
    const UnevenPlan* pl = static_cast<const UnevenPlan*>(plan);
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != pl->dev) return fail(BMC_ERR_INVALID, "uneven: plan made on device %d, called on %d", pl->dev, dev);
    if (tangents) {
        const int nf = 13 + 5 * pl->n_cest;
        if (tangents->n_tangents < 1 || tangents->n_tangents > BMC_MAX_TANGENTS || !tangents->d_seed || !d_jz)
            return fail(BMC_ERR_INVALID, "uneven: 1..%d tangents with seeds and an output required", BMC_MAX_TANGENTS);
        const int lo = spread ? BMC_SEED_SPREAD_SIGMA : BMC_SEED_NONE;
        for (int t = 0; t < tangents->n_tangents; ++t)
            if (tangents->field_row[t] < lo || tangents->field_row[t] >= nf)
                return fail(BMC_ERR_INVALID, "tangent %d: field row %d outside %d..%d", t, tangents->field_row[t], lo,
                            nf - 1);
    }
    BMC_DISPATCH(pl->n_cest, uneven(*pl, d_params, d_m0, spread, tangents, d_active, d_z, d_jz, (cudaStream_t)stream));
}

bmc_status bmc_uneven_set_dense_switch(void* plan, double norm) {
    if (!plan) return fail(BMC_ERR_INVALID, "uneven: null plan");
    if (!(norm >= 0.0) || norm > 1e6) return fail(BMC_ERR_INVALID, "uneven: dense-path norm %g outside 0..1e6", norm);
    static_cast<UnevenPlan*>(plan)->dense_switch = norm;
    return BMC_OK;
}

bmc_status bmc_uneven_uses_block_kernel(const void* plan, int32_t* out) {
    if (!plan || !out) return fail(BMC_ERR_INVALID, "uneven: null plan or output");
    *out = static_cast<const UnevenPlan*>(plan)->adj_ok &&
           g_tangent_mode.load(std::memory_order_relaxed) == BMC_TANGENTS_AUTO;
    return BMC_OK;
}

bmc_status bmc_uneven_destroy(void* plan) {
    UnevenPlan* pl = static_cast<UnevenPlan*>(plan);
    if (!pl) return BMC_OK;
    void* ptrs[] = {pl->rec, pl->chain_map, pl->vox_table, pl->tab_base, pl->tab_noff, pl->tab_nev, pl->scratch,
                    pl->seg, pl->tab_row0, pl->adj_blk};
    cudaError_t first = cudaSuccess;
    for (void* p : ptrs) {
        if (!p) continue;
        const cudaError_t e = cudaFree(p);
        if (first == cudaSuccess) first = e;
    }
    delete pl;
    if (first != cudaSuccess) return fail(BMC_ERR_CUDA, "uneven plan: %s", cudaGetErrorString(first));
    return BMC_OK;
}

bmc_status bmc_normal_segments(int32_t n_voxels, int32_t n_params, int64_t n_chains, const int64_t* d_chain_start,
                               const double* d_jz, const double* d_r, double* d_H, double* d_g, double* d_c,
                               void* stream) {
    if (n_voxels < 1 || n_params < 1 || n_params > kMaxJointP || n_chains < 0)
        return fail(BMC_ERR_INVALID, "normal segments: %d voxels, %d parameters (1..%d)", n_voxels, n_params, kMaxJointP);
    if (!d_chain_start || !d_jz || !d_r || !d_H || !d_g || !d_c)
        return fail(BMC_ERR_INVALID, "normal segments: null pointer");
    const long long threads = (long long)n_voxels * 32;
    normal_segments_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        n_voxels, n_params, n_chains, reinterpret_cast<const long long*>(d_chain_start), d_jz, d_r, d_H, d_g, d_c);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_schur_step(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_H, const double* d_g,
                          const double* d_free, double lam, const double* d_lam, double* d_dx_local,
                          double* d_dx_shared, double* d_work, void* stream) {
    if (n_voxels < 1 || n_local < 1 || n_local > kMaxJointP - 1 || (n_shared != 0 && n_shared != 1))
        return fail(BMC_ERR_INVALID, "schur step: %d voxels, %d local (1..%d) and %d shared (0 or 1) values",
                    n_voxels, n_local, kMaxJointP - 1, n_shared);
    if (!d_H || !d_g || !d_dx_local || !d_dx_shared || !d_work) return fail(BMC_ERR_INVALID, "schur step: null pointer");
    if (!d_lam && !(lam >= 0.0)) return fail(BMC_ERR_INVALID, "schur step: damping %g", lam);
    double* sums = d_work + (size_t)n_voxels * (2 * n_local + 4);
    bmc_status s = bmc_schur_eliminate(n_voxels, n_local, n_shared, d_H, d_g, d_free, lam, d_lam, d_work, sums, stream);
    if (s != BMC_OK) return s;
    return bmc_schur_back(n_voxels, n_local, n_shared, sums, lam, d_lam, d_work, d_dx_local, d_dx_shared, stream);
}

bmc_status bmc_schur_eliminate(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_H,
                               const double* d_g, const double* d_free, double lam, const double* d_lam,
                               double* d_work, double* d_sums, void* stream) {
    if (n_voxels < 1 || n_local < 1 || n_local > kMaxJointP - 1 || (n_shared != 0 && n_shared != 1))
        return fail(BMC_ERR_INVALID, "schur step: %d voxels, %d local (1..%d) and %d shared (0 or 1) values",
                    n_voxels, n_local, kMaxJointP - 1, n_shared);
    if (!d_H || !d_g || !d_work || !d_sums) return fail(BMC_ERR_INVALID, "schur step: null pointer");
    if (!d_lam && !(lam >= 0.0)) return fail(BMC_ERR_INVALID, "schur step: damping %g", lam);
    const cudaStream_t st = (cudaStream_t)stream;
    double* Y = d_work;
    double* w = Y + (size_t)n_voxels * n_local;
    double* red = w + (size_t)n_voxels * n_local;
    schur_eliminate_kernel<<<(n_voxels + 127) / 128, 128, 0, st>>>(n_voxels, n_local, n_shared, d_H, d_g, d_free, lam,
                                                                   d_lam, Y, w, red);
    CUDA_TRY(cudaGetLastError());
    schur_sum_kernel<<<1, 1024, 0, st>>>(n_voxels, red, d_sums);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_schur_back(int32_t n_voxels, int32_t n_local, int32_t n_shared, const double* d_sums, double lam,
                          const double* d_lam, const double* d_work, double* d_dx_local, double* d_dx_shared,
                          void* stream) {
    if (n_voxels < 1 || n_local < 1 || n_local > kMaxJointP - 1 || (n_shared != 0 && n_shared != 1))
        return fail(BMC_ERR_INVALID, "schur step: %d voxels, %d local (1..%d) and %d shared (0 or 1) values",
                    n_voxels, n_local, kMaxJointP - 1, n_shared);
    if (!d_sums || !d_work || !d_dx_local || !d_dx_shared) return fail(BMC_ERR_INVALID, "schur step: null pointer");
    if (!d_lam && !(lam >= 0.0)) return fail(BMC_ERR_INVALID, "schur step: damping %g", lam);
    const cudaStream_t st = (cudaStream_t)stream;
    const double* Y = d_work;
    const double* w = Y + (size_t)n_voxels * n_local;
    schur_shared_kernel<<<1, 32, 0, st>>>(n_shared, d_sums, lam, d_lam, d_dx_shared);
    CUDA_TRY(cudaGetLastError());
    const long long n = (long long)n_voxels * n_local;
    schur_back_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n_voxels, n_local, Y, w, d_dx_shared, d_dx_local);
    CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_probe_fma_peak(int32_t precision, int32_t blocks, int32_t iters, double* flops_per_launch,
                              void* stream) {
    if (blocks < 1 || iters < 1 || !flops_per_launch) return fail(BMC_ERR_INVALID, "probe: bad arguments");
    if (precision == BMC_F32)
        fma_probe_kernel<float><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0f, nullptr);
    else
        fma_probe_kernel<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 1.0, nullptr);
    CUDA_TRY(cudaGetLastError());
    *flops_per_launch = 2.0 * 8.0 * 256.0 * (double)blocks * (double)iters;
    return BMC_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// bmc_simulate_noalloc: the forward model with no device allocation at all
// ------------------------------------------------------------------------------------------------
// Some callers cannot let a library call cudaMalloc: a handler running inside JAX/XLA (JAX reserves
// most of the GPU's memory for its own allocator up front, so a cudaMalloc there can fail, and memory
// taken behind XLA's back is not accounted for), code running under another framework's caching
// allocator with a fixed memory budget, and latency-bound pipelines, for which cudaMalloc/cudaFree
// are unbounded-latency calls that synchronise the device. For them this entry point takes its only
// scratch -- the preprocessed event records and a status word -- from one static device array,
// g_noalloc_scratch, of kNoAllocScratchBytes on every GPU that loads the library (held until the
// process exits). The chains run in launch order (no cost sort, which would need more scratch); the
// results are bit-identical to bmc_simulate's, since every chain chooses its own Taylor degree, sub-steps
// and float32 switch point whatever chains share its warp. The array is reserved by the driver when it
// loads this library's device code on a device (under lazy loading: the first bmc_* call there), so a
// caller whose framework reserves the GPU up front makes a first call before that (or loads eagerly).
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;     // 32 MiB per GPU
constexpr size_t kNoAllocStatusBytes = 256;
size_t noalloc_seg_bytes(long long n_rows) { return align256(sizeof(int4) * (size_t)n_rows); }
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};               // device address of the array, per device
bool g_noalloc_tables[kNoAllocMaxDevices] = {};

// Once per device, with that device current: the device address of the static array (in host code
// its name is only a host-side stand-in) and the Taylor tables. Runs inside the first call on a
// device, which should therefore come before any stream capture.
bmc_status noalloc_setup(int precision, void** scratch, const TaylorTable** tt) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return fail(BMC_ERR_UNSUPPORTED, "bmc_simulate_noalloc: device %d above %d", dev, kNoAllocMaxDevices - 1);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_tables[dev]) {
        TaylorTable h[3];
        host_tables(h);
        CUDA_TRY(cudaMemcpyToSymbol(g_tables, h, sizeof(h)));
        g_noalloc_tables[dev] = true;
    }
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(BMC_ERR_CUDA, "bmc_simulate_noalloc: cudaGetSymbolAddress of the static scratch: %s",
                        cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    TaylorTable* t = nullptr;
    CUDA_TRY(cudaGetSymbolAddress((void**)&t, g_tables));
    *tt = t + precision;
    *scratch = g_noalloc_ptr[dev];
    return BMC_OK;
}

template <int NC>
struct NoAlloc {
    template <typename R>
    static bmc_status run(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                          const bmc_spread* sp, double* out, void* scratch, const TaylorTable* tt, cudaStream_t st) {
        ChainArgs a{};
        a.n_vox = pr->n_voxels; a.n_off = pr->n_offsets; a.n_ev = pr->n_events; a.n_fields = Layout<NC>::NF;
        a.mz = pr->mz_loc; a.reset_after_adc = pr->reset_after_adc;
        bmc_status s = fill_spread(a, sp);
        if (s != BMC_OK) return s;
        a.params = params; a.m0 = m0; a.out = out;
        a.status = static_cast<int*>(scratch);
        CUDA_TRY(cudaMemsetAsync(a.status, 0, sizeof(int), st));          // must start at zero each call
        // the scratch: the status word, every row's repeated block, the event records
        int4* seg = reinterpret_cast<int4*>(static_cast<char*>(scratch) + kNoAllocStatusBytes);
        EvRec<R>* rec = reinterpret_cast<EvRec<R>*>(static_cast<char*>(scratch) + kNoAllocStatusBytes +
                                                    noalloc_seg_bytes(pr->n_offsets));
        if ((s = prep_events<R>(pr, ev, rec, st)) != BMC_OK) return s;   // overwrites the previous call's
        a.ev = rec;
        if constexpr (std::is_same<R, double>::value) {
            if ((s = scan_blocks(rec, pr->n_offsets, pr->n_events, pr->n_offsets, seg, st)) != BMC_OK) return s;
            a.seg = seg;
        }
        return launch_chain<NC, R, 0>(a, tt, st);
    }

    static bmc_status simulate(const bmc_problem* pr, const double* params, const bmc_events* ev, const double* m0,
                               const bmc_spread* sp, double* out, void* scratch, const TaylorTable* tt,
                               cudaStream_t st) {
        return pr->precision == BMC_F32 ? run<float>(pr, params, ev, m0, sp, out, scratch, tt, st)
                                        : run<double>(pr, params, ev, m0, sp, out, scratch, tt, st);
    }
};

}  // namespace

extern "C" bmc_status bmc_simulate_noalloc(const bmc_problem* prob, const double* d_params, const bmc_events* ev,
                                           const double* d_m0, const bmc_spread* spread, double* d_out,
                                           void* stream) {
    bmc_status s = check_problem(prob, d_params, ev, d_m0);
    if (s != BMC_OK) return s;
    if (!d_out) return fail(BMC_ERR_INVALID, "null output");
    const size_t rec_bytes = prob->precision == BMC_F32 ? sizeof(EvRec<float>) : sizeof(EvRec<double>);
    const size_t nrec = (size_t)prob->n_offsets * (size_t)prob->n_events;
    const size_t fixed = kNoAllocStatusBytes + noalloc_seg_bytes(prob->n_offsets);
    const size_t cap = fixed < kNoAllocScratchBytes ? (kNoAllocScratchBytes - fixed) / rec_bytes : 0;
    if (nrec > cap)
        return fail(BMC_ERR_INVALID,
                    "bmc_simulate_noalloc: the event table (%d offsets x %d events = %zu records of %zu bytes) "
                    "exceeds its static scratch of %zu bytes (at most %zu records); use bmc_simulate",
                    prob->n_offsets, prob->n_events, nrec, rec_bytes, kNoAllocScratchBytes, cap);
    void* scratch = nullptr;
    const TaylorTable* tt = nullptr;
    if ((s = noalloc_setup(prob->precision, &scratch, &tt)) != BMC_OK) return s;
    const cudaStream_t st = (cudaStream_t)stream;
    switch (prob->n_cest) {
        case 0: return NoAlloc<0>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        case 1: return NoAlloc<1>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        case 2: return NoAlloc<2>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        case 3: return NoAlloc<3>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        case 4: return NoAlloc<4>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        case 5: return NoAlloc<5>::simulate(prob, d_params, ev, d_m0, spread, d_out, scratch, tt, st);
        default: return fail(BMC_ERR_UNSUPPORTED, "n_cest %d", prob->n_cest);
    }
}
