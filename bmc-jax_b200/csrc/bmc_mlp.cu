// bmc_mlp.cu -- the learned warm start: a multilayer perceptron that maps a measured saturation ladder
// (Z values) to normalised starting values for the Levenberg-Marquardt fit, trained and evaluated on
// the 5th-generation tensor cores of sm_100a.
//
// Every dense product is one hand-written kernel, `gemm_kernel`: C[M][N] = A[M][K] * B[N][K]^T with
// A and B in bf16 (K contiguous), the product accumulated in fp32 in tensor memory (TMEM) by
// `tcgen05.mma.cta_group::1.kind::f16` (M = 128 rows per CTA, N = the CTA's column tile, K = 16 per
// instruction), issued by one thread. Operand tiles (128 x 64 of A, N x 64 of B) are staged in shared
// memory in the canonical K-major no-swizzle layout (8-row x 16-byte core matrices: 128 B between
// neighbours along K, 1024 B between 8-row groups) by cp.async, two stages deep; an mbarrier that
// `tcgen05.commit` arrives on tells the CTA when a stage may be overwritten and when the accumulator
// is complete. The epilogue reads the accumulator back with `tcgen05.ld` (warp w owns TMEM lanes
// 32w..32w+31 = rows of C) and fuses what follows the product: bias + GELU (+ transposed copy for the
// weight gradient), bias only, GELU' times the back-propagated gradient (+ bias-gradient column sums),
// or split-K accumulation of a weight gradient.
//
// Layers (all padded to multiples of 64; the padding is zero in weights, inputs and gradients):
//   h_1 = gelu(W_1 x + b_1), h_l = gelu(W_l h_{l-1} + b_l) (l = 2..L), y = W_o h_L + b_o
// Loss: mean over the batch and the n_out outputs of (y - t)^2. Optimiser: Adam with bias correction.
//
// Every wait is bounded (about two seconds of SM clock); a CTA that gives up sets bit 0 of the status
// word at the start of the work buffer, waits (bounded) for its MMAs in flight, frees its TMEM and
// returns.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "../../include/bmc_b200.h"

namespace bmc {
bmc_status record_error(bmc_status s, const char* msg);
}

namespace {

using bf16 = __nv_bfloat16;

bmc_status fail(bmc_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return bmc::record_error(s, buf);
}

#define MLP_CUDA_TRY(expr)                                                                      \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return fail(BMC_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------------------------------------
// PTX wrappers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// wait for the phase of the given parity, for at most ~2^32 SM cycles (about two seconds)
__device__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1LL << 32)) return false;
    return true;
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation: executed by one whole warp; the address lands in shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (TMEM, fp32) (+)= A (smem, bf16) * B (smem, bf16)^T, one M=128 x N x K=16 step
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// the mbarrier receives one arrival when every MMA this thread issued so far has completed
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// 16 consecutive fp32 columns of this thread's TMEM lane; the wait is tied to the registers
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                   "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// shared-memory matrix descriptor: K-major, no swizzle, 128 B between core matrices along K (LBO),
// 1024 B between 8-row groups (SBO), descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t(128 >> 4) << 16) | (uint64_t(1024 >> 4) << 32) |
           (uint64_t(1) << 46);
}
// instruction descriptor: fp32 accumulator, bf16 A and B, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

// ------------------------------------------------------------------------------------------------
// activation
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    // d/dz [z Phi(z)] = Phi(z) + z phi(z)
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ------------------------------------------------------------------------------------------------
// the GEMM
// ------------------------------------------------------------------------------------------------
enum : int { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_DHIDDEN = 2, EPI_DW = 3 };

struct GemmArgs {
    const bf16* A;
    int lda;  // [M][K]
    const bf16* B;
    int ldb;  // [N][K]
    int M, N, K;
    int k_split;  // K range of one blockIdx.z (multiple of 64)
    int m_valid;  // rows >= m_valid are computed but not stored
    // epilogue operands (see each EPI_*)
    const float* bias;  // [N]
    float* zf;          // HIDDEN: pre-activation out; DHIDDEN: pre-activation in  [M][ldz]
    int ldz;
    bf16* h;            // HIDDEN: gelu(z); DHIDDEN: dz  [M][ldh]
    int ldh;
    bf16* ht;           // transposed copy of h [N][ldht] (may be null)
    int ldht;
    float* out;         // OUT: y [M][ldo]; DW: gradient accumulated with atomics [M][ldo]
    int ldo;
    float* out2;        // OUT: caller's y [m_valid2][n_valid2]
    int ld2, m_valid2, n_valid2;
    float* dbias;       // DHIDDEN: column sums of dz (atomics) [N]
    int* status;
};

constexpr int kGemmStages = 3;   // K chunks in flight: a CTA's first three are all loaded before its first MMA

template <int BN>
struct GemmSmem {
    static constexpr uint32_t A_BYTES = 128 * 128;  // 128 rows x 64 bf16
    static constexpr uint32_t B_BYTES = BN * 128;
    static constexpr uint32_t STAGE = A_BYTES + B_BYTES;
    static constexpr uint32_t BYTES = kGemmStages * STAGE;
    static constexpr uint32_t NCOLS = BN < 32 ? 32 : BN;  // TMEM columns (power of two >= 32)
};

template <int EPI>
__device__ __forceinline__ void epilogue(const GemmArgs& g, int row, int n, float (&v)[16]) {
    const bool live = row < g.m_valid;
    if constexpr (EPI == EPI_HIDDEN) {
        float hv[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            v[i] += g.bias[n + i];
            hv[i] = gelu(v[i]);
        }
        if (live) {
            if (g.zf) {
                float4* z4 = reinterpret_cast<float4*>(g.zf + size_t(row) * g.ldz + n);
#pragma unroll
                for (int q = 0; q < 4; ++q) z4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
            __align__(16) bf16 hb[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) hb[i] = __float2bfloat16_rn(hv[i]);
            uint4* h4 = reinterpret_cast<uint4*>(g.h + size_t(row) * g.ldh + n);
            h4[0] = reinterpret_cast<const uint4*>(hb)[0];
            h4[1] = reinterpret_cast<const uint4*>(hb)[1];
            if (g.ht) {
#pragma unroll
                for (int i = 0; i < 16; ++i) g.ht[size_t(n + i) * g.ldht + row] = hb[i];
            }
        }
    } else if constexpr (EPI == EPI_OUT) {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += g.bias[n + i];
        if (live) {
            float4* o4 = reinterpret_cast<float4*>(g.out + size_t(row) * g.ldo + n);
#pragma unroll
            for (int q = 0; q < 4; ++q) o4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            if (g.out2 && row < g.m_valid2) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (n + i < g.n_valid2) g.out2[size_t(row) * g.ld2 + n + i] = v[i];
            }
        }
    } else if constexpr (EPI == EPI_DHIDDEN) {
        __align__(16) bf16 db[16];
        float dz[16];
        if (live) {
            const float4* z4 = reinterpret_cast<const float4*>(g.zf + size_t(row) * g.ldz + n);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 z = z4[q];
                dz[4 * q] = v[4 * q] * gelu_grad(z.x);
                dz[4 * q + 1] = v[4 * q + 1] * gelu_grad(z.y);
                dz[4 * q + 2] = v[4 * q + 2] * gelu_grad(z.z);
                dz[4 * q + 3] = v[4 * q + 3] * gelu_grad(z.w);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) dz[i] = 0.0f;
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            db[i] = __float2bfloat16_rn(dz[i]);
            dz[i] = __bfloat162float(db[i]);  // the bias gradient sums what the weight gradient sees
        }
        if (live) {
            uint4* h4 = reinterpret_cast<uint4*>(g.h + size_t(row) * g.ldh + n);
            h4[0] = reinterpret_cast<const uint4*>(db)[0];
            h4[1] = reinterpret_cast<const uint4*>(db)[1];
            if (g.ht) {
#pragma unroll
                for (int i = 0; i < 16; ++i) g.ht[size_t(n + i) * g.ldht + row] = db[i];
            }
        }
        // column sums over the warp's 32 rows, one atomic per column
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float s = dz[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0 && g.dbias) atomicAdd(g.dbias + n + i, s);
        }
    } else {  // EPI_DW
        if (live) {
            float* o = g.out + size_t(row) * g.ldo + n;
            if ((reinterpret_cast<uintptr_t>(o) & 15) == 0) {
                // one 16-byte reduction per four columns (global float4 atomics, sm_90 and later)
                float4* o4 = reinterpret_cast<float4*>(o);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    atomicAdd(o4 + q, make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
            } else {
#pragma unroll
                for (int i = 0; i < 16; ++i) atomicAdd(o + i, v[i]);
            }
        }
    }
}

// 8 warps: the loads and the epilogue are spread over all of them (warps w and w + 4 read the same 32
// TMEM lanes, w & 3, and take the two halves of the tile's columns); one thread issues the MMAs.
constexpr int kGemmThreads = 256;

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 2) gemm_kernel(GemmArgs g) {
    using S = GemmSmem<BN>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[kGemmStages];
    __shared__ uint32_t tmem_slot;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_split;
    const int ke = min(g.K, kb + g.k_split);
    const int nk = (ke - kb) / 64;
    const uint32_t s0 = smem_addr(smem);

    if (warp == 0) tmem_alloc(smem_addr(&tmem_slot), S::NCOLS);
    if (tid == 0) {
#pragma unroll
        for (int i = 0; i < kGemmStages; ++i) mbar_init(smem_addr(&bars[i]), 1);
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    auto load = [&](int stage, int k0) {
        const uint32_t a = s0 + stage * S::STAGE, b = a + S::A_BYTES;
        for (int i = tid; i < 128 * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            cp_async16(a + (r >> 3) * 1024 + c * 128 + (r & 7) * 16, g.A + size_t(m0 + r) * g.lda + k0 + c * 8);
        }
        for (int i = tid; i < BN * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            cp_async16(b + (r >> 3) * 1024 + c * 128 + (r & 7) * 16, g.B + size_t(n0 + r) * g.ldb + k0 + c * 8);
        }
        cp_async_commit();
    };

    // Chunk c uses stage c % kGemmStages; its MMAs are committed to that stage's barrier (phase c / stages),
    // which the CTA waits for before the stage takes chunk c + stages.
    bool ok = true;
    int issued = 0;   // chunks whose loads were issued
    for (; issued < min(nk, kGemmStages); ++issued) load(issued, kb + issued * 64);
    int committed = -1;
    for (int c = 0; ok && c < nk; ++c) {
        const int st = c % kGemmStages;
        const int pending = issued - (c + 1);   // later chunks' load groups that may still be in flight
        if (pending >= 2) cp_async_wait<2>();
        else if (pending == 1) cp_async_wait<1>();
        else cp_async_wait<0>();
        fence_proxy_async();  // this thread's cp.async writes -> visible to the tensor core
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a = s0 + st * S::STAGE, b = a + S::A_BYTES;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                umma_bf16(tmem, smem_desc(a + j * 256), smem_desc(b + j * 256), idesc_bf16(BN), (c | j) != 0);
            umma_commit(smem_addr(&bars[st]));
        }
        committed = c;
        if (issued < nk) {
            // the stage is free once chunk c's MMAs are done
            const bool w = mbar_wait(smem_addr(&bars[st]), (c / kGemmStages) & 1);
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            load(st, kb + issued * 64);
            ++issued;
        }
    }
    if (committed >= 0) {
        // the last commit covers every earlier MMA of the CTA
        const bool w = mbar_wait(smem_addr(&bars[committed % kGemmStages]), (committed / kGemmStages) & 1);
        ok = ok && w;
    }
    ok = __syncthreads_and(ok);
    cp_async_wait<0>();
    tc_fence_after();

    if (ok && nk > 0) {
        const int quarter = warp & 3, half = warp >> 2;
        const int row = m0 + quarter * 32 + lane;
        const uint32_t trow = tmem + (uint32_t(quarter * 32) << 16);
#pragma unroll 1
        for (int cb = half * (BN / 2); cb < (half + 1) * (BN / 2); cb += 16) {
            float v[16];
            tmem_ld16(trow + cb, v);
            epilogue<EPI>(g, row, n0 + cb, v);
        }
    } else if (!ok && tid == 0 && g.status) {
        atomicOr(g.status, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, S::NCOLS);
}

// ------------------------------------------------------------------------------------------------
// element-wise kernels
// ------------------------------------------------------------------------------------------------
// x fp32 [batch][n_in] -> X bf16 [rows][in_pad] and XT bf16 [in_pad][rows], normalised per input
// ((x - shift) * scale), zero in the padding; 32 x 32 tiles through shared memory
__global__ void prep_input_kernel(const float* __restrict__ x, const float* __restrict__ shift,
                                  const float* __restrict__ scale, int batch, int n_in, int rows, int in_pad,
                                  bf16* __restrict__ X, bf16* __restrict__ XT) {
    __shared__ bf16 tile[32][33];
    const int i0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int m = m0 + r, i = i0 + threadIdx.x;
        float v = 0.0f;
        if (m < batch && i < n_in) v = (x[size_t(m) * n_in + i] - (shift ? shift[i] : 0.0f)) * (scale ? scale[i] : 1.0f);
        const bf16 b = __float2bfloat16_rn(v);
        if (m < rows && i < in_pad) X[size_t(m) * in_pad + i] = b;
        tile[r][threadIdx.x] = b;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int i = i0 + r, m = m0 + threadIdx.x;
        if (i < in_pad && m < rows) XT[size_t(i) * rows + m] = tile[threadIdx.x][r];
    }
}

// gradient of the mean squared error at the output: d = 2 (y - t) / (batch n_out), in bf16 (row and
// transposed copies), its column sums into the output-bias gradient, and the loss into *loss
__global__ void loss_kernel(const float* __restrict__ y, int ldy, const float* __restrict__ t, int batch, int n_out,
                            int rows, int out_pad, bf16* __restrict__ d, bf16* __restrict__ dt,
                            float* __restrict__ dbias, float* __restrict__ loss) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const float inv = 1.0f / (float(batch) * float(n_out));
    float lsum = 0.0f;
    for (int j = 0; j < out_pad; ++j) {
        float g = 0.0f;
        if (m < batch && j < n_out) {
            const float e = y[size_t(m) * ldy + j] - t[size_t(m) * n_out + j];
            lsum += e * e * inv;
            g = 2.0f * e * inv;
        }
        const bf16 gb = __float2bfloat16_rn(g);
        if (m < rows) {
            d[size_t(m) * out_pad + j] = gb;
            dt[size_t(j) * rows + m] = gb;
        }
        float s = __bfloat162float(gb);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && j < n_out && s != 0.0f) atomicAdd(dbias + j, s);
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, lsum);
}

constexpr int kMaxLayers = 9;  // up to 8 hidden layers + the output layer

struct LayerMap {
    int n;
    long long off_w[kMaxLayers], off_b[kMaxLayers];
    int rows[kMaxLayers], cols[kMaxLayers];  // padded out x in
    long long sh_w[kMaxLayers], sh_wt[kMaxLayers];  // element offsets of W and W^T in the shadow
};

__device__ __forceinline__ void refresh_shadow(const LayerMap& L, long long p, float w, bf16* shadow) {
    for (int l = 0; l < L.n; ++l) {
        const long long q = p - L.off_w[l];
        if (q >= 0 && q < (long long)L.rows[l] * L.cols[l]) {
            const int o = int(q / L.cols[l]), i = int(q % L.cols[l]);
            const bf16 b = __float2bfloat16_rn(w);
            shadow[L.sh_w[l] + q] = b;
            shadow[L.sh_wt[l] + (long long)i * L.rows[l] + o] = b;
            return;
        }
    }
}

__global__ void sync_kernel(LayerMap L, const float* __restrict__ p, long long n, bf16* __restrict__ shadow) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        refresh_shadow(L, k, p[k], shadow);
}

__global__ void adam_kernel(LayerMap L, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr_t, float b1, float b2, float eps,
                            bf16* __restrict__ shadow) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.0f - b1) * gk;
        const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        const float w = p[k] - lr_t * mk / (sqrtf(vk) + eps);
        p[k] = w;
        refresh_shadow(L, k, w, shadow);
    }
}

// Adam with the step count on the device (a CUDA graph replays it unchanged): the bias-corrected rate of
// step *d_step + 1, computed by every thread as the host entry computes it; the count is advanced by
// step_advance_kernel after the update.
__global__ void adam_dev_kernel(LayerMap L, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, long long n, const int* __restrict__ d_step, float lr, float b1,
                                float b2, float eps, bf16* __restrict__ shadow) {
    const double t = double(*d_step + 1);
    const float lr_t = float(double(lr) * sqrt(1.0 - pow(double(b2), t)) / (1.0 - pow(double(b1), t)));
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const float gk = g[k];
        const float mk = b1 * m[k] + (1.0f - b1) * gk;
        const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        const float w = p[k] - lr_t * mk / (sqrtf(vk) + eps);
        p[k] = w;
        refresh_shadow(L, k, w, shadow);
    }
}

__global__ void step_advance_kernel(int* d_step) { *d_step += 1; }

// ------------------------------------------------------------------------------------------------
// host side: shapes, buffer carving, launches
// ------------------------------------------------------------------------------------------------
long long rup(long long x, long long m) { return (x + m - 1) / m * m; }
size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

struct Shape {
    int n_in, H, L, n_out;  // L hidden layers of width H
    int in_pad, out_pad;
    int layers() const { return L + 1; }
    int in_of(int l) const { return l == 0 ? in_pad : H; }
    int out_of(int l) const { return l == L ? out_pad : H; }
};

bmc_status check_shape(const bmc_mlp_shape* s, Shape* out) {
    if (!s) return fail(BMC_ERR_INVALID, "null MLP shape");
    if (s->n_in < 1 || s->n_out < 1 || s->n_hidden_layers < 1 || s->n_hidden < 128)
        return fail(BMC_ERR_INVALID, "MLP shape: n_in %d, n_out %d, hidden layers %d, width %d", s->n_in, s->n_out,
                    s->n_hidden_layers, s->n_hidden);
    if (s->n_hidden % 128 != 0 || s->n_hidden > 1024)
        return fail(BMC_ERR_UNSUPPORTED, "MLP hidden width %d: a multiple of 128 up to 1024", s->n_hidden);
    if (s->n_hidden_layers > kMaxLayers - 1)
        return fail(BMC_ERR_UNSUPPORTED, "MLP: at most %d hidden layers", kMaxLayers - 1);
    if (s->n_in > 4096 || s->n_out > 128) return fail(BMC_ERR_UNSUPPORTED, "MLP: n_in <= 4096 and n_out <= 128");
    Shape r;
    r.n_in = s->n_in;
    r.H = s->n_hidden;
    r.L = s->n_hidden_layers;
    r.n_out = s->n_out;
    r.in_pad = int(rup(s->n_in, 64));
    r.out_pad = int(rup(s->n_out, 64));
    *out = r;
    return BMC_OK;
}

LayerMap layer_map(const Shape& s) {
    LayerMap m{};
    m.n = s.layers();
    long long off = 0, sh = 0;
    for (int l = 0; l < m.n; ++l) {
        m.rows[l] = s.out_of(l);
        m.cols[l] = s.in_of(l);
        m.off_w[l] = off;
        off += (long long)m.rows[l] * m.cols[l];
        m.off_b[l] = off;
        off += m.rows[l];
        m.sh_w[l] = sh;
        sh += (long long)m.rows[l] * m.cols[l];
        m.sh_wt[l] = sh;
        sh += (long long)m.rows[l] * m.cols[l];
    }
    return m;
}
long long n_params(const Shape& s) {
    const LayerMap m = layer_map(s);
    return m.off_b[m.n - 1] + m.rows[m.n - 1];
}
long long shadow_elems(const Shape& s) {
    const LayerMap m = layer_map(s);
    return m.sh_wt[m.n - 1] + (long long)m.rows[m.n - 1] * m.cols[m.n - 1];
}

// the work buffer of one batch size
struct Work {
    int* status;
    bf16 *X, *XT;
    float* Z[kMaxLayers];
    bf16 *Hb[kMaxLayers], *HT[kMaxLayers];
    float* Y;
    bf16 *dO, *dOT;
    bf16 *dA, *dAT, *dB, *dBT;
    size_t bytes;
    int rows, dot_rows;
};

Work carve(const Shape& s, long long batch, void* base) {
    Work w{};
    w.rows = int(rup(batch, 128));
    w.dot_rows = int(rup(s.out_pad, 128));
    const size_t R = size_t(w.rows);
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t b) {
        void* q = p ? p + off : nullptr;
        off += a256(b);
        return q;
    };
    w.status = static_cast<int*>(take(256));
    w.X = static_cast<bf16*>(take(R * s.in_pad * 2));
    w.XT = static_cast<bf16*>(take(R * s.in_pad * 2));
    for (int l = 0; l < s.L; ++l) {
        w.Z[l] = static_cast<float*>(take(R * s.H * 4));
        w.Hb[l] = static_cast<bf16*>(take(R * s.H * 2));
        w.HT[l] = static_cast<bf16*>(take(R * s.H * 2));
    }
    w.Y = static_cast<float*>(take(R * s.out_pad * 4));
    w.dO = static_cast<bf16*>(take(R * s.out_pad * 2));
    w.dOT = static_cast<bf16*>(take(size_t(w.dot_rows) * R * 2));
    w.dA = static_cast<bf16*>(take(R * s.H * 2));
    w.dAT = static_cast<bf16*>(take(R * s.H * 2));
    w.dB = static_cast<bf16*>(take(R * s.H * 2));
    w.dBT = static_cast<bf16*>(take(R * s.H * 2));
    w.bytes = off;
    return w;
}

template <int BN, int EPI>
bmc_status launch_gemm_t(const GemmArgs& g, int splits, cudaStream_t st) {
    using S = GemmSmem<BN>;
    // the attribute once per device and instantiation (later calls only enqueue work, which keeps them
    // capturable); atomic, as calls on several devices may come from several threads
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    MLP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !((configured.load(std::memory_order_acquire) >> dev) & 1ull)) {
        MLP_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::BYTES));
        if (dev < 64) configured.fetch_or(1ull << dev, std::memory_order_acq_rel);
    }
    dim3 grid(g.M / 128, g.N / BN, splits);
    gemm_kernel<BN, EPI><<<grid, kGemmThreads, S::BYTES, st>>>(g);
    MLP_CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

// C = A B^T with the shapes checked; splits > 1 only for EPI_DW (atomic accumulation)
template <int EPI>
bmc_status gemm(GemmArgs g, int splits, cudaStream_t st) {
    if (g.M % 128 || g.N % 64 || g.K % 64 || g.K < 64 || (g.lda % 8) || (g.ldb % 8))
        return fail(BMC_ERR_INVALID, "gemm %d x %d x %d (lda %d, ldb %d): internal shape error", g.M, g.N, g.K,
                    g.lda, g.ldb);
    if (EPI != EPI_DW) splits = 1;
    const int chunks = g.K / 64;
    splits = std::max(1, std::min(splits, chunks));
    g.k_split = int(rup(chunks, splits) / splits) * 64;
    splits = int((g.K + g.k_split - 1) / g.k_split);
    // 128-wide tiles where they fill the SMs, else 64-wide (twice the CTAs)
    if (g.N % 128 == 0 && (long long)(g.M / 128) * (g.N / 128) * splits >= 148) return launch_gemm_t<128, EPI>(g, splits, st);
    return launch_gemm_t<64, EPI>(g, splits, st);
}

// split-K of a weight gradient: about one CTA per SM over 64-wide tiles (what `gemm` takes for these
// shapes), each CTA accumulating whole 64-deep chunks before its atomics
int dw_splits(int M, int N, int K) {
    const int tiles = (M / 128) * (N / 64);
    return std::max(1, std::min(K / 64, 148 / std::max(1, tiles)));
}

bmc_status forward_impl(const Shape& s, const float* params, const bf16* shadow, const float* x, const float* shift,
                        const float* scale, long long batch, float* y, const Work& w, bool keep,
                        cudaStream_t st) {
    const LayerMap M = layer_map(s);
    {
        dim3 grid(unsigned(rup(s.in_pad, 32) / 32), unsigned(w.rows / 32));
        prep_input_kernel<<<grid, dim3(32, 8), 0, st>>>(x, shift, scale, int(batch), s.n_in, w.rows, s.in_pad,
                                                         w.X, w.XT);
        MLP_CUDA_TRY(cudaGetLastError());
    }
    const bf16* in = w.X;
    int ld_in = s.in_pad;
    for (int l = 0; l < s.L; ++l) {
        GemmArgs g{};
        g.A = in;
        g.lda = ld_in;
        g.B = shadow + M.sh_w[l];
        g.ldb = M.cols[l];
        g.M = w.rows;
        g.N = s.H;
        g.K = M.cols[l];
        g.m_valid = w.rows;
        g.bias = params + M.off_b[l];
        g.zf = keep ? w.Z[l] : nullptr;
        g.ldz = s.H;
        g.h = w.Hb[l];
        g.ldh = s.H;
        g.ht = keep ? w.HT[l] : nullptr;
        g.ldht = w.rows;
        g.status = w.status;
        if (bmc_status e = gemm<EPI_HIDDEN>(g, 1, st)) return e;
        in = w.Hb[l];
        ld_in = s.H;
    }
    GemmArgs g{};
    const int l = s.L;
    g.A = in;
    g.lda = ld_in;
    g.B = shadow + M.sh_w[l];
    g.ldb = M.cols[l];
    g.M = w.rows;
    g.N = s.out_pad;
    g.K = M.cols[l];
    g.m_valid = w.rows;
    g.bias = params + M.off_b[l];
    g.out = w.Y;
    g.ldo = s.out_pad;
    g.out2 = y;
    g.ld2 = s.n_out;
    g.m_valid2 = int(batch);
    g.n_valid2 = s.n_out;
    g.status = w.status;
    return gemm<EPI_OUT>(g, 1, st);
}

bmc_status backward_impl(const Shape& s, const bf16* shadow, const float* target, long long batch, const Work& w,
                         float* grad, float* loss, cudaStream_t st) {
    const LayerMap M = layer_map(s);
    MLP_CUDA_TRY(cudaMemsetAsync(grad, 0, size_t(n_params(s)) * sizeof(float), st));
    MLP_CUDA_TRY(cudaMemsetAsync(w.dOT, 0, size_t(w.dot_rows) * w.rows * 2, st));
    const int lo = s.L;  // output layer index
    loss_kernel<<<unsigned(w.rows / 128), 128, 0, st>>>(w.Y, s.out_pad, target, int(batch), s.n_out, w.rows,
                                                         s.out_pad, w.dO, w.dOT, grad + M.off_b[lo], loss);
    MLP_CUDA_TRY(cudaGetLastError());
    // output layer weight gradient: dW_o = dO^T H_L   (rows of dO^T padded to 128; rows >= out_pad not stored)
    {
        GemmArgs g{};
        g.A = w.dOT;
        g.lda = w.rows;
        g.B = w.HT[s.L - 1];
        g.ldb = w.rows;
        g.M = w.dot_rows;
        g.N = s.H;
        g.K = w.rows;
        g.m_valid = s.out_pad;
        g.out = grad + M.off_w[lo];
        g.ldo = s.H;
        g.status = w.status;
        if (bmc_status e = gemm<EPI_DW>(g, dw_splits(g.M, g.N, g.K), st)) return e;
    }
    // dH_L = dO W_o, times gelu'(Z_L)
    const bf16* dcur = w.dO;
    int ld_cur = s.out_pad;
    bf16 *nxt = w.dA, *nxtT = w.dAT, *oth = w.dB, *othT = w.dBT;
    for (int l = s.L; l >= 1; --l) {
        // gradient wrt the input of layer l (= output of hidden layer l-1)
        GemmArgs g{};
        g.A = dcur;
        g.lda = ld_cur;
        g.B = shadow + M.sh_wt[l];
        g.ldb = M.rows[l];
        g.M = w.rows;
        g.N = s.H;
        g.K = M.rows[l];
        g.m_valid = w.rows;
        g.zf = w.Z[l - 1];
        g.ldz = s.H;
        g.h = nxt;
        g.ldh = s.H;
        g.ht = nxtT;
        g.ldht = w.rows;
        g.dbias = grad + M.off_b[l - 1];
        g.status = w.status;
        if (bmc_status e = gemm<EPI_DHIDDEN>(g, 1, st)) return e;
        // weight gradient of layer l-1: dW = dZ^T (input of layer l-1)
        GemmArgs d{};
        d.A = nxtT;
        d.lda = w.rows;
        d.B = (l - 1 == 0) ? w.XT : w.HT[l - 2];
        d.ldb = w.rows;
        d.M = s.H;
        d.N = M.cols[l - 1];
        d.K = w.rows;
        d.m_valid = s.H;
        d.out = grad + M.off_w[l - 1];
        d.ldo = M.cols[l - 1];
        d.status = w.status;
        if (bmc_status e = gemm<EPI_DW>(d, dw_splits(d.M, d.N, d.K), st)) return e;
        dcur = nxt;
        ld_cur = s.H;
        std::swap(nxt, oth);
        std::swap(nxtT, othT);
    }
    return BMC_OK;
}

}  // namespace

extern "C" {

bmc_status bmc_mlp_sizes(const bmc_mlp_shape* shape, int64_t batch, int64_t* n_param, int64_t* shadow_bytes,
                         int64_t* work_bytes) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (batch < 1 || batch > (int64_t(1) << 24)) return fail(BMC_ERR_INVALID, "MLP batch %lld", (long long)batch);
    if (n_param) *n_param = n_params(s);
    if (shadow_bytes) *shadow_bytes = shadow_elems(s) * 2;
    if (work_bytes) *work_bytes = int64_t(carve(s, batch, nullptr).bytes);
    return BMC_OK;
}

bmc_status bmc_mlp_sync(const bmc_mlp_shape* shape, const float* d_params, void* d_shadow, void* stream) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (!d_params || !d_shadow) return fail(BMC_ERR_INVALID, "null params or shadow");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = n_params(s);
    sync_kernel<<<unsigned(std::min<long long>((n + 255) / 256, 4096)), 256, 0, st>>>(
        layer_map(s), d_params, n, static_cast<bf16*>(d_shadow));
    MLP_CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_mlp_forward(const bmc_mlp_shape* shape, const float* d_params, const void* d_shadow,
                           const float* d_x, const float* d_in_shift, const float* d_in_scale, int64_t batch,
                           float* d_y, void* d_work, int32_t keep_for_backward, void* stream) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (batch < 1 || batch > (int64_t(1) << 24)) return fail(BMC_ERR_INVALID, "MLP batch %lld", (long long)batch);
    if (!d_params || !d_shadow || !d_x || !d_work) return fail(BMC_ERR_INVALID, "null params, shadow, x or work");
    if ((reinterpret_cast<uintptr_t>(d_work) & 255) || (reinterpret_cast<uintptr_t>(d_shadow) & 15))
        return fail(BMC_ERR_INVALID, "work must be 256-byte and shadow 16-byte aligned");
    const Work w = carve(s, batch, d_work);
    return forward_impl(s, d_params, static_cast<const bf16*>(d_shadow), d_x, d_in_shift, d_in_scale, batch, d_y,
                        w, keep_for_backward != 0, static_cast<cudaStream_t>(stream));
}

bmc_status bmc_mlp_backward(const bmc_mlp_shape* shape, const void* d_shadow, const float* d_target, int64_t batch,
                            void* d_work, float* d_grad, float* d_loss, void* stream) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (batch < 1 || batch > (int64_t(1) << 24)) return fail(BMC_ERR_INVALID, "MLP batch %lld", (long long)batch);
    if (!d_shadow || !d_target || !d_work || !d_grad)
        return fail(BMC_ERR_INVALID, "null shadow, target, work or grad");
    if (reinterpret_cast<uintptr_t>(d_work) & 255) return fail(BMC_ERR_INVALID, "work must be 256-byte aligned");
    const Work w = carve(s, batch, d_work);
    return backward_impl(s, static_cast<const bf16*>(d_shadow), d_target, batch, w, d_grad, d_loss,
                         static_cast<cudaStream_t>(stream));
}

bmc_status bmc_mlp_adam_step(const bmc_mlp_shape* shape, float* d_params, const float* d_grad, float* d_m,
                             float* d_v, void* d_shadow, int32_t step, float lr, float beta1, float beta2, float eps,
                             void* stream) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (!d_params || !d_grad || !d_m || !d_v || !d_shadow) return fail(BMC_ERR_INVALID, "null Adam operand");
    if (step < 1 || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0))
        return fail(BMC_ERR_INVALID, "Adam: step %d, lr %g, beta1 %g, beta2 %g, eps %g", step, lr, beta1, beta2,
                    eps);
    const double lr_t = lr * std::sqrt(1.0 - std::pow(double(beta2), step)) / (1.0 - std::pow(double(beta1), step));
    const long long n = n_params(s);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    adam_kernel<<<unsigned(std::min<long long>((n + 255) / 256, 4096)), 256, 0, st>>>(
        layer_map(s), d_params, d_grad, d_m, d_v, n, float(lr_t), beta1, beta2, eps, static_cast<bf16*>(d_shadow));
    MLP_CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

bmc_status bmc_mlp_adam_step_dev(const bmc_mlp_shape* shape, float* d_params, const float* d_grad, float* d_m,
                                 float* d_v, void* d_shadow, int32_t* d_step, float lr, float beta1, float beta2,
                                 float eps, void* stream) {
    Shape s;
    if (bmc_status e = check_shape(shape, &s)) return e;
    if (!d_params || !d_grad || !d_m || !d_v || !d_shadow || !d_step) return fail(BMC_ERR_INVALID, "null Adam operand");
    if (!(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0))
        return fail(BMC_ERR_INVALID, "Adam: lr %g, beta1 %g, beta2 %g, eps %g", lr, beta1, beta2, eps);
    const long long n = n_params(s);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    adam_dev_kernel<<<unsigned(std::min<long long>((n + 255) / 256, 4096)), 256, 0, st>>>(
        layer_map(s), d_params, d_grad, d_m, d_v, n, d_step, lr, beta1, beta2, eps, static_cast<bf16*>(d_shadow));
    MLP_CUDA_TRY(cudaGetLastError());
    step_advance_kernel<<<1, 1, 0, st>>>(d_step);
    MLP_CUDA_TRY(cudaGetLastError());
    return BMC_OK;
}

}  // extern "C"
