// nn_b200.cu -- training and inference kernels of the warm-start network.
//
// The matrix products run on the 5th-generation tensor cores: one CTA of
// 128 threads computes a 128 x BN tile of A B^T (bf16 operands, fp32
// accumulator in tensor memory).  Operands are staged global -> shared
// memory by all threads in the canonical no-swizzle K-major layout that
// tcgen05.mma reads through shared-memory matrix descriptors, two stages
// deep; one elected thread issues the MMAs and commits them to an mbarrier
// per stage; the epilogue reads the accumulator with tcgen05.ld (each warp
// its 32 lanes) and applies bias and activation.  Every mbarrier wait is
// bounded in time: a wait inside the K loop gives up after the launch's
// limit (wait_ns), after which the CTA records error bit 1, stops issuing,
// waits for its issued MMAs to drain (a fixed, separate bound of 2 s),
// frees its tensor memory and returns.  If the drain bound also runs out,
// the CTA still frees its tensor memory (every allocation must be freed
// before the CTA exits) and records error bit 2: MMAs may then have been
// running when it was freed, and the context should not be trusted.
//
// The rest are small memory-bound kernels (im2col / col2im for the 1D
// convolutions, activation adjoint, transposes, column sums, MSE, Adam).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nn_b200.h"
#include "../../include/swe_b200.h"

namespace nn {
namespace {

constexpr int BM = 128;       // tile rows (UMMA M)
constexpr int BK = 64;        // K elements per stage
constexpr int BN_MAX = 128;   // tile columns (UMMA N), multiple of 16
constexpr int NT = 128;       // threads per CTA
constexpr int A_BYTES = BM * BK * 2;      // 16 KB
constexpr int B_BYTES = BN_MAX * BK * 2;  // 16 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
// Two stages use 64 KB; the allocation is 96 KB so that the operand reads
// of every descriptor stay inside it by a wide margin.
constexpr int SMEM_BYTES = 96 * 1024;
// Bound of the final wait for the CTA's own MMAs before its tensor memory is
// freed (independent of the launch's wait limit, so that a short limit
// never frees tensor memory under MMAs that are still running).
constexpr unsigned long long DRAIN_LIMIT_NS = 2000000000ull;  // 2 s

struct GemmArgs {
    const uint16_t* A;
    const uint16_t* B;
    int M, N, K, lda, ldb, kchunk;  // kchunk: K per blockIdx.z (multiple of BK)
    const float* bias;
    int act, ldc;
    float* out_f32;
    uint16_t* out_bf16;
    float* pre_f32;
    float* partial;  // split K: [z][M][N]
    uint32_t* err;
    unsigned long long wait_ns;  // limit of each wait inside the K loop
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Shared-memory matrix descriptor, no swizzle, K-major: 8-row x 16-byte core
// matrices; lbo = byte distance between the two core matrices along K of
// one MMA, sbo = byte distance between 8-row groups; version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: fp32 accumulator (bits 4-5 = 1),
// A and B bf16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24.
__device__ __forceinline__ uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase `parity` of an mbarrier, giving up once `limit`
// nanoseconds have passed (the time is checked before every probe, so a
// limit of 0 gives up at once).
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit) {
    const unsigned long long t0 = global_ns();
    while (global_ns() - t0 < limit) {
        if (mbar_try(bar, parity)) return true;
    }
    return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float x) {
    return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float x) {
    // d/dx x Phi(x) = Phi(x) + x phi(x)
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

__device__ __forceinline__ void epilogue_store(const GemmArgs& g, int r, int c, float acc) {
    float pre = acc + (g.bias ? g.bias[c] : 0.0f);
    const float y = g.act == NN_ACT_GELU ? gelu(pre) : pre;
    const size_t o = (size_t)r * g.ldc + c;
    if (g.pre_f32) g.pre_f32[o] = pre;
    if (g.out_f32) g.out_f32[o] = y;
    if (g.out_bf16) g.out_bf16[o] = __bfloat16_as_ushort(__float2bfloat16_rn(y));
}

__global__ void __launch_bounds__(NT, 1) gemm_kernel(const GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_ok;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM;
    const int bn = min(BN_MAX, ((g.N + 15) / 16) * 16);
    const int n0 = blockIdx.y * BN_MAX;
    const int kbeg = blockIdx.z * g.kchunk;
    const int kend = min(g.K, kbeg + g.kchunk);
    const int nkb = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;
    uint32_t ncols = 32;
    while ((int)ncols < bn) ncols <<= 1;

    if (warp == 0) {  // tensor memory for the accumulator (one full warp)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&s_tmem)), "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(smem_u32(&s_bar[0]));
        mbar_init(smem_u32(&s_bar[1]));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = instr_desc(bn);
    uint32_t phase[2] = {0u, 0u};
    int issued = 0;  // MMA groups committed

    for (int kb = 0; kb < nkb; ++kb) {
        const int s = kb & 1;
        uint8_t* sA = smem + s * STAGE_BYTES;
        uint8_t* sB = sA + A_BYTES;
        if (kb >= 2) {  // the MMAs that read this stage two blocks ago are done
            if (tid == 0) {
                if (!mbar_wait(smem_u32(&s_bar[s]), phase[s], g.wait_ns)) s_ok = 0;
            }
            phase[s] ^= 1u;
            __syncthreads();
            if (!s_ok) break;
        }
        const int k0 = kbeg + kb * BK;
        // A rows: thread t stages row m0 + t, 8 chunks of 8 K-elements.
        {
            const int r = m0 + tid;
#pragma unroll
            for (int kc = 0; kc < BK / 8; ++kc) {
                const int k = k0 + kc * 8;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (r < g.M && k < kend) v = *reinterpret_cast<const uint4*>(g.A + (size_t)r * g.lda + k);
                *reinterpret_cast<uint4*>(sA + kc * (BM * 16) + tid * 16) = v;
            }
        }
        if (tid < bn) {
            const int r = n0 + tid;
#pragma unroll
            for (int kc = 0; kc < BK / 8; ++kc) {
                const int k = k0 + kc * 8;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (r < g.N && k < kend) v = *reinterpret_cast<const uint4*>(g.B + (size_t)r * g.ldb + k);
                *reinterpret_cast<uint4*>(sB + kc * (bn * 16) + tid * 16) = v;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int t = 0; t < BK / 16; ++t) {
                const uint64_t ad = smem_desc(a0 + t * 2 * (BM * 16), BM * 16, 128);
                const uint64_t bd = smem_desc(b0 + t * 2 * (bn * 16), bn * 16, 128);
                mma_bf16(tmem, ad, bd, idesc, (kb > 0 || t > 0) ? 1u : 0u);
            }
            mma_commit(smem_u32(&s_bar[s]));
        }
        issued = kb + 1;
    }

    // Wait for the last commit (it covers every MMA this thread issued).
    __shared__ int s_drained;
    if (tid == 0) s_drained = 1;
    if (issued > 0) {
        const int s = (issued - 1) & 1;
        if (tid == 0) {
            if (!mbar_wait(smem_u32(&s_bar[s]), phase[s], DRAIN_LIMIT_NS)) s_drained = 0;
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool ok = s_ok != 0 && s_drained != 0;
    if (!ok) {
        if (tid == 0 && g.err) atomicOr(g.err, (s_ok ? 0u : 1u) | (s_drained ? 0u : 2u));
    } else {
        const int r = m0 + warp * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < bn; c0 += 8) {
            float v[8];
            if (issued > 0) {
                tmem_ld8(lane_addr + (uint32_t)c0, v);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = 0.0f;
            }
            if (r < g.M) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int c = n0 + c0 + i;
                    if (c >= g.N) continue;
                    if (g.partial) g.partial[((size_t)blockIdx.z * g.M + r) * g.N + c] = v[i];
                    else epilogue_store(g, r, c, v[i]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// Split-K: sum the partial tiles in z order, then the epilogue.
__global__ void splitk_epilogue_kernel(const GemmArgs g, int ksplit) {
    const long long total = (long long)g.M * g.N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (int z = 0; z < ksplit; ++z) acc += g.partial[(size_t)z * total + i];
        const int r = (int)(i / g.N), c = (int)(i - (long long)r * g.N);
        epilogue_store(g, r, c, acc);
    }
}

__device__ __forceinline__ float bf16_to_f(uint16_t u) { return __uint_as_float((uint32_t)u << 16); }
__device__ __forceinline__ uint16_t f_to_bf16(float f) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

__global__ void im2col_kernel(const float* xf, const uint16_t* xb, int Nb, int Lin, int Cin, int sn,
                              int sl, int sc, int k, int stride, int pad, int Lout, float scale,
                              float shift, uint16_t* cols, int ldcols) {
    const long long total = (long long)Nb * Lout * ldcols;
    const int kc = k * Cin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / ldcols;
        const int col = (int)(i - row * ldcols);
        float v = 0.0f;
        if (col < kc) {
            const int n = (int)(row / Lout), lo = (int)(row - (long long)n * Lout);
            const int kk = col / Cin, ci = col - kk * Cin;
            const int l = lo * stride - pad + kk;
            if (l >= 0 && l < Lin) {
                const size_t o = (size_t)n * sn + (size_t)l * sl + (size_t)ci * sc;
                v = (xf ? xf[o] : bf16_to_f(xb[o])) * scale + shift;
            }
        }
        cols[i] = f_to_bf16(v);
    }
}

__global__ void col2im_kernel(const float* dcols, int ld, int Nb, int Lin, int Cin, int k, int stride,
                              int pad, int Lout, float* dX) {
    const long long total = (long long)Nb * Lin * Cin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % Cin);
        const long long nl = i / Cin;
        const int l = (int)(nl % Lin), n = (int)(nl / Lin);
        float acc = 0.0f;
        // kk = l + pad - lo*stride in [0, k)
        for (int kk = (l + pad) % stride; kk < k; kk += stride) {
            const int lo = (l + pad - kk) / stride;
            if (lo < 0 || lo >= Lout) continue;
            acc += dcols[((size_t)n * Lout + lo) * ld + (size_t)kk * Cin + ci];
        }
        dX[i] = acc;
    }
}

__global__ void act_backward_kernel(const float* dact, const float* pre, int M, int N, int ld_in,
                                    int act, uint16_t* d_bf16, int ldd, uint16_t* dT_bf16, int ldt,
                                    float* d_f32) {
    // 32 x 32 tiles through shared memory so the transposed store is coalesced.
    __shared__ uint16_t tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: column (N), by: row (M)
    const int tx = threadIdx.x, ty = threadIdx.y;           // 32 x 8 threads
    for (int j = ty; j < 32; j += 8) {
        const int r = by + j, c = bx + tx;
        uint16_t b = 0;
        if (r < M && c < N) {
            const size_t o = (size_t)r * ld_in + c;
            float d = dact[o];
            if (act == NN_ACT_GELU) d *= gelu_grad(pre[o]);
            b = f_to_bf16(d);
            if (d_bf16) d_bf16[(size_t)r * ldd + c] = b;
            if (d_f32) d_f32[(size_t)r * ld_in + c] = d;
        }
        tile[j][tx] = b;
    }
    __syncthreads();
    if (!dT_bf16) return;
    for (int j = ty; j < 32; j += 8) {
        const int c = bx + j, r = by + tx;  // write dT[c][r]
        if (c < N && r < ldt) dT_bf16[(size_t)c * ldt + r] = r < M ? tile[tx][j] : (uint16_t)0;
    }
}

__global__ void colsum_kernel(const float* x, int M, int N, int ld, float* out) {
    const int c = blockIdx.x;
    __shared__ float s[256];
    float acc = 0.0f;
    for (int r = threadIdx.x; r < M; r += blockDim.x) acc += x[(size_t)r * ld + c];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = s[0];
}

__global__ void transpose_bf16_kernel(const uint16_t* in, int R, int C, int ldi, uint16_t* out,
                                      int ldo) {
    __shared__ uint16_t tile[32][33];
    const int bc = blockIdx.x * 32, br = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int j = ty; j < 32; j += 8) {
        const int r = br + j, c = bc + tx;
        tile[j][tx] = (r < R && c < C) ? in[(size_t)r * ldi + c] : (uint16_t)0;
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int c = bc + j, r = br + tx;
        if (c < C && r < ldo) out[(size_t)c * ldo + r] = r < R ? tile[tx][j] : (uint16_t)0;
    }
}

__global__ void cast_kernel(const float* in, int R, int C, int ldi, uint16_t* out, int ldo) {
    const long long total = (long long)R * ldo;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / ldo;
        const int c = (int)(i - r * ldo);
        out[i] = c < C ? f_to_bf16(in[(size_t)r * ldi + c]) : (uint16_t)0;
    }
}

__global__ void mse_kernel(const float* pred, const float* target, int M, int N, float* loss,
                           float* grad) {
    __shared__ float s[256];
    const long long total = (long long)M * N;
    const float inv = 1.0f / (float)total;
    float acc = 0.0f;
    for (long long i = threadIdx.x; i < total; i += blockDim.x) {
        const float d = pred[i] - target[i];
        acc += d * d;
        if (grad) grad[i] = 2.0f * d * inv;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) loss[0] = s[0] * inv;
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, long long count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (int)(b > 148LL * 16 ? 148LL * 16 : b);
}

bool g_smem_set[64] = {false};

}  // namespace
}  // namespace nn

using namespace nn;

extern "C" int nn_gemm_bf16(const uint16_t* A, int lda, const uint16_t* B, int ldb, int M, int N,
                            int K, const float* bias, int act, float* out_f32, uint16_t* out_bf16,
                            float* pre_f32, int ldc, int ksplit, float* workspace,
                            long long wait_ns, uint32_t* err, void* stream) {
    if (!A || !B || M < 1 || N < 1 || K < 16 || K % 16 || lda % 8 || ldb % 8 || lda < K || ldb < K)
        return SWE_EARG;
    if (wait_ns < 0) return SWE_EARG;
    if (((uintptr_t)A | (uintptr_t)B) & 15u) return SWE_EARG;
    if (act != NN_ACT_NONE && act != NN_ACT_GELU) return SWE_EARG;
    if (!out_f32 && !out_bf16 && !pre_f32) return SWE_EARG;
    if (ldc < N || ksplit < 1 || ksplit > 1024 || (ksplit > 1 && !workspace)) return SWE_EARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SWE_ECUDA;
    if (!g_smem_set[dev]) {
        if (cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 SMEM_BYTES) != cudaSuccess)
            return SWE_ECUDA;
        g_smem_set[dev] = true;
    }
    GemmArgs g{};
    g.A = A;
    g.B = B;
    g.M = M;
    g.N = N;
    g.K = K;
    g.lda = lda;
    g.ldb = ldb;
    // K per split, a multiple of BK
    const int kblocks = (K + BK - 1) / BK;
    const int per = (kblocks + ksplit - 1) / ksplit;
    g.kchunk = per * BK;
    const int zs = (kblocks + per - 1) / per;
    g.bias = bias;
    g.act = act;
    g.ldc = ldc;
    g.out_f32 = out_f32;
    g.out_bf16 = out_bf16;
    g.pre_f32 = pre_f32;
    g.partial = zs > 1 ? workspace : nullptr;
    g.err = err;
    g.wait_ns = (unsigned long long)wait_ns;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((M + BM - 1) / BM, (N + BN_MAX - 1) / BN_MAX, zs);
    gemm_kernel<<<grid, NT, SMEM_BYTES, s>>>(g);
    if (zs > 1) splitk_epilogue_kernel<<<grid_for((long long)M * N, 256), 256, 0, s>>>(g, zs);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_im2col(const float* x_f32, const uint16_t* x_bf16, int Nb, int Lin, int Cin,
                         int x_stride_n, int x_stride_l, int x_stride_c, int k, int stride, int pad,
                         int Lout, float scale, float shift, uint16_t* cols, int ldcols,
                         void* stream) {
    if ((!x_f32 && !x_bf16) || !cols || Nb < 1 || Lin < 1 || Cin < 1 || k < 1 || stride < 1 ||
        pad < 0 || Lout < 1 || ldcols < k * Cin)
        return SWE_EARG;
    const long long total = (long long)Nb * Lout * ldcols;
    im2col_kernel<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(
        x_f32, x_bf16, Nb, Lin, Cin, x_stride_n, x_stride_l, x_stride_c, k, stride, pad, Lout, scale,
        shift, cols, ldcols);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_col2im(const float* dcols, int lddcols, int Nb, int Lin, int Cin, int k, int stride,
                         int pad, int Lout, float* dX, void* stream) {
    if (!dcols || !dX || Nb < 1 || Lin < 1 || Cin < 1 || k < 1 || stride < 1 || pad < 0 || Lout < 1 ||
        lddcols < k * Cin)
        return SWE_EARG;
    const long long total = (long long)Nb * Lin * Cin;
    col2im_kernel<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(dcols, lddcols, Nb, Lin, Cin,
                                                                        k, stride, pad, Lout, dX);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_act_backward(const float* dact, const float* pre, int M, int N, int ld_in, int act,
                               uint16_t* d_bf16, int ldd, uint16_t* dT_bf16, int ldt, float* d_f32,
                               void* stream) {
    if (!dact || M < 1 || N < 1 || ld_in < N || (act == NN_ACT_GELU && !pre)) return SWE_EARG;
    if (act != NN_ACT_NONE && act != NN_ACT_GELU) return SWE_EARG;
    if ((d_bf16 && ldd < N) || (dT_bf16 && ldt < M)) return SWE_EARG;
    const int Mt = dT_bf16 ? (ldt > M ? ldt : M) : M;  // rows covered (zero tail of dT)
    const dim3 grid((N + 31) / 32, (Mt + 31) / 32);
    act_backward_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(dact, pre, M, N, ld_in, act,
                                                                       d_bf16, ldd, dT_bf16, ldt, d_f32);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_colsum(const float* x, int M, int N, int ld, float* out, void* stream) {
    if (!x || !out || M < 1 || N < 1 || ld < N) return SWE_EARG;
    colsum_kernel<<<N, 256, 0, (cudaStream_t)stream>>>(x, M, N, ld, out);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_transpose_bf16(const uint16_t* in, int R, int C, int ldi, uint16_t* out, int ldo,
                                 void* stream) {
    if (!in || !out || R < 1 || C < 1 || ldi < C || ldo < R) return SWE_EARG;
    const dim3 grid((C + 31) / 32, (ldo + 31) / 32);
    transpose_bf16_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(in, R, C, ldi, out, ldo);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_cast_bf16(const float* in, int R, int C, int ldi, uint16_t* out, int ldo,
                            uint16_t* outT, int ldt, void* stream) {
    if (!in || !out || R < 1 || C < 1 || ldi < C || ldo < C || (outT && ldt < R)) return SWE_EARG;
    cudaStream_t s = (cudaStream_t)stream;
    cast_kernel<<<grid_for((long long)R * ldo, 256), 256, 0, s>>>(in, R, C, ldi, out, ldo);
    if (outT) {
        const dim3 grid((C + 31) / 32, (ldt + 31) / 32);
        transpose_bf16_kernel<<<grid, dim3(32, 8), 0, s>>>(out, R, C, ldo, outT, ldt);
    }
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_mse(const float* pred, const float* target, int M, int N, float* loss, float* grad,
                      void* stream) {
    if (!pred || !target || M < 1 || N < 1) return SWE_EARG;
    mse_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(pred, target, M, N, loss, grad);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}

extern "C" int nn_adam(float* params, const float* grads, float* m, float* v, long long count, float lr,
                       float beta1, float beta2, float eps, int step, void* stream) {
    if (!params || !grads || !m || !v || count < 1 || step < 1) return SWE_EARG;
    const float c1 = 1.0f - powf(beta1, (float)step);
    const float c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<grid_for(count, 256), 256, 0, (cudaStream_t)stream>>>(params, grads, m, v, count, lr,
                                                                        beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}
