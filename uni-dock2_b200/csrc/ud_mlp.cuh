// ud_mlp.cuh -- the learned move proposal: a BF16 MLP (672 -> 256 -> 256 -> 256 -> 64,
// ReLU) with FP32 accumulation on the tensor cores, its training kernels (masked Gaussian
// negative log-likelihood, backward pass, Adam) and the host state that drives them.
//
// No reference counterpart: the network replaces the random draw of mutate_pose_tile
// (src/cuda/mc.cu:146-256) by a sample from N(mean, exp(logvar)) over the 6 + T move
// dimensions; Vina scoring and Metropolis stay the judge.  Rounding points (BF16 inputs,
// weights, hidden activations and back-propagated pre-activation gradients; FP32 sums,
// biases, loss and optimiser) are restated in oracle/mlp_oracle.py.
#pragma once
#include <cuda.h>          // CUtensorMap (the TMA descriptor; encoded on the host at run time)
#include <cuda_bf16.h>
#include <random>

namespace mlp {
constexpr int IN = 672, HID = 256, OUT = 64;
constexpr int NDIM = 26;                      // 6 rigid-body + up to 20 torsion dimensions
constexpr int NATOM = 80, NMAP = 8, TMAX = 20;
constexpr float LV_MIN = -8.f, LV_MAX = 4.f;
constexpr long long OFF_W1 = 0, OFF_B1 = OFF_W1 + (long long)IN * HID, OFF_W2 = OFF_B1 + HID,
                    OFF_B2 = OFF_W2 + (long long)HID * HID, OFF_W3 = OFF_B2 + HID,
                    OFF_B3 = OFF_W3 + (long long)HID * HID, OFF_W4 = OFF_B3 + HID,
                    OFF_B4 = OFF_W4 + (long long)HID * OUT, NPARAM = OFF_B4 + OUT;
}  // namespace mlp

// C[m][n] (+bias[n], ReLU) = sum_k A(m,k) B(k,n), A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn]: the strides express the transposes of the backward pass.
struct GemmArgs {
    const __nv_bfloat16* A;
    long long sam, sak;
    const __nv_bfloat16* B;
    long long sbk, sbn;
    int M, N, K;
    float* C;                 // optional FP32 output, row-major, ldc
    int ldc;
    __nv_bfloat16* C16;       // optional BF16 output, row-major, ldc16
    int ldc16;
    const float* bias;        // optional, per output column
    int relu;
};

constexpr int GBM = 64, GBN = 64, GBK = 32, GPAD = 8;

__device__ __forceinline__ uint32_t ld_b32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// 64x64 output tile per CTA of 4 warps (2x2, 32x32 each = 2x4 m16n8k16 tiles), K in
// steps of 32 staged through shared memory (B transposed to [n][k] so both operands'
// fragments are pairs of consecutive k).  Out-of-range elements load as zero.
__global__ void __launch_bounds__(128) k_gemm_bf16(GemmArgs g) {
    __shared__ __align__(16) __nv_bfloat16 As[GBM][GBK + GPAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[GBN][GBK + GPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = warp >> 1, wn = warp & 1;
    const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
    const int g8 = lane >> 2, t4 = lane & 3;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
    for (int k0 = 0; k0 < g.K; k0 += GBK) {
        for (int e = tid; e < GBM * GBK; e += 128) {
            const int r = e / GBK, k = e % GBK, m = m0 + r, kk = k0 + k;
            As[r][k] = (m < g.M && kk < g.K) ? g.A[(long long)m * g.sam + (long long)kk * g.sak] : zero;
        }
        for (int e = tid; e < GBN * GBK; e += 128) {
            const int c = e / GBK, k = e % GBK, n = n0 + c, kk = k0 + k;
            Bs[c][k] = (n < g.N && kk < g.K) ? g.B[(long long)kk * g.sbk + (long long)n * g.sbn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < GBK; ks += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int mi = 0; mi < 2; mi++) {
                const int r = wm * 32 + mi * 16 + g8;
                a[mi][0] = ld_b32(&As[r][ks + 2 * t4]);
                a[mi][1] = ld_b32(&As[r + 8][ks + 2 * t4]);
                a[mi][2] = ld_b32(&As[r][ks + 8 + 2 * t4]);
                a[mi][3] = ld_b32(&As[r + 8][ks + 8 + 2 * t4]);
            }
#pragma unroll
            for (int ni = 0; ni < 4; ni++) {
                const int c = wn * 32 + ni * 8 + g8;
                b[ni][0] = ld_b32(&Bs[c][ks + 2 * t4]);
                b[ni][1] = ld_b32(&Bs[c][ks + 8 + 2 * t4]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++) {
                    float* d = acc[mi][ni];
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                        : "r"(a[mi][0]), "r"(a[mi][1]), "r"(a[mi][2]), "r"(a[mi][3]), "r"(b[ni][0]),
                          "r"(b[ni][1]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++)
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int m = m0 + wm * 32 + mi * 16 + g8 + 8 * h;
                    const int n = n0 + wn * 32 + ni * 8 + 2 * t4 + j;
                    if (m < g.M && n < g.N) {
                        float v = acc[mi][ni][2 * h + j];
                        if (g.bias) v += g.bias[n];
                        if (g.relu) v = fmaxf(v, 0.f);
                        if (g.C) g.C[(long long)m * g.ldc + n] = v;
                        if (g.C16) g.C16[(long long)m * g.ldc16 + n] = __float2bfloat16_rn(v);
                    }
                }
}

// ---------------------------------------------------------------------- tcgen05 GEMM, TMA-staged
// Y[M x N] = act(X[M x K] W[K x N] + b) on the 5th-generation tensor cores: one CTA of 128
// threads per 128-row tile, the FP32 accumulator (128 lanes x N columns) in tensor memory,
// one thread issuing tcgen05.mma (kind::f16, BF16 operands, M = 128, K = 16 per instruction).
// Operands arrive 32 K-values at a time by TMA (cp.async.bulk.tensor, each CTA its own), double
// buffered: while the tensor cores work on one stage the next stage's tiles are loading.  The
// canonical no-swizzle layouts come straight out of 3-D tensor maps:
//  * X (K-major): dims (8 k, rows, K/8 chunks), strides (ld*2 B, 16 B), box (8, 128, 4): four
//    2 KB chunk blocks of 128 rows x 16 B; core matrices K-adjacent 2048 B apart, M-adjacent
//    128 B apart;
//  * W (N-major): dims (8 n, K rows, N/8 chunks), strides (N*2 B, 16 B), box (8, 32, N/8): N/8
//    blocks of 32 k-rows x 16 B; core matrices K-adjacent 128 B, N-adjacent 512 B apart.
// Rows beyond the map's extent arrive as zeros.  Split-K: grid.y CTAs share a tile's K range
// (kchunk each) and write FP32 partials [split][M][N], summed by k_sum_splits in split order.
// Every wait is bounded: on timeout the kernel records an error, waits (bounded) for its own
// copies and MMAs in flight, and releases its tensor memory.  N is 64 or 256, kchunk a
// multiple of 32.
constexpr int TC_BM = 128, TC_BK = 32;
constexpr long long TC_SPIN = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);        // version 1, no swizzle
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < TC_SPIN; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// one 3-D tile of a tensor map into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

template <int N>
__global__ void __launch_bounds__(128) k_gemm_tc(const __grid_constant__ CUtensorMap tmX,
                                                 const __grid_constant__ CUtensorMap tmW,
                                                 const float* __restrict__ bias, int M, int kchunk, int relu,
                                                 __nv_bfloat16* __restrict__ Y16, float* __restrict__ Y32, int* err) {
    static_assert(N == 64 || N == 256, "N");
    constexpr int A_BYTES = TC_BM * TC_BK * 2;              // 8 KB per stage
    constexpr int B_BYTES = N * TC_BK * 2;                  // 4 or 16 KB per stage
    extern __shared__ __align__(16) unsigned char tc_smem_raw[];
    // operand stages from a 1024-byte boundary (the launch requests 1 KB of slack)
    unsigned char* tc_smem = tc_smem_raw + ((1024u - (smem_u32(tc_smem_raw) & 1023u)) & 1023u);
    unsigned char* sA[2] = {tc_smem, tc_smem + A_BYTES};
    unsigned char* sB[2] = {tc_smem + 2 * A_BYTES, tc_smem + 2 * A_BYTES + B_BYTES};
    __shared__ __align__(8) uint64_t mma_bar[2], tma_bar[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail, s_issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM;
    const int kbase = blockIdx.y * kchunk;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&s_tmem)), "r"(N) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < 2; i++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mma_bar[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&tma_bar[i])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
        s_issued = -1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    // instruction descriptor: F32 accumulate, BF16 A and B, A K-major, B N-major, N, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(N >> 3) << 17) |
                           ((uint32_t)(TC_BM >> 4) << 24);
    const int nstage = kchunk / TC_BK;
    if (tid == 0) {
        int loaded = 0, consumed = 0, issued = -1;
        bool fail = false;
        auto load = [&](int s) {
            const int b = s & 1;
            const int k0 = kbase + s * TC_BK;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         :: "r"(smem_u32(&tma_bar[b])), "r"((uint32_t)(A_BYTES + B_BYTES)) : "memory");
            tma_load_3d(sA[b], &tmX, 0, m0, k0 >> 3, smem_u32(&tma_bar[b]));
            tma_load_3d(sB[b], &tmW, 0, k0, 0, smem_u32(&tma_bar[b]));
        };
        if (nstage > 0) { load(0); loaded = 1; }
        for (int s = 0; s < nstage && !fail; s++) {
            const int b = s & 1;
            if (s + 1 < nstage) {
                // the other buffer held stage s - 1: its MMAs finish before it is refilled
                if (s >= 1 && !mbar_wait(smem_u32(&mma_bar[(s - 1) & 1]), (uint32_t)(((s - 1) >> 1) & 1))) {
                    fail = true;
                    break;
                }
                load(s + 1);
                loaded = s + 2;
            }
            if (!mbar_wait(smem_u32(&tma_bar[b]), (uint32_t)((s >> 1) & 1))) {
                fail = true;
                break;
            }
            consumed = s + 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int step = 0; step < TC_BK / 16; step++) {
                const uint64_t da = umma_desc(smem_u32(sA[b] + step * 2 * 2048), 2048, 128);
                const uint64_t db = umma_desc(smem_u32(sB[b] + step * 256), 128, 512);
                const uint32_t acc = (s > 0 || step > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(&mma_bar[b])) : "memory");
            issued = s;
        }
        if (fail) {
            // copies still in flight land before the buffers are released (bounded)
            for (int t = consumed; t < loaded; t++) mbar_wait(smem_u32(&tma_bar[t & 1]), (uint32_t)((t >> 1) & 1));
            s_fail = 1;
        }
        s_issued = issued;
    }
    __syncthreads();
    // all MMAs done when the barrier phase of the last committed stage completes (a commit
    // tracks every MMA issued before it); also after a timeout, so that tensor memory is not
    // released under MMAs still in flight; if this bounded wait times out as well, what the
    // tensor cores still do with the released columns is undefined
    const int issued = s_issued;
    if (issued >= 0 && !mbar_wait(smem_u32(&mma_bar[issued & 1]), (uint32_t)((issued >> 1) & 1))) {
        if (tid == 0) s_fail = 1;
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!s_fail && issued == nstage - 1) {
        const int m = m0 + warp * 32 + lane;                   // this thread's row (TMEM lane)
        float* Yp = Y32 ? Y32 + (size_t)blockIdx.y * M * N : nullptr;
        for (int c = 0; c < N; c += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < M) {
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    v[j] = __uint_as_float(r[j]) + (bias ? bias[c + j] : 0.f);
                    if (relu) v[j] = fmaxf(v[j], 0.f);
                }
                if (Yp) {
#pragma unroll
                    for (int j = 0; j < 8; j++) Yp[(long long)m * N + c + j] = v[j];
                }
                if (Y16) {
                    __nv_bfloat162 h[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    *reinterpret_cast<uint4*>(Y16 + (long long)m * N + c) = *reinterpret_cast<uint4*>(h);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(N) : "memory");
}

// Y[i] = sum over splits s of P[s][i], in split order
__global__ void k_sum_splits(long long n, int splits, const float* __restrict__ P, float* __restrict__ Y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float v = 0.f;
        for (int s = 0; s < splits; s++) v += P[(long long)s * n + i];
        Y[i] = v;
    }
}

// out[c * ldo + r] = in[r * C + c] for r < R, c < C, and 0 for R <= r < ldo: a BF16 transpose
// through 32 x 32 shared-memory tiles (block 32 x 8), zero-padding the new rows' tails so they can
// serve as the K-extended operand of a tensor-core GEMM
__global__ void __launch_bounds__(256) k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C,
                                                        __nv_bfloat16* __restrict__ out, int ldo) {
    __shared__ __nv_bfloat16 tile[32][34];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        tile[i][threadIdx.x] = (r < R && c < C) ? in[(long long)r * C + c] : zero;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < C && r < ldo) out[(long long)c * ldo + r] = tile[threadIdx.x][i];
    }
}

__global__ void k_f32_to_bf16(long long n, const float* __restrict__ s, __nv_bfloat16* __restrict__ d) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        d[i] = __float2bfloat16_rn(s[i]);
}

// masked Gaussian NLL over the n x 64 outputs: dout and the summed loss (mean over rows)
__global__ void k_mlp_nll(int n, const float* __restrict__ out, const float* __restrict__ Y,
                          const float* __restrict__ M, float* __restrict__ dout, double* loss) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < (long long)n * mlp::OUT) {
        const int row = (int)(i / mlp::OUT), col = (int)(i % mlp::OUT);
        const float inv_n = 1.f / (float)n;
        float d = 0.f;
        if (col < 2 * mlp::NDIM) {
            const int j = col < mlp::NDIM ? col : col - mlp::NDIM;
            const float mean = out[(long long)row * mlp::OUT + j];
            const float raw = out[(long long)row * mlp::OUT + mlp::NDIM + j];
            const float lv = fminf(fmaxf(raw, mlp::LV_MIN), mlp::LV_MAX);
            const float r = Y[(long long)row * mlp::NDIM + j] - mean;
            const float iv = expf(-lv);
            const float mk = M[(long long)row * mlp::NDIM + j];
            if (col < mlp::NDIM) {
                d = -mk * r * iv * inv_n;
                l = mk * 0.5f * (lv + r * r * iv) * inv_n;
            } else {
                const bool inside = raw >= mlp::LV_MIN && raw <= mlp::LV_MAX;
                d = inside ? mk * 0.5f * (1.f - r * r * iv) * inv_n : 0.f;
            }
        }
        dout[i] = d;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, (double)l);
}

// dpre = dh * (h > 0), in FP32 and BF16
__global__ void k_relu_bwd(long long n, const float* __restrict__ dh, const __nv_bfloat16* __restrict__ h,
                           float* __restrict__ dpre, __nv_bfloat16* __restrict__ dpre16) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = __bfloat162float(h[i]) > 0.f ? dh[i] : 0.f;
        dpre[i] = v;
        dpre16[i] = __float2bfloat16_rn(v);
    }
}

// column sums of a rows x cols FP32 matrix
__global__ void k_colsum(int rows, int cols, const float* __restrict__ s, float* __restrict__ d) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.f;
    for (int r = 0; r < rows; r++) acc += s[(long long)r * cols + c];
    d[c] = acc;
}

// Adam on the FP32 master parameters; refreshes their BF16 copy
__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ p16, float lr, float c1, float c2) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        p16[i] = __float2bfloat16_rn(pi);
    }
}

// gather rows of a training set into a batch
__global__ void k_gather_rows(int nb, const int* __restrict__ idx, int width, const __nv_bfloat16* __restrict__ src,
                              __nv_bfloat16* __restrict__ dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)nb * width) return;
    const int r = (int)(i / width), c = (int)(i % width);
    dst[i] = src[(long long)idx[r] * width + c];
}
__global__ void k_gather_rows_f32(int nb, const int* __restrict__ idx, int width, const float* __restrict__ src,
                                  float* __restrict__ dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)nb * width) return;
    const int r = (int)(i / width), c = (int)(i % width);
    dst[i] = src[(long long)idx[r] * width + c];
}

