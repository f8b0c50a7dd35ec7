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

