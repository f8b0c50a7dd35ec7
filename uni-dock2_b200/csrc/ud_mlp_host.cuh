// ud_mlp_host.cuh -- host state of the learned move proposal: device buffers of the
// network (FP32 master weights, BF16 copy, Adam moments, activations) and the launch
// sequences of its forward pass, backward pass and Adam step (kernels in ud_mlp.cuh).
// Included by ud_engine.cu after its device-buffer helpers.
#pragma once
#include <cudaTypedefs.h>
#include <random>

struct MlpState {
    bool ready = false;
    int adam_t = 0;
    int cap = 0;
    bool use_tc = true;                     // forward and backward GEMMs on tcgen05 (else mma.sync)
    bool tc_attr = false;
    DBuf<int> tc_err;                       // set by a tcgen05 GEMM whose wait timed out
    DBuf<float> p, g, m, v;                 // NPARAM each
    DBuf<__nv_bfloat16> p16;
    DBuf<__nv_bfloat16> x16, h16[3], d16;   // activations of up to cap rows (d16: cap rounded up to 32)
    DBuf<__nv_bfloat16> xt16, wt16;         // tcgen05 backward: an activation transposed, a weight transposed
    DBuf<float> out, dout, dh, dpre;
    DBuf<double> loss;

    static int blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 4096); }
    static int pad32(int n) { return (n + 31) & ~31; }

    void ensure(int n) {
        if (n <= cap) return;
        x16.ensure((size_t)n * mlp::IN);
        for (auto& h : h16) h.ensure((size_t)n * mlp::HID);
        d16.ensure((size_t)pad32(n) * mlp::HID);
        xt16.ensure((size_t)mlp::IN * pad32(n));
        wt16.ensure((size_t)mlp::HID * mlp::HID);
        out.ensure((size_t)n * mlp::OUT);
        dout.ensure((size_t)n * mlp::OUT);
        dh.ensure((size_t)n * mlp::HID);
        dpre.ensure((size_t)n * mlp::HID);
        cap = n;
    }

    void init(uint64_t seed, cudaStream_t s) {
        std::vector<float> h((size_t)mlp::NPARAM, 0.f);
        std::mt19937_64 rng(seed);
        auto fill = [&](long long off, int fan_in, long long count) {
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (float)fan_in));
            for (long long i = 0; i < count; i++) h[(size_t)(off + i)] = nd(rng);
        };
        fill(mlp::OFF_W1, mlp::IN, (long long)mlp::IN * mlp::HID);
        fill(mlp::OFF_W2, mlp::HID, (long long)mlp::HID * mlp::HID);
        fill(mlp::OFF_W3, mlp::HID, (long long)mlp::HID * mlp::HID);
        fill(mlp::OFF_W4, mlp::HID, (long long)mlp::HID * mlp::OUT);
        for (long long i = 0; i < (long long)mlp::HID * mlp::OUT; i++) h[(size_t)(mlp::OFF_W4 + i)] *= 0.1f;
        set(h.data(), s);
    }

    void set(const float* host, cudaStream_t s) {
        p.upload(host, (size_t)mlp::NPARAM, s);
        g.ensure((size_t)mlp::NPARAM);
        m.ensure((size_t)mlp::NPARAM);
        v.ensure((size_t)mlp::NPARAM);
        p16.ensure((size_t)mlp::NPARAM);
        ck(cudaMemsetAsync(m.p, 0, sizeof(float) * mlp::NPARAM, s), "memset");
        ck(cudaMemsetAsync(v.p, 0, sizeof(float) * mlp::NPARAM, s), "memset");
        k_f32_to_bf16<<<blocks(mlp::NPARAM), 256, 0, s>>>(mlp::NPARAM, p.p, p16.p);
        ck(cudaGetLastError(), "k_f32_to_bf16");
        adam_t = 0;
        ready = true;
    }

    void gemm(cudaStream_t s, const __nv_bfloat16* A, long long sam, long long sak, const __nv_bfloat16* B,
              long long sbk, long long sbn, int M, int N, int K, float* C, int ldc, __nv_bfloat16* C16, int ldc16,
              const float* bias, int relu) {
        GemmArgs a{A, sam, sak, B, sbk, sbn, M, N, K, C, ldc, C16, ldc16, bias, relu};
        dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM);
        k_gemm_bf16<<<grid, 128, 0, s>>>(a);
        ck(cudaGetLastError(), "k_gemm_bf16");
    }

    static constexpr int TC_SMEM = 96 * 1024;   // more than the 48 KB of stages: at most 2 CTAs
                                                // per SM, so 2 x 256 tensor-memory columns fit
    DBuf<float> part;                            // split-K partial sums of the weight gradients

    // the driver's tensor-map encoder, looked up once through the runtime
    static PFN_cuTensorMapEncodeTiled_v12000 encoder() {
        static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
        if (!fn) {
            void* f = nullptr;
            cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
            ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q), "cudaGetDriverEntryPoint");
            if (q != cudaDriverEntryPointSuccess || !f) throw Fail(UD_ECUDA, "cuTensorMapEncodeTiled is not available");
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        }
        return fn;
    }
    static CUtensorMap encode(const __nv_bfloat16* base, const cuuint64_t dim[3], const cuuint64_t str[2],
                              const cuuint32_t box[3], const char* what) {
        CUtensorMap m;
        const cuuint32_t es[3] = {1, 1, 1};
        const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(base), dim, str,
                                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw Fail(UD_ECUDA, std::string("cuTensorMapEncodeTiled failed for ") + what);
        return m;
    }
    // X operand: rows x K (K a multiple of 8) BF16 values, row stride ld; K-major 128-row boxes
    static CUtensorMap map_x(const __nv_bfloat16* base, int rows, int K, int ld) {
        const cuuint64_t dim[3] = {8, (cuuint64_t)rows, (cuuint64_t)(K / 8)};
        const cuuint64_t str[2] = {(cuuint64_t)ld * 2, 16};
        const cuuint32_t box[3] = {8, (cuuint32_t)TC_BM, TC_BK / 8};
        return encode(base, dim, str, box, "a K-major operand");
    }
    // W operand: K rows x N values (row-major); N-major boxes of 32 rows
    static CUtensorMap map_w(const __nv_bfloat16* base, int K, int N) {
        const cuuint64_t dim[3] = {8, (cuuint64_t)K, (cuuint64_t)(N / 8)};
        const cuuint64_t str[2] = {(cuuint64_t)N * 2, 16};
        const cuuint32_t box[3] = {8, (cuuint32_t)TC_BK, (cuuint32_t)(N / 8)};
        return encode(base, dim, str, box, "an N-major operand");
    }

    // one tcgen05 GEMM: Y = act(X W + b); X rows x K with row stride ldx, W K x N; `splits` CTAs
    // per row tile share the K range (FP32 partials summed in split order into Y32)
    void tc_run(cudaStream_t s, const __nv_bfloat16* X, int M, int K, int ldx, const __nv_bfloat16* W, int N,
                const float* bias, int relu, __nv_bfloat16* Y16, float* Y32, int splits) {
        if (K % 8 || ldx % 8 || (N != 64 && N != 256)) throw Fail(UD_EINVAL, "tensor-core GEMM shape");
        const int kchunk = ((K + splits - 1) / splits + TC_BK - 1) / TC_BK * TC_BK;
        const CUtensorMap mx = map_x(X, M, K, ldx), mw = map_w(W, K, N);
        const dim3 grid((unsigned)((M + TC_BM - 1) / TC_BM), (unsigned)splits);
        float* y = Y32;
        if (splits > 1) {
            part.ensure((size_t)splits * M * N);
            y = part.p;
        }
        if (N == 256)
            k_gemm_tc<256><<<grid, 128, TC_SMEM, s>>>(mx, mw, bias, M, kchunk, relu, Y16, y, tc_err.p);
        else
            k_gemm_tc<64><<<grid, 128, TC_SMEM, s>>>(mx, mw, bias, M, kchunk, relu, Y16, y, tc_err.p);
        ck(cudaGetLastError(), "k_gemm_tc");
        if (splits > 1) {
            const long long nmn = (long long)M * N;
            k_sum_splits<<<blocks(nmn), 256, 0, s>>>(nmn, splits, part.p, Y32);
            ck(cudaGetLastError(), "k_sum_splits");
        }
    }

    void tc_layer(cudaStream_t s, int n, const __nv_bfloat16* x, int K, long long off_w, long long off_b, int N,
                  int relu, __nv_bfloat16* y16, float* y32) {
        tc_run(s, x, n, K, K, p16.p + off_w, N, p.p + off_b, relu, y16, y32, 1);
    }

    // errors recorded by the tensor-core GEMM since the last check (call after a sync)
    void check_tc(cudaStream_t s) {
        if (!tc_err.p) return;
        int e = 0;
        ck(cudaMemcpyAsync(&e, tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "tensor-core GEMM check");
        if (e) {
            ck(cudaMemsetAsync(tc_err.p, 0, sizeof(int), s), "memset");
            throw Fail(UD_ECUDA, "tensor-core GEMM: a wait for its MMAs timed out");
        }
    }

    // one-time setup of the tcgen05 path (kernel attributes, error flag); also called before
    // a CUDA graph capture of the forward pass, which must not allocate
    void prepare(cudaStream_t s) {
        if (!use_tc || tc_attr) return;
        ck(cudaFuncSetAttribute(k_gemm_tc<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM), "attr");
        ck(cudaFuncSetAttribute(k_gemm_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM), "attr");
        encoder();                                  // the encoder lookup, before any capture
        tc_err.ensure(1);
        ck(cudaMemsetAsync(tc_err.p, 0, sizeof(int), s), "memset");
        tc_attr = true;
    }

    // out[n x 64] (FP32) from x16[n x 672]
    void forward(cudaStream_t s, int n, const __nv_bfloat16* x) {
        if (use_tc) {
            prepare(s);
            tc_layer(s, n, x, mlp::IN, mlp::OFF_W1, mlp::OFF_B1, mlp::HID, 1, h16[0].p, nullptr);
            tc_layer(s, n, h16[0].p, mlp::HID, mlp::OFF_W2, mlp::OFF_B2, mlp::HID, 1, h16[1].p, nullptr);
            tc_layer(s, n, h16[1].p, mlp::HID, mlp::OFF_W3, mlp::OFF_B3, mlp::HID, 1, h16[2].p, nullptr);
            tc_layer(s, n, h16[2].p, mlp::HID, mlp::OFF_W4, mlp::OFF_B4, mlp::OUT, 0, nullptr, out.p);
            return;
        }
        const __nv_bfloat16* w = p16.p;
        gemm(s, x, mlp::IN, 1, w + mlp::OFF_W1, mlp::HID, 1, n, mlp::HID, mlp::IN, nullptr, 0, h16[0].p, mlp::HID,
             p.p + mlp::OFF_B1, 1);
        gemm(s, h16[0].p, mlp::HID, 1, w + mlp::OFF_W2, mlp::HID, 1, n, mlp::HID, mlp::HID, nullptr, 0, h16[1].p,
             mlp::HID, p.p + mlp::OFF_B2, 1);
        gemm(s, h16[1].p, mlp::HID, 1, w + mlp::OFF_W3, mlp::HID, 1, n, mlp::HID, mlp::HID, nullptr, 0, h16[2].p,
             mlp::HID, p.p + mlp::OFF_B3, 1);
        gemm(s, h16[2].p, mlp::HID, 1, w + mlp::OFF_W4, mlp::OUT, 1, n, mlp::OUT, mlp::HID, out.p, mlp::OUT, nullptr,
             0, p.p + mlp::OFF_B4, 0);
    }

    // in [R x C] (BF16, row-major) -> out [C x ldo], rows zero-padded from R to ldo
    static void transpose(cudaStream_t s, const __nv_bfloat16* in, int R, int C, __nv_bfloat16* out, int ldo) {
        dim3 grid((unsigned)((C + 31) / 32), (unsigned)((ldo + 31) / 32));
        k_transpose_bf16<<<grid, dim3(32, 8), 0, s>>>(in, R, C, out, ldo);
        ck(cudaGetLastError(), "k_transpose_bf16");
    }

    // Y[M x N] (FP32) = X[M x K] W[K x N] on the tensor cores, no bias or activation; a long
    // contraction (the batch, for weight gradients) is split over CTAs to fill the GPU
    void tc_gemm(cudaStream_t s, const __nv_bfloat16* X, int M, int K, int ldx, const __nv_bfloat16* W, int N,
                 float* Y) {
        const int tiles = (M + TC_BM - 1) / TC_BM;
        int splits = 1;
        if (K >= 128) splits = std::max(1, std::min(K / 64, 296 / tiles));
        tc_run(s, X, M, K, ldx, W, N, nullptr, 0, nullptr, Y, splits);
    }

    // The backward products on tcgen05.  Weight gradients dW = h_in^T d contract over the batch:
    // h_in is transposed into [K_in x n32] (n32 = n rounded up to 32, zero tail) and d16 holds
    // n32 rows with a zero tail; the contraction is split over CTAs (tc_gemm).  Input gradients
    // dh = d W^T take W transposed into [N_out x K_in].
    void backward_tc(cudaStream_t s, int n, const __nv_bfloat16* x) {
        prepare(s);
        const int n32 = pad32(n);
        const __nv_bfloat16* w = p16.p;
        // d16 rows n..n32 (in both the 64- and the 256-wide views) stay zero
        if (n32 > n)
            ck(cudaMemsetAsync(d16.p + (size_t)n * mlp::OUT, 0, ((size_t)n32 * mlp::HID - (size_t)n * mlp::OUT) * 2, s),
               "memset");
        const long long no = (long long)n * mlp::OUT;
        k_f32_to_bf16<<<blocks(no), 256, 0, s>>>(no, dout.p, d16.p);
        // output layer: dW4 = h3^T d [256 x 64], db4 = colsum(d), dh3 = d W4^T [n x 256]
        transpose(s, h16[2].p, n, mlp::HID, xt16.p, n32);
        tc_gemm(s, xt16.p, mlp::HID, n32, n32, d16.p, mlp::OUT, g.p + mlp::OFF_W4);
        k_colsum<<<1, 64, 0, s>>>(n, mlp::OUT, dout.p, g.p + mlp::OFF_B4);
        transpose(s, w + mlp::OFF_W4, mlp::HID, mlp::OUT, wt16.p, mlp::HID);
        tc_gemm(s, d16.p, n, mlp::OUT, mlp::OUT, wt16.p, mlp::HID, dh.p);
        const long long off_w[3] = {mlp::OFF_W1, mlp::OFF_W2, mlp::OFF_W3};
        const long long off_b[3] = {mlp::OFF_B1, mlp::OFF_B2, mlp::OFF_B3};
        const long long nh = (long long)n * mlp::HID;
        for (int l = 2; l >= 0; l--) {
            k_relu_bwd<<<blocks(nh), 256, 0, s>>>(nh, dh.p, h16[l].p, dpre.p, d16.p);
            ck(cudaGetLastError(), "k_relu_bwd");
            const __nv_bfloat16* hin = l ? h16[l - 1].p : x;
            const int kin = l ? mlp::HID : mlp::IN;
            transpose(s, hin, n, kin, xt16.p, n32);
            tc_gemm(s, xt16.p, kin, n32, n32, d16.p, mlp::HID, g.p + off_w[l]);
            k_colsum<<<1, 256, 0, s>>>(n, mlp::HID, dpre.p, g.p + off_b[l]);
            if (l > 0) {
                transpose(s, w + off_w[l], mlp::HID, mlp::HID, wt16.p, mlp::HID);
                tc_gemm(s, d16.p, n, mlp::HID, mlp::HID, wt16.p, mlp::HID, dh.p);
            }
        }
        ck(cudaGetLastError(), "mlp backward");
    }

    // gradients of the mean NLL into g (after forward on x); the batch's mean loss is
    // added to loss.p[0] (cleared first when reset)
    void loss_backward(cudaStream_t s, int n, const __nv_bfloat16* x, const float* Y, const float* M, bool reset) {
        loss.ensure(1);
        if (reset) ck(cudaMemsetAsync(loss.p, 0, sizeof(double), s), "memset");
        const long long no = (long long)n * mlp::OUT;
        k_mlp_nll<<<(int)((no + 255) / 256), 256, 0, s>>>(n, out.p, Y, M, dout.p, loss.p);
        ck(cudaGetLastError(), "k_mlp_nll");
        if (use_tc) {
            backward_tc(s, n, x);
            return;
        }
        const __nv_bfloat16* w = p16.p;
        // output layer: dW4 = h3^T d, db4 = colsum(d), dh3 = d W4^T
        k_f32_to_bf16<<<blocks(no), 256, 0, s>>>(no, dout.p, d16.p);
        gemm(s, h16[2].p, 1, mlp::HID, d16.p, mlp::OUT, 1, mlp::HID, mlp::OUT, n, g.p + mlp::OFF_W4, mlp::OUT,
             nullptr, 0, nullptr, 0);
        k_colsum<<<1, 64, 0, s>>>(n, mlp::OUT, dout.p, g.p + mlp::OFF_B4);
        gemm(s, d16.p, mlp::OUT, 1, w + mlp::OFF_W4, 1, mlp::OUT, n, mlp::HID, mlp::OUT, dh.p, mlp::HID, nullptr, 0,
             nullptr, 0);
        const long long off_w[3] = {mlp::OFF_W1, mlp::OFF_W2, mlp::OFF_W3};
        const long long off_b[3] = {mlp::OFF_B1, mlp::OFF_B2, mlp::OFF_B3};
        const long long nh = (long long)n * mlp::HID;
        for (int l = 2; l >= 0; l--) {
            k_relu_bwd<<<blocks(nh), 256, 0, s>>>(nh, dh.p, h16[l].p, dpre.p, d16.p);
            ck(cudaGetLastError(), "k_relu_bwd");
            const __nv_bfloat16* hin = l ? h16[l - 1].p : x;
            const int kin = l ? mlp::HID : mlp::IN;
            gemm(s, hin, 1, kin, d16.p, mlp::HID, 1, kin, mlp::HID, n, g.p + off_w[l], mlp::HID, nullptr, 0, nullptr,
                 0);
            k_colsum<<<1, 256, 0, s>>>(n, mlp::HID, dpre.p, g.p + off_b[l]);
            if (l > 0)
                gemm(s, d16.p, mlp::HID, 1, w + off_w[l], 1, mlp::HID, n, mlp::HID, mlp::HID, dh.p, mlp::HID, nullptr,
                     0, nullptr, 0);
        }
        ck(cudaGetLastError(), "mlp backward");
    }

    void adam(cudaStream_t s, float lr) {
        adam_t++;
        const float c1 = 1.f - std::pow(0.9f, (float)adam_t), c2 = 1.f - std::pow(0.999f, (float)adam_t);
        k_adam<<<blocks(mlp::NPARAM), 256, 0, s>>>(mlp::NPARAM, p.p, g.p, m.p, v.p, p16.p, lr, c1, c2);
        ck(cudaGetLastError(), "k_adam");
    }
};
