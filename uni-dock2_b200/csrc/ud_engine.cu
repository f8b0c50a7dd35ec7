// ud_engine.cu -- kernels and C ABI of the B200 docking engine (libudock_b200.so).
//
// Kernels (all sm_100a, one warp per pose unless noted):
//   k_grid_build   thread per grid point: per-type Vina maps (new; no reference counterpart)
//   k_score        E + generalised gradient of a pose batch   (src/cuda/bfgs_wrapper.cu:51-98)
//   k_terms        final score terms, no curl                 (src/score/score.cpp:12-147)
//   k_bfgs         BFGS / refinement rounds on pose records   (src/cuda/optimize.cu:14-77)
//   k_search       persistent MC search: warp per chain; CTAs take (ligand, chain block)
//                  work items in cost order from a global counter (src/cuda/mc.cu:109-448)
//   k_cluster      CTA per ligand: energy ranking + greedy RMSD leaders (src/cuda/cluster.cu)
//   k_filter       CTA per ligand: energy_range / num_pose filter (src/task/DockTask.cpp:188-220)
//   k_gather       output records of the selected poses
//   k_learn_step   a block of K MC steps of every chain per launch (the learned-proposal
//                  search; the step function is k_search's), with k_learn_features (network input per
//                  chain), k_step_advance, and k_lig_best / k_label_moves (move recording)
//   k_pose_offsets prefix sums for ud_score_batch_noalloc
// Network kernels (tcgen05 forward GEMM, mma.sync GEMM, loss, backward, Adam): ud_mlp.cuh.
// Host orchestration replaces DockTask::run (src/task/DockTask.cpp:39-123).
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <stdexcept>
#include <mutex>
#include <random>
#include <cuda_bf16.h>
#include "ud_device.cuh"
#include "ud_mlp.cuh"
#include "../../include/udock_b200.h"

using namespace ud;

// XS-type vdW radii on the host (src/constants/constants.h:21-43)
static const float kVdwHost[NT] = {1.1f, 1.92f, 1.9f, 1.9f, 1.8f, 1.8f, 1.8f, 1.8f, 1.7f, 1.7f, 1.7f,
                                   1.7f, 1.5f, 2.2f, 2.1f, 2.0f, 1.8f, 2.0f, 2.2f, 2.3f, 1.2f};

// ====================================================================== layout helpers
__host__ __device__ inline int r4(int x) { return (x + 3) & ~3; }
__host__ __device__ inline int rec_floats(int n, int t) { return r4(8 + 3 * n + t); }
// pair buffer floats of a ligand: used on the pair-list path while the list fits PB_MAX
#ifndef PB_MAX_FLOATS
#define PB_MAX_FLOATS 4096
#endif
constexpr int PB_MAX = PB_MAX_FLOATS;
__host__ __device__ inline int pb_floats(int npair) {
    return npair <= PB_MAX ? r4(npair) : 0;
}
__host__ __device__ inline int ws_floats(int n, int t, int npair) {
    int d = 6 + t;
    return 4 * rec_floats(n, t) + r4(3 * n) + 5 * r4(d) + r4(2 * t) + r4(d * (d + 1)) + pb_floats(npair);
}

struct LigDev {
    int blob_off;
    int blob_words;
    int natom, ntors, nheavy;
    int stride;          // record floats
    int lig_uid;
    int stage_words;     // blob prefix the search stages into shared memory
    long long best_off;  // float offset of chain 0's record in the chain-pose buffer
    long long out_off;   // float offset of the output records (num_pose capacity)
};

__device__ __forceinline__ Work work_at(float* ws, const Topo& T) {
    const int natom = T.natom, ntors = T.ntors, d = 6 + ntors;
    Work W;
    W.F = ws + 4 * rec_floats(natom, ntors);
    W.g = W.F + r4(3 * natom);
    W.gn = W.g + r4(d);
    W.p = W.gn + r4(d);
    W.y = W.p + r4(d);
    W.mhy = W.y + r4(d);
    W.sc = W.mhy + r4(d);
    W.H = reinterpret_cast<double*>(W.sc + r4(2 * ntors));
    W.pb = pb_floats(T.nprec) ? reinterpret_cast<float*>(W.H) + r4(d * (d + 1)) : nullptr;
    return W;
}

__device__ __forceinline__ void copy_words(float* dst, const float* src, int n) {
    for (int i = lane_id(); i < n; i += WARP) dst[i] = src[i];
    __syncwarp();
}

// initial pose from the blob: input coordinates, dihedrals, centre = mean, rot_vec = 0,
// energy 999 (src/cuda/task.cu:87-105)
__device__ void load_initial(const int* blob, Slot P, int natom, int ntors) {
    const float* x0 = reinterpret_cast<const float*>(blob + blob[H_X0]);
    const float* d0 = reinterpret_cast<const float*>(blob + blob[H_D0]);
    const float* c0 = reinterpret_cast<const float*>(blob + blob[H_C0]);
    int lane = lane_id();
    if (lane == 0) {
        P.h[0] = 999.f;
        P.h[1] = c0[0]; P.h[2] = c0[1]; P.h[3] = c0[2];
        P.h[4] = P.h[5] = P.h[6] = P.h[7] = 0.f;
    }
    for (int i = lane; i < 3 * natom; i += WARP) P.x[i] = x0[i];
    for (int i = lane; i < ntors; i += WARP) P.d[i] = d0[i];
    __syncwarp();
}

// ====================================================================== grid build
__device__ __forceinline__ float eval_e(float d, int t1, int t2) {
    float f;
    return eval_ef(d, t1, t2, f);
}

constexpr int MAX_MAPS = 20;   // every non-hydrogen XS type
struct MapTypes { int n; int t[MAX_MAPS]; };

__global__ void __launch_bounds__(256) k_grid_build(const float4* __restrict__ rec, int nrec, MapTypes mt,
                                                    float ox, float oy, float oz, float s, int gx, int gy, int gz,
                                                    float* __restrict__ out32, __half* __restrict__ out16) {
    __shared__ float4 tile[256];
    long long npt = (long long)gx * gy * gz;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int ix = (int)(idx % gx), iy = (int)((idx / gx) % gy), iz = (int)(idx / ((long long)gx * gy));
    // grid point in float via one rounded fma; the cutoff test below is done in FP64
    // from the float inputs, so it is bit-identical to the oracle's
    float px = __fmaf_rn((float)ix, s, ox), py = __fmaf_rn((float)iy, s, oy), pz = __fmaf_rn((float)iz, s, oz);
    float acc[MAX_MAPS];
    float rm[MAX_MAPS];
#pragma unroll
    for (int m = 0; m < MAX_MAPS; m++) { acc[m] = 0.f; rm[m] = m < mt.n ? vdw(mt.t[m]) : 0.f; }
    for (int base = 0; base < nrec; base += 256) {
        int j = base + threadIdx.x;
        if (j < nrec) tile[threadIdx.x] = rec[j];
        __syncthreads();
        int nt = min(256, nrec - base);
        if (idx < npt) {
            for (int k = 0; k < nt; k++) {
                float4 r = tile[k];
                double rr = cutoff_r2(r.x, r.y, r.z, px, py, pz);
                if (rr < 64.0) {
                    float rn = sqrtf((float)rr);
                    int tj = (int)r.w;
                    float rj = vdw(tj);
#pragma unroll
                    for (int m = 0; m < MAX_MAPS; m++)
                        if (m < mt.n) acc[m] += eval_e(rn - (rm[m] + rj), mt.t[m], tj);
                }
            }
        }
        __syncthreads();
    }
    if (idx < npt) {
#pragma unroll
        for (int m = 0; m < MAX_MAPS; m++) {
            if (m < mt.n) {
                out32[(long long)m * npt + idx] = acc[m];
                if (out16) out16[(long long)m * npt + idx] = __float2half_rn(acc[m]);
            }
        }
    }
}

// ====================================================================== scoring kernels
struct PoseIO {
    const int* lig;          // per pose
    const long long* xoff;   // per pose: float offset of coords in xyz
    const float* xyz;
    const float* centers;    // 3 per pose
    const float* rotvecs;    // 3 per pose
    const long long* goff;   // per pose: offset of gradient in out_g
};

// CELLS: the direct sums walk the receptor cell list.  Grid scoring never reaches the direct
// sums, so its launches take the <false> instance and keep the smaller register budget (the cell
// walk costs k_score 14 registers, which is one resident CTA per SM fewer).
template <bool CELLS>
__global__ void k_score(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int n, PoseIO io, Env env,
                        float vcap, float slope, int ws_max, float* out_e, float* out_g) {
    extern __shared__ __align__(16) float smem[];
    int warp = threadIdx.x >> 5, lane = lane_id();
    int pose = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pose >= n) return;
    float* ws = smem + (size_t)warp * ws_max;
    const LigDev L = ligs[io.lig[pose]];
    const int* blob = blobs + L.blob_off;
    Topo T = topo_view(blob);
    Slot P = slot_at(ws, L.stride, 0, T.natom);
    Work W = work_at(ws, T);
    const float* x = io.xyz + io.xoff[pose];
    for (int i = lane; i < 3 * T.natom; i += WARP) P.x[i] = x[i];
    if (lane < 3) { P.h[1 + lane] = io.centers[3 * pose + lane]; P.h[4 + lane] = io.rotvecs[3 * pose + lane]; }
    __syncwarp();
    float e = eval_e_grad<CELLS>(T, env, P, W.F, W.g, vcap, slope, W.pb);
    if (lane == 0) out_e[pose] = e;
    float* g = out_g + io.goff[pose];
    for (int i = lane; i < 6 + T.ntors; i += WARP) g[i] = W.g[i];
}

// ---------------------------------------------------------------------- bandwidth probe
// Streaming read of a buffer (16-byte loads, grid-stride), summed so the loads are kept;
// one partial sum per thread block.  With a buffer that fits the L2 the repeated reads are
// L2 hits (the L2 read bandwidth); with one far larger, HBM reads.
__global__ void __launch_bounds__(512) k_read_probe(const float4* __restrict__ buf, long long n4, int passes,
                                                    float* out) {
    float s = 0.f;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int r = 0; r < passes; r++)
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            s += (v.x + v.y) + (v.z + v.w);
        }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + blockIdx.x, s);
}

// ---------------------------------------------------------------------- no-allocation scoring
// Staging area of ud_score_batch_noalloc: one per device (module-scope, allocated when the
// module loads), shared by every context on that device.  Holds, 256-byte aligned in
// this order: pose ligand ids (int), coordinate and gradient offsets (int64), coordinates,
// centres, rotation vectors, energies and gradients (float).
static __device__ __align__(256) unsigned char g_noalloc_scratch[UD_NOALLOC_SCRATCH_BYTES];

// exclusive prefix sums of 3*natom and 6+ntors over the poses (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) k_pose_offsets(const LigDev* __restrict__ ligs, int n,
                                                       const int* __restrict__ pose_lig, long long* xoff,
                                                       long long* goff) {
    __shared__ long long sx[32], sg[32];
    __shared__ long long carry_x, carry_g;
    const int warp = threadIdx.x >> 5, lane = lane_id();
    if (threadIdx.x == 0) { carry_x = 0; carry_g = 0; }
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        long long vx = 0, vg = 0;
        if (i < n) {
            const LigDev L = ligs[pose_lig[i]];
            vx = 3LL * L.natom;
            vg = 6LL + L.ntors;
        }
        long long ix = vx, ig = vg;          // inclusive warp scan
        for (int d = 1; d < WARP; d <<= 1) {
            long long tx = __shfl_up_sync(FULL, ix, d), tg = __shfl_up_sync(FULL, ig, d);
            if (lane >= d) { ix += tx; ig += tg; }
        }
        if (lane == WARP - 1) { sx[warp] = ix; sg[warp] = ig; }
        __syncthreads();
        if (warp == 0) {                     // scan of the warp totals
            long long wx = lane < (int)(blockDim.x >> 5) ? sx[lane] : 0;
            long long wg = lane < (int)(blockDim.x >> 5) ? sg[lane] : 0;
            for (int d = 1; d < WARP; d <<= 1) {
                long long tx = __shfl_up_sync(FULL, wx, d), tg = __shfl_up_sync(FULL, wg, d);
                if (lane >= d) { wx += tx; wg += tg; }
            }
            sx[lane] = wx;
            sg[lane] = wg;
        }
        __syncthreads();
        const long long px = (warp ? sx[warp - 1] : 0) + carry_x, pg = (warp ? sg[warp - 1] : 0) + carry_g;
        if (i < n) {
            xoff[i] = px + ix - vx;
            goff[i] = pg + ig - vg;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            carry_x = px + ix;
            carry_g = pg + ig;
        }
        __syncthreads();
    }
}

// score() without curl: intra over i<j, inter, penalty (slope 1e6), bias (score.cpp:12-108);
// decomp = per-atom inter terms (score.cpp:115-147)
__global__ void k_terms(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int n, const int* pose_lig,
                        const long long* xoff, const float* xyz, Env env, float* out4, float* decomp,
                        const long long* doff) {
    int warp = threadIdx.x >> 5, lane = lane_id();
    int pose = blockIdx.x * (blockDim.x >> 5) + warp;
    if (pose >= n) return;
    const LigDev L = ligs[pose_lig[pose]];
    Topo T = topo_view(blobs + L.blob_off);
    const float* X = xyz + xoff[pose];
    float e_intra = 0.f, e_inter = 0.f, e_pen = 0.f, e_bias = 0.f;
    for (int i = lane; i < T.natom; i += WARP) {
        int ti = T.type(i);
        float xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
        for (int k = T.pair_off(i); k < T.pair_off(i + 1); k++) {
            int j = T.pair(k) & 0xFFFF;
            if (j <= i) continue;
            float d0 = X[3 * j] - xi, d1 = X[3 * j + 1] - yi, d2 = X[3 * j + 2] - zi;
            float rr = d0 * d0 + d1 * d1 + d2 * d2;
            if (rr < 64.f) e_intra += eval_e(sqrtf(rr) - (vdw(ti) + vdw(T.type(j))), ti, T.type(j));
        }
        if (ti == VN_H) continue;
        float dec[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        if (env.mode == 1) {
            int m = T.map_index(i);
            float gx, gy, gz;
            if (m >= 0) e_inter += grid_sample(env.grid, m, xi, yi, zi, gx, gy, gz);
        } else {
            near_receptor(env, xi, yi, zi, [&](const float4 r) {
                double rr = cutoff_r2(r.x, r.y, r.z, xi, yi, zi);
                if (rr < 64.0) {
                    int tj = (int)r.w;
                    float d = sqrtf((float)rr) - (vdw(ti) + vdw(tj));
                    e_inter += eval_e(d, ti, tj);
                    if (decomp) {
                        float x1 = d * 2.f, x2 = (d - 3.f) * 0.5f;
                        dec[0] += -0.035579f * __expf(-x1 * x1);
                        dec[1] += -0.005156f * __expf(-x2 * x2);
                        dec[2] += d < 0.f ? 0.840245f * d * d : 0.f;
                        unsigned b1 = 1u << ti, b2 = 1u << tj;
                        if ((b1 & HYD_MASK) && (b2 & HYD_MASK))
                            dec[3] += -0.035069f * (d <= 0.5f ? 1.f : (d >= 1.5f ? 0.f : 1.5f - d));
                        if (((b1 & ACC_MASK) && (b2 & DON_MASK)) || ((b1 & DON_MASK) && (b2 & ACC_MASK)))
                            dec[4] += -0.587439f * (d <= -0.7f ? 1.f : (d >= 0.f ? 0.f : -d / 0.7f));
                    }
                }
            });
        }
        if (decomp) {
            float* o = decomp + doff[pose] + 5 * i;
            for (int q = 0; q < 5; q++) o[q] = dec[q];
        }
        float pen = 0.f;
        if (xi < env.box_lo[0]) pen += env.box_lo[0] - xi;
        if (xi > env.box_hi[0]) pen += xi - env.box_hi[0];
        if (yi < env.box_lo[1]) pen += env.box_lo[1] - yi;
        if (yi > env.box_hi[1]) pen += yi - env.box_hi[1];
        if (zi < env.box_lo[2]) pen += env.box_lo[2] - zi;
        if (zi > env.box_hi[2]) pen += zi - env.box_hi[2];
        e_pen += pen * PENALTY_SLOPE;
    }
    if (decomp) {  // hydrogens get zero rows
        for (int i = lane; i < T.natom; i += WARP)
            if (T.type(i) == VN_H)
                for (int q = 0; q < 5; q++) decomp[doff[pose] + 5 * i + q] = 0.f;
    }
    if (env.bias_type != 0) {
        for (int i = lane; i < T.natom; i += WARP) {
            for (int b = T.bias_off(i); b < T.bias_off(i + 1); b++) {
                const float* bp = T.bias() + 5 * b;
                float r[3] = {bp[0] - X[3 * i], bp[1] - X[3 * i + 1], bp[2] - X[3 * i + 2]};
                if (env.bias_type == 1) {
                    float rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                    e_bias += bp[3] * env.bias_k * expf(-rr / bp[4]);
                } else {
                    float ka = T.type(i) == VN_H ? 0.1f : 30.f;
                    float rn = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                    float ei = expf(3.f * (1.f - rn));
                    e_bias += bp[3] * env.bias_k * ka / (1.f + ei);
                }
            }
        }
    }
    e_intra = warp_sum(e_intra);
    e_inter = warp_sum(e_inter);
    e_pen = warp_sum(e_pen);
    e_bias = warp_sum(e_bias);
    if (lane == 0) {
        out4[4 * pose] = e_intra; out4[4 * pose + 1] = e_inter;
        out4[4 * pose + 2] = e_pen; out4[4 * pose + 3] = e_bias;
    }
}

// ====================================================================== BFGS batch
// CELLS as in k_score: refinement on the grid maps takes the <false> instance.
template <bool CELLS>
__global__ void k_bfgs(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int n, const int* item_lig,
                       const long long* item_off, float* recs, Env env, int max_steps, int rounds, float vcap,
                       float slope0, int ramp, int ws_max, int* nevals) {
    extern __shared__ __align__(16) float smem[];
    int warp = threadIdx.x >> 5, lane = lane_id();
    int item = blockIdx.x * (blockDim.x >> 5) + warp;
    if (item >= n) return;
    float* ws = smem + (size_t)warp * ws_max;
    const LigDev L = ligs[item_lig[item]];
    Topo T = topo_view(blobs + L.blob_off);
    Work W = work_at(ws, T);
    float* rec = recs + item_off[item];
    int nrec = 8 + 3 * T.natom + T.ntors;
    copy_words(ws, rec, nrec);
    int cur = 0, ne = 0;
    float slope = slope0;
    for (int r = 0; r < rounds; r++) {
        int others[3], k = 0;
        for (int s = 0; s < 4; s++) if (s != cur) others[k++] = s;
        cur = bfgs<CELLS>(T, env, ws, L.stride, cur, others[0], others[1], W, max_steps, vcap, slope, ne);
        if (ramp) slope = fminf(slope * 100.f, PENALTY_SLOPE);
    }
    copy_words(rec, ws + (size_t)cur * L.stride, nrec);
    if (nevals && lane == 0) nevals[item] = ne;
}

// ====================================================================== MC search
struct SearchP {
    uint32_t k0, k1;
    int nchain, mc_steps, opt_steps, randomize;
    int retain;        // poses kept per chain (1..4)
    int ws_max;        // floats per warp
    int blob_max;      // words reserved for the blob
};

__device__ __forceinline__ bool metropolis(float e_old, float e_new, float temp, float rx) {  // mc.h:12-18
    if (e_new < e_old) return true;
    return rx < expf((e_old - e_new) / temp);
}

__device__ __forceinline__ void store_record(float* dst, Slot P, int nrec) { copy_words(dst, P.h, nrec); }

// a chain's best record before its first improvement: the start pose, energy 1e9 (the
// bound every chain's first accepted pose is compared against)
__device__ __forceinline__ void init_best(float* out, Slot P, int nrec) {
    copy_words(out, P.h, nrec);
    if (lane_id() == 0) out[0] = 1e9f;
    __syncwarp();
}

// The poses a chain keeps in records out[r * stride]: its last R (1..4) new best poses,
// i.e. its R lowest-energy refined poses, each new best replacing the highest kept (1e9
// marks an unused record).  best() is the bound a refined pose has to beat, so the chain's
// moves do not depend on R; with R = 1 this is the reference's best pose per chain
// (mc.cu:376-393).
// RMAX: 1 (one pose, the common case, no extra registers) or 4 (R <= 4 at run time).
template <int RMAX>
struct Retained {
    float* out;
    int stride, R;
    float e0, e1, e2, e3;
    __device__ __forceinline__ float best() const {
        if constexpr (RMAX == 1) {
            return e0;
        } else {
            float m = e0;
            if (R > 1) m = fminf(m, e1);
            if (R > 2) m = fminf(m, e2);
            if (R > 3) m = fminf(m, e3);
            return m;
        }
    }
    __device__ __forceinline__ float worst() const {
        float m = e0;
        if (R > 1) m = fmaxf(m, e1);
        if (R > 2) m = fmaxf(m, e2);
        if (R > 3) m = fmaxf(m, e3);
        return m;
    }
    __device__ __forceinline__ void store(Slot P, int nrec, float energy) {
        if constexpr (RMAX == 1) {
            copy_words(out, P.h, nrec);
            e0 = energy;
        } else {
            const float t = worst();
            int r = 0;                               // the first record holding the highest energy
            if (!(e0 == t)) r = (R > 1 && e1 == t) ? 1 : ((R > 2 && e2 == t) ? 2 : 3);
            copy_words(out + (long long)r * stride, P.h, nrec);
            if (r == 0) e0 = energy; else if (r == 1) e1 = energy; else if (r == 2) e2 = energy; else e3 = energy;
        }
    }
};

// A learned move for one MC step: the proposal network's Gaussian (mean, raw log-variance
// per dimension, 6 + T used) and the probability of taking it instead of a random move.
struct Proposal {
    const float* out;     // 64 floats: mean[0:26], raw log-variance[26:52]; null: random moves only
    float p_learned;
};

// One MC step of a chain (mc.cu:323-393): the candidate (slot A+1) is the accepted pose
// with one move applied (a random move, or a sample of the learned proposal), optimised by
// BFGS with curl 10; Metropolis at T = 1.2 (step 0 always accepts); an accepted new best is
// optimised again with curl 1000 and recorded.  Returns the accepted slot; sets *accepted.
template <class Keep>
__device__ __forceinline__ int mc_step(const Topo& T, const Env& env, float* ws, int stride, int A, const Work& W,
                                       const Rng& rng, int step, int opt_steps, int nrec, Keep& keep,
                                       int& ne, const Proposal& prop, bool& accepted) {
    const int lane = lane_id();
    const int C = (A + 1) & 3;
    Slot SC = slot_at(ws, stride, C, T.natom);
    slot_copy(SC, slot_at(ws, stride, A, T.natom), T.natom, T.ntors);
    bool learned = false;
    if (prop.out) learned = u01(rng.draw((uint32_t)step, P_LEARN).x) < prop.p_learned;
    if (learned) {
        // One degree of freedom moves, chosen as the random move chooses it (mc.cu:158-169):
        // the centre, the orientation or one torsion.  Its change is a sample of the
        // network's Gaussian for those dimensions, m ~ N(mean, exp(logvar)) (Box-Muller on
        // Philox draws), in place of the random move's uniform draw; the rigid part is
        // clamped to a step of the random move's size.  Applied as one update of the
        // candidate.
        const int dim = 6 + T.ntors;
        const int nmut = 2 + T.ntors;
        const uint32_t uw = rng.draw((uint32_t)step, P_WHICH).x;
        const int which = env.constraint ? (nmut < 3 ? 3 : 2 + (int)(uw % (uint32_t)(nmut - 2)))
                                         : (int)(uw % (uint32_t)nmut);
        const bool mine = which == 0 ? lane < 3 : (which == 1 ? (lane >= 3 && lane < 6) : lane == 4 + which);
        if (lane < dim) {
            const U4 u = rng.draw((uint32_t)step, P_LNORM + (lane >> 2));
            const uint32_t ua = (lane & 2) ? u.z : u.x, ub = (lane & 2) ? u.w : u.y;
            const float r = sqrtf(-2.f * __logf(u01(ua))), th = 2.f * PI_F * u01(ub);
            float sn, cs;
            __sincosf(th, &sn, &cs);
            const float z = (lane & 1) ? r * sn : r * cs;
            const float lv = fminf(fmaxf(prop.out[26 + lane], -8.f), 4.f);
            float m = prop.out[lane] + __expf(0.5f * lv) * z;
            if (lane < 3) m = fminf(fmaxf(m, -2.f), 2.f);
            else if (lane < 6) m = fminf(fmaxf(m, -PI_F), PI_F);
            else m = fminf(fmaxf(m, -2.f * PI_F), 2.f * PI_F);
            if ((lane < 6 && env.constraint) || !mine) m = 0.f;
            if (!(m == m)) m = 0.f;
            W.p[lane] = m;
        }
        __syncwarp();
        // with BFGS the move is applied by its first line-search call (LS_MOVE)
        if (opt_steps == 0) apply_update(T, env, SC, W.p, 1.f, W.sc);
    } else {
        mutate(T, env, rng, (uint32_t)step, SC);
    }
    const float e_acc = ws[A * stride];
    const float rx = u01(rng.draw((uint32_t)step, P_METRO).x);
    accepted = false;
    if (opt_steps == 0) {
        float e = eval_e_grad(T, env, SC, W.F, W.g, VCAP_SEARCH, PENALTY_SLOPE, W.pb);
        ne++;
        if (lane == 0) SC.h[0] = e;
        __syncwarp();
        if (step == 0 || metropolis(e_acc, e, 1.2f, rx)) {
            A = C;
            accepted = true;
            if (e < keep.best()) keep.store(SC, nrec, e);
        }
        return A;
    }
    // slots: A holds the accepted pose; the other three serve the candidate and the
    // optimiser.  Both BFGS runs of a step (candidate with curl 10, accepted new best with
    // curl 1000) go through one call site (phase 0 / 1).
    for (int phase = 0; phase < 2; phase++) {
        const int X = (A + 1 - phase) & 3;
        const int R = bfgs(T, env, ws, stride, X, (X + 1) & 3, (X + 2) & 3, W, opt_steps,
                           phase ? VCAP_AUTH : VCAP_SEARCH, PENALTY_SLOPE, ne, (phase == 0 && learned) ? A : -1);
        const float e_new = ws[R * stride];
        if (phase == 0) {
            if (!(step == 0 || metropolis(e_acc, e_new, 1.2f, rx))) break;
            A = R;
            accepted = true;
            if (!(e_new < keep.best())) break;
        } else {
            A = R;
            if (e_new < keep.best()) keep.store(slot_at(ws, stride, A, T.natom), nrec, e_new);
        }
    }
    return A;
}

// Work items are (ligand, first chain, chain count) in descending ligand cost; CTAs take
// items from a global counter, re-stage the topology blob only when the ligand changes,
// and their warps take the item's chains from a shared counter.  Large ligands are so
// spread over many CTAs and the launch ends with the cheapest items.
// NT, MINB: the largest CTA and the CTAs per SM the register budget is sized for (256
// threads: 4 CTAs = 64 registers, 3 = 80; 384 threads: 2 CTAs = 80 registers); the host
// picks the width and instantiation that keep the most warps resident (shared memory
// holds one topology blob per CTA, so wide CTAs pay when the blob is large).
template <int MINB, int RMAX, int NT = 256>
__global__ void __launch_bounds__(NT, MINB) k_search(const int* __restrict__ blobs,
                                                const LigDev* __restrict__ ligs, const int4* __restrict__ items,
                                                int nitems, Env env, SearchP sp, float* best, int* work_counter,
                                                unsigned long long* nevals) {
    extern __shared__ __align__(16) float smem[];
    __shared__ int s_item, s_next, s_lig;
    int* sblob = reinterpret_cast<int*>(smem);
    float* wsbase = smem + sp.blob_max;
    const int warp = threadIdx.x >> 5, lane = lane_id();
    float* ws = wsbase + (size_t)warp * sp.ws_max;
    unsigned long long my_evals = 0, my_heavy = 0;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_flag;
    uint32_t phase = 0;
    if (threadIdx.x == 0) { s_lig = -1; stage_bar_init(&s_bar); }
    while (true) {
        if (threadIdx.x == 0) { s_item = atomicAdd(work_counter, 1); s_next = 0; }
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int4 item = items[it];          // (ligand, first chain, count, -)
        const LigDev L = ligs[item.x];
        if (item.x != s_lig && !stage_blob(sblob, blobs + L.blob_off, L.stage_words, &s_bar, phase, &s_flag)) {
            if (threadIdx.x == 0 && nevals) atomicAdd(nevals + 2, 1ull);
            break;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_lig = item.x;
        const Topo T = topo_view(sblob);
        const int nrec = 8 + 3 * T.natom + T.ntors;
        const Work W = work_at(ws, T);
        while (true) {
            int ci = 0;
            if (lane == 0) ci = atomicAdd(&s_next, 1);
            ci = __shfl_sync(FULL, ci, 0);
            if (ci >= item.z) break;
            const int c = item.y + ci;
            float* out = best + L.best_off + (long long)c * sp.retain * L.stride;
            Rng rng{sp.k0, sp.k1, (uint32_t)c, (uint32_t)L.lig_uid};
            int A = 0;
            Slot SA = slot_at(ws, L.stride, A, T.natom);
            load_initial(sblob, SA, T.natom, T.ntors);
            if (sp.randomize) randomize(T, env, rng, c, sp.nchain, SA, W.g, W.sc);
            for (int r = 0; r < sp.retain; r++) init_best(out + (long long)r * L.stride, SA, nrec);
            Retained<RMAX> keep{out, L.stride, sp.retain, 1e9f, 1e9f, 1e9f, 1e9f};
            int ne = 0;
            if (sp.mc_steps == 0) {
                float e = eval_e_f(T, env, SA.x, W.F, VCAP_SEARCH, PENALTY_SLOPE, W.pb);
                ne++;
                if (lane == 0) SA.h[0] = e;
                __syncwarp();
                store_record(out, SA, nrec);
            } else {
                const Proposal none{nullptr, 0.f};
                bool acc;
                for (int step = 0; step < sp.mc_steps; step++)
                    A = mc_step(T, env, ws, L.stride, A, W, rng, step, sp.opt_steps, nrec, keep, ne, none, acc);
            }
            my_evals += ne;
            my_heavy += (unsigned long long)ne * T.nheavy;
        }
        __syncthreads();
    }
    if (lane == 0 && nevals) {
        atomicAdd(nevals, my_evals);
        atomicAdd(nevals + 1, my_heavy);
    }
}

// ====================================================================== learned search
// The same MC chains as k_search, advanced a block of K steps per launch so that the
// proposals of all chains come from one batched evaluation of the proposal network: the
// accepted pose of each chain stays in HBM (`acc`, laid out as the best records) between
// launches; a block is k_learn_features -> network forward -> k_learn_step ->
// k_step_advance, captured once as a CUDA graph and replayed ceil(mc_steps / K) times.
// The network sees the block's first pose, so a learned move can replace only the block's
// first random move, with probability q = p_learned * K (p_learned stays the expected share
// of learned moves).  With p_learned = 0 the chains follow exactly the moves of k_search
// (same counter-based random stream, same step function).
struct LearnP {
    uint32_t k0, k1;
    int nchain, opt_steps, randomize;
    int retain;               // poses kept per chain (1..4)
    int ws_max, blob_max;
    float p_learned;          // q: probability of a learned move at a block's first step
    int nfeat_maps;           // grid maps used as features (<= 8)
    int block;                // K: MC steps per launch
    int mc_steps;
};
struct MoveSet {              // recorded accepted moves (training data)
    __nv_bfloat16* x;         // [max][672] features of the pose before the move
    float* y;                 // [max][26] move: centre shift, rotation vector, torsion changes
    float* m;                 // [max][26] mask of the dimensions that apply
    int* count;
    int max;
    int target;               // 0: the move to the next accepted pose; 1: to the ligand's best pose
    float* aux;               // target 1: [max][32] centre, rigid-frame atoms, dihedrals of the pose
    long long* chain;         // target 1: [max] chain of the sample
    // per-chain staging of one step ([chain] rows); k_move_scan / k_move_copy append the
    // staged rows in chain order, so the set's row order is (step, chain) on every run
    int* sflag;               // [nch] 1: the chain recorded a move this step
    int* spos;                // [nch] row in the set, or -1
    float* sy;                // [nch][26] move (target 0) or [nch][32] pose (target 1)
    float* sm;                // [nch][26] mask (target 0)
};
constexpr int AUX = 32;

// Features of a pose record (672 values): for each of up to 80 atoms the energies of the
// first 8 grid maps at the atom, squashed v / (1 + |v|); torsion angles / pi; the pose's
// energy squashed E / (10 + |E|); a constant 1; the centre relative to the box centre in
// units of 15 A (clamped to +-2); zero padding.
__device__ void pose_features(const Topo& T, const Env& env, const float* rec, int nmaps, __nv_bfloat16* row) {
    const int lane = lane_id();
    const float* x = rec + 8;
    const float* d = rec + 8 + 3 * T.natom;
    for (int i = lane; i < mlp::NATOM * mlp::NMAP; i += WARP) {
        const int a = i >> 3, m = i & 7;
        float v = 0.f;
        if (a < T.natom && m < nmaps) {
            float gx, gy, gz;
            v = grid_sample(env.grid, m, x[3 * a], x[3 * a + 1], x[3 * a + 2], gx, gy, gz);
            v = __fdividef(v, 1.f + fabsf(v));
            if (!(v == v)) v = 0.f;
        }
        row[i] = __float2bfloat16_rn(v);
    }
    for (int k = lane; k < mlp::IN - mlp::NATOM * mlp::NMAP; k += WARP) {
        float v = 0.f;
        if (k < mlp::TMAX) v = k < T.ntors ? d[k] * (1.f / PI_F) : 0.f;
        else if (k == mlp::TMAX) { const float e = rec[0]; v = __fdividef(e, 10.f + fabsf(e)); if (!(v == v)) v = 0.f; }
        else if (k == mlp::TMAX + 1) v = 1.f;
        else if (k < mlp::TMAX + 5) {               // centre relative to the box centre / 15 A
            const int a = k - mlp::TMAX - 2;
            v = fminf(fmaxf((rec[1 + a] - 0.5f * (env.box_lo[a] + env.box_hi[a])) * (1.f / 15.f), -2.f), 2.f);
            if (!(v == v)) v = 0.f;
        }
        row[mlp::NATOM * mlp::NMAP + k] = __float2bfloat16_rn(v);
    }
}

__global__ void k_learn_features(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int nlig, int nchain,
                                 Env env, const float* __restrict__ acc, const int* __restrict__ step_p, int nmaps,
                                 __nv_bfloat16* __restrict__ X) {
    if (*step_p == 0) return;                      // no accepted pose before the first step
    const long long nch = (long long)nlig * nchain;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long g = w0; g < nch; g += nw) {
        const int lig = (int)(g / nchain), c = (int)(g % nchain);
        const LigDev L = ligs[lig];
        const Topo T = topo_view(blobs + L.blob_off);
        pose_features(T, env, acc + L.best_off + (long long)c * L.stride, nmaps, X + g * mlp::IN);
    }
}

__global__ void k_step_advance(int* step_p, int block) { *step_p += block; }

// rotation vector of the rotation taking the old frame of atoms (f0, f1, f2) to the new one
// (po, pn: the frame's three points, 9 floats each, before and after)
__device__ void frame_rotvec_pts(const float* po, const float* pn, float* rv) {
    float e[2][3][3];
    const float* xs[2] = {po, pn};
    for (int s = 0; s < 2; s++) {
        const float* x = xs[s];
        float u[3], w[3];
        for (int i = 0; i < 3; i++) { u[i] = x[3 + i] - x[i]; w[i] = x[6 + i] - x[i]; }
        const float iu = rsqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int i = 0; i < 3; i++) u[i] *= iu;
        const float p = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
        for (int i = 0; i < 3; i++) w[i] -= p * u[i];
        const float iw = rsqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        for (int i = 0; i < 3; i++) w[i] *= iw;
        for (int i = 0; i < 3; i++) { e[s][0][i] = u[i]; e[s][1][i] = w[i]; }
        e[s][2][0] = u[1] * w[2] - u[2] * w[1];
        e[s][2][1] = u[2] * w[0] - u[0] * w[2];
        e[s][2][2] = u[0] * w[1] - u[1] * w[0];
    }
    float R[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) R[i][j] = e[1][0][i] * e[0][0][j] + e[1][1][i] * e[0][1][j] + e[1][2][i] * e[0][2][j];
    const float ct = fminf(fmaxf(0.5f * (R[0][0] + R[1][1] + R[2][2] - 1.f), -1.f), 1.f);
    const float th = acosf(ct);
    const float a0 = R[2][1] - R[1][2], a1 = R[0][2] - R[2][0], a2 = R[1][0] - R[0][1];
    const float sn = sinf(th);
    const float k = sn > 1e-4f ? th / (2.f * sn) : 0.5f;
    rv[0] = k * a0; rv[1] = k * a1; rv[2] = k * a2;
    if (!(rv[0] == rv[0] && rv[1] == rv[1] && rv[2] == rv[2])) rv[0] = rv[1] = rv[2] = 0.f;
}
__device__ void frame_rotvec(const float* xo, const float* xn, int f0, int f1, int f2, float* rv) {
    float po[9], pn[9];
    const int f[3] = {f0, f1, f2};
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) { po[3 * j + i] = xo[3 * f[j] + i]; pn[3 * j + i] = xn[3 * f[j] + i]; }
    frame_rotvec_pts(po, pn, rv);
}

// stage (the move, its mask) of chain g for this step; the features of the pose before
// the move are row g of the step's feature matrix.  Moves with a non-finite value (a chain
// whose pose diverged) are not recorded.  Every chain writes its flag every step.
__device__ void record_move(const Topo& T, const Env& env, const float* old_rec, Slot P, bool accepted, MoveSet D,
                            long long g) {
    const int lane = lane_id();
    const int f0 = T.b[H_FRAME0], f1 = T.b[H_FRAME0 + 1], f2 = T.b[H_FRAME0 + 2];
    if (!accepted) {
        if (lane == 0) D.sflag[g] = 0;
        return;
    }
    if (D.target == 1) {
        // the pose before the move; its target is labelled after the run (k_label_moves)
        float a = 0.f;
        if (lane < 3) a = old_rec[1 + lane];
        else if (lane < 12) { const int j = (lane - 3) / 3, i = (lane - 3) % 3; const int f = j == 0 ? f0 : (j == 1 ? f1 : f2);
                              a = f >= 0 ? old_rec[8 + 3 * f + i] : 0.f; }
        else if (lane - 12 < T.ntors) a = old_rec[8 + 3 * T.natom + (lane - 12)];
        const bool ok = __all_sync(FULL, isfinite(a));
        D.sy[g * AUX + lane] = a;
        if (lane == 0) D.sflag[g] = ok ? 1 : 0;
        return;
    }
    const bool rigid = !env.constraint;
    float yv = 0.f, mv = 0.f;                 // lane d < 26 holds dimension d
    float rv[3] = {0.f, 0.f, 0.f};
    const bool frame_ok = rigid && f0 >= 0;
    if (lane == 0 && frame_ok) frame_rotvec(old_rec + 8, P.x, f0, f1, f2, rv);
    rv[0] = __shfl_sync(FULL, rv[0], 0);
    rv[1] = __shfl_sync(FULL, rv[1], 0);
    rv[2] = __shfl_sync(FULL, rv[2], 0);
    if (lane < 3) {
        yv = P.h[1 + lane] - old_rec[1 + lane];
        mv = rigid ? 1.f : 0.f;
    } else if (lane < 6) {
        yv = rv[lane - 3];
        mv = frame_ok ? 1.f : 0.f;
    } else if (lane < mlp::NDIM && lane - 6 < T.ntors) {
        yv = normalize_angle(P.d[lane - 6] - old_rec[8 + 3 * T.natom + (lane - 6)]);
        mv = 1.f;
    }
    const bool ok = __all_sync(FULL, isfinite(yv));
    if (lane < mlp::NDIM) {
        D.sy[g * mlp::NDIM + lane] = yv;
        D.sm[g * mlp::NDIM + lane] = mv;
    }
    if (lane == 0) D.sflag[g] = ok ? 1 : 0;
}

// rows of the staged moves in chain order: spos[g] = count + (flags before g), or -1;
// count += flags (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) k_move_scan(MoveSet D, long long nch) {
    __shared__ int sw[32];
    __shared__ int carry;
    const int warp = threadIdx.x >> 5, lane = lane_id();
    if (threadIdx.x == 0) carry = *D.count;
    __syncthreads();
    for (long long base = 0; base < nch; base += blockDim.x) {
        const long long g = base + threadIdx.x;
        const int f = g < nch ? D.sflag[g] : 0;
        int incl = f;
        for (int d = 1; d < WARP; d <<= 1) {
            const int t = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == WARP - 1) sw[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = lane < (int)(blockDim.x >> 5) ? sw[lane] : 0;
            for (int d = 1; d < WARP; d <<= 1) {
                const int t = __shfl_up_sync(FULL, w, d);
                if (lane >= d) w += t;
            }
            sw[lane] = w;
        }
        __syncthreads();
        const int pre = carry + (warp ? sw[warp - 1] : 0) + incl - f;
        if (g < nch) D.spos[g] = f ? pre : -1;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = pre + f;
        __syncthreads();
    }
    if (threadIdx.x == 0) *D.count = carry;
}

// copy each staged row to its place in the set (warp per chain; rows past max are dropped)
__global__ void k_move_copy(MoveSet D, const __nv_bfloat16* __restrict__ X, long long nch) {
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const int lane = lane_id();
    for (long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; g < nch; g += nw) {
        const int idx = D.spos[g];
        if (idx < 0 || idx >= D.max) continue;
        const uint32_t* xs = reinterpret_cast<const uint32_t*>(X + g * mlp::IN);
        uint32_t* xd = reinterpret_cast<uint32_t*>(D.x + (long long)idx * mlp::IN);
        for (int i = lane; i < mlp::IN / 2; i += WARP) xd[i] = xs[i];
        if (D.target == 1) {
            D.aux[(long long)idx * AUX + lane] = D.sy[g * AUX + lane];
            if (lane == 0) D.chain[idx] = g;
        } else if (lane < mlp::NDIM) {
            D.y[(long long)idx * mlp::NDIM + lane] = D.sy[g * mlp::NDIM + lane];
            D.m[(long long)idx * mlp::NDIM + lane] = D.sm[g * mlp::NDIM + lane];
        }
    }
}

// best chain of every ligand (lowest best energy, NaN as +inf, ties to the lower index)
__global__ void k_lig_best(const LigDev* __restrict__ ligs, int nlig, int nchain, const float* __restrict__ best,
                           int* out) {
    __shared__ float se[256];
    __shared__ int si[256];
    const int lig = blockIdx.x;
    if (lig >= nlig) return;
    const LigDev L = ligs[lig];
    float e = INFINITY;
    int ix = 0x7fffffff;
    for (int c = threadIdx.x; c < nchain; c += blockDim.x) {
        float v = best[L.best_off + (long long)c * L.stride];
        if (!(v == v)) v = INFINITY;
        if (v < e || (v == e && c < ix)) { e = v; ix = c; }
    }
    se[threadIdx.x] = e;
    si[threadIdx.x] = ix;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const float e2 = se[threadIdx.x + o];
            const int i2 = si[threadIdx.x + o];
            if (e2 < se[threadIdx.x] || (e2 == se[threadIdx.x] && i2 < si[threadIdx.x])) { se[threadIdx.x] = e2; si[threadIdx.x] = i2; }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[lig] = si[0] == 0x7fffffff ? 0 : si[0];
}

// targets of recorded poses: the move from each pose to its ligand's best pose
__global__ void k_label_moves(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int nchain,
                              const float* __restrict__ best, const int* __restrict__ lig_best, MoveSet D, int n,
                              int constraint) {
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (w >= n) return;
    const long long g = D.chain[w];
    const int lig = (int)(g / nchain);
    const LigDev L = ligs[lig];
    const Topo T = topo_view(blobs + L.blob_off);
    const float* b = best + L.best_off + (long long)lig_best[lig] * L.stride;
    const float* a = D.aux + w * AUX;
    const int f0 = T.b[H_FRAME0], f1 = T.b[H_FRAME0 + 1], f2 = T.b[H_FRAME0 + 2];
    const bool rigid = !constraint;
    const bool frame_ok = rigid && f0 >= 0;
    float rv[3] = {0.f, 0.f, 0.f};
    if (lane == 0 && frame_ok) {
        float pn[9];
        const int f[3] = {f0, f1, f2};
        for (int j = 0; j < 3; j++)
            for (int i = 0; i < 3; i++) pn[3 * j + i] = b[8 + 3 * f[j] + i];
        frame_rotvec_pts(a + 3, pn, rv);
    }
    float yv = 0.f, mv = 0.f;
    const float r0 = __shfl_sync(FULL, rv[0], 0), r1 = __shfl_sync(FULL, rv[1], 0), r2 = __shfl_sync(FULL, rv[2], 0);
    if (lane < 3) { yv = b[1 + lane] - a[lane]; mv = rigid ? 1.f : 0.f; }
    else if (lane < 6) { yv = lane == 3 ? r0 : (lane == 4 ? r1 : r2); mv = frame_ok ? 1.f : 0.f; }
    else if (lane < mlp::NDIM && lane - 6 < T.ntors) {
        yv = normalize_angle(b[8 + 3 * T.natom + (lane - 6)] - a[12 + (lane - 6)]);
        mv = 1.f;
    }
    if (!isfinite(yv)) { yv = 0.f; mv = 0.f; }
    if (lane < mlp::NDIM) {
        D.y[w * mlp::NDIM + lane] = yv;
        D.m[w * mlp::NDIM + lane] = mv;
    }
}

template <int MINB, int RMAX, int NT = 256>
__global__ void __launch_bounds__(NT, MINB) k_learn_step(const int* __restrict__ blobs,
                                                        const LigDev* __restrict__ ligs, const int4* __restrict__ items,
                                                        int nitems, Env env, LearnP sp, const int* __restrict__ step_p,
                                                        float* acc, float* best, const float* __restrict__ prop_out,
                                                        const __nv_bfloat16* __restrict__ X, MoveSet rec_set,
                                                        int* work_counter, unsigned long long* nevals) {
    extern __shared__ __align__(16) float smem[];
    __shared__ int s_item, s_next, s_lig;
    int* sblob = reinterpret_cast<int*>(smem);
    float* wsbase = smem + sp.blob_max;
    const int warp = threadIdx.x >> 5, lane = lane_id();
    float* ws = wsbase + (size_t)warp * sp.ws_max;
    const int step0 = *step_p;
    const int nsteps = min(sp.block, sp.mc_steps - step0);
    unsigned long long my_evals = 0, my_heavy = 0;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_flag;
    uint32_t phase = 0;
    if (threadIdx.x == 0) { s_lig = -1; stage_bar_init(&s_bar); }
    while (true) {
        if (threadIdx.x == 0) { s_item = atomicAdd(work_counter, 1); s_next = 0; }
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const int4 item = items[it];
        const LigDev L = ligs[item.x];
        if (item.x != s_lig && !stage_blob(sblob, blobs + L.blob_off, L.stage_words, &s_bar, phase, &s_flag)) {
            if (threadIdx.x == 0 && nevals) atomicAdd(nevals + 2, 1ull);
            break;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_lig = item.x;
        const Topo T = topo_view(sblob);
        const int nrec = 8 + 3 * T.natom + T.ntors;
        const Work W = work_at(ws, T);
        while (true) {
            int ci = 0;
            if (lane == 0) ci = atomicAdd(&s_next, 1);
            ci = __shfl_sync(FULL, ci, 0);
            if (ci >= item.z) break;
            const int c = item.y + ci;
            const long long g = (long long)item.x * sp.nchain + c;
            float* out = best + L.best_off + (long long)c * sp.retain * L.stride;
            float* accp = acc + L.best_off + (long long)c * L.stride;
            const Rng rng{sp.k0, sp.k1, (uint32_t)c, (uint32_t)L.lig_uid};
            Slot SA = slot_at(ws, L.stride, 0, T.natom);
            Retained<RMAX> keep{out, L.stride, sp.retain, 1e9f, 1e9f, 1e9f, 1e9f};
            if (step0 == 0) {
                load_initial(sblob, SA, T.natom, T.ntors);
                if (sp.randomize) randomize(T, env, rng, c, sp.nchain, SA, W.g, W.sc);
                for (int r = 0; r < sp.retain; r++) init_best(out + (long long)r * L.stride, SA, nrec);
            } else {
                copy_words(SA.h, accp, nrec);
                keep.e0 = out[0];
                if (sp.retain > 1) keep.e1 = out[L.stride];
                if (sp.retain > 2) keep.e2 = out[2LL * L.stride];
                if (sp.retain > 3) keep.e3 = out[3LL * L.stride];
            }
            __syncwarp();
            int ne = 0, A = 0;
            for (int s = 0; s < nsteps; s++) {
                const int step = step0 + s;
                const Proposal prop{(prop_out && step > 0 && s == 0) ? prop_out + g * mlp::OUT : nullptr,
                                    sp.p_learned};
                bool accepted;
                A = mc_step(T, env, ws, L.stride, A, W, rng, step, sp.opt_steps, nrec, keep, ne, prop, accepted);
                // moves are recorded with blocks of one step (the features are the block's first pose)
                if (rec_set.count && step > 0)
                    record_move(T, env, accp, slot_at(ws, L.stride, A, T.natom), accepted, rec_set, g);
            }
            __syncwarp();
            copy_words(accp, slot_at(ws, L.stride, A, T.natom).h, nrec);
            my_evals += ne;
            my_heavy += (unsigned long long)ne * T.nheavy;
        }
        __syncthreads();
    }
    if (lane == 0 && nevals) {
        atomicAdd(nevals, my_evals);
        atomicAdd(nevals + 1, my_heavy);
    }
}

// ====================================================================== clustering
// CTA per ligand.  Ranking by (energy, index) with NaN as +inf; greedy leaders with
// per-thread fixed-order fmaf sums over heavy atoms (bit-identical to the oracle).
__global__ void k_cluster(const int* __restrict__ blobs, const LigDev* __restrict__ ligs, int nlig, int nchain,
                          const float* __restrict__ best, float rmsd_limit, int* leaders, int* counts) {
    extern __shared__ __align__(16) float smem[];
    float* e = smem;
    int* order = reinterpret_cast<int*>(e + nchain);
    int* lead = order + nchain;
    __shared__ int s_nl;
    int lig = blockIdx.x;
    if (lig >= nlig) return;
    const LigDev L = ligs[lig];
    Topo T = topo_view(blobs + L.blob_off);
    const float* base = best + L.best_off;
    for (int i = threadIdx.x; i < nchain; i += blockDim.x) {
        float v = base[(long long)i * L.stride];
        e[i] = isnan(v) ? INFINITY : v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nchain; i += blockDim.x) {
        float ei = e[i];
        int r = 0;
        for (int j = 0; j < nchain; j++) {
            float ej = e[j];
            r += (ej < ei) || (ej == ei && j < i);
        }
        order[r] = i;
    }
    if (threadIdx.x == 0) s_nl = 0;
    __syncthreads();
    float thr = __fmul_rn(__fmul_rn(rmsd_limit, rmsd_limit), (float)T.nheavy);
    for (int o = 0; o < nchain; o++) {
        int c = order[o];
        int nl = s_nl;
        const float* xc = base + (long long)c * L.stride + 8;
        int close = 0;
        for (int t = threadIdx.x; t < nl; t += blockDim.x) {
            const float* xl = base + (long long)lead[t] * L.stride + 8;
            float acc = 0.f;
            for (int h = 0; h < T.nheavy; h++) {
                int a = T.heavy(h);
                float dx = __fsub_rn(xc[3 * a], xl[3 * a]);
                float dy = __fsub_rn(xc[3 * a + 1], xl[3 * a + 1]);
                float dz = __fsub_rn(xc[3 * a + 2], xl[3 * a + 2]);
                acc = __fmaf_rn(dx, dx, acc);
                acc = __fmaf_rn(dy, dy, acc);
                acc = __fmaf_rn(dz, dz, acc);
            }
            if (acc < thr) close = 1;
        }
        int any = __syncthreads_or(close);
        if (!any && threadIdx.x == 0) { lead[nl] = c; s_nl = nl + 1; }
        __syncthreads();
    }
    int nl = s_nl;
    for (int i = threadIdx.x; i < nchain; i += blockDim.x) leaders[(long long)lig * nchain + i] = i < nl ? lead[i] : -1;
    if (threadIdx.x == 0) counts[lig] = nl;
}

// energy_range / num_pose filter over the refined leaders (DockTask.cpp:188-220);
// out_sel[lig*num_pose + k] = chain index of the k-th output pose
__global__ void k_filter(const LigDev* __restrict__ ligs, int nlig, int nchain, const float* __restrict__ best,
                         const int* leaders, const int* counts, int num_pose, float energy_range, int* out_sel,
                         int* out_count) {
    extern __shared__ __align__(16) float smem[];
    float* e = smem;
    int* order = reinterpret_cast<int*>(e + nchain);
    int lig = blockIdx.x;
    if (lig >= nlig) return;
    const LigDev L = ligs[lig];
    int nl = counts[lig];
    const int* ld = leaders + (long long)lig * nchain;
    for (int i = threadIdx.x; i < nl; i += blockDim.x) {
        float v = best[L.best_off + (long long)ld[i] * L.stride];
        e[i] = isnan(v) ? INFINITY : v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nl; i += blockDim.x) {
        float ei = e[i];
        int r = 0;
        for (int j = 0; j < nl; j++) r += (e[j] < ei) || (e[j] == ei && j < i);
        order[r] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int cnt = 0;
        if (nl > 0) {
            float emin = e[order[0]];
            for (int k = 0; k < nl; k++) {
                float v = e[order[k]];
                if (v > emin + energy_range) break;
                out_sel[(long long)lig * num_pose + cnt] = ld[order[k]];
                cnt++;
                if (cnt >= num_pose) break;
            }
        }
        out_count[lig] = cnt;
    }
}

// gather selected records into the output buffer and list them for scoring
__global__ void k_gather(const LigDev* __restrict__ ligs, int nlig, int num_pose, const float* __restrict__ best,
                         const int* sel, const int* cnt, float* out_rec) {
    int warp = threadIdx.x >> 5;
    long long item = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (item >= (long long)nlig * num_pose) return;
    int lig = (int)(item / num_pose), k = (int)(item % num_pose);
    if (k >= cnt[lig]) return;
    const LigDev L = ligs[lig];
    int c = sel[item];
    const float* src = best + L.best_off + (long long)c * L.stride;
    float* dst = out_rec + L.out_off + (long long)k * L.stride;
    for (int i = lane_id(); i < L.stride; i += WARP) dst[i] = src[i];
}

// ====================================================================== host side
namespace {
thread_local std::string g_err;

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Fail(UD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void ensure(size_t count) {
        if (count <= n && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        if (count == 0) count = 1;
        ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        ensure(count);
        if (count) ck(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s), "H2D");
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
};

struct LigHost {
    int natom, ntors, nheavy, blob_words, stride, nprec, stage_words;
    long long blob_off;
};
inline int lig_ws(const LigHost& h) { return ws_floats(h.natom, h.ntors, h.nprec); }
}  // namespace

#include "ud_mlp_host.cuh"

struct ud_ctx {
    int device = 0;
    int nsm = 148;
    cudaStream_t stream = nullptr;
    float box_lo[3], box_hi[3];
    int constraint = 0, bias_type = 0;
    float bias_k = 0.1f;
    // receptor
    std::vector<float4> h_rec;
    DBuf<float4> d_rec_cells;           // receptor atoms sorted into CELL_A cells (direct sums)
    DBuf<int> d_cell_start;
    float cell_o[3] = {0, 0, 0};
    int cdim[3] = {1, 1, 1};
    DBuf<float4> d_rec;
    // grid
    DBuf<float> d_maps32;
    DBuf<__half> d_maps16;
    int nmaps = 0, gdim[3] = {0, 0, 0}, grid_prec = 0;
    float origin[3] = {0, 0, 0}, spacing = 0.f;
    signed char map_of_type[NT + 3];
    // ligands
    std::vector<int> h_blobs;
    std::vector<LigHost> h_ligs;
    std::vector<LigDev> h_ligdev;
    DBuf<int> d_blobs;
    DBuf<LigDev> d_ligs;
    bool ligs_dirty = true;
    int max_natom = 0, max_ntors = 0, max_blob = 0, max_stage = 0;
    // search state
    int nchain = 0;
    long long best_floats = 0;
    DBuf<float> d_best;
    DBuf<int> d_order, d_counter, d_leaders, d_counts, d_sel, d_selcnt;
    DBuf<int4> d_items;
    DBuf<unsigned long long> d_nevals;
    // results
    int num_pose = 0;
    long long out_floats = 0;
    DBuf<float> d_out, d_terms, d_decomp;
    DBuf<int> d_item_lig;
    DBuf<long long> d_item_off, d_item_off2;
    std::vector<int> h_counts;
    bool has_results = false;
    bool decomp = false;
    // learned move proposal: the network, the learned search's chain state and step
    // counter, the features of every chain, and the recorded accepted moves
    MlpState mlp;
    DBuf<float> d_acc;
    DBuf<int> d_step;
    DBuf<__nv_bfloat16> d_x16, d_mx;
    DBuf<float> d_my, d_mm;
    DBuf<int> d_mcount, d_ligbest;
    DBuf<float> d_maux;
    DBuf<long long> d_mchain;
    DBuf<int> d_sflag, d_spos;          // per-chain move staging of one learned-search step
    DBuf<float> d_sy, d_sm;
    int moves_max = 0, moves_n = 0;
    // chain packing autotuner (warps per CTA, chains per warp per work item)
    int autotune = 0, tune_w = 8, tune_k = 0;
    int pack_w = 0, pack_k = 0;               // ud_set_packing (0: chosen per batch)
    int shape[4] = {0, 0, 0, 0};              // last search: W, CTAs per SM, minb, k
    int retain = 1;                                   // poses kept per chain
    long long tune_key = -1;
    // measurement
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    float stage_ms[6] = {0, 0, 0, 0, 0, 0};
    long long counters[4] = {0, 0, 0, 0};
    void rec(int i) { cudaEventRecord(ev[i], stream); }
};

namespace {

int fail(const Fail& f) {
    g_err = f.what();
    return f.code;
}

Env make_env(ud_ctx* c, int mode) {
    Env e;
    for (int a = 0; a < 3; a++) { e.box_lo[a] = c->box_lo[a]; e.box_hi[a] = c->box_hi[a]; }
    e.mode = mode;
    e.constraint = c->constraint;
    e.bias_type = c->bias_type;
    e.bias_k = c->bias_k;
    e.rec = c->d_rec.p;
    e.nrec = (int)c->h_rec.size();
    e.rec_cells = c->d_rec_cells.p;
    e.cell_start = c->d_cell_start.p;
    for (int a = 0; a < 3; a++) { e.cell_o[a] = c->cell_o[a]; e.cdim[a] = c->cdim[a]; }
    e.grid.f32 = c->d_maps32.p;
    e.grid.f16 = c->d_maps16.p;
    e.grid.use_f16 = (c->grid_prec == UD_GRID_F16 && c->d_maps16.p) ? 1 : 0;
    e.grid.ox = c->origin[0]; e.grid.oy = c->origin[1]; e.grid.oz = c->origin[2];
    e.grid.inv_s = c->spacing > 0 ? 1.f / c->spacing : 0.f;
    e.grid.gx = c->gdim[0]; e.grid.gy = c->gdim[1]; e.grid.gz = c->gdim[2];
    if (mode == UD_MODE_GRID && c->nmaps == 0) throw Fail(UD_ESTATE, "grid mode requested but no grid was built");
    return e;
}

void sync_ligs(ud_ctx* c) {
    if (!c->ligs_dirty) return;
    for (const LigHost& h : c->h_ligs) {       // per-atom grid map slot for the current maps
        int* b = c->h_blobs.data() + h.blob_off;
        for (int i = 0; i < h.natom; i++) b[b[H_MAPIDX] + i] = c->map_of_type[b[b[H_TYPES] + i]];
    }
    c->d_blobs.upload(c->h_blobs.data(), c->h_blobs.size(), c->stream);
    c->h_ligdev.resize(c->h_ligs.size());
    for (size_t i = 0; i < c->h_ligs.size(); i++) {
        const LigHost& h = c->h_ligs[i];
        LigDev& d = c->h_ligdev[i];
        d.blob_off = (int)h.blob_off;
        d.blob_words = h.blob_words;
        d.natom = h.natom;
        d.ntors = h.ntors;
        d.nheavy = h.nheavy;
        d.stride = h.stride;
        d.lig_uid = (int)i;
        d.stage_words = h.stage_words;
        d.best_off = 0;
        d.out_off = 0;
    }
    c->d_ligs.upload(c->h_ligdev.data(), c->h_ligdev.size(), c->stream);
    c->ligs_dirty = false;
}

void upload_ligdev(ud_ctx* c) { c->d_ligs.upload(c->h_ligdev.data(), c->h_ligdev.size(), c->stream); }

int smem_limit(ud_ctx* c) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    return v > 0 ? v : 48 * 1024;
}

// warps per CTA so that W warps of ws floats fit beside `extra` floats
int pick_warps(ud_ctx* c, int ws, int extra, int want) {
    int lim = smem_limit(c) / 4 - extra - 64;
    int w = want;
    while (w > 1 && w * ws > lim) w--;
    if (w * ws > lim) throw Fail(UD_EINVAL, "ligand too large for shared memory");
    return w;
}

template <typename K>
void set_smem(K kernel, size_t bytes) {
    ck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "smem attribute");
}

// The scoring and refinement kernels of a scoring mode: only direct sums walk the cell list.
auto score_kernel(const Env& env) { return env.mode == UD_MODE_GRID ? k_score<false> : k_score<true>; }
auto bfgs_kernel(const Env& env) { return env.mode == UD_MODE_GRID ? k_bfgs<false> : k_bfgs<true>; }

}  // namespace

// ====================================================================== C ABI
extern "C" {

int ud_version(void) { return 100; }

const char* ud_last_error(void) { return g_err.c_str(); }

int ud_device_memory(int device, long long* out_free, long long* out_total) {
    try {
        if (!out_free || !out_total) throw Fail(UD_EINVAL, "null argument");
        int cur = 0;
        ck(cudaGetDevice(&cur), "cudaGetDevice");
        ck(cudaSetDevice(device), "cudaSetDevice");
        size_t fr = 0, tot = 0;
        const cudaError_t e = cudaMemGetInfo(&fr, &tot);
        cudaSetDevice(cur);
        ck(e, "cudaMemGetInfo");
        *out_free = (long long)fr;
        *out_total = (long long)tot;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_create(int device, const float* box6, ud_ctx** out) {
    try {
        if (!out || !box6) throw Fail(UD_EINVAL, "null argument");
        int ndev = 0;
        ck(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
        if (ndev <= 0) throw Fail(UD_ECUDA, "No CUDA device is found!");
        if (device < 0 || device >= ndev) throw Fail(UD_EINVAL, "invalid device id");
        ck(cudaSetDevice(device), "cudaSetDevice");
        ud_ctx* c = new ud_ctx();
        c->device = device;
        cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        for (auto& e : c->ev) ck(cudaEventCreate(&e), "cudaEventCreate");
        c->box_lo[0] = box6[0]; c->box_hi[0] = box6[1];
        c->box_lo[1] = box6[2]; c->box_hi[1] = box6[3];
        c->box_lo[2] = box6[4]; c->box_hi[2] = box6[5];
        for (int i = 0; i < NT + 3; i++) c->map_of_type[i] = -1;
        *out = c;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_destroy(ud_ctx* c) {
    if (!c) return UD_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->d_rec.release(); c->d_rec_cells.release(); c->d_cell_start.release();
    c->d_maps32.release(); c->d_maps16.release();
    c->d_blobs.release(); c->d_ligs.release(); c->d_best.release();
    c->d_order.release(); c->d_items.release(); c->d_counter.release(); c->d_leaders.release(); c->d_counts.release();
    c->d_sel.release(); c->d_selcnt.release(); c->d_nevals.release();
    c->d_out.release(); c->d_terms.release(); c->d_decomp.release();
    c->d_item_lig.release(); c->d_item_off.release(); c->d_item_off2.release();
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return UD_OK;
}

int ud_set_flags(ud_ctx* c, int constraint, int bias_type, float bias_k) {
    if (!c) { g_err = "null context"; return UD_EINVAL; }
    if (bias_type < 0 || bias_type > 2) { g_err = "bias_type must be 0, 1 or 2"; return UD_EINVAL; }
    c->constraint = constraint ? 1 : 0;
    c->bias_type = bias_type;
    c->bias_k = bias_k;
    return UD_OK;
}

int ud_set_receptor(ud_ctx* c, int n, const float* xyz, const int* types) {
    try {
        if (!c || n < 0 || (n > 0 && (!xyz || !types))) throw Fail(UD_EINVAL, "invalid receptor arguments");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        c->h_rec.clear();
        for (int i = 0; i < n; i++) {
            int t = types[i];
            if (t < 0 || t >= NT) throw Fail(UD_EINVAL, "receptor type out of range");
            if (t == VN_H) continue;
            float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
            bool in = (c->box_lo[0] - 8.f <= x && x <= c->box_hi[0] + 8.f) &&
                      (c->box_lo[1] - 8.f <= y && y <= c->box_hi[1] + 8.f) &&
                      (c->box_lo[2] - 8.f <= z && z <= c->box_hi[2] + 8.f);
            if (in) c->h_rec.push_back(make_float4(x, y, z, (float)t));
        }
        c->d_rec.upload(c->h_rec.data(), c->h_rec.size(), c->stream);
        // cell list over the kept region (box +- 8 A): counting sort, stable in receptor order
        int ncell = 1;
        for (int a = 0; a < 3; a++) {
            c->cell_o[a] = c->box_lo[a] - 8.f;
            c->cdim[a] = (int)std::floor((c->box_hi[a] + 8.f - c->cell_o[a]) * (1.f / CELL_A)) + 1;
            ncell *= c->cdim[a];
        }
        auto cell_of = [&](const float4& r) {
            const float p[3] = {r.x, r.y, r.z};
            int q[3];
            for (int a = 0; a < 3; a++) {
                const float f = std::floor((p[a] - c->cell_o[a]) * (1.f / CELL_A));
                q[a] = std::min(std::max((int)f, 0), c->cdim[a] - 1);
            }
            return (q[2] * c->cdim[1] + q[1]) * c->cdim[0] + q[0];
        };
        std::vector<int> start((size_t)ncell + 1, 0);
        for (const float4& r : c->h_rec) start[cell_of(r) + 1]++;
        for (int k = 0; k < ncell; k++) start[k + 1] += start[k];
        std::vector<float4> sorted(c->h_rec.size());
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (const float4& r : c->h_rec) sorted[fill[cell_of(r)]++] = r;
        c->d_rec_cells.upload(sorted.data(), sorted.size(), c->stream);
        c->d_cell_start.upload(start.data(), start.size(), c->stream);
        ck(cudaStreamSynchronize(c->stream), "receptor upload");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_receptor_count(const ud_ctx* c) { return c ? (int)c->h_rec.size() : 0; }

int ud_build_grid(ud_ctx* c, float spacing, int nmaps, const int* map_types, int precision) {
    try {
        if (!c || spacing <= 0.f || nmaps <= 0 || nmaps > MAX_MAPS || !map_types)
            throw Fail(UD_EINVAL, "invalid grid arguments (1..20 maps, spacing > 0)");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        MapTypes mt;
        mt.n = nmaps;
        for (int i = 0; i < NT + 3; i++) c->map_of_type[i] = -1;
        for (int m = 0; m < nmaps; m++) {
            if (map_types[m] <= 0 || map_types[m] >= NT) throw Fail(UD_EINVAL, "map type out of range");
            mt.t[m] = map_types[m];
            c->map_of_type[map_types[m]] = (signed char)m;
        }
        for (int a = 0; a < 3; a++) {
            c->origin[a] = c->box_lo[a];
            c->gdim[a] = (int)ceilf((c->box_hi[a] - c->box_lo[a]) / spacing - 1e-4f) + 1;
            if (c->gdim[a] < 2) c->gdim[a] = 2;
        }
        c->spacing = spacing;
        c->nmaps = nmaps;
        c->ligs_dirty = true;          // map slots of loaded ligands change
        long long npt = (long long)c->gdim[0] * c->gdim[1] * c->gdim[2];
        if (npt * nmaps >= (1LL << 31))
            throw Fail(UD_EINVAL, "grid too large: the maps must hold fewer than 2^31 values (larger spacing or box)");
        c->d_maps32.ensure((size_t)npt * nmaps);
        c->d_maps16.ensure((size_t)npt * nmaps);
        int threads = 256;
        long long blocks = (npt + threads - 1) / threads;
        k_grid_build<<<(unsigned)blocks, threads, 0, c->stream>>>(c->d_rec.p, (int)c->h_rec.size(), mt, c->origin[0],
                                                                  c->origin[1], c->origin[2], spacing, c->gdim[0],
                                                                  c->gdim[1], c->gdim[2], c->d_maps32.p, c->d_maps16.p);
        ck(cudaGetLastError(), "k_grid_build launch");
        ck(cudaStreamSynchronize(c->stream), "k_grid_build");
        c->grid_prec = precision == UD_GRID_F16 ? UD_GRID_F16 : UD_GRID_F32;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_set_grid_precision(ud_ctx* c, int precision) {
    if (!c) { g_err = "null context"; return UD_EINVAL; }
    c->grid_prec = precision == UD_GRID_F16 ? UD_GRID_F16 : UD_GRID_F32;
    return UD_OK;
}

int ud_get_grid(const ud_ctx* c, float* out, int* gdim3, float* origin3) {
    try {
        if (!c || c->nmaps == 0) throw Fail(UD_ESTATE, "no grid built");
        if (gdim3) for (int a = 0; a < 3; a++) gdim3[a] = c->gdim[a];
        if (origin3) for (int a = 0; a < 3; a++) origin3[a] = c->origin[a];
        if (out) {
            ck(cudaSetDevice(c->device), "cudaSetDevice");
            size_t n = (size_t)c->gdim[0] * c->gdim[1] * c->gdim[2] * c->nmaps;
            ck(cudaMemcpy(out, c->d_maps32.p, n * sizeof(float), cudaMemcpyDeviceToHost), "grid D2H");
        }
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_add_ligands(ud_ctx* c, int nlig, const int* atom_off, const float* xyz, const int* types, const int* tors_off,
                   const int* axis, const float* dihedrals, const int* range_off, const float* ranges,
                   const int* rot_off, const int* rot_atoms, const int* pair_off, const int* pairs,
                   const int* bias_off, const float* bias) {
    try {
        if (!c || nlig < 0 || !atom_off || !tors_off || !range_off || !rot_off || !pair_off)
            throw Fail(UD_EINVAL, "invalid ligand arguments");
        for (int l = 0; l < nlig; l++) {
            int a0 = atom_off[l], n = atom_off[l + 1] - a0;
            int t0 = tors_off[l], T = tors_off[l + 1] - t0;
            if (n <= 0 || T < 0) throw Fail(UD_EINVAL, "ligand with no atoms");
            if (n > 4096 || T > 256) throw Fail(UD_EINVAL, "ligand too large (max 4096 atoms, 256 torsions)");
            int nheavy = 0;
            for (int i = 0; i < n; i++) {
                int t = types[a0 + i];
                if (t < 0 || t >= NT) throw Fail(UD_EINVAL, "ligand atom type out of range");
                nheavy += t != VN_H;
            }
            int p0 = pair_off[a0], np = pair_off[a0 + n] - p0;
            int r0 = rot_off[t0], nrot = rot_off[t0 + T] - r0;
            int g0 = range_off[t0], nrange = range_off[t0 + T] - g0;
            int b0 = bias_off ? bias_off[a0] : 0, nb = bias_off ? bias_off[a0 + n] - b0 : 0;
            std::vector<int> blob(H_WORDS, 0);
            auto put = [&](int hdr, int count) {
                blob[hdr] = (int)blob.size();
                blob.resize(blob.size() + ((count + 3) & ~3), 0);
                return blob[hdr];
            };
            blob[H_NATOM] = n; blob[H_NTORS] = T; blob[H_NHEAVY] = nheavy; blob[H_NPAIR] = np;
            blob[H_NROT] = nrot; blob[H_NRANGE] = nrange; blob[H_NBIAS] = nb;
            int o;
            o = put(H_TYPES, n);
            for (int i = 0; i < n; i++) blob[o + i] = types[a0 + i];
            o = put(H_AXIS, 2 * T);
            for (int k = 0; k < 2 * T; k++) {
                int v = axis[2 * t0 + k];
                if (v < 0 || v >= n) throw Fail(UD_EINVAL, "torsion axis atom out of range");
                blob[o + k] = v;
            }
            o = put(H_RANGE_OFF, T + 1);
            for (int k = 0; k <= T; k++) blob[o + k] = range_off[t0 + k] - g0;
            for (int k = 0; k < T; k++)
                if (range_off[t0 + k + 1] - range_off[t0 + k] <= 0) throw Fail(UD_EINVAL, "torsion without range");
            o = put(H_RANGES, 2 * nrange);
            memcpy(&blob[o], ranges + 2 * (size_t)g0, sizeof(float) * 2 * nrange);
            o = put(H_ROT_OFF, T + 1);
            for (int k = 0; k <= T; k++) blob[o + k] = rot_off[t0 + k] - r0;
            o = put(H_ROT, nrot);
            for (int k = 0; k < nrot; k++) {
                int v = rot_atoms[r0 + k];
                if (v < 0 || v >= n) throw Fail(UD_EINVAL, "rotated atom out of range");
                blob[o + k] = v;
            }
            o = put(H_BIAS_OFF, n + 1);
            for (int i = 0; i <= n; i++) blob[o + i] = bias_off ? bias_off[a0 + i] - b0 : 0;
            o = put(H_BIAS, 5 * nb);
            if (nb) memcpy(&blob[o], bias + 5 * (size_t)b0, sizeof(float) * 5 * nb);
            o = put(H_HEAVY, nheavy);
            for (int i = 0, k = 0; i < n; i++) if (types[a0 + i] != VN_H) blob[o + k++] = i;
            o = put(H_X0, 3 * n);
            memcpy(&blob[o], xyz + 3 * (size_t)a0, sizeof(float) * 3 * n);
            o = put(H_D0, T);
            if (T) memcpy(&blob[o], dihedrals + t0, sizeof(float) * T);
            o = put(H_C0, 3);
            {   // centre = float mean of the input coordinates (rapidjson_parser.cpp:67-83,197-199)
                float s[3] = {0.f, 0.f, 0.f};
                for (int i = 0; i < n; i++)
                    for (int a = 0; a < 3; a++) s[a] += xyz[3 * (size_t)(a0 + i) + a];
                float cc[3] = {s[0] / n, s[1] / n, s[2] / n};
                memcpy(&blob[o], cc, sizeof(cc));
            }
            o = put(H_RADII, n);
            for (int i = 0; i < n; i++) {
                const float r = kVdwHost[types[a0 + i]];
                memcpy(&blob[o + i], &r, sizeof(float));
            }
            {   // heavy rotated atoms per torsion, in the reference's loop order
                std::vector<int> rh_off(T + 1, 0), rh;
                for (int k = 0; k < T; k++) {
                    for (int q = rot_off[t0 + k]; q < rot_off[t0 + k + 1]; q++) {
                        const int a = rot_atoms[q];
                        if (types[a0 + a] != VN_H) rh.push_back(a);
                    }
                    rh_off[k + 1] = (int)rh.size();
                }
                o = put(H_RHOFF, T + 1);
                for (int k = 0; k <= T; k++) blob[o + k] = rh_off[k];
                o = put(H_RHEAVY, (int)rh.size());
                for (size_t q = 0; q < rh.size(); q++) blob[o + q] = rh[q];
            }
            o = put(H_MAPIDX, n);      // filled from the current grid at upload (sync_ligs)
            for (int i = 0; i < n; i++) blob[o + i] = -1;
            {   // heavy scored pairs, once each (i < j), for the intra kernels, in round-robin
                // order (pair (a, a+t mod n) for t = 1..n/2) so that 32 consecutive pairs touch
                // each atom about twice (fewer shared-memory bank conflicts in pass 1)
                std::vector<char> scored((size_t)n * n, 0);
                for (int i = 0; i < n; i++)
                    for (int k = pair_off[a0 + i] - p0; k < pair_off[a0 + i + 1] - p0; k++) {
                        const int v = pairs[p0 + k];
                        if (v < 0 || v >= n) throw Fail(UD_EINVAL, "intra pair atom out of range");
                        scored[(size_t)i * n + v] = 1;
                    }
                std::vector<int> rec;
                for (int t = 1; t <= n / 2; t++)
                    for (int a = 0; a < n; a++) {
                        if (2 * t == n && a >= t) break;
                        const int i = std::min(a, (a + t) % n), j = std::max(a, (a + t) % n);
                        if (!scored[(size_t)i * n + j] && !scored[(size_t)j * n + i]) continue;
                        const int ti = types[a0 + i], tj = types[a0 + j];
                        if (ti == VN_H || tj == VN_H) continue;
                        const unsigned b1 = 1u << ti, b2 = 1u << tj;
                        int w0 = i | (j << 12);
                        if ((b1 & HYD_MASK) && (b2 & HYD_MASK)) w0 |= PREC_HYD;
                        if (((b1 & ACC_MASK) && (b2 & DON_MASK)) || ((b1 & DON_MASK) && (b2 & ACC_MASK))) w0 |= PREC_HB;
                        const float rs = kVdwHost[ti] + kVdwHost[tj];
                        int w1;
                        memcpy(&w1, &rs, sizeof(w1));
                        rec.push_back(w0);
                        rec.push_back(w1);
                    }
                const int np2 = (int)rec.size() / 2;
                if (np2 > 0xFFFF) throw Fail(UD_EINVAL, "too many intra pairs (max 65535)");
                blob[H_NPREC] = np2;
                // sections the search reads come first: the pair list and gather lists, then
                // the adjacency only the final scoring reads (not staged)
                o = put(H_PREC, (int)rec.size());
                for (size_t q = 0; q < rec.size(); q++) blob[o + q] = rec[q];
                // gather lists: for each atom, (pair index, partner) in pair-index order
                std::vector<std::vector<int>> g(n);
                for (int p = 0; p < np2; p++) {
                    const int i = rec[2 * p] & 0xFFF, j = (rec[2 * p] >> 12) & 0xFFF;
                    g[i].push_back(p | (j << 16));
                    g[j].push_back(p | (i << 16));
                }
                o = put(H_GOFF, n + 1);
                int acc = 0;
                for (int i = 0; i < n; i++) { blob[o + i] = acc; acc += (int)g[i].size(); }
                blob[o + n] = acc;
                o = put(H_GADJ, acc);
                for (int i = 0, k = 0; i < n; i++)
                    for (int v : g[i]) blob[o + k++] = v;
                blob[H_STAGE] = (int)blob.size();
            }
            o = put(H_PAIR_OFF, n + 1);
            for (int i = 0; i <= n; i++) blob[o + i] = pair_off[a0 + i] - p0;
            o = put(H_PAIRS, np);
            for (int i = 0; i < n; i++) {
                const int ti = types[a0 + i];
                for (int k = pair_off[a0 + i] - p0; k < pair_off[a0 + i + 1] - p0; k++) {
                    const int v = pairs[p0 + k];
                    const int tj = types[a0 + v];
                    const unsigned b1 = 1u << ti, b2 = 1u << tj;
                    int ent = v;
                    if (ti == VN_H || tj == VN_H) ent |= PAIR_ZERO;
                    if ((b1 & HYD_MASK) && (b2 & HYD_MASK)) ent |= PAIR_HYD;
                    if (((b1 & ACC_MASK) && (b2 & DON_MASK)) || ((b1 & DON_MASK) && (b2 & ACC_MASK))) ent |= PAIR_HB;
                    blob[o + k] = ent;
                }
            }
            {   // rigid frame for recorded moves: three non-collinear atoms of the root fragment
                std::vector<char> moved(n, 0);
                for (int q = r0; q < r0 + nrot; q++) moved[rot_atoms[q]] = 1;
                auto X = [&](int a, int k) { return (double)xyz[3 * (size_t)(a0 + a) + k]; };
                int f0 = -1, f1 = -1, f2 = -1;
                for (int i = 0; i < n && f0 < 0; i++) if (!moved[i]) f0 = i;
                double best = 0.0;
                for (int i = 0; i < n && f0 >= 0; i++) {
                    if (moved[i] || i == f0) continue;
                    double d2 = 0.0;
                    for (int k = 0; k < 3; k++) d2 += (X(i, k) - X(f0, k)) * (X(i, k) - X(f0, k));
                    if (d2 > best) { best = d2; f1 = i; }
                }
                best = 0.0;
                for (int i = 0; i < n && f1 >= 0; i++) {
                    if (moved[i] || i == f0 || i == f1) continue;
                    double u[3], w[3];
                    for (int k = 0; k < 3; k++) { u[k] = X(f1, k) - X(f0, k); w[k] = X(i, k) - X(f0, k); }
                    const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
                    const double a2 = cx * cx + cy * cy + cz * cz;
                    if (a2 > best) { best = a2; f2 = i; }
                }
                if (f2 < 0 || best < 0.01) f0 = f1 = f2 = -1;       // no rigid frame
                blob[H_FRAME0] = f0; blob[H_FRAME0 + 1] = f1; blob[H_FRAME0 + 2] = f2;
            }
            blob[H_TOTAL] = (int)blob.size();
            LigHost h;
            h.natom = n; h.ntors = T; h.nheavy = nheavy;
            h.blob_words = (int)blob.size();
            h.stage_words = blob[H_STAGE];
            h.blob_off = (long long)c->h_blobs.size();
            h.stride = rec_floats(n, T);
            h.nprec = blob[H_NPREC];
            c->h_blobs.insert(c->h_blobs.end(), blob.begin(), blob.end());
            c->h_ligs.push_back(h);
            c->max_natom = std::max(c->max_natom, n);
            c->max_ntors = std::max(c->max_ntors, T);
            c->max_blob = std::max(c->max_blob, h.blob_words);
            c->max_stage = std::max(c->max_stage, h.stage_words);
        }
        c->ligs_dirty = true;
        c->has_results = false;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_clear_ligands(ud_ctx* c) {
    if (!c) { g_err = "null context"; return UD_EINVAL; }
    c->h_blobs.clear();
    c->h_ligs.clear();
    c->h_ligdev.clear();
    c->max_natom = c->max_ntors = c->max_blob = c->max_stage = 0;
    c->ligs_dirty = true;
    c->has_results = false;
    c->nchain = 0;
    return UD_OK;
}

int ud_ligand_count(const ud_ctx* c) { return c ? (int)c->h_ligs.size() : 0; }

int ud_record_floats(const ud_ctx* c, int lig) {
    if (!c || lig < 0 || lig >= (int)c->h_ligs.size()) { g_err = "invalid ligand index"; return UD_EINVAL; }
    return c->h_ligs[lig].stride;
}

int ud_score_batch(ud_ctx* c, int n, const int* pose_lig, const float* coords, const float* centers,
                   const float* rotvecs, int mode, float vcap, float slope, float* out_e, float* out_g) {
    try {
        if (!c || n < 0 || (n > 0 && (!pose_lig || !coords || !centers || !rotvecs || !out_e || !out_g)))
            throw Fail(UD_EINVAL, "invalid score arguments");
        if (n == 0) return UD_OK;
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        sync_ligs(c);
        Env env = make_env(c, mode);
        std::vector<long long> xoff(n), goff(n);
        long long xs = 0, gs = 0;
        int wsm = 0;
        for (int i = 0; i < n; i++) {
            int l = pose_lig[i];
            if (l < 0 || l >= (int)c->h_ligs.size()) throw Fail(UD_EINVAL, "pose ligand index out of range");
            xoff[i] = xs;
            goff[i] = gs;
            xs += 3LL * c->h_ligs[l].natom;
            gs += 6 + c->h_ligs[l].ntors;
            wsm = std::max(wsm, lig_ws(c->h_ligs[l]));
        }
        DBuf<int> dl; DBuf<long long> dxo, dgo; DBuf<float> dx, dc, dr, de, dg;
        dl.upload(pose_lig, n, c->stream);
        dxo.upload(xoff.data(), n, c->stream);
        dgo.upload(goff.data(), n, c->stream);
        dx.upload(coords, xs, c->stream);
        dc.upload(centers, 3 * (size_t)n, c->stream);
        dr.upload(rotvecs, 3 * (size_t)n, c->stream);
        de.ensure(n);
        dg.ensure(gs);
        int W = pick_warps(c, wsm, 0, 8);
        size_t smem = (size_t)W * wsm * 4;
        const auto ks = score_kernel(env);
        set_smem(ks, smem);
        PoseIO io{dl.p, dxo.p, dx.p, dc.p, dr.p, dgo.p};
        ks<<<(n + W - 1) / W, 32 * W, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, io, env, vcap, slope, wsm,
                                                              de.p, dg.p);
        ck(cudaGetLastError(), "k_score launch");
        ck(cudaMemcpyAsync(out_e, de.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaMemcpyAsync(out_g, dg.p, gs * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "k_score");
        for (auto* b : {&dx, &dc, &dr, &de, &dg}) b->release();
        dl.release(); dxo.release(); dgo.release();
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_read_bandwidth(int device, long long bytes, int repeats, float* out_gbps) {
    try {
        if (bytes < (1 << 20) || repeats < 1 || !out_gbps) throw Fail(UD_EINVAL, "invalid probe arguments");
        ck(cudaSetDevice(device), "cudaSetDevice");
        int nsm = 0;
        ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device), "attribute");
        const long long n4 = bytes / 16;
        const int grid = nsm * 4;
        DBuf<float4> buf;
        DBuf<float> part;
        buf.ensure((size_t)n4);
        part.ensure((size_t)grid);
        cudaStream_t st;
        ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        ck(cudaMemsetAsync(buf.p, 0, (size_t)n4 * 16, st), "memset");
        ck(cudaMemsetAsync(part.p, 0, (size_t)grid * 4, st), "memset");
        // enough passes per launch that a launch reads at least 1 GiB (launch overhead negligible)
        const int passes = (int)std::max<long long>(1, (1LL << 30) / ((long long)n4 * 16));
        for (int w = 0; w < 3; w++) k_read_probe<<<grid, 512, 0, st>>>(buf.p, n4, passes, part.p);
        ck(cudaEventRecord(e0, st), "event");
        for (int r = 0; r < repeats; r++) k_read_probe<<<grid, 512, 0, st>>>(buf.p, n4, passes, part.p);
        ck(cudaEventRecord(e1, st), "event");
        ck(cudaGetLastError(), "k_read_probe launch");
        ck(cudaEventSynchronize(e1), "probe");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(st);
        *out_gbps = (float)((double)n4 * 16.0 * passes * repeats / (ms * 1e-3) / 1e9);
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_score_batch_timed(ud_ctx* c, int n, const int* pose_lig, const float* coords, const float* centers,
                         const float* rotvecs, int mode, float vcap, float slope, int repeats, float* out_e,
                         float* out_g, float* out_ms) {
    try {
        if (!c || n <= 0 || repeats < 1 || !pose_lig || !coords || !centers || !rotvecs || !out_e || !out_g || !out_ms)
            throw Fail(UD_EINVAL, "invalid score arguments");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        sync_ligs(c);
        Env env = make_env(c, mode);
        std::vector<long long> xoff(n), goff(n);
        long long xs = 0, gs = 0;
        int wsm = 0;
        for (int i = 0; i < n; i++) {
            int l = pose_lig[i];
            if (l < 0 || l >= (int)c->h_ligs.size()) throw Fail(UD_EINVAL, "pose ligand index out of range");
            xoff[i] = xs;
            goff[i] = gs;
            xs += 3LL * c->h_ligs[l].natom;
            gs += 6 + c->h_ligs[l].ntors;
            wsm = std::max(wsm, lig_ws(c->h_ligs[l]));
        }
        DBuf<int> dl; DBuf<long long> dxo, dgo; DBuf<float> dx, dc, dr, de, dg;
        dl.upload(pose_lig, n, c->stream);
        dxo.upload(xoff.data(), n, c->stream);
        dgo.upload(goff.data(), n, c->stream);
        dx.upload(coords, xs, c->stream);
        dc.upload(centers, 3 * (size_t)n, c->stream);
        dr.upload(rotvecs, 3 * (size_t)n, c->stream);
        de.ensure(n);
        dg.ensure(gs);
        int W = pick_warps(c, wsm, 0, 8);
        size_t smem = (size_t)W * wsm * 4;
        const auto ks = score_kernel(env);
        set_smem(ks, smem);
        PoseIO io{dl.p, dxo.p, dx.p, dc.p, dr.p, dgo.p};
        const unsigned grid = (unsigned)((n + W - 1) / W);
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        ks<<<grid, 32 * W, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, io, env, vcap, slope, wsm, de.p, dg.p);
        ck(cudaEventRecord(e0, c->stream), "event");
        for (int r = 0; r < repeats; r++)
            ks<<<grid, 32 * W, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, io, env, vcap, slope, wsm, de.p,
                                                       dg.p);
        ck(cudaEventRecord(e1, c->stream), "event");
        ck(cudaGetLastError(), "k_score launch");
        ck(cudaEventSynchronize(e1), "k_score");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *out_ms = ms / repeats;
        ck(cudaMemcpyAsync(out_e, de.p, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaMemcpyAsync(out_g, dg.p, gs * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "k_score");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_score_terms(ud_ctx* c, int n, const int* pose_lig, const float* coords, int mode, float* out4,
                   float* out_decomp) {
    try {
        if (!c || n < 0 || (n > 0 && (!pose_lig || !coords || !out4))) throw Fail(UD_EINVAL, "invalid arguments");
        if (n == 0) return UD_OK;
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        sync_ligs(c);
        Env env = make_env(c, mode);
        std::vector<long long> xoff(n), doff(n);
        long long xs = 0, ds = 0;
        for (int i = 0; i < n; i++) {
            int l = pose_lig[i];
            if (l < 0 || l >= (int)c->h_ligs.size()) throw Fail(UD_EINVAL, "pose ligand index out of range");
            xoff[i] = xs;
            doff[i] = ds;
            xs += 3LL * c->h_ligs[l].natom;
            ds += 5LL * c->h_ligs[l].natom;
        }
        DBuf<int> dl; DBuf<long long> dxo, ddo; DBuf<float> dx, d4, dd;
        dl.upload(pose_lig, n, c->stream);
        dxo.upload(xoff.data(), n, c->stream);
        ddo.upload(doff.data(), n, c->stream);
        dx.upload(coords, xs, c->stream);
        d4.ensure(4 * (size_t)n);
        if (out_decomp) dd.ensure(ds);
        int W = 8;
        k_terms<<<(n + W - 1) / W, 32 * W, 0, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, dl.p, dxo.p, dx.p, env, d4.p,
                                                           out_decomp ? dd.p : nullptr, ddo.p);
        ck(cudaGetLastError(), "k_terms launch");
        ck(cudaMemcpyAsync(out4, d4.p, 4 * n * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        if (out_decomp)
            ck(cudaMemcpyAsync(out_decomp, dd.p, ds * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "k_terms");
        dl.release(); dxo.release(); ddo.release(); dx.release(); d4.release(); dd.release();
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_bfgs_batch(ud_ctx* c, int n, const int* pose_lig, float* records, int max_steps, int rounds, float vcap,
                  float slope0, int ramp, int mode, int* out_nevals) {
    try {
        if (!c || n < 0 || (n > 0 && (!pose_lig || !records)) || max_steps < 0 || rounds < 0)
            throw Fail(UD_EINVAL, "invalid bfgs arguments");
        if (n == 0) return UD_OK;
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        sync_ligs(c);
        Env env = make_env(c, mode);
        std::vector<long long> off(n);
        long long tot = 0;
        int wsm = 0;
        for (int i = 0; i < n; i++) {
            int l = pose_lig[i];
            if (l < 0 || l >= (int)c->h_ligs.size()) throw Fail(UD_EINVAL, "pose ligand index out of range");
            off[i] = tot;
            tot += c->h_ligs[l].stride;
            wsm = std::max(wsm, lig_ws(c->h_ligs[l]));
        }
        // records are packed at 8+3N+T floats each on the host side
        std::vector<float> packed(tot, 0.f);
        long long hs = 0;
        for (int i = 0; i < n; i++) {
            const LigHost& h = c->h_ligs[pose_lig[i]];
            int nr = 8 + 3 * h.natom + h.ntors;
            memcpy(&packed[off[i]], records + hs, nr * sizeof(float));
            hs += nr;
        }
        DBuf<int> dl, dn; DBuf<long long> dof; DBuf<float> dr;
        dl.upload(pose_lig, n, c->stream);
        dof.upload(off.data(), n, c->stream);
        dr.upload(packed.data(), tot, c->stream);
        dn.ensure(n);
        int W = pick_warps(c, wsm, 0, 8);
        size_t smem = (size_t)W * wsm * 4;
        const auto kb = bfgs_kernel(env);
        set_smem(kb, smem);
        kb<<<(n + W - 1) / W, 32 * W, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, dl.p, dof.p, dr.p, env,
                                                             max_steps, rounds, vcap, slope0, ramp, wsm, dn.p);
        ck(cudaGetLastError(), "k_bfgs launch");
        ck(cudaMemcpyAsync(packed.data(), dr.p, tot * sizeof(float), cudaMemcpyDeviceToHost, c->stream), "D2H");
        if (out_nevals) ck(cudaMemcpyAsync(out_nevals, dn.p, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "k_bfgs");
        hs = 0;
        for (int i = 0; i < n; i++) {
            const LigHost& h = c->h_ligs[pose_lig[i]];
            int nr = 8 + 3 * h.natom + h.ntors;
            memcpy(records + hs, &packed[off[i]], nr * sizeof(float));
            hs += nr;
        }
        dl.release(); dn.release(); dof.release(); dr.release();
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

// Layout and launch shape of a chain search over the loaded ligands: chain records
// ligand-major (best_off), warps per CTA and shared memory for the largest ligand, the
// register budget the shared memory allows, and the work items (ligand, first chain,
// count) in descending ligand cost, uploaded with the work counter cleared.
struct SearchPlan {
    int W = 0, grid = 0, nitems = 0, wsm = 0, blob_max = 0;
    int minb = 3;          // instantiation: 3 or 4 (256-thread bound), 2 (384-thread bound)
    size_t smem = 0;
    long long tot = 0;
};

extern "C++" {
template <typename K>
static SearchPlan plan_search(ud_ctx* c, int nchain, K k3, K k4, K k12, int want_w = 0, int force_k = 0) {
    SearchPlan P;
    const int nlig = (int)c->h_ligs.size();
    std::vector<int> order(nlig);
    std::vector<double> cost(nlig);
    for (int l = 0; l < nlig; l++) {
        const LigHost& h = c->h_ligs[l];
        c->h_ligdev[l].best_off = P.tot;
        P.tot += (long long)nchain * c->retain * h.stride;
        P.wsm = std::max(P.wsm, lig_ws(h));
        order[l] = l;
        // evaluation cost ~ intra pairs + grid atoms + kinematics, times BFGS length
        const double np = (double)(c->h_blobs[h.blob_off + H_NPAIR]);
        cost[l] = (np + 8.0 * h.natom + 40.0 * h.ntors + 200.0) * (6 + h.ntors);
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    P.blob_max = r4(c->max_stage);
    int smem_sm = 0;
    ck(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device), "attribute");
    const long long lim = smem_limit(c) / 4 - 64;       // floats of one CTA's shared memory
    // CTA widths 8, 12 and 4 warps (want_w > 0: that one only): per width the instantiation
    // its shared memory allows (64 registers only where that reaches 32 warps per SM; 1 KB
    // per CTA is reserved by the runtime), kept if it holds the most warps resident
    int per_sm = 0;
    K chosen = k3;
    for (int w : {8, 12, 4}) {
        if (want_w > 0 && w != want_w) continue;
        if ((long long)P.blob_max + (long long)w * P.wsm > lim) continue;
        const size_t smem = ((size_t)P.blob_max + (size_t)w * P.wsm) * 4;
        const int by_smem = (int)((size_t)smem_sm / (smem + 1024));
        const int minb = w == 12 ? 2 : (by_smem * w >= 32 ? 4 : 3);
        K kern = minb == 2 ? k12 : (minb == 4 ? k4 : k3);
        set_smem(kern, smem);
        int n = 0;
        ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 32 * w, smem), "occupancy");
        if (n * w > per_sm * P.W) { P.W = w; P.minb = minb; P.smem = smem; per_sm = n; chosen = kern; }
    }
    if (P.W == 0) {                                    // a ligand too large for 4 warps per CTA
        P.W = pick_warps(c, P.wsm, P.blob_max, 4);
        P.minb = 3;
        P.smem = ((size_t)P.blob_max + (size_t)P.W * P.wsm) * 4;
        chosen = k3;
        set_smem(k3, P.smem);
        ck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k3, 32 * P.W, P.smem), "occupancy");
    }
    set_smem(chosen, P.smem);      // the candidates may have set a smaller size on the same kernel
    if (per_sm < 1) per_sm = 1;
    const long long resident = (long long)c->nsm * per_sm;
    // k chains per warp per item (W*k chains; the warps of a CTA share an item's chains
    // dynamically): one by default.  Larger items shorten the wait at an item's end relative
    // to its length but lengthen the launch's tail; on a 148-ligand screen batch (12-warp
    // CTAs, 400 MC steps) the search took 5.65 s at k = 1, 5.81 s at 2, 5.9-6.1 s at 3 and
    // 5.8-6.3 s at 4.  The autotuner and ud_set_packing can choose others.
    const long long total_chains = (long long)nlig * nchain;
    const int k = force_k > 0 ? force_k : 1;
    const int item_chains = P.W * k;
    std::vector<int4> items;
    for (int l : order)
        for (int c0 = 0; c0 < nchain; c0 += item_chains)
            items.push_back(make_int4(l, c0, std::min(item_chains, nchain - c0), 0));
    upload_ligdev(c);
    c->d_items.upload(items.data(), items.size(), c->stream);
    P.nitems = (int)items.size();
    P.grid = (int)std::min((long long)P.nitems, resident);
    c->shape[0] = P.W; c->shape[1] = per_sm; c->shape[2] = P.minb; c->shape[3] = k;
    c->d_counter.ensure(1);
    c->d_nevals.ensure(3);          // evaluations, heavy-atom evaluations, staging timeouts
    ck(cudaMemsetAsync(c->d_counter.p, 0, sizeof(int), c->stream), "memset");
    ck(cudaMemsetAsync(c->d_nevals.p, 0, 3 * sizeof(unsigned long long), c->stream), "memset");
    c->counters[3] = total_chains;
    return P;
}
}  // extern "C++"

using SearchKernel = void (*)(const int*, const LigDev*, const int4*, int, Env, SearchP, float*, int*,
                              unsigned long long*);
// the k_search instantiation of a plan (minb 3, 4: 256-thread bound; 2: 384-thread bound)
static SearchKernel search_kernel(int minb, int rmax) {
    if (rmax > 1) return minb == 4 ? k_search<4, 4> : (minb == 2 ? k_search<2, 4, 384> : k_search<3, 4>);
    return minb == 4 ? k_search<4, 1> : (minb == 2 ? k_search<2, 1, 384> : k_search<3, 1>);
}
static SearchPlan plan_fused(ud_ctx* c, int nchain, int want_w = 0, int force_k = 0) {
    const int r = c->retain;
    return plan_search(c, nchain, search_kernel(3, r), search_kernel(4, r), search_kernel(2, r), want_w, force_k);
}

static void run_search_plan(ud_ctx* c, const SearchPlan& P, const Env& env, uint64_t seed, int nchain, int mc_steps,
                            int opt_steps, int randomize) {
    SearchP sp;
    sp.k0 = (uint32_t)seed;
    sp.k1 = (uint32_t)(seed >> 32) ^ 0x5DEECE66u;
    sp.nchain = nchain;
    sp.mc_steps = mc_steps;
    sp.opt_steps = opt_steps;
    sp.randomize = randomize;
    sp.retain = c->retain;
    sp.ws_max = P.wsm;
    sp.blob_max = P.blob_max;
    if (P.grid > 0) {
        const SearchKernel kern = search_kernel(P.minb, c->retain);
        kern<<<P.grid, 32 * P.W, P.smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, c->d_items.p, P.nitems, env, sp,
                                                      c->d_best.p, c->d_counter.p, c->d_nevals.p);
        ck(cudaGetLastError(), "k_search launch");
        c->counters[2]++;
    }
}

// Chain packing autotuner: warps per CTA (8, 12 or 4) and chains per warp per work item
// (1, 2 or 4), each timed with CUDA events on a short search of the batch itself
// (3 MC steps); the fastest is kept for batches of the same shape.  A chain's result does
// not depend on the packing (its random stream is indexed by chain, ligand and step).
static void autotune_search(ud_ctx* c, const Env& env, uint64_t seed, int nchain, int opt_steps, int randomize) {
    const long long key = (long long)c->h_ligs.size() * 1000003LL + (long long)nchain * 131LL + c->max_stage * 7LL +
                          c->retain;
    if (c->tune_key == key) return;
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    float best_ms = 1e30f;
    int best_w = 8, best_k = 0;
    for (int w : {8, 12, 4})
        for (int k : {1, 2, 4}) {
            const SearchPlan P = plan_fused(c, nchain, w, k);
            c->d_best.ensure((size_t)P.tot);
            ck(cudaEventRecord(e0, c->stream), "event");
            run_search_plan(c, P, env, seed, nchain, 3, opt_steps, randomize);
            ck(cudaEventRecord(e1, c->stream), "event");
            ck(cudaEventSynchronize(e1), "autotune");
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
            if (ms < best_ms) { best_ms = ms; best_w = w; best_k = k; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tune_key = key;
    c->tune_w = best_w;
    c->tune_k = best_k;
}

static void launch_search(ud_ctx* c, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, int mode) {
    sync_ligs(c);
    Env env = make_env(c, mode);
    c->nchain = nchain * c->retain;                  // records per ligand
    if (c->autotune && !(c->pack_w || c->pack_k)) autotune_search(c, env, seed, nchain, opt_steps, randomize);
    const SearchPlan P = (c->pack_w || c->pack_k) ? plan_fused(c, nchain, c->pack_w, c->pack_k)
                         : c->autotune         ? plan_fused(c, nchain, c->tune_w, c->tune_k)
                                               : plan_fused(c, nchain);
    c->best_floats = P.tot;
    c->d_best.ensure((size_t)P.tot);
    run_search_plan(c, P, env, seed, nchain, mc_steps, opt_steps, randomize);
}

// The learned-proposal search (and, with record, the collection of accepted moves): one
// CUDA graph per block of K MC steps, replayed ceil(mc_steps / K) times.
static void launch_learned(ud_ctx* c, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, int mode,
                           float p_learned, int record_max, int target = 0) {
    if (mc_steps < 1) throw Fail(UD_EINVAL, "the learned search needs mc_steps >= 1");
    if (p_learned < 0.f || p_learned > 1.f) throw Fail(UD_EINVAL, "p_learned must be in [0, 1]");
    if (p_learned > 0.f && !c->mlp.ready)
        throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init, ud_mlp_set_params or train one");
    if (mode != UD_MODE_GRID) throw Fail(UD_EINVAL, "the learned search scores on the grid maps");
    sync_ligs(c);
    Env env = make_env(c, mode);
    c->nchain = nchain * c->retain;                  // records per ligand
    const int nlig = (int)c->h_ligs.size();
    const long long nch = (long long)nlig * nchain;
    for (const LigHost& h : c->h_ligs)
        if (h.natom > mlp::NATOM || h.ntors > mlp::TMAX)
            throw Fail(UD_EINVAL, "the proposal network covers ligands of at most 80 atoms and 20 torsions");
    // two chains per warp per work item unless fixed: a launch runs a block of a few MC steps
    // of every chain, whose lengths vary far more than those of whole chains, and sharing an
    // item's chains among its warps evens them out (148-ligand screen batch, 200 steps,
    // p_learned 0.25, blocks of 4 steps: 1683 ms at k = 2, 1718 at 1, 1808 at 4)
    const int lk = c->pack_k ? c->pack_k : 2;
    const SearchPlan P = c->retain > 1
                             ? plan_search(c, nchain, k_learn_step<3, 4>, k_learn_step<4, 4>, k_learn_step<2, 4, 384>,
                                           c->pack_w, lk)
                             : plan_search(c, nchain, k_learn_step<3, 1>, k_learn_step<4, 1>, k_learn_step<2, 1, 384>,
                                           c->pack_w, lk);
    c->best_floats = P.tot;
    c->d_best.ensure((size_t)P.tot);
    c->d_acc.ensure((size_t)P.tot);
    const bool feats = p_learned > 0.f || record_max > 0;
    if (feats) c->d_x16.ensure((size_t)nch * mlp::IN);
    if (p_learned > 0.f) {
        c->mlp.ensure((int)nch);
        c->mlp.prepare(c->stream);                  // nothing may allocate inside the capture
    }
    MoveSet ms{nullptr, nullptr, nullptr, nullptr, 0, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (record_max > 0) {
        c->d_mx.ensure((size_t)record_max * mlp::IN);
        c->d_my.ensure((size_t)record_max * mlp::NDIM);
        c->d_mm.ensure((size_t)record_max * mlp::NDIM);
        c->d_mcount.ensure(1);
        if (target == 1) {
            c->d_maux.ensure((size_t)record_max * AUX);
            c->d_mchain.ensure((size_t)record_max);
        }
        c->d_sflag.ensure((size_t)nch);
        c->d_spos.ensure((size_t)nch);
        c->d_sy.ensure((size_t)nch * (target == 1 ? AUX : mlp::NDIM));
        if (target == 0) c->d_sm.ensure((size_t)nch * mlp::NDIM);
        ck(cudaMemsetAsync(c->d_mcount.p, 0, sizeof(int), c->stream), "memset");
        ck(cudaMemsetAsync(c->d_sflag.p, 0, sizeof(int) * (size_t)nch, c->stream), "memset");
        ms = MoveSet{c->d_mx.p, c->d_my.p, c->d_mm.p, c->d_mcount.p, record_max, target,
                     target == 1 ? c->d_maux.p : nullptr, target == 1 ? c->d_mchain.p : nullptr,
                     c->d_sflag.p, c->d_spos.p, c->d_sy.p, target == 0 ? c->d_sm.p : nullptr};
        c->moves_max = record_max;
    }
    c->d_step.ensure(1);
    ck(cudaMemsetAsync(c->d_step.p, 0, sizeof(int), c->stream), "memset");
    LearnP sp;
    sp.k0 = (uint32_t)seed;
    sp.k1 = (uint32_t)(seed >> 32) ^ 0x5DEECE66u;
    sp.nchain = nchain;
    sp.opt_steps = opt_steps;
    sp.randomize = randomize;
    sp.ws_max = P.wsm;
    sp.blob_max = P.blob_max;
    sp.p_learned = p_learned;
    sp.retain = c->retain;
    sp.nfeat_maps = std::min(c->nmaps, mlp::NMAP);
    sp.block = ud_learned_block(p_learned, record_max > 0);
    sp.p_learned = std::min(1.f, p_learned * (float)sp.block);
    sp.mc_steps = mc_steps;
    const int nblocks = (mc_steps + sp.block - 1) / sp.block;
    auto kern = c->retain > 1
                    ? (P.minb == 4 ? k_learn_step<4, 4> : (P.minb == 2 ? k_learn_step<2, 4, 384> : k_learn_step<3, 4>))
                    : (P.minb == 4 ? k_learn_step<4, 1> : (P.minb == 2 ? k_learn_step<2, 1, 384> : k_learn_step<3, 1>));
    const int fblocks = (int)std::min<long long>((nch * 32 + 255) / 256, (long long)c->nsm * 16);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ck(cudaStreamSynchronize(c->stream), "learned search setup");
    ck(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    try {
        ck(cudaMemsetAsync(c->d_counter.p, 0, sizeof(int), c->stream), "memset");
        if (feats)
            k_learn_features<<<fblocks, 256, 0, c->stream>>>(c->d_blobs.p, c->d_ligs.p, nlig, nchain, env, c->d_acc.p,
                                                             c->d_step.p, sp.nfeat_maps, c->d_x16.p);
        if (p_learned > 0.f) c->mlp.forward(c->stream, (int)nch, c->d_x16.p);
        kern<<<P.grid, 32 * P.W, P.smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, c->d_items.p, P.nitems, env, sp,
                                                      c->d_step.p, c->d_acc.p, c->d_best.p,
                                                      p_learned > 0.f ? c->mlp.out.p : nullptr, c->d_x16.p, ms,
                                                      c->d_counter.p, c->d_nevals.p);
        if (record_max > 0) {
            k_move_scan<<<1, 1024, 0, c->stream>>>(ms, nch);
            k_move_copy<<<fblocks, 256, 0, c->stream>>>(ms, c->d_x16.p, nch);
        }
        k_step_advance<<<1, 1, 0, c->stream>>>(c->d_step.p, sp.block);
    } catch (...) {
        cudaStreamEndCapture(c->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    ck(cudaStreamEndCapture(c->stream, &graph), "graph capture");
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ck(ie, "graph instantiate");
    cudaError_t le = cudaSuccess;
    for (int b = 0; b < nblocks && le == cudaSuccess; b++) le = cudaGraphLaunch(exec, c->stream);
    const cudaError_t se = cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(exec);
    ck(le, "graph launch");
    ck(se, "learned search");
    if (p_learned > 0.f) c->mlp.check_tc(c->stream);
    c->counters[2] += (long long)nblocks * (3 + (feats ? 1 : 0) + (p_learned > 0.f ? 4 : 0) + (record_max > 0 ? 2 : 0));
}

static void read_search_counters(ud_ctx* c) {
    unsigned long long ne[3] = {0, 0, 0};
    ck(cudaMemcpyAsync(ne, c->d_nevals.p, sizeof(ne), cudaMemcpyDeviceToHost, c->stream), "D2H");
    ck(cudaStreamSynchronize(c->stream), "search counters");
    c->counters[0] = (long long)ne[0];
    c->counters[1] = (long long)ne[1];
    if (ne[2]) throw Fail(UD_ECUDA, "search: a topology bulk copy did not complete within its wait limit");
}

int ud_search(ud_ctx* c, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, int mode,
              long long* out_nevals) {
    try {
        if (!c || nchain <= 0 || mc_steps < 0 || opt_steps < 0) throw Fail(UD_EINVAL, "invalid search arguments");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        c->counters[2] = 0;
        launch_search(c, seed, nchain, mc_steps, opt_steps, randomize, mode);
        read_search_counters(c);
        if (out_nevals) *out_nevals = c->counters[0];
        c->has_results = false;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_get_chain_poses(const ud_ctx* c, int lig, float* out) {
    try {
        if (!c || lig < 0 || lig >= (int)c->h_ligs.size() || !out || c->nchain == 0)
            throw Fail(UD_EINVAL, "invalid arguments or no search results");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        const LigHost& h = c->h_ligs[lig];
        ck(cudaMemcpy(out, c->d_best.p + c->h_ligdev[lig].best_off, (size_t)c->nchain * h.stride * sizeof(float),
                      cudaMemcpyDeviceToHost), "D2H");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

static void launch_cluster(ud_ctx* c, float rmsd_limit) {
    int nlig = (int)c->h_ligs.size();
    int nchain = c->nchain;
    c->d_leaders.ensure((size_t)nlig * nchain);
    c->d_counts.ensure(nlig);
    size_t smem = (size_t)nchain * 12;
    set_smem(k_cluster, smem);
    int threads = std::min(1024, std::max(32, ((nchain + 31) / 32) * 32));
    k_cluster<<<nlig, threads, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, nlig, nchain, c->d_best.p, rmsd_limit,
                                                  c->d_leaders.p, c->d_counts.p);
    ck(cudaGetLastError(), "k_cluster launch");
}

int ud_cluster(ud_ctx* c, float rmsd_limit, int* out_leaders, int* out_counts) {
    try {
        if (!c || c->nchain == 0) throw Fail(UD_ESTATE, "no search results to cluster");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        launch_cluster(c, rmsd_limit);
        int nlig = (int)c->h_ligs.size();
        if (out_leaders)
            ck(cudaMemcpyAsync(out_leaders, c->d_leaders.p, (size_t)nlig * c->nchain * sizeof(int),
                               cudaMemcpyDeviceToHost, c->stream), "D2H");
        if (out_counts)
            ck(cudaMemcpyAsync(out_counts, c->d_counts.p, nlig * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "k_cluster");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

// DockTask::run for the loaded batch; p_learned < 0: the fused search (k_search), else the
// learned-proposal search with that probability of a learned move
static int dock_impl(ud_ctx* c, const ud_dock_params* p, float p_learned, long long* out_nevals) {
    try {
        if (!c || !p || p->nchain <= 0 || p->mc_steps < 0 || p->opt_steps < 0 || p->num_pose <= 0 ||
            p->refine_steps < 0 || (p->refine_mode != UD_MODE_DIRECT && p->refine_mode != UD_MODE_GRID))
            throw Fail(UD_EINVAL, "invalid dock parameters");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        int nlig = (int)c->h_ligs.size();
        if (nlig == 0) throw Fail(UD_ESTATE, "no ligands loaded");
        c->counters[2] = 0;
        sync_ligs(c);
        c->rec(0);
        if (p_learned < 0.f)
            launch_search(c, p->seed, p->nchain, p->mc_steps, p->opt_steps, p->randomize, p->mode);
        else
            launch_learned(c, p->seed, p->nchain, p->mc_steps, p->opt_steps, p->randomize, p->mode, p_learned, 0);
        c->rec(1);
        launch_cluster(c, p->rmsd_limit);
        c->counters[2]++;
        c->rec(2);
        // refinement of every cluster leader (on exact pair sums unless refine_mode says
        // grid): the (ligand, chain) list is built on the host from the leader counts
        Env env = make_env(c, p->refine_mode);
        std::vector<int> counts(nlig);
        ck(cudaMemcpyAsync(counts.data(), c->d_counts.p, nlig * sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H");
        const int nrec_lig = c->nchain;                 // records per ligand (chains x retained)
        std::vector<int> leaders((size_t)nlig * nrec_lig);
        ck(cudaMemcpyAsync(leaders.data(), c->d_leaders.p, leaders.size() * sizeof(int), cudaMemcpyDeviceToHost,
                           c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "search+cluster");
        if (p->refine_steps > 0) {
            std::vector<int> il;
            std::vector<long long> io;
            int wsm = 0;
            for (int l = 0; l < nlig; l++) {
                const LigHost& h = c->h_ligs[l];
                wsm = std::max(wsm, lig_ws(h));
                for (int k = 0; k < counts[l]; k++) {
                    il.push_back(l);
                    io.push_back(c->h_ligdev[l].best_off + (long long)leaders[(size_t)l * nrec_lig + k] * h.stride);
                }
            }
            int n = (int)il.size();
            if (n > 0) {
                c->d_item_lig.upload(il.data(), n, c->stream);
                c->d_item_off.upload(io.data(), n, c->stream);
                int W = pick_warps(c, wsm, 0, 8);
                size_t smem = (size_t)W * wsm * 4;
                const auto kb = bfgs_kernel(env);
                set_smem(kb, smem);
                kb<<<(n + W - 1) / W, 32 * W, smem, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, c->d_item_lig.p,
                                                                     c->d_item_off.p, c->d_best.p, env, 2,
                                                                     p->refine_steps, VCAP_AUTH, 100.f, 1, wsm,
                                                                     nullptr);
                ck(cudaGetLastError(), "k_bfgs launch");
                c->counters[2]++;
            }
        }
        c->rec(3);
        // filter and gather
        c->num_pose = p->num_pose;
        long long of = 0;
        for (int l = 0; l < nlig; l++) {
            c->h_ligdev[l].out_off = of;
            of += (long long)p->num_pose * c->h_ligs[l].stride;
        }
        c->out_floats = of;
        upload_ligdev(c);
        c->d_sel.ensure((size_t)nlig * p->num_pose);
        c->d_selcnt.ensure(nlig);
        c->d_out.ensure((size_t)of);
        size_t fsm = (size_t)nrec_lig * 8;
        set_smem(k_filter, fsm);
        k_filter<<<nlig, 128, fsm, c->stream>>>(c->d_ligs.p, nlig, nrec_lig, c->d_best.p, c->d_leaders.p,
                                                c->d_counts.p, p->num_pose, p->energy_range, c->d_sel.p, c->d_selcnt.p);
        ck(cudaGetLastError(), "k_filter launch");
        long long items = (long long)nlig * p->num_pose;
        k_gather<<<(unsigned)((items + 7) / 8), 256, 0, c->stream>>>(c->d_ligs.p, nlig, p->num_pose, c->d_best.p,
                                                                    c->d_sel.p, c->d_selcnt.p, c->d_out.p);
        ck(cudaGetLastError(), "k_gather launch");
        c->counters[2] += 2;
        c->rec(4);
        c->h_counts.assign(nlig, 0);
        ck(cudaMemcpyAsync(c->h_counts.data(), c->d_selcnt.p, nlig * sizeof(int), cudaMemcpyDeviceToHost, c->stream),
           "D2H");
        read_search_counters(c);
        long long ne = c->counters[0];
        // final scoring of the selected poses (score.cpp semantics)
        std::vector<int> pl;
        std::vector<long long> xo, dof;
        long long ds = 0;
        for (int l = 0; l < nlig; l++)
            for (int k = 0; k < c->h_counts[l]; k++) {
                pl.push_back(l);
                xo.push_back(c->h_ligdev[l].out_off + (long long)k * c->h_ligs[l].stride + 8);
                dof.push_back(ds);
                ds += 5LL * c->h_ligs[l].natom;
            }
        int n = (int)pl.size();
        c->decomp = p->energy_decomp != 0;
        if (n > 0) {
            Env fenv = make_env(c, p->final_mode);
            c->d_item_lig.upload(pl.data(), n, c->stream);
            c->d_item_off.upload(xo.data(), n, c->stream);
            c->d_item_off2.upload(dof.data(), n, c->stream);
            c->d_terms.ensure(4 * (size_t)n);
            if (c->decomp) c->d_decomp.ensure((size_t)ds);
            k_terms<<<(n + 7) / 8, 256, 0, c->stream>>>(c->d_blobs.p, c->d_ligs.p, n, c->d_item_lig.p, c->d_item_off.p,
                                                        c->d_out.p, fenv, c->d_terms.p,
                                                        c->decomp ? c->d_decomp.p : nullptr, c->d_item_off2.p);
            ck(cudaGetLastError(), "k_terms launch");
            c->counters[2]++;
        }
        c->rec(5);
        ck(cudaStreamSynchronize(c->stream), "k_terms");
        float t[5];
        for (int i = 0; i < 5; i++) ck(cudaEventElapsedTime(&t[i], c->ev[i], c->ev[i + 1]), "event time");
        for (int i = 0; i < 5; i++) c->stage_ms[i] = t[i];
        ck(cudaEventElapsedTime(&c->stage_ms[5], c->ev[0], c->ev[5]), "event time");
        if (out_nevals) *out_nevals = ne;
        c->has_results = true;
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_dock(ud_ctx* c, const ud_dock_params* p, long long* out_nevals) { return dock_impl(c, p, -1.f, out_nevals); }

int ud_learned_block(float p_learned, int recording) {
    if (recording || !(p_learned >= 0.f && p_learned <= 1.f)) return 1;
    return p_learned > 0.f ? std::max(1, std::min(8, (int)(1.f / p_learned))) : 8;
}

int ud_dock_learned(ud_ctx* c, const ud_dock_params* p, float p_learned, long long* out_nevals) {
    if (!(p_learned >= 0.f && p_learned <= 1.f)) {
        g_err = "p_learned must be in [0, 1]";
        return UD_EINVAL;
    }
    return dock_impl(c, p, p_learned, out_nevals);
}

int ud_result_counts(const ud_ctx* c, int* out) {
    if (!c || !c->has_results || !out) { g_err = "no docking results"; return UD_ESTATE; }
    memcpy(out, c->h_counts.data(), c->h_counts.size() * sizeof(int));
    return UD_OK;
}

long long ud_result_floats(const ud_ctx* c) {
    if (!c || !c->has_results) return 0;
    long long s = 0;
    for (size_t l = 0; l < c->h_ligs.size(); l++) s += (long long)c->h_counts[l] * c->h_ligs[l].stride;
    return s;
}

int ud_get_results(const ud_ctx* c, float* out_records, float* out_terms4, float* out_decomp) {
    try {
        if (!c || !c->has_results) throw Fail(UD_ESTATE, "no docking results");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        int nlig = (int)c->h_ligs.size();
        std::vector<float> all((size_t)c->out_floats);
        ck(cudaMemcpy(all.data(), c->d_out.p, all.size() * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
        long long w = 0;
        int npose = 0;
        long long ndec = 0;
        for (int l = 0; l < nlig; l++) {
            long long nf = (long long)c->h_counts[l] * c->h_ligs[l].stride;
            if (out_records) memcpy(out_records + w, all.data() + c->h_ligdev[l].out_off, nf * sizeof(float));
            w += nf;
            npose += c->h_counts[l];
            ndec += 5LL * c->h_ligs[l].natom * c->h_counts[l];
        }
        if (out_terms4 && npose)
            ck(cudaMemcpy(out_terms4, c->d_terms.p, 4 * (size_t)npose * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
        if (out_decomp && c->decomp && ndec)
            ck(cudaMemcpy(out_decomp, c->d_decomp.p, ndec * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

void* ud_stream(ud_ctx* c) { return c ? (void*)c->stream : nullptr; }

int ud_stage_times(const ud_ctx* c, float* out6) {
    if (!c || !out6) { g_err = "null argument"; return UD_EINVAL; }
    memcpy(out6, c->stage_ms, sizeof(c->stage_ms));
    return UD_OK;
}

int ud_counters(const ud_ctx* c, long long* out4) {
    if (!c || !out4) { g_err = "null argument"; return UD_EINVAL; }
    memcpy(out4, c->counters, sizeof(c->counters));
    return UD_OK;
}

int ud_sync(ud_ctx* c) {
    try {
        if (!c) throw Fail(UD_EINVAL, "null context");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_set_gemm(ud_ctx* c, int kind) {
    if (!c || (kind != 0 && kind != 1)) { g_err = "kind must be 0 (mma.sync) or 1 (tcgen05)"; return UD_EINVAL; }
    c->mlp.use_tc = kind == 1;
    return UD_OK;
}

int ud_set_retain(ud_ctx* c, int retain) {
    if (!c || retain < 1 || retain > 4) { g_err = "retain must be 1..4"; return UD_EINVAL; }
    c->retain = retain;
    c->tune_key = -1;
    return UD_OK;
}

int ud_set_autotune(ud_ctx* c, int on) {
    if (!c) { g_err = "null context"; return UD_EINVAL; }
    c->autotune = on ? 1 : 0;
    c->tune_key = -1;
    return UD_OK;
}

int ud_set_packing(ud_ctx* c, int warps_per_cta, int chains_per_warp) {
    if (!c) { g_err = "null context"; return UD_EINVAL; }
    if (!(warps_per_cta == 0 || warps_per_cta == 4 || warps_per_cta == 8 || warps_per_cta == 12) ||
        chains_per_warp < 0 || chains_per_warp > 4) {
        g_err = "packing: warps per CTA 0, 4, 8 or 12; chains per warp 0..4";
        return UD_EINVAL;
    }
    c->pack_w = warps_per_cta;
    c->pack_k = chains_per_warp;
    return UD_OK;
}

int ud_search_shape(const ud_ctx* c, int* out4) {
    if (!c || !out4) { g_err = "invalid arguments"; return UD_EINVAL; }
    for (int i = 0; i < 4; i++) out4[i] = c->shape[i];
    return UD_OK;
}

// ---------------------------------------------------------------------- learned proposal
long long ud_mlp_param_count(void) { return mlp::NPARAM; }

int ud_mlp_init(ud_ctx* c, uint64_t seed) {
    try {
        if (!c) throw Fail(UD_EINVAL, "null context");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        c->mlp.init(seed, c->stream);
        ck(cudaStreamSynchronize(c->stream), "mlp init");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_set_params(ud_ctx* c, const float* params) {
    try {
        if (!c || !params) throw Fail(UD_EINVAL, "invalid arguments");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        c->mlp.set(params, c->stream);
        ck(cudaStreamSynchronize(c->stream), "mlp set");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_get_params(ud_ctx* c, float* params) {
    try {
        if (!c || !params) throw Fail(UD_EINVAL, "invalid arguments");
        if (!c->mlp.ready) throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init or ud_mlp_set_params");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        ck(cudaMemcpyAsync(params, c->mlp.p.p, sizeof(float) * mlp::NPARAM, cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "mlp get");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_forward(ud_ctx* c, int n, const float* x, float* out) {
    try {
        if (!c || n < 0 || (n > 0 && (!x || !out))) throw Fail(UD_EINVAL, "invalid arguments");
        if (!c->mlp.ready) throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init or ud_mlp_set_params");
        if (n == 0) return UD_OK;
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        MlpState& m = c->mlp;
        m.ensure(n);
        DBuf<float> dx;
        dx.upload(x, (size_t)n * mlp::IN, c->stream);
        k_f32_to_bf16<<<MlpState::blocks((long long)n * mlp::IN), 256, 0, c->stream>>>((long long)n * mlp::IN, dx.p,
                                                                                        m.x16.p);
        m.forward(c->stream, n, m.x16.p);
        ck(cudaMemcpyAsync(out, m.out.p, sizeof(float) * n * mlp::OUT, cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "mlp forward");
        m.check_tc(c->stream);
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_loss_grad(ud_ctx* c, int n, const float* x, const float* y, const float* mask, double* out_loss,
                     float* out_grad) {
    try {
        if (!c || n <= 0 || !x || !y || !mask || !out_loss || !out_grad) throw Fail(UD_EINVAL, "invalid arguments");
        if (!c->mlp.ready) throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init or ud_mlp_set_params");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        MlpState& m = c->mlp;
        m.ensure(n);
        DBuf<float> dx, dy, dm;
        dx.upload(x, (size_t)n * mlp::IN, c->stream);
        dy.upload(y, (size_t)n * mlp::NDIM, c->stream);
        dm.upload(mask, (size_t)n * mlp::NDIM, c->stream);
        k_f32_to_bf16<<<MlpState::blocks((long long)n * mlp::IN), 256, 0, c->stream>>>((long long)n * mlp::IN, dx.p,
                                                                                        m.x16.p);
        m.forward(c->stream, n, m.x16.p);
        m.loss_backward(c->stream, n, m.x16.p, dy.p, dm.p, true);
        ck(cudaMemcpyAsync(out_loss, m.loss.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaMemcpyAsync(out_grad, m.g.p, sizeof(float) * mlp::NPARAM, cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "mlp loss_grad");
        m.check_tc(c->stream);
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

// epochs of minibatch Adam over n device-resident samples (full batches only)
static void train_on_device(ud_ctx* c, int n, const __nv_bfloat16* x16, const float* y, const float* mk, int epochs,
                            int batch, float lr, uint64_t seed, float* out_epoch_loss) {
    cudaStream_t s = c->stream;
    MlpState& m = c->mlp;
    const int nb = std::min(batch, n);
    m.ensure(nb);
    DBuf<float> by, bm;
    DBuf<int> didx;
    by.ensure((size_t)nb * mlp::NDIM);
    bm.ensure((size_t)nb * mlp::NDIM);
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    std::mt19937_64 rng(seed);
    const int nbatch = n / nb;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        didx.upload(perm.data(), (size_t)n, s);
        for (int b = 0; b < nbatch; b++) {
            const int* ib = didx.p + (size_t)b * nb;
            k_gather_rows<<<(int)(((long long)nb * mlp::IN + 255) / 256), 256, 0, s>>>(nb, ib, mlp::IN, x16, m.x16.p);
            k_gather_rows_f32<<<(nb * mlp::NDIM + 255) / 256, 256, 0, s>>>(nb, ib, mlp::NDIM, y, by.p);
            k_gather_rows_f32<<<(nb * mlp::NDIM + 255) / 256, 256, 0, s>>>(nb, ib, mlp::NDIM, mk, bm.p);
            m.forward(s, nb, m.x16.p);
            m.loss_backward(s, nb, m.x16.p, by.p, bm.p, b == 0);
            m.adam(s, lr);
        }
        double l = 0.0;
        ck(cudaMemcpyAsync(&l, m.loss.p, sizeof(double), cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "mlp train epoch");
        if (out_epoch_loss) out_epoch_loss[ep] = (float)(l / std::max(1, nbatch));
    }
    m.check_tc(s);
}

int ud_mlp_train(ud_ctx* c, int n, const float* x, const float* y, const float* mask, int epochs, int batch, float lr,
                 uint64_t seed, float* out_epoch_loss) {
    try {
        if (!c || n <= 0 || !x || !y || !mask || epochs < 0 || batch <= 0) throw Fail(UD_EINVAL, "invalid arguments");
        if (!c->mlp.ready) throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init or ud_mlp_set_params");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        cudaStream_t s = c->stream;
        DBuf<float> dx, dy, dm;
        DBuf<__nv_bfloat16> x16;
        dx.upload(x, (size_t)n * mlp::IN, s);
        x16.ensure((size_t)n * mlp::IN);
        k_f32_to_bf16<<<MlpState::blocks((long long)n * mlp::IN), 256, 0, s>>>((long long)n * mlp::IN, dx.p, x16.p);
        ck(cudaStreamSynchronize(s), "mlp train upload");
        dx.release();
        dy.upload(y, (size_t)n * mlp::NDIM, s);
        dm.upload(mask, (size_t)n * mlp::NDIM, s);
        train_on_device(c, n, x16.p, dy.p, dm.p, epochs, batch, lr, seed, out_epoch_loss);
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_search_learned(ud_ctx* c, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, float p_learned,
                      long long* out_nevals) {
    try {
        if (!c || nchain <= 0 || mc_steps < 1 || opt_steps < 0) throw Fail(UD_EINVAL, "invalid search arguments");
        if (c->h_ligs.empty()) throw Fail(UD_ESTATE, "no ligands loaded");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        launch_learned(c, seed, nchain, mc_steps, opt_steps, randomize, UD_MODE_GRID, p_learned, 0);
        read_search_counters(c);
        c->has_results = false;
        if (out_nevals) *out_nevals = c->counters[0];
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_collect_moves(ud_ctx* c, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, int target,
                     int max_moves, int* out_count) {
    try {
        if (!c || nchain <= 0 || mc_steps < 1 || opt_steps < 0 || max_moves <= 0 || !out_count ||
            (target != 0 && target != 1))
            throw Fail(UD_EINVAL, "invalid arguments");
        if (c->h_ligs.empty()) throw Fail(UD_ESTATE, "no ligands loaded");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        launch_learned(c, seed, nchain, mc_steps, opt_steps, randomize, UD_MODE_GRID, 0.f, max_moves, target);
        read_search_counters(c);
        c->has_results = false;
        int cnt = 0;
        ck(cudaMemcpyAsync(&cnt, c->d_mcount.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "collect");
        *out_count = std::min(cnt, max_moves);
        c->moves_n = *out_count;
        if (target == 1 && *out_count > 0) {
            const int nlig = (int)c->h_ligs.size();
            c->d_ligbest.ensure((size_t)nlig);
            k_lig_best<<<nlig, 256, 0, c->stream>>>(c->d_ligs.p, nlig, nchain, c->d_best.p, c->d_ligbest.p);
            MoveSet ms{c->d_mx.p,    c->d_my.p,     c->d_mm.p, c->d_mcount.p, max_moves, 1,
                       c->d_maux.p,  c->d_mchain.p, nullptr,   nullptr,        nullptr,   nullptr};
            const long long threads = (long long)*out_count * 32;
            k_label_moves<<<(unsigned)((threads + 255) / 256), 256, 0, c->stream>>>(
                c->d_blobs.p, c->d_ligs.p, nchain, c->d_best.p, c->d_ligbest.p, ms, *out_count, c->constraint);
            ck(cudaGetLastError(), "label moves");
            ck(cudaStreamSynchronize(c->stream), "label moves");
        }
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_get_moves(ud_ctx* c, int n, float* out_x, float* out_y, float* out_mask) {
    try {
        if (!c || n < 0 || n > c->moves_n) throw Fail(UD_EINVAL, "invalid move count");
        if (n == 0) return UD_OK;
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        if (out_x) {
            std::vector<uint16_t> h((size_t)n * mlp::IN);
            ck(cudaMemcpyAsync(h.data(), c->d_mx.p, h.size() * 2, cudaMemcpyDeviceToHost, c->stream), "D2H");
            ck(cudaStreamSynchronize(c->stream), "moves");
            for (size_t i = 0; i < h.size(); i++) {
                const uint32_t u = (uint32_t)h[i] << 16;
                memcpy(&out_x[i], &u, 4);
            }
        }
        if (out_y) ck(cudaMemcpyAsync(out_y, c->d_my.p, sizeof(float) * n * mlp::NDIM, cudaMemcpyDeviceToHost, c->stream), "D2H");
        if (out_mask) ck(cudaMemcpyAsync(out_mask, c->d_mm.p, sizeof(float) * n * mlp::NDIM, cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "moves");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

int ud_mlp_train_moves(ud_ctx* c, int epochs, int batch, float lr, uint64_t seed, float* out_epoch_loss) {
    try {
        if (!c || epochs < 0 || batch <= 0) throw Fail(UD_EINVAL, "invalid arguments");
        if (c->moves_n <= 0) throw Fail(UD_ESTATE, "no recorded moves: call ud_collect_moves first");
        if (!c->mlp.ready) throw Fail(UD_ESTATE, "no proposal network: call ud_mlp_init or ud_mlp_set_params");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        train_on_device(c, c->moves_n, c->d_mx.p, c->d_my.p, c->d_mm.p, epochs, batch, lr, seed, out_epoch_loss);
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}

}  // extern "C"

// ====================================================================== no-allocation scoring
namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// device address of g_noalloc_scratch on `device` (which must be current), looked up once
unsigned char* noalloc_scratch(int device) {
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) throw Fail(UD_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress (no-allocation scratch)");
        g_noalloc_ptr[device] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_ptr[device]);
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
}  // namespace

extern "C" int ud_score_batch_noalloc(ud_ctx* c, int n, const int* pose_lig, const float* coords,
                                      const float* centers, const float* rotvecs, int mode, float vcap, float slope,
                                      float* out_e, float* out_g) {
    try {
        if (!c || n < 0 || (n > 0 && (!pose_lig || !coords || !centers || !rotvecs || !out_e || !out_g)))
            throw Fail(UD_EINVAL, "invalid score arguments");
        if (n == 0) return UD_OK;
        if (n > UD_NOALLOC_MAX_POSES)
            throw Fail(UD_EINVAL, "ud_score_batch_noalloc: " + std::to_string(n) + " poses exceed the limit of " +
                                      std::to_string(UD_NOALLOC_MAX_POSES) + "; split the batch");
        ck(cudaSetDevice(c->device), "cudaSetDevice");
        if (c->ligs_dirty)
            throw Fail(UD_ESTATE, "ud_score_batch_noalloc: the ligand set changed since it was last uploaded; "
                                  "make one ud_score_batch, ud_search or ud_dock call first");
        Env env = make_env(c, mode);
        long long xs = 0, gs = 0;
        int wsm = 0;
        for (int i = 0; i < n; i++) {
            const int l = pose_lig[i];
            if (l < 0 || l >= (int)c->h_ligs.size()) throw Fail(UD_EINVAL, "pose ligand index out of range");
            xs += 3LL * c->h_ligs[l].natom;
            gs += 6 + c->h_ligs[l].ntors;
            wsm = std::max(wsm, lig_ws(c->h_ligs[l]));
        }
        const size_t o_lig = 0;
        const size_t o_xo = align256(o_lig + (size_t)n * sizeof(int));
        const size_t o_go = align256(o_xo + (size_t)n * sizeof(long long));
        const size_t o_x = align256(o_go + (size_t)n * sizeof(long long));
        const size_t o_c = align256(o_x + (size_t)xs * sizeof(float));
        const size_t o_r = align256(o_c + 3 * (size_t)n * sizeof(float));
        const size_t o_e = align256(o_r + 3 * (size_t)n * sizeof(float));
        const size_t o_g = align256(o_e + (size_t)n * sizeof(float));
        const size_t end = o_g + (size_t)gs * sizeof(float);
        if (end > (size_t)UD_NOALLOC_SCRATCH_BYTES)
            throw Fail(UD_EINVAL, "ud_score_batch_noalloc: the batch needs " + std::to_string(end) +
                                      " bytes of staging, above the fixed " +
                                      std::to_string((size_t)UD_NOALLOC_SCRATCH_BYTES) + "; split the batch");
        unsigned char* s = noalloc_scratch(c->device);
        int* d_lig = reinterpret_cast<int*>(s + o_lig);
        long long* d_xo = reinterpret_cast<long long*>(s + o_xo);
        long long* d_go = reinterpret_cast<long long*>(s + o_go);
        float* d_x = reinterpret_cast<float*>(s + o_x);
        float* d_c = reinterpret_cast<float*>(s + o_c);
        float* d_r = reinterpret_cast<float*>(s + o_r);
        float* d_e = reinterpret_cast<float*>(s + o_e);
        float* d_g = reinterpret_cast<float*>(s + o_g);
        cudaStream_t st = c->stream;
        ck(cudaMemcpyAsync(d_lig, pose_lig, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaMemcpyAsync(d_x, coords, (size_t)xs * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaMemcpyAsync(d_c, centers, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
        ck(cudaMemcpyAsync(d_r, rotvecs, 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, st), "H2D");
        // every offset, energy and gradient word is written below: nothing has to start at zero
        k_pose_offsets<<<1, 1024, 0, st>>>(c->d_ligs.p, n, d_lig, d_xo, d_go);
        ck(cudaGetLastError(), "k_pose_offsets launch");
        const int W = pick_warps(c, wsm, 0, 8);
        const size_t smem = (size_t)W * wsm * 4;
        const auto ks = score_kernel(env);
        set_smem(ks, smem);
        PoseIO io{d_lig, d_xo, d_x, d_c, d_r, d_go};
        ks<<<(n + W - 1) / W, 32 * W, smem, st>>>(c->d_blobs.p, c->d_ligs.p, n, io, env, vcap, slope, wsm, d_e,
                                                       d_g);
        ck(cudaGetLastError(), "k_score launch");
        ck(cudaMemcpyAsync(out_e, d_e, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaMemcpyAsync(out_g, d_g, (size_t)gs * sizeof(float), cudaMemcpyDeviceToHost, st), "D2H");
        ck(cudaStreamSynchronize(st), "k_score");
        return UD_OK;
    } catch (const Fail& f) {
        return fail(f);
    }
}
