// ud_device.cuh -- warp-level device code of the B200 docking engine.
//
// One warp owns one pose (a Monte Carlo chain, a BFGS job or a scoring job).  The
// ligand topology is a packed blob of 32-bit words (layout below) that kernels stage
// in shared memory; pose state (coordinates, dihedrals, centre, last rotation
// increment) lives in per-warp shared-memory slots.  Per-atom work is strided over
// the 32 lanes, per-torsion scalar work runs lane-parallel, reductions are fixed
// xor-butterflies (results are deterministic run to run).
//
// The arithmetic follows the reference engine (paths relative to
// unidock/unidock_engine/): Vina terms src/score/vina.h:151-321; E/force
// src/cuda/bfgs.cuh:221-394; reverse gradient pass bfgs.cuh:69-193; kinematics
// bfgs.cuh:443-618; line search bfgs.cuh:623-670; BFGS bfgs.cuh:682-829 (inverse
// Hessian kept in FP64 here); mutation / Metropolis src/cuda/mc.cu:146-256,
// src/search/mc.h:12-18.  The intermolecular term is either the reference's direct
// pair sum or trilinear interpolation of precomputed per-type grid maps.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

namespace ud {

constexpr int WARP = 32;
constexpr unsigned FULL = 0xffffffffu;
constexpr int NT = 21;            // XS types
constexpr int VN_H = 0;
constexpr float PI_F = 3.1415927f;
constexpr float EPS_F = 1.1920929e-07f;   // numeric_limits<float>::epsilon()
constexpr float PENALTY_SLOPE = 1e6f;
constexpr float VCAP_SEARCH = 10.0f;
constexpr float VCAP_AUTH = 1000.0f;
constexpr int LS_STEPS = 10;

// ---------------------------------------------------------------- blob layout
// Header words; section offsets are word offsets from the blob start.
enum BlobHdr {
    H_NATOM = 0, H_NTORS, H_NHEAVY, H_NPAIR, H_NROT, H_NRANGE, H_NBIAS,
    H_TYPES,       // natom ints
    H_AXIS,        // 2T ints (from, to)
    H_RANGE_OFF,   // T+1 ints (in ranges)
    H_RANGES,      // 2*nrange floats
    H_ROT_OFF,     // T+1 ints
    H_ROT,         // rotated atoms of every torsion
    H_PAIR_OFF,    // natom+1 ints: per-atom intra adjacency (both directions)
    H_PAIRS,       // packed entries: j | zero<<16 | hydrophobic pair<<17 | hbond pair<<18
    H_BIAS_OFF,    // natom+1 ints (records)
    H_BIAS,        // 5 floats per record
    H_HEAVY,       // heavy atom indices
    H_X0, H_D0, H_C0,   // initial coordinates, dihedrals, centre
    H_RADII,       // natom floats: vdW radius per atom
    H_RHOFF,       // T+1 ints: heavy rotated atoms per torsion
    H_RHEAVY,
    H_MAPIDX,      // natom ints: grid map slot of each atom (-1: none), set at upload
    H_NPREC,       // number of heavy scored pairs (a count, not an offset)
    H_PREC,        // 2 words per pair: i | j<<12 | hydrophobic<<24 | hbond<<25, and R_i + R_j (float)
    H_GOFF,        // natom+1 ints: per-atom lists of (pair index, partner) for the gather
    H_GADJ,        // entries: pair index | partner << 16
    H_TOTAL,
    H_STAGE,       // words of the blob prefix the search stages into shared memory
    H_FRAME0,      // 3 words: non-collinear atoms no torsion moves (a rigid frame), or -1
    H_WORDS = 36
};
// The search is bound by instruction fetch: its loop body is large and the warps of an SM
// run different parts of it.  Every loop with a run-time trip count therefore carries
// `#pragma unroll 1`; the compiler's default unrolling of those loops made the library's
// code 32 % larger and the search of a 148-ligand screen batch 23 % slower (same results).
// inlining of the large routines of the search loop: a single shared copy (noinline)
// keeps the loop's instruction footprint small, inlining saves the call overhead
#ifndef UD_EVAL_ATTR
#define UD_EVAL_ATTR __forceinline__
#endif
#ifndef UD_KIN_ATTR
#define UD_KIN_ATTR __forceinline__
#endif
#ifndef UD_LS_ATTR
#define UD_LS_ATTR __forceinline__
#endif
constexpr int PREC_HYD = 1 << 24, PREC_HB = 1 << 25;
constexpr int PAIR_ZERO = 1 << 16, PAIR_HYD = 1 << 17, PAIR_HB = 1 << 18;

// Topology view: one base pointer and word offsets (keeps addressing 32-bit).
struct Topo {
    const int* b;
    int natom, ntors, nheavy, nbias;
    int o_types, o_axis, o_roff, o_ranges, o_rot_off, o_rot, o_pair_off, o_pairs, o_bias_off, o_bias, o_heavy,
        o_radii, o_rhoff, o_rheavy, o_mapidx, nprec, o_prec, o_goff, o_gadj;
    __device__ __forceinline__ int type(int i) const { return b[o_types + i]; }
    __device__ __forceinline__ int axis(int k) const { return b[o_axis + k]; }
    __device__ __forceinline__ int range_off(int k) const { return b[o_roff + k]; }
    __device__ __forceinline__ const float* ranges() const { return reinterpret_cast<const float*>(b + o_ranges); }
    __device__ __forceinline__ int rot_off(int k) const { return b[o_rot_off + k]; }
    __device__ __forceinline__ int rot(int q) const { return b[o_rot + q]; }
    __device__ __forceinline__ int pair_off(int i) const { return b[o_pair_off + i]; }
    __device__ __forceinline__ int pair(int k) const { return b[o_pairs + k]; }
    __device__ __forceinline__ int bias_off(int i) const { return b[o_bias_off + i]; }
    __device__ __forceinline__ const float* bias() const { return reinterpret_cast<const float*>(b + o_bias); }
    __device__ __forceinline__ int heavy(int h) const { return b[o_heavy + h]; }
    __device__ __forceinline__ float radius(int i) const { return __int_as_float(b[o_radii + i]); }
    __device__ __forceinline__ int rh_off(int k) const { return b[o_rhoff + k]; }
    __device__ __forceinline__ int rheavy(int q) const { return b[o_rheavy + q]; }
    __device__ __forceinline__ int map_index(int i) const { return b[o_mapidx + i]; }
    __device__ __forceinline__ int2 prec(int p) const { return *reinterpret_cast<const int2*>(b + o_prec + 2 * p); }
    __device__ __forceinline__ int goff(int i) const { return b[o_goff + i]; }
    __device__ __forceinline__ int gadj(int k) const { return b[o_gadj + k]; }
};

__device__ __forceinline__ Topo topo_view(const int* b) {
    Topo t;
    t.b = b;
    t.natom = b[H_NATOM];
    t.ntors = b[H_NTORS];
    t.nheavy = b[H_NHEAVY];
    t.nbias = b[H_NBIAS];
    t.o_types = b[H_TYPES];
    t.o_axis = b[H_AXIS];
    t.o_roff = b[H_RANGE_OFF];
    t.o_ranges = b[H_RANGES];
    t.o_rot_off = b[H_ROT_OFF];
    t.o_rot = b[H_ROT];
    t.o_pair_off = b[H_PAIR_OFF];
    t.o_pairs = b[H_PAIRS];
    t.o_bias_off = b[H_BIAS_OFF];
    t.o_bias = b[H_BIAS];
    t.o_heavy = b[H_HEAVY];
    t.o_radii = b[H_RADII];
    t.o_rhoff = b[H_RHOFF];
    t.o_rheavy = b[H_RHEAVY];
    t.o_mapidx = b[H_MAPIDX];
    t.nprec = b[H_NPREC];
    t.o_prec = b[H_PREC];
    t.o_goff = b[H_GOFF];
    t.o_gadj = b[H_GADJ];
    return t;
}

// ---------------------------------------------------------------- scoring env
struct GridView {
    const float* f32;     // nmaps * npt, x fastest
    const __half* f16;    // same layout, or null
    float ox, oy, oz, inv_s;
    int gx, gy, gz;
    int use_f16;
};

struct Env {
    float box_lo[3], box_hi[3];
    int mode;                 // 0 direct, 1 grid
    int constraint;
    int bias_type;            // 0 none, 1 pos, 2 align
    float bias_k;
    const float4* rec;        // x y z type(as float)
    int nrec;
    GridView grid;
    // the receptor atoms again, sorted into cubic cells of CELL_A (x fastest), for the direct
    // sums: cell_start[c] .. cell_start[c + 1] are cell c's atoms, in receptor order
    const float4* rec_cells;
    const int* cell_start;
    float cell_o[3];
    int cdim[3];
};

// Cell edge of the receptor cell list: a little above the 8 A cutoff, so that two points
// closer than the cutoff are never two cells apart along an axis, whatever the rounding.
constexpr float CELL_A = 8.0625f;

__constant__ float c_vdw[NT] = {1.1f, 1.92f, 1.9f, 1.9f, 1.8f, 1.8f, 1.8f, 1.8f, 1.7f, 1.7f, 1.7f,
                                1.7f, 1.5f, 2.2f, 2.1f, 2.0f, 1.8f, 2.0f, 2.2f, 2.3f, 1.2f};
// bit t set: hydrophobic / acceptor / donor (src/score/vina.h:125-137)
constexpr unsigned HYD_MASK = (1u << 2) | (1u << 12) | (1u << 16) | (1u << 17) | (1u << 18);
constexpr unsigned ACC_MASK = (1u << 6) | (1u << 7) | (1u << 10) | (1u << 11);
constexpr unsigned DON_MASK = (1u << 5) | (1u << 7) | (1u << 9) | (1u << 11) | (1u << 20);

__device__ __forceinline__ float vdw(int t) { return c_vdw[t]; }

__device__ __forceinline__ bool hyd_pair(int t1, int t2) {
    return ((1u << t1) & HYD_MASK) && ((1u << t2) & HYD_MASK);
}
__device__ __forceinline__ bool hb_pair(int t1, int t2) {
    unsigned b1 = 1u << t1, b2 = 1u << t2;
    return ((b1 & ACC_MASK) && (b2 & DON_MASK)) || ((b1 & DON_MASK) && (b2 & ACC_MASK));
}

// Squared distance for the 8 A cutoff test, in FP64 from float inputs with every
// operation rounded separately: the difference of two floats and the product of two
// such differences are exact in double, so the in/out decision at r^2 = 64 is the same
// as the FP64 oracle's (the Vina terms are discontinuous at the cutoff).
__device__ __forceinline__ double cutoff_r2(float ax, float ay, float az, float bx, float by, float bz) {
    double dx = __dsub_rn((double)ax, (double)bx);
    double dy = __dsub_rn((double)ay, (double)by);
    double dz = __dsub_rn((double)az, (double)bz);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// f(r) for every receptor atom in the 27 cells around (px, py, pz): a superset of the atoms
// within the 8 A cutoff (callers keep the cutoff test), cell rows in (z, y) order, each row's
// x cells contiguous in the sorted array, receptor order within a cell.  Nothing for a
// non-finite point (such a pose scores +inf).
template <class F>
__device__ __forceinline__ void near_receptor(const Env& env, float px, float py, float pz, F&& f) {
    if (!env.cell_start || !(isfinite(px) && isfinite(py) && isfinite(pz))) return;
    const int cx = (int)fminf(fmaxf(floorf((px - env.cell_o[0]) * (1.f / CELL_A)), -2.f), (float)env.cdim[0] + 1.f);
    const int cy = (int)fminf(fmaxf(floorf((py - env.cell_o[1]) * (1.f / CELL_A)), -2.f), (float)env.cdim[1] + 1.f);
    const int cz = (int)fminf(fmaxf(floorf((pz - env.cell_o[2]) * (1.f / CELL_A)), -2.f), (float)env.cdim[2] + 1.f);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, env.cdim[0] - 1);
    if (x0 > x1) return;
#pragma unroll 1
    for (int q = 0; q < 9; q++) {                         // the 9 (z, y) rows of cells
        const int y = cy - 1 + q % 3, z = cz - 1 + q / 3;
        if ((unsigned)y >= (unsigned)env.cdim[1] || (unsigned)z >= (unsigned)env.cdim[2]) continue;
        const int row = (z * env.cdim[1] + y) * env.cdim[0];
        const int e = __ldg(env.cell_start + row + x1 + 1);
#pragma unroll 1
        for (int j = __ldg(env.cell_start + row + x0); j < e; j++) f(__ldg(env.rec_cells + j));
    }
}

// Vina pair energy and dE/dd at surface distance d for a heavy pair with the given
// pair flags (vina.h:292-321).
__device__ __forceinline__ float vina_ef(float d, bool hyd, bool hb, float& f) {
    float x1 = d * 2.0f;                    // (d - 0) / 0.5
    float e1 = __expf(-x1 * x1);
    float x2 = (d - 3.0f) * 0.5f;           // (d - 3) / 2
    float e2 = __expf(-x2 * x2);
    float e = -0.035579f * e1 + -0.005156f * e2;
    f = -0.035579f * (e1 * 2.f * (0.f - d) * 4.0f) + -0.005156f * (e2 * 2.f * (3.f - d) * 0.25f);
    if (d < 0.f) {
        e += 0.840245f * d * d;
        f += 0.840245f * 2.f * d;
    }
    if (hyd) {
        if (d <= 0.5f) e += -0.035069f;
        else if (d < 1.5f) { e += -0.035069f * (1.5f - d); f += -0.035069f * -1.0f; }
    }
    if (hb) {
        if (d <= -0.7f) e += -0.587439f;
        else if (d < 0.f) { e += -0.587439f * (0.f - d) / 0.7f; f += -0.587439f * (1.f / -0.7f); }
    }
    return e;
}

// Intra pair term seen from atom a of the pair (a, b), d = x_b - x_a: returns the pair
// energy after the per-pair curl and the scalar s with force on a = -s d.  The reaction
// on b is the negation, bit for bit what the reference computes from b's side (the
// squared distance, radius sum and Vina terms are symmetric).
__device__ __forceinline__ float pair_scalar(float dx, float dy, float dz, float rsum, bool hyd, bool hb, float vcap,
                                             float& s_out) {
    s_out = 0.f;
    const float rr = dx * dx + dy * dy + dz * dz;
    if (!(rr < 64.f)) return 0.f;
    const float rsq = rsqrtf(rr);                       // r and 1/r from one reciprocal root;
    const float rn = rr > 0.f ? rr * rsq : 0.f;         // r is clamped at EPSILON before dividing
    float fdr;
    float ep = vina_ef(rn - rsum, hyd, hb, fdr);
    fdr *= rn < EPS_F ? (1.f / EPS_F) : rsq;
    if (ep > 0.f) {
        const float c = __fdividef(vcap, vcap + ep);
        ep *= c;
        fdr *= c * c;
    }
    s_out = fdr;
    return ep;
}

__device__ __forceinline__ float eval_ef(float d, int t1, int t2, float& f) {
    f = 0.f;
    if (t1 == VN_H || t2 == VN_H) return 0.f;
    return vina_ef(d, hyd_pair(t1, t2), hb_pair(t1, t2), f);
}


// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// ---------------------------------------------------------------- topology staging (TMA)
// A work item's topology blob goes from global to the CTA's shared memory as one bulk
// asynchronous copy on the tensor-memory-access engine (cp.async.bulk, into this CTA only),
// completing on an mbarrier.  Both addresses are 16-byte aligned and the size is a multiple
// of 16 bytes (blobs are padded to 4 words and start at 4-word offsets); every thread waits
// on the barrier's phase with a bounded spin.
constexpr long long STAGE_SPIN = 1LL << 24;

__device__ __forceinline__ uint32_t cta_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void stage_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(cta_smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one thread: arm the barrier for `bytes` and start the copy
__device__ __forceinline__ void stage_bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(cta_smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(cta_smem_addr(dst)), "l"(src), "r"(bytes), "r"(cta_smem_addr(bar)) : "memory");
}

// every thread: wait for the phase with parity `parity`; false after STAGE_SPIN polls
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < STAGE_SPIN; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(cta_smem_addr(bar)), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Stage `words` ints of a blob into sblob: by bulk copy when both ends are 16-byte aligned
// and the size a multiple of 16 bytes, else by the CTA's threads.  Call from every thread
// after a __syncthreads; returns false (in every thread) when the copy did not complete.
__device__ __forceinline__ bool stage_blob(int* sblob, const int* src, int words, uint64_t* bar, uint32_t& phase,
                                           int* s_flag) {
    const bool bulk = ((reinterpret_cast<uintptr_t>(src) | cta_smem_addr(sblob)) & 15u) == 0 && (words & 3) == 0;
    if (!bulk) {
        for (int w = threadIdx.x; w < words; w += blockDim.x) sblob[w] = src[w];
        return true;
    }
    if (threadIdx.x == 0) {
        *s_flag = 0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        stage_bulk_copy(sblob, src, (uint32_t)words * 4u, bar);
    }
    __syncthreads();
    if (!stage_wait(bar, phase & 1u)) atomicOr(s_flag, 1);
    phase++;
    __syncthreads();
    return *s_flag == 0;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
// three warp sums at once: the same butterfly per value (bit-identical to three warp_sum
// calls), interleaved so that their shuffle latencies overlap
__device__ __forceinline__ void warp_sum3(float& a, float& b, float& c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ta = __shfl_xor_sync(FULL, a, o), tb = __shfl_xor_sync(FULL, b, o), tc = __shfl_xor_sync(FULL, c, o);
        a += ta; b += tb; c += tc;
    }
}

// Reduce-scatter of 16 per-lane values: after the call, a[0] of lane L holds the warp
// total of value v = bit4(L)<<3 | bit3(L)<<2 | bit2(L)<<1 | bit1(L).  16 shuffles
// instead of 80 for 16 separate butterflies; the summation order is fixed.
__device__ __forceinline__ void reduce_scatter16(float (&a)[16]) {
    const int lane = lane_id();
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const int o = 16 >> s, m = 16 >> s, h = m >> 1;
        const bool up = lane & o;
#pragma unroll
        for (int j = 0; j < h; j++) {
            float send = up ? a[j] : a[j + h];
            float keep = up ? a[j + h] : a[j];
            a[j] = keep + __shfl_xor_sync(FULL, send, o);
        }
    }
    a[0] += __shfl_xor_sync(FULL, a[0], 1);
}
__device__ __forceinline__ int rs16_lane(int v) {
    return (((v >> 3) & 1) << 4) | (((v >> 2) & 1) << 3) | (((v >> 1) & 1) << 2) | ((v & 1) << 1);
}

// ---------------------------------------------------------------- RNG: Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11.
// Stream: key = (seed lo, seed hi ^ 0x5DEECE66), counter = (chain, ligand, step, purpose).
struct U4 { uint32_t x, y, z, w; };
__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return {c0, c1, c2, c3};
}
__device__ __forceinline__ float u01(uint32_t u) {
    return (float)(u >> 8) * (1.0f / 16777216.0f) + (0.5f / 16777216.0f);
}
enum { P_WHICH = 0, P_TORS = 1, P_METRO = 2, P_LEARN = 3, P_LNORM = 8, P_SPHERE = 16, P_INIT = 256 };
struct Rng {
    uint32_t k0, k1, chain, lig;
    __device__ __forceinline__ U4 draw(uint32_t step, uint32_t purpose) const {
        return philox(chain, lig, step, purpose, k0, k1);
    }
};

// ---------------------------------------------------------------- small math
// fmodf(x, 2 PI) with exact shortcuts for the common magnitudes: |x| < 2 PI is returned
// unchanged and 2 PI <= |x| < 4 PI loses one period, both exactly what fmodf returns
// (the subtraction is exact by Sterbenz's lemma)
__device__ __forceinline__ float fmod_2pi(float x) {
    const float p = 2.f * PI_F, ax = fabsf(x);
    if (ax < p) return x;
    if (ax < 2.f * p) return x > 0.f ? x - p : x + p;
    return fmodf(x, p);
}
__device__ __forceinline__ float normalize_angle(float x) {   // mymath.h:38-47
    x = fmod_2pi(x);
    if (x < -PI_F) x += 2.f * PI_F;
    if (x > PI_F) x -= 2.f * PI_F;
    return x;
}
__device__ __forceinline__ float normalize_angle_2pi(float x) {
    x = fmod_2pi(x);
    if (x < 0.f) x += 2.f * PI_F;
    return x;
}
__device__ __forceinline__ float clamp_by_ranges(float a, const float* r, int n) {  // mymath.h:133-158
#pragma unroll 1
    for (int i = 0; i < n; i++)
        if (a >= r[2 * i] && a <= r[2 * i + 1]) return a;
    float best = a, md = 100.f;
#pragma unroll 1
    for (int i = 0; i < n; i++) {
        float d0 = fabsf(a - r[2 * i]), d1 = fabsf(a - r[2 * i + 1]);
        if (d0 < md) { md = d0; best = r[2 * i]; }
        if (d1 < md) { md = d1; best = r[2 * i + 1]; }
    }
    return best;
}
__device__ __forceinline__ void rotvec_to_quat(float vx, float vy, float vz, float& q0, float& q1, float& q2,
                                               float& q3) {  // quaternion.h:90-107
    float th = sqrtf(vx * vx + vy * vy + vz * vz);
    if (th > EPS_F) {
        float s, c;
        const float h = th * 0.5f;
        if (h <= PI_F) __sincosf(h, &s, &c);     // hardware sine/cosine on [0, pi]
        else sincosf(h, &s, &c);
        const float k = __fdividef(s, th);
        q0 = c;
        q1 = k * vx;
        q2 = k * vy;
        q3 = k * vz;
    } else {
        q0 = 1.f; q1 = q2 = q3 = 0.f;
    }
}
// v' = q v q* expanded (quaternion.h:185-196)
__device__ __forceinline__ void quat_rotate(float q0, float q1, float q2, float q3, float& x, float& y, float& z) {
    float w0 = -q1 * x - q2 * y - q3 * z;
    float w1 = q0 * x + q2 * z - q3 * y;
    float w2 = q0 * y - q1 * z + q3 * x;
    float w3 = q0 * z + q1 * y - q2 * x;
    float nx = -w0 * q1 + w1 * q0 - w2 * q3 + w3 * q2;
    float ny = -w0 * q2 + w1 * q3 + w2 * q0 - w3 * q1;
    float nz = -w0 * q3 - w1 * q2 + w2 * q1 + w3 * q0;
    x = nx; y = ny; z = nz;
}
__device__ __forceinline__ void quat_to_rotvec(float q0, float q1, float q2, float q3, float* v) {
    float th = 2.f * acosf(q0);
    float s = sinf(th * 0.5f);
    if (s > EPS_F) {
        float k = th / s;
        v[0] = q1 * k; v[1] = q2 * k; v[2] = q3 * k;
    } else {
        v[0] = v[1] = v[2] = 0.f;
    }
}

// <M, dR/dv_ind>_F with dR/dv from rotation.h:80-144 (Bailey et al. 2013), the shared
// angle terms precomputed by the caller; M row major.
struct RotGradBasis { float s, c, sdt, omc, vb0, vb1, vb2; };
__device__ __forceinline__ RotGradBasis rot_grad_basis(float vx, float vy, float vz) {
    RotGradBasis B;
    float ang = sqrtf(vx * vx + vy * vy + vz * vz);
    float th;
    if (ang > EPS_F) {
        th = normalize_angle_2pi(ang);
        if (th > PI_F) { th = 2.f * PI_F - th; ang = -ang; }
        B.vb0 = __fdividef(vx, ang); B.vb1 = __fdividef(vy, ang); B.vb2 = __fdividef(vz, ang);
    } else {
        th = 0.f; B.vb0 = B.vb1 = B.vb2 = 0.f;
    }
    __sincosf(th, &B.s, &B.c);                   // th in [0, pi]
    if (th > EPS_F) { B.sdt = __fdividef(B.s, th); B.omc = __fdividef(1.f - B.c, th); }
    else { float t2 = th * th; B.sdt = 1.f - t2 / 6.f; B.omc = th / 2.f - th * t2 / 24.f; }
    return B;
}
__device__ __forceinline__ float frob_drdv(const RotGradBasis& B, int ind, float m0, float m1, float m2, float m3,
                                           float m4, float m5, float m6, float m7, float m8) {
    const float vb[3] = {B.vb0, B.vb1, B.vb2};
    const float vi = ind == 0 ? B.vb0 : (ind == 1 ? B.vb1 : B.vb2);
    const float e0 = ind == 0 ? 1.f : 0.f, e1 = ind == 1 ? 1.f : 0.f, e2 = ind == 2 ? 1.f : 0.f;
    const float e[3] = {e0, e1, e2};
    const float sk[9] = {0.f, -vb[2], vb[1], vb[2], 0.f, -vb[0], -vb[1], vb[0], 0.f};
    const float a = vb[0] * vb[0], bq = vb[1] * vb[1], cq = vb[2] * vb[2];
    const float sk2[9] = {-bq - cq, vb[0] * vb[1], vb[0] * vb[2], vb[0] * vb[1], -a - cq, vb[1] * vb[2],
                          vb[0] * vb[2], vb[1] * vb[2], -a - bq};
    const float vs[3] = {e0 - vi * vb[0], e1 - vi * vb[1], e2 - vi * vb[2]};
    const float ts[9] = {0.f, -vs[2], vs[1], vs[2], 0.f, -vs[0], -vs[1], vs[0], 0.f};
    const float m[9] = {m0, m1, m2, m3, m4, m5, m6, m7, m8};
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int k = i * 3 + j;
            float g = B.c * vi * sk[k] + B.s * vi * sk2[k];
            float mc = e[i] * vb[j] + vb[i] * e[j] - 2.f * vi * vb[i] * vb[j];
            g += B.sdt * ts[k] + B.omc * mc;
            acc += m[k] * g;
        }
    }
    return acc;
}

// ---------------------------------------------------------------- pose slots
// A pose slot in shared memory: [energy, cx, cy, cz, rx, ry, rz, pad] + coords[3N] + dihe[T]
struct Slot {
    float* h;    // header (8 floats)
    float* x;    // coords 3N
    float* d;    // dihedrals T
};
__device__ __forceinline__ Slot slot_at(float* base, int stride, int idx, int natom) {
    float* p = base + idx * stride;
    return {p, p + 8, p + 8 + 3 * natom};
}
__device__ __forceinline__ void slot_copy(Slot dst, Slot src, int natom, int ntors) {
    int n = 8 + 3 * natom + ntors;
#pragma unroll 1
    for (int i = lane_id(); i < n; i += WARP) dst.h[i] = src.h[i];
    __syncwarp();
}

// ---------------------------------------------------------------- grid sample
__device__ __forceinline__ float grid_sample(const GridView& g, int map, float x, float y, float z,
                                             float& gx_, float& gy_, float& gz_) {
    float u0 = (x - g.ox) * g.inv_s, u1 = (y - g.oy) * g.inv_s, u2 = (z - g.oz) * g.inv_s;
    bool c0 = false, c1 = false, c2 = false;
    if (!(u0 >= 0.f)) { u0 = 0.f; c0 = true; }      // also catches NaN
    if (!(u1 >= 0.f)) { u1 = 0.f; c1 = true; }
    if (!(u2 >= 0.f)) { u2 = 0.f; c2 = true; }
    const float h0 = (float)(g.gx - 1), h1 = (float)(g.gy - 1), h2 = (float)(g.gz - 1);
    if (u0 > h0) { u0 = h0; c0 = true; }
    if (u1 > h1) { u1 = h1; c1 = true; }
    if (u2 > h2) { u2 = h2; c2 = true; }
    int i0 = min(max((int)floorf(u0), 0), g.gx - 2);
    int i1 = min(max((int)floorf(u1), 0), g.gy - 2);
    int i2 = min(max((int)floorf(u2), 0), g.gz - 2);
    const float fx = u0 - (float)i0, fy = u1 - (float)i1, fz = u2 - (float)i2;
    // 32-bit indices: the maps of one grid hold fewer than 2^31 values (20 x 81^3 at 30 A)
    const int sy = g.gx, sz = g.gx * g.gy;
    const int base = (map * g.gz + i2) * sz + i1 * sy + i0;
    float v0, v1, v2, v3, v4, v5, v6, v7;
    if (g.use_f16) {
        const __half* m = g.f16 + base;
        v0 = __half2float(m[0]); v1 = __half2float(m[1]);
        v2 = __half2float(m[sy]); v3 = __half2float(m[sy + 1]);
        v4 = __half2float(m[sz]); v5 = __half2float(m[sz + 1]);
        v6 = __half2float(m[sz + sy]); v7 = __half2float(m[sz + sy + 1]);
    } else {
        const float* m = g.f32 + base;
        v0 = __ldg(m); v1 = __ldg(m + 1);
        v2 = __ldg(m + sy); v3 = __ldg(m + sy + 1);
        v4 = __ldg(m + sz); v5 = __ldg(m + sz + 1);
        v6 = __ldg(m + sz + sy); v7 = __ldg(m + sz + sy + 1);
    }
    const float hx = 1.f - fx, hy = 1.f - fy, hz = 1.f - fz;
    const float c00 = v0 * hx + v1 * fx, c10 = v2 * hx + v3 * fx;
    const float c01 = v4 * hx + v5 * fx, c11 = v6 * hx + v7 * fx;
    const float cc0 = c00 * hy + c10 * fy, cc1 = c01 * hy + c11 * fy;
    const float e = cc0 * hz + cc1 * fz;
    const float ddx = ((v1 - v0) * hy + (v3 - v2) * fy) * hz + ((v5 - v4) * hy + (v7 - v6) * fy) * fz;
    const float ddy = (c10 - c00) * hz + (c11 - c01) * fz;
    const float ddz = cc1 - cc0;
    gx_ = c0 ? 0.f : ddx * g.inv_s;
    gy_ = c1 ? 0.f : ddy * g.inv_s;
    gz_ = c2 ? 0.f : ddz * g.inv_s;
    return e;
}

// ---------------------------------------------------------------- intra pairs
// The reference visits every scored pair from both atoms (per-pair curl, energy halved,
// bfgs.cuh:305-352).  Both visits give the same energy and opposite forces, so each
// heavy pair is evaluated once here.  The functions add the intra forces to F (which
// holds the inter forces of the lane's own atoms) and return the lane's share of the
// intra energy.  The kernel is issue bound, so both variants evaluate exactly the listed
// pairs, spread evenly over the lanes.  (A round robin in registers for ligands of up to 32
// atoms, one atom per lane and partners fetched by shuffle, visited every atom pair slot and
// was measured 11 % slower on the plain search of a screen batch, 17 % on the learned one.)

// Pass 1 evaluates every pair once and stores the force scalar of each pair in the warp's
// pair buffer PB; pass 2 gathers F_a += s_p (x_a - x_b) over the atom's pairs in pair-index
// order
__device__ __forceinline__ float intra_buffered(const Topo& T, const float* X, float* F, float vcap, float* PB) {
    const int lane = lane_id();
    float e = 0.f;
#pragma unroll 1
    for (int p = lane; p < T.nprec; p += WARP) {
        const int2 pr = T.prec(p);
        const int i = pr.x & 0xFFF, j = (pr.x >> 12) & 0xFFF;
        float sc;
        e += pair_scalar(X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2],
                         __int_as_float(pr.y), pr.x & PREC_HYD, pr.x & PREC_HB, vcap, sc);
        PB[p] = sc;
    }
    __syncwarp();
#pragma unroll 1
    for (int a = lane; a < T.natom; a += WARP) {
        const float xa = X[3 * a], ya = X[3 * a + 1], za = X[3 * a + 2];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        const int k1 = T.goff(a + 1);
#pragma unroll 1
        for (int k = T.goff(a); k < k1; k++) {
            const int ent = T.gadj(k);
            const float sc = PB[ent & 0xFFFF];
            const int b = ent >> 16;
            fx += sc * (xa - X[3 * b]);
            fy += sc * (ya - X[3 * b + 1]);
            fz += sc * (za - X[3 * b + 2]);
        }
        F[3 * a] += fx; F[3 * a + 1] += fy; F[3 * a + 2] += fz;
    }
    return e;
}

// ligands whose pair list does not fit the pair buffer: pairs spread over the lanes,
// forces accumulated with shared-memory atomic adds
__device__ __forceinline__ float intra_atomic(const Topo& T, const float* X, float* F, float vcap) {
    float e = 0.f;
#pragma unroll 1
    for (int p = lane_id(); p < T.nprec; p += WARP) {
        const int2 pr = T.prec(p);
        const int i = pr.x & 0xFFF, j = (pr.x >> 12) & 0xFFF;
        const float dx = X[3 * j] - X[3 * i], dy = X[3 * j + 1] - X[3 * i + 1], dz = X[3 * j + 2] - X[3 * i + 2];
        float sc;
        e += pair_scalar(dx, dy, dz, __int_as_float(pr.y), pr.x & PREC_HYD, pr.x & PREC_HB, vcap, sc);
        if (sc != 0.f) {
            atomicAdd(F + 3 * i, -sc * dx); atomicAdd(F + 3 * i + 1, -sc * dy); atomicAdd(F + 3 * i + 2, -sc * dz);
            atomicAdd(F + 3 * j, sc * dx); atomicAdd(F + 3 * j + 1, sc * dy); atomicAdd(F + 3 * j + 2, sc * dz);
        }
    }
    return e;
}

// ---------------------------------------------------------------- energy + force
// Fills F (3N, dE/dx per atom) and returns the warp-summed energy (bfgs.cuh:221-394).
// PB: the warp's pair buffer (null when the pair list does not fit it: atomic accumulation).
// A pose with a non-finite coordinate scores +inf.  In the reference such a pose (left by
// a rotation increment whose norm overflows, quaternion.h:90-107 then gives sin(inf))
// escapes every cutoff and box test and gets a finite energy, so Metropolis and the best
// records could take it; +inf makes the line search, the BFGS revert, Metropolis and the
// best records all reject it, and changes nothing for finite poses.
// CELLS: direct sums over the receptor cell list (the refinement and the scoring kernels);
// otherwise over every kept receptor atom (the search kernels, whose default scoring is the
// grid, keep the lighter loop and their register budget).
template <bool CELLS = false>
__device__ __forceinline__ float eval_e_f(const Topo& T, const Env& env, const float* X, float* F, float vcap,
                                          float slope, float* PB) {
    const int lane = lane_id();
    float energy = 0.f;
    bool bad = false;
    // inter + penalty
#pragma unroll 1
    for (int i = lane; i < T.natom; i += WARP) {
        const int ti = T.type(i);
        float fx = 0.f, fy = 0.f, fz = 0.f;
        bad |= !(isfinite(X[3 * i]) && isfinite(X[3 * i + 1]) && isfinite(X[3 * i + 2]));
        if (ti != VN_H) {
            const float px = X[3 * i], py = X[3 * i + 1], pz = X[3 * i + 2];
            float e_atom = 0.f;
            if (env.mode == 1) {
                const int m = T.map_index(i);
                if (m >= 0) e_atom = grid_sample(env.grid, m, px, py, pz, fx, fy, fz);
            } else {
                const float r1 = T.radius(i);
                auto pair = [&](const float4 r) {
                    const float rv0 = r.x - px, rv1 = r.y - py, rv2 = r.z - pz;
                    const double rr = cutoff_r2(r.x, r.y, r.z, px, py, pz);
                    if (rr < 64.0) {
                        const int tj = (int)r.w;
                        float rn = sqrtf((float)rr), fdr;
                        e_atom += eval_ef(rn - (r1 + vdw(tj)), ti, tj, fdr);
                        if (rn < EPS_F) rn = EPS_F;
                        fdr /= rn;
                        fx -= fdr * rv0; fy -= fdr * rv1; fz -= fdr * rv2;
                    }
                };
                if constexpr (CELLS) {
                    near_receptor(env, px, py, pz, pair);
                } else {
                    for (int j = 0; j < env.nrec; j++) pair(__ldg(env.rec + j));
                }
            }
            if (e_atom > 0.f) {
                float s = vcap / (vcap + e_atom);
                e_atom *= s;
                s *= s;
                fx *= s; fy *= s; fz *= s;
            }
            // box penalty (bfgs.cuh:196-218)
            float pen = 0.f;
            if (px < env.box_lo[0]) { pen += env.box_lo[0] - px; fx += -slope; }
            if (px > env.box_hi[0]) { pen += px - env.box_hi[0]; fx += slope; }
            if (py < env.box_lo[1]) { pen += env.box_lo[1] - py; fy += -slope; }
            if (py > env.box_hi[1]) { pen += py - env.box_hi[1]; fy += slope; }
            if (pz < env.box_lo[2]) { pen += env.box_lo[2] - pz; fz += -slope; }
            if (pz > env.box_hi[2]) { pen += pz - env.box_hi[2]; fz += slope; }
            energy += e_atom + pen * slope;
        }
        F[3 * i] = fx; F[3 * i + 1] = fy; F[3 * i + 2] = fz;
    }
    __syncwarp();
    if (PB) energy += intra_buffered(T, X, F, vcap, PB);
    else energy += intra_atomic(T, X, F, vcap);
    // bias (bfgs.cuh:356-388; vina.h:353-400)
    if (env.bias_type != 0 && T.nbias > 0) {
        __syncwarp();
#pragma unroll 1
        for (int i = lane; i < T.natom; i += WARP) {
            const int b0 = T.bias_off(i), b1 = T.bias_off(i + 1);
            if (b0 < b1) {
                float fb0 = 0.f, fb1 = 0.f, fb2 = 0.f;
                const float px = X[3 * i], py = X[3 * i + 1], pz = X[3 * i + 2];
#pragma unroll 1
                for (int b = b0; b < b1; b++) {
                    const float* bp = T.bias() + 5 * b;
                    const float r0 = bp[0] - px, r1 = bp[1] - py, r2 = bp[2] - pz;
                    if (env.bias_type == 1) {
                        float rr = r0 * r0 + r1 * r1 + r2 * r2;
                        float eb = bp[3] * env.bias_k * expf(-rr / bp[4]);
                        fb0 += eb * 2.f * r0 / bp[4];
                        fb1 += eb * 2.f * r1 / bp[4];
                        fb2 += eb * 2.f * r2 / bp[4];
                        energy += eb;
                    } else {
                        float ka = T.type(i) == VN_H ? 0.1f : 30.f;
                        float rn = sqrtf(r0 * r0 + r1 * r1 + r2 * r2);
                        float ei = expf(3.f * (1.f - rn));
                        float eb = bp[3] * env.bias_k * ka / (1.f + ei);
                        float f = -eb * ei / (1.f + ei) * 3.f;
                        fb0 += f * r0 / rn; fb1 += f * r1 / rn; fb2 += f * r2 / rn;
                        energy += eb;
                    }
                }
                F[3 * i] += fb0; F[3 * i + 1] += fb1; F[3 * i + 2] += fb2;
            }
        }
    }
    __syncwarp();
    const float e = warp_sum(energy);
    return __any_sync(FULL, bad) ? INFINITY : e;
}

// Generalised gradient from per-atom dE/dx (bfgs.cuh:69-193).  G has 6+ntors entries.
__device__ __forceinline__ void grad_from_forces(const Topo& T, const Env& env, Slot P, const float* F, float* G) {
    const int lane = lane_id();
    const float* X = P.x;
#pragma unroll 1
    for (int k = lane; k < T.ntors; k += WARP) {
        const int from = T.axis(2 * k), to = T.axis(2 * k + 1);
        const float xt = X[3 * to], yt = X[3 * to + 1], zt = X[3 * to + 2];
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        const int q1 = T.rh_off(k + 1);
#pragma unroll 1
        for (int q = T.rh_off(k); q < q1; q++) {       // heavy rotated atoms, in order
            const int a = T.rheavy(q);
            const float t0 = X[3 * a] - xt, t1 = X[3 * a + 1] - yt, t2 = X[3 * a + 2] - zt;
            const float f0 = F[3 * a], f1 = F[3 * a + 1], f2 = F[3 * a + 2];
            s0 += t1 * f2 - t2 * f1;
            s1 += t2 * f0 - t0 * f2;
            s2 += t0 * f1 - t1 * f0;
        }
        const float a0 = xt - X[3 * from], a1 = yt - X[3 * from + 1], a2 = zt - X[3 * from + 2];
        G[6 + k] = (s0 * a0 + s1 * a1 + s2 * a2) / sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
    }
    if (env.constraint) {
        if (lane < 6) G[lane] = 0.f;
        __syncwarp();
        return;
    }
    float q0, q1, q2, q3;
    rotvec_to_quat(P.h[4], P.h[5], P.h[6], q0, q1, q2, q3);
    q1 = -q1; q2 = -q2; q3 = -q3;
    const float cx = P.h[1], cy = P.h[2], cz = P.h[3];
    float a[16];
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] = 0.f;
#pragma unroll 1
    for (int h = lane; h < T.nheavy; h += WARP) {
        const int i = T.heavy(h);
        float t0 = X[3 * i] - cx, t1 = X[3 * i + 1] - cy, t2 = X[3 * i + 2] - cz;
        quat_rotate(q0, q1, q2, q3, t0, t1, t2);
        const float f0 = F[3 * i], f1 = F[3 * i + 1], f2 = F[3 * i + 2];
        a[0] += f0; a[1] += f1; a[2] += f2;
        a[3] += f0 * t0; a[4] += f0 * t1; a[5] += f0 * t2;
        a[6] += f1 * t0; a[7] += f1 * t1; a[8] += f1 * t2;
        a[9] += f2 * t0; a[10] += f2 * t1; a[11] += f2 * t2;
    }
    reduce_scatter16(a);
    // value v lives in lane rs16_lane(v): gather the 12 sums to every lane
    float s[12];
#pragma unroll
    for (int v = 0; v < 12; v++) s[v] = __shfl_sync(FULL, a[0], rs16_lane(v));
    if (lane < 3) {
        G[lane] = lane == 0 ? s[0] : (lane == 1 ? s[1] : s[2]);
        RotGradBasis B = rot_grad_basis(P.h[4], P.h[5], P.h[6]);
        G[3 + lane] = frob_drdv(B, lane, s[3], s[4], s[5], s[6], s[7], s[8], s[9], s[10], s[11]);
    }
    __syncwarp();
}

template <bool CELLS = false>
__device__ UD_EVAL_ATTR float eval_e_grad(const Topo& T, const Env& env, Slot P, float* F, float* G,
                                             float vcap, float slope, float* PB) {
    float e = eval_e_f<CELLS>(T, env, P.x, F, vcap, slope, PB);
    grad_from_forces(T, env, P, F, G);
    return e;
}

// ---------------------------------------------------------------- kinematics
__device__ __forceinline__ void refresh_center(const Topo& T, Slot P) {
    const int lane = lane_id();
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll 1
    for (int i = lane; i < T.natom; i += WARP) { s0 += P.x[3 * i]; s1 += P.x[3 * i + 1]; s2 += P.x[3 * i + 2]; }
    warp_sum3(s0, s1, s2);
    __syncwarp();
    if (lane == 0) {
        const float n = (float)T.natom;
        P.h[1] = __fdividef(s0, n); P.h[2] = __fdividef(s1, n); P.h[3] = __fdividef(s2, n);
    }
    __syncwarp();
}

// New value of dihedral k after an increment (bfgs.cuh:455-471): returns the applied
// increment and stores the clamped dihedral.
__device__ __forceinline__ float dihedral_step(const Topo& T, Slot P, int k, float incr_raw) {
    const float inc = normalize_angle(incr_raw);
    const int r0 = T.range_off(k), nr = T.range_off(k + 1) - r0;
    const float t = normalize_angle(P.d[k] + inc);
    const float dn = clamp_by_ranges(t, T.ranges() + 2 * r0, nr);
    const float applied = dn - P.d[k];
    P.d[k] = dn;
    return applied;
}

// Rotate the atoms of torsion k by the angle with sine s and cosine c about the axis
// from->to through `to` (bfgs.cuh:477-527); all lanes read the axis atoms directly.
__device__ __forceinline__ void rotate_torsion(const Topo& T, Slot P, int k, float s, float c) {
    const int lane = lane_id();
    const int from = T.axis(2 * k), to = T.axis(2 * k + 1);
    const float tx = P.x[3 * to], ty = P.x[3 * to + 1], tz = P.x[3 * to + 2];
    float ax = tx - P.x[3 * from], ay = ty - P.x[3 * from + 1], az = tz - P.x[3 * from + 2];
    const float l2 = ax * ax + ay * ay + az * az;
    if (!(l2 > EPS_F * EPS_F)) { ax = 1.f; ay = 0.f; az = 0.f; }
    else { const float il = rsqrtf(l2); ax *= il; ay *= il; az *= il; }
    __syncwarp();
    const int q1 = T.rot_off(k + 1);
#pragma unroll 1
    for (int q = T.rot_off(k) + lane; q < q1; q += WARP) {
        const int a = T.rot(q);
        const float v0 = P.x[3 * a] - tx, v1 = P.x[3 * a + 1] - ty, v2 = P.x[3 * a + 2] - tz;
        const float m = (1.f - c) * (ax * v0 + ay * v1 + az * v2);
        const float c0 = ay * v2 - az * v1, c1 = az * v0 - ax * v2, c2 = ax * v1 - ay * v0;
        P.x[3 * a] = c * v0 + m * ax + s * c0 + tx;
        P.x[3 * a + 1] = c * v1 + m * ay + s * c1 + ty;
        P.x[3 * a + 2] = c * v2 + m * az + s * c2 + tz;
    }
    __syncwarp();
}

// One torsion increment as the reference applies it (dihedral, rotation, centre).
__device__ __forceinline__ void apply_dihe(const Topo& T, Slot P, int k, float incr_raw) {
    float applied = 0.f;
    if (lane_id() == 0) applied = dihedral_step(T, P, k, incr_raw);
    applied = __shfl_sync(FULL, applied, 0);
    __syncwarp();
    float s, c;
    __sincosf(applied, &s, &c);
    rotate_torsion(T, P, k, s, c);
    refresh_center(T, P);
}

// pose += alpha * g: torsions in index order, then rotation about the old centre and
// translation (bfgs.cuh:560-618).  SC holds 2 floats per torsion of scratch.  The
// dihedral updates are independent of the coordinates, so they run lane-parallel first;
// the rotations then follow sequentially in index order as in the reference.
__device__ UD_KIN_ATTR void apply_update(const Topo& T, const Env& env, Slot P, const float* G, float alpha,
                                             float* SC) {
    const int lane = lane_id();
#pragma unroll 1
    for (int k = lane; k < T.ntors; k += WARP) {
        const float applied = dihedral_step(T, P, k, G[6 + k] * alpha);
        float s, c;
        __sincosf(applied, &s, &c);       // |applied| <= 2 pi: hardware sine/cosine (~1e-6 abs)
        SC[2 * k] = s;
        SC[2 * k + 1] = c;
    }
    __syncwarp();
#pragma unroll 1
    for (int k = 0; k < T.ntors; k++) rotate_torsion(T, P, k, SC[2 * k], SC[2 * k + 1]);
    if (T.ntors > 0) refresh_center(T, P);
    if (env.constraint) return;
    const float c0x = P.h[1], c0y = P.h[2], c0z = P.h[3];
    const float ncx = c0x + alpha * G[0], ncy = c0y + alpha * G[1], ncz = c0z + alpha * G[2];
    const float rx = G[3] * alpha, ry = G[4] * alpha, rz = G[5] * alpha;
    float q0, q1, q2, q3;
    rotvec_to_quat(rx, ry, rz, q0, q1, q2, q3);
    __syncwarp();
    if (lane == 0) {
        P.h[1] = ncx; P.h[2] = ncy; P.h[3] = ncz;
        P.h[4] = rx; P.h[5] = ry; P.h[6] = rz;
    }
#pragma unroll 1
    for (int i = lane; i < T.natom; i += WARP) {
        float v0 = P.x[3 * i] - c0x, v1 = P.x[3 * i + 1] - c0y, v2 = P.x[3 * i + 2] - c0z;
        quat_rotate(q0, q1, q2, q3, v0, v1, v2);
        P.x[3 * i] = v0 + ncx; P.x[3 * i + 1] = v1 + ncy; P.x[3 * i + 2] = v2 + ncz;
    }
    __syncwarp();
}

// ---------------------------------------------------------------- optimiser
struct Work {        // per-warp scratch in shared memory
    float* F;        // 3N
    float* g;        // D
    float* gn;       // D
    float* p;        // D
    float* y;        // D
    float* mhy;      // D
    float* sc;       // 2T torsion sine/cosine scratch
    double* H;       // D(D+1)/2, packed upper triangle: H[i + j(j+1)/2], i <= j
    float* pb;       // pair buffer (one float per scored pair), or null
};

__device__ __forceinline__ float gdot(const float* a, const float* b, int n) {
    float s = 0.f;
#pragma unroll 1
    for (int i = lane_id(); i < n; i += WARP) s += a[i] * b[i];
    return warp_sum(s);
}

// out = -H v for the packed symmetric H (bfgs.cuh:413-428), lane per row
__device__ __forceinline__ void minus_hv(const double* H, const float* v, float* out, int dim) {
#pragma unroll 1
    for (int i = lane_id(); i < dim; i += WARP) {
        double s = 0.0;
        const int ri = i * (i + 1) / 2;
#pragma unroll 1
        for (int j = 0; j < i; j++) s += H[ri + j] * (double)v[j];              // H[j,i], j < i
#pragma unroll 1
        for (int j = i, cj = ri; j < dim; cj += j + 1, j++) s += H[cj + i] * (double)v[j];  // H[i,j], j >= i
        out[i] = (float)(-s);
    }
    __syncwarp();
}

constexpr int LS_TRIALS = 0, LS_INIT = 1, LS_MOVE = 2;
// Backtracking Armijo line search (bfgs.cuh:623-670).  Trial poses go to Pn.  The start of a
// BFGS run goes through the same call sites, so that the search loop holds one copy of the
// evaluation and kinematics code: mode LS_INIT only evaluates Px (energy, gradient into
// W.g); LS_MOVE sets Pn = Px moved by W.p (a learned MC move) and evaluates Pn likewise.
template <bool CELLS = false>
__device__ UD_LS_ATTR float line_search(const Topo& T, const Env& env, Slot Px, Slot Pn, const Work& W,
                                             int dim, float e0, float vcap, float slope, float& alpha_out,
                                             int& n_eval, int mode) {
    const bool start = mode != LS_TRIALS;
    float alpha = 1.f, e_new = 0.f;
    const float pg = start ? 0.f : gdot(W.p, W.g, dim);
#pragma unroll 1
    for (int trial = 0; trial < LS_STEPS; trial++) {
        if (mode != LS_INIT) {
            slot_copy(Pn, Px, T.natom, T.ntors);
            apply_update(T, env, Pn, W.p, alpha, W.sc);
        }
        const Slot Q = mode == LS_INIT ? Px : Pn;
        e_new = eval_e_grad<CELLS>(T, env, Q, W.F, start ? W.g : W.gn, vcap, slope, W.pb);
        n_eval++;
        if (start || e_new - e0 < 1e-4f * alpha * pg) break;
        alpha *= 0.5f;
    }
    alpha_out = alpha;
    return e_new;
}

// BFGS on the pose in slot ix (bfgs.cuh:729-829).  Uses slots ix / ialt / iori; returns
// the slot index holding the result, whose header[0] is the final energy.
template <bool CELLS = false>
__device__ __forceinline__ int bfgs(const Topo& T, const Env& env, float* slots, int stride, int ix, int ialt,
                                    int iori, const Work& W, int max_steps, float vcap, float slope, int& n_eval,
                                    int move_from = -1) {
    const int lane = lane_id();
    const int dim = 6 + T.ntors;
    const Slot X = slot_at(slots, stride, ix, T.natom);
    float E_ori = 0.f, E = 0.f;
    const int ntri = dim * (dim + 1) / 2;
    int cur = ix, alt = ialt;
    // step -1 evaluates the start pose and sets H = I; move_from >= 0: the start pose is
    // that slot moved by W.p (line_search LS_MOVE)
#pragma unroll 1
    for (int step = -1; step < max_steps; step++) {
        if (step >= 0) minus_hv(W.H, W.g, W.p, dim);          // p = -H g
        float alpha;
        const bool mv = step < 0 && move_from >= 0;
        const float E1 = line_search<CELLS>(T, env, slot_at(slots, stride, mv ? move_from : cur, T.natom),
                                     slot_at(slots, stride, mv ? cur : alt, T.natom), W, dim, E, vcap, slope, alpha,
                                     n_eval, step < 0 ? (mv ? LS_MOVE : LS_INIT) : LS_TRIALS);
        if (step < 0) {
            E_ori = E = E1;
#pragma unroll 1
            for (int i = lane; i < ntri; i += WARP) W.H[i] = 0.0;
            __syncwarp();
#pragma unroll 1
            for (int i = lane; i < dim; i += WARP) W.H[i + i * (i + 1) / 2] = 1.0;
            slot_copy(slot_at(slots, stride, iori, T.natom), X, T.natom, T.ntors);
            continue;
        }
        // y = g_new - g with g.g (the reference tests the old gradient), y.p and y.y in one
        // reduction (each the same sum as a separate dot product)
        float gg = 0.f, yp = 0.f, yy = 0.f;
#pragma unroll 1
        for (int i = lane; i < dim; i += WARP) {
            const float gi = W.g[i], yi = W.gn[i] - gi;
            W.y[i] = yi;
            gg += gi * gi;
            yp += yi * W.p[i];
            yy += yi * yi;
        }
        warp_sum3(gg, yp, yy);
        __syncwarp();
        E = E1;
        const int t = cur; cur = alt; alt = t;                // x := x_new
        if (sqrtf(gg) < 1e-5f) break;
#pragma unroll 1
        for (int i = lane; i < dim; i += WARP) W.g[i] = W.gn[i];
        __syncwarp();
        if (step == 0 && fabsf(yy) > EPS_F) {
#pragma unroll 1
            for (int i = lane; i < dim; i += WARP) W.H[i + i * (i + 1) / 2] = (double)(alpha * yp / yy);
            __syncwarp();
        }
        if (alpha * yp < EPS_F) continue;
        minus_hv(W.H, W.y, W.mhy, dim);
        const double yhy = -(double)gdot(W.y, W.mhy, dim);
        const double r = 1.0 / ((double)alpha * (double)yp);
        const double a = alpha;
        const double c1 = a * r, c2 = a * a * (r * r * yhy + r);
        int i = lane, j = 0;                                  // idx = i + j(j+1)/2, i <= j
        while (i > j) { j++; i -= j; }
#pragma unroll 1
        for (int idx = lane; idx < ntri; idx += WARP) {
            const double pi = W.p[i], pj = W.p[j];
            W.H[idx] += c1 * ((double)W.mhy[i] * pj + (double)W.mhy[j] * pi) + c2 * pi * pj;
            i += WARP;
            while (i > j) { j++; i -= j; }
        }
        __syncwarp();
    }
    const Slot R = slot_at(slots, stride, cur, T.natom);
    if (E > E_ori) {
        E = E_ori;
        slot_copy(R, slot_at(slots, stride, iori, T.natom), T.natom, T.ntors);
    }
    if (lane == 0) R.h[0] = E;
    __syncwarp();
    return cur;
}

// ---------------------------------------------------------------- MC moves
__device__ __forceinline__ float gyration_radius(const Topo& T, Slot P) {
    const int lane = lane_id();
    float s = 0.f;
#pragma unroll 1
    for (int h = lane; h < T.nheavy; h += WARP) {
        const int i = T.heavy(h);
        const float d0 = P.x[3 * i] - P.h[1], d1 = P.x[3 * i + 1] - P.h[2], d2 = P.x[3 * i + 2] - P.h[3];
        s += d0 * d0 + d1 * d1 + d2 * d2;
    }
    s = warp_sum(s);
    const float r = T.nheavy > 0 ? sqrtf(s / T.nheavy) : 0.f;
    return r > 0.f ? r : 1.f;
}

__device__ __forceinline__ void rand_in_sphere(const Rng& rng, uint32_t step, float& v0, float& v1, float& v2) {
#pragma unroll 1
    for (int a = 0; a < 64; a++) {
        const U4 u = rng.draw(step, P_SPHERE + a);
        v0 = (u01(u.x) - 0.5f) * 2.f;
        v1 = (u01(u.y) - 0.5f) * 2.f;
        v2 = (u01(u.z) - 0.5f) * 2.f;
        if (sqrtf(v0 * v0 + v1 * v1 + v2 * v2) < 1.f) return;
    }
    v0 = v1 = v2 = 0.f;
}

// mc.cu:146-256 with the counter-based generator
__device__ __forceinline__ void mutate(const Topo& T, const Env& env, const Rng& rng, uint32_t step, Slot P) {
    const int lane = lane_id();
    const float amp = 2.f;
    const int nmut = 2 + T.ntors;
    const U4 u = rng.draw(step, P_WHICH);
    int which;
    if (env.constraint) which = nmut < 3 ? 3 : 2 + (int)(u.x % (uint32_t)(nmut - 2));
    else which = (int)(u.x % (uint32_t)nmut);
    if (which == 0) {
        float v0, v1, v2;
        rand_in_sphere(rng, step, v0, v1, v2);
        const float c0 = P.h[1], c1 = P.h[2], c2 = P.h[3];
        const float t0 = fminf(fmaxf(amp * v0 + c0, env.box_lo[0]), env.box_hi[0]);
        const float t1 = fminf(fmaxf(amp * v1 + c1, env.box_lo[1]), env.box_hi[1]);
        const float t2 = fminf(fmaxf(amp * v2 + c2, env.box_lo[2]), env.box_hi[2]);
        const float d0 = t0 - c0, d1 = t1 - c1, d2 = t2 - c2;
        __syncwarp();
        if (lane == 0) { P.h[1] = c0 + d0; P.h[2] = c1 + d1; P.h[3] = c2 + d2; }
#pragma unroll 1
        for (int i = lane; i < T.natom; i += WARP) {
            P.x[3 * i] += d0; P.x[3 * i + 1] += d1; P.x[3 * i + 2] += d2;
        }
        __syncwarp();
    } else if (which == 1) {
        float v0, v1, v2;
        rand_in_sphere(rng, step, v0, v1, v2);
        const float a = gyration_radius(T, P);
        const float rv0 = amp / a * v0, rv1 = amp / a * v1, rv2 = amp / a * v2;
        float q0, q1, q2, q3;
        rotvec_to_quat(rv0, rv1, rv2, q0, q1, q2, q3);
        const float cx = P.h[1], cy = P.h[2], cz = P.h[3];
        __syncwarp();
        if (lane == 0) { P.h[4] = rv0; P.h[5] = rv1; P.h[6] = rv2; }
#pragma unroll 1
        for (int i = lane; i < T.natom; i += WARP) {
            float t0 = P.x[3 * i] - cx, t1 = P.x[3 * i + 1] - cy, t2 = P.x[3 * i + 2] - cz;
            quat_rotate(q0, q1, q2, q3, t0, t1, t2);
            P.x[3 * i] = t0 + cx; P.x[3 * i + 1] = t1 + cy; P.x[3 * i + 2] = t2 + cz;
        }
        __syncwarp();
    } else if (which - 2 < T.ntors) {
        const int k = which - 2;
        const U4 w = rng.draw(step, P_TORS);
        const float r0 = u01(w.x), r1 = u01(w.y);
        const int b = T.range_off(k), nr = T.range_off(k + 1) - b;
        int ir = (int)ceilf(r0 * nr - 1.f);
        ir = ir < 0 ? 0 : (ir > nr - 1 ? nr - 1 : ir);
        const float lo = T.ranges()[2 * (b + ir)], hi = T.ranges()[2 * (b + ir) + 1];
        const float a = lo + (hi - lo) * r1 - P.d[k];
        apply_dihe(T, P, k, a);
    }
}

// initial randomisation (mc.cu:18-104); G is D floats of scratch, SC 2T floats
__device__ __forceinline__ void randomize(const Topo& T, const Env& env, const Rng& rng, int chain, int nchain,
                                          Slot P, float* G, float* SC) {
    const int lane = lane_id();
    if (lane == 0) {
        const U4 u = rng.draw(0, P_INIT);
        if (env.constraint) {
            G[0] = G[1] = G[2] = G[3] = G[4] = G[5] = 0.f;
        } else {
            const float s = chain + 0.5f, n = (float)nchain;
            const float r = sqrtf(s / n), R = sqrtf(1.f - s / n);
            const float al = 2.f * PI_F * s / 1.4142136f, be = 2.f * PI_F * s / 1.5337512f;
            if (env.bias_type == 2) {
                G[0] = G[1] = G[2] = 0.f;
            } else {
                G[0] = (env.box_lo[0] + (env.box_hi[0] - env.box_lo[0]) * u01(u.x)) - P.h[1];
                G[1] = (env.box_lo[1] + (env.box_hi[1] - env.box_lo[1]) * u01(u.y)) - P.h[2];
                G[2] = (env.box_lo[2] + (env.box_hi[2] - env.box_lo[2]) * u01(u.z)) - P.h[3];
            }
            quat_to_rotvec(r * sinf(al), r * cosf(al), R * sinf(be), R * cosf(be), G + 3);
        }
    }
#pragma unroll 1
    for (int k = lane; k < T.ntors; k += WARP) {
        const U4 u = rng.draw(0, P_INIT + 1 + k);
        const int b = T.range_off(k), nr = T.range_off(k + 1) - b;
        int j = (int)(u01(u.x) * nr);
        if (j > nr - 1) j = nr - 1;
        const float lo = T.ranges()[2 * (b + j)], hi = T.ranges()[2 * (b + j) + 1];
        G[6 + k] = lo + (hi - lo) * u01(u.y) - P.d[k];
    }
    __syncwarp();
    apply_update(T, env, P, G, 1.f, SC);
}

}  // namespace ud
