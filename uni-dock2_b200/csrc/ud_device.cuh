// ud_device.cuh -- warp-level device code of the B200 docking engine.
//
// One warp owns one pose (a Monte Carlo chain, a BFGS job or a scoring job).  The
// ligand topology is a packed blob of 32-bit words (layout below) that kernels stage
// in shared memory; pose state (coordinates, dihedrals, centre, last rotation
// increment) lives in per-warp shared memory slots.  All per-atom work is strided
// over the 32 lanes; scalar decisions are taken by lane 0 and broadcast by shuffle;
// reductions are xor-butterflies, so results are deterministic.
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
enum BlobHdr {
    H_NATOM = 0, H_NTORS, H_NHEAVY, H_NPAIR, H_NROT, H_NRANGE, H_NBIAS,
    H_TYPES, H_AXIS, H_RANGE_OFF, H_RANGES, H_ROT_OFF, H_ROT, H_PAIR_OFF, H_PAIRS,
    H_BIAS_OFF, H_BIAS, H_HEAVY, H_X0, H_D0, H_C0, H_TOTAL, H_RES1, H_RES2,
    H_WORDS = 24
};

struct Topo {
    int natom, ntors, nheavy, nbias;
    const int* types;
    const int* axis;
    const int* range_off;
    const float* ranges;
    const int* rot_off;
    const int* rot;
    const int* pair_off;
    const int* pairs;
    const int* bias_off;
    const float* bias;
    const int* heavy;
};

__device__ __forceinline__ Topo topo_view(const int* b) {
    Topo t;
    t.natom = b[H_NATOM];
    t.ntors = b[H_NTORS];
    t.nheavy = b[H_NHEAVY];
    t.nbias = b[H_NBIAS];
    t.types = b + b[H_TYPES];
    t.axis = b + b[H_AXIS];
    t.range_off = b + b[H_RANGE_OFF];
    t.ranges = reinterpret_cast<const float*>(b + b[H_RANGES]);
    t.rot_off = b + b[H_ROT_OFF];
    t.rot = b + b[H_ROT];
    t.pair_off = b + b[H_PAIR_OFF];
    t.pairs = b + b[H_PAIRS];
    t.bias_off = b + b[H_BIAS_OFF];
    t.bias = reinterpret_cast<const float*>(b + b[H_BIAS]);
    t.heavy = b + b[H_HEAVY];
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
    signed char map_of_type[NT + 3];
};

__constant__ float c_vdw[NT] = {1.1f, 1.92f, 1.9f, 1.9f, 1.8f, 1.8f, 1.8f, 1.8f, 1.7f, 1.7f, 1.7f,
                                1.7f, 1.5f, 2.2f, 2.1f, 2.0f, 1.8f, 2.0f, 2.2f, 2.3f, 1.2f};
// bit t set: hydrophobic / acceptor / donor (src/score/vina.h:125-137)
constexpr unsigned HYD_MASK = (1u << 2) | (1u << 12) | (1u << 16) | (1u << 17) | (1u << 18);
constexpr unsigned ACC_MASK = (1u << 6) | (1u << 7) | (1u << 10) | (1u << 11);
constexpr unsigned DON_MASK = (1u << 5) | (1u << 7) | (1u << 9) | (1u << 11) | (1u << 20);

__device__ __forceinline__ float vdw(int t) { return c_vdw[t]; }

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

// Vina pair energy and dE/dd for surface distance d (vina.h:292-321).
__device__ __forceinline__ float eval_ef(float d, int t1, int t2, float& f) {
    f = 0.f;
    if (t1 == VN_H || t2 == VN_H) return 0.f;
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
    unsigned b1 = 1u << t1, b2 = 1u << t2;
    if ((b1 & HYD_MASK) && (b2 & HYD_MASK)) {
        if (d <= 0.5f) e += -0.035069f;
        else if (d < 1.5f) { e += -0.035069f * (1.5f - d); f += -0.035069f * -1.0f; }
    }
    if (((b1 & ACC_MASK) && (b2 & DON_MASK)) || ((b1 & DON_MASK) && (b2 & ACC_MASK))) {
        if (d <= -0.7f) e += -0.587439f;
        else if (d < 0.f) { e += -0.587439f * (0.f - d) / 0.7f; f += -0.587439f * (1.f / -0.7f); }
    }
    return e;
}

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
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
enum { P_WHICH = 0, P_TORS = 1, P_METRO = 2, P_SPHERE = 16, P_INIT = 256 };
struct Rng {
    uint32_t k0, k1, chain, lig;
    __device__ __forceinline__ U4 draw(uint32_t step, uint32_t purpose) const {
        return philox(chain, lig, step, purpose, k0, k1);
    }
};

// ---------------------------------------------------------------- small math
__device__ __forceinline__ float normalize_angle(float x) {   // mymath.h:38-47
    x = fmodf(x, 2.f * PI_F);
    if (x < -PI_F) x += 2.f * PI_F;
    if (x > PI_F) x -= 2.f * PI_F;
    return x;
}
__device__ __forceinline__ float normalize_angle_2pi(float x) {
    x = fmodf(x, 2.f * PI_F);
    if (x < 0.f) x += 2.f * PI_F;
    return x;
}
__device__ __forceinline__ float clamp_by_ranges(float a, const float* r, int n) {  // mymath.h:133-158
    for (int i = 0; i < n; i++)
        if (a >= r[2 * i] && a <= r[2 * i + 1]) return a;
    float best = a, md = 100.f;
    for (int i = 0; i < n; i++) {
        float d0 = fabsf(a - r[2 * i]), d1 = fabsf(a - r[2 * i + 1]);
        if (d0 < md) { md = d0; best = r[2 * i]; }
        if (d1 < md) { md = d1; best = r[2 * i + 1]; }
    }
    return best;
}
__device__ __forceinline__ void rotvec_to_quat(float vx, float vy, float vz, float* q) {  // quaternion.h:90-107
    float th = sqrtf(vx * vx + vy * vy + vz * vz);
    if (th > EPS_F) {
        float s, c;
        sincosf(th * 0.5f, &s, &c);
        q[0] = c;
        q[1] = s * (vx / th);
        q[2] = s * (vy / th);
        q[3] = s * (vz / th);
    } else {
        q[0] = 1.f; q[1] = q[2] = q[3] = 0.f;
    }
}
// v' = q v q* expanded (quaternion.h:185-196)
__device__ __forceinline__ void quat_rotate(const float* q, float& x, float& y, float& z) {
    float w0 = -q[1] * x - q[2] * y - q[3] * z;
    float w1 = q[0] * x + q[2] * z - q[3] * y;
    float w2 = q[0] * y - q[1] * z + q[3] * x;
    float w3 = q[0] * z + q[1] * y - q[2] * x;
    // (w) * conj(q)
    float nx = -w0 * q[1] + w1 * q[0] - w2 * q[3] + w3 * q[2];
    float ny = -w0 * q[2] + w1 * q[3] + w2 * q[0] - w3 * q[1];
    float nz = -w0 * q[3] - w1 * q[2] + w2 * q[1] + w3 * q[0];
    x = nx; y = ny; z = nz;
}
__device__ __forceinline__ void quat_to_rotvec(const float* q, float* v) {  // quaternion.h:115-130
    float th = 2.f * acosf(q[0]);
    float s = sinf(th * 0.5f);
    if (s > EPS_F) {
        float k = th / s;
        v[0] = q[1] * k; v[1] = q[2] * k; v[2] = q[3] * k;
    } else {
        v[0] = v[1] = v[2] = 0.f;
    }
}

// dR/dv_ind (rotation.h:80-144) contracted with a 3x3 matrix (row major)
__device__ float frob_drdv(const float* mat, float vx, float vy, float vz, int ind) {
    float v[3] = {vx, vy, vz};
    float ang = sqrtf(vx * vx + vy * vy + vz * vz);
    float th, vb[3];
    if (ang > EPS_F) {
        th = normalize_angle_2pi(ang);
        if (th > PI_F) { th = 2.f * PI_F - th; ang = -ang; }
        vb[0] = v[0] / ang; vb[1] = v[1] / ang; vb[2] = v[2] / ang;
    } else {
        th = 0.f; vb[0] = vb[1] = vb[2] = 0.f;
    }
    float s, c;
    sincosf(th, &s, &c);
    float e[3] = {0.f, 0.f, 0.f};
    e[ind] = 1.f;
    float sk[9] = {0.f, -vb[2], vb[1], vb[2], 0.f, -vb[0], -vb[1], vb[0], 0.f};
    float a = vb[0] * vb[0], b = vb[1] * vb[1], cc = vb[2] * vb[2];
    float sk2[9] = {-b - cc, vb[0] * vb[1], vb[0] * vb[2], vb[0] * vb[1], -a - cc, vb[1] * vb[2],
                    vb[0] * vb[2], vb[1] * vb[2], -a - b};
    float sdt, omc;
    if (th > EPS_F) { sdt = s / th; omc = (1.f - c) / th; }
    else { float t2 = th * th; sdt = 1.f - t2 / 6.f; omc = th / 2.f - th * t2 / 24.f; }
    float vs[3] = {e[0] - vb[ind] * vb[0], e[1] - vb[ind] * vb[1], e[2] - vb[ind] * vb[2]};
    float ts[9] = {0.f, -vs[2], vs[1], vs[2], 0.f, -vs[0], -vs[1], vs[0], 0.f};
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            int k = i * 3 + j;
            float g = c * vb[ind] * sk[k] + s * vb[ind] * sk2[k];
            float mc = e[i] * vb[j] + vb[i] * e[j] - 2.f * vb[ind] * vb[i] * vb[j];
            g += sdt * ts[k] + omc * mc;
            acc += mat[k] * g;
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
    float* p = base + (size_t)idx * stride;
    return {p, p + 8, p + 8 + 3 * natom};
}
__device__ __forceinline__ int slot_stride(int natom, int ntors) {
    return (8 + 3 * natom + ntors + 3) & ~3;
}
__device__ __forceinline__ void slot_copy(Slot dst, Slot src, int natom, int ntors) {
    int n = 8 + 3 * natom + ntors;
    for (int i = lane_id(); i < n; i += WARP) dst.h[i] = src.h[i];
    __syncwarp();
}

// ---------------------------------------------------------------- grid sample
__device__ __forceinline__ float grid_sample(const GridView& g, int map, float x, float y, float z,
                                             float& gx_, float& gy_, float& gz_) {
    float u[3] = {(x - g.ox) * g.inv_s, (y - g.oy) * g.inv_s, (z - g.oz) * g.inv_s};
    int dim[3] = {g.gx, g.gy, g.gz};
    int i0[3];
    float fr[3];
    bool cl[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float v = u[a];
        cl[a] = false;
        if (!(v >= 0.f)) { v = 0.f; cl[a] = true; }      // also catches NaN
        float hi = (float)(dim[a] - 1);
        if (v > hi) { v = hi; cl[a] = true; }
        int i = (int)floorf(v);
        if (i > dim[a] - 2) i = dim[a] - 2;
        if (i < 0) i = 0;
        i0[a] = i;
        fr[a] = v - (float)i;
    }
    size_t npt = (size_t)g.gx * g.gy * g.gz;
    size_t base = (size_t)map * npt + ((size_t)i0[2] * g.gy + i0[1]) * g.gx + i0[0];
    size_t sy = g.gx, sz = (size_t)g.gx * g.gy;
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
    float fx = fr[0], fy = fr[1], fz = fr[2];
    float hx = 1.f - fx, hy = 1.f - fy, hz = 1.f - fz;
    float c00 = v0 * hx + v1 * fx, c10 = v2 * hx + v3 * fx;
    float c01 = v4 * hx + v5 * fx, c11 = v6 * hx + v7 * fx;
    float c0 = c00 * hy + c10 * fy, c1 = c01 * hy + c11 * fy;
    float e = c0 * hz + c1 * fz;
    float ddx = ((v1 - v0) * hy + (v3 - v2) * fy) * hz + ((v5 - v4) * hy + (v7 - v6) * fy) * fz;
    float ddy = (c10 - c00) * hz + (c11 - c01) * fz;
    float ddz = c1 - c0;
    gx_ = cl[0] ? 0.f : ddx * g.inv_s;
    gy_ = cl[1] ? 0.f : ddy * g.inv_s;
    gz_ = cl[2] ? 0.f : ddz * g.inv_s;
    return e;
}

// ---------------------------------------------------------------- energy + force
// Fills F (3N, dE/dx per atom) and returns the warp-summed energy (bfgs.cuh:221-394).
__device__ float eval_e_f(const Topo& T, const Env& env, const float* X, float* F, float vcap, float slope) {
    const int lane = lane_id();
    float energy = 0.f;
    // inter + penalty
    for (int i = lane; i < T.natom; i += WARP) {
        int ti = T.types[i];
        float fx = 0.f, fy = 0.f, fz = 0.f;
        if (ti != VN_H) {
            float px = X[3 * i], py = X[3 * i + 1], pz = X[3 * i + 2];
            float e_atom = 0.f;
            if (env.mode == 1) {
                int m = env.map_of_type[ti];
                if (m >= 0) e_atom = grid_sample(env.grid, m, px, py, pz, fx, fy, fz);
            } else {
                float r1 = vdw(ti);
                for (int j = 0; j < env.nrec; j++) {
                    float4 r = __ldg(env.rec + j);
                    float rv0 = r.x - px, rv1 = r.y - py, rv2 = r.z - pz;
                    double rr = cutoff_r2(r.x, r.y, r.z, px, py, pz);
                    if (rr < 64.0) {
                        int tj = (int)r.w;
                        float rn = sqrtf((float)rr), fdr;
                        e_atom += eval_ef(rn - (r1 + vdw(tj)), ti, tj, fdr);
                        if (rn < EPS_F) rn = EPS_F;
                        fdr /= rn;
                        fx -= fdr * rv0; fy -= fdr * rv1; fz -= fdr * rv2;
                    }
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
    // intra (bfgs.cuh:305-352)
    float e_intra = 0.f;
    for (int i = lane; i < T.natom; i += WARP) {
        int ti = T.types[i];
        float r1 = vdw(ti);
        float xi = X[3 * i], yi = X[3 * i + 1], zi = X[3 * i + 2];
        float fx = 0.f, fy = 0.f, fz = 0.f, ea = 0.f;
        int k1 = T.pair_off[i + 1];
        for (int k = T.pair_off[i]; k < k1; k++) {
            int j = T.pairs[k];
            float rv0 = X[3 * j] - xi, rv1 = X[3 * j + 1] - yi, rv2 = X[3 * j + 2] - zi;
            float rr = rv0 * rv0 + rv1 * rv1 + rv2 * rv2;
            if (rr < 64.f) {
                int tj = T.types[j];
                float rn = sqrtf(rr), fdr;
                float ep = eval_ef(rn - (r1 + vdw(tj)), ti, tj, fdr);
                if (rn < EPS_F) rn = EPS_F;
                fdr /= rn;
                float px = -fdr * rv0, py = -fdr * rv1, pz = -fdr * rv2;
                if (ep > 0.f) {
                    float s = vcap / (vcap + ep);
                    ep *= s;
                    s *= s;
                    px *= s; py *= s; pz *= s;
                }
                ea += ep;
                fx += px; fy += py; fz += pz;
            }
        }
        e_intra += ea;
        F[3 * i] += fx; F[3 * i + 1] += fy; F[3 * i + 2] += fz;
    }
    energy += 0.5f * e_intra;
    // bias (bfgs.cuh:356-388; vina.h:353-400)
    if (env.bias_type != 0 && T.nbias > 0) {
        __syncwarp();
        for (int i = lane; i < T.natom; i += WARP) {
            int b0 = T.bias_off[i], b1 = T.bias_off[i + 1];
            if (b0 < b1) {
                float fb[3] = {0.f, 0.f, 0.f};
                float px = X[3 * i], py = X[3 * i + 1], pz = X[3 * i + 2];
                for (int b = b0; b < b1; b++) {
                    const float* bp = T.bias + 5 * b;
                    float r[3] = {bp[0] - px, bp[1] - py, bp[2] - pz};
                    if (env.bias_type == 1) {
                        float rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                        float eb = bp[3] * env.bias_k * expf(-rr / bp[4]);
                        fb[0] += eb * 2.f * r[0] / bp[4];
                        fb[1] += eb * 2.f * r[1] / bp[4];
                        fb[2] += eb * 2.f * r[2] / bp[4];
                        energy += eb;
                    } else {
                        float ka = T.types[i] == VN_H ? 0.1f : 30.f;
                        float rn = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                        float ei = expf(3.f * (1.f - rn));
                        float eb = bp[3] * env.bias_k * ka / (1.f + ei);
                        float f = -eb * ei / (1.f + ei) * 3.f;
                        fb[0] += f * r[0] / rn; fb[1] += f * r[1] / rn; fb[2] += f * r[2] / rn;
                        energy += eb;
                    }
                }
                F[3 * i] += fb[0]; F[3 * i + 1] += fb[1]; F[3 * i + 2] += fb[2];
            }
        }
    }
    __syncwarp();
    return warp_sum(energy);
}

// Generalised gradient from per-atom dE/dx (bfgs.cuh:69-193).  G has 6+ntors entries.
__device__ void grad_from_forces(const Topo& T, const Env& env, Slot P, const float* F, float* G) {
    const int lane = lane_id();
    const float* X = P.x;
    for (int k = lane; k < T.ntors; k += WARP) {
        int from = T.axis[2 * k], to = T.axis[2 * k + 1];
        float xt = X[3 * to], yt = X[3 * to + 1], zt = X[3 * to + 2];
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        int q1 = T.rot_off[k + 1];
        for (int q = T.rot_off[k]; q < q1; q++) {
            int a = T.rot[q];
            if (T.types[a] == VN_H) continue;
            float t0 = X[3 * a] - xt, t1 = X[3 * a + 1] - yt, t2 = X[3 * a + 2] - zt;
            float f0 = F[3 * a], f1 = F[3 * a + 1], f2 = F[3 * a + 2];
            s0 += t1 * f2 - t2 * f1;
            s1 += t2 * f0 - t0 * f2;
            s2 += t0 * f1 - t1 * f0;
        }
        float a0 = xt - X[3 * from], a1 = yt - X[3 * from + 1], a2 = zt - X[3 * from + 2];
        G[6 + k] = (s0 * a0 + s1 * a1 + s2 * a2) / sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
    }
    if (env.constraint) {
        if (lane < 6) G[lane] = 0.f;
        __syncwarp();
        return;
    }
    float q[4];
    rotvec_to_quat(P.h[4], P.h[5], P.h[6], q);
    q[1] = -q[1]; q[2] = -q[2]; q[3] = -q[3];
    float cx = P.h[1], cy = P.h[2], cz = P.h[3];
    float fs0 = 0.f, fs1 = 0.f, fs2 = 0.f;
    float m[9];
#pragma unroll
    for (int j = 0; j < 9; j++) m[j] = 0.f;
    for (int h = lane; h < T.nheavy; h += WARP) {
        int i = T.heavy[h];
        float t0 = X[3 * i] - cx, t1 = X[3 * i + 1] - cy, t2 = X[3 * i + 2] - cz;
        quat_rotate(q, t0, t1, t2);
        float f0 = F[3 * i], f1 = F[3 * i + 1], f2 = F[3 * i + 2];
        fs0 += f0; fs1 += f1; fs2 += f2;
        m[0] += f0 * t0; m[1] += f0 * t1; m[2] += f0 * t2;
        m[3] += f1 * t0; m[4] += f1 * t1; m[5] += f1 * t2;
        m[6] += f2 * t0; m[7] += f2 * t1; m[8] += f2 * t2;
    }
    fs0 = warp_sum(fs0); fs1 = warp_sum(fs1); fs2 = warp_sum(fs2);
#pragma unroll
    for (int j = 0; j < 9; j++) m[j] = warp_sum(m[j]);
    if (lane == 0) { G[0] = fs0; G[1] = fs1; G[2] = fs2; }
    if (lane < 3) G[3 + lane] = frob_drdv(m, P.h[4], P.h[5], P.h[6], lane);
    __syncwarp();
}

__device__ __forceinline__ float eval_e_grad(const Topo& T, const Env& env, Slot P, float* F, float* G,
                                             float vcap, float slope) {
    float e = eval_e_f(T, env, P.x, F, vcap, slope);
    grad_from_forces(T, env, P, F, G);
    return e;
}

// ---------------------------------------------------------------- kinematics
// One torsion increment (bfgs.cuh:443-549); the centre is refreshed by the caller.
__device__ void apply_dihe(const Topo& T, Slot P, int k, float incr_raw) {
    const int lane = lane_id();
    float incr = 0.f, ax = 0.f, ay = 0.f, az = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
    if (lane == 0) {
        float inc = normalize_angle(incr_raw);
        int r0 = T.range_off[k], nr = T.range_off[k + 1] - r0;
        float t = normalize_angle(P.d[k] + inc);
        float dn = clamp_by_ranges(t, T.ranges + 2 * r0, nr);
        incr = dn - P.d[k];
        P.d[k] = dn;
        int from = T.axis[2 * k], to = T.axis[2 * k + 1];
        tx = P.x[3 * to]; ty = P.x[3 * to + 1]; tz = P.x[3 * to + 2];
        ax = tx - P.x[3 * from]; ay = ty - P.x[3 * from + 1]; az = tz - P.x[3 * from + 2];
        float l = sqrtf(ax * ax + ay * ay + az * az);
        if (l <= EPS_F) { ax = 1.f; ay = 0.f; az = 0.f; }
        else { ax /= l; ay /= l; az /= l; }
    }
    incr = __shfl_sync(FULL, incr, 0);
    ax = __shfl_sync(FULL, ax, 0); ay = __shfl_sync(FULL, ay, 0); az = __shfl_sync(FULL, az, 0);
    tx = __shfl_sync(FULL, tx, 0); ty = __shfl_sync(FULL, ty, 0); tz = __shfl_sync(FULL, tz, 0);
    float s, c;
    sincosf(incr, &s, &c);
    int q1 = T.rot_off[k + 1];
    for (int q = T.rot_off[k] + lane; q < q1; q += WARP) {
        int a = T.rot[q];
        float v0 = P.x[3 * a] - tx, v1 = P.x[3 * a + 1] - ty, v2 = P.x[3 * a + 2] - tz;
        float m = (1.f - c) * (ax * v0 + ay * v1 + az * v2);
        float c0 = ay * v2 - az * v1, c1 = az * v0 - ax * v2, c2 = ax * v1 - ay * v0;
        P.x[3 * a] = c * v0 + m * ax + s * c0 + tx;
        P.x[3 * a + 1] = c * v1 + m * ay + s * c1 + ty;
        P.x[3 * a + 2] = c * v2 + m * az + s * c2 + tz;
    }
    __syncwarp();
}

__device__ void refresh_center(const Topo& T, Slot P) {
    const int lane = lane_id();
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int i = lane; i < T.natom; i += WARP) { s0 += P.x[3 * i]; s1 += P.x[3 * i + 1]; s2 += P.x[3 * i + 2]; }
    s0 = warp_sum(s0); s1 = warp_sum(s1); s2 = warp_sum(s2);
    if (lane == 0) {
        P.h[1] = s0 / T.natom; P.h[2] = s1 / T.natom; P.h[3] = s2 / T.natom;
    }
    __syncwarp();
}

// pose += alpha * g: torsions in index order, then rotation about the old centre and
// translation (bfgs.cuh:560-618)
__device__ void apply_update(const Topo& T, const Env& env, Slot P, const float* G, float alpha) {
    for (int k = 0; k < T.ntors; k++) apply_dihe(T, P, k, G[6 + k] * alpha);
    if (T.ntors > 0) refresh_center(T, P);
    if (env.constraint) return;
    const int lane = lane_id();
    float c0x = P.h[1], c0y = P.h[2], c0z = P.h[3];
    float ncx = c0x + alpha * G[0], ncy = c0y + alpha * G[1], ncz = c0z + alpha * G[2];
    float rx = G[3] * alpha, ry = G[4] * alpha, rz = G[5] * alpha;
    float q[4];
    rotvec_to_quat(rx, ry, rz, q);
    __syncwarp();
    if (lane == 0) {
        P.h[1] = ncx; P.h[2] = ncy; P.h[3] = ncz;
        P.h[4] = rx; P.h[5] = ry; P.h[6] = rz;
    }
    for (int i = lane; i < T.natom; i += WARP) {
        float v0 = P.x[3 * i] - c0x, v1 = P.x[3 * i + 1] - c0y, v2 = P.x[3 * i + 2] - c0z;
        quat_rotate(q, v0, v1, v2);
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
    double* H;       // D(D+1)/2
};

__device__ __forceinline__ float gdot(const float* a, const float* b, int n) {
    float s = 0.f;
    for (int i = lane_id(); i < n; i += WARP) s += a[i] * b[i];
    return warp_sum(s);
}

__device__ __forceinline__ int tri(int i, int j) { return i <= j ? i + j * (j + 1) / 2 : j + i * (i + 1) / 2; }

// Backtracking Armijo line search (bfgs.cuh:623-670).  Trial poses go to Pn.
__device__ float line_search(const Topo& T, const Env& env, Slot Px, Slot Pn, const Work& W, int dim,
                             float e0, float vcap, float slope, float& alpha_out, int& n_eval) {
    float alpha = 1.f, e_new = 0.f;
    float pg = gdot(W.p, W.g, dim);
    for (int trial = 0; trial < LS_STEPS; trial++) {
        slot_copy(Pn, Px, T.natom, T.ntors);
        apply_update(T, env, Pn, W.p, alpha);
        e_new = eval_e_grad(T, env, Pn, W.F, W.gn, vcap, slope);
        n_eval++;
        if (e_new - e0 < 1e-4f * alpha * pg) break;
        alpha *= 0.5f;
    }
    alpha_out = alpha;
    return e_new;
}

// BFGS on the pose in slot ix (bfgs.cuh:729-829).  Uses slots in / alt / ori; returns
// the slot index holding the result, whose header[0] is the final energy.
__device__ int bfgs(const Topo& T, const Env& env, float* slots, int stride, int ix, int ialt, int iori,
                    const Work& W, int max_steps, float vcap, float slope, int& n_eval) {
    const int lane = lane_id();
    const int dim = 6 + T.ntors;
    Slot X = slot_at(slots, stride, ix, T.natom);
    float E_ori = eval_e_grad(T, env, X, W.F, W.g, vcap, slope);
    n_eval++;
    float E = E_ori;
    const int ntri = dim * (dim + 1) / 2;
    for (int i = lane; i < ntri; i += WARP) W.H[i] = 0.0;
    __syncwarp();
    for (int i = lane; i < dim; i += WARP) W.H[i + i * (i + 1) / 2] = 1.0;
    slot_copy(slot_at(slots, stride, iori, T.natom), X, T.natom, T.ntors);
    int cur = ix, alt = ialt;
    for (int step = 0; step < max_steps; step++) {
        // p = -H g
        for (int i = lane; i < dim; i += WARP) {
            double s = 0.0;
            for (int j = 0; j < dim; j++) s += W.H[tri(i, j)] * (double)W.g[j];
            W.p[i] = (float)(-s);
        }
        __syncwarp();
        float alpha;
        Slot Pc = slot_at(slots, stride, cur, T.natom);
        Slot Pa = slot_at(slots, stride, alt, T.natom);
        float E1 = line_search(T, env, Pc, Pa, W, dim, E, vcap, slope, alpha, n_eval);
        for (int i = lane; i < dim; i += WARP) W.y[i] = W.gn[i] - W.g[i];
        __syncwarp();
        E = E1;
        int t = cur; cur = alt; alt = t;       // x := x_new
        float gg = gdot(W.g, W.g, dim);
        if (sqrtf(gg) < 1e-5f) break;
        for (int i = lane; i < dim; i += WARP) W.g[i] = W.gn[i];
        __syncwarp();
        if (step == 0) {
            float yy = gdot(W.y, W.y, dim);
            if (fabsf(yy) > EPS_F) {
                float yp0 = gdot(W.y, W.p, dim);
                for (int i = lane; i < dim; i += WARP) W.H[i + i * (i + 1) / 2] = (double)(alpha * yp0 / yy);
                __syncwarp();
            }
        }
        float yp = gdot(W.y, W.p, dim);
        if (alpha * yp < EPS_F) continue;
        for (int i = lane; i < dim; i += WARP) {
            double s = 0.0;
            for (int j = 0; j < dim; j++) s += W.H[tri(i, j)] * (double)W.y[j];
            W.mhy[i] = (float)(-s);
        }
        __syncwarp();
        double yhy = -(double)gdot(W.y, W.mhy, dim);
        double r = 1.0 / ((double)alpha * (double)yp);
        double a = alpha;
        double c2 = a * a * (r * r * yhy + r);
        for (int idx = lane; idx < ntri; idx += WARP) {
            // packed upper triangle: idx = i + j(j+1)/2 with i <= j
            int j = (int)((sqrtf(8.f * idx + 1.f) - 1.f) * 0.5f);
            while (j * (j + 1) / 2 > idx) j--;
            while ((j + 1) * (j + 2) / 2 <= idx) j++;
            int i = idx - j * (j + 1) / 2;
            double pi = W.p[i], pj = W.p[j];
            W.H[idx] += a * r * ((double)W.mhy[i] * pj + (double)W.mhy[j] * pi) + c2 * pi * pj;
        }
        __syncwarp();
    }
    Slot R = slot_at(slots, stride, cur, T.natom);
    if (E > E_ori) {
        E = E_ori;
        slot_copy(R, slot_at(slots, stride, iori, T.natom), T.natom, T.ntors);
    }
    if (lane == 0) R.h[0] = E;
    __syncwarp();
    return cur;
}

// ---------------------------------------------------------------- MC moves
__device__ float gyration_radius(const Topo& T, Slot P) {
    const int lane = lane_id();
    float s = 0.f;
    for (int h = lane; h < T.nheavy; h += WARP) {
        int i = T.heavy[h];
        float d0 = P.x[3 * i] - P.h[1], d1 = P.x[3 * i + 1] - P.h[2], d2 = P.x[3 * i + 2] - P.h[3];
        s += d0 * d0 + d1 * d1 + d2 * d2;
    }
    s = warp_sum(s);
    float r = T.nheavy > 0 ? sqrtf(s / T.nheavy) : 0.f;
    return r > 0.f ? r : 1.f;
}

__device__ __forceinline__ void rand_in_sphere(const Rng& rng, uint32_t step, float* v) {
    for (int a = 0; a < 64; a++) {
        U4 u = rng.draw(step, P_SPHERE + a);
        v[0] = (u01(u.x) - 0.5f) * 2.f;
        v[1] = (u01(u.y) - 0.5f) * 2.f;
        v[2] = (u01(u.z) - 0.5f) * 2.f;
        if (sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) < 1.f) return;
    }
    v[0] = v[1] = v[2] = 0.f;
}

// mc.cu:146-256 with the counter-based generator
__device__ void mutate(const Topo& T, const Env& env, const Rng& rng, uint32_t step, Slot P) {
    const int lane = lane_id();
    const float amp = 2.f;
    int nmut = 2 + T.ntors;
    U4 u = rng.draw(step, P_WHICH);
    int which;
    if (env.constraint) which = nmut < 3 ? 3 : 2 + (int)(u.x % (uint32_t)(nmut - 2));
    else which = (int)(u.x % (uint32_t)nmut);
    if (which == 0) {
        float v[3];
        rand_in_sphere(rng, step, v);
        float d[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float c = P.h[1 + a];
            float t = amp * v[a] + c;
            if (t > env.box_hi[a]) t = env.box_hi[a];
            if (t < env.box_lo[a]) t = env.box_lo[a];
            d[a] = t - c;
        }
        __syncwarp();
        if (lane == 0) { P.h[1] += d[0]; P.h[2] += d[1]; P.h[3] += d[2]; }
        for (int i = lane; i < T.natom; i += WARP) {
            P.x[3 * i] += d[0]; P.x[3 * i + 1] += d[1]; P.x[3 * i + 2] += d[2];
        }
        __syncwarp();
    } else if (which == 1) {
        float v[3];
        rand_in_sphere(rng, step, v);
        float a = gyration_radius(T, P);
        float rv[3] = {amp / a * v[0], amp / a * v[1], amp / a * v[2]};
        float q[4];
        rotvec_to_quat(rv[0], rv[1], rv[2], q);
        float cx = P.h[1], cy = P.h[2], cz = P.h[3];
        __syncwarp();
        if (lane == 0) { P.h[4] = rv[0]; P.h[5] = rv[1]; P.h[6] = rv[2]; }
        for (int i = lane; i < T.natom; i += WARP) {
            float t0 = P.x[3 * i] - cx, t1 = P.x[3 * i + 1] - cy, t2 = P.x[3 * i + 2] - cz;
            quat_rotate(q, t0, t1, t2);
            P.x[3 * i] = t0 + cx; P.x[3 * i + 1] = t1 + cy; P.x[3 * i + 2] = t2 + cz;
        }
        __syncwarp();
    } else if (which - 2 < T.ntors) {
        int k = which - 2;
        U4 w = rng.draw(step, P_TORS);
        float r0 = u01(w.x), r1 = u01(w.y);
        int b = T.range_off[k], nr = T.range_off[k + 1] - b;
        int ir = (int)ceilf(r0 * nr - 1.f);
        ir = ir < 0 ? 0 : (ir > nr - 1 ? nr - 1 : ir);
        float lo = T.ranges[2 * (b + ir)], hi = T.ranges[2 * (b + ir) + 1];
        float a = lo + (hi - lo) * r1 - P.d[k];
        apply_dihe(T, P, k, a);
        refresh_center(T, P);
    }
}

// initial randomisation (mc.cu:18-104); G is D floats of scratch
__device__ void randomize(const Topo& T, const Env& env, const Rng& rng, int chain, int nchain, Slot P, float* G) {
    const int lane = lane_id();
    if (lane == 0) {
        U4 u = rng.draw(0, P_INIT);
        if (env.constraint) {
            G[0] = G[1] = G[2] = G[3] = G[4] = G[5] = 0.f;
        } else {
            float s = chain + 0.5f, n = (float)nchain;
            float r = sqrtf(s / n), R = sqrtf(1.f - s / n);
            float al = 2.f * PI_F * s / 1.4142136f, be = 2.f * PI_F * s / 1.5337512f;
            float q[4] = {r * sinf(al), r * cosf(al), R * sinf(be), R * cosf(be)};
            if (env.bias_type == 2) {
                G[0] = G[1] = G[2] = 0.f;
            } else {
                G[0] = (env.box_lo[0] + (env.box_hi[0] - env.box_lo[0]) * u01(u.x)) - P.h[1];
                G[1] = (env.box_lo[1] + (env.box_hi[1] - env.box_lo[1]) * u01(u.y)) - P.h[2];
                G[2] = (env.box_lo[2] + (env.box_hi[2] - env.box_lo[2]) * u01(u.z)) - P.h[3];
            }
            quat_to_rotvec(q, G + 3);
        }
    }
    for (int k = lane; k < T.ntors; k += WARP) {
        U4 u = rng.draw(0, P_INIT + 1 + k);
        int b = T.range_off[k], nr = T.range_off[k + 1] - b;
        int j = (int)(u01(u.x) * nr);
        if (j > nr - 1) j = nr - 1;
        float lo = T.ranges[2 * (b + j)], hi = T.ranges[2 * (b + j) + 1];
        G[6 + k] = lo + (hi - lo) * u01(u.y) - P.d[k];
    }
    __syncwarp();
    apply_update(T, env, P, G, 1.f);
}

}  // namespace ud
