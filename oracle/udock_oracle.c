/*
 * udock_oracle.c -- CPU restatement of the Uni-Dock2 docking-engine hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * udock_oracle.h for the list of reference functions restated here; each
 * function below cites the reference file:line it follows (paths relative to
 * unidock/unidock_engine/ in the reference project).
 *
 * Arithmetic type: orc_real = double (default) or float (-DORC_FLOAT).
 * Constants follow the reference: PI = Real(3.1415927) (src/myutils/common.h:44),
 * EPSILON = numeric_limits<Real>::epsilon() (common.h:12).
 */
#include "udock_oracle.h"
#include <math.h>
#include <float.h>
#include <string.h>
#include <stdlib.h>

typedef orc_real R;

#ifdef ORC_FLOAT
#define EPS FLT_EPSILON
#define RSQRT(x) sqrtf(x)
#else
#define EPS DBL_EPSILON
#define RSQRT(x) sqrt(x)
#endif
#define PI_R ((R)3.1415927)
#define PHI_R ((R)1.4142136)
#define PSI_R ((R)1.5337512)

#define VN_H 0
#define NTYPES 21

/* src/constants/constants.h:21-43 */
static const double VDW[NTYPES] = {1.1, 1.92, 1.9, 1.9, 1.8, 1.8, 1.8, 1.8, 1.7, 1.7, 1.7,
                                   1.7, 1.5, 2.2, 2.1, 2.0, 1.8, 2.0, 2.2, 2.3, 1.2};

R orc_vdw_radius(int t) { return (R)VDW[t]; }

/* src/score/vina.h:125-141 */
static int is_hydrophobic(int t) { return t == 2 || t == 12 || t == 16 || t == 17 || t == 18; }
static int is_acceptor(int t) { return t == 6 || t == 7 || t == 10 || t == 11; }
static int is_donor(int t) { return t == 5 || t == 7 || t == 9 || t == 11 || t == 20; }
static int hbond_possible(int a, int b) {
    return (is_acceptor(a) && is_donor(b)) || (is_donor(a) && is_acceptor(b));
}

/* src/myutils/mymath.h:210-214 */
R orc_gaussian(R d, R offset, R width, R* out_f) {
    R t = (d - offset) / width;
    R e = exp(-(t * t));
    *out_f = e * 2 * (offset - d) / width / width;
    return e;
}

/* src/score/vina.h:151-163 */
static R slope_interp(R lo, R hi, R x, R* out_f) {
    if (x <= lo) { *out_f = 0; return 1; }
    if (x >= hi) { *out_f = 0; return 0; }
    *out_f = 1 / (lo - hi);
    return (hi - x) / (hi - lo);
}

/* src/score/vina.h:174-199 weights */
#define W_G1 ((R)-0.035579)
#define W_G2 ((R)-0.005156)
#define W_REP ((R)0.840245)
#define W_HYD ((R)-0.035069)
#define W_HB ((R)-0.587439)
#define W_CONF ((R)0.05846)

/* src/score/vina.h:292-321 */
R orc_eval_ef(R d, int t1, int t2, R* out_f) {
    R e = 0, f = 0;
    *out_f = 0;
    if (t1 == VN_H || t2 == VN_H) return 0;
    e += W_G1 * orc_gaussian(d, 0, (R)0.5, &f);
    *out_f += W_G1 * f;
    e += W_G2 * orc_gaussian(d, 3, 2, &f);
    *out_f += W_G2 * f;
    if (d < 0) { e += W_REP * d * d; *out_f += W_REP * 2 * d; }
    if (is_hydrophobic(t1) && is_hydrophobic(t2)) {
        e += W_HYD * slope_interp((R)0.5, (R)1.5, d, &f);
        *out_f += W_HYD * f;
    }
    if (hbond_possible(t1, t2)) {
        e += W_HB * slope_interp((R)-0.7, 0, d, &f);
        *out_f += W_HB * f;
    }
    return e;
}

/* unweighted single terms (vina.h:215-268): 0 gauss1, 1 gauss2, 2 repulsion,
   3 hydrophobic ramp, 4 hbond ramp */
R orc_vina_term(int which, R d, R* f) {
    switch (which) {
    case 0: return orc_gaussian(d, 0, (R)0.5, f);
    case 1: return orc_gaussian(d, 3, 2, f);
    case 2: if (d >= 0) { *f = 0; return 0; } *f = 2 * d; return d * d;
    case 3: return slope_interp((R)0.5, (R)1.5, d, f);
    default: return slope_interp((R)-0.7, 0, d, f);
    }
}

/* src/score/vina.h:332-350 */
void orc_eval_decomp(R d, int t1, int t2, R out[5]) {
    R f;
    out[0] = out[1] = out[2] = out[3] = out[4] = 0;
    if (t1 == VN_H || t2 == VN_H) return;
    out[0] = W_G1 * orc_gaussian(d, 0, (R)0.5, &f);
    out[1] = W_G2 * orc_gaussian(d, 3, 2, &f);
    out[2] = d < 0 ? W_REP * d * d : 0;
    if (is_hydrophobic(t1) && is_hydrophobic(t2)) out[3] = W_HYD * slope_interp((R)0.5, (R)1.5, d, &f);
    if (hbond_possible(t1, t2)) out[4] = W_HB * slope_interp((R)-0.7, 0, d, &f);
}

/* src/score/vina.h:353-365 */
R orc_eval_ef_pos(const R* r, R v, R r2, R* out_f) {
    R rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    R e = v * exp(-rr / r2);
    out_f[0] += e * 2 * r[0] / r2;
    out_f[1] += e * 2 * r[1] / r2;
    out_f[2] += e * 2 * r[2] / r2;
    return e;
}

/* src/score/vina.h:382-400 */
R orc_eval_ef_zalign(const R* r, R a_qt, int t, R* out_f) {
    const R s_a = 3, c_a = 1;
    R k_a = (t == VN_H ? (R)0.1 : (R)30);
    R rn = RSQRT(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    R ei = exp(s_a * (c_a - rn));
    R e = a_qt * k_a / (1 + ei);
    R f = -e * ei / (1 + ei) * s_a;
    out_f[0] += f * r[0] / rn;
    out_f[1] += f * r[1] / rn;
    out_f[2] += f * r[2] / rn;
    return e;
}

/* ---------------- math helpers: src/myutils/mymath.h ---------------- */
static R norm3(const R* a) { return RSQRT(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static R dot3(const R* a, const R* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const R* a, const R* b, R* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* mymath.h:38-47 */
R orc_normalize_angle(R x) {
    x = fmod(x, 2 * PI_R);
    if (x < -PI_R) x += 2 * PI_R;
    if (x > PI_R) x -= 2 * PI_R;
    return x;
}
/* mymath.h:24-30 */
R orc_normalize_angle_2pi(R x) {
    x = fmod(x, 2 * PI_R);
    if (x < 0) x += 2 * PI_R;
    return x;
}
/* mymath.h:133-158 */
R orc_clamp_by_ranges(R ang, const R* ranges, int nrange) {
    for (int i = 0; i < nrange; i++)
        if (ang >= ranges[2 * i] && ang <= ranges[2 * i + 1]) return ang;
    R closest = ang, mind = 100;
    for (int i = 0; i < nrange; i++) {
        R d0 = fabs(ang - ranges[2 * i]);
        R d1 = fabs(ang - ranges[2 * i + 1]);
        if (d0 < mind) { mind = d0; closest = ranges[2 * i]; }
        if (d1 < mind) { mind = d1; closest = ranges[2 * i + 1]; }
    }
    return closest;
}
/* mymath.h:103-110 */
R orc_get_radian_in_ranges(const R* ranges, int nrange, const R* rand2) {
    int i = (int)ceil(rand2[0] * nrange - 1);
    if (i < 0) i = 0;
    if (i > nrange - 1) i = nrange - 1;
    R from = ranges[2 * i], to = ranges[2 * i + 1];
    return from + (to - from) * rand2[1];
}
/* src/cuda/common.cuh:59-68 */
R orc_get_real_within_by_int(int c, R min, R max, int n) {
    R v = (R)(c % n) * (max - min) / n + min;
    if (v < min) return min;
    if (v > max) return max;
    return v;
}

/* ---------------- geometry: src/geometry/quaternion.h, rotation.h ---------------- */
/* quaternion.h:46-52 */
void orc_quaternion_multiply_left(const R* q2, R* q1) {
    R t[4] = {q1[0], q1[1], q1[2], q1[3]};
    q1[0] = q2[0] * t[0] - q2[1] * t[1] - q2[2] * t[2] - q2[3] * t[3];
    q1[1] = q2[0] * t[1] + q2[1] * t[0] + q2[2] * t[3] - q2[3] * t[2];
    q1[2] = q2[0] * t[2] - q2[1] * t[3] + q2[2] * t[0] + q2[3] * t[1];
    q1[3] = q2[0] * t[3] + q2[1] * t[2] - q2[2] * t[1] + q2[3] * t[0];
}
/* quaternion.h:59-69 */
void orc_quaternion_normalize(R* q) {
    R s = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (fabs(s - 1) < EPS) return;
    R a = RSQRT(s);
    for (int i = 0; i < 4; i++) q[i] /= a;
}
/* quaternion.h:90-107 */
void orc_rotvec_to_quaternion(R* q, const R* rv) {
    R th = norm3(rv);
    if (th > EPS) {
        R s = sin(th / 2);
        q[0] = cos(th / 2);
        q[1] = s * (rv[0] / th);
        q[2] = s * (rv[1] / th);
        q[3] = s * (rv[2] / th);
    } else {
        q[0] = 1; q[1] = q[2] = q[3] = 0;
    }
}
/* quaternion.h:115-130 */
void orc_quaternion_to_rotvec(R* v, const R* q) {
    R th = 2 * acos(q[0]);
    R s = sin(th / 2);
    if (s > EPS) {
        R k = th / s;
        v[0] = q[1] * k; v[1] = q[2] * k; v[2] = q[3] * k;
    } else {
        v[0] = v[1] = v[2] = 0;
    }
}
/* quaternion.h:185-196: v' = q v q* */
void orc_rotate_vec_by_quaternion(R* v, const R* q) {
    R v4[4] = {0, v[0], v[1], v[2]};
    R qc[4] = {q[0], -q[1], -q[2], -q[3]};
    orc_quaternion_multiply_left(q, v4);
    orc_quaternion_multiply_left(v4, qc);
    v[0] = qc[1]; v[1] = qc[2]; v[2] = qc[3];
}
/* rotation.h:56-66 */
void orc_rotate_vec_by_rodrigues(R* v, const R* axis, R theta) {
    R t[3];
    R c = cos(theta), s = sin(theta);
    R m = (1 - c) * dot3(axis, v);
    cross3(axis, v, t);
    v[0] = c * v[0] + m * axis[0] + s * t[0];
    v[1] = c * v[1] + m * axis[1] + s * t[1];
    v[2] = c * v[2] + m * axis[2] + s * t[2];
}
/* rotation.h:19-46 with norm=true */
static void rotvec_to_axis_angle_norm(R* out, const R* rv) {
    R angle = norm3(rv);
    if (angle > EPS) {
        out[0] = orc_normalize_angle_2pi(angle);
        if (out[0] > PI_R) { out[0] = 2 * PI_R - out[0]; angle = -angle; }
        out[1] = rv[0] / angle; out[2] = rv[1] / angle; out[3] = rv[2] / angle;
    } else {
        out[0] = out[1] = out[2] = out[3] = 0;
    }
}
static void skew(R* m, const R* v) {
    m[0] = 0; m[1] = -v[2]; m[2] = v[1];
    m[3] = v[2]; m[4] = 0; m[5] = -v[0];
    m[6] = -v[1]; m[7] = v[0]; m[8] = 0;
}
static void skew_sq(R* m, const R* v) {
    R v01 = v[0] * v[1], v12 = v[1] * v[2], v02 = v[0] * v[2];
    R a = v[0] * v[0], b = v[1] * v[1], c = v[2] * v[2];
    m[0] = -b - c; m[1] = v01; m[2] = v02;
    m[3] = v01; m[4] = -a - c; m[5] = v12;
    m[6] = v02; m[7] = v12; m[8] = -a - b;
}
static void outer3(const R* a, const R* b, R* o) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) o[i * 3 + j] = a[i] * b[j];
}
/* rotation.h:80-144 (Bailey et al. 2013 / Mirzaei et al. 2012) */
void orc_grad_rot_over_vec(R* g, const R* v, int ind) {
    R aa[4];
    rotvec_to_axis_angle_norm(aa, v);
    R th = aa[0];
    const R* vb = aa + 1;
    R e[3] = {0, 0, 0};
    e[ind] = 1;
    R s = sin(th), c = cos(th);
    R sk[9], sk2[9];
    skew(sk, vb);
    skew_sq(sk2, vb);
    for (int j = 0; j < 9; j++) g[j] = c * vb[ind] * sk[j] + s * vb[ind] * sk2[j];
    R sdt, omcdt;
    if (th > EPS) { sdt = s / th; omcdt = (1 - c) / th; }
    else { R t2 = th * th; sdt = 1 - t2 / 6; omcdt = th / 2 - th * t2 / 24; }
    R vs[3];
    for (int j = 0; j < 3; j++) vs[j] = e[j] - vb[ind] * vb[j];
    R ts[9], mc[9] = {0}, mt[9];
    skew(ts, vs);
    outer3(e, vb, mt);
    for (int j = 0; j < 9; j++) mc[j] += mt[j];
    outer3(vb, e, mt);
    for (int j = 0; j < 9; j++) mc[j] += mt[j];
    outer3(vb, vb, mt);
    for (int j = 0; j < 9; j++) mc[j] -= 2 * vb[ind] * mt[j];
    for (int j = 0; j < 9; j++) g[j] += sdt * ts[j] + omcdt * mc[j];
}

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ---------------- */
#define PH_M0 0xD2511F53u
#define PH_M1 0xCD9E8D57u
#define PH_W0 0x9E3779B9u
#define PH_W1 0xBB67AE85u
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)PH_M0 * c0;
        uint64_t p1 = (uint64_t)PH_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += PH_W0;
        k1 += PH_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
/* uniform in (0,1): top 24 bits, centred in their bucket; exact in float */
float orc_u01(uint32_t u) { return (float)(u >> 8) * (1.0f / 16777216.0f) + (0.5f / 16777216.0f); }

/* RNG stream layout shared with the CUDA path:
   key = (seed lo, seed hi ^ 0x5DEECE66), ctr = (chain, ligand, step, purpose) */
enum { P_WHICH = 0, P_TORS = 1, P_METRO = 2, P_SPHERE = 16, P_INIT = 256 };
static void rng4(const orc_search_param* sp, int chain, uint32_t step, uint32_t purpose, uint32_t out[4]) {
    uint32_t key[2] = {(uint32_t)sp->seed, (uint32_t)(sp->seed >> 32) ^ 0x5DEECE66u};
    uint32_t ctr[4] = {(uint32_t)chain, (uint32_t)sp->lig_uid, step, purpose};
    orc_philox4x32_10(ctr, key, out);
}

/* Squared distance for the 8 A cutoff test (r^2 < 64, vina.h:206), computed in double
   with separately rounded operations.  For float-valued inputs it is exact up to the
   final additions and identical to the engine's, so both take the same side of the
   discontinuous cutoff. */
static double cut_r2(double ax, double ay, double az, double bx, double by, double bz) {
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    return (dx * dx + dy * dy) + dz * dz;
}

/* ---------------- grid model (no reference counterpart) ---------------- */
/* map value for probe type t at point p = the reference inter pair sum for one atom of
   type t at p, without curl: sum_j eval_ef(|p-r_j| - (R_t+R_j)), |p-r_j|^2 < 64
   (semantics of src/cuda/bfgs.cuh:252-273) */
void orc_grid_build(int nrec, const R* rx, const int* rt, int nmaps, const int* map_types,
                    const R* origin, R spacing, const int* gd, R* out) {
    size_t npt = (size_t)gd[0] * gd[1] * gd[2];
#pragma omp parallel for schedule(static)
    for (long long idx = 0; idx < (long long)npt; idx++) {
        int ix = (int)(idx % gd[0]);
        int iy = (int)((idx / gd[0]) % gd[1]);
        int iz = (int)(idx / ((size_t)gd[0] * gd[1]));
        /* grid points are float (one rounded fma), as the engine lays them out */
        float p[3] = {fmaf((float)ix, (float)spacing, (float)origin[0]), fmaf((float)iy, (float)spacing, (float)origin[1]),
                      fmaf((float)iz, (float)spacing, (float)origin[2])};
        for (int m = 0; m < nmaps; m++) {
            int t = map_types[m];
            R acc = 0, f;
            for (int j = 0; j < nrec; j++) {
                if (rt[j] == VN_H) continue;
                double rr = cut_r2(rx[3 * j], rx[3 * j + 1], rx[3 * j + 2], p[0], p[1], p[2]);
                if (rr < 64) {
                    R r = RSQRT((R)rr);
                    acc += orc_eval_ef(r - (orc_vdw_radius(t) + orc_vdw_radius(rt[j])), t, rt[j], &f);
                }
            }
            out[(size_t)m * npt + idx] = acc;
        }
    }
}

/* trilinear value + analytic gradient of map `map` at x; coordinates outside the
   grid are clamped to it and the gradient along a clamped axis is zero */
R orc_grid_interp(const orc_env* env, int map, const R* x, R* g) {
    const int* gd = env->gdim;
    int i0[3];
    R fr[3];
    int clamped[3];
    for (int a = 0; a < 3; a++) {
        R u = (x[a] - env->origin[a]) / env->spacing;
        clamped[a] = 0;
        if (!(u >= 0)) { u = 0; clamped[a] = 1; }   /* also catches NaN */
        if (u > (R)(gd[a] - 1)) { u = (R)(gd[a] - 1); clamped[a] = 1; }
        int i = (int)floor(u);
        if (i > gd[a] - 2) i = gd[a] - 2;
        if (i < 0) i = 0;
        i0[a] = i;
        fr[a] = u - (R)i;
    }
    size_t npt = (size_t)gd[0] * gd[1] * gd[2];
    const R* m = env->maps + (size_t)map * npt;
    R v[8];
    for (int c = 0; c < 8; c++) {
        int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
        v[c] = m[((size_t)(i0[2] + dz) * gd[1] + (i0[1] + dy)) * gd[0] + (i0[0] + dx)];
    }
    R fx = fr[0], fy = fr[1], fz = fr[2];
    R gx = 1 - fx, gy = 1 - fy, gz = 1 - fz;
    /* along x */
    R c00 = v[0] * gx + v[1] * fx, c10 = v[2] * gx + v[3] * fx;
    R c01 = v[4] * gx + v[5] * fx, c11 = v[6] * gx + v[7] * fx;
    R c0 = c00 * gy + c10 * fy, c1 = c01 * gy + c11 * fy;
    R e = c0 * gz + c1 * fz;
    R dx00 = v[1] - v[0], dx10 = v[3] - v[2], dx01 = v[5] - v[4], dx11 = v[7] - v[6];
    R ddx = (dx00 * gy + dx10 * fy) * gz + (dx01 * gy + dx11 * fy) * fz;
    R ddy = (c10 - c00) * gz + (c11 - c01) * fz;
    R ddz = c1 - c0;
    R inv = 1 / env->spacing;
    g[0] = clamped[0] ? 0 : ddx * inv;
    g[1] = clamped[1] ? 0 : ddy * inv;
    g[2] = clamped[2] ? 0 : ddz * inv;
    return e;
}

/* ---------------- scoring ---------------- */
/* src/cuda/bfgs.cuh:196-218 */
static R box_penalty(const R* c, const orc_env* env, R* f, R slope) {
    R p = 0;
    for (int a = 0; a < 3; a++) {
        if (c[a] < env->box_lo[a]) { p += env->box_lo[a] - c[a]; f[a] += -slope; }
        if (c[a] > env->box_hi[a]) { p += c[a] - env->box_hi[a]; f[a] += slope; }
    }
    return p * slope;
}

/* src/cuda/bfgs.cuh:221-394 (cal_e_f_tile), with the inter block replaced by the grid
   model when env->mode == 1 */
R orc_e_f(const orc_lig* lig, const orc_env* env, const orc_pose* pose, R vcap, R slope, R* aux_f) {
    int n = lig->natom;
    const R* X = pose->coords;
    R energy = 0;
    for (int i = 0; i < 3 * n; i++) aux_f[i] = 0;
    /* inter */
    for (int i = 0; i < n; i++) {
        int ti = lig->types[i];
        if (ti == VN_H) continue;
        R e_atom = 0, fx = 0, fy = 0, fz = 0;
        if (env->mode == 0) {
            R r1 = orc_vdw_radius(ti), fdr;
            for (int j = 0; j < env->nrec; j++) {
                int tj = env->rec_types[j];
                if (tj == VN_H) continue;
                R rv0 = env->rec_xyz[3 * j] - X[3 * i];
                R rv1 = env->rec_xyz[3 * j + 1] - X[3 * i + 1];
                R rv2 = env->rec_xyz[3 * j + 2] - X[3 * i + 2];
                double rr = cut_r2(env->rec_xyz[3 * j], env->rec_xyz[3 * j + 1], env->rec_xyz[3 * j + 2],
                                   X[3 * i], X[3 * i + 1], X[3 * i + 2]);
                if (rr < 64) {
                    R r = RSQRT((R)rr);
                    e_atom += orc_eval_ef(r - (r1 + orc_vdw_radius(tj)), ti, tj, &fdr);
                    if (r < EPS) r = EPS;
                    fdr /= r;
                    fx -= fdr * rv0; fy -= fdr * rv1; fz -= fdr * rv2;
                }
            }
        } else {
            int m = env->map_of_type[ti];
            if (m >= 0) {
                R g[3];
                e_atom = orc_grid_interp(env, m, X + 3 * i, g);
                fx = g[0]; fy = g[1]; fz = g[2];
            }
        }
        if (e_atom > 0) {   /* bfgs.cuh:276-283 */
            R s = vcap / (vcap + e_atom);
            e_atom *= s;
            s *= s;
            fx *= s; fy *= s; fz *= s;
        }
        energy += e_atom;
        aux_f[3 * i] += fx; aux_f[3 * i + 1] += fy; aux_f[3 * i + 2] += fz;
    }
    /* penalty: bfgs.cuh:293-300 */
    for (int i = 0; i < n; i++)
        if (lig->types[i] != VN_H) energy += box_penalty(X + 3 * i, env, aux_f + 3 * i, slope);
    /* intra: bfgs.cuh:305-352 */
    R e_intra = 0;
    for (int i = 0; i < n; i++) {
        int ti = lig->types[i];
        R r1 = orc_vdw_radius(ti);
        R e_atom = 0, fx = 0, fy = 0, fz = 0, fdr;
        for (int k = lig->pair_off[i]; k < lig->pair_off[i + 1]; k++) {
            int j = lig->pairs[k];
            R rv0 = X[3 * j] - X[3 * i], rv1 = X[3 * j + 1] - X[3 * i + 1], rv2 = X[3 * j + 2] - X[3 * i + 2];
            R rr = rv0 * rv0 + rv1 * rv1 + rv2 * rv2;
            if (rr < 64) {
                R r = RSQRT(rr);
                R ep = orc_eval_ef(r - (r1 + orc_vdw_radius(lig->types[j])), ti, lig->types[j], &fdr);
                if (r < EPS) r = EPS;
                fdr /= r;
                R px = -fdr * rv0, py = -fdr * rv1, pz = -fdr * rv2;
                if (ep > 0) {
                    R s = vcap / (vcap + ep);
                    ep *= s;
                    s *= s;
                    px *= s; py *= s; pz *= s;
                }
                e_atom += ep;
                fx += px; fy += py; fz += pz;
            }
        }
        e_intra += e_atom;
        aux_f[3 * i] += fx; aux_f[3 * i + 1] += fy; aux_f[3 * i + 2] += fz;
    }
    energy += (R)0.5 * e_intra;
    /* bias: bfgs.cuh:356-388 */
    if (env->bias_type != 0 && lig->bias_off) {
        for (int i = 0; i < n; i++) {
            R fb[3] = {0, 0, 0};
            for (int b = lig->bias_off[i]; b < lig->bias_off[i + 1]; b++) {
                const R* bp = lig->bias + 5 * b;
                R r[3] = {bp[0] - X[3 * i], bp[1] - X[3 * i + 1], bp[2] - X[3 * i + 2]};
                if (env->bias_type == 1) energy += orc_eval_ef_pos(r, bp[3] * env->bias_k, bp[4], fb);
                else energy += orc_eval_ef_zalign(r, bp[3] * env->bias_k, lig->types[i], fb);
            }
            aux_f[3 * i] += fb[0]; aux_f[3 * i + 1] += fb[1]; aux_f[3 * i + 2] += fb[2];
        }
    }
    /* A pose with a non-finite coordinate scores +inf (the engine's rule; the reference's
       cutoff and box tests all fail on NaN and give such a pose a finite energy). */
    for (int i = 0; i < 3 * n; i++)
        if (!isfinite(X[i])) return (R)INFINITY;
    return energy;
}

/* src/cuda/bfgs.cuh:69-193 (cal_grad_tile) */
static void grad_from_forces(const orc_lig* lig, const orc_env* env, const orc_pose* pose,
                             const R* aux_f, R* g) {
    const R* X = pose->coords;
    for (int k = 0; k < lig->ntors; k++) {
        int from = lig->axis[2 * k], to = lig->axis[2 * k + 1];
        R t5[3] = {0, 0, 0}, t1[3], t3[3];
        for (int q = lig->rot_off[k]; q < lig->rot_off[k + 1]; q++) {
            int a = lig->rot_atoms[q];
            if (lig->types[a] == VN_H) continue;
            t1[0] = X[3 * a] - X[3 * to]; t1[1] = X[3 * a + 1] - X[3 * to + 1]; t1[2] = X[3 * a + 2] - X[3 * to + 2];
            cross3(t1, aux_f + 3 * a, t3);
            t5[0] += t3[0]; t5[1] += t3[1]; t5[2] += t3[2];
        }
        t3[0] = X[3 * to] - X[3 * from]; t3[1] = X[3 * to + 1] - X[3 * from + 1]; t3[2] = X[3 * to + 2] - X[3 * from + 2];
        g[6 + k] = dot3(t5, t3) / norm3(t3);
    }
    R q[4];
    orc_rotvec_to_quaternion(q, pose->rot_vec);
    q[1] = -q[1]; q[2] = -q[2]; q[3] = -q[3];
    R fs[3] = {0, 0, 0}, mat[9] = {0};
    for (int i = 0; i < lig->natom; i++) {
        if (lig->types[i] == VN_H) continue;
        R t1[3] = {X[3 * i] - pose->center[0], X[3 * i + 1] - pose->center[1], X[3 * i + 2] - pose->center[2]};
        orc_rotate_vec_by_quaternion(t1, q);
        const R* f = aux_f + 3 * i;
        fs[0] += f[0]; fs[1] += f[1]; fs[2] += f[2];
        R mt[9];
        outer3(f, t1, mt);
        for (int j = 0; j < 9; j++) mat[j] += mt[j];
    }
    if (!env->constraint) {
        g[0] = fs[0]; g[1] = fs[1]; g[2] = fs[2];
        for (int i = 0; i < 3; i++) {
            R d[9];
            orc_grad_rot_over_vec(d, pose->rot_vec, i);
            R s = 0;
            for (int j = 0; j < 9; j++) s += mat[j] * d[j];
            g[3 + i] = s;
        }
    } else {
        g[0] = g[1] = g[2] = g[3] = g[4] = g[5] = 0;
    }
}

R orc_e_grad(const orc_lig* lig, const orc_env* env, const orc_pose* pose, R vcap, R slope,
             R* out_g, R* aux_f) {
    R e = orc_e_f(lig, env, pose, vcap, slope, aux_f);
    grad_from_forces(lig, env, pose, aux_f, out_g);
    return e;
}

/* src/score/score.cpp:12-108 (no curl; intra over i<j) */
void orc_score_terms(const orc_lig* lig, const orc_env* env, const R* X, R* out) {
    R f;
    R e_intra = 0, e_inter = 0, e_pen = 0, e_bias = 0;
    for (int i = 0; i < lig->natom; i++) {
        for (int k = lig->pair_off[i]; k < lig->pair_off[i + 1]; k++) {
            int j = lig->pairs[k];
            if (j <= i) continue;
            R d0 = X[3 * j] - X[3 * i], d1 = X[3 * j + 1] - X[3 * i + 1], d2 = X[3 * j + 2] - X[3 * i + 2];
            R rr = d0 * d0 + d1 * d1 + d2 * d2;
            if (rr < 64)
                e_intra += orc_eval_ef(RSQRT(rr) - (orc_vdw_radius(lig->types[i]) + orc_vdw_radius(lig->types[j])),
                                       lig->types[i], lig->types[j], &f);
        }
    }
    for (int i = 0; i < lig->natom; i++) {
        int ti = lig->types[i];
        if (ti == VN_H) continue;
        if (env->mode == 0) {
            for (int j = 0; j < env->nrec; j++) {
                int tj = env->rec_types[j];
                if (tj == VN_H) continue;
                double rr = cut_r2(env->rec_xyz[3 * j], env->rec_xyz[3 * j + 1], env->rec_xyz[3 * j + 2],
                                   X[3 * i], X[3 * i + 1], X[3 * i + 2]);
                if (rr < 64)
                    e_inter += orc_eval_ef(RSQRT((R)rr) - (orc_vdw_radius(ti) + orc_vdw_radius(tj)), ti, tj, &f);
            }
        } else {
            int m = env->map_of_type[ti];
            R g[3];
            if (m >= 0) e_inter += orc_grid_interp(env, m, X + 3 * i, g);
        }
        R t3[3] = {0, 0, 0};
        e_pen += box_penalty(X + 3 * i, env, t3, (R)1e6);
    }
    if (env->bias_type != 0 && lig->bias_off) {
        for (int i = 0; i < lig->natom; i++) {
            for (int b = lig->bias_off[i]; b < lig->bias_off[i + 1]; b++) {
                const R* bp = lig->bias + 5 * b;
                R r[3] = {bp[0] - X[3 * i], bp[1] - X[3 * i + 1], bp[2] - X[3 * i + 2]}, fb[3] = {0, 0, 0};
                if (env->bias_type == 1) e_bias += orc_eval_ef_pos(r, bp[3] * env->bias_k, bp[4], fb);
                else e_bias += orc_eval_ef_zalign(r, bp[3] * env->bias_k, lig->types[i], fb);
            }
        }
    }
    out[0] = e_intra; out[1] = e_inter; out[2] = e_pen; out[3] = e_bias;
}

/* ---------------- kinematics ---------------- */
static void pose_copy(const orc_lig* lig, orc_pose* dst, const orc_pose* src) {
    dst->energy = src->energy;
    memcpy(dst->center, src->center, sizeof(src->center));
    memcpy(dst->rot_vec, src->rot_vec, sizeof(src->rot_vec));
    memcpy(dst->coords, src->coords, sizeof(R) * 3 * lig->natom);
    if (lig->ntors) memcpy(dst->dihedrals, src->dihedrals, sizeof(R) * lig->ntors);
}

/* src/cuda/bfgs.cuh:443-549 */
void orc_apply_dihe(const orc_lig* lig, orc_pose* x, int k, R incr_raw) {
    R incr = orc_normalize_angle(incr_raw);
    int nr = lig->range_off[k + 1] - lig->range_off[k];
    R t = orc_normalize_angle(x->dihedrals[k] + incr);
    R dnew = orc_clamp_by_ranges(t, lig->ranges + 2 * lig->range_off[k], nr);
    incr = dnew - x->dihedrals[k];
    x->dihedrals[k] = dnew;
    int from = lig->axis[2 * k], to = lig->axis[2 * k + 1];
    R* X = x->coords;
    R cto[3] = {X[3 * to], X[3 * to + 1], X[3 * to + 2]};
    R ax[3] = {cto[0] - X[3 * from], cto[1] - X[3 * from + 1], cto[2] - X[3 * from + 2]};
    R l = norm3(ax);
    if (l <= EPS) { ax[0] = 1; ax[1] = 0; ax[2] = 0; }
    else { ax[0] /= l; ax[1] /= l; ax[2] /= l; }
    for (int q = lig->rot_off[k]; q < lig->rot_off[k + 1]; q++) {
        int a = lig->rot_atoms[q];
        R v[3] = {X[3 * a] - cto[0], X[3 * a + 1] - cto[1], X[3 * a + 2] - cto[2]};
        orc_rotate_vec_by_rodrigues(v, ax, incr);
        X[3 * a] = v[0] + cto[0]; X[3 * a + 1] = v[1] + cto[1]; X[3 * a + 2] = v[2] + cto[2];
    }
    R c[3] = {0, 0, 0};
    for (int i = 0; i < lig->natom; i++) { c[0] += X[3 * i]; c[1] += X[3 * i + 1]; c[2] += X[3 * i + 2]; }
    x->center[0] = c[0] / lig->natom; x->center[1] = c[1] / lig->natom; x->center[2] = c[2] / lig->natom;
}

/* src/cuda/bfgs.cuh:560-618 */
void orc_apply_update(const orc_lig* lig, const orc_env* env, orc_pose* x, const R* g, R alpha) {
    for (int k = 0; k < lig->ntors; k++) orc_apply_dihe(lig, x, k, g[6 + k] * alpha);
    if (env->constraint) return;
    R c0[3] = {x->center[0], x->center[1], x->center[2]};
    x->center[0] = c0[0] + alpha * g[0];
    x->center[1] = c0[1] + alpha * g[1];
    x->center[2] = c0[2] + alpha * g[2];
    R rv[3] = {g[3] * alpha, g[4] * alpha, g[5] * alpha}, q[4];
    orc_rotvec_to_quaternion(q, rv);
    x->rot_vec[0] = rv[0]; x->rot_vec[1] = rv[1]; x->rot_vec[2] = rv[2];
    R* X = x->coords;
    for (int i = 0; i < lig->natom; i++) {
        R v[3] = {X[3 * i] - c0[0], X[3 * i + 1] - c0[1], X[3 * i + 2] - c0[2]};
        orc_rotate_vec_by_quaternion(v, q);
        X[3 * i] = v[0] + x->center[0]; X[3 * i + 1] = v[1] + x->center[1]; X[3 * i + 2] = v[2] + x->center[2];
    }
}

/* ---------------- line search / BFGS ---------------- */
static R gdot(const R* a, const R* b, int n) {
    R s = 0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* src/cuda/bfgs.cuh:623-670 */
void orc_line_search(const orc_lig* lig, const orc_env* env, const orc_pose* x, const R* g, const R* p,
                     R e0, R vcap, R slope, orc_pose* out_x, R* out_g, R* out_e, R* out_alpha, int* n_eval) {
    int dim = 6 + lig->ntors;
    R alpha = 1, e_new = 0;
    R pg = gdot(p, g, dim);
    R* aux_f = (R*)malloc(sizeof(R) * 3 * lig->natom);
    for (int trial = 0; trial < 10; trial++) {
        pose_copy(lig, out_x, x);
        orc_apply_update(lig, env, out_x, p, alpha);
        e_new = orc_e_grad(lig, env, out_x, vcap, slope, out_g, aux_f);
        if (n_eval) (*n_eval)++;
        if (e_new - e0 < (R)1e-4 * alpha * pg) break;
        alpha *= (R)0.5;
    }
    free(aux_f);
    *out_e = e_new;
    *out_alpha = alpha;
}

static int tri(int i, int j) { return i <= j ? i + j * (j + 1) / 2 : j + i * (i + 1) / 2; }

/* src/cuda/bfgs.cuh:729-829 (with bfgs_update_hessian_tile :682-712 and
   minus_mat_vec_product_tile :413-428); the inverse Hessian is kept in double */
int orc_bfgs(const orc_lig* lig, const orc_env* env, orc_pose* x, int max_steps, R vcap, R slope) {
    int n = lig->natom, T = lig->ntors, dim = 6 + T;
    int n_eval = 0;
    R* buf = (R*)calloc((size_t)(3 * n * 3 + T * 3 + dim * 8), sizeof(R));
    R* aux_f = buf;
    R* cxn = aux_f + 3 * n;
    R* cxo = cxn + 3 * n;
    R* dxn = cxo + 3 * n;
    R* dxo = dxn + T;
    R* g = dxo + T;
    R* gn = g + dim;
    R* go = gn + dim;
    R* p = go + dim;
    R* y = p + dim;
    R* mhy = y + dim;
    double* H = (double*)calloc((size_t)dim * (dim + 1) / 2, sizeof(double));
    orc_pose xn = {0}, xo = {0};
    xn.coords = cxn; xn.dihedrals = dxn;
    xo.coords = cxo; xo.dihedrals = dxo;

    R E_ori = orc_e_grad(lig, env, x, vcap, slope, g, aux_f);
    n_eval++;
    R E = E_ori, E1 = 0, alpha = 0;
    for (int i = 0; i < dim; i++) H[tri(i, i)] = 1;
    memcpy(gn, g, sizeof(R) * dim);
    pose_copy(lig, &xn, x);
    memcpy(go, g, sizeof(R) * dim);
    pose_copy(lig, &xo, x);
    memcpy(p, g, sizeof(R) * dim);
    for (int step = 0; step < max_steps; step++) {
        for (int i = 0; i < dim; i++) {
            double s = 0;
            for (int j = 0; j < dim; j++) s += H[tri(i, j)] * (double)g[j];
            p[i] = (R)(-s);
        }
        orc_line_search(lig, env, x, g, p, E, vcap, slope, &xn, gn, &E1, &alpha, &n_eval);
        for (int i = 0; i < dim; i++) y[i] = gn[i] - g[i];
        E = E1;
        pose_copy(lig, x, &xn);
        R gg = gdot(g, g, dim);
        if (RSQRT(gg) < (R)1e-5) break;
        memcpy(g, gn, sizeof(R) * dim);
        if (step == 0) {
            R yy = gdot(y, y, dim);
            if (fabs(yy) > EPS) {
                R yp = gdot(y, p, dim);
                for (int i = 0; i < dim; i++) H[tri(i, i)] = (double)(alpha * yp / yy);
            }
        }
        /* bfgs_update_hessian_tile */
        R yp = gdot(y, p, dim);
        if (alpha * yp < EPS) continue;
        for (int i = 0; i < dim; i++) {
            double s = 0;
            for (int j = 0; j < dim; j++) s += H[tri(i, j)] * (double)y[j];
            mhy[i] = (R)(-s);
        }
        double yhy = -(double)gdot(y, mhy, dim);
        double r = 1.0 / ((double)alpha * (double)yp);
        double a = alpha;
        for (int i = 0; i < dim; i++)
            for (int j = i; j < dim; j++)
                H[i + j * (j + 1) / 2] += a * r * ((double)mhy[i] * p[j] + (double)mhy[j] * p[i]) +
                                          a * a * (r * r * yhy + r) * (double)p[i] * p[j];
    }
    if (E > E_ori) {
        E = E_ori;
        pose_copy(lig, x, &xo);
    }
    x->energy = E;
    free(H);
    free(buf);
    return n_eval;
}

/* ---------------- MC search ---------------- */
/* src/cuda/common.cuh:106-122 */
static R gyration_radius(const orc_lig* lig, const orc_pose* x) {
    R s = 0;
    int n = 0;
    for (int i = 0; i < lig->natom; i++) {
        if (lig->types[i] == VN_H) continue;
        R d0 = x->coords[3 * i] - x->center[0], d1 = x->coords[3 * i + 1] - x->center[1],
          d2 = x->coords[3 * i + 2] - x->center[2];
        s += d0 * d0 + d1 * d1 + d2 * d2;
        n++;
    }
    R r = n > 0 ? RSQRT(s / n) : 0;
    return r > 0 ? r : 1;
}

/* unit-ball sample by rejection (common.cuh:90-103); attempts are capped at 64,
   after which the zero vector is used */
static void rand_in_sphere(const orc_search_param* sp, int chain, uint32_t step, R* v) {
    for (int a = 0; a < 64; a++) {
        uint32_t u[4];
        rng4(sp, chain, step, P_SPHERE + a, u);
        v[0] = ((R)orc_u01(u[0]) - (R)0.5) * 2;
        v[1] = ((R)orc_u01(u[1]) - (R)0.5) * 2;
        v[2] = ((R)orc_u01(u[2]) - (R)0.5) * 2;
        if (norm3(v) < 1) return;
    }
    v[0] = v[1] = v[2] = 0;
}

/* src/cuda/mc.cu:18-104 */
void orc_randomize(const orc_lig* lig, const orc_env* env, const orc_search_param* sp, int chain, orc_pose* x) {
    int T = lig->ntors;
    R* g = (R*)calloc((size_t)(6 + T), sizeof(R));
    uint32_t u[4];
    rng4(sp, chain, 0, P_INIT, u);
    if (!env->constraint) {
        R s = chain + (R)0.5, n = (R)sp->nchain;
        R r = RSQRT(s / n), Rr = RSQRT(1 - s / n);
        R al = 2 * PI_R * s / PHI_R, be = 2 * PI_R * s / PSI_R;
        R q[4] = {r * sin(al), r * cos(al), Rr * sin(be), Rr * cos(be)};
        if (env->bias_type == 2) {
            g[0] = g[1] = g[2] = 0;
        } else {
            g[0] = (env->box_lo[0] + (env->box_hi[0] - env->box_lo[0]) * (R)orc_u01(u[0])) - x->center[0];
            g[1] = (env->box_lo[1] + (env->box_hi[1] - env->box_lo[1]) * (R)orc_u01(u[1])) - x->center[1];
            g[2] = (env->box_lo[2] + (env->box_hi[2] - env->box_lo[2]) * (R)orc_u01(u[2])) - x->center[2];
        }
        orc_quaternion_to_rotvec(g + 3, q);
    }
    for (int k = 0; k < T; k++) {
        rng4(sp, chain, 0, P_INIT + 1 + k, u);
        int nr = lig->range_off[k + 1] - lig->range_off[k];
        int j = (int)((R)orc_u01(u[0]) * nr);
        if (j > nr - 1) j = nr - 1;
        const R* rg = lig->ranges + 2 * (lig->range_off[k] + j);
        R v = rg[0] + (rg[1] - rg[0]) * (R)orc_u01(u[1]);
        g[6 + k] = v - x->dihedrals[k];
    }
    orc_apply_update(lig, env, x, g, 1);
    free(g);
}

/* src/cuda/mc.cu:146-256; returns nothing, mutates x */
static void mutate(const orc_lig* lig, const orc_env* env, const orc_search_param* sp, int chain,
                   uint32_t step, orc_pose* x) {
    const R amplitude = 2;
    int T = lig->ntors;
    int num_mutable = 2 + T;
    uint32_t u[4];
    rng4(sp, chain, step, P_WHICH, u);
    int which;
    if (env->constraint) {
        if (num_mutable < 3) which = 3;
        else which = 2 + (int)(u[0] % (uint32_t)(num_mutable - 2));
    } else {
        which = (int)(u[0] % (uint32_t)num_mutable);
    }
    if (which == 0) {
        R v[3], d[3];
        rand_in_sphere(sp, chain, step, v);
        for (int a = 0; a < 3; a++) {
            R t = amplitude * v[a] + x->center[a];
            if (t > env->box_hi[a]) t = env->box_hi[a];
            if (t < env->box_lo[a]) t = env->box_lo[a];
            d[a] = t - x->center[a];
            x->center[a] = x->center[a] + d[a];
        }
        for (int i = 0; i < lig->natom; i++)
            for (int a = 0; a < 3; a++) x->coords[3 * i + a] += d[a];
    } else if (which == 1) {
        R v[3], q[4];
        rand_in_sphere(sp, chain, step, v);
        R a = gyration_radius(lig, x);
        R rv[3] = {amplitude / a * v[0], amplitude / a * v[1], amplitude / a * v[2]};
        orc_rotvec_to_quaternion(q, rv);
        x->rot_vec[0] = rv[0]; x->rot_vec[1] = rv[1]; x->rot_vec[2] = rv[2];
        for (int i = 0; i < lig->natom; i++) {
            R t[3] = {x->coords[3 * i] - x->center[0], x->coords[3 * i + 1] - x->center[1],
                      x->coords[3 * i + 2] - x->center[2]};
            orc_rotate_vec_by_quaternion(t, q);
            for (int k = 0; k < 3; k++) x->coords[3 * i + k] = t[k] + x->center[k];
        }
    } else if (which - 2 < T) {
        int k = which - 2;
        rng4(sp, chain, step, P_TORS, u);
        R r2[2] = {(R)orc_u01(u[0]), (R)orc_u01(u[1])};
        int nr = lig->range_off[k + 1] - lig->range_off[k];
        R a = orc_get_radian_in_ranges(lig->ranges + 2 * lig->range_off[k], nr, r2) - x->dihedrals[k];
        orc_apply_dihe(lig, x, k, a);
    }
}

/* src/search/mc.h:12-18 */
static int metropolis_accept(R e_old, R e_new, R temp, R rx) {
    if (e_new < e_old) return 1;
    return rx < exp((e_old - e_new) / temp);
}

static void pose_alloc(const orc_lig* lig, orc_pose* p) {
    p->coords = (R*)calloc((size_t)3 * lig->natom, sizeof(R));
    p->dihedrals = (R*)calloc((size_t)(lig->ntors > 0 ? lig->ntors : 1), sizeof(R));
}
static void pose_free(orc_pose* p) { free(p->coords); free(p->dihedrals); }

/* src/cuda/mc.cu:275-398 (mc_kernel), preceded by randomize_pose when requested */
long orc_mc_chain(const orc_lig* lig, const orc_env* env, const orc_search_param* sp, int chain,
                  const orc_pose* x0, orc_pose* out) {
    long n_eval = 0;
    orc_pose cand, acc;
    pose_alloc(lig, &cand);
    pose_alloc(lig, &acc);
    pose_copy(lig, out, x0);
    if (sp->randomize) orc_randomize(lig, env, sp, chain, out);
    pose_copy(lig, &acc, out);
    R best_e = (R)1e9;
    if (sp->mc_steps == 0) {
        R* aux = (R*)malloc(sizeof(R) * 3 * lig->natom);
        acc.energy = orc_e_f(lig, env, &acc, (R)10, (R)1e6, aux);
        n_eval++;
        free(aux);
        pose_copy(lig, out, &acc);
    } else {
        R* aux = (R*)malloc(sizeof(R) * (3 * lig->natom + 6 + lig->ntors));
        for (int step = 0; step < sp->mc_steps; step++) {
            pose_copy(lig, &cand, &acc);
            mutate(lig, env, sp, chain, (uint32_t)step, &cand);
            if (sp->opt_steps == 0) {
                cand.energy = orc_e_grad(lig, env, &cand, (R)10, (R)1e6, aux + 3 * lig->natom, aux);
                n_eval++;
            } else {
                n_eval += orc_bfgs(lig, env, &cand, sp->opt_steps, (R)10, (R)1e6);
            }
            uint32_t u[4];
            rng4(sp, chain, (uint32_t)step, P_METRO, u);
            int accepted = metropolis_accept(acc.energy, cand.energy, (R)1.2, (R)orc_u01(u[0]));
            if (step == 0 || accepted) {
                pose_copy(lig, &acc, &cand);
                if (acc.energy < best_e) {
                    if (sp->opt_steps > 0) n_eval += orc_bfgs(lig, env, &acc, sp->opt_steps, (R)1000, (R)1e6);
                    if (acc.energy < best_e) {
                        pose_copy(lig, out, &acc);
                        best_e = acc.energy;
                    }
                }
            }
        }
        free(aux);
    }
    pose_free(&cand);
    pose_free(&acc);
    return n_eval;
}

/* ---------------- clustering: src/cuda/cluster.cu:16-135 ----------------
   RMSD over heavy atoms in input order, no superposition.  The pose order is a
   stable sort by energy (ties by index); a pose becomes a leader iff its squared
   deviation sum to every current leader is >= limit^2 * n_heavy.  Sums run over
   heavy atoms in order with explicit fmaf so the CUDA path reproduces them bit for
   bit. */
static const float* g_sort_e;
static int cmp_idx(const void* a, const void* b) {
    int i = *(const int*)a, j = *(const int*)b;
    float ei = g_sort_e[i], ej = g_sort_e[j];
    if (ei < ej) return -1;
    if (ei > ej) return 1;
    return (i > j) - (i < j);
}
int orc_cluster(int natom, const int* types, int npose, const float* coords, const float* energies,
                float rmsd_limit, int* out_leaders) {
    int* order = (int*)malloc(sizeof(int) * npose);
    for (int i = 0; i < npose; i++) order[i] = i;
    g_sort_e = energies;
    qsort(order, npose, sizeof(int), cmp_idx);
    int nh = 0;
    for (int i = 0; i < natom; i++) nh += types[i] != VN_H;
    float thr = (rmsd_limit * rmsd_limit) * (float)nh;
    int nl = 0;
    for (int oi = 0; oi < npose; oi++) {
        int c = order[oi];
        int novel = 1;
        for (int l = 0; l < nl && novel; l++) {
            int b = out_leaders[l];
            float acc = 0.f;
            for (int i = 0; i < natom; i++) {
                if (types[i] == VN_H) continue;
                float dx = coords[(size_t)c * 3 * natom + 3 * i] - coords[(size_t)b * 3 * natom + 3 * i];
                float dy = coords[(size_t)c * 3 * natom + 3 * i + 1] - coords[(size_t)b * 3 * natom + 3 * i + 1];
                float dz = coords[(size_t)c * 3 * natom + 3 * i + 2] - coords[(size_t)b * 3 * natom + 3 * i + 2];
                acc = fmaf(dx, dx, acc);
                acc = fmaf(dy, dy, acc);
                acc = fmaf(dz, dz, acc);
            }
            if (acc < thr) novel = 0;
        }
        if (novel) out_leaders[nl++] = c;
    }
    free(order);
    return nl;
}

/* ---------------- batched helpers ---------------- */
void orc_e_grad_batch(const orc_lig* lig, const orc_env* env, int n, const R* coords, const R* centers,
                      const R* rotvecs, R vcap, R slope, R* out_e, R* out_g) {
    int dim = 6 + lig->ntors;
#pragma omp parallel for schedule(dynamic, 4)
    for (int p = 0; p < n; p++) {
        orc_pose x;
        x.energy = 0;
        x.coords = (R*)(coords + (size_t)p * 3 * lig->natom);
        x.dihedrals = NULL;
        for (int a = 0; a < 3; a++) { x.center[a] = centers[3 * p + a]; x.rot_vec[a] = rotvecs[3 * p + a]; }
        R* aux = (R*)malloc(sizeof(R) * 3 * lig->natom);
        out_e[p] = orc_e_grad(lig, env, &x, vcap, slope, out_g + (size_t)p * dim, aux);
        free(aux);
    }
}
