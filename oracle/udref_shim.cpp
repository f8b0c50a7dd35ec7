// udref_shim.cpp -- C entry points over the reference engine's own host code.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from the
// reference sources where they lie (unidock/unidock_engine/src/...): this file
// includes the reference's inline headers (score/vina.h, myutils/mymath.h,
// geometry/quaternion.h, geometry/rotation.h) and links the reference's
// score/score.cpp, so the values these functions return are the reference's own.
// It is used to pin the oracle restatement and as the reference CPU scoring
// baseline; it is never part of the product.
#include <vector>
#include <cstring>
#include "score/vina.h"
#include "score/score.h"
#include "myutils/mymath.h"
#include "geometry/quaternion.h"
#include "geometry/rotation.h"

static Vina g_vina;

extern "C" {

Real udref_eval_ef(Real d, int t1, int t2, Real* out_f) { return g_vina.eval_ef(d, t1, t2, out_f); }
Real udref_gaussian1(Real d, Real* f) { return g_vina.vina_gaussian1(d, f); }
Real udref_gaussian2(Real d, Real* f) { return g_vina.vina_gaussian2(d, f); }
Real udref_repulsion(Real d, Real* f) { return g_vina.vina_repulsion(d, f); }
Real udref_hydrophobic(Real d, Real* f) { return g_vina.vina_hydrophobic(d, f); }
Real udref_hbond(Real d, Real* f) { return g_vina.vina_hbond(d, f); }
Real udref_conf_indep(Real e, int n) { return g_vina.vina_conf_indep(e, n); }
Real udref_eval_ef_zalign(Real* r, Real a, int t, Real* f) { return g_vina.eval_ef_zalign(r, a, t, f); }
Real udref_eval_ef_pos(Real* r, Real v, Real r2, Real* f) { return g_vina.eval_ef_pos(r, v, r2, f); }
Real udref_normalize_angle(Real x) { return normalize_angle(x); }
Real udref_normalize_angle_2pi(Real x) { return normalize_angle_2pi(x); }
Real udref_clamp_by_ranges(Real a, Real* r, int n) { return clamp_by_ranges(a, r, n); }
Real udref_get_radian_in_ranges(Real* r, int n, Real* rand2) { return get_radian_in_ranges(r, n, rand2); }
void udref_rotvec_to_quaternion(Real* q, const Real* v) { rotvec_to_quaternion(q, v); }
void udref_quaternion_to_rotvec(Real* v, const Real* q) { quaternion_to_rotvec(v, q); }
void udref_rotate_vec_by_quaternion(Real* v, const Real* q) { rotate_vec_by_quaternion(v, q); }
void udref_rotate_vec_by_rodrigues(Real* v, const Real* axis, Real th) { rotate_vec_by_rodrigues(v, axis, th); }
void udref_grad_rot_over_vec(Real* out9, const Real* v, int ind) { cal_grad_of_rot_over_vec(out9, v, ind); }
void udref_quaternion_multiply_left(const Real* q2, Real* q1) { quaternion_multiply_left(q2, q1); }

// The reference's host final score (score.cpp:12-108) for one pose.
// out4 = [intra, inter, penalty, bias]
void udref_score(int natom, const Real* coords, const int* types, const int* pair_off, const int* pairs,
                 int nrec, const Real* rec_xyz, const int* rec_types, const Real* box6,
                 int bias_type, Real bias_k, int nbias, const int* bias_atom, const Real* bias_par,
                 Real* out4) {
    UDFixMol fix;
    fix.natom = nrec;
    fix.coords.assign(rec_xyz, rec_xyz + 3 * nrec);
    fix.vina_types.assign(rec_types, rec_types + nrec);
    UDFlexMol m;
    m.natom = natom;
    m.vina_types.assign(types, types + natom);
    m.intra_range.resize(2 * natom);
    for (int i = 0; i < natom; i++) {
        m.intra_range[2 * i] = pair_off[i];
        m.intra_range[2 * i + 1] = pair_off[i + 1] - pair_off[i];
    }
    m.intra_pairs.assign(pairs, pairs + pair_off[natom]);
    for (int b = 0; b < nbias; b++) {
        Bias bb;
        bb.i = bias_atom[b];
        for (int k = 0; k < 5; k++) bb.param[k] = (float)bias_par[5 * b + k];
        m.biases.push_back(bb);
    }
    DockParam dp;
    dp.box.x_lo = box6[0]; dp.box.x_hi = box6[1];
    dp.box.y_lo = box6[2]; dp.box.y_hi = box6[3];
    dp.box.z_lo = box6[4]; dp.box.z_hi = box6[5];
    dp.bias_type = bias_type == 1 ? BT_POS : (bias_type == 2 ? BT_ALIGN : BT_NO);
    dp.bias_k = bias_k;
    FlexPose pose;
    std::vector<Real> c(coords, coords + 3 * natom);
    pose.coords = c.data();
    score(&pose, c.data(), fix, m, dp);
    out4[0] = pose.center[0];
    out4[1] = pose.center[1];
    out4[2] = pose.center[2];
    out4[3] = pose.rot_vec[3];
}

// Many poses of one ligand through the reference's score(), OpenMP over poses:
// the reference CPU scoring throughput baseline.
void udref_score_batch(int npose, int natom, const Real* coords, const int* types, const int* pair_off,
                       const int* pairs, int nrec, const Real* rec_xyz, const int* rec_types,
                       const Real* box6, Real* out4) {
    UDFixMol fix;
    fix.natom = nrec;
    fix.coords.assign(rec_xyz, rec_xyz + 3 * nrec);
    fix.vina_types.assign(rec_types, rec_types + nrec);
    UDFlexMol m;
    m.natom = natom;
    m.vina_types.assign(types, types + natom);
    m.intra_range.resize(2 * natom);
    for (int i = 0; i < natom; i++) {
        m.intra_range[2 * i] = pair_off[i];
        m.intra_range[2 * i + 1] = pair_off[i + 1] - pair_off[i];
    }
    m.intra_pairs.assign(pairs, pairs + pair_off[natom]);
    DockParam dp;
    dp.box.x_lo = box6[0]; dp.box.x_hi = box6[1];
    dp.box.y_lo = box6[2]; dp.box.y_hi = box6[3];
    dp.box.z_lo = box6[4]; dp.box.z_hi = box6[5];
    dp.bias_type = BT_NO;
#pragma omp parallel for schedule(dynamic, 16)
    for (int p = 0; p < npose; p++) {
        FlexPose pose;
        score(&pose, coords + (size_t)p * 3 * natom, fix, m, dp);
        out4[4 * p + 0] = pose.center[0];
        out4[4 * p + 1] = pose.center[1];
        out4[4 * p + 2] = pose.center[2];
        out4[4 * p + 3] = pose.rot_vec[3];
    }
}

// The reference's per-atom decomposition of the intermolecular energy
// (score_decomp, score.cpp:114-147): out5[natom][5] = gauss1, gauss2, repulsion,
// hydrophobic, hbond.
void udref_score_decomp(int natom, const Real* coords, const int* types, int nrec, const Real* rec_xyz,
                        const int* rec_types, Real* out5) {
    UDFixMol fix;
    fix.natom = nrec;
    fix.coords.assign(rec_xyz, rec_xyz + 3 * nrec);
    fix.vina_types.assign(rec_types, rec_types + nrec);
    UDFlexMol m;
    m.natom = natom;
    m.vina_types.assign(types, types + natom);
    std::vector<AtomEnergyDecomp> d;
    score_decomp(d, coords, fix, m);
    for (int i = 0; i < natom; i++) {
        out5[5 * i + 0] = d[i].gauss1;
        out5[5 * i + 1] = d[i].gauss2;
        out5[5 * i + 2] = d[i].repulsion;
        out5[5 * i + 3] = d[i].hydrophobic;
        out5[5 * i + 4] = d[i].hbond;
    }
}

}  // extern "C"
