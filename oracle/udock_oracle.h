/*
 * udock_oracle.h -- CPU oracle for the Uni-Dock2 docking-engine hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the
 * product (uni-dock2_b200/).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may use it.
 *
 * It restates, in plain C at FP64 (or FP32 with -DORC_FLOAT), the reference
 * engine's algorithm for the hot path (reference paths relative to
 * unidock/unidock_engine/):
 *   - Vina pair terms               src/score/vina.h:151-321, src/myutils/mymath.h:210-214
 *   - direct-sum inter E/force      src/cuda/bfgs.cuh:242-289 (per-atom curl :276-283)
 *   - box penalty                   src/cuda/bfgs.cuh:196-218
 *   - intra pair terms              src/cuda/bfgs.cuh:305-352
 *   - bias terms                    src/cuda/bfgs.cuh:356-388, src/score/vina.h:353-400
 *   - reverse gradient pass         src/cuda/bfgs.cuh:69-193, src/geometry/rotation.h:80-144
 *   - kinematics                    src/cuda/bfgs.cuh:443-618
 *   - line search / BFGS            src/cuda/bfgs.cuh:623-829
 *   - MC chain / mutation / init    src/cuda/mc.cu:18-398, src/search/mc.h:12-18
 *   - RMSD + greedy clustering      src/cuda/cluster.cu:16-135
 *   - host final score              src/score/score.cpp:12-108
 * plus the grid model that has no reference counterpart (grid build and
 * trilinear interpolation of per-type maps) and the counter-based Philox4x32-10
 * generator (Salmon et al., SC'11) that both the oracle and the CUDA path use.
 */
#ifndef UDOCK_ORACLE_H
#define UDOCK_ORACLE_H

#include <stdint.h>

#ifdef ORC_FLOAT
typedef float orc_real;
#else
typedef double orc_real;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ligand topology, flat arrays; all indices are local to the ligand */
typedef struct {
    int natom, ntors;
    const int* types;        /* natom XS types */
    const int* axis;         /* 2*ntors: (from, to) */
    const int* range_off;    /* ntors+1: offsets (in ranges, not values) into ranges */
    const orc_real* ranges;  /* 2 values per range, radians */
    const int* rot_off;      /* ntors+1: offsets into rot_atoms */
    const int* rot_atoms;    /* rotated atom indices per torsion */
    const int* pair_off;     /* natom+1: per-atom intra adjacency (both directions) */
    const int* pairs;
    const int* bias_off;     /* natom+1 offsets into bias params (in records of 5), may be NULL */
    const orc_real* bias;    /* 5 per record: x y z V r2 */
} orc_lig;

/* scoring environment */
typedef struct {
    int nrec;
    const orc_real* rec_xyz;  /* 3*nrec */
    const int* rec_types;
    orc_real box_lo[3], box_hi[3];
    int mode;                 /* 0 = direct sum, 1 = grid */
    /* grid */
    int nmaps;
    const int* map_of_type;   /* 21 entries: map slot per XS type or -1 */
    const orc_real* maps;     /* nmaps * gz*gy*gx, x fastest */
    orc_real origin[3];
    orc_real spacing;
    int gdim[3];
    /* flags */
    int constraint;           /* constraint docking: no translation/rotation */
    int bias_type;            /* 0 none, 1 pos, 2 align */
    orc_real bias_k;
} orc_env;

/* a pose; coords/dihedrals are caller-owned */
typedef struct {
    orc_real energy;
    orc_real center[3];
    orc_real rot_vec[3];
    orc_real* coords;     /* 3*natom */
    orc_real* dihedrals;  /* ntors */
} orc_pose;

/* ---- building blocks ---- */
orc_real orc_eval_ef(orc_real d, int t1, int t2, orc_real* out_f);
orc_real orc_vina_term(int which, orc_real d, orc_real* out_f);
void orc_eval_decomp(orc_real d, int t1, int t2, orc_real out_terms[5]);
orc_real orc_gaussian(orc_real d, orc_real offset, orc_real width, orc_real* out_f);
orc_real orc_vdw_radius(int t);
orc_real orc_normalize_angle(orc_real x);
orc_real orc_normalize_angle_2pi(orc_real x);
orc_real orc_clamp_by_ranges(orc_real ang, const orc_real* ranges, int nrange);
orc_real orc_get_radian_in_ranges(const orc_real* ranges, int nrange, const orc_real* rand2);
orc_real orc_get_real_within_by_int(int c, orc_real min, orc_real max, int n);
void orc_rotvec_to_quaternion(orc_real* out_q, const orc_real* rv);
void orc_quaternion_to_rotvec(orc_real* out_v, const orc_real* q);
void orc_rotate_vec_by_quaternion(orc_real* v, const orc_real* q);
void orc_rotate_vec_by_rodrigues(orc_real* v, const orc_real* axis, orc_real theta);
void orc_quaternion_multiply_left(const orc_real* q2, orc_real* q1);
void orc_quaternion_normalize(orc_real* q);
void orc_grad_rot_over_vec(orc_real* out9, const orc_real* v, int ind);
orc_real orc_eval_ef_zalign(const orc_real* r, orc_real a_qt, int t, orc_real* out_f);
orc_real orc_eval_ef_pos(const orc_real* r, orc_real v, orc_real r2, orc_real* out_f);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float orc_u01(uint32_t u);

/* ---- grid ---- */
void orc_grid_build(int nrec, const orc_real* rec_xyz, const int* rec_types,
                    int nmaps, const int* map_types, const orc_real* origin, orc_real spacing,
                    const int* gdim, orc_real* out_maps);
orc_real orc_grid_interp(const orc_env* env, int map, const orc_real* x, orc_real* out_g);

/* ---- scoring ---- */
/* E + per-atom gradient (aux_f, 3*natom); returns total energy (reference cal_e_f_tile) */
orc_real orc_e_f(const orc_lig* lig, const orc_env* env, const orc_pose* pose,
                 orc_real vcap, orc_real slope, orc_real* aux_f);
/* E + generalised gradient (6+ntors), reference cal_e_grad_tile */
orc_real orc_e_grad(const orc_lig* lig, const orc_env* env, const orc_pose* pose,
                    orc_real vcap, orc_real slope, orc_real* out_g, orc_real* aux_f);
/* energy terms without curl: out[0]=intra(i<j) out[1]=inter out[2]=penalty out[3]=bias
   (reference score.cpp:12-108; uses env->mode for inter) */
void orc_score_terms(const orc_lig* lig, const orc_env* env, const orc_real* coords, orc_real* out4);

/* ---- kinematics / optimisation ---- */
void orc_apply_update(const orc_lig* lig, const orc_env* env, orc_pose* x,
                      const orc_real* g, orc_real alpha);
void orc_apply_dihe(const orc_lig* lig, orc_pose* x, int itor, orc_real incr);
void orc_line_search(const orc_lig* lig, const orc_env* env, const orc_pose* x, const orc_real* g,
                     const orc_real* p, orc_real e0, orc_real vcap, orc_real slope,
                     orc_pose* out_x, orc_real* out_g, orc_real* out_e, orc_real* out_alpha,
                     int* n_eval);
/* in-place BFGS; returns number of energy evaluations */
int orc_bfgs(const orc_lig* lig, const orc_env* env, orc_pose* x, int max_steps,
             orc_real vcap, orc_real slope);

/* ---- search ---- */
typedef struct {
    uint64_t seed;
    int lig_uid;          /* ligand id in the RNG counter */
    int nchain;           /* chains per ligand (Super-Fibonacci n) */
    int mc_steps;
    int opt_steps;
    int randomize;
} orc_search_param;

/* one MC chain; x is the input pose, out_best receives the best pose.
   returns the number of energy evaluations. */
long orc_mc_chain(const orc_lig* lig, const orc_env* env, const orc_search_param* sp,
                  int chain, const orc_pose* x0, orc_pose* out_best);
void orc_randomize(const orc_lig* lig, const orc_env* env, const orc_search_param* sp,
                   int chain, orc_pose* x);

/* ---- clustering ---- */
/* greedy leader clustering on FP32 coordinates; returns number of leaders.
   order: stable sort of energies (ties by index). compare in squared space:
   keep iff sum_sq >= limit^2 * n_heavy for every leader (fixed-order fmaf sums). */
int orc_cluster(int natom, const int* types, int npose, const float* coords,
                const float* energies, float rmsd_limit, int* out_leaders);

/* batched helpers for Python (OpenMP over items when built with -fopenmp) */
void orc_e_grad_batch(const orc_lig* lig, const orc_env* env, int n,
                      const orc_real* coords, const orc_real* centers, const orc_real* rotvecs,
                      orc_real vcap, orc_real slope, orc_real* out_e, orc_real* out_g);

#ifdef __cplusplus
}
#endif
#endif
