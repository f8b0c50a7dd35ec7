/*
 * udock_b200.h -- C ABI of the B200 docking engine (libudock_b200.so).
 *
 * The engine replaces the hot path behind the reference's pybind module
 * `unidock_engine.api.python.pipeline` (reference: unidock/unidock_engine/api/python/
 * pipeline.cpp:56-151).  The reference binds C++ classes; this library exports plain
 * C functions over pointers and sizes so any FFI (ctypes, cffi, JNI, cgo) can bind it.
 * Each function below names the reference interface it replaces.
 *
 * Conventions
 *  - Every function returns 0 on success and a negative code on failure; the message
 *    of the last failure on the calling thread is returned by ud_last_error()
 *    (reference: exceptions -> core_pipeline() returns 1 -> RuntimeError,
 *    src/screening/core.cpp:218-222, api/python/pipeline.cpp:141-143).
 *  - All arrays are caller-owned host memory, C-contiguous; the engine copies what it
 *    keeps.  Device memory is owned by the context and freed by ud_destroy.
 *  - Calls on one context are synchronous and not re-entrant; different contexts may
 *    be used from different threads.
 *  - Angles are radians; coordinates Angstrom; energies kcal/mol.
 *  - A pose record is [energy, cx, cy, cz, rvx, rvy, rvz, 0, coords(3N), dihedrals(T)]:
 *    the reference's FlexPose (src/model/model.h:18-24) flattened.
 */
#ifndef UDOCK_B200_H
#define UDOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ud_ctx ud_ctx;

enum { UD_OK = 0, UD_EINVAL = -1, UD_ECUDA = -2, UD_ESTATE = -3, UD_ENOMEM = -4 };
enum { UD_MODE_DIRECT = 0, UD_MODE_GRID = 1 };
enum { UD_GRID_F32 = 0, UD_GRID_F16 = 1 };

/* Library version (major*10000 + minor*100 + patch). */
int ud_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* ud_last_error(void);

/* Free and total device memory of CUDA device `device`, in bytes (the budget of the
 * memory-bounded batches when no max_gpu_mem is given).
 * Replaces: the device-memory query of decide_memory_limit_mb (src/screening/core.cpp:32-63). */
int ud_device_memory(int device, long long* out_free, long long* out_total);

/* Create a context on CUDA device `device` for the docking box
 * box6 = {x_lo, x_hi, y_lo, y_hi, z_lo, z_hi}.
 * Replaces: DockingPipeline(...) construction + decide_memory_limit_mb/cudaSetDevice
 * (api/python/pipeline.cpp:58-111, src/screening/core.cpp:32-63). */
int ud_create(int device, const float* box6, ud_ctx** out);

/* Free all device memory of the context (src/task/DockTask.cpp free_memory_all). */
int ud_destroy(ud_ctx* ctx);

/* Search flags: constraint docking (no translation/rotation), bias type
 * (0 none, 1 position, 2 z-align) and bias scale.
 * Replaces: apply_bias / constraint_docking handling (src/screening/core.cpp:86-97,142-146). */
int ud_set_flags(ud_ctx* ctx, int constraint_docking, int bias_type, float bias_k);

/* Receptor atoms; hydrogens and atoms outside the box grown by 8 A are dropped here.
 * Replaces: DockingPipeline.set_receptor + RapidJsonParser::parse_receptor_info
 * (api/python/pipeline.cpp:113-116, src/format/rapidjson_parser.cpp:25-52). */
int ud_set_receptor(ud_ctx* ctx, int n, const float* xyz, const int* types);

/* Number of receptor atoms kept. */
int ud_receptor_count(const ud_ctx* ctx);

/* Build per-type grid maps covering the box at `spacing` for the XS types in
 * map_types[nmaps] (1..20 non-hydrogen types); precision selects the map storage used by searches
 * (UD_GRID_F32, or UD_GRID_F16 kept beside the FP32 master).
 * New component (the reference scores by direct pair sum, src/cuda/bfgs.cuh:242-289). */
int ud_build_grid(ud_ctx* ctx, float spacing, int nmaps, const int* map_types, int precision);

/* Copy the FP32 maps to the host (out: nmaps*gz*gy*gx floats, x fastest); gdim3 and
 * origin3 receive the grid shape and origin.  Pass out=NULL to query the shape only. */
int ud_get_grid(const ud_ctx* ctx, float* out, int* gdim3, float* origin3);

/* Select the map storage used for grid-mode scoring (UD_GRID_F32 / UD_GRID_F16). */
int ud_set_grid_precision(ud_ctx* ctx, int precision);

/* Append ligands.  All index arrays are local to the ligand.  Offsets are prefix sums
 * of length count+1 into the following array:
 *   atom_off[nlig+1]   -> xyz (3 per atom), types
 *   tors_off[nlig+1]   -> axis (2 per torsion: from,to), dihedrals (radians)
 *   range_off[T+1]     -> ranges (2 per range, radians); T = tors_off[nlig]
 *   rot_off[T+1]       -> rot_atoms (atoms moved by each torsion)
 *   pair_off[A+1]      -> pairs (per-atom intra neighbours, both directions); A = atom_off[nlig]
 *   bias_off[A+1]      -> bias (5 per record: x y z V r2); bias_off/bias may be NULL
 * Replaces: DockingPipeline.add_ligands + RapidJsonParser::parse_ligands_info and the
 * GPU upload of DockTask::alloc_gpu (api/python/pipeline.cpp:118-123,
 * src/format/rapidjson_parser.cpp:54-225, src/cuda/task.cu:304-402). */
int ud_add_ligands(ud_ctx* ctx, int nlig, const int* atom_off, const float* xyz, const int* types,
                   const int* tors_off, const int* axis, const float* dihedrals,
                   const int* range_off, const float* ranges, const int* rot_off, const int* rot_atoms,
                   const int* pair_off, const int* pairs, const int* bias_off, const float* bias);

/* Bulk ligand input (host only, no GPU needed).  Parses a JSON document in the engine's
 * ligand schema (an object of ligands; the reserved keys "receptor" and "score" are
 * skipped) and builds, for every ligand, the 1-2/1-3 and 1-4 pair sets, the rigid
 * fragments of the torsion tree and the scored intra pair lists, on `nthreads` host
 * threads (0 = all cores).  The result is a ligand set in exactly the packed layout of
 * ud_add_ligands (plus ff types, charges and the pair-set sizes), in document order.
 * Replaces: the json.dumps + rapidjson hand-off and RapidJsonParser::parse_ligands_info
 * with split_torsions_into_frags (api/python/pipeline.cpp:125-139,
 * src/format/rapidjson_parser.cpp:54-225,227-296).
 * Errors (malformed document or schema) return UD_EINVAL; the message is in
 * ud_ligset_last_error(). */
typedef struct ud_ligset ud_ligset;
int ud_ligset_parse_json(const char* json, size_t len, int use_tor_lib, int nthreads, ud_ligset** out);
/* out8 = [ligands, atoms, torsions, ranges, rotated atoms, pair entries, bias records,
 * bytes of all names]: the lengths of the export arrays (offset arrays have one more). */
int ud_ligset_sizes(const ud_ligset* set, long long* out8);
/* Copy the set out; any pointer may be NULL to skip that array.  name_off[ligands+1]
 * indexes `names` (UTF-8, not NUL-terminated). */
int ud_ligset_export(const ud_ligset* set, int* atom_off, float* xyz, int* types, int* ff_types, float* charges,
                     int* tors_off, int* axis, float* dihedrals, int* range_off, float* ranges, int* rot_off,
                     int* rot_atoms, int* pair_off, int* pairs, int* bias_off, float* bias, int* n_pairs_1213,
                     int* n_pairs_14, long long* name_off, char* names);
void ud_ligset_free(ud_ligset* set);
const char* ud_ligset_last_error(void);

/* Drop all ligands and search results. */
int ud_clear_ligands(ud_ctx* ctx);

/* Number of ligands loaded. */
int ud_ligand_count(const ud_ctx* ctx);

/* Energy and generalised gradient (6+T: centre, orientation, torsions) of n poses.
 * pose_lig[n] ligand index per pose; coords concatenated per pose (3*natom each);
 * centers/rotvecs 3 per pose (rotvec = last rotation increment, the reference's
 * FlexPose::rot_vec); out_g concatenated 6+T per pose.
 * mode UD_MODE_DIRECT (reference pair sum) or UD_MODE_GRID.
 * Replaces: cal_e_grad_one_gpu (src/cuda/bfgs_wrapper.cu:63-98), batched. */
int ud_score_batch(ud_ctx* ctx, int n, const int* pose_lig, const float* coords, const float* centers,
                   const float* rotvecs, int mode, float vcap, float slope, float* out_e, float* out_g);

/* ud_score_batch without any device-memory allocation.  No counterpart in the reference.
 * For callers that must not allocate device memory inside the call: a host whose device
 * memory is already handed to its own pool allocator, or a loop that cannot afford the
 * device-wide synchronisation that cudaFree implies.  Same arguments, results and errors
 * as ud_score_batch; the per-call staging lives in one fixed module-scope device array
 * of UD_NOALLOC_SCRATCH_BYTES per device instead of fresh buffers.
 * - Limits: n <= UD_NOALLOC_MAX_POSES, and the batch's staging (ids, 2 int64 offsets,
 *   coordinates, centres, rotation vectors, energies, gradients; each 256-byte aligned)
 *   must fit UD_NOALLOC_SCRATCH_BYTES; larger batches fail with UD_EINVAL: split them.
 * - The ligand set must already be on the device: after ud_add_ligands / ud_build_grid,
 *   one ud_score_batch, ud_search or ud_dock call uploads it; otherwise UD_ESTATE.
 * - First call on a device: looks the array's address up (cudaGetSymbolAddress) with
 *   that device current, once; make this first call before any stream capture begins.
 * - Nothing in the array has to start at zero: every word a call reads it wrote first.
 * - All contexts on a device share the one array: calls that overlap in time (from
 *   several threads, or several contexts on one device) race on it and must be
 *   serialised by the caller. */
#ifndef UD_NOALLOC_MAX_POSES
#define UD_NOALLOC_MAX_POSES 16384
#endif
#ifndef UD_NOALLOC_SCRATCH_BYTES
#define UD_NOALLOC_SCRATCH_BYTES (8u << 20)
#endif
int ud_score_batch_noalloc(ud_ctx* ctx, int n, const int* pose_lig, const float* coords, const float* centers,
                           const float* rotvecs, int mode, float vcap, float slope, float* out_e, float* out_g);

/* Measurement helpers (used by bench.py for the roofline; not part of the reference path).
 * ud_read_bandwidth: streaming 16-byte reads of a `bytes` buffer (each launch reads it as
 * many times as make at least 1 GiB), `repeats` launches after 3 warm-up ones, timed with
 * CUDA events: the L2 read bandwidth when the buffer fits the L2 (126 MB on B200), the HBM
 * read bandwidth when it is far larger.
 * ud_score_batch_timed: ud_score_batch with the inputs uploaded once and the scoring
 * kernel launched `repeats` times back to back (after one warm-up launch); out_ms is the
 * mean kernel time.  Results as ud_score_batch.  No counterpart in the reference. */
int ud_read_bandwidth(int device, long long bytes, int repeats, float* out_gbps);
int ud_score_batch_timed(ud_ctx* ctx, int n, const int* pose_lig, const float* coords, const float* centers,
                         const float* rotvecs, int mode, float vcap, float slope, int repeats, float* out_e,
                         float* out_g, float* out_ms);

/* Final-score terms of n poses without curl: out_terms4 = [intra(i<j), inter, penalty, bias]
 * per pose; out_decomp (nullable) = 5 inter terms per atom
 * [gauss1, gauss2, repulsion, hydrophobic, hbond].
 * Replaces: score() / score_decomp() (src/score/score.cpp:12-147). */
int ud_score_terms(ud_ctx* ctx, int n, const int* pose_lig, const float* coords, int mode,
                   float* out_terms4, float* out_decomp);

/* In-place BFGS of n pose records (see header comment; records concatenated, record of a
 * pose sized for its ligand).  `rounds` consecutive optimisations of max_steps each,
 * round r using penalty slope min(slope0 * 100^r, 1e6) when ramp != 0, else slope0.
 * out_nevals (nullable) receives energy evaluations per pose.
 * Replaces: opt_kernel / optimize_cu and DockTask::run_refine
 * (src/cuda/optimize.cu:14-77, src/task/DockTask.cpp:155-186). */
int ud_bfgs_batch(ud_ctx* ctx, int n, const int* pose_lig, float* records, int max_steps, int rounds,
                  float vcap, float slope0, int ramp, int mode, int* out_nevals);

/* Monte Carlo search: nchain chains per loaded ligand, one persistent launch; each
 * chain keeps its best pose.  opt_steps >= 0 (resolve the reference's -1 heuristic
 * on the host).  out_nevals (nullable) receives the total energy evaluations.
 * Replaces: mc_cu / mc_kernel / randomize_pose (src/cuda/mc.cu:18-448). */
int ud_search(ud_ctx* ctx, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize,
              int mode, long long* out_nevals);

/* Best pose record of every chain of ligand `lig` (nchain records, ligand-sized). */
int ud_get_chain_poses(const ud_ctx* ctx, int lig, float* out_records);

/* Size in floats of one pose record of ligand `lig`. */
int ud_record_floats(const ud_ctx* ctx, int lig);

/* Greedy RMSD clustering of each ligand's chain poses (heavy atoms, no fit; stable
 * energy order, ties by index; a pose is kept iff its squared deviation sum to every
 * kept pose is >= limit^2 * n_heavy).  out_leaders[nlig*nchain] (chain indices, sorted
 * by energy), out_counts[nlig].
 * Replaces: cluster_cu (src/cuda/cluster.cu:74-135). */
int ud_cluster(ud_ctx* ctx, float rmsd_limit, int* out_leaders, int* out_counts);

/* Full docking of all loaded ligands: search, clustering, refinement of the cluster
 * leaders (refine_steps rounds x 2 BFGS steps, slope ramp 1e2..1e6, vcap 1000), filter
 * by energy_range and num_pose, final scoring (no curl, direct sum).
 * Replaces: DockTask::run (src/task/DockTask.cpp:39-123) over all batches. */
typedef struct {
    uint64_t seed;
    int nchain;          /* exhaustiveness */
    int mc_steps;
    int opt_steps;       /* resolved, >= 0 */
    int refine_steps;
    int num_pose;
    float rmsd_limit;
    float energy_range;
    int randomize;
    int mode;            /* UD_MODE_GRID or UD_MODE_DIRECT for the search */
    int final_mode;      /* scoring of output poses: UD_MODE_DIRECT (reference) or grid */
    int energy_decomp;
    int refine_mode;     /* scoring of the refinement BFGS: UD_MODE_DIRECT (exact pair sums, as
                            the reference's optimize_cu, src/cuda/optimize.cu:14-77) or grid */
} ud_dock_params;

int ud_dock(ud_ctx* ctx, const ud_dock_params* params, long long* out_nevals);

/* Output pose counts per ligand after ud_dock (out_counts[nlig]). */
int ud_result_counts(const ud_ctx* ctx, int* out_counts);

/* Output poses after ud_dock, ligand-major, in rank order:
 * out_records: pose records (ligand-sized, concatenated);
 * out_terms4: [intra, inter, penalty, bias] per pose;
 * out_decomp (nullable, only if energy_decomp): 5 per atom per pose. */
int ud_get_results(const ud_ctx* ctx, float* out_records, float* out_terms4, float* out_decomp);

/* Total floats of all output records (sizing helper for ud_get_results). */
long long ud_result_floats(const ud_ctx* ctx);

/* Synchronise the context's stream; returns an error if a kernel failed. */
int ud_sync(ud_ctx* ctx);

/* The cudaStream_t the context launches on (for callers that time with CUDA events).
 * No reference counterpart (the reference uses the legacy default stream). */
void* ud_stream(ud_ctx* ctx);

/* Device times (ms, CUDA events on the context's stream) of the stages of the last
 * ud_dock: out6 = [search, cluster, refine, filter+gather, final score, total].
 * No reference counterpart (the reference logs host wall time, screening.cpp:204-214). */
int ud_stage_times(const ud_ctx* ctx, float* out6);

/* Work counters of the last ud_search / ud_dock: out4 = [energy evaluations in the search,
 * heavy-atom evaluations in the search (sum over evaluations of heavy atoms),
 * kernel launches, chains].  Replaces the reference's managed line-search counter
 * (src/cuda/common.cu:6, src/cuda/mc.cu:443). */
int ud_counters(const ud_ctx* ctx, long long* out4);

/* Poses kept per chain by ud_search / ud_search_learned / ud_dock (1..4, default 1): each
 * chain keeps its last `retain` new best poses (its lowest-energy refined poses; records
 * never filled keep the start pose with energy 1e9); with 1, the reference's one best pose
 * per chain (src/cuda/mc.cu:389-392).  The chains' moves do not depend on it.  Chain poses,
 * clustering, refinement and the filter then see nchain * retain poses per ligand, chain
 * c's at c*retain .. c*retain+retain-1.  No reference counterpart. */
int ud_set_retain(ud_ctx* ctx, int retain);

/* Chain packing autotuner for ud_search / ud_dock (on != 0): before a batch of a new
 * shape, times short searches (3 MC steps) with 8, 12 or 4 warps per CTA and 1, 2 or 4
 * chains per warp per work item and keeps the fastest.  Results do not depend on the
 * packing.  Without it (and without ud_set_packing) the search takes the CTA width that
 * keeps the most warps resident.
 * No reference counterpart (the reference launches one fixed shape, src/cuda/mc.cu:424-440). */
int ud_set_autotune(ud_ctx* ctx, int on);

/* Fixed chain packing for the searches of this context: warps per CTA (4, 8 or 12; 0 =
 * chosen per batch) and chains per warp per work item (1..4; 0 = chosen per batch).  Takes
 * precedence over the autotuner; a width whose CTA does not fit the shared memory falls back
 * to the widest of at most 4 warps that fits (ud_search_shape reports what ran).  Results do
 * not depend on the packing.
 * No reference counterpart. */
int ud_set_packing(ud_ctx* ctx, int warps_per_cta, int chains_per_warp);

/* Launch shape of the last search (fused or learned): out4 = [warps per CTA, CTAs per SM,
 * register class (3, 4: 256-thread bound; 2: 384-thread bound), chains per warp per item].
 * No reference counterpart. */
int ud_search_shape(const ud_ctx* ctx, int* out4);

/* ---------------------------------------------------------------------------------------
 * Learned move proposal.  No reference counterpart: a BF16 MLP (672 -> 256 -> 256 -> 256
 * -> 64, ReLU, FP32 accumulation on the tensor cores) predicts from a chain's accepted
 * pose a Gaussian (mean, log-variance) over its 6 + T move dimensions [centre shift (3),
 * rotation vector (3), torsion changes (T)]; a sampled move replaces the random draw of
 * mutate_pose_tile (src/cuda/mc.cu:146-256); p_learned is the expected share of MC steps
 * whose move is learned.  BFGS, Vina scoring and Metropolis stay as in the plain search.
 * Features of a pose (672): energies of the first 8 grid maps at each of up to 80 atoms,
 * squashed v/(1+|v|); torsion angles / pi (up to 20); E/(10+|E|); 1; zero padding.
 * Parameters (flat FP32, ud_mlp_param_count of them): W1[672x256], b1, W2[256x256], b2,
 * W3[256x256], b3, W4[256x64], b4; W row-major [in x out].  Output row (64): mean[0:26],
 * raw log-variance[26:52] (clamped to [-8, 4] where used), 12 unused. */
long long ud_mlp_param_count(void);
/* Tensor-core path of the network's GEMMs (forward pass and the training backward pass):
 * 1 = tcgen05.mma with a tensor-memory accumulator (default; the backward contracts over the
 * batch through transposed operands), 0 = mma.sync. */
int ud_mlp_set_gemm(ud_ctx* ctx, int kind);
/* He-normal weights (last layer scaled by 0.1), zero biases, Adam state cleared. */
int ud_mlp_init(ud_ctx* ctx, uint64_t seed);
int ud_mlp_set_params(ud_ctx* ctx, const float* params);
int ud_mlp_get_params(ud_ctx* ctx, float* params);
/* out[n x 64] for features x[n x 672]. */
int ud_mlp_forward(ud_ctx* ctx, int n, const float* x, float* out);
/* Mean masked Gaussian negative log-likelihood of targets y[n x 26] under mask[n x 26],
 * and its gradient with respect to every parameter (flat, param_count floats). */
int ud_mlp_loss_grad(ud_ctx* ctx, int n, const float* x, const float* y, const float* mask, double* out_loss,
                     float* out_grad);
/* Adam (lr; betas 0.9, 0.999; eps 1e-8) over shuffled full minibatches for `epochs`;
 * out_epoch_loss[epochs] (nullable) receives the mean minibatch loss of each epoch. */
int ud_mlp_train(ud_ctx* ctx, int n, const float* x, const float* y, const float* mask, int epochs, int batch,
                 float lr, uint64_t seed, float* out_epoch_loss);
/* The MC search of ud_search with learned moves (grid scoring; ligands of at most 80
 * atoms and 20 torsions): the steps run in blocks of K = floor(1 / p_learned) (at most 8),
 * each block one launch of all chains after one batched forward pass of the network over
 * every chain's accepted pose; the learned move replaces the random move of a block's
 * first step with probability p_learned * K.  p_learned = 0 gives exactly ud_search's
 * chains.  Results as ud_search (ud_get_chain_poses, ud_cluster). */
int ud_search_learned(ud_ctx* ctx, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize,
                      float p_learned, long long* out_nevals);
/* K, the MC steps per launch of the learned search: floor(1 / p_learned) clamped to 1..8
 * (8 at p_learned = 0); 1 while moves are recorded (recording != 0) or for p_learned
 * outside [0, 1].  Needs no device. */
int ud_learned_block(float p_learned, int recording);
/* Run the plain search (as ud_search_learned with p_learned = 0) and record up to
 * max_moves accepted moves: the features of the pose before the step, a move (centre
 * shift, rotation vector of a rigid frame of the ligand, wrapped torsion changes) and the
 * mask of the dimensions that apply.  target 0: the move to the accepted pose; target 1:
 * the move to the best pose of the ligand at the end of the run (over all its chains).
 * Replaces nothing. */
int ud_collect_moves(ud_ctx* ctx, uint64_t seed, int nchain, int mc_steps, int opt_steps, int randomize, int target,
                     int max_moves, int* out_count);
/* ud_dock with the learned-proposal search (ud_search_learned) in place of ud_search;
 * mode must be UD_MODE_GRID. */
int ud_dock_learned(ud_ctx* ctx, const ud_dock_params* params, float p_learned, long long* out_nevals);
/* Copy the first n recorded moves: x[n x 672], y[n x 26], mask[n x 26] (each nullable). */
int ud_get_moves(ud_ctx* ctx, int n, float* out_x, float* out_y, float* out_mask);
/* ud_mlp_train on the recorded moves, on the device. */
int ud_mlp_train_moves(ud_ctx* ctx, int epochs, int batch, float lr, uint64_t seed, float* out_epoch_loss);

#ifdef __cplusplus
}
#endif
#endif
