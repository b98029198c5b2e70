/*
 * unidock_b200 -- C ABI of the B200 docking engine.
 *
 * The reference (dptech-corp/Uni-Dock) has no C ABI: its batched search sits
 * behind internal C++ calls.  Each entry point below names the reference
 * interface it replaces.  All arguments are plain pointers and sizes; device
 * memory is owned by the library behind opaque handles; host arrays are owned
 * by the caller.  Every function returns UD_OK (0) or an error code and never
 * throws or exits; ud_last_error() describes the last failure of the calling
 * thread.  A `stream` argument is a cudaStream_t (NULL = default stream).
 */
#ifndef UNIDOCK_B200_H
#define UNIDOCK_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UD_OK 0
#define UD_ERR_ARG 1      /* invalid argument */
#define UD_ERR_PARSE 2    /* malformed PDBQT input */
#define UD_ERR_CUDA 3     /* CUDA runtime failure (message has the CUDA error) */
#define UD_ERR_CAPACITY 4 /* ligand exceeds a capacity limit (atoms, torsions) */
#define UD_ERR_STATE 5    /* call out of order (e.g. results before a search) */
#define UD_ERR_TIMEOUT 6  /* a device-side wait ran past its time limit (streaming screen) */

#define UD_SF_VINA 0
#define UD_SF_AD4 1
#define UD_SF_VINARDO 2

typedef struct ud_maps_s* ud_maps;
typedef struct ud_ligand_s* ud_ligand;
typedef struct ud_batch_s* ud_batch;
typedef struct ud_stream_s* ud_stream;

/* Library version (major*10000 + minor*100 + patch). */
int ud_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* ud_last_error(void);

/* ---------------------------------------------------------------- receptor
 * Parse a rigid receptor PDBQT and assign X-Score types from its bonds.
 * Replaces parse_receptor_pdbqt (unidock/src/lib/parse_pdbqt.cpp:1214) +
 * model::assign_types (unidock/src/lib/model.cpp:408).  With xyz/xs NULL only
 * *n_atoms is set.  Untyped atoms (hydrogens) get xs = 36. */
int ud_receptor_parse(const char* pdbqt, size_t len, float* xyz, int* xs, int capacity,
                      int* n_atoms);

/* Receptor parse with AutoDock types and partial charges as well (the inputs
 * of AD4 maps); any output pointer may be NULL.  Untyped atoms get ad = 35. */
int ud_receptor_parse_ex(const char* pdbqt, size_t len, float* xyz, int* xs, int* ad, float* charge,
                         int capacity, int* n_atoms);

/* ---------------------------------------------------------------- grid maps
 * Build grid maps on the GPU for the listed XS types (all 24 Vina map types
 * when types == NULL) over the box center +- size/2 at `spacing`.
 * Replaces Vina::compute_vina_maps (unidock/src/lib/vina.cpp:491-567) and
 * cache::populate_no_bias (unidock/src/lib/cache.cpp:471-549).  `sf` is
 * UD_SF_VINA or UD_SF_VINARDO; weights follow the reference's order
 * (Vina: gauss1, gauss2, repulsion, hydrophobic, hbond, glue, rot) with the
 * rotatable weight in raw form (e.g. 0.05846); NULL = defaults. */
int ud_maps_create(int sf, const float* weights, int n_weights, const float* rec_xyz,
                   const int* rec_xs, int n_rec, const float center[3], const float size[3],
                   float spacing, const int* types, int n_types, void* stream, ud_maps* out);
/* AutoDock 4.2 maps built on the GPU (the reference reads them from AutoGrid
 * files instead, ad4cache::read, unidock/src/lib/ad4cache.cpp:391-437): one
 * map per AD type of `types` (NULL = every AD kind a ligand atom can read; CG
 * carbons read C), then the electrostatic map (per unit ligand charge) and the
 * desolvation map (per unit |ligand charge|), the three ad4cache::eval_deriv
 * combines (ad4cache.cpp:227-269).  Map values are the reference's AD4.2 pair
 * terms (potentials.h:346-486, scoring_function.h:74-86) summed over receptor
 * atoms at the exact probe distances.  Weights in the reference's order
 * (vdW, H-bond, electrostatics, desolvation, glue, torsional -- the last raw,
 * as ad4_tors_add uses it); NULL = defaults.  The box has an even number of
 * voxels per axis, as AutoGrid maps do.  Replaces the external autogrid4 step. */
int ud_maps_create_ad4(const float* weights, int n_weights, const float* rec_xyz, const int* rec_ad,
                       const float* rec_q, int n_rec, const float center[3], const float size[3], float spacing,
                       const int* types, int n_types, void* stream, ud_maps* out);
/* Write the maps as AutoGrid .map text files <prefix>.<type>.map (AD4 maps:
 * AD type names plus <prefix>.e.map and <prefix>.d.map; Vina maps: X-Score type
 * names), header as ad4cache::write (ad4cache.cpp:439-521), values at full
 * float precision.  --write_maps of the reference CLI. */
int ud_maps_write(ud_maps maps, const char* prefix);
/* Maps read from AutoGrid .map files <prefix>.<type>.map (the reference's
 * --maps: cache::read, cache.cpp:325-379, for Vina / Vinardo by X-Score type
 * names; ad4cache::read, ad4cache.cpp:391-437, for AD4 by AD type names plus
 * the required .e.map and .d.map).  Weights as ud_maps_create / _ad4. */
int ud_maps_load(int sf, const float* weights, int n_weights, const char* prefix, void* stream, ud_maps* out);
/* dims[3] sample points, init[3] box corner, factor[3] samples per Angstrom. */
int ud_maps_info(ud_maps maps, int dims[3], float init[3], float factor[3], int* n_maps);
/* Copy the map of XS type `xs` to host memory (dims[0]*dims[1]*dims[2] floats,
 * x fastest); for AD4 maps `xs` is an AD type, 35 the electrostatic and 36 the
 * desolvation map.  Replaces igrid::get_grids (unidock/src/lib/igrid.h:39). */
int ud_maps_read(ud_maps maps, int xs, float* out, size_t n);
int ud_maps_destroy(ud_maps maps);

/* ---------------------------------------------------------------- ligands
 * Parse a ligand into a torsion-tree model (host memory): a V2000 SDF
 * record (4th line ends in V2000) or else a Vina PDBQT.
 * Replaces parse_ligand_from_file_no_failure with hydrogens kept, as the
 * reference CLI calls it (unidock/src/lib/parse_pdbqt.cpp:1076-1140,
 * unidock/src/main/main.cpp:858-863) + model::initialize
 * (unidock/src/lib/model.cpp:613-619).  A ligand with more than 48 torsions
 * or 256 atoms returns UD_ERR_CAPACITY, as the reference refuses more than
 * MAX_NUM_OF_LIG_TORSION torsions and MAX_NUM_OF_ATOMS (150) atoms
 * (parse_pdbqt.cpp:1107-1120); the same holds for the two calls below. */
int ud_ligand_parse(const char* text, size_t len, ud_ligand* out);
/* SDF record with the fragInfo / torsionInfo / atomInfo properties of the
 * reference's ligand preparation.  keep_h = 0 leaves atoms of AutoDock type H
 * out of the model (parse_sdf_ligand's keep_H, parse_pdbqt.cpp:612-873).
 * Results of such a ligand are written back as its own SDF record. */
int ud_ligand_parse_sdf(const char* sdf, size_t len, int keep_h, ud_ligand* out);
/* The ligand's own input record (SDF or PDBQT, as parsed) with the atom
 * coordinates of `pose` ([x y z qw qx qy qz torsions...]) and no result block,
 * into buf (cap bytes, NUL-terminated); *len = full length.  Replaces
 * model::write_structure / write_sdf_structure (unidock/src/lib/model.h:125-144)
 * as Vina::write_pose uses them for --local_only (vina.cpp:1018-1030). */
int ud_ligand_write(ud_ligand lig, const float* pose, char* buf, size_t cap, size_t* len);
/* Parse n ligands on `threads` host threads (0 = all): out[i] is the handle
 * or NULL, status[i] its error code (may be NULL: then any failure makes the
 * call return UD_ERR_PARSE, the successful handles still set).  The batch form
 * of the OpenMP-parallel parse of the reference CLI (main.cpp:975-983). */
int ud_ligand_parse_many(const char* const* texts, const size_t* lens, int n, int threads, ud_ligand* out,
                         int* status);
/* counts[0] atoms, [1] heavy atoms, [2] torsions, [3] rigid nodes,
 * [4] intramolecular pairs, [5] TORSDOF, [6] glue pairs, [7] BFGS steps. */
int ud_ligand_counts(ud_ligand lig, int counts[8]);
/* Flat export of the model; any pointer may be NULL.  node_rel holds 6 floats
 * per node (origin relative to parent, unit axis), input frame. */
int ud_ligand_export(ud_ligand lig, float* lab_xyz, float* local_xyz, int* xs, int* ad, int* el,
                     float* charge, int* atom_node, int* node_parent, int* node_begin,
                     int* node_end, float* node_rel, int* pair_a, int* pair_b);
/* Pose of the input coordinates: [x y z qw qx qy qz t0 .. t(T-1)]. */
int ud_ligand_initial_pose(ud_ligand lig, float* pose);
/* Lab coordinates (3 per atom) of a pose (host forward kinematics,
 * model::set, unidock/src/lib/model.cpp:848-851). */
int ud_ligand_coords(ud_ligand lig, const float* pose, float* xyz);
/* Conformation-independent inputs (num_tors, num_rotors, heavy atoms,
 * hydrophobic atoms, h-bond atoms, ligands, length). */
int ud_ligand_conf_indep(ud_ligand lig, float out[7]);
int ud_ligand_destroy(ud_ligand lig);

/* ---------------------------------------------------------------- batches
 * Upload the topology of n ligands to device memory for scoring and search
 * against `maps`.  Replaces the per-batch marshalling of do_docking_base
 * (unidock/src/cuda/monte_carlo.cu:2397-2900) and precalculate_parallel
 * (unidock/src/cuda/precalculate.cu:169-326): type-pair tables of the
 * scoring function are shared by all ligands. */
int ud_batch_create(ud_maps maps, const ud_ligand* ligs, int n, void* stream, ud_batch* out);
/* The batch's handle and device buffers reused for n other ligands (no
 * counterpart in the reference): buffers grow to the largest batch seen and
 * are never freed in between, so a streaming screen that cycles a few batch
 * handles makes no device allocation or free -- which would synchronise the
 * device -- once warm.  A launched search must have been collected first
 * (UD_ERR_STATE otherwise); the results of the previous ligands are dropped. */
int ud_batch_reset(ud_batch batch, const ud_ligand* ligs, int n, void* stream);
int ud_batch_destroy(ud_batch batch);

/* Energy and pose gradient at fixed poses, host buffers.  pose_ligand[i]
 * selects the ligand of pose i; poses has pose_stride floats per pose in the
 * layout of ud_ligand_initial_pose; g_out receives 6 + T floats per pose in
 * the reference's change layout (d/dposition, torque, d/dtorsions) with
 * stride g_stride.  v_intra / v_inter are the curl caps of the intramolecular
 * and grid terms (1000 = scoring, 10 = search); entries of g_out past a
 * pose's 6 + T are set to 0.  Replaces model::eval_deriv
 * (unidock/src/lib/model.cpp:935-962). */
int ud_score_grad(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses,
                  int pose_stride, float v_intra, float v_inter, float* e_out, float* g_out,
                  int g_stride, void* stream);
/* Same with device pointers; asynchronous on `stream`; entries of g_out past
 * a pose's 6 + T are left as they are. */
int ud_score_grad_device(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses,
                         int pose_stride, float v_intra, float v_inter, float* e_out,
                         float* g_out, int g_stride, void* stream);
/* Scoring-path energies: out[2*i] grid (cache::eval, cache.cpp:84-120),
 * out[2*i+1] intramolecular pairs from the nearest-bin table (model::evali,
 * model.cpp:927-933), both with curl cap v. */
int ud_score(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses,
             int pose_stride, float v, float* out, void* stream);

/* Score of fixed poses as Vina::score reports it (vina.cpp:1168-1240,
 * rigid receptor): 8 floats per pose = {estimated free energy of binding,
 * ligand-receptor, ligand-flex (0), flex-receptor (0), flex-flex (0), ligand
 * intramolecular, torsional (conf-independent) term, unbound system's energy
 * (the pose's own intramolecular energy)}.  Used by --score_only and
 * --local_only. */
int ud_score_terms(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                   float* out, void* stream);

/* ---------------------------------------------------------------- differentiation
 * No counterpart in the reference (its gradient is internal to BFGS).
 *
 * Term weights of the maps' scoring function, in the reference's order
 * (Vina: gauss1, gauss2, repulsion, hydrophobic, hbond, glue; Vinardo:
 * gauss1, repulsion, hydrophobic, hbond, glue); the rotatable-bond weight is
 * not a term (it enters only the final conf-independent score). */
int ud_maps_term_count(ud_maps maps, int* n_terms);
int ud_maps_get_weights(ud_maps maps, float* w, int n);
/* Replace the term weights: maps and pair tables become the weight-sum of
 * per-term maps and tables (built on the GPU on first use, about
 * n_terms x (maps + 27 MB) of device memory), so searches and scores that
 * follow use the new weights.  Equal to maps built with those weights up to
 * FP32 rounding of the sum. */
int ud_maps_set_weights(ud_maps maps, const float* w, int n, void* stream);

#define UD_ADJOINT_EXACT 1  /* pair forces: exact derivative of the lerped energy */
/* Energy at fixed poses with its gradient in the POSE layout and its weight
 * gradient (the adjoint of the energy; conformer coordinates recomputed from
 * the pose, not stored).
 *   g_out  (optional) 7 + T floats per pose, stride g_stride:
 *          d/dposition[3], d/dq[4], d/dtorsions[T]; d/dq is tangent to the
 *          unit sphere at q (the orientation is meant as q/|q|, and the
 *          poses are expected to carry unit quaternions);
 *   dw_out (optional) n_terms floats per pose, stride dw_stride: d/d(term
 *          weight), with the maps' current weights.
 * Pair forces follow the reference (model::eval_deriv, the table's dE/dr / r
 * column, model.cpp:935-962) unless flags has UD_ADJOINT_EXACT, which takes the
 * exact derivative of the computed (lerped) energy -- the gradient that
 * finite differences of the energy converge to.  Poses whose pose_ligand is
 * out of range get a NaN energy (device form) or UD_ERR_ARG (host form). */
int ud_score_adjoint(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                     float v_intra, float v_inter, int flags, float* e_out, float* g_out, int g_stride,
                     float* dw_out, int dw_stride, void* stream);
/* Same with device pointers; asynchronous on `stream`. */
int ud_score_adjoint_device(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses,
                            int pose_stride, float v_intra, float v_inter, int flags, float* e_out, float* g_out,
                            int g_stride, float* dw_out, int dw_stride, void* stream);

/* ---------------------------------------------------------------- search */
typedef struct {
    int exhaustiveness;     /* MC chains per ligand (--exhaustiveness) */
    int max_step;           /* cap on MC steps per chain, 0 = heuristic only (--max_step) */
    int num_modes;          /* poses kept per ligand (--num_modes) */
    float min_rmsd;         /* clustering radius (--min_rmsd) */
    float energy_range;     /* output energy window (--energy_range) */
    unsigned long long seed;/* --seed */
    int form;               /* 0 = plain (one launch per ligand), 1 = batched persistent */
    int chains_per_block;   /* warps per CTA, 1..4; 0 = the batch's autotuned value, else the CTA size of
                               4, 2 or 1 warps that keeps the most chains resident per SM at the
                               batch's layout (the plain form: 4) */
    int bfgs_cap;           /* 0 = per-ligand (25 + atoms)/3 BFGS steps; >0 caps it;
                               <0 = the batch's autotuned cap (per-ligand when not tuned) */
    int use_graph;          /* batched form: the per-batch sequence (queue reset, search
                               kernel, result copies) captured once as a CUDA graph and
                               replayed while parameters and buffers are unchanged */
    int refine_step;        /* > 0: each mode is refined against the receptor atoms in up
                               to refine_step rounds and scored against them, as the
                               reference does unless --no_refine (--refine_step, CLI
                               default 3; vina.h:251-272).  Vina / Vinardo maps built
                               from a receptor only; otherwise, and at 0, the modes keep
                               their grid energies (--no_refine). */
    int lanes_per_chain;    /* batched form: 32 = one chain per warp, 16 = two chains per
                               warp (half a warp each); 0 = the batch's autotuned value,
                               else 32.  The plain form ignores it. */
} ud_search_params;

/* Device bytes a batch of these n ligands holds through a search with
 * `params` (exhaustiveness, num_modes) under scoring `sf`: topology, chain
 * results and mode buffers, headroom included; the maps, pair tables and
 * receptor cells belong to the maps handle and are not counted.  Host-only.
 * The batch packing of the CLI's --max_gpu_memory uses it, as the reference
 * packs batches by predict_peak_memory (unidock/src/main/main.cpp:139-206). */
int ud_batch_device_bytes(const ud_ligand* ligs, int n, int sf, const ud_search_params* params, size_t* bytes);

/* Launch configuration picked by ud_autotune. */
typedef struct {
    int chains_per_block;      /* warps per CTA */
    int lanes_per_chain;       /* lanes per chain: 32 (a warp) or 16 (half a warp) */
    int bfgs_cap;              /* BFGS iteration cap: always 0 (caps are not tuned) */
    int n_sample;              /* ligands of the batch in the tuning sample */
    int n_tried;               /* configurations timed */
    float ligands_per_s;       /* sample throughput of the picked configuration */
    float base_ligands_per_s;  /* sample throughput of the default (4 chains/CTA, no cap) */
    float energy_shift;        /* mean best-energy change against the default (<= 0.1) */
} ud_tune_result;

/* Autotuner (no counterpart in the reference): times the batched search on a
 * sample of the batch (ligands spread over its size order, enough chains to
 * fill the GPU twice, the caller's exhaustiveness, at most 40 MC steps) at
 * each launch shape, warps per CTA in {4, 2, 1} x lanes per chain in {32, 16}.
 * A shape replaces the best so far only when it is more than 3% faster and its
 * mean best energy is within 0.1 kcal/mol of the default's (4 warps, 32
 * lanes).  BFGS iteration caps are not tuned (bfgs_cap in the result is 0):
 * every cap tried moved the search's best-energy distribution away from the
 * reference's at the fast screen settings.  Searches of this batch with
 * chains_per_block = 0 and lanes_per_chain = 0 then use the shape picked.
 * Synchronous; takes about 7 short searches. */
int ud_autotune(ud_batch batch, const ud_search_params* params, ud_tune_result* out, void* stream);

/* Run the Monte-Carlo + BFGS search of every ligand of the batch.
 * Replaces Vina::global_search_gpu (unidock/src/lib/vina.h:154-354) and
 * monte_carlo_template::do_docking (unidock/src/cuda/monte_carlo.cu:2975-3010).
 * Synchronous: returns after the results are on the host. */
int ud_search(ud_batch batch, const ud_search_params* params, void* stream);
/* ud_search split in two: the asynchronous device part (search kernel, then
 * the clustering of every ligand's chains into modes and, with refine_step,
 * their refinement against the receptor atoms, all enqueued on `stream` with
 * inputs already resident) and the host part (final scores, ordering, RMSD
 * bounds).  ud_search == ud_search_launch + ud_search_collect. */
int ud_search_launch(ud_batch batch, const ud_search_params* params, void* stream);
/* The set-up of ud_search_launch without the launch: result buffers (device
 * and page-locked host), the ligand order and, with use_graph, the captured
 * graph.  A following ud_search_launch with the same params only launches. */
int ud_search_prepare(ud_batch batch, const ud_search_params* params, void* stream);
int ud_search_collect(ud_batch batch, void* stream);
/* Raw per-chain results of the last search: best pose (pose_stride floats
 * per chain, chain-major per ligand), best energy and evaluations spent. */
int ud_search_chains(ud_batch batch, float* poses, int pose_stride, float* e, int* evals);
/* Allocation-free batched search.  No counterpart in the reference: added
 * for callers that cannot let the library allocate device memory while they
 * search -- applications whose device memory belongs to their own pool
 * allocator (a cudaMalloc behind its back fragments or overcommits the pool),
 * and latency-critical loops where an allocation's implicit device-wide
 * synchronisation is not acceptable.
 *
 * Runs the batched persistent search (form 1; params->form and use_graph are
 * ignored) on `stream` and returns without waiting.  chains_per_block,
 * lanes_per_chain and bfgs_cap resolve as in ud_search (0 / 0 / <0 = the
 * batch's autotuned values when it was tuned).  The caller owns every output,
 * all in device memory of the current device:
 *   d_poses     [n_ligands * exhaustiveness][pose_stride] best pose per chain
 *               (chain-major per ligand, as ud_search_chains), pose_stride >=
 *               7 + the batch's largest torsion count; only the first 7 + T
 *               floats of a row (T = that ligand's torsions) are written;
 *   d_energies  [n_ligands * exhaustiveness] best energy per chain;
 *   d_evals     [n_ligands * exhaustiveness] evaluations per chain, or NULL.
 * Results equal those of ud_search_launch + ud_search_chains with the same
 * params.  No clustering or rescoring is done (that host part allocates).
 * An empty batch is refused (UD_ERR_ARG), as ud_search refuses it.
 *
 * Scratch (the work-queue counter and one record per chain) lives in one
 * static device array of 3,145,984 bytes (about 3.1 MB) that each GPU using
 * the library holds until the process exits; the call clears what must start
 * at zero.  The ligand order comes from the batch's own device memory, filled
 * when the batch was created.  Limit: at most 131072 chains (ligands x
 * exhaustiveness) per call, beyond which it returns UD_ERR_CAPACITY without
 * launching anything.  All calls on one device share that scratch, so calls
 * whose work overlaps on that device (issued on two streams, or from two
 * threads) race: order them on one stream or synchronise between them.  Each
 * device has its own copy, so calls on different devices do not interfere.
 * The first call on each device looks up the scratch's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture. */
int ud_search_device_noalloc(ud_batch batch, const ud_search_params* params, float* d_poses, int pose_stride,
                             float* d_energies, int* d_evals, void* stream);
/* Number of modes kept for ligand `lig` after clustering and rescoring. */
int ud_result_count(ud_batch batch, int lig, int* n_modes);
/* Mode k of ligand `lig`: pose (7+T floats) and
 * energies[8] = {affinity, rmsd_lb, rmsd_ub, inter+intra, inter, intra,
 * conf_independent, unbound} as written in "REMARK VINA RESULT"
 * (unidock/src/lib/vina.cpp:725-748). */
int ud_result_mode(ud_batch batch, int lig, int k, float* pose, float energies[8]);
/* Output text of ligand `lig` (format 0 = PDBQT MODEL blocks, 1 = SDF),
 * written into buf (cap bytes, NUL-terminated); *len = full length.
 * Replaces Vina::get_poses_gpu / get_sdf_poses_gpu (vina.cpp:872-996). */
int ud_result_write(ud_batch batch, int lig, int format, char* buf, size_t cap, size_t* len);
/* Local optimisation (BFGS at curl cap v, max_steps iterations or the
 * per-ligand (25 + atoms)/3 when 0) from the given poses, updated in place.
 * Replaces quasi_newton::operator() (unidock/src/lib/quasi_newton.cpp:42-53),
 * the --local_only path of Vina::optimize (unidock/src/lib/vina.cpp:1385-1428). */
int ud_optimize(ud_batch batch, const int* pose_ligand, float* poses, int n_poses, int pose_stride,
                int max_steps, float v, float* e_out, int* evals_out, void* stream);
/* ---------------------------------------------------------------- bias wells
 * AutoDock-bias style wells (BPF text, unidock/src/lib/bias.h: a header line,
 * then "x y z Vset r type [AD types]" with type don, acc, aro or map).
 * Added to Vina / Vinardo maps built from a receptor, as --bias does
 * (Vina::set_bias + cache::compute_bias, vina.cpp:1472-1480, cache.cpp:789-957):
 * every map point gets Vset exp(-d^2/r^2) on the maps the well reaches when it
 * is below -0.01; the wells also enter the scoring against the receptor atoms
 * (refinement, ud_score_terms_receptor).  On AutoDock 4.2 maps the wells go
 * into the maps only, as ad4cache::set_bias (ad4cache.cpp:54-88) places them:
 * don -> HD, acc -> OA and NA, aro -> A, map -> the AD types named, or every
 * map with the electrostatic and desolvation maps when none is named.  Wells
 * accumulate over calls.  The maps then have no term decomposition
 * (ud_maps_set_weights, weight gradients: UD_ERR_STATE). */
int ud_maps_add_bias(ud_maps maps, const char* bpf, size_t len, void* stream);
/* Ligand `lig`'s own wells (--multi_bias, Vina::set_batch_bias,
 * vina.cpp:1482-1493), used instead of the maps' when it is scored against
 * the receptor atoms, as model::bias_list is.  As in the reference's GPU
 * search, they do not change the maps the search uses.  Empty text clears
 * them; ud_batch_reset clears all. */
int ud_batch_set_bias(ud_batch batch, int lig, const char* bpf, size_t len);

/* ---------------------------------------------------------------- receptor atoms
 * Scoring against the receptor atoms the maps were built from, instead of the
 * maps: the reference's non_cache (unidock/src/lib/non_cache.cpp), which it
 * uses after the search and for --score_only / --local_only scores unless
 * --no_refine.  An atom outside the box is scored at its position clamped into
 * the box plus a penalty of slope per Angstrom.  Vina / Vinardo maps built
 * from a receptor (ud_maps_create) only; others give UD_ERR_STATE.
 *
 * Energy and gradient (change layout, 6 + T floats per pose) at fixed poses:
 * model::eval_deriv with non_cache::eval_deriv (non_cache.cpp:420-500) at
 * out-of-box slope `slope` and curl cap v. */
int ud_score_grad_receptor(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                           float slope, float v, float* e_out, float* g_out, int g_stride, void* stream);
/* Refinement of poses (updated in place), as the reference refines each mode
 * after its search (vina.h:251-272): up to refine_step rounds of BFGS
 * ((25 + atoms)/3 steps, curl cap 1000) against the receptor atoms at slope
 * 100, 1e4, 1e6, ..., stopping once every heavy atom is inside the box; then
 * the scoring energies.  out4 per pose: {last BFGS energy, inter (receptor
 * atoms, slope 1e6, curl cap 1000, nearest-bin table), intra (model::evali),
 * 1 if inside the box else 0}. */
int ud_refine(ud_batch batch, const int* pose_ligand, float* poses, int n_poses, int pose_stride, int refine_step,
              float* out4, void* stream);
/* ud_score_terms with the inter energy from the receptor atoms: Vina::score
 * without --no_refine (vina.cpp:1168-1243). */
int ud_score_terms_receptor(ud_batch batch, const int* pose_ligand, const float* poses, int n_poses, int pose_stride,
                            float* out, void* stream);
/* ---------------------------------------------------------------- streaming screen
 * One persistent search kernel fed slot by slot while it runs.  The reference
 * CLI has no such mode; it parses and docks one batch after another
 * (unidock/src/main/main.cpp:975-1070).  The host packs each slot of ligands
 * into page-locked memory, copies it into a device arena and publishes it;
 * the kernel, launched by ud_stream_create, takes the published slots' (ligand,
 * chain) items as they arrive, waiting at most timeout_ms for the next slot;
 * each finished slot's modes are clustered and refined on SMs the kernel
 * leaves free and scored on the host.  Every buffer is allocated at creation,
 * so pushing and collecting never synchronise the device.  Not thread-safe
 * per stream.  Ligand handles must live until their slot is collected and its
 * results read. */
typedef struct {
    int slot_ligands;   /* ligands per slot (rounded up to a multiple of 16) */
    int max_slots;      /* slots the stream takes in all (size of the device arena) */
    int ring;           /* result areas: slot s writes area s % ring, so slot s may be pushed
                           only after slot s - ring was collected */
    int max_atoms;      /* largest ligand the stream takes (shared memory per chain is sized by it) */
    int max_torsions;
    int timeout_ms;     /* longest time the kernel waits with no new slot published (0 = 60000) */
} ud_stream_config;

/* Create the stream and launch its kernel.  params: exhaustiveness, max_step
 * (1..11655 required: a chain's step count must not depend on its slot),
 * num_modes, min_rmsd, energy_range, seed, chains_per_block, bfgs_cap (> 0
 * caps, else per-ligand), refine_step; one chain per warp.  A ligand of
 * global id g (slot s, position i: g = s * slot_ligands + i) draws the same
 * random streams as ligand g of a batch with ud_search, so a stream of full
 * slots gives the chains of one batch of all its ligands. */
int ud_stream_create(ud_maps maps, const ud_search_params* params, const ud_stream_config* cfg, ud_stream* out);
/* Pack, copy and publish the next slot (1..slot_ligands ligands); *slot = its
 * index.  UD_ERR_STATE while slot (index - ring) is not collected;
 * UD_ERR_CAPACITY past max_slots, for a ligand beyond max_atoms /
 * max_torsions, or when the arena is full. */
int ud_stream_push(ud_stream stream, const ud_ligand* ligs, int n, int* slot);
/* No further slot: the kernel ends once the published slots are done. */
int ud_stream_close(ud_stream stream);
/* Wait until every chain of the slot is done, cluster and refine its modes
 * and compute the final scores (as ud_search_collect for a batch). */
int ud_stream_collect(ud_stream stream, int slot);
/* Results of a collected slot, as ud_result_count / ud_result_mode /
 * ud_result_write and ud_search_chains for a batch (lig = position in the slot). */
int ud_stream_result_count(ud_stream stream, int slot, int lig, int* n_modes);
int ud_stream_result_mode(ud_stream stream, int slot, int lig, int k, float* pose, float energies[8]);
int ud_stream_result_write(ud_stream stream, int slot, int lig, int format, char* buf, size_t cap, size_t* len);
int ud_stream_chains(ud_stream stream, int slot, float* poses, int pose_stride, float* e, int* evals);
/* Wait for the kernel to end (close the stream first, or it ends when a
 * wait for the next slot runs out: UD_ERR_TIMEOUT); *evals = evaluations of
 * the collected slots. */
int ud_stream_finish(ud_stream stream, long long* evals);
int ud_stream_destroy(ud_stream stream);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (roofline
 * denominator of the search kernels).  No counterpart in the reference. */
int ud_device_fp32_peak(float* tflops);
/* Measured L2 read bandwidth of the current device in GB/s: a 32 MB buffer
 * held in L2 read with L2-only 16-byte loads by every SM (the roofline
 * denominator of the search kernel, whose grid maps and pair tables stay
 * L2-resident).  Allocates 32 MB of device memory for the duration of the
 * call.  No counterpart in the reference. */
int ud_device_l2_peak(float* gbs);
/* Evaluations and device time of the last search: the search kernel's own
 * time (between events recorded around it; in the graph form, event nodes
 * inside the graph), without the clustering, refinement and copies after it. */
int ud_search_stats(ud_batch batch, long long* evals, float* kernel_ms);
/* Host-to-device bytes of the batch's last topology upload (ud_batch_create /
 * ud_batch_reset): ligand records, atoms, nodes, pair slots and incidence
 * lists, grid-atom list, work order (and AD4 charges / pair coefficients).
 * No counterpart in the reference (measurement). */
int ud_batch_upload_bytes(ud_batch batch, size_t* bytes);

#ifdef __cplusplus
}
#endif
#endif /* UNIDOCK_B200_H */
