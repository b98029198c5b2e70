// Device-side data layout of the docking engine and the host entry points
// into ud_engine.cu.  Host C++ (CUDA runtime types only) so the C-ABI layer
// and the host model code can include it.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace ud {

constexpr int kMaxLigAtoms = 256;  // atom indices packed in 8 bits in pair records
constexpr int kMaxLigTorsions = 48;
constexpr int kMaxNodes = kMaxLigTorsions + 1;
constexpr int kTableBins = 2051;   // Vina/Vinardo r^2 bins (factor 32, cutoff 8 A)

// Grid maps of one receptor box: x fastest, one map per requested XS type.
struct MapsDesc {
    int dims[3];           // sample points per axis (n_voxels + 1)
    float init[3];         // box corner (grid::m_init)
    float factor[3];       // samples per Angstrom (grid::m_factor)
    float factor_inv[3];
    float dim_m1[3];       // dims - 1 as float
    float corner2[3];      // box end
    float slope;           // out-of-box penalty slope
    int n_maps;
    int8_t slot_of_xs[36]; // map slot per XS grid type (per AD type for AD4), -1 when absent
    int ad4;               // AutoDock 4.2 maps: type maps, then the electrostatic and desolvation maps
    int e_slot, d_slot;    // AD4: slots of the electrostatic and desolvation maps
};

// AD4 pair-table rows scaled per pair (after the AD type-pair rows)
constexpr int kAd4TableRowElec = 35 * 36 / 2;
constexpr int kAd4TableRowDesolv = kAd4TableRowElec + 1;

// One ligand's topology as it sits in device memory (offsets into the batch
// arrays).  Nodes are in DFS pre-order: node k >= 1 owns torsion k - 1.
struct LigDesc {
    int atom_off, n_atoms;
    int node_off, n_nodes;
    int pair_off, n_pairs;
    int n_heavy;
    int max_depth;
    int local_steps;       // BFGS iteration cap of this ligand
    int grid_off, n_grid;  // atoms with a grid map: list of atom | slot << 8
    int pad;
};
static_assert(sizeof(LigDesc) == 48, "LigDesc layout");

struct NodeRec {            // 40 bytes
    float rel_origin[3];
    float rel_axis[3];
    int parent;
    int depth;
    int atoms;             // atoms of the node's subtree (DFS order): begin | end << 16
    int subtree_end;       // one past the last node of this node's subtree
};

// Pair records are a | b << 8 | type_pair << 16; this value pads a 32-pair
// group of the conflict-free pair order and is skipped.
constexpr uint32_t kPairPad = 0xFFFF0000u;
// A 32-slot pair group is kPairPasses lane ranges of 32 / kPairPasses slots,
// each a matching (no atom twice), whose forces are added one range at a time.
constexpr int kPairPasses = 4;
constexpr int kPairPassWidth = 32 / kPairPasses;

// Atom record: local xyz and packed fields (node | (map slot + 1) << 8 |
// heavy << 16 | (xs + 1) << 24).
struct AtomRec {
    float x, y, z;
    int packed;
};

struct SearchParams {
    int global_steps;
    int exhaustiveness;    // chains per ligand
    unsigned long long seed;
    float hunt_cap;        // curl cap during the search (10)
    float authentic_v;     // curl cap of the refinement (1000)
    float temperature;     // Metropolis temperature (1.2)
    float mutation_amplitude;
    int lanes_per_chain;   // 32 (a warp per chain) or 16 (two chains per warp)
    int chains_per_block;  // warps per CTA (1..4)
    int persistent;        // 0: plain fixed-tiling launch, 1: persistent queue
    int bfgs_cap;          // 0: per-ligand local_steps; >0: min(local_steps, cap)
};

// Control of a streaming screen (ud_stream_*): one persistent search over an
// append-only device arena that the host fills slot by slot.  Slot s holds up
// to slot_ligands ligands with global ids s * slot_ligands + local index; its
// chains are the items [s * slot_ligands * E, (s + 1) * slot_ligands * E) of
// the work counter.  The host copies a slot's topology, order, ligand count
// and chain count into device memory, then the new published count (the
// copies are ordered on one stream); a warp whose item lies in an unpublished
// slot waits, with a time limit, for the count to pass it.  Chain results go
// to a ring of `ring` result areas (slot s to area s % ring; the host reuses an
// area only after it has taken the results out), and the warp finishing a
// slot's last chain sets done_host[s] in host-mapped memory.
struct StreamView {
    const unsigned int* published;   // slots whose data is in device memory
    const unsigned int* closed;      // 1 once the host publishes nothing more
    unsigned int* next_item;         // work counter
    unsigned int* slot_left;         // per slot: chains not finished yet
    const int* slot_nlig;            // per slot: ligands
    const int* order;                // per slot, slot_ligands entries: global ligand ids, costliest first
    unsigned int* done_host;         // host-mapped, per slot: 1 when all its chains are finished
    int* status;                     // 0, or kStreamTimeout when a wait ran out
    int slot_ligands;
    int max_slots;
    int ring;
    int reserve_every;               // blocks on SMs whose id is a multiple of this return at once (0: none)
    unsigned long long timeout_ns;   // longest wait for a publication
};
constexpr int kStreamTimeout = 1;

// AutoDock 4.2 atom-kind parameters indexed by AD type (atom_constants.h
// ad_type_property) and the set of maps an AD4 map build computes.
constexpr int kAdTypes = 35;
struct Ad4Params {
    float radius[kAdTypes], depth[kAdTypes], hb_depth[kAdTypes], hb_radius[kAdTypes];
    float solvation[kAdTypes], volume[kAdTypes];
};
struct Ad4MapSpec {
    int n_slots;           // type maps; the electrostatic and desolvation maps follow them
    int slot_ad[36];       // AD type of each type map
    float w_vdw, w_hb, w_elec, w_dsolv;
};

// Capacity of the allocation-free search (ud_search_device_noalloc): chains
// (ligands x exhaustiveness) per call.
constexpr int kNoAllocMaxChains = 131072;

// Result record of one chain.
struct ChainResult {
    float e;               // best energy (refined, authentic cap)
    int evals;             // energy+gradient evaluations spent
    int ligand;
    int chain;
    float e_grid;          // scoring-path energies of the best pose at the authentic cap:
    float e_intra;         // grid (cache::eval) and intramolecular (nearest-bin table)
};

// ---------------------------------------------------------------- device views
// Device pointers of one batch, one set of maps, the scoring tables and the
// per-term data of weight gradients, as handed to the launchers below.
struct DeviceBatchView {
    const LigDesc* ligs;
    const AtomRec* atoms;
    const NodeRec* nodes;
    const uint32_t* pairs;
    const uint32_t* grid_list;
    int max_atoms, max_torsions;
    const float* charges;    // AD4: per atom
    const float* pair_coef;  // AD4: float2 per pair slot
    int ad4;
};

struct DeviceMapsView {
    const float* data;
    MapsDesc desc;
    const float2* xpairs;  // [slot][z][y][x] = (data at x, data at x + 1; x + 1 clamped to the last point)
};

struct DeviceTablesView {
    const float* smooth;   // float4 per bin: (e, dor) of the bin and the next
    const float* fast;
    int n_bins;
    float factor;
    float cutoff2;
};

struct DeviceTermsView {
    const float* maps;     // [term][slot][z][y][x], unweighted term maps
    const float* rows;     // float4 per bin: [term][tp][bin], laid out as DeviceTablesView::smooth
    int n_terms;
    long long map_block;   // floats per term in `maps`
    long long row_block;   // float4 per term in `rows`
};

// A bias well as the receptor-atom scoring adds it to a ligand atom: the well
// (x, y, z, Vset, r) and, per XS type of the atom, how many times it counts
// (a CG carbon counts as its C_H / C_P type).
struct BiasRec {
    float x, y, z, vset;
    float r;
    float pad[3];
    unsigned char mult[36];
    unsigned char pad2[12];
};
static_assert(sizeof(BiasRec) == 80, "BiasRec layout");

// A bias well as a map build adds it: the well and the map slots it reaches.
struct BiasMapRec {
    float x, y, z, vset, r;
    unsigned int slots_lo, slots_hi;  // bit s: map slot s
    float pad;
};

// Receptor atoms for scoring without maps (the reference's non_cache, used to
// refine and rescore poses): a uniform grid of cubic cells over the box; cell c
// lists, in receptor order, every typed receptor atom within the cutoff of some
// point of the cell, as (x, y, z, XS type as int bits).  Positions are clamped
// into the box before the lookup, so every query lands in a cell.
struct DeviceReceptorView {
    const float* atoms;    // float4 per entry, grouped by cell
    const int* start;      // [cells + 1] entry offsets
    int n[3];              // cells per axis
    float begin[3], end[3];// the box (grid_dims begin / end)
    float inv_cell;        // 1 / cell edge
    const BiasRec* bias;   // bias wells of the maps (used for ligands without their own)
    int n_bias;
    const BiasRec* lig_bias;       // per-ligand bias wells, all ligands' lists back to back
    const int* lig_bias_span;      // per ligand: offset | count << 16 into lig_bias (0: none)
};

// Modes of the receptor-atom kernel.
enum ReceptorMode : int {
    kRecEnergyGrad = 0,    // energy and gradient at fixed poses (model::eval_deriv with non_cache)
    kRecRefine = 1,        // refinement rounds, then the final scoring energies
    kRecScore = 2          // scoring energies only (non_cache::eval, model::evali)
};

// ---------------------------------------------------------------- launchers (ud_engine.cu)
cudaError_t launch_maps(const float* rec_xyzt, int n_rec, const float* fastT, int n_bins, int n_slots,
                        int n_slots_pad, float factor, float cutoff2, const MapsDesc& d, float* out,
                        cudaStream_t stream);
cudaError_t launch_score(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                         const int* pose_lig, const float* poses, int pose_stride, int n_poses,
                         float v_intra, float v_inter, float* e_out, float* g_out, int g_stride,
                         float* score_out, cudaStream_t stream);
cudaError_t launch_adjoint(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                           const DeviceTermsView& terms, int n_ligands, const int* pose_lig, const float* poses,
                           int pose_stride, int n_poses, float v_intra, float v_inter, int exact, float* e_out,
                           float* g_out, int g_stride, float* dw_out, int dw_stride, cudaStream_t stream);
// AD4 maps: type maps of spec.slot_ad, then the electrostatic and desolvation
// maps; receptor atoms as (x, y, z, charge) plus their AD types
cudaError_t launch_maps_ad4(const float* rec_xyzq, const int* rec_ad, int n_rec, const Ad4Params& params,
                            const Ad4MapSpec& spec, const MapsDesc& d, float* out, cudaStream_t stream);
// out[i] = sum_t w[t] * in[t * block + i], i < block (a multiple of 4, 16-byte aligned buffers)
cudaError_t launch_combine_terms(const float* in, long long block, int n_terms, const float* w, float* out,
                                 cudaStream_t stream);
cudaError_t launch_search(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                          const SearchParams& P, const int* order, int n_items, int first_item,
                          unsigned int* queue, float* poses, int pose_stride, ChainResult* results,
                          int grid_blocks, cudaStream_t stream);
// CTAs of `warps` warps (chains of lanes_per_chain = 32 or 16 lanes) resident per SM
int search_blocks_per_sm(const DeviceBatchView& b, int warps, int lanes_per_chain = 32);
cudaError_t launch_optimize(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                            const int* pose_lig, float* poses, int pose_stride, int n_poses, int max_steps,
                            float v, float* e_out, int* evals_out, cudaStream_t stream);
// The x-pair copy of the maps (DeviceMapsView::xpairs) from `maps`.
cudaError_t launch_map_xpairs(const float* maps, const MapsDesc& d, float2* out, cudaStream_t stream);
float measure_fp32_peak_tflops();
float measure_l2_read_gbs();
// The persistent search of a streaming screen (StreamView) on `blocks` CTAs:
// the batch view is the arena (LigDesc offsets absolute), the poses and
// results are the ring of result areas.
cudaError_t launch_search_stream(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                                 const SearchParams& P, const StreamView& sv, float* poses, int pose_stride,
                                 ChainResult* results, int blocks, cudaStream_t stream);
int stream_blocks_per_sm(const DeviceBatchView& b, int warps);
// Loads the per-slot clustering kernel (and the refinement kernel when
// `refine`) into the context and raises their shared-memory limits to the
// stream's largest layout (`b`), so that launching them while the persistent
// stream kernel runs needs no module load (a lazy load waits for the kernels
// running in the context, the persistent one included) and no attribute change.
cudaError_t prepare_stream_post(const DeviceBatchView& b, int cap, bool refine);
// The persistent search over the batch's device-resident work order `d_order`
// with the library's static scratch (queue counter, per-chain records) in
// place of device allocations; per-chain energies / evaluations written to
// the caller's device buffers.
cudaError_t launch_search_noalloc(const DeviceBatchView& b, const DeviceMapsView& m, const DeviceTablesView& t,
                                  const SearchParams& P, const int* d_order, int n_ligands, int grid_blocks,
                                  float* poses, int pose_stride, float* e_out, int* evals_out,
                                  cudaStream_t stream);
int engine_chain_smem_bytes(int max_atoms, int max_torsions);
// Bias wells added to the maps (cache::compute_bias): every map point of every
// slot a well reaches gets Vset exp(-d^2 / r^2) when that is below -0.01,
// wells in list order.
cudaError_t launch_bias_maps(const BiasMapRec* bias, int n_bias, const MapsDesc& d, float* maps,
                             cudaStream_t stream);
// Per-ligand clustering of the chain results (warp per ligand) into at most
// `cap` modes: n_modes[lig], and per mode slot lig * cap + k its chain, its
// ligand (-1 for an unused slot) and a copy of the chain's pose.
// scratch: n_ligands * cap * 3 * max_atoms floats.
cudaError_t launch_cluster(const DeviceBatchView& b, const float* poses, int pose_stride, const ChainResult* results,
                           int n_ligands, int exhaustiveness, int cap, float min_rmsd, float* scratch, int* n_modes,
                           int* mode_chain, int* mode_lig, float* mode_pose, cudaStream_t stream);
// Receptor-atom scoring of poses (one warp per pose, pose_lig < 0 skipped):
//   kRecEnergyGrad: e_out[i] and g_out (6 + T per pose, stride g_stride) at slope / cap v;
//   kRecRefine:     refinement rounds (slope 100 * 100^p, curl cap v) updating poses in place,
//                   out4[i] = (last BFGS energy, inter at slope 1e6, intra, inside box 1/0);
//   kRecScore:      out4[i] = (0, inter at slope 1e6, intra, inside box 1/0), caps v.
cudaError_t launch_receptor(int mode, const DeviceBatchView& b, const DeviceTablesView& t,
                            const DeviceReceptorView& r, const int* pose_lig, float* poses, int pose_stride,
                            int n_poses, int refine_step, float slope, float v, float* e_out, float* g_out,
                            int g_stride, float* out4, cudaStream_t stream);

}  // namespace ud
