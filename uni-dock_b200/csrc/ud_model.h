// Host-side model of the docking engine: atom typing constants, scoring
// functions and their r^2 tables, ligand torsion trees, receptor atoms and
// pose post-processing.  Everything here runs on the CPU once per input; the
// per-pose arithmetic lives in ud_engine.cu.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

namespace ud {

// ---------------------------------------------------------------- atom types
// Element, AutoDock and X-Score type ids (the ids are an interface shared with
// PDBQT files and the reference's tables: unidock/src/lib/atom_constants.h:28-116).
enum { EL_H = 0, EL_C, EL_N, EL_O, EL_S, EL_P, EL_F, EL_Cl, EL_Br, EL_I, EL_Si, EL_At, EL_Met,
       EL_Dummy, EL_SIZE };
enum { AD_C = 0, AD_A, AD_N, AD_O, AD_P, AD_S, AD_H, AD_F, AD_I, AD_NA, AD_OA, AD_SA, AD_HD,
       AD_Mg, AD_Mn, AD_Zn, AD_Ca, AD_Fe, AD_Cl, AD_Br, AD_Si, AD_At, AD_G0, AD_G1, AD_G2, AD_G3,
       AD_CG0, AD_CG1, AD_CG2, AD_CG3, AD_W, AD_OXA, AD_NXA, AD_OXD, AD_NXD, AD_SIZE };
enum { XS_C_H = 0, XS_C_P, XS_N_P, XS_N_D, XS_N_A, XS_N_DA, XS_O_P, XS_O_D, XS_O_A, XS_O_DA,
       XS_S_P, XS_P_P, XS_F_H, XS_Cl_H, XS_Br_H, XS_I_H, XS_Si, XS_At, XS_Met_D, XS_C_H_CG0,
       XS_C_P_CG0, XS_G0, XS_C_H_CG1, XS_C_P_CG1, XS_G1, XS_C_H_CG2, XS_C_P_CG2, XS_G2,
       XS_C_H_CG3, XS_C_P_CG3, XS_G3, XS_W, XS_O_XA, XS_N_XA, XS_O_XD, XS_N_XD, XS_SIZE };

struct AdKind {
    const char* name;
    float radius, depth, hb_depth, hb_radius, solvation, volume, covalent_radius;
};
const AdKind& ad_kind(int ad);
int ad_type_from_name(const std::string& name);  // AD_SIZE when unknown
bool is_non_ad_metal(const std::string& name);
int ad_to_el(int ad);
float xs_radius(int xs);
float xs_vinardo_radius(int xs);
bool xs_is_hydrophobic(int xs);
bool xs_is_acceptor(int xs);
bool xs_is_donor(int xs);
bool xs_h_bond_possible(int a, int b);
const char* xs_name(int xs);
int xs_from_name(const std::string& s);
float max_covalent_radius();
// Grid map a ligand atom of XS type t reads (CG carbons fold onto C_H/C_P,
// glue atoms and untyped atoms read none: -1).
int xs_grid_type(int t);

inline int tri_index(int i, int j) {  // upper-triangular (i <= j) packed index
    if (i > j) std::swap(i, j);
    return i + j * (j + 1) / 2;
}

// ---------------------------------------------------------------- scoring
enum ScoringChoice { SF_VINA = 0, SF_AD42 = 1, SF_VINARDO = 2 };

struct Scoring {
    int choice = SF_VINA;
    std::vector<float> weights;      // term weights followed by the rotatable-bond weight
    float cutoff = 8.0f;             // pair cutoff (Angstrom)
    float max_cutoff = 8.0f;
    int n_terms = 0;                 // distance-dependent terms (excluding conf-independent)
    static Scoring make(int choice, const float* w, int nw);
    static std::vector<float> default_weights(int choice);
    // Weighted pair energy of XS types (t1,t2) at distance r (type form, Vina/Vinardo).
    float eval_types(int t1, int t2, float r) const;
    // One unweighted term k of the type form.
    float term_types(int k, int t1, int t2, float r) const;
    // Final score from inter+intra energy (num_tors_div / ad4_tors_add).
    float conf_independent(float e, float num_tors, float torsdof) const;
};

// AutoDock 4.2 terms between AD-typed atoms, unweighted (potentials.h:346-486
// with the parameters of scoring_function.h:74-86).
constexpr float kAd4ShortCutoff = 8.0f;   // vdW and H-bond
constexpr float kAd4LongCutoff = 20.48f;  // electrostatics and desolvation
constexpr float kAd4Qsolv = 0.01097f;     // charge-dependent solvation factor
float ad4_vdw(int t1, int t2, float r);
float ad4_hb(int t1, int t2, float r);
float ad4_elec_unit(float r);      // electrostatic energy of two unit charges
float ad4_desolv_gauss(float r);   // distance factor exp(-r^2 / (2 sigma^2)) of desolvation
float ad4_solvation(int ad);
float ad4_volume(int ad);
// AD4 pair-table rows: AD type pairs tri_index(t1, t2), then two rows shared by
// all pairs and scaled per pair: electrostatics (times q1 q2) and the
// charge-dependent desolvation (times |q1| V2 + |q2| V1).
constexpr int kAd4TypePairs = AD_SIZE * (AD_SIZE + 1) / 2;
constexpr int kAd4RowElec = kAd4TypePairs;
constexpr int kAd4RowDesolv = kAd4TypePairs + 1;
constexpr int kAd4Rows = kAd4TypePairs + 2;

// r^2-binned tables with factor 32 (points per A^2): `fast` is the midpoint
// average used for maps/scoring, `smooth` the (e, dE/dr / r) pairs for lerp.
struct PairTable {
    int n = 0;           // bins per type pair
    float factor = 32.f;
    int n_types = 0;     // XS_SIZE
    std::vector<float> fast;    // [tp][bin]
    std::vector<float> smooth;  // [tp][bin][2]
    void build(const Scoring& sf, int term = -1);  // term >= 0: one unweighted term
};
// smooth/fast construction of one row from the tabulated energies at r = sqrt(i/factor)
void table_row_from_energies(const float* e, const float* rs, int n, float* fast, float* smooth);

// ---------------------------------------------------------------- bias
// One entry of an AutoDock-bias style file (BPF; unidock/src/lib/bias.h):
// "x y z Vset r type [AD types...]", a Gaussian well Vset exp(-d^2 / r^2)
// around (x, y, z) for the atoms its type selects.
enum BiasType { BIAS_DON = 0, BIAS_ACC, BIAS_ARO, BIAS_MAP, BIAS_UNKNOWN };
struct BiasElement {
    float xyz[3] = {0, 0, 0};
    float vset = 0, r = 1;
    int type = BIAS_UNKNOWN;
    std::vector<int> ad_list;  // BIAS_MAP: the AD types named (empty: every type)
};
// The entries of a bias file (its first line is a header; blank lines skipped).
std::vector<BiasElement> parse_bias(const std::string& text);
// AD types whose AutoDock 4.2 maps get the well (ad4cache::set_bias,
// ad4cache.cpp:54-88): don HD; acc OA and NA; aro A; map the AD types named,
// or with none named every map, the electrostatic and desolvation maps
// included (all bits set).
uint64_t bias_ad4_map_types(const BiasElement& b);
// XS types whose maps get the well (cache::compute_bias, cache.cpp:789-957):
// acceptor wells the acceptor maps, map wells every map or the types of the
// named AD types' elements; donor and aromatic wells none.
uint64_t bias_map_types(const BiasElement& b);
// Times the well is added to a ligand atom of XS type t when it is scored
// against the receptor atoms (non_cache::eval / eval_deriv, non_cache.cpp:
// 112-400): a CG carbon counts as its C_H / C_P type; a map well counts once
// per named AD type that selects t.
void bias_atom_multiplicity(const BiasElement& b, unsigned char mult[XS_SIZE]);

// ---------------------------------------------------------------- ligand model
struct Atom {
    float lab[3];      // coordinates as read (lab frame of the input pose)
    float local[3];    // coordinates relative to the owning node origin (input frame)
    float charge = 0;
    int ad = AD_SIZE, el = EL_SIZE, xs = XS_SIZE;
    int node = 0;
    int serial = 0;
    std::vector<int> bonds;        // bonded atom indices in bond-detection order
    std::vector<char> bond_rot;    // rotatable flags of the bonds
};

struct Node {
    int parent = -1;
    int begin = 0, end = 0;        // atom range [begin, end)
    float rel_origin[3] = {0, 0, 0};  // origin relative to parent origin (input frame)
    float rel_axis[3] = {0, 0, 0};    // unit rotation axis (input frame)
    float origin0[3] = {0, 0, 0};     // input-frame origin
};

struct Pair {
    int a, b, tp;
};

struct Ligand {
    std::string name;
    std::vector<Atom> atoms;
    std::vector<Node> nodes;           // DFS pre-order; node k >= 1 owns torsion k-1
    std::vector<Pair> pairs;           // intramolecular pairs (1-4 and beyond), XS typing
    std::vector<Pair> glue_pairs;
    std::vector<Pair> pairs_ad;        // the same with AutoDock typing (hydrogens included)
    std::vector<Pair> glue_pairs_ad;
    std::vector<std::pair<std::string, int>> context;  // input lines; atom index or -1
    int torsdof = 0;
    bool sdf = false;
    int n_torsions() const { return (int)nodes.size() - 1; }
    int n_heavy() const;
    // conf_independent_inputs (num_tors, num_rotors, heavy, hydrophobic, h-bond, ligands, length)
    std::array<float, 7> conf_indep_inputs() const;
};

// Parse a Vina PDBQT ligand (ROOT/BRANCH/TORSDOF) and build torsion tree,
// bonds, types and pairs.  Throws std::runtime_error on malformed input.
Ligand parse_ligand_pdbqt(const std::string& text, int atom_typing_xs = 1);

// SDF (V2000) ligand carrying fragInfo / torsionInfo / atomInfo properties;
// keep_h keeps AutoDock type H atoms in the fragments (the reference CLI always does).
Ligand parse_ligand_sdf(const std::string& text, bool keep_h = true, int atom_typing_xs = 1);
bool looks_like_sdf(const std::string& text);
// SDF when the text is a V2000 molfile, PDBQT otherwise.
Ligand parse_ligand(const std::string& text, bool keep_h = true, int atom_typing_xs = 1);

// Receptor atoms with types assigned from bonds (rigid receptor).
struct Receptor {
    std::vector<std::array<float, 3>> xyz;
    std::vector<int> ad, el, xs;
    std::vector<float> charge;
};
Receptor parse_receptor_pdbqt(const std::string& text);

// Forward kinematics on the host (used for output writing and clustering):
// pose = [x y z qw qx qy qz t0 ...]; fills lab coordinates of all atoms.
void ligand_coords(const Ligand& lig, const float* pose, float* xyz_out);

// ---------------------------------------------------------------- output
struct PoseResult {
    std::vector<float> pose;  // 7 + T
    float e = 0, inter = 0, intra = 0, total = 0, conf_indep = 0, unbound = 0, lb = 0, ub = 0;
    std::vector<float> heavy_xyz;
};
// Input record of the ligand with the coordinates of one pose, no remarks.
std::string write_structure(const Ligand& lig, const float* pose);
std::string write_pdbqt_models(const Ligand& lig, const std::vector<PoseResult>& poses,
                               bool ad4);
std::string write_sdf_models(const Ligand& lig, const std::vector<PoseResult>& poses, bool ad4);

}  // namespace ud
