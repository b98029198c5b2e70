// Test-only C interface over the REFERENCE's own CPU sources (unidock/src/lib),
// compiled by oracle/Makefile into oracle/_ref/libudref.so.  It is the checker
// that pins the oracle restatement and the CUDA engine to the reference: maps
// (cache::populate_no_bias), ligand parsing (parse_ligand_pdbqt_from_file_no_failure),
// fixed-pose energy/gradient (model::eval_deriv, model::eval_intramolecular,
// cache::eval), local optimisation (quasi_newton) and the CPU Monte-Carlo chain
// (the loop of monte_carlo::operator(), unidock/src/cuda/monte_carlo.cu:2319-2356,
// restated here around the reference's mutate_conf / quasi_newton / output container).
//
// Only tests/, the oracle leg of bench.py and __graft_entry__.smoke() load this.
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <vector>

#include "ad4cache.h"
#include "cache.h"
#include "coords.h"
#include "model.h"
#include "mutate.h"
#include "non_cache.h"
#include "parse_pdbqt.h"
#include "precalculate.h"
#include "quasi_newton.h"
#include "ref_driver.h"
#include "scoring_function.h"

namespace {

thread_local std::string g_err;

flv to_flv(const float* w, int n) { return flv(w, w + n); }

conf make_conf(const model& m, const float* pos, const float* quat, const float* tors) {
    conf c(m.get_size());
    c.ligands[0].rigid.position = vec(pos[0], pos[1], pos[2]);
    c.ligands[0].rigid.orientation = qt(quat[0], quat[1], quat[2], quat[3]);
    for (sz i = 0; i < c.ligands[0].torsions.size(); ++i) c.ligands[0].torsions[i] = tors[i];
    return c;
}

void read_conf(const conf& c, float* pos, float* quat, float* tors) {
    const auto& r = c.ligands[0].rigid;
    for (int i = 0; i < 3; ++i) pos[i] = r.position[i];
    quat[0] = r.orientation.R_component_1();
    quat[1] = r.orientation.R_component_2();
    quat[2] = r.orientation.R_component_3();
    quat[3] = r.orientation.R_component_4();
    for (sz i = 0; i < c.ligands[0].torsions.size(); ++i) tors[i] = c.ligands[0].torsions[i];
}

bool metropolis(fl old_f, fl new_f, fl temperature, rng& generator) {
    if (new_f < old_f) return true;
    const fl p = std::exp((old_f - new_f) / temperature);
    return random_fl(0, 1, generator) < p;
}

}  // namespace

extern "C" {

const char* udref_last_error() { return g_err.c_str(); }

// Grid maps of cache::populate_no_bias for a typed receptor given as arrays.
// Box set up as Vina::compute_vina_maps (unidock/src/lib/vina.cpp:528-539).
void* udref_maps_new(int sf_choice, const float* weights, int n_weights, const float* xyz,
                     const int* xs, int n_atoms, const float* center, const float* size,
                     float spacing, const int* types, int n_types) {
    try {
        auto h = new RefMaps();
        h->sf = std::make_shared<ScoringFunction>((scoring_function_choice)sf_choice,
                                                  to_flv(weights, n_weights));
        h->rec = model(atom_type::XS);
        for (int i = 0; i < n_atoms; ++i) {
            atom a;
            a.coords = vec(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
            a.xs = (sz)xs[i];
            a.ad = AD_TYPE_C;
            a.el = EL_TYPE_C;
            h->rec.grid_atoms.push_back(a);
        }
        VINA_FOR_IN(i, h->gd) {
            h->gd[i].n_voxels = sz(std::ceil(fl(size[i]) / fl(spacing)));
            fl real_span = fl(spacing) * h->gd[i].n_voxels;
            h->gd[i].begin = fl(center[i]) - real_span / 2;
            h->gd[i].end = h->gd[i].begin + real_span;
        }
        h->pre.reset(new precalculate(*h->sf));
        h->grid = cache(h->gd, 1e6);
        szv needed(types, types + n_types);
        h->grid.populate_no_bias(h->rec, *h->pre, needed);
        return h;
    } catch (...) {
        g_err = "udref_maps_new failed";
        return nullptr;
    }
}

void udref_maps_free(void* h) { delete (RefMaps*)h; }

// dims[3] = sample points per axis; begin[3]; factor[3] (points per Angstrom as grid::m_factor)
int udref_maps_dims(void* hh, int* dims, float* begin, float* factor, float* factor_inv) {
    auto h = (RefMaps*)hh;
    const grid& g = h->grid.m_grids[XS_TYPE_C_H].initialized() ? h->grid.m_grids[XS_TYPE_C_H]
                                                                 : h->grid.m_grids[XS_TYPE_O_A];
    dims[0] = (int)g.m_data.dim0();
    dims[1] = (int)g.m_data.dim1();
    dims[2] = (int)g.m_data.dim2();
    for (int i = 0; i < 3; ++i) {
        begin[i] = g.m_init[i];
        factor[i] = g.m_factor[i];
        factor_inv[i] = g.m_factor_inv[i];
    }
    return 0;
}

int udref_maps_get(void* hh, int xs_type, float* out) {
    auto h = (RefMaps*)hh;
    const grid& g = h->grid.m_grids[xs_type];
    if (!g.initialized()) return -1;
    std::memcpy(out, g.m_data.m_data.data(), g.m_data.m_data.size() * sizeof(float));
    return (int)g.m_data.m_data.size();
}

// eval_fast of the type-pair table precalculate::eval_fast (precalculate.h:40-47, 169-172)
float udref_table_fast(void* hh, int t1, int t2, float r2) {
    auto h = (RefMaps*)hh;
    sz n = num_atom_types(h->sf->get_atom_typing());
    return h->pre->eval_fast(triangular_matrix_index_permissive(n, t1, t2), r2);
}

// Ligand parsed by the reference parser (parse_pdbqt.cpp:1076-1140), per-atom-pair tables
// precalculate_byatom (precalculate.h:206-241).
void* udref_ligand_new(const char* path, int sf_choice, const float* weights, int n_weights) {
    try {
        auto h = new RefLigand();
        h->sf = std::make_shared<ScoringFunction>((scoring_function_choice)sf_choice,
                                                  to_flv(weights, n_weights));
        // .pdbqt / .sdf dispatch on the file name with hydrogens kept, as the
        // reference CLI loads ligands (main.cpp:858-863, parse_pdbqt.cpp:1076-1087)
        h->m = parse_ligand_from_file_no_failure(path, h->sf->get_atom_typing(), true);
        if (h->m.num_ligands() != 1) {
            delete h;
            g_err = "parse failed";
            return nullptr;
        }
        h->pre.reset(new precalculate_byatom(*h->sf, h->m));
        return h;
    } catch (...) {
        g_err = "udref_ligand_new failed";
        return nullptr;
    }
}

void udref_ligand_free(void* h) { delete (RefLigand*)h; }

// counts[0]=atoms, [1]=movable atoms, [2]=torsions, [3]=intra pairs, [4]=rigid nodes
int udref_ligand_counts(void* hh, int* counts) {
    auto h = (RefLigand*)hh;
    const ligand& lig = h->m.ligands[0];
    counts[0] = (int)h->m.num_atoms();
    counts[1] = (int)h->m.num_movable_atoms();
    counts[2] = (int)h->m.get_size().ligands[0];
    counts[3] = (int)lig.pairs.size();
    int nodes = 1 + counts[2];
    counts[4] = nodes;
    return 0;
}

// Per atom: lab coords of the initial pose, local coords (atom::coords), xs, ad, el, charge.
int udref_ligand_atoms(void* hh, float* lab, float* local, int* xs, int* ad, int* el,
                       float* charge) {
    auto h = (RefLigand*)hh;
    for (sz i = 0; i < h->m.num_atoms(); ++i) {
        const atom& a = h->m.atoms[i];
        for (int k = 0; k < 3; ++k) {
            lab[3 * i + k] = h->m.coords[i][k];
            local[3 * i + k] = a.coords[k];
        }
        xs[i] = (int)a.xs;
        ad[i] = (int)a.ad;
        el[i] = (int)a.el;
        charge[i] = a.charge;
    }
    return 0;
}

int udref_ligand_pairs(void* hh, int* a, int* b) {
    auto h = (RefLigand*)hh;
    const auto& pairs = h->m.ligands[0].pairs;
    for (sz i = 0; i < pairs.size(); ++i) {
        a[i] = (int)pairs[i].a;
        b[i] = (int)pairs[i].b;
    }
    return (int)pairs.size();
}

namespace {
void walk_tree(const branch& b, int parent, std::vector<int>& par, std::vector<int>& beg,
               std::vector<int>& end, std::vector<float>& org) {
    int me = (int)par.size();
    par.push_back(parent);
    beg.push_back((int)b.node.begin);
    end.push_back((int)b.node.end);
    for (int k = 0; k < 3; ++k) org.push_back(b.node.relative_origin[k]);
    for (int k = 0; k < 3; ++k) org.push_back(b.node.relative_axis[k]);
    for (const auto& c : b.children) walk_tree(c, me, par, beg, end, org);
}
}  // namespace

// Torsion tree in DFS pre-order: parent[], atom ranges, relative origin/axis (6 floats).
int udref_ligand_tree(void* hh, int* parent, int* begin, int* end, float* rel) {
    auto h = (RefLigand*)hh;
    const ligand& lig = h->m.ligands[0];
    std::vector<int> par{-1}, beg{(int)lig.node.begin}, en{(int)lig.node.end};
    std::vector<float> org{0, 0, 0, 0, 0, 0};
    for (const auto& c : lig.children) walk_tree(c, 0, par, beg, en, org);
    for (sz i = 0; i < par.size(); ++i) {
        parent[i] = par[i];
        begin[i] = beg[i];
        end[i] = en[i];
        for (int k = 0; k < 6; ++k) rel[6 * i + k] = org[6 * i + k];
    }
    return (int)par.size();
}

int udref_initial_conf(void* hh, float* pos, float* quat, float* tors) {
    auto h = (RefLigand*)hh;
    read_conf(h->m.get_initial_conf(), pos, quat, tors);
    return 0;
}

// Conformation-independent inputs (conf_independent.cpp:65-99): num_tors etc.
int udref_ligand_conf_indep(void* hh, float* out7) {
    auto h = (RefLigand*)hh;
    conf_independent_inputs in(h->m);
    flv v = in;
    for (int i = 0; i < 7; ++i) out7[i] = v[i];
    return 0;
}

// model::set + model::eval_deriv (model.cpp:935-962); g has 6+T floats in change order.
float udref_eval_deriv(void* lh, void* mh, const float* pos, const float* quat,
                       const float* tors, float v_intra, float v_inter, float* g,
                       float* coords_out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    conf c = make_conf(L->m, pos, quat, tors);
    L->m.set(c);
    change ch(L->m.get_size());
    vec v(v_intra, v_inter, v_inter);
    fl e = L->m.eval_deriv(*L->pre, *M->ig, v, ch);
    for (sz i = 0; i < ch.num_floats(); ++i) g[i] = ch(i);
    if (coords_out)
        for (sz i = 0; i < L->m.num_atoms(); ++i)
            for (int k = 0; k < 3; ++k) coords_out[3 * i + k] = L->m.coords[i][k];
    return e;
}

// Scoring-path energies at a fixed pose: out[0] = cache::eval (grid, cache.cpp:84-120),
// out[1] = model::evali (intra pairs with eval_fast, model.cpp:927-933),
// out[2] = model::eval_intramolecular (model.cpp:964-1000), out[3] = final Vina score
// conf_independent(inter + intra - intra_best) with intra_best = out[2] (vina.cpp:1168-1243).
int udref_score(void* lh, void* mh, const float* pos, const float* quat, const float* tors,
                float v, float* out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    conf c = make_conf(L->m, pos, quat, tors);
    L->m.set(c);
    vec vv(v, v, v);
    fl grid_e = M->ig->eval(L->m, v);
    fl lig_intra = L->m.evali(*L->pre, vv);
    fl intra_mol = L->m.eval_intramolecular(*L->pre, *M->ig, vv);
    out[0] = grid_e;
    out[1] = lig_intra;
    out[2] = intra_mol;
    out[3] = L->sf->conf_independent(L->m, grid_e + lig_intra - intra_mol);
    return 0;
}

// quasi_newton (quasi_newton.cpp:42-53) from the given pose; pose updated in place.
float udref_bfgs(void* lh, void* mh, float* pos, float* quat, float* tors, float v,
                 int max_steps, int* evalcount) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    conf c = make_conf(L->m, pos, quat, tors);
    output_type out(c, 0);
    change g(L->m.get_size());
    quasi_newton qn;
    qn.max_steps = (unsigned)max_steps;
    int ec = 0;
    qn(L->m, *L->pre, *M->ig, out, g, vec(v, v, v), ec);
    read_conf(out.c, pos, quat, tors);
    if (evalcount) *evalcount = ec;
    return out.e;
}

// The receptor-atom scorer Vina::compute_vina_maps keeps unless --no_refine
// (vina.cpp:557-562), and the docking model it scores: the receptor with the
// ligand appended, as set_ligand_from_object_gpu builds each ligand's model.
static non_cache& nc_of(RefMaps* M) {
    if (!M->nc) M->nc.reset(new non_cache(M->rec, M->gd, M->pre.get(), 1e6, M->bias));
    return *M->nc;
}
static model docking_model(RefMaps* M, RefLigand* L) {
    model mm = M->rec;
    mm.append(L->m);
    mm.bias_list = L->bias;  // as set_ligand_from_object_gpu sets it for --multi_bias
    return mm;
}

// Bias wells of a BPF text: header line, then one well per line (Vina::set_bias, vina.cpp:1472-1480).
static std::vector<bias_element> parse_bpf(const char* text) {
    std::vector<bias_element> out;
    std::istringstream in(text);
    std::string line;
    std::getline(in, line);
    while (std::getline(in, line)) {
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        std::istringstream l(line);
        out.emplace_back(l);
    }
    return out;
}

// --bias: the wells added to the maps (cache::compute_bias) and kept for non_cache.
int udref_maps_bias(void* mh, const char* text) {
    auto M = (RefMaps*)mh;
    std::vector<bias_element> wells = parse_bpf(text);
    M->grid.compute_bias(M->rec, wells);
    M->bias.insert(M->bias.end(), wells.begin(), wells.end());
    M->nc.reset();
    return (int)M->bias.size();
}

// --bias on AutoDock 4.2 maps read from files: ad4cache::set_bias
// (ad4cache.cpp:54-88), as Vina::load_maps applies it (vina.cpp:577-586).
int udref_ad4_bias(void* mh, const char* text) {
    auto M = (RefMaps*)mh;
    const std::vector<bias_element> wells = parse_bpf(text);
    M->ad4.set_bias(wells);
    return (int)wells.size();
}

// Values of AD4 map t (an AD type, or AD_TYPE_SIZE / AD_TYPE_SIZE + 1 for the
// electrostatic / desolvation map), x fastest; -1 when the map is absent.
int udref_ad4_map_get(void* mh, int t, float* out) {
    auto M = (RefMaps*)mh;
    if (t < 0 || t >= (int)M->ad4.m_grids.size()) return -1;
    const grid& g = M->ad4.m_grids[t];
    if (!g.initialized()) return -1;
    const auto& v = g.m_data.m_data;
    for (size_t i = 0; i < v.size(); ++i) out[i] = (float)v[i];
    return (int)v.size();
}

// --multi_bias: the ligand's own wells.
int udref_ligand_bias(void* lh, const char* text) {
    auto L = (RefLigand*)lh;
    L->bias = parse_bpf(text);
    return (int)L->bias.size();
}

// model::eval_deriv against the receptor atoms (non_cache::eval_deriv,
// non_cache.cpp:420-500) at out-of-box slope `slope`, curl caps v.
float udref_nc_eval_deriv(void* lh, void* mh, const float* pos, const float* quat, const float* tors, float slope,
                          float v, float* g) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    non_cache& nc = nc_of(M);
    nc.slope = slope;
    model mm = docking_model(M, L);
    conf c = make_conf(mm, pos, quat, tors);
    mm.set(c);
    change ch(mm.get_size());
    fl e = mm.eval_deriv(*L->pre, nc, vec(v, v, v), ch);
    for (sz i = 0; i < ch.num_floats(); ++i) g[i] = ch(i);
    nc.slope = 1e6;
    return e;
}

// The refinement of one pose in Vina::global_search_gpu (vina.h:251-272): up to
// refine_step rounds of quasi_newton against the receptor atoms at slope
// 100 * 10^(2p), stopping once the heavy atoms are inside the box; then
// non_cache::eval at slope 1e6 and model::evali at the authentic cap
// (score_gpu, vina.cpp:1245-1283).  Pose updated in place; out[0] = the last
// quasi_newton energy, out[1] = inter (receptor atoms), out[2] = intra;
// returns 1 when the pose ended inside the box.
int udref_refine(void* lh, void* mh, float* pos, float* quat, float* tors, int refine_step, float* out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    non_cache& nc = nc_of(M);
    model mm = docking_model(M, L);
    conf c = make_conf(mm, pos, quat, tors);
    output_type o(c, 0);
    change g(mm.get_size());
    quasi_newton qn;
    qn.max_steps = unsigned((25 + mm.num_movable_atoms()) / 3);
    const vec authentic_v(1000, 1000, 1000);
    int evalcount = 0;
    VINA_FOR(p, refine_step) {
        nc.slope = 100 * std::pow(10.0, 2.0 * p);
        qn(mm, *L->pre, nc, o, g, authentic_v, evalcount);
        if (nc.within(mm)) break;
    }
    const int within = nc.within(mm) ? 1 : 0;
    nc.slope = 1e6;
    read_conf(o.c, pos, quat, tors);
    mm.set(o.c);
    out[0] = o.e;
    out[1] = nc.eval(mm, authentic_v[1]);
    out[2] = mm.evali(*L->pre, authentic_v);
    return within;
}

// Scoring-path energies against the receptor atoms at a fixed pose (Vina::score
// without --no_refine, vina.cpp:1168-1243): out[0] = non_cache::eval (slope 1e6,
// cap v), out[1] = model::evali, out[2] = model::eval_intramolecular.
int udref_nc_score(void* lh, void* mh, const float* pos, const float* quat, const float* tors, float v, float* out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    non_cache& nc = nc_of(M);
    nc.slope = 1e6;
    model mm = docking_model(M, L);
    conf c = make_conf(mm, pos, quat, tors);
    mm.set(c);
    vec vv(v, v, v);
    out[0] = nc.eval(mm, v);
    out[1] = mm.evali(*L->pre, vv);
    out[2] = mm.eval_intramolecular(*L->pre, nc, vv);
    return 0;
}

// Final scores of one ligand's modes as Vina::global_search_gpu computes them
// after its search (vina.h:232-343 with score_gpu, vina.cpp:1245-1322), from
// the modes' poses as they stand after any refinement:
//   Vina / Vinardo: the poses are ordered by `order_e` (the refinement's last
//     energy, or max when a pose ended outside the box), the intramolecular
//     energy of the first is taken (model::eval_intramolecular against the
//     receptor atoms when `receptor`, else the maps), and each pose scores
//     conf_independent(inter + intra - that energy), inter from non_cache::eval
//     (slope 1e6) or the maps at cap 1000;
//   AD4: inter from the maps, total = inter + conf_independent(0), unbound -intra.
// The poses are then sorted by that total and the RMSD bounds taken against
// the best.  out (9 floats per mode, in final order): input index, total,
// rmsd lb, rmsd ub, inter + intra, inter, intra, conf-independent part, unbound.
int udref_final_scores(void* lh, void* mh, int n, const float* poses, int pose_stride, const float* order_e,
                       int receptor, float* out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    const bool ad4 = L->sf->get_atom_typing() == atom_type::AD;
    const vec authentic_v(1000, 1000, 1000);
    model mm = receptor ? docking_model(M, L) : L->m;
    const igrid& scorer = receptor ? static_cast<const igrid&>(nc_of(M)) : *M->ig;
    if (receptor) nc_of(M).slope = 1e6;
    struct Mode { conf c; fl e; int src; fl inter, intra, conf_indep, unbound, lb, ub; };
    std::vector<Mode> v;
    for (int i = 0; i < n; ++i) {
        const float* p = poses + (size_t)i * pose_stride;
        v.push_back(Mode{make_conf(mm, p, p + 3, p + 7), order_e ? (fl)order_e[i] : 0, i, 0, 0, 0, 0, 0, 0});
    }
    if (v.empty()) return 0;
    double intramolecular = 0;
    if (!ad4) {
        std::stable_sort(v.begin(), v.end(), [](const Mode& a, const Mode& b) { return a.e < b.e; });
        mm.set(v[0].c);
        intramolecular = mm.eval_intramolecular(*L->pre, scorer, authentic_v);
    }
    for (auto& x : v) {
        mm.set(x.c);
        const double grids = scorer.eval(mm, authentic_v[1]);
        const double lig_intra = mm.evali(*L->pre, authentic_v);
        x.inter = grids;
        x.intra = lig_intra;
        if (ad4) {
            x.conf_indep = L->sf->conf_independent(mm, 0);
            x.e = grids + x.conf_indep;
            x.unbound = -lig_intra;
        } else {
            const double total = L->sf->conf_independent(mm, grids + lig_intra - intramolecular);
            x.e = total;
            x.conf_indep = total - (grids + lig_intra - intramolecular);
            x.unbound = intramolecular;
        }
    }
    std::stable_sort(v.begin(), v.end(), [](const Mode& a, const Mode& b) { return a.e < b.e; });
    mm.set(v[0].c);
    const model best = mm;
    for (size_t k = 0; k < v.size(); ++k) {
        mm.set(v[k].c);
        float* o = out + 9 * k;
        o[0] = (float)v[k].src;
        o[1] = v[k].e;
        o[2] = mm.rmsd_lower_bound(best);
        o[3] = mm.rmsd_upper_bound(best);
        o[4] = v[k].inter + v[k].intra;
        o[5] = v[k].inter;
        o[6] = v[k].intra;
        o[7] = v[k].conf_indep;
        o[8] = v[k].unbound;
    }
    return (int)v.size();
}

// Clustering of one ligand's chain results as the reference's GPU path does
// it: each chain's best pose through add_to_output_container (coords.cpp:44-68)
// with num_saved_mins = max_modes, then Vina::remove_redundant (vina.cpp:
// 1465-1470).  Writes the chain indices of the modes in their final order and
// returns their count.
int udref_cluster(void* lh, int n_chains, const float* poses, int pose_stride, const float* energies, float min_rmsd,
                  int max_modes, int* out_chain) {
    auto L = (RefLigand*)lh;
    model& m = L->m;
    output_container out;
    for (int k = 0; k < n_chains; ++k) {
        const float* p = poses + (size_t)k * pose_stride;
        conf c = make_conf(m, p, p + 3, p + 7);
        m.set(c);
        output_type t(c, energies[k]);
        t.coords = m.get_heavy_atom_movable_coords();
        t.lb = (fl)k;  // the chain index travels in a field clustering does not read
        add_to_output_container(out, t, min_rmsd, (sz)max_modes);
    }
    output_container tmp;
    VINA_FOR_IN(i, out) add_to_output_container(tmp, out[i], min_rmsd, out.size());
    for (sz i = 0; i < tmp.size(); ++i) out_chain[i] = (int)tmp[i].lb;
    return (int)tmp.size();
}

// Monte-Carlo chains of the CPU search (monte_carlo.cu:2319-2356): chains run on
// `threads` host threads, each chain with its own mt19937 seeded by seed + chain.
// Returns per chain the best energy found (search energy, hunt cap v) and its pose.
int udref_mc(void* lh, void* mh, unsigned seed, int n_chains, int global_steps,
             int local_steps, int threads, float hunt_cap, float* best_e, float* best_pose,
             int pose_stride, long long* evals_out) {
    auto L = (RefLigand*)lh;
    auto M = (RefMaps*)mh;
    if (threads < 1) threads = 1;
    std::atomic<int> next{0};
    std::atomic<long long> evals{0};
    vec corner1 = M->corner1(), corner2 = M->corner2();
    auto worker = [&]() {
        model m = L->m;
        for (;;) {
            int chain = next.fetch_add(1);
            if (chain >= n_chains) break;
            rng generator(static_cast<rng::result_type>(seed + (unsigned)chain));
            int evalcount = 0;
            vec authentic_v(1000, 1000, 1000);
            vec hunt(hunt_cap, hunt_cap, hunt_cap);
            conf_size s = m.get_size();
            change g(s);
            output_type tmp(s, 0);
            tmp.c.randomize(corner1, corner2, generator);
            fl best = max_fl;
            output_type best_out = tmp;
            quasi_newton qn;
            qn.max_steps = (unsigned)local_steps;
            for (int step = 0; step < global_steps; ++step) {
                output_type candidate = tmp;
                mutate_conf(candidate.c, m, 2.0, generator);
                qn(m, *L->pre, *M->ig, candidate, g, hunt, evalcount);
                if (step == 0 || metropolis(tmp.e, candidate.e, 1.2, generator)) {
                    tmp = candidate;
                    m.set(tmp.c);
                    if (tmp.e < best) {
                        qn(m, *L->pre, *M->ig, tmp, g, authentic_v, evalcount);
                        m.set(tmp.c);
                        if (tmp.e < best) {
                            best = tmp.e;
                            best_out = tmp;
                        }
                    }
                }
            }
            best_e[chain] = best;
            read_conf(best_out.c, best_pose + (size_t)chain * pose_stride,
                      best_pose + (size_t)chain * pose_stride + 3,
                      best_pose + (size_t)chain * pose_stride + 7);
            evals += evalcount;
        }
    };
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t) ts.emplace_back(worker);
    for (auto& t : ts) t.join();
    if (evals_out) *evals_out = evals.load();
    return 0;
}

// AutoDock 4.2 maps from AutoGrid .map files <prefix>.<type>.map, .e.map,
// .d.map (ad4cache::read, ad4cache.cpp:391-437), scored with the AD4.2
// scoring function of the given weights.
void* udref_ad4_maps_read(const char* prefix, const float* weights, int n_weights) {
    try {
        auto h = new RefMaps();
        h->sf = std::make_shared<ScoringFunction>(SF_AD42, to_flv(weights, n_weights));
        h->ad4 = ad4cache(1e6);
        h->ad4.read(prefix);
        h->ig = &h->ad4;
        return h;
    } catch (...) {
        g_err = "udref_ad4_maps_read failed";
        return nullptr;
    }
}

namespace {
atom ad4_atom(int ad, float q) {
    atom a;
    a.ad = (sz)ad;
    a.xs = XS_TYPE_SIZE;  // no X-Score type: no glue term
    a.el = EL_TYPE_SIZE;
    a.charge = q;
    return a;
}
}  // namespace

// ScoringFunction(SF_AD42)::eval of two AD-typed atoms at distance r
// (scoring_function.h:113-117): the weighted sum of the AD4.2 terms.
float udref_ad4_pair(int ad1, float q1, int ad2, float q2, float r, const float* weights, int n_weights) {
    ScoringFunction sf(SF_AD42, to_flv(weights, n_weights));
    atom a = ad4_atom(ad1, q1), b = ad4_atom(ad2, q2);
    return sf.eval(a, b, r);
}

// Energy of a probe atom (AD type, charge) at point p against every receptor
// atom within the AD4 cutoff: the sum of the reference's pairwise
// ScoringFunction(SF_AD42)::eval, i.e. the value an AD4 grid map of that probe
// holds at p (type map + q * electrostatic map + |q| * desolvation map).
double udref_ad4_probe(const float* xyz, const int* ad, const float* q, int n, const float* p, int probe_ad,
                       float probe_q, const float* weights, int n_weights) {
    ScoringFunction sf(SF_AD42, to_flv(weights, n_weights));
    atom pr = ad4_atom(probe_ad, probe_q);
    const fl cut2 = sf.get_cutoff() * sf.get_cutoff();
    double acc = 0;
    for (int i = 0; i < n; ++i) {
        vec d(xyz[3 * i] - p[0], xyz[3 * i + 1] - p[1], xyz[3 * i + 2] - p[2]);
        fl r2 = d.norm_sqr();
        if (r2 >= cut2) continue;
        atom b = ad4_atom(ad[i], q[i]);
        acc += sf.eval(pr, b, std::sqrt(r2));
    }
    return acc;
}

}  // extern "C"
