// Ligand and receptor input: PDBQT and SDF parsing, torsion tree, covalent bonds,
// X-Score typing and the intramolecular pair list.
//
// The result has to be the model the reference builds from the same file,
// atom for atom (order, local frames, types, pairs), because poses and
// energies are exchanged in that atom order.  Semantics followed:
//   parsing + tree:  unidock/src/lib/parse_pdbqt.cpp:182-282 (parsing_struct),
//                    :323-456 (ROOT/BRANCH/TORSDOF), :498-542 (postprocess_branch),
//                    :924-960 (branch records), unidock/src/lib/tree.h:116-128 (segment frames)
//   bonds:           unidock/src/lib/model.cpp:288-390 (assign_bonds, atom_exists_between)
//   typing:          unidock/src/lib/model.cpp:408-506 (assign_types)
//   pairs:           unidock/src/lib/model.cpp:508-611 (bonded_to, initialize_pairs)
//   SDF input:       unidock/src/lib/parse_pdbqt.cpp:129-144, 400-420, 612-873, 962-1000
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

#include "ud_model.h"

namespace ud {

namespace {

enum Mob : uint8_t { MOB_VARIABLE = 0, MOB_FIXED = 1, MOB_ROTOR = 2 };

struct ParsedAtom {
    unsigned number = 0;
    int ad = AD_SIZE;
    int xs = XS_SIZE;
    float charge = 0;
    float xyz[3] = {0, 0, 0};
    int context = -1;
};

// One ROOT or BRANCH block: its atoms in file order, each with the branches
// that hang off it; `immobile` is the atom of this block bonded to its parent.
struct Block {
    struct Entry {
        ParsedAtom a;
        std::vector<std::unique_ptr<Block>> children;
    };
    std::vector<Entry> atoms;
    int immobile = -1;
    int axis_begin = -1;  // parent-side atom of the rotatable bond (flat index)
    int axis_end = -1;    // this block's immobile atom (flat index)
    bool essentially_empty() const {
        for (std::size_t i = 0; i < atoms.size(); ++i) {
            if (immobile >= 0 && immobile != (int)i) return false;
            if (!atoms[i].children.empty()) return false;
        }
        return true;
    }
};

std::string trim(const std::string& s) {
    std::size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

bool starts_with(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }

// Fixed-column field [i, j] (1-based, inclusive) of a PDB line.
std::string column(const std::string& s, std::size_t i, std::size_t j, bool required,
                   const char* what) {
    if (j > s.size()) {
        if (required) throw std::runtime_error(std::string("line too short for ") + what + ": " + s);
        if (i > s.size()) return "";
        j = s.size();
    }
    return trim(s.substr(i - 1, j - i + 1));
}

template <class T> T convert(const std::string& s, const std::string& line, const char* what) {
    std::istringstream in(s);
    T v;
    in >> v;
    char c;
    if (in.fail() || (in >> c)) throw std::runtime_error(std::string(what) + " \"" + s + "\" is not valid: " + line);
    return v;
}

ParsedAtom parse_atom_line(const std::string& line) {
    ParsedAtom a;
    a.number = convert<unsigned>(column(line, 7, 11, true, "atom number"), line, "Atom number");
    for (int k = 0; k < 3; ++k)
        a.xyz[k] = convert<float>(column(line, 31 + 8 * k, 38 + 8 * k, true, "coordinate"), line,
                                  "Coordinate");
    std::string q = column(line, 69, 76, false, "charge");
    if (!q.empty()) a.charge = convert<float>(q, line, "Charge");
    std::string name = (line.size() >= 78) ? trim(line.substr(77, 2)) : std::string();
    a.ad = ad_type_from_name(name);
    if (is_non_ad_metal(name)) a.xs = XS_Met_D;
    if (!(a.ad < AD_SIZE || a.xs == XS_Met_D))
        throw std::runtime_error("Atom type " + name + " is not a valid AutoDock type: " + line);
    return a;
}

void two_unsigned(const std::string& line, std::size_t skip, unsigned& a, unsigned& b) {
    std::istringstream in(line.substr(skip));
    int x, y;
    in >> x >> y;
    if (!in || x < 0 || y < 0) throw std::runtime_error("Syntax error: " + line);
    a = (unsigned)x;
    b = (unsigned)y;
}

struct LineReader {
    std::vector<std::string> lines;
    std::size_t pos = 0;
    bool next(std::string& s) {
        if (pos >= lines.size()) return false;
        s = lines[pos++];
        return true;
    }
};

struct Builder {
    Ligand& lig;
    std::vector<std::vector<uint8_t>> mob;  // symmetric mobility matrix
    explicit Builder(Ligand& l) : lig(l) {}

    int add_context(const std::string& s) {
        lig.context.emplace_back(s, -1);
        return (int)lig.context.size() - 1;
    }

    void parse_branch(LineReader& in, Block& b, unsigned from, unsigned to) {
        std::string s;
        while (in.next(s)) {
            add_context(s);
            if (s.empty() || starts_with(s, "WARNING") || starts_with(s, "REMARK")) {
            } else if (starts_with(s, "BRANCH")) {
                branch_record(in, s, b);
            } else if (starts_with(s, "ENDBRANCH")) {
                unsigned f, t;
                two_unsigned(s, 9, f, t);
                if (f != from || t != to) throw std::runtime_error("Inconsistent branch numbers.");
                if (b.immobile < 0)
                    throw std::runtime_error("Atom " + std::to_string(to) + " has not been found in this branch.");
                return;
            } else if (starts_with(s, "ATOM  ") || starts_with(s, "HETATM")) {
                ParsedAtom a = parse_atom_line(s);
                a.context = (int)lig.context.size() - 1;
                if (a.number == to) b.immobile = (int)b.atoms.size();
                b.atoms.push_back(Block::Entry{a, {}});
            } else if (starts_with(s, "MODEL")) {
                throw std::runtime_error("Unexpected multi-MODEL tag in ligand PDBQT.");
            } else {
                throw std::runtime_error("Unknown or inappropriate tag in ligand: " + s);
            }
        }
        throw std::runtime_error("Unterminated BRANCH.");
    }

    void branch_record(LineReader& in, const std::string& s, Block& b) {
        unsigned first, second;
        two_unsigned(s, 6, first, second);
        for (auto& e : b.atoms) {
            if (e.a.number == first) {
                e.children.emplace_back(new Block());
                parse_branch(in, *e.children.back(), first, second);
                return;
            }
        }
        throw std::runtime_error("Atom number " + std::to_string(first) + " is missing in this branch.");
    }

    void grow_mob() {
        std::size_t n = lig.atoms.size();
        for (auto& row : mob) row.resize(n, MOB_VARIABLE);
        while (mob.size() < n) mob.emplace_back(n, MOB_VARIABLE);
    }
    void set_mob(int i, int j, uint8_t v) {
        mob[i][j] = v;
        mob[j][i] = v;
    }

    // Append an atom to the flat list with coordinates relative to `origin`.
    int insert_atom(Block::Entry& e, const float* origin) {
        int idx = (int)lig.atoms.size();
        for (auto& c : e.children) c->axis_begin = idx;
        Atom a;
        for (int k = 0; k < 3; ++k) {
            a.lab[k] = e.a.xyz[k];
            a.local[k] = e.a.xyz[k] - origin[k];
        }
        a.charge = e.a.charge;
        a.ad = e.a.ad;
        a.xs = e.a.xs;
        a.serial = (int)e.a.number;
        lig.atoms.push_back(a);
        if (e.a.context >= 0) lig.context[e.a.context].second = idx;
        return idx;
    }

    void insert_immobiles(Block::Entry& e, const float* origin) {
        for (auto& c : e.children) {
            if (!c->atoms.empty()) {
                c->axis_end = (int)lig.atoms.size();
                insert_atom(c->atoms[c->immobile], origin);
            }
        }
    }

    void postprocess(Block& b, int node) {
        // copy: lig.nodes grows (and may reallocate) while children are added
        const float origin[3] = {lig.nodes[node].origin0[0], lig.nodes[node].origin0[1],
                                 lig.nodes[node].origin0[2]};
        lig.nodes[node].begin = (int)lig.atoms.size();
        for (std::size_t i = 0; i < b.atoms.size(); ++i) {
            if (!(b.immobile >= 0 && (int)i == b.immobile)) insert_atom(b.atoms[i], origin);
            insert_immobiles(b.atoms[i], origin);
        }
        lig.nodes[node].end = (int)lig.atoms.size();
        grow_mob();
        const int nb = lig.nodes[node].begin, ne = lig.nodes[node].end;
        if (b.axis_begin >= 0)
            for (int i = nb; i < ne; ++i) set_mob(b.axis_begin, i, MOB_FIXED);
        if (b.axis_end >= 0)
            for (int i = nb; i < ne; ++i) set_mob(b.axis_end, i, MOB_FIXED);
        if (b.axis_begin >= 0 && b.axis_end >= 0) set_mob(b.axis_begin, b.axis_end, MOB_ROTOR);
        for (int i = nb; i < ne; ++i)
            for (int j = i + 1; j < ne; ++j) set_mob(i, j, MOB_FIXED);
        for (auto& e : b.atoms) {
            for (auto& c : e.children) {
                if (c->essentially_empty()) continue;
                Node nd;
                nd.parent = node;
                const float* imm = c->atoms[c->immobile].a.xyz;
                float d[3];
                for (int k = 0; k < 3; ++k) {
                    nd.origin0[k] = imm[k];
                    d[k] = imm[k] - e.a.xyz[k];
                }
                float nrm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                if (nrm < std::numeric_limits<float>::epsilon())
                    throw std::runtime_error("Ligand with zero-length rotatable bond.");
                for (int k = 0; k < 3; ++k) {
                    nd.rel_axis[k] = (1 / nrm) * d[k];
                    nd.rel_origin[k] = nd.origin0[k] - origin[k];
                }
                lig.nodes.push_back(nd);
                postprocess(*c, (int)lig.nodes.size() - 1);
            }
        }
    }

    uint8_t dist_type(int i, int j) const {
        if (i == j) return MOB_FIXED;
        return mob[i][j];
    }

    static float cov_radius(const Atom& a) {
        if (a.ad < AD_SIZE) return ad_kind(a.ad).covalent_radius;
        if (a.xs == XS_Met_D) return 1.75f;
        return ad_kind(0).covalent_radius;
    }

    static float dist2(const float* a, const float* b) {
        float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        return dx * dx + dy * dy + dz * dz;
    }

    // Covalent bonds between atoms that cannot move relative to each other.
    void assign_bonds() {
        const float allowance = 1.1f;
        const int n = (int)lig.atoms.size();
        const float max_cov = max_covalent_radius();
        // 15 A beads fix the order in which candidate neighbours are visited
        const float bead_r2 = 15.0f * 15.0f;
        std::vector<std::pair<std::array<float, 3>, std::vector<int>>> beads;
        for (int i = 0; i < n; ++i) {
            const float* c = lig.atoms[i].lab;
            bool placed = false;
            for (auto& b : beads)
                if (dist2(c, b.first.data()) < bead_r2) {
                    b.second.push_back(i);
                    placed = true;
                    break;
                }
            if (!placed) beads.push_back({{c[0], c[1], c[2]}, {i}});
        }
        for (int i = 0; i < n; ++i) {
            Atom& ai = lig.atoms[i];
            float icov = (ai.ad < AD_SIZE) ? ad_kind(ai.ad).covalent_radius : max_cov;
            std::vector<int> relevant;
            const float bead_cut = 15.0f + allowance * (icov + max_cov);
            const float bead_cut2 = bead_cut * bead_cut;
            for (auto& b : beads) {
                if (dist2(b.first.data(), ai.lab) > bead_cut2) continue;
                for (int j : b.second) {
                    if (dist_type(i, j) != MOB_VARIABLE && i != j) {
                        float r2 = dist2(ai.lab, lig.atoms[j].lab);
                        float lim = allowance * (icov + max_cov);
                        if (r2 < lim * lim) relevant.push_back(j);
                    }
                }
            }
            for (int j : relevant) {
                if (j <= i) continue;
                Atom& aj = lig.atoms[j];
                float bl = cov_radius(ai) + cov_radius(aj);
                uint8_t dt = dist_type(i, j);
                float r2 = dist2(ai.lab, aj.lab);
                float lim = allowance * bl;
                if (r2 < lim * lim && !atom_between(i, j, relevant)) {
                    bool rot = (dt == MOB_ROTOR);
                    ai.bonds.push_back(j);
                    ai.bond_rot.push_back(rot);
                    aj.bonds.push_back(i);
                    aj.bond_rot.push_back(rot);
                }
            }
        }
    }

    bool atom_between(int a, int b, const std::vector<int>& relevant) const {
        float r2 = dist2(lig.atoms[a].lab, lig.atoms[b].lab);
        for (int c : relevant) {
            if (c == a || c == b) continue;
            if (dist_type(a, c) != MOB_VARIABLE && dist_type(b, c) != MOB_VARIABLE &&
                dist2(lig.atoms[a].lab, lig.atoms[c].lab) < r2 &&
                dist2(lig.atoms[b].lab, lig.atoms[c].lab) < r2)
                return true;
        }
        return false;
    }

    void bonded_to(int a, int depth, std::vector<int>& out) const {
        if (std::find(out.begin(), out.end(), a) != out.end()) return;
        out.push_back(a);
        if (depth > 0)
            for (int b : lig.atoms[a].bonds) bonded_to(b, depth - 1, out);
    }

    bool closure_clash(int i, int j) const {
        int t1 = lig.atoms[i].ad, t2 = lig.atoms[j].ad;
        auto gcg = [&](int cg, int g) { return (t1 == cg && t2 == g) || (t2 == cg && t1 == g); };
        if (gcg(AD_CG0, AD_G0) || gcg(AD_CG1, AD_G1) || gcg(AD_CG2, AD_G2) || gcg(AD_CG3, AD_G3))
            return false;
        std::vector<int> ni, nj;
        bonded_to(i, 1, ni);
        bonded_to(j, 1, nj);
        bool has[4] = {false, false, false, false};
        for (int k : ni) {
            int t = lig.atoms[k].ad;
            if (t >= AD_CG0 && t <= AD_CG3) has[t - AD_CG0] = true;
        }
        for (int k : nj) {
            int t = lig.atoms[k].ad;
            if (t >= AD_CG0 && t <= AD_CG3 && has[t - AD_CG0]) return true;
        }
        return false;
    }

    bool glue_pair(int i, int j) const {
        int t1 = lig.atoms[i].ad, t2 = lig.atoms[j].ad;
        auto gcg = [&](int cg, int g) { return (t1 == cg && t2 == g) || (t2 == cg && t1 == g); };
        return gcg(AD_CG0, AD_G0) || gcg(AD_CG1, AD_G1) || gcg(AD_CG2, AD_G2) || gcg(AD_CG3, AD_G3);
    }

    void make_pairs(bool xs_typing) {
        const int n = (int)lig.atoms.size();
        const int nt = xs_typing ? XS_SIZE : AD_SIZE;
        for (int i = 0; i < n; ++i) {
            std::vector<int> near;
            bonded_to(i, 3, near);
            for (int j = i + 1; j < n; ++j) {
                if (mob[i][j] != MOB_VARIABLE) continue;
                if (std::find(near.begin(), near.end(), j) != near.end()) continue;
                if (closure_clash(i, j)) continue;
                int t1 = xs_typing ? lig.atoms[i].xs : lig.atoms[i].ad;
                int t2 = xs_typing ? lig.atoms[j].xs : lig.atoms[j].ad;
                if (t1 < nt && t2 < nt) {
                    Pair p{i, j, tri_index(t1, t2)};
                    auto& dst = glue_pair(i, j) ? (xs_typing ? lig.glue_pairs : lig.glue_pairs_ad)
                                                : (xs_typing ? lig.pairs : lig.pairs_ad);
                    dst.push_back(p);
                }
            }
        }
    }
};

bool bonded_to_hd(const std::vector<Atom>& atoms, const Atom& a) {
    for (int b : a.bonds)
        if (atoms[b].ad == AD_HD) return true;
    return false;
}

bool is_heteroatom(const Atom& a) {
    bool het = a.ad != AD_A && a.ad != AD_C && a.ad != AD_H && a.ad != AD_HD && a.ad < AD_SIZE;
    return het || a.xs == XS_Met_D;
}

bool bonded_to_heteroatom(const std::vector<Atom>& atoms, const Atom& a) {
    for (int b : a.bonds)
        if (is_heteroatom(atoms[b])) return true;
    return false;
}

// X-Score typing from element, AutoDock type and bonds.
void assign_types(std::vector<Atom>& atoms) {
    for (auto& a : atoms) {
        a.el = ad_to_el(a.ad);
        if (a.ad == AD_SIZE && a.xs == XS_Met_D) a.el = EL_Met;
        const bool acceptor = (a.ad == AD_OA || a.ad == AD_NA);
        const bool donor = (a.el == EL_Met || bonded_to_hd(atoms, a));
        int& x = a.xs;
        switch (a.el) {
            case EL_H: break;
            case EL_C: {
                bool het = bonded_to_heteroatom(atoms, a);
                if (a.ad == AD_CG0) x = het ? XS_C_P_CG0 : XS_C_H_CG0;
                else if (a.ad == AD_CG1) x = het ? XS_C_P_CG1 : XS_C_H_CG1;
                else if (a.ad == AD_CG2) x = het ? XS_C_P_CG2 : XS_C_H_CG2;
                else if (a.ad == AD_CG3) x = het ? XS_C_P_CG3 : XS_C_H_CG3;
                else x = het ? XS_C_P : XS_C_H;
                break;
            }
            case EL_N:
                if (a.ad == AD_NXA) x = XS_N_XA;
                else if (a.ad == AD_NXD) x = XS_N_XD;
                else x = (acceptor && donor) ? XS_N_DA : (acceptor ? XS_N_A : (donor ? XS_N_D : XS_N_P));
                break;
            case EL_O:
                // the reference maps OXA/OXD onto the nitrogen biased types (model.cpp:448-452)
                if (a.ad == AD_OXA) x = XS_N_XA;
                else if (a.ad == AD_OXD) x = XS_N_XD;
                else x = (acceptor && donor) ? XS_O_DA : (acceptor ? XS_O_A : (donor ? XS_O_D : XS_O_P));
                break;
            case EL_S: x = XS_S_P; break;
            case EL_P: x = XS_P_P; break;
            case EL_F: x = XS_F_H; break;
            case EL_Cl: x = XS_Cl_H; break;
            case EL_Br: x = XS_Br_H; break;
            case EL_I: x = XS_I_H; break;
            case EL_Si: x = XS_Si; break;
            case EL_At: x = XS_At; break;
            case EL_Met: x = XS_Met_D; break;
            case EL_Dummy:
                if (a.ad == AD_G0) x = XS_G0;
                else if (a.ad == AD_G1) x = XS_G1;
                else if (a.ad == AD_G2) x = XS_G2;
                else if (a.ad == AD_G3) x = XS_G3;
                else x = XS_SIZE;
                break;
            default: break;
        }
    }
}

// Rigid-body frames, bonds, X-Score types and intramolecular pairs from the
// parsed ROOT block (postprocess_ligand, parse_pdbqt.cpp:525-542, then
// model.cpp:initialize); shared by the PDBQT and SDF front ends.
void finish_ligand(Builder& B, Block& root, int atom_typing_xs) {
    Ligand& lig = B.lig;
    Node r;
    for (int k = 0; k < 3; ++k) r.origin0[k] = root.atoms[0].a.xyz[k];
    lig.nodes.push_back(r);
    B.postprocess(root, 0);
    B.grow_mob();
    for (std::size_t k = 0; k < lig.nodes.size(); ++k)
        for (int i = lig.nodes[k].begin; i < lig.nodes[k].end; ++i) lig.atoms[i].node = (int)k;
    B.assign_bonds();
    assign_types(lig.atoms);
    // both typings: the pair list of a batch follows its maps' scoring function
    B.make_pairs(true);
    B.make_pairs(false);
    if (!atom_typing_xs) {
        lig.pairs = lig.pairs_ad;
        lig.glue_pairs = lig.glue_pairs_ad;
    }
}

// Whitespace-separated unsigned integers of an SDF property line.
std::vector<int> sdf_ints(const std::string& line) {
    std::vector<int> v;
    std::istringstream in(line);
    std::string tok;
    while (in >> tok) {
        for (char c : tok)
            if (!std::isdigit((unsigned char)c)) throw std::runtime_error("Invalid SDF property line: " + line);
        v.push_back(std::stoi(tok));
    }
    return v;
}

}  // namespace

int Ligand::n_heavy() const {
    int k = 0;
    for (auto& a : atoms) k += (a.el != EL_H);
    return k;
}

// conf_independent_inputs(model) of unidock/src/lib/conf_independent.cpp:65-99
std::array<float, 7> Ligand::conf_indep_inputs() const {
    std::array<float, 7> v{};
    auto heavy_neighbours = [&](int i) {
        unsigned k = 0;
        for (int b : atoms[i].bonds)
            if (!(atoms[b].ad == AD_H || atoms[b].ad == AD_HD)) ++k;
        return k;
    };
    float num_tors = 0, num_rotors = 0, heavy = 0, hydrophobic = 0, hb = 0;
    for (std::size_t i = 0; i < atoms.size(); ++i) {
        const Atom& a = atoms[i];
        if (a.el == EL_H) continue;
        unsigned ar = 0;
        for (std::size_t k = 0; k < a.bonds.size(); ++k) {
            const Atom& b = atoms[a.bonds[k]];
            if (a.bond_rot[k] && !(b.ad == AD_H || b.ad == AD_HD) && heavy_neighbours(a.bonds[k]) > 1) ++ar;
        }
        num_tors += 0.5f * ar;
        if (ar > 2) num_rotors += 0.5f;
        else num_rotors += 0.5f * ar;
        if (xs_is_hydrophobic(a.xs)) hydrophobic += 1;
        if (xs_is_acceptor(a.xs) || xs_is_donor(a.xs)) hb += 1;
        heavy += 1;
    }
    v[0] = num_tors;
    v[1] = num_rotors;
    v[2] = heavy;
    v[3] = hydrophobic;
    v[4] = hb;
    v[5] = 1;
    v[6] = 0;
    return v;
}

Ligand parse_ligand_pdbqt(const std::string& text, int atom_typing_xs) {
    Ligand lig;
    LineReader in;
    {
        std::istringstream ss(text);
        std::string s;
        while (std::getline(ss, s)) {
            if (!s.empty() && s.back() == '\r') s.pop_back();
            in.lines.push_back(s);
        }
    }
    Builder B(lig);
    Block root;
    std::string s;
    // header up to ROOT
    bool got_root = false;
    while (in.next(s)) {
        B.add_context(s);
        if (s.empty() || starts_with(s, "WARNING") || starts_with(s, "REMARK")) continue;
        if (starts_with(s, "ROOT")) {
            got_root = true;
            break;
        }
        if (starts_with(s, "MODEL")) throw std::runtime_error("Unexpected multi-MODEL tag in ligand PDBQT.");
        throw std::runtime_error("Unknown or inappropriate tag in ligand: " + s);
    }
    if (got_root) {
        while (in.next(s)) {
            B.add_context(s);
            if (s.empty() || starts_with(s, "WARNING") || starts_with(s, "REMARK")) continue;
            if (starts_with(s, "ATOM  ") || starts_with(s, "HETATM")) {
                ParsedAtom a = parse_atom_line(s);
                a.context = (int)lig.context.size() - 1;
                root.atoms.push_back(Block::Entry{a, {}});
            } else if (starts_with(s, "ENDROOT")) {
                break;
            } else {
                throw std::runtime_error("Unknown or inappropriate tag in ligand: " + s);
            }
        }
    }
    bool have_torsdof = false;
    while (in.next(s)) {
        B.add_context(s);
        if (s.empty() || s[0] == '\0' || starts_with(s, "WARNING") || starts_with(s, "REMARK")) continue;
        if (starts_with(s, "BRANCH")) {
            B.branch_record(in, s, root);
        } else if (starts_with(s, "TORSDOF")) {
            if (have_torsdof) throw std::runtime_error("TORSDOF keyword can be defined only once.");
            std::istringstream t(s.substr(7));
            int v;
            t >> v;
            if (!t || v < 0) throw std::runtime_error("Syntax error: " + s);
            lig.torsdof = v;
            have_torsdof = true;
        } else if (starts_with(s, "MODEL")) {
            throw std::runtime_error("Unexpected multi-MODEL tag in ligand PDBQT.");
        } else {
            throw std::runtime_error("Unknown or inappropriate tag in ligand: " + s);
        }
    }
    if (root.atoms.empty()) throw std::runtime_error("No atoms in this ligand.");
    if (!have_torsdof) throw std::runtime_error("Missing TORSDOF keyword in this ligand.");
    finish_ligand(B, root, atom_typing_xs);
    return lig;
}

bool looks_like_sdf(const std::string& text) {
    // a V2000 molfile: the counts line (4th line) ends in "V2000"
    std::size_t pos = 0;
    for (int k = 0; k < 3; ++k) {
        pos = text.find('\n', pos);
        if (pos == std::string::npos) return false;
        ++pos;
    }
    std::size_t end = text.find('\n', pos);
    std::string counts = text.substr(pos, end == std::string::npos ? std::string::npos : end - pos);
    return counts.find("V2000") != std::string::npos || counts.find("V3000") != std::string::npos;
}

// SDF (V2000) ligand with the torsion tree written by the reference's ligand
// preparation (unidock_tools torsion_tree.py): the property blocks "fragInfo"
// (the SDF atom numbers of each rigid fragment; fragment 0 is the root),
// "torsionInfo" (lines "a b fa fb": rotatable bond a-b with a in fragment fa
// and b in fragment fb) and "atomInfo" (atom number, partial charge in columns
// 4-13, AutoDock type from column 14).  Followed:
//   atom lines       parse_pdbqt.cpp:129-144 (x/y/z in columns 1-30, element at 32-33)
//   property blocks  parse_pdbqt.cpp:612-733 (a block runs to the next empty line;
//                    "$$$$" lines are dropped; every other line is kept as context)
//   tree             parse_pdbqt.cpp:735-859 and :400-420, :962-1000: root = fragment 0
//                    in listed order; for each atom of a fragment in order and each
//                    torsion naming it, the fragment on the other side becomes a branch
//                    of that atom unless already placed; the branch's immobile atom is
//                    the torsion's other atom.
// Without keep_h, atoms of AutoDock type H are left out of every fragment (their
// lines stay in the context with the input coordinates).  Without fragInfo the
// ligand is one rigid body of all atoms and TORSDOF 0.  TORSDOF is the number of
// torsionInfo lines.
Ligand parse_ligand_sdf(const std::string& text, bool keep_h, int atom_typing_xs) {
    Ligand lig;
    lig.sdf = true;
    LineReader in;
    {
        std::istringstream ss(text);
        std::string s;
        while (std::getline(ss, s)) {
            if (!s.empty() && s.back() == '\r') s.pop_back();
            in.lines.push_back(s);
        }
    }
    Builder B(lig);
    std::string s;
    for (int k = 0; k < 3; ++k) {
        if (!in.next(s)) throw std::runtime_error("SDF record ends inside its header.");
        B.add_context(s);
        if (k == 0) lig.name = trim(s);
    }
    if (!in.next(s)) throw std::runtime_error("SDF record has no counts line.");
    B.add_context(s);
    if (s.find("V3000") != std::string::npos) throw std::runtime_error("V3000 molfiles are not supported.");
    const int n_atoms = (int)convert<float>(column(s, 1, 3, true, "atom count"), s, "Atom num");
    const int n_bonds = (int)convert<float>(column(s, 4, 6, true, "bond count"), s, "Bond num");
    if (n_atoms <= 0) throw std::runtime_error("No atoms in this ligand.");
    std::vector<ParsedAtom> atoms(n_atoms);
    for (int i = 0; i < n_atoms; ++i) {
        if (!in.next(s)) throw std::runtime_error("SDF record ends inside its atom block.");
        B.add_context(s);
        ParsedAtom& a = atoms[i];
        for (int k = 0; k < 3; ++k)
            a.xyz[k] = convert<float>(column(s, 1 + 10 * k, 10 + 10 * k, true, "coordinate"), s, "Coordinate");
        if (s.size() < 32) throw std::runtime_error("line too short for the element: " + s);
        std::string name = s.substr(31, 2);
        if (name.size() == 2 && name[1] == ' ') name = name.substr(0, 1);
        a.ad = ad_type_from_name(name);
        a.number = (unsigned)(i + 1);
        a.context = (int)lig.context.size() - 1;
    }
    for (int i = 0; i < n_bonds; ++i) {
        if (!in.next(s)) throw std::runtime_error("SDF record ends inside its bond block.");
        B.add_context(s);
    }
    while (in.next(s)) {
        B.add_context(s);
        if (s.find("M  END") != std::string::npos) break;
    }
    std::vector<std::vector<int>> frags, torsions;
    while (in.next(s)) {
        if (s.find("$$$$") != std::string::npos) continue;
        B.add_context(s);
        if (s.empty() || s[0] != '>') continue;
        const bool atom_info = s.find("atomInfo") != std::string::npos || s.find("atom_info") != std::string::npos;
        const bool torsion = !atom_info && s.find("torsion") != std::string::npos;
        const bool frag = !atom_info && !torsion && s.find("frag") != std::string::npos;
        while (in.next(s)) {
            B.add_context(s);
            if (s.empty()) break;
            if (atom_info) {
                std::size_t sp = s.find(' ');
                std::size_t idlen = std::min<std::size_t>(sp == std::string::npos ? 3 : sp, 3);
                if (idlen == 0 || s.size() < 14) throw std::runtime_error("Invalid atomInfo line: " + s);
                int id = convert<int>(column(s, 1, idlen, true, "atom id"), s, "AtomId");
                float q = convert<float>(column(s, 4, 13, true, "partial charge"), s, "Partial Charge");
                if (id < 1 || id > n_atoms) throw std::runtime_error("atomInfo names a missing atom: " + s);
                atoms[id - 1].charge = q;
                atoms[id - 1].ad = ad_type_from_name(trim(s.substr(13)));
            } else if (torsion) {
                std::vector<int> t = sdf_ints(s);
                if (t.size() < 4) throw std::runtime_error("Invalid torsionInfo line: " + s);
                torsions.push_back(t);
            } else if (frag) {
                frags.push_back(sdf_ints(s));
            }
        }
    }
    for (auto& a : atoms)
        if (a.ad >= AD_SIZE)
            throw std::runtime_error("SDF atom " + std::to_string(a.number) + " has no valid AutoDock type.");
    for (auto& f : frags)
        for (int id : f)
            if (id < 1 || id > n_atoms) throw std::runtime_error("fragInfo names a missing atom.");
    for (auto& t : torsions)
        if (t[2] < 0 || t[3] < 0 || (frags.size() && (t[2] >= (int)frags.size() || t[3] >= (int)frags.size())))
            throw std::runtime_error("torsionInfo names a missing fragment.");
    lig.torsdof = (int)torsions.size();
    if (!keep_h)
        for (auto& f : frags)
            f.erase(std::remove_if(f.begin(), f.end(), [&](int id) { return atoms[id - 1].ad == AD_H; }), f.end());

    Block root;
    if (frags.empty()) {
        lig.torsdof = 0;
        for (auto& a : atoms) root.atoms.push_back(Block::Entry{a, {}});
    } else {
        std::vector<char> placed(frags.size(), 0);
        placed[0] = 1;
        // fill block `b` with fragment f (immobile atom `to`, 0 for the root) and its branches
        std::function<void(Block&, int, int)> fill = [&](Block& b, int f, int to) {
            for (int id : frags[f]) {
                if (id == to) b.immobile = (int)b.atoms.size();
                b.atoms.push_back(Block::Entry{atoms[id - 1], {}});
            }
            for (int id : frags[f]) {
                for (const auto& t : torsions) {
                    int from, next_to, nf;
                    if (t[0] == id) {
                        from = t[0], next_to = t[1], nf = t[3];
                    } else if (t[1] == id) {
                        from = t[1], next_to = t[0], nf = t[2];
                    } else {
                        continue;
                    }
                    if (placed[nf]) continue;
                    for (auto& e : b.atoms) {
                        if ((int)e.a.number != from) continue;
                        placed[nf] = 1;
                        e.children.emplace_back(new Block());
                        fill(*e.children.back(), nf, next_to);
                        break;
                    }
                }
            }
            if (to > 0 && b.immobile < 0)
                throw std::runtime_error("Atom " + std::to_string(to) + " has not been found in this branch.");
        };
        fill(root, 0, 0);
    }
    if (root.atoms.empty()) throw std::runtime_error("No atoms in this ligand.");
    finish_ligand(B, root, atom_typing_xs);
    return lig;
}

Ligand parse_ligand(const std::string& text, bool keep_h, int atom_typing_xs) {
    return looks_like_sdf(text) ? parse_ligand_sdf(text, keep_h, atom_typing_xs)
                                : parse_ligand_pdbqt(text, atom_typing_xs);
}

// Rigid receptor: atoms in file order, bonds from distances (all receptor
// atoms are mutually fixed) and X-Score types (model.cpp:288-506).
Receptor parse_receptor_pdbqt(const std::string& text) {
    Receptor R;
    std::istringstream ss(text);
    std::string s;
    std::vector<Atom> atoms;
    while (std::getline(ss, s)) {
        if (!s.empty() && s.back() == '\r') s.pop_back();
        if (s.empty() || starts_with(s, "TER") || starts_with(s, "END") || starts_with(s, "WARNING") ||
            starts_with(s, "REMARK"))
            continue;
        if (starts_with(s, "ATOM  ") || starts_with(s, "HETATM")) {
            ParsedAtom p = parse_atom_line(s);
            Atom a;
            for (int k = 0; k < 3; ++k) a.lab[k] = p.xyz[k];
            a.ad = p.ad;
            a.xs = p.xs;
            a.charge = p.charge;
            atoms.push_back(a);
        } else if (starts_with(s, "MODEL")) {
            throw std::runtime_error("Unexpected multi-MODEL tag in rigid receptor.");
        } else {
            throw std::runtime_error("Unknown or inappropriate tag in rigid receptor: " + s);
        }
    }
    // bonds through a 3 A cell list; only the bond set matters for typing
    const float allowance = 1.1f;
    const float max_cov = max_covalent_radius();
    const int n = (int)atoms.size();
    const float cell = 4.0f;  // >= 1.1 * (2 * max covalent radius)
    std::unordered_map<long long, std::vector<int>> cells;
    auto key = [&](const float* p, int dx, int dy, int dz) {
        long long x = (long long)std::floor(p[0] / cell) + dx, y = (long long)std::floor(p[1] / cell) + dy,
                  z = (long long)std::floor(p[2] / cell) + dz;
        return (x * 1000003LL + y) * 1000033LL + z;
    };
    for (int i = 0; i < n; ++i) cells[key(atoms[i].lab, 0, 0, 0)].push_back(i);
    auto d2 = [](const float* a, const float* b) {
        float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        return dx * dx + dy * dy + dz * dz;
    };
    auto cov = [&](const Atom& a) {
        if (a.ad < AD_SIZE) return ad_kind(a.ad).covalent_radius;
        if (a.xs == XS_Met_D) return 1.75f;
        return ad_kind(0).covalent_radius;
    };
    for (int i = 0; i < n; ++i) {
        Atom& ai = atoms[i];
        float icov = (ai.ad < AD_SIZE) ? ad_kind(ai.ad).covalent_radius : max_cov;
        float lim = allowance * (icov + max_cov);
        std::vector<int> relevant;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = cells.find(key(ai.lab, dx, dy, dz));
                    if (it == cells.end()) continue;
                    for (int j : it->second)
                        if (j != i && d2(ai.lab, atoms[j].lab) < lim * lim) relevant.push_back(j);
                }
        std::sort(relevant.begin(), relevant.end());
        for (int j : relevant) {
            if (j <= i) continue;
            float bl = cov(ai) + cov(atoms[j]);
            float r2 = d2(ai.lab, atoms[j].lab);
            float blim = allowance * bl;
            if (!(r2 < blim * blim)) continue;
            bool between = false;
            for (int c : relevant) {
                if (c == i || c == j) continue;
                if (d2(ai.lab, atoms[c].lab) < r2 && d2(atoms[j].lab, atoms[c].lab) < r2) {
                    between = true;
                    break;
                }
            }
            if (!between) {
                ai.bonds.push_back(j);
                ai.bond_rot.push_back(0);
                atoms[j].bonds.push_back(i);
                atoms[j].bond_rot.push_back(0);
            }
        }
    }
    assign_types(atoms);
    for (auto& a : atoms) {
        R.xyz.push_back({a.lab[0], a.lab[1], a.lab[2]});
        R.ad.push_back(a.ad);
        R.el.push_back(a.el);
        R.xs.push_back(a.xs);
        R.charge.push_back(a.charge);
    }
    return R;
}

// Host forward kinematics (tree.h:89-93,116-128; quaternion.cpp:116-132).
void ligand_coords(const Ligand& lig, const float* pose, float* xyz) {
    const int R = (int)lig.nodes.size();
    std::vector<float> org(3 * R), q(4 * R), rot(9 * R);
    auto q2r = [](const float* qq, float* m) {
        float a = qq[0], b = qq[1], c = qq[2], d = qq[3];
        float aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d,
              cc = c * c, cd = c * d, dd = d * d;
        // row-major m[3*i+j] = R(i,j)
        m[0] = aa + bb - cc - dd; m[1] = 2 * (-ad + bc); m[2] = 2 * (ac + bd);
        m[3] = 2 * (ad + bc); m[4] = aa - bb + cc - dd; m[5] = 2 * (-ab + cd);
        m[6] = 2 * (-ac + bd); m[7] = 2 * (ab + cd); m[8] = aa - bb - cc + dd;
    };
    for (int k = 0; k < 3; ++k) org[k] = pose[k];
    for (int k = 0; k < 4; ++k) q[k] = pose[3 + k];
    q2r(&q[0], &rot[0]);
    const float pi = 3.1415926535897931f;
    for (int n = 1; n < R; ++n) {
        const Node& nd = lig.nodes[n];
        int p = nd.parent;
        const float* pr = &rot[9 * p];
        float ax[3];
        for (int i = 0; i < 3; ++i) {
            org[3 * n + i] = org[3 * p + i] + (pr[3 * i] * nd.rel_origin[0] + pr[3 * i + 1] * nd.rel_origin[1] +
                                               pr[3 * i + 2] * nd.rel_origin[2]);
            ax[i] = pr[3 * i] * nd.rel_axis[0] + pr[3 * i + 1] * nd.rel_axis[1] + pr[3 * i + 2] * nd.rel_axis[2];
        }
        float ang = pose[7 + n - 1];
        // normalize_angle
        for (int it = 0; it < 8 && (ang > pi || ang < -pi); ++it) ang += (ang > pi) ? -2 * pi : 2 * pi;
        float c = std::cos(ang / 2), s = std::sin(ang / 2);
        float t[4] = {c, s * ax[0], s * ax[1], s * ax[2]};
        const float* pq = &q[4 * p];
        float r4[4] = {t[0] * pq[0] - t[1] * pq[1] - t[2] * pq[2] - t[3] * pq[3],
                       t[0] * pq[1] + t[1] * pq[0] + t[2] * pq[3] - t[3] * pq[2],
                       t[0] * pq[2] - t[1] * pq[3] + t[2] * pq[0] + t[3] * pq[1],
                       t[0] * pq[3] + t[1] * pq[2] - t[2] * pq[1] + t[3] * pq[0]};
        float s2 = r4[0] * r4[0] + r4[1] * r4[1] + r4[2] * r4[2] + r4[3] * r4[3];
        if (std::abs(s2 - 1) >= 1e-6f) {
            float a = std::sqrt(s2);
            for (int k = 0; k < 4; ++k) r4[k] *= 1 / a;
        }
        for (int k = 0; k < 4; ++k) q[4 * n + k] = r4[k];
        q2r(&q[4 * n], &rot[9 * n]);
    }
    for (std::size_t i = 0; i < lig.atoms.size(); ++i) {
        int n = lig.atoms[i].node;
        const float* m = &rot[9 * n];
        const float* l = lig.atoms[i].local;
        for (int k = 0; k < 3; ++k)
            xyz[3 * i + k] = org[3 * n + k] + (m[3 * k] * l[0] + m[3 * k + 1] * l[1] + m[3 * k + 2] * l[2]);
    }
}

}  // namespace ud
