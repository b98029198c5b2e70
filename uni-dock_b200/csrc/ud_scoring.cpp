// Atom-type constants, scoring-function terms and their r^2 tables.
//
// The parameter tables (AutoDock 4 atom kinds, X-Score radii) and the term
// formulas must be the same numbers as the reference's for results to agree;
// they follow unidock/src/lib/atom_constants.h:143-470 and
// unidock/src/lib/potentials.h:27-509.  Arithmetic is FP32 with the same
// operation order as the reference so that the tables match bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "ud_model.h"

namespace ud {

static const AdKind kAdKinds[AD_SIZE] = {
    {"C", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00143f, 33.51030f, 0.77f},
    {"A", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00052f, 33.51030f, 0.77f},
    {"N", 1.75000f, 0.16000f, 0.0f, 0.0f, -0.00162f, 22.44930f, 0.75f},
    {"O", 1.60000f, 0.20000f, 0.0f, 0.0f, -0.00251f, 17.15730f, 0.73f},
    {"P", 2.10000f, 0.20000f, 0.0f, 0.0f, -0.00110f, 38.79240f, 1.06f},
    {"S", 2.00000f, 0.20000f, 0.0f, 0.0f, -0.00214f, 33.51030f, 1.02f},
    {"H", 1.00000f, 0.02000f, 0.0f, 0.0f, 0.00051f, 0.00000f, 0.37f},
    {"F", 1.54500f, 0.08000f, 0.0f, 0.0f, -0.00110f, 15.44800f, 0.71f},
    {"I", 2.36000f, 0.55000f, 0.0f, 0.0f, -0.00110f, 55.05850f, 1.33f},
    {"NA", 1.75000f, 0.16000f, -5.0f, 1.9f, -0.00162f, 22.44930f, 0.75f},
    {"OA", 1.60000f, 0.20000f, -5.0f, 1.9f, -0.00251f, 17.15730f, 0.73f},
    {"SA", 2.00000f, 0.20000f, -1.0f, 2.5f, -0.00214f, 33.51030f, 1.02f},
    {"HD", 1.00000f, 0.02000f, 1.0f, 0.0f, 0.00051f, 0.00000f, 0.37f},
    {"Mg", 0.65000f, 0.87500f, 0.0f, 0.0f, -0.00110f, 1.56000f, 1.30f},
    {"Mn", 0.65000f, 0.87500f, 0.0f, 0.0f, -0.00110f, 2.14000f, 1.39f},
    {"Zn", 0.74000f, 0.55000f, 0.0f, 0.0f, -0.00110f, 1.70000f, 1.31f},
    {"Ca", 0.99000f, 0.55000f, 0.0f, 0.0f, -0.00110f, 2.77000f, 1.74f},
    {"Fe", 0.65000f, 0.01000f, 0.0f, 0.0f, -0.00110f, 1.84000f, 1.25f},
    {"Cl", 2.04500f, 0.27600f, 0.0f, 0.0f, -0.00110f, 35.82350f, 0.99f},
    {"Br", 2.16500f, 0.38900f, 0.0f, 0.0f, -0.00110f, 42.56610f, 1.14f},
    {"Si", 2.30000f, 0.20000f, 0.0f, 0.0f, -0.00143f, 50.96500f, 1.11f},
    {"At", 2.40000f, 0.55000f, 0.0f, 0.0f, -0.00110f, 57.90580f, 1.44f},
    {"G0", 0.00000f, 0.00000f, 0.0f, 0.0f, 0.00000f, 0.00000f, 0.77f},
    {"G1", 0.00000f, 0.00000f, 0.0f, 0.0f, 0.00000f, 0.00000f, 0.77f},
    {"G2", 0.00000f, 0.00000f, 0.0f, 0.0f, 0.00000f, 0.00000f, 0.77f},
    {"G3", 0.00000f, 0.00000f, 0.0f, 0.0f, 0.00000f, 0.00000f, 0.77f},
    {"CG0", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00143f, 33.51030f, 0.77f},
    {"CG1", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00143f, 33.51030f, 0.77f},
    {"CG2", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00143f, 33.51030f, 0.77f},
    {"CG3", 2.00000f, 0.15000f, 0.0f, 0.0f, -0.00143f, 33.51030f, 0.77f},
    {"W", 0.00000f, 0.00000f, 0.0f, 0.0f, 0.00000f, 0.00000f, 0.00f},
    {"OXA", 1.60000f, 0.20000f, 0.0f, 0.0f, -0.00251f, 17.15730f, 0.73f},
    {"NXA", 1.75000f, 0.16000f, 0.0f, 0.0f, -0.00162f, 22.44930f, 0.75f},
    {"OXD", 1.60000f, 0.20000f, 0.0f, 0.0f, -0.00251f, 17.15730f, 0.73f},
    {"NXD", 1.75000f, 0.16000f, 0.0f, 0.0f, -0.00162f, 22.44930f, 0.75f},
};

static const float kXsRadius[XS_SIZE] = {1.9f, 1.9f, 1.8f, 1.8f, 1.8f, 1.8f, 1.7f, 1.7f, 1.7f,
                                         1.7f, 2.0f, 2.1f, 1.5f, 1.8f, 2.0f, 2.2f, 2.2f, 2.3f,
                                         1.2f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f,
                                         0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.7f, 1.8f, 1.7f, 1.8f};
static const float kXsVinardoRadius[XS_SIZE] = {
    2.0f, 2.0f, 1.7f, 1.7f, 1.7f, 1.7f, 1.6f, 1.6f, 1.6f, 1.6f, 2.0f, 2.1f,
    1.5f, 1.8f, 2.0f, 2.2f, 2.2f, 2.3f, 1.2f, 2.0f, 2.0f, 2.0f, 2.0f, 2.0f,
    2.0f, 2.0f, 2.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.6f, 1.7f, 1.6f, 1.7f};

static const char* kXsNames[XS_SIZE] = {
    "C_H", "C_P", "N_P", "N_D", "N_A", "N_DA", "O_P", "O_D", "O_A", "O_DA", "S_P", "P_P",
    "F_H", "Cl_H", "Br_H", "I_H", "Si", "At", "Met_D", "C_H_CG0", "C_P_CG0", "G0", "C_H_CG1",
    "C_P_CG1", "G1", "C_H_CG2", "C_P_CG2", "G2", "C_H_CG3", "C_P_CG3", "G3", "W", "O_XA",
    "N_XA", "O_XD", "N_XD"};

const AdKind& ad_kind(int ad) { return kAdKinds[ad]; }

int ad_type_from_name(const std::string& name) {
    for (int i = 0; i < AD_SIZE; ++i)
        if (name == kAdKinds[i].name) return i;
    if (name == "Se") return AD_S;
    if (name == "CL") return AD_Cl;
    return AD_SIZE;
}

bool is_non_ad_metal(const std::string& name) {
    static const char* names[] = {"Cu", "Fe", "Na", "K", "Hg", "Co", "U", "Cd", "Ni"};
    for (auto n : names)
        if (name == n) return true;
    return false;
}

int ad_to_el(int t) {
    switch (t) {
        case AD_C: case AD_A: case AD_CG0: case AD_CG1: case AD_CG2: case AD_CG3: return EL_C;
        case AD_N: case AD_NA: case AD_NXA: case AD_NXD: return EL_N;
        case AD_O: case AD_OA: case AD_OXA: case AD_OXD: return EL_O;
        case AD_P: return EL_P;
        case AD_S: case AD_SA: return EL_S;
        case AD_H: case AD_HD: return EL_H;
        case AD_F: return EL_F;
        case AD_I: return EL_I;
        case AD_Mg: case AD_Mn: case AD_Zn: case AD_Ca: case AD_Fe: return EL_Met;
        case AD_Cl: return EL_Cl;
        case AD_Br: return EL_Br;
        case AD_Si: return EL_Si;
        case AD_At: return EL_At;
        case AD_G0: case AD_G1: case AD_G2: case AD_G3: case AD_W: return EL_Dummy;
        default: return EL_SIZE;
    }
}

float xs_radius(int xs) { return kXsRadius[xs]; }
float xs_vinardo_radius(int xs) { return kXsVinardoRadius[xs]; }
const char* xs_name(int xs) { return (xs >= 0 && xs < XS_SIZE) ? kXsNames[xs] : "?"; }
int xs_from_name(const std::string& s) {
    for (int i = 0; i < XS_SIZE; ++i)
        if (s == kXsNames[i]) return i;
    return -1;
}

bool xs_is_hydrophobic(int xs) {
    return xs == XS_C_H || xs == XS_F_H || xs == XS_Cl_H || xs == XS_Br_H || xs == XS_I_H;
}
bool xs_is_acceptor(int xs) {
    return xs == XS_N_A || xs == XS_N_DA || xs == XS_O_A || xs == XS_O_DA || xs == XS_O_XA ||
           xs == XS_N_XA;
}
bool xs_is_donor(int xs) {
    return xs == XS_N_D || xs == XS_N_DA || xs == XS_O_D || xs == XS_O_DA || xs == XS_Met_D ||
           xs == XS_N_XD || xs == XS_O_XD;
}
bool xs_h_bond_possible(int a, int b) {
    return (xs_is_donor(a) && xs_is_acceptor(b)) || (xs_is_donor(b) && xs_is_acceptor(a));
}

float max_covalent_radius() {
    float m = 0;
    for (int i = 0; i < AD_SIZE; ++i) m = std::max(m, kAdKinds[i].covalent_radius);
    return m;
}

int xs_grid_type(int t) {
    switch (t) {
        case XS_G0: case XS_G1: case XS_G2: case XS_G3: return -1;
        case XS_C_H_CG0: case XS_C_H_CG1: case XS_C_H_CG2: case XS_C_H_CG3: return XS_C_H;
        case XS_C_P_CG0: case XS_C_P_CG1: case XS_C_P_CG2: case XS_C_P_CG3: return XS_C_P;
        default: return (t >= 0 && t < XS_SIZE) ? t : -1;
    }
}

// ------------------------------------------------------------------ terms
static inline bool is_glue(int t) { return t == XS_G0 || t == XS_G1 || t == XS_G2 || t == XS_G3; }

static inline bool is_glued(int a, int b) {
    auto g = [](int g, int ch, int cp, int x, int y) {
        return (x == g && (y == ch || y == cp)) || (y == g && (x == ch || x == cp));
    };
    return g(XS_G0, XS_C_H_CG0, XS_C_P_CG0, a, b) || g(XS_G1, XS_C_H_CG1, XS_C_P_CG1, a, b) ||
           g(XS_G2, XS_C_H_CG2, XS_C_P_CG2, a, b) || g(XS_G3, XS_C_H_CG3, XS_C_P_CG3, a, b);
}

static inline float slope_step(float x_bad, float x_good, float x) {
    if (x_bad < x_good) {
        if (x <= x_bad) return 0;
        if (x >= x_good) return 1;
    } else {
        if (x >= x_bad) return 0;
        if (x <= x_good) return 1;
    }
    return (x - x_bad) / (x_good - x_bad);
}

static inline float opt_dist(int a, int b, bool vinardo) {
    if (is_glue(a) || is_glue(b)) return 0.0f;
    return vinardo ? xs_vinardo_radius(a) + xs_vinardo_radius(b) : xs_radius(a) + xs_radius(b);
}

static inline float gauss(float x, float width) { return std::exp(-((x / width) * (x / width))); }

static inline bool xs_biased(int t) {
    return t == XS_O_XA || t == XS_N_XA || t == XS_O_XD || t == XS_N_XD;
}

// Term k of the type form at distance r.  Vina: gauss(0,0.5), gauss(3,2),
// repulsion(0), hydrophobic(0.5,1.5), h-bond(-0.7,0), glue.  Vinardo:
// gauss(0,0.8), repulsion(0), hydrophobic(0,2.5), h-bond(-0.6,0), glue.
float Scoring::term_types(int k, int t1, int t2, float r) const {
    const bool vinardo = (choice == SF_VINARDO);
    if (choice == SF_AD42) return 0.0f;  // AD4 terms depend on charges: per-atom form only
    int kind;  // 0 gauss1 1 gauss2 2 repulsion 3 hydrophobic 4 hbond 5 glue
    if (!vinardo) kind = k;
    else kind = (k == 0) ? 0 : k + 1;
    const float cutoff = (kind == 5) ? 20.0f : 8.0f;
    if (r >= cutoff) return 0.0f;
    switch (kind) {
        case 0: {
            float offset = 0.0f, width = vinardo ? 0.8f : 0.5f;
            return gauss(r - (opt_dist(t1, t2, vinardo) + offset), width);
        }
        case 1: return gauss(r - (opt_dist(t1, t2, false) + 3.0f), 2.0f);
        case 2: {
            float d = r - (opt_dist(t1, t2, vinardo) + 0.0f);
            if (d > 0.0f) return 0.0f;
            return d * d;
        }
        case 3: {
            if (xs_is_hydrophobic(t1) && xs_is_hydrophobic(t2)) {
                float good = vinardo ? 0.0f : 0.5f, bad = vinardo ? 2.5f : 1.5f;
                return slope_step(bad, good, r - opt_dist(t1, t2, vinardo));
            }
            return 0.0f;
        }
        case 4: {
            if (!xs_h_bond_possible(t1, t2)) return 0.0f;
            float good = vinardo ? -0.6f : -0.7f, bad = 0.0f;
            float s = slope_step(bad, good, r - opt_dist(t1, t2, vinardo));
            if (!vinardo && (xs_biased(t1) || xs_biased(t2))) return (float)(10.0 * (double)s);
            return s;
        }
        case 5: return is_glued(t1, t2) ? r : 0.0f;
    }
    return 0.0f;
}

// ---------------------------------------------------------------- AutoDock 4.2
// potentials.h:346-486.  The reference computes in float (fl) with double
// literals promoting some subexpressions; the same promotions are kept.
static float int_pow_f(float x, int n) {
    float p = 1.0f;
    for (int i = 0; i < n; ++i) p = p * x;
    return p;
}

static float ad4_smoothen(float r, float rij, float smoothing) {  // potentials.h:66-77
    smoothing *= 0.5f;
    if (r > rij + smoothing) return r - smoothing;
    if (r < rij - smoothing) return r + smoothing;
    return rij;
}

float ad4_vdw(int t1, int t2, float r) {
    const float cap = 100000.0f, smoothing = 0.5f;
    if (r >= kAd4ShortCutoff) return 0.0f;
    const AdKind &a = ad_kind(t1), &b = ad_kind(t2);
    const float hb_depth = a.hb_depth * b.hb_depth;
    const float vdw_rij = a.radius + b.radius;
    const float vdw_depth = std::sqrt(a.depth * b.depth);
    if (hb_depth < 0) return 0.0f;  // an H-bond pair, not vdW
    r = ad4_smoothen(r, vdw_rij, smoothing);
    const float c_12 = int_pow_f(vdw_rij, 12) * vdw_depth;
    const float c_6 = (float)((double)(int_pow_f(vdw_rij, 6) * vdw_depth) * 2.0);
    const float r6 = int_pow_f(r, 6), r12 = int_pow_f(r, 12);
    const float eps = std::numeric_limits<float>::epsilon();
    if (r12 > eps && r6 > eps) return std::min(cap, c_12 / r12 - c_6 / r6);
    return cap;
}

float ad4_hb(int t1, int t2, float r) {
    const float cap = 100000.0f, smoothing = 0.5f;
    if (r >= kAd4ShortCutoff) return 0.0f;
    const AdKind &a = ad_kind(t1), &b = ad_kind(t2);
    const float hb_rij = a.hb_radius + b.hb_radius;
    const float hb_depth = a.hb_depth * b.hb_depth;
    if (hb_depth >= 0) return 0.0f;  // a vdW pair, not H-bond
    r = ad4_smoothen(r, hb_rij, smoothing);
    const float c_12 = (float)((double)(int_pow_f(hb_rij, 12) * -hb_depth * 10) / 2.0);
    const float c_10 = (float)((double)(int_pow_f(hb_rij, 10) * -hb_depth * 12) / 2.0);
    const float r10 = int_pow_f(r, 10), r12 = int_pow_f(r, 12);
    const float eps = std::numeric_limits<float>::epsilon();
    if (r12 > eps && r10 > eps) return std::min(cap, c_12 / r12 - c_10 / r10);
    return cap;
}

float ad4_elec_unit(float r) {
    const float cap = 100.0f;
    if (r >= kAd4LongCutoff) return 0.0f;
    const float q1q2 = (float)(1.0 * 332.0);
    const float B = (float)(78.4 + 8.5525);
    const float lB = (float)(-(double)B * 0.003627);
    const float diel = (float)(-8.5525 + ((double)B / (1 + 7.7839 * (double)std::exp(lB * r))));
    if (r < std::numeric_limits<float>::epsilon()) return q1q2 * cap / diel;
    return q1q2 * std::min(cap, 1.0f / (r * diel));
}

float ad4_desolv_gauss(float r) {
    const float sigma = 3.6f;
    if (r >= kAd4LongCutoff) return 0.0f;
    const float x = r / sigma;
    return (float)std::exp(-0.5 * (double)(x * x));
}

float ad4_solvation(int ad) { return ad < AD_SIZE ? ad_kind(ad).solvation : -0.00110f; }
float ad4_volume(int ad) { return ad < AD_SIZE ? ad_kind(ad).volume : 0.0f; }

// AD4 row `row` (kAd4Rows layout) at r for term k (< 0: weighted sum of all).
static float ad4_row_value(const Scoring& sf, int row, int k, float r) {
    auto w = [&](int t) { return k < 0 ? sf.weights[t] : (k == t ? 1.0f : 0.0f); };
    if (row == kAd4RowElec) return w(2) * ad4_elec_unit(r);
    if (row == kAd4RowDesolv) return w(3) * (float)((double)kAd4Qsolv * ad4_desolv_gauss(r));
    int t1 = 0, t2 = 0;  // invert tri_index
    while ((t2 + 1) * (t2 + 2) / 2 <= row) ++t2;
    t1 = row - t2 * (t2 + 1) / 2;
    float acc = 0.0f;
    acc += w(0) * ad4_vdw(t1, t2, r);
    acc += w(1) * ad4_hb(t1, t2, r);
    const float s1 = ad4_solvation(t1), s2 = ad4_solvation(t2), v1 = ad4_volume(t1), v2 = ad4_volume(t2);
    acc += w(3) * ((s1 * v2 + s2 * v1) * ad4_desolv_gauss(r));
    const bool glued = (t1 == AD_G0 && t2 == AD_CG0) || (t1 == AD_G1 && t2 == AD_CG1) ||
                       (t1 == AD_G2 && t2 == AD_CG2) || (t1 == AD_G3 && t2 == AD_CG3) ||
                       (t2 == AD_G0 && t1 == AD_CG0) || (t2 == AD_G1 && t1 == AD_CG1) ||
                       (t2 == AD_G2 && t1 == AD_CG2) || (t2 == AD_G3 && t1 == AD_CG3);
    if (glued && r < 20.0f) acc += w(4) * r;
    return acc;
}

float Scoring::eval_types(int t1, int t2, float r) const {
    float acc = 0;
    for (int k = 0; k < n_terms; ++k) acc += weights[k] * term_types(k, t1, t2, r);
    return acc;
}

std::vector<float> Scoring::default_weights(int choice) {
    // unidock/src/main/main.cpp:373-395 defaults; the rotatable weight is stored
    // in the transformed form 5*w/0.1-1 (vina.cpp:392-412) for Vina/Vinardo.
    if (choice == SF_VINA)
        return {-0.035579f, -0.005156f, 0.840245f, -0.035069f, -0.587439f, 50.0f,
                (float)(5 * 0.05846 / 0.1 - 1)};
    if (choice == SF_VINARDO)
        return {-0.045f, 0.8f, -0.035f, -0.6f, 50.0f, (float)(5 * 0.05846 / 0.1 - 1)};
    return {0.1662f, 0.1209f, 0.1406f, 0.1322f, 50.0f, 0.2983f};
}

Scoring Scoring::make(int choice, const float* w, int nw) {
    Scoring s;
    s.choice = choice;
    s.weights = (w && nw > 0) ? std::vector<float>(w, w + nw) : default_weights(choice);
    s.n_terms = (choice == SF_VINA) ? 6 : 5;
    if ((int)s.weights.size() != s.n_terms + 1)
        throw std::runtime_error("wrong number of scoring weights");
    if (choice == SF_AD42) {
        s.cutoff = 20.48f;
        s.max_cutoff = 20.48f;
    }
    return s;
}

// conf_independent.cpp:153-156 (num_tors_div) and :184-187 (ad4_tors_add)
float Scoring::conf_independent(float e, float num_tors, float torsdof) const {
    float w = weights[n_terms];
    if (choice == SF_AD42) return e + w * torsdof;
    float weight = (float)(0.1 * (double)(w + 1));
    float y = (float)(1.0 + (double)(weight * num_tors) / 5.0);
    if (std::abs(e) < std::numeric_limits<float>::epsilon()) return 0;
    if (std::abs(y) < std::numeric_limits<float>::epsilon())
        return (e * y > 0) ? std::numeric_limits<float>::max() : -std::numeric_limits<float>::max();
    return e / y;
}

// ------------------------------------------------------------------ tables
// Row construction of precalculate_element::init_from_smooth_fst
// (unidock/src/lib/precalculate.h:66-85).
void table_row_from_energies(const float* e, const float* rs, int n, float* fast, float* smooth) {
    for (int i = 0; i < n; ++i) smooth[2 * i] = e[i];
    for (int i = 0; i < n; ++i) {
        float dor;
        if (i == 0 || i == n - 1) {
            dor = 0;
        } else {
            float delta = rs[i + 1] - rs[i - 1];
            float r = rs[i];
            dor = (smooth[2 * (i + 1)] - smooth[2 * (i - 1)]) / (delta * r);
        }
        smooth[2 * i + 1] = dor;
        float f1 = smooth[2 * i];
        float f2 = (i + 1 >= n) ? 0 : smooth[2 * (i + 1)];
        fast[i] = (f2 + f1) / 2;
    }
}

void PairTable::build(const Scoring& sf, int term) {
    factor = 32.0f;
    const float cut2 = sf.max_cutoff * sf.max_cutoff;
    n = (int)(std::size_t)(factor * cut2) + 3;
    if (sf.choice == SF_AD42) {  // AD type pairs + the two per-pair scaled rows
        n_types = AD_SIZE;
        const int rows = kAd4Rows;
        fast.assign((std::size_t)rows * n, 0.0f);
        smooth.assign((std::size_t)rows * n * 2, 0.0f);
        std::vector<float> rs(n), e(n);
        for (int i = 0; i < n; ++i) rs[i] = std::sqrt((float)i / factor);
        for (int row = 0; row < rows; ++row) {
            for (int i = 0; i < n; ++i) e[i] = ad4_row_value(sf, row, term, rs[i]);
            table_row_from_energies(e.data(), rs.data(), n, &fast[(std::size_t)row * n],
                                    &smooth[(std::size_t)row * n * 2]);
        }
        return;
    }
    n_types = XS_SIZE;
    const int ntp = n_types * (n_types + 1) / 2;
    fast.assign((std::size_t)ntp * n, 0.0f);
    smooth.assign((std::size_t)ntp * n * 2, 0.0f);
    std::vector<float> rs(n), e(n);
    for (int i = 0; i < n; ++i) rs[i] = std::sqrt((float)i / factor);
    const float vmax = std::numeric_limits<float>::max();
    for (int t1 = 0; t1 < n_types; ++t1)
        for (int t2 = t1; t2 < n_types; ++t2) {
            const int tp = tri_index(t1, t2);
            for (int i = 0; i < n; ++i) {
                float v = (term < 0) ? sf.eval_types(t1, t2, rs[i]) : sf.term_types(term, t1, t2, rs[i]);
                e[i] = std::min(vmax, v);
            }
            table_row_from_energies(e.data(), rs.data(), n, &fast[(std::size_t)tp * n],
                                    &smooth[(std::size_t)tp * n * 2]);
        }
}

}  // namespace ud

// ---------------------------------------------------------------- bias

namespace ud {

std::vector<BiasElement> parse_bias(const std::string& text) {
    std::vector<BiasElement> out;
    std::istringstream in(text);
    std::string line;
    std::getline(in, line);  // header
    while (std::getline(in, line)) {
        std::istringstream l(line);
        BiasElement b;
        if (!(l >> b.xyz[0] >> b.xyz[1] >> b.xyz[2] >> b.vset >> b.r)) continue;
        std::string t;
        l >> t;
        if (t == "don") b.type = BIAS_DON;
        else if (t == "acc") b.type = BIAS_ACC;
        else if (t == "aro") b.type = BIAS_ARO;
        else if (t == "map") {
            b.type = BIAS_MAP;
            for (std::string a; l >> a;) {  // AD types; metals and unknown names are not kept (bias.h)
                const int ad = ad_type_from_name(a);
                if (ad < AD_SIZE) b.ad_list.push_back(ad);
            }
        } else b.type = BIAS_UNKNOWN;
        out.push_back(b);
    }
    return out;
}

uint64_t bias_ad4_map_types(const BiasElement& b) {
    auto bit = [](int t) { return (uint64_t)1 << t; };
    switch (b.type) {
        case BIAS_DON: return bit(AD_HD);
        case BIAS_ACC: return bit(AD_OA) | bit(AD_NA);
        case BIAS_ARO: return bit(AD_A);
        case BIAS_MAP: {
            if (b.ad_list.empty()) return ~(uint64_t)0;
            uint64_t m = 0;
            for (int ad : b.ad_list) m |= bit(ad);
            return m;
        }
        default: return 0;
    }
}

uint64_t bias_map_types(const BiasElement& b) {
    auto bit = [](int t) { return (uint64_t)1 << t; };
    uint64_t m = 0;
    if (b.type == BIAS_ACC) return bit(XS_O_A) | bit(XS_N_A) | bit(XS_O_DA) | bit(XS_N_DA);
    if (b.type != BIAS_MAP) return 0;
    if (b.ad_list.empty()) return (bit(XS_SIZE) - 1);
    for (int ad : b.ad_list) {
        switch (ad_to_el(ad)) {
            case EL_C:
                if (ad == AD_CG0) m |= bit(XS_C_P_CG0) | bit(XS_C_H_CG0);
                else if (ad == AD_CG1) m |= bit(XS_C_P_CG1) | bit(XS_C_H_CG1);
                else if (ad == AD_CG2) m |= bit(XS_C_P_CG2) | bit(XS_C_H_CG2);
                else if (ad == AD_CG3) m |= bit(XS_C_P_CG3) | bit(XS_C_H_CG3);
                else if (ad == AD_C)
                    m |= bit(XS_C_P_CG0) | bit(XS_C_H_CG0) | bit(XS_C_P_CG1) | bit(XS_C_H_CG1) | bit(XS_C_P_CG2) |
                         bit(XS_C_H_CG2) | bit(XS_C_P_CG3) | bit(XS_C_H_CG3) | bit(XS_C_P) | bit(XS_C_H);
                else m |= bit(XS_C_P) | bit(XS_C_H);
                break;
            case EL_N: m |= bit(XS_N_DA) | bit(XS_N_A) | bit(XS_N_D) | bit(XS_N_P); break;
            case EL_O: m |= bit(XS_O_DA) | bit(XS_O_A) | bit(XS_O_D) | bit(XS_O_P); break;
            case EL_S: m |= bit(XS_S_P); break;
            case EL_P: m |= bit(XS_P_P); break;
            case EL_F: m |= bit(XS_F_H); break;
            case EL_Cl: m |= bit(XS_Cl_H); break;
            case EL_Br: m |= bit(XS_Br_H); break;
            case EL_I: m |= bit(XS_I_H); break;
            case EL_Si: m |= bit(XS_Si); break;
            case EL_At: m |= bit(XS_At); break;
            case EL_Met: m |= bit(XS_Met_D); break;
            case EL_Dummy:
                if (ad == AD_G0) m |= bit(XS_G0);
                else if (ad == AD_G1) m |= bit(XS_G1);
                else if (ad == AD_G2) m |= bit(XS_G2);
                else if (ad == AD_G3) m |= bit(XS_G3);
                break;  // W: no XS type
            default: break;
        }
    }
    return m;
}

void bias_atom_multiplicity(const BiasElement& b, unsigned char mult[XS_SIZE]) {
    for (int t = 0; t < XS_SIZE; ++t) mult[t] = 0;
    auto add = [&](int t) {
        if (mult[t] < 255) ++mult[t];
    };
    if (b.type == BIAS_ACC) {
        for (int t : {XS_O_A, XS_N_A, XS_O_DA, XS_N_DA}) add(t);
        return;
    }
    if (b.type != BIAS_MAP) return;  // donor: no polar H in XS scoring; aromatic: CG types never remain
    if (b.ad_list.empty()) {  // every scored atom (glue atoms are not scored)
        for (int t = 0; t < XS_SIZE; ++t) add(t);
        return;
    }
    for (int ad : b.ad_list) {
        switch (ad_to_el(ad)) {
            case EL_C: add(XS_C_P); add(XS_C_H); break;  // atoms' CG types were folded into C_H / C_P
            case EL_N: for (int t : {XS_N_DA, XS_N_A, XS_N_D, XS_N_P}) add(t); break;
            case EL_O: for (int t : {XS_O_DA, XS_O_A, XS_O_D, XS_O_P}) add(t); break;
            case EL_S: add(XS_S_P); break;
            case EL_P: add(XS_P_P); break;
            case EL_F: add(XS_F_H); break;
            case EL_Cl: add(XS_Cl_H); break;
            case EL_Br: add(XS_Br_H); break;
            case EL_I: add(XS_I_H); break;
            case EL_Si: add(XS_Si); break;
            case EL_At: add(XS_At); break;
            case EL_Met: add(XS_Met_D); break;
            default: break;  // hydrogen, glue and W select no scored atom
        }
    }
    for (int t : {XS_C_H_CG0, XS_C_H_CG1, XS_C_H_CG2, XS_C_H_CG3}) mult[t] = mult[XS_C_H];
    for (int t : {XS_C_P_CG0, XS_C_P_CG1, XS_C_P_CG2, XS_C_P_CG3}) mult[t] = mult[XS_C_P];
}

}  // namespace ud
