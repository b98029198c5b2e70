/*
 * CPU restatement (oracle) of the reference's docking arithmetic.
 * Test infrastructure only: it checks the CUDA engine and is never part of
 * the product path.  Each function names the reference code it restates;
 * paths are relative to the reference repository (dptech-corp/Uni-Dock).
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define XS_SIZE 36
/* FP32 build: the float libm functions the reference calls (std::exp/sqrt/cos/sin on float) */
#if ORACLE_IS_FLOAT
#define RX(fn) fn##f
#else
#define RX(fn) fn
#endif
static const real PI_R = (real)3.1415926535897931;
static const real EPS_R = (real)FLT_EPSILON;   /* the reference's fl is float */
static const real MAXF = (real)FLT_MAX;

/* unidock/src/lib/atom_constants.h:313-350 (X-Score radii), :352-389 (Vinardo) */
static const float xs_r[XS_SIZE] = {1.9f, 1.9f, 1.8f, 1.8f, 1.8f, 1.8f, 1.7f, 1.7f, 1.7f, 1.7f, 2.0f, 2.1f,
                                    1.5f, 1.8f, 2.0f, 2.2f, 2.2f, 2.3f, 1.2f, 1.9f, 1.9f, 1.9f, 1.9f, 1.9f,
                                    1.9f, 1.9f, 1.9f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.7f, 1.8f, 1.7f, 1.8f};
static const float xs_vr[XS_SIZE] = {2.0f, 2.0f, 1.7f, 1.7f, 1.7f, 1.7f, 1.6f, 1.6f, 1.6f, 1.6f, 2.0f, 2.1f,
                                     1.5f, 1.8f, 2.0f, 2.2f, 2.2f, 2.3f, 1.2f, 2.0f, 2.0f, 2.0f, 2.0f, 2.0f,
                                     2.0f, 2.0f, 2.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.6f, 1.7f, 1.6f, 1.7f};
/* the reference indexes these arrays by type id (xs_radius, atom_constants.h:391-401);
 * glue types (ids 21, 24, 27, 30) never reach them (optimal_distance returns 0) */
static int is_glue(int t) { return t == 21 || t == 24 || t == 27 || t == 30; }
static real xs_radius(int t, int vinardo) { return (real)(vinardo ? xs_vr[t] : xs_r[t]); }
static int hydrophobic(int t) { return t == 0 || t == 12 || t == 13 || t == 14 || t == 15; }
static int acceptor(int t) { return t == 4 || t == 5 || t == 8 || t == 9 || t == 32 || t == 33; }
static int donor(int t) { return t == 3 || t == 5 || t == 7 || t == 9 || t == 18 || t == 33 || t == 34 || t == 35; }
static int hbond_possible(int a, int b) { return (donor(a) && acceptor(b)) || (donor(b) && acceptor(a)); }
static int biased(int t) { return t >= 32 && t <= 35; }
static int glued(int a, int b) {
    /* potentials.h:100-121: G0..G3 with their CG carbons */
    const int g[4] = {21, 24, 27, 30}, ch[4] = {19, 22, 25, 28}, cp[4] = {20, 23, 26, 29};
    for (int k = 0; k < 4; ++k)
        if ((a == g[k] && (b == ch[k] || b == cp[k])) || (b == g[k] && (a == ch[k] || a == cp[k]))) return 1;
    return 0;
}

/* potentials.h:29-38 */
static real slope_step(real bad, real good, real x) {
    if (bad < good) {
        if (x <= bad) return 0;
        if (x >= good) return 1;
    } else {
        if (x >= bad) return 0;
        if (x <= good) return 1;
    }
    return (x - bad) / (good - bad);
}

static real opt_dist(int a, int b, int vinardo) {
    if (is_glue(a) || is_glue(b)) return 0;
    return xs_radius(a, vinardo) + xs_radius(b, vinardo);
}

/* Weighted type-pair energy: scoring_function.h:47-68 terms, potentials.h:137-345,487-509 */
static real pair_energy(int sf, const double* w, int t1, int t2, real r) {
    const int vin = (sf == 2);
    real acc = 0;
    if (!vin) {
        real terms[6] = {0, 0, 0, 0, 0, 0};
        if (r < 8) {
            real d0 = r - (opt_dist(t1, t2, 0) + 0);
            terms[0] = RX(exp)(-((d0 / (real)0.5) * (d0 / (real)0.5)));
            real d3 = r - (opt_dist(t1, t2, 0) + 3);
            terms[1] = RX(exp)(-((d3 / 2) * (d3 / 2)));
            if (d0 <= 0) terms[2] = d0 * d0;
            if (hydrophobic(t1) && hydrophobic(t2)) terms[3] = slope_step((real)1.5, (real)0.5, r - opt_dist(t1, t2, 0));
            if (hbond_possible(t1, t2)) {
                real s = slope_step(0, (real)-0.7, r - opt_dist(t1, t2, 0));
                terms[4] = (biased(t1) || biased(t2)) ? (real)(10.0 * (double)s) : s;
            }
        }
        if (r < 20 && glued(t1, t2)) terms[5] = r;
        for (int k = 0; k < 6; ++k) acc += (real)(float)w[k] * terms[k];
    } else {
        real terms[5] = {0, 0, 0, 0, 0};
        if (r < 8) {
            real d0 = r - (opt_dist(t1, t2, 1) + 0);
            terms[0] = RX(exp)(-((d0 / (real)0.8) * (d0 / (real)0.8)));
            if (d0 <= 0) terms[1] = d0 * d0;
            if (hydrophobic(t1) && hydrophobic(t2)) terms[2] = slope_step((real)2.5, 0, r - opt_dist(t1, t2, 1));
            if (hbond_possible(t1, t2)) terms[3] = slope_step(0, (real)-0.6, r - opt_dist(t1, t2, 1));
        }
        if (r < 20 && glued(t1, t2)) terms[4] = r;
        for (int k = 0; k < 5; ++k) acc += (real)(float)w[k] * terms[k];
    }
    return acc;
}

int orc_table_bins(int sf) { (void)sf; return (int)(32.0f * 64.0f) + 3; }

/* precalculate::precalculate + precalculate_element::init_from_smooth_fst
 * (unidock/src/lib/precalculate.h:66-85, 133-168, 188-193) */
int orc_table_row(int sf, const double* w, int nw, int t1, int t2, real* fast, real* smooth) {
    (void)nw;
    const int n = orc_table_bins(sf);
    const real factor = 32;
    real* rs = (real*)malloc(sizeof(real) * n);
    for (int i = 0; i < n; ++i) rs[i] = RX(sqrt)((real)i / factor);
    for (int i = 0; i < n; ++i) {
        real e = pair_energy(sf, w, t1, t2, rs[i]);
        smooth[2 * i] = e < MAXF ? e : MAXF;
    }
    for (int i = 0; i < n; ++i) {
        real dor;
        if (i == 0 || i == n - 1) dor = 0;
        else dor = (smooth[2 * (i + 1)] - smooth[2 * (i - 1)]) / ((rs[i + 1] - rs[i - 1]) * rs[i]);
        smooth[2 * i + 1] = dor;
        real f1 = smooth[2 * i], f2 = (i + 1 >= n) ? 0 : smooth[2 * (i + 1)];
        fast[i] = (f2 + f1) / 2;
    }
    free(rs);
    return n;
}

static int tri(int a, int b) { return a <= b ? a + b * (b + 1) / 2 : b + a * (a + 1) / 2; }

/* cache::populate_no_bias (unidock/src/lib/cache.cpp:471-549): each grid point
 * sums the fast-table energy of every typed receptor atom with r^2 <= cutoff^2,
 * in ascending atom order (the szv_grid candidate order). */
void orc_maps(int sf, const double* w, int nw, const real* rx, const int* rt, int n_rec, const int* dims,
              const real* init, const real* finv, const int* types, int n_types, real* out) {
    const int nb = orc_table_bins(sf);
    real* tab = (real*)malloc(sizeof(real) * (size_t)XS_SIZE * n_types * nb);
    real* sm = (real*)malloc(sizeof(real) * 2 * nb);
    for (int t1 = 0; t1 < XS_SIZE; ++t1)
        for (int k = 0; k < n_types; ++k) orc_table_row(sf, w, nw, t1, types[k], tab + ((size_t)t1 * n_types + k) * nb, sm);
    free(sm);
    /* 8 A cell list keeps the candidate scan short; candidates are re-sorted by index */
    const real cell = 8;
    real lo[3] = {init[0] - 8, init[1] - 8, init[2] - 8};
    int nc[3];
    for (int d = 0; d < 3; ++d) nc[d] = (int)((finv[d] * (dims[d] - 1) + 16) / cell) + 1;
    int ncell = nc[0] * nc[1] * nc[2];
    int* head = (int*)malloc(sizeof(int) * (ncell + 1));
    int* cnt = (int*)calloc(ncell + 1, sizeof(int));
    int* cid = (int*)malloc(sizeof(int) * (n_rec > 0 ? n_rec : 1));
    for (int i = 0; i < n_rec; ++i) {
        cid[i] = -1;
        if (rt[i] < 0 || rt[i] >= XS_SIZE) continue;
        int c[3], ok = 1;
        for (int d = 0; d < 3; ++d) {
            c[d] = (int)floor((double)((rx[3 * i + d] - lo[d]) / cell));
            if (c[d] < 0 || c[d] >= nc[d]) ok = 0;
        }
        if (!ok) continue;
        cid[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cnt[cid[i]]++;
    }
    head[0] = 0;
    for (int k = 0; k < ncell; ++k) head[k + 1] = head[k] + cnt[k];
    int* list = (int*)malloc(sizeof(int) * (head[ncell] + 1));
    int* fill = (int*)calloc(ncell, sizeof(int));
    for (int i = 0; i < n_rec; ++i)
        if (cid[i] >= 0) list[head[cid[i]] + fill[cid[i]]++] = i;  /* ascending within a cell */
    int* cand = (int*)malloc(sizeof(int) * (n_rec > 0 ? n_rec : 1));
    real* acc = (real*)malloc(sizeof(real) * n_types);
    const size_t plane = (size_t)dims[0] * dims[1] * dims[2];
    for (int z = 0; z < dims[2]; ++z)
        for (int y = 0; y < dims[1]; ++y)
            for (int x = 0; x < dims[0]; ++x) {
                real p[3] = {init[0] + finv[0] * (real)x, init[1] + finv[1] * (real)y, init[2] + finv[2] * (real)z};
                int c[3];
                for (int d = 0; d < 3; ++d) c[d] = (int)floor((double)((p[d] - lo[d]) / cell));
                int nca = 0;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx) {
                            int a = c[0] + dx, b = c[1] + dy, cc = c[2] + dz;
                            if (a < 0 || b < 0 || cc < 0 || a >= nc[0] || b >= nc[1] || cc >= nc[2]) continue;
                            int k = (cc * nc[1] + b) * nc[0] + a;
                            for (int q = head[k]; q < head[k + 1]; ++q) cand[nca++] = list[q];
                        }
                /* insertion sort: candidate lists are short */
                for (int i = 1; i < nca; ++i) {
                    int v = cand[i], j = i - 1;
                    while (j >= 0 && cand[j] > v) { cand[j + 1] = cand[j]; --j; }
                    cand[j + 1] = v;
                }
                for (int k = 0; k < n_types; ++k) acc[k] = 0;
                for (int q = 0; q < nca; ++q) {
                    int i = cand[q];
                    real dx = rx[3 * i] - p[0], dy = rx[3 * i + 1] - p[1], dz = rx[3 * i + 2] - p[2];
                    real r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 <= 64) {
                        int bin = (int)((real)32 * r2);
                        const real* row = tab + (size_t)rt[i] * n_types * nb;
                        for (int k = 0; k < n_types; ++k) acc[k] += row[(size_t)k * nb + bin];
                    }
                }
                size_t idx = x + (size_t)dims[0] * (y + (size_t)dims[1] * z);
                for (int k = 0; k < n_types; ++k) out[k * plane + idx] = acc[k];
            }
    free(tab); free(head); free(cnt); free(cid); free(list); free(fill); free(cand); free(acc);
}

/* ---------------------------------------------------------------- kinematics */
static void q2r(const real* q, real* m) { /* quaternion_to_r3, quaternion.cpp:84-115 (row-major) */
    real a = q[0], b = q[1], c = q[2], d = q[3];
    real aa = a * a, ab = a * b, ac = a * c, ad = a * d, bb = b * b, bc = b * c, bd = b * d, cc = c * c, cd = c * d,
         dd = d * d;
    m[0] = aa + bb - cc - dd; m[1] = 2 * (-ad + bc); m[2] = 2 * (ac + bd);
    m[3] = 2 * (ad + bc); m[4] = aa - bb + cc - dd; m[5] = 2 * (-ab + cd);
    m[6] = 2 * (-ac + bd); m[7] = 2 * (ab + cd); m[8] = aa - bb - cc + dd;
}
static void qmul(const real* a, const real* b, real* o) {
    real t0 = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    real t1 = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
    real t2 = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
    real t3 = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}
static real norm_angle(real x) { /* normalize_angle, common.h:252-270 */
    if (x > 3 * PI_R) { real n = (x - PI_R) / (2 * PI_R); x -= 2 * PI_R * (real)ceil((double)n); return norm_angle(x); }
    if (x < -3 * PI_R) { real n = (-x - PI_R) / (2 * PI_R); x += 2 * PI_R * (real)ceil((double)n); return norm_angle(x); }
    if (x > PI_R) return x - 2 * PI_R;
    if (x < -PI_R) return x + 2 * PI_R;
    return x;
}
static void axis_angle(const real* ax, real ang, real* q) { /* angle_to_quaternion, quaternion.cpp:33-44 */
    ang = norm_angle(ang);
    real c = RX(cos)(ang / 2), s = RX(sin)(ang / 2);
    q[0] = c; q[1] = s * ax[0]; q[2] = s * ax[1]; q[3] = s * ax[2];
}
static void qnorm_approx(real* q) { /* quaternion_normalize_approx, quaternion.h:80-92 */
    real s = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (!(fabs((double)(s - 1)) < 1e-6)) {
        real a = RX(sqrt)(s);
        for (int k = 0; k < 4; ++k) q[k] *= 1 / a;
    }
}

typedef struct {
    real o[3], q[4], m[9], axis[3];
} frame;

/* model::set / tree::set_conf (tree.h:89-93,116-128,199-208) */
static void set_conf(const orc_ligand* L, const real* pose, frame* F, real* xyz) {
    for (int k = 0; k < 3; ++k) F[0].o[k] = pose[k];
    for (int k = 0; k < 4; ++k) F[0].q[k] = pose[3 + k];
    q2r(F[0].q, F[0].m);
    for (int n = 1; n < L->n_nodes; ++n) {
        const frame* P = &F[L->parent[n]];
        const real* rel = L->rel + 6 * n;
        for (int i = 0; i < 3; ++i) {
            F[n].o[i] = P->o[i] + (P->m[3 * i] * rel[0] + P->m[3 * i + 1] * rel[1] + P->m[3 * i + 2] * rel[2]);
            F[n].axis[i] = P->m[3 * i] * rel[3] + P->m[3 * i + 1] * rel[4] + P->m[3 * i + 2] * rel[5];
        }
        real t[4];
        axis_angle(F[n].axis, pose[7 + n - 1], t);
        qmul(t, P->q, F[n].q);
        qnorm_approx(F[n].q);
        q2r(F[n].q, F[n].m);
    }
    for (int a = 0; a < L->n_atoms; ++a) {
        const frame* f = &F[L->node[a]];
        const real* l = L->local + 3 * a;
        for (int i = 0; i < 3; ++i) xyz[3 * a + i] = f->o[i] + (f->m[3 * i] * l[0] + f->m[3 * i + 1] * l[1] + f->m[3 * i + 2] * l[2]);
    }
}

/* grid::evaluate_aux with curl (grid.cpp:40-129, curl.h:28-43) */
static real grid_eval(const orc_grid* G, int t, const real* p, real v, real* d) {
    real s[3], miss[3];
    int reg[3], a[3];
    for (int i = 0; i < 3; ++i) {
        s[i] = (p[i] - G->init[i]) * G->factor[i];
        if (s[i] < 0) { miss[i] = -s[i]; reg[i] = -1; a[i] = 0; s[i] = 0; }
        else if (s[i] >= G->dim_m1[i]) { miss[i] = s[i] - G->dim_m1[i]; reg[i] = 1; a[i] = G->dims[i] - 2; s[i] = 1; }
        else { miss[i] = 0; reg[i] = 0; a[i] = (int)s[i]; s[i] -= a[i]; }
    }
    const real penalty = G->slope * (miss[0] * G->factor_inv[0] + miss[1] * G->factor_inv[1] + miss[2] * G->factor_inv[2]);
    const real* m = G->maps + (size_t)t * G->dims[0] * G->dims[1] * G->dims[2];
#define AT(x, y, z) m[(x) + (size_t)G->dims[0] * ((y) + (size_t)G->dims[1] * (z))]
    real f000 = AT(a[0], a[1], a[2]), f100 = AT(a[0] + 1, a[1], a[2]), f010 = AT(a[0], a[1] + 1, a[2]),
         f110 = AT(a[0] + 1, a[1] + 1, a[2]), f001 = AT(a[0], a[1], a[2] + 1), f101 = AT(a[0] + 1, a[1], a[2] + 1),
         f011 = AT(a[0], a[1] + 1, a[2] + 1), f111 = AT(a[0] + 1, a[1] + 1, a[2] + 1);
#undef AT
    real x = s[0], y = s[1], z = s[2], mx = 1 - x, my = 1 - y, mz = 1 - z;
    real f = f000 * mx * my * mz + f100 * x * my * mz + f010 * mx * y * mz + f110 * x * y * mz + f001 * mx * my * z +
             f101 * x * my * z + f011 * mx * y * z + f111 * x * y * z;
    if (d) {
        real gx = f000 * (-1) * my * mz + f100 * 1 * my * mz + f010 * (-1) * y * mz + f110 * 1 * y * mz +
                  f001 * (-1) * my * z + f101 * 1 * my * z + f011 * (-1) * y * z + f111 * 1 * y * z;
        real gy = f000 * mx * (-1) * mz + f100 * x * (-1) * mz + f010 * mx * 1 * mz + f110 * x * 1 * mz +
                  f001 * mx * (-1) * z + f101 * x * (-1) * z + f011 * mx * 1 * z + f111 * x * 1 * z;
        real gz = f000 * mx * my * (-1) + f100 * x * my * (-1) + f010 * mx * y * (-1) + f110 * x * y * (-1) +
                  f001 * mx * my * 1 + f101 * x * my * 1 + f011 * mx * y * 1 + f111 * x * y * 1;
        real g[3] = {gx, gy, gz};
        if (f > 0 && v < (real)0.1 * MAXF) {
            real tmp = (v < EPS_R) ? 0 : (v / (v + f));
            f *= tmp;
            for (int i = 0; i < 3; ++i) g[i] *= tmp * tmp;
        }
        for (int i = 0; i < 3; ++i) d[i] = G->factor[i] * (reg[i] == 0 ? g[i] : 0) + G->slope * reg[i];
    } else if (f > 0 && v < (real)0.1 * MAXF) {
        f *= (v < EPS_R) ? 0 : (v / (v + f));
    }
    return f + penalty;
}

/* tree::derivative / branches_derivative (tree.h:75-84,164-192): returns the
 * subtree force and torque of node n about its origin, fills torsion slots. */
static void derivative(const orc_ligand* L, const frame* F, const real* xyz, const real* frc, int n, real* out6,
                       real* g) {
    real ft[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < L->n_atoms; ++a) {
        if (L->node[a] != n) continue;
        real r[3] = {xyz[3 * a] - F[n].o[0], xyz[3 * a + 1] - F[n].o[1], xyz[3 * a + 2] - F[n].o[2]};
        const real* f = frc + 3 * a;
        ft[0] += f[0]; ft[1] += f[1]; ft[2] += f[2];
        ft[3] += r[1] * f[2] - r[2] * f[1];
        ft[4] += r[2] * f[0] - r[0] * f[2];
        ft[5] += r[0] * f[1] - r[1] * f[0];
    }
    for (int c = n + 1; c < L->n_nodes; ++c) {
        if (L->parent[c] != n) continue;
        real ch[6];
        derivative(L, F, xyz, frc, c, ch, g);
        real r[3] = {F[c].o[0] - F[n].o[0], F[c].o[1] - F[n].o[1], F[c].o[2] - F[n].o[2]};
        ft[0] += ch[0]; ft[1] += ch[1]; ft[2] += ch[2];
        ft[3] += (r[1] * ch[2] - r[2] * ch[1]) + ch[3];
        ft[4] += (r[2] * ch[0] - r[0] * ch[2]) + ch[4];
        ft[5] += (r[0] * ch[1] - r[1] * ch[0]) + ch[5];
    }
    if (n > 0) g[6 + n - 1] = ft[3] * F[n].axis[0] + ft[4] * F[n].axis[1] + ft[5] * F[n].axis[2];
    memcpy(out6, ft, sizeof ft);
}

/* model::eval_deriv (model.cpp:935-962) with cache::eval_deriv (cache.cpp:160-199)
 * and eval_interacting_pairs_deriv (model.cpp:888-915). */
real orc_eval_deriv(const orc_ligand* L, const orc_grid* G, const real* smooth, int nb, const real* pose, real v_intra,
                    real v_inter, real* g, real* xyz_out) {
    frame* F = (frame*)calloc(L->n_nodes, sizeof(frame));
    real* xyz = (real*)malloc(sizeof(real) * 3 * L->n_atoms);
    real* frc = (real*)calloc(3 * L->n_atoms, sizeof(real));
    set_conf(L, pose, F, xyz);
    real e = 0;
    for (int a = 0; a < L->n_atoms; ++a) {
        if (L->gtype[a] < 0) continue;
        e += grid_eval(G, L->gtype[a], xyz + 3 * a, v_inter, frc + 3 * a);
    }
    for (int k = 0; k < L->n_pairs; ++k) {
        int a = L->pa[k], b = L->pb[k];
        real r[3] = {xyz[3 * b] - xyz[3 * a], xyz[3 * b + 1] - xyz[3 * a + 1], xyz[3 * b + 2] - xyz[3 * a + 2]};
        real r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        if (r2 < 64) {
            real rf = 32 * r2;
            int i1 = (int)rf;
            real rem = rf - i1;
            const real* row = smooth + (size_t)L->ptp[k] * nb * 2;
            real pe = row[2 * i1] + rem * (row[2 * i1 + 2] - row[2 * i1]);
            real dor = row[2 * i1 + 1] + rem * (row[2 * i1 + 3] - row[2 * i1 + 1]);
            real f[3] = {dor * r[0], dor * r[1], dor * r[2]};
            if (pe > 0 && v_intra < (real)0.1 * MAXF) {
                real tmp = (v_intra < EPS_R) ? 0 : (v_intra / (v_intra + pe));
                pe *= tmp;
                for (int i = 0; i < 3; ++i) f[i] *= tmp * tmp;
            }
            e += pe;
            for (int i = 0; i < 3; ++i) {
                frc[3 * a + i] -= f[i];
                frc[3 * b + i] += f[i];
            }
        }
    }
    real root[6];
    derivative(L, F, xyz, frc, 0, root, g);
    for (int i = 0; i < 6; ++i) g[i] = root[i];
    if (xyz_out) memcpy(xyz_out, xyz, sizeof(real) * 3 * L->n_atoms);
    free(F); free(xyz); free(frc);
    return e;
}

/* cache::eval (cache.cpp:84-120) + model::evali (model.cpp:867-886, 927-933) */
void orc_eval_score(const orc_ligand* L, const orc_grid* G, const real* fast, int nb, const real* pose, real v,
                    real* out) {
    frame* F = (frame*)calloc(L->n_nodes, sizeof(frame));
    real* xyz = (real*)malloc(sizeof(real) * 3 * L->n_atoms);
    set_conf(L, pose, F, xyz);
    real eg = 0, ei = 0;
    for (int a = 0; a < L->n_atoms; ++a)
        if (L->gtype[a] >= 0) eg += grid_eval(G, L->gtype[a], xyz + 3 * a, v, NULL);
    for (int k = 0; k < L->n_pairs; ++k) {
        int a = L->pa[k], b = L->pb[k];
        real dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1], dz = xyz[3 * a + 2] - xyz[3 * b + 2];
        real r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < 64) {
            real t = fast[(size_t)L->ptp[k] * nb + (int)(32 * r2)];
            if (t > 0 && v < (real)0.1 * MAXF) t *= (v < EPS_R) ? 0 : (v / (v + t));
            ei += t;
        }
    }
    out[0] = eg;
    out[1] = ei;
    free(F); free(xyz);
}

/* ---------------------------------------------------------------- BFGS (bfgs.h:27-146) */
static void increment(const real* x, const real* p, real alpha, int T, real* out) { /* conf.h:98-104,146-150 */
    for (int i = 0; i < 3; ++i) out[i] = x[i] + alpha * p[i];
    real rot[3] = {alpha * p[3], alpha * p[4], alpha * p[5]};
    real ang = RX(sqrt)(rot[0] * rot[0] + rot[1] * rot[1] + rot[2] * rot[2]);
    real t[4] = {1, 0, 0, 0};
    if (ang > EPS_R) {
        real ax[3] = {rot[0] / ang, rot[1] / ang, rot[2] / ang};
        axis_angle(ax, ang, t);
    }
    qmul(t, x + 3, out + 3);
    qnorm_approx(out + 3);
    for (int k = 0; k < T; ++k) out[7 + k] = norm_angle(x[7 + k] + norm_angle(alpha * p[6 + k]));
}

static real dot(const real* a, const real* b, int n) {
    real s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

real orc_bfgs(const orc_ligand* L, const orc_grid* G, const real* smooth, int nb, real* x, int max_steps, real v,
              int* evals) {
    const int T = L->n_nodes - 1, n = 6 + T, cs = 7 + T;
    real* H = (real*)calloc((size_t)n * (n + 1) / 2, sizeof(real));
    real *g = (real*)calloc(n, sizeof(real)), *gn = (real*)calloc(n, sizeof(real)), *g0 = (real*)calloc(n, sizeof(real));
    real *p = (real*)calloc(n, sizeof(real)), *y = (real*)calloc(n, sizeof(real)), *mhy = (real*)calloc(n, sizeof(real));
    real *xn = (real*)calloc(cs, sizeof(real)), *x0 = (real*)calloc(cs, sizeof(real));
    int ev = 0;
    for (int i = 0; i < n; ++i) H[tri(i, i)] = 1;
    real f0 = orc_eval_deriv(L, G, smooth, nb, x, v, v, g, NULL);
    ++ev;
    const real forig = f0;
    memcpy(g0, g, sizeof(real) * n);
    memcpy(x0, x, sizeof(real) * cs);
    for (int step = 0; step < max_steps; ++step) {
        for (int i = 0; i < n; ++i) {
            real s = 0;
            for (int j = 0; j < n; ++j) s += H[tri(i, j)] * g[j];
            p[i] = -s;
        }
        const real pg = dot(p, g, n);
        real alpha = 1, f1 = 0;
        for (int trial = 0; trial < 10; ++trial) {
            increment(x, p, alpha, T, xn);
            f1 = orc_eval_deriv(L, G, smooth, nb, xn, v, v, gn, NULL);
            ++ev;
            if (f1 - f0 < (real)0.0001 * alpha * pg) break;
            alpha *= (real)0.5;
        }
        for (int i = 0; i < n; ++i) y[i] = gn[i] - g[i];
        f0 = f1;
        memcpy(x, xn, sizeof(real) * cs);
        if (!(RX(sqrt)(dot(g, g, n)) >= (real)1e-5)) break;
        memcpy(g, gn, sizeof(real) * n);
        if (step == 0) {
            real yy = dot(y, y, n);
            if (fabs((double)yy) > EPS_R)
                for (int i = 0; i < n; ++i) H[tri(i, i)] = alpha * dot(y, p, n) / yy;
        }
        const real yp = dot(y, p, n);
        if (alpha * yp < EPS_R) continue;
        for (int i = 0; i < n; ++i) {
            real s = 0;
            for (int j = 0; j < n; ++j) s += H[tri(i, j)] * y[j];
            mhy[i] = -s;
        }
        const real yhy = -dot(y, mhy, n);
        const real r = 1 / (alpha * yp);
        for (int i = 0; i < n; ++i)
            for (int j = i; j < n; ++j)
                H[tri(i, j)] += alpha * r * (mhy[i] * p[j] + mhy[j] * p[i]) + alpha * alpha * (r * r * yhy + r) * p[i] * p[j];
    }
    if (!(f0 <= forig)) {
        f0 = forig;
        memcpy(x, x0, sizeof(real) * cs);
    }
    if (evals) *evals = ev;
    free(H); free(g); free(gn); free(g0); free(p); free(y); free(mhy); free(xn); free(x0);
    return f0;
}

/* ------------------------------------------------------------ AutoDock 4.2
 * unidock/src/lib/atom_constants.h:158-194 (ad_type_property: radius, depth,
 * hb_depth, hb_radius, solvation, volume) and potentials.h:346-486 (terms),
 * scoring_function.h:74-86 (smoothing 0.5, caps 100000 / 100, cutoffs 8 /
 * 20.48, desolvation sigma 3.6 and charge factor 0.01097). */
static const float ad_par[35][6] = {
    {2.00f, 0.150f, 0.0f, 0.0f, -0.00143f, 33.51030f}, {2.00f, 0.150f, 0.0f, 0.0f, -0.00052f, 33.51030f},
    {1.75f, 0.160f, 0.0f, 0.0f, -0.00162f, 22.44930f}, {1.60f, 0.200f, 0.0f, 0.0f, -0.00251f, 17.15730f},
    {2.10f, 0.200f, 0.0f, 0.0f, -0.00110f, 38.79240f}, {2.00f, 0.200f, 0.0f, 0.0f, -0.00214f, 33.51030f},
    {1.00f, 0.020f, 0.0f, 0.0f, 0.00051f, 0.00000f},   {1.545f, 0.080f, 0.0f, 0.0f, -0.00110f, 15.44800f},
    {2.36f, 0.550f, 0.0f, 0.0f, -0.00110f, 55.05850f}, {1.75f, 0.160f, -5.0f, 1.9f, -0.00162f, 22.44930f},
    {1.60f, 0.200f, -5.0f, 1.9f, -0.00251f, 17.15730f}, {2.00f, 0.200f, -1.0f, 2.5f, -0.00214f, 33.51030f},
    {1.00f, 0.020f, 1.0f, 0.0f, 0.00051f, 0.00000f},   {0.65f, 0.875f, 0.0f, 0.0f, -0.00110f, 1.56000f},
    {0.65f, 0.875f, 0.0f, 0.0f, -0.00110f, 2.14000f},  {0.74f, 0.550f, 0.0f, 0.0f, -0.00110f, 1.70000f},
    {0.99f, 0.550f, 0.0f, 0.0f, -0.00110f, 2.77000f},  {0.65f, 0.010f, 0.0f, 0.0f, -0.00110f, 1.84000f},
    {2.045f, 0.276f, 0.0f, 0.0f, -0.00110f, 35.82350f}, {2.165f, 0.389f, 0.0f, 0.0f, -0.00110f, 42.56610f},
    {2.30f, 0.200f, 0.0f, 0.0f, -0.00143f, 50.96500f}, {2.40f, 0.550f, 0.0f, 0.0f, -0.00110f, 57.90580f},
    {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {2.00f, 0.150f, 0.0f, 0.0f, -0.00143f, 33.51030f}, {2.00f, 0.150f, 0.0f, 0.0f, -0.00143f, 33.51030f},
    {2.00f, 0.150f, 0.0f, 0.0f, -0.00143f, 33.51030f}, {2.00f, 0.150f, 0.0f, 0.0f, -0.00143f, 33.51030f},
    {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {1.60f, 0.200f, 0.0f, 0.0f, -0.00251f, 17.15730f}, {1.75f, 0.160f, 0.0f, 0.0f, -0.00162f, 22.44930f},
    {1.60f, 0.200f, 0.0f, 0.0f, -0.00251f, 17.15730f}, {1.75f, 0.160f, 0.0f, 0.0f, -0.00162f, 22.44930f}};

static real ipow_r(real x, int n) {
    real p = 1;
    for (int i = 0; i < n; ++i) p = p * x;
    return p;
}

static real ad4_smooth(real r, real rij) {  /* potentials.h smoothen, smoothing 0.5 */
    const real h = (real)0.25;
    if (r > rij + h) return r - h;
    if (r < rij - h) return r + h;
    return rij;
}

real orc_ad4_pair(int t1, real q1, int t2, real q2, real r, const double* w) {
    real e = 0;
    const real cap = (real)100000;
    /* vdW 12-6 / H-bond 12-10, cutoff 8 */
    if (r < 8) {
        const real hbd = (real)ad_par[t1][2] * (real)ad_par[t2][2];
        if (hbd >= 0) {
            const real rij = (real)ad_par[t1][0] + (real)ad_par[t2][0];
            const real depth = RX(sqrt)((real)ad_par[t1][1] * (real)ad_par[t2][1]);
            const real rs = ad4_smooth(r, rij);
            const real c12 = ipow_r(rij, 12) * depth, c6 = ipow_r(rij, 6) * depth * 2;
            const real r6 = ipow_r(rs, 6), r12 = ipow_r(rs, 12);
            const real v = (r12 > EPS_R && r6 > EPS_R) ? (c12 / r12 - c6 / r6 < cap ? c12 / r12 - c6 / r6 : cap) : cap;
            e += (real)(float)w[0] * v;
        } else {
            const real rij = (real)ad_par[t1][3] + (real)ad_par[t2][3];
            const real rs = ad4_smooth(r, rij);
            const real c12 = ipow_r(rij, 12) * -hbd * 10 / 2, c10 = ipow_r(rij, 10) * -hbd * 12 / 2;
            const real r10 = ipow_r(rs, 10), r12 = ipow_r(rs, 12);
            const real v = (r12 > EPS_R && r10 > EPS_R) ? (c12 / r12 - c10 / r10 < cap ? c12 / r12 - c10 / r10 : cap)
                                                        : cap;
            e += (real)(float)w[1] * v;
        }
    }
    if (r < (real)20.48) {
        /* electrostatics, distance-dependent dielectric, cap 100 */
        const real B = (real)(78.4 + 8.5525);
        const real lB = -B * (real)0.003627;
        const real diel = (real)-8.5525 + B / (1 + (real)7.7839 * RX(exp)(lB * r));
        const real inv = r < EPS_R ? (real)100 / diel : ((real)1 / (r * diel) < 100 ? (real)1 / (r * diel) : (real)100);
        e += (real)(float)w[2] * (q1 * q2 * 332 * inv);
        /* desolvation */
        const real k = (real)0.01097, x = r / (real)3.6;
        const real g = RX(exp)((real)-0.5 * x * x);
        const real s1 = (real)ad_par[t1][4], s2 = (real)ad_par[t2][4], v1 = (real)ad_par[t1][5], v2 = (real)ad_par[t2][5];
        const real aq1 = q1 < 0 ? -q1 : q1, aq2 = q2 < 0 ? -q2 : q2;
        e += (real)(float)w[3] * (((s1 + k * aq1) * v2 + (s2 + k * aq2) * v1) * g);
    }
    return e;
}

real orc_ad4_probe(const real* rx, const int* rad, const real* rq, int n, const real* p, int probe_ad, real probe_q,
                   const double* w) {
    real acc = 0;
    for (int i = 0; i < n; ++i) {
        const real dx = rx[3 * i] - p[0], dy = rx[3 * i + 1] - p[1], dz = rx[3 * i + 2] - p[2];
        const real r2 = dx * dx + dy * dy + dz * dz;
        if (r2 >= (real)20.48 * (real)20.48) continue;
        acc += orc_ad4_pair(probe_ad, probe_q, rad[i], rq[i], RX(sqrt)(r2), w);
    }
    return acc;
}
