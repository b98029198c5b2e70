/*
 * CPU restatement of the reference's docking arithmetic (test infrastructure
 * only: tests/, the oracle leg of bench.py and __graft_entry__.smoke() use it
 * as the checker; the product never calls it).  Built twice by oracle/Makefile:
 * ORACLE_REAL=float (liboracle32.so, the reference's FP32 arithmetic) and
 * ORACLE_REAL=double (liboracle64.so, the FP64 oracle used to state errors).
 */
#ifndef UD_ORACLE_H
#define UD_ORACLE_H

#ifndef ORACLE_REAL
#define ORACLE_REAL float
/* AutoDock 4.2: weighted pair energy of two AD-typed atoms with charges
 * (w = vdW, H-bond, electrostatics, desolvation, glue), and the energy of a
 * probe atom against receptor atoms within the 20.48 A cutoff. */
real orc_ad4_pair(int t1, real q1, int t2, real q2, real r, const double* w);
real orc_ad4_probe(const real* rec_xyz, const int* rec_ad, const real* rec_q, int n_rec, const real* p,
                   int probe_ad, real probe_q, const double* w);

#endif
typedef ORACLE_REAL real;

/* Flat ligand topology (the layout exported by ud_ligand_export). */
typedef struct {
    int n_atoms, n_nodes, n_pairs;
    const real* local;     /* 3 per atom: coordinates relative to the owning node origin */
    const int* node;       /* owning node of each atom */
    const int* gtype;      /* grid map index of each atom, -1 = none */
    const int* heavy;      /* 1 for non-hydrogen atoms */
    const int* parent;     /* parent node (DFS pre-order, root = 0) */
    const real* rel;       /* 6 per node: origin relative to parent, unit axis */
    const int* pa;         /* pair atoms */
    const int* pb;
    const int* ptp;        /* type-pair index of each pair */
} orc_ligand;

typedef struct {
    int dims[3];
    real init[3], factor[3], factor_inv[3], dim_m1[3];
    real slope;
    const real* maps;      /* [map][z][y][x] */
} orc_grid;

/* One type-pair row of the r^2 tables (fast[n], smooth[n][2]) of scoring
 * function sf (0 Vina, 2 Vinardo) with weights w (rotatable weight last,
 * already transformed); returns n. */
int orc_table_row(int sf, const double* w, int nw, int t1, int t2, real* fast, real* smooth);
int orc_table_bins(int sf);

/* Grid maps of XS types `types` for typed receptor atoms. */
void orc_maps(int sf, const double* w, int nw, const real* rec_xyz, const int* rec_xs, int n_rec,
              const int* dims, const real* init, const real* factor_inv, const int* types,
              int n_types, real* out);

/* Energy and gradient (6 + T, change layout) of pose [x y z qw qx qy qz t...]. */
real orc_eval_deriv(const orc_ligand* L, const orc_grid* G, const real* smooth, int n_bins,
                    const real* pose, real v_intra, real v_inter, real* g, real* xyz_out);
/* Scoring energies: out[0] grid, out[1] intramolecular pairs (nearest-bin table). */
void orc_eval_score(const orc_ligand* L, const orc_grid* G, const real* fast, int n_bins,
                    const real* pose, real v, real* out);
/* BFGS local optimisation from `pose` (updated); returns the energy. */
real orc_bfgs(const orc_ligand* L, const orc_grid* G, const real* smooth, int n_bins, real* pose,
              int max_steps, real v, int* evals);

/* AutoDock 4.2: weighted pair energy of two AD-typed atoms with charges
 * (w = vdW, H-bond, electrostatics, desolvation, glue), and the energy of a
 * probe atom against receptor atoms within the 20.48 A cutoff. */
real orc_ad4_pair(int t1, real q1, int t2, real q2, real r, const double* w);
real orc_ad4_probe(const real* rec_xyz, const int* rec_ad, const real* rec_q, int n_rec, const real* p,
                   int probe_ad, real probe_q, const double* w);

#endif
