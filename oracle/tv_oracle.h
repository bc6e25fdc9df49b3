/*
 * tv_oracle.h -- CPU restatement of the Tandav gravity hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it. Each function restates the reference algorithm it cites; parity of
 * this restatement with the real reference (oracle/_ref/<variant>/ref_harness)
 * is itself checked by tests/test_oracle_vs_reference.py and the committed
 * fixtures in tests/golden/.
 *
 * Positions and masses are passed as "Float" arrays, whose width (4 or 8
 * bytes) is given by `fsize`, as in the reference's DOUBLE_PRECISION switch
 * (src/globals.h:46-54). 128-bit Peano keys are passed as pairs of uint64
 * (hi, lo).
 */
#ifndef TV_ORACLE_H
#define TV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Top node as in src/domain.h:40-52 (union Domain_Node_List, TNode part). */
typedef struct {
	uint64_t key;
	int32_t target, level, first_part, npart;
	float pos[3], mass, com[3], dp[3];
} tvo_topnode;

/* Walk parameters shared by both walks (tree_accel.c / tree_periodic.c). */
typedef struct {
	double gravity;        /* Const.Gravity */
	double softening;      /* Param.Grav_Softening[1] (Plummer equivalent) */
	double domain_size;    /* Domain.Size */
	double boxsize;        /* Sim.Boxsize[0]; <= 0 for isolated */
	double open_bh;        /* TREE_OPEN_PARAM_BH (theta^2) */
	double open_rel;       /* TREE_OPEN_PARAM_REL */
	int32_t use_bh;        /* Sig.Use_BH_Criterion */
	int32_t vector_size;   /* VECTOR_SIZE */
} tvo_walk_params;

/* Peano_Key / Reversed_Peano_Key (peano.c:122-276) for n particles. */
void tvo_peano_keys(int64_t n, int32_t fsize, const void *x, const void *y,
                    const void *z, const double origin[3], double size,
                    uint64_t *std_key, uint64_t *rev_key);

/* Index permutation ordering 128-bit keys ascending (Qsort_Index with
 * cmp_peanoKeys, sort.c:90-116 / peano.c:6-12); equal keys keep input order. */
void tvo_sort_keys(int64_t n, const uint64_t *key, uint32_t *perm);

/* Single-target domain decomposition (domain.c:67-145 with NTarget = 1):
 * all non-empty level-2 cells, ordered by descending short key, with the
 * node centre of transform_bunches_into_top_nodes (domain.c:220-250).
 * Keys must be sorted std keys. Returns the number of top nodes. */
int32_t tvo_top_nodes(int64_t n, int32_t fsize, const uint64_t *std_key,
                      const void *x, const void *y, const void *z,
                      const double origin[3], double size, tvo_topnode *out);

/* Gravity_Tree_Build (tree_build.c:47-572), sequential per top node, built
 * as if every subtree fits the thread buffer: subtrees are concatenated in
 * top-node order. tree must hold tree_cap nodes of the reference layout
 * (56 B FP32 / 96 B FP64). Returns the node count, or -1 when tree_cap is too
 * small, -2 on coincident particles (keys equal to 42 levels). */
int64_t tvo_tree_build(int64_t n, int32_t fsize, const uint64_t *rev_key,
                       const void *x, const void *y, const void *z,
                       const void *mass, double domain_size,
                       tvo_topnode *top, int32_t ntop, void *tree,
                       int64_t tree_cap, int32_t *tree_parent, int32_t vector_size);

/* Gravity_Tree_Acceleration walk part for the active particles
 * (tree_accel.c:32-394): acc += per-particle sum (double), cost = count.
 * last_acc is P.Last_Acc_Mag (relative criterion). */
void tvo_walk_gravity(int64_t n, int32_t fsize, const void *x, const void *y,
                      const void *z, const void *mass, const void *last_acc,
                      const tvo_topnode *top, int32_t ntop, const void *tree,
                      const tvo_walk_params *prm, double *acc, double *cost);

/* Gravity_Tree_Periodic (tree_periodic.c:23-450) with the table lookup of
 * Ewald_Correction (Gravity/periodic.c:35-113). ewald_fx/fy/fz are the 65^3
 * Float tables already divided by Boxsize^2. */
void tvo_walk_ewald(int64_t n, int32_t fsize, const void *x, const void *y,
                    const void *z, const void *mass, const void *last_acc,
                    const tvo_topnode *top, int32_t ntop, const void *tree,
                    const tvo_walk_params *prm, const void *ewald_fx,
                    const void *ewald_fy, const void *ewald_fz, double *acc,
                    double *cost);

/* The two walks with GRAVITY_POTENTIAL: pot[i] = the double sum of the
 * potential terms of particle i (interact(), tree_accel.c:362-389;
 * interact_with_ewald_cube with Ewald_Potential, tree_periodic.c:439-447,
 * Gravity/periodic.c:115-170; ewald_fp is the potential table divided by
 * Boxsize). pot may be NULL. */
void tvo_walk_gravity_pot(int64_t n, int32_t fsize, const void *x, const void *y,
                          const void *z, const void *mass, const void *last_acc,
                          const tvo_topnode *top, int32_t ntop, const void *tree,
                          const tvo_walk_params *prm, double *acc, double *cost,
                          double *pot);
void tvo_walk_ewald_pot(int64_t n, int32_t fsize, const void *x, const void *y,
                        const void *z, const void *mass, const void *last_acc,
                        const tvo_topnode *top, int32_t ntop, const void *tree,
                        const tvo_walk_params *prm, const void *ewald_fx,
                        const void *ewald_fy, const void *ewald_fz, const void *ewald_fp,
                        double *acc, double *cost, double *pot);

/* compute_ewald_force / compute_ewald_potential (Gravity/periodic.c:235-461)
 * in box units on the (N_EWALD+1)^3 octant grid, FP64 (not yet divided by
 * Boxsize^2 / Boxsize). */
void tvo_ewald_table(int32_t n_ewald, double *fx, double *fy, double *fz,
                     double *fp);

/* The same Ewald correction force at arbitrary separations x (box units),
 * with real-space images |n|<=nreal per axis and k-space |h|<=nk per axis. */
void tvo_ewald_force(int64_t m, const double *x, int32_t nreal, int32_t nk,
                     double *f);

/* FP64 direct summation onto `nt` targets with the reference's softened
 * kernel (interact(), tree_accel.c:362-394, h = -41/32 eps). When box > 0
 * the nearest image is used and, if corr_table != NULL, the Ewald correction
 * is added from a fine FP64 octant table (corr_n+1)^3 x 3 with tricubic
 * interpolation. */
void tvo_direct(int64_t n, const double *pos, const double *mass, int64_t nt,
                const int64_t *targets, double gravity, double softening,
                double box, const double *corr_table, int32_t corr_n,
                double *acc);

#ifdef __cplusplus
}
#endif
#endif
