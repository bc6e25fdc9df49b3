/*
 * tandav_gpu.h -- C ABI of the B200 (sm_100a) gravity hot path for Tandav.
 *
 * Each entry point replaces the body of one reference C entry point (paths
 * relative to the reference's src/); a reference build with GPU gravity calls
 * these from the original functions, inside one `#pragma omp single` (the
 * reference's entry points are orphaned OpenMP worksharing functions run by
 * every thread of the team, src/main.c:37).
 *
 * All pointers in this interface are host pointers to plain arrays; device
 * memory is owned by the context. "Float" arrays have the width given by
 * tvg_config.float_bytes (4, or 8 under DOUBLE_PRECISION, src/globals.h:46-54).
 * Every function returns TVG_OK or an error code; tvg_last_error() gives the
 * message. Nothing here falls back to the CPU: without a usable GPU the calls
 * fail with TVG_E_CUDA.
 */
#ifndef TANDAV_GPU_H
#define TANDAV_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the reference's fatal Assert, src/aux.c:49-77, becomes a
 * return value the host maps to Assert) */
enum {
	TVG_OK = 0,
	TVG_E_CUDA = 1,        /* CUDA runtime error or no device */
	TVG_E_NOMEM = 2,       /* device allocation failed */
	TVG_E_TREE_FULL = 3,   /* node capacity exceeded */
	TVG_E_TIMEOUT = 4,     /* a bounded device-side wait gave up */
	TVG_E_BADINPUT = 5,    /* invalid argument, NaN/Inf or out-of-domain position */
	TVG_E_COINCIDENT = 6,  /* particles equal to 41 key levels (tree_build.c:337) */
	TVG_E_STATE = 7        /* call out of order (e.g. walk before tree build) */
};

/* Largest capacity a context accepts: node and particle indices are 32-bit. */
#define TVG_MAX_PARTICLES (((int64_t) 1 << 30) - 4096)

typedef struct tvg_context tvg_context;

/* Compile-time Config and run-time parameters of the reference that the hot
 * path reads. */
typedef struct {
	int32_t float_bytes;   /* sizeof(Float) */
	int32_t periodic;      /* PERIODIC */
	double boxsize;        /* Sim.Boxsize[0] (periodic) */
	double gravity;        /* Const.Gravity (src/constants.c:5) */
	double softening;      /* Param.Grav_Softening[1]; tree_build.c:134-139 */
	double open_bh;        /* TREE_OPEN_PARAM_BH (theta^2) */
	double open_rel;       /* TREE_OPEN_PARAM_REL */
	int32_t vector_size;   /* VECTOR_SIZE */
	int32_t flags;         /* TVG_CFG_* */
	int64_t max_particles; /* device capacity (Task.Npart_Total_Max), <= TVG_MAX_PARTICLES */
} tvg_config;

enum {
	/* interact_with_topnode_particles indexes particles from the top node's
	 * Target (tree_accel.c:185, tree_periodic.c:188), which for top nodes with
	 * <= VECTOR_SIZE particles holds a tree index (tree_build.c:91). Set this
	 * flag to use First_Part instead. Default: the reference's behaviour. */
	TVG_CFG_FIX_SMALL_TOPNODES = 1,
	/* Group form: interact every particle of a bundle (a tree leaf of <=
	 * VECTOR_SIZE particles) that the walk reaches below the top level, as the
	 * reference's walks do (tree_accel.c:221-243). Default: such a bundle is a
	 * monopole like any other node when the opening criterion accepts it. */
	TVG_CFG_OPEN_BUNDLES = 2,
	/* GRAVITY_POTENTIAL: the plain form also computes Grav_Pot (the Dehnen K1
	 * potential of interact(), tree_accel.c:362-389, plus G m times the
	 * trilinear lookup of the Ewald potential table, Gravity/periodic.c:
	 * 115-170, tree_periodic.c:439-447), in the reference's sign convention
	 * (+G m / r). The group form computes no potential and refuses a walk
	 * while this flag is set. */
	TVG_CFG_POTENTIAL = 4,
	/* Isolated runs: every domain decomposition of tvg_compute_acceleration
	 * and tvg_force_step first recomputes the domain from the current order
	 * (tvg_find_domain), as Domain_Decomposition does (domain.c:67-71);
	 * tvg_step_graph then runs such steps directly. Without it the domain is
	 * the one last set (tvg_set_domain / tvg_find_domain). */
	TVG_CFG_FIND_DOMAIN = 8,
	/* Group form (no reference counterpart; the reference's walks use node
	 * monopoles): every accepted node also carries its traceless quadrupole
	 * moment about its centre of mass, summed from its particles in FP64 for
	 * each walk tree, and the relative criterion bounds the next (octupole)
	 * term instead: a node of mass M and size s at distance r from the group
	 * box is accepted when M s^3 <= r^5 |a_old|_min TREE_OPEN_PARAM_REL / G.
	 * The Ewald walk (groups without per-target images) adds each accepted
	 * node's quadrupole term to its correction and bounds the next term,
	 * G M s^3 max|d3 T| / (48 L^5) <= alpha_E |a_old|_min
	 * (tvg_set_ewald_opening). The plain form is unaffected. */
	TVG_CFG_QUADRUPOLE = 16
};

/* Host view of struct Particle_Data (src/Gravity/../particles.h:17-37). Any
 * pointer may be NULL when the matching field bit is not requested. */
typedef struct {
	int32_t *type;
	int32_t *time_bin;
	uint32_t *it_drift_pos;
	uint32_t *it_kick_pos;
	void *key;             /* peanoKey, 16 bytes per particle (little endian) */
	uint32_t *id;
	void *cost;
	void *pos[3];
	void *vel[3];
	void *acc[3];
	void *mass;
	void *grav_acc[3];
	void *last_acc_mag;
	int32_t *tree_parent;
	void *grav_pot;        /* Grav_Pot (TVG_CFG_POTENTIAL) */
} tvg_particles;

enum {
	TVG_F_TYPE = 1 << 0, TVG_F_TIME_BIN = 1 << 1, TVG_F_IT_DRIFT = 1 << 2,
	TVG_F_IT_KICK = 1 << 3, TVG_F_KEY = 1 << 4, TVG_F_ID = 1 << 5, TVG_F_COST = 1 << 6,
	TVG_F_POS = 1 << 7, TVG_F_VEL = 1 << 8, TVG_F_ACC = 1 << 9, TVG_F_MASS = 1 << 10,
	TVG_F_GRAV_ACC = 1 << 11, TVG_F_LAST_ACC = 1 << 12, TVG_F_TREE_PARENT = 1 << 13,
	TVG_F_ALL = (1 << 14) - 1,
	/* not in TVG_F_ALL: the reference has Grav_Pot only with GRAVITY_POTENTIAL */
	TVG_F_GRAV_POT = 1 << 14
};

/* Top node as dumped from union Domain_Node_List (src/domain.h:40-52). */
typedef struct {
	uint64_t key;
	int32_t target, level, first_part, npart;
	float pos[3], mass, com[3], dp[3];
} tvg_topnode;

/* ------------------------------------------------------------ lifecycle */

/* Creates a context on `device` and allocates device memory for
 * cfg->max_particles particles. Replaces the device side of
 * Allocate_Particle_Structures (src/particles.c:28) and Setup_Gravity_Tree
 * (src/Gravity/tree_build.c:124-142). */
int tvg_init(int device, const tvg_config *cfg, tvg_context **ctx);
void tvg_finalize(tvg_context *ctx);
const char *tvg_last_error(const tvg_context *ctx);
/* Library version string. */
const char *tvg_version(void);

/* Copies host particle fields (bitmask TVG_F_*) of n particles to the
 * device mirror; n becomes the active particle count (Task.Npart_Total). */
int tvg_upload(tvg_context *ctx, int64_t n, const tvg_particles *p, uint32_t fields);
/* Copies device fields back to the host arrays. */
int tvg_download(tvg_context *ctx, tvg_particles *p, uint32_t fields);

/* ------------------------------------------------ keys, sort, top nodes */

/* Domain.Origin / Domain.Size used by the keys (set_computational_domain,
 * src/domain.c:732-762). */
int tvg_set_domain(tvg_context *ctx, const double origin[3], double size);
/* set_computational_domain (domain.c:732-847) from the resident positions,
 * then tvg_set_domain with the result. Periodic: origin 0, size the box.
 * Isolated: centre = the median of each coordinate as the reference's Median
 * computes it (the (n >> 1)-th smallest of particles 1 .. n-1 in the current
 * order, kept in Float; select.c:19-107), size = 2.001 * the largest
 * |x - centre| over particles and axes (double), origin = centre - size / 2. */
int tvg_find_domain(tvg_context *ctx, double origin[3], double *size);

/* Replaces the Peano_Key loop of Sort_Particles_By_Peano_Key
 * (src/peano.c:27-30): P.Key = standard 128-bit key of P.Pos. */
int tvg_peano_keys(tvg_context *ctx);

/* Replaces Qsort_Index + reorder_collisionless_particles
 * (src/peano.c:32-35, src/sort.c:90-116, src/aux.c:187-301): sorts all
 * device particle fields by P.Key. Equal 128-bit keys keep input order. If
 * perm is not NULL it receives the index permutation (new i <- old perm[i]). */
int tvg_sort_particles(tvg_context *ctx, uint32_t *perm);

/* Replaces Reverse_Peano_Keys (src/peano.c:84-97): P.Key = reversed key. */
int tvg_reverse_keys(tvg_context *ctx);

/* Replaces the bunch loop of Domain_Decomposition (src/domain.c:67-145) and
 * transform_bunches_into_top_nodes (:220-250): the top nodes, in descending
 * key order, for the particles sorted by standard keys. With one target
 * (NTask = 1, the default, or NTask >= 65 on one rank, domain.c:151-156)
 * every non-empty level-2 cell; with NTask = 2 .. 64 targets (set by
 * tvg_set_domain_decomposition) the cells balanced by P.Cost as the
 * reference balances them over its threads. ntop receives the count. */
int tvg_top_nodes(tvg_context *ctx, int32_t *ntop);

/* NTask of Setup_Domain_Decomposition (src/domain.c:151-156; one rank: the
 * OpenMP threads of the reference's team), Param.Part_Alloc_Factor and
 * DOMAIN_IMBAL_CEIL (Config). The decomposition then weighs the particles by
 * cost_metric (domain.c:533-536: the integer part of max(1, P.Cost), P.Cost as
 * left by the last walk or uploaded with TVG_F_COST) and sums the costs as
 * the reference's threads do: each of NTask static shares of a range in
 * float, the shares added in thread order. Defaults: 1, 1.1, 0.05. */
int tvg_set_domain_decomposition(tvg_context *ctx, int32_t ntask, double part_alloc_factor,
                                 double imbal_ceil);
/* Refinement rounds of the last balanced decomposition. */
int tvg_decomposition_rounds(tvg_context *ctx, int32_t *rounds);

/* ----------------------------------------------------------- tree build */

enum {
	/* node Mass/CoM summed in particle order in Float, as the reference does
	 * (tree_build.c:561-572); otherwise in FP64 and rounded once. */
	TVG_BUILD_EXACT_MOMENTS = 1
};

/* Replaces Gravity_Tree_Build (src/Gravity/tree_build.c:47-122): builds the
 * subtree of every top node, the top nodes' Target/Mass/CoM and
 * P.Tree_Parent, on the device. */
int tvg_tree_build(tvg_context *ctx, uint32_t flags);

/* Copies the tree in the reference layout (struct Tree_Node, 56 B FP32 /
 * 96 B FP64, src/Gravity/tree.h:23-32) and the top nodes to the host. */
int tvg_download_tree(tvg_context *ctx, void *tree, int64_t tree_cap, int64_t *nnodes,
                      tvg_topnode *top, int32_t top_cap, int32_t *ntop);

/* ----------------------------------------------------------- tree walk */

enum {
	/* the reference algorithm, one thread per active particle, in Float */
	TVG_FORM_PLAIN = 0,
	/* one warp per PH group, FP32 on integer-offset positions */
	TVG_FORM_GROUP = 1
};
enum { TVG_WALK_GRAVITY = 1, TVG_WALK_EWALD = 2 };
enum { TVG_EWALD_TABLE = 0, TVG_EWALD_MLP = 1 };

/* Replaces Gravity_Periodic_Init (src/Gravity/periodic.c:180-233): the
 * 65^3 Ewald force (and potential) tables, computed in FP64 on the device and
 * stored as Float divided by Boxsize^2 (Boxsize). */
int tvg_ewald_init(tvg_context *ctx);
/* Copies the four raw (box-unit) Float tables Fx, Fy, Fz, Fp, in the layout of
 * the reference's ./ewald_tables.dat (Gravity/periodic.c:325-342). */
int tvg_download_ewald_table(tvg_context *ctx, void *fx, void *fy, void *fz, void *fp);

/* Loads raw (box-unit) Float tables as read from ./ewald_tables.dat
 * (read_ewald_correction_table, Gravity/periodic.c:303-323) instead of
 * computing them, then divides by Boxsize^2 / Boxsize as the reference does. */
int tvg_upload_ewald_table(tvg_context *ctx, const void *fx, const void *fy, const void *fz,
                           const void *fp);

/* Replaces Gravity_Tree_Acceleration (src/Gravity/tree_accel.c:32-91) and,
 * with TVG_WALK_EWALD, Gravity_Tree_Periodic (src/Gravity/tree_periodic.c:
 * 23-72), for the active particles: Acc += walk, Grav_Acc = walk (gravity
 * part) / Grav_Acc += walk (Ewald part), Cost = / += interaction count. The
 * criterion is Barnes & Hut when use_bh != 0 (Sig.Use_BH_Criterion), else the
 * relative criterion with P.Last_Acc_Mag. */
int tvg_walk(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts, int32_t ewald_kind);

/* accel.c:28-43 (safe_last_accel): Last_Acc_Mag = |Acc|, Acc = 0. */
int tvg_save_last_accel(tvg_context *ctx);

/* Zero Acc, Grav_Acc and Cost of all particles. */
int tvg_zero_accel(tvg_context *ctx);

/* ---------------------------------------------------- whole force step */

/* One tree-force evaluation on device-resident particles: keys, sort,
 * top nodes, tree build and the walk(s) of `parts` (accel.c:51-71 without
 * the BH prepare pass when use_bh == 0). */
int tvg_force_step(tvg_context *ctx, int32_t form, int32_t use_bh, uint32_t parts,
                   int32_t ewald_kind);

/* tvg_force_step end to end from host buffers, for a host code whose
 * particles live in host memory (the reference's P, Gravity_Tree_Acceleration
 * after Domain_Decomposition, accel.c:15-71): uploads the `in_fields` of n
 * particles (positions required), runs the same keys, sort, top nodes, build
 * and walks, and downloads the `out_fields` (in the new PH order, like the
 * reference's reordered P). The copies overlap the kernels: the positions go
 * first, the other inputs while the keys and radix passes run (the field
 * gather waits for them), and outputs that the walks do not write (ID, ...)
 * while the walks run. Returns when `out` holds the results. Page-locked
 * host memory (tvg_host_alloc / tvg_host_register) gives full copy speed. */
int tvg_force_step_host(tvg_context *ctx, int64_t n, const tvg_particles *in, uint32_t in_fields,
                        tvg_particles *out, uint32_t out_fields, int32_t form, int32_t use_bh,
                        uint32_t parts, int32_t ewald_kind);

/* Active_Particle_List / NActive_Particles (src/timestep.c:280-299): the walks
 * compute forces for these particles only (indices into the current, sorted
 * order, ascending). NULL selects all particles. Sorting resets it to all. */
int tvg_set_active(tvg_context *ctx, const int32_t *list, int64_t n_active);

/* Per-phase device times (ms) of the last calls, CUDA events on the
 * context stream: [keys, sort, top, build, walk, ewald walk, total]. */
int tvg_phase_times(tvg_context *ctx, double *ms, int32_t n);

/* Device-timed region on the context stream: stop = 0 records the start
 * event, stop = 1 records the end event, waits for it and returns the
 * elapsed milliseconds in *ms. */
int tvg_timer(tvg_context *ctx, int32_t stop, double *ms);

/* Number of kernels this context has launched since it was created. */
int tvg_launch_count(tvg_context *ctx, int64_t *count);

/* Page-locked host memory for transfers that overlap with device work. */
int tvg_host_alloc(size_t bytes, void **ptr);
int tvg_host_free(void *ptr);
/* Page-locks an existing host range (cudaHostRegister), so that uploads from
 * and downloads into it run as direct transfers: the reference's memory pool
 * (`Memory`, posix_memalign in Init_Memory_Management, memory.c:209), which
 * holds P, is registered once after it is allocated and unregistered before
 * it is freed. TVG_E_BADINPUT for a NULL or empty range, TVG_E_STATE when
 * (part of) the range is registered already, TVG_E_CUDA otherwise. */
int tvg_host_register(void *ptr, size_t bytes);
int tvg_host_unregister(void *ptr);

/* Measured FP32 FFMA throughput of the device (TFLOP/s, FMA = 2 flop) over
 * `ms_target` milliseconds: the denominator of the walk's roofline. */
int tvg_fp32_peak(tvg_context *ctx, double ms_target, double *tflops);

/* ---------------------------------------------- sort without allocation */

/* Largest n accepted by tvg_sort_keys_noalloc. */
#define TVG_NOALLOC_MAX_KEYS (1 << 18)

/* This entry point has no counterpart in the reference. It is the PH-key
 * sort of tvg_sort_particles for callers that cannot allocate device memory:
 * a host code whose own memory manager reserves the GPU's memory up front and
 * admits no allocation behind its back (as the reference reserves its whole
 * host pool once), or a step loop that cannot take the device-wide
 * synchronisation that cudaMalloc and cudaFree imply. It needs no context.
 *
 * key_hi, key_lo: n 128-bit keys (high and low 64-bit words), device memory;
 * perm: n uint32, device memory, receives the permutation that orders the
 * keys ascending (perm[i] = input index of the i-th smallest key; equal keys
 * keep input order) -- the same permutation tvg_sort_particles returns.
 * Runs on the calling thread's current device, on the legacy default stream
 * (stream 0), and synchronises that stream before it returns, so the result
 * is in perm on return.
 *
 * Its scratch (about 6.4 MB) is one statically sized device array that every
 * GPU loading this library holds until the process exits; nothing is
 * allocated or freed by a call. The first call on each device looks up that
 * array's device address (cudaGetSymbolAddress), so make that first call
 * before any stream capture begins. All calls on a device share the array,
 * which keeps the last call's contents; calls that overlap on the same GPU
 * (from several host threads) race and give wrong results.
 * Returns TVG_E_BADINPUT for n < 0 or n > TVG_NOALLOC_MAX_KEYS, TVG_E_CUDA
 * on a CUDA error. */
int tvg_sort_keys_noalloc(const uint64_t *key_hi, const uint64_t *key_lo, int64_t n, uint32_t *perm);

/* Counters of the last walk: total gravity and Ewald interactions. */
int tvg_walk_counters(tvg_context *ctx, double *grav_interactions, double *ewald_interactions);
/* Of the last group walk's gravity interactions, those with a node's
 * quadrupole (TVG_CFG_QUADRUPOLE; 0 otherwise). No reference counterpart. */
int tvg_walk_quad_interactions(tvg_context *ctx, double *quad_interactions);

/* Largest n_targets accepted by tvg_forcetest. */
#define TVG_FORCETEST_MAX_TARGETS (1 << 20)

/* Replaces Gravity_Forcetest (Gravity/forcetest.c:25-172), which checks
 * NTEST = 10 random active particles on the host: FP64 direct summation over
 * all resident particles for n_targets targets (indices into the current,
 * i.e. PH-sorted, particle order), with the reference's softened kernel on
 * the nearest image; with TVG_WALK_EWALD in parts (periodic box) the periodic
 * images are Ewald-summed (alpha L = 12, real space on the nearest image,
 * k space |h|^2 <= 576). parts must include TVG_WALK_GRAVITY. Outputs, each optional:
 * acc_direct and acc_tree (3 * n_targets doubles, x block then y then z) hold
 * the direct sum and the resident Grav_Acc; err[4] = rms, 99th percentile
 * (nearest rank), mean and max of |a_tree - a_direct| / |a_direct|.
 * Allocates and frees its own device scratch. */
int tvg_forcetest(tvg_context *ctx, uint32_t parts, int64_t n_targets, const int64_t *targets,
                  double *acc_direct, double *acc_tree, double *err);

/* Sets the opening parameters (the reference's compile-time constants
 * TREE_OPEN_PARAM_BH, used as theta^2, and TREE_OPEN_PARAM_REL) for the
 * following walks; no reference counterpart. Values must be > 0. */
int tvg_set_opening(tvg_context *ctx, double open_bh, double open_rel);

/* Opening of the group form's Ewald walk (no reference counterpart): a node
 * is opened for the Ewald correction when the monopole error of the
 * correction, G M h2 s^2 / (8 L^4) (h2: bound of its second derivatives in
 * box units), exceeds rel_alpha |a_old| (relative mode), or when
 * h2 s^2 / L^2 exceeds bh_factor times TREE_OPEN_PARAM_BH (Barnes-Hut mode).
 * Defaults 2.5e-4 and 0.5. */
int tvg_set_ewald_opening(tvg_context *ctx, double rel_alpha, double bh_factor);

/* Iteration limit of the group form's traversal loops (no reference
 * counterpart; the reference's walks run unbounded, tree_accel.c:211-353):
 * a warp that pops more than `max_iterations` node batches for one group
 * stops, and the walk returns TVG_E_TIMEOUT with the context still usable.
 * Default 2^24, far above any walk (a group pops at most a few 10^4
 * batches). Accepts 1 .. 2^31 - 1. */
int tvg_set_walk_limit(tvg_context *ctx, int64_t max_iterations);

/* ------------------------------------------- hierarchical time stepping */

/* Parameters of the timeline and background cosmology that the kick, drift
 * and time-step code reads (Time.Begin/End, Cosmo, Param; src/timestep.c,
 * src/cosmology.c, src/comoving.c). */
typedef struct {
	int32_t comoving;          /* COMOVING: time is the expansion factor a */
	double time_begin;         /* Time.Begin */
	double time_end;           /* Time.End */
	double hubble_constant;    /* Cosmo.Hubble_Constant (code units: 0.1 for km/s/kpc) */
	double omega_matter;       /* Cosmo.Omega_Matter */
	double omega_lambda;       /* Cosmo.Omega_Lambda */
	double omega_rad;          /* Cosmo.Omega_Rad */
	double omega_0;            /* Cosmo.Omega_0 = Omega_Matter + Omega_Lambda + OMEGA_RAD */
	double omega_baryon;       /* Cosmo.Omega_Baryon */
	double rho_crit0;          /* Cosmo.Rho_Crit0 (code units) */
	double time_int_accuracy;  /* Param.Time_Int_Accuracy */
	double max_timestep;       /* Param.Max_Timestep */
	double displ_constraint;   /* TIME_DISPL_CONSTRAINT (Config) */
} tvg_timeline_config;

/* struct IntegerTimeLine Int_Time, the parts of struct TimeData Time and of
 * Cosmo that change, and the step signals (src/timestep.h:24-32,
 * src/signal.h). */
typedef struct {
	uint32_t beg, current, next, end, step, next_sync_point;   /* Int_Time */
	double time_current, time_next, time_step;                 /* Time.Current/Next/Step */
	double step_max, step_min;                                 /* Time.Step_Max/Min */
	double expansion_factor, hubble_parameter;                 /* Cosmo (Set_Current_Cosmology) */
	float dt_max_global;                                       /* Dt_Max_Global */
	int32_t max_active_bin;                                    /* Time.Max_Active_Bin */
	int32_t time_bin_min, time_bin_max;
	int32_t sync_point, first_step, prepare_step;              /* Sig */
	int64_t n_active;                                          /* NActive_Particles */
	int64_t step_counter;                                      /* Time.Step_Counter */
} tvg_timeline_state;

/* Setup_Time_Integration (timestep.c:108-178) and setup_kick_drift_factors
 * (comoving.c:109-153): the integer timeline, and with COMOVING the 512-knot
 * kick/drift factor tables (FP64 quadrature on the device, natural cubic
 * spline; knot 0 at a = 0 as in the reference). All particles start active. */
int tvg_timeline_init(tvg_context *ctx, const tvg_timeline_config *cfg);
/* The 512 knots a_i and the tabulated kick and drift integrals (comoving). */
int tvg_download_kick_drift_table(tvg_context *ctx, double *a, double *kick, double *drift);
/* Particle_Kick_Step / Particle_Drift_Step (comoving.c:30-50, kick.c:78-84,
 * drift.c:115-121) for two points of the integer timeline. */
int tvg_kick_drift_factors(tvg_context *ctx, uint32_t it_curr, uint32_t it_next, double *kick,
                           double *drift);
/* Set_New_Timesteps (timestep.c:35-89): new time bins of all particles from
 * |Grav_Acc| (set_new_particle_timebins, timestep.c:200-236), the system step
 * and the Active_Particle_List of the next step, kept on the device. */
int tvg_set_new_timesteps(tvg_context *ctx);
/* Kick_First_Halfstep / Kick_Second_Halfstep (kick.c:9-70) over the active
 * particles; the second also ends the step (Sig.First_Step = false, as
 * Update(AFTER_STEP) does). After tvg_time_for_domain_update, and while no
 * domain update is due, each kick also adds the particles' momentum to the
 * kept tree (Gravity_Tree_Update_Kicks, tree_update.c:12-54): Dp of every
 * node above them and of their top node, summed in particle order. */
int tvg_kick_first_halfstep(tvg_context *ctx);
int tvg_kick_second_halfstep(tvg_context *ctx);
/* Drift_To_Sync_Point (drift.c:12-62): drifts the active particles to
 * Int_Time.Next, wraps all particles into the box, advances the clock; with
 * tree updates and no domain update due, moves the kicked nodes by
 * Time.Step * Dp (Gravity_Tree_Update_Drift, tree_update.c:62-101). */
int tvg_drift_to_sync_point(tvg_context *ctx);
/* Time_For_Domain_Update (signal.c:85-116): adds NActive_Particles to the
 * particle updates since the last domain decomposition; a decomposition (and
 * a new tree) is due at a sync point or when they exceed
 * domain_update_param * N (DOMAIN_UPDATE_PARAM, 0.1 in the reference's
 * Config). *domain_update receives Sig.Domain_Update. The first call turns on
 * the reference's tree updates between rebuilds for this context: until a
 * due update, the kicks and the drift update the kept tree and
 * tvg_compute_acceleration / tvg_step_graph walk it without keys, sort or
 * build. A context that never calls it rebuilds at every force computation.
 * The node sums follow the particle order, which is the order of the
 * Active_Particle_List that Set_New_Timesteps makes. */
int tvg_time_for_domain_update(tvg_context *ctx, double domain_update_param, int32_t *domain_update);
/* Reads / replaces the timeline state (e.g. to restart). */
int tvg_timeline_get(tvg_context *ctx, tvg_timeline_state *st);
int tvg_timeline_set(tvg_context *ctx, const tvg_timeline_state *st);
/* Number of particles in each of the 32 time bins. */
int tvg_rung_histogram(tvg_context *ctx, int32_t *hist);
/* Compute_Acceleration (accel.c:15-71) with the domain decomposition of the
 * single-rank reference: keys, sort (Sort_Particles_By_Peano_Key rebuilds
 * the Active_Particle_List, peano.c:42), top nodes, tree build, then for the
 * active particles safe_last_accel (Last_Acc_Mag = |Acc|, Acc = 0), with
 * prepare (Sig.Prepare_Step) a Barnes-Hut walk and safe_last_accel again, and
 * the relative-criterion walk. Without a timeline every particle is active.
 * With tree updates (tvg_time_for_domain_update) and no domain update due,
 * the walks run on the kept, updated tree (accel.c:53). */
int tvg_compute_acceleration(tvg_context *ctx, int32_t form, uint32_t parts, int32_t ewald_kind,
                             int32_t prepare);
/* tvg_compute_acceleration of the group form (prepare = 0) with the step's
 * whole launch sequence as one CUDA graph (no host round trip inside: the
 * counts of the step stay on the device). The first call with a given
 * configuration (parts, ewald_kind, group size, timeline, particle count)
 * runs the step directly; later calls capture it once for each of the two
 * buffer states the sort alternates between, then launch the captured graph.
 * The timeline's active-bin limit is passed to the device before each launch.
 * Results, phase times and counters as tvg_compute_acceleration. */
int tvg_step_graph(tvg_context *ctx, uint32_t parts, int32_t ewald_kind);
/* Releases the captured step graphs (tvg_finalize does too). */
int tvg_step_graph_reset(tvg_context *ctx);

/* Autotuner of the group form (no reference counterpart): on the current tree
 * and active set, times the gravity + Ewald walks with 32-, 64- and
 * 128-particle groups (one, two or four targets per lane) over a sample --
 * the active particles in every 8th window of 128 particles -- and keeps the
 * fastest for the later walks of this context. choice receives 1, 2 or 4,
 * ms[3] the three sample times. The chosen walk then runs over the whole
 * active set: Acc, Grav_Acc and Cost are left as that one walk leaves them
 * (Acc as it was plus the walk's contribution). */
int tvg_autotune(tvg_context *ctx, int32_t use_bh, uint32_t parts, int32_t ewald_kind,
                 int32_t *choice, double *ms);

/* ---------------------------------------------- learned Ewald correction */

/* Training of the 3 -> 64 -> 64 -> 3 network (tanh) that stands in for the
 * Ewald table interpolation (no reference counterpart): n_samples points
 * uniform on the folded octant with FP64 Ewald-sum targets, Adam over
 * minibatches of `batch`, cosine learning-rate decay from lr to lr_final.
 * resume != 0 continues from the current weights. */
typedef struct {
	int32_t steps;
	int32_t batch;
	int64_t n_samples;
	float lr, lr_final;
	uint64_t seed;
	int32_t resume;
} tvg_mlp_train_config;

/* Number of parameters (float): the 3-64-64-3 network (4611, trained), then
 * the cubic fit of the correction's smooth part (3 x 20) and the network's
 * output scale (fitted). The model is T(x) = 4 pi x / 3 + S(x) + C . m(4x-1)
 * + s N(4x-1), S the seven lattice images nearest to the octant. */
#define TVG_MLP_NPARAM 4672

/* Trains on the device (fits C and s first unless resume != 0);
 * final_loss = mean square error per component of T (box units) with the
 * FP32 weights over all samples. Leaves the weights unvalidated (see
 * tvg_ewald_mlp_validate). */
int tvg_ewald_mlp_train(tvg_context *ctx, const tvg_mlp_train_config *cfg, float *final_loss);
/* Copies the FP32 parameters out (set = 0) or in (set != 0). */
int tvg_ewald_mlp_weights(tvg_context *ctx, float *params, int32_t set);
/* Gradient of the network's mean-square loss over n samples x[3n] (octant,
 * box units) with targets y[3n] for N (what the rest of the model leaves,
 * divided by s), from the training kernels; the fitted entries get 0. */
int tvg_ewald_mlp_grad(tvg_context *ctx, int64_t n, const float *x, const float *y, float *grad,
                       float *loss);
/* T(x) at n octant points x[3n] (box units) from the BF16 weights. */
int tvg_ewald_mlp_eval(tvg_context *ctx, int64_t n, const double *x, double *t);
/* The exact FP64 table (tvg_ewald_init) validates the BF16 network at its 65^3
 * nodes: max and rms |T_mlp - T|; the walk accepts TVG_EWALD_MLP only while
 * the max error is at most max_allowed. */
int tvg_ewald_mlp_validate(tvg_context *ctx, double max_allowed, double *max_err, double *rms_err);

/* ---------------------------------------------------------- snapshots */

/* Header of a Gadget format-2 snapshot (struct gadget_header, IO/io.h:24-44):
 * particles per type in this file and in the simulation, mass per type (0:
 * the MASS block holds it), Time, Redshift (the reference writes
 * 1/Time - 1 with COMOVING), the number of files, and the box and cosmology
 * constants. */
typedef struct {
	uint32_t npart[6];
	uint64_t nall[6];
	double massarr[6];
	double time;
	double redshift;
	int32_t num_files;
	double boxsize, omega0, omega_lambda, hubble_param;
} tvg_snapshot_header;

/* Optional blocks after POS, VEL, ID, MASS (IO/io.h:69-84). */
enum {
	TVG_SNAP_ACC = 1,      /* "ACC ": one component, Acc[0], as the reference's table declares */
	TVG_SNAP_GACC = 2,     /* "GACC": Grav_Acc[3] (OUTPUT_PARTIAL_ACCELERATIONS) */
	TVG_SNAP_GPOT = 4,     /* "GPOT": Grav_Pot (OUTPUT_GRAV_POTENTIAL) */
	TVG_SNAP_MASS = 8      /* reading: the MASS block was present */
};

/* Write_Snapshot (IO/write_snapshot.c:13-328) for one rank and one file:
 * the header and the blocks in the reference's format (4-byte Fortran record
 * markers, format-2 label records, 32-bit IDs, fields interleaved per
 * particle) of the n particles in the host arrays of p (Float of
 * float_bytes). The header's 64 fill and padding bytes are written as zero. */
int tvg_write_snapshot_host(const char *path, const tvg_snapshot_header *header, int64_t n,
                            int32_t float_bytes, const tvg_particles *p, uint32_t blocks);
/* The same for the context's particles, downloaded from the device in their
 * current order (PH order after a sort, as the reference writes them). */
int tvg_write_snapshot(tvg_context *ctx, const char *path, const tvg_snapshot_header *header,
                       uint32_t blocks);
/* read_header_data (IO/read_snapshot.c:313-402): the header of the snapshot
 * `path`, or of `path.0` when the snapshot is split into files path.0,
 * path.1, ... (find_files, :544-575); *num_files receives their number.
 * Files of either byte order are read. */
int tvg_read_snapshot_header(const char *path, tvg_snapshot_header *header, int32_t *num_files);
/* Read_Snapshot (IO/read_snapshot.c:19-123) for one rank: the particles of
 * all files into the host arrays of p (cap entries each, Float of
 * float_bytes; IDs 32-bit). POS, VEL and ID are required; MASS, ACC
 * (component 0), GACC and GPOT are read when present and p has the array.
 * As the reference stores them (Reallocate_P): one section per type in
 * increasing type order, each in file order. Masses come from the header's
 * Massarr of the type's section when any Massarr is nonzero
 * (generate_masses_from_header, :412-437), else from the MASS block; p->type
 * from the ID ranges of the header's per-type totals (set_particle_types,
 * :444-474), or the section's type where no range holds the ID (the
 * reference leaves it unset). *n receives the particle count, *blocks the
 * TVG_SNAP_* bits of the optional blocks found in every file. A block whose
 * size disagrees with the file's particle count and the Float width, a
 * missing required block or n > cap are TVG_E_BADINPUT. */
int tvg_read_snapshot_host(const char *path, int32_t float_bytes, int64_t cap, tvg_particles *p,
                           int64_t *n, uint32_t *blocks);
/* tvg_read_snapshot_host into host staging, then tvg_upload of Pos, Vel, ID,
 * Mass, Type and the optional fields found (Acc with Acc[0] from the ACC
 * block, Grav_Acc, Grav_Pot) to the context. */
int tvg_read_snapshot(tvg_context *ctx, const char *path, int64_t *n, uint32_t *blocks);

#ifdef __cplusplus
}
#endif
#endif
