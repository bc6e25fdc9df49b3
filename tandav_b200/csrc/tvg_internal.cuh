// tvg_internal.cuh -- shared definitions of the B200 gravity hot path.
//
// Device data layout (HBM, all arrays structure-of-arrays, capacity `cap`):
//   particle fields mirror struct Particle_Data (particles.h:17-37) in the
//   host's Float width, each with a second "alt" buffer so that the PH
//   permutation is a gather into alt followed by a pointer swap;
//   keys are split into key_hi / key_lo (uint64) for the radix sort;
//   the tree is kept twice: in the reference layout (struct Tree_Node, for
//   download and the plain walk) and, for the group walk, as level-ordered
//   node records with integer (box-fraction) coordinates.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/tandav_gpu.h"

// top nodes: 64 level-2 cells on one target; up to 512 + 20 rounds x 64
// splits x 7 when Domain_Decomposition balances 64 targets
#define TVG_MAX_TOP 16384
#define TVG_MAX_DEVICES 64         // per-device caches of launch attributes
#define TVG_MAX_LEVEL 42

// ---------------------------------------------------------------- errors

#define TVG_CUDA(ctx, call)                                                        \
	do {                                                                           \
		cudaError_t e_ = (call);                                                   \
		if (e_ != cudaSuccess)                                                     \
			return tvg_fail((ctx), TVG_E_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,  \
			                #call, cudaGetErrorString(e_));                         \
	} while (0)

// wraps the grid argument of every kernel launch: counts the launch
#define TVG_CNT(ctx, grid) ((ctx)->launches++, (grid))

#define TVG_CHECK(expr)                                                            \
	do {                                                                           \
		int rc_ = (expr);                                                          \
		if (rc_ != TVG_OK) return rc_;                                             \
	} while (0)

// device status word bits (written by kernels, read by the host after a phase)
enum {
	TVG_ST_COINCIDENT = 1,
	TVG_ST_BADPOS = 2,
	TVG_ST_TREE_FULL = 4,
	TVG_ST_TIMEOUT = 8,
	TVG_ST_LIST_OVERFLOW = 16,
	TVG_ST_TIMESTEP = 32,
	TVG_ST_TREE_STALE = 64,    // a kept tree's ranges do not fit the particles
	TVG_ST_OFF_GRID = 128      // group form: a position off its integer grid
};

struct tvg_buf {
	void *p = nullptr;
	size_t bytes = 0;
};

// Walk node record of the group walk (level-ordered tree, 48 bytes).
struct __align__(16) tvg_wnode {
	uint32_t cx, cy, cz;    // centre of mass, integer box coordinates
	float mass;
	uint32_t gx, gy, gz;    // geometric centre (reference Tree.Pos), integer coords
	float size;             // node size (box units scaled to length)
	int32_t child;          // first child (walk index) or first particle
	int32_t nchild;         // > 0: children; < 0: -(number of particles) of a bundle
	float size2;            // size^2
	int32_t level;
};

// Counts of the current step kept on the device: the kernels of a step read
// them, so a step needs no host round trip between its phases and can be
// captured as one CUDA graph (tvg_step_graph). The host reads them back once,
// after the step.
struct tvg_devcount {
	int64_t nu;              // uncollapsed nodes of the build
	int64_t nnodes;          // tree nodes, terminators included
	int64_t n_active;        // active particles
	int64_t ngroups;         // groups of the group walk
	double mass_total;       // sum of the masses (Ewald uniform remainder)
	int32_t ntop;            // top nodes
	int32_t max_active_bin;  // bins <= this are active
	int32_t sort_skip[8];    // radix digit d is the same for all keys
	int64_t nwchild;         // walk nodes below the top nodes (TVG_CFG_QUADRUPOLE)
};

// Per top node tables of the tree build, on the device (TVG_MAX_TOP
// entries each, one allocation): the subtree's first node and node count,
// the offset from a node's rank among the build's survivors to its tree
// index, and the first particle after the top node.
struct TopTables {
	int32_t *target;
	int32_t *nsurv;
	int32_t *toff;
	int32_t *end;
};


struct tvg_graph_entry;

// field slots in ctx->f[]
enum {
	FS_TYPE = 0, FS_TIME_BIN, FS_IT_DRIFT, FS_IT_KICK, FS_ID, FS_COST,
	FS_POS0, FS_POS1, FS_POS2, FS_VEL0, FS_VEL1, FS_VEL2,
	FS_ACC0, FS_ACC1, FS_ACC2, FS_MASS, FS_GACC0, FS_GACC1, FS_GACC2,
	FS_LAST_ACC, FS_TREE_PARENT, FS_GRAV_POT, FS_NFIELDS
};

struct tvg_context {
	int device = 0;
	tvg_config cfg{};
	cudaStream_t stream = nullptr;
	// tvg_force_step_host: copies that overlap the step's kernels, and the
	// events that order them against the context stream (created on first use)
	cudaStream_t copy_stream = nullptr;
	cudaEvent_t xev[3] = { nullptr, nullptr, nullptr };
	// when set, the sort's field gather waits for this event (inputs still
	// uploading on copy_stream)
	cudaEvent_t gather_wait = nullptr;
	int64_t cap = 0;          // particle capacity
	int64_t n = 0;            // active particle count
	double origin[3] = { 0, 0, 0 };
	double dsize = 0;         // Domain.Size
	bool have_domain = false;
	bool keys_std = false;    // key holds standard keys
	bool sorted = false;
	bool have_top = false;
	bool have_tree = false;
	bool have_ewald = false;
	bool have_walktree = false;
	char err[512] = { 0 };

	// particle fields (two buffers each for the permutation)
	void *f[FS_NFIELDS] = { nullptr };
	void *falt[FS_NFIELDS] = { nullptr };
	// key split for the sort
	uint64_t *key_hi = nullptr, *key_lo = nullptr, *key_tmp = nullptr;
	uint32_t *perm = nullptr, *perm_tmp = nullptr;
	uint32_t *sort_hist = nullptr;     // per-tile digit histograms
	uint32_t *sort_off = nullptr;      // scanned
	uint32_t *digit_count = nullptr;   // 8 x 256 global digit histogram
	void *scan_tmp = nullptr;
	size_t scan_tmp_bytes = 0;
	int *status = nullptr;             // device status word
	int *h_status = nullptr;           // pinned mirror

	// top nodes
	int32_t ntop = 0;
	tvg_topnode *d_top = nullptr;
	tvg_topnode h_top[TVG_MAX_TOP];
	int32_t *top_first = nullptr;      // [64] first particle of level-2 cell c
	int32_t *top_count = nullptr;      // [64]
	int32_t *top_of = nullptr;         // top node of every particle (cap)
	// Domain_Decomposition balanced over NTask targets (tvg_set_domain_decomposition)
	int32_t dd_ntask = 1;
	double dd_part_alloc_factor = 1.1; // Param.Part_Alloc_Factor
	double dd_imbal_ceil = 0.05;       // DOMAIN_IMBAL_CEIL
	void *dd_scratch = nullptr;        // fill jobs, bunch keys and partial sums
	int32_t dd_rounds = 0;             // refinement rounds of the last decomposition

	// tree build scratch
	uint8_t *lvl = nullptr;            // LCA level with the previous particle
	int32_t *ncnt = nullptr;           // nodes starting at each particle; then scan
	uint8_t *lvl_min64 = nullptr;      // min of lvl over 64-blocks
	int64_t ucap = 0;                  // capacity of uncollapsed node arrays
	int32_t *u_start = nullptr, *u_count = nullptr, *u_endu = nullptr, *u_diff = nullptr;
	int32_t *u_final = nullptr;
	uint8_t *u_level = nullptr, *u_flag = nullptr;
	int64_t nu = 0;                    // uncollapsed node count
	// final tree
	int64_t tcap = 0;                  // node capacity
	int64_t nnodes = 0;
	void *tree = nullptr;              // reference layout
	int32_t *tree_u = nullptr;         // final node -> uncollapsed index
	double *pref = nullptr;            // prefix sums of m, m*x, m*y, m*z (FP64)


	// Ewald tables (Float, divided by box^2) and raw FP64
	void *ewald_f[4] = { nullptr, nullptr, nullptr, nullptr };
	double *ewald_raw = nullptr;
	float *ewald32 = nullptr;          // FP32 copy for the group form (FP64 builds)
	float *ewald_ext = nullptr;        // (Tx, Ty, Tz, 0) on 68^3 points, x = 0.5 i / 64, i = -1..66
	float *ewald_taylor = nullptr;     // T and 3 derivatives at TVG_TAYLOR_NODES^3 nodes, 64 floats each
	// Ewald-walk opening of the group form: the monopole error of the
	// correction may reach ewald_open_rel |a_old| (relative mode); the limit of
	// h2 s^2 / L^2 in units of TREE_OPEN_PARAM_BH (Barnes-Hut mode)
	double ewald_open_rel = 2.5e-4;
	double ewald_open_bh = 0.5;
	// iteration limit of the group walks' traversal loops (tvg_set_walk_limit)
	int32_t walk_limit = 1 << 24;

	// group walk data
	uint32_t *ipos[3] = { nullptr, nullptr, nullptr };
	tvg_wnode *wtree = nullptr;
	float4 *wquad = nullptr;           // TVG_CFG_QUADRUPOLE: G Q of every walk node, 2 float4
	int32_t *wrange = nullptr;         // first particle and count of every walk node (2 int32)
	int64_t nw = 0;
	int32_t *group_first = nullptr;
	int64_t ngroups = 0;
	int32_t *work_counter = nullptr;
	double *counters = nullptr;        // device interaction counters [4]

	// active particles (Active_Particle_List); all particles when !use_active
	int32_t *active = nullptr;
	int32_t *tune_active = nullptr;    // the autotuner's sample of the active set
	int64_t n_active = 0;
	bool use_active = false;
	int64_t launches = 0;              // kernels launched by this context
	int group_tpl = 0;                 // group form targets per lane (0: default)

	// learned Ewald correction (tvg_ewald_mlp.cu)
	float *mlp_prm = nullptr;          // FP32 parameters (4611)
	void *mlp_bf16 = nullptr;          // BF16 copy used for inference
	bool have_mlp = false, mlp_ok = false;
	double mlp_max_err = 0;

	// hierarchical time integration (tvg_integrate.cu)
	bool have_timeline = false;
	struct {
		tvg_timeline_config cfg;
		tvg_timeline_state state;
	} tl{};
	double *kd_x = nullptr, *kd_kick = nullptr, *kd_drift = nullptr;   // 512 knots
	double *kd_m2k = nullptr, *kd_m2d = nullptr, *kd_work = nullptr;   // spline second derivatives
	void *tl_scratch = nullptr;        // reductions (256 B)
	int32_t *act_flag = nullptr, *act_off = nullptr;

	// tree updates between rebuilds (tvg_tree_update.cu)
	bool tree_updates = false;         // tvg_time_for_domain_update has been called
	bool domain_update = true;         // Sig.Domain_Update (= Sig.Tree_Update)
	int64_t npart_updates = 0;         // Local_NPart_Updates (signal.c:80)
	int32_t *tu_first = nullptr;       // first particle of every tree node
	int32_t *tu_big = nullptr;         // [0]: count, then the nodes the node kick leaves to a warp each
	int32_t *big_list = nullptr;       // [0]: count, then the nodes whose moments a block each sums
	void *tu_dp = nullptr;             // dp of the active particles by slot, 3 x cap Float

	// device-resident counts and top-node tables of the step
	tvg_devcount *dc = nullptr;
	int32_t *d_toptab = nullptr;       // TopTables storage: 4 x TVG_MAX_TOP
	// stream capture in progress: the step's functions skip every host read
	// and synchronisation
	bool capturing = false;
	// CUDA graphs of the step (tvg_step.cu): one per buffer parity
	tvg_graph_entry *graphs[2] = { nullptr, nullptr };
	uint64_t graph_warm_key = 0;

	// timings
	cudaEvent_t ev[16];
	double phase_ms[8] = { 0 };
	double last_counts[3] = { 0, 0, 0 };   // gravity, Ewald, of the gravity ones quadrupole
};


int tvg_fail(tvg_context *ctx, int code, const char *fmt, ...);
int tvg_sync_status(tvg_context *ctx, const char *phase);
int tvg_device_scan_i32(tvg_context *ctx, const int32_t *in, int32_t *out, int64_t n,
                        int64_t *total);
// as tvg_device_scan_i32, the total written to device memory (no host read)
int tvg_device_scan_i32_dev(tvg_context *ctx, const int32_t *in, int32_t *out, int64_t n,
                            int64_t *total_dev);
// reads the device counts back into the host mirrors (top nodes, node
// counts); synchronises the stream
int tvg_read_counts(tvg_context *ctx);
// times and interaction counts of the last group walk (synchronises)
int tvg_walk_group_results(tvg_context *ctx);
// the active-bin limit of the timeline into the device counts
int tvg_set_device_max_bin(tvg_context *ctx);
void tvg_graph_release(tvg_context *ctx);
// tree updates between rebuilds (tvg_tree_update.cu): due when the context
// follows Time_For_Domain_Update and no domain update is due
bool tvg_tree_update_due(const tvg_context *ctx);
int tvg_tree_update_check(tvg_context *ctx, const char *what);
// active flags and their exclusive scan (act_flag, act_off) for the current
// active set, in particle order; *na = its size
int tvg_impl_active_slots(tvg_context *ctx, int64_t *na);
int tvg_impl_tree_dp_buffer(tvg_context *ctx, void **dp);
int tvg_impl_tree_kick(tvg_context *ctx, int64_t na);
int tvg_impl_tree_drift(tvg_context *ctx, double dt);

// phase implementations (one translation unit each)
int tvg_impl_keys(tvg_context *ctx, bool reversed);
int tvg_impl_sort(tvg_context *ctx, uint32_t *perm_out);
int tvg_impl_top_nodes(tvg_context *ctx);
// Domain_Decomposition's cost-driven top nodes for NTask > 1 (tvg_decompose.cu)
int tvg_impl_top_nodes_balanced(tvg_context *ctx);
// the top node of every particle (top_of) from the device top-node list
int tvg_impl_top_of(tvg_context *ctx);
int tvg_impl_tree_build(tvg_context *ctx, uint32_t flags);
int tvg_impl_download_tree(tvg_context *ctx, void *tree, int64_t cap, int64_t *nnodes);
int tvg_impl_ewald_init(tvg_context *ctx);
int tvg_impl_ewald_ext(tvg_context *ctx);
int tvg_impl_ewald_taylor(tvg_context *ctx);
// nodes per axis of the group form's Taylor table of the Ewald correction
#ifndef TVG_TAYLOR_NODES
#define TVG_TAYLOR_NODES 33
#endif
int tvg_impl_walk_plain(tvg_context *ctx, int use_bh, uint32_t parts);
int tvg_impl_walk_group(tvg_context *ctx, int use_bh, uint32_t parts, int ewald_kind);
int tvg_impl_save_last_accel(tvg_context *ctx);
int tvg_impl_zero_accel(tvg_context *ctx);
int tvg_impl_active_from_bins(tvg_context *ctx);

static inline size_t tvg_fsize(const tvg_context *ctx) { return (size_t) ctx->cfg.float_bytes; }

static inline TopTables tvg_top_tables(const tvg_context *ctx)
{
	TopTables t;
	t.target = ctx->d_toptab;
	t.nsurv = ctx->d_toptab + TVG_MAX_TOP;
	t.toff = ctx->d_toptab + 2 * TVG_MAX_TOP;
	t.end = ctx->d_toptab + 3 * TVG_MAX_TOP;
	return t;
}

// records a timing event on the context stream; while a capture is in
// progress as an event-record node of the graph (a plain record would only
// mark a dependency inside the capture)
static inline cudaError_t tvg_record(tvg_context *ctx, cudaEvent_t e)
{
	return ctx->capturing ? cudaEventRecordWithFlags(e, ctx->stream, cudaEventRecordExternal)
	                      : cudaEventRecord(e, ctx->stream);
}

// element size of field slot
static inline size_t tvg_field_bytes(const tvg_context *ctx, int slot)
{
	switch (slot) {
	case FS_TYPE: case FS_TIME_BIN: case FS_IT_DRIFT: case FS_IT_KICK: case FS_ID:
	case FS_TREE_PARENT:
		return 4;
	default:
		return tvg_fsize(ctx);
	}
}

// host pointer of a field slot in a tvg_particles, and the TVG_F_* bit of a slot
void *tvg_host_field(const tvg_particles *p, int slot);
uint32_t tvg_slot_bit(int slot);

static inline unsigned tvg_blocks(int64_t n, int threads)
{
	int64_t b = (n + threads - 1) / threads;
	return (unsigned) (b < 1 ? 1 : b);
}

// ------------------------------------------------------- device helpers

__device__ __forceinline__ int tvg_clz128(uint64_t hi, uint64_t lo)
{
	return hi ? __clzll(hi) : 64 + (lo ? __clzll(lo) : 64);
}

// triplet of the standard key at level l (1..42): bits 130-3l .. 128-3l
__device__ __forceinline__ int tvg_std_triplet(uint64_t hi, uint64_t lo, int l)
{
	int sh = 128 - 3 * l;      // lowest bit of the triplet
	if (sh >= 64) return (int) ((hi >> (sh - 64)) & 7);
	if (sh >= 62) return (int) (((hi << (64 - sh)) | (lo >> sh)) & 7);
	return (int) ((lo >> sh) & 7);
}
