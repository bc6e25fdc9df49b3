// tvg_decompose.cu -- Domain_Decomposition's cost-balanced top nodes on one
// rank (src/domain.c:67-145 with NTarget = NTask > 1, :151-156).
//
// The reference cuts the PH-sorted particles into "bunches" (octree cells
// along the curve), gives each to one of NTarget targets (its OpenMP threads)
// by cost and splits the costliest bunch of every target until the targets'
// costs agree within DOMAIN_IMBAL_CEIL and their particle counts within
// Part_Alloc_Factor - 1. Its bunches become the top nodes, so a drop-in has
// to repeat the decision exactly: the tree below every top node, and with it
// the walk's interaction order, follows from them.
//
// Split between the device and the host:
// * k_fill_bunches (fill_new_bunches, domain.c:472-531) counts the particles
//   of every bunch from the sorted short keys (binary search of each bunch's
//   key range) and sums cost_metric (domain.c:533-536: the integer part of
//   max(1, P.Cost)) as the reference does: every one of its T threads sums
//   its static share of the range (the first n % T threads one particle more)
//   sequentially in float, one device thread per (share, bunch).
// * The host adds the T partial sums of a bunch in thread order (the
//   reference adds them in a critical section in the threads' order of
//   arrival; the order matters only when three or more partial sums of one
//   bunch cannot be added exactly, above 2^24), then runs the loop on the
//   bunch list (at most a few thousand entries): remove_empty_bunches, the
//   sorts by key and by cost with the reference's comparators through the C
//   library's qsort, distribute, find_global_imbalances,
//   mark_bunches_to_split, make_new_bunchlist.
// * k_bunch_top turns the final bunches into top nodes (centre of the first
//   particle's cell at the bunch level, transform_bunches_into_top_nodes,
//   domain.c:220-250) in the final order, by descending key.
//
// One decomposition costs one kernel launch and one host round trip per
// refinement round (at most N_SHORT_TRIPLETS - MIN_LEVEL + 2); it cannot be
// captured in the step graph, which then runs its steps directly.
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "tvg_internal.cuh"

namespace {

constexpr int MIN_LEVEL = 2;                 // domain.c:3
constexpr int N_SHORT_TRIPLETS = 64 / 3;     // peano.h
constexpr int MAX_JOB_OUT = 1 << 16;         // (bunch, thread share) sums per launch

// the members of struct Bunch_Node (domain.h:29-38) the loop uses
struct Bunch {
	uint64_t key;      // largest short key the bunch can hold
	int target;        // -task - 1
	int level;
	int first;         // first particle (INT_MAX: none)
	uint64_t npart;
	float cost;
	int modify;        // split in the next round
};

// compare_bunches_by_key / _by_cost (domain.c:678-692): descending
int cmp_key(const void *a, const void *b)
{
	const Bunch *x = (const Bunch *) a, *y = (const Bunch *) b;
	return (int) (x->key < y->key) - (int) (x->key > y->key);
}

int cmp_cost(const void *a, const void *b)
{
	const Bunch *x = (const Bunch *) a, *y = (const Bunch *) b;
	return (int) (x->cost < y->cost) - (int) (x->cost > y->cost);
}

// a range of particles counted into nb consecutive bunches
struct FillJob {
	int64_t first_part;
	int64_t npart;
	int32_t nb;
	int32_t key0;      // offset of the bunch keys in the key table
	int32_t out0;      // offset of the outputs: (share t, bunch c) at out0 + t * nb + c
	int32_t pad;
};

// first index in [a, b) whose key exceeds k (b if none)
__device__ __forceinline__ int64_t after_key(const uint64_t *__restrict__ key, int64_t a, int64_t b,
                                             uint64_t k)
{
	while (a < b) {
		const int64_t m = a + ((b - a) >> 1);
		if (key[m] <= k) a = m + 1;
		else b = m;
	}
	return a;
}

// one thread per (job, thread share t, bunch c)
template <typename F>
__global__ void k_fill_bunches(const uint64_t *__restrict__ key_hi, const F *__restrict__ cost,
                               const FillJob *__restrict__ jobs, int njobs, int nthreads, int maxnb,
                               const uint64_t *__restrict__ bkey, int64_t *__restrict__ out_cnt,
                               int64_t *__restrict__ out_first, float *__restrict__ out_cost)
{
	const int64_t g = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	const int64_t per_job = (int64_t) nthreads * maxnb;
	if (g >= per_job * njobs) return;
	const FillJob jb = jobs[g / per_job];
	const int r = (int) (g % per_job);
	const int t = r / maxnb, c = r % maxnb;
	if (c >= jb.nb) return;
	// the static share of thread t (schedule(static) without a chunk)
	const int64_t q = jb.npart / nthreads, rem = jb.npart % nthreads;
	const int64_t s = jb.first_part + (t < rem ? (q + 1) * t : q * t + rem);
	const int64_t e = s + (t < rem ? q + 1 : q);
	// a particle belongs to the first bunch whose key is >= its short key
	const uint64_t *k = bkey + jb.key0;
	const int64_t a = c == 0 ? s : after_key(key_hi, s, e, k[c - 1]);
	const int64_t b = after_key(key_hi, a, e, k[c]);
	float sum = 0.f;
#pragma unroll 4
	for (int64_t i = a; i < b; i++) {
		const unsigned int m = (unsigned int) fmax(1.0, (double) cost[i]);   // cost_metric
		sum = __fadd_rn(sum, __uint2float_rn(m));
	}
	const int64_t o = jb.out0 + (int64_t) t * jb.nb + c;
	out_cnt[o] = b - a;
	out_first[o] = b > a ? a : (int64_t) INT32_MAX;
	out_cost[o] = sum;
}

// transform_bunches_into_top_nodes (domain.c:220-250)
template <typename F>
__global__ void k_bunch_top(int ntop, const F *__restrict__ x, const F *__restrict__ y,
                            const F *__restrict__ z, double ox, double oy, double oz, double size,
                            tvg_topnode *top, tvg_devcount *dc)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t == 0) dc->ntop = ntop;
	if (t >= ntop) return;
	tvg_topnode tn = top[t];
	const int64_t ip = tn.first_part;
	const double sz = size / (double) (1ULL << tn.level);
	const double px = (double) x[ip] - ox, py = (double) y[ip] - oy, pz = (double) z[ip] - oz;
	tn.pos[0] = (float) __dadd_rn(__dmul_rn(floor(px / sz) + 0.5, sz), ox);
	tn.pos[1] = (float) __dadd_rn(__dmul_rn(floor(py / sz) + 0.5, sz), oy);
	tn.pos[2] = (float) __dadd_rn(__dmul_rn(floor(pz / sz) + 0.5, sz), oz);
	tn.mass = 0;
	for (int k = 0; k < 3; k++) { tn.com[k] = 0; tn.dp[k] = 0; }
	top[t] = tn;
}

struct Scratch {
	FillJob *jobs;
	uint64_t *keys;
	int64_t *cnt, *first;
	float *cost;
};

Scratch scratch_of(void *base)
{
	Scratch s;
	char *p = (char *) base;
	s.jobs = (FillJob *) p;
	p += sizeof(FillJob) * 4096;
	s.keys = (uint64_t *) p;
	p += sizeof(uint64_t) * 8192;
	s.cnt = (int64_t *) p;
	p += sizeof(int64_t) * MAX_JOB_OUT;
	s.first = (int64_t *) p;
	p += sizeof(int64_t) * MAX_JOB_OUT;
	s.cost = (float *) p;
	return s;
}

constexpr size_t SCRATCH_BYTES = sizeof(FillJob) * 4096 + sizeof(uint64_t) * 8192
                                 + (2 * sizeof(int64_t) + sizeof(float)) * MAX_JOB_OUT;

// fill_new_bunches for a set of (parent range, bunches) jobs; every bunch of
// the jobs is reset and then receives its counts, first particle and cost
template <typename F>
int fill(tvg_context *ctx, std::vector<Bunch> &D, const std::vector<FillJob> &jobs_in,
         const std::vector<int> &bunch0, int nthreads)
{
	const Scratch sc = scratch_of(ctx->dd_scratch);
	cudaStream_t s = ctx->stream;
	std::vector<FillJob> jobs = jobs_in;
	std::vector<uint64_t> keys;
	int maxnb = 0, out = 0;
	for (size_t j = 0; j < jobs.size(); j++) {
		jobs[j].key0 = (int32_t) keys.size();
		jobs[j].out0 = out;
		for (int c = 0; c < jobs[j].nb; c++) keys.push_back(D[bunch0[j] + c].key);
		out += nthreads * jobs[j].nb;
		if (jobs[j].nb > maxnb) maxnb = jobs[j].nb;
	}
	if (jobs.size() > 4096 || keys.size() > 8192 || out > MAX_JOB_OUT)
		return tvg_fail(ctx, TVG_E_CUDA, "decomposition: fill of %zu bunches too large", keys.size());
	TVG_CUDA(ctx, cudaMemcpyAsync(sc.jobs, jobs.data(), sizeof(FillJob) * jobs.size(),
	                              cudaMemcpyHostToDevice, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(sc.keys, keys.data(), sizeof(uint64_t) * keys.size(),
	                              cudaMemcpyHostToDevice, s));
	const int64_t nthr = (int64_t) jobs.size() * nthreads * maxnb;
	k_fill_bunches<F><<<TVG_CNT(ctx, tvg_blocks(nthr, 128)), 128, 0, s>>>(
	    ctx->key_hi, (const F *) ctx->f[FS_COST], sc.jobs, (int) jobs.size(), nthreads, maxnb, sc.keys,
	    sc.cnt, sc.first, sc.cost);
	TVG_CUDA(ctx, cudaGetLastError());
	std::vector<int64_t> cnt(out), first(out);
	std::vector<float> cost(out);
	TVG_CUDA(ctx, cudaMemcpyAsync(cnt.data(), sc.cnt, 8 * out, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(first.data(), sc.first, 8 * out, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(cost.data(), sc.cost, 4 * out, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	for (size_t j = 0; j < jobs.size(); j++) {
		for (int c = 0; c < jobs[j].nb; c++) {
			Bunch &b = D[bunch0[j] + c];
			b.npart = 0;
			b.cost = 0.f;
			b.first = INT32_MAX;
			// the critical section of fill_new_bunches, in thread order
			for (int t = 0; t < nthreads; t++) {
				const int o = jobs[j].out0 + t * jobs[j].nb + c;
				b.npart += (uint64_t) cnt[o];
				b.cost = b.cost + cost[o];
				if (first[o] < b.first) b.first = (int) first[o];
			}
		}
	}
	return TVG_OK;
}

template <typename F>
int decompose_typed(tvg_context *ctx)
{
	const int64_t n = ctx->n;
	const int ntask = ctx->dd_ntask;
	const int ntarget = ntask;                 // NTask < 65 (domain.c:153-156)
	const int nthreads = ntask;                // one rank: NTask = NThreads
	// find_min_level (domain.c:309-313), reset_bunchlist (:281-307)
	const int level = (int) fmax((double) MIN_LEVEL, log((double) ntarget) / log(8.0) + 1);
	const int nb0 = 1 << (3 * level);
	const int shift = 3 * level;
	std::vector<Bunch> D(nb0);
	for (int i = 0; i < nb0; i++) {
		D[i].key = ((uint64_t) i << (64 - shift)) | (0xFFFFFFFFFFFFFFFFULL >> shift);
		D[i].level = level;
		D[i].npart = 0;
		D[i].first = INT32_MAX;
		D[i].target = -1;
		D[i].modify = 0;
		D[i].cost = 0.f;
	}
	FillJob j0 = { 0, n, nb0, 0, 0, 0 };
	TVG_CHECK(fill<F>(ctx, D, std::vector<FillJob>(1, j0), std::vector<int>(1, 0), nthreads));
	// find_mean_cost (domain.c:538-556)
	double mean_cost = 0;
	for (const Bunch &b : D) mean_cost += b.cost;
	mean_cost /= ntarget;
	const double mean_npart = (double) n / ntarget;
	std::vector<float> tcost(ntarget);
	std::vector<int> tnpart(ntarget), split(ntarget);
	int cnt = 0;
	for (;;) {
		// remove_empty_bunches (domain.c:435-470)
		std::vector<Bunch> kept;
		kept.reserve(D.size());
		for (const Bunch &b : D)
			if (b.npart != 0) kept.push_back(b);
		D.swap(kept);
		qsort(D.data(), D.size(), sizeof(Bunch), cmp_key);
		// distribute (domain.c:573-628)
		for (int t = 0; t < ntarget; t++) { tcost[t] = 0.f; tnpart[t] = 0; }
		qsort(D.data(), D.size(), sizeof(Bunch), cmp_cost);
		for (Bunch &b : D) {
			int task = 0;
			double max_delta = 0;
			for (int t = 0; t < ntarget; t++) {
				const double delta = mean_cost - tcost[t];
				if (delta > max_delta) { task = t; max_delta = delta; }
			}
			tcost[task] += b.cost;
			tnpart[task] += (int) b.npart;
			b.target = -task - 1;
		}
		qsort(D.data(), D.size(), sizeof(Bunch), cmp_key);
		for (int t = 0; t < ntarget; t++) split[t] = t;
		for (size_t i = 0; i < D.size(); i++) {
			const int task = -(D[i].target + 1);
			const int idx = split[task];
			// (idx beyond the list: fewer bunches than targets, tiny inputs)
			if (idx >= (int) D.size() || D[i].cost > D[idx].cost) split[task] = (int) i;
		}
		// find_global_imbalances (domain.c:630-652)
		double cost_imbal = -1e300, mem_imbal = -1e300;
		for (int t = 0; t < ntarget; t++) {
			cost_imbal = fmax(cost_imbal, fabs(tcost[t] - mean_cost) / mean_cost);
			mem_imbal = fmax(mem_imbal, fabs(tnpart[t] - mean_npart) / mean_npart);
		}
		if (cost_imbal < ctx->dd_imbal_ceil && mem_imbal < ctx->dd_part_alloc_factor - 1) break;
		if (cnt++ > N_SHORT_TRIPLETS - MIN_LEVEL) break;
		// mark_bunches_to_split (domain.c:654-676)
		for (int t = 0; t < ntarget; t++) {
			const int jx = split[t];
			if (jx < 0 || jx >= (int) D.size() || D[jx].level == N_SHORT_TRIPLETS) continue;
			D[jx].modify = 1;
		}
		// make_new_bunchlist (domain.c:374-406), split_bunch (:408-433)
		std::vector<FillJob> jobs;
		std::vector<int> bunch0;
		const size_t old = D.size();
		for (size_t i = 0; i < old; i++) {
			if (!D[i].modify) continue;
			const int first_new = (int) D.size();
			for (int c = 0; c < 8; c++) {
				Bunch b;
				b.level = D[i].level + 1;
				const int sh = 64 - 3 * b.level;
				const uint64_t mask = 0x7ULL << sh;
				b.key = (D[i].key & ~mask) | ((uint64_t) c << sh);
				b.npart = 0;
				b.first = INT32_MAX;
				b.target = -1;
				b.modify = 0;
				b.cost = 0.f;
				D.push_back(b);
			}
			FillJob jb = { D[i].first, (int64_t) D[i].npart, 8, 0, 0, 0 };
			jobs.push_back(jb);
			bunch0.push_back(first_new);
			D[i].npart = 0;                    // removed in the next round
		}
		if (!jobs.empty()) TVG_CHECK(fill<F>(ctx, D, jobs, bunch0, nthreads));
		if (D.size() > (size_t) TVG_MAX_TOP)
			return tvg_fail(ctx, TVG_E_TREE_FULL, "decomposition: more than %d bunches", TVG_MAX_TOP);
	}
	if (D.size() > (size_t) TVG_MAX_TOP)
		return tvg_fail(ctx, TVG_E_TREE_FULL, "decomposition: more than %d top nodes", TVG_MAX_TOP);
	ctx->dd_rounds = cnt;
	// the top nodes in the final order
	const int ntop = (int) D.size();
	std::vector<tvg_topnode> top(ntop);
	for (int t = 0; t < ntop; t++) {
		memset(&top[t], 0, sizeof(tvg_topnode));
		top[t].key = D[t].key;
		top[t].target = D[t].target;
		top[t].level = D[t].level;
		top[t].first_part = D[t].first;
		top[t].npart = (int32_t) D[t].npart;
	}
	cudaStream_t s = ctx->stream;
	TVG_CUDA(ctx, cudaMemcpyAsync(ctx->d_top, top.data(), sizeof(tvg_topnode) * ntop,
	                              cudaMemcpyHostToDevice, s));
	k_bunch_top<F><<<TVG_CNT(ctx, tvg_blocks(ntop, 128)), 128, 0, s>>>(
	    ntop, (const F *) ctx->f[FS_POS0], (const F *) ctx->f[FS_POS1], (const F *) ctx->f[FS_POS2],
	    ctx->origin[0], ctx->origin[1], ctx->origin[2], ctx->dsize, ctx->d_top, ctx->dc);
	TVG_CUDA(ctx, cudaGetLastError());
	// the host copy of the list must outlive the asynchronous copy
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	return TVG_OK;
}

} // namespace

int tvg_impl_top_nodes_balanced(tvg_context *ctx)
{
	if (ctx->capturing)
		return tvg_fail(ctx, TVG_E_STATE, "a balanced domain decomposition cannot be captured");
	if (ctx->n <= 0) return tvg_fail(ctx, TVG_E_STATE, "top_nodes: no particles");
	if (!ctx->dd_scratch) {
		cudaError_t e = cudaMalloc(&ctx->dd_scratch, SCRATCH_BYTES);
		if (e != cudaSuccess) {
			ctx->dd_scratch = nullptr;
			return tvg_fail(ctx, TVG_E_NOMEM, "decomposition scratch: %s", cudaGetErrorString(e));
		}
	}
	const int rc = ctx->cfg.float_bytes == 4 ? decompose_typed<float>(ctx) : decompose_typed<double>(ctx);
	if (rc != TVG_OK) return rc;
	TVG_CHECK(tvg_impl_top_of(ctx));
	return tvg_read_counts(ctx);
}

extern "C" int tvg_set_domain_decomposition(tvg_context *ctx, int32_t ntask, double part_alloc_factor,
                                            double imbal_ceil)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (ntask < 1 || !(part_alloc_factor > 1.0) || !(imbal_ceil > 0.0))
		return tvg_fail(ctx, TVG_E_BADINPUT, "set_domain_decomposition: ntask >= 1, "
		                "part_alloc_factor > 1 and imbal_ceil > 0 required");
	ctx->dd_ntask = ntask;
	ctx->dd_part_alloc_factor = part_alloc_factor;
	ctx->dd_imbal_ceil = imbal_ceil;
	ctx->have_top = ctx->have_tree = ctx->have_walktree = false;
	return TVG_OK;
}

extern "C" int tvg_decomposition_rounds(tvg_context *ctx, int32_t *rounds)
{
	if (!ctx || !rounds) return TVG_E_BADINPUT;
	*rounds = ctx->dd_rounds;
	return TVG_OK;
}
