// Host build of the tree-update arithmetic of the library
// (tandav_b200/csrc/tvg_tree_update.cuh): the same per-node functions the
// kernels of tvg_tree_update.cu run, looped over the nodes on the CPU, so a
// CPU test can hold them against the reference's own tree updates.
// Test infrastructure only; built by tests/test_tree_update_host.py.
#include <vector>

#include "../tandav_b200/csrc/tvg_tree_update.cuh"

template <typename F>
static int kick(void *tree_v, int64_t nnodes, tvg_topnode *top, int ntop, const int32_t *act_off, int64_t n,
                int64_t na, const void *dp_v, int64_t cap)
{
	TuNode<F> *tree = (TuNode<F> *) tree_v;
	const F *dp = (const F *) dp_v;
	std::vector<int32_t> first((size_t) (nnodes > 0 ? nnodes : 1));
	for (int64_t i = 0; i < nnodes; i++) first[i] = tu_node_first(tree, nnodes, i);
	int bad = 0;
	for (int64_t i = 0; i < nnodes; i++)
		bad += !tu_kick_node_at(tree, i, first.data(), act_off, n, na, dp, dp + cap, dp + 2 * cap);
	for (int t = 0; t < ntop; t++) bad += !tu_kick_top_at(top, t, act_off, n, na, dp, dp + cap, dp + 2 * cap);
	return bad;
}

template <typename F>
static void particle_dp(int64_t n, const int32_t *flag, const int32_t *off, const void *mass_v, const void *dt_v,
                        const void *acc_v, void *dp_v, int64_t cap)
{
	const F *mass = (const F *) mass_v, *dt = (const F *) dt_v, *acc = (const F *) acc_v;
	F *dp = (F *) dp_v;
	for (int64_t i = 0; i < n; i++) {
		if (!flag[i]) continue;
		F d[3];
		tu_particle_dp(mass[i], dt[i], acc[i], acc[n + i], acc[2 * n + i], d);
		for (int c = 0; c < 3; c++) dp[c * cap + off[i]] = d[c];
	}
}

template <typename F>
static void drift(void *tree_v, int64_t nnodes, tvg_topnode *top, int ntop, double dt)
{
	TuNode<F> *tree = (TuNode<F> *) tree_v;
	for (int64_t i = 0; i < nnodes; i++) tu_drift_node(tree[i], dt);
	for (int t = 0; t < ntop; t++) tu_drift_top(top[t], dt);
}

extern "C" int tu_host_kick(int fsize, void *tree, int64_t nnodes, tvg_topnode *top, int ntop,
                            const int32_t *act_off, int64_t n, int64_t na, const void *dp, int64_t cap)
{
	return fsize == 4 ? kick<float>(tree, nnodes, top, ntop, act_off, n, na, dp, cap)
	                  : kick<double>(tree, nnodes, top, ntop, act_off, n, na, dp, cap);
}

extern "C" void tu_host_dp(int fsize, int64_t n, const int32_t *flag, const int32_t *off, const void *mass,
                           const void *dt, const void *acc, void *dp, int64_t cap)
{
	if (fsize == 4) particle_dp<float>(n, flag, off, mass, dt, acc, dp, cap);
	else particle_dp<double>(n, flag, off, mass, dt, acc, dp, cap);
}

extern "C" void tu_host_drift(int fsize, void *tree, int64_t nnodes, tvg_topnode *top, int ntop, double dt)
{
	if (fsize == 4) drift<float>(tree, nnodes, top, ntop, dt);
	else drift<double>(tree, nnodes, top, ntop, dt);
}
