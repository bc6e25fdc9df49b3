// tvg_tree_update.cuh -- per-node arithmetic of the tree updates between
// rebuilds (Gravity_Tree_Update_Kicks / Gravity_Tree_Update_Drift,
// src/Gravity/tree_update.c:12-104), shared by the kernels of
// tvg_tree_update.cu and a host build of the same functions.
//
// The reference kicks one active particle at a time and walks from its
// Tree_Parent up to (not including) the subtree's TOP node, adding
// dp / node mass to Dp of every node on the way, then to its top node. A
// node's particles are the contiguous index range [first, first + Npart),
// first being the first particle of the first bundle or leaf at or after the
// node in pre-order (a node's first child is the next node). So each node
// receives the active particles of its range in index order, which is the
// Active_Particle_List order: one thread per node that sums them serially
// repeats the reference's additions exactly, with no atomics.
#pragma once

#include <stdint.h>

#include "tandav_gpu.h"

#define TVG_NODE_TOP (1u << 10)      // Tree_Bitfield TOP (tree.h:64)
#define TVG_NODE_UPDATED (1u << 11)  // Tree_Bitfield UPDATED

// struct Tree_Node (tree.h:23-32)
template <typename F> struct TuNode {
	int32_t DNext;
	uint32_t Bitfield;
	int32_t DUp;
	int32_t Npart;
	F Pos[3];
	F Mass;
	F CoM[3];
	F Dp[3];
};

__host__ __device__ inline double tu_dadd(double a, double b)
{
#ifdef __CUDA_ARCH__
	return __dadd_rn(a, b);
#else
	return a + b;
#endif
}

__host__ __device__ inline double tu_dmul(double a, double b)
{
#ifdef __CUDA_ARCH__
	return __dmul_rn(a, b);
#else
	return a * b;
#endif
}

// first particle of node n (-1 for TOP nodes and terminators, which no kick
// reaches); the scan stays below nnodes
template <typename F>
__host__ __device__ inline int32_t tu_node_first(const TuNode<F> *tree, int64_t nnodes, int64_t n)
{
	if (tree[n].Bitfield & TVG_NODE_TOP) return -1;
	int64_t m = n;
	while (m < nnodes && tree[m].DNext > 0) m++;
	if (m >= nnodes || tree[m].DNext == 0) return -1;
	return -tree[m].DNext - 1;
}

// slots [*a0, *a1) of the active particles with index in [lo, hi): act_off is
// the exclusive scan of the active flags of the n particles, na their total;
// clamped into [0, na]
__host__ __device__ inline void tu_active_slots(const int32_t *act_off, int64_t n, int64_t na, int64_t lo,
                                                int64_t hi, int64_t *a0, int64_t *a1)
{
	int64_t b = (lo >= 0 && lo < n) ? act_off[lo] : na;
	int64_t e = (hi >= 0 && hi < n) ? act_off[hi] : na;
	b = b < 0 ? 0 : (b > na ? na : b);
	e = e < b ? b : (e > na ? na : e);
	*a0 = b;
	*a1 = e;
}

// tree_update.c:14-17: m_dt = Mass * (double) dt rounded to Float, dp = m_dt * Acc
template <typename F>
__host__ __device__ inline void tu_particle_dp(F mass, F dt, F a0, F a1, F a2, F *dp)
{
	const F m_dt = (F) tu_dmul((double) mass, (double) dt);
	dp[0] = m_dt * a0;
	dp[1] = m_dt * a1;
	dp[2] = m_dt * a2;
}

// tree_update.c:24-33 for the active slots [a0, a1) of one subtree node
template <typename F>
__host__ __device__ inline void tu_kick_node(TuNode<F> &nd, const F *dp0, const F *dp1, const F *dp2,
                                             int64_t a0, int64_t a1)
{
	if (a0 >= a1) return;
	const F m = nd.Mass;
	F d0 = nd.Dp[0], d1 = nd.Dp[1], d2 = nd.Dp[2];
	for (int64_t k = a0; k < a1; k++) {
		d0 = d0 + dp0[k] / m;
		d1 = d1 + dp1[k] / m;
		d2 = d2 + dp2[k] / m;
	}
	nd.Dp[0] = d0;
	nd.Dp[1] = d1;
	nd.Dp[2] = d2;
	nd.Bitfield |= TVG_NODE_UPDATED;
}

// tree_update.c:44-52 for one top node (float fields; the quotient is taken in
// Float, so in double for FP64 builds)
template <typename F>
__host__ __device__ inline void tu_kick_top(tvg_topnode &t, const F *dp0, const F *dp1, const F *dp2,
                                            int64_t a0, int64_t a1)
{
	if (a0 >= a1) return;
	if (t.level > 0) t.level = -t.level;
	const F m = (F) t.mass;
	float d0 = t.dp[0], d1 = t.dp[1], d2 = t.dp[2];
	for (int64_t k = a0; k < a1; k++) {
		d0 = (float) ((F) d0 + dp0[k] / m);
		d1 = (float) ((F) d1 + dp1[k] / m);
		d2 = (float) ((F) d2 + dp2[k] / m);
	}
	t.dp[0] = d0;
	t.dp[1] = d1;
	t.dp[2] = d2;
}

// node i of the node kicks (first: tu_node_first of every node); false when
// its particle range does not fit the n particles
template <typename F>
__host__ __device__ inline bool tu_kick_node_at(TuNode<F> *tree, int64_t i, const int32_t *first,
                                                const int32_t *act_off, int64_t n, int64_t na, const F *dp0,
                                                const F *dp1, const F *dp2)
{
	const int64_t lo = first[i];
	if (lo < 0) return true;
	const int64_t hi = lo + tree[i].Npart;
	if (tree[i].Npart <= 0 || hi > n) return false;
	int64_t a0, a1;
	tu_active_slots(act_off, n, na, lo, hi, &a0, &a1);
	tu_kick_node(tree[i], dp0, dp1, dp2, a0, a1);
	return true;
}

// top node t of the top-node kicks; false when its range does not fit
template <typename F>
__host__ __device__ inline bool tu_kick_top_at(tvg_topnode *top, int t, const int32_t *act_off, int64_t n,
                                               int64_t na, const F *dp0, const F *dp1, const F *dp2)
{
	const int64_t lo = top[t].first_part, hi = lo + top[t].npart;
	if (lo < 0 || top[t].npart < 0 || hi > n) return false;
	int64_t a0, a1;
	tu_active_slots(act_off, n, na, lo, hi, &a0, &a1);
	tu_kick_top(top[t], dp0, dp1, dp2, a0, a1);
	return true;
}

// tree_update.c:70-79: a kicked node moves by dt * Dp (in double)
template <typename F>
__host__ __device__ inline void tu_drift_node(TuNode<F> &nd, double dt)
{
	if (!(nd.Bitfield & TVG_NODE_UPDATED)) return;
	for (int c = 0; c < 3; c++) {
		nd.CoM[c] = (F) tu_dadd((double) nd.CoM[c], tu_dmul(dt, (double) nd.Dp[c]));
		nd.Dp[c] = 0;
	}
	nd.Bitfield &= ~TVG_NODE_UPDATED;
}

// tree_update.c:84-97: the same for a kicked top node (negative level)
__host__ __device__ inline void tu_drift_top(tvg_topnode &t, double dt)
{
	if (t.level >= 0) return;
	for (int c = 0; c < 3; c++) {
		t.com[c] = (float) tu_dadd((double) t.com[c], tu_dmul(dt, (double) t.dp[c]));
		t.dp[c] = 0;
	}
	t.level = -t.level;
}
