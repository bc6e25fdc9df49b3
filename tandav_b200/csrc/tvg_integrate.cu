// tvg_integrate.cu -- hierarchical (power-of-two rung) time integration of
// the active particles: Set_New_Timesteps (timestep.c:35-89, 200-299),
// Kick_First/Second_Halfstep (kick.c:9-70), Drift_To_Sync_Point
// (drift.c:12-62), Periodic_Constrain_Particles_To_Box (periodic.c:30-55), and
// the comoving kick/drift factors (comoving.c:30-153).
//
// Timeline: 2^31 integer ticks (Int_Time.End = 1 << 31, timestep.c:127-136);
// with COMOVING a tick is Step_Min = ln(a_end / a_beg) / 2^31 in ln a and
// a(it) = a_beg exp(it Step_Min) (timestep.c:371-374), otherwise
// t(it) = t_beg + it Step_Min.
//
// Kick and drift factors (COMOVING): K(a) = int da / (H a^2) and
// D(a) = int da / (H a^3) from 0.95 a_beg, tabulated at the reference's 512
// knots a_i = 0.95 a_beg exp(i da), da = ln(1.05 a_end / 0.95 a_beg) / 511,
// with knot 0 left at a = 0 and value 0 (the reference's table loop starts at
// i = 1, comoving.c:119-137), and interpolated by a natural cubic spline
// through all 512 knots (gsl cspline, comoving.c:146-150). The reference
// integrates with GSL QAG (GAUSS41, relative 1e-8); here each knot's integral
// is a composite 16-point Gauss-Legendre rule over 32 equal intervals in ln a,
// in FP64 on the device (the integrands are smooth in ln a; the rule is exact
// to FP64 round-off), and the spline's tridiagonal system is solved in FP64
// on the device. The per-particle factor is K(a_next) - K(a_curr) from that
// spline, in FP64, as in Particle_Kick_Step / Particle_Drift_Step.
//
// The particle updates replay the reference's arithmetic (Float kick,
// double drift step) and the file is compiled without FMA contraction.
#include <float.h>
#include <math.h>

#include <vector>

#include "tvg_internal.cuh"
#include "tvg_tree_update.cuh"

#define KD_TABLE 512
#define KD_GL 16
#define KD_SUB 32
#define N_INT_BINS 32

struct Cosmo {
	double h0, om_l, om_m, om_r, om_0;
};

__device__ __host__ inline double hubble(const Cosmo &c, double a)
{
	// E_Hubble, cosmology.c:70-74
	return c.h0 * sqrt(c.om_l + (1.0 - c.om_0) / (a * a) + c.om_m / (a * a * a)
	                   + c.om_r / (a * a * a * a));
}

struct GLRule {
	double x[KD_GL], w[KD_GL];
};

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's iteration on the
// Legendre polynomial (Golub & Welsch 1969 give the same rule)
static GLRule gauss_legendre()
{
	GLRule r;
	const int n = KD_GL;
	for (int i = 0; i < (n + 1) / 2; i++) {
		double z = cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 0;
		for (int it = 0; it < 100; it++) {
			double p1 = 1, p2 = 0;
			for (int j = 1; j <= n; j++) {
				const double p3 = p2;
				p2 = p1;
				p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
			}
			pp = n * (z * p1 - p2) / (z * z - 1.0);
			const double z1 = z;
			z = z1 - p1 / pp;
			if (fabs(z - z1) < 1e-16) break;
		}
		r.x[i] = -z;
		r.x[n - 1 - i] = z;
		r.w[i] = r.w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
	}
	return r;
}

// knot abscissae and the two integrals, one thread per knot
__global__ void k_kd_table(Cosmo c, double a0, double da, GLRule gl, double *x, double *kick,
                           double *drift)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= KD_TABLE) return;
	if (i == 0) {
		x[0] = kick[0] = drift[0] = 0;
		return;
	}
	const double amax = a0 * exp(da * i);
	x[i] = amax;
	const double s0 = log(a0), s1 = log(amax), h = (s1 - s0) / KD_SUB;
	double sk = 0, sd = 0;
	for (int j = 0; j < KD_SUB; j++) {
		const double mid = s0 + (j + 0.5) * h;
		for (int q = 0; q < KD_GL; q++) {
			const double s = mid + 0.5 * h * gl.x[q];
			const double a = exp(s);
			const double f = 0.5 * h * gl.w[q] / hubble(c, a);   // da = a ds
			sk += f / a;             // 1 / (H a^2) da
			sd += f / (a * a);       // 1 / (H a^3) da
		}
	}
	kick[i] = sk;
	drift[i] = sd;
}

// natural cubic spline: second derivatives (Thomas algorithm), one thread
__global__ void k_kd_spline(const double *x, const double *y, double *m2, double *work)
{
	if (blockIdx.x || threadIdx.x) return;
	const int n = KD_TABLE;
	double *cp = work, *dp = work + n;
	m2[0] = m2[n - 1] = 0;
	// rows i = 1..n-2: h_{i-1} M_{i-1} + 2 (h_{i-1} + h_i) M_i + h_i M_{i+1} = r_i
	for (int i = 1; i < n - 1; i++) {
		const double hl = x[i] - x[i - 1], hr = x[i + 1] - x[i];
		const double r = 6.0 * ((y[i + 1] - y[i]) / hr - (y[i] - y[i - 1]) / hl);
		const double b = 2.0 * (hl + hr);
		if (i == 1) {
			cp[i] = hr / b;
			dp[i] = r / b;
		} else {
			const double den = b - hl * cp[i - 1];
			cp[i] = hr / den;
			dp[i] = (r - hl * dp[i - 1]) / den;
		}
	}
	m2[n - 2] = dp[n - 2];
	for (int i = n - 3; i >= 1; i--) m2[i] = dp[i] - cp[i] * m2[i + 1];
}

struct KDTables {
	const double *x, *kick, *drift, *m2k, *m2d;
	double a0, da;       // knot i >= 1 at a0 exp(i da)
};

// spline value at a, in the knot interval [x_i, x_{i+1}) that holds a
__device__ __forceinline__ double spline_eval(const KDTables &t, const double *y,
                                              const double *m2, double a)
{
	int i = (a > t.a0) ? (int) floor(log(a / t.a0) / t.da) : 0;
	i = max(0, min(i, KD_TABLE - 2));
	while (i < KD_TABLE - 2 && a >= t.x[i + 1]) i++;
	while (i > 0 && a < t.x[i]) i--;
	const double h = t.x[i + 1] - t.x[i], d = a - t.x[i];
	const double b = (y[i + 1] - y[i]) / h - h * (2.0 * m2[i] + m2[i + 1]) / 6.0;
	return y[i] + d * (b + d * (0.5 * m2[i] + d * (m2[i + 1] - m2[i]) / (6.0 * h)));
}

struct TimeParams {
	int comoving;
	double t_begin, step_min;
	KDTables tab;
};

__device__ __forceinline__ double it2time(const TimeParams &p, uint32_t it)
{
	// Integer_Time2Integration_Time, timestep.c:371-401
	return p.comoving ? p.t_begin * exp((double) it * p.step_min)
	                  : p.t_begin + (double) it * p.step_min;
}

__device__ __forceinline__ double kick_step(const TimeParams &p, uint32_t c, uint32_t n)
{
	const double a0 = it2time(p, c), a1 = it2time(p, n);
	if (!p.comoving) return a1 - a0;
	return spline_eval(p.tab, p.tab.kick, p.tab.m2k, a1) - spline_eval(p.tab, p.tab.kick, p.tab.m2k, a0);
}

__device__ __forceinline__ double drift_step(const TimeParams &p, uint32_t c, uint32_t n)
{
	const double a0 = it2time(p, c), a1 = it2time(p, n);
	if (!p.comoving) return a1 - a0;
	return spline_eval(p.tab, p.tab.drift, p.tab.m2d, a1) - spline_eval(p.tab, p.tab.drift, p.tab.m2d, a0);
}

// Kick_First_Halfstep / Kick_Second_Halfstep (kick.c:9-70). The kick factor
// (an exponential and a spline in FP64) depends only on It_Kick_Pos and the
// time bin, and the particles of one bin share their It_Kick_Pos in a step.
// So a block keeps one slot per bin: the first thread that claims a bin's
// slot for its particle's It_Kick_Pos evaluates the factor there, and every
// particle of the block with that bin and position takes it (the same
// function, so the same bits); a particle whose position differs evaluates
// its own. KD_IPT particles per thread.
#define KD_THREADS 256
#define KD_IPT 4
#define KD_EMPTY 0xFFFFFFFFu          // no integer time reaches it (the timeline ends at 2^31)

// claims the bin's slot for it_curr; true for the thread that must evaluate
__device__ __forceinline__ bool kd_claim(uint32_t *s_curr, int b, uint32_t it_curr)
{
	return b >= 0 && b < N_INT_BINS && atomicCAS(&s_curr[b], KD_EMPTY, it_curr) == KD_EMPTY;
}

template <typename F>
__global__ void __launch_bounds__(KD_THREADS) k_kick(int64_t n_act, const int32_t *__restrict__ active,
                                                     TimeParams p, const int32_t *__restrict__ bin,
                                                     uint32_t *it_kick, const F *a0, const F *a1, const F *a2,
                                                     F *v0, F *v1, F *v2)
{
	__shared__ uint32_t s_curr[N_INT_BINS];
	__shared__ double s_dt[N_INT_BINS];
	if (threadIdx.x < N_INT_BINS) s_curr[threadIdx.x] = KD_EMPTY;
	__syncthreads();
	const int64_t k0 = (int64_t) blockIdx.x * (KD_THREADS * KD_IPT);
	int64_t idx[KD_IPT];
	int b[KD_IPT];
	uint32_t cur[KD_IPT];
#pragma unroll
	for (int u = 0; u < KD_IPT; u++) {
		const int64_t k = k0 + u * KD_THREADS + threadIdx.x;
		idx[u] = -1;
		if (k < n_act) {
			idx[u] = active ? active[k] : k;
			b[u] = bin[idx[u]];
			cur[u] = it_kick[idx[u]];
			if (kd_claim(s_curr, b[u], cur[u]))
				s_dt[b[u]] = kick_step(p, cur[u], cur[u] + ((1u << b[u]) >> 1));
		}
	}
	__syncthreads();
#pragma unroll
	for (int u = 0; u < KD_IPT; u++) {
		if (idx[u] < 0) continue;
		const int64_t i = idx[u];
		const uint32_t it_step = 1u << b[u];
		const uint32_t it_curr = cur[u], it_next = it_curr + (it_step >> 1);
		const bool hit = b[u] >= 0 && b[u] < N_INT_BINS && s_curr[b[u]] == it_curr;
		const F dt = (F) (hit ? s_dt[b[u]] : kick_step(p, it_curr, it_next));
		v0[i] += dt * a0[i];
		v1[i] += dt * a1[i];
		v2[i] += dt * a2[i];
		it_kick[i] += it_step >> 1;
	}
}

// the momentum change of each active particle for the tree updates
// (tree_update.c:14-17), stored by its slot in particle order; taken with the
// kick step of k_kick, before k_kick advances It_Kick_Pos
template <typename F>
__global__ void k_kick_dp(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ off,
                          TimeParams p, const int32_t *__restrict__ bin, const uint32_t *__restrict__ it_kick,
                          const F *__restrict__ mass, const F *__restrict__ a0, const F *__restrict__ a1,
                          const F *__restrict__ a2, F *dp0, F *dp1, F *dp2)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n || !flag[i]) return;
	const uint32_t it_step = 1u << bin[i];
	const uint32_t it_curr = it_kick[i], it_next = it_curr + (it_step >> 1);
	const F dt = (F) kick_step(p, it_curr, it_next);
	F d[3];
	tu_particle_dp(mass[i], dt, a0[i], a1[i], a2[i], d);
	const int64_t k = off[i];
	dp0[k] = d[0];
	dp1[k] = d[1];
	dp2[k] = d[2];
}

// Drift_To_Sync_Point (drift.c:12-40): the active particles only. The drift
// factor depends only on It_Drift_Pos (it_next is the step's); as in k_kick,
// a block evaluates it once per distinct position of each time bin.
template <typename F>
__global__ void __launch_bounds__(KD_THREADS) k_drift(int64_t n_act, const int32_t *__restrict__ active,
                                                      TimeParams p, uint32_t it_next, uint32_t it_end,
                                                      const int32_t *__restrict__ bin, uint32_t *it_drift,
                                                      const F *v0, const F *v1, const F *v2, F *x0, F *x1, F *x2,
                                                      int *status)
{
	__shared__ uint32_t s_curr[N_INT_BINS];
	__shared__ double s_dt[N_INT_BINS];
	if (threadIdx.x < N_INT_BINS) s_curr[threadIdx.x] = KD_EMPTY;
	__syncthreads();
	const int64_t k0 = (int64_t) blockIdx.x * (KD_THREADS * KD_IPT);
	int64_t idx[KD_IPT];
	int b[KD_IPT];
	uint32_t cur[KD_IPT];
#pragma unroll
	for (int u = 0; u < KD_IPT; u++) {
		const int64_t k = k0 + u * KD_THREADS + threadIdx.x;
		idx[u] = -1;
		if (k < n_act) {
			idx[u] = active ? active[k] : k;
			b[u] = bin[idx[u]];
			cur[u] = it_drift[idx[u]];
			const bool valid = !(it_next > it_end || it_next < cur[u]);
			if (valid && kd_claim(s_curr, b[u], cur[u])) s_dt[b[u]] = drift_step(p, cur[u], it_next);
		}
	}
	__syncthreads();
#pragma unroll
	for (int u = 0; u < KD_IPT; u++) {
		if (idx[u] < 0) continue;
		const int64_t i = idx[u];
		const uint32_t it_curr = cur[u];
		if (it_next > it_end || it_next < it_curr) {            // drift.c:22-27
			atomicOr(status, TVG_ST_BADPOS);
			continue;
		}
		const bool hit = b[u] >= 0 && b[u] < N_INT_BINS && s_curr[b[u]] == it_curr;
		const double dt = hit ? s_dt[b[u]] : drift_step(p, it_curr, it_next);
		x0[i] = (F) ((double) x0[i] + dt * (double) v0[i]);
		x1[i] = (F) ((double) x1[i] + dt * (double) v1[i]);
		x2[i] = (F) ((double) x2[i] + dt * (double) v2[i]);
		it_drift[i] += it_next - it_curr;
	}
}

// Periodic_Constrain_Particles_To_Box (periodic.c:30-55), all particles; the
// loops are bounded (a non-finite or far-out position sets a status bit)
template <typename F>
__global__ void k_wrap(int64_t n, F box, F *x0, F *x1, F *x2, int *status)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	F *x[3] = { x0, x1, x2 };
#pragma unroll
	for (int d = 0; d < 3; d++) {
		F v = x[d][i];
		int it = 0;
		while (v < 0 && it < 64) { v += box; it++; }
		while (v >= box && it < 64) { v -= box; it++; }
		if (it >= 64 || !(v >= 0 && v < box)) atomicOr(status, TVG_ST_BADPOS);
		x[d][i] = v;
	}
}

struct BinParams {
	double grav_accel_factor;   // Cosmo.Grav_Accel_Factor = 1 / a^2 (1 without COMOVING)
	double expansion_factor;    // Cosmo.Expansion_Factor
	double hubble;              // Cosmo.Hubble_Parameter (COMOVING) or 1
	double time_int_accuracy;
	double softening;           // Param.Grav_Softening[1]
	double step_max, step_min;
	float dt_max_global;        // Dt_Max_Global (a float in the reference)
	int comoving;
	int max_active_bin;
};

// set_new_particle_timebins (timestep.c:200-236) with get_physical_timestep,
// cosmological_timestep, Acceleration_Physical (unit.c:55-71) and
// timestep2timebin, in the reference's Float / float / double order
template <typename F>
__global__ void k_timebins(int64_t n, BinParams p, const F *g0, const F *g1, const F *g2,
                           int32_t *bin, int32_t *minmax, int *status)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	int bmin = N_INT_BINS - 1, bmax = 0;
	if (i < n) {
		const F a0 = g0[i], a1 = g1[i], a2 = g2[i];
		double grav = sqrt((double) (a0 * a0 + a1 * a1 + a2 * a2));
		if (p.comoving) grav *= p.grav_accel_factor;
		const F acc_phys = (F) grav;
		const F eps = (F) (105.0 / 32.0 * p.softening);
		const float dt_cosmo = p.comoving
		    ? (float) (p.time_int_accuracy * sqrt(2 * p.expansion_factor * (double) eps / (double) acc_phys))
		    : (float) (p.time_int_accuracy * sqrt(2 * (double) eps / (double) acc_phys));
		float dtf = FLT_MAX;
		dtf = (float) fmin((double) dtf, (double) dt_cosmo);
		F dt = (F) dtf;
		if (p.comoving) dt = (F) ((double) dt * p.hubble);      // convert_dt_to_dlna
		dt = (F) fmin((double) dt, (double) p.dt_max_global);
		if (!((double) dt >= p.step_min)) atomicOr(status, TVG_ST_TIMESTEP);
		int e = 0;
		frexp(p.step_max / (double) dt, &e);
		const int want = N_INT_BINS - 1 - e;
		const int allowed = max(p.max_active_bin, bin[i]);
		const int b = min(want, allowed);
		bin[i] = b;
		bmin = b;
		bmax = b;
	}
	bmin = __reduce_min_sync(0xFFFFFFFFu, bmin);
	bmax = __reduce_max_sync(0xFFFFFFFFu, bmax);
	if ((threadIdx.x & 31) == 0) {
		atomicMin(minmax, bmin);
		atomicMax(minmax + 1, bmax);
	}
}

// rung histogram of all particles
__global__ void k_bin_hist(int64_t n, const int32_t *__restrict__ bin, int32_t *hist)
{
	__shared__ int32_t h[N_INT_BINS];
	if (threadIdx.x < N_INT_BINS) h[threadIdx.x] = 0;
	__syncthreads();
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		const int b = bin[i];
		if (b >= 0 && b < N_INT_BINS) atomicAdd(&h[b], 1);
	}
	__syncthreads();
	if (threadIdx.x < N_INT_BINS && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

// per-type sums of |v|^2 (Float squares summed in Float, added in FP64),
// minimum mass and count (Comoving_VelDisp_Timestep_Constraint, comoving.c:195-223).
// Like the reference's per-thread partial sums, each thread sums its
// particles in registers; the warp and then the block combine them, and one
// atomic per block and type adds the block's share (one atomic per particle
// on six addresses serialises: 43 ms at 256^3). The FP64 sum's order is not
// the reference's either way (its threads' partial sums meet in a critical
// section in any order).
#define VD_THREADS 256
template <typename F>
__global__ void __launch_bounds__(VD_THREADS) k_veldisp(int64_t n, const int32_t *__restrict__ type,
                                                        const F *__restrict__ v0, const F *__restrict__ v1,
                                                        const F *__restrict__ v2, const F *__restrict__ mass,
                                                        double *vel2, uint32_t *min_mass_bits,
                                                        unsigned long long *npart)
{
	__shared__ double s_v[VD_THREADS / 32][6];
	__shared__ uint32_t s_m[VD_THREADS / 32][6];
	__shared__ unsigned long long s_n[VD_THREADS / 32][6];
	double sv[6];
	uint32_t sm[6];
	unsigned long long sn[6];
#pragma unroll
	for (int t = 0; t < 6; t++) {
		sv[t] = 0.0;
		sm[t] = 0xFFFFFFFFu;
		sn[t] = 0ull;
	}
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		const int ty = type[i];
		const F a = v0[i], b = v1[i], c = v2[i];
		const double q = (double) (a * a + b * b + c * c);
		const uint32_t m = __float_as_uint((float) mass[i]);     // masses > 0
#pragma unroll
		for (int t = 0; t < 6; t++)
			if (ty == t) {
				sv[t] += q;
				sm[t] = min(sm[t], m);
				sn[t] += 1ull;
			}
	}
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
	for (int t = 0; t < 6; t++) {
#pragma unroll
		for (int o = 16; o; o >>= 1) {
			sv[t] += __shfl_xor_sync(0xFFFFFFFFu, sv[t], o);
			sm[t] = min(sm[t], __shfl_xor_sync(0xFFFFFFFFu, sm[t], o));
			sn[t] += __shfl_xor_sync(0xFFFFFFFFu, sn[t], o);
		}
		if (lane == 0) {
			s_v[w][t] = sv[t];
			s_m[w][t] = sm[t];
			s_n[w][t] = sn[t];
		}
	}
	__syncthreads();
	if (threadIdx.x < 6) {
		const int t = threadIdx.x;
		double v = 0.0;
		uint32_t m = 0xFFFFFFFFu;
		unsigned long long c = 0ull;
		for (int k = 0; k < VD_THREADS / 32; k++) {
			v += s_v[k][t];
			m = min(m, s_m[k][t]);
			c += s_n[k][t];
		}
		if (c) {
			atomicAdd(&vel2[t], v);
			atomicMin(&min_mass_bits[t], m);
			atomicAdd(&npart[t], c);
		}
	}
}

// Make_Active_Particle_List (timestep.c:280-299): flags, scan, scatter
// the bin limit from the device counts (set before the step, so that a
// captured step reads the current one)
__global__ void k_active_flags(int64_t n, const int32_t *__restrict__ bin,
                               const tvg_devcount *__restrict__ dc, int32_t *flag)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) flag[i] = bin[i] <= dc->max_active_bin;
}

__global__ void k_set_max_bin(tvg_devcount *dc, int32_t b) { dc->max_active_bin = b; }

int tvg_set_device_max_bin(tvg_context *ctx)
{
	k_set_max_bin<<<TVG_CNT(ctx, 1), 1, 0, ctx->stream>>>(ctx->dc, ctx->tl.state.max_active_bin);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

__global__ void k_active_scatter(int64_t n, const int32_t *__restrict__ flag,
                                 const int32_t *__restrict__ off, int32_t *active)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n && flag[i]) active[off[i]] = (int32_t) i;
}

// ------------------------------------------------------------------ host

static int ensure(tvg_context *ctx, void **p, size_t bytes)
{
	if (*p) return TVG_OK;
	TVG_CUDA(ctx, cudaMalloc(p, bytes));
	return TVG_OK;
}

static TimeParams time_params(const tvg_context *ctx)
{
	TimeParams p;
	p.comoving = ctx->tl.cfg.comoving;
	p.t_begin = ctx->tl.cfg.time_begin;
	p.step_min = ctx->tl.state.step_min;
	p.tab.x = ctx->kd_x;
	p.tab.kick = ctx->kd_kick;
	p.tab.drift = ctx->kd_drift;
	p.tab.m2k = ctx->kd_m2k;
	p.tab.m2d = ctx->kd_m2d;
	p.tab.a0 = 0.95 * ctx->tl.cfg.time_begin;
	p.tab.da = log((1.05 * ctx->tl.cfg.time_end) / (0.95 * ctx->tl.cfg.time_begin)) / (KD_TABLE - 1);
	return p;
}

static Cosmo cosmo(const tvg_timeline_config &c)
{
	return Cosmo{ c.hubble_constant, c.omega_lambda, c.omega_matter, c.omega_rad, c.omega_0 };
}

static double host_it2time(const tvg_context *ctx, uint32_t it)
{
	const tvg_timeline_config &c = ctx->tl.cfg;
	return c.comoving ? c.time_begin * exp((double) it * ctx->tl.state.step_min)
	                  : c.time_begin + (double) it * ctx->tl.state.step_min;
}

// Set_Current_Cosmology (cosmology.c:40-58): the parts the time step reads
static void set_current_cosmology(tvg_context *ctx)
{
	tvg_timeline_state &s = ctx->tl.state;
	const tvg_timeline_config &c = ctx->tl.cfg;
	if (c.comoving) {
		s.expansion_factor = s.time_current;
		s.hubble_parameter = hubble(cosmo(c), s.time_current);
	} else {
		s.expansion_factor = 1;
		s.hubble_parameter = c.hubble_constant;
	}
}

extern "C" int tvg_timeline_init(tvg_context *ctx, const tvg_timeline_config *cfg)
{
	if (!ctx || !cfg) return TVG_E_BADINPUT;
	if (!(cfg->time_end > cfg->time_begin) || (cfg->comoving && !(cfg->time_begin > 0)))
		return tvg_fail(ctx, TVG_E_BADINPUT, "timeline: need time_end > time_begin (> 0 when comoving)");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	cudaStream_t s = ctx->stream;
	ctx->tl.cfg = *cfg;
	tvg_timeline_state &st = ctx->tl.state;
	memset(&st, 0, sizeof(st));
	// Setup_Time_Integration, timestep.c:127-158
	st.beg = 0;
	st.end = 1u << (N_INT_BINS - 1);
	st.step_max = cfg->comoving ? log(cfg->time_end) - log(cfg->time_begin)
	                            : cfg->time_end - cfg->time_begin;
	st.step_min = st.step_max / (double) (st.end - st.beg);
	st.current = st.beg;
	st.time_current = host_it2time(ctx, st.current);
	st.max_active_bin = N_INT_BINS - 1;
	st.first_step = 1;
	st.prepare_step = 0;
	st.sync_point = 0;
	st.next_sync_point = 0;
	st.dt_max_global = FLT_MAX;
	set_current_cosmology(ctx);
	// kick / drift factor tables (setup_kick_drift_factors, comoving.c:109-153)
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_x, 8 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_kick, 8 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_drift, 8 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_m2k, 8 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_m2d, 8 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->kd_work, 16 * KD_TABLE));
	TVG_CHECK(ensure(ctx, (void **) &ctx->tl_scratch, 256));
	if (cfg->comoving) {
		const double a0 = 0.95 * cfg->time_begin;
		const double da = log((1.05 * cfg->time_end) / a0) / (KD_TABLE - 1);
		k_kd_table<<<TVG_CNT(ctx, (KD_TABLE + 127) / 128), 128, 0, s>>>(
		    cosmo(*cfg), a0, da, gauss_legendre(), ctx->kd_x, ctx->kd_kick, ctx->kd_drift);
		TVG_CUDA(ctx, cudaGetLastError());
		k_kd_spline<<<TVG_CNT(ctx, 1), 1, 0, s>>>(ctx->kd_x, ctx->kd_kick, ctx->kd_m2k, ctx->kd_work);
		k_kd_spline<<<TVG_CNT(ctx, 1), 1, 0, s>>>(ctx->kd_x, ctx->kd_drift, ctx->kd_m2d, ctx->kd_work);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	ctx->have_timeline = true;
	return TVG_OK;
}

extern "C" int tvg_download_kick_drift_table(tvg_context *ctx, double *a, double *kick,
                                             double *drift)
{
	if (!ctx || !a || !kick || !drift) return TVG_E_BADINPUT;
	if (!ctx->have_timeline || !ctx->tl.cfg.comoving)
		return tvg_fail(ctx, TVG_E_STATE, "kick/drift table: comoving timeline not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	TVG_CUDA(ctx, cudaMemcpy(a, ctx->kd_x, 8 * KD_TABLE, cudaMemcpyDeviceToHost));
	TVG_CUDA(ctx, cudaMemcpy(kick, ctx->kd_kick, 8 * KD_TABLE, cudaMemcpyDeviceToHost));
	TVG_CUDA(ctx, cudaMemcpy(drift, ctx->kd_drift, 8 * KD_TABLE, cudaMemcpyDeviceToHost));
	return TVG_OK;
}

// Particle_Kick_Step / Particle_Drift_Step for given integer times, from the
// device tables (one thread)
__global__ void k_factor(TimeParams p, uint32_t c, uint32_t n, double *out)
{
	out[0] = kick_step(p, c, n);
	out[1] = drift_step(p, c, n);
}

extern "C" int tvg_kick_drift_factors(tvg_context *ctx, uint32_t it_curr, uint32_t it_next,
                                      double *kick, double *drift)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	double *d = (double *) ctx->tl_scratch, h[2];
	k_factor<<<TVG_CNT(ctx, 1), 1, 0, ctx->stream>>>(time_params(ctx), it_curr, it_next, d);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CUDA(ctx, cudaMemcpyAsync(h, d, 16, cudaMemcpyDeviceToHost, ctx->stream));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	if (kick) *kick = h[0];
	if (drift) *drift = h[1];
	return TVG_OK;
}

// Make_Active_Particle_List on the device; n_active to the host
int tvg_impl_active_from_bins(tvg_context *ctx)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	if (!ctx->active) TVG_CUDA(ctx, cudaMalloc((void **) &ctx->active, 4 * (size_t) ctx->cap));
	TVG_CHECK(ensure(ctx, (void **) &ctx->act_flag, 4 * (size_t) ctx->cap));
	TVG_CHECK(ensure(ctx, (void **) &ctx->act_off, 4 * (size_t) ctx->cap));
	int32_t *flag = ctx->act_flag, *off = ctx->act_off;
	// a captured step is given the limit before its launch (tvg_step_graph)
	if (!ctx->capturing) TVG_CHECK(tvg_set_device_max_bin(ctx));
	k_active_flags<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(
	    n, (const int32_t *) ctx->f[FS_TIME_BIN], ctx->dc, flag);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CHECK(tvg_device_scan_i32_dev(ctx, flag, off, n, &ctx->dc->n_active));
	k_active_scatter<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, flag, off, ctx->active);
	TVG_CUDA(ctx, cudaGetLastError());
	ctx->use_active = true;
	if (ctx->capturing) return TVG_OK;
	int64_t total = 0;
	TVG_CUDA(ctx, cudaMemcpyAsync(&total, &ctx->dc->n_active, 8, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	ctx->n_active = total;
	ctx->tl.state.n_active = total;
	if (total == 0)
		return tvg_fail(ctx, TVG_E_STATE, "no active particles (max active bin %d)",
		                ctx->tl.state.max_active_bin);
	return TVG_OK;
}

template <typename F>
static int velocity_constraint(tvg_context *ctx, double *dt_out)
{
	// Comoving_VelDisp_Timestep_Constraint (comoving.c:195-287)
	const tvg_timeline_config &c = ctx->tl.cfg;
	tvg_timeline_state &st = ctx->tl.state;
	cudaStream_t s = ctx->stream;
	char *scr = (char *) ctx->tl_scratch;
	double *vel2 = (double *) scr;                              // [6]
	uint32_t *mmin = (uint32_t *) (scr + 48);                   // [6]
	unsigned long long *np = (unsigned long long *) (scr + 72); // [6]
	TVG_CUDA(ctx, cudaMemsetAsync(vel2, 0, 48, s));
	TVG_CUDA(ctx, cudaMemsetAsync(mmin, 0x7F, 24, s));
	TVG_CUDA(ctx, cudaMemsetAsync(np, 0, 48, s));
	const int64_t n = ctx->n;
	const unsigned nb = tvg_blocks(n, VD_THREADS * 8) < 148u * 8u ? tvg_blocks(n, VD_THREADS * 8) : 148u * 8u;
	k_veldisp<F><<<TVG_CNT(ctx, nb), VD_THREADS, 0, s>>>(
	    n, (const int32_t *) ctx->f[FS_TYPE], (const F *) ctx->f[FS_VEL0], (const F *) ctx->f[FS_VEL1],
	    (const F *) ctx->f[FS_VEL2], (const F *) ctx->f[FS_MASS], vel2, mmin, np);
	TVG_CUDA(ctx, cudaGetLastError());
	double hv[6];
	uint32_t hm[6];
	unsigned long long hn[6];
	TVG_CUDA(ctx, cudaMemcpyAsync(hv, vel2, 48, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(hm, mmin, 24, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaMemcpyAsync(hn, np, 48, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	const double rho_b = c.omega_baryon * c.rho_crit0;
	const double rho_nb = c.omega_matter * c.rho_crit0 - rho_b;
	double dt_max = DBL_MAX;
	for (int t = 0; t < 6; t++) {
		if (hn[t] == 0) continue;
		float mf;
		memcpy(&mf, &hm[t], 4);
		const double dmean = pow((double) mf / (t == 0 ? rho_b : rho_nb), 1.0 / 3.0);
		const double vrms = sqrt(hv[t] / (double) hn[t]);
		const double dt = c.displ_constraint * dmean / vrms * st.expansion_factor
		                * st.expansion_factor * st.hubble_parameter;
		dt_max = fmin(dt, dt_max);
	}
	*dt_out = dt_max;
	return TVG_OK;
}

template <typename F>
static int set_new_timesteps_typed(tvg_context *ctx)
{
	tvg_timeline_state &st = ctx->tl.state;
	const tvg_timeline_config &c = ctx->tl.cfg;
	cudaStream_t s = ctx->stream;
	const int64_t n = ctx->n;
	if (st.sync_point || st.prepare_step || st.first_step) {
		// set_global_timestep_constraint (timestep.c:533-550)
		double dt = c.max_timestep;
		if (c.comoving) {
			double dv = DBL_MAX;
			TVG_CHECK(velocity_constraint<F>(ctx, &dv));
			dt = fmin(dt, dv);
		}
		st.dt_max_global = (float) dt;
	}
	// set_new_particle_timebins
	BinParams bp;
	bp.grav_accel_factor = c.comoving ? 1.0 / (st.expansion_factor * st.expansion_factor) : 1.0;
	bp.expansion_factor = st.expansion_factor;
	bp.hubble = st.hubble_parameter;
	bp.time_int_accuracy = c.time_int_accuracy;
	bp.softening = ctx->cfg.softening;
	bp.step_max = st.step_max;
	bp.step_min = st.step_min;
	bp.dt_max_global = st.dt_max_global;
	bp.comoving = c.comoving;
	bp.max_active_bin = st.max_active_bin;
	int32_t *mm = (int32_t *) ((char *) ctx->tl_scratch + 128);
	const int32_t init[2] = { N_INT_BINS - 1, 0 };
	TVG_CUDA(ctx, cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, s));
	k_timebins<F><<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(
	    n, bp, (const F *) ctx->f[FS_GACC0], (const F *) ctx->f[FS_GACC1], (const F *) ctx->f[FS_GACC2],
	    (int32_t *) ctx->f[FS_TIME_BIN], mm, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	int32_t h[2];
	TVG_CUDA(ctx, cudaMemcpyAsync(h, mm, 8, cudaMemcpyDeviceToHost, s));
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	TVG_CHECK(tvg_sync_status(ctx, "set_new_timesteps"));
	st.time_bin_min = h[0];
	st.time_bin_max = h[1];
	// set_system_timestep (timestep.c:245-268)
	const uint32_t step_bin = 1u << st.time_bin_min;
	uint32_t step_sync = st.current ? (1u << __builtin_ctz(st.current)) : 0;
	if (st.current == st.beg) step_sync = step_bin;
	const uint32_t step_end = st.end - st.current;
	st.step = step_end < step_bin ? step_end : step_bin;
	if (step_sync < st.step) st.step = step_sync;
	st.next = st.current + st.step;
	st.time_next = host_it2time(ctx, st.next);
	st.time_step = st.time_next - st.time_current;
	// (the reference sets Max_Active_Bin = Time_Bin_Min on the first step,
	// timestep.c:264-265, and overwrites it right after, timestep.c:55)
	// max_active_time_bin (timestep.c:275-278); Int_Time.Next is never 0 here
	st.max_active_bin = st.next ? __builtin_ctz(st.next) : N_INT_BINS - 1;
	st.sync_point = 0;
	if (st.current == st.next_sync_point) {
		st.sync_point = 1;
		st.next_sync_point += 1u << st.time_bin_max;
	}
	return tvg_impl_active_from_bins(ctx);
}

extern "C" int tvg_set_new_timesteps(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (ctx->cfg.float_bytes == 4) TVG_CHECK(set_new_timesteps_typed<float>(ctx));
	else TVG_CHECK(set_new_timesteps_typed<double>(ctx));
	return TVG_OK;
}

template <typename F>
static int kick_typed(tvg_context *ctx)
{
	const int64_t na = ctx->use_active ? ctx->n_active : ctx->n;
	if (na == 0) return TVG_OK;
	// Gravity_Tree_Update_Kicks (kick.c:31-32, 61-62) without a due domain update
	const bool nodes = tvg_tree_update_due(ctx);
	int64_t slots = 0;
	if (nodes) {
		TVG_CHECK(tvg_tree_update_check(ctx, "kick"));
		TVG_CHECK(tvg_impl_active_slots(ctx, &slots));
		void *dpv = nullptr;
		TVG_CHECK(tvg_impl_tree_dp_buffer(ctx, &dpv));
		F *dp = (F *) dpv;
		const int64_t cap = ctx->cap;
		k_kick_dp<F><<<TVG_CNT(ctx, tvg_blocks(ctx->n, 256)), 256, 0, ctx->stream>>>(
		    ctx->n, ctx->act_flag, ctx->act_off, time_params(ctx), (const int32_t *) ctx->f[FS_TIME_BIN],
		    (const uint32_t *) ctx->f[FS_IT_KICK], (const F *) ctx->f[FS_MASS], (const F *) ctx->f[FS_ACC0],
		    (const F *) ctx->f[FS_ACC1], (const F *) ctx->f[FS_ACC2], dp, dp + cap, dp + 2 * cap);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	k_kick<F><<<TVG_CNT(ctx, tvg_blocks(na, KD_THREADS * KD_IPT)), KD_THREADS, 0, ctx->stream>>>(
	    na, ctx->use_active ? ctx->active : nullptr, time_params(ctx),
	    (const int32_t *) ctx->f[FS_TIME_BIN], (uint32_t *) ctx->f[FS_IT_KICK],
	    (const F *) ctx->f[FS_ACC0], (const F *) ctx->f[FS_ACC1], (const F *) ctx->f[FS_ACC2],
	    (F *) ctx->f[FS_VEL0], (F *) ctx->f[FS_VEL1], (F *) ctx->f[FS_VEL2]);
	TVG_CUDA(ctx, cudaGetLastError());
	if (nodes) TVG_CHECK(tvg_impl_tree_kick(ctx, slots));
	return TVG_OK;
}

static int kick(tvg_context *ctx)
{
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (ctx->cfg.float_bytes == 4) TVG_CHECK(kick_typed<float>(ctx));
	else TVG_CHECK(kick_typed<double>(ctx));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}

extern "C" int tvg_kick_first_halfstep(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	return kick(ctx);
}

extern "C" int tvg_kick_second_halfstep(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	TVG_CHECK(kick(ctx));
	ctx->tl.state.first_step = 0;          // Update(AFTER_STEP), update.c
	return TVG_OK;
}

template <typename F>
static int drift_typed(tvg_context *ctx)
{
	tvg_timeline_state &st = ctx->tl.state;
	cudaStream_t s = ctx->stream;
	const int64_t na = ctx->use_active ? ctx->n_active : ctx->n;
	if (na > 0) {
		k_drift<F><<<TVG_CNT(ctx, tvg_blocks(na, KD_THREADS * KD_IPT)), KD_THREADS, 0, s>>>(
		    na, ctx->use_active ? ctx->active : nullptr, time_params(ctx), st.next, st.end,
		    (const int32_t *) ctx->f[FS_TIME_BIN], (uint32_t *) ctx->f[FS_IT_DRIFT], (const F *) ctx->f[FS_VEL0], (const F *) ctx->f[FS_VEL1],
		    (const F *) ctx->f[FS_VEL2], (F *) ctx->f[FS_POS0], (F *) ctx->f[FS_POS1],
		    (F *) ctx->f[FS_POS2], ctx->status);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	// Gravity_Tree_Update_Drift(Time.Step) (drift.c:41-42)
	if (tvg_tree_update_due(ctx)) {
		TVG_CHECK(tvg_tree_update_check(ctx, "drift"));
		TVG_CHECK(tvg_impl_tree_drift(ctx, st.time_step));
	}
	if (ctx->cfg.periodic) {
		k_wrap<F><<<TVG_CNT(ctx, tvg_blocks(ctx->n, 256)), 256, 0, s>>>(
		    ctx->n, (F) ctx->cfg.boxsize, (F *) ctx->f[FS_POS0], (F *) ctx->f[FS_POS1],
		    (F *) ctx->f[FS_POS2], ctx->status);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	TVG_CUDA(ctx, cudaStreamSynchronize(s));
	TVG_CHECK(tvg_sync_status(ctx, "drift"));
	// clock (drift.c:46-59)
	st.current += st.step;
	st.next += st.step;
	st.time_current = host_it2time(ctx, st.current);
	st.time_next = host_it2time(ctx, st.next);
	st.step_counter++;
	set_current_cosmology(ctx);
	if (ctx->tree_updates) {
		// the reference walks the tree it keeps until the next domain update
		ctx->have_walktree = false;
	} else {
		// positions moved: keys, order and tree are stale
		ctx->keys_std = ctx->sorted = ctx->have_top = ctx->have_tree = ctx->have_walktree = false;
	}
	return TVG_OK;
}

extern "C" int tvg_drift_to_sync_point(tvg_context *ctx)
{
	if (!ctx) return TVG_E_BADINPUT;
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	if (ctx->cfg.float_bytes == 4) return drift_typed<float>(ctx);
	return drift_typed<double>(ctx);
}

extern "C" int tvg_timeline_get(tvg_context *ctx, tvg_timeline_state *st)
{
	if (!ctx || !st) return TVG_E_BADINPUT;
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	*st = ctx->tl.state;
	return TVG_OK;
}

extern "C" int tvg_timeline_set(tvg_context *ctx, const tvg_timeline_state *st)
{
	if (!ctx || !st) return TVG_E_BADINPUT;
	if (!ctx->have_timeline) return tvg_fail(ctx, TVG_E_STATE, "timeline not initialised");
	ctx->tl.state = *st;
	return TVG_OK;
}

extern "C" int tvg_rung_histogram(tvg_context *ctx, int32_t *hist)
{
	if (!ctx || !hist) return TVG_E_BADINPUT;
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	int32_t *d = (int32_t *) ((char *) ctx->tl_scratch + 128);
	TVG_CUDA(ctx, cudaMemsetAsync(d, 0, 4 * N_INT_BINS, ctx->stream));
	if (ctx->n > 0) {
		k_bin_hist<<<TVG_CNT(ctx, 148 * 4), 256, 0, ctx->stream>>>(
		    ctx->n, (const int32_t *) ctx->f[FS_TIME_BIN], d);
		TVG_CUDA(ctx, cudaGetLastError());
	}
	TVG_CUDA(ctx, cudaMemcpyAsync(hist, d, 4 * N_INT_BINS, cudaMemcpyDeviceToHost, ctx->stream));
	TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
	return TVG_OK;
}
