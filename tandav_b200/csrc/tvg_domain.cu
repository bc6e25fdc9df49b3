// tvg_domain.cu -- set_computational_domain (src/domain.c:732-847): the cube
// the keys and node sizes refer to.
//
// Periodic: origin 0, size the box. Isolated: the centre is the median of
// each coordinate (find_domain_center, domain.c:763-801), the size 2.001
// times the largest |x - centre| over all particles and axes, in double
// (find_largest_particle_distance, :805-835), and origin = centre - size / 2.
//
// Median (select.c:95-107) is Select(n >> 1, n, data), the Numerical Recipes
// selection written for arrays indexed from 1 (l = 1, ir = n - 1) and run on
// an array indexed from 0: it returns the (n >> 1)-th smallest of
// data[1 .. n-1] (the first particle in the current order takes no part),
// and data[0] for n = 1. Here that order statistic is found exactly by a
// radix select over the coordinates mapped to ordered unsigned integers: one
// histogram pass per byte, most significant first, each keeping the bucket
// that holds the wanted rank. The centre is kept in Float, as the reference
// keeps it.
// Roofline: HBM bound, one read of a coordinate array per byte of the Float
// (4 or 8 passes per axis) plus one read of the positions for the distance.
#include "tvg_internal.cuh"

namespace {

__device__ __forceinline__ uint32_t ordered(float v)
{
	const uint32_t u = __float_as_uint(v);
	return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ uint64_t ordered(double v)
{
	const uint64_t u = (uint64_t) __double_as_longlong(v);
	return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

// 256-bin histogram of byte `shift` of the ordered values of x[1 .. n-1]
// whose bits under `mask` equal `prefix`
template <typename F, typename U>
__global__ void k_select_hist(int64_t n, const F *__restrict__ x, U prefix, U mask, int shift,
                              uint32_t *__restrict__ hist)
{
	__shared__ uint32_t h[256];
	for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0;
	__syncthreads();
	for (int64_t i = 1 + blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		const U u = ordered(x[i]);
		if ((u & mask) == prefix) atomicAdd(&h[(u >> shift) & 0xFF], 1u);
	}
	__syncthreads();
	for (int b = threadIdx.x; b < 256; b += blockDim.x)
		if (h[b]) atomicAdd(&hist[b], h[b]);
}

// largest |x - c| over the particles and the three axes, in double; the
// non-negative doubles order like their bit patterns
template <typename F>
__global__ void k_max_distance(int64_t n, const F *__restrict__ x, const F *__restrict__ y,
                               const F *__restrict__ z, double cx, double cy, double cz,
                               unsigned long long *__restrict__ out)
{
	double m = 0;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		m = fmax(m, fabs((double) x[i] - cx));
		m = fmax(m, fabs((double) y[i] - cy));
		m = fmax(m, fabs((double) z[i] - cz));
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
	if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long) __double_as_longlong(m));
}

template <typename U> U unordered_bits(U u);
template <> uint32_t unordered_bits(uint32_t u) { return (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u; }
template <> uint64_t unordered_bits(uint64_t u)
{
	return (u & 0x8000000000000000ull) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
}

template <typename F> struct Bits;
template <> struct Bits<float> { typedef uint32_t U; };
template <> struct Bits<double> { typedef uint64_t U; };

// Median of one coordinate array: the (n >> 1)-th smallest of x[1 .. n-1]
template <typename F>
int select_median(tvg_context *ctx, const F *x, int64_t n, uint32_t *d_hist, F *out)
{
	typedef typename Bits<F>::U U;
	cudaStream_t s = ctx->stream;
	if (n == 1) {
		TVG_CUDA(ctx, cudaMemcpyAsync(out, x, sizeof(F), cudaMemcpyDeviceToHost, s));
		TVG_CUDA(ctx, cudaStreamSynchronize(s));
		return TVG_OK;
	}
	uint64_t rank = (uint64_t) (n >> 1) - 1;          // 0-based among x[1 .. n-1]
	U prefix = 0, mask = 0;
	uint32_t h[256];
	const int grid = (int) (tvg_blocks(n, 256) < 148 * 8 ? tvg_blocks(n, 256) : 148 * 8);
	for (int shift = 8 * (int) sizeof(U) - 8; shift >= 0; shift -= 8) {
		TVG_CUDA(ctx, cudaMemsetAsync(d_hist, 0, sizeof(h), s));
		k_select_hist<F, U><<<TVG_CNT(ctx, grid), 256, 0, s>>>(n, x, prefix, mask, shift, d_hist);
		TVG_CUDA(ctx, cudaGetLastError());
		TVG_CUDA(ctx, cudaMemcpyAsync(h, d_hist, sizeof(h), cudaMemcpyDeviceToHost, s));
		TVG_CUDA(ctx, cudaStreamSynchronize(s));
		int b = 0;
		while (b < 255 && rank >= h[b]) rank -= h[b++];
		if (rank >= h[b]) return tvg_fail(ctx, TVG_E_CUDA, "find_domain: selection lost the rank");
		prefix |= (U) b << shift;
		mask |= (U) 0xFF << shift;
	}
	const U bits = unordered_bits<U>(prefix);
	memcpy(out, &bits, sizeof(F));
	return TVG_OK;
}

template <typename F>
int find_domain_typed(tvg_context *ctx, double origin[3], double *size)
{
	const int64_t n = ctx->n;
	cudaStream_t s = ctx->stream;
	const F *x[3] = { (const F *) ctx->f[FS_POS0], (const F *) ctx->f[FS_POS1], (const F *) ctx->f[FS_POS2] };
	// scratch: the sort's tile histograms (at least 2 x 1 KB, free between
	// sorts) hold the 256 digit counts and the maximum distance
	void *scratch = ctx->sort_hist;
	uint32_t *d_hist = (uint32_t *) scratch;
	unsigned long long *d_max = (unsigned long long *) ((char *) scratch + 256 * 4);
	double center[3];
	int rc = TVG_OK;
	for (int d = 0; d < 3 && rc == TVG_OK; d++) {
		F c = 0;
		rc = select_median<F>(ctx, x[d], n, d_hist, &c);
		center[d] = (double) c;                       // Float center[3] (domain.c:767)
	}
	if (rc == TVG_OK) {
		const int grid = (int) (tvg_blocks(n, 256) < 148 * 8 ? tvg_blocks(n, 256) : 148 * 8);
		unsigned long long m = 0;
		cudaError_t e = cudaMemsetAsync(d_max, 0, 8, s);
		if (e == cudaSuccess) {
			k_max_distance<F><<<TVG_CNT(ctx, grid), 256, 0, s>>>(n, x[0], x[1], x[2], center[0],
			                                                       center[1], center[2], d_max);
			e = cudaGetLastError();
		}
		if (e == cudaSuccess) e = cudaMemcpyAsync(&m, d_max, 8, cudaMemcpyDeviceToHost, s);
		if (e == cudaSuccess) e = cudaStreamSynchronize(s);
		if (e != cudaSuccess) rc = tvg_fail(ctx, TVG_E_CUDA, "find_domain: %s", cudaGetErrorString(e));
		double maxd;
		memcpy(&maxd, &m, 8);
		*size = 2.001 * maxd;                           // domain.c:832
		for (int d = 0; d < 3; d++) origin[d] = center[d] - 0.5 * *size;
	}
	return rc;
}

} // namespace

extern "C" int tvg_find_domain(tvg_context *ctx, double origin[3], double *size)
{
	if (!ctx || !origin || !size) return TVG_E_BADINPUT;
	if (ctx->n <= 0) return tvg_fail(ctx, TVG_E_STATE, "find_domain: no particles");
	TVG_CUDA(ctx, cudaSetDevice(ctx->device));
	double o[3], sz = 0;
	if (ctx->cfg.periodic) {                            // domain.c:732-747
		sz = ctx->cfg.boxsize;
		o[0] = o[1] = o[2] = 0;
	} else {
		const int rc = ctx->cfg.float_bytes == 4 ? find_domain_typed<float>(ctx, o, &sz)
		                                         : find_domain_typed<double>(ctx, o, &sz);
		if (rc != TVG_OK) return rc;
	}
	for (int d = 0; d < 3; d++) origin[d] = o[d];
	*size = sz;
	return tvg_set_domain(ctx, o, sz);
}
