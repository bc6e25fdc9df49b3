// tvg_scan.cu -- device-wide exclusive prefix sum of int32 (reduce, scan of
// block sums, apply), 4096 items per block, warp-shuffle block scans.
// No inter-block waits: every phase is its own launch.
#include "tvg_internal.cuh"

#define SCAN_THREADS 512
#define SCAN_IPT 8
#define SCAN_TILE (SCAN_THREADS * SCAN_IPT)

__device__ __forceinline__ int32_t warp_incl_scan(int32_t v)
{
	const int lane = threadIdx.x & 31;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		int32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
		if (lane >= o) v += u;
	}
	return v;
}

// exclusive scan of one value per thread across the block; returns the block total
__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t *excl, int32_t *s_warp)
{
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
	int32_t inc = warp_incl_scan(v);
	if (lane == 31) s_warp[w] = inc;
	__syncthreads();
	if (w == 0) {
		int32_t t = lane < nw ? s_warp[lane] : 0;
		int32_t ti = warp_incl_scan(t);
		if (lane < nw) s_warp[lane] = ti - t;
		if (lane == nw - 1) s_warp[32] = ti;
	}
	__syncthreads();
	*excl = inc - v + s_warp[w];
	int32_t total = s_warp[32];
	__syncthreads();
	return total;
}

__global__ void k_scan_reduce(const int32_t *__restrict__ in, int64_t n, int32_t *__restrict__ sums)
{
	__shared__ int32_t s_warp[33];
	const int64_t base = (int64_t) blockIdx.x * SCAN_TILE;
	int32_t acc = 0;
#pragma unroll
	for (int k = 0; k < SCAN_IPT; k++) {
		int64_t i = base + (int64_t) k * SCAN_THREADS + threadIdx.x;
		if (i < n) acc += in[i];
	}
	int32_t ex;
	int32_t tot = block_excl_scan(acc, &ex, s_warp);
	if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_apply(const int32_t *__restrict__ in, int32_t *__restrict__ out, int64_t n,
                             const int32_t *__restrict__ offs, int64_t *total_out)
{
	__shared__ int32_t s_warp[33];
	const int64_t base = (int64_t) blockIdx.x * SCAN_TILE + (int64_t) threadIdx.x * SCAN_IPT;
	int32_t v[SCAN_IPT];
	int32_t acc = 0;
#pragma unroll
	for (int k = 0; k < SCAN_IPT; k++) {
		int64_t i = base + k;
		v[k] = i < n ? in[i] : 0;
		acc += v[k];
	}
	int32_t ex;
	block_excl_scan(acc, &ex, s_warp);
	int32_t run = ex + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
	for (int k = 0; k < SCAN_IPT; k++) {
		int64_t i = base + k;
		if (i < n) out[i] = run;
		run += v[k];
	}
	// the thread holding the last element: the inclusive sum of everything
	if (total_out && base <= n - 1 && n - 1 < base + SCAN_IPT) *total_out = run;
}

// Recursive exclusive scan; `tmp` must hold the block sums of every level.
static int scan_rec(tvg_context *ctx, const int32_t *in, int32_t *out, int64_t n, int32_t *tmp,
                    size_t tmp_elems, int64_t *total_dev)
{
	const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
	if (nb <= 1) {
		k_scan_apply<<<TVG_CNT(ctx, 1), SCAN_THREADS, 0, ctx->stream>>>(in, out, n, nullptr, total_dev);
		TVG_CUDA(ctx, cudaGetLastError());
		return TVG_OK;
	}
	if ((size_t) (2 * nb) > tmp_elems)
		return tvg_fail(ctx, TVG_E_NOMEM, "scan scratch too small (%lld blocks)", (long long) nb);
	int32_t *sums = tmp, *offs = tmp + nb;
	k_scan_reduce<<<TVG_CNT(ctx, (unsigned) nb), SCAN_THREADS, 0, ctx->stream>>>(in, n, sums);
	TVG_CUDA(ctx, cudaGetLastError());
	TVG_CHECK(scan_rec(ctx, sums, offs, nb, tmp + 2 * nb, tmp_elems - 2 * nb, nullptr));
	k_scan_apply<<<TVG_CNT(ctx, (unsigned) nb), SCAN_THREADS, 0, ctx->stream>>>(in, out, n, offs, total_dev);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}

// out[i] = sum(in[0..i)); *total (if not NULL) receives the full sum, read
// back synchronously. in and out may alias.
int tvg_device_scan_i32(tvg_context *ctx, const int32_t *in, int32_t *out, int64_t n,
                        int64_t *total)
{
	if (n <= 0) {
		if (total) *total = 0;
		return TVG_OK;
	}
	int32_t last_in = 0;
	if (total)
		TVG_CUDA(ctx, cudaMemcpyAsync(&last_in, in + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
	TVG_CHECK(scan_rec(ctx, in, out, n, (int32_t *) ctx->scan_tmp, ctx->scan_tmp_bytes / 4, nullptr));
	if (total) {
		int32_t last_out = 0;
		TVG_CUDA(ctx, cudaMemcpyAsync(&last_out, out + n - 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
		TVG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
		*total = (int64_t) last_out + last_in;
	}
	return TVG_OK;
}

// the total stays on the device (int64 at total_dev); no synchronisation
int tvg_device_scan_i32_dev(tvg_context *ctx, const int32_t *in, int32_t *out, int64_t n,
                            int64_t *total_dev)
{
	if (n <= 0) {
		TVG_CUDA(ctx, cudaMemsetAsync(total_dev, 0, 8, ctx->stream));
		return TVG_OK;
	}
	return scan_rec(ctx, in, out, n, (int32_t *) ctx->scan_tmp, ctx->scan_tmp_bytes / 4, total_dev);
}
