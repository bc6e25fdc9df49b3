// tvg_sort.cu -- PH-order sort of all particle fields.
//
// Replaces Qsort_Index on the 128-bit keys (sort.c:90-341, cmp_peanoKeys at
// peano.c:6-12) and reorder_collisionless_particles (peano.c:50-82).
//  1. LSD radix sort of (key_hi, index) on the 64-bit high key word: 8-bit
//     digits; a digit that is equal for every key (decided on the device) is
//     not ranked: its pass copies the keys through, so the number of passes,
//     and with it the buffer a step ends in, never depends on the data. Each
//     pass is
//     reduce-then-scan: per-tile (4096 keys) digit histograms, one device
//     scan of the digit-major histogram, then a scatter in which every tile
//     ranks its keys stably with warp __match_any_sync and writes them through
//     a shared-memory staging sort (coalesced runs per digit).
//  2. Runs of equal high words are ordered by the low word (insertion sort
//     per run, one thread per run; runs are rare and short unless positions
//     coincide).
//  3. Every particle field is gathered through the permutation in one launch,
//     four particles per thread with 128-bit stores (and 128-bit loads where
//     the permutation keeps an aligned run of four in place).
// The resulting order is the ascending 128-bit key order, equal keys in
// input order (the reference's quicksort leaves equal keys in an
// unspecified order).
// Roofline: HBM bound; per pass 8 B read (histogram) + 12 B read + 12 B write
// per key.
#include <mutex>

#include "tvg_internal.cuh"

#define RS_THREADS 256
#define RS_IPT 16
#define RS_TILE (RS_THREADS * RS_IPT)
#define RS_WARPS (RS_THREADS / 32)

__global__ void k_iota(int64_t n, uint32_t *p)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) p[i] = (uint32_t) i;
}

// global histogram of all 8 digits of key_hi (to skip constant digits)
__global__ void k_digit_counts(int64_t n, const uint64_t *__restrict__ key, uint32_t *count)
{
	__shared__ uint32_t h[8 * 256];
	for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) h[i] = 0;
	__syncthreads();
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		uint64_t k = key[i];
#pragma unroll
		for (int d = 0; d < 8; d++) atomicAdd(&h[d * 256 + ((k >> (8 * d)) & 0xFF)], 1u);
	}
	__syncthreads();
	for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x)
		if (h[i]) atomicAdd(&count[i], h[i]);
}

// skip[d] = 1 when digit d has the same value in all n keys
__global__ void k_digit_skip(int64_t n, const uint32_t *__restrict__ count, int32_t *skip)
{
	const int d = threadIdx.x;
	if (d >= 8) return;
	int sk = 0;
	for (int b = 0; b < 256; b++)
		if (count[d * 256 + b] == (uint32_t) n) sk = 1;
	skip[d] = sk;
}

// per-tile digit histogram, stored digit-major: hist[d * ntiles + tile]
// (zeros for a digit that skip marks)
__global__ void k_tile_hist(int64_t n, int shift, const uint64_t *__restrict__ key,
                            uint32_t *__restrict__ hist, int64_t ntiles,
                            const int32_t *__restrict__ skip = nullptr)
{
	if (skip && skip[shift >> 3]) {
		hist[(int64_t) threadIdx.x * ntiles + blockIdx.x] = 0;
		return;
	}
	__shared__ uint32_t h[256];
	h[threadIdx.x] = 0;
	__syncthreads();
	const int64_t base = (int64_t) blockIdx.x * RS_TILE;
#pragma unroll 4
	for (int k = 0; k < RS_IPT; k++) {
		int64_t i = base + (int64_t) k * RS_THREADS + threadIdx.x;
		if (i < n) {
			uint32_t d = (uint32_t) (key[i] >> shift) & 0xFF;
			unsigned peers = __match_any_sync(__activemask(), d);
			int leader = __ffs(peers) - 1;
			if ((int) (threadIdx.x & 31) == leader) atomicAdd(&h[d], (uint32_t) __popc(peers));
		}
	}
	__syncthreads();
	hist[(int64_t) threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS)
k_radix_scatter(int64_t n, int shift, const uint64_t *__restrict__ kin,
                const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
                uint32_t *__restrict__ vout, const uint32_t *__restrict__ off, int64_t ntiles,
                const int32_t *__restrict__ skip = nullptr)
{
	if (skip && skip[shift >> 3]) {     // constant digit: the order stays
		const int64_t b0 = (int64_t) blockIdx.x * RS_TILE;
		const int c0 = (int) min((int64_t) RS_TILE, n - b0);
		for (int p = threadIdx.x; p < c0; p += RS_THREADS) {
			kout[b0 + p] = kin[b0 + p];
			vout[b0 + p] = vin[b0 + p];
		}
		return;
	}
	extern __shared__ __align__(16) unsigned char smem[];
	uint64_t *skey = (uint64_t *) smem;                          // RS_TILE
	uint32_t *sval = (uint32_t *) (skey + RS_TILE);              // RS_TILE
	uint32_t *whist = sval + RS_TILE;                            // RS_WARPS * 256
	uint32_t *dstart = whist + RS_WARPS * 256;                   // 256
	uint32_t *gstart = dstart + 256;                             // 256
	uint32_t *running = gstart + 256;                            // 256
	int32_t *s_warp = (int32_t *) (running + 256);               // 33

	const int t = threadIdx.x, lane = t & 31, w = t >> 5;
	const int64_t base = (int64_t) blockIdx.x * RS_TILE;
	const int cnt = (int) min((int64_t) RS_TILE, n - base);
	for (int i = t; i < RS_WARPS * 256; i += RS_THREADS) whist[i] = 0;
	running[t] = 0;
	gstart[t] = off[(int64_t) t * ntiles + blockIdx.x];
	__syncthreads();
	// tile digit counts -> tile-local exclusive offsets
	for (int r = 0; r < RS_IPT; r++) {
		int idx = r * RS_THREADS + t;
		if (idx < cnt) {
			uint32_t d = (uint32_t) (kin[base + idx] >> shift) & 0xFF;
			unsigned peers = __match_any_sync(__activemask(), d);
			if (lane == __ffs(peers) - 1) atomicAdd(&running[d], (uint32_t) __popc(peers));
		}
	}
	__syncthreads();
	{
		int32_t c = (int32_t) running[t], ex;
		// 256 threads: reuse the generic block scan pattern
		int32_t inc = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			int32_t u = __shfl_up_sync(0xFFFFFFFFu, inc, o);
			if (lane >= o) inc += u;
		}
		if (lane == 31) s_warp[w] = inc;
		__syncthreads();
		if (w == 0) {
			int32_t v = lane < RS_WARPS ? s_warp[lane] : 0;
			int32_t vi = v;
#pragma unroll
			for (int o = 1; o < 32; o <<= 1) {
				int32_t u = __shfl_up_sync(0xFFFFFFFFu, vi, o);
				if (lane >= o) vi += u;
			}
			if (lane < RS_WARPS) s_warp[lane] = vi - v;
		}
		__syncthreads();
		ex = inc - c + s_warp[w];
		dstart[t] = (uint32_t) ex;
		running[t] = 0;
	}
	__syncthreads();
	const unsigned lt_mask = (1u << lane) - 1u;
	for (int r = 0; r < RS_IPT; r++) {
		const int idx = r * RS_THREADS + t;
		const bool valid = idx < cnt;
		uint64_t k = 0;
		uint32_t v = 0, d = 256 + lane;      // invalid lanes match nobody
		if (valid) {
			k = kin[base + idx];
			v = vin[base + idx];
			d = (uint32_t) (k >> shift) & 0xFF;
		}
		unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
		int rank_w = __popc(peers & lt_mask);
		if (valid && rank_w == 0) whist[w * 256 + d] = (uint32_t) __popc(peers);
		__syncthreads();
		{   // per digit: exclusive prefix over warps, continuing the running count
			uint32_t run = running[t];
#pragma unroll
			for (int ww = 0; ww < RS_WARPS; ww++) {
				uint32_t c = whist[ww * 256 + t];
				whist[ww * 256 + t] = run;
				run += c;
			}
			running[t] = run;
		}
		__syncthreads();
		if (valid) {
			uint32_t pos = dstart[d] + whist[w * 256 + d] + (uint32_t) rank_w;
			skey[pos] = k;
			sval[pos] = v;
		}
		__syncthreads();
		for (int ww = 0; ww < RS_WARPS; ww++) whist[ww * 256 + t] = 0;
		__syncthreads();
	}
	for (int p = t; p < cnt; p += RS_THREADS) {
		uint64_t k = skey[p];
		uint32_t d = (uint32_t) (k >> shift) & 0xFF;
		int64_t dest = (int64_t) gstart[d] + (p - (int) dstart[d]);
		kout[dest] = k;
		vout[dest] = sval[p];
	}
}

// Orders runs of equal key_hi by the low key word, stably (the radix passes
// sort the high words only): out = perm with each run reordered. Every
// element of a run finds the run's ends and its rank by one pass over the run,
// in parallel, so a run of r equal high words costs O(r) time on r threads;
// elements outside runs are copied.
__global__ void k_tie_rank(int64_t n, const uint64_t *__restrict__ hi, const uint64_t *__restrict__ lo_orig,
                           const uint32_t *__restrict__ perm, uint32_t *__restrict__ out)
{
	const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	const uint64_t h = hi[i];
	const uint32_t pv = perm[i];
	if (!((i > 0 && hi[i - 1] == h) || (i + 1 < n && hi[i + 1] == h))) {
		out[i] = pv;
		return;
	}
	int64_t a = i, e = i + 1;
	while (a > 0 && hi[a - 1] == h) a--;
	while (e < n && hi[e] == h) e++;
	const uint64_t kv = lo_orig[pv];
	int64_t r = 0;
	for (int64_t j = a; j < e; j++) {
		const uint64_t kj = lo_orig[perm[j]];
		r += (kj < kv || (kj == kv && j < i)) ? 1 : 0;
	}
	out[a + r] = pv;
}

__global__ void k_gather_u64(int64_t n, const uint32_t *__restrict__ perm, const uint64_t *__restrict__ in,
                             uint64_t *__restrict__ out)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i < n) out[i] = in[perm[i]];
}

struct GatherList {
	const void *in[FS_NFIELDS];
	void *out[FS_NFIELDS];
	int bytes[FS_NFIELDS];
	int nf;
};

// All particle fields through the permutation in one pass (perm read once).
// A thread moves four consecutive particles i .. i+3 (i a multiple of 4):
// their permutation entries come in one 128-bit load, and every field is
// written with 128-bit stores (one per 4-byte field, two per 8-byte field).
// Where the four sources are one aligned run (perm[i] a multiple of 4 and
// perm[i+k] = perm[i] + k: particles that kept their place in the order,
// nearly all of them between the steps of a run) the loads are 128-bit too;
// elsewhere the four elements are gathered one by one. Buffers start
// 256-byte aligned, so every vector access is aligned.
__global__ void k_gather_fields(int64_t n, const uint32_t *__restrict__ perm, GatherList g)
{
	const int64_t i = 4 * (blockIdx.x * (int64_t) blockDim.x + threadIdx.x);
	if (i >= n) return;
	if (i + 4 > n) {                               // ragged end: scalar
		for (int64_t j = i; j < n; j++) {
			const uint32_t src = perm[j];
			for (int f = 0; f < g.nf; f++) {
				if (g.bytes[f] == 8) ((uint64_t *) g.out[f])[j] = ((const uint64_t *) g.in[f])[src];
				else ((uint32_t *) g.out[f])[j] = ((const uint32_t *) g.in[f])[src];
			}
		}
		return;
	}
	const uint4 p = *(const uint4 *) (perm + i);
	const bool run = (p.x & 3u) == 0 && p.y == p.x + 1 && p.z == p.x + 2 && p.w == p.x + 3;
	for (int f = 0; f < g.nf; f++) {
		if (g.bytes[f] == 8) {
			const uint64_t *in = (const uint64_t *) g.in[f];
			uint4 *out = (uint4 *) ((uint64_t *) g.out[f] + i);
			if (run) {
				const uint4 *v = (const uint4 *) (in + p.x);
				out[0] = __ldg(v);
				out[1] = __ldg(v + 1);
			} else {
				const uint64_t a = in[p.x], b = in[p.y], c = in[p.z], d = in[p.w];
				out[0] = make_uint4((uint32_t) a, (uint32_t) (a >> 32), (uint32_t) b, (uint32_t) (b >> 32));
				out[1] = make_uint4((uint32_t) c, (uint32_t) (c >> 32), (uint32_t) d, (uint32_t) (d >> 32));
			}
		} else {
			const uint32_t *in = (const uint32_t *) g.in[f];
			uint4 *out = (uint4 *) ((uint32_t *) g.out[f] + i);
			if (run) *out = __ldg((const uint4 *) (in + p.x));
			else *out = make_uint4(in[p.x], in[p.y], in[p.z], in[p.w]);
		}
	}
}

// k_radix_scatter's dynamic shared memory (above the 48 KB default) is a
// function attribute of each device: set it once for every device the
// process sorts on
static cudaError_t radix_smem_attr(size_t smem)
{
	static std::mutex mu;
	static bool done[TVG_MAX_DEVICES] = { false };
	int device = 0;
	cudaError_t e = cudaGetDevice(&device);
	if (e != cudaSuccess) return e;
	if (device < 0 || device >= TVG_MAX_DEVICES) return cudaErrorInvalidDevice;
	std::lock_guard<std::mutex> lock(mu);
	if (done[device]) return cudaSuccess;
	e = cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
	if (e == cudaSuccess) done[device] = true;
	return e;
}

int tvg_impl_sort(tvg_context *ctx, uint32_t *perm_out)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	cudaStream_t s = ctx->stream;
	const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
	k_iota<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->perm);
	TVG_CUDA(ctx, cudaMemsetAsync(ctx->digit_count, 0, 4 * 8 * 256, s));
	k_digit_counts<<<TVG_CNT(ctx, 296), 512, 0, s>>>(n, ctx->key_hi, ctx->digit_count);
	int32_t *skip = ctx->dc->sort_skip;
	k_digit_skip<<<TVG_CNT(ctx, 1), 32, 0, s>>>(n, ctx->digit_count, skip);
	TVG_CUDA(ctx, cudaGetLastError());
	const size_t smem = RS_TILE * 12 + (RS_WARPS * 256 + 3 * 256 + 33) * 4;
	TVG_CUDA(ctx, radix_smem_attr(smem));
	uint64_t *kin = ctx->key_hi, *kout = ctx->key_tmp;
	uint32_t *vin = ctx->perm, *vout = ctx->perm_tmp;
	for (int d = 0; d < 8; d++) {
		const int shift = 8 * d;
		k_tile_hist<<<TVG_CNT(ctx, (unsigned) ntiles), RS_THREADS, 0, s>>>(n, shift, kin, ctx->sort_hist, ntiles,
		                                                                   skip);
		TVG_CUDA(ctx, cudaGetLastError());
		TVG_CHECK(tvg_device_scan_i32(ctx, (const int32_t *) ctx->sort_hist, (int32_t *) ctx->sort_off,
		                              256 * ntiles, nullptr));
		k_radix_scatter<<<TVG_CNT(ctx, (unsigned) ntiles), RS_THREADS, smem, s>>>(n, shift, kin, vin, kout, vout,
		                                                            ctx->sort_off, ntiles, skip);
		TVG_CUDA(ctx, cudaGetLastError());
		uint64_t *kt = kin; kin = kout; kout = kt;
		uint32_t *vt = vin; vin = vout; vout = vt;
	}
	ctx->key_hi = kin; ctx->key_tmp = kout;
	// runs of equal high words by the low words, into the other buffer
	k_tie_rank<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, kin, ctx->key_lo, vin, vout);
	ctx->perm = vout; ctx->perm_tmp = vin;
	k_gather_u64<<<TVG_CNT(ctx, tvg_blocks(n, 256)), 256, 0, s>>>(n, ctx->perm, ctx->key_lo, ctx->key_tmp);
	{ uint64_t *t = ctx->key_lo; ctx->key_lo = ctx->key_tmp; ctx->key_tmp = t; }
	GatherList g;
	g.nf = 0;
	for (int f = 0; f < FS_NFIELDS; f++) {
		g.in[g.nf] = ctx->f[f];
		g.out[g.nf] = ctx->falt[f];
		g.bytes[g.nf] = (int) tvg_field_bytes(ctx, f);
		g.nf++;
	}
	if (ctx->gather_wait) TVG_CUDA(ctx, cudaStreamWaitEvent(s, ctx->gather_wait, 0));
	k_gather_fields<<<TVG_CNT(ctx, tvg_blocks((n + 3) / 4, 256)), 256, 0, s>>>(n, ctx->perm, g);
	TVG_CUDA(ctx, cudaGetLastError());
	for (int f = 0; f < FS_NFIELDS; f++) { void *t = ctx->f[f]; ctx->f[f] = ctx->falt[f]; ctx->falt[f] = t; }
	if (perm_out)
		TVG_CUDA(ctx, cudaMemcpyAsync(perm_out, ctx->perm, 4 * n, cudaMemcpyDeviceToHost, s));
	return TVG_OK;
}

// ------------------------------------------------------------------------
// Sort without any allocation (tvg_sort_keys_noalloc).
//
// Some callers cannot allocate device memory: a host code whose own memory
// manager reserves the GPU's memory up front and forbids allocations behind
// its back, or a latency-bound step loop that cannot pay the device-wide
// synchronisation that cudaMalloc and cudaFree imply. For them this variant
// of the sort keeps its scratch (the
// key and index ping-pong buffers and the digit histograms) in one file-scope
// device array of fixed size, so a call allocates nothing; the caller passes
// the keys and receives the permutation in its own device buffers.
//
// The array belongs to every GPU that loads this library, for the life of the
// process (about 6.4 MB). All calls on a device share it and it keeps the
// last call's contents: each pass rewrites every histogram entry it reads, so
// nothing has to start at zero. Two calls that overlap on the same GPU (from
// two host threads, or on two streams) corrupt each other's scratch.
// ------------------------------------------------------------------------

#define NOALLOC_TILES (TVG_NOALLOC_MAX_KEYS / RS_TILE)

struct NoallocScratch {
	uint64_t key[2][TVG_NOALLOC_MAX_KEYS];   // sorted high words, ping-pong
	uint32_t idx[2][TVG_NOALLOC_MAX_KEYS];   // permutation, ping-pong
	uint32_t hist[256 * NOALLOC_TILES];      // per-tile digit counts (digit-major)
	uint32_t off[256 * NOALLOC_TILES];       // their exclusive prefix sum
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoallocScratch)];

// single-block exclusive prefix sum of up to 1024 * 16 counts
__global__ void __launch_bounds__(1024) k_scan_small(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, int n)
{
	__shared__ uint32_t s_warp[32];
	const int t = threadIdx.x, lane = t & 31, w = t >> 5;
	uint32_t v[16], sum = 0;
#pragma unroll
	for (int k = 0; k < 16; k++) {
		const int i = t * 16 + k;
		v[k] = i < n ? in[i] : 0u;
		sum += v[k];
	}
	uint32_t inc = sum;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint32_t u = __shfl_up_sync(0xFFFFFFFFu, inc, o);
		if (lane >= o) inc += u;
	}
	if (lane == 31) s_warp[w] = inc;
	__syncthreads();
	if (w == 0) {
		uint32_t x = s_warp[lane], xi = x;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			uint32_t u = __shfl_up_sync(0xFFFFFFFFu, xi, o);
			if (lane >= o) xi += u;
		}
		s_warp[lane] = xi - x;
	}
	__syncthreads();
	uint32_t run = inc - sum + s_warp[w];
#pragma unroll
	for (int k = 0; k < 16; k++) {
		const int i = t * 16 + k;
		if (i < n) out[i] = run;
		run += v[k];
	}
}

// Device address of the scratch array, looked up once per device with that
// device current (the host-side symbol is not a device address).
static NoallocScratch *noalloc_scratch(int device)
{
	static std::mutex mu;
	static NoallocScratch *addr[64] = { nullptr };
	if (device < 0 || device >= 64) return nullptr;
	std::lock_guard<std::mutex> lock(mu);
	if (!addr[device]) {
		void *p = nullptr;
		if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
			cudaGetLastError();
			return nullptr;
		}
		addr[device] = (NoallocScratch *) p;
	}
	return addr[device];
}

extern "C" int tvg_sort_keys_noalloc(const uint64_t *key_hi, const uint64_t *key_lo, int64_t n,
                                     uint32_t *perm)
{
	if (n < 0 || n > TVG_NOALLOC_MAX_KEYS) return TVG_E_BADINPUT;
	if (n == 0) return TVG_OK;
	if (!key_hi || !key_lo || !perm) return TVG_E_BADINPUT;
	int device = 0;
	if (cudaGetDevice(&device) != cudaSuccess) { cudaGetLastError(); return TVG_E_CUDA; }
	NoallocScratch *S = noalloc_scratch(device);
	if (!S) return TVG_E_CUDA;
	const size_t smem = RS_TILE * 12 + (RS_WARPS * 256 + 3 * 256 + 33) * 4;
	if (radix_smem_attr(smem) != cudaSuccess) { cudaGetLastError(); return TVG_E_CUDA; }
	const int64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
	cudaStream_t s = 0;
	k_iota<<<tvg_blocks(n, 256), 256, 0, s>>>(n, S->idx[0]);
	const uint64_t *kin = key_hi;
	int cur = 0;
	for (int d = 0; d < 8; d++) {
		const int shift = 8 * d;
		uint64_t *kout = S->key[d & 1];
		k_tile_hist<<<(unsigned) ntiles, RS_THREADS, 0, s>>>(n, shift, kin, S->hist, ntiles);
		k_scan_small<<<1, 1024, 0, s>>>(S->hist, S->off, (int) (256 * ntiles));
		k_radix_scatter<<<(unsigned) ntiles, RS_THREADS, smem, s>>>(n, shift, kin, S->idx[cur], kout,
		                                                            S->idx[cur ^ 1], S->off, ntiles);
		kin = kout;
		cur ^= 1;
	}
	k_tie_rank<<<tvg_blocks(n, 256), 256, 0, s>>>(n, kin, key_lo, S->idx[cur], perm);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaStreamSynchronize(s);
	return e == cudaSuccess ? TVG_OK : TVG_E_CUDA;
}
