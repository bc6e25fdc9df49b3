// tvg_keys.cu -- Peano-Hilbert keys.
//
// Bit-exact with Peano_Key / Reversed_Peano_Key (peano.c:122-276): the
// coordinate is scaled in FP64 exactly as the reference does
// ((p - origin) * (2^63 / size), truncated to uint64) and mapped onto the
// curve of Skilling's Hilbert transpose (2004, AIP Conf. Proc. 707, 381).
// The curve is walked as a finite automaton (tvg_ph_table.inc, generated by
// gen_ph_table.py from the transpose): 24 states, two levels per lookup in a
// shared-memory table, 21 lookups for the key's 42 levels, instead of the
// transpose's 63 conditional 64-bit steps per coordinate. Standard key:
// level k (1..42) at bits 130-3k..128-3k. Reversed key: level k at bits
// 3k+2..3k (levels 1..41, level 42 truncated to its two low bits).
// Roofline: HBM (3 Float in, 16 B out per particle).
#include "tvg_internal.cuh"
#include "tvg_ph_table.inc"

// spread the low 21 bits of v to every third bit (bit i -> bit 3i)
__device__ __forceinline__ uint64_t spread3(uint64_t v)
{
	v &= 0x1FFFFFULL;
	v = (v | (v << 32)) & 0x1F00000000FFFFULL;
	v = (v | (v << 16)) & 0x1F0000FF0000FFULL;
	v = (v | (v << 8)) & 0x100F00F00F00F00FULL;
	v = (v | (v << 4)) & 0x10C30C30C30C30C3ULL;
	v = (v | (v << 2)) & 0x1249249249249249ULL;
	return v;
}

// the two digits of a table entry, first level in the low three bits (the
// order of the reversed key)
__device__ __forceinline__ uint64_t swap_digits(unsigned e)
{
	return (uint64_t) (((e >> 3) & 7u) | ((e & 7u) << 3));
}

// grid-stride: every block copies the 3 KB table into shared memory once
template <typename F, bool REV>
__global__ void __launch_bounds__(256) k_ph_keys(int64_t n, const F *__restrict__ x, const F *__restrict__ y,
                                                 const F *__restrict__ z, double ox, double oy, double oz,
                                                 double fac, uint64_t *__restrict__ key_hi,
                                                 uint64_t *__restrict__ key_lo, int *status)
{
	__shared__ uint16_t tab[TVG_PH_STATES * 64];
	__shared__ uint8_t start[8];
	for (int k = threadIdx.x; k < TVG_PH_STATES * 64; k += blockDim.x) tab[k] = tvg_ph_table2[k];
	if (threadIdx.x < 8) start[threadIdx.x] = tvg_ph_start[threadIdx.x];
	__syncthreads();
	bool bad = false;
	for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
	     i += (int64_t) gridDim.x * blockDim.x) {
		const double px = (double) x[i], py = (double) y[i], pz = (double) z[i];
		const double sx = (px - ox) * fac, sy = (py - oy) * fac, sz = (pz - oz) * fac;
		// the reference converts out-of-range values with undefined results;
		// report them instead (NaN fails both comparisons)
		if (!(sx >= 0.0 && sx < 18446744073709551616.0 && sy >= 0.0 && sy < 18446744073709551616.0
		      && sz >= 0.0 && sz < 18446744073709551616.0))
			bad = true;
		const uint64_t x0 = (uint64_t) sx, x1 = (uint64_t) sy, x2 = (uint64_t) sz;
		// octants of levels 1..21 (coordinate bits 62..42) and 22..42 (41..21),
		// three bits a level, the first level highest
		const uint64_t mh = (spread3(x0 >> 42) << 2) | (spread3(x1 >> 42) << 1) | spread3(x2 >> 42);
		const uint64_t ml = (spread3(x0 >> 21) << 2) | (spread3(x1 >> 21) << 1) | spread3(x2 >> 21);
		// bit 63 (level 0) selects the state of the curve below it
		unsigned st = start[(unsigned) (((x0 >> 63) << 2) | ((x1 >> 63) << 1) | (x2 >> 63))];
		// digits: standard order in dh (levels 1..21) and dl (22..42) like mh,
		// ml; reversed order, level k at bit 3(k-1) of r1 (levels 1..21) and
		// 3(k-22) of r2 (22..42)
		uint64_t dh = 0, dl = 0;
#pragma unroll
		for (int j = 0; j < 10; j++) {             // levels 2j+1, 2j+2
			const unsigned e = tab[st * 64 + (unsigned) ((mh >> (57 - 6 * j)) & 63)];
			st = e >> 6;
			if (REV) dh |= swap_digits(e) << (6 * j);
			else dh |= (uint64_t) (e & 63u) << (57 - 6 * j);
		}
		{                                          // levels 21 and 22 straddle the words
			const unsigned e = tab[st * 64 + (unsigned) (((mh & 7) << 3) | ((ml >> 60) & 7))];
			st = e >> 6;
			if (REV) {
				dh |= (uint64_t) ((e >> 3) & 7u) << 60;
				dl |= (uint64_t) (e & 7u);
			} else {
				dh |= (uint64_t) ((e >> 3) & 7u);
				dl |= (uint64_t) (e & 7u) << 60;
			}
		}
#pragma unroll
		for (int j = 0; j < 10; j++) {             // levels 2j+23, 2j+24
			const unsigned e = tab[st * 64 + (unsigned) ((ml >> (54 - 6 * j)) & 63)];
			st = e >> 6;
			if (REV) dl |= swap_digits(e) << (3 + 6 * j);
			else dl |= (uint64_t) (e & 63u) << (54 - 6 * j);
		}
		if (REV) {
			key_lo[i] = dh << 3;
			key_hi[i] = (dh >> 61) | (dl << 2);
		} else {
			key_hi[i] = (dh << 1) | (dl >> 62);
			key_lo[i] = dl << 2;
		}
	}
	if (bad) atomicOr(status, TVG_ST_BADPOS);
}

template <typename F>
static void launch_keys(tvg_context *ctx, unsigned nb, bool reversed)
{
	const int64_t n = ctx->n;
	const double fac = (double) (1ULL << 63) / ctx->dsize;
	const F *x = (const F *) ctx->f[FS_POS0], *y = (const F *) ctx->f[FS_POS1], *z = (const F *) ctx->f[FS_POS2];
	if (reversed)
		k_ph_keys<F, true><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    n, x, y, z, ctx->origin[0], ctx->origin[1], ctx->origin[2], fac, ctx->key_hi, ctx->key_lo,
		    ctx->status);
	else
		k_ph_keys<F, false><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    n, x, y, z, ctx->origin[0], ctx->origin[1], ctx->origin[2], fac, ctx->key_hi, ctx->key_lo,
		    ctx->status);
}

int tvg_impl_keys(tvg_context *ctx, bool reversed)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	// four particles per thread or 16 blocks per SM, whichever is fewer
	const unsigned nb4 = tvg_blocks(n, 256 * 4), nb = nb4 < 148u * 16u ? nb4 : 148u * 16u;
	if (ctx->cfg.float_bytes == 4) launch_keys<float>(ctx, nb, reversed);
	else launch_keys<double>(ctx, nb, reversed);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}
