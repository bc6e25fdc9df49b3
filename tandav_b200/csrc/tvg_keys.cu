// tvg_keys.cu -- Peano-Hilbert keys, one thread per particle.
//
// Bit-exact with Peano_Key / Reversed_Peano_Key (peano.c:122-276): the
// coordinate is scaled in FP64 exactly as the reference does
// ((p - origin) * (2^63 / size), truncated to uint64), converted to the
// Hilbert transpose of Skilling (2004, AIP Conf. Proc. 707, 381), and
// interleaved. Standard key: level k (1..42) at bits 130-3k..128-3k.
// Reversed key: level k at bits 3k+2..3k (levels 0..41, level 42 truncated).
// Roofline: HBM-bound on paper (3 Float in, 16 B out per particle); the 189
// conditional 64-bit XOR steps make it issue-bound at small Float widths.
#include "tvg_internal.cuh"

__device__ __forceinline__ void hilbert_transpose(uint64_t &x0, uint64_t &x1, uint64_t &x2)
{
#pragma unroll 4
	for (int b = 63; b >= 1; b--) {
		const uint64_t q = 1ULL << b, mask = q - 1;
		// i = 0: invert low bits of x0 when its bit b is set
		if (x0 & q) x0 ^= mask;
		// i = 1, 2: invert x0 or exchange low bits with x0
		if (x1 & q) {
			x0 ^= mask;
		} else {
			uint64_t t = (x0 ^ x1) & mask;
			x0 ^= t;
			x1 ^= t;
		}
		if (x2 & q) {
			x0 ^= mask;
		} else {
			uint64_t t = (x0 ^ x2) & mask;
			x0 ^= t;
			x2 ^= t;
		}
	}
	// Gray encode
	x1 ^= x0;
	x2 ^= x1;
	// bit b of `above` = parity of the bits of x2 strictly above b
	uint64_t p = x2;
	p ^= p >> 1;
	p ^= p >> 2;
	p ^= p >> 4;
	p ^= p >> 8;
	p ^= p >> 16;
	p ^= p >> 32;           // bit b = parity of bits >= b
	uint64_t above = p ^ x2;
	x0 ^= above;
	x1 ^= above;
	x2 ^= above;
}

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

// reverse the order of the low 21 bits
__device__ __forceinline__ uint64_t rev21(uint64_t v)
{
	return __brevll(v) >> 43;
}

template <typename F>
__global__ void k_ph_keys(int64_t n, const F *__restrict__ x, const F *__restrict__ y,
                          const F *__restrict__ z, double ox, double oy, double oz, double fac,
                          int reversed, uint64_t *__restrict__ key_hi,
                          uint64_t *__restrict__ key_lo, int *status)
{
	int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
	if (i >= n) return;
	const double px = (double) x[i], py = (double) y[i], pz = (double) z[i];
	const double sx = (px - ox) * fac, sy = (py - oy) * fac, sz = (pz - oz) * fac;
	// the reference converts out-of-range values with undefined results;
	// report them instead (NaN fails both comparisons)
	if (!(sx >= 0.0 && sx < 18446744073709551616.0 && sy >= 0.0 && sy < 18446744073709551616.0
	      && sz >= 0.0 && sz < 18446744073709551616.0))
		atomicOr(status, TVG_ST_BADPOS);
	uint64_t x0 = (uint64_t) sx, x1 = (uint64_t) sy, x2 = (uint64_t) sz;
	hilbert_transpose(x0, x1, x2);
	uint64_t hi, lo;
	if (!reversed) {
		// levels 1..21 (bits 62..42 of X) -> key bits 127..65; level 22
		// (bit 41) straddles the words; levels 23..42 (bits 40..21) -> 63..2
		uint64_t a = (x0 >> 42) & 0x1FFFFF, b = (x1 >> 42) & 0x1FFFFF, c = (x2 >> 42) & 0x1FFFFF;
		uint64_t top = (spread3(a) << 2) | (spread3(b) << 1) | spread3(c);   // 63 bits
		uint64_t t22 = (((x0 >> 41) & 1) << 2) | (((x1 >> 41) & 1) << 1) | ((x2 >> 41) & 1);
		uint64_t d = (x0 >> 21) & 0xFFFFF, e = (x1 >> 21) & 0xFFFFF, f = (x2 >> 21) & 0xFFFFF;
		uint64_t low = (spread3(d) << 2) | (spread3(e) << 1) | spread3(f);   // 60 bits
		hi = (top << 1) | (t22 >> 2);
		lo = (t22 << 62) | (low << 2);
	} else {
		// level k (bit 63-k of X) at key bits 3k+2..3k, k = 1..41; level 42
		// keeps its two low bits at 127..126
		// levels 1..21 -> bits 5..65: reversed order of X bits 62..42
		uint64_t a = rev21((x0 >> 42) & 0x1FFFFF), b = rev21((x1 >> 42) & 0x1FFFFF),
		         c = rev21((x2 >> 42) & 0x1FFFFF);
		// after reversal, bit j (0..20) holds level j+1
		uint64_t s1 = (spread3(a) << 2) | (spread3(b) << 1) | spread3(c);  // level j+1 at 3j
		// levels 22..41 -> bits 66..125: X bits 41..22, reversed (20 bits)
		uint64_t d = __brevll((x0 >> 22) & 0xFFFFF) >> 44, e = __brevll((x1 >> 22) & 0xFFFFF) >> 44,
		         f = __brevll((x2 >> 22) & 0xFFFFF) >> 44;
		uint64_t s2 = (spread3(d) << 2) | (spread3(e) << 1) | spread3(f);  // level j+22 at 3j
		uint64_t t42 = (((x1 >> 21) & 1) << 1) | ((x2 >> 21) & 1);            // low 2 bits
		// s1 placed at bit 3 (level 1 at bits 5..3); s2 at bit 66
		lo = s1 << 3;
		hi = (s1 >> 61) | (s2 << 2) | (t42 << 62);
	}
	key_hi[i] = hi;
	key_lo[i] = lo;
}

int tvg_impl_keys(tvg_context *ctx, bool reversed)
{
	const int64_t n = ctx->n;
	if (n == 0) return TVG_OK;
	const double fac = (double) (1ULL << 63) / ctx->dsize;
	const unsigned nb = tvg_blocks(n, 256);
	if (ctx->cfg.float_bytes == 4)
		k_ph_keys<float><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    n, (const float *) ctx->f[FS_POS0], (const float *) ctx->f[FS_POS1],
		    (const float *) ctx->f[FS_POS2], ctx->origin[0], ctx->origin[1], ctx->origin[2], fac,
		    reversed, ctx->key_hi, ctx->key_lo, ctx->status);
	else
		k_ph_keys<double><<<TVG_CNT(ctx, nb), 256, 0, ctx->stream>>>(
		    n, (const double *) ctx->f[FS_POS0], (const double *) ctx->f[FS_POS1],
		    (const double *) ctx->f[FS_POS2], ctx->origin[0], ctx->origin[1], ctx->origin[2], fac,
		    reversed, ctx->key_hi, ctx->key_lo, ctx->status);
	TVG_CUDA(ctx, cudaGetLastError());
	return TVG_OK;
}
