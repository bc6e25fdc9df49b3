// tvg_snapshot.cu -- Gadget format-2 snapshot files (Write_Snapshot,
// IO/write_snapshot.c:13-328; block table IO/io.h:68-89) for one rank and
// one file: the 256-byte header, then POS, VEL, ID, MASS and the optional
// ACC, GACC, GPOT blocks, each preceded by the format-2 label record
// ("NAME", size + 8) and framed by 4-byte Fortran record markers. Multi-
// component fields are interleaved per particle (fill_data_buffer,
// write_snapshot.c:230-272). Host code: the context variant downloads one
// block's fields at a time (in the device order, which after a sort is the
// PH order the reference writes in), so it stages three components of n
// particles at most, as the reference's write buffer does.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "tvg_internal.cuh"

namespace {

struct Writer {
	FILE *fp;
	bool ok = true;
	void raw(const void *d, size_t n)
	{
		if (ok && n && fwrite(d, 1, n, fp) != n) ok = false;
	}
	void u32(uint32_t v) { raw(&v, 4); }
	// format-2 label record, then the record marker that opens the data
	void begin(const char *label, uint32_t bytes)
	{
		u32(8);
		raw(label, 4);
		u32(bytes + 8);
		u32(8);
		u32(bytes);
	}
};

// the header as struct gadget_header (io.h:24-44) lays it out; the fill bytes
// (which the reference leaves unset) are zero
void header_bytes(const tvg_snapshot_header *h, unsigned char out[256])
{
	memset(out, 0, 256);
	for (int t = 0; t < 6; t++) {
		const uint32_t lo = (uint32_t) h->nall[t], hi = (uint32_t) (h->nall[t] >> 32);
		memcpy(out + 4 * t, &h->npart[t], 4);
		memcpy(out + 24 + 8 * t, &h->massarr[t], 8);
		memcpy(out + 96 + 4 * t, &lo, 4);
		memcpy(out + 168 + 4 * t, &hi, 4);
	}
	memcpy(out + 72, &h->time, 8);
	memcpy(out + 80, &h->redshift, 8);
	memcpy(out + 124, &h->num_files, 4);
	memcpy(out + 128, &h->boxsize, 8);
	memcpy(out + 136, &h->omega0, 8);
	memcpy(out + 144, &h->omega_lambda, 8);
	memcpy(out + 152, &h->hubble_param, 8);
}

// one block of n particles with ncomp components of fb bytes each
bool block(Writer &w, const char *label, int64_t n, int ncomp, size_t fb, void *const *src)
{
	for (int c = 0; c < ncomp; c++)
		if (!src[c]) return false;
	const uint64_t bytes = (uint64_t) n * ncomp * fb;
	if (bytes > 0xFFFFFFFFull - 8) return false;     // Fortran record size (write_snapshot.c:282)
	w.begin(label, (uint32_t) bytes);
	if (ncomp == 1) {
		w.raw(src[0], (size_t) bytes);
	} else {
		// interleaved per particle, a chunk of particles at a time
		const int64_t chunk = 65536;
		std::vector<unsigned char> buf((size_t) (n < chunk ? n : chunk) * ncomp * fb);
		for (int64_t i0 = 0; i0 < n; i0 += chunk) {
			const int64_t m = n - i0 < chunk ? n - i0 : chunk;
			for (int64_t i = 0; i < m; i++)
				for (int c = 0; c < ncomp; c++)
					memcpy(&buf[((size_t) i * ncomp + c) * fb],
					       (const unsigned char *) src[c] + (size_t) (i0 + i) * fb, fb);
			w.raw(buf.data(), (size_t) m * ncomp * fb);
		}
	}
	w.u32((uint32_t) bytes);
	return true;
}

// the blocks of a snapshot in file order (IO/io.h:68-89)
enum { SB_POS, SB_VEL, SB_ID, SB_MASS, SB_ACC, SB_GACC, SB_GPOT, SB_N };
const char *const SB_LABEL[SB_N] = { "POS ", "VEL ", "ID  ", "MASS", "ACC ", "GACC", "GPOT" };
const int SB_NCOMP[SB_N] = { 3, 3, 1, 1, 1, 3, 1 };

bool block_wanted(int b, uint32_t blocks)
{
	if (b == SB_ACC) return blocks & TVG_SNAP_ACC;
	if (b == SB_GACC) return blocks & TVG_SNAP_GACC;
	if (b == SB_GPOT) return blocks & TVG_SNAP_GPOT;
	return true;
}

// Supplies the host arrays of one block's components; false if it cannot.
struct Fetch {
	virtual bool get(int block, void **comp) = 0;
	virtual ~Fetch() = default;
};

// the fields of a host tvg_particles view
struct HostFetch : Fetch {
	const tvg_particles *p;
	explicit HostFetch(const tvg_particles *q) : p(q) {}
	bool get(int b, void **c) override
	{
		switch (b) {
		case SB_POS: for (int k = 0; k < 3; k++) c[k] = p->pos[k]; break;
		case SB_VEL: for (int k = 0; k < 3; k++) c[k] = p->vel[k]; break;
		case SB_ID: c[0] = p->id; break;
		case SB_MASS: c[0] = p->mass; break;
		case SB_ACC: c[0] = p->acc[0]; break;      // one component: Acc[0] (io.h:75)
		case SB_GACC: for (int k = 0; k < 3; k++) c[k] = p->grav_acc[k]; break;
		case SB_GPOT: c[0] = p->grav_pot; break;
		default: return false;
		}
		return true;
	}
};

int write_file(const char *path, const tvg_snapshot_header *h, int64_t n, int32_t fb, uint32_t blocks,
               Fetch &fetch, char *err, size_t errlen)
{
	auto fail = [&](const char *m) {
		if (err) snprintf(err, errlen, "write_snapshot: %s", m);
		return TVG_E_BADINPUT;
	};
	if (!path || !h || n < 0 || (fb != 4 && fb != 8)) return fail("bad arguments");
	FILE *fp = fopen(path, "wb");
	if (!fp) return fail("cannot open the file");
	Writer w{ fp };
	unsigned char head[256];
	header_bytes(h, head);
	w.u32(8);
	w.raw("HEAD", 4);
	w.u32(256 + 8);
	w.u32(8);
	w.u32(256);
	w.raw(head, 256);
	w.u32(256);
	bool good = true;
	for (int b = 0; good && b < SB_N; b++) {
		if (!block_wanted(b, blocks)) continue;
		void *comp[3] = { nullptr, nullptr, nullptr };
		good = fetch.get(b, comp) && block(w, SB_LABEL[b], n, SB_NCOMP[b], b == SB_ID ? 4 : fb, comp);
	}
	const bool closed = fclose(fp) == 0;
	if (!good) return fail("a requested field is NULL, cannot be read, or a block exceeds 4 GB");
	if (!w.ok || !closed) return fail("write error");
	return TVG_OK;
}

} // namespace

extern "C" int tvg_write_snapshot_host(const char *path, const tvg_snapshot_header *header, int64_t n,
                                       int32_t float_bytes, const tvg_particles *p, uint32_t blocks)
{
	if (!p) return TVG_E_BADINPUT;
	HostFetch f(p);
	return write_file(path, header, n, float_bytes, blocks, f, nullptr, 0);
}

namespace {

// the context's fields, downloaded one block at a time into one staging
// buffer (three components at most)
struct DeviceFetch : Fetch {
	tvg_context *ctx;
	std::vector<unsigned char> stage;
	int rc = TVG_OK;                   // status of a failed download
	char msg[sizeof(((tvg_context *) nullptr)->err)] = { 0 };
	explicit DeviceFetch(tvg_context *c) : ctx(c) {}
	bool get(int b, void **c) override
	{
		const size_t fb = tvg_fsize(ctx), n = (size_t) (ctx->n > 0 ? ctx->n : 1);
		stage.resize(3 * n * fb);
		tvg_particles p;
		memset(&p, 0, sizeof(p));
		uint32_t field = 0;
		unsigned char *q = stage.data();
		switch (b) {
		case SB_POS: for (int k = 0; k < 3; k++) p.pos[k] = q + k * n * fb; field = TVG_F_POS; break;
		case SB_VEL: for (int k = 0; k < 3; k++) p.vel[k] = q + k * n * fb; field = TVG_F_VEL; break;
		case SB_ID: p.id = (uint32_t *) q; field = TVG_F_ID; break;
		case SB_MASS: p.mass = q; field = TVG_F_MASS; break;
		case SB_ACC: for (int k = 0; k < 3; k++) p.acc[k] = q + k * n * fb; field = TVG_F_ACC; break;
		case SB_GACC: for (int k = 0; k < 3; k++) p.grav_acc[k] = q + k * n * fb; field = TVG_F_GRAV_ACC; break;
		case SB_GPOT: p.grav_pot = q; field = TVG_F_GRAV_POT; break;
		default: return false;
		}
		rc = tvg_download(ctx, &p, field);
		if (rc != TVG_OK) {
			memcpy(msg, ctx->err, sizeof(msg));
			return false;
		}
		HostFetch h(&p);
		return h.get(b, c);
	}
};

} // namespace

extern "C" int tvg_write_snapshot(tvg_context *ctx, const char *path, const tvg_snapshot_header *header,
                                  uint32_t blocks)
{
	if (!ctx) return TVG_E_BADINPUT;
	DeviceFetch f(ctx);
	const int rc = write_file(path, header, ctx->n, (int32_t) tvg_fsize(ctx), blocks, f, ctx->err,
	                          sizeof(ctx->err));
	if (f.rc != TVG_OK) {               // the download's own error
		memcpy(ctx->err, f.msg, sizeof(ctx->err));
		return f.rc;
	}
	return rc;
}
