// tvg_snapshot.cu -- Gadget format-2 snapshot files (Write_Snapshot,
// IO/write_snapshot.c:13-328; block table IO/io.h:68-89) for one rank and
// one file: the 256-byte header, then POS, VEL, ID, MASS and the optional
// ACC, GACC, GPOT blocks, each preceded by the format-2 label record
// ("NAME", size + 8) and framed by 4-byte Fortran record markers. Multi-
// component fields are interleaved per particle (fill_data_buffer,
// write_snapshot.c:230-272). Host code: the context variant downloads the
// fields (in the device order, which after a sort is the PH order the
// reference writes in) and writes them.
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
		std::vector<unsigned char> buf((size_t) bytes);
		for (int64_t i = 0; i < n; i++)
			for (int c = 0; c < ncomp; c++)
				memcpy(&buf[((size_t) i * ncomp + c) * fb], (const unsigned char *) src[c] + (size_t) i * fb,
				       fb);
		w.raw(buf.data(), buf.size());
	}
	w.u32((uint32_t) bytes);
	return true;
}

int write_host(const char *path, const tvg_snapshot_header *h, int64_t n, int32_t fb,
               const tvg_particles *p, uint32_t blocks, char *err, size_t errlen)
{
	auto fail = [&](const char *m) {
		if (err) snprintf(err, errlen, "write_snapshot: %s", m);
		return TVG_E_BADINPUT;
	};
	if (!path || !h || !p || n < 0 || (fb != 4 && fb != 8)) return fail("bad arguments");
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
	void *pos[3] = { p->pos[0], p->pos[1], p->pos[2] }, *vel[3] = { p->vel[0], p->vel[1], p->vel[2] };
	void *id[1] = { p->id }, *mass[1] = { p->mass };
	bool good = block(w, "POS ", n, 3, fb, pos) && block(w, "VEL ", n, 3, fb, vel)
	         && block(w, "ID  ", n, 1, 4, id) && block(w, "MASS", n, 1, fb, mass);
	if (good && (blocks & TVG_SNAP_ACC)) {
		// the reference's ACC block has one component: Acc[0] (io.h:75)
		void *acc[1] = { p->acc[0] };
		good = block(w, "ACC ", n, 1, fb, acc);
	}
	if (good && (blocks & TVG_SNAP_GACC)) {
		void *g[3] = { p->grav_acc[0], p->grav_acc[1], p->grav_acc[2] };
		good = block(w, "GACC", n, 3, fb, g);
	}
	if (good && (blocks & TVG_SNAP_GPOT)) {
		void *g[1] = { p->grav_pot };
		good = block(w, "GPOT", n, 1, fb, g);
	}
	const bool closed = fclose(fp) == 0;
	if (!good) return fail("a requested field is NULL or a block exceeds 4 GB");
	if (!w.ok || !closed) return fail("write error");
	return TVG_OK;
}

} // namespace

extern "C" int tvg_write_snapshot_host(const char *path, const tvg_snapshot_header *header, int64_t n,
                                       int32_t float_bytes, const tvg_particles *p, uint32_t blocks)
{
	return write_host(path, header, n, float_bytes, p, blocks, nullptr, 0);
}

extern "C" int tvg_write_snapshot(tvg_context *ctx, const char *path, const tvg_snapshot_header *header,
                                  uint32_t blocks)
{
	if (!ctx) return TVG_E_BADINPUT;
	const int64_t n = ctx->n;
	const size_t fb = tvg_fsize(ctx);
	// host copies of the fields the file needs
	uint32_t fields = TVG_F_POS | TVG_F_VEL | TVG_F_ID | TVG_F_MASS;
	if (blocks & TVG_SNAP_ACC) fields |= TVG_F_ACC;
	if (blocks & TVG_SNAP_GACC) fields |= TVG_F_GRAV_ACC;
	if (blocks & TVG_SNAP_GPOT) fields |= TVG_F_GRAV_POT;
	std::vector<unsigned char> store;
	int nbuf = 8 + ((blocks & TVG_SNAP_ACC) ? 3 : 0) + ((blocks & TVG_SNAP_GACC) ? 3 : 0)
	         + ((blocks & TVG_SNAP_GPOT) ? 1 : 0);
	store.resize((size_t) nbuf * (size_t) (n > 0 ? n : 1) * 8);
	unsigned char *q = store.data();
	auto take = [&](size_t bytes) {
		void *r = q;
		q += bytes * (size_t) (n > 0 ? n : 1);
		return r;
	};
	tvg_particles p;
	memset(&p, 0, sizeof(p));
	for (int k = 0; k < 3; k++) p.pos[k] = take(fb);
	for (int k = 0; k < 3; k++) p.vel[k] = take(fb);
	p.id = (uint32_t *) take(4);
	p.mass = take(fb);
	if (blocks & TVG_SNAP_ACC)
		for (int k = 0; k < 3; k++) p.acc[k] = take(fb);
	if (blocks & TVG_SNAP_GACC)
		for (int k = 0; k < 3; k++) p.grav_acc[k] = take(fb);
	if (blocks & TVG_SNAP_GPOT) p.grav_pot = take(fb);
	TVG_CHECK(tvg_download(ctx, &p, fields));
	return write_host(path, header, n, (int32_t) fb, &p, blocks, ctx->err, sizeof(ctx->err));
}
