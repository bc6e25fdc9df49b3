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

#include <array>
#include <string>
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

// ------------------------------------------------------------------ reading

namespace {

uint32_t bswap32(uint32_t v) { return __builtin_bswap32(v); }

void swap_words(unsigned char *d, size_t bytes, size_t word)
{
	for (size_t o = 0; o + word <= bytes; o += word)
		for (size_t a = 0, b = word - 1; a < b; a++, b--) {
			const unsigned char t = d[o + a];
			d[o + a] = d[o + b];
			d[o + b] = t;
		}
}

// one format-2 file: its blocks by label (payload offset and size)
struct SnapFile {
	FILE *fp = nullptr;
	bool swap = false;
	struct Blk { char label[4]; long off; uint32_t size; };
	std::vector<Blk> blocks;
	~SnapFile() { if (fp) fclose(fp); }

	bool u32(uint32_t *v)
	{
		if (fread(v, 4, 1, fp) != 1) return false;
		if (swap) *v = bswap32(*v);
		return true;
	}
	// the byte order from the first record marker (find_endianess,
	// read_snapshot.c:519-541), then every block's label record
	bool open(const char *path)
	{
		fp = fopen(path, "rb");
		if (!fp) return false;
		uint32_t first = 0;
		if (fread(&first, 4, 1, fp) != 1) return false;
		if (first == 8) swap = false;
		else if (bswap32(first) == 8) swap = true;
		else return false;                      // not a format-2 file
		rewind(fp);
		for (;;) {
			uint32_t m0, size8, m1, a, b;
			Blk k;
			if (!u32(&m0)) break;                   // end of file
			if (m0 != 8 || fread(k.label, 1, 4, fp) != 4 || !u32(&size8) || !u32(&m1) || m1 != 8)
				return false;
			if (!u32(&a) || a + 8 != size8) return false;
			k.off = ftell(fp);
			k.size = a;
			if (fseek(fp, (long) a, SEEK_CUR) != 0 || !u32(&b) || b != a) return false;
			blocks.push_back(k);
		}
		return true;
	}
	const Blk *find(const char *label) const
	{
		for (const Blk &k : blocks)
			if (!memcmp(k.label, label, 4)) return &k;
		return nullptr;
	}
	bool read(const Blk *k, void *dst, size_t word)
	{
		if (fseek(fp, k->off, SEEK_SET) != 0 || fread(dst, 1, k->size, fp) != k->size) return false;
		if (swap) swap_words((unsigned char *) dst, k->size, word);
		return true;
	}
};

// the 256-byte header (struct gadget_header, io.h:24-44)
bool parse_header(SnapFile &f, tvg_snapshot_header *h, uint32_t npart[6])
{
	const SnapFile::Blk *k = f.find("HEAD");
	if (!k || k->size != 256) return false;
	unsigned char b[256];
	if (fseek(f.fp, k->off, SEEK_SET) != 0 || fread(b, 1, 256, f.fp) != 256) return false;
	if (f.swap) {
		swap_words(b, 24, 4);                  // Npart
		swap_words(b + 24, 64, 8);             // Massarr, Time, Redshift
		swap_words(b + 88, 40, 4);             // Flag_Sfr .. Num_Files
		swap_words(b + 128, 32, 8);            // Boxsize .. Hubble_Param
		swap_words(b + 160, 32, 4);            // Flag_Age, Flag_Metals, Nall_High_Word
	}
	memset(h, 0, sizeof(*h));
	for (int t = 0; t < 6; t++) {
		uint32_t lo, hi;
		memcpy(&npart[t], b + 4 * t, 4);
		memcpy(&h->massarr[t], b + 24 + 8 * t, 8);
		memcpy(&lo, b + 96 + 4 * t, 4);
		memcpy(&hi, b + 168 + 4 * t, 4);
		h->npart[t] = npart[t];
		h->nall[t] = (uint64_t) lo | ((uint64_t) hi << 32);
	}
	memcpy(&h->time, b + 72, 8);
	memcpy(&h->redshift, b + 80, 8);
	memcpy(&h->num_files, b + 124, 4);
	memcpy(&h->boxsize, b + 128, 8);
	memcpy(&h->omega0, b + 136, 8);
	memcpy(&h->omega_lambda, b + 144, 8);
	memcpy(&h->hubble_param, b + 152, 8);
	return true;
}

// find_files (read_snapshot.c:544-575): path itself, else path.0, path.1, ...
std::vector<std::string> snapshot_files(const char *path)
{
	std::vector<std::string> out;
	if (FILE *fp = fopen(path, "rb")) {
		fclose(fp);
		out.push_back(path);
		return out;
	}
	for (int i = 0; i < 10000; i++) {
		std::string name = std::string(path) + "." + std::to_string(i);
		FILE *fp = fopen(name.c_str(), "rb");
		if (!fp) break;
		fclose(fp);
		out.push_back(name);
	}
	return out;
}

} // namespace

extern "C" int tvg_read_snapshot_header(const char *path, tvg_snapshot_header *header, int32_t *num_files)
{
	if (!path || !header) return TVG_E_BADINPUT;
	const std::vector<std::string> files = snapshot_files(path);
	if (files.empty()) return TVG_E_BADINPUT;
	SnapFile f;
	uint32_t np[6];
	if (!f.open(files[0].c_str()) || !parse_header(f, header, np)) return TVG_E_BADINPUT;
	if (num_files) *num_files = (int32_t) files.size();
	return TVG_OK;
}

extern "C" int tvg_read_snapshot_host(const char *path, int32_t float_bytes, int64_t cap, tvg_particles *p,
                                      int64_t *n_out, uint32_t *blocks_out)
{
	if (!path || !p || cap < 0 || (float_bytes != 4 && float_bytes != 8)) return TVG_E_BADINPUT;
	if (!p->pos[0] || !p->pos[1] || !p->pos[2] || !p->vel[0] || !p->vel[1] || !p->vel[2] || !p->id)
		return TVG_E_BADINPUT;
	const std::vector<std::string> files = snapshot_files(path);
	if (files.empty()) return TVG_E_BADINPUT;
	const size_t fb = (size_t) float_bytes;
	// per-file and total counts per type; the first file's header gives the
	// masses and the ID ranges (Sim.Mpart, Sim.Npart)
	std::vector<std::array<uint32_t, 6>> per_file(files.size());
	tvg_snapshot_header h0;
	uint64_t total[6] = { 0 };
	for (size_t f = 0; f < files.size(); f++) {
		SnapFile sf;
		tvg_snapshot_header h;
		uint32_t np[6];
		if (!sf.open(files[f].c_str()) || !parse_header(sf, &h, np)) return TVG_E_BADINPUT;
		if (f == 0) h0 = h;
		for (int t = 0; t < 6; t++) {
			per_file[f][t] = np[t];
			total[t] += np[t];
		}
	}
	uint64_t n = 0, off[6];
	for (int t = 0; t < 6; t++) {
		off[t] = n;
		n += total[t];
	}
	if ((int64_t) n > cap) return TVG_E_BADINPUT;
	// blocks: label, components, bytes per component, destinations
	struct Want { const char *label; int ncomp; size_t bytes; void *dst[3]; uint32_t bit; bool required; };
	Want want[] = {
		{ "POS ", 3, fb, { p->pos[0], p->pos[1], p->pos[2] }, 0, true },
		{ "VEL ", 3, fb, { p->vel[0], p->vel[1], p->vel[2] }, 0, true },
		{ "ID  ", 1, 4, { p->id, nullptr, nullptr }, 0, true },
		{ "MASS", 1, fb, { p->mass, nullptr, nullptr }, TVG_SNAP_MASS, false },
		{ "ACC ", 1, fb, { p->acc[0], nullptr, nullptr }, TVG_SNAP_ACC, false },
		{ "GACC", 3, fb, { p->grav_acc[0], p->grav_acc[1], p->grav_acc[2] }, TVG_SNAP_GACC, false },
		{ "GPOT", 1, fb, { p->grav_pot, nullptr, nullptr }, TVG_SNAP_GPOT, false },
	};
	uint32_t found = TVG_SNAP_MASS | TVG_SNAP_ACC | TVG_SNAP_GACC | TVG_SNAP_GPOT;
	uint64_t run[6] = { 0 };
	std::vector<unsigned char> buf;
	for (size_t f = 0; f < files.size(); f++) {
		SnapFile sf;
		if (!sf.open(files[f].c_str())) return TVG_E_BADINPUT;
		uint64_t nf = 0, first[6];
		for (int t = 0; t < 6; t++) {
			first[t] = nf;
			nf += per_file[f][t];
		}
		for (const Want &w : want) {
			const SnapFile::Blk *k = sf.find(w.label);
			if (!k) {
				if (w.required) return TVG_E_BADINPUT;   // "Can't find required block"
				found &= ~w.bit;
				continue;
			}
			if ((uint64_t) k->size != nf * w.ncomp * w.bytes) return TVG_E_BADINPUT;
			if (!w.dst[0]) continue;                    // present, not wanted
			buf.resize(k->size > 0 ? k->size : 1);
			if (k->size && !sf.read(k, buf.data(), w.bytes)) return TVG_E_BADINPUT;
			// particle j of type t goes to its type's section, after the
			// particles of that type from the earlier files
			for (int t = 0; t < 6; t++)
				for (uint64_t j = 0; j < per_file[f][t]; j++) {
					const uint64_t src = first[t] + j, dst = off[t] + run[t] + j;
					for (int c = 0; c < w.ncomp; c++)
						memcpy((unsigned char *) w.dst[c] + dst * w.bytes,
						       &buf[(src * w.ncomp + c) * w.bytes], w.bytes);
				}
		}
		for (int t = 0; t < 6; t++) run[t] += per_file[f][t];
	}
	// masses from the header (generate_masses_from_header)
	bool header_mass = false;
	for (int t = 0; t < 6; t++) header_mass |= h0.massarr[t] != 0;
	if (header_mass && p->mass)
		for (int t = 0; t < 6; t++)
			for (uint64_t i = off[t]; i < off[t] + total[t]; i++) {
				if (fb == 4) ((float *) p->mass)[i] = (float) h0.massarr[t];
				else ((double *) p->mass)[i] = h0.massarr[t];
			}
	// types from the ID ranges of the header's totals (set_particle_types)
	if (p->type) {
		uint64_t lo[6], hi[6], r = 0;
		bool any[6];
		for (int t = 0; t < 6; t++) {
			any[t] = h0.nall[t] != 0;
			lo[t] = r;
			r += h0.nall[t];
			hi[t] = r - 1;
		}
		for (int t = 0; t < 6; t++)
			for (uint64_t i = off[t]; i < off[t] + total[t]; i++) {
				const uint64_t id = p->id[i];
				int32_t type = t;
				for (int u = 0; u < 6; u++)
					if (any[u] && id >= lo[u] && id <= hi[u]) type = u;
				p->type[i] = type;
			}
	}
	if (n_out) *n_out = (int64_t) n;
	if (blocks_out) *blocks_out = found;
	return TVG_OK;
}

extern "C" int tvg_read_snapshot(tvg_context *ctx, const char *path, int64_t *n_out, uint32_t *blocks_out)
{
	if (!ctx || !path) return TVG_E_BADINPUT;
	tvg_snapshot_header h;
	int32_t nfiles = 0;
	if (tvg_read_snapshot_header(path, &h, &nfiles) != TVG_OK)
		return tvg_fail(ctx, TVG_E_BADINPUT, "read_snapshot: cannot read the header of %s", path);
	uint64_t cap = 0;
	for (int t = 0; t < 6; t++) cap += h.nall[t];
	if ((int64_t) cap > ctx->cap)
		return tvg_fail(ctx, TVG_E_BADINPUT, "read_snapshot: %llu particles > capacity %lld",
		                (unsigned long long) cap, (long long) ctx->cap);
	const size_t fb = tvg_fsize(ctx), m = cap > 0 ? (size_t) cap : 1;
	// staging: pos 3, vel 3, mass 1, acc 3, grav_acc 3, grav_pot 1 Floats; id, type 4 B
	std::vector<unsigned char> fl(14 * m * fb, 0), id(4 * m), type(4 * m);
	tvg_particles p;
	memset(&p, 0, sizeof(p));
	unsigned char *q = fl.data();
	for (int k = 0; k < 3; k++) p.pos[k] = q + (size_t) k * m * fb;
	for (int k = 0; k < 3; k++) p.vel[k] = q + (size_t) (3 + k) * m * fb;
	p.mass = q + 6 * m * fb;
	for (int k = 0; k < 3; k++) p.acc[k] = q + (size_t) (7 + k) * m * fb;
	for (int k = 0; k < 3; k++) p.grav_acc[k] = q + (size_t) (10 + k) * m * fb;
	p.grav_pot = q + 13 * m * fb;
	p.id = (uint32_t *) id.data();
	p.type = (int32_t *) type.data();
	int64_t n = 0;
	uint32_t blocks = 0;
	if (tvg_read_snapshot_host(path, (int32_t) fb, (int64_t) cap, &p, &n, &blocks) != TVG_OK)
		return tvg_fail(ctx, TVG_E_BADINPUT, "read_snapshot: cannot read %s", path);
	uint32_t fields = TVG_F_POS | TVG_F_VEL | TVG_F_ID | TVG_F_MASS | TVG_F_TYPE;
	if (blocks & TVG_SNAP_ACC) fields |= TVG_F_ACC;
	if (blocks & TVG_SNAP_GACC) fields |= TVG_F_GRAV_ACC;
	if (blocks & TVG_SNAP_GPOT) fields |= TVG_F_GRAV_POT;
	TVG_CHECK(tvg_upload(ctx, n, &p, fields));
	if (n_out) *n_out = n;
	if (blocks_out) *blocks_out = blocks;
	return TVG_OK;
}
