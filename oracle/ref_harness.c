/*
 * ref_harness.c -- drives the UNMODIFIED reference C sources (Tandav) for one
 * gravity evaluation and dumps every hot-path intermediate to a binary file.
 *
 * Test infrastructure only: this program is the oracle's view of the real
 * reference. It is linked against the reference's own objects (all of its
 * src/ except main.c) by oracle/Makefile and is never part of the product.
 *
 * Sequence (mirrors src/main.c:112-191 preamble, src/init.c:11-76,
 * src/setup.c:9-32, src/update.c:13-34 and src/accel.c:15-71):
 *   preamble (threads, Task) -> memory -> particles -> periodic init + Ewald
 *   table -> Setup_Domain_Decomposition -> Setup_Gravity_Tree ->
 *   [omp parallel] Domain_Decomposition -> Gravity_Tree_Build ->
 *   BH pass (Gravity_Tree_Acceleration with Use_BH_Criterion) ->
 *   |a| into Last_Acc_Mag, Acc = 0 (accel.c:28-43) -> relative pass.
 * For the periodic build the Ewald-only walks (Gravity_Tree_Periodic) are run
 * once more on zeroed accumulators so that the correction can be compared on
 * its own.
 *
 * Usage: ref_harness <mode> <input.bin> <output.bin>
 *   mode "force": the sequence above.
 *   mode "keys":  Peano_Key / Reversed_Peano_Key for the input positions with
 *                 the domain taken from the input header (no decomposition).
 *   mode "force2": one force computation on the first tree, then a second
 *                 Domain_Decomposition (balanced on the P.Cost it left) and
 *                 tree; the dumps and walks are those of the second.
 *   mode "update": "force" with the tree updates between rebuilds applied
 *                 to the built tree before the walks (tree_update_sequence).
 *   mode "snap":  Write_Snapshot of the input particles (run_snap).
 *   mode "read":  Read_Snapshot of a snapshot file given in place of the
 *                 input file (run_read).
 *
 * Input  (little endian): "TVIN", int32 version(1), int64 n, double box
 *   (<=0: isolated), double softening, double origin[3], double size,
 *   int32 flags (bit0 BH pass, bit1 relative pass), int32 pad,
 *   double pos[3][n], double vel[3][n], double mass[n].
 * Output: a list of records {char name[16]; int64 nbytes; bytes}.
 */
#include "includes.h"
#include "domain.h"
#include "peano.h"
#include "timestep.h"
#include "Gravity/tree.h"
#include "Gravity/periodic.h"
#include "periodic.h"
#include "vector.h"
#include "IO/io.h"

void Init_Memory_Management(void);
void Setup_Leaf_Vectors(void);

struct dump_topnode {
	uint64_t key;
	int32_t target, level, first_part, npart;
	float pos[3], mass, com[3], dp[3];
};

static FILE *Out = NULL;
static bool Dump_Bulk = true;     /* false: timing run, no per-particle dumps */

static void put(const char *name, const void *data, int64_t nbytes)
{
	char tag[16] = { 0 };
	strncpy(tag, name, 15);
	fwrite(tag, 1, 16, Out);
	fwrite(&nbytes, sizeof(nbytes), 1, Out);
	if (nbytes > 0)
		fwrite(data, 1, (size_t) nbytes, Out);
}

static double now(void) { return omp_get_wtime(); }

struct input {
	int64_t n;
	double box, soft, origin[3], size;
	int32_t flags;
	double *pos, *vel, *mass;
};

static struct input read_input(const char *fname)
{
	struct input in = { 0 };
	FILE *fp = fopen(fname, "rb");
	if (!fp) { fprintf(stderr, "cannot open %s\n", fname); exit(2); }
	char magic[4];
	int32_t version = 0, pad = 0;
	if (fread(magic, 1, 4, fp) != 4 || memcmp(magic, "TVIN", 4)) { fprintf(stderr, "bad magic\n"); exit(2); }
	if (fread(&version, 4, 1, fp) != 1 || version != 1) { fprintf(stderr, "bad version\n"); exit(2); }
	size_t ok = fread(&in.n, 8, 1, fp);
	ok += fread(&in.box, 8, 1, fp);
	ok += fread(&in.soft, 8, 1, fp);
	ok += fread(in.origin, 8, 3, fp);
	ok += fread(&in.size, 8, 1, fp);
	ok += fread(&in.flags, 4, 1, fp);
	ok += fread(&pad, 4, 1, fp);
	if (ok != 9) { fprintf(stderr, "short header\n"); exit(2); }
	in.pos = malloc(3 * in.n * sizeof(double));
	in.vel = malloc(3 * in.n * sizeof(double));
	in.mass = malloc(in.n * sizeof(double));
	if (fread(in.pos, 8, 3 * in.n, fp) != (size_t) (3 * in.n)
	    || fread(in.vel, 8, 3 * in.n, fp) != (size_t) (3 * in.n)
	    || fread(in.mass, 8, in.n, fp) != (size_t) in.n) {
		fprintf(stderr, "short body\n");
		exit(2);
	}
	fclose(fp);
	return in;
}

/* Same thread/rank bookkeeping as the reference's preamble (main.c:112-191). */
static void preamble(void)
{
	NRank = 1;
	#pragma omp parallel
	{
		#pragma omp single
		{
			NThreads = omp_get_num_threads();
			NTask = NRank * NThreads;
		}
		Task.Rank = 0;
		Task.Thread_ID = omp_get_thread_num();
		Task.ID = Task.Thread_ID;
		Task.Is_Thread_Main = (Task.Thread_ID == 0);
		Task.Is_Master = (Task.Thread_ID == 0);
		Task.Is_MPI_Master = true;
		Task.Seed[2] = 14041981L * Task.Thread_ID;
		erand48(Task.Seed);
	}
}

static void set_particle_counts(int64_t n)
{
	Sim.Npart_Total = n;
	memset(Sim.Npart, 0, sizeof(Sim.Npart));
	Sim.Npart[1] = n;
	#pragma omp parallel
	{
		Task.Npart_Total = (int) n;
		memset(Task.Npart, 0, sizeof(Task.Npart));
		Task.Npart[1] = (int) n;
	}
}

static void load_particles(const struct input *in)
{
	int64_t n = in->n;
	for (int64_t i = 0; i < n; i++) {
		P.Type[i] = 1;
		P.Time_Bin[i] = 0;
		P.It_Drift_Pos[i] = P.It_Kick_Pos[i] = 0;
		P.Key[i] = 0;
		P.ID[i] = (ID_t) i;
		P.Cost[i] = 0;
		for (int k = 0; k < 3; k++) {
			P.Pos[k][i] = (Float) in->pos[k * n + i];
			P.Vel[k][i] = (Float) in->vel[k * n + i];
			P.Acc[k][i] = 0;
			P.Grav_Acc[k][i] = 0;
		}
		P.Mass[i] = (Float) in->mass[i];
#ifdef GRAVITY_POTENTIAL
		P.Grav_Pot[i] = 0;
#endif
		P.Last_Acc_Mag[i] = 0;
		P.Tree_Parent[i] = 0;
	}
}

static void zero_accumulators(void)
{
	#pragma omp for
	for (int i = 0; i < Task.Npart_Total; i++) {
		P.Acc[0][i] = P.Acc[1][i] = P.Acc[2][i] = 0;
		P.Grav_Acc[0][i] = P.Grav_Acc[1][i] = P.Grav_Acc[2][i] = 0;
		P.Cost[i] = 0;
#ifdef GRAVITY_POTENTIAL
		P.Grav_Pot[i] = 0;
#endif
	}
}

/* Dump Acc/Grav_Acc/Cost (and Grav_Pot with GRAVITY_POTENTIAL) as doubles
 * under a name prefix. */
static void dump_forces(const char *prefix, int64_t n)
{
	if (!Dump_Bulk) return;
	double *buf = malloc(3 * n * sizeof(double));
	char name[16];
	for (int k = 0; k < 3; k++)
		for (int64_t i = 0; i < n; i++)
			buf[k * n + i] = P.Acc[k][i];
	snprintf(name, 16, "%s_acc", prefix);
	put(name, buf, 3 * n * sizeof(double));
	for (int k = 0; k < 3; k++)
		for (int64_t i = 0; i < n; i++)
			buf[k * n + i] = P.Grav_Acc[k][i];
	snprintf(name, 16, "%s_gacc", prefix);
	put(name, buf, 3 * n * sizeof(double));
	for (int64_t i = 0; i < n; i++)
		buf[i] = P.Cost[i];
	snprintf(name, 16, "%s_cost", prefix);
	put(name, buf, n * sizeof(double));
#ifdef GRAVITY_POTENTIAL
	for (int64_t i = 0; i < n; i++)
		buf[i] = P.Grav_Pot[i];
	snprintf(name, 16, "%s_pot", prefix);
	put(name, buf, n * sizeof(double));
#endif
	free(buf);
}

static void init_memory(int64_t n)
{
	size_t tree_bytes = sizeof(struct Tree_Node);
	/* per-thread scratch: the PH reorder needs N*8 bytes (peano.c:56-58) and
	 * a subtree is built in the buffer when it fits (tree_build.c:65-96) */
	double per_thread = fmax(1.05 * n * 8.0, 0.1 * n * tree_bytes) + (16 << 20);
	Param.Buffer_Size = (int) ceil(per_thread * NThreads / (1 << 20));
	double pool = (double) n * 1.3 * (sizeof_P + 64.0 + 16.0) + 1.2 * 0.3 * n * tree_bytes;
	Param.Max_Mem_Size = Param.Buffer_Size + (int) ceil(pool / (1 << 20)) + 512;
	Param.Part_Alloc_Factor = 1.1;
	Init_Memory_Management();
}

static int run_keys(const struct input *in)
{
	int64_t n = in->n;
	Domain.Size = in->size;
	for (int k = 0; k < 3; k++) Domain.Origin[k] = in->origin[k];
	peanoKey *std = malloc(n * sizeof(peanoKey));
	peanoKey *rev = malloc(n * sizeof(peanoKey));
	for (int64_t i = 0; i < n; i++) {
		Float x = (Float) in->pos[i], y = (Float) in->pos[n + i], z = (Float) in->pos[2 * n + i];
		std[i] = Peano_Key(x, y, z);
		rev[i] = Reversed_Peano_Key(x, y, z);
	}
	put("std_key", std, n * sizeof(peanoKey));
	put("rev_key", rev, n * sizeof(peanoKey));
	free(std); free(rev);
	return 0;
}

/* The top nodes and the tree under a name prefix ("<p>_top", "<p>_tree"). */
static void dump_tree_state(const char *prefix)
{
	char name[16];
	struct dump_topnode *tn = calloc(NTop_Nodes, sizeof(*tn));
	for (uint32_t j = 0; j < NTop_Nodes; j++) {
		tn[j].key = D[j].TNode.Key;
		tn[j].target = D[j].TNode.Target;
		tn[j].level = D[j].TNode.Level;
		tn[j].first_part = D[j].TNode.First_Part;
		tn[j].npart = D[j].TNode.Npart;
		for (int k = 0; k < 3; k++) {
			tn[j].pos[k] = D[j].TNode.Pos[k];
			tn[j].com[k] = D[j].TNode.CoM[k];
			tn[j].dp[k] = D[j].TNode.Dp[k];
		}
		tn[j].mass = D[j].TNode.Mass;
	}
	snprintf(name, 16, "%s_top", prefix);
	put(name, tn, (int64_t) NTop_Nodes * sizeof(*tn));
	free(tn);
	snprintf(name, 16, "%s_tree", prefix);
	put(name, Tree, (int64_t) NNodes * sizeof(struct Tree_Node));
}

/* Mode "update": the tree updates between rebuilds (Gravity/tree_update.c,
 * called from kick.c:31-32,61-62 and drift.c:41-42) on the tree just built.
 * Acc = Vel; the active particles are those with ID % 3 != 1, in index
 * order; two kick passes of Gravity_Tree_Update_Kicks, with the Float kick
 * step size * (1 + ID % 4) / 4 and then size * (1 + ID % 3) / 3; then
 * Gravity_Tree_Update_Drift(origin[0]). The state after the kicks is dumped
 * as "upk_*", after the drift as "upd_*"; the walks then run on the updated
 * tree for all particles. */
static void tree_update_sequence(const struct input *in, int64_t n)
{
	for (int64_t i = 0; i < n; i++)
		for (int k = 0; k < 3; k++) P.Acc[k][i] = P.Vel[k][i];
	int na = 0;
	for (int64_t i = 0; i < n; i++)
		if (P.ID[i] % 3 != 1) Active_Particle_List[na++] = (int) i;
	for (int pass = 0; pass < 2; pass++) {
		const int q = pass == 0 ? 4 : 3;
		for (int j = 0; j < na; j++) {
			const int ipart = Active_Particle_List[j];
			const Float dt = (Float) (in->size * (1 + P.ID[ipart] % q) / q);
			Gravity_Tree_Update_Kicks(ipart, dt);
		}
	}
	dump_tree_state("upk");
	#pragma omp parallel
	Gravity_Tree_Update_Drift(in->origin[0]);
	dump_tree_state("upd");
	for (int64_t i = 0; i < n; i++) Active_Particle_List[i] = (int) i;
	NActive_Particles = (int) n;
}

/* One force computation on the current tree as Compute_Acceleration does it
 * with Sig.Prepare_Step (accel.c:15-71): Barnes-Hut pass, |Acc| into
 * Last_Acc_Mag, zeroed accumulators, relative pass. P.Cost then holds the
 * relative pass's interaction counts (incl. the Ewald walk when periodic),
 * the cost the next Domain_Decomposition balances (domain.c:533-536). */
static void force_for_cost(void)
{
	#pragma omp parallel
	{
		zero_accumulators();
		Sig.Use_BH_Criterion = true;
		Gravity_Tree_Acceleration();
		#pragma omp barrier
		#pragma omp for
		for (int i = 0; i < Task.Npart_Total; i++)
			P.Last_Acc_Mag[i] = SQRT(p2(P.Acc[0][i]) + p2(P.Acc[1][i]) + p2(P.Acc[2][i]));
		zero_accumulators();
		Sig.Use_BH_Criterion = false;
		Gravity_Tree_Acceleration();
	}
}

static int run_force(const struct input *in, bool update, bool redecompose)
{
	int64_t n = in->n;
	bool periodic = in->box > 0;
#ifdef PERIODIC
	if (!periodic) { fprintf(stderr, "periodic build needs box > 0\n"); return 3; }
#else
	if (periodic) { fprintf(stderr, "isolated build needs box <= 0\n"); return 3; }
#endif
	set_particle_counts(n);
	for (int t = 0; t < NPARTYPE; t++) Param.Grav_Softening[t] = in->soft;
	/* sizeof_P is set by Allocate_Particle_Structures; size the pool first */
	sizeof_P = 0;
	for (int i = 0; i < NP_Fields; i++) sizeof_P += P_Fields[i].Bytes * P_Fields[i].N;
	init_memory(n);
	Allocate_Particle_Structures();
	load_particles(in);
	Time.Max_Active_Bin = 31;
	Active_Particle_List = Malloc(Task.Npart_Total_Max * sizeof(*Active_Particle_List), "APL");
	NActive_Particles = (int) n;
	for (int64_t i = 0; i < n; i++) Active_Particle_List[i] = (int) i;

	double t0 = now();
	if (periodic) {
		Sim.Boxsize[0] = Sim.Boxsize[1] = Sim.Boxsize[2] = in->box;
		Init_Periodic();
		#pragma omp parallel
		Periodic_Constrain_Particles_To_Box();
		Gravity_Periodic_Init();
	}
	double t_ewald_init = now() - t0;

	Setup_Leaf_Vectors();
	Setup_Domain_Decomposition();
	Setup_Gravity_Tree();

	double t_dd = 0, t_build = 0, t_bh = 0, t_rel = 0, t_bh_ew = 0, t_rel_ew = 0;
	int flags = in->flags;
	double *acc_bh = malloc(3 * n * sizeof(double));

	#pragma omp parallel
	{
		#pragma omp master
		t0 = now();
		Sig.Prepare_Step = true;
		Sig.Domain_Update = true;
		Domain_Decomposition();
		#pragma omp barrier
		#pragma omp master
		{ t_dd = now() - t0; t0 = now(); }
		Gravity_Tree_Build();
		#pragma omp barrier
		#pragma omp master
		t_build = now() - t0;
	}

	/* mode "force2": one force computation, then the next decomposition and
	 * tree (the main loop's second step, main.c:43-70): the dumps below
	 * describe that second decomposition, balanced on P.Cost. cost_in / id_in
	 * are P.Cost and P.ID in the order the second decomposition starts from. */
	if (redecompose) {
		force_for_cost();
		const int64_t nn = Task.Npart_Total;
		double *c = malloc(nn * sizeof(double));
		uint32_t *ids = malloc(nn * sizeof(uint32_t));
		for (int64_t i = 0; i < nn; i++) { c[i] = P.Cost[i]; ids[i] = (uint32_t) P.ID[i]; }
		put("cost_in", c, nn * sizeof(double));
		put("id_in", ids, nn * sizeof(uint32_t));
		free(c);
		free(ids);
		#pragma omp parallel
		{
			Sig.Domain_Update = true;
			Domain_Decomposition();
		}
		/* Gravity_Tree_Build places each subtree where its thread reserves
		 * memory (tree_build.c:59-96), so with several threads the node
		 * indices (Target, Tree_Parent, and through quirk Q3 the particles a
		 * small top node's walk reads) depend on the threads' timing. A
		 * one-thread team places the subtrees in top-node order, as every
		 * run with one thread does; the subtrees themselves do not change. */
		#pragma omp parallel num_threads(1)
		Gravity_Tree_Build();
	}

	/* bounded CPU sample (flags bits 8..23 = stride s > 1): the walks run for
	 * every s-th particle only, as a reduced Active_Particle_List. Bits 24..30
	 * = repetitions R <= s: the BH pass runs for the particles i with
	 * i % s < R, then the relative pass R times, repetition r for the
	 * particles i % s == r, each timed ("rel_times") */
	const int stride = ((flags >> 8) & 0xFFFF) > 1 ? ((flags >> 8) & 0xFFFF) : 1;
	int reps = (flags >> 24) & 0x7F;
	if (reps < 1) reps = 1;
	if (reps > stride) reps = stride;
	double rel_times[128] = { 0 };
	if (stride > 1) {
		int na = 0;
		for (int64_t i = 0; i < n; i++)
			if (i % stride < reps) Active_Particle_List[na++] = (int) i;
		NActive_Particles = na;
	}
	const bool dump_bulk = (flags & 4) == 0;
	Dump_Bulk = dump_bulk;

	/* ---- dump decomposition and tree ---- */
	if (dump_bulk) {
		put("domain_size", &Domain.Size, sizeof(double));
		put("domain_origin", Domain.Origin, 3 * sizeof(double));
		uint32_t *ids = malloc(n * sizeof(uint32_t));
		for (int64_t i = 0; i < n; i++) ids[i] = (uint32_t) P.ID[i];
		put("perm", ids, n * sizeof(uint32_t));
		free(ids);
		put("rev_key", P.Key, n * sizeof(peanoKey));
		peanoKey *std = malloc(n * sizeof(peanoKey));
		for (int64_t i = 0; i < n; i++)
			std[i] = Peano_Key(P.Pos[0][i], P.Pos[1][i], P.Pos[2][i]);
		put("std_key", std, n * sizeof(peanoKey));
		free(std);
		double *pos = malloc(3 * n * sizeof(double));
		for (int k = 0; k < 3; k++)
			for (int64_t i = 0; i < n; i++) pos[k * n + i] = P.Pos[k][i];
		put("pos", pos, 3 * n * sizeof(double));
		free(pos);
		struct dump_topnode *tn = calloc(NTop_Nodes, sizeof(*tn));
		for (uint32_t j = 0; j < NTop_Nodes; j++) {
			tn[j].key = D[j].TNode.Key;
			tn[j].target = D[j].TNode.Target;
			tn[j].level = D[j].TNode.Level;
			tn[j].first_part = D[j].TNode.First_Part;
			tn[j].npart = D[j].TNode.Npart;
			for (int k = 0; k < 3; k++) {
				tn[j].pos[k] = D[j].TNode.Pos[k];
				tn[j].com[k] = D[j].TNode.CoM[k];
				tn[j].dp[k] = D[j].TNode.Dp[k];
			}
			tn[j].mass = D[j].TNode.Mass;
		}
		put("topnodes", tn, (int64_t) NTop_Nodes * sizeof(*tn));
		free(tn);
		put("tree", Tree, (int64_t) NNodes * sizeof(struct Tree_Node));
		put("tree_parent", P.Tree_Parent, n * sizeof(*P.Tree_Parent));
		int32_t fsize = (int32_t) sizeof(Float);
		put("float_size", &fsize, 4);
	}
	if (update) tree_update_sequence(in, n);

	#pragma omp parallel
	{
		if (flags & 1) {
			zero_accumulators();
			#pragma omp master
			t0 = now();
			Sig.Use_BH_Criterion = true;
			Gravity_Tree_Acceleration();
			#pragma omp barrier
			#pragma omp master
			{
				t_bh = now() - t0;
				dump_forces("bh", n);
				for (int k = 0; k < 3; k++)
					for (int64_t i = 0; i < n; i++) acc_bh[k * n + i] = P.Acc[k][i];
			}
			#pragma omp barrier
			if (periodic && dump_bulk) {
				zero_accumulators();
				#pragma omp master
				t0 = now();
				Gravity_Tree_Periodic();
				#pragma omp barrier
				#pragma omp master
				{ t_bh_ew = now() - t0; dump_forces("bhew", n); }
				#pragma omp barrier
			}
			/* accel.c:28-43: |a| of the BH pass becomes Last_Acc_Mag */
			#pragma omp for
			for (int i = 0; i < (int) n; i++) {
				P.Acc[0][i] = (Float) acc_bh[i];
				P.Acc[1][i] = (Float) acc_bh[n + i];
				P.Acc[2][i] = (Float) acc_bh[2 * n + i];
				P.Last_Acc_Mag[i] = SQRT(p2(P.Acc[0][i]) + p2(P.Acc[1][i]) + p2(P.Acc[2][i]));
			}
		}
		if (flags & 2) {
			for (int r = 0; r < reps; r++) {
				if (reps > 1) {
					#pragma omp single
					{
						int na = 0;
						for (int64_t i = r; i < n; i += stride) Active_Particle_List[na++] = (int) i;
						NActive_Particles = na;
					}
				}
				zero_accumulators();
				#pragma omp master
				t0 = now();
				Sig.Use_BH_Criterion = false;
				Gravity_Tree_Acceleration();
				#pragma omp barrier
				#pragma omp master
				{
					rel_times[r] = now() - t0;
					if (r == 0) { t_rel = rel_times[0]; dump_forces("rel", n); }
				}
				#pragma omp barrier
			}
			if (periodic && dump_bulk) {
				zero_accumulators();
				#pragma omp master
				t0 = now();
				Gravity_Tree_Periodic();
				#pragma omp barrier
				#pragma omp master
				{ t_rel_ew = now() - t0; dump_forces("relew", n); }
				#pragma omp barrier
			}
		}
	}
	if (dump_bulk) {
		double *lam = malloc(n * sizeof(double));
		for (int64_t i = 0; i < n; i++) lam[i] = P.Last_Acc_Mag[i];
		put("last_acc_mag", lam, n * sizeof(double));
		free(lam);
	}
	double timings[8] = { t_ewald_init, t_dd, t_build, t_bh, t_bh_ew, t_rel, t_rel_ew, (double) NThreads };
	put("timings", timings, sizeof(timings));
	put("rel_times", rel_times, (int64_t) reps * sizeof(double));
	double gconst = Const.Gravity;
	put("gravity", &gconst, sizeof(double));
	double eps[3] = { Epsilon[1], Epsilon2[1], Epsilon3[1] };
	put("epsilon", eps, sizeof(eps));
	free(acc_bh);
	return 0;
}

/* Write_Snapshot (IO/write_snapshot.c:13-60) of the input particles in
 * input order, to "<output>_000", with Acc[k] = (k+1) Pos[k] and
 * Grav_Acc[k] = (k+2) Vel[k] (and Grav_Pot = Pos[0] - 3 Mass). In this mode the input's size field is
 * Time.Current and box is Sim.Boxsize; the Cosmo constants (compile-time in
 * the reference) are reported as the record "cosmo" in <output>. */
static int run_snap(const struct input *in, const char *out_base)
{
	int64_t n = in->n;
	set_particle_counts(n);
	sizeof_P = 0;
	for (int i = 0; i < NP_Fields; i++) sizeof_P += P_Fields[i].Bytes * P_Fields[i].N;
	init_memory(n);
	Allocate_Particle_Structures();
	load_particles(in);
	for (int64_t i = 0; i < n; i++)    /* distinct per component, for the ACC/GACC blocks */
		for (int k = 0; k < 3; k++) {
			P.Acc[k][i] = (Float) ((k + 1) * in->pos[k * n + i]);
			P.Grav_Acc[k][i] = (Float) ((k + 2) * in->vel[k * n + i]);
		}
#ifdef GRAVITY_POTENTIAL
	for (int64_t i = 0; i < n; i++) P.Grav_Pot[i] = (Float) (in->pos[i] - 3 * in->mass[i]);
#endif
	for (int t = 0; t < NPARTYPE; t++) Sim.Mpart[t] = 0;
	Sim.Boxsize[0] = Sim.Boxsize[1] = Sim.Boxsize[2] = in->box;
	Time.Current = in->size;
	Time.NSnap = 10;
	Time.Snap_Counter = 0;
	Param.Num_Output_Files = 1;
	Param.Num_IO_Tasks = 1;
	snprintf(Param.Output_File_Base, sizeof(Param.Output_File_Base), "%s", out_base);
	Write_Snapshot();
	double cosmo[3] = { Cosmo.Omega_0, Cosmo.Omega_Lambda, Cosmo.Hubble_Constant };
	put("cosmo", cosmo, sizeof(cosmo));
	int32_t fsize = (int32_t) sizeof(Float);
	put("float_size", &fsize, 4);
	return 0;
}

/* Read_Snapshot (IO/read_snapshot.c:19-123) of the snapshot at `path` (or
 * path.0, path.1, ...): the memory pool is sized from the header's totals,
 * then the reference reads the file(s) into P. Dumps the particles in the
 * order read (ID, Type, Pos, Vel, Mass, Acc[0], Grav_Acc as doubles) and
 * Sim's per-type counts and masses. */
static int run_read(const char *path)
{
	char first[CHARBUFSIZE];
	snprintf(first, sizeof(first), "%s", path);
	FILE *fp = fopen(first, "rb");
	if (!fp) {
		snprintf(first, sizeof(first), "%s.0", path);
		fp = fopen(first, "rb");
	}
	if (!fp) { fprintf(stderr, "cannot open %s\n", path); return 2; }
	unsigned char head[20 + 256];
	if (fread(head, 1, sizeof(head), fp) != sizeof(head)) { fclose(fp); return 2; }
	fclose(fp);
	int64_t total = 0;
	for (int t = 0; t < 6; t++) {
		uint32_t lo, hi;
		memcpy(&lo, head + 20 + 96 + 4 * t, 4);
		memcpy(&hi, head + 20 + 168 + 4 * t, 4);
		total += (int64_t) lo + ((int64_t) hi << 32);
	}
	sizeof_P = 0;
	for (int i = 0; i < NP_Fields; i++) sizeof_P += P_Fields[i].Bytes * P_Fields[i].N;
	init_memory(total > 0 ? total : 1);
	Param.Num_IO_Tasks = 1;
	Read_Snapshot((char *) path);
	const int64_t n = Task.Npart_Total;
	put("read_n", &n, 8);
	uint32_t *id = malloc((n ? n : 1) * sizeof(uint32_t));
	int32_t *type = malloc((n ? n : 1) * sizeof(int32_t));
	double *buf = malloc((n ? 3 * n : 1) * sizeof(double));
	for (int64_t i = 0; i < n; i++) { id[i] = (uint32_t) P.ID[i]; type[i] = P.Type[i]; }
	put("read_id", id, n * sizeof(uint32_t));
	put("read_type", type, n * sizeof(int32_t));
	for (int k = 0; k < 3; k++) for (int64_t i = 0; i < n; i++) buf[k * n + i] = P.Pos[k][i];
	put("read_pos", buf, 3 * n * sizeof(double));
	for (int k = 0; k < 3; k++) for (int64_t i = 0; i < n; i++) buf[k * n + i] = P.Vel[k][i];
	put("read_vel", buf, 3 * n * sizeof(double));
	for (int64_t i = 0; i < n; i++) buf[i] = P.Mass[i];
	put("read_mass", buf, n * sizeof(double));
	for (int64_t i = 0; i < n; i++) buf[i] = P.Acc[0][i];
	put("read_acc0", buf, n * sizeof(double));
	for (int k = 0; k < 3; k++) for (int64_t i = 0; i < n; i++) buf[k * n + i] = P.Grav_Acc[k][i];
	put("read_gacc", buf, 3 * n * sizeof(double));
	int64_t npart[6];
	double mpart[6];
	for (int t = 0; t < 6; t++) { npart[t] = (int64_t) Sim.Npart[t]; mpart[t] = Sim.Mpart[t]; }
	put("sim_npart", npart, sizeof(npart));
	put("sim_mpart", mpart, sizeof(mpart));
	int32_t fsize = (int32_t) sizeof(Float);
	put("float_size", &fsize, 4);
	free(id); free(type); free(buf);
	return 0;
}

int main(int argc, char *argv[])
{
	if (argc != 4) {
		fprintf(stderr, "usage: %s force|keys|snap|update input.bin output.bin\n"
		                "       %s read snapshot output.bin\n", argv[0], argv[0]);
		return 1;
	}
	preamble();
	if (!strcmp(argv[1], "read")) {       /* argv[2] is a snapshot, not an input file */
		Out = fopen(argv[3], "wb");
		if (!Out) { fprintf(stderr, "cannot write %s\n", argv[3]); return 2; }
		int rc = run_read(argv[2]);
		fclose(Out);
		return rc;
	}
	struct input in = read_input(argv[2]);
	Out = fopen(argv[3], "wb");
	if (!Out) { fprintf(stderr, "cannot write %s\n", argv[3]); return 2; }
	int rc = 1;
	if (!strcmp(argv[1], "keys"))
		rc = run_keys(&in);
	else if (!strcmp(argv[1], "force"))
		rc = run_force(&in, false, false);
	else if (!strcmp(argv[1], "force2"))
		rc = run_force(&in, false, true);
	else if (!strcmp(argv[1], "update"))
		rc = run_force(&in, true, false);
	else if (!strcmp(argv[1], "snap"))
		rc = run_snap(&in, argv[3]);
	fclose(Out);
	return rc;
}
