/* awsem_gpu.h -- C ABI of the B200 AWSEM-MD engine (libawsem_gpu.so).
 *
 * Replaces, for one single-GPU system, the per-step force and energy path of
 * the reference LAMMPS plugins of adavtyan/awsemmd:
 *   fix backbone      FixBackbone::pre_force -> compute_backbone
 *                     (src/fix_backbone.cpp:8181-8189, :7047-7673)
 *   pair vexcluded    PairExcludedVolume::compute (src/pair_excluded_volume.cpp:50-138)
 * and the LAMMPS pieces the benchmark step needs around them (bond_style
 * harmonic, fix nve, fix langevin, units real).
 *
 * Conventions
 *   - Every call returns 0 on success and a negative AWSEM_E* code on error;
 *     awsem_last_error() then holds the message (thread local).  Parse and
 *     topology errors carry the reference's own error texts.
 *   - Host arrays of positions, velocities and forces are [natoms][3] doubles
 *     in the caller's atom order (the data file's atom-id order).
 *   - energies[21]: [0..17] the reference fix's energy[] vector
 *     (fix_backbone.h:330-332: total, chain, shake, chi, rama, excluded,
 *     dssp, p_ap, water, burial, helix, amh-go, frag_mem, vec_fm,
 *     contact_restraints, membrane, ssb, dh), [18] pair vexcluded,
 *     [19] harmonic bonds, [20] kinetic energy.  kcal/mol.
 *   - A handle is used by one host thread at a time; distinct handles are
 *     independent.  Each handle owns one CUDA stream on its device.
 */
#ifndef AWSEM_GPU_H
#define AWSEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define AWSEM_OK 0
#define AWSEM_EINVAL -1   /* bad argument */
#define AWSEM_EPARSE -2   /* input file or parameter error */
#define AWSEM_ECUDA -3    /* CUDA runtime error */
#define AWSEM_ESTATE -4   /* invalid state (e.g. pair-list overflow detected) */
#define AWSEM_ENOMEM -5   /* device memory budget exceeded */
#define AWSEM_EBUSY -6    /* serving handle: the request does not fit now (retry after a collect) */

/* arithmetic forms */
#define AWSEM_FP64 0   /* plain form: FP64 throughout */
#define AWSEM_MIXED 1  /* FP32 pair geometry / Gaussians / switches, FP64 accumulation and integration */

/* term groups for awsem_compute */
#define AWSEM_TERMS_FIX 1   /* fix backbone terms */
#define AWSEM_TERMS_PAIR 2  /* pair vexcluded */
#define AWSEM_TERMS_BOND 4  /* bond_style harmonic */
#define AWSEM_TERMS_ALL 7

typedef struct awsem_system awsem_system;

/* Selection records (awsem_debug_selections): one 64-bit key per selected
 * item, key = kind << 56 | aux << 44 | i << 22 | j, with residue indices
 * i, j (internal order: the data file's residues in id order).  These are
 * the discrete decisions of the reference's pair passes, each at the line
 * that takes it in src/fix_backbone.cpp:
 *   DENS_WATER  (i<j) contact beads inside water well 0's support, |i-j|>1
 *               or another chain (DL1 :7759)
 *   DENS_HELIX  the same for the helix well (DL1 :7768)
 *   XI_WATER    aux = well: gamma0 != gamma1, separated, inside the well's
 *               support (DL2 :7925)
 *   WATER       aux = well: separated, inside the well's support (DL3 :8009)
 *   XI_FORCE    pair inside well 0's support with |xi_water(i)| > 1e-8
 *               (aux bit 0) or |xi_water(j)| > 1e-8 (bit 1) (:8027, :8033)
 *   HELIX_FORCE pair inside the helix support with |xi-helix sum| > 1e-6 (:8052)
 *   HELIX_PAIR  (i, i + helix_i_diff): |O_i - N_j|^2 < cutoff^2 (:7864);
 *               aux bit 0: |O_i - N_j| <= cutoff as well (:3708)
 *   DSSP        (acceptor O of i, donor N-H of j): candidate (:8064-8094);
 *               aux bit 0: r_NO <= cutoff (:2904), bit 1: both nu switches
 *               >= 1e-4 (:3052)
 *   PAP         (i<j) CA pair inside the P_AP cutoff (:8096-8103) and
 *               separated enough for some P_AP class; aux bit 0:
 *               nu(i, j) >= 1e-12 (:3281), bits 1-3: antiparallel medium,
 *               antiparallel long, parallel (:3290-3295)
 *   EV          bead pair (i, b0), (j, b1), i <= j, inside its pair
 *               vexcluded cutoff with a non-zero prefactor
 *               (src/pair_excluded_volume.cpp:98-110); aux = 3 b0 + b1
 *               (beads 0 CA, 1 CB or H-beta, 2 O) */
#define AWSEM_SEL_DENS_WATER 1
#define AWSEM_SEL_DENS_HELIX 2
#define AWSEM_SEL_XI_WATER 3
#define AWSEM_SEL_WATER 4
#define AWSEM_SEL_XI_FORCE 5
#define AWSEM_SEL_HELIX_FORCE 6
#define AWSEM_SEL_HELIX_PAIR 7
#define AWSEM_SEL_DSSP 8
#define AWSEM_SEL_PAP 9
#define AWSEM_SEL_EV 10

typedef struct awsem_run_params {
  double dt;                 /* fs (units real) */
  int langevin;              /* 0: fix nve only; 1: fix nve + fix langevin */
  double t_start, t_stop;    /* K, linear ramp over the run */
  double damp;               /* fs */
  unsigned long long seed;   /* Langevin stream seed */
  double skin;               /* pair-list skin, A (applied at the next rebuild) */
  int neigh_every;           /* forced rebuild period in steps; 0: displacement check only */
} awsem_run_params;

const char *awsem_last_error(void);
int awsem_version(void);

/* Build a system from a run directory laid out like a reference run:
 * coefficient file (fix_backbone_coeff.data sections), sequence file, the
 * tables read from the working directory (anti_HB, anti_NHB, para_HB,
 * para_one, anti_one, ssweight, gamma.dat, burial_gamma.dat), fragment
 * memories (.mem + .gro + gamma file) and an atom_style awsemmd data file.
 * pair_style: "p cut_short cut_long"; pair_coeffs: ';'-separated
 * "itype jtype lambda [cut_short cut_long]" records (pair_style vexcluded).
 * Replaces the FixBackbone constructor (src/fix_backbone.cpp:86-1072),
 * PairExcludedVolume::settings/coeff (src/pair_excluded_volume.cpp:175-232)
 * and read_data. */
int awsem_create_from_files(const char *workdir, const char *data_file, const char *coeff_file,
                            const char *seq_file, const char *pair_style, const char *pair_coeffs,
                            int precision, int device, awsem_system **out);
void awsem_destroy(awsem_system *sys);

/* The same system from a host code's own atom arrays instead of a data file
 * (what a LAMMPS fix has in memory): per atom, in the caller's order, its
 * role (0 CA, 1 CB or H-beta, 2 O, -1 other: the CA / CB / O groups of
 * `fix backbone`), residue and molecule ids, type and tag; masses by type
 * (mass_by_type[1..ntypes]); x (may be NULL); bonds as caller indices
 * (nbonds may be 0 when the host computes the bonds itself).  The
 * coefficient and sequence files and the tables are read from `workdir`, as
 * by the FixBackbone constructor (src/fix_backbone.cpp:86-1072).  With both
 * coeff_file and seq_file NULL the handle carries no fix backbone terms: it
 * evaluates pair vexcluded (AWSEM_TERMS_PAIR) and the given bonds only, its
 * chains being the runs of equal molecule id along the residues (what
 * PairExcludedVolume alone needs, src/pair_excluded_volume.cpp:50-138). */
int awsem_create_from_atoms(const char *workdir, const char *coeff_file, const char *seq_file, int natoms,
                            const int *role, const int *residue, const int *molecule, const int *type, const int *tag,
                            const double *mass_by_type, int ntypes, const double *x, int nbonds, const int *bond_a,
                            const int *bond_b, const double *bond_k, const double *bond_r0, const char *pair_style,
                            const char *pair_coeffs, int precision, int device, awsem_system **out);

/* Batches of independent replicas (one launch sequence advances them all).
 * Create an empty handle, add replicas (each a reference-style run
 * directory; all must share one coefficient file, tables and pair_style),
 * then commit.  `seed` is the replica's own Langevin seed (0: use the run's
 * seed).  A replica's trajectory does not depend on which other replicas
 * share the batch: every cross-thread sum is an exact fixed-point sum and
 * the noise stream is keyed by (seed, step, atom id).  No counterpart in the
 * reference (it runs one system per LAMMPS process). */
int awsem_batch_create(int precision, int device, awsem_system **out);
int awsem_batch_add_files(awsem_system *sys, const char *workdir, const char *data_file, const char *coeff_file,
                          const char *seq_file, const char *pair_style, const char *pair_coeffs,
                          unsigned long long seed, int *replica);
int awsem_batch_commit(awsem_system *sys);

/* Replicas given as arrays instead of files.  The force field (coefficient
 * file, the tables in `workdir`, the fragment-memory gamma file, pair_style
 * vexcluded settings) is read once; atoms follow the awsemmd data-file
 * conventions: per residue CA (type 1), O (type 3), CB (type 4) or H-beta
 * for glycine (type 5), atom ids 1..3n in that order, masses 27/28/60/2,
 * harmonic bonds CA-CA 3.816, CA-O 2.40, O-CA 2.76, CA-CB 1.53, CA-HB 1.09
 * with K = 60 kcal/mol/A^2. */
typedef struct awsem_replica_desc {
  int n_res;
  int n_chains;
  const int *chain_len;        /* [n_chains] residues per chain */
  const char *seq;             /* [n_res] one-letter residue codes */
  const double *ssweight;      /* [n_res][enabled SSWeight columns], or NULL */
  const double *x;             /* [n_res][3][3]: CA, O, CB/H-beta of each residue (A) */
  const double *v;             /* same layout (A/fs), or NULL for zero */
  int n_mem;                   /* fragment memories */
  const int *mem_pos;          /* [n_mem] first target residue, 0-based */
  const int *mem_len;          /* [n_mem] */
  const double *mem_weight;    /* [n_mem] */
  const char *mem_seq;         /* concatenated memory residue codes */
  const double *mem_ca;        /* concatenated [len][3] CA coordinates (A) */
  const double *mem_cb;        /* concatenated [len][3] CB coordinates (A; ignored for glycine) */
  unsigned long long seed;     /* Langevin seed of the replica (0: the run's) */
} awsem_replica_desc;

int awsem_batch_set_forcefield(awsem_system *sys, const char *workdir, const char *coeff_file,
                               const char *pair_style, const char *pair_coeffs);
int awsem_batch_add_replica(awsem_system *sys, const awsem_replica_desc *desc, int *replica);
int awsem_nreplicas(const awsem_system *sys);
int awsem_replica_natoms(const awsem_system *sys, int replica);
int awsem_replica_nres(const awsem_system *sys, int replica);
int awsem_replica_set_state(awsem_system *sys, int replica, const double *x, const double *v);
int awsem_replica_get_state(awsem_system *sys, int replica, double *x, double *v);
int awsem_replica_energies(awsem_system *sys, int replica, double *energies);
/* Every replica's state in one call each way: x and v are [natoms][3] with
 * the replicas concatenated in replica order, each in its caller atom order
 * (replica r starts at atom 3 * (residues of replicas before r)).  One
 * host-device copy per array (pinned host memory makes it a DMA at full
 * bandwidth) plus a reordering kernel.  Either pointer may be NULL. */
int awsem_batch_set_state(awsem_system *sys, const double *x, const double *v);
int awsem_batch_get_state(awsem_system *sys, double *x, double *v);
int awsem_replica_forces(awsem_system *sys, int replica, double *f);

/* totals over the whole batch (one replica: that system) */
int awsem_natoms(const awsem_system *sys);
int awsem_nres(const awsem_system *sys);

/* Drop-in force call: forces at the caller's positions x are ADDED into f
 * (the fix adds into atom->f during pre_force), energies (may be NULL) are
 * written.  `terms` selects AWSEM_TERMS_* groups.  The residue pair list is
 * kept between calls and rebuilt when the displacement check requires it;
 * when it outgrows its capacity it is enlarged and the evaluation repeated
 * (with LAMMPS's lists emulated the call returns AWSEM_ESTATE instead and
 * the next one runs on the enlarged list).  Non-finite positions make the
 * call return AWSEM_ESTATE.  Replaces FixBackbone::pre_force
 * (src/fix_backbone.cpp:8181) and, with AWSEM_TERMS_PAIR,
 * PairExcludedVolume::compute. */
int awsem_compute(awsem_system *sys, long long step, const double *x, double *f, double *energies, int terms);

/* Device-resident state of a single-system handle (caller atom order);
 * the awsem_replica_* forms address one replica of a batch. */
int awsem_set_state(awsem_system *sys, const double *x, const double *v);
int awsem_get_state(awsem_system *sys, double *x, double *v);

/* `run nsteps`: velocity Verlet (+ Langevin) with every force evaluated on
 * the GPU; the step sequence is captured in a CUDA graph.  thermo (may be
 * NULL) receives, per replica, (nsteps+1) rows of [fix total, vexcluded,
 * bonds, kinetic] (replica-major).  The first row is the setup evaluation
 * at the current step counter.  Advances every replica of a batch. */
int awsem_run(awsem_system *sys, long long nsteps, const awsem_run_params *rp, double *thermo);

/* One part of a LAMMPS `run` whose output (thermo, dumps, fix print) falls
 * between its steps: the window [window_begin, window_end] (absolute steps)
 * is the whole run -- the fix langevin ramp t_start -> t_stop spans it, as
 * LAMMPS's fix langevin interpolates over beginstep..endstep, the setup
 * evaluation is at window_begin and nothing drifts after window_end -- and
 * this call advances nsteps of it.  cont = 0: the call starts the window with
 * its setup evaluation (the current step must be window_begin); cont = 1: it
 * continues a call on this handle that stopped at the current step inside the
 * same window, so that the parts together are the single call bit for bit.
 * After each call the state (awsem_get_state) and energies are those of the
 * full step reached, as LAMMPS has them at end_of_step.  thermo rows: nsteps
 * + 1 (cont = 0) or nsteps (cont = 1) per replica.  awsem_run(n) is the
 * window [step, step + n] in one call.  A set_state, compute or profile call
 * in between ends the possibility to continue (AWSEM_EINVAL). */
int awsem_run_window(awsem_system *sys, long long nsteps, const awsem_run_params *rp, long long window_begin,
                     long long window_end, int cont, double *thermo);

/* Device time (ms) of the last awsem_run, from CUDA events recorded on the
 * engine's stream around the launched step graphs. */
double awsem_last_run_ms(const awsem_system *sys);

/* Energies and total forces (incl. Langevin) of the last evaluation. */
int awsem_energies(awsem_system *sys, double *energies);
int awsem_forces(awsem_system *sys, double *f);

/* Per-residue pair-pass intermediates of the last evaluation, [nres][8]:
 * rho_water, rho_helix, xi_water, xi1_helix, xi2_helix, burial coefficient,
 * sigma_water, sigma_helix. */
int awsem_residue_arrays(awsem_system *sys, double *out);

/* One force evaluation of a single-system handle at positions x (as
 * awsem_compute with AWSEM_TERMS_ALL) that also records its selections
 * (AWSEM_SEL_* keys above, in no particular order) into keys[cap].  *count
 * receives the number recorded; when it exceeds cap only the first cap
 * keys are stored and the call returns AWSEM_ESTATE.  The evaluation
 * reuses the handle's pair list when it is still valid, as a step does.  A
 * diagnostic for parity tests: the reference keeps these decisions inside
 * compute_pair (src/fix_backbone.cpp:7677-8135), compute_dssp_hdrgn (:2902),
 * compute_P_AP_potential (:3279), compute_helix_dtheta_pair (:3706) and
 * PairExcludedVolume::compute (src/pair_excluded_volume.cpp:50-138). */
int awsem_debug_selections(awsem_system *sys, long long step, const double *x, unsigned long long *keys,
                           long long cap, long long *count);

/* Limits of the bounded waits in device code, in SM clock cycles (0: the
 * defaults, about two seconds for a fragment-memory warp waiting on its
 * shared-memory copies and one second for a block of the persistent step
 * form waiting at a grid barrier).  A wait that runs out gives up, the kernel
 * ends normally (a fragment-memory warp first lets its copies in flight land,
 * waiting a fixed quarter second at most) and the call returns AWSEM_ESTATE
 * ("results of this call are invalid"); the next call runs clean.  hold, for
 * tests of those paths only, makes the waits' conditions unreachable so that
 * every wait runs out: bit 0 the copy waits (each stage expects 16 bytes that
 * never arrive), bit 1 the grid barriers (each waits for one block more than
 * the grid); hold 0 restores normal waits.  No counterpart in the reference
 * (LAMMPS has no device waits). */
int awsem_set_wait_limits(awsem_system *sys, long long fm_copy_wait_cycles, long long grid_barrier_wait_cycles,
                          int hold);

/* Pair-list statistics: builds so far, current list radius (A), largest
 * number of higher-numbered partners of one residue, overflow marker (0 when
 * the list never overflowed, else the pair count it needed). */
int awsem_neighbor_stats(awsem_system *sys, int *nbuilds, double *radius, int *max_count, int *overflow);

/* Current MD step counter. */
long long awsem_step(const awsem_system *sys);

/* Kernels of one MD step, in launch order (names for awsem_profile_step). */
#define AWSEM_NKERNELS 12
const char *awsem_kernel_name(int k);

/* Average device time (ms) of each kernel of one MD step, measured with CUDA
 * events on the engine's stream(s) over `reps` steps launched one kernel at
 * a time (the step advances; no graph).  Uses the last run's parameters. */
int awsem_profile_step(awsem_system *sys, int reps, double *ms);

/* Launch-shape autotuner (no counterpart in the reference): times `reps`
 * profiled steps of this handle's own system for each candidate shape of the
 * tunable kernels and keeps the fastest -- separations per fragment-memory
 * warp (1, 2, 3, 6 or all), and the grids of the pair-parallel passes and of
 * the hydrogen-bond pass (1 to 32 blocks per SM).  The state and the step
 * counter are restored afterwards; results do not depend on the shapes (all
 * sums are exact).  The grid of the fragment-memory kernel (1 to 4 blocks
 * per SM looping over the work, or one warp per unit) is judged on whole
 * steps, since that kernel overlaps the pair passes.  Last, the step form
 * (awsem_set_step_form) is chosen on whole steps: the chain of per-pass
 * kernels with those shapes against the persistent step kernel at several
 * grid sizes and stream-warp counts (handles without cell-grid replicas).
 * chosen (may be NULL): [separations per warp, pair-pass blocks,
 * hydrogen-bond blocks, fragment-memory blocks (0: one warp per unit)]; the
 * step form is read with awsem_get_step_form.  Not available on serving
 * handles. */
int awsem_autotune(awsem_system *sys, int reps, int *chosen);

/* Launch shapes in awsem_autotune's `chosen` layout, e.g. ones tuned
 * earlier on the same workload (no counterpart in the reference).  Results
 * do not depend on them.  AWSEM_EINVAL when a value is out of range. */
int awsem_set_launch_shapes(awsem_system *sys, const int *shapes);

/* LAMMPS `neighbor SKIN bin` and `neigh_modify delay D every E check
 * yes|no`.  skin > 0 sets the skin of the engine's lists (as
 * awsem_run_params.skin does for a run; <= 0 keeps it); the rest applies to
 * the neighbour list that [AMH-Go] reads.  The reference evaluates AMH-Go over the fix's full
 * neighbour list (fix_backbone.cpp:1809-1813 requests it, :3874-3972 walks
 * it), whose pairs are those within the pair-list cutoff plus the skin when
 * LAMMPS last rebuilt it; the engine keeps that membership per replica and
 * rebuilds it by LAMMPS's rule: at each run setup (and each awsem_compute),
 * then once at least `delay` steps have passed, on multiples of `every`, and
 * with check=1 only after some atom moved more than half the skin.
 * Defaults: skin 2.0, delay 0, every 1, check 1 (LAMMPS's).  AWSEM_EINVAL
 * for delay < 0, every < 1 or check not 0/1. */
int awsem_set_neighbor(awsem_system *sys, double skin, int delay, int every, int check);

/* For a host that runs the MD loop itself and calls awsem_compute once per
 * step (LAMMPS with `fix backbone/gpu`): whether the host rebuilt its
 * neighbour lists on the step of the next awsem_compute (LAMMPS:
 * neighbor->ago == 0).  With [AMH-Go] that evaluation then records a new
 * list (built = 1) or keeps the one recorded at the last build (built = 0),
 * as the reference fix reads LAMMPS's list (fix_backbone.cpp:3874-3880).
 * Applies to the next awsem_compute only; without a call every
 * awsem_compute builds.  AWSEM_EINVAL unless built is 0 or 1. */
int awsem_set_list_built(awsem_system *sys, int built);

/* Q order parameters, as LAMMPS's `compute ID group qwolynes datafile sep
 * exp` (src/compute_q_wolynes.cpp:50-238) and `compute ID group qonuchic
 * cutoff r_contact datafile factor | cutoff/gauss r_contact datafile |
 * shadow datafile factor | shadow/gauss datafile` (src/compute_q_onuchic.cpp:
 * 27-317) define them: `words` are the words after `compute`, the group is
 * the CA atoms of replica `rep` (the fix's first group), data files are
 * opened as named (relative to the process's working directory).  Errors
 * carry the reference's messages.  awsem_q_value evaluates a definition on
 * the replica's current positions (its compute_scalar): pair sums in FP64 in
 * a fixed order on the device. */
int awsem_q_create(awsem_system *sys, int rep, const char *words, int *qid);
int awsem_q_value(awsem_system *sys, int qid, double *value);

/* Step form of awsem_run / awsem_server_advance (no counterpart in the
 * reference, which evaluates on the CPU inside LAMMPS's pre_force hook).
 * form 0: each MD step is a chain of per-pass kernels (prepare, list
 * decision and build, density, residue, water_xi, pair, hbond, fragment
 * memory on a second stream, finish), captured in a CUDA graph.  form 1: each
 * MD step is ONE cooperative launch of a persistent kernel whose blocks pass
 * through the same passes separated by grid barriers; `stream_warps` (1..7)
 * of each block's 8 warps stream fragment-memory units concurrently with the
 * pair passes.  `blocks` is the persistent grid (0: every block that fits on
 * the device).  Results are identical bit for bit in both forms (all sums
 * are exact fixed point).  Form 1 is refused (AWSEM_EINVAL) on handles with a
 * replica above 2,048 residues (those build cell grids).  A barrier wait that
 * gives up (about one second) makes the call fail with AWSEM_ESTATE. */
int awsem_set_step_form(awsem_system *sys, int form, int blocks, int stream_warps);

/* form[3] = {form, persistent grid (blocks; 0 until first used when set to
 * "all that fit"), stream warps per block}. */
int awsem_get_step_form(awsem_system *sys, int *form);

/* Sizes behind the roofline's algorithmic-byte counts:
 * info[0] residues, [1] atoms, [2] fragment-memory records (4 distances
 * each), [3] bytes per stored distance (8 FP64, 4 mixed), [4] rows per
 * residue, [5] pair-list capacity (pairs), [6] residue pairs i < j in the
 * list of the last build, [7] non-uniform memory coefficients stored (0/1). */
int awsem_model_info(awsem_system *sys, long long *info);

/* Serving: continuous batching of MD runs (annealing or structure
 * prediction requests) on one GPU.  No counterpart in the reference (one
 * system per LAMMPS process); each request runs exactly what `run nsteps`
 * with fix langevin (ramp t_start -> t_stop) and fix nve would run on it
 * alone, and its result does not depend on which other requests share the
 * GPU: forces are exact fixed-point sums and the noise is keyed by the
 * request's own step count and atom ids.
 *
 * A serving handle is created with fixed capacities, all device memory
 * allocated at creation (the memory budget): max_residues residues (handed
 * out in 32-residue groups), max_requests requests in flight, and
 * max_memory_records fragment-memory records (one per memory and target
 * pair; 16 bytes each in the mixed form, 32 in FP64, plus 4 or 8 when the
 * memory coefficients differ between records).  The force field is read
 * once, as in awsem_batch_set_forcefield; requests are array-described
 * replicas (awsem_replica_desc, `seed` = the request's Langevin seed).
 *
 * awsem_server_admit places a request (AWSEM_EBUSY when it does not fit
 * now); it starts with the next step.  awsem_server_advance runs nsteps
 * steps of every admitted request (finished requests stay frozen).
 * awsem_server_progress reports steps done / requested; awsem_server_collect
 * copies a finished request's final x, v ([natoms][3], the request's atom
 * order) and energies[21] (either may be NULL) and frees its room.
 * usage: [0] requests held, [1] residues held (group-rounded), [2] residue
 * capacity, [3] memory records held (stripe-rounded), [4] record capacity,
 * [5] device bytes allocated, [6] step counter, [7] request capacity. */
int awsem_server_create(const char *workdir, const char *coeff_file, const char *pair_style, const char *pair_coeffs,
                        int precision, int device, long long max_residues, int max_requests,
                        long long max_memory_records, double dt, double damp, awsem_system **out);
int awsem_server_admit(awsem_system *srv, const awsem_replica_desc *request, long long nsteps, double t_start,
                       double t_stop, int *slot);
/* Admission in two parts, so that a serving loop can prepare the next
 * arrivals while the GPU advances: awsem_server_prepare builds a request's
 * host-side data (topology, fragment-memory table slices in the handle's
 * arithmetic type; no device work, and it may run on another host thread
 * while awsem_server_advance runs on this handle); awsem_server_admit_prepared
 * places it (AWSEM_EBUSY when it does not fit now: the prepared request stays
 * valid and may be admitted later; AWSEM_EINVAL for a request prepared for
 * another handle).  awsem_request_free releases a prepared request, admitted
 * or not, and may be called after the handle is destroyed.
 * awsem_server_admit is prepare + admit_prepared + free. */
typedef struct awsem_request awsem_request;
int awsem_server_prepare(awsem_system *srv, const awsem_replica_desc *request, awsem_request **out);
int awsem_server_admit_prepared(awsem_system *srv, awsem_request *request, long long nsteps, double t_start,
                                double t_stop, int *slot);
void awsem_request_free(awsem_request *request);
int awsem_server_advance(awsem_system *srv, long long nsteps);
int awsem_server_progress(awsem_system *srv, int slot, long long *done, long long *total);
int awsem_server_collect(awsem_system *srv, int slot, double *x, double *v, double *energies);
int awsem_server_usage(awsem_system *srv, long long *info);

/* Fragment-memory forces and energy through an entry point that allocates
 * nothing: for callers that cannot call cudaMalloc when forces are needed
 * (a host code that owns all device memory through its own pool, a step
 * being recorded into a CUDA graph, an allocation-free real-time loop).
 * No counterpart in the reference (its fragment-memory term,
 * FixBackbone::compute_fragment_memory_potential, only runs inside the fix).
 *
 * d_x: device array [natoms][3] in the handle's internal order (per residue
 * CA, CB or H-beta, O; residues in handle order); d_f: device array
 * [natoms][3], overwritten with the fragment-memory forces; d_energy: one
 * device double, overwritten with the fragment-memory energy; stream: a
 * cudaStream_t (NULL: the default stream); the call is asynchronous on it.
 * The handle's memory tables are used as they are resident since commit.
 *
 * Scratch: a fixed-size __device__ array of AWSEM_NOALLOC_MAX_ATOMS atoms
 * (576 KiB, held by every GPU that loads the library until exit); larger
 * handles are rejected with AWSEM_EINVAL.  The first call on a device looks
 * up that array's device address (cudaGetSymbolAddress); make that first
 * call before any stream capture.  A device reset (cudaDeviceReset) ends the
 * context that address belongs to: the next call on that device looks it up
 * again, so it too should come before any capture.  All calls share the
 * array and each clears what it uses first; calls whose kernels overlap on
 * the GPU race on it and must be serialised by the caller.  The caller's
 * buffers and stream belong to the handle's device; like every entry point,
 * the call leaves the caller's current device as it found it. */
#define AWSEM_NOALLOC_MAX_ATOMS 24576
int awsem_fragmem_noalloc(awsem_system *sys, const double *d_x, double *d_f, double *d_energy, void *stream);

#ifdef __cplusplus
}
#endif
#endif
