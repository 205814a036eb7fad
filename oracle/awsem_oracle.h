/* FP64 CPU restatement of the AWSEM-MD per-step force and energy path
   (oracle; test infrastructure only -- never part of the product path).

   C ABI, loaded with ctypes by tests/ and bench.py's CPU baseline.  Arrays
   of positions, velocities and forces are [natoms][3] doubles in data-file
   atom order (sorted by atom id).  Energies: out[0..17] follow the reference
   energy[] enum (fix_backbone.h:330-332: total, chain, shake, chi, rama,
   excluded, dssp, p_ap, water, burial, helix, amh-go, frag_mem, vec_fm,
   contact_restraints, membrane, ssb, dh), out[18] = pair vexcluded,
   out[19] = harmonic bonds, out[20] = kinetic energy. */
#ifndef AWSEM_ORACLE_H
#define AWSEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

void *oracle_create(const char *workdir, const char *data_file, const char *coeff_file,
                    const char *seq_file, const char *pair_style, const char *pair_coeffs);
void oracle_destroy(void *h);
const char *oracle_last_error(void);
int oracle_natoms(void *h);
int oracle_nres(void *h);
/* positions / velocities in, forces and energies out (no Langevin force) */
int oracle_compute(void *h, const double *x, double *f, double *energies);
/* per-residue intermediates of the last compute: rho_w, rho_h, xi_w, xi1_h,
   xi2_h, burial_coefficient, sigma_w, sigma_h ([n][8]) */
int oracle_residue_arrays(void *h, double *out);
/* One evaluation at x recording its selections; returns the number of
   distinct keys of the set `which` (0: AWSEM_SEL_* selection records,
   include/awsem_gpu.h; 1: distance predicates decided within 2e-6 of their
   threshold; 2: the reference's n x n cache entries the evaluation touches,
   kinds 32-36) and stores up to cap of them, sorted, in out; -1 on error */
long long oracle_selections(void *h, const double *x, int which, unsigned long long *out, long long cap);
/* nsteps of velocity Verlet (+ Langevin); x and v updated in place.
   thermo (optional): (nsteps+1) x 4 rows of [fix total, vexcluded, bonds, ke]. */
int oracle_run(void *h, double *x, double *v, long long step0, long long nsteps, double dt,
               int langevin, double t_start, double t_stop, double damp,
               unsigned long long seed, double *thermo);
/* LAMMPS neighbor skin and neigh_modify delay / every / check of the fix's
   full neighbour list that [AMH-Go] reads (defaults 2.0, 0, 1, 1) */
int oracle_set_neighbor(void *h, double skin, int delay, int every, int check);
/* compute qwolynes / qonuchic over the CA atoms at positions x ([natoms][3]);
   `words` as after LAMMPS's `compute`, data files opened as named */
int oracle_q(void *h, const double *x, const char *words, double *out);
double oracle_uniform(unsigned long long seed, long long step, long long tag, int comp);

#ifdef __cplusplus
}
#endif
#endif
