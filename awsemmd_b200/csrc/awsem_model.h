// Host-side AWSEM model: force-field parameters, system topology and
// fragment-memory tables, built from the reference's input formats
// (fix_backbone_coeff.data sections, gamma.dat / burial_gamma.dat / DSSP
// tables / ssweight, the sequence file, atom_style awsemmd data files and
// .mem/.gro fragment memories).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace awsem {

// Energy slots: 0..17 follow the reference fix's energy[] enum
// (fix_backbone.h:330-332); 18 pair vexcluded, 19 harmonic bonds, 20 kinetic.
enum Energy {
  E_TOTAL = 0, E_CHAIN, E_SHAKE, E_CHI, E_RAMA, E_VEXCLUDED, E_DSSP, E_PAP, E_WATER, E_BURIAL,
  E_HELIX, E_AMHGO, E_FRAGMEM, E_VFRAGMEM, E_CONT_REST, E_MEMB, E_SSB, E_DH,
  E_FIX_TERMS = 18, E_PAIR = 18, E_BOND = 19, E_KIN = 20, E_SLOTS = 21
};

enum TermFlag : uint32_t {
  T_CHAIN = 1u << 0, T_CHI = 1u << 1, T_RAMA = 1u << 2, T_RAMA_P = 1u << 3, T_SSW = 1u << 4,
  T_DSSP = 1u << 5, T_PAP = 1u << 6, T_WATER = 1u << 7, T_BURIAL = 1u << 8, T_HELIX = 1u << 9,
  T_FM = 1u << 10, T_FM_TABLE = 1u << 11, T_AMHGO = 1u << 12, T_SSB = 1u << 13, T_DH = 1u << 14,
  T_CONTREST = 1u << 15, T_SHAKE = 1u << 16, T_MEMB = 1u << 17, T_PHOSPH = 1u << 18, T_VFM = 1u << 19
};

// Residue flags
enum ResFlag : uint32_t { R_GLY = 1u, R_PRO = 2u, R_FIRST = 4u, R_LAST = 8u, R_PHOSPH = 16u };

// Offsets of the lookup tables inside the device table buffer (doubles)
enum TableOffset {
  TB_ANTI_HB = 0, TB_ANTI_NHB = 800, TB_PARA_HB = 1600, TB_PARA_ONE = 2400, TB_ANTI_ONE = 2420,
  TB_BURIAL = 2440, TB_WATER = 2500, TB_WATER_PHOSPH = 2500 + 5 * 800, TB_SIZE = 2500 + 10 * 800
};

// Scalar parameters, passed to kernels by value.  Names follow the reference.
struct FFParams {
  uint32_t terms;
  int n_wells, contact_cutoff, helix_i_diff, i_med_min, i_med_max, i_diff_pap;
  int n_rama, n_rama_p, pro_acc_flag, fm_min_sep, fm_max_sep, fm_nd;
  int well_flag[5];
  int ssweight[12];
  double epsilon;
  double an, bn, cn, ap, bp, cp, ah, bh, ch;
  double k_chain[3], r_ncb0, r_cpcb0, r_ncp0, k_chi, chi0;
  double w[12], phiw[12], phi0[12], psiw[12], psi0[12];
  double cphi0[12], sphi0[12], cpsi0[12], spsi0[12];  // cos / sin of phi0, psi0 (angle-sum form of rama)
  double hbscl[4][9];
  double sigma_NO_sqinv, sigma_HO_sqinv, NO_zero, HO_zero, k_dssp, dssp_cut, dssp_cut_sq;
  double pref[2], d_nu0, nu_cut_sq[2];
  double k_global_pap, k_betapred_pap, k_pap[3], pap_cut, pap_pref, pap_cutoff_sq, pap_drmin_sq, pap_drmax_sq;
  double water_kappa, water_kappa_sigma, treshold;
  double well_rmin[5], well_rmax[5], w_rmin_th[5], w_rmax_th[5], w_rmin_sq[5], w_rmax_sq[5];
  double k_burial, burial_kappa, burial_ro_min[3], burial_ro_max[3];
  double k_helix, helix_gamma_p, helix_gamma_w, helix_kappa, helix_kappa_sigma, helix_treshold;
  double helix_cutoff, helix_cutoff_sq, helix_rmin, helix_rmax, h_rmin_th, h_rmax_th, h_rmin_sq, h_rmax_sq;
  double h4prob[20], h4prob_pro, helix_sigma_HO_sqinv, helix_sigma_NO_sqinv, helix_HO_zero, helix_NO_zero;
  double k_fm, fm_sigma_exp;
  double fm_sigma_sq[64];  // |i-j|^(2 * fm_sigma_exp) by separation
  // table fragment memory ([Fragment_Memory_Table]): grid tb_rmin + ir * tb_dr, ir < tb_size
  double tb_rmin, tb_rmax, tb_dr;
  int tb_size, tb_nbrs;
  // AMH-Go ([AMH-Go], fix_backbone.cpp:297-303): strength (epsilon-scaled), power, native cutoff;
  // pairs count only within the reference's fix pair-list cutoff plus the neighbour skin
  double k_amh_go, amh_go_p, amh_go_rc, pair_list_cutoff;
  double helix_sigma_HO, helix_sigma_NO;  // as read (the pair-list cutoff uses them)
  // [Solvent_Barrier] (fix_backbone.cpp:334-345): two wells, kappa, separation, radius correction
  double k_ssb1, k_ssb2, ssb_rmin1, ssb_rmax1, ssb_rmin2, ssb_rmax2, ssb_kappa, ssb_rshift[20];
  int ssb_ij_sep, ssb_rad_cor, dh_min_sep;
  // [DebyeHuckel] (:467-477): strengths by charge signs, screening, minimum separation
  double k_plusplus, k_minusminus, k_plusminus, k_screening, screening_length;
  // [Contact_Restraints] (:321-327, :1106-1150): epsilon-scaled strength, width and its cutoffs
  double k_cont_rest, cr_sigma, cr_sigma_sq_inv, cr_dr_cut, cr_cut_sq;
  // [Shake] (:180-183): strength and the CA(i)-CA(i+1), CA(i)-O(i), O(i)-CA(i+1) lengths
  double k_shake, r_sh1, r_sh2, r_sh3;
  // [Membrane] (:346-358): strength, switching steepness, centre, pore, thickness, radii, gammas
  double k_overall_memb, k_bin, memb_xo[3], memb_len, rho0_max, rho0_distor, g_memb[3][4];
  int memb_pore_type;
  // [Phosphorylation] (:413-421): hypercharge factor; the residues are flagged R_PHOSPH
  double k_hypercharge;
  int n_phosph_res, phosph_res[20];
  // [Vector_Fragment_Memory] (:328-333): strength and angle width (rad)
  double k_vfm, vfm_sigma_sq;
};

struct ForceField {
  FFParams p{};
  std::vector<double> tables;  // TB_SIZE doubles
  // one memory file, gamma file and strength serve both [Fragment_Memory] and
  // [Fragment_Memory_Table] (the reference reads them into the same variables)
  std::string fm_file, fm_gamma_file;
  double k_fm_raw = 0.0;
  double tb_width = 0.0;  // [Fragment_Memory_Table] well width (scales the Gaussian variance)
  int tb_use_file = 0;    // read the tables from fm_table.energy/.force when present, else write them
  int amh_go_censor = 0;  // [AMH-Go] frustration censoring flag (0 or 1)
  std::string cr_file;    // [Contact_Restraints] restraints file
  double k_water = 0.0;  // epsilon-scaled [Water] strength, applied to gamma.dat
};

// Gamma_Array (fragment-memory gamma by sequence separation and residue class)
struct GammaTable {
  int nseq_cl = 0, nres_cl = 0;
  bool frag_resty = false;
  int i_sep[10] = {0};
  std::vector<double> g;
  int min_sep() const { return i_sep[0]; }
  int max_sep() const { return i_sep[nseq_cl]; }
  double get(int ti, int tj, int tfi, int tfj, int ires, int jres) const;
};

struct Memory {
  int pos = 0, len = 0;
  double weight = 1.0;
  std::string se;
  std::vector<double> xca, xcb;  // [len*3], angstrom
};

// Per-system topology in the engine's internal atom order: atom 3*r + b with
// b = 0 CA, 1 CB (or H-beta), 2 O, residues in residue-id order.
struct Topology {
  int n_res = 0, n_atoms = 0, n_chains = 0;
  std::string seq;
  std::vector<int> res_type, res_flags, res_chain, chain_start, chain_end;  // chain_* per chain, inclusive
  std::vector<double> aps;  // [12][n_res]
  // external (caller) atom order
  std::vector<int> ext_of;      // internal atom -> external index
  std::vector<int> atom_type;   // internal atom -> LAMMPS type
  std::vector<int> atom_tag;    // internal atom -> atom id (Langevin stream key)
  std::vector<double> mass;     // internal atom
  // harmonic bonds (internal atom indices)
  std::vector<int> bond_i, bond_j;
  std::vector<double> bond_k, bond_r0;
  // pair vexcluded
  int ntypes = 0, ev_p = 2;
  std::vector<double> ev_pref, ev_cs, ev_cl;  // [(ntypes+1)^2]: lambda*sign, cut_short, cut_long
  // 1-2 exclusions between beads of residue r and r (self) / r+1 (next): 9-bit masks
  std::vector<uint32_t> excl_self, excl_next;
};

// Fragment memory in pair-major form: one row per (target residue i, sep d),
// each row a run of records (one per covering memory) of 4 distances
// (CA-CA, CA-CB, CB-CA, CB-CB); skipped glycine pairs hold FM_SKIP.
struct FMTable {
  static constexpr double FM_SKIP = 1e30;
  int nd = 0;                        // rows per residue (d = min_sep .. min_sep+nd-1)
  std::vector<int> row_start;        // [n_res*nd + 1] record offsets
  std::vector<double> rf;            // [records*4]
  std::vector<double> coef;          // [records] eps*k*w*gamma (empty when uniform)
  double uniform_coef = 0.0;
  bool uniform = true;
  long long records() const { return row_start.empty() ? 0 : row_start.back(); }
};

// Table fragment memory (FixBackbone::compute_fragment_memory_table,
// fix_backbone.cpp:4238-4322): for target residue i, separation slot
// jo = j - i - min_sep (< nbrs) and atom pair k, the energy and radial-force
// factor of every memory covering (i, j) summed on the grid r = tb_rmin +
// ir * tb_dr.  `present` marks the tables the reference allocates (some
// memory has the atom pair; a table read from files is always present).
struct FMTableTB {
  int nbrs = 0, size = 0;
  std::vector<double> data;      // [n_res][nbrs][4][size][2]: energy, force
  std::vector<uint8_t> present;  // [n_res][nbrs][4]
};

// AMH-Go (FixBackbone::compute_amh_go_model, fix_backbone.cpp:3850-3992):
// for atom slot 2 r + b (b = 0 CA, 1 CB) of target residue r, the native
// contacts it interacts with (the full list's partners j with
// |r - res(j)| >= min_sep or another molecule, not censored, native distance
// below rc), each with its native distance, gamma and Gaussian variance
// |r - res(j)|^0.3; and per residue the system's normalisation (:3787-3848).
struct AmhGoContacts {
  std::vector<int> start;                    // [2 n_res + 1]
  std::vector<int> partner;                  // internal atom 3 j + b
  std::vector<double> rnat, gamma, sig_sq;   // per contact
  std::vector<double> norm;                  // [n_res]: normalisation of the residue's system
};

// Contact restraints in residue-pair order: restraints of residue i (with a
// partner j > i) at [start[i], start[i+1]), sorted by j (fix_backbone.cpp:1106-1171)
struct ContactRestraints {
  std::vector<int> start, j;
  std::vector<double> w, r0;
};

// Vector fragment memory records of residue i: [start[i], start[i+1]), each
// a partner j and the memory's CA-CB angle between i and j (radians)
struct VfmRecords {
  std::vector<int> start, j;
  std::vector<double> angle;
};

struct SystemInput {
  ForceField ff;
  Topology top;
  GammaTable gamma;
  std::vector<Memory> mems;
  FMTable fm;
  FMTableTB tb;
  AmhGoContacts go;
  std::vector<double> charge;  // [n_res] Debye-Hueckel charges (charge_on_residues.dat)
  ContactRestraints cr;
  std::vector<int> zim;        // [n_res] membrane zone of each residue (file zim: 1, 2 or 3)
  VfmRecords vfm;
  std::vector<double> x, v;  // internal order [n_atoms*3]
};

// Parsers (throw std::runtime_error with the reference's message on errors)
void read_coeff_file(const std::string &path, ForceField &ff);
void read_tables(const std::string &dir, ForceField &ff, Topology &top);
void read_sequence(const std::string &path, Topology &top);
void read_gamma_table(const std::string &path, GammaTable &g);
void read_memories(const std::string &dir, const std::string &mem_file, int n_res, std::vector<Memory> &mems);

// Topology from per-atom arrays (any order).  role: 0 CA, 1 CB/H-beta, 2 O, -1 other.
void build_topology(Topology &top, int n_atoms, const int *role, const int *residue, const int *molecule,
                    const int *type, const int *tag, const double *mass_by_type, int ntypes);
void set_bonds(Topology &top, int nb, const int *bi, const int *bj, const double *k, const double *r0,
               const int *ext_to_int);
void set_pair_coeffs(Topology &top, const std::string &style, const std::string &coeffs);
void build_fm_table(const ForceField &ff, const Topology &top, const GammaTable &g,
                    const std::vector<Memory> &mems, FMTable &out);
// `dir`: where fm_table.energy / fm_table.force are read or written
void build_fm_table_tb(const ForceField &ff, const Topology &top, const GammaTable &g,
                       const std::vector<Memory> &mems, const std::string &dir, FMTableTB &out);
// AMH-Go native contacts and normalisation from `dir`'s amh-go.gamma, amh-go.gro
// (and frustration_censored_contacts.dat with censoring 1)
void build_amh_go(const ForceField &ff, const Topology &top, const std::string &dir, AmhGoContacts &out);
// FixBackbone's pair-list cutoff (fix_backbone.cpp:1051-1067) for the enabled terms
double pair_list_cutoff(const FFParams &p);

// A system from per-atom arrays in the caller's order (a host code's own
// atom data: roles 0 CA, 1 CB/H-beta, 2 O, -1 other; residue and molecule
// ids, types, tags, masses by type, x and v (either may be null), bonds as
// caller indices), with the coefficient file, sequence and tables of `dir`
// (read_files: also read the coefficient and sequence files).
void load_system_atoms(const std::string &dir, const std::string &coeff_file, const std::string &seq_file,
                       int natoms, const int *role, const int *res, const int *mol, const int *typ, const int *tag,
                       const double *mass, int ntypes, const double *xe, const double *ve, int nbonds,
                       const int *bond_a, const int *bond_b, const double *bond_k, const double *bond_r0,
                       const std::string &pair_style, const std::string &pair_coeffs, SystemInput &S,
                       bool read_files);

// Whole system from a directory laid out like a reference run directory.
void load_system_dir(const std::string &dir, const std::string &data_file, const std::string &coeff_file,
                     const std::string &seq_file, const std::string &pair_style, const std::string &pair_coeffs,
                     SystemInput &out);

// A batch of independent replicas concatenated for the device: residues,
// chains and atoms of replica k follow those of replica k-1; chain ids are
// global so different replicas never count as the same chain.  All replicas
// share one force field (same coefficient file, tables and pair_style).
struct Batch {
  ForceField ff;
  Topology top;       // concatenated topology (ext_of is per replica, see below)
  FMTable fm;         // concatenated fragment-memory rows
  FMTableTB tb;       // concatenated fragment-memory tables (per residue)
  AmhGoContacts go;   // concatenated AMH-Go contacts (partners offset to batch atoms)
  std::vector<double> charge;  // concatenated Debye-Hueckel charges
  ContactRestraints cr;        // concatenated contact restraints (residues offset)
  std::vector<int> zim;        // concatenated membrane zones
  VfmRecords vfm;              // concatenated vector fragment memory records (residues offset)
  std::vector<double> x, v;
  std::vector<int> res_sys;              // residue -> replica
  std::vector<int> sys_res_begin, sys_res_end;    // [n_sys]
  std::vector<int> sys_atom_begin;       // [n_sys + 1]
  std::vector<std::vector<int>> ext_of;  // per replica: local internal atom -> caller index
  int n_sys = 0;
};

// A Q order parameter over the CA atoms of one replica: compute qwolynes
// (src/compute_q_wolynes.cpp) or compute qonuchic (src/compute_q_onuchic.cpp)
// from the words after LAMMPS's `compute`.  kind 0: Q_W, sum over |i-j| > sep
// of exp(-(r - mat)^2 / 2 sigma^2), sigma = (1 + |i-j|)^sigma_exp; kind 1:
// count of native pairs (mat >= 0, |i-j| > 3) with r^2 < mat; kind 2: sum over
// them of exp(-(r - sqrt(mat))^2 / 2 sigma^2), sigma^2 = (1 + |i-j|)^(2 sigma_exp).
// The value is the sum times qnorm; only entries i < j of mat are read.
struct QDefinition {
  int kind = 0, n = 0, sep = 0;
  double sigma_exp = 0.15, qnorm = 0.0;
  std::vector<double> mat;  // [n*n]
};
QDefinition parse_q_compute(const std::string &words, int n_res);

// Concatenate replicas (each already loaded); throws if their force fields differ.
void assemble_batch(const std::vector<const SystemInput *> &reps, Batch &out);

// Force field shared by replicas given as arrays: coefficient file and the
// tables of a run directory, the fragment-memory gamma file, pair_style
// vexcluded settings, and the data-file conventions of the atom types
// (1 CA, 3 O, 4 CB, 5 H-beta), their masses and the five bond types.
struct SharedForceField {
  ForceField ff;
  GammaTable gamma;
  std::string pair_style, pair_coeffs;
  double mass[6] = {0, 27.0, 14.0, 28.0, 60.0, 2.0};
  double bond_k[6] = {0, 60, 60, 60, 60, 60}, bond_r0[6] = {0, 3.816, 2.40, 2.76, 1.53, 1.09};
};

void load_shared_forcefield(const std::string &dir, const std::string &coeff_file, const std::string &pair_style,
                            const std::string &pair_coeffs, SharedForceField &out);

// One replica from arrays (see awsem_replica_desc in awsem_gpu.h).
struct ReplicaArrays {
  int n_res, n_chains;
  const int *chain_len;
  const char *seq;
  const double *ssweight;  // [n_res][number of enabled SSWeight columns] or null
  const double *x, *v;     // [n_res][3 beads: CA, O, CB/HB][3] (data-file order)
  int n_mem;
  const int *mem_pos, *mem_len;
  const double *mem_weight;
  const char *mem_seq;
  const double *mem_ca, *mem_cb;
};
void load_system_arrays(const SharedForceField &sf, const ReplicaArrays &ra, SystemInput &out);

}  // namespace awsem
