/* FP64 CPU restatement of AWSEM-MD's per-step force and energy evaluation.

   ORACLE -- test infrastructure.  Only tests/, the package smoke check and
   bench.py's CPU-baseline leg load this library, and only as the checker.

   It restates, in plain loops over residue pairs (no neighbour list, no
   caches), the reference algorithm of:
     fix backbone      src/fix_backbone.cpp (adavtyan/awsemmd)
     fragment memory   src/fragment_memory.cpp
     pair vexcluded    src/pair_excluded_volume.cpp
   for the terms enabled by the default parameter file plus fragment memory:
   Chain, Chi, Rama (+Rama_P, SSWeight), ABC, Dssp_Hdrgn, P_AP, Water,
   Burial, Helix, Fragment_Memory, Epsilon.  Each function cites the
   reference lines it follows.  The LAMMPS pieces around the fix (harmonic
   bonds, velocity Verlet, Langevin, units real) are restated from the LAMMPS
   documentation; the Langevin noise uses the same counter-based uniform
   stream as the GPU engine (SplitMix64 finaliser keyed by seed, step, atom
   id and component).

   The restatement is checked against the reference compiled against the
   LAMMPS-API shim (oracle/_ref) on the same inputs. */
#include "awsem_oracle.h"
#include "../include/awsem_gpu.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>

namespace {

const double BOLTZ = 0.0019872067;
const double MVV2E = 48.88821291 * 48.88821291;
const double FTM2V = 1.0 / 48.88821291 / 48.88821291;

const char AA[] = "ARNDCQEGHILKMFPSTWYV";

int aa_index(char c)
{
  for (int k = 0; k < 20; k++)
    if (AA[k] == c) return k;
  return 0;  // the reference maps unknown letters to 0 (se_map, fix_backbone.cpp:55)
}

/* four residue classes of Gamma_Array (fragment_memory.cpp:28): 1 SHL,
   2 AHL, 3 BAS, 4 HPB, indexed by the AA order above */
int four_class(int t)
{
  static const int m[20] = {1, 3, 2, 2, 4, 2, 2, 1, 3, 4, 4, 3, 4, 4, 1, 1, 1, 4, 4, 4};
  return m[t];
}

inline uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, int64_t step, int64_t tag, int comp)
{
  uint64_t key = mix64(seed ^ mix64((uint64_t) step));
  uint64_t r = mix64(key ^ ((uint64_t) tag * 4ULL + (uint64_t) comp));
  return (double) (r >> 11) * (1.0 / 9007199254740992.0);
}

/* selection keys: kind << 56 | aux << 44 | i << 22 | j (awsem_gpu.h) */
inline uint64_t sel_key(int kind, int aux, int i, int j)
{
  return (uint64_t) kind << 56 | (uint64_t) aux << 44 | (uint64_t) i << 22 | (uint64_t) j;
}
/* reference cache entries (oracle and reference host only) */
enum { TOUCH_WELL = 32, TOUCH_HWELL = 33, TOUCH_RNO = 34, TOUCH_RHO = 35, TOUCH_NU = 36 };
/* v within 2e-6 (relative) of the threshold t: FP32 geometry may decide otherwise */
inline bool near_thr(double v, double t) { return fabs(v - t) <= 2e-6 * fabs(t); }

std::vector<std::string> words(const std::string &s)
{
  std::istringstream is(s);
  std::vector<std::string> v;
  std::string t;
  while (is >> t) v.push_back(t);
  return v;
}

std::string join(const std::string &dir, const std::string &f)
{
  if (f.empty() || f[0] == '/' || dir.empty()) return f;
  return dir + "/" + f;
}

enum { ET_TOTAL = 0, ET_CHAIN, ET_SHAKE, ET_CHI, ET_RAMA, ET_VEXCLUDED, ET_DSSP, ET_PAP, ET_WATER,
       ET_BURIAL, ET_HELIX, ET_AMHGO, ET_FRAGMEM, ET_VFRAGMEM, ET_CONT_REST, ET_MEMB, ET_SSB, ET_DH, NET };

struct Params {
  double epsilon = 1.0;
  bool abc = 0, chain = 0, chi = 0, rama = 0, rama_p = 0, ssw = 0, dssp = 0, pap = 0, water = 0,
       burial = 0, helix = 0, fm = 0, fm_tb = 0;
  // defaults of fix_backbone.cpp:136-143
  double an = 0.4831806, bn = 0.7032820, cn = -0.1864262;
  double ap = 0.4436538, bp = 0.2352006, cp = 0.3211455;
  double ah = 0.8409657, bh = 0.8929599, ch = -0.7338894;
  double k_chain[3] = {0, 0, 0}, r_ncb0 = 0, r_cpcb0 = 0, r_ncp0 = 0;
  double k_chi = 0, chi0 = 0;
  double k_rama = 0;
  int n_rama = 0, n_rama_p = 0;
  static const int i_rp = 6;
  double w[12] = {0}, sigma[12] = {0}, phiw[12] = {0}, phi0[12] = {0}, psiw[12] = {0}, psi0[12] = {0};
  bool ssweight[12] = {0};
  double hbscl[4][9] = {{0}};
  double sigma_NO = 0, sigma_HO = 0, NO_zero = 0, HO_zero = 0, k_dssp = 0, dssp_cut = 0, dssp_cut_sq = 0;
  double pref[2] = {0, 0}, d_nu0 = 0, nu_cut1_sq = 0, nu_cut2_sq = 0, sigma_NO_sqinv = 0, sigma_HO_sqinv = 0;
  double k_global_pap = 0, k_betapred_pap = 0, k_pap[3] = {0, 0, 0}, pap_cut = 0, pap_pref = 0,
         pap_cutoff_sq = 0;
  int i_med_min = 0, i_med_max = 0, i_diff_pap = 0;
  double k_water = 0, water_kappa = 0, water_kappa_sigma = 0, treshold = 0;
  int contact_cutoff = 0, n_wells = 0, well_flag[5] = {0};
  double well_rmin[5] = {0}, well_rmax[5] = {0};
  double k_burial = 0, burial_kappa = 0, burial_ro_min[3] = {0}, burial_ro_max[3] = {0};
  double k_helix = 0, helix_gamma_p = 0, helix_gamma_w = 0, helix_kappa = 0, helix_kappa_sigma = 0,
         helix_treshold = 0, helix_cutoff = 0, helix_cutoff_sq = 0;
  int helix_i_diff = 0, pro_acc_flag = 0;
  double helix_rmin = 0, helix_rmax = 0, h4prob[20] = {0}, h4prob_pro = 0;
  double helix_sigma_HO = 0, helix_sigma_NO = 0, helix_HO_zero = 0, helix_NO_zero = 0,
         helix_sigma_HO_sqinv = 0, helix_sigma_NO_sqinv = 0;
  double k_fm = 0, fm_sigma_exp = 0.15;
  std::string fm_file, fm_gamma_file;
  // [AMH-Go] (fix_backbone.cpp:297-303)
  bool amhgo = 0;
  double k_amh_go = 0, amh_go_p = 0, amh_go_rc = 0;
  int censoring = 0;
  // [Solvent_Barrier] (:334-345), [DebyeHuckel] (:467-477), [Contact_Restraints] (:321-327)
  bool ssb = 0, huckel = 0, cont_rest = 0;
  double k_solventb1 = 0, k_solventb2 = 0, ssb_rmin1 = 0, ssb_rmax1 = 0, ssb_rmin2 = 0, ssb_rmax2 = 0, ssb_kappa = 0;
  double ssb_rshift[20] = {0};
  int ssb_ij_sep = 0, ssb_rad_cor = 0, debye_huckel_min_sep = 0;
  double k_PlusPlus = 0, k_MinusMinus = 0, k_PlusMinus = 0, k_screening = 0, screening_length = 0;
  double k_cont_rest = 0, cr_sigma = 0, cr_sigma_sq_inv = 0, cr_dr_cutoff = 0, cr_glob_cutoff_sq = 0;
  std::string cr_file;
  // [Shake] (:180-183), [Membrane] (:346-358), [Phosphorylation] (:413-421)
  bool shake = 0, memb = 0, phosph = 0;
  double k_shake = 0, r_sh1 = 0, r_sh2 = 0, r_sh3 = 0;
  double k_overall_memb = 0, k_bin = 0, memb_xo[3] = {0, 0, 0}, memb_len = 0, rho0_max = 0, rho0_distor = 0;
  double g_memb[3][4] = {{0}};
  int memb_pore_type = 0;
  double k_hypercharge = 0;
  int n_phosph_res = 0, phosph_res[20] = {0};
  double phosph_water_gamma[5][20][20][2];
  // [Vector_Fragment_Memory] (:328-333)
  bool vfm = 0;
  double k_vec_frag_mem = 0, vfm_sigma = 0, vfm_sigma_sq = 0;
  // [Fragment_Memory_Table] (fix_backbone.cpp:310-321)
  double tb_rmin = 0, tb_rmax = 0, tb_dr = 0, tb_width = 0;
  int tb_size = 0, tb_use_file = 0;
  double m_anti_HB[20][20][2], m_anti_NHB[20][20][2], m_para_HB[20][20][2], m_para_one[20], m_anti_one[20];
  double water_gamma[5][20][20][2];
  double burial_gamma[20][3];
  // derived well supports (smart_matrix_lib.h:363-368)
  double w_rmin_th[5], w_rmax_th[5], w_rmin_sq[5], w_rmax_sq[5];
  double h_rmin_th, h_rmax_th, h_rmin_sq, h_rmax_sq;
  double pap_drmin_sq, pap_drmax_sq;
};

/* Gamma_Array (fragment_memory.cpp:275-454) */
struct GammaArray {
  int nseq_cl = 0, nres_cl = 0;
  bool frag_resty = false;
  int i_sep[10];
  std::vector<double> g;

  int min_sep() const { return i_sep[0]; }
  int max_sep() const { return i_sep[nseq_cl]; }

  void idx_list(const std::string &t, std::vector<int> &out)
  {
    out.clear();
    if (t == "ALL") {
      for (int i = 0; i < nres_cl; i++) out.push_back(i);
    } else if (t.size() == 1) {
      if (nres_cl < 20) throw std::runtime_error("gamma file: residue code needs 20 classes");
      out.push_back(aa_index(t[0]));
    } else if (t.size() == 3) {
      int c = t == "SHL" ? 1 : t == "AHL" ? 2 : t == "BAS" ? 3 : t == "HPB" ? 4 : 0;
      if (!c) throw std::runtime_error("gamma file: unknown residue class " + t);
      if (nres_cl == 4) out.push_back(c - 1);
      else
        for (int i = 0; i < 20; i++)
          if (four_class(i) == c) out.push_back(i);
    } else
      throw std::runtime_error("gamma file: bad residue code " + t);
  }

  void load(const std::string &path)
  {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Fragment_Memory: Cannot read gamma file " + path);
    std::vector<std::vector<std::string>> rows;
    std::string line;
    bool first = true;
    while (std::getline(in, line)) {
      if (!line.empty() && line[0] == '#') continue;
      auto v = words(line);
      if (v.empty()) continue;
      if (first) {
        int ns = 0;
        for (auto &t : v) {
          ns++;
          if (t == "inf") {
            i_sep[ns - 1] = -1;
            break;
          }
          i_sep[ns - 1] = atoi(t.c_str());
        }
        nseq_cl = ns - 1;
        if (nseq_cl == 0) throw std::runtime_error("gamma file: no separation classes");
        first = false;
        continue;
      }
      if (v.size() != 4 && v.size() != 6) throw std::runtime_error("gamma file: bad entry");
      rows.push_back(v);
    }
    if (rows.empty()) throw std::runtime_error("gamma file: no entries");
    frag_resty = rows[0].size() == 6;
    for (auto &r : rows) {
      if ((r.size() == 6) != frag_resty) throw std::runtime_error("gamma file: mixed entry forms");
      for (size_t k = 0; k + 2 < r.size(); k++) {
        const std::string &t = r[k];
        if (t == "ALL") nres_cl = std::max(nres_cl, 1);
        else if (t.size() == 3) nres_cl = std::max(nres_cl, 4);
        else if (t.size() == 1) nres_cl = std::max(nres_cl, 20);
      }
    }
    int n2 = nres_cl * nres_cl;
    g.assign((size_t) nseq_cl * (frag_resty ? n2 * n2 : n2), 0.0);
    std::vector<int> is, js, ks, ls;
    for (auto &r : rows) {
      if (!frag_resty) {
        int cl = atoi(r[2].c_str());
        double gm = atof(r[3].c_str());
        idx_list(r[0], is);
        idx_list(r[1], js);
        for (int a : is)
          for (int b : js) {
            g[(size_t) (cl - 1) * n2 + a * nres_cl + b] = gm;
            g[(size_t) (cl - 1) * n2 + b * nres_cl + a] = gm;
          }
      } else {
        // the reference passes the i-fragment class twice (fragment_memory.cpp:369)
        int cl = atoi(r[4].c_str());
        double gm = atof(r[5].c_str());
        idx_list(r[0], is);
        idx_list(r[1], js);
        idx_list(r[2], ks);
        idx_list(r[2], ls);
        size_t base = (size_t) (cl - 1) * n2 * n2;
        for (int a : is)
          for (int b : js)
            for (int c : ks)
              for (int d : ls) {
                g[base + ((size_t) a * nres_cl + b) * n2 + c * nres_cl + d] = gm;
                g[base + ((size_t) b * nres_cl + a) * n2 + c * nres_cl + d] = gm;
                g[base + ((size_t) a * nres_cl + b) * n2 + d * nres_cl + c] = gm;
                g[base + ((size_t) b * nres_cl + a) * n2 + d * nres_cl + c] = gm;
              }
      }
    }
  }

  /* getGamma, fragment_memory.cpp:400-454 */
  double get(int ti, int tj, int tfi, int tfj, int ires, int jres) const
  {
    int dij = abs(ires - jres);
    if (dij < i_sep[0] || (i_sep[nseq_cl] != -1 && dij > i_sep[nseq_cl])) return 0.0;
    int cl;
    for (cl = 1; cl < nseq_cl && dij >= i_sep[cl]; cl++) {}
    if (nres_cl == 1) return g[cl - 1];
    auto c = [&](int t) { return nres_cl == 4 ? four_class(t) - 1 : t; };
    int n2 = nres_cl * nres_cl;
    if (!frag_resty) return g[(size_t) (cl - 1) * n2 + c(ti) * nres_cl + c(tj)];
    return g[(size_t) (cl - 1) * n2 * n2 + ((size_t) c(ti) * nres_cl + c(tj)) * n2 + c(tfi) * nres_cl + c(tfj)];
  }
};

/* one fragment memory (fragment_memory.cpp:34-176): residues pos..pos+len-1
   of the target, CA/CB coordinates read from a .gro file (nm -> A) */
struct Memory {
  int pos, len;
  double weight;
  std::string se;
  std::vector<double> rf0, rf1;  // [len*len]: CA-CA (i<j) / CB-CB (i>j); CA_i-CB_j
  std::vector<double> vmf;       // [len*len]: angle between the CA->CB vectors of i and j (VM)

  double R(const double *a, const double *b) const
  {
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
  }

  /* Rf(ires, iatom, jres, jatom), fragment_memory.cpp:190-202; atom 1 CA, 2 CB */
  double rf(int ires, int iat, int jres, int jat) const
  {
    ires -= pos;
    jres -= pos;
    if (iat == 1 && jat == 1) return rf0[std::min(ires, jres) * len + std::max(ires, jres)];
    if (iat == 2 && jat == 2) return rf0[std::max(ires, jres) * len + std::min(ires, jres)];
    return iat == 1 ? rf1[ires * len + jres] : rf1[jres * len + ires];
  }
};

char three_to_one(const std::string &t)
{
  static const char *names[20] = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
                                  "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"};
  for (int k = 0; k < 20; k++)
    if (t == names[k]) return AA[k];
  return '?';
}

struct System {
  std::string workdir;
  Params P;
  GammaArray G;
  std::vector<Memory> mems;
  std::vector<std::vector<int>> fm_map;  // per residue: memories listing it
  // table fragment memory: [4 * n * tb_nbrs] tables of tb_size points (empty: not allocated)
  int tb_nbrs = 0;
  std::vector<std::vector<double>> tb_e, tb_f;
  bool tb_files() const;
  void build_tb();
  void tb_term(int i, double *f);

  // AMH-Go: native structure, gamma, normalisation, censored residue pairs
  GammaArray go_gamma;
  Memory go_mem;                   // the native structure, amh-go.gro (all n residues)
  std::vector<char> go_censored;   // [n*n]
  double go_norm = 0.0;
  double plc = 0.0;  // the fix's pair-list cutoff (fix_backbone.cpp:1048-1066)
  // The fix's full neighbour list (cut plc + skin) and LAMMPS's rebuild rule
  // (Neighbor::decide with delay / every / check, the half-skin trigger).
  double nb_skin = 2.0;
  int nb_delay = 0, nb_every = 1, nb_check = 1;
  bool list_setup = true;  // the next compute is a run setup: the list is built
  long long list_ago = 0;
  std::vector<double> xhold;  // positions at the last build
  bool lists_used() const { return P.amhgo || P.ssb || P.huckel || P.cont_rest; }
  void list_update(const double *x);
  bool in_list(int a, int b) const;
  // Debye-Hueckel charges and contact restraints (per residue min(i1, i2), sorted by the other)
  std::vector<int> phosph_map;  // [n]: phosphorylated residues
  std::vector<int> z_res;       // [n]: membrane zones (zim)
  /* get_water_gamma, fix_backbone.cpp:2872-2885 */
  double water_gamma(int i, int j, int w, int ti, int tj, int c) const
  {
    if (P.phosph && (phosph_map[i] || phosph_map[j])) return P.phosph_water_gamma[w][ti][tj][c];
    return P.water_gamma[w][ti][tj][c];
  }
  void shake_term(int i, double *f);
  void vfm_term(int i, double *f);
  void membrane_term(int i, double *f);
  std::vector<double> charge;
  struct Restraint { int i2; double w, r0; };
  std::vector<std::vector<Restraint>> cr_map;
  void read_pair_extras();
  void pair_extras(const double *x, double *f);
  void solvent_barrier(int i, int j, const double *x, double *f);
  void debye_huckel(int i, int j, const double *x, double *f);
  void read_amh_go();
  void amhgo_normalization();
  void amhgo_term(const double *x, double *f);

  // topology
  int natoms = 0, n = 0, nch = 0;
  std::vector<int> ch_pos1, ch_len;  // 1-based first residue, length
  std::string se;
  std::vector<int> ca, cb, o;  // atom index per residue (cb = CB or H-beta)
  std::vector<int> chain_of;   // 0-based chain of residue
  std::vector<double> aps[12];
  std::vector<int> atype, amol, ares, tag;
  std::vector<double> mass;  // by type
  // bonds
  std::vector<int> b_t, b_i, b_j;
  std::vector<double> bk, br0;
  std::vector<std::vector<int>> special;
  // pair vexcluded
  int ev_p = 2;
  double ev_cs_glob = 0, ev_cl_glob = 0;
  std::vector<double> ev_lambda, ev_cs, ev_cl;  // [(ntypes+1)^2]
  std::vector<int> ev_set;
  int ntypes = 0;

  // per-step working arrays
  std::vector<double> xca, xcb, xo, xn, xh, xcp;  // [n*3]
  std::vector<double> rho_w, rho_h, sig_w, sigp_w, sig_h, sigp_h, xi_w, xi1, xi2, bur;
  double E[NET];
  double e_pair = 0, e_bond = 0;
  // Selections of the last compute, recorded when sel_on: sel_keys holds one
  // AWSEM_SEL_* key per selected item (include/awsem_gpu.h), near_keys the
  // distance predicates decided within 2e-6 (relative) of their threshold
  // (where FP32 geometry may decide otherwise), touch_keys the entries of the
  // reference's n x n caches (cWell, cR, cP_AP, smart_matrix_lib.h) that the
  // reference evaluation reads or fills, in its own index order.
  bool sel_on = false;
  std::vector<uint64_t> sel_keys, near_keys, touch_keys;
  void sel(int kind, int aux, int i, int j)
  {
    if (sel_on) sel_keys.push_back(sel_key(kind, aux, i, j));
  }
  void near(int kind, int aux, int i, int j)
  {
    if (sel_on) near_keys.push_back(sel_key(kind, aux, i, j));
  }
  void touch(int kind, int aux, int i, int j)
  {
    if (sel_on) touch_keys.push_back(sel_key(kind, aux, i, j));
  }

  bool first(int i) const { return ch_pos1[chain_of[i]] == i + 1; }
  bool last(int i) const { return ch_pos1[chain_of[i]] + ch_len[chain_of[i]] - 1 == i + 1; }
  int type_of(int i) const { return aa_index(se[i]); }
  int contact_atom(int i) const { return se[i] == 'G' ? ca[i] : cb[i]; }
  bool bonded(int a, int b) const { return std::find(special[a].begin(), special[a].end(), b) != special[a].end(); }

  void read_coeff(const std::string &path);
  void read_tables();
  void read_data(const std::string &path);
  void read_seq(const std::string &path);
  void read_mems();
  void pair_setup(const std::string &style, const std::string &coeffs);
  void compute(const double *x, double *f);
  void backbone_atoms(const double *x);
  void chain_term(int i, double *f);
  void chi_term(int i, double *f);
  void rama_term(int i, double *f);
  void dihedral_slopes(int i, int iang, double &angle, double ys[5][3], double xs[5][3]);
  int dssp_term(int i, int j, double *f);
  void pap_nu(int i, int j, double &nu, double &prd);
  int pap_term(int i, int j, double *f);
  int helix_pair(int i, int j, double *f);
  void fm_term(int i, double *f);
  void pair_terms(const double *x, double *f);
  void excluded_volume(const double *x, double *f);
  void bonds(const double *x, double *f);
};

/* coefficient file: section loop and epsilon scaling, fix_backbone.cpp:164-516 */
void System::read_coeff(const std::string &path)
{
  std::ifstream in(path);
  if (!in) throw std::runtime_error("Coefficient file was not found!");
  Params &p = P;
  std::string s;
  static const char *unsupported[] = {"[Excluded]", "[Excluded_P]", "[Excluded_R6]",
                                      "[Fragment_Frustratometer]", "[Tertiary_Frustratometer]",
                                      "[Nmer_Frustratometer]", "[Amylometer]",
                                      "[Selection_Temperature]", "[Monte_Carlo_Seq_Opt]", "[Optimization]",
                                      "[Burial_Optimization]", "[DebyeHuckel_Optimization]",
                                      "[Shuffler]", "[Mutate_Sequence]"};
  while (in >> s) {
    if (s == "[ABC]") {
      p.abc = 1;
      in >> p.an >> p.bn >> p.cn >> p.ap >> p.bp >> p.cp >> p.ah >> p.bh >> p.ch;
    } else if (s == "[Chain]") {
      p.chain = 1;
      in >> p.k_chain[0] >> p.k_chain[1] >> p.k_chain[2] >> p.r_ncb0 >> p.r_cpcb0 >> p.r_ncp0;
    } else if (s == "[Chi]") {
      p.chi = 1;
      in >> p.k_chi >> p.chi0;
    } else if (s == "[Rama]") {
      p.rama = 1;
      in >> p.k_rama >> p.n_rama;
      for (int j = 0; j < p.n_rama; j++) {
        in >> p.w[j] >> p.sigma[j] >> p.phiw[j] >> p.phi0[j] >> p.psiw[j] >> p.psi0[j];
        p.phiw[j] *= p.sigma[j];
        p.psiw[j] *= p.sigma[j];
      }
    } else if (s == "[Rama_P]") {
      p.rama_p = 1;
      in >> p.n_rama_p;
      for (int j = 0; j < p.n_rama_p; j++) {
        int q = j + Params::i_rp;
        in >> p.w[q] >> p.sigma[q] >> p.phiw[q] >> p.phi0[q] >> p.psiw[q] >> p.psi0[q];
        p.phiw[q] *= p.sigma[q];
        p.psiw[q] *= p.sigma[q];
      }
    } else if (s == "[SSWeight]") {
      p.ssw = 1;
      for (int j = 0; j < 12; j++) {
        int v;
        in >> v;
        p.ssweight[j] = v != 0;
      }
    } else if (s == "[Dssp_Hdrgn]") {
      p.dssp = 1;
      in >> p.k_dssp >> p.hbscl[0][0] >> p.hbscl[0][1];
      for (int j = 0; j < 7; j++) in >> p.hbscl[1][j];
      for (int j = 0; j < 9; j++) in >> p.hbscl[2][j];
      for (int j = 0; j < 9; j++) in >> p.hbscl[3][j];
      in >> p.sigma_HO >> p.sigma_NO >> p.HO_zero >> p.NO_zero >> p.dssp_cut >> p.pref[0] >> p.pref[1] >> p.d_nu0;
      p.dssp_cut_sq = p.dssp_cut * p.dssp_cut;
      p.nu_cut1_sq = pow(p.d_nu0 + atanh(2.0 * 1e-4 - 1.0) / p.pref[0], 2);
      p.nu_cut2_sq = pow(p.d_nu0 + atanh(2.0 * 1e-4 - 1.0) / p.pref[1], 2);
      p.sigma_HO_sqinv = 1.0 / (p.sigma_HO * p.sigma_HO);
      p.sigma_NO_sqinv = 1.0 / (p.sigma_NO * p.sigma_NO);
    } else if (s == "[P_AP]") {
      p.pap = 1;
      in >> p.k_global_pap >> p.k_betapred_pap >> p.k_pap[0] >> p.k_pap[1] >> p.k_pap[2] >> p.pap_cut >>
          p.pap_pref >> p.i_med_min >> p.i_med_max >> p.i_diff_pap;
      p.pap_cutoff_sq = pow(p.pap_cut + atanh(1.0 - 2.0 * 1e-12) / p.pap_pref, 2);
    } else if (s == "[Water]") {
      p.water = 1;
      in >> p.k_water >> p.water_kappa >> p.water_kappa_sigma >> p.treshold >> p.contact_cutoff >> p.n_wells;
      for (int j = 0; j < p.n_wells; j++) in >> p.well_rmin[j] >> p.well_rmax[j] >> p.well_flag[j];
    } else if (s == "[Burial]") {
      p.burial = 1;
      in >> p.k_burial >> p.burial_kappa;
      for (int j = 0; j < 3; j++) in >> p.burial_ro_min[j] >> p.burial_ro_max[j];
    } else if (s == "[Helix]") {
      p.helix = 1;
      in >> p.k_helix >> p.helix_gamma_p >> p.helix_gamma_w >> p.helix_kappa >> p.helix_kappa_sigma >>
          p.helix_treshold >> p.helix_i_diff >> p.helix_cutoff;
      p.helix_cutoff_sq = p.helix_cutoff * p.helix_cutoff;
      in >> p.helix_rmin >> p.helix_rmax;
      for (int j = 0; j < 20; j++) in >> p.h4prob[j];
      in >> p.pro_acc_flag >> p.h4prob_pro >> p.helix_sigma_HO >> p.helix_sigma_NO >> p.helix_HO_zero >>
          p.helix_NO_zero;
      p.helix_sigma_HO_sqinv = 1.0 / (p.helix_sigma_HO * p.helix_sigma_HO);
      p.helix_sigma_NO_sqinv = 1.0 / (p.helix_sigma_NO * p.helix_sigma_NO);
    } else if (s == "[Fragment_Memory]") {
      p.fm = 1;
      in >> p.k_fm >> p.fm_file >> p.fm_gamma_file;
    } else if (s == "[Fragment_Memory_Table]") {
      p.fm_tb = 1;
      in >> p.k_fm >> p.fm_file >> p.fm_gamma_file;
      in >> p.tb_rmin >> p.tb_rmax >> p.tb_dr;
      p.tb_size = (int) ((p.tb_rmax - p.tb_rmin) / p.tb_dr) + 2;
      in >> p.tb_width >> p.tb_use_file >> p.fm_sigma_exp;
    } else if (s == "[AMH-Go]") {
      p.amhgo = 1;
      in >> p.k_amh_go >> p.amh_go_p >> p.amh_go_rc;
      // the reference reads the censoring flag unconditionally; a file without
      // it leaves its stream failed, so the oracle asks for it
      if (!(in >> p.censoring)) throw std::runtime_error("[AMH-Go]: the frustration censoring flag is missing");
      if (p.censoring == 2) throw std::runtime_error("oracle: [AMH-Go] censoring 2 is not part of the restated path");
    } else if (s == "[Vector_Fragment_Memory]") {
      p.vfm = 1;
      in >> p.k_vec_frag_mem >> p.vfm_sigma;
      p.vfm_sigma_sq = p.vfm_sigma * p.vfm_sigma;
    } else if (s == "[Shake]") {
      p.shake = 1;
      in >> p.k_shake >> p.r_sh1 >> p.r_sh2 >> p.r_sh3;
    } else if (s == "[Membrane]") {
      p.memb = 1;
      in >> p.k_overall_memb >> p.k_bin >> p.memb_xo[0] >> p.memb_xo[1] >> p.memb_xo[2] >> p.memb_pore_type >>
          p.memb_len >> p.rho0_max >> p.rho0_distor;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 4; ++j) in >> p.g_memb[i][j];
    } else if (s == "[Phosphorylation]") {
      if (!p.water) throw std::runtime_error("Cannot run phosphorylation without water potential");
      p.phosph = 1;
      in >> p.k_hypercharge >> p.n_phosph_res;
      if (p.n_phosph_res > 20) throw std::runtime_error("Number of phosphorylated residues may not exceed 20");
      for (int i = 0; i < p.n_phosph_res; ++i) in >> p.phosph_res[i];
    } else if (s == "[Solvent_Barrier]") {
      p.ssb = 1;
      in >> p.k_solventb1 >> p.ssb_rmin1 >> p.ssb_rmax1 >> p.k_solventb2 >> p.ssb_rmin2 >> p.ssb_rmax2 >> p.ssb_kappa >>
          p.ssb_ij_sep >> p.ssb_rad_cor;
      for (int j = 0; j < 20; ++j) in >> p.ssb_rshift[j];
    } else if (s == "[DebyeHuckel]") {
      p.huckel = 1;
      in >> p.k_PlusPlus >> p.k_MinusMinus >> p.k_PlusMinus >> p.k_screening >> p.screening_length >>
          p.debye_huckel_min_sep;
    } else if (s == "[Contact_Restraints]") {
      p.cont_rest = 1;
      in >> p.k_cont_rest >> p.cr_sigma >> p.cr_file;
      p.cr_sigma_sq_inv = pow(p.cr_sigma, -2);
    } else if (s == "[Epsilon]") {
      in >> p.epsilon;
    } else {
      for (const char *u : unsupported)
        if (s == u) throw std::runtime_error("oracle: section " + s + " is not part of the restated path");
    }
  }
  // epsilon scaling (fix_backbone.cpp:501-516)
  for (double &k : p.k_chain) k *= p.epsilon;
  p.k_chi *= p.epsilon;
  p.k_rama *= p.epsilon;
  p.k_water *= p.epsilon;
  p.k_burial *= p.epsilon;
  p.k_helix *= p.epsilon;
  p.k_dssp *= p.epsilon;
  p.k_global_pap *= p.epsilon;
  p.k_amh_go *= p.epsilon;
  p.k_cont_rest *= p.epsilon;
  for (int j = 0; j < p.n_rama; j++) p.w[j] *= p.k_rama;
  for (int j = 0; j < p.n_rama_p; j++) p.w[j + Params::i_rp] *= p.k_rama;
  // well supports: rmin - 8 ln10/kappa, rmax + 8 ln10/kappa (smart_matrix_lib.h:363-368)
  for (int k = 0; k < p.n_wells; k++) {
    p.w_rmin_th[k] = p.well_rmin[k] - 8.0 * 2.302585 / p.water_kappa;
    p.w_rmax_th[k] = p.well_rmax[k] + 8.0 * 2.302585 / p.water_kappa;
    p.w_rmin_sq[k] = p.w_rmin_th[k] * p.w_rmin_th[k];
    p.w_rmax_sq[k] = p.w_rmax_th[k] * p.w_rmax_th[k];
  }
  if (p.helix) {
    p.h_rmin_th = p.helix_rmin - 8.0 * 2.302585 / p.helix_kappa;
    p.h_rmax_th = p.helix_rmax + 8.0 * 2.302585 / p.helix_kappa;
    p.h_rmin_sq = p.h_rmin_th * p.h_rmin_th;
    p.h_rmax_sq = p.h_rmax_th * p.h_rmax_th;
  }
  if (p.pap) {
    // smart_matrix_lib.h:110-115
    double drmax = p.pap_cut + double(int(8.0 * 2.302585 / p.pap_pref) + 1);
    double drmin = p.pap_cut - double(int(8.0 * 2.302585 / p.pap_pref) + 1);
    p.pap_drmax_sq = drmax * drmax;
    p.pap_drmin_sq = drmin * drmin;
  }
}

/* parameter tables read from the working directory (fix_backbone.cpp:555-693) */
void System::read_tables()
{
  Params &p = P;
  if (p.dssp) {
    std::ifstream a(join(workdir, "anti_HB")), b(join(workdir, "anti_NHB")), c(join(workdir, "para_HB")),
        d(join(workdir, "para_one")), e(join(workdir, "anti_one"));
    if (!a || !b || !c || !d || !e) throw std::runtime_error("DSSP table file missing");
    for (int i = 0; i < 20; i++) {
      d >> p.m_para_one[i];
      e >> p.m_anti_one[i];
      for (int j = 0; j < 20; j++) {
        a >> p.m_anti_HB[i][j][0];
        b >> p.m_anti_NHB[i][j][0];
        c >> p.m_para_HB[i][j][0];
      }
    }
    for (int i = 0; i < 20; i++)
      for (int j = 0; j < 20; j++) {
        a >> p.m_anti_HB[i][j][1];
        b >> p.m_anti_NHB[i][j][1];
        c >> p.m_para_HB[i][j][1];
      }
    if (!a || !b || !c || !d || !e) throw std::runtime_error("DSSP file format error");
  }
  for (int k = 0; k < 12; k++) aps[k].assign(n, 0.0);
  if (p.ssw) {
    std::ifstream in(join(workdir, "ssweight"));
    if (!in) throw std::runtime_error("File ssweight doesn't exist");
    for (int j = 0; j < n; j++)
      for (int k = 0; k < 12; k++)
        if (p.ssweight[k]) in >> aps[k][j];
  }
  if (p.water) {
    std::ifstream in(join(workdir, "gamma.dat"));
    if (!in) throw std::runtime_error("File gamma.dat doesn't exist");
    for (int w = 0; w < p.n_wells; w++)
      for (int i = 0; i < 20; i++)
        for (int j = i; j < 20; j++) {
          in >> p.water_gamma[w][i][j][0] >> p.water_gamma[w][i][j][1];
          if (!in) throw std::runtime_error("gamma.dat format error");
          p.water_gamma[w][i][j][0] *= p.k_water;
          p.water_gamma[w][i][j][1] *= p.k_water;
          p.water_gamma[w][j][i][0] = p.water_gamma[w][i][j][0];
          p.water_gamma[w][j][i][1] = p.water_gamma[w][i][j][1];
        }
  }
  if (p.phosph) {
    // fix_backbone.cpp:643-670
    static const int bb_four_letter_map[20] = {1, 3, 2, 2, 4, 2, 2, 1, 3, 4, 4, 3, 4, 4, 1, 1, 1, 4, 4, 4};
    for (int w = 0; w < p.n_wells; ++w)
      for (int i = 0; i < 20; ++i)
        for (int j = i; j < 20; ++j)
          for (int c = 0; c < 2; c++)
            p.phosph_water_gamma[w][i][j][c] = p.phosph_water_gamma[w][j][i][c] = p.water_gamma[w][i][j][c];
    for (int w = 0; w < p.n_wells; ++w)
      for (int i = 0; i < 20; ++i)
        for (int c = 0; c < 2; c++) {
          double g = p.phosph_water_gamma[w][i][6][c];
          if (bb_four_letter_map[i] == 1) g *= p.k_hypercharge;
          else if (bb_four_letter_map[i] == 2 || bb_four_letter_map[i] == 3) g *= pow(p.k_hypercharge, 2);
          p.phosph_water_gamma[w][i][15][c] = p.phosph_water_gamma[w][15][i][c] = g;
        }
    phosph_map.assign(n, 0);
    for (int j = 0; j < p.n_phosph_res; ++j)
      if (p.phosph_res[j] != 0) {
        if (p.phosph_res[j] < 1 || p.phosph_res[j] > n) throw std::runtime_error("oracle: phosphorylated residue out of range");
        phosph_map[p.phosph_res[j] - 1] = 1;
      }
  }
  if (p.burial) {
    std::ifstream in(join(workdir, "burial_gamma.dat"));
    if (!in) throw std::runtime_error("File burial_gamma.dat doesn't exist");
    for (int i = 0; i < 20; i++) in >> p.burial_gamma[i][0] >> p.burial_gamma[i][1] >> p.burial_gamma[i][2];
    if (!in) throw std::runtime_error("burial_gamma.dat format error");
  }
}

void System::read_seq(const std::string &path)
{
  std::ifstream in(path);
  if (!in) throw std::runtime_error("Sequence file was not found");
  std::string t;
  while (in >> t) {
    if (t[0] == '#') continue;
    ch_pos1.push_back((int) se.size() + 1);
    ch_len.push_back((int) t.size());
    se += t;
  }
  nch = (int) ch_len.size();
}

/* LAMMPS data file, atom_style awsemmd */
void System::read_data(const std::string &path)
{
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open data file " + path);
  std::string line;
  std::getline(in, line);
  int nbonds = 0, nbt = 0;
  std::vector<std::string> section;
  std::map<std::string, std::vector<std::string>> sections;
  std::string cur;
  while (std::getline(in, line)) {
    auto h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    auto v = words(line);
    if (v.empty()) continue;
    if (cur.empty()) {
      if (v.size() >= 2 && v[1] == "atoms") { natoms = atoi(v[0].c_str()); continue; }
      if (v.size() >= 2 && v[1] == "bonds") { nbonds = atoi(v[0].c_str()); continue; }
      if (v.size() >= 3 && v[1] == "atom" && v[2] == "types") { ntypes = atoi(v[0].c_str()); continue; }
      if (v.size() >= 3 && v[1] == "bond" && v[2] == "types") { nbt = atoi(v[0].c_str()); continue; }
      if (v.size() >= 3 && (v[2] == "types" || v[2] == "xlo" || v[2] == "ylo" || v[2] == "zlo")) continue;
      if (v.size() >= 2 && (v[1] == "angles" || v[1] == "dihedrals" || v[1] == "impropers")) continue;
    }
    if (v[0] == "Masses" || v[0] == "Atoms" || v[0] == "Velocities" || v[0] == "Bonds" ||
        (v[0] == "Bond" && v.size() > 1 && v[1] == "Coeffs")) {
      cur = v[0] == "Bond" ? "Bond Coeffs" : v[0];
      continue;
    }
    if (cur.empty()) throw std::runtime_error("data file: unexpected line " + line);
    sections[cur].push_back(line);
  }
  mass.assign(ntypes + 1, 0.0);
  for (auto &l : sections["Masses"]) {
    auto v = words(l);
    mass[atoi(v[0].c_str())] = atof(v[1].c_str());
  }
  std::vector<std::pair<int, std::vector<std::string>>> rows;
  for (auto &l : sections["Atoms"]) {
    auto v = words(l);
    rows.push_back({atoi(v[0].c_str()), v});
  }
  std::sort(rows.begin(), rows.end(), [](auto &a, auto &b) { return a.first < b.first; });
  if ((int) rows.size() != natoms) throw std::runtime_error("data file: atom count mismatch");
  atype.resize(natoms);
  amol.resize(natoms);
  ares.resize(natoms);
  tag.resize(natoms);
  std::map<int, int> t2i;
  for (int i = 0; i < natoms; i++) {
    auto &v = rows[i].second;
    tag[i] = atoi(v[0].c_str());
    amol[i] = atoi(v[1].c_str());
    ares[i] = atoi(v[2].c_str());
    atype[i] = atoi(v[3].c_str());
    t2i[tag[i]] = i;
  }
  bk.assign(nbt + 1, 0.0);
  br0.assign(nbt + 1, 0.0);
  for (auto &l : sections["Bond Coeffs"]) {
    auto v = words(l);
    bk[atoi(v[0].c_str())] = atof(v[1].c_str());
    br0[atoi(v[0].c_str())] = atof(v[2].c_str());
  }
  special.assign(natoms, {});
  for (auto &l : sections["Bonds"]) {
    auto v = words(l);
    int i = t2i.at(atoi(v[2].c_str())), j = t2i.at(atoi(v[3].c_str()));
    b_t.push_back(atoi(v[1].c_str()));
    b_i.push_back(i);
    b_j.push_back(j);
    special[i].push_back(j);
    special[j].push_back(i);
  }
  (void) nbonds;
}

/* a .gro structure read as Fragment_Memory's constructor does
   (fragment_memory.cpp:60-172): residues fpos+1..fpos+len, CA and CB
   coordinates (nm -> A), then the CA-CA / CB-CB and CA-CB distance tables */
void load_gro(const std::string &path, int fpos, Memory &m, const std::string &open_msg, const std::string &who)
{
  m.se.assign(m.len, '?');
  std::vector<double> xa((size_t) m.len * 3, 0.0), xb((size_t) m.len * 3, 0.0);
  FILE *fg = fopen(path.c_str(), "r");
  if (!fg) throw std::runtime_error(open_msg);
  char buf[256];
  if (!fgets(buf, sizeof buf, fg)) throw std::runtime_error("bad gro");
  int nat = 0;
  if (fscanf(fg, "%d", &nat) != 1) throw std::runtime_error("bad gro");
  int nca = 0;
  for (int a = 0; a < nat; a++) {
    int ires, iatom;
    char resty[16], atomty[16];
    double x, y, z;
    if (fscanf(fg, "%d %15s %15s %d %lf %lf %lf", &ires, resty, atomty, &iatom, &x, &y, &z) != 7) break;
    if (ires > fpos + m.len) break;
    if (ires > fpos && ires <= fpos + m.len) {
      int r = ires - fpos - 1;
      x *= 10;
      y *= 10;
      z *= 10;
      if (!strcmp(atomty, "CA")) {
        m.se[r] = three_to_one(resty);
        if (m.se[r] == '?') {
          fclose(fg);
          throw std::runtime_error(who + ": Unknown residue");
        }
        xa[3 * r] = x;
        xa[3 * r + 1] = y;
        xa[3 * r + 2] = z;
        nca++;
      } else if (!strcmp(atomty, "CB")) {
        xb[3 * r] = x;
        xb[3 * r + 1] = y;
        xb[3 * r + 2] = z;
      }
    }
  }
  fclose(fg);
  if (nca != m.len) throw std::runtime_error(who + ": Wrong atom count in memory structure file");
  m.rf0.assign((size_t) m.len * m.len, 0.0);
  m.rf1.assign((size_t) m.len * m.len, 0.0);
  for (int i = 0; i < m.len; i++)
    for (int j = 0; j < m.len; j++) {
      m.rf0[i * m.len + j] = i < j ? m.R(&xa[3 * i], &xa[3 * j]) : (i > j ? m.R(&xb[3 * i], &xb[3 * j]) : 0.0);
      m.rf1[i * m.len + j] = m.R(&xa[3 * i], &xb[3 * j]);
    }
  // Fragment_Memory::VM (fragment_memory.cpp:240-243)
  m.vmf.assign((size_t) m.len * m.len, 0.0);
  for (int i = 0; i < m.len; i++)
    for (int j = 0; j < m.len; j++) {
      const double *a = &xa[3 * i], *b = &xb[3 * i], *c = &xa[3 * j], *d = &xb[3 * j];
      m.vmf[i * m.len + j] = acos(((b[0] - a[0]) * (d[0] - c[0]) + (b[1] - a[1]) * (d[1] - c[1]) + (b[2] - a[2]) * (d[2] - c[2])) /
                                  (m.R(a, b) * m.R(c, d)));
    }
}

/* .mem list and .gro memories (fix_backbone.cpp:1966-2042,
   fragment_memory.cpp:34-176) and the residue -> memory map (:749-791) */
void System::read_mems()
{
  std::ifstream in(join(workdir, P.fm_file));
  if (!in) throw std::runtime_error("Fragment_Memory: Error opening mem file");
  std::string line;
  int state = 0;  // 0 none, 1 target, 2 memories
  while (std::getline(in, line)) {
    auto v = words(line);
    std::string t = v.empty() ? "" : v[0];
    if (!t.empty() && t[0] == '#') continue;
    if (!t.empty() && t[0] == '[') state = 0;
    if (v.empty()) {
      state = 0;
      continue;
    }
    if (state == 2) {
      if (v.size() != 5) throw std::runtime_error("Fragment_Memory: Error reading mem file");
      Memory m;
      m.pos = atoi(v[1].c_str()) - 1;
      int fpos = atoi(v[2].c_str()) - 1;
      m.len = atoi(v[3].c_str());
      m.weight = atof(v[4].c_str());
      load_gro(join(workdir, v[0]), fpos, m, "Fragment_Memory: Cannot read the file " + v[0], "Fragment_Memory");
      if (m.pos + m.len > n) throw std::runtime_error("Fragment_Memory: Incorrectly defined memory fragment");
      mems.push_back(m);
    } else if (state == 0) {
      if (t == "[Target]") state = 1;
      else if (t == "[Memories]") state = 2;
    }
  }
  G.load(join(workdir, P.fm_gamma_file));
  fm_map.assign(n, {});
  if (P.fm_tb && !P.fm && tb_files()) return;  // the tables come from files (fix_backbone.cpp:758)
  int min_sep = G.min_sep();
  for (int k = 0; k < (int) mems.size(); k++)
    for (int i = mems[k].pos; i < mems[k].pos + mems[k].len - min_sep; i++) fm_map[i].push_back(k);
}

bool System::tb_files() const
{
  return P.tb_use_file && std::ifstream(join(workdir, "fm_table.energy")).good() &&
         std::ifstream(join(workdir, "fm_table.force")).good();
}

/* the FM tables: read_fragment_memory_table (fix_backbone.cpp:4179-4236) or
   compute_fragment_memory_table (:4238-4322) */
void System::build_tb()
{
  const Params &p = P;
  if (!fm_map.size()) fm_map.assign(n, {});
  if (G.min_sep() == 0 && G.max_sep() == 0) G.load(join(workdir, p.fm_gamma_file));
  tb_nbrs = G.max_sep() != -1 ? G.max_sep() - G.min_sep() + 1 : n - G.min_sep();
  const size_t ntb = (size_t) 4 * n * tb_nbrs;
  tb_e.assign(ntb, {});
  tb_f.assign(ntb, {});
  if (tb_files()) {
    for (int pass = 0; pass < 2; pass++) {
      std::ifstream in(join(workdir, pass ? "fm_table.force" : "fm_table.energy"));
      size_t ir = 0, itb = 0;
      double val;
      while (in >> val) {
        if (ir != 0 && ir % p.tb_size == 0) {
          ir = 0;
          itb++;
        }
        if (itb >= ntb) throw std::runtime_error("Fragment memory table file format error!");
        std::vector<double> &t = pass ? tb_f[itb] : tb_e[itb];
        if (t.empty()) t.assign(p.tb_size, 0.0);
        if (pass && tb_e[itb].empty()) tb_e[itb].assign(p.tb_size, 0.0);
        t[ir++] = val;
      }
    }
    return;
  }
  static const int it[4] = {1, 1, 2, 2}, jt[4] = {1, 2, 1, 2};
  for (int i = 0; i < n; i++)
    for (int km : fm_map[i]) {
      const Memory &m = mems[km];
      double ekw = p.epsilon * p.k_fm * m.weight;
      int js = i + G.min_sep();
      int je = m.pos + m.len - 1;
      if (G.max_sep() != -1) je = std::min(je, i + G.max_sep());
      if (je >= n) throw std::runtime_error("Missing residues in memory potential");
      for (int j = js; j <= je; j++) {
        double sig_sq = pow(abs(i - j), 2 * p.fm_sigma_exp);
        sig_sq = sig_sq * p.tb_width * p.tb_width;
        double gam = G.get(type_of(i), type_of(j), aa_index(m.se[i - m.pos]), aa_index(m.se[j - m.pos]), i, j);
        double ekwg = ekw * gam;
        for (int k = 0; k < 4; k++) {
          if (it[k] == 2 && (se[i] == 'G' || m.se[i - m.pos] == 'G')) continue;
          if (jt[k] == 2 && (se[j] == 'G' || m.se[j - m.pos] == 'G')) continue;
          size_t itb = (size_t) 4 * tb_nbrs * i + 4 * (j - js) + k;
          if (tb_e[itb].empty()) {
            tb_e[itb].assign(p.tb_size, 0.0);
            tb_f[itb].assign(p.tb_size, 0.0);
          }
          double rf = m.rf(i, it[k], j, jt[k]);
          for (int ir = 0; ir < p.tb_size; ir++) {
            double r = p.tb_rmin + ir * p.tb_dr;
            double dr = r - rf;
            double drsq = dr * dr;
            double V = -ekwg * exp(-drsq / (2 * sig_sq));
            tb_e[itb][ir] += V;
            tb_f[itb][ir] += V * dr / (sig_sq * r);
          }
        }
      }
    }
}

/* pair_style vexcluded settings/coeff/init_one (pair_excluded_volume.cpp:175-265) */
void System::pair_setup(const std::string &style, const std::string &coeffs)
{
  auto v = words(style);
  ev_p = atoi(v[0].c_str());
  ev_cs_glob = atof(v[1].c_str());
  ev_cl_glob = atof(v[2].c_str());
  int N = ntypes + 1;
  ev_lambda.assign(N * N, 0.0);
  ev_cs.assign(N * N, 0.0);
  ev_cl.assign(N * N, 0.0);
  ev_set.assign(N * N, 0);
  std::stringstream ss(coeffs);
  std::string rec;
  auto range = [&](const std::string &t, int &lo, int &hi) {
    size_t s = t.find('*');
    if (s == std::string::npos) lo = hi = atoi(t.c_str());
    else {
      lo = s == 0 ? 1 : atoi(t.substr(0, s).c_str());
      hi = s == t.size() - 1 ? ntypes : atoi(t.substr(s + 1).c_str());
    }
  };
  while (std::getline(ss, rec, ';')) {
    auto c = words(rec);
    if (c.empty()) continue;
    int ilo, ihi, jlo, jhi;
    range(c[0], ilo, ihi);
    range(c[1], jlo, jhi);
    double lam = atof(c[2].c_str());
    double cs = c.size() == 5 ? atof(c[3].c_str()) : ev_cs_glob;
    double cl = c.size() == 5 ? atof(c[4].c_str()) : ev_cl_glob;
    for (int i = ilo; i <= ihi; i++)
      for (int j = std::max(jlo, i); j <= jhi; j++) {
        ev_lambda[i * N + j] = lam;
        ev_cs[i * N + j] = cs;
        ev_cl[i * N + j] = cl;
        ev_set[i * N + j] = 1;
      }
  }
  for (int i = 1; i <= ntypes; i++)
    for (int j = i; j <= ntypes; j++) {
      if (!ev_set[i * N + j]) {
        ev_lambda[i * N + j] = sqrt(ev_lambda[i * N + i] * ev_lambda[j * N + j]);
        ev_cs[i * N + j] = sqrt(ev_cs[i * N + i] * ev_cs[j * N + j]);
        ev_cl[i * N + j] = sqrt(ev_cl[i * N + i] * ev_cl[j * N + j]);
      }
      ev_lambda[j * N + i] = ev_lambda[i * N + j];
      ev_cs[j * N + i] = ev_cs[i * N + j];
      ev_cl[j * N + i] = ev_cl[i * N + j];
    }
}

/* residue bookkeeping from atom groups: CA type 1, CB/H-beta types 4/5,
   O type 3, residue order by residue id (Construct_Computational_Arrays,
   fix_backbone.cpp:1590-1698, for a serial system with every residue local) */
static void build_residues(System &S)
{
  S.n = (int) S.se.size();
  S.ca.assign(S.n, -1);
  S.cb.assign(S.n, -1);
  S.o.assign(S.n, -1);
  S.chain_of.assign(S.n, -1);
  for (int a = 0; a < S.natoms; a++) {
    int r = S.ares[a] - 1;
    if (r < 0 || r >= S.n) throw std::runtime_error("Residue tag is out of range");
    int t = S.atype[a];
    if (t == 1) S.ca[r] = a;
    else if (t == 4 || t == 5) S.cb[r] = a;
    else if (t == 3) S.o[r] = a;
    S.chain_of[r] = S.amol[a] - 1;
  }
  for (int r = 0; r < S.n; r++) {
    if (S.ca[r] < 0 || S.cb[r] < 0 || S.o[r] < 0) throw std::runtime_error("Missing neighbor atoms in fix backbone");
    int c = S.chain_of[r];
    if (c < 0 || c >= S.nch) throw std::runtime_error("Chain tag is out of range");
    if (r + 1 < S.ch_pos1[c] || r + 1 > S.ch_pos1[c] + S.ch_len[c] - 1)
      throw std::runtime_error("Residue tag is out of range");
  }
}

/* coordinates and virtual N, H, C' (fix_backbone.cpp:7067-7138) */
void System::backbone_atoms(const double *x)
{
  const Params &p = P;
  xca.assign(3 * n, 0.0);
  xcb.assign(3 * n, 0.0);
  xo.assign(3 * n, 0.0);
  xn.assign(3 * n, 0.0);
  xh.assign(3 * n, 0.0);
  xcp.assign(3 * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      xca[3 * i + k] = x[3 * ca[i] + k];
      xcb[3 * i + k] = x[3 * cb[i] + k];
      xo[3 * i + k] = x[3 * o[i] + k];
    }
  for (int i = 0; i < n; i++) {
    int im1 = i > 0 ? i - 1 : -1;
    if (im1 != -1 && !first(i)) {
      for (int k = 0; k < 3; k++) {
        xn[3 * i + k] = p.an * xca[3 * im1 + k] + p.bn * xca[3 * i + k] + p.cn * xo[3 * im1 + k];
        xh[3 * i + k] = p.ah * xca[3 * im1 + k] + p.bh * xca[3 * i + k] + p.ch * xo[3 * im1 + k];
        xcp[3 * im1 + k] = p.ap * xca[3 * im1 + k] + p.bp * xca[3 * i + k] + p.cp * xo[3 * im1 + k];
      }
    } else if (im1 != -1) {
      for (int k = 0; k < 3; k++) xcp[3 * im1 + k] = 0.0;
    }
  }
}

inline void addf(double *f, int atom, double a, double b, double c)
{
  f[3 * atom] += a;
  f[3 * atom + 1] += b;
  f[3 * atom + 2] += c;
}

/* compute_chain_potential, fix_backbone.cpp:2062-2170 */
void System::chain_term(int i, double *f)
{
  const Params &p = P;
  double dx[3], r, dr, force;
  if (!first(i) && se[i] != 'G') {
    int im1 = i - 1;
    for (int k = 0; k < 3; k++) dx[k] = xn[3 * i + k] - xcb[3 * i + k];
    r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    dr = r - p.r_ncb0;
    force = 2 * p.k_chain[0] * dr / r;
    E[ET_CHAIN] += p.k_chain[0] * dr * dr;
    for (int k = 0; k < 3; k++) {
      f[3 * ca[im1] + k] -= p.an * dx[k] * force;
      f[3 * o[im1] + k] -= p.cn * dx[k] * force;
      f[3 * ca[i] + k] -= p.bn * dx[k] * force;
      f[3 * cb[i] + k] -= -dx[k] * force;
    }
  }
  if (!last(i) && se[i] != 'G') {
    int ip1 = i + 1;
    for (int k = 0; k < 3; k++) dx[k] = xcp[3 * i + k] - xcb[3 * i + k];
    r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    dr = r - p.r_cpcb0;
    force = 2 * p.k_chain[1] * dr / r;
    E[ET_CHAIN] += p.k_chain[1] * dr * dr;
    for (int k = 0; k < 3; k++) {
      f[3 * ca[ip1] + k] -= p.bp * dx[k] * force;
      f[3 * ca[i] + k] -= p.ap * dx[k] * force;
      f[3 * o[i] + k] -= p.cp * dx[k] * force;
      f[3 * cb[i] + k] -= -dx[k] * force;
    }
  }
  if (!first(i) && !last(i)) {
    int im1 = i - 1, ip1 = i + 1;
    for (int k = 0; k < 3; k++) dx[k] = xn[3 * i + k] - xcp[3 * i + k];
    r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    dr = r - p.r_ncp0;
    force = 2 * p.k_chain[2] * dr / r;
    E[ET_CHAIN] += p.k_chain[2] * dr * dr;
    for (int k = 0; k < 3; k++) {
      f[3 * ca[im1] + k] -= p.an * dx[k] * force;
      f[3 * o[im1] + k] -= p.cn * dx[k] * force;
      f[3 * ca[ip1] + k] -= -p.bp * dx[k] * force;
      f[3 * ca[i] + k] -= (p.bn - p.ap) * dx[k] * force;
      f[3 * o[i] + k] -= -p.cp * dx[k] * force;
    }
  }
}

inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double *a, const double *b, double *c)
{
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* compute_chi_potential, fix_backbone.cpp:2239-2339 */
void System::chi_term(int i, double *f)
{
  const Params &p = P;
  double a[3], b[3], c[3], axb[3], cxa[3], bxc[3], aprl[3], bprl[3], cprl[3];
  for (int k = 0; k < 3; k++) {
    a[k] = xcp[3 * i + k] - xca[3 * i + k];
    b[k] = xca[3 * i + k] - xn[3 * i + k];
    c[k] = xca[3 * i + k] - xcb[3 * i + k];
  }
  double arvsq = 1.0 / dot3(a, a), brvsq = 1.0 / dot3(b, b), crvsq = 1.0 / dot3(c, c);
  double norm = sqrt(arvsq * brvsq * crvsq);
  cross3(a, b, axb);
  cross3(c, a, cxa);
  cross3(b, c, bxc);
  double chi = dot3(axb, c) * norm;
  for (int k = 0; k < 3; k++) {
    aprl[k] = norm * bxc[k] - arvsq * chi * a[k];
    bprl[k] = norm * cxa[k] - brvsq * chi * b[k];
    cprl[k] = norm * axb[k] - crvsq * chi * c[k];
  }
  double dchi = chi - p.chi0;
  double force = 2 * p.k_chi * dchi;
  E[ET_CHI] += p.k_chi * dchi * dchi;
  int im1 = i - 1, ip1 = i + 1;
  for (int k = 0; k < 3; k++) {
    f[3 * ca[im1] + k] -= -p.an * bprl[k] * force;
    f[3 * o[im1] + k] -= -p.cn * bprl[k] * force;
    f[3 * ca[ip1] + k] -= p.bp * aprl[k] * force;
    f[3 * ca[i] + k] -= (cprl[k] + (1 - p.bn) * bprl[k] + (p.ap - 1) * aprl[k]) * force;
    f[3 * o[i] + k] -= p.cp * aprl[k] * force;
    f[3 * cb[i] + k] -= -cprl[k] * force;
  }
}

/* calcDihedralAndSlopes, fix_backbone.cpp:2341-2453; atoms CA0, CA1, CA2, O0, O1 */
void System::dihedral_slopes(int i, int iang, double &angle, double ys[5][3], double xs[5][3])
{
  const Params &p = P;
  double a[3], b[3], c[3], bxa[3], cxa[3], cxb[3];
  for (int k = 0; k < 3; k++) {
    if (iang == 0) {
      a[k] = xcp[3 * i + k] - xca[3 * i + k];
      b[k] = xca[3 * i + k] - xn[3 * i + k];
      c[k] = xn[3 * i + k] - xcp[3 * (i - 1) + k];
    } else {
      a[k] = xn[3 * (i + 1) + k] - xcp[3 * i + k];
      b[k] = xcp[3 * i + k] - xca[3 * i + k];
      c[k] = xca[3 * i + k] - xn[3 * i + k];
    }
  }
  double adb = dot3(a, b), bdc = dot3(b, c), adc = dot3(a, c), b2 = dot3(b, b), bm = sqrt(b2);
  cross3(b, a, bxa);
  cross3(c, a, cxa);
  cross3(c, b, cxb);
  double cdbxa = dot3(c, bxa);
  double Y = bm * cdbxa, X = adb * bdc - b2 * adc;
  angle = atan2(Y, X);
  double X2Y2 = 1.0 / (X * X + Y * Y);
  double dy = X * X2Y2, dxx = -Y * X2Y2;
  b2 *= dxx;
  adb *= dxx;
  adc *= dxx;
  bdc *= dxx;
  cdbxa *= dy / bm;
  bm *= dy;
  const double an = p.an, bn = p.bn, cn = p.cn, ap = p.ap, bp = p.bp, cp = p.cp;
  for (int l = 0; l < 3; l++) {
    double h1, h2, h3, h4;
    if (iang == 0) {
      h1 = cxb[l] * bm;
      h2 = cxa[l] * bm;
      h3 = bxa[l] * bm;
      h4 = b[l] * cdbxa;
      ys[0][l] = -an * h4 + (an - ap) * h3 + an * h2;
      ys[1][l] = (1.0 - bn) * h4 + (bn - bp) * h3 + (ap - 1.0) * h1 - (1.0 - bn) * h2;
      ys[2][l] = bp * h1;
      ys[3][l] = -cn * h4 + (cn - cp) * h3 + cn * h2;
      ys[4][l] = cp * h1;
      h1 = b[l] * bdc - c[l] * b2;
      h2 = a[l] * bdc - 2.0 * b[l] * adc + c[l] * adb;
      h3 = b[l] * adb - a[l] * b2;
      xs[0][l] = -an * h2 + (an - ap) * h3;
      xs[1][l] = (ap - 1.0) * h1 + (1.0 - bn) * h2 + (bn - bp) * h3;
      xs[2][l] = bp * h1;
      xs[3][l] = -cn * h2 + (cn - cp) * h3;
      xs[4][l] = cp * h1;
    } else {
      h1 = bxa[l] * bm;
      h2 = cxb[l] * bm;
      h3 = cxa[l] * bm;
      h4 = b[l] * cdbxa;
      ys[0][l] = -an * h1;
      ys[1][l] = (ap - 1.0) * h4 + (1.0 - bn) * h1 + (an - ap) * h2 - (ap - 1) * h3;
      ys[2][l] = bp * h4 + (bn - bp) * h2 - bp * h3;
      ys[3][l] = -cn * h1;
      ys[4][l] = cp * h4 + (cn - cp) * h2 - cp * h3;
      h1 = b[l] * bdc - c[l] * b2;
      h2 = a[l] * bdc - 2.0 * b[l] * adc + c[l] * adb;
      h3 = b[l] * adb - a[l] * b2;
      xs[0][l] = -an * h3;
      xs[1][l] = (an - ap) * h1 + (ap - 1.0) * h2 + (1.0 - bn) * h3;
      xs[2][l] = (bn - bp) * h1 + bp * h2;
      xs[3][l] = -cn * h3;
      xs[4][l] = (cn - cp) * h1 + cp * h2;
    }
  }
}

/* compute_rama_potential + compute_rama_force, fix_backbone.cpp:2455-2546 */
void System::rama_term(int i, double *f)
{
  const Params &p = P;
  double phi, psi, ys[2][5][3], xs[2][5][3];
  dihedral_slopes(i, 0, phi, ys[0], xs[0]);
  dihedral_slopes(i, 1, psi, ys[1], xs[1]);
  int j0 = 0, j1 = p.n_rama;
  if (se[i] == 'P' && p.rama_p) {
    j0 = Params::i_rp;
    j1 = Params::i_rp + p.n_rama_p;
  }
  int atoms[5] = {ca[i - 1], ca[i], ca[i + 1], o[i - 1], o[i]};
  for (int j = j0; j < j1; j++) {
    if (p.ssweight[j] && aps[j][i] == 0.0) continue;
    double cos_phi = cos(phi + p.phi0[j]) - 1.0;
    double cos_psi = cos(psi + p.psi0[j]) - 1.0;
    double pc = p.phiw[j] * cos_phi, sc = p.psiw[j] * cos_psi;
    double V = p.w[j] * exp(-cos_phi * pc - cos_psi * sc);
    if (p.ssweight[j]) V *= aps[j][i];
    double force = 2.0 * V;
    double f1[2] = {force * pc * sin(phi + p.phi0[j]), force * sc * sin(psi + p.psi0[j])};
    E[ET_RAMA] += -V;
    for (int ia = 0; ia < 2; ia++)
      for (int at = 0; at < 5; at++)
        for (int l = 0; l < 3; l++) f[3 * atoms[at] + l] += f1[ia] * (ys[ia][at][l] + xs[ia][at][l]);
  }
}

/* compute_dssp_hdrgn(i, j), fix_backbone.cpp:2902-3277 (O of i, N-H of j) */
/* returns the gates passed: bit 0 r_NO <= cutoff (:2904), bit 1 both nu >= 1e-4 (:3052) */
int System::dssp_term(int i, int j, double *f)
{
  const Params &p = P;
  auto rNO = [&](int a, int b) {
    return sqrt(pow(xo[3 * a] - xn[3 * b], 2) + pow(xo[3 * a + 1] - xn[3 * b + 1], 2) +
                pow(xo[3 * a + 2] - xn[3 * b + 2], 2));
  };
  auto rHO = [&](int a, int b) {
    return sqrt(pow(xo[3 * a] - xh[3 * b], 2) + pow(xo[3 * a + 1] - xh[3 * b + 1], 2) +
                pow(xo[3 * a + 2] - xh[3 * b + 2], 2));
  };
  touch(TOUCH_RNO, 0, i, j);
  const double rno0 = rNO(i, j);
  if (near_thr(rno0, p.dssp_cut)) near(AWSEM_SEL_DSSP, 0, i, j);
  if (rno0 > p.dssp_cut) return 0;
  int ic = chain_of[i], jc = chain_of[j];
  int i_ch_start = ch_pos1[ic], j_ch_start = ch_pos1[jc];
  int i_ch_end = ch_pos1[ic] + ch_len[ic] - 1, j_ch_end = ch_pos1[jc] + ch_len[jc] - 1;
  bool i_rep = true, i_AP = true, i_P = true;
  if (last(j) || se[j + 1] == 'P') i_rep = false;
  if (first(i) || last(j) || se[i] == 'P') i_AP = false;
  if (i >= i_ch_end - 2 || last(j) || se[i + 2] == 'P') i_P = false;
  auto aHB = [&](char a, char b, int k) { return p.m_anti_HB[aa_index(a)][aa_index(b)][k]; };
  auto aNHB = [&](char a, char b, int k) { return p.m_anti_NHB[aa_index(a)][aa_index(b)][k]; };
  auto pHB = [&](char a, char b, int k) { return p.m_para_HB[aa_index(a)][aa_index(b)][k]; };
  auto p1 = [&](char a) { return p.m_para_one[aa_index(a)]; };
  auto a1 = [&](char a) { return p.m_anti_one[aa_index(a)]; };
  double ts_aHB[2], ts_aNHB[2], ts_pHB[2];
  for (int k = 0; k < 2; k++) {
    if (i_AP) {
      ts_aHB[k] = 0.5 * aHB(se[i], se[j], k);
      ts_aNHB[k] = 0.25 * (aNHB(se[i + 1], se[j - 1], k) + aNHB(se[i - 1], se[j + 1], k));
    } else
      ts_aHB[k] = ts_aNHB[k] = 0.0;
    ts_pHB[k] = i_P ? pHB(se[i + 1], se[j], k) : 0.0;
  }
  double lambda[4];
  int hb_class;
  if (ic == jc && abs(j - i) < 45) {
    if (abs(j - i) < 4) {
      lambda[0] = -p.hbscl[0][0];
      lambda[1] = -p.hbscl[0][1];
      lambda[2] = 0.0;
      lambda[3] = 0.0;
      hb_class = 1;
    } else if (abs(j - i) < 18) {
      if (p.n_rama > 0 && aps[p.n_rama - 1][i] == 1.0 && aps[p.n_rama - 1][j] == 1.0) {
        lambda[0] = -p.hbscl[1][0];
        lambda[1] = -p.hbscl[1][1];
        lambda[2] = -p.hbscl[1][2] - p.hbscl[1][3] * ts_aHB[0] - p.hbscl[1][4] * ts_aNHB[0] -
                    p.hbscl[1][5] * (a1(se[i]) + a1(se[j]));
        lambda[3] = -p.hbscl[1][6];
      } else {
        lambda[0] = 0.0;
        lambda[1] = -p.hbscl[1][1];
        lambda[2] = 0.0;
        lambda[3] = 0.0;
      }
      hb_class = 2;
    } else {
      lambda[0] = -p.hbscl[2][0];
      lambda[1] = -p.hbscl[2][1];
      lambda[2] = -p.hbscl[2][2] - p.hbscl[2][3] * ts_aHB[1] - p.hbscl[2][4] * ts_aNHB[1] -
                  p.hbscl[2][5] * (a1(se[i]) + a1(se[j]));
      lambda[3] = -p.hbscl[2][6] - p.hbscl[2][7] * ts_pHB[1] - p.hbscl[2][8] * (p1(se[i + 1]) + p1(se[j]));
      hb_class = 3;
    }
  } else {
    lambda[0] = -p.hbscl[3][0];
    lambda[1] = -p.hbscl[3][1];
    lambda[2] = -p.hbscl[3][2] - p.hbscl[3][3] * ts_aHB[1] - p.hbscl[3][4] * ts_aNHB[1] -
                p.hbscl[3][5] * (a1(se[i]) + a1(se[j]));
    lambda[3] = -p.hbscl[3][6] - p.hbscl[3][7] * ts_pHB[1] - p.hbscl[3][8] * (p1(se[i + 1]) + p1(se[j]));
    hb_class = 4;
  }
  double nu[2], prdnu[2], dxnu[2][3], r_nu;
  bool use_nu[2];
  use_nu[0] = i - 2 >= i_ch_start - 1 && i + 2 < i_ch_end && hb_class != 2;
  use_nu[1] = j - 2 >= j_ch_start - 1 && j + 2 < j_ch_end && hb_class != 2;
  int cen[2] = {i, j};
  for (int s = 0; s < 2; s++) {
    nu[s] = prdnu[s] = 0.0;
    if (use_nu[s]) {
      int c = cen[s];
      for (int k = 0; k < 3; k++) dxnu[s][k] = xca[3 * (c + 2) + k] - xca[3 * (c - 2) + k];
      r_nu = dxnu[s][0] * dxnu[s][0] + dxnu[s][1] * dxnu[s][1] + dxnu[s][2] * dxnu[s][2];
      if (r_nu > (s == 0 ? p.nu_cut1_sq : p.nu_cut2_sq)) {
        r_nu = sqrt(r_nu);
        double th = tanh(p.pref[s] * (r_nu - p.d_nu0));
        nu[s] = 0.5 * (1.0 + th);
        prdnu[s] = p.pref[s] * nu[s] * (1.0 - th) / r_nu;
      }
    } else
      nu[s] = 1.0;
  }
  if (nu[0] < 1e-4 || nu[1] < 1e-4) return 1;
  bool i_theta[4] = {true, i_rep, i_AP, i_P};
  // (acceptor O residue, donor N-H residue) of the four Gaussians
  int acc[4] = {i, i, j, j}, don[4] = {j, j + 1, i, i + 2};
  double R_NO[4], R_HO[4], xNO[4][3], xHO[4][3], theta[4], prd[4][2];
  for (int k = 0; k < 4; k++) {
    if (!i_theta[k]) {
      theta[k] = 0.0;
      prd[k][0] = prd[k][1] = 0.0;
      continue;
    }
    int a = acc[k], d = don[k];
    touch(TOUCH_RNO, 0, a, d);
    touch(TOUCH_RHO, 0, a, d);
    R_NO[k] = rNO(a, d);
    R_HO[k] = rHO(a, d);
    for (int l = 0; l < 3; l++) {
      xNO[k][l] = xo[3 * a + l] - xn[3 * d + l];
      xHO[k][l] = xo[3 * a + l] - xh[3 * d + l];
    }
    double dNO = (R_NO[k] - p.NO_zero) * p.sigma_NO_sqinv;
    double dHO = (R_HO[k] - p.HO_zero) * p.sigma_HO_sqinv;
    theta[k] = exp(-0.5 * ((R_NO[k] - p.NO_zero) * dNO + (R_HO[k] - p.HO_zero) * dHO));
    prd[k][0] = -dNO / R_NO[k];
    prd[k][1] = -dHO / R_HO[k];
  }
  double ff1 = p.k_dssp * theta[0];
  double V[4] = {lambda[0], lambda[1] * theta[1], lambda[2] * theta[2], lambda[3] * theta[3]};
  double theta_sum = ff1 * (V[0] + V[1] + V[2] + V[3]);
  ff1 *= nu[0] * nu[1];
  for (double &v : V) v *= ff1;
  double VT = V[0] + V[1] + V[2] + V[3];
  E[ET_DSSP] += VT;
  if (use_nu[0]) {
    double g = theta_sum * prdnu[0] * nu[1];
    for (int k = 0; k < 3; k++) {
      f[3 * ca[i - 2] + k] -= -g * dxnu[0][k];
      f[3 * ca[i + 2] + k] -= g * dxnu[0][k];
    }
  }
  if (use_nu[1]) {
    double g = theta_sum * nu[0] * prdnu[1];
    for (int k = 0; k < 3; k++) {
      f[3 * ca[j - 2] + k] -= -g * dxnu[1][k];
      f[3 * ca[j + 2] + k] -= g * dxnu[1][k];
    }
  }
  double scale[4] = {VT, V[1], V[2], V[3]};
  for (int k = 0; k < 4; k++) {
    if (!i_theta[k]) continue;
    double q0 = prd[k][0] * scale[k], q1 = prd[k][1] * scale[k];
    int a = acc[k], d = don[k];
    for (int l = 0; l < 3; l++) {
      f[3 * o[a] + l] -= q0 * xNO[k][l] + q1 * xHO[k][l];
      f[3 * ca[d - 1] + l] += p.an * q0 * xNO[k][l] + p.ah * q1 * xHO[k][l];
      f[3 * ca[d] + l] += p.bn * q0 * xNO[k][l] + p.bh * q1 * xHO[k][l];
      f[3 * o[d - 1] + l] += p.cn * q0 * xNO[k][l] + p.ch * q1 * xHO[k][l];
    }
  }
  return 3;
}

/* cP_AP::compute, smart_matrix_lib.h:178-203 */
void System::pap_nu(int i, int j, double &nu, double &prd)
{
  const Params &p = P;
  double dx0 = xca[3 * i] - xca[3 * j], dx1 = xca[3 * i + 1] - xca[3 * j + 1], dx2 = xca[3 * i + 2] - xca[3 * j + 2];
  double drsq = pow(dx0, 2) + pow(dx1, 2) + pow(dx2, 2);
  if (drsq > p.pap_drmax_sq) {
    nu = 0.0;
    prd = 0.0;
  } else if (drsq < p.pap_drmin_sq) {
    nu = 1.0;
    prd = 0.0;
  } else {
    double dr = sqrt(drsq);
    double th = tanh(p.pap_pref * (p.pap_cut - dr));
    nu = 0.5 * (1 + th);
    prd = 0.5 * p.pap_pref * (1 - pow(th, 2)) / dr;
  }
}

/* compute_P_AP_potential(i, j), i < j, fix_backbone.cpp:3279-3383; returns
   bit 0 nu(i, j) >= 1e-12 (:3281), bits 1-3 the classes antiparallel medium,
   antiparallel long, parallel (:3290-3295) */
int System::pap_term(int i, int j, double *f)
{
  const Params &p = P;
  double nu_ij, prd_ij;
  touch(TOUCH_NU, 0, i, j);
  pap_nu(i, j, nu_ij, prd_ij);
  if (nu_ij < 1e-12) return 0;
  int ic = chain_of[i], jc = chain_of[j], d = p.i_diff_pap;
  int i_ch_end = ch_pos1[ic] + ch_len[ic] - 1, j_ch_end = ch_pos1[jc] + ch_len[jc] - 1;
  bool ap_med = ic == jc && i < i_ch_end - (p.i_med_min + 2 * d) && j >= i + (p.i_med_min + 2 * d) &&
                j <= std::min(i + p.i_med_max + 2 * d, i_ch_end - 1);
  bool ap_long = (ic == jc && i < i_ch_end - (p.i_med_max + 2 * d + 1) && j >= i + (p.i_med_max + 2 * d + 1) &&
                  j < j_ch_end) ||
                 (ic != jc && i + d < n && j - d >= 0 && chain_of[i + d] == ic && chain_of[j - d] == jc);
  bool par = (ic == jc && i < i_ch_end - (p.i_med_max + 1 + d) && j >= i + (p.i_med_max + 1) && j < i_ch_end - d) ||
             (ic != jc && i + d < n && j + d < n && chain_of[i + d] == ic && chain_of[j + d] == jc);
  bool beta = p.n_rama > 0 && aps[p.n_rama - 1][i] == 1.0 && aps[p.n_rama - 1][j] == 1.0;
  auto apply = [&](double K, int i2, int j2) {
    double nu2, prd2;
    touch(TOUCH_NU, 0, i2, j2);
    pap_nu(i2, j2, nu2, prd2);
    E[ET_PAP] += -p.k_global_pap * K * nu_ij * nu2;
    double f0 = p.k_global_pap * K * prd_ij * nu2;
    double f1 = p.k_global_pap * K * nu_ij * prd2;
    for (int k = 0; k < 3; k++) {
      double d0 = xca[3 * i + k] - xca[3 * j + k];
      double d1 = xca[3 * i2 + k] - xca[3 * j2 + k];
      f[3 * ca[i] + k] -= f0 * d0;
      f[3 * ca[j] + k] -= -f0 * d0;
      f[3 * ca[i2] + k] -= f1 * d1;
      f[3 * ca[j2] + k] -= -f1 * d1;
    }
  };
  if (ap_med || ap_long) {
    double K = beta ? (ap_med ? p.k_pap[0] : 0.0) + (ap_long ? p.k_pap[1] * p.k_betapred_pap : 0.0)
                    : (ap_med ? p.k_pap[0] : 0.0) + (ap_long ? p.k_pap[1] : 0.0);
    apply(K, i + d, j - d);
  }
  if (par) {
    double K = beta ? p.k_pap[2] * p.k_betapred_pap : p.k_pap[2];
    apply(K, i + d, j + d);
  }
  return 1 | (ap_med ? 2 : 0) | (ap_long ? 4 : 0) | (par ? 8 : 0);
}

/* compute_helix_dtheta_pair(i, j = i + 4), fix_backbone.cpp:3706-3785;
   returns 1 when |O_i - N_j| <= cutoff (:3708) */
int System::helix_pair(int i, int j, double *f)
{
  const Params &p = P;
  double xNO[3], xHO[3];
  for (int k = 0; k < 3; k++) {
    xNO[k] = xo[3 * i + k] - xn[3 * j + k];
    xHO[k] = xo[3 * i + k] - xh[3 * j + k];
  }
  double R_NO = sqrt(pow(xNO[0], 2) + pow(xNO[1], 2) + pow(xNO[2], 2));
  touch(TOUCH_RNO, 0, i, j);
  if (near_thr(R_NO, p.helix_cutoff)) near(AWSEM_SEL_HELIX_PAIR, 0, i, j);
  if (R_NO > p.helix_cutoff) return 0;
  if (chain_of[i] != chain_of[j]) return 1;
  touch(TOUCH_RHO, 0, i, j);
  double R_HO = sqrt(pow(xHO[0], 2) + pow(xHO[1], 2) + pow(xHO[2], 2));
  double h4i = p.h4prob[type_of(i)];
  if (se[i] == 'P' && p.pro_acc_flag) h4i = p.h4prob_pro;
  double prob_sum = h4i + p.h4prob[type_of(j)];
  double dNO = R_NO - p.helix_NO_zero, dHO = R_HO - p.helix_HO_zero;
  double dNOs = dNO * p.helix_sigma_NO_sqinv, dHOs = dHO * p.helix_sigma_HO_sqinv;
  double pair_theta = -p.k_helix * prob_sum * exp(-0.5 * (dNO * dNOs + dHO * dHOs));
  double prd0 = -dNOs / R_NO, prd1 = -dHOs / R_HO;
  double sigma_gamma = p.helix_gamma_p + (p.helix_gamma_w - p.helix_gamma_p) * sig_h[i] * sig_h[j];
  xi1[i] = (p.helix_gamma_w - p.helix_gamma_p) * pair_theta * sigp_h[i] * sig_h[j];
  xi2[i] = (p.helix_gamma_w - p.helix_gamma_p) * pair_theta * sig_h[i] * sigp_h[j];
  double V = sigma_gamma * pair_theta;
  E[ET_HELIX] += V;
  for (int k = 0; k < 3; k++) {
    f[3 * ca[j - 1] + k] -= -V * (p.an * prd0 * xNO[k] + p.ah * prd1 * xHO[k]);
    f[3 * ca[j] + k] -= -V * (p.bn * prd0 * xNO[k] + p.bh * prd1 * xHO[k]);
    f[3 * o[j - 1] + k] -= -V * (p.cn * prd0 * xNO[k] + p.ch * prd1 * xHO[k]);
    f[3 * o[i] + k] -= V * (prd0 * xNO[k] + prd1 * xHO[k]);
  }
  return 1;
}

/* compute_fragment_memory_potential(i), fix_backbone.cpp:4079-4177 */
void System::fm_term(int i, double *f)
{
  const Params &p = P;
  static const int it[4] = {1, 1, 2, 2}, jt[4] = {1, 2, 1, 2};
  for (int km : fm_map[i]) {
    const Memory &m = mems[km];
    double ekw = p.epsilon * p.k_fm * m.weight;
    int js = i + G.min_sep();
    int je = m.pos + m.len - 1;
    if (G.max_sep() != -1) je = std::min(je, i + G.max_sep());
    if (je >= n) throw std::runtime_error("Missing residues in memory potential");
    for (int j = js; j <= je; j++) {
      if (chain_of[i] != chain_of[j])
        throw std::runtime_error("Fragment Memory: Interaction between residues of different chains");
      double sig_sq = pow(abs(i - j), 2 * p.fm_sigma_exp);
      double gam = G.get(type_of(i), type_of(j), aa_index(m.se[i - m.pos]), aa_index(m.se[j - m.pos]), i, j);
      double ekwg = ekw * gam;
      int ia[4] = {ca[i], ca[i], cb[i], cb[i]}, ja[4] = {ca[j], cb[j], ca[j], cb[j]};
      const double *xi[4] = {&xca[3 * i], &xca[3 * i], &xcb[3 * i], &xcb[3 * i]};
      const double *xj[4] = {&xca[3 * j], &xcb[3 * j], &xca[3 * j], &xcb[3 * j]};
      for (int k = 0; k < 4; k++) {
        if (it[k] == 2 && (se[i] == 'G' || m.se[i - m.pos] == 'G')) continue;
        if (jt[k] == 2 && (se[j] == 'G' || m.se[j - m.pos] == 'G')) continue;
        double dx[3] = {xi[k][0] - xj[k][0], xi[k][1] - xj[k][1], xi[k][2] - xj[k][2]};
        double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
        double dr = r - m.rf(i, it[k], j, jt[k]);
        double V = -ekwg * exp(-dr * dr / (2.0 * sig_sq));
        E[ET_FRAGMEM] += V;
        double force = V * dr / (sig_sq * r);
        addf(f, ia[k], force * dx[0], force * dx[1], force * dx[2]);
        addf(f, ja[k], -force * dx[0], -force * dx[1], -force * dx[2]);
      }
    }
  }
}

/* table_fragment_memory(i, j) for j = i + min_sep .. min(i + max_sep, the
   chain's last residue) (fix_backbone.cpp:4325-4429, :7513-7527) */
void System::tb_term(int i, double *f)
{
  const Params &p = P;
  int jr0 = i + G.min_sep();
  int jrn = ch_pos1[chain_of[i]] + ch_len[chain_of[i]] - 2;
  if (G.max_sep() != -1) jrn = std::min(i + G.max_sep(), jrn);
  static const int it[4] = {1, 1, 2, 2}, jt[4] = {1, 2, 1, 2};
  for (int j = jr0; j <= jrn; j++) {
    int tb_j = j - i - G.min_sep();
    size_t itb0 = (size_t) 4 * tb_nbrs * i + 4 * tb_j;
    if (tb_e[itb0].empty()) continue;
    int ia[4] = {ca[i], ca[i], cb[i], cb[i]}, ja[4] = {ca[j], cb[j], ca[j], cb[j]};
    const double *xi[4] = {&xca[3 * i], &xca[3 * i], &xcb[3 * i], &xcb[3 * i]};
    const double *xj[4] = {&xca[3 * j], &xcb[3 * j], &xca[3 * j], &xcb[3 * j]};
    for (int k = 0; k < 4; k++) {
      if (se[i] == 'G' && it[k] == 2) continue;
      if (se[j] == 'G' && jt[k] == 2) continue;
      double dx[3] = {xi[k][0] - xj[k][0], xi[k][1] - xj[k][1], xi[k][2] - xj[k][2]};
      double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      if (!(r >= p.tb_rmin && r <= p.tb_rmax)) throw std::runtime_error("Table Fragment Memory: r is out of computed range.");
      int ir = int((r - p.tb_rmin) / p.tb_dr);
      size_t itb = itb0 + k;
      if (tb_e[itb].empty()) break;
      if (ir < 0 || ir >= p.tb_size) throw std::runtime_error("Table Fragment Memory: ir is out of range.");
      double r1 = p.tb_rmin + (double) ir * p.tb_dr, r2 = p.tb_rmin + (double) (ir + 1) * p.tb_dr;
      double v1 = tb_e[itb][ir], v2 = tb_e[itb][ir + 1];
      double V = ((v2 - v1) * r + v1 * r2 - v2 * r1) / (r2 - r1);
      double f1 = tb_f[itb][ir], f2 = tb_f[itb][ir + 1];
      double ff = ((f2 - f1) * r + f1 * r2 - f2 * r1) / (r2 - r1);
      E[ET_FRAGMEM] += V;
      addf(f, ia[k], ff * dx[0], ff * dx[1], ff * dx[2]);
      addf(f, ja[k], -ff * dx[0], -ff * dx[1], -ff * dx[2]);
    }
  }
}

/* theta of a density well and its radial derivative over r
   (cWell::compute_theta_pair, smart_matrix_lib.h:612-628) */
inline void well_theta(double r, double rmin_th, double rmax_th, double kappa, double rmin, double rmax,
                       double &theta, double &prd)
{
  if (r < rmin_th || r > rmax_th) {
    theta = prd = 0.0;
    return;
  }
  double t_min = tanh(kappa * (r - rmin));
  double t_max = tanh(kappa * (rmax - r));
  theta = 0.25 * (1.0 + t_min) * (1.0 + t_max);
  prd = kappa * theta * (t_max - t_min) / r;
}

/* compute_pair, fix_backbone.cpp:7677-8135: densities (DL1), switching
   functions, burial and helix pairs (SL), water xi (DL2), main loop (DL3) */
void System::pair_terms(const double *x, double *f)
{
  const Params &p = P;
  rho_w.assign(n, 0.0);
  rho_h.assign(n, 0.0);
  sig_w.assign(n, 0.0);
  sigp_w.assign(n, 0.0);
  sig_h.assign(n, 0.0);
  sigp_h.assign(n, 0.0);
  xi_w.assign(n, 0.0);
  xi1.assign(n, 0.0);
  xi2.assign(n, 0.0);
  bur.assign(n, 0.0);
  auto in_win = [&](double rsq, double lo, double hi, int kind, int aux, int i, int j) {
    if (near_thr(rsq, lo) || near_thr(rsq, hi)) near(kind, aux, i, j);
    return rsq > lo && rsq < hi;
  };
  auto cpos = [&](int i) { return &x[3 * contact_atom(i)]; };
  // DL1
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++) {
      if (!(chain_of[i] != chain_of[j] || abs(i - j) > 1)) continue;
      const double *a = cpos(i), *b = cpos(j);
      double dx0 = a[0] - b[0], dx1 = a[1] - b[1], dx2 = a[2] - b[2];
      double rsq = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
      if (p.water && in_win(rsq, p.w_rmin_sq[0], p.w_rmax_sq[0], AWSEM_SEL_DENS_WATER, 0, i, j)) {
        double th, pr;
        well_theta(sqrt(rsq), p.w_rmin_th[0], p.w_rmax_th[0], p.water_kappa, p.well_rmin[0], p.well_rmax[0], th, pr);
        rho_w[i] += th;
        rho_w[j] += th;
        sel(AWSEM_SEL_DENS_WATER, 0, i, j);
        touch(TOUCH_WELL, 0, i, j);
      }
      if (p.helix && in_win(rsq, p.h_rmin_sq, p.h_rmax_sq, AWSEM_SEL_DENS_HELIX, 0, i, j)) {
        double th, pr;
        well_theta(sqrt(rsq), p.h_rmin_th, p.h_rmax_th, p.helix_kappa, p.helix_rmin, p.helix_rmax, th, pr);
        rho_h[i] += th;
        rho_h[j] += th;
        sel(AWSEM_SEL_DENS_HELIX, 0, i, j);
        touch(TOUCH_HWELL, 0, i, j);
      }
    }
  // SL: switching functions and burial (:7795-7841)
  for (int i = 0; i < n; i++) {
    if (p.water) {
      double th = tanh(p.water_kappa_sigma * (rho_w[i] - p.treshold));
      sig_w[i] = 0.5 * (1.0 - th);
      sigp_w[i] = -p.water_kappa_sigma * sig_w[i] * (1.0 + th);
    }
    if (p.helix) {
      double th = tanh(p.helix_kappa_sigma * (rho_h[i] - p.helix_treshold));
      sig_h[i] = 0.5 * (1.0 - th);
      sigp_h[i] = -p.helix_kappa_sigma * sig_h[i] * (1.0 + th);
    }
    if (p.burial) {
      double t[3][2];
      for (int k = 0; k < 3; k++) {
        t[k][0] = tanh(p.burial_kappa * (rho_w[i] - p.burial_ro_min[k]));
        t[k][1] = tanh(p.burial_kappa * (p.burial_ro_max[k] - rho_w[i]));
      }
      // get_burial_gamma (fix_backbone.cpp:2887-2899): glutamate's gammas for a phosphorylated residue
      int ty = (p.phosph && phosph_map[i]) ? 6 : type_of(i);
      for (int k = 0; k < 3; k++) E[ET_BURIAL] += -0.5 * p.k_burial * p.burial_gamma[ty][k] * (t[k][0] + t[k][1]);
      bur[i] = p.burial_gamma[ty][0] * (t[0][1] * t[0][1] - t[0][0] * t[0][0]);
      bur[i] += p.burial_gamma[ty][1] * (t[1][1] * t[1][1] - t[1][0] * t[1][0]);
      bur[i] += p.burial_gamma[ty][2] * (t[2][1] * t[2][1] - t[2][0] * t[2][0]);
      bur[i] *= 0.5 * p.k_burial * p.burial_kappa;
    }
  }
  // SL: helical (i, i+4) pairs (:7843-7868)
  if (p.helix) {
    int d = p.helix_i_diff;
    for (int i = 0; i < n; i++) {
      int j = i + d;
      if (j >= n || chain_of[j] != chain_of[i]) continue;
      double dx0 = xo[3 * i] - xn[3 * j], dx1 = xo[3 * i + 1] - xn[3 * j + 1], dx2 = xo[3 * i + 2] - xn[3 * j + 2];
      const double r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
      if (near_thr(r2, p.helix_cutoff_sq)) near(AWSEM_SEL_HELIX_PAIR, 0, i, j);
      if (r2 < p.helix_cutoff_sq) sel(AWSEM_SEL_HELIX_PAIR, helix_pair(i, j, f), i, j);
    }
  }
  // DL2: water xi (:7877-7954)
  if (p.water) {
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) {
        if (!(chain_of[i] != chain_of[j] || abs(i - j) >= p.contact_cutoff)) continue;
        const double *a = cpos(i), *b = cpos(j);
        double dx0 = a[0] - b[0], dx1 = a[1] - b[1], dx2 = a[2] - b[2];
        double rsq = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
        int ti = type_of(i), tj = type_of(j);
        for (int w = 0; w < p.n_wells; w++) {
          if (!p.well_flag[w]) continue;
          double g0 = water_gamma(i, j, w, ti, tj, 0), g1 = water_gamma(i, j, w, ti, tj, 1);
          // `!fabs(g0 - g1) < delta` in the reference is true exactly when g0 != g1
          if (g0 != g1 && in_win(rsq, p.w_rmin_sq[w], p.w_rmax_sq[w], AWSEM_SEL_XI_WATER, w, i, j)) {
            sel(AWSEM_SEL_XI_WATER, w, i, j);
            touch(TOUCH_WELL, w, i, j);
            double th, pr;
            well_theta(sqrt(rsq), p.w_rmin_th[w], p.w_rmax_th[w], p.water_kappa, p.well_rmin[w], p.well_rmax[w], th, pr);
            double tg = (g1 - g0) * th;
            xi_w[i] += tg * sig_w[j];
            xi_w[j] += tg * sig_w[i];
          }
        }
      }
    for (int i = 0; i < n; i++) xi_w[i] *= sigp_w[i];
  }
  // DL3: water, burial, helix-density radial forces (:7958-8057, 8116-8128)
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++) {
      if (!(chain_of[i] != chain_of[j] || abs(i - j) > 1)) continue;
      int ai = contact_atom(i), aj = contact_atom(j);
      const double *a = &x[3 * ai], *b = &x[3 * aj];
      double dx[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
      double rsq = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
      double force = 0.0;
      bool other = chain_of[i] != chain_of[j];
      double r = sqrt(rsq);
      if (p.water) {
        int ti = type_of(i), tj = type_of(j);
        for (int w = 0; w < p.n_wells; w++) {
          if (!p.well_flag[w]) continue;
          if ((other || abs(j - i) >= p.contact_cutoff) &&
              in_win(rsq, p.w_rmin_sq[w], p.w_rmax_sq[w], AWSEM_SEL_WATER, w, i, j)) {
            sel(AWSEM_SEL_WATER, w, i, j);
            touch(TOUCH_WELL, w, i, j);
            double g0 = water_gamma(i, j, w, ti, tj, 0), g1 = water_gamma(i, j, w, ti, tj, 1);
            double sg = fabs(g0 - g1) < 1e-5 ? 0.5 * (g0 + g1) : g0 + (g1 - g0) * sig_w[i] * sig_w[j];
            double th, pr;
            well_theta(r, p.w_rmin_th[w], p.w_rmax_th[w], p.water_kappa, p.well_rmin[w], p.well_rmax[w], th, pr);
            E[ET_WATER] += -sg * th;
            force += sg * pr;
          }
        }
        if (in_win(rsq, p.w_rmin_sq[0], p.w_rmax_sq[0], AWSEM_SEL_XI_FORCE, 0, i, j)) {
          double th, pr;
          well_theta(r, p.w_rmin_th[0], p.w_rmax_th[0], p.water_kappa, p.well_rmin[0], p.well_rmax[0], th, pr);
          const int on = (fabs(xi_w[i]) > 1e-8 ? 1 : 0) | (fabs(xi_w[j]) > 1e-8 ? 2 : 0);
          if (on & 1) force += pr * xi_w[i];
          if (on & 2) force += pr * xi_w[j];
          if (on) {
            sel(AWSEM_SEL_XI_FORCE, on, i, j);
            touch(TOUCH_WELL, 0, i, j);
          }
        }
      }
      if (p.burial && rsq > p.w_rmin_sq[0] && rsq < p.w_rmax_sq[0]) {
        touch(TOUCH_WELL, 0, i, j);
        double th, pr;
        well_theta(r, p.w_rmin_th[0], p.w_rmax_th[0], p.water_kappa, p.well_rmin[0], p.well_rmax[0], th, pr);
        force += (bur[i] + bur[j]) * pr;
      }
      if (p.helix && in_win(rsq, p.h_rmin_sq, p.h_rmax_sq, AWSEM_SEL_HELIX_FORCE, 0, i, j)) {
        int d = p.helix_i_diff;
        double fac = xi1[i] + xi1[j];
        if (i - d >= 0) fac += xi2[i - d];
        if (j - d >= 0) fac += xi2[j - d];
        if (fabs(fac) > 1e-6) {
          sel(AWSEM_SEL_HELIX_FORCE, 0, i, j);
          touch(TOUCH_HWELL, 0, i, j);
          double th, pr;
          well_theta(r, p.h_rmin_th, p.h_rmax_th, p.helix_kappa, p.helix_rmin, p.helix_rmax, th, pr);
          force += -fac * pr;
        }
      }
      if (force != 0.0) {
        addf(f, ai, force * dx[0], force * dx[1], force * dx[2]);
        addf(f, aj, -force * dx[0], -force * dx[1], -force * dx[2]);
      }
    }
  // DL3: DSSP, (O_i, N_j) for ordered residue pairs (:8064-8094)
  if (p.dssp)
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        if (i == j) continue;
        if (!(chain_of[i] != chain_of[j] || abs(j - i) > 2)) continue;
        if (se[j] == 'P' || last(i) || first(j)) continue;
        if (j == 0) continue;
        double dx0 = xo[3 * i] - xn[3 * j], dx1 = xo[3 * i + 1] - xn[3 * j + 1], dx2 = xo[3 * i + 2] - xn[3 * j + 2];
        const double r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
        if (near_thr(r2, p.dssp_cut_sq)) near(AWSEM_SEL_DSSP, 0, i, j);
        if (r2 < p.dssp_cut_sq) sel(AWSEM_SEL_DSSP, dssp_term(i, j, f), i, j);
      }
  // DL3: P_AP on CA pairs (:8096-8103)
  // the selection records list the CA pairs separated enough for some P_AP
  // class (other chains, or at least the smallest class separation)
  const int pap_sep = std::min(p.i_med_min + 2 * p.i_diff_pap, p.i_med_max + 1);
  if (p.pap)
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) {
        const double *a = &x[3 * ca[i]], *b = &x[3 * ca[j]];
        double dx0 = a[0] - b[0], dx1 = a[1] - b[1], dx2 = a[2] - b[2];
        const double rsq = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
        const bool listed = chain_of[i] != chain_of[j] || j - i >= pap_sep;
        if (listed && near_thr(rsq, p.pap_cutoff_sq)) near(AWSEM_SEL_PAP, 0, i, j);
        // 1-2 bonded CA pairs are not in LAMMPS's list (special_bonds fene):
        // the reference never evaluates them (no P_AP class holds them anyway)
        if (rsq < p.pap_cutoff_sq && !bonded(ca[i], ca[j])) {
          const int g = pap_term(i, j, f);
          if (listed) sel(AWSEM_SEL_PAP, g, i, j);
        }
      }
}

/* PairExcludedVolume::compute, pair_excluded_volume.cpp:50-138, over all
   atom pairs except 1-2 bonded ones (special_bonds fene) */
void System::excluded_volume(const double *x, double *f)
{
  // a bead pair as (residue, bead) with the lower residue (then bead) first
  auto ev_sel = [&](int a, int b, bool near_only) {
    auto bead = [&](int at) {
      const int r = ares[at] - 1;
      return at == ca[r] ? 0 : at == cb[r] ? 1 : at == o[r] ? 2 : -1;
    };
    int ri = ares[a] - 1, rj = ares[b] - 1, bi = bead(a), bj = bead(b);
    if (bi < 0 || bj < 0) return;
    if (ri > rj || (ri == rj && bi > bj)) {
      std::swap(ri, rj);
      std::swap(bi, bj);
    }
    if (near_only) near(AWSEM_SEL_EV, 3 * bi + bj, ri, rj);
    else sel(AWSEM_SEL_EV, 3 * bi + bj, ri, rj);
  };
  int N = ntypes + 1;
  int sign = ev_p % 2 == 0 ? 1 : -1;
  e_pair = 0.0;
  for (int i = 0; i < natoms; i++)
    for (int j = i + 1; j < natoms; j++) {
      int ti = atype[i], tj = atype[j];
      double rc = (abs(ares[i] - ares[j]) < 5 && amol[i] == amol[j]) ? ev_cs[ti * N + tj] : ev_cl[ti * N + tj];
      double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
      double rsq = dx * dx + dy * dy + dz * dz;
      double r = sqrt(rsq);
      const bool counted = sel_on && ev_lambda[ti * N + tj] != 0.0;
      if (counted && near_thr(r, rc)) ev_sel(i, j, true);
      if (!(r < rc)) continue;
      bool excl = false;
      for (int s : special[i])
        if (s == j) excl = true;
      if (excl) continue;
      if (counted) ev_sel(i, j, false);
      double dr = r - rc;
      double pref = ev_lambda[ti * N + tj] * sign * pow(dr, ev_p - 1);
      double fpair = r > 0.0 ? -pref * ev_p / r : 0.0;
      addf(f, i, dx * fpair, dy * fpair, dz * fpair);
      addf(f, j, -dx * fpair, -dy * fpair, -dz * fpair);
      e_pair += pref * dr;
    }
}

/* bond_style harmonic (LAMMPS documentation: E = K (r - r0)^2) */
void System::bonds(const double *x, double *f)
{
  e_bond = 0.0;
  for (size_t b = 0; b < b_t.size(); b++) {
    int i = b_i[b], j = b_j[b];
    double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double dr = r - br0[b_t[b]];
    double rk = bk[b_t[b]] * dr;
    double fb = r > 0.0 ? -2.0 * rk / r : 0.0;
    e_bond += rk * dr;
    addf(f, i, dx * fb, dy * fb, dz * fb);
    addf(f, j, -dx * fb, -dy * fb, -dz * fb);
  }
}

/* The fix's pair-list cutoff, fix_backbone.cpp:1048-1066: 8 A, or the
   DSSP / P_AP cutoffs, the outer theta radii of the water and helix wells
   and, with [Helix], calc_exp_helix_cutoff (:1074-1103), if larger. */
double pair_list_cut(const Params &p)
{
  double cut = 8.0;
  if (p.dssp) cut = std::max(cut, p.dssp_cut);
  if (p.pap) cut = std::max(cut, sqrt(p.pap_cutoff_sq));
  if (p.water)
    for (int k = 0; k < p.n_wells; k++) cut = std::max(cut, p.w_rmax_th[k]);
  if (p.helix) {
    cut = std::max(cut, p.h_rmax_th);
    // O(i) to virtual N(j) / H(j): the farthest of the atoms they are built from
    const double r0[3] = {3.77, 2.5, 2.41};
    auto reach = [&](double a, double b, double c) {
      double r[3];
      r[0] = sqrt(pow(a * r0[0], 2) + pow(c * r0[1], 2) + a * c * (r0[0] * r0[0] + r0[1] * r0[1] - r0[2] * r0[2]));
      r[1] = sqrt(pow(a * r0[2], 2) + pow(b * r0[1], 2) + a * b * (r0[2] * r0[2] + r0[1] * r0[1] - r0[0] * r0[0]));
      r[2] = sqrt(pow(b * r0[0], 2) + pow(c * r0[2], 2) + b * c * (r0[0] * r0[0] + r0[2] * r0[2] - r0[1] * r0[1]));
      return std::max(r[0], std::max(r[1], r[2]));
    };
    double r1 = 1.1 * reach(p.an, p.bn, p.cn) + p.helix_NO_zero + p.helix_sigma_NO * sqrt(6.0 * log(10.0));
    double r2 = 1.1 * reach(p.ah, p.bh, p.ch) + p.helix_HO_zero + p.helix_sigma_HO * sqrt(6.0 * log(10.0));
    cut = std::max(cut, std::max(r1, r2));
    cut = std::max(cut, p.helix_cutoff);
  }
  if (p.cont_rest) cut = std::max(cut, sqrt(p.cr_glob_cutoff_sq));
  if (p.huckel) cut = std::max(cut, 2.0 * p.screening_length / p.k_screening);
  if (p.ssb) {
    double c = 0.0;
    if (p.ssb_rad_cor)
      for (int i = 0; i < 20; ++i) c = std::max(c, 2.0 * p.ssb_rshift[i]);
    c += std::max(p.ssb_rmax1, p.ssb_rmax2) + 10.0 / p.ssb_kappa;
    cut = std::max(cut, c);
  }
  return cut;
}

/* [AMH-Go] inputs (fix_backbone.cpp:695-742): amh-go.gamma, the native
   structure amh-go.gro as Fragment_Memory(0, 0, n, 1.0, ...), the censored
   residue pairs of frustration_censored_contacts.dat (flag 1), the fix's
   pair-list cutoff, and the normalisation. */
void System::read_amh_go()
{
  go_gamma.load(join(workdir, "amh-go.gamma"));
  if (go_gamma.frag_resty) throw std::runtime_error("AMH-Go: Wrong call of getGamma() function");
  go_mem.pos = 0;
  go_mem.len = n;
  go_mem.weight = 1.0;
  load_gro(join(workdir, "amh-go.gro"), 0, go_mem, "Cannot read file amh-go.gro", "AMH_Go");
  go_censored.assign((size_t) n * n, 0);
  if (P.censoring == 1) {
    std::ifstream cf(join(workdir, "frustration_censored_contacts.dat"));
    int a, b;
    while (cf >> a >> b)
      if (a >= 1 && a <= n && b >= 1 && b <= n) go_censored[(size_t) (a - 1) * n + (b - 1)] = 1;
  }
  amhgo_normalization();
}

/* compute_amhgo_normalization, fix_backbone.cpp:3787-3854:
   a = (1 / 8N) sum over CA / CB atoms i of |sum over native contacts of gamma|^p,
   the power taken of the running sum after each partner chain (the
   reference's loop nesting), N the last chain's last residue number. */
void System::amhgo_normalization()
{
  const Params &p = P;
  go_norm = 0.0;
  int iresn = 0;
  for (int ich = 0; ich < nch; ++ich) {
    const int ires0 = ch_pos1[ich] - 1;
    iresn = ch_pos1[ich] + ch_len[ich] - 1;
    for (int i = ires0; i < iresn; ++i) {
      const int it = aa_index(se[i]);
      for (int iatom = 1; iatom <= 2 - (se[i] == 'G' ? 1 : 0); ++iatom) {
        double normi = 0.0;
        for (int jch = 0; jch < nch; ++jch) {
          const int jres0 = ch_pos1[jch] - 1, jresn = ch_pos1[jch] + ch_len[jch] - 1;
          for (int j = jres0; j < jresn; ++j) {
            const int jt = aa_index(se[j]);
            for (int jatom = 1; jatom <= 2 - (se[j] == 'G' ? 1 : 0); ++jatom) {
              if (abs(i - j) < go_gamma.min_sep()) continue;
              if (go_mem.rf(i, iatom, j, jatom) < p.amh_go_rc) normi += go_gamma.get(it, jt, 0, 0, i, j);
            }
          }
          go_norm += pow(fabs(normi), p.amh_go_p);
        }
      }
    }
  }
  go_norm /= 8 * iresn;
}

/* compute_amh_go_model, fix_backbone.cpp:3856-3992, over the fix's full
   neighbour list: for each atom i, every atom j != i in the list (in_list),
   in atom order. */
void System::amhgo_term(const double *x, double *f)
{
  const Params &p = P;
  const int min_sep = go_gamma.min_sep();
  double Etot = 0.0;
  std::vector<int> fmap;
  std::vector<double> fbuf;
  for (int i = 0; i < natoms; i++) {
    const int ires = ares[i], ri = ires - 1;
    const bool i_ca = i == ca[ri], i_cb = i == cb[ri] && se[ri] != 'G';
    if (!i_ca && !i_cb) continue;
    const int it = aa_index(se[ri]);
    fmap.assign(1, i);
    fbuf.assign(3, 0.0);
    double Ei = 0.0;
    for (int j = 0; j < natoms; j++) {
      if (j == i || !in_list(i, j)) continue;
      const int jres = ares[j], rj = jres - 1;
      if (p.censoring == 1 && (go_censored[(size_t) ri * n + rj] || go_censored[(size_t) rj * n + ri])) continue;
      const bool j_ca = j == ca[rj], j_cb = j == cb[rj] && se[rj] != 'G';
      if (!(j_ca || j_cb) || !(abs(ires - jres) >= min_sep || amol[i] != amol[j])) continue;
      const double rnative = go_mem.rf(ri, i_ca ? 1 : 2, rj, j_ca ? 1 : 2);
      if (!(rnative < p.amh_go_rc)) continue;
      const double dx[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
      const double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      const double dr = r - rnative, drsq = dr * dr;
      const double sigma_sq = pow(abs(ires - jres), 0.3);
      if (drsq < 27.6 * sigma_sq) {
        const double gamma = go_gamma.get(it, aa_index(se[rj]), 0, 0, ri, rj);
        const double Eij = gamma * exp(-drsq / (2.0 * sigma_sq));
        const double force = Eij * dr / (sigma_sq * r);
        fmap.push_back(j);
        for (int k = 0; k < 3; k++) {
          fbuf[k] += force * dx[k];
          fbuf.push_back(-force * dx[k]);
        }
        Ei += Eij;
      }
    }
    const double factor = -0.5 * p.k_amh_go * p.amh_go_p * pow(Ei, p.amh_go_p - 1) / go_norm;
    for (size_t k = 0; k < fmap.size(); k++)
      for (int c = 0; c < 3; c++) f[3 * fmap[k] + c] += factor * fbuf[3 * k + c];
    Etot += -0.5 * p.k_amh_go * pow(Ei, p.amh_go_p) / go_norm;
  }
  E[ET_AMHGO] += Etot;
}

/* The fix's neighbour lists (cut plc + skin; fix_backbone.cpp:1805-1813)
   as LAMMPS keeps them: built at a run setup, then by Neighbor::decide() --
   after `delay` steps, on multiples of `every`, and with `check` only once an
   atom has moved more than half the skin since the last build. */
void System::list_update(const double *x)
{
  bool build = list_setup;
  list_setup = false;
  if (!build) {
    list_ago++;
    if (list_ago >= nb_delay && list_ago % nb_every == 0) {
      if (!nb_check) {
        build = true;
      } else {
        const double trigger = 0.25 * nb_skin * nb_skin;
        for (int a = 0; a < natoms && !build; a++) {
          double dx = x[3 * a] - xhold[3 * a], dy = x[3 * a + 1] - xhold[3 * a + 1], dz = x[3 * a + 2] - xhold[3 * a + 2];
          if (dx * dx + dy * dy + dz * dz > trigger) build = true;
        }
      }
    }
  }
  if (build) {
    xhold.assign(x, x + 3 * natoms);
    list_ago = 0;
  }
}

/* atoms a and b are neighbours in those lists: within plc + skin at the last
   build, not 1-2 bonded (special_bonds fene) */
bool System::in_list(int a, int b) const
{
  const double cut = plc + nb_skin, cutsq = cut * cut;
  double dx = xhold[3 * a] - xhold[3 * b], dy = xhold[3 * a + 1] - xhold[3 * b + 1], dz = xhold[3 * a + 2] - xhold[3 * b + 2];
  if (!(dx * dx + dy * dy + dz * dz < cutsq)) return false;
  for (int s : special[a])
    if (s == b) return false;
  return true;
}

/* charge_on_residues.dat (fix_backbone.cpp:1022-1045) and the contact
   restraints file (read_contact_restraints_file, :1106-1171) */
void System::read_pair_extras()
{
  Params &p = P;
  if (p.huckel) {
    charge.assign(n, 0.0);
    std::ifstream in(join(workdir, "charge_on_residues.dat"));
    if (!in) throw std::runtime_error("File charge_on_residues.dat doesn't exist");
    int total = 0;
    in >> total;
    for (int k = 0; k < total; k++) {
      int r;
      double q;
      in >> r >> q;
      if (r < 1 || r > n) throw std::runtime_error("oracle: charge_on_residues.dat residue out of range");
      charge[r - 1] = q;
    }
  }
  if (p.cont_rest) {
    std::ifstream in(join(workdir, p.cr_file));
    if (!in) throw std::runtime_error("File for Contact Restraints potential doesn't exist");
    cr_map.assign(n, {});
    int i1, i2;
    double ww, r0, r0_max = 0.0;
    while (in >> i1 >> i2 >> ww >> r0) {
      if (in.eof()) throw std::runtime_error("Contact Restraints potential parameter file format error");
      int j1 = std::min(i1, i2) - 1, j2 = std::max(i1, i2) - 1;
      if (j1 < 0 || j1 >= n || j2 < 0 || j2 >= n)
        throw std::runtime_error("Indices out of range in Contact Restraints potential file");
      cr_map[j1].push_back({j2, ww * p.k_cont_rest, r0});
      if (r0 > r0_max) r0_max = r0;
    }
    p.cr_dr_cutoff = p.cr_sigma * 4.29;
    p.cr_glob_cutoff_sq = pow(r0_max + p.cr_dr_cutoff, 2);
    for (auto &m : cr_map)
      std::stable_sort(m.begin(), m.end(), [](const Restraint &a, const Restraint &b) { return a.i2 < b.i2; });
  }
}

/* compute_solvent_barrier, fix_backbone.cpp:6237-6305 (residues i < j) */
void System::solvent_barrier(int i, int j, const double *x, double *f)
{
  const Params &p = P;
  if (chain_of[i] == chain_of[j] && j - i < p.ssb_ij_sep) return;
  const int iatom = contact_atom(i), jatom = contact_atom(j);
  double dx[3] = {x[3 * iatom] - x[3 * jatom], x[3 * iatom + 1] - x[3 * jatom + 1], x[3 * iatom + 2] - x[3 * jatom + 2]};
  double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
  double rmin1 = p.ssb_rmin1, rmax1 = p.ssb_rmax1, rmin2 = p.ssb_rmin2, rmax2 = p.ssb_rmax2;
  if (p.ssb_rad_cor) {
    double rshift = p.ssb_rshift[type_of(i)] + p.ssb_rshift[type_of(j)];
    rmin1 += rshift;
    rmax1 += rshift;
    rmin2 += rshift;
    rmax2 += rshift;
  }
  if (r > rmax1 + 10 / p.ssb_kappa && r > rmax2 + 10 / p.ssb_kappa) return;
  double t_min1 = tanh(p.ssb_kappa * (r - rmin1)), t_max1 = tanh(p.ssb_kappa * (rmax1 - r));
  double t_min2 = tanh(p.ssb_kappa * (r - rmin2)), t_max2 = tanh(p.ssb_kappa * (rmax2 - r));
  double theta1 = 0.5 * (t_min1 + t_max1), theta2 = 0.5 * (t_min2 + t_max2);
  E[ET_SSB] += p.epsilon * p.k_solventb1 * theta1;
  E[ET_SSB] += p.epsilon * p.k_solventb2 * theta2;
  double force1 = -p.epsilon * p.k_solventb1 * p.ssb_kappa * theta1 * (t_max1 - t_min1) / r;
  double force2 = -p.epsilon * p.k_solventb2 * p.ssb_kappa * theta2 * (t_max2 - t_min2) / r;
  for (int k = 0; k < 3; k++) {
    f[3 * iatom + k] += force1 * dx[k];
    f[3 * iatom + k] += force2 * dx[k];
    f[3 * jatom + k] += -force1 * dx[k];
    f[3 * jatom + k] += -force2 * dx[k];
  }
}

/* compute_DebyeHuckel_Interaction, fix_backbone.cpp:6307-6363 (residues i < j) */
void System::debye_huckel(int i, int j, const double *x, double *f)
{
  const Params &p = P;
  if (abs(i - j) < p.debye_huckel_min_sep) return;
  double qi = charge[i], qj = charge[j];
  if (qi == 0 && qj == 0) return;
  const int iatom = contact_atom(i), jatom = contact_atom(j);
  double dx[3] = {x[3 * iatom] - x[3 * jatom], x[3 * iatom + 1] - x[3 * jatom + 1], x[3 * iatom + 2] - x[3 * jatom + 2]};
  double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
  double qq = 0.0;
  if (qi > 0.0 && qj > 0.0) qq = p.k_PlusPlus * qi * qj / r;
  else if (qi < 0.0 && qj < 0.0) qq = p.k_MinusMinus * qi * qj / r;
  else if ((qi < 0.0 && qj > 0.0) || (qi > 0.0 && qj < 0.0)) qq = p.k_PlusMinus * qi * qj / r;
  double e = p.epsilon * qq * exp(-p.k_screening * r / p.screening_length);
  E[ET_DH] += e;
  double force = (e / r) * (1.0 / r + p.k_screening / p.screening_length);
  for (int k = 0; k < 3; k++) {
    f[3 * iatom + k] += force * dx[k];
    f[3 * jatom + k] += -force * dx[k];
  }
}

/* The DL3 loop's contact restraints (fix_backbone.cpp:8058-8060, :8137-8177)
   on contact-bead pairs, solvent barrier and Debye-Hueckel (:8105-8114) on
   CA pairs, each pair as the fix's half list holds it. */
void System::pair_extras(const double *x, double *f)
{
  const Params &p = P;
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++) {
      const int ci = contact_atom(i), cj = contact_atom(j);
      if (p.cont_rest && (amol[ci] != amol[cj] || j - i > 1) && !cr_map[i].empty()) {
        double dx[3] = {x[3 * ci] - x[3 * cj], x[3 * ci + 1] - x[3 * cj + 1], x[3 * ci + 2] - x[3 * cj + 2]};
        double rsq = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (rsq < p.cr_glob_cutoff_sq && in_list(ci, cj)) {
          for (const Restraint &c : cr_map[i]) {
            if (c.i2 != j) continue;
            double r = sqrt(rsq), dr = r - c.r0;
            if (fabs(dr) < p.cr_dr_cutoff) {
              double V = -c.w * exp(-0.5 * (dr * dr) * p.cr_sigma_sq_inv);
              double force = V * dr * p.cr_sigma_sq_inv / r;
              E[ET_CONT_REST] += V;
              for (int k = 0; k < 3; k++) {
                f[3 * ci + k] += force * dx[k];
                f[3 * cj + k] -= force * dx[k];
              }
            }
            break;
          }
        }
      }
      if ((p.ssb || p.huckel) && in_list(ca[i], ca[j])) {
        if (p.ssb && (amol[ca[i]] != amol[ca[j]] || j - i >= p.ssb_ij_sep)) solvent_barrier(i, j, x, f);
        if (p.huckel && j - i > 1) debye_huckel(i, j, x, f);
      }
    }
}

/* compute_shake, fix_backbone.cpp:2172-2237 */
void System::shake_term(int i, double *f)
{
  const Params &p = P;
  auto bond = [&](const double *u, const double *v, int au, int av, double r0) {
    double dx[3] = {u[0] - v[0], u[1] - v[1], u[2] - v[2]};
    double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    double dr = r - r0;
    double force = 2 * p.epsilon * p.k_shake * dr / r;
    E[ET_SHAKE] += p.epsilon * p.k_shake * dr * dr;
    for (int k = 0; k < 3; k++) {
      f[3 * au + k] -= dx[k] * force;
      f[3 * av + k] -= -dx[k] * force;
    }
  };
  if (!last(i)) bond(&xca[3 * i], &xca[3 * (i + 1)], ca[i], ca[i + 1], p.r_sh1);
  bond(&xca[3 * i], &xo[3 * i], ca[i], o[i], p.r_sh2);
  if (!last(i)) bond(&xo[3 * i], &xca[3 * (i + 1)], o[i], ca[i + 1], p.r_sh3);
}

/* compute_membrane_potential, fix_backbone.cpp:6107-6235 (pore type 0) */
void System::membrane_term(int i, double *f)
{
  const Params &p = P;
  const double *xi = se[i] == 'G' ? &xca[3 * i] : &xcb[3 * i];
  const int iatom = contact_atom(i);
  double dx = xi[0] - p.memb_xo[0], dy = xi[1] - p.memb_xo[1], dz = xi[2] - p.memb_xo[2];
  double memb_a = p.rho0_distor * p.rho0_max, memb_b = p.memb_len / 2;
  double rho_actual = sqrt(dx * dx + dy * dy);
  double rho0 = (p.rho0_max - memb_a) + ((memb_a) / (p.memb_len)) * (dz + memb_b);
  const double kb = p.k_bin;
  double s_per = 0.5 * (1 + tanh(kb * (dz - memb_b)));
  double s_mem = 0.5 * ((tanh(kb * (dz + memb_b))) + (tanh(kb * (memb_b - dz))));
  double s_cyt = 0.5 * (1 + tanh(kb * (-memb_b - dz)));
  double s_por = 0.5 * (1 - (tanh(kb * (rho_actual - rho0))));
  double s_nopor = (1 - s_por);
  const double(*g)[4] = p.g_memb;
  double V = 0.0;
  if (z_res[i] == 1) V = (-g[0][0] * s_per) + (-g[0][1] * s_cyt) + (g[0][2] * s_mem * s_nopor) + (-g[0][3] * s_mem * s_por);
  else if (z_res[i] == 2) V = (g[1][0] * s_per) + (g[1][1] * s_cyt) + (-g[1][2] * s_mem * s_nopor) + (g[1][3] * s_mem * s_por);
  else V = (-g[2][0] * s_per) + (-g[2][1] * s_cyt) + (g[2][2] * s_mem * s_nopor) + (-g[2][3] * s_mem * s_por);
  E[ET_MEMB] += p.epsilon * p.k_overall_memb * V;
  double dz_per = 0.5 * kb * (1 - pow((tanh(kb * (dz - memb_b))), 2));
  double dz_mem = -0.5 * kb * pow(tanh(kb * (dz + memb_b)), 2) + 0.5 * kb * pow(tanh(kb * (memb_b - dz)), 2);
  double dz_cyt = -0.5 * kb * (1 - pow((tanh(kb * (-memb_b - dz))), 2));
  double dr1_dz = ((memb_a) / (p.memb_len));
  double dz_s_por = 0.5 * kb * (1 - pow(tanh(kb * (rho_actual - rho0)), 2)) * dr1_dz;
  double dx_s_por = ((-0.5 * kb * dx) / rho_actual) * (1 - pow(tanh(kb * (rho_actual - rho0)), 2));
  double dy_s_por = ((-0.5 * kb * dy) / rho_actual) * (1 - pow(tanh(kb * (rho_actual - rho0)), 2));
  double dx_s_nopor = -dx_s_por, dy_s_nopor = -dy_s_por, dz_s_nopor = -dz_s_por;
  double dz_s_por_smem = s_mem * dz_s_por + dz_mem * s_por;
  double dz_s_nopor_smem = s_mem * dz_s_nopor + dz_mem * s_nopor;
  double dV_dx, dV_dy, dV_dz;
  if (z_res[i] == 1) {
    dV_dx = g[0][2] * s_mem * dx_s_nopor + (-g[0][3]) * s_mem * dx_s_por;
    dV_dy = g[0][2] * s_mem * dy_s_nopor + (-g[0][3]) * s_mem * dy_s_por;
    dV_dz = -g[0][0] * dz_per + (-g[0][1]) * dz_cyt + g[0][2] * dz_s_nopor_smem + (-g[0][3]) * dz_s_por_smem;
  } else if (z_res[i] == 2) {
    dV_dx = -g[1][2] * s_mem * dx_s_nopor + g[1][3] * s_mem * dx_s_por;
    dV_dy = -g[1][2] * s_mem * dy_s_nopor + g[1][3] * s_mem * dy_s_por;
    dV_dz = g[1][0] * dz_per + g[1][1] * dz_cyt + (-g[1][2]) * dz_s_nopor_smem + g[1][3] * dz_s_por_smem;
  } else {
    dV_dx = g[2][2] * s_mem * dx_s_nopor + (-g[2][3]) * s_mem * dx_s_por;
    dV_dy = g[2][2] * s_mem * dy_s_nopor + (-g[2][3]) * s_mem * dy_s_por;
    dV_dz = -g[2][0] * dz_per + (-g[2][1]) * dz_cyt + g[2][2] * dz_s_nopor_smem + (-g[2][3]) * dz_s_por_smem;
  }
  f[3 * iatom + 0] += -p.epsilon * p.k_overall_memb * dV_dx;
  f[3 * iatom + 1] += -p.epsilon * p.k_overall_memb * dV_dy;
  f[3 * iatom + 2] += -p.epsilon * p.k_overall_memb * dV_dz;
}

/* compute_vector_fragment_memory_potential, fix_backbone.cpp:3994-4077 */
void System::vfm_term(int i, double *f)
{
  const Params &p = P;
  for (int k : fm_map[i]) {
    const Memory &m = mems[k];
    const double epsilon_k_weight = p.epsilon * p.k_vec_frag_mem;
    int js = i + G.min_sep(), je = m.pos + m.len - 1;
    if (G.max_sep() != -1) je = std::min(je, i + G.max_sep());
    if (je >= n) throw std::runtime_error("Missing residues in memory potential");
    for (int j = js; j <= je; ++j) {
      if (chain_of[i] != chain_of[j])
        throw std::runtime_error("Fragment Memory: Interaction between residues of different chains");
      if (se[i] == 'G' || se[j] == 'G' || m.se[i - m.pos] == 'G' || m.se[j - m.pos] == 'G') continue;
      double vi[3], vj[3];
      for (int c = 0; c < 3; c++) {
        vi[c] = xcb[3 * i + c] - xca[3 * i + c];
        vj[c] = xcb[3 * j + c] - xca[3 * j + c];
      }
      double vmsqi = vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2];
      double vmsqj = vj[0] * vj[0] + vj[1] * vj[1] + vj[2] * vj[2];
      double vmi = sqrt(vmsqi), vmj = sqrt(vmsqj);
      double vp = vi[0] * vj[0] + vi[1] * vj[1] + vi[2] * vj[2];
      double vpn = vp / (vmi * vmj);
      double gc = acos(vpn);
      double gf = m.vmf[(i - m.pos) * m.len + (j - m.pos)];
      double dg = gc - gf;
      double V = -epsilon_k_weight * exp(-dg * dg / (2 * p.vfm_sigma_sq));
      E[ET_VFRAGMEM] += V;
      double force = -V * dg / (p.vfm_sigma_sq * vmi * vmj * sqrt(1 - vpn * vpn));
      for (int c = 0; c < 3; c++) {
        double fi = force * (vj[c] - vi[c] * vp / vmsqi), fj = force * (vi[c] - vj[c] * vp / vmsqj);
        f[3 * ca[i] + c] += -fi;
        f[3 * cb[i] + c] += fi;
        f[3 * ca[j] + c] += -fj;
        f[3 * cb[j] + c] += fj;
      }
    }
  }
}

/* compute_backbone, fix_backbone.cpp:7047-7673, then vexcluded and bonds */
void System::compute(const double *x, double *f)
{
  const Params &p = P;
  for (double &e : E) e = 0.0;
  for (int k = 0; k < 3 * natoms; k++) f[k] = 0.0;
  if (lists_used()) list_update(x);
  backbone_atoms(x);
  for (int i = 0; i < n; i++) {
    if (p.chain) chain_term(i, f);
    if (!first(i) && !last(i) && p.chi && se[i] != 'G') chi_term(i, f);
    if (!first(i) && !last(i) && p.rama && se[i] != 'G') rama_term(i, f);
    if (p.shake) shake_term(i, f);
    if (p.memb) membrane_term(i, f);
    if (p.vfm) vfm_term(i, f);
    if (p.fm) fm_term(i, f);
    if (p.fm_tb) tb_term(i, f);
  }
  pair_terms(x, f);
  if (p.ssb || p.huckel || p.cont_rest) pair_extras(x, f);
  if (p.amhgo) amhgo_term(x, f);
  for (int k = 1; k < NET; k++) E[ET_TOTAL] += E[k];
  excluded_volume(x, f);
  bonds(x, f);
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char *oracle_last_error(void) { return g_err.c_str(); }

void *oracle_create(const char *workdir, const char *data_file, const char *coeff_file, const char *seq_file,
                    const char *pair_style, const char *pair_coeffs)
{
  System *S = new System();
  try {
    S->workdir = workdir ? workdir : "";
    S->read_coeff(join(S->workdir, coeff_file));
    S->read_seq(join(S->workdir, seq_file));
    S->read_data(join(S->workdir, data_file));
    build_residues(*S);
    S->read_tables();
    if (S->P.vfm && !S->P.fm && !S->P.fm_tb)
      throw std::runtime_error("oracle: Vector_Fragment_Memory needs the fragment-memory memories");
    if (S->P.fm || S->P.fm_tb) S->read_mems();
    if (S->P.fm_tb) S->build_tb();
    if (S->P.ssb || S->P.huckel || S->P.cont_rest) S->read_pair_extras();
    if (S->P.memb) {
      // zim (fix_backbone.cpp:611-619)
      std::ifstream in(join(S->workdir, "zim"));
      if (!in) throw std::runtime_error("File zim doesn't exist");
      S->z_res.assign(S->n, 0);
      for (int i = 0; i < S->n; ++i) {
        in >> S->z_res[i];
        if (in.eof()) throw std::runtime_error("Membrane potential parameter file format error");
        if (S->z_res[i] < 1 || S->z_res[i] > 3) throw std::runtime_error("oracle: zim values must be 1, 2 or 3");
      }
    }
    if (S->lists_used()) S->plc = pair_list_cut(S->P);
    if (S->P.amhgo) S->read_amh_go();
    S->pair_setup(pair_style, pair_coeffs ? pair_coeffs : "");
  } catch (std::exception &e) {
    g_err = e.what();
    delete S;
    return nullptr;
  }
  return S;
}

void oracle_destroy(void *h) { delete (System *) h; }
int oracle_natoms(void *h) { return ((System *) h)->natoms; }
int oracle_nres(void *h) { return ((System *) h)->n; }

int oracle_compute(void *h, const double *x, double *f, double *energies)
{
  System *S = (System *) h;
  try {
    std::vector<double> tmp;
    if (!f) {
      tmp.resize(3 * S->natoms);
      f = tmp.data();
    }
    S->list_setup = true;  // a single evaluation builds its lists
    S->compute(x, f);
    if (energies) {
      for (int k = 0; k < NET; k++) energies[k] = S->E[k];
      energies[18] = S->e_pair;
      energies[19] = S->e_bond;
      energies[20] = 0.0;
    }
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

int oracle_residue_arrays(void *h, double *out)
{
  System *S = (System *) h;
  for (int i = 0; i < S->n; i++) {
    out[8 * i + 0] = S->rho_w[i];
    out[8 * i + 1] = S->rho_h[i];
    out[8 * i + 2] = S->xi_w[i];
    out[8 * i + 3] = S->xi1[i];
    out[8 * i + 4] = S->xi2[i];
    out[8 * i + 5] = S->bur[i];
    out[8 * i + 6] = S->sig_w[i];
    out[8 * i + 7] = S->sig_h[i];
  }
  return S->n;
}

long long oracle_selections(void *h, const double *x, int which, unsigned long long *out, long long cap)
{
  System *S = (System *) h;
  try {
    std::vector<double> f((size_t) 3 * S->natoms);
    S->sel_keys.clear();
    S->near_keys.clear();
    S->touch_keys.clear();
    S->sel_on = true;
    S->list_setup = true;
    S->compute(x, f.data());
    S->sel_on = false;
  } catch (std::exception &e) {
    S->sel_on = false;
    g_err = e.what();
    return -1;
  }
  std::vector<uint64_t> &v = which == 0 ? S->sel_keys : which == 1 ? S->near_keys : S->touch_keys;
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  for (long long k = 0; k < (long long) v.size() && k < cap; k++) out[k] = v[k];
  return (long long) v.size();
}

int oracle_run(void *h, double *x, double *v, long long step0, long long nsteps, double dt, int langevin,
               double t_start, double t_stop, double damp, unsigned long long seed, double *thermo)
{
  System *S = (System *) h;
  try {
    int N = S->natoms;
    std::vector<double> f(3 * N);
    long long begin = step0, end = step0 + nsteps;
    auto ke = [&]() {
      double s = 0.0;
      for (int i = 0; i < N; i++) {
        double m = S->mass[S->atype[i]];
        s += m * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
      }
      return 0.5 * MVV2E * s;
    };
    /* fix langevin post_force: uniform noise, units real */
    auto langevin_force = [&](long long step) {
      if (!langevin) return;
      double delta = end != begin ? (double) (step - begin) / (double) (end - begin) : 0.0;
      double tsqrt = sqrt(t_start + delta * (t_stop - t_start));
      for (int i = 0; i < N; i++) {
        double m = S->mass[S->atype[i]];
        double g1 = -m / damp / FTM2V;
        double g2 = sqrt(m) * sqrt(24.0 * BOLTZ / damp / dt / MVV2E) / FTM2V * tsqrt;
        for (int k = 0; k < 3; k++)
          f[3 * i + k] += g1 * v[3 * i + k] + g2 * (uniform01(seed, step, S->tag[i], k) - 0.5);
      }
    };
    auto row = [&](long long r) {
      if (!thermo) return;
      thermo[4 * r + 0] = S->E[ET_TOTAL];
      thermo[4 * r + 1] = S->e_pair;
      thermo[4 * r + 2] = S->e_bond;
      thermo[4 * r + 3] = ke();
    };
    S->list_setup = true;  // the run's setup builds the lists
    S->compute(x, f.data());
    langevin_force(begin);
    row(0);
    double dtf = 0.5 * dt * FTM2V;
    for (long long s = 1; s <= nsteps; s++) {
      for (int i = 0; i < N; i++) {
        double dtfm = dtf / S->mass[S->atype[i]];
        for (int k = 0; k < 3; k++) {
          v[3 * i + k] += dtfm * f[3 * i + k];
          x[3 * i + k] += dt * v[3 * i + k];
        }
      }
      S->compute(x, f.data());
      langevin_force(begin + s);
      for (int i = 0; i < N; i++) {
        double dtfm = dtf / S->mass[S->atype[i]];
        for (int k = 0; k < 3; k++) v[3 * i + k] += dtfm * f[3 * i + k];
      }
      row(s);
    }
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

int oracle_set_neighbor(void *h, double skin, int delay, int every, int check)
{
  System *S = (System *) h;
  if (!(skin >= 0.0) || delay < 0 || every < 1) {
    g_err = "oracle_set_neighbor: skin >= 0, delay >= 0, every >= 1";
    return -1;
  }
  S->nb_skin = skin;
  S->nb_delay = delay;
  S->nb_every = every;
  S->nb_check = check ? 1 : 0;
  return 0;
}

/* compute qwolynes (compute_q_wolynes.cpp:50-238) and compute qonuchic
   (compute_q_onuchic.cpp:27-317) over the CA atoms (group alpha_carbons),
   `words` as after LAMMPS's `compute`, data files opened as named. */
int oracle_q(void *h, const double *x, const char *words_c, double *out)
{
  System *S = (System *) h;
  try {
    std::vector<std::string> w = words(words_c);
    if (w.size() < 3) throw std::runtime_error("compute: ID group style ...");
    if (w[1] != "alpha_carbons") throw std::runtime_error("oracle: Q over the group alpha_carbons only");
    const int n = S->n;
    auto xca = [&](int r, int k) { return x[3 * S->ca[r] + k]; };
    double q = 0.0;
    if (w[2] == "qwolynes") {
      if (w.size() != 6) throw std::runtime_error("Illegal compute qwolynes command");
      int sep = atoi(w[4].c_str());
      double sigmaexp = atof(w[5].c_str());
      std::vector<double> r_native((size_t) n * n);
      std::ifstream in(w[3]);
      if (!in) throw std::runtime_error("Native distance file can't be read");
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) in >> r_native[(size_t) i * n + j];
      for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
          if (!(abs(j - i) > sep)) continue;
          double sigmaij = pow(1 + abs(i - j), sigmaexp);
          double rijn = r_native[(size_t) i * n + j];
          double rij = sqrt(pow(xca(i, 0) - xca(j, 0), 2) + pow(xca(i, 1) - xca(j, 1), 2) + pow(xca(i, 2) - xca(j, 2), 2));
          q += exp(-pow(rij - rijn, 2) / (2.0 * pow(sigmaij, 2)));
        }
      *out = q * (2.0 / (((double) n - (double) sep) * ((double) n - ((double) sep + 1.0))));
      return 0;
    }
    if (w[2] != "qonuchic") throw std::runtime_error("oracle: compute style " + w[2]);
    int narg = (int) w.size();
    if (narg != 5 && narg != 6 && narg != 7) throw std::runtime_error("Illegal compute qonuchic command");
    enum { T_CUTOFF = 0, T_SHADOW = 1, T_CUTOFF_GAUSS = 2, T_SHADOW_GAUSS = 3 };
    int cp_type;
    double factor = 1.0, r_consq = 0.0;
    std::string datafile;
    if (w[3] == "cutoff" || w[3] == "cutoff/gauss") {
      cp_type = w[3] == "cutoff" ? T_CUTOFF : T_CUTOFF_GAUSS;
      if (narg != (cp_type == T_CUTOFF ? 7 : 6)) throw std::runtime_error("Illegal compute qonuchic command");
      double r_contact = atof(w[4].c_str());
      r_consq = r_contact * r_contact;
      datafile = w[5];
      if (cp_type == T_CUTOFF) factor = atof(w[6].c_str());
    } else if (w[3] == "shadow" || w[3] == "shadow/gauss") {
      cp_type = w[3] == "shadow" ? T_SHADOW : T_SHADOW_GAUSS;
      if (narg != (cp_type == T_SHADOW ? 6 : 5)) throw std::runtime_error("Illegal compute qonuchic command");
      datafile = w[4];
      if (cp_type == T_SHADOW) factor = atof(w[5].c_str());
    } else {
      throw std::runtime_error("Wrong type for compute qonuchic");
    }
    const double sigmaexp = 0.15;
    std::vector<double> rsq_native((size_t) n * n, 0.0);
    std::vector<char> is_native((size_t) n * n, 0);
    double qnorm = 0.0;
    if (cp_type == T_CUTOFF || cp_type == T_CUTOFF_GAUSS) {
      FILE *f = fopen(datafile.c_str(), "r");
      if (!f) throw std::runtime_error("Compute qonuchic: can't read native coordinates");
      int nAtoms = 0;
      if (fscanf(f, "%d", &nAtoms) != 1 || nAtoms != n) {
        fclose(f);
        throw std::runtime_error("Compute qonuchic: atom number mismatch");
      }
      std::vector<double> xn((size_t) 3 * n);
      for (int i = 0; i < n; ++i)
        if (fscanf(f, "%lf %lf %lf", &xn[3 * i], &xn[3 * i + 1], &xn[3 * i + 2]) != 3) {
          fclose(f);
          throw std::runtime_error("Compute qonuchic: can't read native coordinates");
        }
      fclose(f);
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          double dx0 = xn[3 * j] - xn[3 * i], dx1 = xn[3 * j + 1] - xn[3 * i + 1], dx2 = xn[3 * j + 2] - xn[3 * i + 2];
          double &r = rsq_native[(size_t) i * n + j];
          r = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
          if (r < r_consq && j - i > 3) {
            is_native[(size_t) i * n + j] = 1;
            qnorm += 1.0;
          }
          if (cp_type == T_CUTOFF && is_native[(size_t) i * n + j]) r *= factor * factor;
        }
    } else {
      FILE *f = fopen(datafile.c_str(), "r");
      if (!f) throw std::runtime_error("Compute qonuchic: can't read contact map file");
      int ires, jres;
      double rn;
      while (fscanf(f, "%d %d %lf", &ires, &jres, &rn) == 3) {
        ires--;
        jres--;
        if (ires >= n || jres >= n || ires < 0 || jres < 0 || abs(jres - ires) <= 3) {
          fclose(f);
          throw std::runtime_error("Compute qonuchic: wrong residue index in shadow contact map file");
        }
        is_native[(size_t) ires * n + jres] = 1;
        rsq_native[(size_t) ires * n + jres] = rn * rn;
        if (cp_type == T_SHADOW) rsq_native[(size_t) ires * n + jres] *= factor * factor;
        qnorm += 1.0;
      }
      fclose(f);
    }
    qnorm = 1 / qnorm;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) {
        if (!(is_native[(size_t) i * n + j] && abs(j - i) > 3)) continue;
        double dx0 = xca(i, 0) - xca(j, 0), dx1 = xca(i, 1) - xca(j, 1), dx2 = xca(i, 2) - xca(j, 2);
        double rsq = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
        if (cp_type == T_CUTOFF || cp_type == T_SHADOW) {
          if (rsq < rsq_native[(size_t) i * n + j]) q += 1.0;
        } else {
          double sigma_sq = pow(1 + abs(i - j), 2.0 * sigmaexp);
          q += exp(-pow(sqrt(rsq) - sqrt(rsq_native[(size_t) i * n + j]), 2) / (2.0 * sigma_sq));
        }
      }
    *out = q * qnorm;
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
  return 0;
}

double oracle_uniform(unsigned long long seed, long long step, long long tag, int comp)
{
  return uniform01(seed, step, tag, comp);
}

}  // extern "C"
