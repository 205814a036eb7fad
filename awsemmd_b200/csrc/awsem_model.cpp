// Host-side model construction: parsers for the reference's input formats and
// the builders that turn them into the engine's device layouts.
//
// Formats and semantics follow the reference:
//   coefficient file section loop + epsilon scaling   fix_backbone.cpp:164-516
//   DSSP tables, ssweight, gamma.dat, burial_gamma.dat fix_backbone.cpp:555-693
//   sequence file                                     fix_backbone.cpp:537-553
//   .mem list / .gro memories                         fix_backbone.cpp:1966-2042,
//                                                     fragment_memory.cpp:34-176
//   gamma file (Gamma_Array)                          fragment_memory.cpp:275-454
//   residue -> memory map                             fix_backbone.cpp:749-791
//   pair_style/pair_coeff vexcluded                   pair_excluded_volume.cpp:175-265
#include "awsem_model.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>

namespace awsem {

namespace {

const char kAA[] = "ARNDCQEGHILKMFPSTWYV";

int residue_code(char c)
{
  const char *p = strchr(kAA, c);
  return (p && c) ? int(p - kAA) : 0;
}

int residue_class4(int t)
{
  // SHL 1 (A G P S T), AHL 2 (N D Q E), BAS 3 (R H K), HPB 4 (C I L M F W Y V)
  static const int cls[20] = {1, 3, 2, 2, 4, 2, 2, 1, 3, 4, 4, 3, 4, 4, 1, 1, 1, 4, 4, 4};
  return cls[t];
}

std::vector<std::string> tokens(const std::string &line)
{
  std::vector<std::string> out;
  std::istringstream in(line);
  for (std::string t; in >> t;) out.push_back(t);
  return out;
}

std::string path_in(const std::string &dir, const std::string &name)
{
  if (name.empty() || name[0] == '/' || dir.empty()) return name;
  return dir + "/" + name;
}

[[noreturn]] void fail(const std::string &msg) { throw std::runtime_error(msg); }

char residue_from_three(const char *s)
{
  static const char *names[20] = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
                                  "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"};
  for (int k = 0; k < 20; k++)
    if (!strcmp(s, names[k])) return kAA[k];
  return '?';
}

}  // namespace

void read_coeff_file(const std::string &path, ForceField &ff)
{
  std::ifstream in(path);
  if (!in) fail("Coefficient file was not found!");
  FFParams &p = ff.p;
  p = FFParams{};
  p.epsilon = 1.0;
  p.an = 0.4831806; p.bn = 0.7032820; p.cn = -0.1864262;
  p.ap = 0.4436538; p.bp = 0.2352006; p.cp = 0.3211455;
  p.ah = 0.8409657; p.bh = 0.8929599; p.ch = -0.7338894;
  p.fm_sigma_exp = 0.15;
  const int i_rp = 6;  // first proline Ramachandran well
  double k_rama = 0.0, k_water = 0.0;
  static const char *outside[] = {
      "[Excluded]", "[Excluded_P]", "[Excluded_R6]",
      "[Fragment_Frustratometer]", "[Tertiary_Frustratometer]", "[Nmer_Frustratometer]",
      "[Amylometer]", "[Selection_Temperature]", "[Monte_Carlo_Seq_Opt]", "[Optimization]",
      "[Burial_Optimization]", "[DebyeHuckel_Optimization]", "[Shuffler]", "[Mutate_Sequence]"};
  std::string s, pending;
  // a section that omits a trailing value leaves its successor's header as the
  // next token (`pending`)
  while (!pending.empty() ? (s = pending, pending.clear(), true) : (bool) (in >> s)) {
    if (s == "[ABC]") {
      in >> p.an >> p.bn >> p.cn >> p.ap >> p.bp >> p.cp >> p.ah >> p.bh >> p.ch;
    } else if (s == "[Chain]") {
      p.terms |= T_CHAIN;
      in >> p.k_chain[0] >> p.k_chain[1] >> p.k_chain[2] >> p.r_ncb0 >> p.r_cpcb0 >> p.r_ncp0;
    } else if (s == "[Chi]") {
      p.terms |= T_CHI;
      in >> p.k_chi >> p.chi0;
    } else if (s == "[Rama]") {
      p.terms |= T_RAMA;
      in >> k_rama >> p.n_rama;
      if (p.n_rama > i_rp) fail("Rama: too many wells");
      for (int j = 0; j < p.n_rama; j++) {
        double sigma;
        in >> p.w[j] >> sigma >> p.phiw[j] >> p.phi0[j] >> p.psiw[j] >> p.psi0[j];
        p.phiw[j] *= sigma;
        p.psiw[j] *= sigma;
      }
    } else if (s == "[Rama_P]") {
      p.terms |= T_RAMA_P;
      in >> p.n_rama_p;
      if (p.n_rama_p > 12 - i_rp) fail("Rama_P: too many wells");
      for (int j = i_rp; j < i_rp + p.n_rama_p; j++) {
        double sigma;
        in >> p.w[j] >> sigma >> p.phiw[j] >> p.phi0[j] >> p.psiw[j] >> p.psi0[j];
        p.phiw[j] *= sigma;
        p.psiw[j] *= sigma;
      }
    } else if (s == "[SSWeight]") {
      p.terms |= T_SSW;
      for (int j = 0; j < 12; j++) in >> p.ssweight[j];
    } else if (s == "[Dssp_Hdrgn]") {
      p.terms |= T_DSSP;
      double sHO, sNO;
      in >> p.k_dssp >> p.hbscl[0][0] >> p.hbscl[0][1];
      for (int j = 0; j < 7; j++) in >> p.hbscl[1][j];
      for (int j = 0; j < 9; j++) in >> p.hbscl[2][j];
      for (int j = 0; j < 9; j++) in >> p.hbscl[3][j];
      in >> sHO >> sNO >> p.HO_zero >> p.NO_zero >> p.dssp_cut >> p.pref[0] >> p.pref[1] >> p.d_nu0;
      p.dssp_cut_sq = p.dssp_cut * p.dssp_cut;
      for (int k = 0; k < 2; k++) p.nu_cut_sq[k] = pow(p.d_nu0 + atanh(2.0 * 1e-4 - 1.0) / p.pref[k], 2);
      p.sigma_HO_sqinv = 1.0 / (sHO * sHO);
      p.sigma_NO_sqinv = 1.0 / (sNO * sNO);
    } else if (s == "[P_AP]") {
      p.terms |= T_PAP;
      in >> p.k_global_pap >> p.k_betapred_pap >> p.k_pap[0] >> p.k_pap[1] >> p.k_pap[2] >> p.pap_cut >>
          p.pap_pref >> p.i_med_min >> p.i_med_max >> p.i_diff_pap;
      p.pap_cutoff_sq = pow(p.pap_cut + atanh(1.0 - 2.0 * 1e-12) / p.pap_pref, 2);
    } else if (s == "[Water]") {
      p.terms |= T_WATER;
      in >> k_water >> p.water_kappa >> p.water_kappa_sigma >> p.treshold >> p.contact_cutoff >> p.n_wells;
      if (p.n_wells > 5) fail("Water: at most 5 wells");
      for (int j = 0; j < p.n_wells; j++) in >> p.well_rmin[j] >> p.well_rmax[j] >> p.well_flag[j];
    } else if (s == "[Burial]") {
      p.terms |= T_BURIAL;
      in >> p.k_burial >> p.burial_kappa;
      for (int j = 0; j < 3; j++) in >> p.burial_ro_min[j] >> p.burial_ro_max[j];
    } else if (s == "[Helix]") {
      p.terms |= T_HELIX;
      double sHO, sNO;
      in >> p.k_helix >> p.helix_gamma_p >> p.helix_gamma_w >> p.helix_kappa >> p.helix_kappa_sigma >>
          p.helix_treshold >> p.helix_i_diff >> p.helix_cutoff >> p.helix_rmin >> p.helix_rmax;
      for (int j = 0; j < 20; j++) in >> p.h4prob[j];
      in >> p.pro_acc_flag >> p.h4prob_pro >> sHO >> sNO >> p.helix_HO_zero >> p.helix_NO_zero;
      p.helix_sigma_HO = sHO;
      p.helix_sigma_NO = sNO;
      p.helix_cutoff_sq = p.helix_cutoff * p.helix_cutoff;
      p.helix_sigma_HO_sqinv = 1.0 / (sHO * sHO);
      p.helix_sigma_NO_sqinv = 1.0 / (sNO * sNO);
    } else if (s == "[AMH-Go]") {
      // fix_backbone.cpp:297-303
      p.terms |= T_AMHGO;
      in >> p.k_amh_go >> p.amh_go_p >> p.amh_go_rc;
      std::string t;
      ff.amh_go_censor = 0;
      if (in >> t) {
        if (t[0] == '[') pending = t;  // the censoring flag is absent (older coefficient files)
        else ff.amh_go_censor = atoi(t.c_str());
      }
      if (ff.amh_go_censor == 2)
        fail("AMH-Go: frustration censoring 2 (native distances from go_rnative*.dat) is not supported");
    } else if (s == "[Vector_Fragment_Memory]") {
      // fix_backbone.cpp:328-333
      p.terms |= T_VFM;
      double sigma;
      in >> p.k_vfm >> sigma;
      p.vfm_sigma_sq = sigma * sigma;
    } else if (s == "[Shake]") {
      // fix_backbone.cpp:180-183
      p.terms |= T_SHAKE;
      in >> p.k_shake >> p.r_sh1 >> p.r_sh2 >> p.r_sh3;
    } else if (s == "[Membrane]") {
      // fix_backbone.cpp:346-358
      p.terms |= T_MEMB;
      in >> p.k_overall_memb >> p.k_bin >> p.memb_xo[0] >> p.memb_xo[1] >> p.memb_xo[2] >> p.memb_pore_type >>
          p.memb_len >> p.rho0_max >> p.rho0_distor;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 4; j++) in >> p.g_memb[i][j];
    } else if (s == "[Phosphorylation]") {
      // fix_backbone.cpp:413-421 (the water section must come first)
      if (!(p.terms & T_WATER)) fail("Cannot run phosphorylation without water potential");
      p.terms |= T_PHOSPH;
      in >> p.k_hypercharge >> p.n_phosph_res;
      if (p.n_phosph_res > 20) fail("Number of phosphorylated residues may not exceed 20");
      for (int i = 0; i < p.n_phosph_res; i++) in >> p.phosph_res[i];
    } else if (s == "[Solvent_Barrier]") {
      // fix_backbone.cpp:334-345 (the 20 radius shifts are read whatever the correction flag)
      p.terms |= T_SSB;
      in >> p.k_ssb1 >> p.ssb_rmin1 >> p.ssb_rmax1 >> p.k_ssb2 >> p.ssb_rmin2 >> p.ssb_rmax2 >> p.ssb_kappa >>
          p.ssb_ij_sep >> p.ssb_rad_cor;
      for (int j = 0; j < 20; j++) in >> p.ssb_rshift[j];
    } else if (s == "[DebyeHuckel]") {
      // fix_backbone.cpp:467-477
      p.terms |= T_DH;
      in >> p.k_plusplus >> p.k_minusminus >> p.k_plusminus >> p.k_screening >> p.screening_length >> p.dh_min_sep;
    } else if (s == "[Contact_Restraints]") {
      // fix_backbone.cpp:321-327
      p.terms |= T_CONTREST;
      in >> p.k_cont_rest >> p.cr_sigma >> ff.cr_file;
      p.cr_sigma_sq_inv = pow(p.cr_sigma, -2);
    } else if (s == "[Fragment_Memory]") {
      p.terms |= T_FM;
      in >> ff.k_fm_raw >> ff.fm_file >> ff.fm_gamma_file;
    } else if (s == "[Fragment_Memory_Table]") {
      // fix_backbone.cpp:310-321
      p.terms |= T_FM_TABLE;
      in >> ff.k_fm_raw >> ff.fm_file >> ff.fm_gamma_file;
      in >> p.tb_rmin >> p.tb_rmax >> p.tb_dr;
      p.tb_size = (int) ((p.tb_rmax - p.tb_rmin) / p.tb_dr) + 2;
      in >> ff.tb_width >> ff.tb_use_file >> p.fm_sigma_exp;
    } else if (s == "[Epsilon]") {
      in >> p.epsilon;
    } else {
      for (const char *o : outside)
        if (s == o) fail("section " + s + " is not supported by the GPU engine");
    }
  }
  // epsilon scaling (fix_backbone.cpp:501-516)
  for (double &k : p.k_chain) k *= p.epsilon;
  p.k_chi *= p.epsilon;
  k_rama *= p.epsilon;
  k_water *= p.epsilon;
  p.k_burial *= p.epsilon;
  p.k_helix *= p.epsilon;
  p.k_dssp *= p.epsilon;
  p.k_global_pap *= p.epsilon;
  for (int j = 0; j < p.n_rama; j++) p.w[j] *= k_rama;
  for (int j = 0; j < p.n_rama_p; j++) p.w[j + i_rp] *= k_rama;
  for (int j = 0; j < 12; j++) {
    p.cphi0[j] = cos(p.phi0[j]), p.sphi0[j] = sin(p.phi0[j]);
    p.cpsi0[j] = cos(p.psi0[j]), p.spsi0[j] = sin(p.psi0[j]);
  }
  p.k_fm = ff.k_fm_raw;
  p.k_amh_go *= p.epsilon;
  p.k_cont_rest *= p.epsilon;
  // density-well supports (smart_matrix_lib.h:363-368) and P_AP saturation (:110-115)
  for (int k = 0; k < p.n_wells; k++) {
    p.w_rmin_th[k] = p.well_rmin[k] - 8.0 * 2.302585 / p.water_kappa;
    p.w_rmax_th[k] = p.well_rmax[k] + 8.0 * 2.302585 / p.water_kappa;
    p.w_rmin_sq[k] = p.w_rmin_th[k] * p.w_rmin_th[k];
    p.w_rmax_sq[k] = p.w_rmax_th[k] * p.w_rmax_th[k];
  }
  if (p.terms & T_HELIX) {
    p.h_rmin_th = p.helix_rmin - 8.0 * 2.302585 / p.helix_kappa;
    p.h_rmax_th = p.helix_rmax + 8.0 * 2.302585 / p.helix_kappa;
    p.h_rmin_sq = p.h_rmin_th * p.h_rmin_th;
    p.h_rmax_sq = p.h_rmax_th * p.h_rmax_th;
  }
  if (p.terms & T_PAP) {
    double span = double(int(8.0 * 2.302585 / p.pap_pref) + 1);
    p.pap_drmax_sq = (p.pap_cut + span) * (p.pap_cut + span);
    p.pap_drmin_sq = (p.pap_cut - span) * (p.pap_cut - span);
  }
  ff.k_water = k_water;
  ff.tables.assign(TB_SIZE, 0.0);
  p.pair_list_cutoff = pair_list_cutoff(p);
}

double pair_list_cutoff(const FFParams &p)
{
  double cut = 8.0;  // fix_backbone.cpp:1051-1057
  if (p.terms & T_DSSP) cut = std::max(cut, p.dssp_cut);
  if (p.terms & T_PAP) cut = std::max(cut, sqrt(p.pap_cutoff_sq));
  if (p.terms & T_WATER)
    for (int k = 0; k < p.n_wells; k++) cut = std::max(cut, p.w_rmax_th[k]);
  if (p.terms & T_HELIX) {
    cut = std::max(cut, p.h_rmax_th);
    // calc_exp_helix_cutoff (:1074-1103): O(i) to the atoms behind the virtual N(j) and H(j)
    const double r0[3] = {3.77, 2.5, 2.41};
    double r1[3], r2[3];
    r1[0] = sqrt(pow(p.an * r0[0], 2) + pow(p.cn * r0[1], 2) + p.an * p.cn * (r0[0] * r0[0] + r0[1] * r0[1] - r0[2] * r0[2]));
    r1[1] = sqrt(pow(p.an * r0[2], 2) + pow(p.bn * r0[1], 2) + p.an * p.bn * (r0[2] * r0[2] + r0[1] * r0[1] - r0[0] * r0[0]));
    r1[2] = sqrt(pow(p.bn * r0[0], 2) + pow(p.cn * r0[2], 2) + p.bn * p.cn * (r0[0] * r0[0] + r0[2] * r0[2] - r0[1] * r0[1]));
    r2[0] = sqrt(pow(p.ah * r0[0], 2) + pow(p.ch * r0[1], 2) + p.ah * p.ch * (r0[0] * r0[0] + r0[1] * r0[1] - r0[2] * r0[2]));
    r2[1] = sqrt(pow(p.ah * r0[2], 2) + pow(p.bh * r0[1], 2) + p.ah * p.bh * (r0[2] * r0[2] + r0[1] * r0[1] - r0[0] * r0[0]));
    r2[2] = sqrt(pow(p.bh * r0[0], 2) + pow(p.ch * r0[2], 2) + p.bh * p.ch * (r0[0] * r0[0] + r0[2] * r0[2] - r0[1] * r0[1]));
    double r1_max = std::max(r1[0], std::max(r1[1], r1[2])), r2_max = std::max(r2[0], std::max(r2[1], r2[2]));
    r1_max = 1.1 * r1_max + p.helix_NO_zero + p.helix_sigma_NO * sqrt(6.0 * log(10.0));
    r2_max = 1.1 * r2_max + p.helix_HO_zero + p.helix_sigma_HO * sqrt(6.0 * log(10.0));
    cut = std::max(cut, std::max(r1_max, r2_max));
    cut = std::max(cut, p.helix_cutoff);
  }
  if (p.terms & T_CONTREST) cut = std::max(cut, sqrt(p.cr_cut_sq));
  if (p.terms & T_DH) cut = std::max(cut, 2.0 * p.screening_length / p.k_screening);
  if (p.terms & T_SSB) {
    double c = 0.0;
    if (p.ssb_rad_cor)
      for (int k = 0; k < 20; k++) c = std::max(c, 2.0 * p.ssb_rshift[k]);
    c += std::max(p.ssb_rmax1, p.ssb_rmax2) + 10.0 / p.ssb_kappa;
    cut = std::max(cut, c);
  }
  return cut;
}

void read_sequence(const std::string &path, Topology &top)
{
  std::ifstream in(path);
  if (!in) fail("Sequence file was not found");
  top.seq.clear();
  top.chain_start.clear();
  top.chain_end.clear();
  for (std::string t; in >> t;) {
    if (t[0] == '#') continue;
    top.chain_start.push_back((int) top.seq.size());
    top.seq += t;
    top.chain_end.push_back((int) top.seq.size() - 1);
  }
  top.n_chains = (int) top.chain_start.size();
  top.n_res = (int) top.seq.size();
}

void read_tables(const std::string &dir, ForceField &ff, Topology &top)
{
  FFParams &p = ff.p;
  double k_water = ff.k_water;
  std::vector<double> &T = ff.tables;
  T.assign(TB_SIZE, 0.0);
  if (p.terms & T_DSSP) {
    const char *names[5] = {"anti_HB", "anti_NHB", "para_HB", "para_one", "anti_one"};
    std::ifstream f[5];
    for (int k = 0; k < 5; k++) {
      f[k].open(path_in(dir, names[k]));
      if (!f[k]) fail(std::string("File ") + names[k] + " doesn't exist");
    }
    for (int blk = 0; blk < 2; blk++)
      for (int i = 0; i < 20; i++) {
        if (blk == 0) {
          f[3] >> T[TB_PARA_ONE + i];
          f[4] >> T[TB_ANTI_ONE + i];
        }
        for (int j = 0; j < 20; j++) {
          int at = (i * 20 + j) * 2 + blk;
          f[0] >> T[TB_ANTI_HB + at];
          f[1] >> T[TB_ANTI_NHB + at];
          f[2] >> T[TB_PARA_HB + at];
        }
      }
    for (auto &s : f)
      if (!s) fail("DSSP file format error");
  }
  top.aps.assign((size_t) 12 * top.n_res, 0.0);
  if (p.terms & T_SSW) {
    std::ifstream in(path_in(dir, "ssweight"));
    if (!in) fail("File ssweight doesn't exist");
    for (int r = 0; r < top.n_res; r++)
      for (int k = 0; k < 12; k++)
        if (p.ssweight[k]) in >> top.aps[(size_t) k * top.n_res + r];
  }
  if (p.terms & T_WATER) {
    std::ifstream in(path_in(dir, "gamma.dat"));
    if (!in) fail("File gamma.dat doesn't exist");
    for (int w = 0; w < p.n_wells; w++)
      for (int i = 0; i < 20; i++)
        for (int j = i; j < 20; j++) {
          double g0, g1;
          in >> g0 >> g1;
          if (!in) fail("Water potential gamma.dat file format error");
          g0 *= k_water;
          g1 *= k_water;
          for (int s = 0; s < 2; s++) {
            int a = s ? j : i, b = s ? i : j;
            T[TB_WATER + w * 800 + (a * 20 + b) * 2 + 0] = g0;
            T[TB_WATER + w * 800 + (a * 20 + b) * 2 + 1] = g1;
          }
        }
  }
  if (p.terms & T_PHOSPH) {
    // fix_backbone.cpp:643-670: pairs with a phosphorylated residue take the
    // serine (15) rows and columns from glutamate (6), scaled by the
    // hypercharge factor once (partner class 1) or twice (classes 2, 3), in the
    // reference's loop order
    static const int bb_class[20] = {1, 3, 2, 2, 4, 2, 2, 1, 3, 4, 4, 3, 4, 4, 1, 1, 1, 4, 4, 4};
    for (int w = 0; w < p.n_wells; w++) {
      double *P = &T[TB_WATER_PHOSPH + w * 800];
      std::copy(&T[TB_WATER + w * 800], &T[TB_WATER + w * 800] + 800, P);
      for (int i = 0; i < 20; i++) {
        const double fac = bb_class[i] == 1 ? p.k_hypercharge
                         : (bb_class[i] == 2 || bb_class[i] == 3) ? pow(p.k_hypercharge, 2) : 1.0;
        for (int c = 0; c < 2; c++) {
          const double g = bb_class[i] == 4 ? P[(i * 20 + 6) * 2 + c] : P[(i * 20 + 6) * 2 + c] * fac;
          P[(i * 20 + 15) * 2 + c] = P[(15 * 20 + i) * 2 + c] = g;
        }
      }
    }
  }
  if (p.terms & T_BURIAL) {
    if (!(p.terms & T_WATER)) fail("Cannot use burial without water potential");
    std::ifstream in(path_in(dir, "burial_gamma.dat"));
    if (!in) fail("File burial_gamma.dat doesn't exist");
    for (int i = 0; i < 60; i++) in >> T[TB_BURIAL + i];
    if (!in) fail("Burial potential burial_gamma.dat file format error");
  }
}

double GammaTable::get(int ti, int tj, int tfi, int tfj, int ires, int jres) const
{
  int d = std::abs(ires - jres);
  if (d < i_sep[0] || (i_sep[nseq_cl] != -1 && d > i_sep[nseq_cl])) return 0.0;
  int cl = 1;
  while (cl < nseq_cl && d >= i_sep[cl]) cl++;
  if (nres_cl == 1) return g[cl - 1];
  auto c = [&](int t) { return nres_cl == 4 ? residue_class4(t) - 1 : t; };
  size_t n2 = (size_t) nres_cl * nres_cl;
  if (!frag_resty) return g[(cl - 1) * n2 + c(ti) * nres_cl + c(tj)];
  return g[(cl - 1) * n2 * n2 + (c(ti) * nres_cl + c(tj)) * n2 + c(tfi) * nres_cl + c(tfj)];
}

void read_gamma_table(const std::string &path, GammaTable &G)
{
  FILE *f = fopen(path.c_str(), "r");
  if (!f) fail("Fragment_Memory: Cannot read gamma file");
  char line[512];
  std::vector<std::vector<std::string>> entries;
  bool header = true;
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    auto t = tokens(line);
    if (t.empty()) continue;
    if (header) {
      int ns = 0;
      for (auto &s : t) {
        if (ns >= 10) fail("Fragment_Memory: Wrong definition of sequance separation classes");
        G.i_sep[ns++] = s == "inf" ? -1 : atoi(s.c_str());
        if (s == "inf") break;
      }
      G.nseq_cl = ns - 1;
      if (G.nseq_cl <= 0) fail("Fragment_Memory: Wrong definition of sequance separation classes");
      header = false;
    } else {
      if (t.size() != 4 && t.size() != 6) fail("Fragment_Memory: Incorrect entery in gamma file");
      entries.push_back(t);
    }
  }
  fclose(f);
  if (entries.empty()) fail("Fragment_Memory: Incorrect entery in gamma file");
  G.frag_resty = entries[0].size() == 6;
  G.nres_cl = 0;
  for (auto &e : entries) {
    if ((e.size() == 6) != G.frag_resty) fail("Fragment_Memory: Incorrect entery in gamma file");
    for (size_t k = 0; k + 2 < e.size(); k++) {
      size_t L = e[k].size();
      if (e[k] == "ALL") G.nres_cl = std::max(G.nres_cl, 1);
      else if (L == 3) G.nres_cl = std::max(G.nres_cl, 4);
      else if (L == 1) G.nres_cl = std::max(G.nres_cl, 20);
      else fail("Fragment_Memory: Incorrect entery in gamma file");
    }
  }
  size_t n2 = (size_t) G.nres_cl * G.nres_cl;
  G.g.assign(G.nseq_cl * (G.frag_resty ? n2 * n2 : n2), 0.0);
  auto expand = [&](const std::string &s) {
    std::vector<int> v;
    if (s == "ALL") {
      for (int i = 0; i < G.nres_cl; i++) v.push_back(i);
    } else if (s.size() == 1) {
      if (G.nres_cl < 20) fail("Fragment_Memory: Cannot build gamma array");
      v.push_back(residue_code(s[0]));
    } else {
      int c = s == "SHL" ? 1 : s == "AHL" ? 2 : s == "BAS" ? 3 : s == "HPB" ? 4 : 0;
      if (!c) fail("Fragment_Memory: Incorrect entery in gamma file");
      if (G.nres_cl == 4) v.push_back(c - 1);
      else
        for (int i = 0; i < 20; i++)
          if (residue_class4(i) == c) v.push_back(i);
    }
    return v;
  };
  for (auto &e : entries) {
    if (!G.frag_resty) {
      int cl = atoi(e[2].c_str());
      if (cl > G.nseq_cl) fail("Fragment_Memory: Wrong sequance separation class tag");
      double gm = atof(e[3].c_str());
      for (int a : expand(e[0]))
        for (int b : expand(e[1])) {
          G.g[(cl - 1) * n2 + a * G.nres_cl + b] = gm;
          G.g[(cl - 1) * n2 + b * G.nres_cl + a] = gm;
        }
    } else {
      int cl = atoi(e[4].c_str());
      if (cl > G.nseq_cl) fail("Fragment_Memory: Cannot build gamma array");
      double gm = atof(e[5].c_str());
      // the reference hands the i-fragment class in for both fragment slots
      // (fragment_memory.cpp:369); kept as is
      auto fi = expand(e[2]);
      for (int a : expand(e[0]))
        for (int b : expand(e[1]))
          for (int c : fi)
            for (int d : fi) {
              size_t base = (cl - 1) * n2 * n2;
              G.g[base + (a * G.nres_cl + b) * n2 + c * G.nres_cl + d] = gm;
              G.g[base + (b * G.nres_cl + a) * n2 + c * G.nres_cl + d] = gm;
              G.g[base + (a * G.nres_cl + b) * n2 + d * G.nres_cl + c] = gm;
              G.g[base + (b * G.nres_cl + a) * n2 + d * G.nres_cl + c] = gm;
            }
    }
  }
}

// CA / CB coordinates (nm -> A) and residue names of residues fpos+1 ..
// fpos+len of a .gro file (Fragment_Memory::loadGro, fragment_memory.cpp:
// 34-176); m.len and m.pos are set by the caller.
static void load_gro(const std::string &path, int fpos, Memory &m, const std::string &open_msg,
                     const std::string &who)
{
  m.se.assign(m.len, '-');
  m.xca.assign((size_t) m.len * 3, 0.0);
  m.xcb.assign((size_t) m.len * 3, 0.0);
  FILE *g = fopen(path.c_str(), "r");
  if (!g) fail(open_msg);
  char title[256];
  int nat = 0, nca = 0;
  if (!fgets(title, sizeof title, g) || fscanf(g, "%d", &nat) != 1) {
    fclose(g);
    fail(who + ": Wrong atom count in memory structure file");
  }
  for (int a = 0; a < nat; a++) {
    int ires, iat;
    char rn[32], an[32];
    double x, y, z;
    if (fscanf(g, "%d %31s %31s %d %lf %lf %lf", &ires, rn, an, &iat, &x, &y, &z) != 7) break;
    if (ires > fpos + m.len) break;
    if (ires <= fpos) continue;
    int r = ires - fpos - 1;
    double *dst = nullptr;
    if (!strcmp(an, "CA")) {
      m.se[r] = residue_from_three(rn);
      if (m.se[r] == '?') {
        fclose(g);
        fail(who + ": Unknown residue");
      }
      dst = &m.xca[3 * r];
      nca++;
    } else if (!strcmp(an, "CB")) {
      dst = &m.xcb[3 * r];
    }
    if (dst) {
      dst[0] = x * 10;
      dst[1] = y * 10;
      dst[2] = z * 10;
    }
  }
  fclose(g);
  if (nca != m.len) fail(who + ": Wrong atom count in memory structure file");
}

void read_memories(const std::string &dir, const std::string &mem_file, int n_res, std::vector<Memory> &mems)
{
  FILE *f = fopen(path_in(dir, mem_file).c_str(), "r");
  if (!f) fail("Fragment_Memory: Error opening mem file");
  char buf[1024];
  enum { NONE, TARGET, MEMS } state = NONE;
  std::map<std::string, std::vector<std::string>> gro_cache;
  while (fgets(buf, sizeof buf, f)) {
    auto t = tokens(buf);
    if (!t.empty() && t[0][0] == '#') continue;
    if (!t.empty() && t[0][0] == '[') state = NONE;
    if (t.empty()) {
      state = NONE;
      continue;
    }
    if (state == MEMS) {
      if (t.size() != 5) fail("Fragment_Memory: Error reading mem file");
      Memory m;
      m.pos = atoi(t[1].c_str()) - 1;
      int fpos = atoi(t[2].c_str()) - 1;
      m.len = atoi(t[3].c_str());
      m.weight = atof(t[4].c_str());
      if (m.len <= 0) fail("Fragment_Memory: Incorrectly defined memory fragment");
      load_gro(path_in(dir, t[0]), fpos, m, "Fragment_Memory: Cannot read the file", "Fragment_Memory");
      if (m.pos + m.len > n_res) fail("read_mems: Fragment_Memory: Incorrectly defined memory fragment");
      mems.push_back(std::move(m));
    } else if (state == NONE) {
      if (t[0] == "[Target]") state = TARGET;
      else if (t[0] == "[Memories]") state = MEMS;
    }
  }
  fclose(f);
}

void build_topology(Topology &top, int n_atoms, const int *role, const int *residue, const int *molecule,
                    const int *type, const int *tag, const double *mass_by_type, int ntypes)
{
  int n = top.n_res;
  if (n <= 0) fail("sequence must be read before the topology");
  top.n_atoms = 3 * n;
  top.ntypes = ntypes;
  top.ext_of.assign(top.n_atoms, -1);
  top.atom_type.assign(top.n_atoms, 0);
  top.atom_tag.assign(top.n_atoms, 0);
  top.mass.assign(top.n_atoms, 0.0);
  top.res_chain.assign(n, -1);
  for (int a = 0; a < n_atoms; a++) {
    if (role[a] < 0) continue;
    int r = residue[a] - 1;
    if (r < 0 || r >= n) fail("Residue tag is out of range");
    if (residue[a] <= 0) fail("Molecular tag must be positive in fix backbone");
    int slot = 3 * r + role[a];
    if (top.ext_of[slot] != -1) fail("two atoms of the same role in one residue");
    top.ext_of[slot] = a;
    top.atom_type[slot] = type[a];
    top.atom_tag[slot] = tag ? tag[a] : a + 1;
    top.mass[slot] = mass_by_type[type[a]];
    int c = molecule[a] - 1;
    if (c < 0 || c >= top.n_chains) fail("Chain tag is out of range");
    if (top.res_chain[r] == -1) top.res_chain[r] = c;
    else if (top.res_chain[r] != c) fail("Atoms in a residue have different chain tag");
  }
  if (n_atoms != top.n_atoms) fail("every atom must be a CA, CB/H-beta or O of a residue");
  for (int slot = 0; slot < top.n_atoms; slot++)
    if (top.ext_of[slot] == -1) fail("Missing neighbor atoms in fix backbone (Code 001)");
  top.res_type.assign(n, 0);
  top.res_flags.assign(n, 0);
  for (int r = 0; r < n; r++) {
    int c = top.res_chain[r];
    if (r < top.chain_start[c] || r > top.chain_end[c]) fail("Residue tag is out of range");
    char s = top.seq[r];
    top.res_type[r] = residue_code(s);
    uint32_t fl = 0;
    if (s == 'G') fl |= R_GLY;
    if (s == 'P') fl |= R_PRO;
    if (r == top.chain_start[c]) fl |= R_FIRST;
    if (r == top.chain_end[c]) fl |= R_LAST;
    top.res_flags[r] = (int) fl;
  }
}

void set_bonds(Topology &top, int nb, const int *bi, const int *bj, const double *k, const double *r0,
               const int *ext_to_int)
{
  top.bond_i.clear();
  top.bond_j.clear();
  top.bond_k.clear();
  top.bond_r0.clear();
  top.excl_self.assign(top.n_res, 0u);
  top.excl_next.assign(top.n_res, 0u);
  for (int b = 0; b < nb; b++) {
    int a1 = ext_to_int[bi[b]], a2 = ext_to_int[bj[b]];
    top.bond_i.push_back(a1);
    top.bond_j.push_back(a2);
    top.bond_k.push_back(k[b]);
    top.bond_r0.push_back(r0[b]);
    int r1 = a1 / 3, r2 = a2 / 3, b1 = a1 % 3, b2 = a2 % 3;
    if (r1 == r2) {
      top.excl_self[r1] |= 1u << (b1 * 3 + b2);
      top.excl_self[r1] |= 1u << (b2 * 3 + b1);
    } else if (r2 == r1 + 1) {
      top.excl_next[r1] |= 1u << (b1 * 3 + b2);
    } else if (r1 == r2 + 1) {
      top.excl_next[r2] |= 1u << (b2 * 3 + b1);
    } else {
      fail("bonds must join beads of the same or adjacent residues");
    }
  }
}

void set_pair_coeffs(Topology &top, const std::string &style, const std::string &coeffs)
{
  auto s = tokens(style);
  if (s.size() != 3) fail("Illegal pair_style command");
  top.ev_p = atoi(s[0].c_str());
  double cs_glob = atof(s[1].c_str()), cl_glob = atof(s[2].c_str());
  int N = top.ntypes + 1;
  std::vector<double> lam(N * N, 0.0), cs(N * N, 0.0), cl(N * N, 0.0);
  std::vector<int> set(N * N, 0);
  std::stringstream ss(coeffs);
  std::string rec;
  auto bounds = [&](const std::string &t, int &lo, int &hi) {
    size_t st = t.find('*');
    if (st == std::string::npos) lo = hi = atoi(t.c_str());
    else {
      lo = st == 0 ? 1 : atoi(t.substr(0, st).c_str());
      hi = st + 1 == t.size() ? top.ntypes : atoi(t.substr(st + 1).c_str());
    }
    if (lo < 1 || hi > top.ntypes || lo > hi) fail("Numeric index is out of bounds");
  };
  while (std::getline(ss, rec, ';')) {
    auto c = tokens(rec);
    if (c.empty()) continue;
    if (c.size() != 3 && c.size() != 5) fail("Incorrect args for pair coefficients");
    int ilo, ihi, jlo, jhi;
    bounds(c[0], ilo, ihi);
    bounds(c[1], jlo, jhi);
    for (int i = ilo; i <= ihi; i++)
      for (int j = std::max(jlo, i); j <= jhi; j++) {
        lam[i * N + j] = atof(c[2].c_str());
        cs[i * N + j] = c.size() == 5 ? atof(c[3].c_str()) : cs_glob;
        cl[i * N + j] = c.size() == 5 ? atof(c[4].c_str()) : cl_glob;
        set[i * N + j] = 1;
      }
  }
  // init_one: geometric mixing for unset pairs, then symmetrise
  int sign = top.ev_p % 2 == 0 ? 1 : -1;
  top.ev_pref.assign(N * N, 0.0);
  top.ev_cs.assign(N * N, 0.0);
  top.ev_cl.assign(N * N, 0.0);
  for (int i = 1; i <= top.ntypes; i++)
    for (int j = i; j <= top.ntypes; j++) {
      if (!set[i * N + j]) {
        lam[i * N + j] = sqrt(lam[i * N + i] * lam[j * N + j]);
        cs[i * N + j] = sqrt(cs[i * N + i] * cs[j * N + j]);
        cl[i * N + j] = sqrt(cl[i * N + i] * cl[j * N + j]);
      }
      for (int s2 = 0; s2 < 2; s2++) {
        int a = s2 ? j : i, b = s2 ? i : j;
        top.ev_pref[a * N + b] = lam[i * N + j] * sign;
        top.ev_cs[a * N + b] = cs[i * N + j];
        top.ev_cl[a * N + b] = cl[i * N + j];
      }
    }
}

void build_fm_table(const ForceField &ff, const Topology &top, const GammaTable &G, const std::vector<Memory> &mems,
                    FMTable &out)
{
  const FFParams &p = ff.p;
  int n = top.n_res;
  int min_sep = G.min_sep(), max_sep = G.max_sep();
  int max_len = 0;
  for (auto &m : mems) max_len = std::max(max_len, m.len);
  int dmax = max_sep == -1 ? max_len - 1 : std::min(max_sep, max_len - 1);
  out.nd = std::max(dmax - min_sep + 1, 0);
  if (min_sep + out.nd > 64) fail("fragment memory: sequence separations above 63 are not supported");
  // memories listing residue i (fix_backbone.cpp:772-789), in memory order
  std::vector<std::vector<int>> listed(n);
  for (int k = 0; k < (int) mems.size(); k++)
    for (int i = mems[k].pos; i < mems[k].pos + mems[k].len - min_sep; i++) listed[i].push_back(k);
  struct Rec {
    double rf[4];
    double c;
  };
  std::vector<std::vector<Rec>> rows((size_t) n * std::max(out.nd, 1));
  auto dist = [](const double *a, const double *b) {
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
  };
  for (int i = 0; i < n; i++) {
    for (int k : listed[i]) {
      const Memory &m = mems[k];
      int je = m.pos + m.len - 1;
      if (max_sep != -1) je = std::min(je, i + max_sep);
      if (je >= n) fail("Missing residues in memory potential");
      double ekw = p.epsilon * p.k_fm * m.weight;
      for (int j = i + min_sep; j <= je; j++) {
        if (top.res_chain[i] != top.res_chain[j])
          fail("Fragment Memory: Interaction between residues of different chains");
        int d = j - i - min_sep;
        int li = i - m.pos, lj = j - m.pos;
        char mi = m.se[li], mj = m.se[lj];
        double gam = G.get(top.res_type[i], top.res_type[j], residue_code(mi), residue_code(mj), i, j);
        Rec rec;
        rec.c = ekw * gam;
        // atom pairs CA-CA, CA-CB, CB-CA, CB-CB (fix_backbone.cpp:4088-4096, fragment_memory.cpp:190-202)
        rec.rf[0] = dist(&m.xca[3 * li], &m.xca[3 * lj]);
        rec.rf[1] = dist(&m.xca[3 * li], &m.xcb[3 * lj]);
        rec.rf[2] = dist(&m.xca[3 * lj], &m.xcb[3 * li]);
        rec.rf[3] = dist(&m.xcb[3 * lj], &m.xcb[3 * li]);
        bool gi = top.seq[i] == 'G' || mi == 'G', gj = top.seq[j] == 'G' || mj == 'G';
        if (gj) rec.rf[1] = FMTable::FM_SKIP;
        if (gi) rec.rf[2] = FMTable::FM_SKIP;
        if (gi || gj) rec.rf[3] = FMTable::FM_SKIP;
        rows[(size_t) i * out.nd + d].push_back(rec);
      }
    }
  }
  out.row_start.assign((size_t) n * out.nd + 1, 0);
  long long tot = 0;
  for (size_t r = 0; r < rows.size() && out.nd > 0; r++) {
    out.row_start[r] = (int) tot;
    tot += (long long) rows[r].size();
  }
  if (tot > 0x7fffffffLL) fail("fragment memory table too large");
  out.row_start[(size_t) n * out.nd] = (int) tot;
  out.rf.resize((size_t) tot * 4);
  out.coef.resize((size_t) tot);
  out.uniform = true;
  bool have = false;
  size_t at = 0;
  for (auto &row : rows)
    for (auto &rec : row) {
      for (int k = 0; k < 4; k++) out.rf[4 * at + k] = rec.rf[k];
      out.coef[at] = rec.c;
      if (!have) {
        out.uniform_coef = rec.c;
        have = true;
      } else if (rec.c != out.uniform_coef) {
        out.uniform = false;
      }
      at++;
    }
  if (out.uniform) out.coef.clear();
}

static bool file_exists(const std::string &path)
{
  std::ifstream f(path);
  return (bool) f;
}

// FixBackbone::compute_fragment_memory_table (fix_backbone.cpp:4238-4322),
// read_fragment_memory_table (:4179-4236) and output_fragment_memory_table
// (:6062-6105), in the reference's loop order and FP64 arithmetic.
void build_fm_table_tb(const ForceField &ff, const Topology &top, const GammaTable &G,
                       const std::vector<Memory> &mems, const std::string &dir, FMTableTB &out)
{
  const FFParams &p = ff.p;
  const int n = top.n_res, min_sep = G.min_sep(), max_sep = G.max_sep();
  out.nbrs = max_sep != -1 ? max_sep - min_sep + 1 : n - min_sep;  // fix_backbone.cpp:999-1002
  out.size = p.tb_size;
  if (out.nbrs <= 0 || out.size < 2 || !(p.tb_dr > 0.0))
    fail("Fragment_Memory_Table: empty table (check rmin, rmax, dr and the gamma file's separations)");
  const size_t ntb = (size_t) n * out.nbrs * 4;
  const double bytes = (double) ntb * out.size * 16.0;
  if (bytes > 96e9)
    fail("Fragment_Memory_Table: the tables would take " + std::to_string(bytes / 1e9) +
         " GB; use a coarser dr or a gamma file with a maximum separation");
  out.data.assign(ntb * out.size * 2, 0.0);
  out.present.assign(ntb, 0);
  const std::string fe = path_in(dir, "fm_table.energy"), ff_ = path_in(dir, "fm_table.force");
  if (ff.tb_use_file && file_exists(fe) && file_exists(ff_)) {
    // tables listed itb-major, tb_size values each (energies, then forces)
    for (int pass = 0; pass < 2; pass++) {
      std::ifstream in(pass ? ff_ : fe);
      size_t ir = 0, itb = 0;
      double val;
      while (in >> val) {
        if (ir != 0 && ir % out.size == 0) {
          ir = 0;
          itb++;
        }
        if (itb >= ntb) fail("Fragment memory table file format error!");
        out.data[(itb * out.size + ir) * 2 + pass] = val;
        out.present[itb] = 1;
        ir++;
      }
      if (itb != ntb - 1 && ir != (size_t) out.size) fail("Fragment memory table file format error!");
    }
    return;
  }
  // memories listing residue i, in memory order (fix_backbone.cpp:772-789)
  std::vector<std::vector<int>> listed(n);
  for (int k = 0; k < (int) mems.size(); k++)
    for (int i = mems[k].pos; i < mems[k].pos + mems[k].len - min_sep; i++) listed[i].push_back(k);
  auto dist = [](const double *a, const double *b) {
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
  };
  const double w = ff.tb_width;
  for (int i = 0; i < n; i++)
    for (int km : listed[i]) {
      const Memory &m = mems[km];
      const double ekw = p.epsilon * p.k_fm * m.weight;
      const int js = i + min_sep;
      int je = m.pos + m.len - 1;
      if (max_sep != -1) je = std::min(je, i + max_sep);
      if (je >= n) fail("Missing residues in memory potential");
      for (int j = js; j <= je; j++) {
        double sig_sq = pow((double) abs(i - j), 2 * p.fm_sigma_exp);
        sig_sq = sig_sq * w * w;
        const int li = i - m.pos, lj = j - m.pos;
        const char mi = m.se[li], mj = m.se[lj];
        const double ekwg = ekw * G.get(top.res_type[i], top.res_type[j], residue_code(mi), residue_code(mj), i, j);
        // atom pairs CA-CA, CA-CB, CB-CA, CB-CB and their memory distances
        const double rf[4] = {dist(&m.xca[3 * li], &m.xca[3 * lj]), dist(&m.xca[3 * li], &m.xcb[3 * lj]),
                              dist(&m.xca[3 * lj], &m.xcb[3 * li]), dist(&m.xcb[3 * lj], &m.xcb[3 * li])};
        const bool gi = top.seq[i] == 'G' || mi == 'G', gj = top.seq[j] == 'G' || mj == 'G';
        for (int k = 0; k < 4; k++) {
          if (k >= 2 && gi) continue;
          if ((k & 1) && gj) continue;
          const size_t itb = ((size_t) i * out.nbrs + (j - js)) * 4 + k;
          out.present[itb] = 1;
          double *t = &out.data[itb * out.size * 2];
          for (int ir = 0; ir < out.size; ir++) {
            const double r = p.tb_rmin + ir * p.tb_dr;
            const double dr = r - rf[k];
            const double drsq = dr * dr;
            const double V = -ekwg * exp(-drsq / (2 * sig_sq));
            t[2 * ir] += V;
            t[2 * ir + 1] += V * dr / (sig_sq * r);
          }
        }
      }
    }
  if (ff.tb_use_file) {
    // saved for later runs; absent tables as zero rows, infinities as 0
    FILE *e = fopen(fe.c_str(), "w"), *f = fopen(ff_.c_str(), "w");
    if (!e || !f) fail("Fragment memory table files not found!");
    for (size_t itb = 0; itb < ntb; itb++) {
      for (int ir = 0; ir < out.size; ir++) {
        double ev = out.present[itb] ? out.data[(itb * out.size + ir) * 2] : 0.0;
        double fv = out.present[itb] ? out.data[(itb * out.size + ir) * 2 + 1] : 0.0;
        if (std::isinf(ev)) ev = 0.0;
        if (std::isinf(fv)) fv = 0.0;
        fprintf(e, "%.12f ", ev);
        fprintf(f, "%.12f ", fv);
      }
      fprintf(e, "\n");
      fprintf(f, "\n");
    }
    fclose(e);
    fclose(f);
  }
}

// compute_vector_fragment_memory_potential's pairs (fix_backbone.cpp:
// 3994-4077): for residue i, each memory covering it (the fragment-memory
// map, :765-790, memories in file order), partners j from i + min_sep to the
// memory's end (and i + max_sep), neither residue nor its memory residue a
// glycine; the memory's angle between the CA->CB vectors of i and j
// (Fragment_Memory::VM, fragment_memory.cpp:240-243)
void build_vfm(const Topology &top, const GammaTable &G, const std::vector<Memory> &mems, VfmRecords &out)
{
  const int n = top.n_res, min_sep = G.min_sep(), max_sep = G.max_sep();
  std::vector<std::vector<std::pair<int, double>>> per(n);
  for (const Memory &m : mems) {
    if (m.pos + m.len > n) fail("Fragment_Memory: Incorrectly defined memory fragment");
    auto vec = [&](int r, double *v) {
      for (int c = 0; c < 3; c++) v[c] = m.xcb[3 * r + c] - m.xca[3 * r + c];
    };
    for (int i = m.pos; i < m.pos + m.len - min_sep; i++) {
      int je = m.pos + m.len - 1;
      if (max_sep != -1) je = std::min(je, i + max_sep);
      for (int j = i + min_sep; j <= je; j++) {
        if (top.res_chain[i] != top.res_chain[j])
          fail("Fragment Memory: Interaction between residues of different chains");
        if (top.seq[i] == 'G' || top.seq[j] == 'G' || m.se[i - m.pos] == 'G' || m.se[j - m.pos] == 'G') continue;
        double u[3], v[3];
        vec(i - m.pos, u);
        vec(j - m.pos, v);
        const double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]), nv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        per[i].push_back({j, acos((u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) / (nu * nv))});
      }
    }
  }
  out = VfmRecords();
  out.start.assign(n + 1, 0);
  for (int i = 0; i < n; i++) {
    out.start[i + 1] = out.start[i] + (int) per[i].size();
    for (auto &e : per[i]) {
      out.j.push_back(e.first);
      out.angle.push_back(e.second);
    }
  }
}

// The constructors of compute qwolynes (compute_q_wolynes.cpp:50-110, file
// read :135-152) and compute qonuchic (compute_q_onuchic.cpp:27-85, contact
// arrays :124-186): argument counts, the native data and the normalisation.
// The group is the replica's CA atoms (n_res of them).
QDefinition parse_q_compute(const std::string &words, int n_res)
{
  auto w = tokens(words);
  QDefinition q;
  q.n = n_res;
  q.mat.assign((size_t) n_res * n_res, 0.0);
  if (w.size() >= 3 && w[2] == "qwolynes") {
    if (w.size() != 6) fail("Illegal compute qwolynes command");
    q.kind = 0;
    q.sep = atoi(w[4].c_str());
    q.sigma_exp = atof(w[5].c_str());
    std::ifstream in(w[3]);
    if (!in) fail("Native distance file can't be read");
    for (size_t k = 0; k < q.mat.size(); k++)
      if (!(in >> q.mat[k])) fail("compute qwolynes: the native distance file holds fewer than n x n values");
    q.qnorm = 2.0 / (((double) n_res - (double) q.sep) * ((double) n_res - ((double) q.sep + 1.0)));
    return q;
  }
  if (w.size() < 3 || w[2] != "qonuchic") fail("compute: only the qwolynes and qonuchic styles are supported");
  const int narg = (int) w.size();
  if (narg != 5 && narg != 6 && narg != 7) fail("Illegal compute qonuchic command");
  const std::string type = w[3];
  q.sigma_exp = 0.15;
  double count = 0.0;
  for (double &m : q.mat) m = -1.0;  // not native
  if (type == "cutoff" || type == "cutoff/gauss") {
    const bool hard = type == "cutoff";
    if (hard ? narg != 7 : narg != 6) fail("Illegal compute qonuchic command");
    q.kind = hard ? 1 : 2;
    const double r_contact = atof(w[4].c_str()), r_consq = r_contact * r_contact;
    const double factor = hard ? atof(w[6].c_str()) : 1.0;
    FILE *f = fopen(w[5].c_str(), "r");
    if (!f) fail("Compute qonuchic: can't read native coordinates");
    int na = 0;
    if (fscanf(f, "%d", &na) != 1) na = -1;
    std::vector<double> xn((size_t) 3 * std::max(na, 0));
    for (int i = 0; i < na; i++)
      if (fscanf(f, "%lf %lf %lf", &xn[3 * i], &xn[3 * i + 1], &xn[3 * i + 2]) != 3) na = -1;
    fclose(f);
    if (na != n_res) fail("Compute qonuchic: atom number mismatch");
    for (int i = 0; i < na; i++)
      for (int j = 0; j < na; j++) {
        const double dx = xn[3 * j] - xn[3 * i], dy = xn[3 * j + 1] - xn[3 * i + 1], dz = xn[3 * j + 2] - xn[3 * i + 2];
        double rsq = dx * dx + dy * dy + dz * dz;
        if (rsq < r_consq && j - i > 3) {
          count += 1.0;
          if (hard) rsq *= factor * factor;
          q.mat[(size_t) i * n_res + j] = rsq;
        }
      }
  } else if (type == "shadow" || type == "shadow/gauss") {
    const bool hard = type == "shadow";
    if (hard ? narg != 6 : narg != 5) fail("Illegal compute qonuchic command");
    q.kind = hard ? 1 : 2;
    const double factor = hard ? atof(w[5].c_str()) : 1.0;
    FILE *f = fopen(w[4].c_str(), "r");
    if (!f) fail("Compute qonuchic: can't read contact map file");
    int ires, jres;
    double rn;
    while (fscanf(f, "%d %d %lf", &ires, &jres, &rn) == 3) {
      ires--;
      jres--;
      if (ires >= n_res || jres >= n_res || ires < 0 || jres < 0 || abs(jres - ires) <= 3) {
        fclose(f);
        fail("Compute qonuchic: wrong residue index in shadow contact map file");
      }
      q.mat[(size_t) ires * n_res + jres] = hard ? rn * rn * (factor * factor) : rn * rn;
      count += 1.0;
    }
    fclose(f);
  } else {
    fail("Wrong type for compute qonuchic");
  }
  q.qnorm = 1 / count;
  return q;
}

// zim (fix_backbone.cpp:611-619): the membrane zone (1, 2 or 3) of each
// residue; the reference leaves the potential undefined for other values
void read_zim(const std::string &path, int n_res, std::vector<int> &z)
{
  std::ifstream in(path);
  if (!in) fail("File zim doesn't exist");
  z.assign(n_res, 0);
  for (int i = 0; i < n_res; i++) {
    in >> z[i];
    if (!in || in.eof()) fail("Membrane potential parameter file format error");
    if (z[i] < 1 || z[i] > 3) fail("Membrane: zim values must be 1, 2 or 3");
  }
}

// phosph_map (fix_backbone.cpp:671-681): residue numbers from 1; 0 entries are ignored
void flag_phosphorylated(const FFParams &p, Topology &top)
{
  for (int k = 0; k < p.n_phosph_res; k++) {
    const int r = p.phosph_res[k];
    if (r == 0) continue;
    if (r < 1 || r > top.n_res) fail("Phosphorylation: residue number out of range");
    top.res_flags[r - 1] |= R_PHOSPH;
  }
}

// charge_on_residues.dat (fix_backbone.cpp:1022-1045): a count, then that
// many (residue number, charge) records; residues not listed carry no charge
void read_charges(const std::string &path, int n_res, std::vector<double> &q)
{
  std::ifstream in(path);
  if (!in) fail("File charge_on_residues.dat doesn't exist");
  int count = 0;
  in >> count;
  q.assign(n_res, 0.0);
  for (int k = 0; k < count; k++) {
    int r;
    double c;
    if (!(in >> r >> c)) fail("DebyeHuckel: charge_on_residues.dat has fewer records than its count");
    if (r < 1 || r > n_res) fail("DebyeHuckel: residue number out of range in charge_on_residues.dat");
    q[r - 1] = c;
  }
}

// read_contact_restraints_file (fix_backbone.cpp:1106-1171): records
// "i1 i2 w r0" (residue numbers from 1), w scaled by the epsilon-scaled
// strength; the global cutoff r0_max + 4.29 sigma; per residue min(i1, i2) the
// restraints sorted by the other residue (a pair listed twice: the first record)
void read_contact_restraints(const std::string &path, FFParams &p, int n_res, ContactRestraints &out)
{
  std::ifstream in(path);
  if (!in) fail("File for Contact Restraints potential doesn't exist");
  struct Rec { int i, j, order; double w, r0; };
  std::vector<Rec> recs;
  int i1, i2;
  double w, r0, r0_max = 0.0;
  while (in >> i1 >> i2 >> w >> r0) {
    const int j1 = std::min(i1, i2) - 1, j2 = std::max(i1, i2) - 1;
    if (j1 < 0 || j1 >= n_res || j2 < 0 || j2 >= n_res) fail("Indices out of range in Contact Restraints potential file");
    recs.push_back({j1, j2, (int) recs.size(), w * p.k_cont_rest, r0});
    if (r0 > r0_max) r0_max = r0;
  }
  p.cr_dr_cut = p.cr_sigma * 4.29;
  p.cr_cut_sq = pow(r0_max + p.cr_dr_cut, 2);
  std::stable_sort(recs.begin(), recs.end(), [](const Rec &a, const Rec &b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });
  out = ContactRestraints();
  out.start.assign(n_res + 1, 0);
  for (const Rec &r : recs) {
    out.start[r.i + 1]++;
    out.j.push_back(r.j);
    out.w.push_back(r.w);
    out.r0.push_back(r.r0);
  }
  for (int k = 0; k < n_res; k++) out.start[k + 1] += out.start[k];
}

// FixBackbone::compute_amhgo_normalization (fix_backbone.cpp:3787-3848) and
// the contact selection of compute_amh_go_model (:3850-3992), with the
// native structure Fragment_Memory(0, 0, n, 1.0, "amh-go.gro") (:695-742).
void build_amh_go(const ForceField &ff, const Topology &top, const std::string &dir, AmhGoContacts &out)
{
  const FFParams &p = ff.p;
  const int n = top.n_res;
  GammaTable G;
  try {
    read_gamma_table(path_in(dir, "amh-go.gamma"), G);
  } catch (std::exception &e) {
    std::string m = e.what();
    fail(m.find("Cannot read") != std::string::npos ? std::string("Cannot read file amh-go.gamma")
                                                     : "AMH_Go" + m.substr(m.find(':')));
  }
  if (G.frag_resty) fail("AMH-Go: Wrong call of getGamma() function");
  Memory nat;
  nat.pos = 0;
  nat.len = n;
  load_gro(path_in(dir, "amh-go.gro"), 0, nat, "Cannot read file amh-go.gro", "AMH_Go");
  std::vector<uint8_t> censored;
  if (ff.amh_go_censor == 1) {
    censored.assign((size_t) n * n, 0);
    std::ifstream cf(path_in(dir, "frustration_censored_contacts.dat"));
    int a, b;
    while (cf >> a >> b)
      if (a >= 1 && a <= n && b >= 1 && b <= n) censored[(size_t) (a - 1) * n + (b - 1)] = 1;
  }
  // native distance of atom ia (0 CA, 1 CB) of residue i and atom ja of j
  // (Fragment_Memory::Rf: CA-CA, CB-CB, CA-CB distances of the structure)
  auto rnative = [&](int i, int ia, int j, int ja) {
    const double *a = ia ? &nat.xcb[3 * i] : &nat.xca[3 * i];
    const double *b = ja ? &nat.xcb[3 * j] : &nat.xca[3 * j];
    if (ia == ja && i > j) std::swap(a, b);
    if (ia != ja && ia == 1) std::swap(a, b);  // the CA-CB table is indexed (CA residue, CB residue)
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
  };
  const int min_sep = G.min_sep();
  // normalisation a = (1 / 8N) sum over atoms i of |sum over native contacts
  // of gamma|^p; the power is taken after each partner chain, of the running
  // sum (the reference's loop nesting), and N is the last chain's last residue
  double norm = 0.0;
  for (int i = 0; i < n; i++)
    for (int ia = 0; ia <= (top.seq[i] == 'G' ? 0 : 1); ia++) {
      double normi = 0.0;
      for (int jc = 0; jc < top.n_chains; jc++) {
        for (int j = top.chain_start[jc]; j <= top.chain_end[jc]; j++)
          for (int ja = 0; ja <= (top.seq[j] == 'G' ? 0 : 1); ja++) {
            if (abs(i - j) < min_sep) continue;
            if (rnative(i, ia, j, ja) < p.amh_go_rc) normi += G.get(top.res_type[i], top.res_type[j], 0, 0, i, j);
          }
        norm += pow(fabs(normi), p.amh_go_p);
      }
    }
  norm /= 8 * (top.chain_end.back() + 1);
  out.norm.assign(n, norm);
  // 1-2 bonded atom pairs: absent from the full neighbour list (special_bonds fene)
  std::set<std::pair<int, int>> bonded;
  for (size_t b = 0; b < top.bond_i.size(); b++)
    bonded.insert({std::min(top.bond_i[b], top.bond_j[b]), std::max(top.bond_i[b], top.bond_j[b])});
  // contacts of each CA / CB atom (the full list's partners, in atom order)
  out.start.assign((size_t) 2 * n + 1, 0);
  out.partner.clear();
  out.rnat.clear();
  out.gamma.clear();
  out.sig_sq.clear();
  for (int i = 0; i < n; i++)
    for (int ia = 0; ia < 2; ia++) {
      out.start[2 * i + ia] = (int) out.partner.size();
      if (ia == 1 && top.seq[i] == 'G') continue;
      for (int j = 0; j < n; j++)
        for (int ja = 0; ja < 2; ja++) {
          if ((ja == 1 && top.seq[j] == 'G') || (i == j && ia == ja)) continue;
          const bool other = top.res_chain[i] != top.res_chain[j];
          if (!(abs(i - j) >= min_sep || other)) continue;
          if (!censored.empty() && (censored[(size_t) i * n + j] || censored[(size_t) j * n + i])) continue;
          if (bonded.count({std::min(3 * i + ia, 3 * j + ja), std::max(3 * i + ia, 3 * j + ja)})) continue;
          const double rn = rnative(i, ia, j, ja);
          if (!(rn < p.amh_go_rc)) continue;
          out.partner.push_back(3 * j + ja);
          out.rnat.push_back(rn);
          out.gamma.push_back(G.get(top.res_type[i], top.res_type[j], 0, 0, i, j));
          out.sig_sq.push_back(pow(abs(i - j), 0.3));
        }
    }
  out.start[(size_t) 2 * n] = (int) out.partner.size();
}

void load_shared_forcefield(const std::string &dir, const std::string &coeff_file, const std::string &pair_style,
                            const std::string &pair_coeffs, SharedForceField &out)
{
  read_coeff_file(path_in(dir, coeff_file), out.ff);
  Topology none;  // ssweight is per replica: read the residue-independent tables only
  FFParams &p = out.ff.p;
  uint32_t ssw = p.terms & T_SSW;
  p.terms &= ~T_SSW;
  read_tables(dir, out.ff, none);
  p.terms |= ssw;
  if (p.terms & (T_FM | T_FM_TABLE)) {
    read_gamma_table(path_in(dir, out.ff.fm_gamma_file), out.gamma);
    p.fm_min_sep = out.gamma.min_sep();
    p.fm_max_sep = out.gamma.max_sep();
    for (int d = 0; d < 64; d++) p.fm_sigma_sq[d] = pow((double) d, 2 * p.fm_sigma_exp);
  }
  if ((p.terms & T_FM_TABLE) && p.fm_max_sep == -1)
    fail("Fragment_Memory_Table: replicas given as arrays need a gamma file with a maximum separation");
  out.pair_style = pair_style;
  out.pair_coeffs = pair_coeffs;
}

void load_system_arrays(const SharedForceField &sf, const ReplicaArrays &ra, SystemInput &S)
{
  if (sf.ff.p.terms & T_AMHGO) fail("AMH-Go needs a run directory (amh-go.gro, amh-go.gamma): load the replica from files");
  if (sf.ff.p.terms & T_DH) fail("DebyeHuckel needs a run directory (charge_on_residues.dat): load the replica from files");
  if (sf.ff.p.terms & T_MEMB) fail("Membrane needs a run directory (zim): load the replica from files");
  if (sf.ff.p.terms & T_CONTREST)
    fail("Contact_Restraints needs a run directory (the restraints file): load the replica from files");
  if (ra.n_res <= 0 || ra.n_chains <= 0 || !ra.chain_len || !ra.seq || !ra.x) fail("replica: empty description");
  S.ff = sf.ff;
  Topology &t = S.top;
  t.seq.assign(ra.seq, ra.seq + ra.n_res);
  int at = 0;
  for (int c = 0; c < ra.n_chains; c++) {
    if (ra.chain_len[c] <= 0) fail("replica: chain lengths must be positive");
    t.chain_start.push_back(at);
    at += ra.chain_len[c];
    t.chain_end.push_back(at - 1);
  }
  if (at != ra.n_res) fail("replica: chain lengths do not add up to n_res");
  t.n_chains = ra.n_chains;
  t.n_res = ra.n_res;
  // atoms in data-file order per residue: CA, O, CB/H-beta; ids 1..3n
  int na = 3 * ra.n_res;
  std::vector<int> role(na), res(na), mol(na), typ(na), tag(na);
  for (int r = 0, c = 0; r < ra.n_res; r++) {
    while (r > t.chain_end[c]) c++;
    const int roles[3] = {0, 2, 1};
    for (int k = 0; k < 3; k++) {
      int a = 3 * r + k;
      role[a] = roles[k];
      res[a] = r + 1;
      mol[a] = c + 1;
      typ[a] = k == 0 ? 1 : k == 1 ? 3 : (ra.seq[r] == 'G' ? 5 : 4);
      tag[a] = a + 1;
    }
  }
  build_topology(t, na, role.data(), res.data(), mol.data(), typ.data(), tag.data(), sf.mass, 5);
  // harmonic bonds of the AWSEM topology: CA-O, CA-CB/HB, CA-CA(+1), O-CA(+1)
  std::vector<int> bi, bj;
  std::vector<double> bk, br;
  auto add = [&](int i, int j, int type) {
    bi.push_back(i);
    bj.push_back(j);
    bk.push_back(sf.bond_k[type]);
    br.push_back(sf.bond_r0[type]);
  };
  for (int r = 0; r < ra.n_res; r++) {
    add(3 * r, 3 * r + 1, 2);
    add(3 * r, 3 * r + 2, ra.seq[r] == 'G' ? 5 : 4);
    if (!(t.res_flags[r] & R_LAST)) {
      add(3 * r, 3 * (r + 1), 1);
      add(3 * r + 1, 3 * (r + 1), 3);
    }
  }
  std::vector<int> ext_to_int(na);
  for (int s = 0; s < t.n_atoms; s++) ext_to_int[t.ext_of[s]] = s;
  set_bonds(t, (int) bi.size(), bi.data(), bj.data(), bk.data(), br.data(), ext_to_int.data());
  set_pair_coeffs(t, sf.pair_style, sf.pair_coeffs);
  // secondary-structure weights of the enabled [SSWeight] columns, in order
  t.aps.assign((size_t) 12 * ra.n_res, 0.0);
  if ((S.ff.p.terms & T_SSW) && ra.ssweight) {
    int ncol = 0;
    for (int k = 0; k < 12; k++) ncol += S.ff.p.ssweight[k] ? 1 : 0;
    for (int r = 0; r < ra.n_res; r++)
      for (int k = 0, c = 0; k < 12; k++)
        if (S.ff.p.ssweight[k]) t.aps[(size_t) k * ra.n_res + r] = ra.ssweight[(size_t) r * ncol + c++];
  }
  // fragment memories
  if (S.ff.p.terms & (T_FM | T_FM_TABLE)) {
    S.gamma = sf.gamma;
    size_t off = 0;
    for (int m = 0; m < ra.n_mem; m++) {
      Memory mm;
      mm.pos = ra.mem_pos[m];
      mm.len = ra.mem_len[m];
      mm.weight = ra.mem_weight[m];
      if (mm.len <= 0 || mm.pos < 0 || mm.pos + mm.len > ra.n_res)
        fail("Fragment_Memory: Incorrectly defined memory fragment");
      mm.se.assign(ra.mem_seq + off, ra.mem_seq + off + mm.len);
      mm.xca.assign(ra.mem_ca + 3 * off, ra.mem_ca + 3 * (off + mm.len));
      mm.xcb.assign(ra.mem_cb + 3 * off, ra.mem_cb + 3 * (off + mm.len));
      off += mm.len;
      S.mems.push_back(std::move(mm));
    }
    if (S.ff.p.terms & T_FM) {
      build_fm_table(S.ff, t, S.gamma, S.mems, S.fm);
      S.ff.p.fm_nd = S.fm.nd;
    }
    if (S.ff.p.terms & T_FM_TABLE) {
      build_fm_table_tb(S.ff, t, S.gamma, S.mems, "", S.tb);
      S.ff.p.tb_nbrs = S.tb.nbrs;
    }
    if (S.ff.p.terms & T_VFM) build_vfm(t, S.gamma, S.mems, S.vfm);
    S.mems.clear();
    S.mems.shrink_to_fit();
  }
  if (S.ff.p.terms & T_PHOSPH) flag_phosphorylated(S.ff.p, t);
  S.x.assign(3 * t.n_atoms, 0.0);
  S.v.assign(3 * t.n_atoms, 0.0);
  for (int s = 0; s < t.n_atoms; s++)
    for (int k = 0; k < 3; k++) {
      S.x[3 * s + k] = ra.x[3 * t.ext_of[s] + k];
      if (ra.v) S.v[3 * s + k] = ra.v[3 * t.ext_of[s] + k];
    }
}

void assemble_batch(const std::vector<const SystemInput *> &reps, Batch &B)
{
  if (reps.empty()) fail("empty batch");
  const SystemInput &r0 = *reps[0];
  B = Batch();
  B.ff = r0.ff;
  B.n_sys = (int) reps.size();
  Topology &T = B.top;
  T.ntypes = r0.top.ntypes;
  T.ev_p = r0.top.ev_p;
  T.ev_pref = r0.top.ev_pref;
  T.ev_cs = r0.top.ev_cs;
  T.ev_cl = r0.top.ev_cl;
  int nd = 0;
  long long nres = 0, nrec = 0;
  auto same_ff = [](const FFParams &a, const FFParams &b) {
    FFParams x = a, y = b;  // rows per residue may differ; everything else must match
    x.fm_nd = y.fm_nd = 0;
    x.tb_nbrs = y.tb_nbrs = 0;
    return memcmp(&x, &y, sizeof x) == 0;
  };
  for (auto *r : reps) {
    if (!same_ff(r->ff.p, r0.ff.p) || r->ff.tables != r0.ff.tables)
      fail("batch replicas must share one force field (coefficient file and tables)");
    if (r->top.ntypes != T.ntypes || r->top.ev_p != T.ev_p || r->top.ev_pref != T.ev_pref ||
        r->top.ev_cs != T.ev_cs || r->top.ev_cl != T.ev_cl)
      fail("batch replicas must share one pair_style vexcluded setup");
    nd = std::max(nd, r->fm.nd);
    nres += r->top.n_res;
    nrec += r->fm.records();
  }
  if (nres > 0x3fffffff || nrec > 0x7fffffffLL) fail("batch too large");
  int N = (int) nres;
  T.n_res = N;
  T.n_atoms = 3 * N;
  T.aps.assign((size_t) 12 * N, 0.0);
  B.fm.nd = nd;
  B.fm.row_start.assign((size_t) N * nd + 1, 0);
  bool uniform = true;
  double ucoef = 0.0;
  bool have = false;
  for (auto *r : reps)
    if (r->fm.records() > 0) {
      if (!r->fm.uniform) uniform = false;
      else if (!have) {
        ucoef = r->fm.uniform_coef;
        have = true;
      } else if (r->fm.uniform_coef != ucoef) uniform = false;
    }
  B.fm.uniform = uniform;
  B.fm.uniform_coef = ucoef;
  B.sys_atom_begin.push_back(0);
  int roff = 0, coff = 0;
  long long rec_off = 0;
  for (int k = 0; k < B.n_sys; k++) {
    const SystemInput &S = *reps[k];
    const Topology &t = S.top;
    int n = t.n_res;
    B.sys_res_begin.push_back(roff);
    B.sys_res_end.push_back(roff + n);
    B.sys_atom_begin.push_back(3 * (roff + n));
    B.ext_of.push_back(t.ext_of);
    T.seq += t.seq;
    for (int i = 0; i < n; i++) {
      T.res_type.push_back(t.res_type[i]);
      T.res_flags.push_back(t.res_flags[i]);
      T.res_chain.push_back(t.res_chain[i] + coff);
      B.res_sys.push_back(k);
      T.excl_self.push_back(t.excl_self[i]);
      T.excl_next.push_back(t.excl_next[i]);
      for (int q = 0; q < 12; q++) T.aps[(size_t) q * N + roff + i] = t.aps[(size_t) q * n + i];
    }
    for (int c = 0; c < t.n_chains; c++) {
      T.chain_start.push_back(t.chain_start[c] + roff);
      T.chain_end.push_back(t.chain_end[c] + roff);
    }
    for (int a = 0; a < t.n_atoms; a++) {
      T.atom_type.push_back(t.atom_type[a]);
      T.atom_tag.push_back(t.atom_tag[a]);
      T.mass.push_back(t.mass[a]);
    }
    for (size_t b = 0; b < t.bond_i.size(); b++) {
      T.bond_i.push_back(t.bond_i[b] + 3 * roff);
      T.bond_j.push_back(t.bond_j[b] + 3 * roff);
      T.bond_k.push_back(t.bond_k[b]);
      T.bond_r0.push_back(t.bond_r0[b]);
    }
    B.x.insert(B.x.end(), S.x.begin(), S.x.end());
    B.v.insert(B.v.end(), S.v.begin(), S.v.end());
    // fragment-memory rows, re-laid to the batch's rows per residue
    const FMTable &f = S.fm;
    for (int i = 0; i < n; i++)
      for (int d = 0; d < nd; d++) {
        size_t dst = (size_t) (roff + i) * nd + d;
        long long cnt = 0, src0 = 0;
        if (d < f.nd && f.records() > 0) {
          src0 = f.row_start[(size_t) i * f.nd + d];
          cnt = f.row_start[(size_t) i * f.nd + d + 1] - src0;
        }
        B.fm.row_start[dst] = (int) rec_off;
        for (long long q = 0; q < cnt; q++) {
          for (int c = 0; c < 4; c++) B.fm.rf.push_back(f.rf[(size_t) (src0 + q) * 4 + c]);
          if (!uniform) B.fm.coef.push_back(f.uniform ? f.uniform_coef : f.coef[src0 + q]);
        }
        rec_off += cnt;
      }
    roff += n;
    coff += t.n_chains;
  }
  B.fm.row_start[(size_t) N * nd] = (int) rec_off;
  if (B.ff.p.terms & T_AMHGO) {
    B.go.start.push_back(0);
    int res_off = 0;
    for (auto *r : reps) {
      const AmhGoContacts &g = r->go;
      const int base = (int) B.go.partner.size();
      for (size_t k = 1; k < g.start.size(); k++) B.go.start.push_back(base + g.start[k]);
      for (int q : g.partner) B.go.partner.push_back(q + 3 * res_off);
      B.go.rnat.insert(B.go.rnat.end(), g.rnat.begin(), g.rnat.end());
      B.go.gamma.insert(B.go.gamma.end(), g.gamma.begin(), g.gamma.end());
      B.go.sig_sq.insert(B.go.sig_sq.end(), g.sig_sq.begin(), g.sig_sq.end());
      B.go.norm.insert(B.go.norm.end(), g.norm.begin(), g.norm.end());
      res_off += r->top.n_res;
    }
  }
  if (B.ff.p.terms & T_DH)
    for (auto *r : reps) B.charge.insert(B.charge.end(), r->charge.begin(), r->charge.end());
  if (B.ff.p.terms & T_MEMB)
    for (auto *r : reps) B.zim.insert(B.zim.end(), r->zim.begin(), r->zim.end());
  if (B.ff.p.terms & T_VFM) {
    B.vfm.start.push_back(0);
    int res_off = 0;
    for (auto *r : reps) {
      const int base = (int) B.vfm.j.size();
      for (size_t k = 1; k < r->vfm.start.size(); k++) B.vfm.start.push_back(base + r->vfm.start[k]);
      for (int q : r->vfm.j) B.vfm.j.push_back(q + res_off);
      B.vfm.angle.insert(B.vfm.angle.end(), r->vfm.angle.begin(), r->vfm.angle.end());
      res_off += r->top.n_res;
    }
  }
  if (B.ff.p.terms & T_CONTREST) {
    B.cr.start.push_back(0);
    int res_off = 0;
    for (auto *r : reps) {
      const int base = (int) B.cr.j.size();
      for (size_t k = 1; k < r->cr.start.size(); k++) B.cr.start.push_back(base + r->cr.start[k]);
      for (int q : r->cr.j) B.cr.j.push_back(q + res_off);
      B.cr.w.insert(B.cr.w.end(), r->cr.w.begin(), r->cr.w.end());
      B.cr.r0.insert(B.cr.r0.end(), r->cr.r0.begin(), r->cr.r0.end());
      res_off += r->top.n_res;
    }
  }
  if (B.ff.p.terms & T_FM_TABLE) {
    B.tb.nbrs = r0.tb.nbrs;
    B.tb.size = r0.tb.size;
    for (auto *r : reps) {
      if (r->tb.nbrs != B.tb.nbrs || r->tb.size != B.tb.size)
        fail("batch replicas must share one fragment-memory table shape (a gamma file with a maximum separation)");
      B.tb.data.insert(B.tb.data.end(), r->tb.data.begin(), r->tb.data.end());
      B.tb.present.insert(B.tb.present.end(), r->tb.present.begin(), r->tb.present.end());
    }
  }
  T.n_chains = coff;
  B.ff.p.fm_nd = nd;
  if (!(B.ff.p.terms & T_FM)) B.ff.p.fm_nd = 0;
}

void load_system_dir(const std::string &dir, const std::string &data_file, const std::string &coeff_file,
                     const std::string &seq_file, const std::string &pair_style, const std::string &pair_coeffs,
                     SystemInput &S)
{
  read_coeff_file(path_in(dir, coeff_file), S.ff);
  read_sequence(path_in(dir, seq_file), S.top);
  // LAMMPS data file, atom_style awsemmd
  std::ifstream in(path_in(dir, data_file));
  if (!in) fail("cannot open data file " + data_file);
  std::string line;
  std::getline(in, line);
  int natoms = 0, ntypes = 0, nbt = 0;
  std::map<std::string, std::vector<std::string>> sec;
  std::string cur;
  while (std::getline(in, line)) {
    size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    auto t = tokens(line);
    if (t.empty()) continue;
    if (cur.empty()) {
      if (t.size() >= 2 && t[1] == "atoms") { natoms = atoi(t[0].c_str()); continue; }
      if (t.size() >= 3 && t[1] == "atom" && t[2] == "types") { ntypes = atoi(t[0].c_str()); continue; }
      if (t.size() >= 3 && t[1] == "bond" && t[2] == "types") { nbt = atoi(t[0].c_str()); continue; }
      if (t.size() >= 2 && (t[1] == "bonds" || t[1] == "angles" || t[1] == "dihedrals" || t[1] == "impropers")) continue;
      if (t.size() >= 3 && (t[2] == "types" || t[2] == "xlo" || t[2] == "ylo" || t[2] == "zlo")) continue;
    }
    if (t[0] == "Masses" || t[0] == "Atoms" || t[0] == "Velocities" || t[0] == "Bonds") {
      cur = t[0];
      continue;
    }
    if (t[0] == "Bond" && t.size() > 1 && t[1] == "Coeffs") {
      cur = "Bond Coeffs";
      continue;
    }
    if (cur.empty()) fail("data file: unexpected line: " + line);
    sec[cur].push_back(line);
  }
  std::vector<double> mass(ntypes + 1, 0.0);
  for (auto &l : sec["Masses"]) {
    auto t = tokens(l);
    mass.at(atoi(t[0].c_str())) = atof(t[1].c_str());
  }
  if ((int) sec["Atoms"].size() != natoms) fail("data file: Atoms section incomplete");
  std::vector<std::pair<int, std::vector<std::string>>> rows;
  for (auto &l : sec["Atoms"]) {
    auto t = tokens(l);
    if (t.size() < 8) fail("data file: Atoms line needs id molecule residue type q x y z");
    rows.push_back({atoi(t[0].c_str()), t});
  }
  std::sort(rows.begin(), rows.end(), [](auto &a, auto &b) { return a.first < b.first; });
  std::vector<int> role(natoms), res(natoms), mol(natoms), typ(natoms), tag(natoms);
  std::vector<double> xe(3 * natoms), ve(3 * natoms, 0.0);
  std::map<int, int> tag_to_ext;
  for (int a = 0; a < natoms; a++) {
    auto &t = rows[a].second;
    tag[a] = atoi(t[0].c_str());
    mol[a] = atoi(t[1].c_str());
    res[a] = atoi(t[2].c_str());
    typ[a] = atoi(t[3].c_str());
    for (int k = 0; k < 3; k++) xe[3 * a + k] = atof(t[5 + k].c_str());
    // awsemmd type convention: 1 CA, 3 O, 4 CB, 5 H-beta
    role[a] = typ[a] == 1 ? 0 : (typ[a] == 4 || typ[a] == 5) ? 1 : typ[a] == 3 ? 2 : -1;
    tag_to_ext[tag[a]] = a;
  }
  for (auto &l : sec["Velocities"]) {
    auto t = tokens(l);
    int a = tag_to_ext.at(atoi(t[0].c_str()));
    for (int k = 0; k < 3; k++) ve[3 * a + k] = atof(t[1 + k].c_str());
  }
  std::vector<double> bk(nbt + 1, 0.0), br(nbt + 1, 0.0);
  for (auto &l : sec["Bond Coeffs"]) {
    auto t = tokens(l);
    bk.at(atoi(t[0].c_str())) = atof(t[1].c_str());
    br.at(atoi(t[0].c_str())) = atof(t[2].c_str());
  }
  std::vector<int> bi, bj;
  std::vector<double> kk, rr;
  for (auto &l : sec["Bonds"]) {
    auto t = tokens(l);
    int bt = atoi(t[1].c_str());
    bi.push_back(tag_to_ext.at(atoi(t[2].c_str())));
    bj.push_back(tag_to_ext.at(atoi(t[3].c_str())));
    kk.push_back(bk.at(bt));
    rr.push_back(br.at(bt));
  }
  load_system_atoms(dir, coeff_file, seq_file, natoms, role.data(), res.data(), mol.data(), typ.data(), tag.data(),
                    mass.data(), ntypes, xe.data(), ve.data(), (int) bi.size(), bi.data(), bj.data(), kk.data(),
                    rr.data(), pair_style, pair_coeffs, S, false);
}

void load_system_atoms(const std::string &dir, const std::string &coeff_file, const std::string &seq_file,
                       int natoms, const int *role, const int *res, const int *mol, const int *typ, const int *tag,
                       const double *mass, int ntypes, const double *xe, const double *ve, int nbonds,
                       const int *bond_a, const int *bond_b, const double *bond_k, const double *bond_r0,
                       const std::string &pair_style, const std::string &pair_coeffs, SystemInput &S,
                       bool read_files)
{
  if (read_files && coeff_file.empty() && seq_file.empty()) {
    // pair vexcluded (and bonds) only: no fix backbone terms, so no
    // coefficient or sequence file; residues 1..max id, chains as runs of
    // equal molecule id along the residues, every residue read as alanine
    // (residue kinds matter to fix backbone terms only)
    S.ff.p.terms = 0;
    int n = 0;
    for (int a = 0; a < natoms; a++) n = std::max(n, res[a]);
    if (n <= 0) fail("Residue tag is out of range");
    std::vector<int> mol_of(n, -1);
    for (int a = 0; a < natoms; a++)
      if (role[a] >= 0 && res[a] >= 1) mol_of[res[a] - 1] = mol[a];
    S.top.seq.assign(n, 'A');
    S.top.chain_start.clear();
    S.top.chain_end.clear();
    for (int r = 0; r < n; r++) {
      if (r == 0 || mol_of[r] != mol_of[r - 1]) S.top.chain_start.push_back(r);
      if (r == n - 1 || mol_of[r + 1] != mol_of[r]) S.top.chain_end.push_back(r);
    }
    S.top.n_chains = (int) S.top.chain_start.size();
    S.top.n_res = n;
  } else if (read_files) {
    read_coeff_file(path_in(dir, coeff_file), S.ff);
    read_sequence(path_in(dir, seq_file), S.top);
  }
  build_topology(S.top, natoms, role, res, mol, typ, tag, mass, ntypes);
  std::vector<int> ext_to_int(natoms);
  for (int s = 0; s < S.top.n_atoms; s++) ext_to_int[S.top.ext_of[s]] = s;
  set_bonds(S.top, nbonds, bond_a, bond_b, bond_k, bond_r0, ext_to_int.data());
  set_pair_coeffs(S.top, pair_style, pair_coeffs);
  read_tables(dir, S.ff, S.top);
  if (S.ff.p.terms & (T_FM | T_FM_TABLE)) {
    read_gamma_table(path_in(dir, S.ff.fm_gamma_file), S.gamma);
    const bool tb_from_file = (S.ff.p.terms & T_FM_TABLE) && S.ff.tb_use_file && !(S.ff.p.terms & T_FM) &&
                              file_exists(path_in(dir, "fm_table.energy")) &&
                              file_exists(path_in(dir, "fm_table.force"));
    // the reference reads the memories unless the tables come from files (fix_backbone.cpp:758)
    if (!tb_from_file) read_memories(dir, S.ff.fm_file, S.top.n_res, S.mems);
    S.ff.p.fm_min_sep = S.gamma.min_sep();
    S.ff.p.fm_max_sep = S.gamma.max_sep();
    for (int d = 0; d < 64; d++) S.ff.p.fm_sigma_sq[d] = pow((double) d, 2 * S.ff.p.fm_sigma_exp);
    if (S.ff.p.terms & T_FM) {
      build_fm_table(S.ff, S.top, S.gamma, S.mems, S.fm);
      S.ff.p.fm_nd = S.fm.nd;
    }
    if (S.ff.p.terms & T_FM_TABLE) {
      build_fm_table_tb(S.ff, S.top, S.gamma, S.mems, dir, S.tb);
      S.ff.p.tb_nbrs = S.tb.nbrs;
    }
    if (S.ff.p.terms & T_VFM) {
      if (tb_from_file) fail("Vector_Fragment_Memory needs the memories (the fragment-memory tables came from files)");
      build_vfm(S.top, S.gamma, S.mems, S.vfm);
    }
  }
  if ((S.ff.p.terms & T_VFM) && !(S.ff.p.terms & (T_FM | T_FM_TABLE)))
    fail("Vector_Fragment_Memory needs the memories of [Fragment_Memory] or [Fragment_Memory_Table]");
  if (S.ff.p.terms & T_DH) read_charges(path_in(dir, "charge_on_residues.dat"), S.top.n_res, S.charge);
  if (S.ff.p.terms & T_MEMB) read_zim(path_in(dir, "zim"), S.top.n_res, S.zim);
  if (S.ff.p.terms & T_PHOSPH) flag_phosphorylated(S.ff.p, S.top);
  if (S.ff.p.terms & T_CONTREST) {
    read_contact_restraints(path_in(dir, S.ff.cr_file), S.ff.p, S.top.n_res, S.cr);
    S.ff.p.pair_list_cutoff = pair_list_cutoff(S.ff.p);  // the restraints set their cutoff
  }
  if (S.ff.p.terms & T_AMHGO) build_amh_go(S.ff, S.top, dir, S.go);
  S.x.assign(3 * S.top.n_atoms, 0.0);
  S.v.assign(3 * S.top.n_atoms, 0.0);
  for (int s = 0; s < S.top.n_atoms; s++)
    for (int k = 0; k < 3; k++) {
      if (xe) S.x[3 * s + k] = xe[3 * S.top.ext_of[s] + k];
      if (ve) S.v[3 * s + k] = ve[3 * S.top.ext_of[s] + k];
    }
}

}  // namespace awsem
