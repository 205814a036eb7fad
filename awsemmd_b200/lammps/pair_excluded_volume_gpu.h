/* pair_style vexcluded/gpu: PairExcludedVolume (src/pair_excluded_volume.h:12,
   src/pair_excluded_volume.cpp:50-370) evaluated by libawsem_gpu.so.

   A LAMMPS style class a maintainer adds beside pair_excluded_volume.h
   (registered as vexcluded/gpu and as excluded_volume/gpu).  The input
   script keeps the reference commands and only renames the style:

     pair_style vexcluded/gpu p cut_short cut_long [fp64|mixed] [device N] [groups CA-group CB-group O-group]
     pair_coeff i j lambda [cut_short cut_long]

   settings, coeff and init_one (geometric mixing of lambda and of both
   cutoffs) are the reference's; compute adds lambda (r - r_c)^p forces
   (r_c = cut_short for two atoms of one molecule less than 5 residues apart,
   cut_long otherwise) into atom->f and reports the energy in eng_vdwl.  The
   pairs are the GPU's own (every atom pair within its cutoff), with the 1-2
   bonded pairs left out as `special_bonds fene` leaves them out of LAMMPS's
   list; the other special weights must be 1.  Roles of the atoms (CA,
   CB or H-beta, O; residues of three beads) come from the three groups,
   alpha_carbons beta_atoms oxygens unless named.  The whole system lives on
   one GPU: every atom on one MPI rank; positions are unwrapped with the
   image flags.  Per-atom energy and virial tallies are not supported; the
   global virial comes from f . r (LAMMPS's fdotr). */
#ifdef PAIR_CLASS
// clang-format off
PairStyle(vexcluded/gpu,PairExcludedVolumeGPU);
PairStyle(excluded_volume/gpu,PairExcludedVolumeGPU);
// clang-format on
#else

#ifndef LMP_PAIR_EXCLUDED_VOLUME_GPU_H
#define LMP_PAIR_EXCLUDED_VOLUME_GPU_H

#include <string>
#include <vector>

#include "awsem_gpu.h"
#include "pair.h"

namespace LAMMPS_NS {

class PairExcludedVolumeGPU : public Pair {
 public:
  PairExcludedVolumeGPU(class LAMMPS *);
  ~PairExcludedVolumeGPU() override;
  void compute(int, int) override;
  void settings(int, char **) override;
  void coeff(int, char **) override;
  void init_style() override;
  double init_one(int, int) override;

 private:
  int p = 2;
  double cut_global[2] = {0.0, 0.0};
  double **lambda = nullptr, **cut_short = nullptr, **cut_long = nullptr;
  int precision = AWSEM_FP64, device = 0;
  std::string groups[3] = {"alpha_carbons", "beta_atoms", "oxygens"};
  awsem_system *handle = nullptr;
  std::string handle_coeffs;   // the coefficients the handle was built with
  std::vector<double> xg, fg;  // [natoms][3] in tag order

  void allocate();
  std::string coeff_text() const;
  void create_handle();
};

}  // namespace LAMMPS_NS

#endif
#endif
