/* fix backbone/gpu: the fix backbone force path (FixBackbone::pre_force,
   src/fix_backbone.cpp:8181-8203) evaluated by libawsem_gpu.so.

   A LAMMPS style class a maintainer adds beside fix_backbone.h; it keeps the
   reference argument list so that an input script only renames the style:

     fix ID CA-group backbone/gpu CB-group O-group coeff-file seq-file [fp64|mixed] [device N]

   Like the reference fix it adds its forces to atom->f during pre_force and
   reports the 18-term energy vector through compute_scalar / compute_vector
   (scalar = total, vector(i) = term i + 1).  The whole system lives on one
   GPU: the fix runs on one MPI rank holding every atom (no ghost atoms are
   used; coordinates are unwrapped with the image flags as the reference
   does, src/fix_backbone.cpp:7067-7138). */
#ifdef FIX_CLASS
// clang-format off
FixStyle(backbone/gpu,FixBackboneGPU);
// clang-format on
#else

#ifndef LMP_FIX_BACKBONE_GPU_H
#define LMP_FIX_BACKBONE_GPU_H

#include <string>
#include <vector>

#include "awsem_gpu.h"
#include "fix.h"

namespace LAMMPS_NS {

class FixBackboneGPU : public Fix {
 public:
  FixBackboneGPU(class LAMMPS *, int, char **);
  ~FixBackboneGPU() override;
  int setmask() override;
  void init() override;
  void setup(int) override;
  void min_setup(int) override;
  void setup_pre_force(int) override;
  void pre_force(int) override;
  void pre_force_respa(int, int, int) override;
  void min_pre_force(int) override;
  double compute_scalar() override;
  double compute_vector(int) override;

 private:
  std::string coeff_file, seq_file;
  int cb_bit = 0, o_bit = 0, precision = AWSEM_FP64, device = 0;
  awsem_system *handle = nullptr;
  bigint evaluated_step = -1;
  double energy[21] = {0};
  std::vector<double> xg, fg;  // [natoms][3] in tag order

  void create_handle();
  void evaluate();
};

}  // namespace LAMMPS_NS

#endif
#endif
