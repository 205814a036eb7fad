/* LAMMPS-API shim: the awsemmd atom style as the reference plugins see it.
   The per-atom `molecule` and `residue` fields live in Atom (lmp_shim.h);
   data-file parsing of the `id molecule residue type q x y z` line is done by
   the shim host, so the class carries no behaviour here. */
#ifndef AWSEM_ORACLE_ATOM_VEC_AWSEMMD_H
#define AWSEM_ORACLE_ATOM_VEC_AWSEMMD_H
#include "lmp_shim.h"
namespace LAMMPS_NS {
class AtomVecAWSEM : public AtomVec {
 public:
  AtomVecAWSEM() { style = "awsemmd"; }
};
}
#endif
