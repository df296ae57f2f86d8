// md_simulator b200 / b200_fp64 -- the reference's Md_simulator with its
// run() done by the B200 path through the C ABI (include/caviar_b200.h).
//
// This header belongs to the integration layer a maintainer adds to the
// reference (CAVIAR) tree; it is compiled against the reference's own
// headers.  The object keeps every keyword of `md_simulator basic`
// (Md_simulator::read, src/caviar/objects/md_simulator.cpp:58-233); only
// run() (md_simulator.cpp:235-274) is replaced: the whole run of velocity-
// Verlet steps, with the neighbour list, LJ, Ewald real-space and k-space
// forces of the simulator's objects, goes to one GPU context, and the final
// owned positions, velocities and accelerations come back into Atom_data.
#ifndef CAVIAR_OBJECTS_MDSIMULATOR_B200_H
#define CAVIAR_OBJECTS_MDSIMULATOR_B200_H

#include "caviar/objects/md_simulator.h"

CAVIAR_NAMESPACE_OPEN

namespace md_simulator
{

  // Mixed precision (CVR_PREC_MIXED): FP32 pair and k-space arithmetic, FP64
  // positions, velocities, S(k) and energy/virial sums.
  class B200 : public Md_simulator
  {
  public:
    B200(class CAVIAR *);
    ~B200();
    bool run() override;

  protected:
    B200(class CAVIAR *, int precision);
    int precision_;
  };

  // Everything FP64 (CVR_PREC_FP64).
  class B200_fp64 : public B200
  {
  public:
    B200_fp64(class CAVIAR *);
  };

} // md_simulator

CAVIAR_NAMESPACE_CLOSE

#endif
