// The reference's md_simulator factory entries plus `md_simulator b200` and
// `md_simulator b200_fp64`.  Stands in for the reference's own
// include/caviar/objects/md_simulator/macro/all.h (which lists basic.h only)
// when this directory precedes the reference's on the include path; the
// object factory (src/caviar/interpreter/object_creator/objects_types.cpp)
// includes it inside its md_simulator creator.
#include "caviar/objects/md_simulator/macro/basic.h"

#ifdef FC_CHECK_AND_CREATE_ACTIVATED
FC_CHECK_AND_CREATE(B200, b200, md_simulator::B200)
FC_CHECK_AND_CREATE(B200_fp64, b200_fp64, md_simulator::B200_fp64)
#endif
