// The reference's md_simulator class list plus the B200 simulators.  Placed
// before the reference's include directory on the compiler's include path,
// this file stands in for the reference's own
// include/caviar/objects/md_simulator/all.h, which lists basic.h only.
#include "caviar/objects/md_simulator/basic.h"
#include "caviar/objects/md_simulator/b200.h"
