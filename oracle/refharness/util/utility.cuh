// Stand-in for the reference's missing util/utility.cuh (see ../refshim.h).
#include "../refshim.h"
