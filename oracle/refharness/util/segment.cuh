// Stand-in for the reference's missing util/segment.cuh (see ../refshim.h).
#include "../refshim.h"
