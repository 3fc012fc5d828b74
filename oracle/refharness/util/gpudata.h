// Stand-in for the reference's missing util/gpudata.h (see ../refshim.h).
#include "../refshim.h"
