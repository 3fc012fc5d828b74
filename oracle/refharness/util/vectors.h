// Stand-in for the reference's missing util/vectors.h (see ../refshim.h).
#include "../refshim.h"
