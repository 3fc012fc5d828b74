// Stand-in for the reference's missing util/ckt.h (see ../refshim.h).
#include "../refshim.h"
