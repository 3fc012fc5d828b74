// Stand-in for the reference's missing util/gpuckt.h (see ../refshim.h).
#include "../refshim.h"
