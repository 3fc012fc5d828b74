// Stand-in for the reference's missing util/subckt.h (see ../refshim.h).
#include "../refshim.h"
