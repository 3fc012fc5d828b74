// Stand-in for the reference's missing util/g_utility.h (see ../refshim.h).
#include "../refshim.h"
