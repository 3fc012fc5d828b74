// Stand-in for the reference's missing util/utility.h (see ../refshim.h).
#include "../refshim.h"
