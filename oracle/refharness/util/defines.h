// Stand-in for the reference's missing util/defines.h (see ../refshim.h).
#include "../refshim.h"
