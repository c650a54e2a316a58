// Stand-in (oracle harness only): Vector.h defines Matrix too.
#include "Vector.h"
