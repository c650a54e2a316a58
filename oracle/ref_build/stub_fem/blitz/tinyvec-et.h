// Stand-in (oracle harness only).
#include "array.h"
