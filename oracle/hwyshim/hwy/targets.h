/* Single-target stand-in for Highway's targets.h (see highway.h). */
#include "hwy/highway.h"
