/* Single-target stand-in for Highway's foreach_target.h (see highway.h).
   One target means the including file is compiled once, and that pass is
   also the last one, so HWY_ONCE is true. */
#ifndef HWY_ONCE
#define HWY_ONCE 1
#endif
