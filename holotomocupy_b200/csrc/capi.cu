// Library-wide entry points: version and last-error message.
#include "common.cuh"
#include "holotomo_b200_internal.h"

extern "C" int ht_version(void) { return 100; }

extern "C" const char* ht_last_error(void) { return ht::last_error(); }

extern "C" long ht_launch_count(void) { return ht::launch_count(); }
