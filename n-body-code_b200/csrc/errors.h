// Internal (not part of the C-ABI): records the thread-local message that
// nbody_last_error() returns, and passes the status through.
#pragma once
#include "../../include/nbody_cuda.h"

nbody_status nbody_set_error(nbody_status s, const char* fmt, ...)
    __attribute__((format(printf, 2, 3), visibility("hidden")));
