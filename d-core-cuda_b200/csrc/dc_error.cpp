// Thread-local error message store behind dc_last_error().
#include <cstdarg>
#include <cstdio>

#include "dc_internal.h"

namespace dc {

static thread_local char g_last_error[1024] = "";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_last_error[0] = '\0'; }

}  // namespace dc

extern "C" const char* dc_last_error(void) { return dc::g_last_error; }

extern "C" const char* dc_version(void) { return "d-core-b200 0.1.0 (sm_100a)"; }
