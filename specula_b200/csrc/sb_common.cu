// Status reporting of the specula_b200 C ABI.
#include "sb_common.cuh"

namespace sb {

static thread_local char g_last_error[512] = "";

int fail(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() { g_last_error[0] = '\0'; }

}  // namespace sb

extern "C" int sb_version(void) { return 100; }

extern "C" const char *sb_last_error(void) { return sb::g_last_error; }
