// Last-error slot of the C ABI: one message per host thread.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "opb200.h"
#include "opb_errors.h"

namespace opb {
namespace {
thread_local std::string g_last_error;
}

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

const char *last_error() { return g_last_error.c_str(); }
}  // namespace opb

extern "C" const char *opb_last_error(void) { return opb::last_error(); }
