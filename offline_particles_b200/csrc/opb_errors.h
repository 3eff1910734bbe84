// Last-error slot shared by every entry point of the library (opb_last_error).
#pragma once

namespace opb {
// Record a formatted message for opb_last_error() and return `code`.
int fail(int code, const char *fmt, ...);
// Clear the message after a successful call.
void clear_error();
}  // namespace opb
