// cc_error.h — error reporting shared by the library's translation units.
#pragma once

namespace cc {
// Record msg as the calling thread's last error (returned by cc_last_error) and return code.
int set_error(int code, const char *msg);
}  // namespace cc
