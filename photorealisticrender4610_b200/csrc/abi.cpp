// Library-level entry points: ABI version and per-thread error messages.
#include "prr_internal.h"

#include <cstring>

namespace prr {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

} // namespace prr

extern "C" {

int prr_abi_version(void) { return PRR_ABI_VERSION; }

int prr_last_error(char *buf, size_t len) {
    const std::string &e = prr::g_last_error;
    if (buf && len > 0) {
        const size_t n = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), n);
        buf[n] = '\0';
    }
    return (int) e.size();
}

} // extern "C"
