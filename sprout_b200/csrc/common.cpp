#include "common.hpp"

#include <algorithm>
#include <cstdarg>

namespace spb {

namespace {
thread_local std::string last_error;
}

int32_t fail(int32_t code, char const* fmt, ...) {
    char    buf[1024];
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    last_error = buf;
    return code;
}

void clear_error() {
    last_error.clear();
}

uint32_t resolve_threads(uint32_t requested) {
    uint32_t const hw = std::max(1u, std::thread::hardware_concurrency());
    return requested == 0 ? hw : std::min(requested, hw);
}

}  // namespace spb

extern "C" SPB_API char const* spb_last_error(void) {
    return spb::last_error.c_str();
}

extern "C" SPB_API char const* spb_version(void) {
    return "sprout_b200 0.1 (sm_100a)";
}
