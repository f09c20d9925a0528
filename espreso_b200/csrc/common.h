// Shared helpers of the FETI4I B200 library: error state, timing, small utilities.
#pragma once

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace feti {

// Library errors never call exit(): the C entry points catch this exception,
// store its text for FETI4IGetLastError() and return.
struct Error : std::runtime_error {
    explicit Error(const std::string &m) : std::runtime_error(m) {}
};

#define FETI_CHECK(cond, msg)                                                    \
    do {                                                                         \
        if (!(cond)) throw ::feti::Error(std::string(msg));                      \
    } while (0)

void set_last_error(const std::string &m);
const char *last_error();
void clear_last_error();

inline double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Verbosity of the FETI4I_VERBOSE_LEVEL option (0 silent, 1 overview, >=2 convergence).
extern int g_verbose;
#define FETI_LOG(level, ...)                                                     \
    do {                                                                         \
        if (::feti::g_verbose >= (level)) { std::fprintf(stderr, __VA_ARGS__); } \
    } while (0)

}  // namespace feti
