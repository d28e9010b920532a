// Minimal single-process helpers standing in for the external atlc library,
// written from how the reference uses them (src/qcs.cu:36-43 includes and
// their call sites). Test infrastructure for building the reference only.
#pragma once
#include <cstdio>
#include <stdexcept>
#include <string>
#include <unistd.h>

namespace atlc
{
template <typename... Args>
std::string format(const char *fmt, Args... args)
{
    char buf[4096];
    std::snprintf(buf, sizeof(buf), fmt, args...);
    return std::string(buf);
}

inline std::string format(const char *fmt) { return std::string(fmt); }

template <typename T>
int log2_int(T x)
{
    int r = -1;
    unsigned long long v = (unsigned long long)x;
    while (v)
    {
        v >>= 1;
        ++r;
    }
    return r;
}

template <typename F>
struct defer_guard
{
    F f;
    ~defer_guard() { f(); }
};
template <typename F>
defer_guard<F> make_defer(F f) { return defer_guard<F>{f}; }

template <typename Code>
inline void check_code(Code code, Code ok, const char *what, const char *file, int line)
{
    if (code != ok)
        throw std::runtime_error(format("%s failed with code %d at %s:%d", what, (int)code, file, line));
}
} // namespace atlc

#define ATLC_CONCAT_INNER(a, b) a##b
#define ATLC_CONCAT(a, b) ATLC_CONCAT_INNER(a, b)
#define ATLC_DEFER_FUNC(func, ...) \
    auto ATLC_CONCAT(atlc_defer_, __LINE__) = ::atlc::make_defer([&]() { func(__VA_ARGS__); })
