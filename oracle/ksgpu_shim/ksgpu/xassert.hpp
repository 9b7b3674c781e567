// Minimal stand-in for ksgpu's xassert.hpp (ksgpu is not vendored with pirate), written for the
// oracle/_ref build only. Each macro throws std::runtime_error with the failed condition.
#ifndef _KSGPU_SHIM_XASSERT_HPP
#define _KSGPU_SHIM_XASSERT_HPP

#include <sstream>
#include <stdexcept>
#include <string>

namespace ksgpu {

[[noreturn]] inline void _xassert_fail(const char *what, const char *file, int line, const std::string &extra = "")
{
    std::stringstream ss;
    ss << file << ":" << line << ": assertion '" << what << "' failed";
    if (!extra.empty())
        ss << " (" << extra << ")";
    throw std::runtime_error(ss.str());
}

template<typename A, typename B>
inline std::string _xassert_pair(const A &a, const B &b)
{
    std::stringstream ss;
    ss << "lhs=" << a << ", rhs=" << b;
    return ss.str();
}

}  // namespace ksgpu

#define xassert(c) do { if (!(c)) ::ksgpu::_xassert_fail(#c, __FILE__, __LINE__); } while (0)
#define xassert_msg(c, msg) do { if (!(c)) ::ksgpu::_xassert_fail(#c, __FILE__, __LINE__, msg); } while (0)
#define _xassert_cmp(a, b, op) do { auto _xa = (a); auto _xb = (b); \
    if (!(_xa op _xb)) ::ksgpu::_xassert_fail(#a " " #op " " #b, __FILE__, __LINE__, ::ksgpu::_xassert_pair(_xa, _xb)); } while (0)
#define xassert_eq(a, b) _xassert_cmp(a, b, ==)
#define xassert_ne(a, b) _xassert_cmp(a, b, !=)
#define xassert_lt(a, b) _xassert_cmp(a, b, <)
#define xassert_le(a, b) _xassert_cmp(a, b, <=)
#define xassert_gt(a, b) _xassert_cmp(a, b, >)
#define xassert_ge(a, b) _xassert_cmp(a, b, >=)
#define xassert_divisible(a, b) do { auto _xa = (a); auto _xb = (b); \
    if ((_xb == 0) || (_xa % _xb) != 0) ::ksgpu::_xassert_fail(#a " divisible by " #b, __FILE__, __LINE__, ::ksgpu::_xassert_pair(_xa, _xb)); } while (0)
#define xassert_iff(a, b) do { if (bool(a) != bool(b)) ::ksgpu::_xassert_fail(#a " iff " #b, __FILE__, __LINE__); } while (0)
#define xassert_shape_eq(arr, shp) do { if (!(arr).shape_equals(std::vector<long> shp)) \
    ::ksgpu::_xassert_fail(#arr ".shape == " #shp, __FILE__, __LINE__, (arr).shape_str()); } while (0)

#endif
