// Minimal stand-in for ksgpu's string_utils.hpp (oracle/_ref build only).
#ifndef _KSGPU_SHIM_STRING_UTILS_HPP
#define _KSGPU_SHIM_STRING_UTILS_HPP

#include <initializer_list>
#include <sstream>
#include <string>
#include <typeinfo>
#include <vector>

namespace ksgpu {

template<typename T>
inline std::string tuple_str(const std::vector<T> &v, const char *sep = ",")
{
    std::stringstream ss;
    ss << "(";
    for (size_t i = 0; i < v.size(); i++) ss << (i ? sep : "") << v[i];
    ss << ")";
    return ss.str();
}
template<typename T>
inline std::string tuple_str(std::initializer_list<T> v, const char *sep = ",")
{
    return tuple_str(std::vector<T>(v), sep);
}
template<typename T>
inline std::string tuple_str(int n, const T *v)
{
    return tuple_str(std::vector<T>(v, v + n));
}

template<typename T>
inline std::string brace_str(const std::vector<T> &v)
{
    std::stringstream ss;
    ss << "{";
    for (size_t i = 0; i < v.size(); i++) ss << (i ? "," : "") << v[i];
    ss << "}";
    return ss.str();
}

template<typename T> inline std::string type_name() { return typeid(T).name(); }
template<> inline std::string type_name<float>() { return "float"; }
template<> inline std::string type_name<double>() { return "double"; }
template<> inline std::string type_name<int>() { return "int"; }
template<> inline std::string type_name<long>() { return "long"; }
template<> inline std::string type_name<bool>() { return "bool"; }
template<> inline std::string type_name<std::string>() { return "string"; }

inline std::string nbytes_to_str(long nbytes)
{
    std::stringstream ss;
    const char *u[] = {"bytes", "KiB", "MiB", "GiB", "TiB"};
    double x = double(nbytes);
    int i = 0;
    while (x >= 1024.0 && i < 4) { x /= 1024.0; i++; }
    ss << x << " " << u[i];
    return ss.str();
}

}  // namespace ksgpu

#endif
