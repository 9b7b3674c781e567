// Minimal stand-in for ksgpu's Dtype (oracle/_ref build only): a (kind, nbits) pair.
#ifndef _KSGPU_SHIM_DTYPE_HPP
#define _KSGPU_SHIM_DTYPE_HPP

#include <cstdint>
#include <ostream>
#include <stdexcept>
#include <string>
#include <cuda_fp16.h>

namespace ksgpu {

enum DtypeFlags : unsigned short { df_none = 0, df_int = 1, df_uint = 2, df_float = 4, df_complex = 8 };

struct Dtype
{
    unsigned short flags = df_none;
    unsigned short nbits = 0;

    Dtype() = default;
    Dtype(unsigned short flags_, int nbits_) : flags(flags_), nbits((unsigned short) nbits_) {}

    template<typename T> static Dtype native();

    bool is_empty() const { return nbits == 0; }
    bool operator==(const Dtype &d) const { return flags == d.flags && nbits == d.nbits; }
    bool operator!=(const Dtype &d) const { return !(*this == d); }

    std::string str() const
    {
        std::string k = (flags & df_complex) ? "complex" : (flags & df_float) ? "float" : (flags & df_uint) ? "uint" : (flags & df_int) ? "int" : "none";
        return k + std::to_string(nbits);
    }

    // Unit roundoff of a floating-point type (2^-p, p = stored mantissa bits + 1).
    double precision() const
    {
        if (!(flags & df_float)) throw std::runtime_error("Dtype::precision(): not a floating-point type");
        int nb = (flags & df_complex) ? nbits / 2 : nbits;
        if (nb == 16) return 1.0 / 2048.0;
        if (nb == 32) return 1.0 / 16777216.0;
        if (nb == 64) return 1.0 / 9007199254740992.0;
        throw std::runtime_error("Dtype::precision(): unsupported width");
    }

    static Dtype from_str(const std::string &s)
    {
        static const struct { const char *name; unsigned short f; int n; } tab[] = {
            {"float16", df_float, 16}, {"float32", df_float, 32}, {"float64", df_float, 64},
            {"int8", df_int, 8}, {"int16", df_int, 16}, {"int32", df_int, 32}, {"int64", df_int, 64},
            {"uint8", df_uint, 8}, {"uint16", df_uint, 16}, {"uint32", df_uint, 32}, {"uint64", df_uint, 64},
            {"complex64", df_float | df_complex, 64}, {"complex128", df_float | df_complex, 128}};
        for (auto &t : tab)
            if (s == t.name) return Dtype(t.f, t.n);
        throw std::runtime_error("Dtype::from_str(): unknown dtype '" + s + "'");
    }
};

template<> inline Dtype Dtype::native<float>() { return Dtype(df_float, 32); }
template<> inline Dtype Dtype::native<double>() { return Dtype(df_float, 64); }
template<> inline Dtype Dtype::native<__half>() { return Dtype(df_float, 16); }
template<> inline Dtype Dtype::native<int8_t>() { return Dtype(df_int, 8); }
template<> inline Dtype Dtype::native<int16_t>() { return Dtype(df_int, 16); }
template<> inline Dtype Dtype::native<int>() { return Dtype(df_int, 32); }
template<> inline Dtype Dtype::native<long>() { return Dtype(df_int, 64); }
template<> inline Dtype Dtype::native<uint8_t>() { return Dtype(df_uint, 8); }
template<> inline Dtype Dtype::native<uint16_t>() { return Dtype(df_uint, 16); }
template<> inline Dtype Dtype::native<unsigned int>() { return Dtype(df_uint, 32); }
template<> inline Dtype Dtype::native<unsigned long>() { return Dtype(df_uint, 64); }
template<> inline Dtype Dtype::native<char>() { return Dtype(df_int, 8); }

inline std::ostream &operator<<(std::ostream &os, const Dtype &d) { return os << d.str(); }

template<typename T>
inline void _check_dtype(const Dtype &d, const char *where)
{
    if (d != Dtype::native<T>())
        throw std::runtime_error(std::string(where) + ": dtype " + d.str() + " does not match " + Dtype::native<T>().str());
}
template<> inline void _check_dtype<void>(const Dtype &, const char *) {}

}  // namespace ksgpu

#endif
