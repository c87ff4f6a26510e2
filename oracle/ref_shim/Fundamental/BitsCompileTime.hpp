/*
 * oracle/ref_shim/Fundamental/BitsCompileTime.hpp -- TEST INFRASTRUCTURE.
 *
 * Stand-in for the un-vendored "Fundamental" submodule (.gitmodules:4-6) so
 * that the reference's UpdaterGPUScBFM_AB_Type.cu compiles from its own
 * sources.  It provides only the compile-time helpers used by diluteBits
 * (UpdaterGPUScBFM_AB_Type.cu:204-230): an all-ones mask, a rectangular bit
 * wave (nOn ones then nOff zeros, repeated from bit 0), an integer ceiling
 * division and an integer ceiling logarithm.  Their meaning is fixed by the
 * Morton masks quoted in the reference's comment at .cu:240-249.
 */
#pragma once
#include <climits>

namespace CompileTimeFunctions {

template <typename A, typename B>
constexpr auto ceilDiv(A a, B b) -> decltype(a / b)
{
    return (a + b - 1) / b;
}

template <unsigned long long B, unsigned long long N, bool done = (N <= 1)>
struct CeilLog {
    static constexpr unsigned long long value = 1 + CeilLog<B, (N + B - 1) / B>::value;
};
template <unsigned long long B, unsigned long long N>
struct CeilLog<B, N, true> {
    static constexpr unsigned long long value = 0;
};

} // namespace CompileTimeFunctions

namespace BitPatterns {

template <typename T, unsigned long long n>
struct Ones {
    static constexpr T value = (n >= sizeof(T) * CHAR_BIT) ? T(~T(0)) : T((T(1) << n) - T(1));
};

template <typename T, unsigned long long nOn, unsigned long long nOff>
struct RectangularWave {
    static constexpr T make()
    {
        T v = 0;
        for (unsigned long long b = 0; b < sizeof(T) * CHAR_BIT; ++b)
            if (b % (nOn + nOff) < nOn) v = T(v | (T(1) << b));
        return v;
    }
    static constexpr T value = make();
};

} // namespace BitPatterns
