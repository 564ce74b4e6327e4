// Stand-in for core/elsaDefines.h with only the scalar types and helpers the projector kernels
// use (the real header needs Eigen, which this toolchain does not have).
#pragma once
#include <cstddef>
#include <stdexcept>
namespace elsa
{
    using real_t = float;
    using index_t = std::ptrdiff_t;
    template <typename T>
    constexpr T pi = static_cast<T>(3.14159265358979323846);
    template <typename T>
    struct SelfType {
        using type = T;
    };
    template <typename T>
    using SelfType_t = typename SelfType<T>::type;
} // namespace elsa
