// Stand-in for core/Error.h: the exception names core/Utilities/TypeCasts.hpp throws.
#pragma once
#include <stdexcept>
namespace elsa
{
    struct InvalidArgumentError : std::invalid_argument {
        using std::invalid_argument::invalid_argument;
    };
    struct LogicError : std::logic_error {
        using std::logic_error::logic_error;
    };
    struct BadCastError : std::runtime_error {
        using std::runtime_error::runtime_error;
    };
} // namespace elsa
