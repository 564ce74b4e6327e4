// Stand-in for logging/Logger.h: the projector kernels' headers only call
// Logger::get(name)->debug(...) (projectors/Luts.hpp:18); spdlog is not available here.
#pragma once
#include <functional>
namespace elsa
{
    struct Logger {
        struct Sink {
            template <class... A>
            void debug(A&&...)
            {
            }
            template <class... A>
            void info(A&&...)
            {
            }
            template <class... A>
            void error(A&&...)
            {
            }
        };
        static Sink* get(const char*)
        {
            static Sink s;
            return &s;
        }
    };
} // namespace elsa
