// Internal helpers shared by the host and device translation units.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "cola_spmm.h"

namespace cola {

// Records a thread-local message for cola_last_error() and returns s.
cola_status fail(cola_status s, const char *fmt, ...);
void clear_error();

}  // namespace cola

#define COLA_REQUIRE(cond, status, ...)            \
    do {                                           \
        if (!(cond))                               \
            return ::cola::fail((status), __VA_ARGS__); \
    } while (0)

#define COLA_TRY(expr)                        \
    do {                                      \
        cola_status _s = (expr);              \
        if (_s != COLA_SUCCESS)               \
            return _s;                        \
    } while (0)
