// Force-included compatibility shim that lets g++ 13 build the reference
// sources unmodified.  The reference targets g++ 15 (C++23 <print> and
// std::sqrtf/std::powf from <cmath>); g++ 13's libstdc++ ships neither.
// This header adds exactly those names and nothing else.
#pragma once
#ifdef __cplusplus
#include <cmath>
#include <format>
#include <sstream>
#include <functional>
#include <unistd.h>
namespace std {
using ::sqrtf;
using ::powf;
}
#endif
