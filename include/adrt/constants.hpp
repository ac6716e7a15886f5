/// @file constants.hpp
/// @brief Shared constants of the adrt API (same name and value as the
///        reference's src/constants.hpp:8, so code written against the
///        reference's headers compiles unchanged).
#pragma once

namespace adrt {

inline constexpr double PI = 3.14159265358979323846;

}  // namespace adrt
