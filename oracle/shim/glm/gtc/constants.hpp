// Stand-in for GLM's gtc/constants.hpp (test infrastructure for the reference build only).
// The constants are the mathematical values of pi, 2*pi and pi/4, rounded to the requested type.
#ifndef MRT_ORACLE_SHIM_GLM_CONSTANTS_HPP
#define MRT_ORACLE_SHIM_GLM_CONSTANTS_HPP

namespace glm {
template <typename T> constexpr T pi() noexcept { return static_cast<T>(3.14159265358979323846264338327950288L); }
template <typename T> constexpr T two_pi() noexcept { return static_cast<T>(6.28318530717958647692528676655900576L); }
template <typename T> constexpr T quarter_pi() noexcept { return static_cast<T>(0.785398163397448309615660845819875721L); }
}  // namespace glm

#endif
