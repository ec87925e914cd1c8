// Platform layer for the reference build used as the checker: the reference's LOG() lines are
// dropped unless MRT_ORACLE_LOG is set in the environment (the Linux layer of the reference prints
// them to stdout, app/System_dependent/Linux/Utils_dependent.hpp:14-16).
#ifndef UTILS_DEPENDENT_HPP
#define UTILS_DEPENDENT_HPP

#include <cstdlib>
#include <iostream>
#include <string>

namespace Dependent {
inline void printString(const ::std::string &log) noexcept {
    static const bool enabled = ::std::getenv("MRT_ORACLE_LOG") != nullptr;
    if (enabled) {
        ::std::cerr << log;
    }
}
}  // namespace Dependent

#endif
