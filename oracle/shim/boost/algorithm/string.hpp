// Minimal stand-in for the one Boost function the reference's filetype_typedefs.h uses
// (boost::iequals, case-insensitive string equality).  Boost is not installed in this
// toolchain; this shim exists only so oracle/ref_io.cpp can compile the reference's file
// readers.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cctype>
#include <string>

namespace boost {
inline bool iequals(const std::string &a, const std::string &b)
{
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); i++)
        if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
    return true;
}
}  // namespace boost
