// Minimal stand-in for an external header the reference sources include
// (psrdada_cpp / Boost are not installed); test infrastructure for oracle/_ref only.
#pragma once
#include <string>
namespace boost { namespace algorithm {
inline void trim(std::string& s) { const char* ws = " \t\n\r\f\v"; s.erase(0, s.find_first_not_of(ws)); s.erase(s.find_last_not_of(ws) + 1); }
} using algorithm::trim; }
