// Minimal stand-in for an external header the reference sources include
// (psrdada_cpp / Boost are not installed); test infrastructure for oracle/_ref only.
#pragma once
#include <ostream>
namespace swref_log { struct Null { template <typename T> Null& operator<<(const T&) { return *this; } Null& operator<<(std::ostream& (*)(std::ostream&)) { return *this; } }; inline Null& null() { static Null n; return n; } }
#define BOOST_LOG_TRIVIAL(level) ::swref_log::null()
#define BOOST_LOG_NAMED_SCOPE(name)
