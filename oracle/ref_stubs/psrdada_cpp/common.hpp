// Minimal stand-in for an external header the reference sources include
// (psrdada_cpp / Boost are not installed); test infrastructure for oracle/_ref only.
#pragma once
#include <algorithm>
#include <cstring>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include "boost/log/trivial.hpp"
