// Minimal stand-in for an external header the reference sources include
// (psrdada_cpp / Boost are not installed); test infrastructure for oracle/_ref only.
#pragma once
#include <cuda_runtime.h>
#include <stdexcept>
#include <string>
#define CUDA_ERROR_CHECK(ans) do { cudaError_t e_ = (ans); if(e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_)); } while(0)
