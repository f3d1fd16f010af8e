// Shared helpers for the skyweaver_b200 CUDA library: status handling, the
// thread-local error string behind sw_last_error(), the device error word
// used by bounded waits, and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <string>

#include "../../include/skyweaver_b200.h"

namespace swb {

// Thread-local last-error message (defined in sw_capi.cu).
void set_error(const char* fmt, ...);
const char* last_error();

// Device address of the error word that kernels with bounded waits write
// when they give up (defined in sw_capi.cu; read by sw_read_device_error).
int* device_error_ptr();
enum DeviceError {
    DEV_ERR_NONE = 0,
    DEV_ERR_CB_TIMEOUT = 1, // coherent beamformer pipeline wait timed out
};

inline cudaStream_t as_cuda(sw_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace swb

// Return an SW status from a C ABI function on a CUDA error.
#define SW_CUDA_CHECK(call)                                                    \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if(_e != cudaSuccess) {                                                \
            swb::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,         \
                           cudaGetErrorString(_e));                            \
            return SW_ERR_CUDA;                                                \
        }                                                                      \
    } while(0)

#define SW_REQUIRE(cond, ...)                                                  \
    do {                                                                       \
        if(!(cond)) {                                                          \
            swb::set_error(__VA_ARGS__);                                       \
            return SW_ERR_INVALID;                                             \
        }                                                                      \
    } while(0)

#define SW_LAUNCH_CHECK() SW_CUDA_CHECK(cudaGetLastError())

// Propagate a non-OK SW status.
#define SW_TRY(expr)                 \
    do {                             \
        int _rc = (expr);            \
        if(_rc != SW_OK) return _rc; \
    } while(0)

namespace swb {

// Largest channel count for which the incoherent beam's channel order is
// computed (one CTA ranks all channels in shared memory).
constexpr int kIbOrderMaxChans = 1024;

// ceil division
template <typename T>
__host__ __device__ constexpr T cdiv(T a, T b) { return (a + b - 1) / b; }

// IEEE single operations that the compiler may not contract into FMAs.
// The reference's CPU implementations round every multiply and add.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// SingleStokesBeamformerTraits::clamp (beamformer_utils.cuh:186-195)
__device__ __forceinline__ int8_t clamp_i8(float v)
{
    return static_cast<int8_t>(fmaxf(-128.0f, fminf(127.0f, v)));
}

}  // namespace swb
