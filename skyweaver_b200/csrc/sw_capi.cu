// Library-wide C ABI pieces: version, thread-local error string and the
// device error word that bounded device-side waits report through.
#include <stdarg.h>

#include "sw_common.cuh"

namespace swb {

static thread_local std::string t_last_error;

void set_error(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
}

const char* last_error() { return t_last_error.c_str(); }

__device__ int g_device_error = 0;

// Device address of g_device_error on the current device.  Every device that
// loads the library has its own copy, so the address is looked up on each
// launch (a runtime table lookup) instead of cached: a cache would hand one
// device's address to kernels on another, or go stale after cudaDeviceReset.
int* device_error_ptr()
{
    void* p = nullptr;
    return cudaGetSymbolAddress(&p, g_device_error) == cudaSuccess ? static_cast<int*>(p)
                                                                   : nullptr;
}

}  // namespace swb

extern "C" {

int sw_version(void) { return 100; }

const char* sw_last_error(void) { return swb::last_error(); }

int sw_read_device_error(int* h_code)
{
    SW_REQUIRE(h_code != nullptr, "sw_read_device_error: null output");
    SW_CUDA_CHECK(cudaMemcpyFromSymbol(h_code, swb::g_device_error, sizeof(int)));
    return SW_OK;
}

int sw_reset_device_error(void)
{
    int zero = 0;
    SW_CUDA_CHECK(cudaMemcpyToSymbol(swb::g_device_error, &zero, sizeof(int)));
    return SW_OK;
}

}  // extern "C"
