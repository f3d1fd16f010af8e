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

int* device_error_ptr()
{
    static int* ptr = nullptr;
    if(ptr == nullptr) {
        void* p = nullptr;
        if(cudaGetSymbolAddress(&p, g_device_error) == cudaSuccess) ptr = static_cast<int*>(p);
    }
    return ptr;
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
