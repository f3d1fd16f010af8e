// WeightsManager on the B200 (cpp/skyweaver/src/WeightsManager.cu:16-87).
//
// w = clamp(rn(127 * a * cos(2 pi phi))), clamp(rn(-127 * a * sin(2 pi phi)))
// with phi = ((t - t0) * rate + offset) * f in FP64, exactly the reference
// formula.  Besides the reference [F][B][A] char2 layout the kernel emits the
// A operand of the tensor-core beamformer: for each channel a "re" block of
// rows (w_re, -w_im) and an "im" block of rows (w_im, w_re) per antenna, so
// that D_re = sum(w_re v_re - w_im v_im) and D_im = sum(w_im v_re + w_re v_im)
// are plain int8 GEMMs against the (v_re, v_im) interleaved K dimension.
#include "sw_common.cuh"

namespace swb {
namespace {

constexpr double kTwoPi = 6.283185307179586;  // TWOPI in WeightsManager.cu:9

__device__ __forceinline__ int8_t clamp_int(int v)
{
    // clamp<int8_t, int> (types.cuh:211-221)
    return static_cast<int8_t>(fmaxf(-128.0f, fminf(127.0f, static_cast<float>(v))));
}

__device__ __forceinline__ int8_t neg_sat(int8_t v)
{
    // -(-128) is not representable; it only arises for |antenna weight| > 1.
    return v == -128 ? (int8_t)127 : (int8_t)(-v);
}

__device__ __forceinline__ void store_gemm(char2* gemm, int f, int b, int a,
                                           int nbeams, int nant, int8_t wr,
                                           int8_t wi)
{
    const size_t re_row = ((size_t)(f * 2 + 0) * nbeams + b) * nant + a;
    const size_t im_row = ((size_t)(f * 2 + 1) * nbeams + b) * nant + a;
    gemm[re_row] = make_char2(wr, neg_sat(wi));
    gemm[im_row] = make_char2(wi, wr);
}

__global__ void generate_weights_k(const float3* __restrict__ delays,
                                   const double* __restrict__ freqs, int nant,
                                   int nbeams, int nchans, double current_epoch,
                                   double delay_epoch, const double* __restrict__ d_epochs,
                                   char2* __restrict__ fba, char2* __restrict__ gemm)
{
    const size_t total = (size_t)nchans * nbeams * nant;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
        i += (size_t)gridDim.x * blockDim.x) {
        const int a = (int)(i % nant);
        const int b = (int)((i / nant) % nbeams);
        const int f = (int)(i / ((size_t)nant * nbeams));
        const float3 dm     = delays[(size_t)b * nant + a];
        // d_epochs (optional) = {current, delay} on the device, so a captured
        // graph can follow the epoch without re-instantiation
        const double t = d_epochs ? (d_epochs[0] - d_epochs[1]) : (current_epoch - delay_epoch);
        const double phase  = (t * (double)dm.z + (double)dm.y) * freqs[f];
        double sn, cs;
        sincos(kTwoPi * phase, &sn, &cs);
        const int8_t wr = clamp_int(__double2int_rn(cs * 127.0 * (double)dm.x));
        const int8_t wi = clamp_int(__double2int_rn(-1.0 * sn * 127.0 * (double)dm.x));
        if(fba) fba[i] = make_char2(wr, wi);
        if(gemm) store_gemm(gemm, f, b, a, nbeams, nant, wr, wi);
    }
}

__global__ void pack_weights_k(const char2* __restrict__ fba,
                               char2* __restrict__ gemm, int nchans, int nbeams,
                               int nant)
{
    const size_t total = (size_t)nchans * nbeams * nant;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
        i += (size_t)gridDim.x * blockDim.x) {
        const int a = (int)(i % nant);
        const int b = (int)((i / nant) % nbeams);
        const int f = (int)(i / ((size_t)nant * nbeams));
        const char2 w = fba[i];
        store_gemm(gemm, f, b, a, nbeams, nant, w.x, w.y);
    }
}

int grid_size(size_t n)
{
    size_t g = (n + 255) / 256;
    return (int)(g > 148 * 16 ? 148 * 16 : (g ? g : 1));
}

}  // namespace

int launch_weights(const float* d_delays, const double* d_freqs, int nant,
                   int nbeams, int nchans, double current_epoch, double delay_epoch,
                   const double* d_epochs, void* d_fba, void* d_gemm,
                   cudaStream_t stream)
{
    SW_REQUIRE(d_delays && d_freqs, "sw_generate_weights: null input");
    SW_REQUIRE(d_fba || d_gemm, "sw_generate_weights: no output");
    SW_REQUIRE(nant > 0 && nbeams > 0 && nchans > 0, "sw_generate_weights: empty shape");
    const size_t n = (size_t)nchans * nbeams * nant;
    generate_weights_k<<<grid_size(n), 256, 0, stream>>>(
        reinterpret_cast<const float3*>(d_delays), d_freqs, nant, nbeams, nchans,
        current_epoch, delay_epoch, d_epochs, static_cast<char2*>(d_fba),
        static_cast<char2*>(d_gemm));
    SW_LAUNCH_CHECK();
    return SW_OK;
}

}  // namespace swb

using namespace swb;

extern "C" {

int sw_generate_weights(const float* d_delays, const double* d_freqs,
                        int nant, int nbeams, int nchans, double current_epoch,
                        double delay_epoch, void* d_weights_fba,
                        void* d_weights_gemm, sw_stream_t stream)
{
    return launch_weights(d_delays, d_freqs, nant, nbeams, nchans, current_epoch,
                          delay_epoch, nullptr, d_weights_fba, d_weights_gemm,
                          as_cuda(stream));
}

int sw_pack_weights(const void* d_weights_fba, void* d_weights_gemm,
                    int nchans, int nbeams, int nant, sw_stream_t stream)
{
    SW_REQUIRE(d_weights_fba && d_weights_gemm, "sw_pack_weights: null pointer");
    const size_t n = (size_t)nchans * nbeams * nant;
    pack_weights_k<<<grid_size(n), 256, 0, as_cuda(stream)>>>(
        static_cast<const char2*>(d_weights_fba), static_cast<char2*>(d_weights_gemm),
        nchans, nbeams, nant);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

}  // extern "C"
