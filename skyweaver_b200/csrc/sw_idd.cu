// IncoherentDedisperser on the B200
// (cpp/skyweaver/src/IncoherentDedisperser.cu:66-125, a host OpenMP loop in
// the reference).
//
// out[t', d, b] = clamp(sum_{tau < ts} sum_f in[t + tau - delay[d,f], f, b]
//                       / scale_factor),   t = max_delay + t' * ts
// with truncation toward zero (types.cuh:211-221).  The int8 sums are exact
// integers (the reference accumulates them in float, exact below 2^24), so
// the kernel sums bytes with SWAR arithmetic: each 32-bit word of 4 beams is
// biased to unsigned (x + 128) and split into two pairs of 16-bit lanes,
// flushed into 32-bit accumulators every 256 additions.  The final
// float divide is the reference's single IEEE division.
#include "sw_common.cuh"

namespace swb {
namespace {

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

// grid: x = beam quads, y = output samples, z = trial DMs
__global__ void idd_k(const uint32_t* __restrict__ tfb, int nchans, int nquads,
                      const int* __restrict__ delays, int max_delay,
                      int tscrunch, float scale_factor,
                      uint32_t* __restrict__ tdb, int ndms, int nout)
{
    const int q  = blockIdx.x * blockDim.x + threadIdx.x;
    const int to = blockIdx.y;
    const int d  = blockIdx.z;
    if(q >= nquads || to >= nout) return;
    const int t = max_delay + to * tscrunch;
    const int* dl = delays + (size_t)d * nchans;
    int acc[4] = {0, 0, 0, 0};
    uint32_t lo = 0, hi = 0;
    int pending = 0;
    for(int tau = 0; tau < tscrunch; ++tau) {
        for(int f = 0; f < nchans; ++f) {
            const size_t row = (size_t)(t + tau - dl[f]) * nchans + f;
            const uint32_t w = tfb[row * nquads + q] ^ 0x80808080u;
            lo += prmt(w, 0, 0x4240);  // bytes 0,2 -> 16-bit lanes
            hi += prmt(w, 0, 0x4341);  // bytes 1,3
            if(++pending == 256) {
                acc[0] += (int)(lo & 0xffff); acc[2] += (int)(lo >> 16);
                acc[1] += (int)(hi & 0xffff); acc[3] += (int)(hi >> 16);
                lo = hi = 0;
                pending = 0;
            }
        }
    }
    acc[0] += (int)(lo & 0xffff); acc[2] += (int)(lo >> 16);
    acc[1] += (int)(hi & 0xffff); acc[3] += (int)(hi >> 16);
    const int bias = 128 * tscrunch * nchans;
    uint32_t packed = 0;
#pragma unroll
    for(int k = 0; k < 4; ++k) {
        const float v = fdiv((float)(acc[k] - bias), scale_factor);
        packed |= ((uint32_t)(uint8_t)clamp_i8(v)) << (8 * k);
    }
    tdb[((size_t)to * ndms + d) * nquads + q] = packed;
}

}  // namespace
}  // namespace swb

extern "C" int sw_incoherent_dedisperse(const int8_t* d_tfb, int nsamples,
                                        int nchans, int nbeams,
                                        const int* d_delays, int ndms,
                                        int max_delay, int tscrunch,
                                        float scale_factor, int8_t* d_tdb,
                                        sw_stream_t stream)
{
    SW_REQUIRE(d_tfb && d_delays && d_tdb, "sw_incoherent_dedisperse: null pointer");
    SW_REQUIRE(nsamples > max_delay,
               "Fewer than max_sample_delay samples passed to dedisperse method");
    SW_REQUIRE(tscrunch > 0 && (nsamples - max_delay) % tscrunch == 0,
               "(nsamples - max_sample_delay) must be a multiple of tscrunch;");
    SW_REQUIRE(nbeams % 4 == 0, "sw_incoherent_dedisperse: nbeams must be a multiple of 4");
    SW_REQUIRE(ndms > 0 && ndms <= 65535, "sw_incoherent_dedisperse: bad DM count");
    const int nout = (nsamples - max_delay) / tscrunch;
    SW_REQUIRE(nout <= 65535 * 1024, "sw_incoherent_dedisperse: too many samples");
    const int nquads = nbeams / 4;
    // nout may exceed the 65535 y-grid limit: chunk the launch over y
    for(int base = 0; base < nout; base += 65535) {
        const int n = nout - base < 65535 ? nout - base : 65535;
        dim3 grid(swb::cdiv(nquads, 128), n, ndms);
        swb::idd_k<<<grid, 128, 0, swb::as_cuda(stream)>>>(
            reinterpret_cast<const uint32_t*>(d_tfb) +
                (size_t)base * tscrunch * nchans * nquads,
            nchans, nquads, d_delays, max_delay, tscrunch, scale_factor,
            reinterpret_cast<uint32_t*>(d_tdb) + (size_t)base * ndms * nquads,
            ndms, n);
        SW_LAUNCH_CHECK();
    }
    return SW_OK;
}
