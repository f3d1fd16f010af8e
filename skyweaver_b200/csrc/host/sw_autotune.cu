// Autotuner for the per-gulp chain, keyed on (nantennas, nbeams, nchans,
// nsamples, tscrunch, DM set): times the coherent dedisperser at every FFT
// length that fits the DM smear, and the coherent beamformer at several
// work-item sizes (the extent of its tiles in time) and then several
// pipeline depths (voltage and weight copies in flight) on synthetic int8
// data of that exact shape, and caches the fastest choice per key for the
// life of the process.
//
// The reference has no autotuner (its kernel shapes are compile-time
// constants, skyweaver_constants.hpp:28-135); it is what picks the B200
// kernels' launch shapes here.
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../sw_common.cuh"
#include "sw_host.hpp"

namespace swb {
namespace {

// deterministic pseudo-random int8 bytes in [-64, 63]
__global__ void fill_k(uint8_t* p, size_t n, uint32_t seed)
{
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
        i += (size_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)i * 2654435761u ^ seed;
        x ^= x >> 15;
        x *= 2246822519u;
        x ^= x >> 13;
        p[i] = (uint8_t)((x & 0x7f) - 64);
    }
}

struct Dev {
    void* p = nullptr;
    ~Dev() { cudaFree(p); }
    int alloc(size_t n)
    {
        SW_CUDA_CHECK(cudaMalloc(&p, n));
        return SW_OK;
    }
};

using Key = std::tuple<int, int, int, int, int, int, int>;
std::mutex g_mu;
std::map<Key, sw_tuning> g_cache;

// average time of `reps` calls after one warm-up, in ms
template <typename F>
int time_ms(F fn, cudaStream_t s, int reps, float* ms)
{
    SW_TRY(fn());
    cudaEvent_t e0, e1;
    SW_CUDA_CHECK(cudaEventCreate(&e0));
    SW_CUDA_CHECK(cudaEventCreate(&e1));
    SW_CUDA_CHECK(cudaEventRecord(e0, s));
    int rc = SW_OK;
    for(int i = 0; i < reps && rc == SW_OK; ++i) rc = fn();
    SW_CUDA_CHECK(cudaEventRecord(e1, s));
    SW_CUDA_CHECK(cudaEventSynchronize(e1));
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / reps;
    return rc;
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" int sw_autotune(int nantennas, int nbeams, int nchans, int nsamples, int tscrunch,
                           int ndms, const float* h_dms, double centre_frequency,
                           double bandwidth, sw_tuning* out, sw_stream_t stream)
{
    SW_REQUIRE(out && h_dms && ndms > 0, "sw_autotune: null argument");
    SW_REQUIRE(nantennas == 16 || nantennas == 32 || nantennas == 64,
               "sw_autotune: nantennas must be 16, 32 or 64");
    SW_REQUIRE(nchans > 0 && nbeams > 0 && nsamples > 0 && nsamples % 64 == 0 && tscrunch > 0,
               "sw_autotune: bad shape");
    // the pipeline's default overlap-save plan (sw_host.hpp)
    const int head    = cdd_head(centre_frequency, bandwidth, nchans, h_dms, ndms);
    const int lag     = cdd_round_lag(0, head);
    const int overlap = head + lag;
    const Key key{nantennas, nbeams, nchans, nsamples, tscrunch, ndms, overlap};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cache.find(key);
        if(it != g_cache.end()) {
            *out = it->second;
            return SW_OK;
        }
    }
    cudaStream_t s = as_cuda(stream);
    const int A = nantennas, F = nchans, T = nsamples, ndm = ndms;
    const size_t nrows = (size_t)F * 2 * A * 2;
    const size_t stride = ((size_t)overlap + T + 15) / 16 * 16;
    Dev in, outs, ws, wgemm, scl, ib, map, cb;
    SW_TRY(in.alloc(nrows * stride));
    SW_TRY(outs.alloc(nrows * (size_t)T * ndm));
    fill_k<<<1024, 256, 0, s>>>(static_cast<uint8_t*>(in.p), nrows * stride, 12345u);
    SW_LAUNCH_CHECK();
    std::vector<void*> dd(ndm);
    for(int d = 0; d < ndm; ++d) dd[d] = static_cast<uint8_t*>(outs.p) + nrows * (size_t)T * d;

    // ---- coherent dedispersion: every power-of-two FFT the smear allows
    // (on-chip sizes when any fits, the split sizes otherwise)
    sw_tuning best{};
    best.overlap = overlap;
    best.lag     = lag;
    best.cdd_ms = 1e30f;
    std::vector<int> lens;
    for(int n = 1024; n <= 8192; n *= 2)
        if(n > overlap) lens.push_back(n);
    if(lens.empty())
        for(int n = 16384; n <= 65536; n *= 2)
            if(n > overlap) lens.push_back(n);
    SW_REQUIRE(!lens.empty(), "sw_autotune: DM smear of %d samples exceeds the longest FFT",
               overlap);
    const double low = (double)(float)(centre_frequency - bandwidth / 2.0f);
    size_t ws_bytes = 0;
    for(int n : lens) {
        const size_t need = sw_cdd_workspace_bytes(F, 2, A, T, n, overlap, ndm);
        const size_t per_seg = (size_t)ndm * n * 8;
        if(need) ws_bytes = std::max(ws_bytes, std::max(per_seg, std::min(need, (size_t)1 << 30)));
    }
    if(ws_bytes) SW_TRY(ws.alloc(ws_bytes));
    for(int n : lens) {
        Dev st;
        SW_TRY(st.alloc(sw_cdd_setup_bytes(ndm, F, n)));
        SW_TRY(sw_cdd_chirps(h_dms, ndm, F, n, low, bandwidth, st.p, stream));
        const size_t per_seg = (size_t)ndm * n * 8;
        const size_t wsn = sw_cdd_workspace_bytes(F, 2, A, T, n, overlap, ndm)
                               ? ws_bytes / per_seg * per_seg
                               : 0;
        float ms = 0.0f;
        SW_TRY(time_ms([&] {
            return sw_coherent_dedisperse_ws(in.p, stride, F, 2, A, T, n, overlap, lag, st.p, ndm,
                                             dd.data(), (size_t)T, wsn ? ws.p : nullptr, wsn,
                                             nullptr, stream);
        }, s, 3, &ms));
        if(ms < best.cdd_ms) {
            best.cdd_ms = ms;
            best.fft_len = n;
        }
    }

    // ---- coherent beamformer: work-item sizes (64-sample tiles per item)
    const size_t wbytes = (size_t)F * 2 * nbeams * 2 * A;
    const int ts = tscrunch <= 32 && (tscrunch & (tscrunch - 1)) == 0 ? tscrunch : 16;
    const int nout = T / ts;
    SW_TRY(wgemm.alloc(wbytes));
    SW_TRY(scl.alloc((size_t)F * sizeof(float)));
    SW_TRY(ib.alloc((size_t)nout * F * sizeof(float)));
    SW_TRY(map.alloc((size_t)nbeams * sizeof(int)));
    SW_TRY(cb.alloc((size_t)ndm * nout * F * nbeams));
    fill_k<<<256, 256, 0, s>>>(static_cast<uint8_t*>(wgemm.p), wbytes, 777u);
    SW_LAUNCH_CHECK();
    SW_CUDA_CHECK(cudaMemsetAsync(map.p, 0, (size_t)nbeams * sizeof(int), s));
    SW_CUDA_CHECK(cudaMemsetAsync(ib.p, 0, (size_t)nout * F * sizeof(float), s));
    {
        std::vector<float> one(F, 1e9f);
        SW_CUDA_CHECK(cudaMemcpyAsync(scl.p, one.data(), F * sizeof(float),
                                      cudaMemcpyHostToDevice, s));
        SW_CUDA_CHECK(cudaStreamSynchronize(s));
    }
    best.cb_ms = 1e30f;
    auto time_cb = [&](int tpi, int vst, int wst, float* ms) {
        sw_cb_shape shape{F, T, A, nbeams, ts, 0, 1, (size_t)T, 0, tpi, vst, wst};
        std::vector<sw_cb_problem> probs;
        for(int d = 0; d < ndm; ++d)
            probs.push_back({dd[d], static_cast<int8_t*>(cb.p) + (size_t)d * nout * F * nbeams,
                             static_cast<float*>(ib.p), 0, nbeams});
        return time_ms([&] {
            return sw_coherent_beamform_grouped(&shape, probs.data(), ndm, wgemm.p,
                                                static_cast<float*>(scl.p),
                                                static_cast<float*>(scl.p),
                                                static_cast<int*>(map.p), stream);
        }, s, 3, ms);
    };
    // work-item size (the tile's extent in time) at the default depths ...
    for(int tpi : {4, 8, 16, 32, 64, 128}) {
        if(tpi > T / 64 && tpi != 4) break;
        float ms = 0.0f;
        SW_TRY(time_cb(tpi, 4, 2, &ms));
        if(ms < best.cb_ms) {
            best.cb_ms = ms;
            best.cb_tiles_per_item = tpi;
            best.cb_voltage_stages = 4;
            best.cb_weight_stages = 2;
        }
    }
    // ... then the pipeline depths at that size
    for(auto vw : {std::pair<int, int>{2, 2}, {3, 2}, {6, 2}, {8, 2}, {4, 3}, {6, 3}}) {
        float ms = 0.0f;
        SW_TRY(time_cb(best.cb_tiles_per_item, vw.first, vw.second, &ms));
        if(ms < best.cb_ms) {
            best.cb_ms = ms;
            best.cb_voltage_stages = vw.first;
            best.cb_weight_stages = vw.second;
        }
    }
    SW_CUDA_CHECK(cudaStreamSynchronize(s));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_cache[key] = best;
    }
    *out = best;
    return SW_OK;
}
