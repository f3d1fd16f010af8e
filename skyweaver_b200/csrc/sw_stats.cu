// StatisticsCalculator on the B200.
//
// The reference (cpp/skyweaver/src/StatisticsCalculator.cu:54-85) walks each
// (channel, pol, antenna) series serially in one thread with FP64 running
// moments.  Here the int8 inputs make the raw power sums S1..S4 exact in
// 64-bit integers, so the series is split over many CTAs that add their
// partial sums into an int64 workspace, and a finalize kernel forms mean,
// std (n-1), skewness and kurtosis in FP64 from the exact sums.  The kernel
// streams the FPACT rows once with 16-byte loads (HBM bound).
//
// update_scalings (cpp/skyweaver/src/StatisticsCalculator.cu:132-239) runs
// on the device with the same IEEE single operations in the same order; its
// outputs are indexed [beamset][chan] (the reference writes [chan] for every
// beamset).
#include <mutex>
#include <vector>

#include "sw_common.cuh"

namespace swb {
namespace {

constexpr int kStatsThreads = 256;
constexpr int kChunkSamples = 16384;  // samples per CTA per row pair

// S1 and S2 by dp4a; the cubes (|x^3| <= 2^21) go into a 32-bit partial
// that the caller widens once per 16-byte load, and the four fourth powers of
// a word (x^4 <= 2^28, four of them < 2^31) are summed in 32 bits before one
// 64-bit add.
__device__ __forceinline__ void accum_word(uint32_t w, int& s1, int& s2, int& s3w,
                                           long long& s4)
{
    s1 = __dp4a((int)w, 0x01010101, s1);
    s2 = __dp4a((int)w, (int)w, s2);
    int q4 = 0;
#pragma unroll
    for(int k = 0; k < 4; ++k) {
        const int x  = (int)(int8_t)(w >> (8 * k));
        const int x2 = x * x;
        s3w += x2 * x;
        q4 += x2 * x2;
    }
    s4 += q4;
}

// grid: (chunks per series, F*P*A series).  Each series is the pair of
// planar rows (re, im) of one (f, p, a).
__global__ void __launch_bounds__(kStatsThreads)
stats_partial_k(const uint8_t* __restrict__ fpact, size_t row_stride,
                size_t sample_offset, int nsamples,
                unsigned long long* __restrict__ sums)
{
    const size_t series = blockIdx.y;
    const int t0 = blockIdx.x * kChunkSamples;
    const int t1 = min(nsamples, t0 + kChunkSamples);
    int s1 = 0, s2 = 0;
    long long s3 = 0, s4 = 0;
    for(int c = 0; c < 2; ++c) {
        const uint8_t* row = fpact + (series * 2 + c) * row_stride + sample_offset;
        for(int t = t0 + threadIdx.x * 16; t < t1; t += kStatsThreads * 16) {
            const uint4 v = *reinterpret_cast<const uint4*>(row + t);
            int s3w = 0;  // 16 cubes: |sum| <= 2^25
            accum_word(v.x, s1, s2, s3w, s4);
            accum_word(v.y, s1, s2, s3w, s4);
            accum_word(v.z, s1, s2, s3w, s4);
            accum_word(v.w, s1, s2, s3w, s4);
            s3 += s3w;
        }
    }
    long long v1 = s1, v2 = s2, v3 = s3, v4 = s4;
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) {
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        v2 += __shfl_xor_sync(0xffffffffu, v2, o);
        v3 += __shfl_xor_sync(0xffffffffu, v3, o);
        v4 += __shfl_xor_sync(0xffffffffu, v4, o);
    }
    __shared__ long long red[kStatsThreads / 32][4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(lane == 0) {
        red[warp][0] = v1; red[warp][1] = v2; red[warp][2] = v3; red[warp][3] = v4;
    }
    __syncthreads();
    if(threadIdx.x < 4) {
        long long acc = 0;
        for(int w = 0; w < kStatsThreads / 32; ++w) acc += red[w][threadIdx.x];
        atomicAdd(&sums[series * 4 + threadIdx.x], (unsigned long long)acc);
    }
}

// TAFTP -> FPACT transpose with the statistics of the same pass: the
// transpose of sw_layout.cu (16 input bytes = 4 samples x 2 pols x re/im of
// one antenna -> one 32-bit word in each of the four planar rows) plus the
// exact S1..S4 sums of those words, so the gulp is read once for both.  A
// CTA is (hpc heaps, one channel); its 256 threads take 4 antennas x
// 64 16-byte chunks of a heap, walk the CTA's heaps for each antenna group
// and add one warp-reduced set of sums per (antenna, pol) into the int64
// workspace (the two warps of an antenna both add).  Padded antennas (a >=
// in_nant) are written as zeros and summed as zeros, like the separate
// stages.  The sums cost more issue than the copy, so the kernel is
// issue-bound: on a 64 ant x 64 ch x 65536-sample gulp (with its memset) 16,
// 8, 4, 2 and 1 heaps per CTA took 0.542, 0.498, 0.526, 0.633 and 1.042 ms,
// against 0.342 + 0.278 ms for the separate transpose and statistics (16
// heaps leave a second wave of CTAs that fills a third of the SMs).
constexpr int kFuseHeaps = 8;
constexpr int kHeapSamples = 256;

__device__ __forceinline__ uint32_t bperm(uint32_t a, uint32_t b, uint32_t sel)
{
    return __byte_perm(a, b, sel);
}

__global__ void __launch_bounds__(256)
transpose_stats_k(const uint4* __restrict__ taftp, uint8_t* __restrict__ fpact,
                  int in_nant, int out_nant, int nchans, int nheaps, size_t row_stride,
                  size_t sample_offset, unsigned long long* __restrict__ sums, int hpc)
{
    const int f  = blockIdx.y;
    const int h0 = blockIdx.x * hpc;
    const int h1 = min(nheaps, h0 + hpc);
    const int c = threadIdx.x & 63, lane = threadIdx.x & 31;
    for(int ag = 0; ag < out_nant; ag += 4) {
        const int a = ag + (int)(threadIdx.x >> 6);  // uniform across a warp
        int s1[2] = {0, 0}, s2[2] = {0, 0};
        long long s3[2] = {0, 0}, s4[2] = {0, 0};
        if(a < out_nant) {
            const size_t base0 = (((size_t)f * 2 + 0) * out_nant + a) * 2 * row_stride + sample_offset;
            const size_t base1 = (((size_t)f * 2 + 1) * out_nant + a) * 2 * row_stride + sample_offset;
            for(int h = h0; h < h1; ++h) {
                uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
                if(a < in_nant) {
                    const uint4 v = taftp[(((size_t)h * in_nant + a) * nchans + f) * 64 + c];
                    const uint32_t t0 = bperm(v.x, v.y, 0x5140), t1 = bperm(v.z, v.w, 0x5140);
                    const uint32_t t2 = bperm(v.x, v.y, 0x7362), t3 = bperm(v.z, v.w, 0x7362);
                    r0 = bperm(t0, t1, 0x5410);  // p0 re
                    r1 = bperm(t0, t1, 0x7632);  // p0 im
                    r2 = bperm(t2, t3, 0x5410);  // p1 re
                    r3 = bperm(t2, t3, 0x7632);  // p1 im
                }
                const size_t s = (size_t)h * kHeapSamples + c * 4;
                *reinterpret_cast<uint32_t*>(fpact + base0 + s)              = r0;
                *reinterpret_cast<uint32_t*>(fpact + base0 + row_stride + s) = r1;
                *reinterpret_cast<uint32_t*>(fpact + base1 + s)              = r2;
                *reinterpret_cast<uint32_t*>(fpact + base1 + row_stride + s) = r3;
                int s3w = 0;  // 8 cubes per pol: |sum| <= 2^24
                accum_word(r0, s1[0], s2[0], s3w, s4[0]);
                accum_word(r1, s1[0], s2[0], s3w, s4[0]);
                s3[0] += s3w;
                s3w = 0;
                accum_word(r2, s1[1], s2[1], s3w, s4[1]);
                accum_word(r3, s1[1], s2[1], s3w, s4[1]);
                s3[1] += s3w;
            }
        }
        long long v[8] = {s1[0], s2[0], s3[0], s4[0], s1[1], s2[1], s3[1], s4[1]};
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
#pragma unroll
            for(int k = 0; k < 8; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if(lane == 0 && a < out_nant) {
#pragma unroll
            for(int p = 0; p < 2; ++p)
#pragma unroll
                for(int k = 0; k < 4; ++k)
                    atomicAdd(&sums[(((size_t)f * 2 + p) * out_nant + a) * 4 + k],
                              (unsigned long long)v[4 * p + k]);
        }
    }
}

__global__ void stats_finalize_k(const long long* __restrict__ sums,
                                 float4* __restrict__ stats, int nseries,
                                 int nsamples)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nseries) return;
    const double n  = 2.0 * nsamples;
    const double S1 = (double)sums[4 * i + 0];
    const double S2 = (double)sums[4 * i + 1];
    const double S3 = (double)sums[4 * i + 2];
    const double S4 = (double)sums[4 * i + 3];
    const double m  = S1 / n;
    const double M2 = S2 - S1 * m;
    const double M3 = S3 - 3.0 * m * S2 + 3.0 * m * m * S1 - n * m * m * m;
    const double M4 = S4 - 4.0 * m * S3 + 6.0 * m * m * S2 - 4.0 * m * m * m * S1 +
                      n * m * m * m * m;
    float4 r;
    r.x = (float)m;
    r.y = (float)sqrt(M2 / (n - 1.0));
    r.z = (float)(sqrt(n) * M3 / pow(M2, 1.5));
    r.w = (float)(n * M4 / (M2 * M2) - 3.0);
    stats[i] = r;
}

// One thread per (beamset, channel); sequential over (pol, antenna) exactly
// like the reference's host loop.
__global__ void scalings_k(const float4* __restrict__ stats,
                           const float* __restrict__ bw, int nbeamsets,
                           int nchans, int npol, int nant, int cb_tscrunch,
                           int ib_tscrunch, float output_level,
                           float* __restrict__ cb_off, float* __restrict__ cb_scl,
                           float* __restrict__ ib_off, float* __restrict__ ib_scl)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nbeamsets * nchans) return;
    const int s = i / nchans, f = i % nchans;
    float sum = 0.0f, count = 0.0f;
    for(int p = 0; p < npol; ++p)
        for(int a = 0; a < nant; ++a) {
            const float w = bw[(size_t)nant * s + a];
            sum   = fadd(sum, fmul(w, stats[((size_t)f * npol + p) * nant + a].y));
            count = fadd(count, w);
        }
    const float avg_std = fdiv(sum, count);
    const float eff     = fdiv(count, (float)npol);
    {
        const float x     = fmul(fmul(127.0f, avg_std), sqrtf(eff));
        const float scale = fmul(x, x);
        const float dof   = (float)(2 * cb_tscrunch * npol);
        cb_off[i] = fmul(scale, dof);
        cb_scl[i] = fdiv(fmul(scale, sqrtf(fmul(2.0f, dof))), output_level);
    }
    {
        const float scale = fmul(avg_std, avg_std);
        const float dof   = fmul(fmul((float)(2 * ib_tscrunch), eff), (float)npol);
        ib_off[i] = fmul(scale, dof);
        ib_scl[i] = fdiv(fmul(scale, sqrtf(fmul(2.0f, dof))), output_level);
    }
}

}  // namespace

int launch_statistics(const void* d_fpact, size_t row_stride,
                      size_t sample_offset, int nchans, int npol, int nant,
                      int nsamples, void* d_scratch, float* d_stats,
                      cudaStream_t stream)
{
    SW_REQUIRE(d_fpact && d_scratch && d_stats, "sw_statistics: null pointer");
    SW_REQUIRE(nsamples > 0 && nsamples % 16 == 0,
               "sw_statistics: nsamples must be a positive multiple of 16");
    SW_REQUIRE(row_stride % 16 == 0 && sample_offset % 16 == 0,
               "sw_statistics: stride and offset must be multiples of 16");
    const int nseries = nchans * npol * nant;
    SW_REQUIRE(nseries > 0 && nseries <= 65535, "sw_statistics: too many series");
    const size_t sum_bytes = (size_t)nseries * 4 * sizeof(long long);
    SW_CUDA_CHECK(cudaMemsetAsync(d_scratch, 0, sum_bytes, stream));
    dim3 grid(cdiv(nsamples, kChunkSamples), nseries);
    stats_partial_k<<<grid, kStatsThreads, 0, stream>>>(
        static_cast<const uint8_t*>(d_fpact), row_stride, sample_offset,
        nsamples, static_cast<unsigned long long*>(d_scratch));
    SW_LAUNCH_CHECK();
    stats_finalize_k<<<cdiv(nseries, 256), 256, 0, stream>>>(
        static_cast<const long long*>(d_scratch),
        reinterpret_cast<float4*>(d_stats), nseries, nsamples);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free statistics.  Some callers cannot call cudaMalloc/cudaFree:
// a real-time ingest loop where the implicit device synchronisation of an
// allocation would stall the transfers and kernels already in flight, or a
// host process whose device memory is owned up front by another component
// (a ring-buffer manager, a memory pool) and gives this library no
// allocation rights.  For them sw_statistics_noalloc keeps its workspace in
// the file-scope array below, which every GPU that loads the library holds
// until the process exits.
constexpr int kNoAllocMaxSeries = 16384;  // channels x pols x antennas
static __device__ __align__(256) long long g_stats_noalloc_sums[kNoAllocMaxSeries * 4];

namespace {

// Device address of g_stats_noalloc_sums on the current device.  The host
// symbol is only a stand-in, so the address is looked up once per device
// (with that device current) and cached for the process; cudaDeviceReset
// would make the cached address stale, which the header documents.
int noalloc_sums(long long** out)
{
    static std::mutex mu;
    static std::vector<long long*> per_device;
    int dev = -1;
    SW_CUDA_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if((size_t)dev >= per_device.size()) per_device.resize(dev + 1, nullptr);
    if(per_device[dev] == nullptr) {
        void* p = nullptr;
        SW_CUDA_CHECK(cudaGetSymbolAddress(&p, g_stats_noalloc_sums));
        per_device[dev] = static_cast<long long*>(p);
    }
    *out = per_device[dev];
    return SW_OK;
}

}  // namespace

}  // namespace swb

using namespace swb;

extern "C" {

int sw_statistics_noalloc(const void* d_fpact, size_t row_stride, size_t sample_offset,
                          int nchans, int npol, int nant, int nsamples, float* d_stats,
                          sw_stream_t stream)
{
    const long long nseries = (long long)nchans * npol * nant;
    SW_REQUIRE(nseries > 0 && nseries <= kNoAllocMaxSeries,
               "sw_statistics_noalloc: %lld (channel, pol, antenna) series exceed the "
               "built-in workspace of %d; use sw_statistics with a caller workspace",
               nseries, kNoAllocMaxSeries);
    long long* sums = nullptr;
    const int rc = noalloc_sums(&sums);
    if(rc != SW_OK) return rc;
    // launch_statistics clears the sums before accumulating into them
    return launch_statistics(d_fpact, row_stride, sample_offset, nchans, npol, nant, nsamples,
                             sums, d_stats, as_cuda(stream));
}

int sw_transpose_fpact_statistics(const void* d_taftp, void* d_fpact, int nheaps,
                                  int input_nantennas, int output_nantennas, int nchans,
                                  size_t row_stride, size_t sample_offset, void* d_scratch,
                                  float* d_stats, sw_stream_t stream)
{
    SW_REQUIRE(d_taftp && d_fpact && d_scratch && d_stats,
               "sw_transpose_fpact_statistics: null pointer");
    SW_REQUIRE(nheaps > 0 && nchans > 0, "sw_transpose_fpact_statistics: empty input");
    SW_REQUIRE(input_nantennas > 0 && input_nantennas <= output_nantennas,
               "Input number of antennas must be <= to the maximum nantennas");
    SW_REQUIRE(row_stride % 16 == 0 && sample_offset % 16 == 0,
               "sw_transpose_fpact_statistics: row stride and offset must be multiples of 16");
    SW_REQUIRE(sample_offset + (size_t)nheaps * kHeapSamples <= row_stride,
               "sw_transpose_fpact_statistics: rows too short for the gulp");
    SW_REQUIRE(nchans <= 65535, "sw_transpose_fpact_statistics: too many channels");
    const int nseries = nchans * 2 * output_nantennas;
    const size_t sum_bytes = (size_t)nseries * 4 * sizeof(long long);
    cudaStream_t s = as_cuda(stream);
    SW_CUDA_CHECK(cudaMemsetAsync(d_scratch, 0, sum_bytes, s));
    dim3 grid(cdiv(nheaps, kFuseHeaps), nchans);
    transpose_stats_k<<<grid, 256, 0, s>>>(static_cast<const uint4*>(d_taftp),
                                          static_cast<uint8_t*>(d_fpact), input_nantennas,
                                          output_nantennas, nchans, nheaps, row_stride,
                                          sample_offset,
                                          static_cast<unsigned long long*>(d_scratch),
                                          kFuseHeaps);
    SW_LAUNCH_CHECK();
    stats_finalize_k<<<cdiv(nseries, 256), 256, 0, s>>>(
        static_cast<const long long*>(d_scratch), reinterpret_cast<float4*>(d_stats), nseries,
        nheaps * kHeapSamples);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

size_t sw_statistics_scratch_bytes(int nchans, int npol, int nant)
{
    return (size_t)nchans * npol * nant * 4 * sizeof(long long);
}

int sw_statistics(const void* d_fpact, size_t row_stride, size_t sample_offset,
                  int nchans, int npol, int nant, int nsamples,
                  void* d_scratch, float* d_stats, sw_stream_t stream)
{
    return launch_statistics(d_fpact, row_stride, sample_offset, nchans, npol,
                             nant, nsamples, d_scratch, d_stats, as_cuda(stream));
}

int sw_update_scalings(const float* d_stats, const float* d_beamset_weights,
                       int nbeamsets, int nchans, int npol, int nant,
                       int cb_tscrunch, int ib_tscrunch, float output_level,
                       float* d_cb_offsets, float* d_cb_scaling,
                       float* d_ib_offsets, float* d_ib_scaling,
                       sw_stream_t stream)
{
    SW_REQUIRE(d_stats && d_beamset_weights && d_cb_offsets && d_cb_scaling &&
                   d_ib_offsets && d_ib_scaling,
               "sw_update_scalings: null pointer");
    SW_REQUIRE(nbeamsets > 0 && nchans > 0, "sw_update_scalings: empty shape");
    const int n = nbeamsets * nchans;
    scalings_k<<<cdiv(n, 128), 128, 0, as_cuda(stream)>>>(
        reinterpret_cast<const float4*>(d_stats), d_beamset_weights, nbeamsets,
        nchans, npol, nant, cb_tscrunch, ib_tscrunch, output_level,
        d_cb_offsets, d_cb_scaling, d_ib_offsets, d_ib_scaling);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

}  // extern "C"
