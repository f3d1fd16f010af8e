// Voltage layout kernels: the TAFTP -> FTPA transpose of the reference
// Transposer (cpp/skyweaver/src/Transposer.cu:13-104,117-184), the B200
// TAFTP -> FPACT (planar stream-major) transpose used by the pipeline,
// converters between FTPA and FPACT, and the overlap-save history copy.
//
// Both transposes are pure HBM streaming: every input byte is read once with
// 16-byte loads and every output byte written once with 16- or 4-byte
// stores, so their roofline is the HBM copy bandwidth.
#include "sw_common.cuh"

namespace swb {
namespace {

constexpr int kHeap = 256;  // SKYWEAVER_NSAMPLES_PER_HEAP
constexpr int kPol  = 2;    // SKYWEAVER_NPOL

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

// ---------------------------------------------------------------------------
// TAFTP -> FTPA.  One CTA per (heap, channel).  The heap's A_in x 256 x P
// char2 block (1 KiB per antenna) is staged in shared memory as 32-bit words
// w[a][s] = (p0.re, p0.im, p1.re, p1.im); the word index within a row is
// XOR-swizzled by the antenna group so that the column reads below are
// bank-conflict free.  Each thread then emits 16-byte output chunks
// (8 antennas of one (sample, pol) row).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int swz_word(int a, int s)
{
    return a * kHeap + (s ^ (((a >> 3) & 7) << 2));
}

__global__ void __launch_bounds__(256)
transpose_ftpa_k(const uint4* __restrict__ taftp, uint4* __restrict__ ftpa,
                 int in_nant, int out_nant, int nchans, int nheaps)
{
    extern __shared__ uint32_t sm_words[];
    const int h = blockIdx.x;
    const int f = blockIdx.y;
    // stage: A_in x 64 chunks of 16 bytes (4 samples x 2 pols x char2)
    for(int idx = threadIdx.x; idx < in_nant * 64; idx += blockDim.x) {
        const int a = idx >> 6, c = idx & 63;
        const size_t src = (((size_t)h * in_nant + a) * nchans + f) * 64 + c;
        uint4 v = taftp[src];
        uint4* dst = reinterpret_cast<uint4*>(&sm_words[swz_word(a, c * 4)]);
        *dst = v;
    }
    __syncthreads();
    const int groups = out_nant >> 3;  // 8 antennas -> 16 bytes per row
    const size_t nsamp = (size_t)nheaps * kHeap;
    for(int idx = threadIdx.x; idx < groups * kHeap; idx += blockDim.x) {
        const int g = idx % groups;
        const int s = idx / groups;
        uint32_t w[8];
#pragma unroll
        for(int i = 0; i < 8; ++i) {
            const int a = g * 8 + i;
            w[i] = (a < in_nant) ? sm_words[swz_word(a, s)] : 0u;
        }
        uint4 o0, o1;
        o0.x = prmt(w[0], w[1], 0x5410); o1.x = prmt(w[0], w[1], 0x7632);
        o0.y = prmt(w[2], w[3], 0x5410); o1.y = prmt(w[2], w[3], 0x7632);
        o0.z = prmt(w[4], w[5], 0x5410); o1.z = prmt(w[4], w[5], 0x7632);
        o0.w = prmt(w[6], w[7], 0x5410); o1.w = prmt(w[6], w[7], 0x7632);
        const size_t t   = (size_t)h * kHeap + s;
        const size_t row = ((size_t)f * nsamp + t) * kPol;  // (f, t, p=0)
        // row of out_nant char2 = out_nant/8 uint4
        ftpa[row * groups + g]           = o0;
        ftpa[(row + 1) * groups + g]     = o1;
    }
}

// ---------------------------------------------------------------------------
// TAFTP -> FPACT.  One CTA per (heap, channel); 64 threads per antenna, each
// turning 16 input bytes (4 samples x 2 pols x re/im) into one 32-bit word
// in each of the four planar rows (p0.re, p0.im, p1.re, p1.im).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
transpose_fpact_k(const uint4* __restrict__ taftp, uint8_t* __restrict__ fpact,
                  int in_nant, int out_nant, int nchans, size_t row_stride,
                  size_t sample_offset)
{
    const int h = blockIdx.x;
    const int f = blockIdx.y;
    for(int idx = threadIdx.x; idx < out_nant * 64; idx += blockDim.x) {
        const int a = idx >> 6, c = idx & 63;
        uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0;
        if(a < in_nant) {
            const size_t src = (((size_t)h * in_nant + a) * nchans + f) * 64 + c;
            uint4 v = taftp[src];
            uint32_t t0 = prmt(v.x, v.y, 0x5140), t1 = prmt(v.z, v.w, 0x5140);
            uint32_t t2 = prmt(v.x, v.y, 0x7362), t3 = prmt(v.z, v.w, 0x7362);
            r0 = prmt(t0, t1, 0x5410);  // p0 re
            r1 = prmt(t0, t1, 0x7632);  // p0 im
            r2 = prmt(t2, t3, 0x5410);  // p1 re
            r3 = prmt(t2, t3, 0x7632);  // p1 im
        }
        const size_t s = sample_offset + (size_t)h * kHeap + c * 4;
        const size_t base0 = ((((size_t)f * kPol + 0) * out_nant + a) * 2) * row_stride + s;
        const size_t base1 = ((((size_t)f * kPol + 1) * out_nant + a) * 2) * row_stride + s;
        *reinterpret_cast<uint32_t*>(fpact + base0)              = r0;
        *reinterpret_cast<uint32_t*>(fpact + base0 + row_stride) = r1;
        *reinterpret_cast<uint32_t*>(fpact + base1)              = r2;
        *reinterpret_cast<uint32_t*>(fpact + base1 + row_stride) = r3;
    }
}

// FTPA <-> FPACT converters (reference-layout stage wrappers and tests).
// One thread per 4 consecutive samples of one planar row (fewer in the last
// group when nsamples is not a multiple of 4).
__global__ void ftpa_to_fpact_k(const int8_t* __restrict__ ftpa,
                                int8_t* __restrict__ fpact, int nchans,
                                int nsamples, int nant, size_t row_stride,
                                size_t sample_offset, int to_fpact)
{
    const size_t nrows  = (size_t)nchans * kPol * nant * 2;
    const size_t nquads = nrows * ((nsamples + 3) / 4);
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nquads;
        i += (size_t)gridDim.x * blockDim.x) {
        const size_t row = i % nrows;  // row fastest -> coalesced FTPA reads
        const int t      = (int)(i / nrows) * 4;
        const int c  = (int)(row & 1);
        const int a  = (int)((row >> 1) % nant);
        const int p  = (int)((row / (2 * nant)) % kPol);
        const int f  = (int)(row / (2 * nant * kPol));
        int8_t* prow = fpact + row * row_stride + sample_offset + t;
#pragma unroll
        for(int k = 0; k < 4; ++k) {
            if(t + k >= nsamples) break;  // ragged last group
            const size_t fi = ((((size_t)f * nsamples + t + k) * kPol + p) * nant + a) * 2 + c;
            if(to_fpact) prow[k] = ftpa[fi];
            else const_cast<int8_t*>(ftpa)[fi] = prow[k];
        }
    }
}

// the last history16 16-byte chunks of every row of `src` to the front of
// the same row of `dst` (src == dst: in place)
__global__ void keep_history_k(const uint4* src, uint4* dst, size_t nrows,
                               size_t row_stride16, size_t history16,
                               size_t nsamples16)
{
    const size_t total = nrows * history16;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
        i += (size_t)gridDim.x * blockDim.x) {
        const size_t row = i / history16, k = i % history16;
        dst[row * row_stride16 + k] = src[row * row_stride16 + nsamples16 + k];
    }
}

int grid_for(size_t work, int block)
{
    size_t g = (work + block - 1) / block;
    if(g > 148 * 32) g = 148 * 32;
    return (int)(g ? g : 1);
}

}  // namespace
}  // namespace swb

using namespace swb;

extern "C" {

int sw_transpose_ftpa(const void* d_taftp, void* d_ftpa, int nheaps,
                      int input_nantennas, int output_nantennas, int nchans,
                      sw_stream_t stream)
{
    SW_REQUIRE(d_taftp && d_ftpa, "sw_transpose_ftpa: null pointer");
    SW_REQUIRE(nheaps > 0 && nchans > 0, "sw_transpose_ftpa: empty input");
    SW_REQUIRE(input_nantennas > 0 && input_nantennas <= output_nantennas,
               "Input number of antennas must be <= to the maximum nantennas");
    SW_REQUIRE(output_nantennas % 8 == 0 && output_nantennas <= 256,
               "sw_transpose_ftpa: output antennas must be a multiple of 8 and <= 256");
    SW_REQUIRE(nheaps <= 65535 && nchans <= 65535, "sw_transpose_ftpa: grid too large");
    const size_t smem = (size_t)input_nantennas * kHeap * 4;
    SW_CUDA_CHECK(cudaFuncSetAttribute(transpose_ftpa_k,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    dim3 grid(nheaps, nchans);
    transpose_ftpa_k<<<grid, 256, smem, as_cuda(stream)>>>(
        static_cast<const uint4*>(d_taftp), static_cast<uint4*>(d_ftpa),
        input_nantennas, output_nantennas, nchans, nheaps);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

int sw_transpose_fpact(const void* d_taftp, void* d_fpact, int nheaps,
                       int input_nantennas, int output_nantennas, int nchans,
                       size_t row_stride, size_t sample_offset,
                       sw_stream_t stream)
{
    SW_REQUIRE(d_taftp && d_fpact, "sw_transpose_fpact: null pointer");
    SW_REQUIRE(nheaps > 0 && nchans > 0, "sw_transpose_fpact: empty input");
    SW_REQUIRE(input_nantennas > 0 && input_nantennas <= output_nantennas,
               "Input number of antennas must be <= to the maximum nantennas");
    SW_REQUIRE(row_stride % 16 == 0 && sample_offset % 16 == 0,
               "sw_transpose_fpact: row stride and offset must be multiples of 16");
    SW_REQUIRE(sample_offset + (size_t)nheaps * kHeap <= row_stride,
               "sw_transpose_fpact: rows too short for the gulp");
    SW_REQUIRE(nheaps <= 65535 && nchans <= 65535, "sw_transpose_fpact: grid too large");
    dim3 grid(nheaps, nchans);
    transpose_fpact_k<<<grid, 256, 0, as_cuda(stream)>>>(
        static_cast<const uint4*>(d_taftp), static_cast<uint8_t*>(d_fpact),
        input_nantennas, output_nantennas, nchans, row_stride, sample_offset);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

static int convert(const void* ftpa, void* fpact, int nchans, int nsamples,
                   int nant, size_t row_stride, size_t off, sw_stream_t stream,
                   int to_fpact)
{
    SW_REQUIRE(ftpa && fpact, "FTPA/FPACT conversion: null pointer");
    SW_REQUIRE(nsamples > 0 && nchans > 0 && nant > 0, "FTPA/FPACT conversion: empty shape");
    SW_REQUIRE(off + nsamples <= row_stride, "FTPA/FPACT conversion: rows too short");
    const size_t work = (size_t)nchans * kPol * nant * 2 * ((nsamples + 3) / 4);
    ftpa_to_fpact_k<<<grid_for(work, 256), 256, 0, as_cuda(stream)>>>(
        static_cast<const int8_t*>(ftpa), static_cast<int8_t*>(fpact), nchans,
        nsamples, nant, row_stride, off, to_fpact);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

int sw_ftpa_to_fpact(const void* d_ftpa, void* d_fpact, int nchans,
                     int nsamples, int nantennas, size_t row_stride,
                     size_t sample_offset, sw_stream_t stream)
{
    return convert(d_ftpa, d_fpact, nchans, nsamples, nantennas, row_stride,
                   sample_offset, stream, 1);
}

int sw_fpact_to_ftpa(const void* d_fpact, void* d_ftpa, int nchans,
                     int nsamples, int nantennas, size_t row_stride,
                     size_t sample_offset, sw_stream_t stream)
{
    return convert(d_ftpa, const_cast<void*>(d_fpact), nchans, nsamples,
                   nantennas, row_stride, sample_offset, stream, 0);
}

int sw_fpact_keep_history(void* d_fpact, size_t nrows, size_t row_stride,
                          size_t history, sw_stream_t stream)
{
    SW_REQUIRE(d_fpact, "sw_fpact_keep_history: null pointer");
    SW_REQUIRE(row_stride % 16 == 0 && history % 16 == 0,
               "sw_fpact_keep_history: stride and history must be multiples of 16");
    if(history == 0 || nrows == 0) return SW_OK;
    SW_REQUIRE(row_stride >= 2 * history,
               "sw_fpact_keep_history: rows must hold at least twice the history");
    // rows hold [history | nsamples] with nsamples = row_stride - history
    const size_t nsamples = row_stride - history;
    const size_t work = nrows * (history / 16);
    keep_history_k<<<grid_for(work, 256), 256, 0, as_cuda(stream)>>>(
        static_cast<const uint4*>(d_fpact), static_cast<uint4*>(d_fpact), nrows,
        row_stride / 16, history / 16, nsamples / 16);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

int sw_fpact_copy_history(const void* d_prev, void* d_next, size_t nrows, size_t row_stride,
                          size_t history, sw_stream_t stream)
{
    SW_REQUIRE(d_prev && d_next, "sw_fpact_copy_history: null pointer");
    SW_REQUIRE(row_stride % 16 == 0 && history % 16 == 0 &&
                   (reinterpret_cast<uintptr_t>(d_prev) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(d_next) & 15) == 0,
               "sw_fpact_copy_history: pointers, stride and history must be multiples of 16");
    if(history == 0 || nrows == 0) return SW_OK;
    SW_REQUIRE(row_stride >= 2 * history,
               "sw_fpact_copy_history: rows must hold at least twice the history");
    const size_t nsamples = row_stride - history;
    const size_t work = nrows * (history / 16);
    keep_history_k<<<grid_for(work, 256), 256, 0, as_cuda(stream)>>>(
        static_cast<const uint4*>(d_prev), static_cast<uint4*>(d_next), nrows,
        row_stride / 16, history / 16, nsamples / 16);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

}  // extern "C"
