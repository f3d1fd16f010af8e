// IncoherentBeamformer on the B200
// (cpp/skyweaver/src/IncoherentBeamformer.cu:15-91; CPU form
//  cpp/skyweaver/test/src/IncoherentBeamformerTester.cu:41-103).
//
// P[s,t',f] = sum_{t in t'} sum_a w[s,a] * Stokes(v_p0, v_p1)  (float, in the
// reference's (t outer, a inner) order), then int8 = clamp(rint(rescale)).
//
// Every Stokes term of int8 voltages is an exact integer, so when the
// antenna weights are integers the float chain is exact as long as the sum
// of |terms| stays below 2^24.  The kernel therefore sums the terms with
// dp4a in integers, checks that bound, and only walks the float chain in the
// reference order (slow path) for outputs that fail it.  The result is
// bit-identical to the reference's CPU implementation in both cases.
//
// One thread per (channel, output sample); the planar FPACT rows make each
// thread's tscrunch samples a contiguous 4/8/16-byte load, coalesced across
// the warp.  The kernel is HBM bound (one read of the voltages).
#include "sw_common.cuh"

namespace swb {
namespace {

constexpr int kMaxBs = 8;          // beamsets per pass (registers)
constexpr int kMaxAnt = 256;
constexpr int kTableAnt = 64;  // antennas of the float-chain product table (4 KB a thread)

// signed byte k (0..15, unrolled) of a 16-byte load
__device__ __forceinline__ int sbyte(const uint4& v, int k)
{
    const uint32_t w = k < 4 ? v.x : k < 8 ? v.y : k < 12 ? v.z : v.w;
    return (int)(int8_t)(w >> (8 * (k & 3)));
}

struct IbArgs {
    const uint8_t* fpact;
    size_t row_stride, offset;
    int nchans, nsamples, nant, tscrunch, nbeamsets, stokes;
    const float *scale, *offset_v, *weights;
    float* raw;
    int8_t* out;
    const int* chan_order;  // CTA row -> channel (nullptr: identity)
};

__device__ __forceinline__ float stokes_f(int stokes, float r0, float i0,
                                          float r1, float i1)
{
    // beamformer_utils.cuh:125-140 with the reference's op order
    switch(stokes) {
    case 0: return fadd(fadd(fmul(r0, r0), fmul(i0, i0)), fadd(fmul(r1, r1), fmul(i1, i1)));
    case 1: return fsub(fadd(fmul(r0, r0), fmul(i0, i0)), fadd(fmul(r1, r1), fmul(i1, i1)));
    case 2: return fmul(2.0f, fsub(fmul(r0, r1), fmul(i0, -i1)));
    default: return fmul(2.0f, fadd(fmul(r0, -i1), fmul(i0, r1)));
    }
}

// NC = 1: one Stokes parameter (args.stokes); NC = 4: I, Q, U, V
// (FullStokesBeamformerTraits, beamformer_utils.cuh:198-278: float4 raw power,
// char4 output, component c computed exactly like single-Stokes mode c).
template <int NC>
__global__ void __launch_bounds__(128)
ib_k(IbArgs args, int bs0)
{
    constexpr int kBs = kMaxBs / NC;  // beamsets per pass
    __shared__ float sw[kBs][kMaxAnt];
    __shared__ int s_intw[kBs];
    const int nbs = min(kBs, args.nbeamsets - bs0);
    for(int i = threadIdx.x; i < kBs * args.nant; i += blockDim.x) {
        const int s = i / args.nant, a = i % args.nant;
        sw[s][a] = (s < nbs) ? args.weights[(size_t)(bs0 + s) * args.nant + a] : 0.0f;
    }
    __syncthreads();
    if(threadIdx.x < kBs) {
        int ok = 1;
        for(int a = 0; a < args.nant; ++a) {
            const float w = sw[threadIdx.x][a];
            ok &= (w == rintf(w)) && fabsf(w) <= 1024.0f;
        }
        s_intw[threadIdx.x] = ok;
    }
    __syncthreads();

    const int nout = args.nsamples / args.tscrunch;
    const int tp = blockIdx.x * blockDim.x + threadIdx.x;
    const int f  = args.chan_order ? args.chan_order[blockIdx.y] : (int)blockIdx.y;
    if(tp >= nout) return;
    const int t0 = tp * args.tscrunch;
    const size_t P = 2;
    long long S[kBs * NC], B[kBs];
#pragma unroll
    for(int s = 0; s < kBs; ++s) {
        B[s] = 0;
#pragma unroll
        for(int c = 0; c < NC; ++c) S[s * NC + c] = 0;
    }

    const bool words = (args.tscrunch % 4) == 0;
    // 16-byte loads when each thread's samples are whole aligned 16-byte runs
    const bool quads = (args.tscrunch % 16) == 0 && (args.row_stride % 16) == 0 &&
                       (args.offset % 16) == 0 &&
                       (reinterpret_cast<uintptr_t>(args.fpact) & 15) == 0;
#pragma unroll 2  // two antennas' loads in flight: 3 % faster on 64 channels
    for(int a = 0; a < args.nant; ++a) {
        const uint8_t* r0 = args.fpact + (((size_t)f * P + 0) * args.nant + a) * 2 * args.row_stride + args.offset + t0;
        const uint8_t* r1 = args.fpact + (((size_t)f * P + 1) * args.nant + a) * 2 * args.row_stride + args.offset + t0;
        int pI = 0, pQ = 0, pU = 0, pV = 0;
        if(quads) {
            for(int k = 0; k < args.tscrunch; k += 16) {
                const uint4 R0 = *reinterpret_cast<const uint4*>(r0 + k);
                const uint4 I0 = *reinterpret_cast<const uint4*>(r0 + args.row_stride + k);
                const uint4 R1 = *reinterpret_cast<const uint4*>(r1 + k);
                const uint4 I1 = *reinterpret_cast<const uint4*>(r1 + args.row_stride + k);
                const int xr0[4] = {(int)R0.x, (int)R0.y, (int)R0.z, (int)R0.w};
                const int xi0[4] = {(int)I0.x, (int)I0.y, (int)I0.z, (int)I0.w};
                const int xr1[4] = {(int)R1.x, (int)R1.y, (int)R1.z, (int)R1.w};
                const int xi1[4] = {(int)I1.x, (int)I1.y, (int)I1.z, (int)I1.w};
#pragma unroll
                for(int q = 0; q < 4; ++q) {
                    const int e0 = __dp4a(xi0[q], xi0[q], __dp4a(xr0[q], xr0[q], 0));
                    const int e1 = __dp4a(xi1[q], xi1[q], __dp4a(xr1[q], xr1[q], 0));
                    pI += e0 + e1;
                    pQ += e0 - e1;
                    pU += __dp4a(xi0[q], xi1[q], __dp4a(xr0[q], xr1[q], 0));
                    pV += __dp4a(xi0[q], xr1[q], 0) - __dp4a(xr0[q], xi1[q], 0);
                }
            }
        } else if(words) {
            for(int k = 0; k < args.tscrunch; k += 4) {
                const int xr0 = *reinterpret_cast<const int*>(r0 + k);
                const int xi0 = *reinterpret_cast<const int*>(r0 + args.row_stride + k);
                const int xr1 = *reinterpret_cast<const int*>(r1 + k);
                const int xi1 = *reinterpret_cast<const int*>(r1 + args.row_stride + k);
                const int e0 = __dp4a(xi0, xi0, __dp4a(xr0, xr0, 0));
                const int e1 = __dp4a(xi1, xi1, __dp4a(xr1, xr1, 0));
                pI += e0 + e1;
                pQ += e0 - e1;
                pU += __dp4a(xi0, xi1, __dp4a(xr0, xr1, 0));
                pV += __dp4a(xi0, xr1, 0) - __dp4a(xr0, xi1, 0);
            }
        } else {
            for(int k = 0; k < args.tscrunch; ++k) {
                const int xr0 = (int8_t)r0[k], xi0 = (int8_t)r0[args.row_stride + k];
                const int xr1 = (int8_t)r1[k], xi1 = (int8_t)r1[args.row_stride + k];
                const int e0 = xr0 * xr0 + xi0 * xi0, e1 = xr1 * xr1 + xi1 * xi1;
                pI += e0 + e1;
                pQ += e0 - e1;
                pU += xr0 * xr1 + xi0 * xi1;
                pV += xi0 * xr1 - xr0 * xi1;
            }
        }
        int pv[NC];
        if constexpr(NC == 4) {
            pv[0] = pI; pv[1] = pQ; pv[2] = 2 * pU; pv[3] = 2 * pV;
        } else {
            pv[0] = args.stokes == 0 ? pI : args.stokes == 1 ? pQ
                  : args.stokes == 2 ? 2 * pU : 2 * pV;
        }
#pragma unroll
        for(int s = 0; s < kBs; ++s) {
            const int wi = (int)sw[s][a];
#pragma unroll
            for(int c = 0; c < NC; ++c) S[s * NC + c] += (long long)wi * pv[c];
            B[s] += (long long)abs(wi) * pI;  // |Q|,|U|,|V| <= I per sample
        }
    }

    for(int s = 0; s < nbs; ++s) {
        const int bs = bs0 + s;
        const size_t o  = ((size_t)bs * nout + tp) * args.nchans + f;
        const size_t so = (size_t)bs * args.nchans + f;
        for(int c = 0; c < NC; ++c) {
            const int stokes = NC == 4 ? c : args.stokes;
            float power;
            if(s_intw[s] && B[s] <= (1ll << 24)) {
                power = (float)S[s * NC + c];  // the float chain is exact
            } else if(quads && args.nant <= kTableAnt) {
                // reference order (t outer, a inner) from a table of the
                // products: each antenna's four 16-sample rows are read once
                // with 16-byte loads, the 16 x nant products go to a
                // per-thread table in local memory (lane-interleaved, so
                // coalesced and mostly L1/L2 resident), and the chain then
                // walks the table.  Walking the rows byte by byte in chain
                // order instead re-reads every row once per sample, because
                // the warp's 4 rows x nant windows do not stay in L1.
                power = 0.0f;
                for(int tc = 0; tc < args.tscrunch; tc += 16) {
                    float x[16][kTableAnt];
#pragma unroll 4
                    for(int a = 0; a < args.nant; ++a) {
                        const uint8_t* q0 = args.fpact + (((size_t)f * P + 0) * args.nant + a) * 2 * args.row_stride + args.offset + t0 + tc;
                        const uint8_t* q1 = args.fpact + (((size_t)f * P + 1) * args.nant + a) * 2 * args.row_stride + args.offset + t0 + tc;
                        const uint4 R0 = *reinterpret_cast<const uint4*>(q0);
                        const uint4 I0 = *reinterpret_cast<const uint4*>(q0 + args.row_stride);
                        const uint4 R1 = *reinterpret_cast<const uint4*>(q1);
                        const uint4 I1 = *reinterpret_cast<const uint4*>(q1 + args.row_stride);
                        const float w = sw[s][a];
#pragma unroll
                        for(int k = 0; k < 16; ++k)
                            x[k][a] = fmul(stokes_f(stokes, (float)sbyte(R0, k), (float)sbyte(I0, k),
                                                    (float)sbyte(R1, k), (float)sbyte(I1, k)),
                                           w);
                    }
                    for(int k = 0; k < 16; ++k)
                        for(int a = 0; a < args.nant; ++a) power = fadd(power, x[k][a]);
                }
            } else {
                // reference order: t outer, a inner, float multiply and add
                power = 0.0f;
                for(int t = t0; t < t0 + args.tscrunch; ++t)
                    for(int a = 0; a < args.nant; ++a) {
                        const uint8_t* q0 = args.fpact + (((size_t)f * P + 0) * args.nant + a) * 2 * args.row_stride + args.offset + t;
                        const uint8_t* q1 = args.fpact + (((size_t)f * P + 1) * args.nant + a) * 2 * args.row_stride + args.offset + t;
                        const float st = stokes_f(stokes, (float)(int8_t)q0[0],
                                                  (float)(int8_t)q0[args.row_stride],
                                                  (float)(int8_t)q1[0],
                                                  (float)(int8_t)q1[args.row_stride]);
                        power = fadd(power, fmul(st, sw[s][a]));
                    }
            }
            args.raw[o * NC + c] = power;
            const float sc = stokes == 0
                                 ? rintf(fdiv(fsub(power, args.offset_v[so]), args.scale[so]))
                                 : rintf(fdiv(power, args.scale[so]));
            args.out[o * NC + c] = clamp_i8(sc);
        }
    }
}

}  // namespace

int launch_incoherent_beamform(const void* d_fpact, size_t row_stride,
                               size_t sample_offset, int nchans, int nsamples,
                               int nant, int tscrunch, const float* d_scale,
                               const float* d_offset,
                               const float* d_beamset_weights, int nbeamsets,
                               int stokes, float* d_raw, int8_t* d_out,
                               cudaStream_t stream, const int* d_chan_order)
{
    SW_REQUIRE(d_fpact && d_scale && d_offset && d_beamset_weights && d_raw && d_out,
               "sw_incoherent_beamform: null pointer");
    SW_REQUIRE(nbeamsets > 0, "Number of beamsets must be greater than zero");
    SW_REQUIRE(nant > 0 && nant <= kMaxAnt, "sw_incoherent_beamform: bad antenna count");
    SW_REQUIRE(tscrunch > 0 && nsamples % tscrunch == 0,
               "sw_incoherent_beamform: nsamples must be a multiple of tscrunch");
    SW_REQUIRE(stokes >= 0 && stokes <= 4, "sw_incoherent_beamform: bad Stokes mode");
    SW_REQUIRE(tscrunch % 4 != 0 || (row_stride % 4 == 0 && sample_offset % 4 == 0 &&
                                     (reinterpret_cast<uintptr_t>(d_fpact) & 3) == 0),
               "sw_incoherent_beamform: with tscrunch a multiple of 4 the voltage pointer, "
               "row stride and sample offset must be multiples of 4 bytes");
    SW_REQUIRE(nchans > 0 && nchans <= 65535, "sw_incoherent_beamform: bad channel count");
    IbArgs args{static_cast<const uint8_t*>(d_fpact), row_stride, sample_offset,
                nchans, nsamples, nant, tscrunch, nbeamsets, stokes, d_scale,
                d_offset, d_beamset_weights, d_raw, d_out, d_chan_order};
    const int nout = nsamples / tscrunch;
    dim3 grid(cdiv(nout, 128), nchans);
    if(stokes == 4) {
        for(int bs0 = 0; bs0 < nbeamsets; bs0 += kMaxBs / 4) {
            ib_k<4><<<grid, 128, 0, stream>>>(args, bs0);
            SW_LAUNCH_CHECK();
        }
    } else {
        for(int bs0 = 0; bs0 < nbeamsets; bs0 += kMaxBs) {
            ib_k<1><<<grid, 128, 0, stream>>>(args, bs0);
            SW_LAUNCH_CHECK();
        }
    }
    return SW_OK;
}

namespace {

// Channels in descending order of voltage power (sum over pols and antennas
// of mean^2 + std^2, from the statistics stage).  The incoherent beam maps
// its CTA rows through this order, so the channels most likely to need the
// float chain (RFI-saturated ones, whose CTAs take longest) start first and
// overlap the others instead of trailing behind them.  Ties go by channel
// index and a NaN power counts as lowest, so the order is a permutation.
__global__ void ib_channel_order_k(const float4* __restrict__ stats, int nchans, int npa,
                                   int* __restrict__ order)
{
    extern __shared__ float pw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for(int c = warp; c < nchans; c += nwarps) {  // one warp per channel
        float s = 0.0f;
        for(int i = lane; i < npa; i += 32) {
            const float4 v = stats[(size_t)c * npa + i];
            s += v.x * v.x + v.y * v.y;
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if(lane == 0) pw[c] = isnan(s) ? -1.0f : s;
    }
    __syncthreads();
    for(int c = threadIdx.x; c < nchans; c += blockDim.x) {
        int r = 0;
        for(int k = 0; k < nchans; ++k) r += (pw[k] > pw[c]) || (pw[k] == pw[c] && k < c);
        order[r] = c;
    }
}

}  // namespace

int launch_ib_channel_order(const float* d_stats, int nchans, int npol, int nant,
                            int* d_order, cudaStream_t stream)
{
    SW_REQUIRE(d_stats && d_order, "ib channel order: null pointer");
    SW_REQUIRE(nchans > 0 && nchans <= kIbOrderMaxChans, "ib channel order: bad channel count");
    ib_channel_order_k<<<1, 256, nchans * sizeof(float), stream>>>(
        reinterpret_cast<const float4*>(d_stats), nchans, npol * nant, d_order);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

}  // namespace swb

extern "C" int sw_incoherent_beamform(const void* d_fpact, size_t row_stride,
                                      size_t sample_offset, int nchans,
                                      int nsamples, int nant, int tscrunch,
                                      const float* d_scale, const float* d_offset,
                                      const float* d_beamset_weights,
                                      int nbeamsets, int stokes, float* d_raw,
                                      int8_t* d_out, sw_stream_t stream)
{
    return swb::launch_incoherent_beamform(
        d_fpact, row_stride, sample_offset, nchans, nsamples, nant, tscrunch,
        d_scale, d_offset, d_beamset_weights, nbeamsets, stokes, d_raw, d_out,
        swb::as_cuda(stream), nullptr);
}
