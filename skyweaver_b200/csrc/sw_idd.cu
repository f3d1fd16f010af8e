// IncoherentDedisperser on the B200
// (cpp/skyweaver/src/IncoherentDedisperser.cu:66-125, a host OpenMP loop in
// the reference).
//
// out[t', d, b] = clamp(sum_{tau < ts} sum_f in[t + tau - delay[d,f], f, b]
//                       / scale_factor),   t = max_delay + t' * ts
// with truncation toward zero (types.cuh:211-221).  The int8 sums are exact
// integers (the reference accumulates them in float, exact below 2^24), so
// the kernels sum bytes in int32 with dp4a: dp4a(word, 1 << 8b, acc) adds
// beam b of a 32-bit word of 4 beams, and on byte-transposed words one dp4a
// adds two or four channels of one beam.  (Biasing each word to unsigned and
// adding pairs of 16-bit lanes, two per instruction, measured 8 % slower
// than one dp4a per addition: it needs a xor and two byte permutes per word
// on the pipe that also issues the adds.)  The final float divide is the
// reference's single IEEE division.
#include "sw_common.cuh"

namespace swb {
namespace {

// One CTA = (trial DM, output sample, block of 128 beam quads).  The linear
// block index runs over the DMs of a group of `group` DMs fastest, then
// output samples, then beam-quad blocks, then DM groups, so the CTAs resident
// at any moment are neighbouring DMs at neighbouring times of one 512-beam
// block: they read nearly the same (time - delay) rows of every channel, a
// window that fits in L2, instead of streaming the rows from HBM once per DM.
__global__ void __launch_bounds__(128)
idd_k(const uint32_t* __restrict__ tfb, int nchans, int nquads,
      const int* __restrict__ delays, int max_delay, int tscrunch,
      float scale_factor, uint32_t* __restrict__ tdb, int ndms, int nout,
      int nqb, int group, long long blk0)
{
    long long blk = blk0 + blockIdx.x;
    const int dl = (int)(blk % group);
    blk /= group;
    const int to = (int)(blk % nout);
    blk /= nout;
    const int qb = (int)(blk % nqb);
    const int d  = (int)(blk / nqb) * group + dl;
    const int q  = qb * blockDim.x + threadIdx.x;
    if(d >= ndms || q >= nquads) return;
    const int t = max_delay + to * tscrunch;
    const int* dl_f = delays + (size_t)d * nchans;
    int acc[4] = {0, 0, 0, 0};
    for(int tau = 0; tau < tscrunch; ++tau) {
#pragma unroll 4
        for(int f = 0; f < nchans; ++f) {
            const size_t row = (size_t)(t + tau - dl_f[f]) * nchans + f;
            const int w = (int)tfb[row * nquads + q];
#pragma unroll
            for(int b = 0; b < 4; ++b) acc[b] = __dp4a(w, 1 << (8 * b), acc[b]);
        }
    }
    uint32_t packed = 0;
#pragma unroll
    for(int k = 0; k < 4; ++k) {
        const float v = fdiv((float)acc[k], scale_factor);
        packed |= ((uint32_t)(uint8_t)clamp_i8(v)) << (8 * k);
    }
    tdb[((size_t)to * ndms + d) * nquads + q] = packed;
}

// Same sums, 16 beams per thread (one 16-byte load per row): the per-load
// address work is shared by 16 beams and each channel's row offset comes
// from a per-CTA table in shared memory.  Needs nbeams % 16 == 0 and 16-byte
// aligned buffers.  A CTA is 128 threads = `tpc` consecutive output samples
// x `lw` lanes of 16 beams (lw <= 32: at most 512 beams), one trial DM.
// Block order as idd_k (DMs of a group fastest, then output chunks, then
// beam blocks, then DM groups), so the CTAs resident at any moment read the
// (time - delay) rows of one 512-beam block, a working set that mostly stays
// in L2.  (All 2048 beams per CTA measured a 38 % L2 hit rate and HBM reads
// of 22x the input; on 4096 samples x 128 DMs x 2048 beams x 256 channels,
// 64/128/256/512/1024/2048 beams per CTA took 44/31/21/20/24/29 ms, and two
// 16-byte loads per thread instead of one 129 -> 154 ms.)
//
// Fewer multiply-add instructions than one dp4a per addition: the words of
// four channels for the same four beams are byte-transposed with PRMT
// (integer ALU pipe) so that one dp4a adds two or four channels of a beam.
// Pair form (words of channels f, f+1 -> [a0 b0 a1 b1], [a2 b2 a3 b3]): 2
// PRMT + 4 dp4a per 8 additions; full form (a second PRMT stage -> [a0 b0 c0
// d0] ...): 8 PRMT + 4 dp4a per 16.  The first NT of the four words of each
// 16-byte load take the full form, the rest the pair form, which splits the
// work between the ALU and the multiply-add pipes.  Channels past the last
// multiple of 4 take one dp4a per addition.  On the case above: one dp4a
// per addition (12 CTAs per SM) 17.3 ms; NT = 0..4 with 8 CTAs per SM 16.3,
// 15.4, 14.9, 15.6, 15.3 ms; NT = 2 with 10 CTAs per SM 14.8 ms, with 12
// (register spills) 23.6 ms.  L2 bandwidth then bounds it: every addition
// reads its byte from L2.
template <int NT, int MINB>
__global__ void __launch_bounds__(128, MINB)
idd16q_k(const uint4* __restrict__ tfb, int nchans, int nq16,
         const int* __restrict__ delays, int max_delay, int tscrunch,
         float scale_factor, uint4* __restrict__ tdb, int ndms, int nout,
         int nqb, int group, int lw, int ntc, long long blk0)
{
    extern __shared__ long long s_off[];  // [nchans] row offsets in uint4 units
    long long blk = blk0 + blockIdx.x;
    const int dl = (int)(blk % group);
    blk /= group;
    const int tc = (int)(blk % ntc);
    blk /= ntc;
    const int qb = (int)(blk % nqb);
    const int d  = (int)(blk / nqb) * group + dl;
    if(d >= ndms) return;  // uniform across the CTA
    const int tpc = blockDim.x / lw;
    const int to = tc * tpc + (int)threadIdx.x / lw;
    const int* dl_f = delays + (size_t)d * nchans;
    const long long row = (long long)nchans * nq16;  // uint4 per time sample
    for(int f = threadIdx.x; f < nchans; f += blockDim.x)
        s_off[f] = (long long)f * nq16 - (long long)dl_f[f] * row;
    __syncthreads();
    const int q = qb * lw + (int)threadIdx.x % lw;  // uint4 of this thread
    if((int)threadIdx.x >= tpc * lw || q >= nq16 || to >= nout) return;
    const int t = max_delay + to * tscrunch;
    int acc[16];
#pragma unroll
    for(int k = 0; k < 16; ++k) acc[k] = 0;
    const int nc4 = nchans & ~3;
    for(int tau = 0; tau < tscrunch; ++tau) {
        const uint4* bt = tfb + (long long)(t + tau) * row + q;
#pragma unroll 2
        for(int f = 0; f < nc4; f += 4) {
            const uint4 va = bt[s_off[f]];
            const uint4 vb = bt[s_off[f + 1]];
            const uint4 vc = bt[s_off[f + 2]];
            const uint4 vd = bt[s_off[f + 3]];
            const uint32_t wa[4] = {va.x, va.y, va.z, va.w};
            const uint32_t wb[4] = {vb.x, vb.y, vb.z, vb.w};
            const uint32_t wc[4] = {vc.x, vc.y, vc.z, vc.w};
            const uint32_t wd[4] = {vd.x, vd.y, vd.z, vd.w};
#pragma unroll
            for(int k = 0; k < 4; ++k) {
                const int t0 = (int)__byte_perm(wa[k], wb[k], 0x5140);  // a0 b0 a1 b1
                const int t1 = (int)__byte_perm(wa[k], wb[k], 0x7362);  // a2 b2 a3 b3
                const int t2 = (int)__byte_perm(wc[k], wd[k], 0x5140);  // c0 d0 c1 d1
                const int t3 = (int)__byte_perm(wc[k], wd[k], 0x7362);  // c2 d2 c3 d3
                int* a = acc + 4 * k;
                if(k < NT) {
                    a[0] = __dp4a((int)__byte_perm(t0, t2, 0x5410), 0x01010101, a[0]);
                    a[1] = __dp4a((int)__byte_perm(t0, t2, 0x7632), 0x01010101, a[1]);
                    a[2] = __dp4a((int)__byte_perm(t1, t3, 0x5410), 0x01010101, a[2]);
                    a[3] = __dp4a((int)__byte_perm(t1, t3, 0x7632), 0x01010101, a[3]);
                } else {
                    a[0] = __dp4a(t2, 0x00000101, __dp4a(t0, 0x00000101, a[0]));
                    a[1] = __dp4a(t2, 0x01010000, __dp4a(t0, 0x01010000, a[1]));
                    a[2] = __dp4a(t3, 0x00000101, __dp4a(t1, 0x00000101, a[2]));
                    a[3] = __dp4a(t3, 0x01010000, __dp4a(t1, 0x01010000, a[3]));
                }
            }
        }
        for(int f = nc4; f < nchans; ++f) {
            const uint4 v = bt[s_off[f]];
            const int w[4] = {(int)v.x, (int)v.y, (int)v.z, (int)v.w};
#pragma unroll
            for(int k = 0; k < 4; ++k)
#pragma unroll
                for(int b = 0; b < 4; ++b)
                    acc[4 * k + b] = __dp4a(w[k], 1 << (8 * b), acc[4 * k + b]);
        }
    }
    uint32_t packed[4];
#pragma unroll
    for(int k = 0; k < 4; ++k) {
        packed[k] = 0;
#pragma unroll
        for(int b = 0; b < 4; ++b) {
            const float v = fdiv((float)acc[4 * k + b], scale_factor);
            packed[k] |= ((uint32_t)(uint8_t)clamp_i8(v)) << (8 * b);
        }
    }
    tdb[((size_t)to * ndms + d) * nq16 + q] =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
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
    const int nquads = nbeams / 4;
    const bool wide = nbeams % 16 == 0 && (reinterpret_cast<uintptr_t>(d_tfb) & 15) == 0 &&
                      (reinterpret_cast<uintptr_t>(d_tdb) & 15) == 0 &&
                      (size_t)nchans * sizeof(long long) <= 48 * 1024;
    const int nlanes = wide ? nbeams / 16 : nquads;  // threads per (DM, sample)
    // wide: CTAs of (128 / lw) output samples x lw lanes of 16 beams
    const int lw = wide ? (nlanes < 32 ? nlanes : 32) : 128;
    const int nqb = swb::cdiv(nlanes, lw);
    const int ntc = wide ? swb::cdiv(nout, 128 / lw) : nout;
    const int group = ndms < 16 ? ndms : 16;
    const long long ngroups = swb::cdiv(ndms, group);
    const long long total = ngroups * ntc * nqb * group;
    const long long chunk = 1ll << 30;  // blocks per launch (grid.x limit 2^31 - 1)
    for(long long b0 = 0; b0 < total; b0 += chunk) {
        const long long n = total - b0 < chunk ? total - b0 : chunk;
        if(wide)  // two of four words transposed in full, 10 CTAs per SM
            swb::idd16q_k<2, 10><<<(unsigned)n, 128, nchans * sizeof(long long), swb::as_cuda(stream)>>>(
                reinterpret_cast<const uint4*>(d_tfb), nchans, nbeams / 16, d_delays, max_delay,
                tscrunch, scale_factor, reinterpret_cast<uint4*>(d_tdb), ndms, nout, nqb,
                group, lw, ntc, b0);
        else
            swb::idd_k<<<(unsigned)n, 128, 0, swb::as_cuda(stream)>>>(
                reinterpret_cast<const uint32_t*>(d_tfb), nchans, nquads, d_delays, max_delay,
                tscrunch, scale_factor, reinterpret_cast<uint32_t*>(d_tdb), ndms, nout, nqb,
                group, b0);
        SW_LAUNCH_CHECK();
    }
    return SW_OK;
}
