// CoherentDedisperser on the B200.
//
// Reference: cpp/skyweaver/src/CoherentDedisperser.cu:142-225 (per channel:
// int8 -> complex64, cuFFT forward, chirp multiply, cuFFT inverse, trim
// overlap/2 each side, /N, round, int8 wrap) with the chirp of
// DMResponse (:293-336) and the golden-vector generator
// python/skyweaver_test_utils/dedisperse.py:58-80,143-173.
//
// B200 design: one CTA transforms one overlap-save segment of one
// (channel, pol, antenna) stream entirely in shared memory and registers:
//   * the forward FFT is an in-place mixed-radix decimation-in-frequency
//     FFT (first pass radix 2/4/8/16 read straight from the planar int8
//     rows, then radix-16 passes); its last pass leaves each thread's 16
//     spectral bins in registers, in digit-reversed order;
//   * for every coherent DM the thread multiplies those bins by the chirp
//     (FP64 phases, stored as complex float in the same digit-reversed
//     order), runs the exact inverse passes (decimation in time, conjugate
//     twiddles) and the last pass writes the trimmed, scaled, rounded and
//     int8-wrapped samples straight to the planar output rows.
// So the forward transform is done once per segment for all DMs, there is
// no spectrum in HBM, and all global traffic is coalesced byte rows.
//
// Trim.  The reference trims overlap/2 samples at each end of a window.  Its
// chirp's impulse response is one-sided (nearly all of it at lags 0 .. the
// intra-channel smear), so a window here trims `overlap - lag` samples at its
// start (the causal part) and `lag` at its end (the short anti-causal part);
// output sample m is the dedispersed voltage at gulp position m - lag.
// lag = overlap / 2 is the reference's own per-window trim.
// Twiddles come from per-pass tables (FP64-computed) staged in shared
// memory; FFT arithmetic is FP32.
#include <algorithm>

#include "sw_common.cuh"

namespace swb {
namespace cdd {

constexpr int kMaxDms = 64;

// ---------------------------------------------------------------- plan
struct Plan {
    int logn, n, r0, npass;
    int radix[8];
    int span[8];    // G_p
    int stride[8];  // s_p = G_p / R_p
    int tw_off[8];  // offset (complex entries) of pass p's table
    int tw_total;
};

__host__ __device__ constexpr Plan make_plan(int logn)
{
    Plan P{};
    P.logn = logn;
    P.n    = 1 << logn;
    const int rem = logn % 4;
    P.r0 = rem ? (1 << rem) : 16;
    int g = P.n, off = 0, p = 0;
    int r = P.r0;
    while(g > 1) {
        P.radix[p]  = r;
        P.span[p]   = g;
        P.stride[p] = g / r;
        P.tw_off[p] = off;
        // radix-16 tables hold twiddle pairs (w1,w2),(w3,w4),..,(w15,0) per j,
        // read with one 16-byte load per pair; other radices hold w1..w(R-1)
        if(P.stride[p] > 1) off += (r == 16 ? 16 : r - 1) * P.stride[p];
        g /= r;
        r = 16;
        ++p;
    }
    P.npass    = p;
    P.tw_total = off;
    return P;
}

// DIF output position -> natural frequency bin
__host__ __device__ inline int digit_reverse(const Plan& P, int pos)
{
    int k = 0, mult = 1;
    for(int p = 0; p < P.npass; ++p) {
        const int q = (pos / P.stride[p]) % P.radix[p];
        k += q * mult;
        mult *= P.radix[p];
    }
    return k;
}

// ------------------------------------------------------- complex helpers
struct c32 {
    float x, y;
};
__device__ __forceinline__ c32 cadd(c32 a, c32 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ c32 csub(c32 a, c32 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ c32 cmul(c32 a, c32 b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__device__ __forceinline__ c32 cmulc(c32 a, c32 b)  // a * conj(b)
{
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ c32 rot90(c32 a)
{
    return INV ? c32{-a.y, a.x} : c32{a.y, -a.x};
}

template <bool INV>
__device__ __forceinline__ void dft2(c32* x)
{
    c32 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(c32& x0, c32& x1, c32& x2, c32& x3)
{
    const c32 t0 = cadd(x0, x2), t1 = csub(x0, x2);
    const c32 t2 = cadd(x1, x3), t3 = rot90<INV>(csub(x1, x3));
    x0 = cadd(t0, t2);
    x2 = csub(t0, t2);
    x1 = cadd(t1, t3);
    x3 = csub(t1, t3);
}

// W_16^k for k = 0..9 (forward sign); constants rounded once by the compiler
__device__ __forceinline__ c32 w16(int k)
{
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float c2 = 0.70710678118654752440f;
    switch(k) {
    case 0: return {1.0f, 0.0f};
    case 1: return {c1, -s1};
    case 2: return {c2, -c2};
    case 3: return {s1, -c1};
    case 4: return {0.0f, -1.0f};
    case 5: return {-s1, -c1};
    case 6: return {-c2, -c2};
    case 7: return {-c1, -s1};
    case 8: return {-1.0f, 0.0f};
    default: return {-c1, s1};  // k == 9
    }
}

// In-register DFT of size 16, natural order in and out.
template <bool INV>
__device__ __forceinline__ void dft16(c32* x)
{
#pragma unroll
    for(int r2 = 0; r2 < 4; ++r2) dft4<INV>(x[r2], x[4 + r2], x[8 + r2], x[12 + r2]);
    // now x[4*q1 + r2] holds A[r2][q1]; twiddle by W16^(r2*q1)
#pragma unroll
    for(int r2 = 1; r2 < 4; ++r2)
#pragma unroll
        for(int q1 = 1; q1 < 4; ++q1) {
            c32 w = w16(r2 * q1);
            if(INV) w.y = -w.y;
            x[4 * q1 + r2] = cmul(x[4 * q1 + r2], w);
        }
#pragma unroll
    for(int q1 = 0; q1 < 4; ++q1) dft4<INV>(x[4 * q1], x[4 * q1 + 1], x[4 * q1 + 2], x[4 * q1 + 3]);
    // x[4*q1 + q2] holds X[q1 + 4*q2]; transpose to natural order
    c32 t[16];
#pragma unroll
    for(int q1 = 0; q1 < 4; ++q1)
#pragma unroll
        for(int q2 = 0; q2 < 4; ++q2) t[q1 + 4 * q2] = x[4 * q1 + q2];
#pragma unroll
    for(int i = 0; i < 16; ++i) x[i] = t[i];
}

template <bool INV>
__device__ __forceinline__ void dft8(c32* x)
{
    // radix 2 x 4: r = 4*r1 + r2, q = q1 + 2*q2
#pragma unroll
    for(int r2 = 0; r2 < 4; ++r2) {
        c32 a = x[r2], b = x[4 + r2];
        x[r2] = cadd(a, b);
        x[4 + r2] = csub(a, b);
    }
    // twiddle W8^(r2*q1) on the q1 = 1 half
    const float c2 = 0.70710678118654752440f;
    x[5] = cmul(x[5], c32{c2, INV ? c2 : -c2});
    x[6] = rot90<INV>(x[6]);
    x[7] = cmul(x[7], c32{-c2, INV ? c2 : -c2});
    dft4<INV>(x[0], x[1], x[2], x[3]);
    dft4<INV>(x[4], x[5], x[6], x[7]);
    c32 t[8];
#pragma unroll
    for(int q2 = 0; q2 < 4; ++q2) {
        t[2 * q2]     = x[q2];
        t[2 * q2 + 1] = x[4 + q2];
    }
#pragma unroll
    for(int i = 0; i < 8; ++i) x[i] = t[i];
}

template <int R, bool INV>
__device__ __forceinline__ void dft(c32* x)
{
    if constexpr(R == 16) dft16<INV>(x);
    else if constexpr(R == 8) dft8<INV>(x);
    else if constexpr(R == 4) dft4<INV>(x[0], x[1], x[2], x[3]);
    else dft2<INV>(x);
}

// one padding slot per 16 complex values keeps the strided radix-16 passes
// free of shared-memory bank conflicts
__host__ __device__ constexpr int pad(int i) { return i + (i >> 4); }
// pad(b + q * s) for a stride s that is a multiple of 16: the padding of
// b + q s is pad(b) + q (s + s / 16), i.e. one base plus constant offsets
// (the compiler folds them into the shared-memory instructions).
__device__ __forceinline__ int pad_at(int b, int pb, int q, int s)
{
    return (s & 15) == 0 ? pb + q * (s + (s >> 4)) : pad(b + q * s);
}

struct Args {
    const uint8_t* in;
    size_t row_stride;
    int nstreams;      // F * P * A
    int nsamples;      // T
    int overlap;       // O: samples of history in front of the gulp
    int lag;           // trimmed at the end of each window (output delay)
    int nseg;
    int ndms;
    const c32* tw;     // twiddle tables
    const c32* chirp;  // [ndms][F][N] in per-thread load order (chirp_k)
    size_t chirp_dm_stride;    // complex entries between two DMs' tables
    const uint32_t* zero_flags;  // [ndms]: non-zero if the DM is 0 (chirp exactly 1)
    int npa;           // P * A (streams per channel)
    uint8_t* out[kMaxDms];
    size_t out_stride;
    float2* dbg;  // optional [ndms][nstreams][nsamples] scaled values before rounding
};

// Twiddles w[1..R-1] of butterfly column j for a pass with stride s.
template <int R>
__device__ __forceinline__ void load_tw(const c32* tw_s, int tw_off, int s, int j, c32* w)
{
    if constexpr(R == 16) {
        const float4* p = reinterpret_cast<const float4*>(tw_s + tw_off);
#pragma unroll
        for(int k = 0; k < 8; ++k) {
            const float4 v = p[k * s + j];
            w[2 * k + 1] = c32{v.x, v.y};
            if(k < 7) w[2 * k + 2] = c32{v.z, v.w};
        }
    } else {
#pragma unroll
        for(int q = 1; q < R; ++q) w[q] = tw_s[tw_off + (q - 1) * s + j];
    }
}

// One radix-R pass of the inverse (DIT) on shared memory.
template <int LOGN, int R>
__device__ __forceinline__ void inv_pass(c32* buf, const c32* tw_s, int G, int s,
                                         int tw_off)
{
    constexpr int N   = 1 << LOGN;
    constexpr int NT  = N / 16;
    constexpr int BPT = 16 / R;  // butterflies per thread
#pragma unroll
    for(int u = 0; u < BPT; ++u) {
        const int beta = threadIdx.x + u * NT;
        const int g = beta / s, j = beta - g * s;
        const int base = g * G + j;
        const int pb = pad(base);
        c32 z[R];
#pragma unroll
        for(int q = 0; q < R; ++q) z[q] = buf[pad_at(base, pb, q, s)];
        if(s > 1) {
{
                c32 w[R];
                load_tw<R>(tw_s, tw_off, s, j, w);
#pragma unroll
                for(int q = 1; q < R; ++q) z[q] = cmulc(z[q], w[q]);
            }
        }
        dft<R, true>(z);
#pragma unroll
        for(int r = 0; r < R; ++r) buf[pad_at(base, pb, r, s)] = z[r];
    }
}

template <int LOGN, int R>
__device__ __forceinline__ void fwd_pass(c32* buf, const c32* tw_s, int G, int s,
                                         int tw_off)
{
    constexpr int N   = 1 << LOGN;
    constexpr int NT  = N / 16;
    constexpr int BPT = 16 / R;
#pragma unroll
    for(int u = 0; u < BPT; ++u) {
        const int beta = threadIdx.x + u * NT;
        const int g = beta / s, j = beta - g * s;
        const int base = g * G + j;
        const int pb = pad(base);
        c32 x[R];
#pragma unroll
        for(int r = 0; r < R; ++r) x[r] = buf[pad_at(base, pb, r, s)];
        dft<R, false>(x);
        if(s > 1) {
{
                c32 w[R];
                load_tw<R>(tw_s, tw_off, s, j, w);
#pragma unroll
                for(int q = 1; q < R; ++q) x[q] = cmul(x[q], w[q]);
            }
        }
#pragma unroll
        for(int q = 0; q < R; ++q) buf[pad_at(base, pb, q, s)] = x[q];
    }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Stage the int8 window of one work item (re row then im row, N bytes each)
// into shared memory: asynchronously with 16-byte cp.async (zero-filled past
// the end of the rows) when the rows and segment starts are 16-byte aligned,
// otherwise with plain byte copies.
template <int N, int NT>
__device__ __forceinline__ void stage_input(uint8_t* st, const Args& A, int item, int L,
                                            bool aligned)
{
    const int stream = item / A.nseg;
    const int seg    = item - stream * A.nseg;
    const uint8_t* row_re = A.in + (size_t)stream * 2 * A.row_stride;
    const uint8_t* row_im = row_re + A.row_stride;
    const int start = seg * L;
    const int avail = A.overlap + A.nsamples;
    if(aligned) {
        constexpr int kChunks = N / 16;
        for(int c = threadIdx.x; c < 2 * kChunks; c += NT) {
            const int plane = c >= kChunks;
            const int k     = (c - plane * kChunks) * 16;
            const int left  = avail - (start + k);
            const int bytes = left <= 0 ? 0 : (left >= 16 ? 16 : left);
            const uint8_t* src = bytes > 0 ? (plane ? row_im : row_re) + start + k : row_re;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                             smem_addr(st + plane * N + k)),
                         "l"(src), "r"(bytes)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    } else {
        for(int i = threadIdx.x; i < N; i += NT) {
            const int idx = start + i;
            st[i]     = idx < avail ? row_re[idx] : 0;
            st[N + i] = idx < avail ? row_im[idx] : 0;
        }
    }
}

// at least two resident CTAs per SM below N = 8192 (latency hiding across
// the per-pass barriers); N = 8192 needs 512 threads and fits one.
template <int LOGN, bool DBG>
__global__ void __launch_bounds__((1 << LOGN) / 16, LOGN >= 13 ? 1 : (LOGN == 12 ? 2 : 4))
cdd_kernel(const __grid_constant__ Args A)
{
    constexpr int N  = 1 << LOGN;
    constexpr int NT = N / 16;
    constexpr Plan P = make_plan(LOGN);
    constexpr int R0 = P.r0;
    constexpr int B0 = 16 / R0;  // first-pass butterflies per thread
    extern __shared__ __align__(16) uint8_t smem[];
    c32* buf  = reinterpret_cast<c32*>(smem);
    c32* tw_s = buf + pad(N) + 16;
    uint8_t* stage = reinterpret_cast<uint8_t*>(tw_s + ((P.tw_total + 1) & ~1));
    for(int i = threadIdx.x; i < P.tw_total; i += NT) tw_s[i] = A.tw[i];

    const int L = N - A.overlap;
    const int head = A.overlap - A.lag;  // trimmed at the start of each window
    const float inv_n = 1.0f / (float)N;  // exact (power of two)
    const int nitems = A.nstreams * A.nseg;
    const bool aligned = (A.row_stride % 16 == 0) && (L % 16 == 0) &&
                         ((reinterpret_cast<uintptr_t>(A.in) & 15) == 0);
    // DMs of exactly 0 (chirp 1): the dedispersed window is the input itself
    // (the FP32 round trip of int8 samples rounds back to them exactly), so
    // they are copied from the staged window instead of transformed.  The
    // debug instance transforms them to report the float round trip.
    uint32_t zero_dms = 0;
    if constexpr(!DBG)
        for(int d = 0; d < A.ndms && d < 32; ++d) zero_dms |= (A.zero_flags[d] ? 1u : 0u) << d;
    const bool copy16 = aligned && (head % 16) == 0 && (A.out_stride % 16) == 0;
    if(blockIdx.x < nitems) stage_input<N, NT>(stage, A, blockIdx.x, L, aligned);
    for(int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int stream = item / A.nseg;
        const int seg    = item - stream * A.nseg;
        const int f      = stream / A.npa;
        const int start  = seg * L;  // first input sample of the window
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();

        // ---- forward pass 0 (radix R0, span N) from the staged int8 window
        {
            constexpr int s0 = N / R0;
#pragma unroll
            for(int u = 0; u < B0; ++u) {
                const int j = threadIdx.x + u * NT;
                c32 x[R0];
#pragma unroll
                for(int r = 0; r < R0; ++r) {
                    const int i = j + r * s0;
                    x[r] = c32{(float)(int8_t)stage[i], (float)(int8_t)stage[N + i]};
                }
                dft<R0, false>(x);
{
                    c32 w[R0];
                    load_tw<R0>(tw_s, P.tw_off[0], s0, j, w);
#pragma unroll
                    for(int q = 1; q < R0; ++q) x[q] = cmul(x[q], w[q]);
                }
#pragma unroll
                for(int q = 0; q < R0; ++q) buf[pad_at(j, pad(j), q, s0)] = x[q];
            }
        }
        for(uint32_t zm = zero_dms; zm; zm &= zm - 1) {
            const int d = __ffs(zm) - 1;
            uint8_t* o_re = A.out[d] + (size_t)stream * 2 * A.out_stride;
            const int n = min(L, A.nsamples - start);  // kept samples of this window
            if(copy16 && ((reinterpret_cast<uintptr_t>(A.out[d]) & 15) == 0)) {
                const int chunks = (n + 15) / 16;
                for(int c = threadIdx.x; c < 2 * chunks; c += NT) {
                    const int plane = c >= chunks;
                    const int k = (c - plane * chunks) * 16;
                    const uint8_t* src = stage + plane * N + head + k;
                    uint8_t* dst = o_re + plane * A.out_stride + start + k;
                    if(k + 16 <= n) {
                        *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
                    } else {
                        for(int b = 0; b < n - k; ++b) dst[b] = src[b];
                    }
                }
            } else {
                for(int i = threadIdx.x; i < 2 * n; i += NT) {
                    const int plane = i >= n, k = i - plane * n;
                    o_re[plane * A.out_stride + start + k] = stage[plane * N + head + k];
                }
            }
        }
        __syncthreads();
        // the staging buffer is free: fetch the next work item's window now so
        // that its global-memory latency hides behind this item's transforms
        if(item + (int)gridDim.x < nitems)
            stage_input<N, NT>(stage, A, item + gridDim.x, L, aligned);
        // ---- forward radix-16 passes except the last
#pragma unroll
        for(int p = 1; p < P.npass - 1; ++p) {
            fwd_pass<LOGN, 16>(buf, tw_s, P.span[p], P.stride[p], P.tw_off[p]);
            __syncthreads();
        }
        // ---- last forward pass (span 16, no twiddles): spectrum -> registers
        c32 spec[16];
#pragma unroll
        for(int r = 0; r < 16; ++r) spec[r] = buf[pad(threadIdx.x * 16 + r)];
        dft16<false>(spec);

        const size_t chirp_stride = A.chirp_dm_stride;  // complex entries per DM
        const float4* chp = reinterpret_cast<const float4*>(A.chirp + (size_t)f * N) + threadIdx.x;
        // the transformed DMs in order; chn holds the chirp of DM `d`
        int d = 0;
        while(d < A.ndms && d < 32 && ((zero_dms >> d) & 1u)) ++d;
        float4 chn[8];
        if(d < A.ndms) {
            const float4* cur = chp + (size_t)d * chirp_stride / 2;
#pragma unroll
            for(int k = 0; k < 8; ++k) chn[k] = cur[k * NT];
        }
        __syncthreads();
        for(; d < A.ndms;) {
            int dn = d + 1;
            while(dn < A.ndms && dn < 32 && ((zero_dms >> dn) & 1u)) ++dn;
            c32 y[16];
#pragma unroll
            for(int k = 0; k < 8; ++k) {
                y[2 * k]     = cmul(spec[2 * k], c32{chn[k].x, chn[k].y});
                y[2 * k + 1] = cmul(spec[2 * k + 1], c32{chn[k].z, chn[k].w});
            }
            if(dn < A.ndms) {  // next DM's chirp, in flight during this inverse
                const float4* nxt = chp + (size_t)dn * chirp_stride / 2;
#pragma unroll
                for(int k = 0; k < 8; ++k) chn[k] = nxt[k * NT];
            }
            dft16<true>(y);
#pragma unroll
            for(int r = 0; r < 16; ++r) buf[pad(threadIdx.x * 16 + r)] = y[r];
            __syncthreads();
#pragma unroll
            for(int p = P.npass - 2; p >= 1; --p) {
                inv_pass<LOGN, 16>(buf, tw_s, P.span[p], P.stride[p], P.tw_off[p]);
                __syncthreads();
            }
            // ---- inverse pass 0 (radix R0, span N): natural-order output
            uint8_t* o_re = A.out[d] + (size_t)stream * 2 * A.out_stride;
            uint8_t* o_im = o_re + A.out_stride;
            constexpr int s0 = N / R0;
#pragma unroll
            for(int u = 0; u < B0; ++u) {
                const int j = threadIdx.x + u * NT;
                c32 z[R0];
#pragma unroll
                for(int q = 0; q < R0; ++q) z[q] = buf[pad_at(j, pad(j), q, s0)];
{
                    c32 w[R0];
                    load_tw<R0>(tw_s, P.tw_off[0], s0, j, w);
#pragma unroll
                    for(int q = 1; q < R0; ++q) z[q] = cmulc(z[q], w[q]);
                }
                dft<R0, true>(z);
#pragma unroll
                for(int r = 0; r < R0; ++r) {
                    const int i = j + r * s0;           // index within the window
                    const int m = start + i - head;     // output sample in the gulp
                    if(i >= head && i < head + L && m < A.nsamples) {
                        const float fr = z[r].x * inv_n, fi = z[r].y * inv_n;
                        o_re[m] = (uint8_t)__float2int_rn(fr);  // int8 wrap, like static_cast<char>
                        o_im[m] = (uint8_t)__float2int_rn(fi);
                        if constexpr(DBG)
                            A.dbg[((size_t)d * A.nstreams + stream) * A.nsamples + m] =
                                make_float2(fr, fi);
                    }
                }
            }
            __syncthreads();
            d = dn;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// ------------------------------------------------- long FFTs (N = S x 8192)
// Overlap-save windows longer than one CTA's shared memory are split four-step
// style into S = N / 8192 sub-transforms of M = 8192 points:
//   n = M n1 + n2, k = k1 + S k2 (n1, k1 < S; n2, k2 < M)
//   forward:  X[k1 + S k2] = DFT_M over n2 of
//                 W_N^(n2 k1) * sum_n1 x[M n1 + n2] W_S^(n1 k1)
//   inverse:  x[n2 + M n1] = sum_k1 W_S^(-n1 k1) *
//                 W_N^(-n2 k1) * IDFT_M over k2 of Y[k1 + S k2]
// cdd_split_kernel runs one (segment, k1) per CTA: the S-point partial DFT
// straight from the int8 rows, the M-point forward FFT, and for every DM the
// chirp of bins k1 + S k2 and the M-point inverse FFT, leaving
// W_N^(-n2 k1) * z in a complex workspace; cdd_split_combine then does the
// S-point inverse DFT over k1, the overlap-save trim, /N, rint and int8 wrap.
constexpr int kSplitLog = 13;
constexpr int kSplitM   = 1 << kSplitLog;

struct SplitArgs {
    const uint8_t* in;
    size_t row_stride;
    int nstreams, nsamples, overlap, lag, nseg, ndms, npa;
    size_t chirp_dm_stride;  // complex entries between two DMs' tables
    int item0, nitems;  // work items [item0, item0 + nitems) of this chunk
    const c32* tw;      // M-point plan tables
    const c32* chirp;   // [ndms][F][S][M]: bin k1 + S k2 at k1's per-thread load order
    const c32* tws;     // [S][M]: W_N^(n2 k1)
    c32* z;             // [ndms][nitems][S][M]
    uint8_t* out[kMaxDms];
    size_t out_stride;
    float2* dbg;
};

// W_S^m (forward sign) for S in {2, 4, 8}
template <int S>
__device__ __forceinline__ c32 wsm(int m)
{
    const float c2 = 0.70710678118654752440f;
    switch((m % S) * (8 / S)) {
    case 0: return {1.0f, 0.0f};
    case 1: return {c2, -c2};
    case 2: return {0.0f, -1.0f};
    case 3: return {-c2, -c2};
    case 4: return {-1.0f, 0.0f};
    case 5: return {-c2, c2};
    case 6: return {0.0f, 1.0f};
    default: return {c2, c2};
    }
}

template <int S>
__global__ void __launch_bounds__(kSplitM / 16, 1)
cdd_split_kernel(const __grid_constant__ SplitArgs A)
{
    constexpr int LOGN = kSplitLog;
    constexpr int M  = kSplitM;
    constexpr int N  = S * M;
    constexpr int NT = M / 16;
    constexpr Plan P = make_plan(LOGN);
    constexpr int R0 = P.r0;
    constexpr int B0 = 16 / R0;
    extern __shared__ __align__(16) uint8_t smem[];
    c32* buf  = reinterpret_cast<c32*>(smem);
    c32* tw_s = buf + pad(M) + 16;
    for(int i = threadIdx.x; i < P.tw_total; i += NT) tw_s[i] = A.tw[i];
    const int L = N - A.overlap;
    const int avail = A.overlap + A.nsamples;

    for(int u = blockIdx.x; u < A.nitems * S; u += gridDim.x) {
        const int il = u / S, k1 = u - il * S;
        const int item   = A.item0 + il;
        const int stream = item / A.nseg;
        const int seg    = item - stream * A.nseg;
        const int f      = stream / A.npa;
        const int start  = seg * L;
        const int8_t* row_re = reinterpret_cast<const int8_t*>(A.in) + (size_t)stream * 2 * A.row_stride;
        const int8_t* row_im = row_re + A.row_stride;
        __syncthreads();  // previous unit's last reads of buf are done
        // ---- S-point partial DFT for this k1, times W_N^(n2 k1)
#pragma unroll 4
        for(int v = 0; v < 16; ++v) {
            const int n2 = threadIdx.x + v * NT;
            c32 acc{0.0f, 0.0f};
#pragma unroll
            for(int n1 = 0; n1 < S; ++n1) {
                const int idx = start + n1 * M + n2;
                const c32 x = idx < avail ? c32{(float)row_re[idx], (float)row_im[idx]}
                                          : c32{0.0f, 0.0f};
                acc = cadd(acc, cmul(x, wsm<S>(n1 * k1)));
            }
            buf[pad(n2)] = cmul(acc, A.tws[(size_t)k1 * M + n2]);
        }
        __syncthreads();
        // ---- M-point forward FFT (DIF) in shared memory
        fwd_pass<LOGN, R0>(buf, tw_s, P.span[0], P.stride[0], P.tw_off[0]);
        __syncthreads();
#pragma unroll
        for(int p = 1; p < P.npass - 1; ++p) {
            fwd_pass<LOGN, 16>(buf, tw_s, P.span[p], P.stride[p], P.tw_off[p]);
            __syncthreads();
        }
        c32 spec[16];
#pragma unroll
        for(int r = 0; r < 16; ++r) spec[r] = buf[pad(threadIdx.x * 16 + r)];
        dft16<false>(spec);
        const size_t chirp_dm = A.chirp_dm_stride;  // complex per DM
        const float4* chp = reinterpret_cast<const float4*>(A.chirp + (size_t)f * N + (size_t)k1 * M) + threadIdx.x;
        __syncthreads();
        for(int d = 0; d < A.ndms; ++d) {
            const float4* cd = chp + (size_t)d * chirp_dm / 2;
            c32 y[16];
#pragma unroll
            for(int k = 0; k < 8; ++k) {
                const float4 c = cd[k * NT];
                y[2 * k]     = cmul(spec[2 * k], c32{c.x, c.y});
                y[2 * k + 1] = cmul(spec[2 * k + 1], c32{c.z, c.w});
            }
            dft16<true>(y);
#pragma unroll
            for(int r = 0; r < 16; ++r) buf[pad(threadIdx.x * 16 + r)] = y[r];
            __syncthreads();
#pragma unroll
            for(int p = P.npass - 2; p >= 1; --p) {
                inv_pass<LOGN, 16>(buf, tw_s, P.span[p], P.stride[p], P.tw_off[p]);
                __syncthreads();
            }
            // last inverse pass, then W_N^(-n2 k1), to the workspace
            c32* zo = A.z + (((size_t)d * A.nitems + il) * S + k1) * M;
            constexpr int s0 = M / R0;
#pragma unroll
            for(int v = 0; v < B0; ++v) {
                const int j = threadIdx.x + v * NT;
                c32 z[R0];
#pragma unroll
                for(int q = 0; q < R0; ++q) z[q] = buf[pad_at(j, pad(j), q, s0)];
                {
                    c32 w[R0];
                    load_tw<R0>(tw_s, P.tw_off[0], s0, j, w);
#pragma unroll
                    for(int q = 1; q < R0; ++q) z[q] = cmulc(z[q], w[q]);
                }
                dft<R0, true>(z);
#pragma unroll
                for(int r = 0; r < R0; ++r) {
                    const int n2 = j + r * s0;
                    zo[n2] = cmulc(z[r], A.tws[(size_t)k1 * M + n2]);
                }
            }
            __syncthreads();
        }
    }
}

template <int S>
__global__ void __launch_bounds__(256)
cdd_split_combine(const __grid_constant__ SplitArgs A)
{
    constexpr int M = kSplitM, N = S * M;
    const int L = N - A.overlap, head = A.overlap - A.lag;
    const float inv_n = 1.0f / (float)N;  // exact (power of two)
    const size_t total = (size_t)A.ndms * A.nitems * M;
    for(size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
        idx += (size_t)gridDim.x * blockDim.x) {
        const int n2 = (int)(idx % M);
        const size_t rest = idx / M;
        const int il = (int)(rest % A.nitems);
        const int d  = (int)(rest / A.nitems);
        const int item   = A.item0 + il;
        const int stream = item / A.nseg;
        const int seg    = item - stream * A.nseg;
        const int start  = seg * L;
        const c32* zi = A.z + ((size_t)d * A.nitems + il) * S * M + n2;
        c32 z[S];
#pragma unroll
        for(int k1 = 0; k1 < S; ++k1) z[k1] = zi[(size_t)k1 * M];
        dft<S, true>(z);  // z[n1] = sum_k1 W_S^(-n1 k1) z'[k1]
        uint8_t* o_re = A.out[d] + (size_t)stream * 2 * A.out_stride;
        uint8_t* o_im = o_re + A.out_stride;
#pragma unroll
        for(int n1 = 0; n1 < S; ++n1) {
            const int i = n2 + n1 * M;
            const int m = start + i - head;
            if(i >= head && i < head + L && m < A.nsamples) {
                const float fr = z[n1].x * inv_n, fi = z[n1].y * inv_n;
                o_re[m] = (uint8_t)__float2int_rn(fr);
                o_im[m] = (uint8_t)__float2int_rn(fi);
                if(A.dbg)
                    A.dbg[((size_t)d * A.nstreams + stream) * A.nsamples + m] = make_float2(fr, fi);
            }
        }
    }
}

template <int S>
int launch_split(SplitArgs a, int total_items, size_t ws_items, cudaStream_t stream)
{
    constexpr Plan P = make_plan(kSplitLog);
    const size_t smem = (size_t)(pad(kSplitM) + 16 + ((P.tw_total + 1) & ~1)) * sizeof(c32);
    SW_CUDA_CHECK(cudaFuncSetAttribute(cdd_split_kernel<S>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    for(int i0 = 0; i0 < total_items; i0 += (int)ws_items) {
        a.item0  = i0;
        a.nitems = (int)std::min<size_t>(ws_items, (size_t)(total_items - i0));
        const long units = (long)a.nitems * S;
        cdd_split_kernel<S><<<(int)std::min<long>(units, nsm), kSplitM / 16, smem, stream>>>(a);
        SW_LAUNCH_CHECK();
        const size_t total = (size_t)a.ndms * a.nitems * kSplitM;
        const size_t blocks = std::min<size_t>(cdiv(total, (size_t)256), (size_t)nsm * 16);
        cdd_split_combine<S><<<(int)blocks, 256, 0, stream>>>(a);
        SW_LAUNCH_CHECK();
    }
    return SW_OK;
}

// ------------------------------------------------------------- setup
struct SetupArgs {
    int logn, ndms, nchans;
    double low_freq, coarse_bw, fine_bw;
    double prefactor[kMaxDms];
};

struct ZeroFlags {
    uint32_t f[kMaxDms];
};
__global__ void set_flags_k(uint32_t* p, ZeroFlags z) { p[threadIdx.x] = z.f[threadIdx.x]; }

__global__ void twiddle_k(c32* tw, int logn)
{
    const Plan P = make_plan(logn);
    for(int p = 0; p < P.npass; ++p) {
        const int s = P.stride[p], R = P.radix[p], G = P.span[p];
        if(s <= 1) continue;
        const int entries = (R == 16 ? 16 : R - 1) * s;
        for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < entries;
            i += gridDim.x * blockDim.x) {
            int q, j;
            if(R == 16) {  // c32 index i = 2*(k*s + j) + h holds w_(2k+1+h)
                const int m = i >> 1, h = i & 1;
                q = 2 * (m / s) + 1 + h;
                j = m % s;
            } else {
                q = i / s + 1;
                j = i % s;
            }
            double sn = 0.0, cs = 0.0;
            // exp(-2 pi i j q / G) in FP64
            if(q < R) sincospi(-2.0 * (double)(j * q) / (double)G, &sn, &cs);
            tw[P.tw_off[p] + i] = c32{(float)cs, (float)sn};
        }
    }
}

// DMResponse (CoherentDedisperser.cu:313-335) in FP64.  The transform
// leaves bin digit_reverse(16 t + r) in register r of thread t; the table
// stores the chirp of that bin at ((r / 2) * (N / 16) + t) * 2 + r % 2, so
// that the k-th 16-byte load of every thread (registers 2k and 2k+1) reads
// one contiguous 512-byte span per warp.
__global__ void chirp_k(c32* chirp, SetupArgs S)
{
    const Plan P = make_plan(S.logn);
    const int nt = P.n / 16;
    const size_t total = (size_t)S.ndms * S.nchans * P.n;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
        i += (size_t)gridDim.x * blockDim.x) {
        const int q   = (int)(i % P.n);
        const int c   = (int)((i / P.n) % S.nchans);
        const int d   = (int)(i / ((size_t)P.n * S.nchans));
        const int t   = (q >> 1) % nt;
        const int r   = 2 * ((q >> 1) / nt) + (q & 1);
        const int k   = digit_reverse(P, 16 * t + r);
        const double nu0   = S.low_freq + c * S.coarse_bw - 0.5 * S.coarse_bw;
        const double nu    = k * S.fine_bw;
        const double phase = (nu * nu * S.prefactor[d]) / ((nu0 + nu) * nu0 * nu0);
        double sn, cs;
        sincos(phase, &sn, &cs);
        chirp[i] = c32{(float)cs, (float)sn};
    }
}

// Chirp tables for the split transform: bin k1 + S k2 of sub-transform k1
// at k1 * M + (the M-point per-thread load order of k2).
__global__ void chirp_split_k(c32* chirp, SetupArgs S, int split)
{
    const Plan P = make_plan(kSplitLog);
    const int nt = kSplitM / 16;
    const int n  = split * kSplitM;
    const size_t total = (size_t)S.ndms * S.nchans * n;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
        i += (size_t)gridDim.x * blockDim.x) {
        const int q  = (int)(i % n);
        const int c  = (int)((i / n) % S.nchans);
        const int d  = (int)(i / ((size_t)n * S.nchans));
        const int k1 = q / kSplitM, qq = q % kSplitM;
        const int t  = (qq >> 1) % nt;
        const int r  = 2 * ((qq >> 1) / nt) + (qq & 1);
        const int k  = k1 + split * digit_reverse(P, 16 * t + r);
        const double nu0   = S.low_freq + c * S.coarse_bw - 0.5 * S.coarse_bw;
        const double nu    = k * S.fine_bw;
        const double phase = (nu * nu * S.prefactor[d]) / ((nu0 + nu) * nu0 * nu0);
        double sn, cs;
        sincos(phase, &sn, &cs);
        chirp[i] = c32{(float)cs, (float)sn};
    }
}

// W_N^(n2 k1) = exp(-2 pi i n2 k1 / N) in FP64, [k1][n2]
__global__ void split_twiddle_k(c32* tws, int split)
{
    const int n = split * kSplitM;
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int k1 = i / kSplitM, n2 = i % kSplitM;
        double sn, cs;
        sincospi(-2.0 * (double)((long long)n2 * k1) / (double)n, &sn, &cs);
        tws[i] = c32{(float)cs, (float)sn};
    }
}

template <int LOGN, bool DBG>
int launch_logn_dbg(const Args& a, cudaStream_t stream)
{
    constexpr int N = 1 << LOGN;
    constexpr Plan P = make_plan(LOGN);
    const size_t smem = (size_t)(pad(N) + 16 + ((P.tw_total + 1) & ~1)) * sizeof(c32) + 2 * N;
    SW_CUDA_CHECK(cudaFuncSetAttribute(cdd_kernel<LOGN, DBG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    SW_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cdd_kernel<LOGN, DBG>,
                                                                 N / 16, smem));
    if(per_sm < 1) per_sm = 1;
    const long items = (long)a.nstreams * a.nseg;
    const long grid  = items < (long)nsm * per_sm ? items : (long)nsm * per_sm;
    cdd_kernel<LOGN, DBG><<<(int)grid, N / 16, smem, stream>>>(a);
    SW_LAUNCH_CHECK();
    return SW_OK;
}

// the float output for precision studies is a separate instance, so the
// production kernel carries none of its registers
template <int LOGN>
int launch_logn(const Args& a, cudaStream_t stream)
{
    return a.dbg ? launch_logn_dbg<LOGN, true>(a, stream) : launch_logn_dbg<LOGN, false>(a, stream);
}

int log2_exact(int n)
{
    int l = 0;
    while((1 << l) < n) ++l;
    return (1 << l) == n ? l : -1;
}

// Setup block: per-pass twiddles, a gap of kSetupGap complex entries whose
// first words flag the DMs of exactly 0, the chirp tables [ndms][nchans][N]
// and, for split transforms, the W_N^(n2 k1) table.
constexpr int kSetupGap = 64;  // >= kMaxDms 32-bit flags

// Dedisperse `nchans` channels (of a setup built for setup_nchans channels
// and setup_ndms DMs, starting at channel chan0) for `ndms` DMs starting at
// dm0 of the setup.
int launch_cdd(const void* d_fpact_in, size_t row_stride, int nchans, int npol, int nant,
               int nsamples, int fft_len, int overlap, int lag, const void* d_setup,
               int setup_ndms, int setup_nchans, int chan0, int dm0, int ndms,
               void* const* h_d_out, size_t out_row_stride, void* d_workspace,
               size_t workspace_bytes, float* d_debug_f32, sw_stream_t stream)
{
    const int logn = log2_exact(fft_len);
    SW_REQUIRE(logn >= 8 && logn <= 16,
               "coherent dedispersion: fft_len must be a power of two in [256, 65536]");
    SW_REQUIRE(d_fpact_in && d_setup && h_d_out, "coherent dedispersion: null pointer");
    SW_REQUIRE(ndms > 0 && ndms <= kMaxDms, "coherent dedispersion: 1..%d DMs", kMaxDms);
    SW_REQUIRE(overlap >= 0 && overlap < fft_len,
               "coherent dedispersion: overlap must be smaller than the FFT");
    SW_REQUIRE(lag >= 0 && lag <= overlap,
               "coherent dedispersion: the lag (%d) must lie in [0, overlap = %d]", lag, overlap);
    SW_REQUIRE(nsamples > 0 && (size_t)overlap + nsamples <= row_stride,
               "coherent dedispersion: input rows must hold history + gulp");
    SW_REQUIRE((size_t)nsamples <= out_row_stride, "coherent dedispersion: output rows too short");
    SW_REQUIRE(nchans > 0 && npol > 0 && nant > 0, "coherent dedispersion: empty shape");
    const int plog = logn > kSplitLog ? kSplitLog : logn;
    const Plan P = make_plan(plog);
    const c32* tw = static_cast<const c32*>(d_setup);
    const c32* ch_all = tw + P.tw_total + kSetupGap;
    const c32* ch = ch_all + ((size_t)dm0 * setup_nchans + chan0) * fft_len;
    const uint32_t* zero_flags = reinterpret_cast<const uint32_t*>(tw + P.tw_total) + dm0;
    const int nstreams = nchans * npol * nant;
    const int nseg = cdiv(nsamples, fft_len - overlap);
    cudaStream_t s = as_cuda(stream);
    if(logn > kSplitLog) {
        const size_t per_item = (size_t)ndms * fft_len * sizeof(c32);
        SW_REQUIRE(d_workspace && workspace_bytes >= per_item,
                   "coherent dedispersion: fft_len %d needs a workspace of at least %zu bytes "
                   "(sw_cdd_workspace_bytes)", fft_len, per_item);
        SplitArgs a{};
        a.in = static_cast<const uint8_t*>(d_fpact_in);
        a.row_stride = row_stride;
        a.nstreams = nstreams;
        a.nsamples = nsamples;
        a.overlap = overlap;
        a.lag = lag;
        a.nseg = nseg;
        a.ndms = ndms;
        a.npa = npol * nant;
        a.chirp_dm_stride = (size_t)setup_nchans * fft_len;
        a.tw = tw;
        a.chirp = ch;
        a.tws = ch_all + (size_t)setup_ndms * setup_nchans * fft_len;
        a.z = static_cast<c32*>(d_workspace);
        for(int d = 0; d < ndms; ++d) {
            SW_REQUIRE(h_d_out[d], "coherent dedispersion: null output for DM %d", d);
            a.out[d] = static_cast<uint8_t*>(h_d_out[d]);
        }
        a.out_stride = out_row_stride;
        a.dbg = reinterpret_cast<float2*>(d_debug_f32);
        const int items = nstreams * nseg;
        const size_t ws_items = std::min<size_t>(workspace_bytes / per_item, (size_t)items);
        switch(fft_len / kSplitM) {
        case 2: return launch_split<2>(a, items, ws_items, s);
        case 4: return launch_split<4>(a, items, ws_items, s);
        default: return launch_split<8>(a, items, ws_items, s);
        }
    }
    Args a{};
    a.in         = static_cast<const uint8_t*>(d_fpact_in);
    a.row_stride = row_stride;
    a.npa        = npol * nant;
    a.nstreams   = nstreams;
    a.nsamples   = nsamples;
    a.overlap    = overlap;
    a.lag        = lag;
    a.nseg       = nseg;
    a.ndms       = ndms;
    a.chirp_dm_stride = (size_t)setup_nchans * fft_len;
    a.tw         = tw;
    a.chirp      = ch;
    a.zero_flags = zero_flags;
    for(int d = 0; d < ndms; ++d) {
        SW_REQUIRE(h_d_out[d], "coherent dedispersion: null output for DM %d", d);
        a.out[d] = static_cast<uint8_t*>(h_d_out[d]);
    }
    a.out_stride = out_row_stride;
    a.dbg        = reinterpret_cast<float2*>(d_debug_f32);
    switch(logn) {
    case 8: return launch_logn<8>(a, s);
    case 9: return launch_logn<9>(a, s);
    case 10: return launch_logn<10>(a, s);
    case 11: return launch_logn<11>(a, s);
    case 12: return launch_logn<12>(a, s);
    default: return launch_logn<13>(a, s);
    }
}

}  // namespace cdd
}  // namespace swb

using namespace swb;
using namespace swb::cdd;

extern "C" {

size_t sw_cdd_setup_bytes(int ndms, int nchans, int fft_len)
{
    const int logn = log2_exact(fft_len);
    if(logn < 8 || logn > 16 || ndms <= 0 || nchans <= 0) return 0;
    const Plan P = make_plan(logn > kSplitLog ? kSplitLog : logn);
    const size_t split_tw = logn > kSplitLog ? (size_t)fft_len : 0;
    return ((size_t)P.tw_total + kSetupGap + (size_t)ndms * nchans * fft_len + split_tw) *
           sizeof(c32);
}

int sw_cdd_chirps(const float* h_dms, int ndms, int nchans, int fft_len,
                  double low_freq, double bw, void* d_setup, sw_stream_t stream)
{
    const int logn = log2_exact(fft_len);
    SW_REQUIRE(logn >= 8 && logn <= 16,
               "coherent dedispersion: fft_len must be a power of two in [256, 65536]");
    SW_REQUIRE(h_dms && ndms > 0 && ndms <= kMaxDms, "coherent dedispersion: 1..%d DMs", kMaxDms);
    SW_REQUIRE(d_setup && nchans > 0, "coherent dedispersion: bad setup arguments");
    const int plog = logn > kSplitLog ? kSplitLog : logn;
    const Plan P = make_plan(plog);
    c32* tw = static_cast<c32*>(d_setup);
    c32* ch = tw + P.tw_total + kSetupGap;
    twiddle_k<<<64, 256, 0, as_cuda(stream)>>>(tw, plog);
    SW_LAUNCH_CHECK();
    // the words after the twiddle tables flag the DMs of exactly 0
    ZeroFlags zf{};
    for(int d = 0; d < ndms; ++d) zf.f[d] = h_dms[d] == 0.0f ? 1u : 0u;
    set_flags_k<<<1, kMaxDms, 0, as_cuda(stream)>>>(reinterpret_cast<uint32_t*>(tw + P.tw_total),
                                                     zf);
    SW_LAUNCH_CHECK();
    SetupArgs S{};
    S.logn      = logn;
    S.ndms      = ndms;
    S.nchans    = nchans;
    S.low_freq  = low_freq;
    S.coarse_bw = bw / nchans;
    S.fine_bw   = S.coarse_bw / fft_len;
    for(int d = 0; d < ndms; ++d)
        S.prefactor[d] = -1.0 * (2.0 * 3.1415926535897932385) * 4.148806423e15 * (double)h_dms[d];
    if(logn > kSplitLog) {
        const int split = fft_len / kSplitM;
        chirp_split_k<<<148 * 4, 256, 0, as_cuda(stream)>>>(ch, S, split);
        SW_LAUNCH_CHECK();
        split_twiddle_k<<<64, 256, 0, as_cuda(stream)>>>(ch + (size_t)ndms * nchans * fft_len,
                                                         split);
        SW_LAUNCH_CHECK();
    } else {
        chirp_k<<<148 * 4, 256, 0, as_cuda(stream)>>>(ch, S);
        SW_LAUNCH_CHECK();
    }
    return SW_OK;
}

size_t sw_cdd_workspace_bytes(int nchans, int npol, int nant, int nsamples, int fft_len,
                              int overlap, int ndms)
{
    const int logn = log2_exact(fft_len);
    if(logn <= kSplitLog) return 0;
    if(logn > 16 || overlap < 0 || overlap >= fft_len || nsamples <= 0 || ndms <= 0) return 0;
    const size_t items = (size_t)nchans * npol * nant * cdiv(nsamples, fft_len - overlap);
    return items * ndms * fft_len * sizeof(c32);
}

int sw_coherent_dedisperse_ws(const void* d_fpact_in, size_t row_stride, int nchans, int npol,
                              int nant, int nsamples, int fft_len, int overlap, int lag,
                              const void* d_setup, int ndms, void* const* h_d_out,
                              size_t out_row_stride, void* d_workspace,
                              size_t workspace_bytes, float* d_debug_f32,
                              sw_stream_t stream)
{
    SW_REQUIRE(d_setup, "coherent dedispersion: null setup");
    return launch_cdd(d_fpact_in, row_stride, nchans, npol, nant, nsamples, fft_len, overlap,
                      lag, d_setup, ndms, nchans, 0, 0, ndms, h_d_out, out_row_stride,
                      d_workspace, workspace_bytes, d_debug_f32, stream);
}

int sw_coherent_dedisperse_channel(const void* d_fpact_in, size_t row_stride, int npol,
                                   int nant, int nsamples, int fft_len, int overlap, int lag,
                                   const void* d_setup, int setup_ndms, int setup_nchans,
                                   int freq_idx, int dm_idx, void* d_out,
                                   size_t out_row_stride, void* d_workspace,
                                   size_t workspace_bytes, sw_stream_t stream)
{
    SW_REQUIRE(d_setup && d_out, "coherent dedispersion: null pointer");
    SW_REQUIRE(setup_ndms > 0 && setup_nchans > 0 && freq_idx >= 0 && freq_idx < setup_nchans &&
                   dm_idx >= 0 && dm_idx < setup_ndms,
               "coherent dedispersion: channel %d / DM %d outside the setup (%d channels, %d DMs)",
               freq_idx, dm_idx, setup_nchans, setup_ndms);
    void* outs[1] = {d_out};
    return launch_cdd(d_fpact_in, row_stride, 1, npol, nant, nsamples, fft_len, overlap, lag,
                      d_setup, setup_ndms, setup_nchans, freq_idx, dm_idx, 1, outs,
                      out_row_stride, d_workspace, workspace_bytes, nullptr, stream);
}

int sw_coherent_dedisperse(const void* d_fpact_in, size_t row_stride,
                           int nchans, int npol, int nant, int nsamples,
                           int fft_len, int overlap, int lag, const void* d_setup,
                           int ndms, void* const* h_d_out,
                           size_t out_row_stride, sw_stream_t stream)
{
    SW_REQUIRE(fft_len <= kSplitM,
               "coherent dedispersion: fft_len %d > %d needs sw_coherent_dedisperse_ws", fft_len,
               kSplitM);
    return sw_coherent_dedisperse_ws(d_fpact_in, row_stride, nchans, npol, nant, nsamples,
                                     fft_len, overlap, lag, d_setup, ndms, h_d_out, out_row_stride,
                                     nullptr, 0, nullptr, stream);
}

}  // extern "C"
