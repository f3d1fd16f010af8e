// CoherentBeamformer on the B200: tcgen05 int8 tensor-core GEMM with a fused
// detection / tscrunch / IB-subtraction / quantisation epilogue.
//
// Reference: cpp/skyweaver/src/CoherentBeamformer.cu:12-174 (dp4a on CUDA
// cores) and its CPU form cpp/skyweaver/test/src/CoherentBeamformerTester.cu
// :43-152.
//
// Formulation (per channel f):
//   A  (M = 128 beams x K = 2*nant int8, K-major, SMEM via TMA):
//        re block rows (w_re, -w_im) per antenna, im block rows (w_im, w_re)
//   B  (N = 2 pols x 64 samples, K = (antenna, re|im), MN-major): the planar
//        FPACT voltage rows, one TMA box [2 pols][2*nant rows][64 samples]
//   D_re = A_re . B, D_im = A_im . B  (int32 in TMEM, exact)
// so TMEM lane b holds Re and Im of beam b for both pols and all 64 samples
// of the tile and the whole Stokes / tscrunch reduction is thread local.
// The epilogue repeats the reference's float operations in the reference's
// order with IEEE single rounding, so the int8 output is bit-identical to
// the CPU implementation.
//
// Roles (one CTA per SM, persistent over a ragged work queue):
//   warp 0      TMA producer (weights double buffered, voltages 4 stages)
//   warp 1      TMEM allocator + single-thread MMA issuer
//   warps 2..17 epilogue, two groups of 8 taking alternate tiles (group g
//               drains accumulator buffer g, and frees the tile's voltage
//               stage once its accumulators are complete); in a group two
//               warps per TMEM lane quarter, 32 samples of the tile apiece
// TMEM: 512 columns = 2 accumulator buffers x (D_re 128 | D_im 128).
// Every wait is bounded by a kernel-wide deadline; on expiry the CTA records
// DEV_ERR_CB_TIMEOUT in the device error word, stops issuing work, waits
// (bounded) for the copies and MMAs it has in flight and exits.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "sw_common.cuh"

namespace swb {
namespace cb {

constexpr int kM           = 128;  // beams per tile
constexpr int kTileT       = 64;   // samples per tile
constexpr int kN           = 2 * kTileT;
// Pipeline depths (copies in flight ahead of the MMAs): runtime choices,
// voltage stages 2..8 (default 4) and weight stages 2..3 (default 2), picked
// per shape by sw_autotune.
constexpr int kVStagesDefault = 4, kVStagesMax = 8;
constexpr int kWStagesDefault = 2, kWStagesMax = 3;
constexpr int kTilesPerItem = 64;  // default work item: 4096 samples of one channel
constexpr int kMaxDm       = 16;
constexpr int kMaxProblems = 96;
// Epilogue warps: two groups of 8, one per accumulator buffer, so that each
// warp reduces 32 samples of every other tile (per-tile overheads are paid
// once per 32 samples instead of once per 16: measured 2.6 % faster than
// 16 warps sharing every tile).
constexpr int kEpiWarps    = 16;
static_assert(kEpiWarps == 8 || kEpiWarps == 16, "one or two epilogue warps per TMEM lane quarter");
constexpr int kThreads     = 32 * (2 + kEpiWarps);
constexpr int kTmemCols    = 512;

struct Problem {
    int8_t* out;
    const float* ib_raw;
    int dm;
    int beam_start;
    int beam_count;
    int item_start;
};

struct Params {
    CUtensorMap vmap[kMaxDm];
    CUtensorMap wmap;
    Problem prob[kMaxProblems];
    int nproblems, nitems;
    int nchans, nsamples, nant, nbeams, tscrunch, stokes, ib_subtract;
    int kbytes, ntc, tpi;
    size_t sample_offset;
    const float* scale;
    const float* offset;
    const int* mapping;
    int32_t* debug;
    int* err;
    uint32_t idesc;
    uint32_t w_layout, w_sbo16, v_lbo16;
    int vstages, wstages;  // pipeline depths
    unsigned long long timeout_ns;
    int test_stall;  // self-test: the producer issues nothing, so waits run out
};

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Barrier and copy helpers take shared-window addresses (uint32_t), so that
// the single-thread producer and MMA roles step through their stages with
// plain adds.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the kernel-wide deadline passed or another role
// already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          volatile int* abort_flag,
                                          unsigned long long deadline, int* err)
{
    if(mbar_try_wait(bar, parity)) return true;
    // Slow path: suspend in the barrier (up to 20 us per poll, woken when the
    // phase completes) instead of spinning, so that waiting warps do not take
    // issue slots from the warps doing the work; the abort flag and the
    // deadline are checked every 16 polls.
    for(uint32_t n = 1;; ++n) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(20000u)
            : "memory");
        if(ok) return true;
        if((n & 15u) == 0) {
            if(*abort_flag) return false;
            if(globaltimer() > deadline) {
                *abort_flag = 1;
                if(err) atomicExch(err, DEV_ERR_CB_TIMEOUT);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map,
                                            uint32_t bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map,
                                            uint32_t bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// tcgen05 shared-memory matrix descriptor (sm_100 "version 1" format),
// kept as its two 32-bit words.  The low word holds the start address >> 4
// (bits 0-13) and the leading byte offset >> 4 (bits 16-29); the high word
// the stride byte offset >> 4 (bits 0-13), the version bit (14) and the
// swizzle mode (bits 29-31).  Shared-memory addresses are below 2^18, so a
// K step or a pipeline stage is a plain add on the low word.
__device__ __forceinline__ uint32_t desc_lo(uint32_t saddr, uint32_t lbo16)
{
    return ((saddr >> 4) & 0x3FFFu) | ((lbo16 & 0x3FFFu) << 16);
}
__device__ __forceinline__ uint32_t desc_hi(uint32_t sbo16, uint32_t layout)
{
    return (sbo16 & 0x3FFFu) | (1u << 14) | ((layout & 7u) << 29);
}

// D (+)= A.B; ACC = 0 overwrites the accumulator (first K step).
template <int ACC>
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint32_t a_lo, uint32_t a_hi,
                                       uint32_t b_lo, uint32_t b_hi, uint32_t idesc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t.reg .b64 ad, bd;\n\t"
        "setp.ne.b32 p, %6, 0;\n\t"
        "mov.b64 ad, {%1, %2};\n\t"
        "mov.b64 bd, {%3, %4};\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], ad, bd, %5, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_lo), "r"(a_hi), "r"(b_lo), "r"(b_hi), "r"(idesc), "n"(ACC));
}

// All MMAs of one tile: KS K steps of 32 bytes, D_re then D_im per step.
// A K step is +32 bytes along the K-major weights and +2048 bytes (32
// voltage rows x 64 samples) along the MN-major voltages.
template <int KS>
__device__ __forceinline__ void mma_tile(uint32_t d_re, uint32_t a_re, uint32_t a_im,
                                         uint32_t a_hi, uint32_t b_lo, uint32_t b_hi,
                                         uint32_t idesc)
{
    mma_i8<0>(d_re, a_re, a_hi, b_lo, b_hi, idesc);
    mma_i8<0>(d_re + 128, a_im, a_hi, b_lo, b_hi, idesc);
#pragma unroll
    for(int ks = 1; ks < KS; ++ks) {
        mma_i8<1>(d_re, a_re + 2 * ks, a_hi, b_lo + 128 * ks, b_hi, idesc);
        mma_i8<1>(d_re + 128, a_im + 2 * ks, a_hi, b_lo + 128 * ks, b_hi, idesc);
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

#define SW_TMEM_LD16(taddr, r)                                                             \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "                                 \
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"        \
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), \
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),            \
                   "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])         \
                 : "r"(taddr))

#define SW_TMEM_LD8(taddr, r)                                                              \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"    \
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),  \
                   "=r"(r[6]), "=r"(r[7])                                                   \
                 : "r"(taddr))

// ------------------------------------------------- exact packed arithmetic
// Pairs of IEEE single operations (.rn, never contracted into an FMA), so
// each element is rounded exactly like the reference's scalar host code.
__device__ __forceinline__ uint64_t pack2(float lo, float hi)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack2(uint64_t v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c)
{
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b)
{
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Exact int32 -> float: every beam voltage is below 2^21 in magnitude, so the
// round-to-nearest conversion is exact.  (Measured against a magic-constant
// scheme, 1.5*2^23 preloaded into TMEM and subtracted in float, and against
// an integer add of that constant: the plain conversion was fastest, since
// it needs no TMEM re-arm and no constant registers.)
__device__ __forceinline__ uint64_t pair_f(const uint32_t* w, int t)
{
    return pack2(__int2float_rn((int)w[t]), __int2float_rn((int)w[t + 1]));
}

// Stokes of L consecutive samples from the exact beam voltages
// (p0 = r0 + i i0, p1 = r1 + i i1) with the reference's operation order
// (beamformer_utils.cuh:125-140: cuCmagf, cuCmulf with cuConjf), two samples
// per packed instruction.  Products are fma(a, b, +0): one rounding exactly
// like a multiply, and since an FMA result cannot be contracted into the
// packed add that consumes it, every sum is also a single rounding.  (A
// packed multiply feeding a packed add was measured to be contracted into an
// FMA, which moved 1 in ~1e5 outputs by one LSB.)
template <int STOKES, int L>
__device__ __forceinline__ void stokes_n(const uint32_t* r0, const uint32_t* r1,
                                         const uint32_t* i0, const uint32_t* i1, float* st)
{
    const uint64_t Z = pack2(0.0f, 0.0f);
#pragma unroll
    for(int t = 0; t < L; t += 2) {
        const uint64_t R0 = pair_f(r0, t), R1 = pair_f(r1, t);
        const uint64_t I0 = pair_f(i0, t), I1 = pair_f(i1, t);
        uint64_t S;
        if constexpr(STOKES <= 1) {
            const uint64_t E0 = add2(fma2(R0, R0, Z), fma2(I0, I0, Z));  // |p0|^2
            const uint64_t E1 = add2(fma2(R1, R1, Z), fma2(I1, I1, Z));  // |p1|^2
            S = STOKES == 0 ? add2(E0, E1) : sub2(E0, E1);
        } else if constexpr(STOKES == 2) {
            // 2*Re(p0 conj p1) = 2*(r0 r1 - i0 (-i1)) = 2*(r0 r1 + i0 i1)
            S = mul2(add2(fma2(R0, R1, Z), fma2(I0, I1, Z)), pack2(2.0f, 2.0f));
        } else {
            // 2*Im(p0 conj p1) = 2*(r0 (-i1) + i0 r1) = 2*(i0 r1 - r0 i1)
            S = mul2(sub2(fma2(I0, R1, Z), fma2(R0, I1, Z)), pack2(2.0f, 2.0f));
        }
        unpack2(S, st[t], st[t + 1]);
    }
}

// All four Stokes parameters (FullStokesBeamformerTraits,
// beamformer_utils.cuh:198-278): component c is computed exactly like the
// single-Stokes mode c, so st[c] equals stokes_n<c> element for element.
template <int L>
__device__ __forceinline__ void stokes_iquv(const uint32_t* r0, const uint32_t* r1,
                                            const uint32_t* i0, const uint32_t* i1,
                                            float (*st)[L])
{
    const uint64_t Z = pack2(0.0f, 0.0f), two = pack2(2.0f, 2.0f);
#pragma unroll
    for(int t = 0; t < L; t += 2) {
        const uint64_t R0 = pair_f(r0, t), R1 = pair_f(r1, t);
        const uint64_t I0 = pair_f(i0, t), I1 = pair_f(i1, t);
        const uint64_t E0 = add2(fma2(R0, R0, Z), fma2(I0, I0, Z));
        const uint64_t E1 = add2(fma2(R1, R1, Z), fma2(I1, I1, Z));
        unpack2(add2(E0, E1), st[0][t], st[0][t + 1]);
        unpack2(sub2(E0, E1), st[1][t], st[1][t + 1]);
        unpack2(mul2(add2(fma2(R0, R1, Z), fma2(I0, I1, Z)), two), st[2][t], st[2][t + 1]);
        unpack2(mul2(sub2(fma2(I0, R1, Z), fma2(R0, I1, Z)), two), st[3][t], st[3][t + 1]);
    }
}

struct Item {
    int p, f, tc, b0;
};

__device__ __forceinline__ Item decode(const Params& P, int item)
{
    int p = 0;
    while(p + 1 < P.nproblems && P.prob[p + 1].item_start <= item) ++p;
    const Problem& pr = P.prob[p];
    const int nblk  = (pr.beam_count + kM - 1) / kM;
    const int local = item - pr.item_start;
    Item it;
    it.p  = p;
    const int mb = local % nblk;
    const int rest = local / nblk;
    it.tc = rest % P.ntc;
    it.f  = rest / P.ntc;
    it.b0 = pr.beam_start + mb * kM;
    return it;
}

// DBG instances also write the exact int32 beam voltages to P.debug; the
// production instances carry no debug path (it costs ~20 registers and a
// branch per load group).
template <int TS, int STOKES, bool DBG>
__global__ void __launch_bounds__(kThreads, 1)
cb_kernel(const __grid_constant__ Params P)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte aligned carve-up
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int wtile = kM * P.kbytes;              // one A block
    const int vtile = 2 * P.kbytes * kTileT;       // one B stage
    const int nvs = P.vstages, nws = P.wstages;
    uint8_t* wbuf = base;                          // [nws][2][wtile]
    uint8_t* vbuf = wbuf + nws * 2 * wtile;        // [nvs][vtile]
    uint64_t* bars = reinterpret_cast<uint64_t*>(vbuf + nvs * vtile);
    uint64_t* v_full    = bars;
    uint64_t* v_empty   = v_full + nvs;
    uint64_t* w_full    = v_empty + nvs;
    uint64_t* w_empty   = w_full + nws;
    uint64_t* acc_full  = w_empty + nws;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain     = acc_empty + 2;  // MMA completion on abort
    uint32_t* s_tmem    = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* s_abort = reinterpret_cast<volatile int*>(s_tmem + 1);

    // shared-window addresses: barrier k of an array is at base + 8 k
    const uint32_t v_full_s = smem_u32(v_full), v_empty_s = smem_u32(v_empty);
    const uint32_t w_full_s = smem_u32(w_full), w_empty_s = smem_u32(w_empty);
    const uint32_t acc_full_s = smem_u32(acc_full), acc_empty_s = smem_u32(acc_empty);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const unsigned long long deadline = globaltimer() + P.timeout_ns;

    if(threadIdx.x == 0) {
        for(int i = 0; i < nvs; ++i) { mbar_init(&v_full[i], 1); mbar_init(&v_empty[i], 1); }
        for(int i = 0; i < nws; ++i) { mbar_init(&w_full[i], 1); mbar_init(&w_empty[i], 1); }
        for(int i = 0; i < 2; ++i) { mbar_init(&acc_full[i], 1); mbar_init(&acc_empty[i], kEpiWarps / 2); }
        mbar_init(drain, 1);
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_tmem;
    const int ntiles_gulp = P.nsamples / kTileT;

    if(warp == 0) {
        if(lane == 0 && !P.test_stall) {
            // ---------------------------------------------------- producer
            const uint32_t wbuf_s = smem_u32(wbuf), vbuf_s = smem_u32(vbuf);
            int vs = 0, ws = 0;
            uint32_t vph = 0, wph = 0;
            // stages armed so far and the phase parity of each one's last arm
            uint32_t v_armed = 0, v_par = 0, w_armed = 0, w_par = 0;
            for(int item = blockIdx.x; item < P.nitems && !*s_abort; item += gridDim.x) {
                const Item it = decode(P, item);
                const Problem& pr = P.prob[it.p];
                if(!mbar_wait(w_empty_s + 8 * ws, wph ^ 1, s_abort, deadline, P.err)) break;
                const uint32_t wbar = w_full_s + 8 * ws;
                mbar_expect_tx(wbar, 2 * wtile);
                w_armed |= 1u << ws;
                w_par = (w_par & ~(1u << ws)) | (wph << ws);
                const uint32_t wdst = wbuf_s + ws * 2 * wtile;
                tma_load_2d(wdst, &P.wmap, wbar, 0, (it.f * 2 + 0) * P.nbeams + it.b0);
                tma_load_2d(wdst + wtile, &P.wmap, wbar, 0, (it.f * 2 + 1) * P.nbeams + it.b0);
                if(++ws == nws) { ws = 0; wph ^= 1; }
                const int tile0 = it.tc * P.tpi;
                const int tile1 = min(ntiles_gulp, tile0 + P.tpi);
                const CUtensorMap* vmap = &P.vmap[pr.dm];
                int x = (int)(P.sample_offset + (size_t)tile0 * kTileT);
                for(int tile = tile0; tile < tile1; ++tile, x += kTileT) {
                    if(!mbar_wait(v_empty_s + 8 * vs, vph ^ 1, s_abort, deadline, P.err)) break;
                    const uint32_t vbar = v_full_s + 8 * vs;
                    mbar_expect_tx(vbar, vtile);
                    v_armed |= 1u << vs;
                    v_par = (v_par & ~(1u << vs)) | (vph << vs);
                    tma_load_3d(vbuf_s + vs * vtile, vmap, vbar, x, 0, it.f * 2);
                    if(++vs == nvs) { vs = 0; vph ^= 1; }
                }
            }
            // After an abort, let every copy still in flight land before the
            // CTA exits (each stage's last armed phase completes when its
            // bytes arrive; bounded like every other wait).
            if(*s_abort) {
                const unsigned long long until = globaltimer() + 100ull * 1000 * 1000;
                for(int i = 0; i < nvs; ++i)
                    if(v_armed >> i & 1)
                        while(!mbar_try_wait(v_full_s + 8 * i, v_par >> i & 1) && globaltimer() < until) {}
                for(int i = 0; i < nws; ++i)
                    if(w_armed >> i & 1)
                        while(!mbar_try_wait(w_full_s + 8 * i, w_par >> i & 1) && globaltimer() < until) {}
            }
        }
    } else if(warp == 1) {
        if(lane == 0) {
            // ------------------------------------------------- MMA issuer
            // This thread shares its SM sub-partition with four busy
            // epilogue warps, so its per-tile instruction count bounds how
            // fast the tensor pipe is fed: descriptors are precomputed words
            // and each tile is one straight run of MMAs.
            int vs = 0, ws = 0, ab = 0;
            uint32_t vph = 0, wph = 0, aph = 0;
            const int ksteps = P.kbytes / 32;
            const uint32_t a_hi = desc_hi(P.w_sbo16, P.w_layout);
            const uint32_t b_hi = desc_hi(32, 4 /*SW64*/);
            const uint32_t a_lo0 = desc_lo(smem_u32(wbuf), 1);
            const uint32_t b_lo0 = desc_lo(smem_u32(vbuf), P.v_lbo16);
            for(int item = blockIdx.x; item < P.nitems && !*s_abort; item += gridDim.x) {
                const Item it = decode(P, item);
                if(!mbar_wait(w_full_s + 8 * ws, wph, s_abort, deadline, P.err)) break;
                const uint32_t a_re = a_lo0 + ((ws * 2 * wtile) >> 4);
                const uint32_t a_im = a_re + (wtile >> 4);
                const int tile0 = it.tc * P.tpi;
                const int tile1 = min(ntiles_gulp, tile0 + P.tpi);
                bool ok = true;
                for(int tile = tile0; tile < tile1; ++tile) {
                    if(!mbar_wait(v_full_s + 8 * vs, vph, s_abort, deadline, P.err)) { ok = false; break; }
                    // phase 0 of acc_empty is completed by the epilogue
                    // warps' initial arrival (both buffers start free)
                    if(!mbar_wait(acc_empty_s + 8 * ab, aph, s_abort, deadline, P.err)) { ok = false; break; }
                    fence_after();
                    const uint32_t b_lo = b_lo0 + ((vs * vtile) >> 4);
                    const uint32_t d_re = tmem + ab * 256;  // D_im at d_re + 128
                    if(ksteps == 4) mma_tile<4>(d_re, a_re, a_im, a_hi, b_lo, b_hi, P.idesc);
                    else if(ksteps == 2) mma_tile<2>(d_re, a_re, a_im, a_hi, b_lo, b_hi, P.idesc);
                    else mma_tile<1>(d_re, a_re, a_im, a_hi, b_lo, b_hi, P.idesc);
                    // one commit per tile: the epilogue frees the voltage stage when
                    // it sees the accumulators (a second commit per tile, for the
                    // stage, measured 2.5 % slower)
                    mma_commit(acc_full_s + 8 * ab);
                    if(++vs == nvs) { vs = 0; vph ^= 1; }
                    if(++ab == 2) { ab = 0; aph ^= 1; }
                }
                mma_commit(w_empty_s + 8 * ws);
                if(++ws == nws) { ws = 0; wph ^= 1; }
                if(!ok) break;
            }
            // After an abort, wait (bounded) for the MMAs already issued, so
            // that none is still reading shared memory or writing TMEM when
            // the CTA frees them.
            if(*s_abort) {
                const uint32_t drain_s = smem_u32(drain);
                mma_commit(drain_s);
                const unsigned long long until = globaltimer() + 100ull * 1000 * 1000;
                while(!mbar_try_wait(drain_s, 0) && globaltimer() < until) {}
            }
        }
    } else {
        // ------------------------------------------------------ epilogue
        constexpr int kHalves = kEpiWarps / 8;       // warps per TMEM lane quarter and group
        constexpr int kSlice  = kTileT / kHalves;    // samples per warp per tile
        // TMEM columns per load group: 16 (measured 1.5 % faster than 8),
        // except for full Stokes at tscrunch <= 4, whose many outputs per
        // group leave too few registers for it
        constexpr int kG      = (STOKES == 4 && TS <= 4) ? 8 : 16;
        constexpr int kGroups = kSlice / kG;         // column groups per warp
        // Release the accumulator buffer as soon as the tile's last column
        // group is in registers, before its arithmetic, when several outputs
        // per group follow the last load (tscrunch <= 8: measured 3.4 %
        // faster at tscrunch 8); at tscrunch 16 the release after the
        // arithmetic measured 0.9 % faster.
        constexpr bool kEarlyRelease = TS <= 8;
        const int q   = warp & 3;               // TMEM lane quarter of this warp
        const int h   = ((warp - 2) >> 2) % kHalves;  // which part of the tile's samples
        const int grp = (warp - 2) / (kEpiWarps / 2); // accumulator buffer this warp drains
        const int F = P.nchans;
        const int nout = P.nsamples / TS;
        const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
        // release this group's accumulator buffer to the MMA warp (phase 0)
        fence_before();
        __syncwarp();
        if(lane == 0) mbar_arrive(&acc_empty[grp]);
        int ab = 0;        // accumulator buffer of the CTA's next tile
        int seq = 0;       // CTA tile sequence number of the item's first tile
        uint32_t aph = 0;  // phase parity of this group's buffer
        for(int item = blockIdx.x; item < P.nitems && !*s_abort; item += gridDim.x) {
            const Item it = decode(P, item);
            const Problem& pr = P.prob[it.p];
            const int b = it.b0 + q * 32 + lane;
            const bool valid = (b < pr.beam_start + pr.beam_count) && (b < P.nbeams);
            const int bs = valid ? P.mapping[b] : 0;
            const float scale = P.scale[bs * F + it.f];
            const float offs  = P.offset[bs * F + it.f];
            const int tile0 = it.tc * P.tpi;
            const int tile1 = min(ntiles_gulp, tile0 + P.tpi);
            // tiles alternate between the buffers: this group takes every
            // other tile, starting with the first one that lands in its buffer
            const int first = tile0 + ((ab ^ grp) & 1);
            bool ok = true;
            constexpr int NC = STOKES == 4 ? 4 : 1;  // output components
            constexpr int kEmits = kSlice / TS;      // outputs per warp per tile
            // Output and IB-power elements of this warp's first output in
            // its first tile; both advance by 2 kTileT / TS output samples.
            const int to0 = (first * kTileT + h * kSlice) / TS;
            int8_t* outp = pr.out + (((size_t)to0 * F + it.f) * P.nbeams + b) * NC;
            const float* ibq =
                P.ib_subtract ? pr.ib_raw + (((size_t)bs * nout + to0) * F + it.f) * NC : nullptr;
            const size_t out_emit = (size_t)F * P.nbeams * NC;  // next output sample
            const size_t ib_emit  = (size_t)F * NC;
            // IB powers of this warp's outputs in the tile, fetched before the
            // accumulator wait so that their latency hides behind it
            constexpr bool kPrefetch = kEmits * NC <= 4;
            float ibp[kPrefetch ? kEmits * NC : 1];
            for(int tile = first; tile < tile1; tile += 2) {
                if constexpr(kPrefetch) {
                    if(P.ib_subtract) {
#pragma unroll
                        for(int e = 0; e < kEmits; ++e) {
                            if constexpr(NC == 1) {
                                ibp[e] = ibq[e * ib_emit];
                            } else {
                                const float4 v = reinterpret_cast<const float4*>(ibq)[e * F];
                                ibp[4 * e] = v.x; ibp[4 * e + 1] = v.y;
                                ibp[4 * e + 2] = v.z; ibp[4 * e + 3] = v.w;
                            }
                        }
                    }
                }
                if(!mbar_wait(acc_full_s + 8 * grp, aph, s_abort, deadline, P.err)) { ok = false; break; }
                // the tile's MMAs are complete, so its voltage stage is free
                if(warp == 2 + (kEpiWarps / 2) * grp && lane == 0)
                    mbar_arrive(&v_empty[(seq + tile - tile0) % nvs]);
                fence_after();
                float power[NC];  // carried across groups while tscrunch > 8
#pragma unroll
                for(int c = 0; c < NC; ++c) power[c] = 0.0f;
                // One column group at a time: load, wait, reduce.  (Loading
                // the next group ahead of the arithmetic, or both groups at
                // once, was measured 1-2.5 % slower.)
                const uint32_t ta0 = lane_base + grp * 256 + h * kSlice;
#pragma unroll
                for(int g = 0; g < kGroups; ++g) {
                    uint32_t r0[kG], r1[kG], i0[kG], i1[kG];
                    const uint32_t ta = ta0 + g * kG;
                    if constexpr(kG == 16) {
                        SW_TMEM_LD16(ta, r0);
                        SW_TMEM_LD16(ta + 64, r1);
                        SW_TMEM_LD16(ta + 128, i0);
                        SW_TMEM_LD16(ta + 192, i1);
                    } else {
                        SW_TMEM_LD8(ta, r0);
                        SW_TMEM_LD8(ta + 64, r1);
                        SW_TMEM_LD8(ta + 128, i0);
                        SW_TMEM_LD8(ta + 192, i1);
                    }
                    tmem_wait_ld();
                    if(kEarlyRelease && g == kGroups - 1) {
                        fence_before();
                        __syncwarp();
                        if(lane == 0) mbar_arrive(&acc_empty[grp]);
                    }
                    const int tbase = tile * kTileT + h * kSlice + g * kG;
                    if(DBG && valid) {
                        int2* dbg = reinterpret_cast<int2*>(P.debug);
                        for(int t = 0; t < kG; ++t) {
                            const size_t base_t = (size_t)it.f * P.nsamples + tbase + t;
                            dbg[(base_t * 2 + 0) * P.nbeams + b] =
                                make_int2((int)r0[t], (int)i0[t]);
                            dbg[(base_t * 2 + 1) * P.nbeams + b] =
                                make_int2((int)r1[t], (int)i1[t]);
                        }
                    }
                    float st[NC][kG];
                    if constexpr(STOKES == 4) stokes_iquv<kG>(r0, r1, i0, i1, st);
                    else stokes_n<STOKES, kG>(r0, r1, i0, i1, st[0]);
#pragma unroll
                    for(int t = 0; t < kG; ++t) {
#pragma unroll
                        for(int c = 0; c < NC; ++c) power[c] = fadd(power[c], st[c][t]);
                        const int u = g * kG + t;  // sample within this warp's slice
                        const bool emit = ((u + 1) % TS) == 0;
                        if(emit) {
                            const int e = u / TS;  // emit index within the slice
                            if constexpr(NC == 1) {
                                float v;
                                if(P.ib_subtract) {
                                    const float ib = kPrefetch ? ibp[kPrefetch ? e : 0] : ibq[e * ib_emit];
                                    v = rintf(fdiv(fsub(power[0], fmul(ib, 16129.0f)), scale));
                                } else if(STOKES == 0) {
                                    v = rintf(fdiv(fsub(power[0], offs), scale));
                                } else {
                                    v = rintf(fdiv(power[0], scale));
                                }
                                if(valid) outp[e * out_emit] = clamp_i8(v);
                            } else {
                                // char4 {I, Q, U, V}; the IB power is float4
                                float v[4];
                                if(P.ib_subtract) {
                                    const float4 ib = kPrefetch
                                        ? make_float4(ibp[0], ibp[1], ibp[2], ibp[3])
                                        : reinterpret_cast<const float4*>(ibq)[e * F];
                                    v[0] = rintf(fdiv(fsub(power[0], fmul(ib.x, 16129.0f)), scale));
                                    v[1] = rintf(fdiv(fsub(power[1], fmul(ib.y, 16129.0f)), scale));
                                    v[2] = rintf(fdiv(fsub(power[2], fmul(ib.z, 16129.0f)), scale));
                                    v[3] = rintf(fdiv(fsub(power[3], fmul(ib.w, 16129.0f)), scale));
                                } else {
                                    v[0] = rintf(fdiv(fsub(power[0], offs), scale));
                                    v[1] = rintf(fdiv(power[1], scale));
                                    v[2] = rintf(fdiv(power[2], scale));
                                    v[3] = rintf(fdiv(power[3], scale));
                                }
                                if(valid)
                                    reinterpret_cast<char4*>(outp)[e * F * P.nbeams] =
                                        make_char4(clamp_i8(v[0]), clamp_i8(v[1]),
                                                   clamp_i8(v[2]), clamp_i8(v[3]));
                            }
#pragma unroll
                            for(int c = 0; c < NC; ++c) power[c] = 0.0f;
                        }
                    }
                }
                if(!kEarlyRelease) {
                    fence_before();
                    __syncwarp();
                    if(lane == 0) mbar_arrive(&acc_empty[grp]);
                }
                aph ^= 1;
                outp += (2 * kTileT / TS) * out_emit;
                if(P.ib_subtract) ibq += (2 * kTileT / TS) * ib_emit;
            }
            if(!ok) break;
            ab ^= (tile1 - tile0) & 1;
            seq += tile1 - tile0;
        }
    }
    fence_before();
    __syncthreads();
    if(warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
    }
}

// ------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
               cudaSuccess &&
           q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

int make_vmap(CUtensorMap* map, const void* fpact, const sw_cb_shape& s)
{
    auto fn = encode_fn();
    SW_REQUIRE(fn != nullptr, "cuTensorMapEncodeTiled is unavailable");
    const cuuint64_t dims[3]    = {(cuuint64_t)s.row_stride, (cuuint64_t)(2 * s.nantennas),
                                   (cuuint64_t)(2 * s.nchans)};
    const cuuint64_t strides[2] = {(cuuint64_t)s.row_stride,
                                   (cuuint64_t)(2 * s.nantennas) * s.row_stride};
    const cuuint32_t box[3]     = {(cuuint32_t)kTileT, (cuuint32_t)(2 * s.nantennas), 2};
    const cuuint32_t es[3]      = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(fpact), dims,
                    strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (voltages) failed: %d", (int)r);
        return SW_ERR_CUDA;
    }
    return SW_OK;
}

int make_wmap(CUtensorMap* map, const void* w, const sw_cb_shape& s)
{
    auto fn = encode_fn();
    SW_REQUIRE(fn != nullptr, "cuTensorMapEncodeTiled is unavailable");
    const int kb = 2 * s.nantennas;
    const cuuint64_t dims[2]    = {(cuuint64_t)kb, (cuuint64_t)(2 * s.nchans) * s.nbeams};
    const cuuint64_t strides[1] = {(cuuint64_t)kb};
    const cuuint32_t box[2]     = {(cuuint32_t)kb, (cuuint32_t)kM};
    const cuuint32_t es[2]      = {1, 1};
    const CUtensorMapSwizzle sw = kb == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                : kb == 64  ? CU_TENSOR_MAP_SWIZZLE_64B
                                            : CU_TENSOR_MAP_SWIZZLE_32B;
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(w), dims, strides,
                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled (weights) failed: %d", (int)r);
        return SW_ERR_CUDA;
    }
    return SW_OK;
}

// Kernel parameter block of the launch being prepared on this host thread
// (~6 KB, kept off the stack; copied into the launch).
Params& launch_params()
{
    static thread_local Params P;
    return P;
}

int dispatch_ts(int ts, int stokes, int grid, size_t smem, cudaStream_t stream);

size_t smem_bytes(int kbytes, int vstages, int wstages)
{
    return 1024 + (size_t)wstages * 2 * kM * kbytes + (size_t)vstages * 2 * kbytes * kTileT +
           (2 * vstages + 2 * wstages + 5) * 8 + 16;
}

int num_sms()
{
    static int n = 0;
    if(n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if(n <= 0) n = 148;
    }
    return n;
}

int launch(const sw_cb_shape* s, const sw_cb_problem* probs, int nprob,
           const void* w, const float* scale, const float* offset,
           const int* mapping, int32_t* debug, cudaStream_t stream,
           unsigned long long timeout_ns = 5ull * 1000 * 1000 * 1000, int test_stall = 0)
{
    SW_REQUIRE(s && probs && nprob > 0 && w && scale && offset && mapping,
               "CoherentBeamformer: null argument");
    SW_REQUIRE(nprob <= kMaxProblems, "CoherentBeamformer: at most %d problems", kMaxProblems);
    SW_REQUIRE(s->nantennas == 16 || s->nantennas == 32 || s->nantennas == 64,
               "CoherentBeamformer: nantennas must be 16, 32 or 64 (got %d)", s->nantennas);
    SW_REQUIRE(s->nsamples > 0 && s->nsamples % kTileT == 0,
               "Number of samples must be a multiple of %d", kTileT);
    SW_REQUIRE(s->tscrunch >= 1 && s->tscrunch <= 32 && (s->tscrunch & (s->tscrunch - 1)) == 0,
               "CoherentBeamformer: tscrunch must be a power of two <= 32");
    SW_REQUIRE(s->stokes >= 0 && s->stokes <= 4, "CoherentBeamformer: bad Stokes mode");
    SW_REQUIRE(s->row_stride % 16 == 0 && s->sample_offset % 16 == 0,
               "CoherentBeamformer: FPACT stride/offset must be multiples of 16");
    SW_REQUIRE(s->sample_offset + (size_t)s->nsamples <= s->row_stride,
               "CoherentBeamformer: rows shorter than the gulp");
    SW_REQUIRE(s->nbeams > 0 && s->nchans > 0, "CoherentBeamformer: empty shape");
    SW_REQUIRE(s->row_stride <= 0x7fffffffULL, "CoherentBeamformer: row stride too large");
    const int vstages = s->voltage_stages > 0 ? s->voltage_stages : kVStagesDefault;
    const int wstages = s->weight_stages > 0 ? s->weight_stages : kWStagesDefault;
    SW_REQUIRE(vstages >= 2 && vstages <= kVStagesMax && wstages >= 2 && wstages <= kWStagesMax,
               "CoherentBeamformer: voltage stages must be 2..%d and weight stages 2..%d",
               kVStagesMax, kWStagesMax);

    Params& P = launch_params();
    memset(&P, 0, sizeof(P));
    const void* dms[kMaxDm];
    int ndm = 0, item = 0;
    SW_REQUIRE(s->tiles_per_item >= 0 && s->tiles_per_item <= 1024,
               "CoherentBeamformer: tiles_per_item must be in [0, 1024]");
    const int tpi = s->tiles_per_item > 0 ? s->tiles_per_item : kTilesPerItem;
    const int ntc = cdiv(s->nsamples / kTileT, tpi);
    for(int i = 0; i < nprob; ++i) {
        const sw_cb_problem& pr = probs[i];
        SW_REQUIRE(pr.d_fpact && pr.d_out && (pr.d_ib_raw || !s->ib_subtract),
                   "CoherentBeamformer: problem %d has a null pointer", i);
        SW_REQUIRE(s->stokes != 4 || ((reinterpret_cast<uintptr_t>(pr.d_out) & 3) == 0 &&
                                      (reinterpret_cast<uintptr_t>(pr.d_ib_raw) & 15) == 0),
                   "CoherentBeamformer: IQUV needs 4-byte aligned output and 16-byte aligned "
                   "IB powers");
        SW_REQUIRE(pr.beam_start >= 0 && pr.beam_count > 0 &&
                       pr.beam_start + pr.beam_count <= s->nbeams,
                   "CoherentBeamformer: problem %d beam range out of bounds", i);
        int d = 0;
        while(d < ndm && dms[d] != pr.d_fpact) ++d;
        if(d == ndm) {
            SW_REQUIRE(ndm < kMaxDm, "CoherentBeamformer: at most %d voltage blocks", kMaxDm);
            dms[ndm] = pr.d_fpact;
            int rc = make_vmap(&P.vmap[ndm], pr.d_fpact, *s);
            if(rc) return rc;
            ++ndm;
        }
        P.prob[i].out        = pr.d_out;
        P.prob[i].ib_raw     = pr.d_ib_raw;
        P.prob[i].dm         = d;
        P.prob[i].beam_start = pr.beam_start;
        P.prob[i].beam_count = pr.beam_count;
        P.prob[i].item_start = item;
        item += s->nchans * ntc * cdiv(pr.beam_count, kM);
    }
    int rc = make_wmap(&P.wmap, w, *s);
    if(rc) return rc;
    P.nproblems   = nprob;
    P.nitems      = item;
    P.nchans      = s->nchans;
    P.nsamples    = s->nsamples;
    P.nant        = s->nantennas;
    P.nbeams      = s->nbeams;
    P.tscrunch    = s->tscrunch;
    P.stokes      = s->stokes;
    P.ib_subtract = s->ib_subtract;
    P.kbytes      = 2 * s->nantennas;
    P.ntc         = ntc;
    P.tpi = tpi;
    P.sample_offset = s->sample_offset;
    P.scale   = scale;
    P.offset  = offset;
    P.mapping = mapping;
    P.debug   = debug;
    P.err     = device_error_ptr();
    SW_REQUIRE(P.err != nullptr, "coherent beamformer: the device error word has no address");
    // kind::i8 instruction descriptor: D=S32, A=B=S8, A K-major, B MN-major,
    // N=128 (bits 17-22: N>>3), M=128 (bits 24-28: M>>4)
    P.idesc = (2u << 4) | (1u << 7) | (1u << 10) | (0u << 15) | (1u << 16) |
              ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
    P.w_layout = P.kbytes == 128 ? 2u : P.kbytes == 64 ? 4u : 6u;  // SW128/SW64/SW32
    P.w_sbo16  = (uint32_t)(8 * P.kbytes / 16);                       // 8-row group stride
    P.v_lbo16  = (uint32_t)(2 * s->nantennas * kTileT / 16);          // pol plane stride
    P.timeout_ns = timeout_ns;                                        // 5 s by default
    P.test_stall = test_stall;
    P.vstages = vstages;
    P.wstages = wstages;

    const size_t smem = smem_bytes(P.kbytes, P.vstages, P.wstages);
    SW_REQUIRE(smem <= 227 * 1024,
               "CoherentBeamformer: %d voltage and %d weight stages need %zu bytes of shared "
               "memory (at most 232448)", P.vstages, P.wstages, smem);
    const int grid = P.nitems < num_sms() ? P.nitems : num_sms();
    return dispatch_ts(s->tscrunch, s->stokes, grid, smem, stream);
}

template <int TS, int STOKES, bool DBG>
int launch_instance(int grid, size_t smem, cudaStream_t stream)
{
    SW_CUDA_CHECK(cudaFuncSetAttribute(cb_kernel<TS, STOKES, DBG>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cb_kernel<TS, STOKES, DBG><<<grid, kThreads, smem, stream>>>(launch_params());
    SW_LAUNCH_CHECK();
    return SW_OK;
}

template <int TS, int STOKES>
int launch_variant(int grid, size_t smem, cudaStream_t stream)
{
    return launch_params().debug != nullptr ? launch_instance<TS, STOKES, true>(grid, smem, stream)
                                            : launch_instance<TS, STOKES, false>(grid, smem, stream);
}

template <int TS>
int dispatch_stokes(int stokes, int grid, size_t smem, cudaStream_t stream)
{
    switch(stokes) {
    case 0: return launch_variant<TS, 0>(grid, smem, stream);
    case 1: return launch_variant<TS, 1>(grid, smem, stream);
    case 2: return launch_variant<TS, 2>(grid, smem, stream);
    case 3: return launch_variant<TS, 3>(grid, smem, stream);
    default: return launch_variant<TS, 4>(grid, smem, stream);
    }
}

int dispatch_ts(int ts, int stokes, int grid, size_t smem, cudaStream_t stream)
{
    switch(ts) {
    case 1: return dispatch_stokes<1>(stokes, grid, smem, stream);
    case 2: return dispatch_stokes<2>(stokes, grid, smem, stream);
    case 4: return dispatch_stokes<4>(stokes, grid, smem, stream);
    case 8: return dispatch_stokes<8>(stokes, grid, smem, stream);
    case 16: return dispatch_stokes<16>(stokes, grid, smem, stream);
    default: return dispatch_stokes<32>(stokes, grid, smem, stream);
    }
}

}  // namespace cb
}  // namespace swb

extern "C" {

int sw_coherent_beamform(const sw_cb_shape* shape, const sw_cb_problem* problem,
                         const void* d_weights_gemm, const float* d_scale,
                         const float* d_offset, const int* d_mapping,
                         int32_t* d_debug_voltages, sw_stream_t stream)
{
    return swb::cb::launch(shape, problem, 1, d_weights_gemm, d_scale, d_offset, d_mapping,
                           d_debug_voltages, swb::as_cuda(stream));
}

int sw_coherent_beamform_grouped(const sw_cb_shape* shape,
                                 const sw_cb_problem* h_problems, int nproblems,
                                 const void* d_weights_gemm, const float* d_scale,
                                 const float* d_offset, const int* d_mapping,
                                 sw_stream_t stream)
{
    return swb::cb::launch(shape, h_problems, nproblems, d_weights_gemm, d_scale, d_offset,
                           d_mapping, nullptr, swb::as_cuda(stream));
}

// Bounded-wait self-test: a minimal grouped launch (16 antennas, 1 channel,
// 128 beams, 64 samples) whose producer issues no copies, so the MMA role's
// first weights wait can only end at its deadline.  The kernel must record
// its timeout in the device error word and return; the context stays usable.
int sw_cb_timeout_selftest(int timeout_us, sw_stream_t stream)
{
    SW_REQUIRE(timeout_us > 0 && timeout_us <= 10 * 1000 * 1000,
               "sw_cb_timeout_selftest: timeout must be in (0, 10 s]");
    const cudaStream_t st = swb::as_cuda(stream);
    sw_cb_shape shape{};
    shape.nantennas = 16;
    shape.nbeams = 128;
    shape.nchans = 1;
    shape.nsamples = 64;
    shape.tscrunch = 16;
    shape.stokes = 0;
    shape.ib_subtract = 1;
    shape.row_stride = 64;
    shape.sample_offset = 0;
    const size_t v_bytes = (size_t)shape.row_stride * 2 * shape.nantennas * 2 * shape.nchans;
    const size_t w_bytes = (size_t)shape.nchans * 2 * shape.nbeams * 2 * shape.nantennas;
    void *v = nullptr, *w = nullptr, *f = nullptr, *o = nullptr, *m = nullptr;
    int rc = SW_OK;
    auto fail = [](int code, const char* msg) {
        swb::set_error("sw_cb_timeout_selftest: %s", msg);
        return code;
    };
    if(cudaMalloc(&v, v_bytes) != cudaSuccess || cudaMalloc(&w, w_bytes) != cudaSuccess ||
       cudaMalloc(&f, 64 * sizeof(float)) != cudaSuccess || cudaMalloc(&o, 4096) != cudaSuccess ||
       cudaMalloc(&m, shape.nbeams * sizeof(int)) != cudaSuccess)
        rc = fail(SW_ERR_CUDA, "allocation failed");
    if(rc == SW_OK && (cudaMemsetAsync(v, 0, v_bytes, st) != cudaSuccess ||
                       cudaMemsetAsync(w, 0, w_bytes, st) != cudaSuccess ||
                       cudaMemsetAsync(f, 0, 64 * sizeof(float), st) != cudaSuccess ||
                       cudaMemsetAsync(m, 0, shape.nbeams * sizeof(int), st) != cudaSuccess))
        rc = fail(SW_ERR_CUDA, "memset failed");
    if(rc == SW_OK) {
        sw_cb_problem pr{};
        pr.d_fpact = v;
        pr.d_out = static_cast<int8_t*>(o);
        pr.d_ib_raw = static_cast<const float*>(f);
        pr.beam_start = 0;
        pr.beam_count = shape.nbeams;
        rc = swb::cb::launch(&shape, &pr, 1, w, static_cast<const float*>(f),
                             static_cast<const float*>(f), static_cast<const int*>(m), nullptr,
                             st, 1000ull * (unsigned long long)timeout_us, 1);
    }
    if(rc == SW_OK && cudaStreamSynchronize(st) != cudaSuccess)
        rc = fail(SW_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    if(rc == SW_OK) {
        int code = 0;
        rc = sw_read_device_error(&code);
        if(rc == SW_OK) {
            sw_reset_device_error();
            rc = code == swb::DEV_ERR_CB_TIMEOUT
                     ? fail(SW_ERR_TIMEOUT, "the coherent beamformer's bounded wait timed out")
                     : fail(SW_ERR_STATE, "no timeout recorded in the device error word");
        }
    }
    cudaFree(v); cudaFree(w); cudaFree(f); cudaFree(o); cudaFree(m);
    return rc;
}

}  // extern "C"
