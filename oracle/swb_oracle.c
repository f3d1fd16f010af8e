/*
 * swb_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * Plain-C restatement of the skyweaver reference's CPU test implementations
 * for the beamforming hot path.  It is the checker for the CUDA library: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product path (libskyweaver_b200.so) never links or calls this file.
 *
 * Floating-point semantics: the reference's CPU references are host C++
 * compiled for x86-64 without FMA, so every float multiply/add is rounded
 * separately.  This file is compiled with -ffp-contract=off -fno-fast-math to
 * keep exactly that behaviour (see oracle/Makefile).
 *
 * Reference files restated (paths relative to the skyweaver project root):
 *   transpose     cpp/skyweaver/test/src/TransposerTester.cu:30-72
 *   statistics    cpp/skyweaver/test/src/StatisticsCalculatorTester.cu:25-99,120-171
 *   scalings      cpp/skyweaver/src/StatisticsCalculator.cu:132-239
 *   IB            cpp/skyweaver/test/src/IncoherentBeamformerTester.cu:41-103
 *   CB            cpp/skyweaver/test/src/CoherentBeamformerTester.cu:43-152
 *   Stokes/quant  cpp/skyweaver/beamformer_utils.cuh:100-196
 *   weights       cpp/skyweaver/test/src/WeightsManagerTester.cu:33-71
 *   chirp         cpp/skyweaver/src/CoherentDedisperser.cu:293-336,340-359
 *   coherent DD   cpp/skyweaver/src/CoherentDedisperser.cu:142-225 and
 *                 python/skyweaver_test_utils/dedisperse.py:58-80,143-173
 *   DM delays     cpp/skyweaver/dedispersion_utils.cuh:7-48
 *   IDD           cpp/skyweaver/src/IncoherentDedisperser.cu:36-125
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SWO_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Stokes helpers: beamformer_utils.cuh:100-140                         */
/* ------------------------------------------------------------------ */
typedef struct {
    float x, y;
} cf32;

static inline float cmagf(cf32 v) { return v.x * v.x + v.y * v.y; }

/* stokes: 0=I, 1=Q, 2=U, 3=V  (beamformer_utils.cuh:108,125-140) */
static inline float calc_stokes(int stokes, cf32 p0, cf32 p1)
{
    switch(stokes) {
    case 0: return cmagf(p0) + cmagf(p1);
    case 1: return cmagf(p0) - cmagf(p1);
    case 2: {
        /* 2 * Re(cuCmulf(p0, conj(p1))) */
        float re = p0.x * p1.x - p0.y * (-p1.y);
        return 2.0f * re;
    }
    default: {
        float im = p0.x * (-p1.y) + p0.y * p1.x;
        return 2.0f * im;
    }
    }
}

/* SingleStokesBeamformerTraits::clamp (beamformer_utils.cuh:186-195) */
static inline int8_t clamp_i8(float v)
{
    return (int8_t)fmaxf(-128.0f, fminf(127.0f, v));
}

/* ------------------------------------------------------------------ */
/* Transposer: TransposerTester.cu:30-72                                */
/* TAFTP (heap time, antenna, channel, 256 samples, pol) char2 ->       */
/* FTPA (channel, sample, pol, antenna) char2, antennas zero padded.    */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_transpose(const int8_t* taftp, int8_t* ftpa, int in_nant,
                              int out_nant, int nchans, int ntimestamps,
                              int nsamples_per_heap, int npol)
{
    size_t tp   = (size_t)nsamples_per_heap * npol;
    size_t ftp  = (size_t)nchans * tp;
    size_t aftp = (size_t)in_nant * ftp;
    size_t pa   = (size_t)npol * out_nant;
    size_t tpa  = (size_t)nsamples_per_heap * ntimestamps * pa;
    memset(ftpa, 0, (size_t)nchans * tpa * 2);
    for(int ts = 0; ts < ntimestamps; ++ts)
        for(int a = 0; a < in_nant; ++a)
            for(int c = 0; c < nchans; ++c)
                for(int s = 0; s < nsamples_per_heap; ++s)
                    for(int p = 0; p < npol; ++p) {
                        size_t in = ts * aftp + a * ftp + c * tp + s * npol + p;
                        size_t os = (size_t)ts * nsamples_per_heap + s;
                        size_t out = c * tpa + os * pa + (size_t)p * out_nant + a;
                        ftpa[2 * out]     = taftp[2 * in];
                        ftpa[2 * out + 1] = taftp[2 * in + 1];
                    }
}

/* ------------------------------------------------------------------ */
/* Statistics: RunningStats, StatisticsCalculatorTester.cu:25-99,       */
/* iterated in the tester's order f, t, p, a; push(re) then push(im).   */
/* Output per (f,p,a): {mean, std, skew, kurtosis} as float.            */
/* ------------------------------------------------------------------ */
typedef struct {
    long long n;
    double M1, M2, M3, M4;
} running_stats;

static void rs_push(running_stats* s, double x)
{
    double delta, delta_n, delta_n2, term1;
    long long n1 = s->n;
    s->n++;
    long long n = s->n;
    delta    = x - s->M1;
    delta_n  = delta / n;
    delta_n2 = delta_n * delta_n;
    term1    = delta * delta_n * n1;
    s->M1 += delta_n;
    s->M4 += term1 * delta_n2 * (n * n - 3 * n + 3) + 6 * delta_n2 * s->M2 -
             4 * delta_n * s->M3;
    s->M3 += term1 * delta_n * (n - 2) - 3 * delta_n * s->M2;
    s->M2 += term1;
}

SWO_EXPORT void swo_statistics(const int8_t* ftpa, float* stats, int nchans,
                               int nsamples, int npol, int nant)
{
    size_t fpa = (size_t)nchans * npol * nant;
    running_stats* rs = (running_stats*)calloc(fpa, sizeof(running_stats));
    size_t idx = 0;
    for(int f = 0; f < nchans; ++f)
        for(int t = 0; t < nsamples; ++t)
            for(int p = 0; p < npol; ++p)
                for(int a = 0; a < nant; ++a) {
                    size_t o = (size_t)f * nant * npol + (size_t)p * nant + a;
                    rs_push(&rs[o], (double)ftpa[2 * idx]);
                    rs_push(&rs[o], (double)ftpa[2 * idx + 1]);
                    ++idx;
                }
    for(size_t i = 0; i < fpa; ++i) {
        double n = (double)rs[i].n;
        stats[4 * i + 0] = (float)rs[i].M1;
        stats[4 * i + 1] = (float)sqrt(rs[i].M2 / (n - 1.0));
        stats[4 * i + 2] = (float)(sqrt(n) * rs[i].M3 / pow(rs[i].M2, 1.5));
        stats[4 * i + 3] = (float)(n * rs[i].M4 / (rs[i].M2 * rs[i].M2) - 3.0);
    }
    free(rs);
}

/* ------------------------------------------------------------------ */
/* Scalings: StatisticsCalculator.cu:132-239.  The reference writes     */
/* index [f_idx] for every beamset (a bug); this restatement uses the   */
/* intended [beamset*nchans + f] index.  Float op order is preserved.   */
/* std::pow(float,int) promotes to double and is rounded back to float. */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_scalings(const float* stats, const float* beamset_weights,
                             int nbeamsets, int nchans, int npol, int nant,
                             int cb_tscrunch, int ib_tscrunch,
                             float output_level, float* cb_offsets,
                             float* cb_scaling, float* ib_offsets,
                             float* ib_scaling)
{
    const float weights_amp = 127.0f;
    size_t pa = (size_t)npol * nant;
    for(int s = 0; s < nbeamsets; ++s) {
        for(int f = 0; f < nchans; ++f) {
            float sum = 0.0f, count = 0.0f;
            for(int p = 0; p < npol; ++p)
                for(int a = 0; a < nant; ++a) {
                    float w = beamset_weights[(size_t)nant * s + a];
                    sum += w * stats[4 * (f * pa + (size_t)p * nant + a) + 1];
                    count += w;
                }
            float avg_std = sum / count;
            float eff     = count / (float)npol;
            size_t o      = (size_t)s * nchans + f;
            {
                double b = (double)(weights_amp * avg_std * sqrtf(eff));
                float scale = (float)(b * b);
                float dof   = (float)(2 * cb_tscrunch * npol);
                cb_offsets[o] = scale * dof;
                cb_scaling[o] = scale * sqrtf(2 * dof) / output_level;
            }
            {
                double b = (double)avg_std;
                float scale = (float)(b * b);
                float dof   = (float)(2 * ib_tscrunch) * eff * (float)npol;
                ib_offsets[o] = scale * dof;
                ib_scaling[o] = scale * sqrtf(2 * dof) / output_level;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Incoherent beamformer: IncoherentBeamformerTester.cu:41-103          */
/* raw/out layout BTF: [beamset][T/tscrunch][F]                         */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_ib(const int8_t* ftpa, float* raw, int8_t* out,
                       int nchans, int tscrunch, int nsamples, int nant,
                       const float* scale, const float* offset,
                       const float* beamset_weights, int nbeamsets, int stokes)
{
    const int nsout = nsamples / tscrunch;
    const size_t pa = 2 * (size_t)nant, tpa = (size_t)nsamples * pa;
    for(int s = 0; s < nbeamsets; ++s)
        for(int F = 0; F < nchans; ++F)
            for(int T = 0; T < nsamples; T += tscrunch) {
                float power = 0.0f;
                for(int t = T; t < T + tscrunch; ++t)
                    for(int a = 0; a < nant; ++a) {
                        float w  = beamset_weights[(size_t)s * nant + a];
                        size_t i0 = F * tpa + t * pa + a, i1 = i0 + nant;
                        cf32 p0 = {(float)ftpa[2 * i0], (float)ftpa[2 * i0 + 1]};
                        cf32 p1 = {(float)ftpa[2 * i1], (float)ftpa[2 * i1 + 1]};
                        power += calc_stokes(stokes, p0, p1) * w;
                    }
                size_t o  = (size_t)s * nsout * nchans + (size_t)(T / tscrunch) * nchans + F;
                size_t so = (size_t)s * nchans + F;
                raw[o]    = power;
                float scaled = (stokes == 0) ? rintf((power - offset[so]) / scale[so])
                                             : rintf(power / scale[so]);
                out[o] = clamp_i8(scaled);
            }
}

/* ------------------------------------------------------------------ */
/* Coherent beamformer: CoherentBeamformerTester.cu:43-152              */
/* weights [F][B][A] char2; output TFB [T/tscrunch][F][B] int8.         */
/* The IB power is recomputed here exactly as the tester does.          */
/* Optional raw_voltages: int32 [F][T][P][B][2] beam voltages (the      */
/* exact complex sums) for bit-exact checks of the tensor-core GEMM.    */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_cb(const int8_t* ftpa, const int8_t* weights, int8_t* out,
                       int nchans, int tscrunch, int nsamples, int nbeams,
                       int nant, const float* scales, const float* offsets,
                       const float* beamset_weights, const int* mapping,
                       int stokes, int ib_subtract, int32_t* raw_voltages)
{
    const int npol = 2;
    for(int c = 0; c < nchans; ++c)
        for(int s0 = 0; s0 < nsamples; s0 += tscrunch)
            for(int b = 0; b < nbeams; ++b) {
                const int bs   = mapping[b];
                float power    = 0.0f;
                float ib_power = 0.0f;
                for(int so = 0; so < tscrunch; ++so) {
                    cf32 acc0 = {0.0f, 0.0f}, acc1 = {0.0f, 0.0f};
                    for(int a = 0; a < nant; ++a) {
                        size_t base = (size_t)nant * npol * nsamples * c +
                                      (size_t)nant * npol * (s0 + so) + a;
                        size_t i0 = base, i1 = base + nant;
                        cf32 v0 = {(float)ftpa[2 * i0], (float)ftpa[2 * i0 + 1]};
                        cf32 v1 = {(float)ftpa[2 * i1], (float)ftpa[2 * i1 + 1]};
                        ib_power += calc_stokes(stokes, v0, v1) *
                                    beamset_weights[(size_t)bs * nant + a];
                        size_t wi = (size_t)nant * nbeams * c + (size_t)nant * b + a;
                        cf32 w = {(float)weights[2 * wi], (float)weights[2 * wi + 1]};
                        /* cuCmulf(weight, v) then cuCaddf */
                        cf32 q0 = {w.x * v0.x - w.y * v0.y, w.x * v0.y + w.y * v0.x};
                        cf32 q1 = {w.x * v1.x - w.y * v1.y, w.x * v1.y + w.y * v1.x};
                        acc0.x += q0.x; acc0.y += q0.y;
                        acc1.x += q1.x; acc1.y += q1.y;
                    }
                    if(raw_voltages) {
                        size_t r = (((size_t)c * nsamples + (s0 + so)) * npol) * nbeams;
                        raw_voltages[2 * (r + b)]              = (int32_t)acc0.x;
                        raw_voltages[2 * (r + b) + 1]          = (int32_t)acc0.y;
                        raw_voltages[2 * (r + nbeams + b)]     = (int32_t)acc1.x;
                        raw_voltages[2 * (r + nbeams + b) + 1] = (int32_t)acc1.y;
                    }
                    power += calc_stokes(stokes, acc0, acc1);
                }
                size_t o  = (size_t)(s0 / tscrunch) * nbeams * nchans + (size_t)c * nbeams + b;
                size_t so = (size_t)bs * nchans + c;
                float v;
                if(ib_subtract)
                    v = rintf((power - ib_power * 16129.0f) / scales[so]);
                else if(stokes == 0)
                    v = rintf((power - offsets[so]) / scales[so]);
                else
                    v = rintf(power / scales[so]);
                out[o] = clamp_i8(v);
            }
}

/* ------------------------------------------------------------------ */
/* Weights: WeightsManagerTester.cu:33-71.  delays float3 [B][A]        */
/* (weight, offset, rate); output [T][F][B][A] char2.                   */
/* ------------------------------------------------------------------ */
#define SWO_TWOPI 6.283185307179586
SWO_EXPORT void swo_weights(const float* delays, int8_t* weights,
                            const double* freqs, int nant, int nbeams,
                            int nchans, double current_epoch,
                            double delay_epoch, double tstep, int ntsteps)
{
    for(int a = 0; a < nant; ++a)
        for(int b = 0; b < nbeams; ++b) {
            const float* dm = &delays[3 * ((size_t)b * nant + a)];
            for(int c = 0; c < nchans; ++c) {
                double frequency = freqs[c];
                for(int ti = 0; ti < ntsteps; ++ti) {
                    double t = (current_epoch - delay_epoch) + ti * tstep;
                    double phase = (t * dm[2] + dm[1]) * frequency;
                    double sn, cs;
                    sincos(SWO_TWOPI * phase, &sn, &cs);
                    size_t o = (size_t)nant * ((size_t)nbeams * ((size_t)ti * nchans + c) + b) + a;
                    weights[2 * o]     = (int8_t)round(cs * 127.0 * dm[0]);
                    weights[2 * o + 1] = (int8_t)round(-1.0 * sn * 127.0 * dm[0]);
                }
            }
        }
}

/* ------------------------------------------------------------------ */
/* DM delays: dedispersion_utils.cuh:7-48                               */
/* ------------------------------------------------------------------ */
#define SWO_DM_CONST_HZ_S 4.148806423e15
SWO_EXPORT double swo_dm_delay(double f_ref, double f, double dm)
{
    return SWO_DM_CONST_HZ_S * (1 / (f_ref * f_ref) - 1 / (f * f)) * dm;
}

SWO_EXPORT int swo_dm_sample_delay(double dm, double f_ref, double tsamp,
                                   double f)
{
    return (int)(swo_dm_delay(f_ref, f, dm) / tsamp + 0.5);
}

/* ------------------------------------------------------------------ */
/* Chirp table: DMResponse, CoherentDedisperser.cu:293-336.             */
/* out [nchans][fft_len] complex double (the FP64 response; the GPU    */
/* path stores it as complex float like the reference).                 */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_chirp(double* out, int nchans, int fft_len,
                          double low_freq, double bw, float dm)
{
    double coarse_bw = bw / nchans;
    double fine_bw   = coarse_bw / fft_len;
    double pref      = -1.0 * (2.0 * 3.1415926535897932385) * SWO_DM_CONST_HZ_S * (double)dm;
    for(int c = 0; c < nchans; ++c) {
        double nu0 = low_freq + c * coarse_bw - 0.5 * coarse_bw;
        for(int k = 0; k < fft_len; ++k) {
            double nu    = k * fine_bw;
            double phase = (nu * nu * pref) / ((nu0 + nu) * nu0 * nu0);
            double s, co;
            sincos(phase, &s, &co);
            out[2 * ((size_t)c * fft_len + k)]     = co;
            out[2 * ((size_t)c * fft_len + k) + 1] = s;
        }
    }
}

/* ------------------------------------------------------------------ */
/* FP64 FFT (iterative radix-2, natural order in and out).              */
/* sign = -1 forward, +1 inverse (unnormalised, like cuFFT).            */
/* ------------------------------------------------------------------ */
static void fft64(double* x, int n, int sign)
{
    for(int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for(; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if(i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j]; x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr; x[2 * j + 1] = ti;
        }
    }
    for(int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        for(int k = 0; k < half; ++k) {
            double ang = sign * 2.0 * 3.1415926535897932385 * k / len;
            double wr = cos(ang), wi = sin(ang);
            for(int i = k; i < n; i += len) {
                int j = i + half;
                double xr = x[2 * j] * wr - x[2 * j + 1] * wi;
                double xi = x[2 * j] * wi + x[2 * j + 1] * wr;
                x[2 * j]     = x[2 * i] - xr;
                x[2 * j + 1] = x[2 * i + 1] - xi;
                x[2 * i] += xr;
                x[2 * i + 1] += xi;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* One overlap-save segment of coherent dedispersion for one stream:    */
/* CoherentDedisperser.cu:142-225 (int8 -> complex, FFT, chirp multiply,*/
/* inverse FFT, trim the overlap, /N, round, int8 wrap) with the FP64   */
/* arithmetic of dedisperse.py:159-164 (complex128 FFT, complex64 cast  */
/* of the normalised result, round-half-even, int8 cast).               */
/* The reference trims overlap/2 samples at each end of the window      */
/* (:196-223); here `lag` samples are trimmed at the end and            */
/* overlap - lag at the start, so lag = overlap / 2 is the reference.   */
/*   in:   int8 char2 [fft_len] (a zero-padded window of the stream)    */
/*   chirp: complex double [fft_len]                                    */
/*   out_i8: char2 [fft_len - overlap]                                  */
/*   out_f64: optional complex double [fft_len - overlap], the FP64     */
/*            dedispersed voltages before requantisation                */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_cdd_segment(const int8_t* in, const double* chirp,
                                int fft_len, int overlap, int lag,
                                int8_t* out_i8, double* out_f64)
{
    double* x = (double*)malloc(sizeof(double) * 2 * (size_t)fft_len);
    for(int i = 0; i < fft_len; ++i) {
        x[2 * i]     = (double)in[2 * i];
        x[2 * i + 1] = (double)in[2 * i + 1];
    }
    fft64(x, fft_len, -1);
    for(int k = 0; k < fft_len; ++k) {
        double a = x[2 * k], b = x[2 * k + 1];
        double c = chirp[2 * k], d = chirp[2 * k + 1];
        x[2 * k]     = a * c - b * d;
        x[2 * k + 1] = a * d + b * c;
    }
    fft64(x, fft_len, +1);
    int head = overlap - lag;
    for(int i = 0; i < fft_len - overlap; ++i) {
        double re = x[2 * (i + head)] / fft_len, im = x[2 * (i + head) + 1] / fft_len;
        if(out_f64) {
            out_f64[2 * i]     = re;
            out_f64[2 * i + 1] = im;
        }
        float fr = (float)re, fi = (float)im;
        out_i8[2 * i]     = (int8_t)(int32_t)rint((double)fr);
        out_i8[2 * i + 1] = (int8_t)(int32_t)rint((double)fi);
    }
    free(x);
}

/* ------------------------------------------------------------------ */
/* Overlap-save over a whole gulp for one stream (the corrected         */
/* buffering of BufferedDispenser.cu:29-72 + CoherentDedisperser).      */
/*   stream: char2 [overlap + nsamples] = history (overlap samples of  */
/*           the previous gulp, zeros for the first gulp) + this gulp   */
/*   out:    char2 [nsamples]; out[m] is the dedispersed voltage at     */
/*           input position m - lag relative to this gulp start         */
/*   Segment k takes input [k*L, k*L + fft_len) of `stream`, zero       */
/*   padded past the end, and yields outputs [k*L, k*L + L) with        */
/*   L = fft_len - overlap.                                             */
/* ------------------------------------------------------------------ */
SWO_EXPORT void swo_cdd_stream(const int8_t* stream, int nsamples,
                               const double* chirp, int fft_len, int overlap,
                               int lag, int8_t* out, double* out_f64)
{
    int L = fft_len - overlap;
    int8_t* seg = (int8_t*)malloc(2 * (size_t)fft_len);
    int8_t* so  = (int8_t*)malloc(2 * (size_t)L);
    double* sf  = out_f64 ? (double*)malloc(sizeof(double) * 2 * (size_t)L) : 0;
    int total = overlap + nsamples;
    for(int k = 0; k * L < nsamples; ++k) {
        int start = k * L;
        for(int i = 0; i < fft_len; ++i) {
            int src = start + i;
            seg[2 * i]     = src < total ? stream[2 * src] : 0;
            seg[2 * i + 1] = src < total ? stream[2 * src + 1] : 0;
        }
        swo_cdd_segment(seg, chirp, fft_len, overlap, lag, so, sf);
        int n = nsamples - start < L ? nsamples - start : L;
        memcpy(out + 2 * (size_t)start, so, 2 * (size_t)n);
        if(out_f64) memcpy(out_f64 + 2 * (size_t)start, sf, sizeof(double) * 2 * (size_t)n);
    }
    free(seg); free(so); free(sf);
}

/* ------------------------------------------------------------------ */
/* Incoherent dedisperser: IncoherentDedisperser.cu:36-125              */
/* ------------------------------------------------------------------ */
SWO_EXPORT int swo_idd_delays(const double* freqs, int nchans,
                              const float* dms, int ndms, double tsamp,
                              int* delays)
{
    int maxd = 0;
    for(int d = 0; d < ndms; ++d)
        for(int c = 0; c < nchans; ++c) {
            int v = swo_dm_sample_delay((double)dms[d], freqs[0], tsamp, freqs[c]);
            delays[(size_t)d * nchans + c] = v;
            if(v > maxd) maxd = v;
        }
    return maxd;
}

/* tfb int8 [nsamples][nchans][nbeams] -> tdb int8                      */
/* [(nsamples-maxd)/tscrunch][ndms][nbeams]; returns 0 or -1 on the     */
/* reference's size errors (IncoherentDedisperser.cu:80-87).            */
SWO_EXPORT int swo_idd(const int8_t* tfb, int8_t* tdb, int nsamples,
                       int nchans, int nbeams, const int* delays, int ndms,
                       int max_delay, int tscrunch, float scale_factor)
{
    if(nsamples <= max_delay) return -1;
    if((nsamples - max_delay) % tscrunch != 0) return -1;
    size_t bf = (size_t)nbeams * nchans;
    float* powers = (float*)malloc(sizeof(float) * (size_t)nbeams);
    for(int t = max_delay; t < nsamples; t += tscrunch) {
        size_t toff = (size_t)(t - max_delay) / tscrunch * nbeams * ndms;
        for(int d = 0; d < ndms; ++d) {
            for(int b = 0; b < nbeams; ++b) powers[b] = 0.0f;
            for(int ts = 0; ts < tscrunch; ++ts)
                for(int f = 0; f < nchans; ++f) {
                    size_t idx = (size_t)((t + ts) - delays[(size_t)d * nchans + f]) * bf +
                                 (size_t)f * nbeams;
                    for(int b = 0; b < nbeams; ++b) powers[b] += (float)tfb[idx + b];
                }
            for(int b = 0; b < nbeams; ++b)
                tdb[toff + (size_t)d * nbeams + b] = clamp_i8(powers[b] / scale_factor);
        }
    }
    free(powers);
    return 0;
}
