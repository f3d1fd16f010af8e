// Host-side planning shared by the pipeline and the autotuner.
#pragma once

#include <algorithm>
#include <cmath>

namespace swb {

constexpr double kDmConst = 4.148806423e15;  // dedispersion_utils.cuh:12-13

// Overlap-save plan of the coherent dedisperser.  The reference's chirp
// (CoherentDedisperser.cu:313-335) has a one-sided impulse response: nearly
// all of it lies at causal lags up to the intra-channel DM smear of the lowest
// channel at the largest DM.  A window therefore trims that smear, rounded up
// to a multiple of 16, at its start (`head`) and `lag` samples (default 128,
// rounded up to 16; none when every DM is 0) at its end, which hold the
// response's short anti-causal part; overlap = head + lag and the output is
// delayed by lag samples.
// Multiples of 16 keep every window start 16-byte aligned.
constexpr int kCddDefaultLag = 128;

inline int cdd_head(double centre_frequency, double bandwidth, int nchans, const float* dms,
                    int ndms)
{
    const double chbw = bandwidth / nchans;
    const float f_low = (float)(centre_frequency - bandwidth / 2.0f);
    double maxdm = 0.0;
    for(int i = 0; i < ndms; ++i) maxdm = std::max(maxdm, (double)dms[i]);
    const double f1 = f_low, f2 = f_low + chbw;
    const double smear = kDmConst * (1.0 / (f1 * f1) - 1.0 / (f2 * f2)) * maxdm;
    const double tsamp = 1.0 / chbw;
    const int ov = (int)std::ceil(smear / tsamp);
    return (ov + 15) / 16 * 16;
}

// The lag for a plan whose head trim is `head`: none when every DM is 0 (the
// chirp is exactly 1, the response a unit impulse), else the request (0 for
// the default) rounded up to 16.
inline int cdd_round_lag(int lag, int head)
{
    if(head == 0) return 0;
    return ((lag > 0 ? lag : kCddDefaultLag) + 15) / 16 * 16;
}

// FFT length by a cost model (log2 N operations per sample over the useful
// fraction 1 - overlap / N), on-chip sizes (<= 8192) when one exceeds the
// overlap, else the smallest split size (16384 .. 65536) that does; 0 if none.
inline int cdd_model_fft_len(int overlap)
{
    int fft_len = 0;
    double best = 1e30;
    for(int n = 1024; n <= 8192; n *= 2) {
        if(n <= overlap) continue;
        const double cost = std::log2((double)n) / (1.0 - (double)overlap / n);
        if(cost < best - 1e-9) { best = cost; fft_len = n; }
    }
    for(int n = 16384; fft_len == 0 && n <= 65536; n *= 2)
        if(n > overlap) fft_len = n;
    return fft_len;
}

}  // namespace swb
