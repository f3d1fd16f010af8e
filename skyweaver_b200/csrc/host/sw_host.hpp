// Host-side planning shared by the pipeline and the autotuner.
#pragma once

#include <algorithm>
#include <cmath>

namespace swb {

constexpr double kDmConst = 4.148806423e15;  // dedispersion_utils.cuh:12-13

// Overlap-save overlap of the coherent dedisperser: the largest intra-channel
// DM smear (lowest channel, largest DM) in samples, rounded up to a multiple
// of 16 so that every segment start stays 16-byte aligned.
inline int cdd_overlap(double centre_frequency, double bandwidth, int nchans, const float* dms,
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

// FFT length by a cost model (log2 N operations per sample over the useful
// fraction 1 - overlap / N), on-chip sizes only; 0 if none fits.
inline int cdd_model_fft_len(int overlap)
{
    int fft_len = 0;
    double best = 1e30;
    for(int n = 1024; n <= 8192; n *= 2) {
        if(n <= overlap) continue;
        const double cost = std::log2((double)n) / (1.0 - (double)overlap / n);
        if(cost < best - 1e-9) { best = cost; fft_len = n; }
    }
    return fft_len;
}

}  // namespace swb
