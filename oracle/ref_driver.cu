// C entry points over the reference's own stage classes, built from the
// reference sources in place (oracle/Makefile, target `ref`) into
// oracle/_ref/libswref.so.  Test infrastructure: the GPU parity tests use it
// to check the oracle restatement (and the B200 kernels) against the
// reference implementation itself.  Shapes are the reference's compile-time
// constants (SKYWEAVER_NANTENNAS, _NCHANS, _NBEAMS, _CB_TSCRUNCH,
// _IB_TSCRUNCH), reported by swref_shape.
//
// Wrapped: Transposer::transpose (src/Transposer.cu:117-184),
// StatisticsCalculator::calculate_statistics (src/StatisticsCalculator.cu:
// 104-130), IncoherentBeamformer / CoherentBeamformer<Stokes I>::beamform
// (src/IncoherentBeamformer.cu:108-182, src/CoherentBeamformer.cu:191-270),
// WeightsManager::weights (src/WeightsManager.cu:109-139),
// IncoherentDedisperser::dedisperse (src/IncoherentDedisperser.cu:66-125) and
// CoherentDedisperser::dedisperse (src/CoherentDedisperser.cu:142-225, one
// window, and timed over a gulp).
#include <cstring>
#include <stdexcept>
#include <vector>

#include "skyweaver/CoherentBeamformer.cuh"
#include "skyweaver/CoherentDedisperser.cuh"
#include "skyweaver/DescribedVector.hpp"
#include "skyweaver/IncoherentBeamformer.cuh"
#include "skyweaver/IncoherentDedisperser.cuh"
#include "skyweaver/PipelineConfig.hpp"
#include "skyweaver/StatisticsCalculator.cuh"
#include "skyweaver/Transposer.cuh"
#include "skyweaver/WeightsManager.cuh"

using namespace skyweaver;
using Traits = SingleStokesBeamformerTraits<StokesParameter::I>;

namespace {
thread_local std::string g_err;

template <typename F>
int guarded(F&& f)
{
    try {
        f();
        return 0;
    } catch(const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

PipelineConfig& config(double centre, double bw)
{
    static PipelineConfig c;
    c.centre_frequency(centre);
    c.bandwidth(bw);
    return c;
}
}  // namespace

extern "C" {

const char* swref_error() { return g_err.c_str(); }

void swref_shape(int* nant, int* nchans, int* nbeams, int* cb_ts, int* ib_ts)
{
    *nant = SKYWEAVER_NANTENNAS;
    *nchans = SKYWEAVER_NCHANS;
    *nbeams = SKYWEAVER_NBEAMS;
    *cb_ts = SKYWEAVER_CB_TSCRUNCH;
    *ib_ts = SKYWEAVER_IB_TSCRUNCH;
}

// TAFTP [heaps][input_nant][F][256][2] char2 -> FTPA [F][T][2][NANT] char2
int swref_transpose(const int8_t* taftp, int nheaps, int input_nant, int8_t* ftpa)
{
    return guarded([&] {
        PipelineConfig& c = config(1284e6, 13.375e6);
        Transposer t(c);
        TAFTPVoltagesH<char2> h({(std::size_t)nheaps, (std::size_t)input_nant, c.nchans(),
                                 c.nsamples_per_heap(), c.npol()});
        std::memcpy(thrust::raw_pointer_cast(h.data()), taftp, h.size() * 2);
        TAFTPVoltagesD<char2> d = h;
        FTPAVoltagesD<char2> out;
        t.transpose(d, out, input_nant, 0);
        thrust::host_vector<char2> back = out.vector();
        std::memcpy(ftpa, thrust::raw_pointer_cast(back.data()), back.size() * 2);
    });
}

// FTPA -> Statistics {mean, std, skew, kurtosis} per (F, P, A)
int swref_statistics(const int8_t* ftpa, int nsamples, float* stats)
{
    return guarded([&] {
        PipelineConfig& c = config(1284e6, 13.375e6);
        StatisticsCalculator calc(c, 0);
        FTPAVoltagesH<char2> h({c.nchans(), (std::size_t)nsamples, c.npol(), c.nantennas()});
        std::memcpy(thrust::raw_pointer_cast(h.data()), ftpa, h.size() * 2);
        FTPAVoltagesD<char2> d = h;
        calc.calculate_statistics(d);
        thrust::host_vector<Statistics> s = calc.statistics().vector();
        std::memcpy(stats, thrust::raw_pointer_cast(s.data()), s.size() * sizeof(Statistics));
    });
}

// Stokes I incoherent beam (raw float and int8 BTF), then the coherent beams
// (int8 TFB) with IB subtraction, exactly like CoherentBeamformerTester.cu:
// 324-352.  weights: FBA char2 [F][NBEAMS][NANT].
int swref_beamform(const int8_t* ftpa, int nsamples, const int8_t* weights, const float* cb_scale,
                   const float* cb_offset, const float* ib_scale, const float* ib_offset,
                   const float* beamset_weights, const int* mapping, int nbeamsets,
                   float* ib_raw, int8_t* ib_out, int8_t* cb_out)
{
    return guarded([&] {
        PipelineConfig& c = config(1284e6, 13.375e6);
        const std::size_t F = c.nchans(), A = c.nantennas(), B = c.nbeams();
        FTPAVoltagesH<char2> h({F, (std::size_t)nsamples, c.npol(), A});
        std::memcpy(thrust::raw_pointer_cast(h.data()), ftpa, h.size() * 2);
        FTPAVoltagesD<char2> d = h;
        thrust::host_vector<char2> wh(F * B * A);
        std::memcpy(thrust::raw_pointer_cast(wh.data()), weights, wh.size() * 2);
        thrust::device_vector<char2> wd = wh;
        const std::size_t ns = F * nbeamsets;
        thrust::device_vector<float> cbs(cb_scale, cb_scale + ns), cbo(cb_offset, cb_offset + ns);
        thrust::device_vector<float> ibs(ib_scale, ib_scale + ns), ibo(ib_offset, ib_offset + ns);
        thrust::device_vector<float> bw(beamset_weights, beamset_weights + A * nbeamsets);
        thrust::device_vector<int> map(mapping, mapping + B);
        IncoherentBeamformer<Traits> ib(c);
        CoherentBeamformer<Traits> cb(c);
        typename IncoherentBeamformer<Traits>::RawPowerVectorTypeD raw;
        typename IncoherentBeamformer<Traits>::PowerVectorTypeD ibq;
        typename CoherentBeamformer<Traits>::PowerVectorTypeD tfb;
        ib.beamform(d, raw, ibq, ibs, ibo, bw, nbeamsets, 0);
        cb.beamform(d, wd, cbs, cbo, map, raw, tfb, nbeamsets, 0);
        thrust::host_vector<float> rh = raw.vector();
        thrust::host_vector<int8_t> ih = ibq.vector(), th = tfb.vector();
        std::memcpy(ib_raw, thrust::raw_pointer_cast(rh.data()), rh.size() * sizeof(float));
        std::memcpy(ib_out, thrust::raw_pointer_cast(ih.data()), ih.size());
        std::memcpy(cb_out, thrust::raw_pointer_cast(th.data()), th.size());
    });
}

// Device time of one IncoherentBeamformer and one CoherentBeamformer
// beamform call on nsamples of synthetic device data (mean over reps after a
// warm-up; the calls synchronise their stream, as in the reference).
int swref_time_beamform(int nsamples, int reps, float* ms_ib, float* ms_cb)
{
    return guarded([&] {
        PipelineConfig& c = config(1284e6, 13.375e6);
        const std::size_t F = c.nchans(), A = c.nantennas(), B = c.nbeams();
        FTPAVoltagesH<char2> h({F, (std::size_t)nsamples, c.npol(), A});
        for(std::size_t i = 0; i < h.size(); ++i)
            h[i] = make_char2((signed char)((i * 2654435761u >> 13) % 31 - 15),
                              (signed char)((i * 40503u >> 7) % 31 - 15));
        FTPAVoltagesD<char2> d = h;
        thrust::device_vector<char2> wd(F * B * A, make_char2(90, -90));
        thrust::device_vector<float> sc(F, 1e9f), of(F, 0.0f), bw(A, 1.0f);
        thrust::device_vector<int> map(B, 0);
        IncoherentBeamformer<Traits> ib(c);
        CoherentBeamformer<Traits> cb(c);
        typename IncoherentBeamformer<Traits>::RawPowerVectorTypeD raw;
        typename IncoherentBeamformer<Traits>::PowerVectorTypeD ibq;
        typename CoherentBeamformer<Traits>::PowerVectorTypeD tfb;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        ib.beamform(d, raw, ibq, sc, of, bw, 1, 0);
        cudaEventRecord(e0, 0);
        for(int r = 0; r < reps; ++r) ib.beamform(d, raw, ibq, sc, of, bw, 1, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms_ib, e0, e1);
        *ms_ib /= reps;
        cb.beamform(d, wd, sc, of, map, raw, tfb, 1, 0);
        cudaEventRecord(e0, 0);
        for(int r = 0; r < reps; ++r) cb.beamform(d, wd, sc, of, map, raw, tfb, 1, 0);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms_cb, e0, e1);
        *ms_cb /= reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

// Device time of the reference's coherent dedispersion of one gulp: one
// CoherentDedisperser::dedisperse call (int8 -> complex, batched cuFFT
// forward, chirp, cuFFT inverse, trim, requantise) per (channel, DM), as its
// pipeline issues them (detail/BeamformerPipeline.cu:192-205).
int swref_time_cdd(int fft_length, int overlap, const float* dms, int ndms, double centre,
                   double bw, int reps, float* ms)
{
    return guarded([&] {
        PipelineConfig& c = config(centre, bw);
        CoherentDedisperserConfig cfg;
        create_coherent_dedisperser_config(cfg, fft_length, overlap, c.nchans(), c.npol(),
                                           c.nantennas(), c.nchans() / bw, centre - bw / 2, bw,
                                           std::vector<float>(dms, dms + ndms));
        CoherentDedisperser cd(cfg);
        TPAVoltagesH<char2> h({(std::size_t)fft_length, c.npol(), c.nantennas()});
        for(std::size_t i = 0; i < h.size(); ++i)
            h[i] = make_char2((signed char)((i * 2654435761u >> 13) % 31 - 15),
                              (signed char)((i * 40503u >> 7) % 31 - 15));
        TPAVoltagesD<char2> in = h;
        FTPAVoltagesD<char2> out({c.nchans(), (std::size_t)(fft_length - overlap), c.npol(),
                                  c.nantennas()});
        cd.dedisperse(in, out, 0, 0);
        cudaDeviceSynchronize();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
        for(int r = 0; r < reps; ++r)
            for(unsigned f = 0; f < c.nchans(); ++f)
                for(int d = 0; d < ndms; ++d) cd.dedisperse(in, out, f, d);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

// One overlap-save window of one channel through the reference's
// CoherentDedisperser::dedisperse (src/CoherentDedisperser.cu:142-225, cuFFT
// in FP32): TPA char2 [fft_length][2][NANT] of channel `chan` in, the trimmed
// [fft_length - overlap][2][NANT] char2 of that channel and DM out.  The
// band is [low, low + bw) over the build's SKYWEAVER_NCHANS channels.
int swref_cdd(int fft_length, int overlap, const float* dms, int ndms, double low, double bw,
              int chan, int dm_idx, const int8_t* tpa, int8_t* out_tpa)
{
    return guarded([&] {
        PipelineConfig& c = config(low + bw / 2, bw);
        CoherentDedisperserConfig cfg;
        create_coherent_dedisperser_config(cfg, fft_length, overlap, c.nchans(), c.npol(),
                                           c.nantennas(), c.nchans() / bw, low, bw,
                                           std::vector<float>(dms, dms + ndms));
        CoherentDedisperser cd(cfg);
        TPAVoltagesH<char2> h({(std::size_t)fft_length, c.npol(), c.nantennas()});
        std::memcpy(thrust::raw_pointer_cast(h.data()), tpa, h.size() * 2);
        TPAVoltagesD<char2> in = h;
        FTPAVoltagesD<char2> out({c.nchans(), (std::size_t)(fft_length - overlap), c.npol(),
                                  c.nantennas()});
        cd.dedisperse(in, out, chan, dm_idx);
        thrust::host_vector<char2> back = out.vector();
        const std::size_t per = (std::size_t)(fft_length - overlap) * c.npol() * c.nantennas();
        std::memcpy(out_tpa, thrust::raw_pointer_cast(back.data()) + chan * per, per * 2);
    });
}

// delays float3 [NBEAMS][NANT] -> weights FBA char2 [F][NBEAMS][NANT]
int swref_weights(const float* delays, double current_epoch, double delay_epoch, double centre,
                  double bw, int8_t* weights)
{
    return guarded([&] {
        PipelineConfig& c = config(centre, bw);
        WeightsManager wm(c, 0);
        const std::size_t n = c.nbeams() * c.nantennas();
        thrust::host_vector<float3> dh(n);
        std::memcpy(thrust::raw_pointer_cast(dh.data()), delays, n * sizeof(float3));
        thrust::device_vector<float3> dd = dh;
        thrust::host_vector<char2> w = wm.weights(dd, current_epoch, delay_epoch);
        std::memcpy(weights, thrust::raw_pointer_cast(w.data()), w.size() * 2);
    });
}

// int8 TFB [T][NCHANS][NBEAMS] -> TDB; also returns the delays and max delay
int swref_idd(const int8_t* tfb, int nsamples, const float* dms, int ndms, int tscrunch,
              double centre, double bw, int8_t* tdb, int* delays, int* max_delay)
{
    return guarded([&] {
        PipelineConfig& c = config(centre, bw);
        IncoherentDedisperser idd(c, std::vector<float>(dms, dms + ndms), (std::size_t)tscrunch);
        const std::size_t n = (std::size_t)nsamples * c.nchans() * c.nbeams();
        thrust::host_vector<int8_t, PinnedAllocator<int8_t>> in(n);
        std::memcpy(thrust::raw_pointer_cast(in.data()), tfb, n);
        TDBPowersH<int8_t> out;
        idd.dedisperse(in, out);
        std::memcpy(tdb, thrust::raw_pointer_cast(out.data()), out.size());
        const auto& dl = idd.delays();
        std::memcpy(delays, dl.data(), dl.size() * sizeof(int));
        *max_delay = idd.max_sample_delay();
    });
}

}  // extern "C"
