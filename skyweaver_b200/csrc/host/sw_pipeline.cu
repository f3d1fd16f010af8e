// BeamformerPipeline on the B200 (C ABI object behind sw_pipeline_*).
//
// Reference: cpp/skyweaver/detail/BeamformerPipeline.cu:44-301.  The
// reference runs ~10 synchronising stage calls per DM per gulp and 64
// serial per-channel dedispersion launches; here one gulp is
//
//   [epoch H2D] -> weights -> history copy -> TAFTP->FPACT transpose
//   -> statistics -> (gulp 0: scalings) -> coherent dedispersion of all
//   channels for every non-zero DM -> incoherent beam per DM -> one
//   persistent grouped tensor-core launch for all (DM x beamset)
//
// A DM of exactly 0 has a chirp of exactly 1: its dedispersed voltages are
// the input delayed by the plan's lag, which the beamformers read straight
// from the transposed rows (at offset overlap - lag), so it costs no
// transform and no copy.
//
// all on one stream, captured once as a CUDA graph per input/output buffer
// pair.  process_host double-buffers the pinned-host input and the outputs
// so that the H2D of gulp g+1 and the D2H of gulp g-1 overlap the compute
// of gulp g on separate copy streams.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "../sw_common.cuh"
#include "sw_host.hpp"

namespace swb {
int launch_weights(const float* d_delays, const double* d_freqs, int nant, int nbeams,
                   int nchans, double current_epoch, double delay_epoch,
                   const double* d_epochs, void* d_fba, void* d_gemm, cudaStream_t stream);
int launch_incoherent_beamform(const void* d_fpact, size_t row_stride, size_t sample_offset,
                               int nchans, int nsamples, int nant, int tscrunch,
                               const float* d_scale, const float* d_offset,
                               const float* d_beamset_weights, int nbeamsets, int stokes,
                               float* d_raw, int8_t* d_out, cudaStream_t stream,
                               const int* d_chan_order);
int launch_ib_channel_order(const float* d_stats, int nchans, int npol, int nant,
                            int* d_order, cudaStream_t stream);
}

namespace {


struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    int alloc(size_t bytes)
    {
        n = bytes;
        if(bytes == 0) return SW_OK;
        SW_CUDA_CHECK(cudaMalloc(&p, bytes));
        return SW_OK;
    }
    ~DevBuf()
    {
        if(p) cudaFree(p);
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

struct sw_pipeline {
    sw_pipeline_config cfg{};
    std::vector<float> dms;
    std::vector<float> bw;  // beamset weights [S][A]
    std::vector<int> mapping;
    std::vector<double> freqs;
    int nheaps = 0, T = 0, F = 0, A = 0, B = 0, S = 0, ndm = 0, ts = 0;
    int fft_len = 0, overlap = 0;  // overlap: multiple of 16
    int lag = 0;                   // of it, trimmed at each window's end
    int cb_tpi = 0;                // CB work-item size (0: kernel default)
    int cb_vst = 0, cb_wst = 0;    // CB pipeline depths (0: kernel defaults)
    size_t ext_stride = 0, ext_off = 0, dd_stride = 0;
    size_t v_off = 0;           // first sample of the beamformers' voltages in a row
    std::vector<int> dd_of;     // per DM: index into dd (-1: DM 0, read from ext)
    std::vector<float> cdd_dms; // the non-zero DMs, in order
    size_t nrows = 0;  // F * P * A * 2

    DevBuf taftp[2];
    DevBuf ext[2];  // transposed rows [overlap history | gulp] per output parity
    std::vector<DevBuf> dd;
    DevBuf stats[2], stats_scratch;  // statistics per output parity
    DevBuf ib_order;  // channels by descending power, for the incoherent beam
    DevBuf cb_off, cb_scl, ib_off, ib_scl;
    DevBuf d_bw, d_map, d_delays, d_freqs, d_wgemm, d_setup, cdd_ws;
    DevBuf epochs;  // [2 parities][2] doubles
    std::vector<DevBuf> ib_raw[2], ib_i8[2], cb[2];
    double* h_epochs = nullptr;  // pinned [2][2]
    double delay_epoch = 0.0;
    bool have_delays = false;

    cudaStream_t compute = nullptr, h2d = nullptr, d2h = nullptr;
    cudaEvent_t h2d_done[2]{}, comp_done[2]{}, d2h_done[2]{}, caller_ready[2]{};
    bool scalings_done = false;
    long gulp = 0;
    int last_par = 0;  // output parity of the last processed gulp
    std::map<std::pair<const void*, int>, cudaGraphExec_t> graphs;

    ~sw_pipeline()
    {
        for(auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        for(int i = 0; i < 2; ++i) {
            if(h2d_done[i]) cudaEventDestroy(h2d_done[i]);
            if(comp_done[i]) cudaEventDestroy(comp_done[i]);
            if(d2h_done[i]) cudaEventDestroy(d2h_done[i]);
            if(caller_ready[i]) cudaEventDestroy(caller_ready[i]);
        }
        if(compute) cudaStreamDestroy(compute);
        if(h2d) cudaStreamDestroy(h2d);
        if(d2h) cudaStreamDestroy(d2h);
        if(h_epochs) cudaFreeHost(h_epochs);
    }

    // IQUV (stokes 4) carries four components per sample: char4 / float4
    int ncomp() const { return cfg.stokes == 4 ? 4 : 1; }
    size_t cb_bytes() const { return (size_t)(T / ts) * F * B * ncomp(); }
    size_t ib_elems() const { return (size_t)S * (T / ts) * F * ncomp(); }

    int init(const sw_pipeline_config& c);
    int enqueue_chain(const void* d_in, int parity, bool first);
    int run(const void* d_in, int parity, double epoch);
};

int sw_pipeline::init(const sw_pipeline_config& c)
{
    cfg = c;
    A = c.nantennas, F = c.nchans, B = c.nbeams, T = c.gulp_samples, ts = c.tscrunch;
    SW_REQUIRE(A == 16 || A == 32 || A == 64, "pipeline: nantennas must be 16, 32 or 64");
    SW_REQUIRE(c.input_nantennas > 0 && c.input_nantennas <= A,
               "Input number of antennas must be <= to the maximum nantennas");
    SW_REQUIRE(T > 0 && T % 256 == 0, "Gulp size is not a multiple of the number of samples per heap");
    SW_REQUIRE(F > 0 && B > 0, "pipeline: empty shape");
    SW_REQUIRE(c.ndms > 0 && c.dms, "No DDPlan set for pipeline");
    SW_REQUIRE(c.nbeamsets > 0 && c.beamset_weights && c.beamset_mapping,
               "pipeline: beamset weights and mapping are required");
    nheaps = T / 256;
    S      = c.nbeamsets;
    ndm    = c.ndms;
    dms.assign(c.dms, c.dms + ndm);
    bw.assign(c.beamset_weights, c.beamset_weights + (size_t)S * A);
    mapping.assign(c.beamset_mapping, c.beamset_mapping + B);
    for(int m : mapping) SW_REQUIRE(m >= 0 && m < S, "pipeline: beamset mapping out of range");
    // PipelineConfig::calculate_channel_frequencies (PipelineConfig.cpp:188-203)
    const double chbw = c.bandwidth / F;
    const double fbottom = c.centre_frequency - c.bandwidth / 2.0;
    for(int i = 0; i < F; ++i) freqs.push_back(fbottom + chbw / 2.0 + chbw * i);

    // Coherent dedispersion plan: each window trims the largest intra-channel
    // DM smear (lowest channel, largest DM) at its start and `lag` samples at
    // its end; overlap = both, multiples of 16.
    if(c.enable_coherent_dedispersion) {
        const int head = swb::cdd_head(c.centre_frequency, c.bandwidth, F, dms.data(), ndm);
        lag     = swb::cdd_round_lag(c.cdd_lag, head);
        overlap = head + lag;
        if(c.fft_len > 0) {
            fft_len = c.fft_len;
        } else if(c.autotune) {
            sw_tuning tu{};
            SW_TRY(sw_autotune(A, B, F, T, ts, ndm, dms.data(), c.centre_frequency, c.bandwidth,
                               &tu, nullptr));
            fft_len = tu.fft_len;
            cb_tpi = tu.cb_tiles_per_item;
            cb_vst = tu.cb_voltage_stages;
            cb_wst = tu.cb_weight_stages;
        } else {
            fft_len = swb::cdd_model_fft_len(overlap);
        }
        SW_REQUIRE(fft_len > overlap && fft_len >= 256 && fft_len <= 65536,
                   "pipeline: fft_len %d does not exceed the DM smear of %d samples or is "
                   "outside [256, 65536]", fft_len, overlap);
        SW_REQUIRE(T >= overlap, "pipeline: gulp shorter than the dedispersion overlap");
    } else {
        overlap = 0;
        lag     = 0;
        fft_len = 0;
    }
    ext_off    = (size_t)overlap;
    ext_stride = (size_t)overlap + T;
    // dedispersed rows share the transposed rows' geometry so that every DM's
    // voltages start at the same offset: overlap - lag = the delayed gulp
    dd_stride  = ext_stride;
    v_off      = (size_t)(overlap - lag);
    dd_of.assign(ndm, -1);
    for(int d = 0; c.enable_coherent_dedispersion && d < ndm; ++d)
        if(dms[d] != 0.0f) {
            dd_of[d] = (int)cdd_dms.size();
            cdd_dms.push_back(dms[d]);
        }
    nrows      = (size_t)F * 2 * A * 2;

    SW_CUDA_CHECK(cudaStreamCreateWithFlags(&compute, cudaStreamNonBlocking));
    SW_CUDA_CHECK(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
    SW_CUDA_CHECK(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    for(int i = 0; i < 2; ++i) {
        SW_CUDA_CHECK(cudaEventCreateWithFlags(&h2d_done[i], cudaEventDisableTiming));
        SW_CUDA_CHECK(cudaEventCreateWithFlags(&comp_done[i], cudaEventDisableTiming));
        SW_CUDA_CHECK(cudaEventCreateWithFlags(&d2h_done[i], cudaEventDisableTiming));
        SW_CUDA_CHECK(cudaEventCreateWithFlags(&caller_ready[i], cudaEventDisableTiming));
    }
    SW_CUDA_CHECK(cudaMallocHost(&h_epochs, 4 * sizeof(double)));
    memset(h_epochs, 0, 4 * sizeof(double));

    const size_t taftp_bytes = (size_t)nheaps * c.input_nantennas * F * 256 * 2 * 2;
    SW_TRY(taftp[0].alloc(taftp_bytes));
    SW_TRY(taftp[1].alloc(taftp_bytes));
    for(DevBuf& b : ext) {
        SW_TRY(b.alloc(nrows * ext_stride));
        SW_CUDA_CHECK(cudaMemset(b.p, 0, b.n));  // zero history for gulp 0
    }
    const int ncdd = (int)cdd_dms.size();
    if(c.enable_coherent_dedispersion && ncdd > 0) {
        dd.resize(ncdd);
        for(int k = 0; k < ncdd; ++k) SW_TRY(dd[k].alloc(nrows * dd_stride));
        SW_TRY(d_setup.alloc(sw_cdd_setup_bytes(ncdd, F, fft_len)));
        // long FFTs (> 8192) pass their sub-transform spectra through a
        // workspace: at most 4 GiB, processed in chunks of segments
        const size_t ws = sw_cdd_workspace_bytes(F, 2, A, T, fft_len, overlap, ncdd);
        if(ws) {
            const size_t per_seg = (size_t)ncdd * fft_len * 8;
            SW_TRY(cdd_ws.alloc(std::max(per_seg, std::min(ws, (size_t)4 << 30) / per_seg * per_seg)));
        }
        const double low = (double)(float)(c.centre_frequency - c.bandwidth / 2.0f);
        SW_TRY(sw_cdd_chirps(cdd_dms.data(), ncdd, F, fft_len, low, c.bandwidth, d_setup.p,
                             (sw_stream_t)compute));
    }
    for(DevBuf& b : stats) SW_TRY(b.alloc((size_t)F * 2 * A * 4 * sizeof(float)));
    SW_TRY(stats_scratch.alloc(sw_statistics_scratch_bytes(F, 2, A)));
    if(F <= swb::kIbOrderMaxChans) SW_TRY(ib_order.alloc((size_t)F * sizeof(int)));
    for(DevBuf* b : {&cb_off, &cb_scl, &ib_off, &ib_scl}) SW_TRY(b->alloc((size_t)S * F * sizeof(float)));
    SW_TRY(d_bw.alloc(bw.size() * sizeof(float)));
    SW_TRY(d_map.alloc(mapping.size() * sizeof(int)));
    SW_TRY(d_delays.alloc((size_t)B * A * 3 * sizeof(float)));
    SW_TRY(d_freqs.alloc(freqs.size() * sizeof(double)));
    SW_TRY(d_wgemm.alloc((size_t)F * 2 * B * 2 * A));
    SW_TRY(epochs.alloc(4 * sizeof(double)));
    SW_CUDA_CHECK(cudaMemcpy(d_bw.p, bw.data(), d_bw.n, cudaMemcpyHostToDevice));
    SW_CUDA_CHECK(cudaMemcpy(d_map.p, mapping.data(), d_map.n, cudaMemcpyHostToDevice));
    SW_CUDA_CHECK(cudaMemcpy(d_freqs.p, freqs.data(), d_freqs.n, cudaMemcpyHostToDevice));
    SW_CUDA_CHECK(cudaMemset(d_delays.p, 0, d_delays.n));
    for(int par = 0; par < 2; ++par) {
        ib_raw[par].resize(ndm);
        ib_i8[par].resize(ndm);
        cb[par].resize(ndm);
        for(int d = 0; d < ndm; ++d) {
            SW_TRY(ib_raw[par][d].alloc(ib_elems() * sizeof(float)));
            SW_TRY(ib_i8[par][d].alloc(ib_elems()));
            SW_TRY(cb[par][d].alloc(cb_bytes()));
        }
    }
    SW_CUDA_CHECK(cudaStreamSynchronize(compute));
    return SW_OK;
}

// One gulp's device chain on `compute` (captured into a graph when enabled).
int sw_pipeline::enqueue_chain(const void* d_in, int parity, bool first)
{
    cudaStream_t s = compute;
    sw_stream_t ss = (sw_stream_t)s;
    double* d_ep = epochs.as<double>() + 2 * parity;
    SW_CUDA_CHECK(cudaMemcpyAsync(d_ep, h_epochs + 2 * parity, 2 * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    SW_TRY(swb::launch_weights(d_delays.as<float>(), d_freqs.as<double>(), A, B, F, 0.0, 0.0,
                               d_ep, nullptr, d_wgemm.p, s));
    // overlap-save history: the previous gulp's last `overlap` samples
    void* rows = ext[parity].p;
    if(overlap > 0)
        SW_TRY(sw_fpact_copy_history(ext[parity ^ 1].p, rows, nrows, ext_stride,
                                     (size_t)overlap, ss));
    // transpose and statistics in one pass over the gulp
    SW_TRY(sw_transpose_fpact_statistics(d_in, rows, nheaps, cfg.input_nantennas, A, F,
                                         ext_stride, ext_off, stats_scratch.p,
                                         stats[parity].as<float>(), ss));
    const int* chan_order = nullptr;
    if(ib_order.p) {
        SW_TRY(swb::launch_ib_channel_order(stats[parity].as<float>(), F, 2, A,
                                            ib_order.as<int>(), s));
        chan_order = ib_order.as<int>();
    }
    if(first) {
        SW_TRY(sw_update_scalings(stats[parity].as<float>(), d_bw.as<float>(), S, F, 2, A, ts, ts,
                                  cfg.output_level, cb_off.as<float>(), cb_scl.as<float>(),
                                  ib_off.as<float>(), ib_scl.as<float>(), ss));
    }
    // every DM's voltages: rows of ext_stride samples from offset v_off
    std::vector<const void*> volt(ndm);
    const size_t vstride = ext_stride, voff = v_off;
    if(!cdd_dms.empty()) {
        std::vector<void*> outs(cdd_dms.size());
        for(size_t k = 0; k < outs.size(); ++k) outs[k] = dd[k].as<uint8_t>() + v_off;
        SW_TRY(sw_coherent_dedisperse_ws(rows, ext_stride, F, 2, A, T, fft_len, overlap, lag,
                                         d_setup.p, (int)outs.size(), outs.data(), dd_stride,
                                         cdd_ws.p, cdd_ws.n, nullptr, ss));
    }
    for(int d = 0; d < ndm; ++d) volt[d] = dd_of[d] < 0 ? rows : dd[dd_of[d]].p;
    for(int d = 0; d < ndm; ++d) {
        SW_TRY(swb::launch_incoherent_beamform(volt[d], vstride, voff, F, T, A, ts,
                                               ib_scl.as<float>(), ib_off.as<float>(),
                                               d_bw.as<float>(), S, cfg.stokes,
                                               ib_raw[parity][d].as<float>(),
                                               ib_i8[parity][d].as<int8_t>(), s, chan_order));
    }
    sw_cb_shape shape{F,     T,    A,    B,      ts,     cfg.stokes, cfg.ib_subtract,
                      vstride, voff, cb_tpi, cb_vst, cb_wst};
    if(cfg.grouped) {
        // one problem per DM over all beams: the epilogue resolves each beam's
        // beamset (scale, offset, IB power) itself, so 128-beam tiles pack
        // across beamset boundaries and every (DM, beamset) shares one queue
        std::vector<sw_cb_problem> probs;
        for(int d = 0; d < ndm; ++d)
            probs.push_back({volt[d], cb[parity][d].as<int8_t>(), ib_raw[parity][d].as<float>(), 0, B});
        SW_TRY(sw_coherent_beamform_grouped(&shape, probs.data(), (int)probs.size(), d_wgemm.p,
                                            cb_scl.as<float>(), cb_off.as<float>(),
                                            d_map.as<int>(), ss));
    } else {
        // plain form: one launch per (DM, contiguous run of beams of one
        // beamset); a mapping with more than 96 runs falls back to one launch
        // per DM
        std::vector<sw_cb_problem> probs;
        for(int d = 0; d < ndm; ++d) {
            int b = 0;
            while(b < B) {
                int e = b + 1;
                while(e < B && mapping[e] == mapping[b]) ++e;
                probs.push_back({volt[d], cb[parity][d].as<int8_t>(),
                                 ib_raw[parity][d].as<float>(), b, e - b});
                b = e;
            }
        }
        if(probs.size() > 96) {
            probs.clear();
            for(int d = 0; d < ndm; ++d)
                probs.push_back({volt[d], cb[parity][d].as<int8_t>(), ib_raw[parity][d].as<float>(), 0, B});
        }
        for(auto& pr : probs)
            SW_TRY(sw_coherent_beamform(&shape, &pr, d_wgemm.p, cb_scl.as<float>(),
                                        cb_off.as<float>(), d_map.as<int>(), nullptr, ss));
    }
    return SW_OK;
}

int sw_pipeline::run(const void* d_in, int parity, double epoch)
{
    SW_REQUIRE(have_delays, "pipeline: no delay model set (sw_pipeline_set_delays)");
    last_par = parity;
    // The chain's first node copies this parity's epoch slot when it runs on
    // the device.  The previous gulp of the same parity must have done so
    // before the slot is overwritten, so the host waits for that gulp (a
    // no-op unless the caller runs more than one gulp ahead of the GPU).
    SW_CUDA_CHECK(cudaEventSynchronize(comp_done[parity]));
    h_epochs[2 * parity + 0] = epoch;
    h_epochs[2 * parity + 1] = delay_epoch;
    if(!scalings_done || !cfg.use_graph) {
        SW_TRY(enqueue_chain(d_in, parity, !scalings_done));
        scalings_done = true;
        return SW_OK;
    }
    auto key = std::make_pair(d_in, parity);
    auto it = graphs.find(key);
    if(it == graphs.end()) {
        cudaGraph_t g;
        SW_CUDA_CHECK(cudaStreamBeginCapture(compute, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_chain(d_in, parity, false);
        cudaError_t e = cudaStreamEndCapture(compute, &g);
        if(rc != SW_OK) return rc;
        SW_CUDA_CHECK(e);
        cudaGraphExec_t ge;
        SW_CUDA_CHECK(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        it = graphs.emplace(key, ge).first;
    }
    SW_CUDA_CHECK(cudaGraphLaunch(it->second, compute));
    return SW_OK;
}

using namespace swb;

extern "C" {

int sw_cdd_plan(double centre_frequency, double bandwidth, int nchans, const float* h_dms,
                int ndms, int lag_request, int* fft_len, int* overlap, int* lag)
{
    SW_REQUIRE(h_dms && ndms > 0 && nchans > 0 && bandwidth > 0.0 && fft_len && overlap && lag,
               "sw_cdd_plan: bad arguments");
    const int head = cdd_head(centre_frequency, bandwidth, nchans, h_dms, ndms);
    const int lg   = cdd_round_lag(lag_request, head);
    const int ov   = head + lg;
    int n = *fft_len > 0 ? *fft_len : cdd_model_fft_len(ov);
    SW_REQUIRE(n > ov && n >= 256 && n <= 65536 && (n & (n - 1)) == 0,
               "coherent dedispersion: no power-of-two FFT length in [256, 65536] exceeds the "
               "overlap of %d samples (requested %d)", ov, *fft_len);
    *fft_len = n;
    *overlap = ov;
    *lag     = lg;
    return SW_OK;
}

int sw_pipeline_create(const sw_pipeline_config* cfg, sw_pipeline** out)
{
    SW_REQUIRE(cfg && out, "sw_pipeline_create: null argument");
    *out = nullptr;
    sw_pipeline* p = new sw_pipeline();
    int rc = p->init(*cfg);
    if(rc != SW_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return SW_OK;
}

int sw_pipeline_destroy(sw_pipeline* p)
{
    if(p) {
        cudaStreamSynchronize(p->compute);
        cudaStreamSynchronize(p->h2d);
        cudaStreamSynchronize(p->d2h);
        delete p;
    }
    return SW_OK;
}

int sw_pipeline_set_delays(sw_pipeline* p, const float* h_delays, double delay_epoch)
{
    SW_REQUIRE(p && h_delays, "sw_pipeline_set_delays: null argument");
    SW_CUDA_CHECK(cudaStreamSynchronize(p->compute));
    SW_CUDA_CHECK(cudaMemcpy(p->d_delays.p, h_delays, p->d_delays.n, cudaMemcpyHostToDevice));
    p->delay_epoch = delay_epoch;
    p->have_delays = true;
    return SW_OK;
}

int sw_pipeline_process_device(sw_pipeline* p, const void* d_taftp, double epoch,
                               sw_stream_t stream)
{
    SW_REQUIRE(p && d_taftp, "sw_pipeline_process_device: null argument");
    cudaStream_t s = as_cuda(stream);
    const int par = (int)(p->gulp & 1);  // outputs alternate between two buffers
    // order after the caller's stream, run, and make the caller's stream wait
    SW_CUDA_CHECK(cudaEventRecord(p->h2d_done[par], s));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->compute, p->h2d_done[par], 0));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->compute, p->d2h_done[par], 0));
    int rc = p->run(d_taftp, par, epoch);
    if(rc != SW_OK) return rc;
    SW_CUDA_CHECK(cudaEventRecord(p->comp_done[par], p->compute));
    SW_CUDA_CHECK(cudaStreamWaitEvent(s, p->comp_done[par], 0));
    ++p->gulp;
    return SW_OK;
}

int sw_pipeline_process_host(sw_pipeline* p, const void* h_taftp, double epoch, void* h_cb_out,
                             sw_stream_t stream)
{
    SW_REQUIRE(p && h_taftp, "sw_pipeline_process_host: null argument");
    const int par = (int)(p->gulp & 1);
    // H2D into this parity's input buffer once its previous gulp consumed it
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->h2d, p->comp_done[par], 0));
    SW_CUDA_CHECK(cudaMemcpyAsync(p->taftp[par].p, h_taftp, p->taftp[par].n,
                                  cudaMemcpyHostToDevice, p->h2d));
    SW_CUDA_CHECK(cudaEventRecord(p->h2d_done[par], p->h2d));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->compute, p->h2d_done[par], 0));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->compute, p->d2h_done[par], 0));
    int rc = p->run(p->taftp[par].p, par, epoch);
    if(rc != SW_OK) return rc;
    SW_CUDA_CHECK(cudaEventRecord(p->comp_done[par], p->compute));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->d2h, p->comp_done[par], 0));
    if(h_cb_out) {
        const size_t nb = p->cb_bytes();
        for(int d = 0; d < p->ndm; ++d)
            SW_CUDA_CHECK(cudaMemcpyAsync(static_cast<uint8_t*>(h_cb_out) + d * nb,
                                          p->cb[par][d].p, nb, cudaMemcpyDeviceToHost, p->d2h));
    }
    SW_CUDA_CHECK(cudaEventRecord(p->d2h_done[par], p->d2h));
    SW_CUDA_CHECK(cudaStreamWaitEvent(as_cuda(stream), p->d2h_done[par], 0));
    ++p->gulp;
    return SW_OK;
}

int sw_pipeline_outputs(sw_pipeline* p, int dm_idx, const int8_t** d_cb_tfb,
                        const float** d_ib_raw, const int8_t** d_ib_btf, const float** d_stats)
{
    SW_REQUIRE(p && dm_idx >= 0 && dm_idx < p->ndm, "sw_pipeline_outputs: bad arguments");
    const int par = p->last_par;
    if(d_cb_tfb) *d_cb_tfb = p->cb[par][dm_idx].as<int8_t>();
    if(d_ib_raw) *d_ib_raw = p->ib_raw[par][dm_idx].as<float>();
    if(d_ib_btf) *d_ib_btf = p->ib_i8[par][dm_idx].as<int8_t>();
    if(d_stats) *d_stats = p->stats[par].as<float>();
    return SW_OK;
}

int sw_pipeline_voltages(sw_pipeline* p, int dm_idx, const int8_t** d_fpact, size_t* row_stride)
{
    SW_REQUIRE(p && dm_idx >= 0 && dm_idx < p->ndm && d_fpact && row_stride,
               "sw_pipeline_voltages: bad arguments");
    const int k = p->dd_of[dm_idx];
    *d_fpact    = (k < 0 ? p->ext[p->last_par].as<int8_t>() : p->dd[k].as<int8_t>()) + p->v_off;
    *row_stride = p->ext_stride;
    return SW_OK;
}

long sw_pipeline_gulp_count(const sw_pipeline* p) { return p ? p->gulp : 0; }

int sw_pipeline_gulp_outputs(sw_pipeline* p, long gulp, int dm_idx, const int8_t** d_cb_tfb,
                             const float** d_ib_raw, const int8_t** d_ib_btf,
                             const float** d_stats)
{
    SW_REQUIRE(p && dm_idx >= 0 && dm_idx < p->ndm, "sw_pipeline_gulp_outputs: bad arguments");
    SW_REQUIRE(gulp >= 0 && gulp < p->gulp && gulp >= p->gulp - 2,
               "sw_pipeline_gulp_outputs: gulp %ld is not one of the last two processed "
               "(%ld processed)", gulp, p->gulp);
    const int par = (int)(gulp & 1);
    SW_CUDA_CHECK(cudaEventSynchronize(p->comp_done[par]));
    if(d_cb_tfb) *d_cb_tfb = p->cb[par][dm_idx].as<int8_t>();
    if(d_ib_raw) *d_ib_raw = p->ib_raw[par][dm_idx].as<float>();
    if(d_ib_btf) *d_ib_btf = p->ib_i8[par][dm_idx].as<int8_t>();
    if(d_stats) *d_stats = p->stats[par].as<float>();
    return SW_OK;
}

int sw_pipeline_order_after(sw_pipeline* p, sw_stream_t stream)
{
    SW_REQUIRE(p, "sw_pipeline_order_after: null pipeline");
    const int par = (int)(p->gulp & 1);
    SW_CUDA_CHECK(cudaEventRecord(p->caller_ready[par], as_cuda(stream)));
    SW_CUDA_CHECK(cudaStreamWaitEvent(p->compute, p->caller_ready[par], 0));
    return SW_OK;
}

int sw_pipeline_wait_input(sw_pipeline* p)
{
    SW_REQUIRE(p, "sw_pipeline_wait_input: null pipeline");
    if(p->gulp > 0) SW_CUDA_CHECK(cudaEventSynchronize(p->h2d_done[(p->gulp - 1) & 1]));
    return SW_OK;
}

size_t sw_pipeline_cb_bytes_per_dm(const sw_pipeline* p) { return p ? p->cb_bytes() : 0; }

int sw_pipeline_fft_len(const sw_pipeline* p, int* fft_len, int* overlap, int* lag)
{
    SW_REQUIRE(p, "sw_pipeline_fft_len: null pipeline");
    if(fft_len) *fft_len = p->fft_len;
    if(overlap) *overlap = p->overlap;
    if(lag) *lag = p->lag;
    return SW_OK;
}

}  // extern "C"
