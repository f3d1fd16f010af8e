// C++ stage-API tests, in the shape of the reference's gtest fixtures
// (cpp/skyweaver/test/src/*Tester.cu), against the oracle library
// (oracle/swb_oracle.c, the C restatement of those testers' CPU code).
// Built and run by tests/test_gpu_cpp_api.py.  Prints "PASS <name>" per case
// and exits non-zero on the first failure.
#include <cmath>
#include <fstream>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "skyweaver_b200.hpp"

using namespace skyweaver_b200;

extern "C" {
void swo_transpose(const int8_t*, int8_t*, int, int, int, int, int, int);
void swo_statistics(const int8_t*, float*, int, int, int, int);
void swo_ib(const int8_t*, float*, int8_t*, int, int, int, int, const float*, const float*,
            const float*, int, int);
void swo_cb(const int8_t*, const int8_t*, int8_t*, int, int, int, int, int, const float*,
            const float*, const float*, const int*, int, int, int32_t*);
void swo_weights(const float*, int8_t*, const double*, int, int, int, double, double, double, int);
}

#define EXPECT(cond)                                                                \
    do {                                                                            \
        if(!(cond)) {                                                               \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);  \
            std::exit(1);                                                           \
        }                                                                           \
    } while(0)

static std::vector<int8_t> normal_int8(std::size_t n, float sigma, unsigned seed)
{
    std::mt19937 g(seed);
    std::normal_distribution<float> d(0.0f, sigma);
    std::vector<int8_t> v(n);
    for(auto& x : v) x = (int8_t)std::max(-127.0f, std::min(127.0f, std::rint(d(g))));
    return v;
}

// host bytes <-> device described vectors
template <typename V>
static void put(V& v, const std::vector<int8_t>& h)
{
    EXPECT(v.size() * sizeof(typename V::value_type) == h.size());
    cuda_check(cudaMemcpy(v.data(), h.data(), h.size(), cudaMemcpyHostToDevice), "put");
}
template <typename V>
static std::vector<int8_t> bytes_of(const V& v)
{
    std::vector<int8_t> h(v.size() * sizeof(typename V::value_type));
    cuda_check(cudaMemcpy(h.data(), v.data(), h.size(), cudaMemcpyDeviceToHost), "get");
    return h;
}
template <typename T, typename V>
static std::vector<T> values_of(const V& v)
{
    std::vector<T> h(v.size() * sizeof(typename V::value_type) / sizeof(T));
    cuda_check(cudaMemcpy(h.data(), v.data(), h.size() * sizeof(T), cudaMemcpyDeviceToHost), "get");
    return h;
}

using StokesI = SingleStokesBeamformerTraits<I>;

static PipelineConfig base_config()
{
    PipelineConfig c;
    c.nantennas(64);
    c.nchans(4);
    c.nbeams(128);
    c.cb_tscrunch(16);
    c.ib_tscrunch(16);
    return c;
}

// TransposerTester.cu:119-122 parameters {12 ant, 12 heaps}, {16, 16}
static void transposer_test()
{
    for(auto p : {std::pair<int, int>{12, 12}, {16, 16}}) {
        PipelineConfig c = base_config();
        const int A_in = p.first, H = p.second, F = (int)c.nchans(), A = (int)c.nantennas();
        auto h = normal_int8((std::size_t)H * A_in * F * 256 * 2 * 2, 40.0f, 1);
        TAFTPVoltagesD<char2> taftp({(std::size_t)H, (std::size_t)A_in, (std::size_t)F, 256, 2});
        taftp.tsamp(4096 / 856e6);
        put(taftp, h);
        FTPAVoltagesD<char2> ftpa;
        Transposer t(c);
        t.transpose(taftp, ftpa, A_in, nullptr);
        std::vector<int8_t> ref((std::size_t)F * H * 256 * 2 * A * 2);
        swo_transpose(h.data(), ref.data(), A_in, A, F, H, 256, 2);
        EXPECT(bytes_of(ftpa) == ref);
        EXPECT(ftpa.dims_as_string() == "FTPA" && ftpa.nsamples() == (std::size_t)H * 256);
        EXPECT(ftpa.nantennas() == (std::size_t)A && ftpa.tsamp() == taftp.tsamp());
    }
    std::puts("PASS transposer");
}

static void statistics_test()
{
    PipelineConfig c = base_config();
    const int F = 4, A = 64, T = 1024;
    auto h = normal_int8((std::size_t)F * T * 2 * A * 2, 20.0f, 1337);
    FTPAVoltagesD<char2> ftpa({(std::size_t)F, (std::size_t)T, 2, (std::size_t)A});
    put(ftpa, h);
    StatisticsCalculator s(c, nullptr);
    s.calculate_statistics(ftpa);
    std::vector<float> ref((std::size_t)F * 2 * A * 4);
    swo_statistics(h.data(), ref.data(), F, T, 2, A);
    EXPECT(s.statistics().dims_as_string() == "FPA" && s.statistics().size() == (std::size_t)F * 2 * A);
    auto got = values_of<float>(s.statistics());
    for(std::size_t i = 0; i < ref.size(); ++i)
        EXPECT(std::fabs(got[i] - ref[i]) <= 1e-5f * std::fabs(ref[i]) + 1e-6f);
    std::puts("PASS statistics");
}

// WeightsManagerTester.cu:99-145
static void weights_test()
{
    PipelineConfig c = base_config();
    const int A = 64, B = 128, F = 4;
    for(int which = 0; which < 3; ++which) {
        std::vector<float3> d((std::size_t)B * A);
        for(int i = 0; i < B * A; ++i) {
            if(which == 0) d[i] = float3{1.0f, 0.0f, 0.0f};
            if(which == 1) d[i] = float3{1.0f, 1e-11f, 1e-10f};
            if(which == 2) d[i] = float3{i * 1e-11f, i * 1e-15f, 0.0f};
        }
        DeviceVector<float3> dd;
        dd.upload(d);
        WeightsManager wm(c, nullptr);
        auto got = bytes_of(wm.weights(dd, 10.0, 9.0));
        std::vector<int8_t> ref((std::size_t)F * B * A * 2);
        swo_weights(reinterpret_cast<const float*>(d.data()), ref.data(),
                    c.channel_frequencies().data(), A, B, F, 10.0, 9.0, 0.0, 1);
        EXPECT(got == ref);
    }
    std::puts("PASS weights");
}

// IncoherentBeamformerTester.cu:154-210 (sigma 32, nbeamsets 1..4) and
// CoherentBeamformerTester.cu:211-361 (weights 127 e^{i theta}, beamset_mapping[0] = 1)
static void beamformer_tests()
{
    PipelineConfig c = base_config();
    c.output_level(32.0f);
    const int F = 4, A = 64, B = 128, T = 2048, ts = 16, S = 2;
    auto v = normal_int8((std::size_t)F * T * 2 * A * 2, 32.0f, 7);
    FTPAVoltagesD<char2> ftpa({(std::size_t)F, (std::size_t)T, 2, (std::size_t)A});
    ftpa.tsamp(4096 / 856e6);
    put(ftpa, v);
    const float level = 32.0f;
    const float ib_dof = 2.0f * ts * A * 2, cb_s = std::pow(127.0f * level * std::sqrt((float)A), 2);
    const float cb_dof = 2.0f * ts * 2;
    std::vector<float> ib_scale(S * F, level * level * std::sqrt(2 * ib_dof) / level),
        ib_off(S * F, level * level * ib_dof), cb_scale(S * F, cb_s * std::sqrt(2 * cb_dof) / level),
        cb_off(S * F, cb_s * cb_dof), bw(S * A, 1.0f);
    std::vector<int> mapping(B, 0);
    mapping[0] = 1;
    DeviceVector<float> d_ibs, d_ibo, d_cbs, d_cbo, d_bw;
    DeviceVector<int> d_map;
    d_ibs.upload(ib_scale); d_ibo.upload(ib_off); d_cbs.upload(cb_scale); d_cbo.upload(cb_off);
    d_bw.upload(bw); d_map.upload(mapping);
    BTFPowersD<float> raw;
    BTFPowersD<int8_t> ib;
    IncoherentBeamformer<StokesI> ibf(c);
    ibf.beamform(ftpa, raw, ib, d_ibs, d_ibo, d_bw, S, nullptr);
    std::vector<float> raw_ref((std::size_t)S * (T / ts) * F);
    std::vector<int8_t> ib_ref(raw_ref.size());
    swo_ib(v.data(), raw_ref.data(), ib_ref.data(), F, ts, T, A, ib_scale.data(), ib_off.data(),
           bw.data(), S, 0);
    EXPECT(values_of<float>(raw) == raw_ref);
    EXPECT(bytes_of(ib) == ib_ref);
    EXPECT(ib.dims_as_string() == "BTF" && ib.nbeams() == (std::size_t)S &&
           std::fabs(ib.tsamp() - ts * ftpa.tsamp()) < 1e-15);
    // full Stokes (FullStokesBeamformerTraits): component k of the float4 /
    // char4 result is the single-Stokes result for parameter k
    BTFPowersD<float4> raw4;
    BTFPowersD<char4> ib4;
    IncoherentBeamformer<FullStokesBeamformerTraits> ibf4(c);
    ibf4.beamform(ftpa, raw4, ib4, d_ibs, d_ibo, d_bw, S, nullptr);
    const auto r4 = values_of<float>(raw4);
    const auto b4 = bytes_of(ib4);
    for(int k = 0; k < 4; ++k) {
        swo_ib(v.data(), raw_ref.data(), ib_ref.data(), F, ts, T, A, ib_scale.data(), ib_off.data(),
               bw.data(), S, k);
        for(std::size_t i = 0; i < raw_ref.size(); ++i) {
            EXPECT(r4[4 * i + k] == raw_ref[i]);
            EXPECT(b4[4 * i + k] == ib_ref[i]);
        }
    }
    std::puts("PASS incoherent_beamformer");

    std::mt19937 g(11);
    std::uniform_real_distribution<float> u(0.0f, 6.283185307f);
    std::vector<int8_t> hw((std::size_t)F * B * A * 2);
    for(std::size_t i = 0; i < hw.size(); i += 2) {
        const float th = u(g);
        hw[i]     = (int8_t)std::lround(127.0 * std::cos(th));
        hw[i + 1] = (int8_t)std::lround(127.0 * std::sin(th));
    }
    DeviceVector<char2> w((std::size_t)F * B * A);
    cuda_check(cudaMemcpy(w.data(), hw.data(), hw.size(), cudaMemcpyHostToDevice), "weights");
    TFBPowersD<int8_t> cb;
    CoherentBeamformer<StokesI> cbf(c);
    cbf.beamform(ftpa, w, d_cbs, d_cbo, d_map, raw, cb, S, nullptr);
    std::vector<int8_t> cb_ref((std::size_t)(T / ts) * F * B);
    swo_cb(v.data(), hw.data(), cb_ref.data(), F, ts, T, B, A, cb_scale.data(), cb_off.data(),
           bw.data(), mapping.data(), 0, 1, nullptr);
    EXPECT(bytes_of(cb) == cb_ref);
    EXPECT(cb.dims_as_string() == "TFB" && cb.nsamples() == (std::size_t)T / ts &&
           cb.nbeams() == (std::size_t)B);
    std::puts("PASS coherent_beamformer");
}

// CoherentDedisperserTester.cu:21-204: the configuration of the reference's
// fixture and its golden vector (DM 1000, one channel, 1024-point FFT), within
// the reference's tolerance of one; DM 0 reproduces the input window.
static void coherent_dedisperser_tests(const std::string& golden)
{
    const std::vector<float> dms = {0.0f, 1000.0f};
    const std::size_t fft_length = 1024, nantennas = 64, nchans = 64, npols = 2;
    const double tsamp = 4096 / 856e6, f_low = 856e6, bridge_bw = 13.375e6;
    const double f2 = f_low + 856e6 / 4096;
    const double delay = 4.148806423e15 * (1.0 / (f_low * f_low) - 1.0 / (f2 * f2)) * 1000.0;
    const std::size_t max_delay_samps = (std::size_t)std::ceil(delay / tsamp);
    EXPECT(max_delay_samps == 578);
    CoherentDedisperserConfig cfg;
    create_coherent_dedisperser_config(cfg, fft_length, max_delay_samps, nchans, npols, nantennas,
                                       tsamp, f_low, bridge_bw, dms);
    EXPECT(std::fabs(cfg.filter_delay - tsamp * 289) < 1e-15 && cfg.high_freq == f_low + bridge_bw);
    CoherentDedisperser cdd(cfg);
    std::ifstream fin(golden + "/codedisp_input_DM1000_1chan.bin", std::ios::binary);
    std::ifstream fout(golden + "/codedisp_output_DM1000_1chan.bin", std::ios::binary);
    std::vector<int8_t> in(1024 * 2 * 64 * 2), want(446 * 2 * 64 * 2);
    fin.read(reinterpret_cast<char*>(in.data()), (std::streamsize)in.size());
    fout.read(reinterpret_cast<char*>(want.data()), (std::streamsize)want.size());
    EXPECT(fin.good() && fout.good());
    TPAVoltagesD<char2> d_in({1024, npols, nantennas});
    put(d_in, in);
    FTPAVoltagesD<char2> d_out({1, fft_length - max_delay_samps, npols, nantennas});
    cdd.dedisperse(d_in, d_out, 0, 1);
    EXPECT(d_out.reference_dm() == 1000.0f);
    const auto got = bytes_of(d_out);
    std::size_t exact = 0;
    for(std::size_t i = 0; i < got.size(); ++i) {
        EXPECT(std::abs((int)got[i] - (int)want[i]) <= 1);
        exact += got[i] == want[i];
    }
    std::printf("coherent dedisperser golden vector: %zu of %zu values exact\n", exact, got.size());
    cdd.dedisperse(d_in, d_out, 0, 0);   // DM 0: the window's middle, unchanged
    const auto id = bytes_of(d_out);
    for(std::size_t i = 0; i < id.size(); ++i) EXPECT(id[i] == in[289 * 2 * 64 * 2 + i]);
    // the gulp-length overload and its limit (CoherentDedisperser.cu:19-57)
    PipelineConfig c = base_config();
    c.nchans(64);
    c.bandwidth(64 * 856e6 / 1024);
    c.gulp_length_samps(65536);
    c.ddplan().add_block(150.0f);
    CoherentDedisperserConfig cfg2;
    create_coherent_dedisperser_config(cfg2, c);
    EXPECT(cfg2.fft_length == 65536 && cfg2.overlap_samps > 1000);
    c.ddplan().add_block(5000.0f);
    bool threw = false;
    try { create_coherent_dedisperser_config(cfg2, c); } catch(const std::runtime_error&) { threw = true; }
    EXPECT(threw);
    std::puts("PASS coherent_dedisperser");
}

// IncoherentDedisperserTester.cu:39-126
static void incoherent_dedisperser_tests()
{
    PipelineConfig c = base_config();
    c.nchans(64);
    c.nbeams(32);
    {
        IncoherentDedisperser d(c, 0.0f);
        for(int x : d.delays()) EXPECT(x == 0);
        EXPECT(d.max_sample_delay() == 0);
    }
    c.bandwidth(32e6);
    c.centre_frequency(580e6);
    std::vector<float> dms = {0.0f, 10.0f, 20.0f, 30.0f, 40.0f};
    for(std::size_t ts : {1, 2}) {
        IncoherentDedisperser d(c, dms, ts);
        EXPECT(d.max_sample_delay() > 0);
        std::size_t T = 3 * d.max_sample_delay();
        T -= (T - d.max_sample_delay()) % ts;
        DeviceVector<int8_t> tfb;
        TDBPowersD<int8_t> tdb;
        tfb.upload(std::vector<int8_t>(T * c.nchans() * c.nbeams(), 1));
        d.dedisperse(tfb, tdb);
        const auto out = bytes_of(tdb);
        EXPECT(out.size() == (T - d.max_sample_delay()) / ts * dms.size() * c.nbeams());
        EXPECT(tdb.ndms() == dms.size() && tdb.nbeams() == c.nbeams());
        for(int8_t x : out) EXPECT(x == (int8_t)std::sqrt((double)(c.nchans() * ts)));
    }
    {
        IncoherentDedisperser d(c, dms);
        DeviceVector<int8_t> tfb;
        TDBPowersD<int8_t> tdb;
        tfb.upload(std::vector<int8_t>(d.max_sample_delay() * c.nchans() * c.nbeams(), 0));
        bool threw = false;
        try { d.dedisperse(tfb, tdb); } catch(const std::runtime_error&) { threw = true; }
        EXPECT(threw);
    }
    std::puts("PASS incoherent_dedisperser");
}

// DelayManagerTester.cu:38-52 with the reference's test_delays.bin
static void delay_manager_tests(const std::string& golden)
{
    PipelineConfig c = base_config();
    c.delay_file(golden + "/test_delays.bin");
    DelayManager dm(c, nullptr);
    EXPECT(dm.nbeamsets() == 2);
    EXPECT(dm.beamset_weights_host().size() == 2 * c.nantennas());
    EXPECT(std::fabs(dm.epoch() - 1708082168.957) < 1e-3);
    const auto& d = dm.delays(dm.epoch() + 1.0);
    EXPECT(d.size() == c.nbeams() * c.nantennas());
    EXPECT(dm.beamset_mapping().size() == c.nbeams() && dm.beamset_weights().size() == 2 * c.nantennas());
    bool threw = false;
    try { dm.delays(dm.epoch() - 10.0); } catch(const InvalidDelayEpoch&) { threw = true; }
    EXPECT(threw);
    threw = false;
    try { dm.delays(1e10); } catch(const std::runtime_error&) { threw = true; }
    EXPECT(threw);
    std::puts("PASS delay_manager");
}

static void dedispersion_plan_tests()
{
    DedispersionPlan p;
    p.add_block("10.0");
    p.add_block("20.0:4");
    p.add_block("30.0:25.0:35.0:2.0:8");
    EXPECT(p.coherent_dms().size() == 3);
    EXPECT(p[1].tscrunch == 4);
    EXPECT(p[2].incoherent_dms.size() == 5);
    bool threw = false;
    try { p.add_block("1:2:3"); } catch(const std::runtime_error&) { threw = true; }
    EXPECT(threw);
    std::puts("PASS dedispersion_plan");
}

// handlers with the reference's concept: init(header), operator()(vector, dm)
struct CbCounter {
    std::size_t inits = 0, calls = 0, bytes = 0;
    std::vector<float> dms_seen;
    double tsamp = 0.0, utc_offset = -1.0;
    std::vector<double> freqs;
    void init(const ObservationHeader&) { ++inits; }
    void operator()(const TFBPowersD<int8_t>& v, std::size_t dm_idx)
    {
        ++calls;
        bytes += v.size();
        dms_seen.push_back(v.reference_dm());
        EXPECT(v.dims_as_string() == "TFB" && dm_idx < 2);
        tsamp = v.tsamp();
        utc_offset = v.utc_offset();
        freqs = v.frequencies();
        (void)bytes_of(v);   // the view is readable on the legacy stream
    }
};
struct IbCounter {
    std::size_t inits = 0, calls = 0, nbeamsets = 0;
    void init(const ObservationHeader&) { ++inits; }
    void operator()(const BTFPowersD<int8_t>& v, std::size_t) { ++calls; nbeamsets = v.nbeams(); }
};
struct StatsCounter {
    std::size_t inits = 0, calls = 0, nseries = 0;
    void init(const ObservationHeader&) { ++inits; }
    void operator()(const FPAStatsD<Statistics>& v) { ++calls; nseries = v.size(); }
};

// BeamformerPipelineTester.cu:119-167 (zeros through the full chain) with the
// reference's handler concept and epoch arithmetic (BeamformerPipeline.cu:
// 100-115, 262-301)
static void pipeline_smoke(const std::string& golden)
{
    PipelineConfig c = base_config();
    c.delay_file(golden + "/test_delays.bin");
    c.gulp_length_samps(4096);
    c.ddplan().add_block(0.0f);
    c.ddplan().add_block(5.0f);
    CbCounter cbh;
    IbCounter ibh;
    StatsCounter sh;
    {
        BeamformerPipeline<CbCounter, IbCounter, StatsCounter> pipe(c, cbh, ibh, sh);
        ObservationHeader hdr{};
        hdr.nantennas = 57;
        hdr.utc_start = 1708082168.957 + 1.0;
        hdr.sample_clock = 1712e6;
        pipe.init(hdr, 0.0);
        EXPECT(cbh.inits == 1 && ibh.inits == 1 && sh.inits == 1);
        TAFTPVoltagesH<char2> taftp({16, 57, c.nchans(), 256, 2});
        std::memset(taftp.data(), 0, taftp.size() * sizeof(char2));
        for(int g = 0; g < 3; ++g) EXPECT(pipe(taftp) == false);
        EXPECT(cbh.calls == 4);   // gulps 0 and 1 delivered, gulp 2 pending
        pipe.flush();
        EXPECT(pipe.call_count() == 3);
    }
    EXPECT(cbh.calls == 6 && ibh.calls == 6 && sh.calls == 3);
    EXPECT(cbh.bytes == 6 * (4096 / 16) * c.nchans() * c.nbeams());
    EXPECT(cbh.dms_seen[0] == 0.0f && cbh.dms_seen[1] == 5.0f);
    EXPECT(cbh.freqs == c.channel_frequencies());
    const double chan_tsamp = (double)c.nchans() / c.bandwidth();
    EXPECT(std::fabs(cbh.tsamp - 16 * chan_tsamp) < 1e-15 && cbh.utc_offset >= 0.0);
    EXPECT(ibh.nbeamsets == 2 && sh.nseries == c.nchans() * 2 * c.nantennas());
    // a pipeline used before init() refuses the gulp
    BeamformerPipeline<CbCounter, IbCounter, StatsCounter> pipe2(c, cbh, ibh, sh);
    TAFTPVoltagesH<char2> taftp({16, 57, c.nchans(), 256, 2});
    bool threw = false;
    try { pipe2(taftp); } catch(const std::runtime_error&) { threw = true; }
    EXPECT(threw);
    std::puts("PASS beamformer_pipeline");
}

struct TdbCollector {
    std::vector<std::vector<int8_t>> got[2];
    std::size_t nbeams = 0, ndms[2] = {0, 0};
    float ref_dm[2] = {0, 0};
    double utc_offset[2] = {0, 0};
    void init(const ObservationHeader&) {}
    void operator()(const TDBPowersD<int8_t>& tdb, std::size_t block)
    {
        got[block].push_back(bytes_of(tdb));
        nbeams = tdb.nbeams();
        ndms[block] = tdb.ndms();
        EXPECT(tdb.dms().size() == tdb.ndms());
        ref_dm[block] = tdb.reference_dm();
        utc_offset[block] = tdb.utc_offset();
    }
};

// IncoherentDedispersionPipeline.cu:6-113 + AggregationBuffer.cu:23-117:
// all-ones TFB gives sqrt(nchans * tscrunch) (truncated) in every output, and
// block b dispatches floor((T - overlap) / dispatch) times
static void idd_pipeline_tests()
{
    PipelineConfig c = base_config();
    c.nchans(64);
    c.nbeams(32);
    c.bandwidth(32e6);
    c.centre_frequency(580e6);
    c.cb_tscrunch(16);
    c.ddplan().add_block("5.0:0.0:20.0:5.0:1");
    c.ddplan().add_block("30.0:25.0:45.0:10.0:2");
    const auto& plan = c.ddplan();
    TdbCollector col;
    IncoherentDedispersionPipeline<int8_t, int8_t, TdbCollector> idd(c, col);
    const std::size_t T = 40000, slot = c.nchans() * c.nbeams();
    DeviceVector<int8_t> ones;
    ones.upload(std::vector<int8_t>(T * slot, 1));
    const double tsamp = 16 / (32e6 / 64);
    for(int b = 0; b < 2; ++b) {
        std::size_t pos = 0;
        for(std::size_t n : {1000u, 17u, 20000u, 18983u}) {
            auto v = TFBPowersD<int8_t>::view(ones.data() + pos * slot, {n, c.nchans(), c.nbeams()});
            v.tsamp(tsamp);
            idd(v, b);
            pos += n;
        }
        EXPECT(pos == T);
    }
    cuda_check(cudaDeviceSynchronize(), "idd pipeline");
    for(int b = 0; b < 2; ++b) {
        const auto& d = idd.dedisperser(b);
        const std::size_t O = d.max_sample_delay();
        std::size_t D = std::max<std::size_t>(O * 10, 8192);
        const std::size_t ts = plan[b].tscrunch;
        D -= D % ts;
        EXPECT(col.got[b].size() == (T - O) / D);
        EXPECT(col.ndms[b] == plan[b].incoherent_dms.size());
        EXPECT(col.ref_dm[b] == plan[b].coherent_dm);
        EXPECT(std::fabs(col.utc_offset[b] - O * tsamp) < 1e-12);
        const int8_t want = (int8_t)std::sqrt((double)(c.nchans() * ts));
        for(const auto& v : col.got[b]) {
            EXPECT(v.size() == D / ts * col.ndms[b] * c.nbeams());
            for(int8_t x : v) EXPECT(x == want);
        }
    }
    std::puts("PASS incoherent_dedispersion_pipeline");
}

// ObservationHeader.cpp:6-33 + MultiFileReader.cu + MultiFileWriter.cu
static void dada_io_tests(const std::string& scratch)
{
    const std::string hdr_text =
        "HEADER DADA\nHDR_SIZE 4096\nNCHAN 64\nOBS_NCHAN 4096\nNPOL 2\nNBIT 8\nNANT 57\n"
        "SAMPLE_CLOCK_START 0\nBW 13375000.0\nOBS_BW 856000000.0\nFREQ 1284000000.0\n"
        "OBS_FREQ 1284000000.0\nTSAMP 4.785\nSAMPLE_CLOCK 1712000000.0\nSYNC_TIME 0\n"
        "UTC_START 1708082229.0\nMJD_START 60356.47\nSOURCE J1644-4559\nRA 16:44:49.27\n"
        "DEC -45:59:09.7\nTELESCOPE MeerKAT\nINSTRUMENT CBF-Feng\nCHAN0_IDX 2688\n";
    std::vector<int8_t> payload = normal_int8(10000, 20.0f, 9);
    std::vector<std::string> files;
    for(int i = 0; i < 2; ++i) {
        std::string h = hdr_text + "OBS_OFFSET " + std::to_string(i * 6000) + "\n";
        h.resize(4096, '\0');
        files.push_back(scratch + "/in" + std::to_string(i) + ".dada");
        std::ofstream f(files.back(), std::ios::binary);
        f.write(h.data(), (std::streamsize)h.size());
        f.write(reinterpret_cast<const char*>(payload.data()) + i * 6000, i ? 4000 : 6000);
    }
    MultiFileReader r(files, 4096, true);
    EXPECT(r.get_total_size() == 10000);
    EXPECT(r.get_header().nantennas == 57 && r.get_header().chan0_idx == 2688);
    std::vector<int8_t> back(10000);
    EXPECT(r.read(reinterpret_cast<char*>(back.data()), 10000) == 10000);
    EXPECT(back == payload && r.eof());
    {
        MultiFileWriter w(scratch + "/out", r.get_header(), 5000, "I", "sw", "cb");
        MultiFileWriter::StreamInfo s{32, 64, 40, 0, {}, 150.0f, 1.9e-5, 0.0, "TFB"};
        for(int k = 0; k < 3; ++k) w(payload.data() + k * 2560, 2560, s, 1);
    }
    const std::string dir = scratch + "/out/2024-02-16-11:17:09/1/1284000000/";
    const std::string base = dir + "sw_2024-02-16-11:17:09_1_00150.000_1284000000_cb_";
    std::ifstream f0(base + "0000000000000000.tfb", std::ios::binary);
    EXPECT(f0.good());
    std::string h0(4096, '\0');
    f0.read(&h0[0], 4096);
    char v[64];
    EXPECT(sw_dada_header_get(h0.data(), 4096, "NBEAM", v, sizeof(v)) == SW_OK && std::string(v) == "32");
    EXPECT(sw_dada_header_get(h0.data(), 4096, "ORDER", v, sizeof(v)) == SW_OK && std::string(v) == "TFB");
    EXPECT(sw_dada_header_get(h0.data(), 4096, "FILE_SIZE", v, sizeof(v)) == SW_OK && std::string(v) == "2560");
    // 5000-byte limit rounded down to whole 2560-byte blocks: three files
    std::ifstream f1(base + "0000000000002560.tfb", std::ios::binary), f2(base + "0000000000005120.tfb", std::ios::binary);
    EXPECT(f1.good() && f2.good());
    std::puts("PASS dada_io");
}

// The coherent beamformer's bounded waits, through the C ABI: a launch whose
// copy producer never issues must report SW_ERR_TIMEOUT and leave the device
// error word clear, and the context must stay usable.
static void bounded_wait_test()
{
    EXPECT(sw_reset_device_error() == SW_OK);
    EXPECT(sw_cb_timeout_selftest(20000, nullptr) == SW_ERR_TIMEOUT);
    int code = -1;
    EXPECT(sw_read_device_error(&code) == SW_OK && code == 0);
    EXPECT(sw_cb_timeout_selftest(0, nullptr) == SW_ERR_INVALID);
    std::puts("PASS bounded_wait");
}

int main(int argc, char** argv)
{
    const std::string golden = argc > 1 ? argv[1] : "tests/golden";
    transposer_test();
    statistics_test();
    weights_test();
    beamformer_tests();
    coherent_dedisperser_tests(golden);
    incoherent_dedisperser_tests();
    delay_manager_tests(golden);
    dedispersion_plan_tests();
    pipeline_smoke(golden);
    idd_pipeline_tests();
    dada_io_tests(argc > 2 ? argv[2] : ".");
    bounded_wait_test();
    beamformer_tests();  // the context is still usable after the timeout
    std::puts("ALL PASS");
    return 0;
}
