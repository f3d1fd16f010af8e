// Host-side C++ API tests that need no GPU: the dedispersion plan parser,
// PipelineConfig, DescribedVector metadata over a view, and the argument
// checks that the coherent dedisperser's configuration makes before it
// touches the device.  Built and run by tests/test_cpp_host_api.py on the
// CPU.  Prints "PASS <name>" per case and exits non-zero on the first
// failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "skyweaver_b200.hpp"

using namespace skyweaver_b200;

#define EXPECT(cond)                                                               \
    do {                                                                           \
        if(!(cond)) {                                                              \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            std::exit(1);                                                          \
        }                                                                          \
    } while(0)

template <typename E, typename F>
static bool throws(F&& f)
{
    try {
        f();
    } catch(const E&) {
        return true;
    } catch(...) {
        return false;
    }
    return false;
}

// DedispersionPlan.cpp:18-78: "cdm", "cdm:tscrunch" and
// "cdm:start:end:step:tscrunch"; an empty range keeps its start; any other
// field count is a runtime_error and a field that is not a number an
// invalid_argument.
static void dedispersion_plan()
{
    DedispersionPlan p;
    p.add_block("0");
    p.add_block("150.5:4");
    p.add_block("300:250:350:10:8");
    p.add_block("40:45:45:1:2");
    EXPECT(p.blocks().size() == 4);
    EXPECT((p.coherent_dms() == std::vector<float>{0.0f, 150.5f, 300.0f, 40.0f}));
    EXPECT(p[0].tscrunch == 1 && p[0].incoherent_dms == std::vector<float>{0.0f});
    EXPECT(p[1].tscrunch == 4 && p[1].incoherent_dms == std::vector<float>{150.5f});
    EXPECT(p[2].tscrunch == 8 && p[2].incoherent_dms.size() == 10);
    EXPECT(p[2].incoherent_dms.front() == 250.0f && p[2].incoherent_dms.back() == 340.0f);
    EXPECT(p[3].incoherent_dms == std::vector<float>{45.0f});
    EXPECT(throws<std::runtime_error>([&] { p.add_block("1:2:3"); }));
    EXPECT(throws<std::runtime_error>([&] { p.add_block("1:2:3:4:5:6"); }));
    EXPECT(throws<std::invalid_argument>([&] { p.add_block("fast"); }));
    EXPECT(throws<std::invalid_argument>([&] { p.add_block("10:x"); }));
    EXPECT(p.blocks().size() == 4);
    std::puts("PASS dedispersion_plan");
}

// PipelineConfig.cpp:188-203: channel centres from the centre frequency and
// bandwidth, recomputed when either changes; Stokes modes by name.
static void pipeline_config()
{
    PipelineConfig c;
    c.centre_frequency(1284e6);
    c.bandwidth(64 * 856e6 / 1024);
    c.nchans(64);
    const auto& f = c.channel_frequencies();
    const double chbw = 856e6 / 1024;
    EXPECT(f.size() == 64);
    EXPECT(std::fabs(f[0] - (1284e6 - 32 * chbw + chbw / 2)) < 1e-3);
    EXPECT(std::fabs(f[63] - (1284e6 + 32 * chbw - chbw / 2)) < 1e-3);
    c.nchans(16);
    c.bandwidth(16 * chbw);
    EXPECT(c.channel_frequencies().size() == 16);
    EXPECT(std::fabs(c.channel_frequencies()[8] - (1284e6 + chbw / 2)) < 1e-3);
    EXPECT(c.npol() == 2 && c.nsamples_per_heap() == 256);
    const char* modes[] = {"I", "Q", "U", "V", "IQUV"};
    for(int i = 0; i < 5; ++i) {
        c.stokes_mode(modes[i]);
        EXPECT(c.stokes_index() == i);
        EXPECT(c.stokes_components() == (i == 4 ? 4u : 1u));
    }
    c.stokes_mode("XY");
    EXPECT(throws<std::runtime_error>([&] { c.stokes_index(); }));
    std::puts("PASS pipeline_config");
}

// DescribedVector.hpp:96-573 over host memory viewed as a device vector: no
// CUDA call is made.  Extents per dimension, metadata that must be set
// before it is read, and the count checks on frequencies and DMs.
static void described_vector()
{
    std::vector<int8_t> mem(4 * 3 * 5 * 2);
    auto v = TDBPowersD<int8_t>::view(mem.data(), {4, 3, 10});
    EXPECT(v.size() == 120 && v.data() == mem.data());
    EXPECT(v.nsamples() == 4 && v.ndms() == 3 && v.nbeams() == 10 && v.nchannels() == 1);
    EXPECT(v.dims_as_string() == "TDB");
    EXPECT(throws<std::runtime_error>([&] { v.dms(); }));
    EXPECT(throws<std::runtime_error>([&] { v.frequencies(); }));
    EXPECT(throws<std::runtime_error>([&] { v.dms(std::vector<float>{1.0f, 2.0f}); }));
    v.dms(std::vector<float>{1.0f, 2.0f, 3.0f});
    v.frequencies(1284e6);
    v.tsamp(4.785e-6 * 16);
    v.utc_offset(0.25);
    v.reference_dm(150.0f);
    EXPECT(v.dms().size() == 3 && v.frequencies()[0] == 1284e6);
    EXPECT(v.reference_dm() == 150.0f && v.utc_offset() == 0.25);
    EXPECT(v.describe().find("TDB") != std::string::npos);
    EXPECT(throws<std::invalid_argument>([&] { TDBPowersD<int8_t>::view(mem.data(), {4, 3}); }));
    EXPECT(throws<std::runtime_error>([&] { v.vector().resize(7); }));  // a view cannot grow
    std::vector<char2> fmem(2 * 8 * 2 * 4);
    auto ftpa = FTPAVoltagesD<char2>::view(fmem.data(), {2, 8, 2, 4});
    EXPECT(ftpa.nchannels() == 2 && ftpa.nsamples() == 8 && ftpa.npol() == 2 &&
           ftpa.nantennas() == 4 && ftpa.dims_as_string() == "FTPA");
    EXPECT(throws<std::runtime_error>([&] { ftpa.frequencies(std::vector<double>{1.0}); }));
    ftpa.frequencies(std::vector<double>{1.0e9, 1.1e9});
    EXPECT(ftpa.frequencies().size() == 2);
    std::puts("PASS described_vector");
}

// CoherentDedisperser.cu:19-57: the configuration from a PipelineConfig
// refuses an empty DM list and a whole-band DM delay above twice the gulp,
// both before any device work.
static void coherent_dedisperser_config_checks()
{
    PipelineConfig c;
    c.centre_frequency(1284e6);
    c.bandwidth(64 * 856e6 / 1024);
    c.nchans(64);
    c.gulp_length_samps(256);
    CoherentDedisperserConfig cfg;
    EXPECT(throws<std::runtime_error>([&] { create_coherent_dedisperser_config(cfg, c); }));
    c.ddplan().add_block(5000.0f);  // ~880 samples of delay across 53.5 MHz at L-band
    bool gulp_error = false;
    try {
        create_coherent_dedisperser_config(cfg, c);
    } catch(const std::runtime_error& e) {
        gulp_error = std::string(e.what()).find("2 times the maximum DM delay") != std::string::npos;
    }
    EXPECT(gulp_error);
    std::vector<float> none;
    EXPECT(throws<std::runtime_error>([&] {
        create_coherent_dedisperser_config(cfg, 8192, 1024, 64, 2, 64, 1.196e-6, 1.257e9, 53.5e6,
                                           none);
    }));
    std::puts("PASS coherent_dedisperser_config_checks");
}

int main()
{
    dedispersion_plan();
    pipeline_config();
    described_vector();
    coherent_dedisperser_config_checks();
    std::puts("ALL PASS");
    return 0;
}
