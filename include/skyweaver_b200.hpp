// skyweaver_b200.hpp -- C++ drop-in layer over the C ABI in skyweaver_b200.h.
//
// Mirrors the reference's stage classes (erc-compact/skyweaver,
// cpp/skyweaver/*.cuh) for the beamforming hot path: same class and method
// names, the same argument meaning, std::runtime_error on the same errors.
// Device buffers are DeviceBuffer<T> (cudaMalloc, RAII) instead of
// DescribedVector<thrust::device_vector>; the dimension metadata of the
// reference's DescribedVector is carried as explicit sizes.
//
// Header only; link with -lskyweaver_b200 -lcudart.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <cctype>
#include <ctime>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "skyweaver_b200.h"

namespace skyweaver_b200 {

inline void check(int status)
{
    if(status != SW_OK) throw std::runtime_error(sw_last_error());
}

inline void cuda_check(cudaError_t e, const char* what)
{
    if(e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ buffers
template <typename T>
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) { resize(n); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : _p(o._p), _n(o._n) { o._p = nullptr; o._n = 0; }
    ~DeviceBuffer() { if(_p) cudaFree(_p); }
    void resize(std::size_t n)
    {
        if(n == _n) return;
        if(_p) cudaFree(_p);
        _p = nullptr;
        _n = n;
        if(n) cuda_check(cudaMalloc(&_p, n * sizeof(T)), "cudaMalloc");
    }
    T* data() { return _p; }
    const T* data() const { return _p; }
    std::size_t size() const { return _n; }
    void upload(const std::vector<T>& h)
    {
        resize(h.size());
        cuda_check(cudaMemcpy(_p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "H2D");
    }
    std::vector<T> download() const
    {
        std::vector<T> h(_n);
        cuda_check(cudaMemcpy(h.data(), _p, _n * sizeof(T), cudaMemcpyDeviceToHost), "D2H");
        return h;
    }

  private:
    T* _p = nullptr;
    std::size_t _n = 0;
};

// --------------------------------------------------------------- Description
// The metadata that the reference's DescribedVector carries beside its data
// (cpp/skyweaver/DescribedVector.hpp:96-573: dimension order and extents,
// channel frequencies, tsamp, utc_offset, dms, reference_dm).  Here the data
// stays a plain device buffer and its description travels beside it, with
// the reference's getter names.
struct Description {
    std::string dims;                  // dimension order, outermost first ("TFB", "BTF", ...)
    std::vector<std::size_t> sizes;    // extent of each dimension in `dims`
    std::vector<double> freqs;         // channel centre frequencies (Hz)
    double sample_period = 0.0;        // seconds per sample of the T dimension
    double offset = 0.0;               // seconds: the dedisperser's filter delay
    std::vector<float> trial_dms;      // DMs of a D dimension
    float coherent_dm = 0.0f;          // DM the voltages were coherently dedispersed to

    const std::vector<std::size_t>& extents() const { return sizes; }
    std::string dims_as_string() const { return dims; }
    const std::vector<double>& frequencies() const { return freqs; }
    double tsamp() const { return sample_period; }
    double utc_offset() const { return offset; }
    const std::vector<float>& dms() const { return trial_dms; }
    float reference_dm() const { return coherent_dm; }
    std::size_t extent(char d) const
    {
        std::size_t n = 1;
        for(std::size_t i = 0; i < dims.size(); ++i)
            if(dims[i] == d) n *= sizes[i];
        return n;
    }
    std::size_t nsamples() const { return extent('T'); }
    std::size_t nchannels() const { return extent('F'); }
    std::size_t nbeams() const { return extent('B'); }
    std::size_t ndms() const { return extent('D'); }
};

// --------------------------------------------------------- DedispersionPlan
// cpp/skyweaver/DedispersionPlan.hpp:11-123, src/DedispersionPlan.cpp:17-78
struct DedispersionPlanBlock {
    float coherent_dm;
    int tscrunch;
    std::vector<float> incoherent_dms;
};

class DedispersionPlan {
  public:
    void add_block(float coherent_dm, float dm_begin, float dm_end, float dm_step, int tscrunch)
    {
        DedispersionPlanBlock b{coherent_dm, tscrunch, {}};
        for(float dm = dm_begin; dm < dm_end; dm += dm_step) b.incoherent_dms.push_back(dm);
        if(b.incoherent_dms.empty()) b.incoherent_dms.push_back(dm_begin);
        add_block(std::move(b));
    }
    void add_block(float coherent_dm, int tscrunch = 1)
    {
        add_block(DedispersionPlanBlock{coherent_dm, tscrunch, {coherent_dm}});
    }
    void add_block(DedispersionPlanBlock&& b)
    {
        _dms.push_back(b.coherent_dm);
        _blocks.emplace_back(std::move(b));
    }
    // "cdm[:start:end:step]:tscrunch" (DedispersionPlan.cpp:50-78)
    void add_block(const std::string& str)
    {
        std::vector<std::string> parts;
        std::stringstream ss(str);
        std::string item;
        while(std::getline(ss, item, ':')) parts.push_back(item);
        try {
            switch(parts.size()) {
            case 1: add_block(std::stof(parts[0])); break;
            case 2: add_block(std::stof(parts[0]), std::stoi(parts[1])); break;
            case 5:
                add_block(std::stof(parts[0]), std::stof(parts[1]), std::stof(parts[2]),
                          std::stof(parts[3]), std::stoi(parts[4]));
                break;
            default:
                throw std::runtime_error("Block defition string of unexpected size: " + str);
            }
        } catch(std::invalid_argument& e) {
            throw std::invalid_argument(std::string("Error parsing block definition string: ") +
                                        e.what());
        }
    }
    const std::vector<float>& coherent_dms() const { return _dms; }
    const std::vector<DedispersionPlanBlock>& blocks() const { return _blocks; }
    const DedispersionPlanBlock& operator[](std::size_t i) const { return _blocks[i]; }

  private:
    std::vector<DedispersionPlanBlock> _blocks;
    std::vector<float> _dms;
};

// ----------------------------------------------------------- PipelineConfig
// cpp/skyweaver/PipelineConfig.hpp; the reference's compile-time sizes
// (skyweaver_constants.hpp:28-94) are runtime fields with the same getters.
class PipelineConfig {
  public:
    std::size_t nantennas() const { return _nant; }
    void nantennas(std::size_t n) { _nant = n; }
    std::size_t nchans() const { return _nchans; }
    void nchans(std::size_t n) { _nchans = n; _stale = true; }
    std::size_t nbeams() const { return _nbeams; }
    void nbeams(std::size_t n) { _nbeams = n; }
    std::size_t npol() const { return 2; }
    std::size_t nsamples_per_heap() const { return 256; }
    std::size_t cb_tscrunch() const { return _cb_ts; }
    void cb_tscrunch(std::size_t t) { _cb_ts = t; }
    std::size_t ib_tscrunch() const { return _ib_ts; }
    void ib_tscrunch(std::size_t t) { _ib_ts = t; }
    std::size_t cb_fscrunch() const { return 1; }
    std::size_t ib_fscrunch() const { return 1; }
    bool ib_subtraction() const { return _ib_sub; }
    void ib_subtraction(bool b) { _ib_sub = b; }
    double centre_frequency() const { return _cfreq; }
    void centre_frequency(double f) { _cfreq = f; _stale = true; }
    double bandwidth() const { return _bw; }
    void bandwidth(double b) { _bw = b; _stale = true; }
    std::size_t gulp_length_samps() const { return _gulp; }
    void gulp_length_samps(std::size_t n) { _gulp = n; }
    float output_level() const { return _level; }
    void output_level(float l) { _level = l; }
    std::string stokes_mode() const { return _stokes; }
    void stokes_mode(const std::string& s) { _stokes = s; }
    const std::string& delay_file() const { return _delay_file; }
    void delay_file(const std::string& f) { _delay_file = f; }
    DedispersionPlan& ddplan() { return _plan; }
    const DedispersionPlan& ddplan() const { return _plan; }
    const std::vector<float>& coherent_dms() const { return _plan.coherent_dms(); }
    // PipelineConfig.cpp:188-203
    const std::vector<double>& channel_frequencies() const
    {
        if(_stale) {
            const double chbw = _bw / _nchans, fbottom = _cfreq - _bw / 2.0;
            _freqs.clear();
            for(std::size_t i = 0; i < _nchans; ++i) _freqs.push_back(fbottom + chbw / 2.0 + chbw * i);
            _stale = false;
        }
        return _freqs;
    }
    // "I", "Q", "U", "V" (SingleStokesBeamformerTraits) or "IQUV"
    // (FullStokesBeamformerTraits: char4 / float4 outputs)
    int stokes_index() const
    {
        static const char* names[] = {"I", "Q", "U", "V", "IQUV"};
        for(int i = 0; i < 5; ++i)
            if(_stokes == names[i]) return i;
        throw std::runtime_error("Unsupported Stokes mode: " + _stokes);
    }
    // values per output sample: 4 for IQUV, else 1
    std::size_t stokes_components() const { return stokes_index() == 4 ? 4 : 1; }

  private:
    std::size_t _nant = 64, _nchans = 64, _nbeams = 32, _cb_ts = 16, _ib_ts = 16, _gulp = 4096;
    bool _ib_sub = true;
    double _cfreq = 1284000000.0, _bw = 13375000.0;
    float _level = 24.0f;
    std::string _stokes = "I", _delay_file;
    bool _autotune = false;

  public:
    // let sw_autotune pick the FFT length and beamformer work-item size
    bool autotune() const { return _autotune; }
    void autotune(bool on) { _autotune = on; }

  private:
    DedispersionPlan _plan;
    mutable bool _stale = true;
    mutable std::vector<double> _freqs;
};

// -------------------------------------------------------------- DelayManager
// cpp/skyweaver/DelayManager.cuh:19-148, src/DelayManager.cu:16-249
class InvalidDelayEpoch : public std::exception {
  public:
    explicit InvalidDelayEpoch(double e) : epoch(e)
    {
        std::ostringstream os;
        os << "No valid delay model for epoch " << e;
        _msg = os.str();
    }
    const char* what() const noexcept override { return _msg.c_str(); }
    double epoch;

  private:
    std::string _msg;
};

#pragma pack(push, 1)
struct DelayModelHeader {
    uint32_t nbeams;
    uint32_t nantennas;
    double start_epoch;
    double end_epoch;
};
#pragma pack(pop)

class DelayManager {
  public:
    DelayManager(const PipelineConfig& config, cudaStream_t stream) : _config(config), _stream(stream)
    {
        _in.open(config.delay_file(), std::ios::in | std::ios::binary);
        if(!_in.is_open())
            throw std::runtime_error("Error: Unable to open file delay file: " + config.delay_file());
        read_next_model();
        _valid_nbeams = _hdr.nbeams;
        _valid_nant   = _hdr.nantennas;
        parse_beamsets();
    }
    // float3 [nbeams][nantennas] on the device, zero padded to the config
    const DeviceBuffer<float>& delays(double epoch)
    {
        if(epoch < _hdr.start_epoch) throw InvalidDelayEpoch(epoch);
        while(!validate_model(epoch)) read_next_model();
        if(_hdr.nantennas > _config.nantennas())
            throw std::runtime_error("Delay model contains too many antennas");
        if(_hdr.nbeams > _config.nbeams()) throw std::runtime_error("Delay model contains too many beams");
        std::vector<float> padded(_config.nbeams() * _config.nantennas() * 3, 0.0f);
        for(uint32_t b = 0; b < _hdr.nbeams; ++b)
            std::memcpy(&padded[3 * (b * _config.nantennas())], &_h[3 * (b * _hdr.nantennas)],
                        3 * sizeof(float) * _hdr.nantennas);
        _d.upload(padded);
        return _d;
    }
    double epoch() const { return _hdr.start_epoch; }
    const std::vector<float>& beamset_weights() const { return _bs_weights; }
    const std::vector<int>& beamset_mapping() const { return _bs_map; }
    int nbeamsets() const { return _nbs; }

  private:
    bool validate_model(double epoch) const
    {
        if(_hdr.nbeams != _valid_nbeams || _hdr.nantennas != _valid_nant)
            throw std::runtime_error("Variable delay model parameters are unsupported");
        return epoch >= _hdr.start_epoch && epoch <= _hdr.end_epoch;
    }
    void safe_read(char* buf, std::size_t n)
    {
        _in.read(buf, n);
        if(_in.eof()) throw std::runtime_error("Reached end of delay model file");
        if(_in.fail() || _in.bad()) throw std::runtime_error("Error: Unable to read from delay file");
    }
    void read_next_model()
    {
        safe_read(reinterpret_cast<char*>(&_hdr), sizeof(_hdr));
        if(_hdr.nbeams > _config.nbeams())
            throw std::runtime_error("Delay model contains too many beams for current skyweaver build");
        _h.resize((std::size_t)_hdr.nbeams * _hdr.nantennas * 3);
        safe_read(reinterpret_cast<char*>(_h.data()), _h.size() * sizeof(float));
    }
    void parse_beamsets()  // DelayManager.cu:162-232 (contiguous beamsets)
    {
        const std::size_t A = _config.nantennas();
        std::vector<std::vector<float>> sets(1, std::vector<float>(A, 0.0f));
        _bs_map.assign(_config.nbeams(), 0);
        for(uint32_t a = 0; a < _hdr.nantennas; ++a) sets[0][a] = _h[3 * a];
        for(uint32_t b = 1; b < _hdr.nbeams; ++b) {
            bool diff = false;
            for(uint32_t a = 0; a < _hdr.nantennas; ++a)
                diff |= _h[3 * (b * _hdr.nantennas + a)] != sets.back()[a];
            if(diff) {
                sets.emplace_back(A, 0.0f);
                for(uint32_t a = 0; a < _hdr.nantennas; ++a) sets.back()[a] = _h[3 * (b * _hdr.nantennas + a)];
            }
            _bs_map[b] = (int)sets.size() - 1;
        }
        _nbs = (int)sets.size();
        _bs_weights.clear();
        for(auto& s : sets) _bs_weights.insert(_bs_weights.end(), s.begin(), s.end());
    }

    const PipelineConfig& _config;
    cudaStream_t _stream;
    std::ifstream _in;
    DelayModelHeader _hdr{};
    std::vector<float> _h;
    DeviceBuffer<float> _d;
    uint32_t _valid_nbeams = 0, _valid_nant = 0;
    std::vector<float> _bs_weights;
    std::vector<int> _bs_map;
    int _nbs = 0;
};

// ------------------------------------------------------------ WeightsManager
// cpp/skyweaver/WeightsManager.cuh:43-65; returns the reference [F][B][A]
// char2 weights and keeps the tensor-core GEMM layout for CoherentBeamformer.
class WeightsManager {
  public:
    WeightsManager(const PipelineConfig& config, cudaStream_t stream) : _config(config), _stream(stream)
    {
        const std::size_t n = config.nchans() * config.nbeams() * config.nantennas() * 2;
        _w.resize(n);
        _gemm.resize(2 * n);
        _freqs.upload(config.channel_frequencies());
    }
    const DeviceBuffer<int8_t>& weights(const DeviceBuffer<float>& delays, double current_epoch,
                                        double delay_epoch)
    {
        check(sw_generate_weights(delays.data(), _freqs.data(), (int)_config.nantennas(),
                                  (int)_config.nbeams(), (int)_config.nchans(), current_epoch,
                                  delay_epoch, _w.data(), _gemm.data(), (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "weights");
        return _w;
    }
    const DeviceBuffer<int8_t>& gemm_weights() const { return _gemm; }

  private:
    const PipelineConfig& _config;
    cudaStream_t _stream;
    DeviceBuffer<int8_t> _w, _gemm;
    DeviceBuffer<double> _freqs;
};

// ---------------------------------------------------------------- Transposer
// cpp/skyweaver/Transposer.cuh:54-69: TAFTP -> FTPA (antennas zero padded)
class Transposer {
  public:
    explicit Transposer(const PipelineConfig& config) : _config(config) {}
    void transpose(const DeviceBuffer<int8_t>& taftp, DeviceBuffer<int8_t>& ftpa,
                   std::size_t input_nantennas, cudaStream_t stream)
    {
        const std::size_t heap = _config.npol() * _config.nsamples_per_heap() * _config.nchans() *
                                 input_nantennas * 2;
        if(taftp.size() % heap != 0) throw std::runtime_error("Voltages are not a multiple of the heap size");
        if(input_nantennas > _config.nantennas())
            throw std::runtime_error("Input number of antennas must be <= to the maximum nantennas");
        const int nheaps = (int)(taftp.size() / heap);
        ftpa.resize((std::size_t)nheaps * 256 * _config.nchans() * 2 * _config.nantennas() * 2);
        check(sw_transpose_ftpa(taftp.data(), ftpa.data(), nheaps, (int)input_nantennas,
                                (int)_config.nantennas(), (int)_config.nchans(), (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "transpose");
    }

  private:
    const PipelineConfig& _config;
};

// -------------------------------------------------------- FTPA -> FPACT helper
inline void ftpa_to_fpact(const DeviceBuffer<int8_t>& ftpa, DeviceBuffer<int8_t>& fpact,
                          std::size_t nchans, std::size_t nsamples, std::size_t nant,
                          cudaStream_t stream)
{
    fpact.resize(nchans * 2 * nant * 2 * nsamples);
    check(sw_ftpa_to_fpact(ftpa.data(), fpact.data(), (int)nchans, (int)nsamples, (int)nant,
                           nsamples, 0, (sw_stream_t)stream));
}

// ------------------------------------------------------ StatisticsCalculator
// cpp/skyweaver/StatisticsCalculator.cuh:58-97 (statistics as float4
// {mean, std, skew, kurtosis} per (channel, pol, antenna))
class StatisticsCalculator {
  public:
    StatisticsCalculator(const PipelineConfig& config, cudaStream_t stream)
        : _config(config), _stream(stream)
    {
    }
    void calculate_statistics(const DeviceBuffer<int8_t>& ftpa)
    {
        const std::size_t F = _config.nchans(), A = _config.nantennas();
        const std::size_t T = ftpa.size() / (F * 2 * A * 2);
        ftpa_to_fpact(ftpa, _fpact, F, T, A, _stream);
        _stats.resize(F * 2 * A * 4);
        _scratch.resize(sw_statistics_scratch_bytes((int)F, 2, (int)A));
        check(sw_statistics(_fpact.data(), T, 0, (int)F, 2, (int)A, (int)T, _scratch.data(),
                            _stats.data(), (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "statistics");
    }
    void update_scalings(const std::vector<float>& beamset_weights, int nbeamsets)
    {
        const std::size_t F = _config.nchans();
        DeviceBuffer<float> bw;
        bw.upload(beamset_weights);
        for(auto* b : {&_cb_off, &_cb_scl, &_ib_off, &_ib_scl}) b->resize(F * nbeamsets);
        check(sw_update_scalings(_stats.data(), bw.data(), nbeamsets, (int)F, 2,
                                 (int)_config.nantennas(), (int)_config.cb_tscrunch(),
                                 (int)_config.ib_tscrunch(), _config.output_level(),
                                 _cb_off.data(), _cb_scl.data(), _ib_off.data(), _ib_scl.data(),
                                 (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "update_scalings");
    }
    const DeviceBuffer<float>& statistics() const { return _stats; }
    const DeviceBuffer<float>& cb_offsets() const { return _cb_off; }
    const DeviceBuffer<float>& cb_scaling() const { return _cb_scl; }
    const DeviceBuffer<float>& ib_offsets() const { return _ib_off; }
    const DeviceBuffer<float>& ib_scaling() const { return _ib_scl; }

  private:
    const PipelineConfig& _config;
    cudaStream_t _stream;
    DeviceBuffer<int8_t> _fpact;
    DeviceBuffer<uint8_t> _scratch;
    DeviceBuffer<float> _stats, _cb_off, _cb_scl, _ib_off, _ib_scl;
};

// ------------------------------------------------------- IncoherentBeamformer
// cpp/skyweaver/IncoherentBeamformer.cuh:84-91 (BTF raw float and int8)
class IncoherentBeamformer {
  public:
    explicit IncoherentBeamformer(const PipelineConfig& config) : _config(config) {}
    void beamform(const DeviceBuffer<int8_t>& ftpa, DeviceBuffer<float>& output_raw,
                  DeviceBuffer<int8_t>& output, const DeviceBuffer<float>& output_scale,
                  const DeviceBuffer<float>& output_offset, const DeviceBuffer<float>& antenna_weights,
                  int nbeamsets, cudaStream_t stream)
    {
        if(nbeamsets <= 0) throw std::runtime_error("Number of beamsets must be greater than zero");
        const std::size_t F = _config.nchans(), A = _config.nantennas(), ts = _config.ib_tscrunch();
        const std::size_t T = ftpa.size() / (F * 2 * A * 2);
        ftpa_to_fpact(ftpa, _fpact, F, T, A, stream);
        output_raw.resize(nbeamsets * (T / ts) * F * _config.stokes_components());
        output.resize(nbeamsets * (T / ts) * F * _config.stokes_components());
        check(sw_incoherent_beamform(_fpact.data(), T, 0, (int)F, (int)T, (int)A, (int)ts,
                                     output_scale.data(), output_offset.data(),
                                     antenna_weights.data(), nbeamsets, _config.stokes_index(),
                                     output_raw.data(), output.data(), (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "incoherent beamformer");
    }

  private:
    const PipelineConfig& _config;
    DeviceBuffer<int8_t> _fpact;
};

// --------------------------------------------------------- CoherentBeamformer
// cpp/skyweaver/CoherentBeamformer.cuh:84-92; weights are the reference
// [F][B][A] char2 vector (packed into the tensor-core layout here).
class CoherentBeamformer {
  public:
    explicit CoherentBeamformer(const PipelineConfig& config) : _config(config) {}
    void beamform(const DeviceBuffer<int8_t>& ftpa, const DeviceBuffer<int8_t>& weights,
                  const DeviceBuffer<float>& output_scale, const DeviceBuffer<float>& output_offset,
                  const DeviceBuffer<int>& beamset_mapping, const DeviceBuffer<float>& ib_powers,
                  DeviceBuffer<int8_t>& output, int nbeamsets, cudaStream_t stream)
    {
        const std::size_t F = _config.nchans(), A = _config.nantennas(), B = _config.nbeams();
        const std::size_t ts = _config.cb_tscrunch();
        if(output_scale.size() != F * nbeamsets)
            throw std::runtime_error("Unexpected number of channels in scaling vector");
        if(output_offset.size() != F * nbeamsets)
            throw std::runtime_error("Unexpected number of channels in offset vector ");
        if(beamset_mapping.size() != B) throw std::runtime_error("Unexpected size of beamset_mapping vector");
        if(weights.size() != F * B * A * 2) throw std::runtime_error("Unexpected size of weights vector");
        const std::size_t T = ftpa.size() / (F * 2 * A * 2);
        ftpa_to_fpact(ftpa, _fpact, F, T, A, stream);
        _gemm.resize(2 * weights.size());
        check(sw_pack_weights(weights.data(), _gemm.data(), (int)F, (int)B, (int)A, (sw_stream_t)stream));
        output.resize((T / ts) * F * B * _config.stokes_components());
        sw_cb_shape shape{(int)F, (int)T, (int)A, (int)B, (int)ts, _config.stokes_index(),
                          _config.ib_subtraction() ? 1 : 0, T, 0};
        sw_cb_problem prob{_fpact.data(), output.data(), ib_powers.data(), 0, (int)B};
        check(sw_coherent_beamform(&shape, &prob, _gemm.data(), output_scale.data(),
                                   output_offset.data(), beamset_mapping.data(), nullptr,
                                   (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "coherent beamformer");
    }

  private:
    const PipelineConfig& _config;
    DeviceBuffer<int8_t> _fpact, _gemm;
};

// ------------------------------------------------------ IncoherentDedisperser
// cpp/skyweaver/IncoherentDedisperser.cuh:14-28, src/IncoherentDedisperser.cu:36-125
class IncoherentDedisperser {
  public:
    IncoherentDedisperser(const PipelineConfig& config, const std::vector<float>& dms,
                          std::size_t tscrunch = 1)
        : _config(config), _dms(dms), _tscrunch(tscrunch)
    {
        const auto& freqs = config.channel_frequencies();
        const double chbw = config.bandwidth() / config.nchans();
        const double tsamp = config.cb_tscrunch() / chbw;
        _delays.resize(dms.size() * freqs.size());
        for(std::size_t d = 0; d < dms.size(); ++d)
            for(std::size_t f = 0; f < freqs.size(); ++f) {
                const double dly = 4.148806423e15 *
                                   (1 / (freqs.front() * freqs.front()) - 1 / (freqs[f] * freqs[f])) *
                                   (double)dms[d];
                _delays[d * freqs.size() + f] = (int)(dly / tsamp + 0.5);
            }
        _max = *std::max_element(_delays.begin(), _delays.end());
        _scale = (float)std::sqrt((double)(config.nchans() * _tscrunch));
        _d_delays.upload(_delays);
    }
    IncoherentDedisperser(const PipelineConfig& config, float dm, std::size_t tscrunch = 1)
        : IncoherentDedisperser(config, std::vector<float>(1, dm), tscrunch)
    {
    }
    const std::vector<int>& delays() const { return _delays; }
    int max_sample_delay() const { return _max; }
    float scale_factor() const { return _scale; }
    // int8 TFB [T][F][B] -> int8 TDB [(T - max_delay)/tscrunch][ndms][B]
    void dedisperse(const DeviceBuffer<int8_t>& tfb, DeviceBuffer<int8_t>& tdb, cudaStream_t stream = 0)
    {
        run(tfb, tdb, 1, stream);
    }
    // char4 (IQUV) TFB -> char4 TDB, each component dedispersed and clamped
    // independently like the reference's char4 instantiation
    // (IncoherentDedisperser.cu:133-137); buffers hold 4 int8 per sample
    void dedisperse_iquv(const DeviceBuffer<int8_t>& tfb, DeviceBuffer<int8_t>& tdb,
                         cudaStream_t stream = 0)
    {
        run(tfb, tdb, 4, stream);
    }

  private:
    void run(const DeviceBuffer<int8_t>& tfb, DeviceBuffer<int8_t>& tdb, std::size_t ncomp,
             cudaStream_t stream)
    {
        const std::size_t F = _config.nchans(), B = _config.nbeams() * ncomp;
        const std::size_t T = tfb.size() / (F * B);
        if(T <= (std::size_t)_max)
            throw std::runtime_error("Fewer than max_sample_delay samples passed to dedisperse method");
        if((T - _max) % _tscrunch != 0)
            throw std::runtime_error("(nsamples - max_sample_delay) must be a multiple of tscrunch;");
        tdb.resize((T - _max) / _tscrunch * _dms.size() * B);
        check(sw_incoherent_dedisperse(tfb.data(), (int)T, (int)F, (int)B, _d_delays.data(),
                                       (int)_dms.size(), _max, (int)_tscrunch, _scale, tdb.data(),
                                       (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "incoherent dedispersion");
    }

    const PipelineConfig& _config;
    std::vector<float> _dms;
    std::size_t _tscrunch;
    std::vector<int> _delays;
    DeviceBuffer<int> _d_delays;
    int _max = 0;
    float _scale = 1.0f;
};

// ------------------------------------------- IncoherentDedispersionPipeline
// IncoherentDedispersionPipeline<In, Out, Handler>
// (detail/IncoherentDedispersionPipeline.cu:6-113) with the AggregationBuffer
// in device memory.  One block per DedispersionPlan block (coherent DM); the
// handler is called as handler(d_tdb, nsamples_out, ndms, nbeams, ref_dm_idx)
// with the TDB result in device memory, ordered on the pushing stream.
template <typename Handler>
class IncoherentDedispersionPipeline {
  public:
    IncoherentDedispersionPipeline(const PipelineConfig& config, const DedispersionPlan& plan,
                                   Handler& handler)
        : _config(config), _handler(handler)
    {
        const auto& blocks = plan.blocks();
        const int ncomp = (int)config.stokes_components();
        std::vector<int> ndms, ts;
        std::vector<float> scale;
        std::vector<const int*> dptr;
        for(const auto& b : blocks) {
            _dedispersers.emplace_back(new IncoherentDedisperser(config, b.incoherent_dms,
                                                                 (std::size_t)b.tscrunch));
            ndms.push_back((int)b.incoherent_dms.size());
            ts.push_back(b.tscrunch);
            scale.push_back(_dedispersers.back()->scale_factor());
        }
        for(auto& d : _dedispersers) dptr.push_back(d->delays().data());
        check(sw_idd_pipeline_create((int)config.nchans(), (int)config.nbeams() * ncomp,
                                     (int)blocks.size(), ndms.data(), dptr.data(), ts.data(),
                                     scale.data(), nullptr, &trampoline, this, &_p));
    }
    ~IncoherentDedispersionPipeline() { sw_idd_pipeline_destroy(_p); }
    IncoherentDedispersionPipeline(const IncoherentDedispersionPipeline&) = delete;
    IncoherentDedispersionPipeline& operator=(const IncoherentDedispersionPipeline&) = delete;

    // operator()(data, ref_dm_idx): push nsamples of device TFB
    void operator()(const int8_t* d_tfb, std::size_t nsamples, std::size_t ref_dm_idx,
                    cudaStream_t stream = 0)
    {
        check(sw_idd_pipeline_push(_p, (int)ref_dm_idx, d_tfb, nsamples, (sw_stream_t)stream));
    }
    const IncoherentDedisperser& dedisperser(std::size_t i) const { return *_dedispersers[i]; }

  private:
    static void trampoline(void* user, int block, const int8_t* d_tdb, int nout, int ndms,
                           int nbeams, sw_stream_t)
    {
        auto* self = static_cast<IncoherentDedispersionPipeline*>(user);
        self->_handler(d_tdb, (std::size_t)nout, (std::size_t)ndms, (std::size_t)nbeams,
                       (std::size_t)block);
    }
    const PipelineConfig& _config;
    Handler& _handler;
    std::vector<std::unique_ptr<IncoherentDedisperser>> _dedispersers;
    sw_idd_pipeline* _p = nullptr;
};

// ------------------------------------------------------------- DADA I/O
// MultiFileReader (src/MultiFileReader.cu:34-303) over sw_dada_reader.
class MultiFileReader {
  public:
    MultiFileReader(const std::vector<std::string>& files, std::size_t header_size = 4096,
                    bool check_contiguity = false)
    {
        std::vector<const char*> names;
        for(const auto& f : files) names.push_back(f.c_str());
        check(sw_dada_reader_open(names.data(), (int)names.size(), header_size,
                                  check_contiguity ? 1 : 0, &_r));
    }
    ~MultiFileReader() { sw_dada_reader_close(_r); }
    MultiFileReader(const MultiFileReader&) = delete;
    MultiFileReader& operator=(const MultiFileReader&) = delete;
    sw_observation_header get_header(int file_idx = 0) const
    {
        sw_observation_header h{};
        check(sw_dada_reader_header(_r, file_idx, &h));
        return h;
    }
    std::size_t get_total_size() const { return sw_dada_reader_total_bytes(_r); }
    std::size_t tellg() const { return sw_dada_reader_tell(_r); }
    bool eof() const { return tellg() >= get_total_size(); }
    void seekg(std::size_t pos) { check(sw_dada_reader_seek(_r, pos)); }
    std::size_t read(char* dst, std::size_t bytes)
    {
        std::size_t got = 0;
        check(sw_dada_reader_read(_r, dst, bytes, &got));
        return got;
    }

  private:
    sw_dada_reader* _r = nullptr;
};

// MultiFileWriter (detail/MultiFileWriter.cu:74-243): one size-split DADA
// stream per stream index (coherent DM), the reference's directory and file
// names and header keys.  Data is host memory.
class MultiFileWriter {
  public:
    struct StreamInfo {
        std::size_t nbeams, nchans, nsamples, ndms;
        std::vector<float> dms;
        float reference_dm;
        double tsamp, utc_offset;
        std::string dims;  // "TFB", "TDB", ...
    };
    MultiFileWriter(const std::string& output_dir, const sw_observation_header& header,
                    std::size_t max_file_bytes, std::string stokes = "I", std::string prefix = "",
                    std::string tag = "")
        : _dir(output_dir), _h(header), _max(max_file_bytes), _stokes(std::move(stokes)),
          _prefix(std::move(prefix)), _tag(std::move(tag))
    {
    }
    ~MultiFileWriter()
    {
        for(auto& w : _w) sw_dada_writer_close(w.second);
    }
    void operator()(const int8_t* data, std::size_t bytes, const StreamInfo& s,
                    std::size_t stream_idx)
    {
        auto it = _w.find(stream_idx);
        if(it == _w.end()) it = _w.emplace(stream_idx, create(s, stream_idx, bytes)).first;
        check(sw_dada_writer_write(it->second, data, bytes));
    }

  private:
    static std::string utc(double t)
    {
        char b[80];
        std::time_t u = (std::time_t)t;
        std::strftime(b, sizeof(b), "%Y-%m-%d-%H:%M:%S", std::gmtime(&u));
        return b;
    }
    sw_dada_writer* create(const StreamInfo& s, std::size_t idx, std::size_t block_bytes)
    {
        std::ostringstream dir, base, dims;
        dir << _dir << "/" << utc(_h.utc_start) << "/" << idx << "/" << std::setfill('0')
            << std::setw(9) << (long long)_h.frequency;
        if(!_prefix.empty()) base << _prefix << "_";
        base << utc(_h.utc_start) << "_" << idx << "_" << std::fixed << std::setprecision(3)
             << std::setfill('0') << std::setw(9) << s.reference_dm << "_"
             << std::setprecision(0) << std::setw(9) << _h.frequency;
        if(!_tag.empty()) base << "_" << _tag;
        std::string ext = "." + s.dims;
        for(auto& c : ext) c = (char)std::tolower((unsigned char)c);
        // file size rounded to a whole number of blocks (MultiFileWriter.cu:103-108)
        const std::size_t filesize = std::max<std::size_t>(1, _max / block_bytes) * block_bytes;
        sw_dada_writer* w = nullptr;
        check(sw_dada_writer_open(dir.str().c_str(), base.str().c_str(), ext.c_str(), filesize,
                                  nullptr, 4096, &w));
        auto set = [&](const char* k, const std::string& v) { check(sw_dada_writer_set(w, k, v.c_str())); };
        auto num = [](double v, int prec) {
            std::ostringstream o;
            o << std::fixed << std::setprecision(prec) << v;
            return o.str();
        };
        set("NBEAM", std::to_string(s.nbeams));
        set("NCHAN", std::to_string(s.nchans));
        set("OBS_NCHAN", std::to_string(_h.obs_nchans));
        set("OBS_FREQUENCY", num(_h.obs_frequency, 6));
        set("OBS_BW", num(_h.obs_bandwidth, 6));
        set("NSAMP", std::to_string(s.nsamples));
        if(s.ndms) {
            set("NDMS", std::to_string(s.ndms));
            std::ostringstream d;
            d << std::setprecision(7);
            for(std::size_t i = 0; i < s.dms.size(); ++i) d << (i ? "," : "") << s.dms[i];
            set("DMS", d.str());
        }
        set("COHERENT_DM", num(s.reference_dm, 6));
        set("FREQ", num(_h.frequency, 6));
        set("BW", num(_h.bandwidth, 6));
        set("TSAMP", num(s.tsamp * 1e6, 6));
        set("NPOL", _stokes == "IQUV" ? "4" : "1");
        set("STOKES_MODE", _stokes);
        set("ORDER", s.dims);
        set("CHAN0_IDX", std::to_string(_h.chan0_idx));
        set("OBS_OVERLAP", "0");
        set("UTC_START", num(_h.utc_start + s.utc_offset, 6));
        return w;
    }
    std::string _dir;
    sw_observation_header _h;
    std::size_t _max;
    std::string _stokes, _prefix, _tag;
    std::map<std::size_t, sw_dada_writer*> _w;
};

// -------------------------------------------------------- BeamformerPipeline
// cpp/skyweaver/BeamformerPipeline.cuh:48-67.  Handlers get host copies:
// cb_handler(const int8_t* tfb, std::size_t bytes, std::size_t dm_idx).
template <typename CBHandler>
class BeamformerPipeline {
  public:
    BeamformerPipeline(const PipelineConfig& config, CBHandler& cb_handler, std::size_t input_nantennas)
        : _config(config), _cb(cb_handler), _delays(config, nullptr)
    {
        if(config.coherent_dms().empty()) throw std::runtime_error("No DDPlan set for pipeline");
        sw_pipeline_config c{};
        c.nantennas       = (int)config.nantennas();
        c.input_nantennas = (int)input_nantennas;
        c.nchans          = (int)config.nchans();
        c.nbeams          = (int)config.nbeams();
        c.gulp_samples    = (int)config.gulp_length_samps();
        c.tscrunch        = (int)config.cb_tscrunch();
        c.stokes          = config.stokes_index();
        c.ib_subtract     = config.ib_subtraction() ? 1 : 0;
        c.output_level    = config.output_level();
        c.centre_frequency = config.centre_frequency();
        c.bandwidth       = config.bandwidth();
        c.ndms            = (int)config.coherent_dms().size();
        c.dms             = config.coherent_dms().data();
        c.enable_coherent_dedispersion = 1;
        c.grouped = 1;
        c.use_graph = 1;
        c.nbeamsets       = _delays.nbeamsets();
        c.beamset_weights = _delays.beamset_weights().data();
        c.beamset_mapping = _delays.beamset_mapping().data();
        c.autotune        = config.autotune() ? 1 : 0;
        check(sw_pipeline_create(&c, &_p));
        _out.resize(sw_pipeline_cb_bytes_per_dm(_p) * c.ndms);
    }
    ~BeamformerPipeline() { sw_pipeline_destroy(_p); }

    // The description of one coherent DM's beams, as the reference's CB
    // handler finds it on its TFBPowersD (CoherentBeamformer.cu:231-235,
    // CoherentDedisperser.cu:224, detail/BeamformerPipeline.cu:191-193):
    // TFB (element char4 for IQUV), tsamp = cb_tscrunch x channel sample,
    // utc_offset = the dedisperser's filter delay, reference_dm = the DM.
    Description describe_cb(std::size_t dm_idx) const
    {
        Description d = describe_base(dm_idx);
        d.dims  = "TFB";
        d.sizes = {_config.gulp_length_samps() / _config.cb_tscrunch(), _config.nchans(),
                   _config.nbeams()};
        d.sample_period *= (double)_config.cb_tscrunch();
        return d;
    }
    // The incoherent beam of the same DM: BTF over beamsets (float raw power
    // and int8), tsamp = ib_tscrunch x channel sample.
    Description describe_ib(std::size_t dm_idx) const
    {
        Description d = describe_base(dm_idx);
        d.dims  = "BTF";
        d.sizes = {(std::size_t)_delays.nbeamsets(),
                   _config.gulp_length_samps() / _config.ib_tscrunch(), _config.nchans()};
        d.sample_period *= (double)_config.ib_tscrunch();
        return d;
    }
    // one gulp of TAFTP voltages already in device memory; each DM's
    // coherent beams stay on the device and go to
    // handler(d_tfb, nsamples, dm_idx, stream), ordered on `stream` (the
    // call signature of IncoherentDedispersionPipeline, which makes the
    // reference's CB handler -> incoherent dedispersion chain device-resident)
    template <typename DeviceHandler>
    void process_device(const void* d_taftp, double epoch, DeviceHandler& handler,
                        cudaStream_t stream = 0)
    {
        const auto& d = _delays.delays(epoch);
        check(sw_pipeline_set_delays(_p, d.download().data(), _delays.epoch()));
        check(sw_pipeline_process_device(_p, d_taftp, epoch, (sw_stream_t)stream));
        const std::size_t nsamp = _config.gulp_length_samps() / _config.cb_tscrunch();
        for(std::size_t dm = 0; dm < _config.coherent_dms().size(); ++dm) {
            const int8_t* cb = nullptr;
            check(sw_pipeline_outputs(_p, (int)dm, &cb, nullptr, nullptr, nullptr));
            handler(cb, nsamp, dm, stream);
        }
    }
    // one gulp of pinned TAFTP voltages; epoch = UNIX time of the gulp start
    void operator()(const void* h_taftp, double epoch)
    {
        const auto& d = _delays.delays(epoch);
        check(sw_pipeline_set_delays(_p, d.download().data(), _delays.epoch()));
        check(sw_pipeline_process_host(_p, h_taftp, epoch, _out.data(), nullptr));
        cuda_check(cudaDeviceSynchronize(), "pipeline");
        const std::size_t per_dm = sw_pipeline_cb_bytes_per_dm(_p);
        for(std::size_t dm = 0; dm < _config.coherent_dms().size(); ++dm)
            _cb(_out.data() + dm * per_dm, per_dm, dm);
    }

  private:
    Description describe_base(std::size_t dm_idx) const
    {
        if(dm_idx >= _config.coherent_dms().size())
            throw std::runtime_error("BeamformerPipeline: DM index out of range");
        int fft_len = 0, overlap = 0, lag = 0;
        check(sw_pipeline_fft_len(_p, &fft_len, &overlap, &lag));
        const double chan_tsamp = (double)_config.nchans() / _config.bandwidth();
        Description d;
        d.freqs         = _config.channel_frequencies();
        d.sample_period = chan_tsamp;
        // the filter delay (CoherentDedisperser.cu:82 sets tsamp * overlap / 2
        // for its symmetric trim): the samples trimmed at each window's end
        d.offset        = chan_tsamp * lag;
        d.coherent_dm   = _config.coherent_dms()[dm_idx];
        return d;
    }

    const PipelineConfig& _config;
    CBHandler& _cb;
    DelayManager _delays;
    sw_pipeline* _p = nullptr;
    std::vector<int8_t> _out;
};

}  // namespace skyweaver_b200
