// skyweaver_b200.hpp -- C++ drop-in layer over the C ABI in skyweaver_b200.h.
//
// Mirrors the reference's C++ API (erc-compact/skyweaver, cpp/skyweaver/*)
// for the beamforming hot path: the same class, type and method names, the
// same argument meaning and std::runtime_error on the same errors.  The
// reference's thrust containers are replaced by DeviceVector (cudaMalloc,
// RAII) and PinnedVector (cudaMallocHost) inside the same DescribedVector
// template, with the same aliases (TAFTPVoltagesH, FTPAVoltagesD,
// TFBPowersD, ...) and metadata getters.
//
// Header only; link with -lskyweaver_b200 -lcudart.
#pragma once

#include <cuda_runtime.h>
#include <vector_types.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <fstream>
#include <initializer_list>
#include <iomanip>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
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

// ---------------------------------------------------------------- containers
// Device memory, owned (cudaMalloc) or a view of memory another object owns
// (the pipeline hands its output buffers to handlers as views).
template <typename T>
class DeviceVector {
  public:
    using value_type = T;
    DeviceVector() = default;
    explicit DeviceVector(std::size_t n) { resize(n); }
    DeviceVector(const DeviceVector&) = delete;
    DeviceVector& operator=(const DeviceVector&) = delete;
    DeviceVector(DeviceVector&& o) noexcept : _p(o._p), _n(o._n), _own(o._own)
    {
        o._p = nullptr;
        o._n = 0;
    }
    DeviceVector& operator=(DeviceVector&& o) noexcept
    {
        if(this != &o) {
            release();
            _p = o._p, _n = o._n, _own = o._own;
            o._p = nullptr, o._n = 0;
        }
        return *this;
    }
    ~DeviceVector() { release(); }
    static DeviceVector view(T* p, std::size_t n)
    {
        DeviceVector v;
        v._p = p, v._n = n, v._own = false;
        return v;
    }
    void resize(std::size_t n)
    {
        if(n == _n) return;
        if(!_own) throw std::runtime_error("DeviceVector: a view cannot be resized");
        release();
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
    void release()
    {
        if(_p && _own) cudaFree(_p);
        _p = nullptr;
        _n = 0;
        _own = true;
    }
    T* _p = nullptr;
    std::size_t _n = 0;
    bool _own = true;
};

// the earlier name of DeviceVector
template <typename T>
using DeviceBuffer = DeviceVector<T>;

// Pinned host memory (the reference's PinnedAllocator host vectors,
// DescribedVector.hpp:588-592): the pipeline's H2D copies run from it.
template <typename T>
class PinnedVector {
  public:
    using value_type = T;
    PinnedVector() = default;
    explicit PinnedVector(std::size_t n) { resize(n); }
    PinnedVector(const PinnedVector&) = delete;
    PinnedVector& operator=(const PinnedVector&) = delete;
    PinnedVector(PinnedVector&& o) noexcept : _p(o._p), _n(o._n) { o._p = nullptr, o._n = 0; }
    ~PinnedVector()
    {
        if(_p) cudaFreeHost(_p);
    }
    void resize(std::size_t n)
    {
        if(n == _n) return;
        T* p = nullptr;
        if(n) cuda_check(cudaMallocHost(reinterpret_cast<void**>(&p), n * sizeof(T)), "cudaMallocHost");
        if(_p) {
            std::memcpy(p, _p, std::min(n, _n) * sizeof(T));
            cudaFreeHost(_p);
        }
        _p = p;
        _n = n;
    }
    T* data() { return _p; }
    const T* data() const { return _p; }
    std::size_t size() const { return _n; }
    T& operator[](std::size_t i) { return _p[i]; }
    const T& operator[](std::size_t i) const { return _p[i]; }
    T* begin() { return _p; }
    T* end() { return _p + _n; }
    const T* begin() const { return _p; }
    const T* end() const { return _p + _n; }

  private:
    T* _p = nullptr;
    std::size_t _n = 0;
};

// ----------------------------------------------------------- DescribedVector
// cpp/skyweaver/DescribedVector.hpp:46-573: a vector with named dimensions
// and the metadata that travels with the data through the pipeline.
enum Dimension { TimeDim, FreqDim, BeamDim, AntennaDim, PolnDim, DispersionDim };

inline std::string dimensions_to_string(const std::vector<Dimension>& dims)
{
    static const char names[] = {'T', 'F', 'B', 'A', 'P', 'D'};
    std::string s;
    for(Dimension d : dims) s += names[d];
    return s;
}

template <typename VectorType_, Dimension... dims>
class DescribedVector {
  public:
    using VectorType             = VectorType_;
    using value_type             = typename VectorType::value_type;
    using FrequenciesType        = std::vector<double>;
    using DispersionMeasuresType = std::vector<float>;

    DescribedVector() : _dims{dims...} {}
    DescribedVector(std::initializer_list<std::size_t> sizes) : _dims{dims...}
    {
        resize(std::vector<std::size_t>(sizes));
    }
    // a vector over memory another object owns (device vectors only)
    static DescribedVector view(value_type* p, std::vector<std::size_t> const& sizes)
    {
        DescribedVector v;
        v.check_sizes(sizes);
        v._sizes  = sizes;
        v._vector = VectorType::view(p, v.calculate_nelements());
        return v;
    }
    void resize(std::initializer_list<std::size_t> sizes) { resize(std::vector<std::size_t>(sizes)); }
    void resize(std::vector<std::size_t> const& sizes)
    {
        check_sizes(sizes);
        _sizes = sizes;
        _vector.resize(calculate_nelements());
    }
    template <typename Other>
    void like(const Other& other)
    {
        resize(other.extents());
        metalike(other);
    }
    template <typename Other>
    void metalike(const Other& other)
    {
        _frequencies       = other._frequencies;
        _frequencies_stale = other._frequencies_stale;
        _dms               = other._dms;
        _dms_stale         = other._dms_stale;
        _tsamp             = other._tsamp;
        _utc_offset        = other._utc_offset;
        _reference_dm      = other._reference_dm;
    }
    std::size_t size() const { return _vector.size(); }
    value_type* data() { return _vector.data(); }
    const value_type* data() const { return _vector.data(); }
    VectorType& vector() { return _vector; }
    const VectorType& vector() const { return _vector; }
    std::size_t calculate_nelements() const
    {
        std::size_t n = 1;
        for(std::size_t s : _sizes) n *= s;
        return _sizes.empty() ? 0 : n;
    }
    template <Dimension dim>
    std::size_t get_dim_extent() const
    {
        std::size_t n = 1;
        for(std::size_t i = 0; i < _dims.size() && i < _sizes.size(); ++i)
            if(_dims[i] == dim) n *= _sizes[i];
        return n;
    }
    FrequenciesType const& frequencies() const
    {
        if(_frequencies_stale)
            throw std::runtime_error("Frequencies must be explicitly set before they can be used");
        return _frequencies;
    }
    void frequencies(FrequenciesType const& freqs)
    {
        if(freqs.size() != get_dim_extent<FreqDim>())
            throw std::runtime_error("Invalid number of frequecies passed.");
        _frequencies = freqs;
        _frequencies_stale = false;
    }
    void frequencies(double freq)
    {
        if(get_dim_extent<FreqDim>() != 1)
            throw std::runtime_error("Invalid number of frequecies passed.");
        _frequencies.assign(1, freq);
        _frequencies_stale = false;
    }
    std::size_t nchannels() const { return get_dim_extent<FreqDim>(); }
    std::size_t nantennas() const { return get_dim_extent<AntennaDim>(); }
    std::size_t nsamples() const { return get_dim_extent<TimeDim>(); }
    std::size_t nbeams() const { return get_dim_extent<BeamDim>(); }
    std::size_t npol() const { return get_dim_extent<PolnDim>(); }
    std::size_t ndms() const { return get_dim_extent<DispersionDim>(); }
    void tsamp(double t) { _tsamp = t; }
    double tsamp() const { return _tsamp; }
    double utc_offset() const { return _utc_offset; }
    void utc_offset(double o) { _utc_offset = o; }
    std::vector<std::size_t> const& extents() const { return _sizes; }
    DispersionMeasuresType const& dms() const
    {
        if(_dms_stale) throw std::runtime_error("Dms must be explicitly set before they can be used");
        return _dms;
    }
    void dms(DispersionMeasuresType const& d)
    {
        if(d.size() != get_dim_extent<DispersionDim>())
            throw std::runtime_error("Invalid number of dispersion measures passed.");
        _dms = d;
        _dms_stale = false;
    }
    void dms(float dm)
    {
        if(get_dim_extent<DispersionDim>() != 1)
            throw std::runtime_error("Invalid number of dispersion measures passed.");
        _dms.assign(1, dm);
        _dms_stale = false;
    }
    void reference_dm(float dm) { _reference_dm = dm; }
    float reference_dm() const { return _reference_dm; }
    std::string dims_as_string() const { return dimensions_to_string(_dims); }
    std::string describe() const
    {
        std::ostringstream os;
        os << "DescribedVector: " << dims_as_string() << " (" << size() << " elements)\n";
        os << "  dimensions:";
        for(std::size_t s : _sizes) os << " " << s;
        os << "\n  nsamples: " << nsamples() << "\n  nchans: " << nchannels()
           << "\n  nantennas: " << nantennas() << "\n  nbeams: " << nbeams()
           << "\n  ndms: " << ndms() << "\n  npol: " << npol() << std::setprecision(15)
           << "\n  frequencies (Hz):";
        for(double f : _frequencies) os << " " << f;
        os << "\n  DMs (pc cm^-3):";
        for(float d : _dms) os << " " << d;
        os << "\n  Coherent DM (pc cm^-3): " << _reference_dm << "\n  Time resolution (s): "
           << _tsamp << "\n  Time offset (s): " << _utc_offset << "\n";
        return os.str();
    }

    // metadata (public for metalike across container types, as in the reference)
    FrequenciesType _frequencies;
    bool _frequencies_stale = true;
    DispersionMeasuresType _dms;
    bool _dms_stale = true;
    double _tsamp = 0.0, _utc_offset = 0.0;
    float _reference_dm = 0.0f;

  private:
    void check_sizes(std::vector<std::size_t> const& sizes) const
    {
        if(sizes.size() != sizeof...(dims))
            throw std::invalid_argument("Number of sizes must match number of dimensions");
    }
    std::vector<std::size_t> _sizes;
    std::vector<Dimension> _dims;
    VectorType _vector;
};

// Copy between host and device described vectors (the reference's implicit
// thrust copies): resizes `dst` like `src`, copies data and metadata.
template <typename Dst, typename Src>
void copy(const Src& src, Dst& dst, cudaStream_t stream = 0)
{
    static_assert(sizeof(typename Dst::value_type) == sizeof(typename Src::value_type),
                  "copy: element types differ");
    dst.like(src);
    cuda_check(cudaMemcpyAsync(dst.data(), src.data(), src.size() * sizeof(typename Src::value_type),
                               cudaMemcpyDefault, stream),
               "copy");
    cuda_check(cudaStreamSynchronize(stream), "copy");
}

// DescribedVector.hpp:594-668
template <typename T>
using TAFTPVoltagesH = DescribedVector<PinnedVector<T>, TimeDim, AntennaDim, FreqDim, TimeDim, PolnDim>;
template <typename T>
using TAFTPVoltagesD = DescribedVector<DeviceVector<T>, TimeDim, AntennaDim, FreqDim, TimeDim, PolnDim>;
template <typename T>
using FTPAVoltagesH = DescribedVector<PinnedVector<T>, FreqDim, TimeDim, PolnDim, AntennaDim>;
template <typename T>
using FTPAVoltagesD = DescribedVector<DeviceVector<T>, FreqDim, TimeDim, PolnDim, AntennaDim>;
template <typename T>
using TPAVoltagesH = DescribedVector<PinnedVector<T>, TimeDim, PolnDim, AntennaDim>;
template <typename T>
using TPAVoltagesD = DescribedVector<DeviceVector<T>, TimeDim, PolnDim, AntennaDim>;
template <typename T>
using TFBPowersH = DescribedVector<PinnedVector<T>, TimeDim, FreqDim, BeamDim>;
template <typename T>
using TFBPowersD = DescribedVector<DeviceVector<T>, TimeDim, FreqDim, BeamDim>;
template <typename T>
using BTFPowersH = DescribedVector<PinnedVector<T>, BeamDim, TimeDim, FreqDim>;
template <typename T>
using BTFPowersD = DescribedVector<DeviceVector<T>, BeamDim, TimeDim, FreqDim>;
template <typename T>
using TDBPowersH = DescribedVector<PinnedVector<T>, TimeDim, DispersionDim, BeamDim>;
template <typename T>
using TDBPowersD = DescribedVector<DeviceVector<T>, TimeDim, DispersionDim, BeamDim>;
template <typename T>
using FPAStatsH = DescribedVector<PinnedVector<T>, FreqDim, PolnDim, AntennaDim>;
template <typename T>
using FPAStatsD = DescribedVector<DeviceVector<T>, FreqDim, PolnDim, AntennaDim>;

// StatisticsCalculator.cuh:14-19
struct Statistics {
    float mean = 0.0f, std = 0.0f, skew = 0.0f, kurtosis = 0.0f;
};

// beamformer_utils.cuh:108,142-278: the output types of each Stokes mode
enum StokesParameter { I, Q, U, V };
template <StokesParameter Stokes>
struct SingleStokesBeamformerTraits {
    typedef int8_t QuantisedPowerType;
    typedef float RawPowerType;
    static constexpr int stokes_index = (int)Stokes;
};
struct FullStokesBeamformerTraits {
    typedef char4 QuantisedPowerType;
    typedef float4 RawPowerType;
    static constexpr int stokes_index = SW_STOKES_IQUV;
};

// ObservationHeader.hpp:9-34
using ObservationHeader = sw_observation_header;

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
    std::size_t _total_nchans = 4096, _cdd_fft = 0;
    int _cdd_lag = 0;

  public:
    // let sw_autotune pick the FFT length and beamformer work-item size
    bool autotune() const { return _autotune; }
    void autotune(bool on) { _autotune = on; }
    // channels of the whole band (PipelineConfig.cpp:245-253, default 4096):
    // with the header's sample clock it sets each gulp's epoch
    std::size_t total_nchans() const { return _total_nchans; }
    void total_nchans(std::size_t n) { _total_nchans = n; }
    // the pipeline's overlap-save plan (no counterpart: the reference ties the
    // FFT length to the gulp and sizes the overlap by the whole subband's DM
    // delay): 0 = automatic (sw_cdd_plan)
    std::size_t cdd_fft_length() const { return _cdd_fft; }
    void cdd_fft_length(std::size_t n) { _cdd_fft = n; }
    int cdd_lag() const { return _cdd_lag; }
    void cdd_lag(int lag) { _cdd_lag = lag; }

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
    using DelayVectorTypeD          = DeviceVector<float3>;
    using BeamsetWeightsVectorTypeD = DeviceVector<float>;
    using BeamsetMappingVectorTypeD = DeviceVector<int>;
    // float3 [nbeams][nantennas] on the device, zero padded to the config.
    // Uploaded only when the epoch moves to another model (the reference
    // copies on every call, DelayManager.cu:56-99).
    const DelayVectorTypeD& delays(double epoch)
    {
        if(epoch < _hdr.start_epoch) throw InvalidDelayEpoch(epoch);
        while(!validate_model(epoch)) read_next_model();
        if(_hdr.nantennas > _config.nantennas())
            throw std::runtime_error("Delay model contains too many antennas");
        if(_hdr.nbeams > _config.nbeams()) throw std::runtime_error("Delay model contains too many beams");
        if(_uploaded != _model) {
            std::vector<float3> padded(_config.nbeams() * _config.nantennas(), float3{0, 0, 0});
            for(uint32_t b = 0; b < _hdr.nbeams; ++b)
                std::memcpy(&padded[b * _config.nantennas()], &_h[3 * (b * _hdr.nantennas)],
                            3 * sizeof(float) * _hdr.nantennas);
            _d.upload(padded);
            _uploaded = _model;
        }
        return _d;
    }
    double epoch() const { return _hdr.start_epoch; }
    // the number of delay models read so far: changes when delays() moves on
    std::size_t model_index() const { return _model; }
    const BeamsetWeightsVectorTypeD& beamset_weights() const { return _d_bs_weights; }
    const BeamsetMappingVectorTypeD& beamset_mapping() const { return _d_bs_map; }
    // the same, on the host
    const std::vector<float>& beamset_weights_host() const { return _bs_weights; }
    const std::vector<int>& beamset_mapping_host() const { return _bs_map; }
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
        ++_model;
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
        _d_bs_weights.upload(_bs_weights);
        _d_bs_map.upload(_bs_map);
    }

    const PipelineConfig& _config;
    cudaStream_t _stream;
    std::ifstream _in;
    DelayModelHeader _hdr{};
    std::vector<float> _h;
    DelayVectorTypeD _d;
    BeamsetWeightsVectorTypeD _d_bs_weights;
    BeamsetMappingVectorTypeD _d_bs_map;
    std::size_t _model = 0, _uploaded = 0;
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
    using DelayVectorTypeD   = DeviceVector<float3>;
    using WeightsVectorTypeD = DeviceVector<char2>;
    WeightsManager(const PipelineConfig& config, cudaStream_t stream) : _config(config), _stream(stream)
    {
        const std::size_t n = config.nchans() * config.nbeams() * config.nantennas();
        _w.resize(n);
        _gemm.resize(4 * n);
        _freqs.upload(config.channel_frequencies());
    }
    // not thread safe: returns the internal buffer (WeightsManager.cuh:58-59)
    const WeightsVectorTypeD& weights(const DelayVectorTypeD& delays, double current_epoch,
                                      double delay_epoch)
    {
        check(sw_generate_weights(reinterpret_cast<const float*>(delays.data()), _freqs.data(),
                                  (int)_config.nantennas(), (int)_config.nbeams(),
                                  (int)_config.nchans(), current_epoch, delay_epoch, _w.data(),
                                  _gemm.data(), (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "weights");
        return _w;
    }
    // the same weights in the tensor-core layout (sw_pack_weights)
    const DeviceVector<int8_t>& gemm_weights() const { return _gemm; }

  private:
    const PipelineConfig& _config;
    cudaStream_t _stream;
    WeightsVectorTypeD _w;
    DeviceVector<int8_t> _gemm;
    DeviceVector<double> _freqs;
};

// FTPA <-> FPACT (the B200 planar layout the kernels read)
inline void ftpa_to_fpact(const char2* ftpa, DeviceVector<int8_t>& fpact, std::size_t nchans,
                          std::size_t nsamples, std::size_t nant, cudaStream_t stream)
{
    fpact.resize(nchans * 2 * nant * 2 * nsamples);
    check(sw_ftpa_to_fpact(ftpa, fpact.data(), (int)nchans, (int)nsamples, (int)nant, nsamples, 0,
                           (sw_stream_t)stream));
}

// ---------------------------------------------------------------- Transposer
// cpp/skyweaver/Transposer.cuh:54-69: TAFTP -> FTPA (antennas zero padded)
class Transposer {
  public:
    explicit Transposer(const PipelineConfig& config) : _config(config) {}
    void transpose(const TAFTPVoltagesD<char2>& taftp, FTPAVoltagesD<char2>& ftpa,
                   std::size_t input_nantennas, cudaStream_t stream)
    {
        const std::size_t heap = _config.npol() * _config.nsamples_per_heap() * _config.nchans() *
                                 input_nantennas;
        if(taftp.size() % heap != 0) throw std::runtime_error("Voltages are not a multiple of the heap size");
        if(input_nantennas > _config.nantennas())
            throw std::runtime_error("Input number of antennas must be <= to the maximum nantennas");
        const std::size_t nheaps = taftp.size() / heap;
        ftpa.resize({_config.nchans(), nheaps * 256, _config.npol(), _config.nantennas()});
        ftpa.metalike(taftp);
        check(sw_transpose_ftpa(taftp.data(), ftpa.data(), (int)nheaps, (int)input_nantennas,
                                (int)_config.nantennas(), (int)_config.nchans(), (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "transpose");
    }

  private:
    const PipelineConfig& _config;
};

// ------------------------------------------------------ StatisticsCalculator
// cpp/skyweaver/StatisticsCalculator.cuh:58-97
class StatisticsCalculator {
  public:
    using StatisticsVectorTypeD = FPAStatsD<Statistics>;
    using ScalingVectorTypeD    = DeviceVector<float>;
    StatisticsCalculator(const PipelineConfig& config, cudaStream_t stream)
        : _config(config), _stream(stream)
    {
    }
    void calculate_statistics(const FTPAVoltagesD<char2>& ftpa)
    {
        const std::size_t F = _config.nchans(), A = _config.nantennas();
        const std::size_t T = ftpa.size() / (F * 2 * A);
        ftpa_to_fpact(ftpa.data(), _fpact, F, T, A, _stream);
        _stats.resize({F, 2, A});
        _stats.metalike(ftpa);
        _scratch.resize(sw_statistics_scratch_bytes((int)F, 2, (int)A));
        check(sw_statistics(_fpact.data(), T, 0, (int)F, 2, (int)A, (int)T, _scratch.data(),
                            reinterpret_cast<float*>(_stats.data()), (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "statistics");
    }
    void update_scalings(const std::vector<float>& beamset_weights, int nbeamsets)
    {
        DeviceVector<float> bw;
        bw.upload(beamset_weights);
        update_scalings(bw, nbeamsets);
    }
    void update_scalings(const DeviceVector<float>& beamset_weights, int nbeamsets)
    {
        const std::size_t F = _config.nchans();
        if(beamset_weights.size() != (std::size_t)nbeamsets * _config.nantennas())
            throw std::runtime_error("Unexpected size of beamset weights vector");
        for(auto* b : {&_cb_off, &_cb_scl, &_ib_off, &_ib_scl}) b->resize(F * nbeamsets);
        check(sw_update_scalings(reinterpret_cast<const float*>(_stats.data()),
                                 beamset_weights.data(), nbeamsets, (int)F, 2,
                                 (int)_config.nantennas(), (int)_config.cb_tscrunch(),
                                 (int)_config.ib_tscrunch(), _config.output_level(),
                                 _cb_off.data(), _cb_scl.data(), _ib_off.data(), _ib_scl.data(),
                                 (sw_stream_t)_stream));
        cuda_check(cudaStreamSynchronize(_stream), "update_scalings");
    }
    const StatisticsVectorTypeD& statistics() const { return _stats; }
    const ScalingVectorTypeD& cb_offsets() const { return _cb_off; }
    const ScalingVectorTypeD& cb_scaling() const { return _cb_scl; }
    const ScalingVectorTypeD& ib_offsets() const { return _ib_off; }
    const ScalingVectorTypeD& ib_scaling() const { return _ib_scl; }

  private:
    const PipelineConfig& _config;
    cudaStream_t _stream;
    DeviceVector<int8_t> _fpact;
    DeviceVector<uint8_t> _scratch;
    StatisticsVectorTypeD _stats;
    ScalingVectorTypeD _cb_off, _cb_scl, _ib_off, _ib_scl;
};

// ------------------------------------------------------- IncoherentBeamformer
// cpp/skyweaver/IncoherentBeamformer.cuh:84-91: BTF raw power and quantised
// power per beamset, with per-beamset antenna weights (the reference's CPU
// implementation, IncoherentBeamformerTester.cu:68-70)
template <typename BfTraits>
class IncoherentBeamformer {
  public:
    using VoltageVectorTypeD  = FTPAVoltagesD<char2>;
    using RawPowerVectorTypeD = BTFPowersD<typename BfTraits::RawPowerType>;
    using PowerVectorTypeD    = BTFPowersD<typename BfTraits::QuantisedPowerType>;
    using ScalingVectorTypeD  = DeviceVector<float>;
    explicit IncoherentBeamformer(const PipelineConfig& config) : _config(config) {}
    void beamform(const VoltageVectorTypeD& input, RawPowerVectorTypeD& output_raw,
                  PowerVectorTypeD& output, const ScalingVectorTypeD& output_scale,
                  const ScalingVectorTypeD& output_offset, const ScalingVectorTypeD& antenna_weights,
                  int nbeamsets, cudaStream_t stream)
    {
        if(nbeamsets <= 0) throw std::runtime_error("Number of beamsets must be greater than zero");
        const std::size_t F = _config.nchans(), A = _config.nantennas(), ts = _config.ib_tscrunch();
        const std::size_t T = input.size() / (F * 2 * A);
        if(output_scale.size() != F * nbeamsets || output_offset.size() != F * nbeamsets)
            throw std::runtime_error("Unexpected number of channels in scaling vector");
        if(antenna_weights.size() != A * nbeamsets)
            throw std::runtime_error("Unexpected size of antenna weights vector");
        ftpa_to_fpact(input.data(), _fpact, F, T, A, stream);
        output_raw.resize({(std::size_t)nbeamsets, T / ts, F});
        output.resize({(std::size_t)nbeamsets, T / ts, F});
        output_raw.metalike(input);
        output.metalike(input);
        output_raw.tsamp(input.tsamp() * ts);
        output.tsamp(input.tsamp() * ts);
        check(sw_incoherent_beamform(_fpact.data(), T, 0, (int)F, (int)T, (int)A, (int)ts,
                                     output_scale.data(), output_offset.data(),
                                     antenna_weights.data(), nbeamsets, BfTraits::stokes_index,
                                     reinterpret_cast<float*>(output_raw.data()),
                                     reinterpret_cast<int8_t*>(output.data()), (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "incoherent beamformer");
    }

  private:
    const PipelineConfig& _config;
    DeviceVector<int8_t> _fpact;
};

// --------------------------------------------------------- CoherentBeamformer
// cpp/skyweaver/CoherentBeamformer.cuh:84-92; weights are the reference
// [F][B][A] char2 vector (packed into the tensor-core layout here).
template <typename BfTraits>
class CoherentBeamformer {
  public:
    using VoltageVectorTypeD  = FTPAVoltagesD<char2>;
    using WeightsVectorTypeD  = DeviceVector<char2>;
    using ScalingVectorTypeD  = DeviceVector<float>;
    using MappingVectorTypeD  = DeviceVector<int>;
    using RawPowerVectorTypeD = BTFPowersD<typename BfTraits::RawPowerType>;
    using PowerVectorTypeD    = TFBPowersD<typename BfTraits::QuantisedPowerType>;
    explicit CoherentBeamformer(const PipelineConfig& config) : _config(config) {}
    void beamform(const VoltageVectorTypeD& input, const WeightsVectorTypeD& weights,
                  const ScalingVectorTypeD& scales, const ScalingVectorTypeD& offsets,
                  const MappingVectorTypeD& beamset_mapping, const RawPowerVectorTypeD& ib_powers,
                  PowerVectorTypeD& output, int nbeamsets, cudaStream_t stream)
    {
        const std::size_t F = _config.nchans(), A = _config.nantennas(), B = _config.nbeams();
        const std::size_t ts = _config.cb_tscrunch();
        if(scales.size() != F * nbeamsets)
            throw std::runtime_error("Unexpected number of channels in scaling vector");
        if(offsets.size() != F * nbeamsets)
            throw std::runtime_error("Unexpected number of channels in offset vector ");
        if(beamset_mapping.size() != B) throw std::runtime_error("Unexpected size of beamset_mapping vector");
        if(weights.size() != F * B * A) throw std::runtime_error("Unexpected size of weights vector");
        const std::size_t T = input.size() / (F * 2 * A);
        ftpa_to_fpact(input.data(), _fpact, F, T, A, stream);
        _gemm.resize(4 * weights.size());
        check(sw_pack_weights(weights.data(), _gemm.data(), (int)F, (int)B, (int)A, (sw_stream_t)stream));
        output.resize({T / ts, F, B});
        output.metalike(input);
        output.tsamp(input.tsamp() * ts);
        sw_cb_shape shape{(int)F, (int)T, (int)A, (int)B, (int)ts, BfTraits::stokes_index,
                          _config.ib_subtraction() ? 1 : 0, T, 0, 0};
        sw_cb_problem prob{_fpact.data(), reinterpret_cast<int8_t*>(output.data()),
                           reinterpret_cast<const float*>(ib_powers.data()), 0, (int)B};
        check(sw_coherent_beamform(&shape, &prob, _gemm.data(), scales.data(), offsets.data(),
                                   beamset_mapping.data(), nullptr, (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "coherent beamformer");
    }

  private:
    const PipelineConfig& _config;
    DeviceVector<int8_t> _fpact, _gemm;
};

// -------------------------------------------------------- CoherentDedisperser
// cpp/skyweaver/CoherentDedisperser.cuh:30-92, src/CoherentDedisperser.cu:
// 19-134,142-225.  The configuration carries the reference's fields; the
// chirp tables of every (DM, channel) live in one device setup block
// (sw_cdd_chirps: FP64 phases of DMResponse, CoherentDedisperser.cu:313-335).
struct CoherentDedisperserConfig {
    std::size_t fft_length = 0;  // number of fine channels (the gulp, in the reference)
    std::size_t overlap_samps = 0;
    std::size_t num_coarse_chans = 0;
    std::size_t npols = 0;
    std::size_t nantennas = 0;
    double filter_delay = 0.0;  // tsamp * overlap_samps / 2 (CoherentDedisperser.cu:82)
    double tsamp = 0.0;
    double bw = 0.0;
    double low_freq = 0.0;
    double high_freq = 0.0;
    double coarse_chan_bw = 0.0;
    double fine_chan_bw = 0.0;
    std::vector<float> _h_dms;
    std::shared_ptr<DeviceVector<uint8_t>> _d_setup;  // twiddles + chirps [dm][chan][fft]
};

// CoherentDedisperser.cu:61-104: every field as the reference computes it,
// then the chirp tables on the device.
inline void create_coherent_dedisperser_config(CoherentDedisperserConfig& config,
                                               std::size_t fft_length, std::size_t overlap_samps,
                                               std::size_t num_coarse_chans, std::size_t npols,
                                               std::size_t nantennas, double tsamp,
                                               double low_freq, double bw, std::vector<float> dms)
{
    if(dms.empty()) throw std::runtime_error("No coherent DMs specified");
    config.fft_length       = fft_length;
    config.overlap_samps    = overlap_samps;
    config.num_coarse_chans = num_coarse_chans;
    config.npols            = npols;
    config.nantennas        = nantennas;
    config.tsamp            = tsamp;
    config.low_freq         = low_freq;
    config.bw               = bw;
    config.high_freq        = low_freq + bw;
    config.coarse_chan_bw   = bw / num_coarse_chans;
    config.filter_delay     = tsamp * overlap_samps / 2.0;
    config.fine_chan_bw     = config.coarse_chan_bw / fft_length;
    config._h_dms           = dms;
    const std::size_t n = sw_cdd_setup_bytes((int)dms.size(), (int)num_coarse_chans, (int)fft_length);
    if(n == 0) throw std::runtime_error("CoherentDedisperser: unsupported FFT length");
    config._d_setup = std::make_shared<DeviceVector<uint8_t>>(n);
    check(sw_cdd_chirps(dms.data(), (int)dms.size(), (int)num_coarse_chans, (int)fft_length, low_freq,
                        bw, config._d_setup->data(), nullptr));
    cuda_check(cudaStreamSynchronize(nullptr), "coherent dedisperser setup");
}

// CoherentDedisperser.cu:19-57.  The reference takes the gulp as the FFT
// length and the DM delay across the whole band as the overlap (and fails
// when that delay exceeds twice the gulp); both are kept here.
inline void create_coherent_dedisperser_config(CoherentDedisperserConfig& config,
                                               const PipelineConfig& pc)
{
    if(pc.coherent_dms().empty()) throw std::runtime_error("No coherent DMs specified");
    const float f_low  = (float)(pc.centre_frequency() - pc.bandwidth() / 2.0f);
    const float f_high = (float)(pc.centre_frequency() + pc.bandwidth() / 2.0f);
    const float tsamp  = (float)(pc.nchans() / pc.bandwidth());
    const float max_dm = *std::max_element(pc.coherent_dms().begin(), pc.coherent_dms().end());
    const double delay = 4.148806423e15 * (1.0 / ((double)f_low * f_low) -
                                           1.0 / ((double)f_high * f_high)) * max_dm;
    const std::size_t max_delay_samps = (std::size_t)(int)(delay / tsamp + 0.5);
    if(max_delay_samps > 2 * pc.gulp_length_samps())
        throw std::runtime_error("Gulp length must be at least 2 times the maximum DM delay");
    create_coherent_dedisperser_config(config, pc.gulp_length_samps(), max_delay_samps, pc.nchans(),
                                       pc.npol(), pc.nantennas(), tsamp, f_low, pc.bandwidth(),
                                       pc.coherent_dms());
}

class CoherentDedisperser {
  public:
    explicit CoherentDedisperser(CoherentDedisperserConfig& config) : _config(config) {}
    // CoherentDedisperser.cu:142-225: the first fft_length samples of one
    // channel's TPA voltages through FFT, chirp of (freq_idx, dm_idx), inverse
    // FFT, overlap_samps / 2 trimmed at each end, /N, rounding and int8 wrap;
    // the fft_length - overlap_samps results land in the FTPA output at
    // freq_idx * (fft_length - overlap_samps) samples, like the reference.
    void dedisperse(const TPAVoltagesD<char2>& d_tpa_voltages_in,
                    FTPAVoltagesD<char2>& d_ftpa_voltages_out, unsigned int freq_idx,
                    unsigned int dm_idx)
    {
        const std::size_t N = _config.fft_length, O = _config.overlap_samps;
        const std::size_t P = _config.npols, A = _config.nantennas, L = N - O;
        if(O >= N) throw std::runtime_error("CoherentDedisperser: overlap must be shorter than the FFT");
        if(d_tpa_voltages_in.size() < N * P * A)
            throw std::runtime_error("CoherentDedisperser: fewer input samples than the FFT length");
        if(freq_idx >= _config.num_coarse_chans || dm_idx >= _config._h_dms.size())
            throw std::runtime_error("CoherentDedisperser: channel or DM index out of range");
        const std::size_t out_offset = freq_idx * P * A * L;
        if(d_ftpa_voltages_out.size() < out_offset + L * P * A)
            throw std::runtime_error("CoherentDedisperser: output vector too small");
        // one window of one channel: rows hold O samples of history then L
        ftpa_to_fpact(d_tpa_voltages_in.data(), _in, 1, N, A, nullptr);
        _out.resize(P * A * 2 * L);
        const std::size_t ws = sw_cdd_workspace_bytes(1, (int)P, (int)A, (int)L, (int)N, (int)O, 1);
        _ws.resize(ws);
        check(sw_coherent_dedisperse_channel(
            _in.data(), N, (int)P, (int)A, (int)L, (int)N, (int)O, (int)(O / 2), _config._d_setup->data(),
            (int)_config._h_dms.size(), (int)_config.num_coarse_chans, (int)freq_idx, (int)dm_idx,
            _out.data(), L, ws ? _ws.data() : nullptr, ws, nullptr));
        check(sw_fpact_to_ftpa(_out.data(), d_ftpa_voltages_out.data() + out_offset, 1, (int)L, (int)A, L,
                               0, nullptr));
        cuda_check(cudaStreamSynchronize(nullptr), "coherent dedispersion");
        d_ftpa_voltages_out.reference_dm(_config._h_dms[dm_idx]);
    }

  private:
    CoherentDedisperserConfig& _config;
    DeviceVector<int8_t> _in, _out;
    DeviceVector<uint8_t> _ws;
};

// ------------------------------------------------------ IncoherentDedisperser
// cpp/skyweaver/IncoherentDedisperser.cuh:14-28, src/IncoherentDedisperser.cu:36-125
// on the device: int8 or char4 (IQUV, each component dedispersed and clamped
// on its own like the reference's char4 instantiation, :133-137) TFB in,
// TDB out.
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
    IncoherentDedisperser(const IncoherentDedisperser&) = delete;
    IncoherentDedisperser& operator=(const IncoherentDedisperser&) = delete;
    const std::vector<int>& delays() const { return _delays; }
    int max_sample_delay() const { return _max; }
    float scale_factor() const { return _scale; }
    // device TFB [T][F][B] (any vector with data() and size() in device
    // memory) -> TDB [(T - max_delay) / tscrunch][ndms][B]
    template <typename InputVectorType, typename OutputVectorType>
    void dedisperse(const InputVectorType& tfb_powers, OutputVectorType& tdb_powers,
                    cudaStream_t stream = 0)
    {
        using T = typename OutputVectorType::value_type;
        static_assert(sizeof(T) == 1 || sizeof(T) == 4, "int8 or char4 powers");
        static_assert(sizeof(typename InputVectorType::value_type) == sizeof(T), "same element type");
        const std::size_t ncomp = sizeof(T);
        const std::size_t F = _config.nchans(), B = _config.nbeams();
        const std::size_t nsamp = tfb_powers.size() / (F * B);
        if(nsamp <= (std::size_t)_max)
            throw std::runtime_error("Fewer than max_sample_delay samples passed to dedisperse method");
        if((nsamp - _max) % _tscrunch != 0)
            throw std::runtime_error("(nsamples - max_sample_delay) must be a multiple of tscrunch;");
        tdb_powers.resize({(nsamp - _max) / _tscrunch, _dms.size(), B});
        check(sw_incoherent_dedisperse(reinterpret_cast<const int8_t*>(tfb_powers.data()), (int)nsamp,
                                       (int)F, (int)(B * ncomp), _d_delays.data(), (int)_dms.size(),
                                       _max, (int)_tscrunch, _scale,
                                       reinterpret_cast<int8_t*>(tdb_powers.data()),
                                       (sw_stream_t)stream));
        cuda_check(cudaStreamSynchronize(stream), "incoherent dedispersion");
    }

  private:
    const PipelineConfig& _config;
    std::vector<float> _dms;
    std::size_t _tscrunch;
    std::vector<int> _delays;
    DeviceVector<int> _d_delays;
    int _max = 0;
    float _scale = 1.0f;
};

// ------------------------------------------- IncoherentDedispersionPipeline
// IncoherentDedispersionPipeline<InputType, OutputType, Handler>
// (IncoherentDedispersionPipeline.cuh:18-60,
// detail/IncoherentDedispersionPipeline.cu:6-113) with the AggregationBuffer
// in device memory: one block per DedispersionPlan block (coherent DM) of the
// config.  The handler gets init(header) and
// handler(TDBPowersD<OutputType> const&, std::size_t ref_dm_idx) with the
// TDB in device memory and the reference's metadata (dms, reference DM,
// centre frequency, tsamp x tscrunch, utc_offset + max delay), ordered on the
// pushing stream.
template <typename InputType, typename OutputType, typename Handler>
class IncoherentDedispersionPipeline {
  public:
    using InputVectorType  = TFBPowersD<InputType>;
    using OutputVectorType = TDBPowersD<OutputType>;
    IncoherentDedispersionPipeline(const PipelineConfig& config, Handler& handler)
        : _config(config), _handler(handler)
    {
        static_assert(sizeof(InputType) == sizeof(OutputType), "same element type");
        const auto& blocks = config.ddplan().blocks();
        const int ncomp = (int)sizeof(InputType);
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
        _meta.resize(blocks.size());
        check(sw_idd_pipeline_create((int)config.nchans(), (int)config.nbeams() * ncomp,
                                     (int)blocks.size(), ndms.data(), dptr.data(), ts.data(),
                                     scale.data(), nullptr, &trampoline, this, &_p));
    }
    ~IncoherentDedispersionPipeline() { sw_idd_pipeline_destroy(_p); }
    IncoherentDedispersionPipeline(const IncoherentDedispersionPipeline&) = delete;
    IncoherentDedispersionPipeline& operator=(const IncoherentDedispersionPipeline&) = delete;

    void init(const ObservationHeader& header) { _handler.init(header); }
    // push one gulp of beams for coherent-DM block ref_dm_idx
    void operator()(const InputVectorType& data, std::size_t ref_dm_idx, cudaStream_t stream = 0)
    {
        if(ref_dm_idx >= _dedispersers.size()) throw std::runtime_error("DM block index out of range");
        Meta& m = _meta[ref_dm_idx];
        m.tsamp = data.tsamp() * _config.ddplan()[ref_dm_idx].tscrunch;
        m.utc_offset = data.utc_offset() + _dedispersers[ref_dm_idx]->max_sample_delay() * data.tsamp();
        check(sw_idd_pipeline_push(_p, (int)ref_dm_idx, reinterpret_cast<const int8_t*>(data.data()),
                                   data.nsamples(), (sw_stream_t)stream));
    }
    const IncoherentDedisperser& dedisperser(std::size_t i) const { return *_dedispersers[i]; }

  private:
    struct Meta {
        double tsamp = 0.0, utc_offset = 0.0;
    };
    static void trampoline(void* user, int block, const int8_t* d_tdb, int nout, int ndms,
                           int nbeams_comp, sw_stream_t)
    {
        auto* self = static_cast<IncoherentDedispersionPipeline*>(user);
        const auto& b = self->_config.ddplan()[block];
        const std::size_t nbeams = (std::size_t)nbeams_comp / sizeof(OutputType);
        OutputVectorType v = OutputVectorType::view(
            reinterpret_cast<OutputType*>(const_cast<int8_t*>(d_tdb)),
            {(std::size_t)nout, (std::size_t)ndms, nbeams});
        v.dms(b.incoherent_dms);
        v.reference_dm(b.coherent_dm);
        v.tsamp(self->_meta[block].tsamp);
        v.utc_offset(self->_meta[block].utc_offset);
        v._frequencies.assign(1, self->_config.centre_frequency());
        v._frequencies_stale = false;
        self->_handler(v, (std::size_t)block);
    }
    const PipelineConfig& _config;
    Handler& _handler;
    std::vector<std::unique_ptr<IncoherentDedisperser>> _dedispersers;
    std::vector<Meta> _meta;
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
// BeamformerPipeline<CBHandler, IBHandler, StatsHandler, BeamformerTraits>
// (cpp/skyweaver/BeamformerPipeline.cuh:24-67,
// detail/BeamformerPipeline.cu:40-301) over the graph-captured device chain
// of sw_pipeline.  The handler concept is the reference's:
//   cb_handler.init(header);    cb_handler(TFBPowersD<Quantised> const&, dm_idx)
//   ib_handler.init(header);    ib_handler(BTFPowersD<Quantised> const&, dm_idx)
//   stats_handler.init(header); stats_handler(FPAStatsD<Statistics> const&)
// with the vectors in device memory and their metadata set (frequencies,
// tsamp, utc_offset = the dedisperser's filter delay, reference_dm).
// Unlike the reference, which synchronises every gulp, operator() queues
// gulp g on the device and then hands gulp g - 1's outputs to the handlers
// while gulp g computes; flush() (and the destructor) hand over the last
// gulp.  The handlers' views stay valid until the next operator() returns.
template <typename CBHandler, typename IBHandler, typename StatsHandler,
          typename BeamformerTraits = SingleStokesBeamformerTraits<I>>
class BeamformerPipeline {
  public:
    using VoltageVectorTypeH = TAFTPVoltagesH<char2>;
    using VoltageVectorTypeD = TAFTPVoltagesD<char2>;
    using TimeType           = long double;
    using Quantised          = typename BeamformerTraits::QuantisedPowerType;

    BeamformerPipeline(const PipelineConfig& config, CBHandler& cb_handler, IBHandler& ib_handler,
                       StatsHandler& stats_handler)
        : _config(config), _cb(cb_handler), _ib(ib_handler), _stats(stats_handler),
          _delays(config, nullptr)
    {
        if(config.coherent_dms().empty()) throw std::runtime_error("No DDPlan set for pipeline");
        if(config.gulp_length_samps() % config.nsamples_per_heap() != 0)
            throw std::runtime_error("Gulp size is not a multiple of the number of samples per heap");
        _tick_per_block = 2 * config.total_nchans() * config.gulp_length_samps();
    }
    ~BeamformerPipeline()
    {
        try {
            flush();
        } catch(...) {
        }
        if(_p) sw_pipeline_destroy(_p);
    }
    BeamformerPipeline(const BeamformerPipeline&) = delete;

    // BeamformerPipeline.cu:100-115: the observation's header (its antenna
    // count, UTC start and sample clock) and a start-time offset
    void init(const ObservationHeader& header, long double utc_offset = 0.0)
    {
        _header     = header;
        _utc_offset = utc_offset;
        if(_p == nullptr) create((int)header.nantennas);
        _cb.init(_header);
        _ib.init(_header);
        _stats.init(_header);
    }
    // one gulp of TAFTP voltages in pinned host memory; the host buffer may be
    // reused once this returns
    bool operator()(const VoltageVectorTypeH& taftp_on_host)
    {
        submit(taftp_on_host.data(), taftp_on_host.size(), true);
        return false;
    }
    // the same from device memory
    bool operator()(const VoltageVectorTypeD& taftp_on_device)
    {
        submit(taftp_on_device.data(), taftp_on_device.size(), false);
        return false;
    }
    // hand the last queued gulp to the handlers
    void flush()
    {
        if(_pending >= 0) deliver(_pending);
        _pending = -1;
    }
    // the coherent-dedispersion plan in use (fft_len, overlap, lag)
    std::vector<int> cdd_plan() const
    {
        int n = 0, o = 0, l = 0;
        if(_p) check(sw_pipeline_fft_len(_p, &n, &o, &l));
        return {n, o, l};
    }
    std::size_t call_count() const { return _call_count; }

  private:
    void create(int input_nantennas)
    {
        sw_pipeline_config c{};
        c.nantennas       = (int)_config.nantennas();
        c.input_nantennas = input_nantennas;
        c.nchans          = (int)_config.nchans();
        c.nbeams          = (int)_config.nbeams();
        c.gulp_samples    = (int)_config.gulp_length_samps();
        c.tscrunch        = (int)_config.cb_tscrunch();
        c.stokes          = BeamformerTraits::stokes_index;
        c.ib_subtract     = _config.ib_subtraction() ? 1 : 0;
        c.output_level    = _config.output_level();
        c.centre_frequency = _config.centre_frequency();
        c.bandwidth       = _config.bandwidth();
        c.ndms            = (int)_config.coherent_dms().size();
        c.dms             = _config.coherent_dms().data();
        c.fft_len         = (int)_config.cdd_fft_length();
        c.enable_coherent_dedispersion = 1;
        c.grouped         = 1;
        c.use_graph       = 1;
        c.nbeamsets       = _delays.nbeamsets();
        c.beamset_weights = _delays.beamset_weights_host().data();
        c.beamset_mapping = _delays.beamset_mapping_host().data();
        c.autotune        = _config.autotune() ? 1 : 0;
        c.cdd_lag         = _config.cdd_lag();
        check(sw_pipeline_create(&c, &_p));
        int n = 0, o = 0, l = 0;
        check(sw_pipeline_fft_len(_p, &n, &o, &l));
        _chan_tsamp = (double)_config.nchans() / _config.bandwidth();
        _filter_delay = _chan_tsamp * l;
    }
    void submit(const void* data, std::size_t n, bool host)
    {
        if(_p == nullptr) throw std::runtime_error("BeamformerPipeline: init() before the first gulp");
        const std::size_t expect = _config.gulp_length_samps() * _header.nantennas * _config.nchans() *
                                   _config.npol();
        if(n != expect)
            throw std::runtime_error("Unexpected buffer size, expected " + std::to_string(expect) +
                                     " but got " + std::to_string(n));
        // BeamformerPipeline.cu:286-291: the epoch of this gulp
        const TimeType epoch = (TimeType)_header.utc_start + _utc_offset +
                               (TimeType)(_call_count * _tick_per_block) / _header.sample_clock;
        const auto& d = _delays.delays((double)epoch);
        if(_delays.model_index() != _uploaded_model) {
            std::vector<float3> h = d.download();
            check(sw_pipeline_set_delays(_p, reinterpret_cast<const float*>(h.data()), _delays.epoch()));
            _uploaded_model = _delays.model_index();
        }
        // the handlers' work on the gulp this one overwrites comes first
        check(sw_pipeline_order_after(_p, nullptr));
        if(host) {
            check(sw_pipeline_process_host(_p, data, (double)epoch, nullptr, nullptr));
            check(sw_pipeline_wait_input(_p));
        } else {
            check(sw_pipeline_process_device(_p, data, (double)epoch, nullptr));
        }
        const long g = sw_pipeline_gulp_count(_p) - 1;
        if(_pending >= 0) deliver(_pending);
        _pending = g;
        ++_call_count;
    }
    void deliver(long g)
    {
        const std::size_t F = _config.nchans(), B = _config.nbeams(), ts = _config.cb_tscrunch();
        const std::size_t T = _config.gulp_length_samps(), A = _config.nantennas();
        const auto& freqs = _config.channel_frequencies();
        const float* d_stats = nullptr;
        for(std::size_t dm = 0; dm < _config.coherent_dms().size(); ++dm) {
            const int8_t *cb = nullptr, *ib = nullptr;
            check(sw_pipeline_gulp_outputs(_p, g, (int)dm, &cb, nullptr, &ib, &d_stats));
            auto cbv = TFBPowersD<Quantised>::view(reinterpret_cast<Quantised*>(const_cast<int8_t*>(cb)),
                                                   {T / ts, F, B});
            auto ibv = BTFPowersD<Quantised>::view(reinterpret_cast<Quantised*>(const_cast<int8_t*>(ib)),
                                                   {(std::size_t)_delays.nbeamsets(), T / ts, F});
            auto describe = [&](auto& v) {
                v.frequencies(freqs);
                v.tsamp(_chan_tsamp * ts);
                v.utc_offset(_filter_delay);
                v.reference_dm(_config.coherent_dms()[dm]);
            };
            describe(cbv);
            describe(ibv);
            _cb(cbv, dm);
            _ib(ibv, dm);
        }
        auto st = FPAStatsD<Statistics>::view(
            reinterpret_cast<Statistics*>(const_cast<float*>(d_stats)), {F, _config.npol(), A});
        st.frequencies(freqs);
        st.tsamp(_chan_tsamp);
        _stats(st);
    }

    const PipelineConfig& _config;
    CBHandler& _cb;
    IBHandler& _ib;
    StatsHandler& _stats;
    DelayManager _delays;
    ObservationHeader _header{};
    TimeType _utc_offset = 0.0;
    std::size_t _tick_per_block = 0, _call_count = 0, _uploaded_model = (std::size_t)-1;
    double _chan_tsamp = 0.0, _filter_delay = 0.0;
    long _pending = -1;
    sw_pipeline* _p = nullptr;
};

}  // namespace skyweaver_b200
