/*
 * skyweaver_b200.h -- C ABI of the B200-native skyweaver beamforming hot path.
 *
 * Conventions
 *   - Every entry point returns an int status (SW_OK == 0).  On failure the
 *     message is available from sw_last_error() (thread local).  No C++
 *     exception crosses this boundary.
 *   - Pointers named d_* are device pointers (caller allocated unless stated),
 *     h_* are host pointers.  Sizes are element counts unless named *_bytes.
 *   - Every kernel entry point is asynchronous on the given stream
 *     (cudaStream_t passed as sw_stream_t; NULL = legacy default stream).
 *   - int8 complex voltages are (re, im) byte pairs ("char2").
 *
 * Layouts
 *   TAFTP  [heap][antenna][channel][256 samples][pol][re,im]   (input files)
 *   FTPA   [channel][sample][pol][antenna][re,im]              (reference stages)
 *   FPACT  [channel][pol][antenna][re|im][row_stride samples]  (B200 planar,
 *          stream-major layout used inside the pipeline; sample s of stream
 *          (f,p,a) lives at byte ((((f*P+p)*A+a)*2+c)*row_stride + offset + s))
 *   weights FBA   [channel][beam][antenna][re,im]              (reference)
 *   weights GEMM  [channel][re-row|im-row][beam][antenna][2]   (tensor-core
 *          A operand: re-row = (w_re, -w_im), im-row = (w_im, w_re))
 *   CB output TFB [sample/tscrunch][channel][beam] int8
 *   IB output BTF [beamset][sample/tscrunch][channel] (float raw and int8)
 *   IDD output TDB [sample][dm][beam] int8
 *
 * Each declaration names the reference (erc-compact/skyweaver, paths relative
 * to the project root) interface it replaces.
 */
#ifndef SKYWEAVER_B200_H
#define SKYWEAVER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct CUstream_st* sw_stream_t;

enum sw_status {
    SW_OK              = 0,
    SW_ERR_INVALID     = 1, /* bad argument or size (std::runtime_error in the reference) */
    SW_ERR_CUDA        = 2, /* CUDA runtime / driver error */
    SW_ERR_UNSUPPORTED = 3, /* shape outside what the kernels implement */
    SW_ERR_TIMEOUT     = 4, /* a bounded device-side wait gave up */
    SW_ERR_STATE       = 5, /* call out of order (e.g. scalings before stats) */
    SW_ERR_EPOCH       = 6  /* InvalidDelayEpoch (DelayManager.cuh:19-34) */
};

/* Stokes modes: one parameter (int8 outputs, float raw IB power) or all four
 * (SW_STOKES_IQUV: char4 {I,Q,U,V} outputs and float4 raw IB power, the
 * reference's FullStokesBeamformerTraits, beamformer_utils.cuh:198-278). */
enum sw_stokes { SW_STOKES_I = 0, SW_STOKES_Q = 1, SW_STOKES_U = 2, SW_STOKES_V = 3,
                 SW_STOKES_IQUV = 4 };

/* Library identification and error reporting. */
int sw_version(void);
const char* sw_last_error(void);
/* Device-side error word shared by the kernels with bounded waits
 * (0 = clean).  sw_reset_device_error clears it. */
int sw_read_device_error(int* h_code);
int sw_reset_device_error(void);

/* Bounded-wait self-test of the coherent beamformer (no reference
 * counterpart: the reference has no device-side waits).  Launches a minimal
 * beamformer whose copy producer issues nothing, so its MMA role's first wait
 * can only end at the given deadline (microseconds, at most 10 s).  Returns
 * SW_ERR_TIMEOUT when the kernel recorded the timeout in the device error
 * word and returned (the word is cleared again), SW_ERR_STATE if it did not. */
int sw_cb_timeout_selftest(int timeout_us, sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* Transposer                                                           */
/* ------------------------------------------------------------------ */
/* Replaces Transposer::transpose (cpp/skyweaver/Transposer.cuh:66-69,
 * cpp/skyweaver/src/Transposer.cu:117-184): TAFTP -> FTPA with the antenna
 * dimension zero padded from input_nantennas to output_nantennas. */
int sw_transpose_ftpa(const void* d_taftp, void* d_ftpa, int nheaps,
                      int input_nantennas, int output_nantennas, int nchans,
                      sw_stream_t stream);

/* B200 form of the same stage: TAFTP -> FPACT written at
 * [sample_offset, sample_offset + nheaps*256) of rows of row_stride samples
 * (the pipeline keeps coherent-dedispersion history in front of the gulp). */
int sw_transpose_fpact(const void* d_taftp, void* d_fpact, int nheaps,
                       int input_nantennas, int output_nantennas, int nchans,
                       size_t row_stride, size_t sample_offset,
                       sw_stream_t stream);

/* Layout converters between the reference FTPA layout and FPACT. */
int sw_ftpa_to_fpact(const void* d_ftpa, void* d_fpact, int nchans,
                     int nsamples, int nantennas, size_t row_stride,
                     size_t sample_offset, sw_stream_t stream);
int sw_fpact_to_ftpa(const void* d_fpact, void* d_ftpa, int nchans,
                     int nsamples, int nantennas, size_t row_stride,
                     size_t sample_offset, sw_stream_t stream);

/* Copy the last `history` samples of every FPACT row to its front
 * (overlap-save history for the next gulp; replaces the per-channel copies of
 * BufferedDispenser::hoard, cpp/skyweaver/src/BufferedDispenser.cu:29-66). */
int sw_fpact_keep_history(void* d_fpact, size_t nrows, size_t row_stride,
                          size_t history, sw_stream_t stream);
/* The same history copy between two row sets: the last `history` samples of
 * every row of d_prev to the front of the same row of d_next (the pipeline
 * alternates two row sets, so a gulp's rows stay intact while the next gulp
 * is transposed). */
int sw_fpact_copy_history(const void* d_prev, void* d_next, size_t nrows,
                          size_t row_stride, size_t history, sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* StatisticsCalculator                                                 */
/* ------------------------------------------------------------------ */
/* Replaces StatisticsCalculator::calculate_statistics
 * (cpp/skyweaver/StatisticsCalculator.cuh:65,
 *  cpp/skyweaver/src/StatisticsCalculator.cu:54-85,104-130).
 * Output d_stats: float [nchans][npol][nant][4] = {mean, std, skew, kurtosis}
 * over the 2*nsamples real and imaginary values of each (f,p,a).
 * d_scratch: caller-provided device workspace of
 * sw_statistics_scratch_bytes() bytes (exact int64 moment sums). */
size_t sw_statistics_scratch_bytes(int nchans, int npol, int nant);
int sw_statistics(const void* d_fpact, size_t row_stride, size_t sample_offset,
                  int nchans, int npol, int nant, int nsamples,
                  void* d_scratch, float* d_stats, sw_stream_t stream);

/* The TAFTP -> FPACT transpose (sw_transpose_fpact) and the statistics of the
 * transposed gulp (sw_statistics with npol 2 over its nheaps * 256 samples)
 * in one pass over the gulp: replaces Transposer::transpose
 * (cpp/skyweaver/src/Transposer.cu:117-184) followed by
 * StatisticsCalculator::calculate_statistics
 * (cpp/skyweaver/src/StatisticsCalculator.cu:54-85,104-130), which read the
 * voltages twice.  d_fpact and d_stats hold exactly what the two separate
 * calls write; d_scratch has sw_statistics_scratch_bytes(nchans, 2,
 * output_nantennas) bytes. */
int sw_transpose_fpact_statistics(const void* d_taftp, void* d_fpact, int nheaps,
                                  int input_nantennas, int output_nantennas, int nchans,
                                  size_t row_stride, size_t sample_offset, void* d_scratch,
                                  float* d_stats, sw_stream_t stream);

/* No counterpart in the reference.  Same result as sw_statistics, for callers
 * that cannot allocate device memory (a real-time ingest loop that must not
 * take cudaMalloc's implicit device synchronisation, or a process whose
 * device memory is owned by another component): the workspace is a
 * file-scope device array of the library, so this call allocates nothing.
 *   - at most 16384 (channel, pol, antenna) series; larger shapes return
 *     SW_ERR_INVALID with a message, nothing is launched;
 *   - the first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress with that device current) and keeps it for the
 *     process; make that first call before capturing any stream.  A
 *     cudaDeviceReset invalidates the kept address, so do not call this
 *     entry point on a device after resetting it;
 *   - every call shares the one array (it is cleared at the start of each
 *     call): calls whose kernels overlap on the GPU, from any stream or
 *     thread, race and give wrong statistics;
 *   - every GPU that loads the library holds the 512 KiB array until exit. */
int sw_statistics_noalloc(const void* d_fpact, size_t row_stride,
                          size_t sample_offset, int nchans, int npol, int nant,
                          int nsamples, float* d_stats, sw_stream_t stream);

/* Replaces StatisticsCalculator::update_scalings
 * (cpp/skyweaver/StatisticsCalculator.cuh:96-97,
 *  cpp/skyweaver/src/StatisticsCalculator.cu:132-239), computed on the
 * device.  Outputs are indexed [beamset*nchans + chan]: the reference writes
 * [chan] for every beamset, which leaves beamsets above 0 with scale 0. */
int sw_update_scalings(const float* d_stats, const float* d_beamset_weights,
                       int nbeamsets, int nchans, int npol, int nant,
                       int cb_tscrunch, int ib_tscrunch, float output_level,
                       float* d_cb_offsets, float* d_cb_scaling,
                       float* d_ib_offsets, float* d_ib_scaling,
                       sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* WeightsManager                                                       */
/* ------------------------------------------------------------------ */
/* Replaces WeightsManager::weights (cpp/skyweaver/WeightsManager.cuh:58-65,
 * cpp/skyweaver/src/WeightsManager.cu:16-87,109-139).
 * d_delays: float3 [nbeams][nant] (weight, offset s, rate s/s);
 * d_freqs: double [nchans] Hz.  Either output may be NULL. */
int sw_generate_weights(const float* d_delays, const double* d_freqs,
                        int nant, int nbeams, int nchans, double current_epoch,
                        double delay_epoch, void* d_weights_fba,
                        void* d_weights_gemm, sw_stream_t stream);
/* Reference FBA weights -> GEMM layout (for caller-supplied weights). */
int sw_pack_weights(const void* d_weights_fba, void* d_weights_gemm,
                    int nchans, int nbeams, int nant, sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* IncoherentBeamformer                                                 */
/* ------------------------------------------------------------------ */
/* Replaces IncoherentBeamformer<BfTraits>::beamform
 * (cpp/skyweaver/IncoherentBeamformer.cuh:84-91,
 *  cpp/skyweaver/src/IncoherentBeamformer.cu:15-91,108-182) for the single
 * Stokes traits.  Uses the per-beamset antenna weights of the reference's
 * CPU implementation (IncoherentBeamformerTester.cu:68-70). */
int sw_incoherent_beamform(const void* d_fpact, size_t row_stride,
                           size_t sample_offset, int nchans, int nsamples,
                           int nant, int tscrunch, const float* d_scale,
                           const float* d_offset,
                           const float* d_beamset_weights, int nbeamsets,
                           int stokes, float* d_raw, int8_t* d_out,
                           sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* CoherentBeamformer (tcgen05 int8 tensor cores)                       */
/* ------------------------------------------------------------------ */
/* One GEMM problem: a coherent DM (voltage block) x a contiguous beam range.
 * The plain form launches one problem; the grouped form runs all problems
 * of a gulp in one persistent launch with a ragged work queue. */
typedef struct sw_cb_problem {
    const void* d_fpact;   /* dedispersed voltages for this DM (FPACT)   */
    int8_t* d_out;         /* TFB output for this DM                      */
    const float* d_ib_raw; /* IB raw power BTF [beamset][T/ts][F] for DM  */
    int beam_start;        /* first beam of the range                     */
    int beam_count;        /* beams in the range                          */
} sw_cb_problem;

typedef struct sw_cb_shape {
    int nchans;
    int nsamples;       /* per gulp; multiple of 64                       */
    int nantennas;      /* 16, 32 or 64                                   */
    int nbeams;         /* total beams (TFB row length)                   */
    int tscrunch;       /* 1..32, power of two                            */
    int stokes;         /* sw_stokes                                      */
    int ib_subtract;    /* SKYWEAVER_IB_SUBTRACTION (default 1)           */
    size_t row_stride;  /* FPACT row stride (samples)                     */
    size_t sample_offset;
    int tiles_per_item; /* 64-sample tiles per work item (0: 64; see sw_autotune) */
    int voltage_stages; /* voltage tiles in flight, 2..8 (0: 4; see sw_autotune) */
    int weight_stages;  /* weight blocks in flight, 2..3 (0: 2)                  */
} sw_cb_shape;

/* Replaces CoherentBeamformer<BfTraits>::beamform
 * (cpp/skyweaver/CoherentBeamformer.cuh:84-92,
 *  cpp/skyweaver/src/CoherentBeamformer.cu:12-174,191-270).
 * d_weights_gemm: sw_generate_weights/sw_pack_weights GEMM layout;
 * d_scale/d_offset: [beamset][chan]; d_mapping: int [nbeams] beam->beamset.
 * d_debug_voltages: optional int32 [F][T][P][B][2] exact beam voltages
 * (test hook; NULL in production). */
int sw_coherent_beamform(const sw_cb_shape* shape, const sw_cb_problem* problem,
                         const void* d_weights_gemm, const float* d_scale,
                         const float* d_offset, const int* d_mapping,
                         int32_t* d_debug_voltages, sw_stream_t stream);
/* Batched form: all (DM x beam range) problems in one persistent launch. */
int sw_coherent_beamform_grouped(const sw_cb_shape* shape,
                                 const sw_cb_problem* h_problems,
                                 int nproblems, const void* d_weights_gemm,
                                 const float* d_scale, const float* d_offset,
                                 const int* d_mapping, sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* CoherentDedisperser (FP64 chirp, FP32 Stockham-class FFT)            */
/* ------------------------------------------------------------------ */
/* Bytes of the device setup block (per-pass FFT twiddle tables followed by
 * the chirp tables) for sw_cdd_chirps / sw_coherent_dedisperse; 0 if
 * fft_len is not a supported power of two (256 .. 65536). */
size_t sw_cdd_setup_bytes(int ndms, int nchans, int fft_len);

/* Replaces create_coherent_dedisperser_config's response tables, i.e.
 * get_dm_responses / DMResponse
 * (cpp/skyweaver/src/CoherentDedisperser.cu:61-104,293-359): FP64 chirp
 * phases stored as complex float [ndms][nchans][fft_len] in the FFT's
 * internal (digit-reversed) bin order, plus FP64-computed twiddles.
 * low_freq is the band's lower edge and bw its width (Hz). */
int sw_cdd_chirps(const float* h_dms, int ndms, int nchans, int fft_len,
                  double low_freq, double bw, void* d_setup,
                  sw_stream_t stream);

/* The overlap-save plan, host only (replaces the overlap and FFT-length
 * choice of create_coherent_dedisperser_config,
 * cpp/skyweaver/src/CoherentDedisperser.cu:19-57, which sizes the overlap by
 * the whole subband's DM delay and takes the gulp as the FFT length).  Each
 * window trims, at its start, the largest intra-channel DM smear (lowest
 * channel, largest DM) rounded up to 16 samples and, at its end, `*lag`
 * samples (lag_request rounded up to 16; 0 = 128; none when every DM is 0,
 * whose chirp is exactly 1): *overlap is their sum.
 * *fft_len > 0 on entry is kept if it exceeds the overlap; 0 picks one by a
 * cost model (on-chip sizes up to 8192 first).  SW_ERR_INVALID if none fits. */
int sw_cdd_plan(double centre_frequency, double bandwidth, int nchans,
                const float* h_dms, int ndms, int lag_request, int* fft_len,
                int* overlap, int* lag);

/* Replaces CoherentDedisperser::dedisperse
 * (cpp/skyweaver/CoherentDedisperser.cuh:77-80,
 *  cpp/skyweaver/src/CoherentDedisperser.cu:142-225) for all channels,
 * antennas, pols and DMs of a gulp with correct overlap-save: input rows
 * hold `overlap` history samples then nsamples new samples
 * (row_stride >= overlap + nsamples); every fft_len-point window advances by
 * fft_len - overlap samples and trims overlap - lag samples at its start and
 * lag at its end, so output d_out[dm] (FPACT, row stride out_row_stride)
 * holds nsamples samples delayed by `lag` (0 <= lag <= overlap).  The
 * reference trims overlap/2 at each end (lag = overlap / 2); its chirp's
 * response lies almost entirely at causal lags up to the intra-channel smear,
 * so a plan with overlap - lag >= that smear and a small lag is wrap-free at
 * a smaller overlap.  Requantisation wraps to int8 like the reference. */
int sw_coherent_dedisperse(const void* d_fpact_in, size_t row_stride,
                           int nchans, int npol, int nant, int nsamples,
                           int fft_len, int overlap, int lag,
                           const void* d_setup, int ndms, void* const* h_d_out,
                           size_t out_row_stride, sw_stream_t stream);

/* Workspace bytes sw_coherent_dedisperse_ws needs to process every
 * overlap-save segment of a gulp in one pass (0 for fft_len <= 8192, which
 * runs entirely on chip). fft_len 16384, 32768 and 65536 are split into
 * 8192-point sub-transforms whose intermediate spectra pass through this
 * complex workspace. */
size_t sw_cdd_workspace_bytes(int nchans, int npol, int nant, int nsamples,
                              int fft_len, int overlap, int ndms);

/* sw_coherent_dedisperse for any fft_len in [256, 65536]. A workspace
 * smaller than sw_cdd_workspace_bytes is used in chunks of segments (at
 * least ndms * fft_len * 8 bytes). d_debug_f32, if not null, receives the
 * dedispersed voltages before rounding: float2 [ndms][nchans][npol][nant]
 * [nsamples] (re, im), for precision studies against an FP64 reference. */
int sw_coherent_dedisperse_ws(const void* d_fpact_in, size_t row_stride,
                              int nchans, int npol, int nant, int nsamples,
                              int fft_len, int overlap, int lag,
                              const void* d_setup,
                              int ndms, void* const* h_d_out,
                              size_t out_row_stride, void* d_workspace,
                              size_t workspace_bytes, float* d_debug_f32,
                              sw_stream_t stream);

/* Replaces CoherentDedisperser::dedisperse(tpa, ftpa, freq_idx, dm_idx)
 * call by call (cpp/skyweaver/CoherentDedisperser.cuh:77-80): one channel,
 * one DM of a setup that sw_cdd_chirps built for setup_nchans channels and
 * setup_ndms DMs; input and output rows as for sw_coherent_dedisperse
 * (npol x nant streams of the one channel).  fft_len > 8192 needs the
 * workspace sw_cdd_workspace_bytes gives for one DM. */
int sw_coherent_dedisperse_channel(const void* d_fpact_in, size_t row_stride,
                                   int npol, int nant, int nsamples,
                                   int fft_len, int overlap, int lag,
                                   const void* d_setup, int setup_ndms,
                                   int setup_nchans, int freq_idx, int dm_idx,
                                   void* d_out, size_t out_row_stride,
                                   void* d_workspace, size_t workspace_bytes,
                                   sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* IncoherentDedisperser                                                */
/* ------------------------------------------------------------------ */
/* Replaces IncoherentDedisperser::dedisperse<int8 TFB, int8 TDB>
 * (cpp/skyweaver/IncoherentDedisperser.cuh:24-26,
 *  cpp/skyweaver/src/IncoherentDedisperser.cu:66-125) on the GPU.
 * d_delays: int [ndms][nchans] sample delays; scale_factor as the
 * reference's prepare() computes it. */
int sw_incoherent_dedisperse(const int8_t* d_tfb, int nsamples, int nchans,
                             int nbeams, const int* d_delays, int ndms,
                             int max_delay, int tscrunch, float scale_factor,
                             int8_t* d_tdb, sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* IncoherentDedispersionPipeline (device-resident AggregationBuffer)   */
/* ------------------------------------------------------------------ */
/* Replaces IncoherentDedispersionPipeline<In,Out,Handler>
 * (cpp/skyweaver/IncoherentDedispersionPipeline.cuh,
 *  cpp/skyweaver/detail/IncoherentDedispersionPipeline.cu:6-113) and its
 * AggregationBuffer (cpp/skyweaver/detail/AggregationBuffer.cu:23-117) with
 * the buffer in device memory. One block per coherent DM of the
 * DedispersionPlan; each block aggregates int8 TFB [T][nchans][nbeams]
 * (nbeams counts Stokes components: 4 x beams for IQUV), and every
 * `dispatch` new samples (after the first dispatch + overlap) runs the
 * incoherent dedisperser on the buffer and calls the handler with the TDB
 * result [dispatch / tscrunch][ndms][nbeams] in device memory, on the
 * pushing stream, before the buffer's overlap moves to its front. */
typedef struct sw_idd_pipeline sw_idd_pipeline;
typedef void (*sw_idd_handler)(void* user, int block, const int8_t* d_tdb,
                               int nsamples_out, int ndms, int nbeams,
                               sw_stream_t stream);

/* h_delays[b]: int [h_ndms[b]][nchans] sample delays of block b (the
 * IncoherentDedisperser's delays(), overlap = their maximum); h_scale[b] its
 * scale factor; h_dispatch may be NULL for the reference's default
 * max(10 x max delay, 8192) rounded down to a multiple of tscrunch. */
int sw_idd_pipeline_create(int nchans, int nbeams, int nblocks,
                           const int* h_ndms, const int* const* h_delays,
                           const int* h_tscrunch, const float* h_scale,
                           const int* h_dispatch, sw_idd_handler handler,
                           void* user, sw_idd_pipeline** out);
void sw_idd_pipeline_destroy(sw_idd_pipeline* p);
/* AggregationBuffer::push_back for block `block` (operator()(data, dm_idx)):
 * nsamples time samples of device TFB. */
int sw_idd_pipeline_push(sw_idd_pipeline* p, int block, const int8_t* d_tfb,
                         size_t nsamples, sw_stream_t stream);
int sw_idd_pipeline_geometry(const sw_idd_pipeline* p, int block,
                             int* dispatch_size, int* overlap,
                             int* nsamples_out, int* ndms);

/* ------------------------------------------------------------------ */
/* Autotuner                                                            */
/* ------------------------------------------------------------------ */
/* Times the coherent dedisperser at every FFT length the DM smear allows
 * and the coherent beamformer at several work-item sizes (its tile shape in
 * time) and pipeline depths (voltage and weight copies in flight), on
 * synthetic data of this exact shape, and returns the fastest choice (cached
 * per key (nantennas, nbeams, nchans, nsamples, tscrunch, ndms, overlap) for
 * the process). The reference's launch shapes are compile-time constants
 * (skyweaver_constants.hpp:28-135); this has no counterpart there. Needs a
 * few GB of device memory while it runs. */
typedef struct sw_tuning {
    int fft_len;            /* coherent dedispersion FFT length          */
    int overlap;            /* overlap-save overlap (samples)            */
    int lag;                /* of it, trimmed at each window's end       */
    int cb_tiles_per_item;  /* sw_cb_shape.tiles_per_item                */
    float cdd_ms, cb_ms;    /* measured per gulp at the chosen settings  */
    int cb_voltage_stages;  /* sw_cb_shape.voltage_stages                */
    int cb_weight_stages;   /* sw_cb_shape.weight_stages                 */
} sw_tuning;

int sw_autotune(int nantennas, int nbeams, int nchans, int nsamples,
                int tscrunch, int ndms, const float* h_dms,
                double centre_frequency, double bandwidth, sw_tuning* out,
                sw_stream_t stream);

/* ------------------------------------------------------------------ */
/* DADA ingest and output (host I/O around the pipeline)                */
/* ------------------------------------------------------------------ */
/* ObservationHeader (cpp/skyweaver/ObservationHeader.hpp:9-34); the
 * reference's long double fields are double here (the raw strings stay
 * available through sw_dada_header_get). */
typedef struct sw_observation_header {
    size_t nchans, npol, nbits, nantennas, sample_clock_start, chan0_idx;
    size_t obs_nchans, obs_offset;
    double bandwidth, obs_bandwidth, frequency, obs_frequency, tsamp;
    double sample_clock, sync_time, utc_start, mjd_start;
    char source_name[64], ra[32], dec[32], telescope[32], instrument[32];
} sw_observation_header;

/* Header::get (cpp/skyweaver/src/Header.cpp:26-70): the value of `key` at
 * the start of a header line; errors on a missing key or "unset". */
int sw_dada_header_get(const char* header, size_t header_size, const char* key,
                       char* value, size_t value_capacity);
/* read_dada_header (cpp/skyweaver/src/ObservationHeader.cpp:6-33). */
int sw_dada_parse_header(const char* header, size_t header_size,
                         sw_observation_header* out);
/* validate_header (cpp/skyweaver/src/ObservationHeader.cpp:35-62). */
int sw_dada_validate_header(const sw_observation_header* h, int nantennas,
                            int nchans, int npol);

/* MultiFileReader (cpp/skyweaver/src/MultiFileReader.cu:34-303): several
 * DADA files read as one contiguous payload (headers skipped), with the
 * optional OBS_OFFSET contiguity check; positions are payload bytes. */
typedef struct sw_dada_reader sw_dada_reader;
int sw_dada_reader_open(const char* const* files, int nfiles, size_t header_size,
                        int check_contiguity, sw_dada_reader** out);
void sw_dada_reader_close(sw_dada_reader* r);
int sw_dada_reader_header(const sw_dada_reader* r, int file_idx,
                          sw_observation_header* out);
size_t sw_dada_reader_total_bytes(const sw_dada_reader* r);
size_t sw_dada_reader_tell(const sw_dada_reader* r);
int sw_dada_reader_seek(sw_dada_reader* r, size_t payload_offset);
/* Reads up to `bytes` (fewer only at the end of the last file). */
int sw_dada_reader_read(sw_dada_reader* r, void* dst, size_t bytes,
                        size_t* nread);

/* FileStream (cpp/skyweaver/src/FileOutputStream.cpp:80-150): a payload
 * split over files of bytes_per_file payload bytes, each led by the header
 * (template + sw_dada_writer_set keys) with FILE_SIZE, FILE_NUMBER and
 * OBS_OFFSET updated, named <dir>/<base>_<offset %016zu><extension>. */
typedef struct sw_dada_writer sw_dada_writer;
int sw_dada_writer_open(const char* directory, const char* base_filename,
                        const char* extension, size_t bytes_per_file,
                        const char* header_template, size_t header_size,
                        sw_dada_writer** out);
int sw_dada_writer_set(sw_dada_writer* w, const char* key, const char* value);
int sw_dada_writer_write(sw_dada_writer* w, const void* data, size_t bytes);
int sw_dada_writer_close(sw_dada_writer* w);

/* ------------------------------------------------------------------ */
/* BeamformerPipeline                                                   */
/* ------------------------------------------------------------------ */
/* Replaces BeamformerPipeline<CBH,IBH,StatsH,BfTraits>
 * (cpp/skyweaver/BeamformerPipeline.cuh:48-67,
 *  cpp/skyweaver/detail/BeamformerPipeline.cu:44-301) with device-buffer
 * handlers: each gulp's stage chain is one CUDA graph. */
typedef struct sw_pipeline sw_pipeline;

typedef struct sw_pipeline_config {
    int nantennas;          /* padded antennas (multiple of 16, <= 64)  */
    int input_nantennas;    /* antennas present in TAFTP input           */
    int nchans;
    int nbeams;
    int gulp_samples;       /* multiple of 256                           */
    int tscrunch;           /* CB and IB tscrunch                        */
    int stokes;
    int ib_subtract;
    float output_level;
    double centre_frequency;
    double bandwidth;
    int ndms;               /* coherent DMs                              */
    const float* dms;       /* host array [ndms]                         */
    int fft_len;            /* 0 = automatic                             */
    int enable_coherent_dedispersion;
    int grouped;            /* 1 = batched persistent CB launch          */
    int use_graph;          /* 1 = capture the gulp chain as a graph     */
    int nbeamsets;
    const float* beamset_weights; /* host [nbeamsets][nantennas]         */
    const int* beamset_mapping;   /* host [nbeams]                       */
    int autotune;           /* 1 = sw_autotune picks fft_len (if 0) and the
                               beamformer work-item size                 */
    int cdd_lag;            /* coherent dedispersion: samples trimmed at the
                               end of each window, i.e. the output delay
                               (0 = 128); the start trim is the largest
                               intra-channel DM smear rounded up to 16   */
} sw_pipeline_config;

int sw_pipeline_create(const sw_pipeline_config* cfg, sw_pipeline** out);
int sw_pipeline_destroy(sw_pipeline* p);
/* Delay model (host float3 [nbeams][nant]) and its epoch. */
int sw_pipeline_set_delays(sw_pipeline* p, const float* h_delays,
                           double delay_epoch);
/* Run one gulp whose TAFTP input is already on the device. */
int sw_pipeline_process_device(sw_pipeline* p, const void* d_taftp,
                               double epoch, sw_stream_t stream);
/* Run one gulp from pinned host memory: H2D copy, chain, and D2H of the
 * coherent-beam output of every DM into h_cb_out (may be NULL); `stream`
 * waits for the D2H. */
int sw_pipeline_process_host(sw_pipeline* p, const void* h_taftp,
                             double epoch, void* h_cb_out,
                             sw_stream_t stream);
/* Device pointers to the last gulp's outputs (ordered on the stream given to
 * the process call; no host wait).  The outputs alternate between two buffer
 * sets, so they stay valid until the next-but-one gulp is processed. */
int sw_pipeline_outputs(sw_pipeline* p, int dm_idx, const int8_t** d_cb_tfb,
                        const float** d_ib_raw, const int8_t** d_ib_btf,
                        const float** d_stats);
/* Gulps processed so far. */
long sw_pipeline_gulp_count(const sw_pipeline* p);
/* The outputs of gulp number `gulp` (one of the last two processed), after a
 * host wait for that gulp's chain to finish on the device: a caller can hand
 * gulp g-1's beams to its handlers while gulp g computes (the reference
 * pipeline synchronises every gulp instead, detail/BeamformerPipeline.cu:
 * 265-301). */
int sw_pipeline_gulp_outputs(sw_pipeline* p, long gulp, int dm_idx,
                             const int8_t** d_cb_tfb, const float** d_ib_raw,
                             const int8_t** d_ib_btf, const float** d_stats);
/* Order the next gulp's chain after the work queued on `stream` so far (e.g.
 * a handler's copies of the outputs that gulp will overwrite: the outputs
 * alternate between two buffer sets). */
int sw_pipeline_order_after(sw_pipeline* p, sw_stream_t stream);
/* Host wait until the last gulp's pinned input has been copied to the device,
 * after which the caller may reuse that host buffer. */
int sw_pipeline_wait_input(sw_pipeline* p);
/* The last gulp's voltages that fed the beamformers for one DM: the
 * dedispersed FPACT rows (nsamples of the gulp from the row start, delayed
 * by the plan's lag), or the transposed gulp without coherent dedispersion
 * (the reference pipeline's _ftpa_dedispersed, detail/BeamformerPipeline.cu:
 * 190-205).  Valid until the next gulp is processed. */
int sw_pipeline_voltages(sw_pipeline* p, int dm_idx, const int8_t** d_fpact,
                         size_t* row_stride);
size_t sw_pipeline_cb_bytes_per_dm(const sw_pipeline* p);
/* The coherent-dedispersion plan: FFT length, overlap (history samples) and
 * lag (trim at each window's end = delay of the dedispersed output; the
 * outputs' utc_offset is lag / channel bandwidth).  Any pointer may be NULL. */
int sw_pipeline_fft_len(const sw_pipeline* p, int* fft_len, int* overlap,
                        int* lag);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* SKYWEAVER_B200_H */
