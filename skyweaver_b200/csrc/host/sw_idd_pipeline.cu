// IncoherentDedispersionPipeline with a device-resident AggregationBuffer
// (C ABI object behind sw_idd_pipeline_*).
//
// Reference: cpp/skyweaver/detail/IncoherentDedispersionPipeline.cu:6-113 and
// cpp/skyweaver/detail/AggregationBuffer.cu:23-117.  The reference copies
// every coherent-DM TFB block to host memory, aggregates it there and runs
// the OpenMP dedisperser on the host.  Here the aggregation buffer lives in
// HBM, pushes are device-to-device copies on the caller's stream, and each
// dispatch runs the incoherent dedispersion kernel on the buffer and hands the
// TDB result (device pointer) to the handler; nothing leaves the GPU.
//
// Buffer semantics follow AggregationBuffer exactly: (dispatch + overlap)
// slots of nchans * nbeams values; filling the last slot dispatches the whole
// buffer, after which the final `overlap` slots move to the front and filling
// resumes behind them.  The first dispatch therefore holds dispatch + overlap
// fresh slots, every later one `dispatch` new slots behind `overlap` old ones.
#include <algorithm>
#include <vector>

#include "../sw_common.cuh"

namespace swb {
namespace {

struct Block {
    int ndms = 0, max_delay = 0, tscrunch = 1, dispatch = 0;
    float scale = 1.0f;
    int* d_delays = nullptr;
    int8_t* d_agg = nullptr;  // (dispatch + max_delay) slots
    int8_t* d_tdb = nullptr;  // dispatch / tscrunch x ndms x nbeams
    size_t fill = 0;          // slots currently held
};

}  // namespace
}  // namespace swb

struct sw_idd_pipeline {
    int nchans = 0, nbeams = 0;
    size_t slot = 0;  // bytes per slot = nchans * nbeams
    std::vector<swb::Block> blocks;
    sw_idd_handler handler = nullptr;
    void* user = nullptr;

    ~sw_idd_pipeline()
    {
        for(auto& b : blocks) {
            cudaFree(b.d_delays);
            cudaFree(b.d_agg);
            cudaFree(b.d_tdb);
        }
    }

    int dispatch(int bi, cudaStream_t s)
    {
        swb::Block& b = blocks[bi];
        const int nsamp = b.dispatch + b.max_delay;
        SW_TRY(sw_incoherent_dedisperse(b.d_agg, nsamp, nchans, nbeams, b.d_delays, b.ndms,
                                        b.max_delay, b.tscrunch, b.scale, b.d_tdb,
                                        reinterpret_cast<sw_stream_t>(s)));
        if(handler)
            handler(user, bi, b.d_tdb, b.dispatch / b.tscrunch, b.ndms, nbeams,
                    reinterpret_cast<sw_stream_t>(s));
        b.fill = 0;
        if(b.max_delay > 0) {
            // dispatch >= max_delay, so source and destination never overlap
            SW_CUDA_CHECK(cudaMemcpyAsync(b.d_agg, b.d_agg + (size_t)b.dispatch * slot,
                                          (size_t)b.max_delay * slot, cudaMemcpyDeviceToDevice,
                                          s));
            b.fill = (size_t)b.max_delay;
        }
        return SW_OK;
    }

    int push(int bi, const int8_t* d_tfb, size_t nslots, cudaStream_t s)
    {
        swb::Block& b = blocks[bi];
        const size_t cap = (size_t)b.dispatch + b.max_delay;
        while(nslots > 0) {
            const size_t room = cap - b.fill;
            const size_t n = std::min(room, nslots);
            SW_CUDA_CHECK(cudaMemcpyAsync(b.d_agg + b.fill * slot, d_tfb, n * slot,
                                          cudaMemcpyDeviceToDevice, s));
            b.fill += n;
            d_tfb += n * slot;
            nslots -= n;
            if(b.fill == cap) SW_TRY(dispatch(bi, s));
        }
        return SW_OK;
    }
};

extern "C" {

int sw_idd_pipeline_create(int nchans, int nbeams, int nblocks, const int* h_ndms,
                           const int* const* h_delays, const int* h_tscrunch,
                           const float* h_scale, const int* h_dispatch,
                           sw_idd_handler handler, void* user, sw_idd_pipeline** out)
{
    SW_REQUIRE(out, "sw_idd_pipeline_create: null output handle");
    *out = nullptr;
    SW_REQUIRE(nchans > 0 && nbeams > 0 && nbeams % 4 == 0,
               "sw_idd_pipeline_create: nbeams (x Stokes components) must be a positive "
               "multiple of 4");
    SW_REQUIRE(nblocks > 0 && h_ndms && h_delays && h_tscrunch && h_scale,
               "sw_idd_pipeline_create: null block description");
    auto* p = new sw_idd_pipeline();
    p->nchans = nchans;
    p->nbeams = nbeams;
    p->slot = (size_t)nchans * nbeams;
    p->handler = handler;
    p->user = user;
    p->blocks.resize(nblocks);
    auto fail = [&](int rc) { delete p; return rc; };
    for(int i = 0; i < nblocks; ++i) {
        swb::Block& b = p->blocks[i];
        if(h_ndms[i] <= 0 || !h_delays[i] || h_tscrunch[i] <= 0) {
            swb::set_error("sw_idd_pipeline_create: block %d is empty", i);
            return fail(SW_ERR_INVALID);
        }
        b.ndms = h_ndms[i];
        b.tscrunch = h_tscrunch[i];
        b.scale = h_scale[i];
        std::vector<int> dl(h_delays[i], h_delays[i] + (size_t)b.ndms * nchans);
        b.max_delay = *std::max_element(dl.begin(), dl.end());
        if(*std::min_element(dl.begin(), dl.end()) < 0) {
            swb::set_error("sw_idd_pipeline_create: negative delay in block %d", i);
            return fail(SW_ERR_INVALID);
        }
        // IncoherentDedispersionPipeline.cu:28-30: max(10 x max delay, 8192),
        // rounded down to a multiple of tscrunch
        int disp = h_dispatch && h_dispatch[i] > 0 ? h_dispatch[i]
                                                   : std::max(b.max_delay * 10, 8192);
        disp -= disp % b.tscrunch;
        if(disp < b.max_delay || disp <= 0) {
            swb::set_error("sw_idd_pipeline_create: dispatch size %d of block %d is smaller "
                           "than its max delay %d", disp, i, b.max_delay);
            return fail(SW_ERR_INVALID);
        }
        b.dispatch = disp;
        if(cudaMalloc(&b.d_delays, dl.size() * sizeof(int)) != cudaSuccess ||
           cudaMalloc(&b.d_agg, (size_t)(disp + b.max_delay) * p->slot) != cudaSuccess ||
           cudaMalloc(&b.d_tdb, (size_t)(disp / b.tscrunch) * b.ndms * nbeams) != cudaSuccess) {
            swb::set_error("sw_idd_pipeline_create: device allocation failed for block %d", i);
            return fail(SW_ERR_CUDA);
        }
        if(cudaMemcpy(b.d_delays, dl.data(), dl.size() * sizeof(int), cudaMemcpyHostToDevice) !=
           cudaSuccess) {
            swb::set_error("sw_idd_pipeline_create: delay upload failed");
            return fail(SW_ERR_CUDA);
        }
    }
    *out = p;
    return SW_OK;
}

void sw_idd_pipeline_destroy(sw_idd_pipeline* p) { delete p; }

int sw_idd_pipeline_push(sw_idd_pipeline* p, int block, const int8_t* d_tfb, size_t nsamples,
                         sw_stream_t stream)
{
    SW_REQUIRE(p && d_tfb, "sw_idd_pipeline_push: null argument");
    SW_REQUIRE(block >= 0 && block < (int)p->blocks.size(), "sw_idd_pipeline_push: bad block");
    return p->push(block, d_tfb, nsamples, swb::as_cuda(stream));
}

int sw_idd_pipeline_geometry(const sw_idd_pipeline* p, int block, int* dispatch_size,
                             int* overlap, int* nsamples_out, int* ndms)
{
    SW_REQUIRE(p && block >= 0 && block < (int)p->blocks.size(),
               "sw_idd_pipeline_geometry: bad pipeline or block");
    const swb::Block& b = p->blocks[block];
    if(dispatch_size) *dispatch_size = b.dispatch;
    if(overlap) *overlap = b.max_delay;
    if(nsamples_out) *nsamples_out = b.dispatch / b.tscrunch;
    if(ndms) *ndms = b.ndms;
    return SW_OK;
}

}  // extern "C"
