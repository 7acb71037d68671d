// kp_noalloc.cu -- kp_batch_riaf_noalloc: the wavefront batch entry point with
// every piece of device scratch (job table, ray records, phase queues,
// counters) in one file-scope static __device__ array, so a call allocates
// nothing.  The kernels are the ones kp_batch_riaf launches; only where their
// scratch lives differs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "kp_launch.h"
#include "kpolaris_b200.h"

namespace kp {

// Helpers of the C-ABI unit (kp_capi.cu).
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);
int job_error(int code, int job);
ImageOutPtrs from_abi(const kp_image_out* o);
int check_outputs(const kp_image_out* out, int npix, int nfreq);
int validate_riaf(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs, int nfreq);
ImageConsts make_consts(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs, int nfreq,
                        int integrator);

namespace {

// Counters of one call, laid out as the batch engine expects them.
struct NoAllocCtrl {
    unsigned long long heads[kMaxWaveCycles * kPhases];
    unsigned counts[kMaxWaveCycles + 1][kPhases];
    int status;
};

struct NoAllocScratch {
    NoAllocCtrl ctrl;
    JobDesc jobs[KP_NOALLOC_MAX_JOBS];
    unsigned ids[kPhases][2][KP_NOALLOC_MAX_RAYS];
    unsigned sorted[KP_NOALLOC_MAX_RAYS];  // near-B queue in longest-first order
    unsigned lpt[512];                     // its bucket counters
    RayRecord pool[KP_NOALLOC_MAX_RAYS];
};

std::mutex g_symbol_mutex;
NoAllocScratch* g_scratch_ptr[64] = {};

}  // namespace
}  // namespace kp

// The scratch of every call on a device (32 MB: 464-byte records and seven id
// queues for KP_NOALLOC_MAX_RAYS rays, a job table of KP_NOALLOC_MAX_JOBS
// descriptors, the counters).  Reserved when this unit's module loads, and
// shared by every call on the device: calls that overlap in time race.
static __device__ __align__(256) unsigned char kp_noalloc_scratch[sizeof(kp::NoAllocScratch)];

namespace kp {

// Device address of the scratch, looked up once per device.  The lookup
// loads the module, which a stream capture would not allow: the first call
// on a device must come before any capture that includes this entry point.
static int scratch_for_device(int device, NoAllocScratch** out) {
    if (device < 0 || device >= 64) return set_error(KP_ERR_INVALID, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_symbol_mutex);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, kp_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_ptr[device] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_scratch_ptr[device];
    return KP_OK;
}

}  // namespace kp

using namespace kp;

extern "C" int kp_batch_riaf_noalloc(const kp_riaf_job* jobs, int njobs, const kp_run_options* options) {
    if (!options) return set_error(KP_ERR_INVALID, "kp_batch_riaf_noalloc needs options with device outputs");
    const kp_run_options opt = *options;
    if (njobs < 0 || (njobs > 0 && !jobs)) return set_error(KP_ERR_INVALID, "invalid job list");
    if (njobs == 0) return KP_OK;
    if (njobs > KP_NOALLOC_MAX_JOBS)
        return set_error(KP_ERR_INVALID, "kp_batch_riaf_noalloc: %d jobs exceed its static limit of %d", njobs,
                         KP_NOALLOC_MAX_JOBS);
    if (!opt.outputs_on_device)
        return set_error(KP_ERR_INVALID, "kp_batch_riaf_noalloc writes device outputs only (outputs_on_device = 1)");
    if (opt.precision != KP_PRECISION_FP64 && opt.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", opt.precision);
    if (opt.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4 && opt.integrator != KP_INTEGRATOR_CASH_KARP)
        return set_error(KP_ERR_INVALID, "unknown integrator %d", opt.integrator);
    if (opt.threads_per_block != 0)
        return set_error(KP_ERR_INVALID, "threads_per_block is fixed by the wavefront kernels (%d far, %d near): pass 0",
                         kFarThreads, kNearThreads);
    long long total = 0;
    int nf_max = 1;
    for (int i = 0; i < njobs; ++i) {
        const kp_riaf_job& jb = jobs[i];
        int st = validate_riaf(&jb.params, &jb.model, jb.frequencies, jb.nfreq);
        if (st != KP_OK) return job_error(st, i);
        if (jb.params.coordinate_system != KP_COORD_CARTESIAN_KS)
            return set_error(KP_ERR_UNSUPPORTED, "job %d: kp_batch_riaf_noalloc traces Cartesian Kerr-Schild images only", i);
        if (jb.radiation_substeps < 1)
            return set_error(KP_ERR_INVALID, "job %d: batch radiation_substeps must be positive", i);
        const int npix = jb.params.camera.nx * jb.params.camera.ny;
        st = check_outputs(&jb.out, npix, jb.nfreq);
        if (st != KP_OK) return job_error(st, i);
        total += npix;
        nf_max = std::max(nf_max, jb.nfreq);
    }
    if (total > KP_NOALLOC_MAX_RAYS)
        return set_error(KP_ERR_INVALID, "kp_batch_riaf_noalloc: %lld rays exceed its static scratch of %d rays",
                         total, KP_NOALLOC_MAX_RAYS);
    if (opt.precision == KP_PRECISION_MIXED) nf_max = KP_MAX_FREQUENCIES;

    cudaError_t e = cudaSetDevice(opt.device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    NoAllocScratch* S = nullptr;
    int st = scratch_for_device(opt.device, &S);
    if (st != KP_OK) return st;
    cudaStream_t stream = static_cast<cudaStream_t>(opt.stream);

    // job table: built on the host stack, copied into the static scratch
    JobDesc table[KP_NOALLOC_MAX_JOBS];
    long long ray = 0;
    for (int i = 0; i < njobs; ++i) {
        const kp_riaf_job& jb = jobs[i];
        JobDesc& d = table[i];
        std::memset(&d, 0, sizeof(d));
        d.c = make_consts(&jb.params, &jb.model, jb.frequencies, jb.nfreq, opt.integrator);
        double fr[5][4];
        host_camera_frame(d.c, fr);
        for (int mu = 0; mu < 4; ++mu) {
            d.frame.x.v[mu] = fr[0][mu];
            d.frame.e0.v[mu] = fr[1][mu];
            d.frame.e1.v[mu] = fr[2][mu];
            d.frame.e2.v[mu] = fr[3][mu];
            d.frame.e3.v[mu] = fr[4][mu];
        }
        d.out = from_abi(&jb.out);
        d.ray_begin = ray;
        d.npix = jb.params.camera.nx * jb.params.camera.ny;
        d.precision = opt.precision;
        ray += d.npix;
    }
    e = cudaMemcpyAsync(S->jobs, table, sizeof(JobDesc) * size_t(njobs), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_error(e, "job table upload");
    // the counters must start at zero; records and queues are written before they are read
    e = cudaMemsetAsync(&S->ctrl, 0, sizeof(NoAllocCtrl), stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync(counters)");

    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt.device);
    const bool mixed = opt.precision == KP_PRECISION_MIXED;
    int blocks[kPhases];
    for (int phase = 0; phase < kPhases; ++phase) {
        int per_sm = opt.blocks_per_sm;
        if (per_sm <= 0) {
            per_sm = mixed ? wave_occupancy_mixed(phase, wave_threads(phase))
                           : wave_occupancy_fp64(phase, nf_max, wave_threads(phase));
            if (per_sm <= 0) per_sm = 1;
        }
        blocks[phase] = std::max(1, sms) * per_sm;
        const long long needed = (total + wave_threads(phase) - 1) / wave_threads(phase);
        if (blocks[phase] > needed) blocks[phase] = int(needed);
    }
    for (int cycle = 0; cycle < kMaxWaveCycles; ++cycle) {
        for (int phase = 0; phase < kPhases; ++phase) {
            WaveDesc W;
            W.jobs = S->jobs;
            W.njobs = njobs;
            W.pool = S->pool;
            W.fresh_begin = 0;
            W.fresh_end = cycle == 0 && phase == kPhaseFar ? total : 0;
            W.in_ids = S->ids[phase][cycle % 2];
            W.in_count = &S->ctrl.counts[cycle][phase];
            W.in_head = &S->ctrl.heads[cycle * kPhases + phase];
            for (int q = 0; q < kPhases; ++q) {
                const int gen = q > phase ? cycle : cycle + 1;
                W.out_ids[q] = S->ids[q][gen % 2];
                W.out_count[q] = &S->ctrl.counts[gen][q];
            }
            W.budget = 0;
            W.status = &S->ctrl.status;
            W.job_done = nullptr;
            if (phase == kPhaseNearB) {
                // longest rays first, as kp_batch_riaf orders its near-B queue
                e = launch_lpt_order(W.in_ids, W.in_count, S->pool, S->lpt, S->sorted, std::max(1, sms), stream);
                if (e != cudaSuccess) return cuda_error(e, "near-B queue order");
                W.in_ids = S->sorted;
            }
            e = mixed ? launch_wave_mixed(phase, W, blocks[phase], wave_threads(phase), stream)
                      : launch_wave_fp64(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
            if (e != cudaSuccess) return cuda_error(e, "wavefront kernel launch");
        }
        unsigned left[kPhases] = {0, 0, 0};
        e = cudaMemcpyAsync(left, S->ctrl.counts[cycle + 1], sizeof(left), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "wavefront kernels");
        if (left[0] == 0 && left[1] == 0 && left[2] == 0) {
            int status_word = 0;
            e = cudaMemcpyAsync(&status_word, &S->ctrl.status, sizeof(int), cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_error(e, "status read");
            if (status_word == 2) return set_error(KP_ERR_TIMEOUT, "a lane exceeded the engine's iteration guard");
            if (status_word != 0)
                return set_error(KP_ERR_CUDA, "wavefront engine invariant violated (status %d)", status_word);
            return KP_OK;
        }
    }
    return set_error(KP_ERR_TIMEOUT, "rays still moving between phases after %d launches", kMaxWaveCycles * kPhases);
}
