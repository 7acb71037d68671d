// kp_server.cu -- the serving loop of include/kpolaris_b200.h: a device-owner
// thread runs the wavefront engine in bounded ticks over a resident pool of
// ray records, admitting jobs by HBM footprint as they arrive.
//
// Tick c: zero the counters of generation c + 1; seed the rays of the jobs
// admitted since the last tick into the far queue of generation c; launch
// far, near-A and near-B with a per-lane budget of RK jobs.  A launch of
// phase p pushes rays for a later phase into generation c and for its own or
// an earlier phase into generation c + 1, so every queue is complete before
// the launch that reads it.  Rays parked by the budget continue in tick c + 1.
// After the tick the host reads the per-job finished-ray counters and copies
// out the jobs whose rays have all finished.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kp_fmks.cuh"
#include "kp_grmhd_setup.h"
#include "kp_launch.h"
#include "kp_range_alloc.h"
#include "kpolaris_b200.h"

namespace kp {

int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);
int check_outputs(const kp_image_out* out, int npix, int nfreq);
int validate_riaf(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs, int nfreq);
int validate_grmhd(const kp_pass_a_params* params, const kp_grid* grid, const double* frequencies, int nfreq,
                   int radiation_substeps, int device);
ImageConsts make_consts(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs, int nfreq,
                        int integrator);
ImageOutPtrs carve_outputs(void* base, int npix, int nfreq);
size_t carved_bytes(int npix, int nfreq);
int copy_outputs_to_host(const ImageOutPtrs& d, const kp_image_out* h, int npix, int nfreq, cudaStream_t s);

namespace {

using Clock = std::chrono::steady_clock;
constexpr long long kOutUnit = 256;  // bytes per output-arena unit

// Scenes the server traces; each has its own phase queues.
enum : int { kServeRiaf = 0, kServeGrmhd = 1, kServeScenes = 2 };

struct ServerJob {
    unsigned long long ticket = 0;
    int scene = kServeRiaf;
    kp_riaf_job req;        // RIAF jobs
    kp_grmhd_job greq;      // GRMHD jobs
    kp_grid* grid = nullptr;  // held (grid_ref) until the job ends
    int nfreq = 1;
    kp_image_out out;
    int state = KP_JOB_PENDING;
    int status = KP_OK;
    bool cancel = false;
    int slot = -1;
    long long npix = 0;
    long long ray_base = -1;
    long long out_base = -1, out_units = 0;
    ImageOutPtrs dout;
    Clock::time_point t_submit, t_admit, t_done;
};

double seconds(Clock::duration d) { return std::chrono::duration<double>(d).count(); }

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * double(v.size() - 1);
    const size_t i = size_t(pos);
    const double f = pos - double(i);
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace
}  // namespace kp

using namespace kp;

struct kp_server {
    kp_server_config cfg;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<ServerJob>> pending;
    std::unordered_map<unsigned long long, std::shared_ptr<ServerJob>> jobs;
    std::vector<std::shared_ptr<ServerJob>> slots;
    unsigned long long next_ticket = 1;
    bool stop = false;
    std::thread worker;
    // statistics
    Clock::time_point t_created;
    long long submitted = 0, completed = 0, cancelled = 0, failed = 0, ticks = 0;
    long long max_rays_inflight = 0;
    int max_jobs_inflight = 0;
    double busy = 0.0;
    std::vector<double> latencies, queue_waits;
    // device state (worker thread only)
    cudaStream_t stream = nullptr;
    RayRecord* pool = nullptr;
    unsigned* ids[kServeScenes][kPhases][2] = {};
    unsigned* counts[kServeScenes] = {};           // per scene [2][kPhases]
    unsigned long long* heads[kServeScenes] = {};  // per scene [kPhases]
    long long scene_cycle[kServeScenes] = {};      // generation parity of each scene's queues
    unsigned* sorted = nullptr;                    // near-B queue in longest-first order (max_rays)
    unsigned* lpt = nullptr;                       // its bucket counters (512)
    int* status = nullptr;
    unsigned* done = nullptr;              // [max_jobs]
    JobDesc* d_jobs = nullptr;
    JobDesc* h_jobs = nullptr;             // pinned staging, one per slot
    SeedEntry* d_seed = nullptr;
    long long* d_prefix = nullptr;
    SeedEntry* h_seed = nullptr;           // pinned
    long long* h_prefix = nullptr;         // pinned
    unsigned* h_done = nullptr;            // pinned
    int* h_status = nullptr;               // pinned
    void* out_arena = nullptr;
    RangeAllocator rays, outs;
    int create_status = KP_OK;
};

namespace {

int footprint_units(const kp_pass_a_params& params, int nfreq, long long* rays, long long* out_units) {
    const long long npix = (long long)params.camera.nx * params.camera.ny;
    *rays = npix;
    *out_units = (long long)((carved_bytes(int(npix), nfreq) + kOutUnit - 1) / kOutUnit);
    return KP_OK;
}

// A job leaves the server (done, cancelled, failed or abandoned): drop its
// hold on the grid.  Callers hold s->mu or own the job alone.
void end_job(ServerJob& j) {
    if (j.grid) {
        grid_unref(j.grid, 1);
        j.grid = nullptr;
    }
}

void release_device(kp_server* s) {
    cudaFree(s->pool);
    cudaFree(s->sorted);
    cudaFree(s->lpt);
    for (int sc = 0; sc < kServeScenes; ++sc) {
        for (auto& q : s->ids[sc]) {
            cudaFree(q[0]);
            cudaFree(q[1]);
        }
        cudaFree(s->counts[sc]);
        cudaFree(s->heads[sc]);
    }
    cudaFree(s->status);
    cudaFree(s->done);
    cudaFree(s->d_jobs);
    cudaFree(s->d_seed);
    cudaFree(s->d_prefix);
    cudaFree(s->out_arena);
    cudaFreeHost(s->h_jobs);
    cudaFreeHost(s->h_seed);
    cudaFreeHost(s->h_prefix);
    cudaFreeHost(s->h_done);
    cudaFreeHost(s->h_status);
    if (s->stream) cudaStreamDestroy(s->stream);
}

int allocate_device(kp_server* s) {
    const kp_server_config& c = s->cfg;
    cudaError_t e = cudaSetDevice(c.device);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamCreate");
    auto dev = [&](void** p, size_t n) {
        if (e == cudaSuccess) e = cudaMalloc(p, n);
    };
    dev((void**)&s->pool, sizeof(RayRecord) * size_t(c.max_rays));
    dev((void**)&s->sorted, sizeof(unsigned) * size_t(c.max_rays));
    dev((void**)&s->lpt, sizeof(unsigned) * 512);
    for (int sc = 0; sc < kServeScenes; ++sc) {
        for (auto& q : s->ids[sc])
            for (auto& b : q) dev((void**)&b, sizeof(unsigned) * size_t(c.max_rays));
        dev((void**)&s->counts[sc], sizeof(unsigned) * 2 * kPhases);
        dev((void**)&s->heads[sc], sizeof(unsigned long long) * kPhases);
    }
    dev((void**)&s->status, sizeof(int));
    dev((void**)&s->done, sizeof(unsigned) * size_t(c.max_jobs));
    dev((void**)&s->d_jobs, sizeof(JobDesc) * size_t(c.max_jobs));
    dev((void**)&s->d_seed, sizeof(SeedEntry) * size_t(c.max_jobs));
    dev((void**)&s->d_prefix, sizeof(long long) * size_t(c.max_jobs + kServeScenes));
    dev(&s->out_arena, c.output_bytes);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_jobs, sizeof(JobDesc) * size_t(c.max_jobs));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_seed, sizeof(SeedEntry) * size_t(c.max_jobs));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_prefix, sizeof(long long) * size_t(c.max_jobs + kServeScenes));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_done, sizeof(unsigned) * size_t(c.max_jobs));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_status, sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(KP_ERR_OOM, "server allocation: %s", cudaGetErrorString(e));
    }
    e = cudaSuccess;
    for (int sc = 0; sc < kServeScenes && e == cudaSuccess; ++sc)
        e = cudaMemset(s->counts[sc], 0, sizeof(unsigned) * 2 * kPhases);
    if (e == cudaSuccess) e = cudaMemset(s->status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->done, 0, sizeof(unsigned) * size_t(c.max_jobs));
    if (e != cudaSuccess) return cuda_error(e, "server initialisation");
    s->rays.reset(c.max_rays);
    s->outs.reset((long long)(c.output_bytes / kOutUnit));
    s->slots.assign(size_t(c.max_jobs), nullptr);
    return KP_OK;
}

JobDesc job_desc(const kp_server* s, const ServerJob& j) {
    JobDesc d;
    std::memset(&d, 0, sizeof(d));
    if (j.scene == kServeGrmhd) {
        const kp_grmhd_job& g = j.greq;
        d.c = image_consts_fmks(&g.params, j.grid->model,
                                grid_consts_of(j.grid->model, j.grid->prims, j.grid->derived), g.frequencies, g.nfreq,
                                s->cfg.integrator);
        fmks_camera_frame(d.c.fmks, g.params.camera.radius, g.params.camera.inclination, d.frame.x, d.frame.e0,
                          d.frame.e1, d.frame.e2, d.frame.e3);
        if (s->cfg.precision == KP_PRECISION_MIXED) grmhd_emission_scale(&g.params, j.grid->model, d.c);
    } else {
        d.c = make_consts(&j.req.params, &j.req.model, j.req.frequencies, j.req.nfreq, s->cfg.integrator);
        double fr[5][4];
        host_camera_frame(d.c, fr);
        for (int mu = 0; mu < 4; ++mu) {
            d.frame.x.v[mu] = fr[0][mu];
            d.frame.e0.v[mu] = fr[1][mu];
            d.frame.e1.v[mu] = fr[2][mu];
            d.frame.e2.v[mu] = fr[3][mu];
            d.frame.e3.v[mu] = fr[4][mu];
        }
    }
    d.out = j.dout;
    d.ray_begin = j.ray_base;
    d.npix = int(j.npix);
    d.precision = s->cfg.precision;
    return d;
}

// Fails every job in flight (a device error ends the server's work).
void fail_inflight(kp_server* s, int status) {
    std::lock_guard<std::mutex> lock(s->mu);
    for (auto& j : s->slots) {
        if (!j) continue;
        j->state = KP_JOB_FAILED;
        j->status = status;
        ++s->failed;
        end_job(*j);
        j = nullptr;
    }
    for (auto& j : s->pending) {
        j->state = KP_JOB_FAILED;
        j->status = status;
        ++s->failed;
        end_job(*j);
    }
    s->pending.clear();
    s->stop = true;
    s->cv_done.notify_all();
}

void worker_main(kp_server* s) {
    cudaSetDevice(s->cfg.device);
    const bool mixed = s->cfg.precision == KP_PRECISION_MIXED;
    const int nf_max = KP_MAX_FREQUENCIES;  // one compiled form for every job
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->cfg.device);
    int blocks[kServeScenes][kPhases];
    for (int p = 0; p < kPhases; ++p) {
        const int th = wave_threads(p);
        const int riaf = mixed ? wave_occupancy_mixed(p, th) : wave_occupancy_fp64(p, nf_max, th);
        const int grmhd = mixed ? wave_occupancy_grmhd_mixed(p, nf_max, th) : wave_occupancy_grmhd(p, nf_max, th);
        blocks[kServeRiaf][p] = std::max(1, sms) * std::max(1, riaf);
        blocks[kServeGrmhd][p] = std::max(1, sms) * std::max(1, grmhd);
    }
    while (true) {
        // ---- admission (FIFO; the head of the queue waits for room)
        std::vector<std::shared_ptr<ServerJob>> admitted;
        bool any_inflight = false;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            for (;;) {
                any_inflight = std::any_of(s->slots.begin(), s->slots.end(), [](const auto& j) { return bool(j); });
                if (!s->pending.empty() || any_inflight || s->stop) break;
                s->cv_work.wait(lock);
            }
            if (s->stop) {
                // stopping: nothing new is started, and jobs in flight are
                // abandoned after the tick that was running
                for (auto& j : s->pending) {
                    j->state = KP_JOB_CANCELLED;
                    ++s->cancelled;
                    end_job(*j);
                }
                s->pending.clear();
                for (auto& j : s->slots) {
                    if (!j) continue;
                    j->state = KP_JOB_CANCELLED;
                    ++s->cancelled;
                    s->rays.release(j->ray_base, j->npix);
                    s->outs.release(j->out_base, j->out_units);
                    end_job(*j);
                    j = nullptr;
                }
                s->cv_done.notify_all();
                break;
            }
            while (!s->pending.empty()) {
                auto& j = s->pending.front();
                auto slot_it = std::find(s->slots.begin(), s->slots.end(), nullptr);
                if (slot_it == s->slots.end()) break;
                long long nr = 0, nu = 0;
                footprint_units(j->scene == kServeGrmhd ? j->greq.params : j->req.params, j->nfreq, &nr, &nu);
                const long long rb = s->rays.alloc(nr);
                if (rb < 0) break;
                const long long ob = s->outs.alloc(nu);
                if (ob < 0) {
                    s->rays.release(rb, nr);
                    break;
                }
                j->slot = int(slot_it - s->slots.begin());
                j->npix = nr;
                j->ray_base = rb;
                j->out_base = ob;
                j->out_units = nu;
                j->dout = carve_outputs(static_cast<char*>(s->out_arena) + ob * kOutUnit, int(nr), j->nfreq);
                j->state = KP_JOB_RUNNING;
                j->t_admit = Clock::now();
                *slot_it = j;
                admitted.push_back(j);
                s->pending.pop_front();
            }
            long long inflight_rays = 0;
            int inflight_jobs = 0;
            for (const auto& j : s->slots)
                if (j) {
                    inflight_rays += j->npix;
                    ++inflight_jobs;
                }
            s->max_rays_inflight = std::max(s->max_rays_inflight, inflight_rays);
            s->max_jobs_inflight = std::max(s->max_jobs_inflight, inflight_jobs);
            if (inflight_jobs == 0) continue;
        }
        const auto t_tick = Clock::now();
        cudaError_t e = cudaSuccess;
        // ---- upload the new jobs; seed their rays per scene (disjoint
        // ranges of the pinned staging, so no copy in flight is overwritten)
        int scene_jobs[kServeScenes] = {0, 0};
        {
            std::lock_guard<std::mutex> lock(s->mu);
            for (const auto& j : s->slots)
                if (j) ++scene_jobs[j->scene];
        }
        int seed_first[kServeScenes] = {0, 0}, seed_count[kServeScenes] = {0, 0};
        long long seeded[kServeScenes] = {0, 0};
        int nseed = 0;
        for (int sc = 0; sc < kServeScenes; ++sc) {
            seed_first[sc] = nseed;
            for (const auto& j : admitted) {
                if (j->scene != sc) continue;
                s->h_jobs[j->slot] = job_desc(s, *j);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(s->d_jobs + j->slot, s->h_jobs + j->slot, sizeof(JobDesc),
                                        cudaMemcpyHostToDevice, s->stream);
                if (e == cudaSuccess) e = cudaMemsetAsync(s->done + j->slot, 0, sizeof(unsigned), s->stream);
                s->h_seed[nseed] = SeedEntry{j->slot, int(j->npix), j->ray_base};
                s->h_prefix[nseed + sc] = seeded[sc];
                seeded[sc] += j->npix;
                ++nseed;
                ++seed_count[sc];
            }
            s->h_prefix[nseed + sc] = seeded[sc];
        }
        if (nseed > 0) {
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->d_seed, s->h_seed, sizeof(SeedEntry) * size_t(nseed), cudaMemcpyHostToDevice,
                                    s->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(s->d_prefix, s->h_prefix, sizeof(long long) * size_t(nseed + kServeScenes),
                                    cudaMemcpyHostToDevice, s->stream);
        }
        // ---- one cycle of the three phases for each scene with jobs in flight;
        // each scene's queues alternate with its own tick count
        for (int sc = 0; sc < kServeScenes && e == cudaSuccess; ++sc) {
            if (scene_jobs[sc] == 0) continue;
            const long long cycle = s->scene_cycle[sc];
            const int cur = int(cycle % 2), nxt = int((cycle + 1) % 2);
            unsigned* cnt = s->counts[sc];
            if (e == cudaSuccess) e = cudaMemsetAsync(cnt + nxt * kPhases, 0, sizeof(unsigned) * kPhases, s->stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(s->heads[sc], 0, sizeof(unsigned long long) * kPhases, s->stream);
            if (seed_count[sc] > 0 && e == cudaSuccess) {
                const SeedEntry* ents = s->d_seed + seed_first[sc];
                const long long* pre = s->d_prefix + seed_first[sc] + sc;
                if (sc == kServeGrmhd)
                    e = (mixed ? launch_seed_grmhd_mixed : launch_seed_grmhd)(
                        s->d_jobs, ents, pre, seed_count[sc], seeded[sc], s->pool, s->ids[sc][kPhaseFar][cur],
                        cnt + cur * kPhases + kPhaseFar, s->stream);
                else if (mixed)
                    e = launch_seed_mixed(s->d_jobs, ents, pre, seed_count[sc], seeded[sc], s->pool,
                                          s->ids[sc][kPhaseFar][cur], cnt + cur * kPhases + kPhaseFar, s->stream);
                else
                    e = launch_seed_fp64(s->d_jobs, ents, pre, seed_count[sc], seeded[sc], s->pool,
                                         s->ids[sc][kPhaseFar][cur], cnt + cur * kPhases + kPhaseFar, s->stream);
            }
            for (int p = 0; p < kPhases && e == cudaSuccess; ++p) {
                WaveDesc W;
                W.jobs = s->d_jobs;
                W.njobs = s->cfg.max_jobs;
                W.pool = s->pool;
                W.fresh_begin = 0;
                W.fresh_end = 0;
                W.in_ids = s->ids[sc][p][cur];
                W.in_count = cnt + cur * kPhases + p;
                W.in_head = s->heads[sc] + p;
                for (int q = 0; q < kPhases; ++q) {
                    const int g = q > p ? cur : nxt;
                    W.out_ids[q] = s->ids[sc][q][g];
                    W.out_count[q] = cnt + g * kPhases + q;
                }
                W.budget = s->cfg.tick_budget;
                W.status = s->status;
                W.job_done = s->done;
                if (p == kPhaseNearB) {
                    // longest rays first (kp_reorder.cu)
                    e = launch_lpt_order(W.in_ids, W.in_count, s->pool, s->lpt, s->sorted, sms, s->stream);
                    if (e != cudaSuccess) break;
                    W.in_ids = s->sorted;
                }
                const int b = blocks[sc][p], th = wave_threads(p);
                if (sc == kServeGrmhd)
                    e = mixed ? launch_wave_grmhd_mixed(p, W, nf_max, b, th, s->stream)
                              : launch_wave_grmhd(p, W, nf_max, b, th, s->stream);
                else
                    e = mixed ? launch_wave_mixed(p, W, b, th, s->stream)
                              : launch_wave_fp64(p, W, nf_max, b, th, s->stream);
            }
            s->scene_cycle[sc] = cycle + 1;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->h_done, s->done, sizeof(unsigned) * size_t(s->cfg.max_jobs),
                                cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->h_status, s->status, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) {
            fail_inflight(s, cuda_error(e, "serving tick"));
            break;
        }
        if (*s->h_status != 0) {
            fail_inflight(s, set_error(*s->h_status == 2 ? KP_ERR_TIMEOUT : KP_ERR_CUDA,
                                       "wavefront engine status %d", *s->h_status));
            break;
        }
        // ---- completions
        std::vector<std::shared_ptr<ServerJob>> finished;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            for (const auto& j : s->slots)
                if (j && (long long)s->h_done[j->slot] >= j->npix) finished.push_back(j);
        }
        for (const auto& j : finished) {
            if (!j->cancel) {
                int st = copy_outputs_to_host(j->dout, &j->out, int(j->npix), j->nfreq, s->stream);
                if (st == KP_OK) {
                    e = cudaStreamSynchronize(s->stream);
                    if (e != cudaSuccess) st = cuda_error(e, "result copy");
                }
                j->status = st;
            }
        }
        {
            std::lock_guard<std::mutex> lock(s->mu);
            const auto now = Clock::now();
            for (const auto& j : finished) {
                s->slots[size_t(j->slot)] = nullptr;
                s->rays.release(j->ray_base, j->npix);
                s->outs.release(j->out_base, j->out_units);
                end_job(*j);
                j->t_done = now;
                if (j->cancel) {
                    j->state = KP_JOB_CANCELLED;
                    ++s->cancelled;
                } else if (j->status != KP_OK) {
                    j->state = KP_JOB_FAILED;
                    ++s->failed;
                } else {
                    j->state = KP_JOB_DONE;
                    ++s->completed;
                    s->latencies.push_back(seconds(j->t_done - j->t_submit));
                    s->queue_waits.push_back(seconds(j->t_admit - j->t_submit));
                }
            }
            ++s->ticks;
            s->busy += seconds(Clock::now() - t_tick);
            if (!finished.empty()) s->cv_done.notify_all();
        }
    }
}

}  // namespace

extern "C" {

void kp_default_server_config(kp_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->precision = KP_PRECISION_MIXED;
    c->integrator = KP_INTEGRATOR_STEP_DOUBLING_RK4;
    c->max_rays = 4ll << 20;
    c->output_bytes = size_t(1) << 30;
    c->max_jobs = 64;
    c->tick_budget = 128;
}

int kp_server_create(const kp_server_config* cfg, kp_server** out) {
    if (!out) return set_error(KP_ERR_INVALID, "kp_server_create: null output handle");
    *out = nullptr;
    kp_server_config c;
    if (cfg) {
        c = *cfg;
    } else {
        kp_default_server_config(&c);
    }
    if (c.precision != KP_PRECISION_FP64 && c.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", c.precision);
    if (c.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4 && c.integrator != KP_INTEGRATOR_CASH_KARP)
        return set_error(KP_ERR_INVALID, "unknown integrator %d", c.integrator);
    if (c.max_rays <= 0 || c.max_rays > (1ll << 31) || c.max_jobs <= 0 || c.max_jobs > 4096 || c.tick_budget <= 0 ||
        c.output_bytes < size_t(kOutUnit))
        return set_error(KP_ERR_INVALID, "invalid server configuration");
    auto* s = new kp_server();
    s->cfg = c;
    s->t_created = Clock::now();
    const int st = allocate_device(s);
    if (st != KP_OK) {
        release_device(s);
        delete s;
        return st;
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return KP_OK;
}

}  // extern "C"

namespace {

int enqueue(kp_server* s, const std::shared_ptr<ServerJob>& j, unsigned long long* ticket) {
    j->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) return set_error(KP_ERR_INVALID, "server is stopping");
        j->ticket = s->next_ticket++;
        s->jobs[j->ticket] = j;
        s->pending.push_back(j);
        ++s->submitted;
    }
    s->cv_work.notify_one();
    *ticket = j->ticket;
    return KP_OK;
}

}  // namespace

extern "C" {

int kp_server_submit(kp_server* s, const kp_riaf_job* job, unsigned long long* ticket) {
    if (!s || !job || !ticket) return set_error(KP_ERR_INVALID, "kp_server_submit: null argument");
    int st = validate_riaf(&job->params, &job->model, job->frequencies, job->nfreq);
    if (st != KP_OK) return st;
    if (job->params.coordinate_system != KP_COORD_CARTESIAN_KS)
        return set_error(KP_ERR_UNSUPPORTED, "the serving loop traces Cartesian Kerr-Schild RIAF images only");
    if (job->radiation_substeps < 1) return set_error(KP_ERR_INVALID, "radiation_substeps must be positive");
    const int npix = job->params.camera.nx * job->params.camera.ny;
    st = check_outputs(&job->out, npix, job->nfreq);
    if (st != KP_OK) return st;
    long long nr = 0, nu = 0;
    footprint_units(job->params, job->nfreq, &nr, &nu);
    if (nr > s->cfg.max_rays || nu * kOutUnit > (long long)s->cfg.output_bytes)
        return set_error(KP_ERR_INVALID, "job footprint (%lld rays, %lld output bytes) exceeds the server's capacity",
                         nr, nu * kOutUnit);
    auto j = std::make_shared<ServerJob>();
    j->scene = kServeRiaf;
    j->req = *job;
    j->nfreq = job->nfreq;
    j->out = job->out;
    return enqueue(s, j, ticket);
}

int kp_server_submit_grmhd(kp_server* s, const kp_grmhd_job* job, unsigned long long* ticket) {
    if (!s || !job || !ticket || !job->grid) return set_error(KP_ERR_INVALID, "kp_server_submit_grmhd: null argument");
    int st = validate_grmhd(&job->params, job->grid, job->frequencies, job->nfreq, job->radiation_substeps,
                            s->cfg.device);
    if (st != KP_OK) return st;
    const int npix = job->params.camera.nx * job->params.camera.ny;
    st = check_outputs(&job->out, npix, job->nfreq);
    if (st != KP_OK) return st;
    long long nr = 0, nu = 0;
    footprint_units(job->params, job->nfreq, &nr, &nu);
    if (nr > s->cfg.max_rays || nu * kOutUnit > (long long)s->cfg.output_bytes)
        return set_error(KP_ERR_INVALID, "job footprint (%lld rays, %lld output bytes) exceeds the server's capacity",
                         nr, nu * kOutUnit);
    auto j = std::make_shared<ServerJob>();
    j->scene = kServeGrmhd;
    j->greq = *job;
    j->nfreq = job->nfreq;
    j->out = job->out;
    j->grid = const_cast<kp_grid*>(job->grid);
    grid_ref(j->grid);
    st = enqueue(s, j, ticket);
    if (st != KP_OK) end_job(*j);
    return st;
}

int kp_server_poll(kp_server* s, unsigned long long ticket, int* state) {
    if (!s || !state) return set_error(KP_ERR_INVALID, "kp_server_poll: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return set_error(KP_ERR_NOT_FOUND, "unknown ticket %llu", ticket);
    *state = it->second->state;
    return KP_OK;
}

int kp_server_wait(kp_server* s, unsigned long long ticket, double timeout_seconds) {
    if (!s) return set_error(KP_ERR_INVALID, "kp_server_wait: null server");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return set_error(KP_ERR_NOT_FOUND, "unknown ticket %llu", ticket);
    auto j = it->second;
    const auto final_state = [&] { return j->state >= KP_JOB_DONE; };
    if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(std::max(0.0, timeout_seconds)), final_state))
        return set_error(KP_ERR_TIMEOUT, "job %llu not finished after %g s", ticket, timeout_seconds);
    if (j->state == KP_JOB_CANCELLED) return set_error(KP_ERR_CANCELLED, "job %llu was cancelled", ticket);
    if (j->state == KP_JOB_FAILED) return j->status != KP_OK ? j->status : set_error(KP_ERR_CUDA, "job failed");
    return KP_OK;
}

int kp_server_cancel(kp_server* s, unsigned long long ticket) {
    if (!s) return set_error(KP_ERR_INVALID, "kp_server_cancel: null server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return set_error(KP_ERR_NOT_FOUND, "unknown ticket %llu", ticket);
    auto j = it->second;
    if (j->state == KP_JOB_PENDING) {
        s->pending.erase(std::find(s->pending.begin(), s->pending.end(), j));
        j->state = KP_JOB_CANCELLED;
        ++s->cancelled;
        end_job(*j);
        s->cv_done.notify_all();
    } else if (j->state == KP_JOB_RUNNING) {
        j->cancel = true;
    }
    return KP_OK;
}

int kp_server_get_stats(kp_server* s, kp_server_stats* out) {
    if (!s || !out) return set_error(KP_ERR_INVALID, "kp_server_get_stats: null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->cancelled = s->cancelled;
    out->failed = s->failed;
    out->ticks = s->ticks;
    out->max_inflight_rays = s->max_rays_inflight;
    out->max_inflight_jobs = s->max_jobs_inflight;
    out->wall_seconds = seconds(Clock::now() - s->t_created);
    out->busy_seconds = s->busy;
    out->latency_p50 = percentile(s->latencies, 0.50);
    out->latency_p99 = percentile(s->latencies, 0.99);
    out->latency_max = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
    out->queue_p50 = percentile(s->queue_waits, 0.50);
    return KP_OK;
}

int kp_server_destroy(kp_server* s) {
    if (!s) return KP_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->cfg.device);
    release_device(s);
    delete s;
    return KP_OK;
}

}  // extern "C"
