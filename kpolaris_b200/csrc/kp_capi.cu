// kp_capi.cu -- host side of the C ABI declared in include/kpolaris_b200.h:
// argument validation with the reference's error semantics, per-image
// constant resolution, device buffers, launches and copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <vector>

#include "kp_fmks.cuh"
#include "kp_grmhd.cuh"
#include "kp_grmhd_setup.h"
#include "kp_launch.h"
#include "kpolaris_b200.h"

namespace {

thread_local char g_error[1024] = "";

}  // namespace

namespace kp {

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return code;
}

// Prefixes the current error message with the index of the job it concerns
// (the message is copied first: it is the buffer being formatted into).
int job_error(int code, int job) {
    char msg[sizeof(g_error)];
    std::memcpy(msg, g_error, sizeof(msg));
    msg[sizeof(msg) - 1] = '\0';
    return set_error(code, "job %d: %s", job, msg);
}

int cuda_error(cudaError_t e, const char* what) {
    return set_error(KP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// engine families (scene x policy) of run_wave_jobs
enum : int {
    kFamilyRiafFP64 = 0,
    kFamilyRiafMixed = 1,
    kFamilyGrmhdFP64 = 2,
    kFamilyGrmhdMixed = 3,
    kFamilyGrmhdSlowFP64 = 4,
    kFamilyGrmhdSlowMixed = 5,
    kFamilyRiafBLFP64 = 6,
    kFamilyRiafBLMixed = 7,
    kFamilyCount = 8
};
constexpr int kDefaultGraphCycles = 3;
constexpr size_t kGraphCacheSize = 8;

// Device-side counters of one batch, zeroed before its first launch.  The
// queue a phase reads in its g-th launch is generation g of that phase:
// counts[g][phase] entries of ids[phase][g % 2].  A launch of cycle c pushes
// a ray for a phase that comes later in the cycle into generation c, for its
// own or an earlier phase into generation c + 1.
struct WaveCtrl {
    unsigned long long heads[kMaxWaveCycles * kPhases];
    unsigned counts[kMaxWaveCycles + 1][kPhases];
    int status;
};

// Per-device library state: a non-blocking stream and grow-only output
// buffers reused across calls.
struct DeviceState {
    int initialised = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    void* out_buf = nullptr;
    size_t out_bytes = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // persistent launches
    JobDesc* d_jobs = nullptr;      // device job table (grow-only)
    JobDesc* h_jobs = nullptr;      // pinned staging of the job table
    int jobs_cap = 0;
    cudaEvent_t staging_free = nullptr;  // last upload from h_jobs has completed
    WaveCtrl* d_ctrl = nullptr;     // queue counters and the status word
    RayRecord* d_pool = nullptr;    // parked ray records, one per ray (grow-only)
    unsigned* d_ids[kPhases][2] = {};  // id queues per phase, by generation parity
    long long pool_cap = 0;
    unsigned* h_left = nullptr;     // pinned: queue counts after a cycle
    unsigned* d_sorted = nullptr;   // near-B queue in longest-first order (pool_cap)
    unsigned* d_lpt = nullptr;      // its bucket counters (2 x 256)
    void* d_series = nullptr;       // slow light: snapshot table and times (grow-only)
    size_t series_bytes = 0;
    // schedule tuning per engine family (kp_autotune_batch): CTAs per SM of
    // each phase kernel (0: occupancy-derived) and cycles per graph launch
    int tuned_per_sm[kFamilyCount][kPhases] = {};
    int tuned_cycles[kFamilyCount] = {};
    // instantiated launch graphs (KP_SCHEDULE_GRAPH), keyed by everything
    // they bake in; the oldest is dropped beyond kGraphCacheSize
    struct GraphEntry {
        int family, nf_max, njobs, cycles;
        long long total;
        int blocks[kPhases];
        const void* jobs;
        const void* pool;
        const void* ctrl;
        const void* ids[kPhases][2];
        const void* sorted;
        const void* lpt;
        cudaGraphExec_t exec;
    };
    std::vector<GraphEntry> graphs;
    cudaEvent_t ev_launch[kMaxWaveCycles * kPhases + 1] = {};  // per-launch timing
};

static std::mutex g_mutex;
static DeviceState g_dev[64];

DeviceState* device_state(int device, int* status) {
    if (device < 0 || device >= 64) {
        *status = set_error(KP_ERR_INVALID, "device ordinal %d out of range", device);
        return nullptr;
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        *status = cuda_error(e, "cudaSetDevice");
        return nullptr;
    }
    DeviceState& d = g_dev[device];
    if (!d.initialised) {
        e = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            *status = cuda_error(e, "cudaStreamCreate");
            return nullptr;
        }
        cudaEventCreate(&d.ev0);
        cudaEventCreate(&d.ev1);
        cudaEventCreateWithFlags(&d.staging_free, cudaEventDisableTiming);
        for (auto& ev : d.ev_launch) cudaEventCreate(&ev);
        cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
        e = cudaMalloc(&d.d_ctrl, sizeof(WaveCtrl));
        if (e != cudaSuccess) {
            *status = cuda_error(e, "cudaMalloc(wave counters)");
            return nullptr;
        }
        e = cudaMallocHost(&d.h_left, sizeof(unsigned) * kPhases);
        if (e != cudaSuccess) {
            *status = cuda_error(e, "cudaMallocHost(queue count)");
            return nullptr;
        }
        d.initialised = 1;
    }
    *status = KP_OK;
    return &d;
}

void* device_output_buffer(DeviceState* d, size_t bytes, int* status) {
    if (bytes > d->out_bytes) {
        if (d->out_buf) cudaFree(d->out_buf);
        d->out_buf = nullptr;
        d->out_bytes = 0;
        cudaError_t e = cudaMalloc(&d->out_buf, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *status = set_error(KP_ERR_OOM, "cudaMalloc(%zu bytes) for image outputs: %s", bytes,
                                cudaGetErrorString(e));
            return nullptr;
        }
        d->out_bytes = bytes;
    }
    *status = KP_OK;
    return d->out_buf;
}

// Carves a kp_image_out-shaped set of device arrays out of one buffer.
ImageOutPtrs carve_outputs(void* base, int npix, int nfreq) {
    char* p = static_cast<char*>(base);
    auto take_d = [&](size_t n) {
        double* r = reinterpret_cast<double*>(p);
        p += ((n * sizeof(double) + 255) / 256) * 256;
        return r;
    };
    auto take_i = [&](size_t n) {
        int32_t* r = reinterpret_cast<int32_t*>(p);
        p += ((n * sizeof(int32_t) + 255) / 256) * 256;
        return r;
    };
    const size_t img = size_t(npix) * size_t(nfreq);
    ImageOutPtrs o;
    o.image_i = take_d(img);
    o.image_q = take_d(img);
    o.image_u = take_d(img);
    o.image_v = take_d(img);
    o.closure_x = take_d(npix);
    o.closure_k = take_d(npix);
    o.final_null = take_d(npix);
    o.frame_error = take_d(npix);
    o.det_r = take_d(npix);
    o.r11 = take_d(npix);
    o.r12 = take_d(npix);
    o.r21 = take_d(npix);
    o.r22 = take_d(npix);
    o.basis_identity_error = take_d(npix);
    o.basis_rotation_angle = take_d(npix);
    o.pass_a_steps = take_i(npix);
    o.steps = take_i(npix);
    o.reason = take_i(npix);
    return o;
}

size_t carved_bytes(int npix, int nfreq) {
    const size_t img = ((size_t(npix) * size_t(nfreq) * 8 + 255) / 256) * 256;
    const size_t dpix = ((size_t(npix) * 8 + 255) / 256) * 256;
    const size_t ipix = ((size_t(npix) * 4 + 255) / 256) * 256;
    return 4 * img + 11 * dpix + 3 * ipix;
}

ImageOutPtrs from_abi(const kp_image_out* o) {
    ImageOutPtrs p;
    p.image_i = o->image_i;
    p.image_q = o->image_q;
    p.image_u = o->image_u;
    p.image_v = o->image_v;
    p.closure_x = o->closure_x;
    p.closure_k = o->closure_k;
    p.final_null = o->final_null;
    p.frame_error = o->frame_error;
    p.det_r = o->det_r;
    p.r11 = o->overlap_r11;
    p.r12 = o->overlap_r12;
    p.r21 = o->overlap_r21;
    p.r22 = o->overlap_r22;
    p.basis_identity_error = o->basis_identity_error;
    p.basis_rotation_angle = o->basis_rotation_angle;
    p.pass_a_steps = o->pass_a_steps;
    p.steps = o->steps;
    p.reason = o->reason;
    return p;
}

int check_outputs(const kp_image_out* out, int npix, int nfreq) {
    if (!out) return set_error(KP_ERR_INVALID, "null output struct");
    if (out->npix != npix || out->nfreq != nfreq)
        return set_error(KP_ERR_INVALID, "output holds npix=%d nfreq=%d, image needs npix=%d nfreq=%d",
                         out->npix, out->nfreq, npix, nfreq);
    const void* ptrs[] = {out->image_i, out->image_q, out->image_u, out->image_v, out->closure_x,
                          out->closure_k, out->final_null, out->frame_error, out->det_r,
                          out->overlap_r11, out->overlap_r12, out->overlap_r21, out->overlap_r22,
                          out->basis_identity_error, out->basis_rotation_angle, out->pass_a_steps,
                          out->steps, out->reason};
    for (const void* p : ptrs)
        if (!p) return set_error(KP_ERR_INVALID, "null output array");
    return KP_OK;
}

int copy_outputs_to_host(const ImageOutPtrs& d, const kp_image_out* h, int npix, int nfreq,
                         cudaStream_t s) {
    const size_t img = size_t(npix) * size_t(nfreq) * sizeof(double);
    const size_t dp = size_t(npix) * sizeof(double);
    const size_t ip = size_t(npix) * sizeof(int32_t);
    struct Item {
        void* dst;
        const void* src;
        size_t n;
    } items[] = {
        {h->image_i, d.image_i, img},          {h->image_q, d.image_q, img},
        {h->image_u, d.image_u, img},          {h->image_v, d.image_v, img},
        {h->closure_x, d.closure_x, dp},       {h->closure_k, d.closure_k, dp},
        {h->final_null, d.final_null, dp},     {h->frame_error, d.frame_error, dp},
        {h->det_r, d.det_r, dp},               {h->overlap_r11, d.r11, dp},
        {h->overlap_r12, d.r12, dp},           {h->overlap_r21, d.r21, dp},
        {h->overlap_r22, d.r22, dp},           {h->basis_identity_error, d.basis_identity_error, dp},
        {h->basis_rotation_angle, d.basis_rotation_angle, dp},
        {h->pass_a_steps, d.pass_a_steps, ip}, {h->steps, d.steps, ip},
        {h->reason, d.reason, ip},
    };
    for (const Item& it : items) {
        cudaError_t e = cudaMemcpyAsync(it.dst, it.src, it.n, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync(device to host)");
    }
    return KP_OK;
}

// isco_radius (src/model/riaf.hpp:166-174), evaluated on the host with libm.
double isco_radius(double spin) {
    const double a = spin;
    const double one = 1.0;
    const double z1 = one + std::cbrt(one - a * a) * (std::cbrt(one + a) + std::cbrt(one - a));
    const double z2 = std::sqrt(3.0 * a * a + z1 * z1);
    const double sign = a < 0.0 ? -1.0 : 1.0;
    return 3.0 + z2 - sign * std::sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
}

// Exponent E of the FP32 emission scale 2^E of one frequency (mixed path).
// The invariant emissivity j ~ n_e e^2 nu_c / (c nu^2) is 1e-38..1e-48 in CGS,
// below FP32 range; E is chosen so that the emission of one radiation step
// at a reference plasma point (r = max(r_min, 3), equator, unit shape
// factor bound 30) is 2^-6.  The transfer equation is linear in (j, S), so
// the image is exactly rescaled by 2^-E in FP64 at the end.
int emission_scale_exponent(const kp_pass_a_params* p, const kp_riaf_model* m, double freq, double dls) {
    const double kPiD = 3.141592653589793, ee = 4.803204712570263e-10, me = 9.1093837015e-28,
                 cl = 2.99792458e10, mp = 1.67262192369e-24, kbol = 1.380649e-16;
    const double r_ref = std::max(m->r_min, 3.0);
    const double ne = std::max(m->ne_unit * m->nth0 * std::pow(r_ref, m->pow_nth), 1e-30);
    const double b = std::sqrt(8.0 * kPiD * 0.1 * ne * mp * cl * cl / (6.0 * r_ref));
    const double nu_c = ee * b / (2.0 * kPiD * me * cl);
    const double j_phys = ne * ee * ee * nu_c / cl * (std::sqrt(2.0) * kPiD / 27.0) * 30.0;
    const double j_inv = j_phys / std::max(freq * freq, 1.0);
    const double step = p->max_radiation_step > 0.0 ? p->max_radiation_step : std::max(p->max_step, 1e-3);
    const double dl = std::max(step * std::fabs(dls), 1e-300);
    (void)kbol;
    double e = std::floor(std::log2(std::ldexp(1.0, -6) / std::max(j_inv * dl, 1e-300)));
    if (!(e == e)) e = 0.0;
    return int(std::min(120.0, std::max(-120.0, e)));
}

int validate_riaf(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs, int nfreq) {
    if (!p || !m) return set_error(KP_ERR_INVALID, "null params or model");
    if (p->camera.nx <= 0 || p->camera.ny <= 0 || p->camera.nx > 2147483647 / p->camera.ny)
        return set_error(KP_ERR_INVALID, "image dimensions must have a positive int-sized product");
    if (nfreq < 1 || nfreq > KP_MAX_FREQUENCIES)
        return set_error(KP_ERR_INVALID,
                         "multifrequency image chunk size must be between 1 and KP_MAX_FREQUENCIES (%d)",
                         KP_MAX_FREQUENCIES);
    if (nfreq > 1 && !freqs) return set_error(KP_ERR_INVALID, "null frequency list");
    switch (p->coordinate_system) {
    case KP_COORD_CARTESIAN_KS: break;
    case KP_COORD_BOYER_LINDQUIST: break;
    case KP_COORD_SPHERICAL_KS:
        return set_error(KP_ERR_UNSUPPORTED, "RIAF image coordinate backend not built: spherical_ks");
    case KP_COORD_FMKS:
        return set_error(KP_ERR_UNSUPPORTED, "RIAF image coordinate backend not built: fmks");
    case KP_COORD_MKS:
        return set_error(KP_ERR_UNSUPPORTED, "RIAF image coordinate backend not built: mks");
    default:
        return set_error(KP_ERR_UNSUPPORTED, "RIAF image coordinate backend not built: unknown");
    }
    if (p->camera.model != KP_CAMERA_PINHOLE)
        return set_error(KP_ERR_UNSUPPORTED, "only the pinhole camera is built for the GPU image path");
    if (p->direct_only) return set_error(KP_ERR_UNSUPPORTED, "direct_only transport is not built");
    if (p->emission_selection.equatorial_h_over_r > 0.0 && p->emission_selection.equatorial_h_over_r < 1.0)
        return set_error(KP_ERR_UNSUPPORTED, "narrow equatorial emission wedge is not built");
    if (m->emission_type != KP_FIT_PANDYA && m->emission_type != KP_FIT_DEXTER)
        return set_error(KP_ERR_UNSUPPORTED,
                         "emission_type %d: only thermal synchrotron (1 Pandya, 4 Dexter) is built",
                         m->emission_type);
    if (p->max_steps < 0) return set_error(KP_ERR_INVALID, "max_steps must be non-negative");
    return KP_OK;
}

// GM/c^2 in cm of the RIAF model's mass (riaf.hpp:76-81).
double riaf_length_unit(const kp_riaf_model* m) {
    const double gnewt = 6.67430e-8, msun = 1.98847e33, cl = 2.99792458e10;
    return gnewt * m->mbh_solar * msun / (cl * cl);
}

// Resolves one image's launch constants on the host.
ImageConsts make_consts(const kp_pass_a_params* p, const kp_riaf_model* m, const double* freqs,
                        int nfreq, int integrator) {
    ImageConsts c;
    std::memset(&c, 0, sizeof(c));
    c.mass = p->mass;
    c.spin = p->spin;
    c.horizon = p->mass + std::sqrt(std::max(p->mass * p->mass - p->spin * p->spin, 0.0));
    c.inner_radius = p->inner_radius;
    c.outer_radius = p->outer_radius;
    c.step = p->step;
    c.min_step_abs = std::fabs(p->min_step);
    c.max_step = p->max_step;
    c.tolerance = p->adaptive_tolerance;
    c.max_radiation_step = p->max_radiation_step;
    c.max_radiation_depth = p->max_radiation_depth;
    c.max_absorption_depth = p->max_absorption_depth;
    c.max_faraday_depth = p->max_faraday_depth;
    c.max_steps = p->max_steps;
    c.adaptive = p->adaptive;
    c.integrator = integrator;
    c.faraday_rotation = p->emission_selection.faraday_rotation;
    c.nx = p->camera.nx;
    c.ny = p->camera.ny;
    c.cam_radius = p->camera.radius;
    c.inclination = p->camera.inclination;
    c.scene = p->coordinate_system == KP_COORD_BOYER_LINDQUIST ? kSceneRiafBL : kSceneRiafCks;
    c.sin_inc = std::sin(p->camera.inclination);
    c.cos_inc = std::cos(p->camera.inclination);
    c.fov = p->camera.fov;
    c.fov_y = p->camera.fov_y;
    c.xspan = p->camera.xspan;
    c.yspan = p->camera.yspan;
    c.x_offset = p->camera.x_offset;
    c.y_offset = p->camera.y_offset;
    c.nth0 = m->nth0;
    c.Te0 = m->Te0;
    c.disk_h = m->disk_h;
    c.pow_nth = m->pow_nth;
    c.pow_T = m->pow_T;
    c.ne_unit = m->ne_unit;
    c.r_min = m->r_min;
    c.r_max = m->r_max;
    c.horizon_buffer = m->horizon_buffer;
    c.emission_scale = m->emission_scale;
    c.absorption_scale = m->absorption_scale;
    c.faraday_scale = m->faraday_scale;
    c.max_pol_frac = m->max_pol_frac;
    c.keplerian_factor = m->keplerian_factor;
    c.infall_factor = m->infall_factor;
    c.min_frequency_scale = m->min_frequency_scale;
    c.min_sin_theta = m->min_sin_theta;
    c.min_thetae = m->min_thetae;
    c.min_radius = m->min_radius;
    {
        const double kbol = 1.380649e-16, me = 9.1093837015e-28, cl = 2.99792458e10;
        c.thetae_unit = m->te_unit * kbol / (me * cl * cl);  // riaf.hpp:67-74
    }
    c.isco = isco_radius(p->spin);
    // Boundary of the far phase: two of the longest steps either pass can
    // take (adaptive steps are clamped to max_step, fixed steps are `step`)
    // beyond the radiating sphere, so no far-phase step reaches the sphere.
    c.fp32_radius = p->outer_radius + 2.0 * std::max(std::fabs(p->max_step), std::fabs(p->step));
    c.fit = m->emission_type == KP_FIT_DEXTER ? 4 : 1;
    c.nfreq = nfreq;
    const double length_unit = riaf_length_unit(m);
    for (int f = 0; f < nfreq; ++f) {
        const double fr = (nfreq == 1 && !freqs) ? m->freq_cgs : freqs[f];
        c.freq[f] = fr;
        c.dlambda_scale[f] = length_unit / std::max(fr, 1.0);  // riaf.hpp:83-85
        const int e = emission_scale_exponent(p, m, fr, c.dlambda_scale[f]);
        c.emission_scale_pow2[f] = std::ldexp(1.0f, e);
        c.inv_emission_scale_pow2[f] = std::ldexp(1.0, -e);
    }
    return c;
}

}  // namespace kp

using namespace kp;

namespace kp {

GridConsts grid_consts(const kp_grid* g) { return grid_consts_of(g->model, g->prims, g->derived); }

// Checks of one GRMHD image request before anything is launched (the FMKS
// backend of run_grmhd_image, src/image/grmhd.cpp:22-59, and this library's
// limits).
int validate_grmhd(const kp_pass_a_params* params, const kp_grid* grid, const double* frequencies, int nfreq,
                   int radiation_substeps, int device) {
    if (!params || !grid) return set_error(KP_ERR_INVALID, "GRMHD image: null argument");
    if (grid->released.load()) return set_error(KP_ERR_INVALID, "the grid has been released");
    if (params->coordinate_system != KP_COORD_FMKS)
        return set_error(KP_ERR_UNSUPPORTED, "GRMHD image coordinate backend not built: only fmks is");
    if (params->camera.nx <= 0 || params->camera.ny <= 0 || params->camera.nx > 2147483647 / params->camera.ny)
        return set_error(KP_ERR_INVALID, "image dimensions must have a positive int-sized product");
    if (nfreq < 1 || nfreq > KP_MAX_FREQUENCIES)
        return set_error(KP_ERR_INVALID, "multifrequency image chunk size must be between 1 and KP_MAX_FREQUENCIES (%d)",
                         KP_MAX_FREQUENCIES);
    if (nfreq > 1 && !frequencies) return set_error(KP_ERR_INVALID, "null frequency list");
    if (params->camera.model != KP_CAMERA_PINHOLE)
        return set_error(KP_ERR_UNSUPPORTED, "only the pinhole camera is built for the GPU image path");
    if (params->direct_only) return set_error(KP_ERR_UNSUPPORTED, "direct_only transport is not built");
    if (radiation_substeps < 1) return set_error(KP_ERR_INVALID, "radiation_substeps must be positive");
    if (grid->model.spin != params->spin) return set_error(KP_ERR_INVALID, "grid spin differs from the metric spin");
    if (device != grid->device) return set_error(KP_ERR_INVALID, "the grid lives on device %d", grid->device);
    return KP_OK;
}

void grid_unref(kp_grid* g, int n) {
    const int left = n ? g->users.fetch_sub(n) - n : g->users.load();
    if (left == 0 && g->released.load() && !g->freed.exchange(true)) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(g->device);
        cudaFree(g->prims);
        cudaFree(g->derived);
        cudaSetDevice(cur);
        delete g;
    }
}

int validate_grmhd_model(const kp_grmhd_model* m) {
    if (!m) return set_error(KP_ERR_INVALID, "null GRMHD model");
    if (m->n1 <= 0 || m->n2 <= 0 || m->n3 <= 0 || double(m->n1) * m->n2 * m->n3 > 4.0e9)
        return set_error(KP_ERR_INVALID, "grid dimensions must be positive (n1 n2 n3 = %d %d %d)", m->n1, m->n2, m->n3);
    if (!(m->dx1 > 0.0) || !(m->dx2 > 0.0) || !(m->dx3 > 0.0))
        return set_error(KP_ERR_INVALID, "grid spacings must be positive");
    if (m->emission_type != KP_FIT_PANDYA && m->emission_type != KP_FIT_DEXTER)
        return set_error(KP_ERR_UNSUPPORTED,
                         "emission_type %d: only thermal synchrotron (1 Pandya, 4 Dexter) is built",
                         m->emission_type);
    return KP_OK;
}

ImageConsts make_consts_grmhd(const kp_pass_a_params* p, const kp_grid* g, const double* freqs, int nfreq,
                              int integrator) {
    return image_consts_fmks(p, g->model, grid_consts(g), freqs, nfreq, integrator);
}

// A step-control frequency list is separate from the image's frequencies
// when its length or any value differs
// (run_multifrequency_image_metric_with_step_control,
// src/image/multifrequency.hpp:174-182); only then is it applied.
int validate_control(const double* ctl, int nctl) {
    if (nctl < 1 || !ctl) return set_error(KP_ERR_INVALID, "multifrequency step-control frequency list must not be empty");
    if (nctl > KP_MAX_CONTROL_FREQUENCIES)
        return set_error(KP_ERR_INVALID, "step-control frequency list longer than KP_MAX_CONTROL_FREQUENCIES (%d)",
                         KP_MAX_CONTROL_FREQUENCIES);
    for (int g = 0; g < nctl; ++g)
        if (!std::isfinite(ctl[g]) || !(ctl[g] > 0.0))
            return set_error(KP_ERR_INVALID, "step-control frequency %d must be finite and positive", g);
    return KP_OK;
}

bool separate_control(const double* freqs, int nfreq, double single_freq, const double* ctl, int nctl) {
    if (nctl != nfreq) return true;
    for (int f = 0; f < nfreq; ++f) {
        const double fr = (nfreq == 1 && !freqs) ? single_freq : freqs[f];
        if (fr != ctl[f]) return true;
    }
    return false;
}

// The control list's frequencies, dlambda scales (length unit / frequency)
// and, for the FP32 fits, 2^E emission scales.
void apply_control_riaf(ImageConsts& c, const kp_pass_a_params* p, const kp_riaf_model* m, const double* ctl,
                        int nctl) {
    const double length_unit = riaf_length_unit(m);
    c.nctl = nctl;
    for (int g = 0; g < nctl; ++g) {
        c.ctl_freq[g] = ctl[g];
        c.ctl_dlambda_scale[g] = length_unit / std::max(ctl[g], 1.0);
        c.ctl_emission_scale_pow2[g] = std::ldexp(1.0f, emission_scale_exponent(p, m, ctl[g], c.ctl_dlambda_scale[g]));
    }
}

}  // namespace kp

// Destroys every cached launch graph of a device.  A graph bakes in the
// addresses of the job table, the ray records, the id queues and the
// longest-first buffers: it must not outlive any of them, so every
// reallocation of those buffers calls this first.  The caller holds g_mutex.
void drop_graphs(DeviceState* dev) {
    for (auto& g : dev->graphs) cudaGraphExecDestroy(g.exec);
    dev->graphs.clear();
}

// Job table storage for njobs descriptors (device table and pinned staging),
// grow-only.  The caller holds g_mutex.
int ensure_job_table(DeviceState* dev, int njobs) {
    if (njobs <= dev->jobs_cap) return KP_OK;
    cudaEventSynchronize(dev->staging_free);
    drop_graphs(dev);
    if (dev->d_jobs) cudaFree(dev->d_jobs);
    if (dev->h_jobs) cudaFreeHost(dev->h_jobs);
    dev->d_jobs = nullptr;
    dev->h_jobs = nullptr;
    dev->jobs_cap = 0;
    const int cap = std::max(njobs, 64);
    cudaError_t e = cudaMalloc(&dev->d_jobs, sizeof(JobDesc) * size_t(cap));
    if (e != cudaSuccess) return set_error(KP_ERR_OOM, "cudaMalloc(job table): %s", cudaGetErrorString(e));
    e = cudaMallocHost(&dev->h_jobs, sizeof(JobDesc) * size_t(cap));
    if (e != cudaSuccess) return set_error(KP_ERR_OOM, "cudaMallocHost(job table): %s", cudaGetErrorString(e));
    dev->jobs_cap = cap;
    return KP_OK;
}

// Runs the wavefront engine over the njobs job descriptors staged in
// dev->h_jobs (total rays): uploads them, grows the record pool, launches
// cycles of (far, near-A, near-B) until no ray is left and checks the status
// word.  The caller holds g_mutex.
int run_wave_jobs(DeviceState* dev, cudaStream_t stream, int njobs, long long total, int family, int nf_max,
                  const kp_run_options& opt, kp_batch_stats* stats) {
    // ray records and id queues, grow-only
    if (total > dev->pool_cap) {
        cudaStreamSynchronize(stream);
        drop_graphs(dev);
        cudaFree(dev->d_pool);
        dev->d_pool = nullptr;
        for (auto& q : dev->d_ids) {
            cudaFree(q[0]);
            cudaFree(q[1]);
            q[0] = q[1] = nullptr;
        }
        cudaFree(dev->d_sorted);
        dev->d_sorted = nullptr;
        dev->pool_cap = 0;
        cudaError_t e = cudaMalloc(&dev->d_pool, sizeof(RayRecord) * size_t(total));
        for (auto& q : dev->d_ids)
            for (auto& b : q)
                if (e == cudaSuccess) e = cudaMalloc(&b, sizeof(unsigned) * size_t(total));
        if (e == cudaSuccess) e = cudaMalloc(&dev->d_sorted, sizeof(unsigned) * size_t(total));
        if (e == cudaSuccess && !dev->d_lpt) e = cudaMalloc(&dev->d_lpt, sizeof(unsigned) * 512);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(KP_ERR_OOM, "cudaMalloc(%lld ray records): %s", total, cudaGetErrorString(e));
        }
        dev->pool_cap = total;
    }
    cudaError_t e = cudaMemcpyAsync(dev->d_jobs, dev->h_jobs, sizeof(JobDesc) * size_t(njobs),
                                    cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync(job table)");
    cudaEventRecord(dev->staging_free, stream);
    // graphs need a capturable stream: not the legacy default stream
    const bool graph = opt.schedule == KP_SCHEDULE_GRAPH && stream != nullptr;
    if (!graph) {
        e = cudaMemsetAsync(dev->d_ctrl, 0, sizeof(WaveCtrl), stream);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync(wave counters)");
    }
    if (opt.threads_per_block != 0)
        return set_error(KP_ERR_INVALID, "threads_per_block is fixed by the wavefront kernels (%d far, %d near): pass 0",
                         kFarThreads, kNearThreads);
    const bool mixed = family == kFamilyRiafMixed;
    int blocks[kPhases];
    for (int phase = 0; phase < kPhases; ++phase) {
        int per_sm = opt.blocks_per_sm;
        if (per_sm <= 0) per_sm = dev->tuned_per_sm[family][phase];
        if (per_sm <= 0) {
            const int th = wave_threads(phase);
            per_sm = family == kFamilyGrmhdFP64        ? wave_occupancy_grmhd(phase, nf_max, th)
                     : family == kFamilyGrmhdMixed     ? wave_occupancy_grmhd_mixed(phase, nf_max, th)
                     : family == kFamilyGrmhdSlowFP64  ? wave_occupancy_grmhd_slow(phase, nf_max, th)
                     : family == kFamilyGrmhdSlowMixed ? wave_occupancy_grmhd_slow_mixed(phase, nf_max, th)
                     : family == kFamilyRiafBLFP64     ? wave_occupancy_bl(phase, nf_max, th)
                     : family == kFamilyRiafBLMixed    ? wave_occupancy_bl_mixed(phase, nf_max, th)
                     : mixed                           ? wave_occupancy_mixed(phase, th)
                                                       : wave_occupancy_fp64(phase, nf_max, th);
            if (per_sm <= 0) per_sm = 1;
        }
        blocks[phase] = dev->sms * per_sm;
        const long long needed = (total + wave_threads(phase) - 1) / wave_threads(phase);
        if (blocks[phase] > needed) blocks[phase] = int(needed);
    }
    WaveCtrl* ctrl = dev->d_ctrl;
    auto launch = [&](int cycle, int phase) -> cudaError_t {
        WaveDesc W;
        W.jobs = dev->d_jobs;
        W.njobs = njobs;
        W.pool = dev->d_pool;
        W.fresh_begin = 0;
        W.fresh_end = cycle == 0 && phase == kPhaseFar ? total : 0;
        W.in_ids = dev->d_ids[phase][cycle % 2];
        W.in_count = &ctrl->counts[cycle][phase];
        W.in_head = &ctrl->heads[cycle * kPhases + phase];
        for (int q = 0; q < kPhases; ++q) {
            const int gen = q > phase ? cycle : cycle + 1;
            W.out_ids[q] = dev->d_ids[q][gen % 2];
            W.out_count[q] = &ctrl->counts[gen][q];
        }
        W.budget = 0;
        W.status = &ctrl->status;
        W.job_done = nullptr;
        if (phase == kPhaseNearB) {
            // longest rays first (kp_reorder.cu): shortens the tail of the launch
            const cudaError_t le = launch_lpt_order(W.in_ids, W.in_count, dev->d_pool, dev->d_lpt, dev->d_sorted,
                                                    dev->sms, stream);
            if (le != cudaSuccess) return le;
            W.in_ids = dev->d_sorted;
        }
        if (family == kFamilyGrmhdFP64) return launch_wave_grmhd(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        if (family == kFamilyGrmhdMixed)
            return launch_wave_grmhd_mixed(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        if (family == kFamilyGrmhdSlowFP64)
            return launch_wave_grmhd_slow(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        if (family == kFamilyRiafBLFP64) return launch_wave_bl(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        if (family == kFamilyRiafBLMixed)
            return launch_wave_bl_mixed(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        if (family == kFamilyGrmhdSlowMixed)
            return launch_wave_grmhd_slow_mixed(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
        return mixed ? launch_wave_mixed(phase, W, blocks[phase], wave_threads(phase), stream)
                     : launch_wave_fp64(phase, W, nf_max, blocks[phase], wave_threads(phase), stream);
    };
    // Rays leave the camera in the far phase, trace the radiating sphere in
    // near-A then near-B and return in the far phase of the next cycle; a few
    // graze the boundary and take one more.  After each cycle the host reads
    // the next generation's queue counts.
    cudaEventRecord(dev->ev0, stream);
    int launches = 0;
    int cycle = 0;
    if (graph) {
        // counter reset, `cycles` cycles of launches and the read-back of the
        // next generation's counts, captured once per workload shape
        const int cycles = dev->tuned_cycles[family] > 0 ? min_val(dev->tuned_cycles[family], kMaxWaveCycles)
                                                        : kDefaultGraphCycles;
        DeviceState::GraphEntry key;
        std::memset(&key, 0, sizeof(key));
        key.family = family;
        key.nf_max = nf_max;
        key.njobs = njobs;
        key.cycles = cycles;
        key.total = total;
        for (int p = 0; p < kPhases; ++p) {
            key.blocks[p] = blocks[p];
            key.ids[p][0] = dev->d_ids[p][0];
            key.ids[p][1] = dev->d_ids[p][1];
        }
        key.jobs = dev->d_jobs;
        key.pool = dev->d_pool;
        key.ctrl = dev->d_ctrl;
        key.sorted = dev->d_sorted;
        key.lpt = dev->d_lpt;
        cudaGraphExec_t exec = nullptr;
        for (const auto& g : dev->graphs) {
            if (g.family == key.family && g.nf_max == key.nf_max && g.njobs == key.njobs && g.cycles == key.cycles &&
                g.total == key.total && std::memcmp(g.blocks, key.blocks, sizeof(key.blocks)) == 0 &&
                g.jobs == key.jobs && g.pool == key.pool && g.ctrl == key.ctrl && g.sorted == key.sorted &&
                g.lpt == key.lpt && std::memcmp(g.ids, key.ids, sizeof(key.ids)) == 0) {
                exec = g.exec;
                break;
            }
        }
        if (!exec) {
            e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_error(e, "cudaStreamBeginCapture");
            cudaError_t ce = cudaMemsetAsync(dev->d_ctrl, 0, sizeof(WaveCtrl), stream);
            for (int c = 0; c < cycles && ce == cudaSuccess; ++c)
                for (int phase = 0; phase < kPhases && ce == cudaSuccess; ++phase) ce = launch(c, phase);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(dev->h_left, ctrl->counts[cycles], sizeof(unsigned) * kPhases,
                                     cudaMemcpyDeviceToHost, stream);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(stream, &g);
            if (ce != cudaSuccess || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                return cuda_error(ce != cudaSuccess ? ce : e, "capturing the launch graph");
            }
            e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_error(e, "cudaGraphInstantiate");
            if (dev->graphs.size() >= kGraphCacheSize) {
                cudaGraphExecDestroy(dev->graphs.front().exec);
                dev->graphs.erase(dev->graphs.begin());
            }
            key.exec = exec;
            dev->graphs.push_back(key);
        }
        e = cudaGraphLaunch(exec, stream);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphLaunch");
        launches = cycles * kPhases;
        cycle = cycles;
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "wavefront graph");
    }
    while (!graph || dev->h_left[0] != 0 || dev->h_left[1] != 0 || dev->h_left[2] != 0) {
        if (cycle >= kMaxWaveCycles)
            return set_error(KP_ERR_TIMEOUT, "rays still moving between phases after %d launches", launches);
        for (int phase = 0; phase < kPhases; ++phase) {
            if (stats && !graph) cudaEventRecord(dev->ev_launch[launches], stream);
            e = launch(cycle, phase);
            if (e != cudaSuccess) return cuda_error(e, "wavefront kernel launch");
            ++launches;
        }
        if (stats && !graph) cudaEventRecord(dev->ev_launch[launches], stream);
        ++cycle;
        e = cudaMemcpyAsync(dev->h_left, ctrl->counts[cycle], sizeof(unsigned) * kPhases, cudaMemcpyDeviceToHost,
                            stream);
        if (e != cudaSuccess) return cuda_error(e, "queue count read");
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "wavefront kernels");
        if (dev->h_left[0] == 0 && dev->h_left[1] == 0 && dev->h_left[2] == 0) break;
    }
    cudaEventRecord(dev->ev1, stream);
    if (stats) {
        stats->rays = total;
        stats->launches = launches;
        stats->blocks = blocks[kPhaseNearB];
        stats->threads_per_block = kNearThreads;
    }
    e = cudaEventSynchronize(dev->ev1);
    if (e != cudaSuccess) return cuda_error(e, "wavefront kernels");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, dev->ev0, dev->ev1);
    if (stats) {
        stats->kernel_seconds = ms * 1e-3;
        // per-launch times need events between launches: eager schedules only
        for (int k = 0; k < launches && !graph; ++k) {
            float lms = 0.f;
            cudaEventElapsedTime(&lms, dev->ev_launch[k], dev->ev_launch[k + 1]);
            stats->phase_seconds[k % kPhases] += lms * 1e-3;
            stats->phase_launches[k % kPhases] += 1;
        }
    }
    if (opt.timing) std::printf("timing image_kernel_batch %g s\n", ms * 1e-3);
    int status_word = 0;
    e = cudaMemcpy(&status_word, &ctrl->status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "status read");
    if (status_word == 2)
        return set_error(KP_ERR_TIMEOUT, "a lane exceeded the engine's iteration guard");
    if (status_word != 0)
        return set_error(KP_ERR_CUDA, "wavefront engine invariant violated (status %d)", status_word);
    return KP_OK;
}

extern "C" {

const char* kp_last_error(void) { return g_error; }

int kp_abi_version(void) { return KP_ABI_VERSION; }

size_t kp_abi_sizeof(int which) {
    switch (which) {
    case 0: return sizeof(kp_camera_params);
    case 1: return sizeof(kp_emission_selection);
    case 2: return sizeof(kp_pass_a_params);
    case 3: return sizeof(kp_riaf_model);
    case 4: return sizeof(kp_image_out);
    case 5: return sizeof(kp_run_options);
    case 6: return sizeof(JobDesc);
    case 7: return sizeof(kp_riaf_job);
    case 8: return sizeof(kp_batch_stats);
    case 9: return sizeof(kp_tuning);
    case 10: return sizeof(kp_grmhd_model);
    case 11: return sizeof(kp_grmhd_job);
    case 12: return sizeof(kp_analysis_config);
    case 13: return sizeof(kp_analysis_out);
    case 14: return sizeof(kp_iharm_options);
    case 15: return sizeof(kp_response_config);
    default: return 0;
    }
}

size_t kp_image_output_bytes(int npix, int nfreq) {
    return size_t(npix) * (size_t(4 * nfreq + 11) * sizeof(double) + 3 * sizeof(int32_t));
}

void kp_default_run_options(kp_run_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = KP_PRECISION_FP64;
    o->schedule = KP_SCHEDULE_PER_PIXEL;
    o->integrator = KP_INTEGRATOR_STEP_DOUBLING_RK4;
}

void kp_default_pass_a_params(kp_pass_a_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->camera.nx = 64;
    p->camera.ny = 64;
    p->camera.radius = 100.0;
    p->camera.inclination = 1.04719755119659774615;
    p->camera.fov = 10.0;
    p->camera.fov_y = -1.0;
    p->camera.xspan = -1.0;
    p->camera.yspan = -1.0;
    p->camera.model = KP_CAMERA_PINHOLE;
    p->emission_selection.equatorial_h_over_r = 0.0;
    p->emission_selection.equatorial_samples = 8;
    p->emission_selection.faraday_rotation = 1;
    p->mass = 1.0;
    p->spin = 0.0;
    p->inner_radius = 2.2;
    p->outer_radius = 200.0;
    p->step = 0.05;
    p->max_steps = 4096;
    p->adaptive_tolerance = 1e-7;
    p->min_step = 1e-5;
    p->max_step = 1.0;
    p->max_radiation_step = 1.0;
    p->max_radiation_depth = 1.0;
    p->max_absorption_depth = -1.0;
    p->max_faraday_depth = -1.0;
    p->fmks_hslope = 0.3;
    p->fmks_mks_smooth = 0.5;
    p->fmks_poly_alpha = 14.0;
    p->fmks_poly_xt = 0.82;
    p->fmks_poly_norm = 1.0;
    p->coordinate_system = KP_COORD_CARTESIAN_KS;
}

void kp_default_riaf_model(kp_riaf_model* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->nth0 = 1.0;
    m->Te0 = 1.0;
    m->disk_h = 0.35;
    m->pow_nth = -1.1;
    m->pow_T = -0.84;
    m->ne_unit = 5.0e6;
    m->te_unit = 1.0e11;
    m->b_unit = 30.0;
    m->freq_cgs = 230.0e9;
    m->mbh_solar = 4.3e6;
    m->r_min = 1.0;
    m->r_max = 100.0;
    m->horizon_buffer = 0.1;
    m->emission_scale = 1.0;
    m->absorption_scale = 1.0;
    m->faraday_scale = 1.0;
    m->max_pol_frac = 0.99;
    m->keplerian_factor = 1.0;
    m->infall_factor = 0.0;
    m->emission_type = KP_FIT_PANDYA;
    m->min_frequency_scale = 1e-6;
    m->min_sin_theta = 1e-4;
    m->min_thetae = 1e-3;
    m->min_radius = 1e-6;
}

static int batch_riaf_impl(const kp_riaf_job* jobs, int njobs, const kp_run_options* options, kp_batch_stats* stats,
                           const double* ctl, int nctl);

// kp_image_riaf with an optional separate step-control list (nctl > 0).
static int image_riaf_impl(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                           const double* frequencies, int nfreq, const kp_run_options* options, kp_image_out* out,
                           const double* ctl, int nctl) {
    (void)radiation_substeps;
    kp_run_options opt;
    if (options) {
        opt = *options;
    } else {
        kp_default_run_options(&opt);
    }
    int st = validate_riaf(params, model, frequencies, nfreq);
    if (st != KP_OK) return st;
    const int npix = params->camera.nx * params->camera.ny;
    st = check_outputs(out, npix, nfreq);
    if (st != KP_OK) return st;
    if (opt.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4 && opt.integrator != KP_INTEGRATOR_CASH_KARP)
        return set_error(KP_ERR_INVALID, "unknown integrator %d", opt.integrator);
    if (opt.precision != KP_PRECISION_FP64 && opt.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", opt.precision);
    if (opt.precision == KP_PRECISION_MIXED || opt.schedule != KP_SCHEDULE_PER_PIXEL ||
        params->coordinate_system != KP_COORD_CARTESIAN_KS) {
        // the persistent engine: a batch of one (the plain per-pixel kernel
        // is the Cartesian Kerr-Schild form)
        kp_riaf_job job;
        std::memset(&job, 0, sizeof(job));
        job.params = *params;
        job.model = *model;
        for (int f = 0; f < nfreq; ++f) job.frequencies[f] = frequencies ? frequencies[f] : model->freq_cgs;
        job.nfreq = nfreq;
        job.radiation_substeps = radiation_substeps;
        job.out = *out;
        return batch_riaf_impl(&job, 1, &opt, nullptr, ctl, nctl);
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState* dev = device_state(opt.device, &st);
    if (!dev) return st;
    cudaStream_t stream = opt.stream ? static_cast<cudaStream_t>(opt.stream) : dev->stream;
    ImageConsts c = make_consts(params, model, frequencies, nfreq, opt.integrator);
    if (nctl > 0) apply_control_riaf(c, params, model, ctl, nctl);
    ImageOutPtrs dptr;
    if (opt.outputs_on_device) {
        dptr = from_abi(out);
    } else {
        void* buf = device_output_buffer(dev, carved_bytes(npix, nfreq), &st);
        if (!buf) return st;
        dptr = carve_outputs(buf, npix, nfreq);
    }
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = launch_image_fp64(c, dptr, stream);
    if (e != cudaSuccess) return cuda_error(e, "image kernel launch");
    if (opt.timing) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "image kernel");
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("timing %s %g s\n", nfreq > 1 ? "image_kernel_multifrequency" : "image_kernel_single", s);
    }
    if (!opt.outputs_on_device) {
        const auto t1 = std::chrono::steady_clock::now();
        st = copy_outputs_to_host(dptr, out, npix, nfreq, stream);
        if (st != KP_OK) return st;
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "image kernel / device-to-host copy");
        if (opt.timing) {
            const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
            std::printf("timing %s %g s\n",
                        nfreq > 1 ? "image_device_to_host_multifrequency" : "image_device_to_host_single", s);
        }
    } else if (!opt.stream) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "image kernel");
    }
    return KP_OK;
}

int kp_image_riaf(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                  const double* frequencies, int nfreq, const kp_run_options* options, kp_image_out* out) {
    return image_riaf_impl(params, model, radiation_substeps, frequencies, nfreq, options, out, nullptr, 0);
}

int kp_image_riaf_step_control(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                               const double* frequencies, int nfreq, const double* control_frequencies,
                               int ncontrol, const kp_run_options* options, kp_image_out* out) {
    int st = validate_control(control_frequencies, ncontrol);
    if (st != KP_OK) return st;
    st = validate_riaf(params, model, frequencies, nfreq);
    if (st != KP_OK) return st;
    if (!separate_control(frequencies, nfreq, model->freq_cgs, control_frequencies, ncontrol))
        return image_riaf_impl(params, model, radiation_substeps, frequencies, nfreq, options, out, nullptr, 0);
    return image_riaf_impl(params, model, radiation_substeps, frequencies, nfreq, options, out, control_frequencies,
                           ncontrol);
}

void kp_default_analysis_config(kp_analysis_config* cfg) {
    if (!cfg) return;
    cfg->radial_bins = 16;  // AnalysisConfig defaults (analysis_driver.hpp:16-23)
    cfg->radial_min = 2.0;
    cfg->radial_max = 100.0;
    cfg->formation_fraction = 0.9;
}

// Checks a response configuration against the bins each partition needs
// (make_response_config, tools/kpolaris_response_options.hpp:10-82, whose
// tool-level checks a caller of the C ABI bypasses); returns the channel
// count or a negative status.
static int validate_response(const kp_response_config* r) {
    if (!r) return set_error(KP_ERR_INVALID, "null response configuration");
    if (r->parameter < KP_RESPONSE_NONE || r->parameter > KP_RESPONSE_COEFFICIENTS)
        return set_error(KP_ERR_INVALID, "unknown response parameter %d", r->parameter);
    if (r->partition < KP_PARTITION_NONE || r->partition > KP_PARTITION_B_CGS)
        return set_error(KP_ERR_INVALID, "unknown source partition %d", r->partition);
    if (r->partition == KP_PARTITION_NONE) {
        if (r->parameter != KP_RESPONSE_NONE)
            return set_error(KP_ERR_INVALID, "a response parameter needs a source partition");
        return 0;
    }
    if (r->parameter != KP_RESPONSE_NONE && !(std::isfinite(r->step) && r->step >= 1e-6 && r->step <= 0.1))
        return set_error(KP_ERR_INVALID, "analysis_response_step must be finite and in [1e-6,0.1]");
    const double half_pi = 0.5 * 3.14159265358979323846;
    if (r->partition == KP_PARTITION_REGION &&
        !(std::isfinite(r->funnel_angle) && std::isfinite(r->disk_angle) && r->funnel_angle > 0.0 &&
          r->funnel_angle < r->disk_angle && r->disk_angle < half_pi))
        return set_error(KP_ERR_INVALID, "analysis region angles must satisfy 0 < funnel < disk < 90 degrees");
    if ((r->partition == KP_PARTITION_REGION || r->partition == KP_PARTITION_NEAR_FAR) &&
        !(std::isfinite(r->observer_theta) && std::isfinite(r->observer_phi)))
        return set_error(KP_ERR_INVALID, "the observer direction must be finite");
    if (r->partition == KP_PARTITION_PLASMA_REGION &&
        !(std::isfinite(r->sigma_boundary) && std::isfinite(r->beta_boundary) && r->sigma_boundary > 0.0 &&
          r->beta_boundary > 0.0))
        return set_error(KP_ERR_INVALID, "analysis sigma/beta boundaries must be finite and positive");
    auto increasing = [&](int n) {
        for (int i = 0; i < n; ++i) {
            if (!(std::isfinite(r->edges[i]) && r->edges[i] > 0.0)) return false;
            if (i > 0 && !(r->edges[i] > r->edges[i - 1])) return false;
        }
        return true;
    };
    int want = 0;
    switch (r->partition) {
    case KP_PARTITION_RADIAL:
        if (r->bins < 1 || r->bins + 1 > KP_MAX_PARTITION_EDGES || r->edge_count != r->bins + 1 ||
            !increasing(r->edge_count))
            return set_error(KP_ERR_INVALID,
                             "radial partition: bins in [1, %d], edge_count = bins + 1 increasing positive edges",
                             KP_MAX_PARTITION_EDGES - 1);
        want = r->bins;
        break;
    case KP_PARTITION_REGION: want = 6; break;
    case KP_PARTITION_PLASMA_REGION: want = 4; break;
    case KP_PARTITION_NEAR_FAR: want = 2; break;
    default:
        if (r->edge_count < 1 || r->edge_count > KP_MAX_PARTITION_EDGES || !increasing(r->edge_count))
            return set_error(KP_ERR_INVALID,
                             "analysis_partition_edges must be finite, positive, strictly increasing "
                             "(at most %d edges)", KP_MAX_PARTITION_EDGES);
        want = r->edge_count + 2;
        break;
    }
    if (r->bins != want)
        return set_error(KP_ERR_INVALID, "partition %d needs bins = %d, got %d", r->partition, want, r->bins);
    const bool responses = r->parameter != KP_RESPONSE_NONE;
    return r->bins * (responses ? 5 : 1) + (responses ? 4 : 0);
}

static int analysis_impl(const kp_pass_a_params* params, const kp_riaf_model* model,
                         const kp_analysis_config* config, const kp_response_config* resp_cfg,
                         const kp_run_options* options, kp_image_out* out, kp_analysis_out* analysis,
                         double* response);

int kp_image_riaf_analysis(const kp_pass_a_params* params, const kp_riaf_model* model, int radiation_substeps,
                           const kp_analysis_config* config, const kp_run_options* options, kp_image_out* out,
                           kp_analysis_out* analysis) {
    (void)radiation_substeps;
    return analysis_impl(params, model, config, nullptr, options, out, analysis, nullptr);
}

void kp_default_response_config(kp_response_config* r) {
    if (!r) return;
    std::memset(r, 0, sizeof(*r));
    r->parameter = KP_RESPONSE_NONE;
    r->partition = KP_PARTITION_NONE;
    r->step = 1e-3;
    r->funnel_angle = 0.3490658503988659;
    r->disk_angle = 1.0471975511965976;
    r->sigma_boundary = 1.0;
    r->beta_boundary = 1.0;
}

int kp_response_channels(const kp_response_config* r) { return validate_response(r); }

int kp_image_riaf_analysis_response(const kp_pass_a_params* params, const kp_riaf_model* model,
                                    int radiation_substeps, const kp_analysis_config* config,
                                    const kp_response_config* response_config, const kp_run_options* options,
                                    kp_image_out* out, kp_analysis_out* analysis, double* response) {
    (void)radiation_substeps;
    return analysis_impl(params, model, config, response_config, options, out, analysis, response);
}

static int analysis_impl(const kp_pass_a_params* params, const kp_riaf_model* model,
                         const kp_analysis_config* config, const kp_response_config* resp_cfg,
                         const kp_run_options* options, kp_image_out* out, kp_analysis_out* analysis,
                         double* response) {
    kp_run_options opt;
    if (options) {
        opt = *options;
    } else {
        kp_default_run_options(&opt);
    }
    int st = validate_riaf(params, model, nullptr, 1);
    if (st == KP_OK && params->coordinate_system != KP_COORD_CARTESIAN_KS)
        return set_error(KP_ERR_UNSUPPORTED, "analysis-mode image coordinate backend not built: boyer_lindquist");
    if (st != KP_OK) return st;
    if (!config || !analysis) return set_error(KP_ERR_INVALID, "null analysis config or outputs");
    // validate_options (tools/kpolaris_model_image_options.cpp:265-284)
    if (config->radial_bins < 1 || config->radial_bins > KP_MAX_ANALYSIS_RADIAL_BINS)
        return set_error(KP_ERR_INVALID, "analysis radial_bins must lie in [1, %d]", KP_MAX_ANALYSIS_RADIAL_BINS);
    if ((config->radial_min > 0.0 && !std::isfinite(config->radial_min)) ||
        (config->radial_max > 0.0 && !std::isfinite(config->radial_max)))
        return set_error(KP_ERR_INVALID, "analysis radial bounds must be finite when specified");
    if (config->radial_min > 0.0 && config->radial_max > 0.0 && !(config->radial_max > config->radial_min))
        return set_error(KP_ERR_INVALID, "analysis radial_max must exceed radial_min");
    if (!std::isfinite(config->formation_fraction) || !(config->formation_fraction > 0.0) ||
        !(config->formation_fraction < 1.0))
        return set_error(KP_ERR_INVALID, "analysis formation_fraction must lie strictly between 0 and 1");
    if (opt.precision != KP_PRECISION_FP64)
        return set_error(KP_ERR_UNSUPPORTED, "analysis mode runs in FP64 only");
    if (opt.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4)
        return set_error(KP_ERR_UNSUPPORTED, "analysis mode uses step-doubling RK4 only");
    if (!(params->min_step > 0.0)) return set_error(KP_ERR_INVALID, "analysis mode needs min_step > 0");
    const int npix = params->camera.nx * params->camera.ny;
    st = check_outputs(out, npix, 1);
    if (st != KP_OK) return st;
    const int channels = resp_cfg ? validate_response(resp_cfg) : 0;
    if (channels < 0) return channels;
    if (channels > 0 && !response) return set_error(KP_ERR_INVALID, "null response output with %d channels", channels);
    const size_t response_bytes = size_t(4) * size_t(channels) * size_t(npix) * sizeof(double);
    // kp_analysis_out and AnalysisPtrs list the same arrays in the same order
    constexpr int kArrays = int(sizeof(kp_analysis_out) / sizeof(void*));
    static_assert(sizeof(kp_analysis_out) == sizeof(AnalysisPtrs), "analysis array lists differ");
    static_assert(kArrays == 52, "analysis array count");
    auto is_int = [](int i) { return i == 10 || i == 22; };
    auto is_radial = [](int i) { return i >= 23 && i < 31; };
    void* host[kArrays];
    std::memcpy(host, analysis, sizeof(host));
    for (int i = 0; i < kArrays; ++i)
        if (!host[i]) return set_error(KP_ERR_INVALID, "analysis output array %d is NULL", i);
    const int bins = config->radial_bins;
    auto bytes_of = [&](int i) {
        return size_t(is_radial(i) ? bins : 1) * size_t(npix) * (is_int(i) ? sizeof(int32_t) : sizeof(double));
    };

    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState* dev = device_state(opt.device, &st);
    if (!dev) return st;
    cudaStream_t stream = opt.stream ? static_cast<cudaStream_t>(opt.stream) : dev->stream;
    const ImageConsts c = make_consts(params, model, nullptr, 1, opt.integrator);
    const AnalysisConsts k{bins, config->radial_min, config->radial_max, config->formation_fraction};
    ImageOutPtrs dptr;
    void* dev_arrays[kArrays];
    void* analysis_buf = nullptr;
    if (opt.outputs_on_device) {
        dptr = from_abi(out);
        std::memcpy(dev_arrays, host, sizeof(dev_arrays));
    } else {
        void* buf = device_output_buffer(dev, carved_bytes(npix, 1), &st);
        if (!buf) return st;
        dptr = carve_outputs(buf, npix, 1);
        size_t total = 0;
        for (int i = 0; i < kArrays; ++i) total += (bytes_of(i) + 255) / 256 * 256;
        cudaError_t e = cudaMalloc(&analysis_buf, total);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(KP_ERR_OOM, "cudaMalloc(%zu bytes) for analysis outputs: %s", total,
                             cudaGetErrorString(e));
        }
        char* p = static_cast<char*>(analysis_buf);
        for (int i = 0; i < kArrays; ++i) {
            dev_arrays[i] = p;
            p += (bytes_of(i) + 255) / 256 * 256;
        }
    }
    AnalysisPtrs an;
    std::memcpy(&an, dev_arrays, sizeof(an));
    // response channels: the configuration and (host outputs) the channel
    // array in one device buffer, the array zeroed before the launch
    void* resp_buf = nullptr;
    kp_response_config* d_resp = nullptr;
    double* d_response = nullptr;
    cudaError_t e = cudaSuccess;
    if (channels > 0) {
        const size_t cfg_bytes = (sizeof(kp_response_config) + 255) / 256 * 256;
        const size_t bytes = cfg_bytes + (opt.outputs_on_device ? 0 : response_bytes);
        e = cudaMalloc(&resp_buf, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (analysis_buf) cudaFree(analysis_buf);
            return set_error(KP_ERR_OOM, "cudaMalloc(%zu bytes) for response channels: %s", bytes,
                             cudaGetErrorString(e));
        }
        d_resp = static_cast<kp_response_config*>(resp_buf);
        d_response = opt.outputs_on_device ? response
                                           : reinterpret_cast<double*>(static_cast<char*>(resp_buf) + cfg_bytes);
        e = cudaMemcpyAsync(d_resp, resp_cfg, sizeof(kp_response_config), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_response, 0, response_bytes, stream);
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (e == cudaSuccess) e = launch_image_fp64_analysis(c, k, dptr, an, d_resp, d_response, stream);
    if (e == cudaSuccess && opt.timing) {
        e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess)
            std::printf("timing image_kernel_analysis %g s\n",
                        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    if (e == cudaSuccess && !opt.outputs_on_device) {
        st = copy_outputs_to_host(dptr, out, npix, 1, stream);
        for (int i = 0; st == KP_OK && e == cudaSuccess && i < kArrays; ++i)
            e = cudaMemcpyAsync(host[i], dev_arrays[i], bytes_of(i), cudaMemcpyDeviceToHost, stream);
        if (st == KP_OK && e == cudaSuccess && channels > 0)
            e = cudaMemcpyAsync(response, d_response, response_bytes, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    } else if (e == cudaSuccess && (!opt.stream || resp_buf)) {
        // the configuration buffer is freed below: the launch must be done
        e = cudaStreamSynchronize(stream);
    }
    if (resp_buf) cudaFree(resp_buf);
    if (analysis_buf) cudaFree(analysis_buf);
    if (e != cudaSuccess) return cuda_error(e, "analysis image");
    return st;
}

int kp_batch_riaf(const kp_riaf_job* jobs, int njobs, const kp_run_options* options, kp_batch_stats* stats) {
    return batch_riaf_impl(jobs, njobs, options, stats, nullptr, 0);
}

// kp_batch_riaf; a step-control list (nctl > 0) applies to every job.
static int batch_riaf_impl(const kp_riaf_job* jobs, int njobs, const kp_run_options* options, kp_batch_stats* stats,
                           const double* ctl, int nctl) {
    kp_run_options opt;
    if (options) {
        opt = *options;
    } else {
        kp_default_run_options(&opt);
        opt.schedule = KP_SCHEDULE_PERSISTENT;
    }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (njobs < 0 || (njobs > 0 && !jobs)) return set_error(KP_ERR_INVALID, "invalid job list");
    if (njobs == 0) return KP_OK;
    if (opt.precision != KP_PRECISION_FP64 && opt.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", opt.precision);
    if (opt.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4 && opt.integrator != KP_INTEGRATOR_CASH_KARP)
        return set_error(KP_ERR_INVALID, "unknown integrator %d", opt.integrator);
    // Validate every job before launching any work (batch_driver.hpp:137-145).
    long long total = 0;
    int nf_max = 1;
    size_t scratch = 0;
    for (int i = 0; i < njobs; ++i) {
        const kp_riaf_job& jb = jobs[i];
        int st = validate_riaf(&jb.params, &jb.model, jb.frequencies, jb.nfreq);
        if (st != KP_OK) return job_error(st, i);
        // one metric per batch, as run_image_batch_metric<Metric> has
        if (jb.params.coordinate_system != jobs[0].params.coordinate_system)
            return set_error(KP_ERR_UNSUPPORTED, "job %d: the jobs of a batch must share one coordinate system", i);
        if (jb.radiation_substeps < 1) return set_error(KP_ERR_INVALID, "job %d: batch radiation_substeps must be positive", i);
        const int npix = jb.params.camera.nx * jb.params.camera.ny;
        st = check_outputs(&jb.out, npix, jb.nfreq);
        if (st != KP_OK) return job_error(st, i);
        total += npix;
        nf_max = std::max(nf_max, jb.nfreq);
        scratch += carved_bytes(npix, jb.nfreq);
    }
    const bool bl = jobs[0].params.coordinate_system == KP_COORD_BOYER_LINDQUIST;
    const bool mixed_policy = opt.precision == KP_PRECISION_MIXED;
    const int family = bl ? (mixed_policy ? kFamilyRiafBLMixed : kFamilyRiafBLFP64)
                          : (mixed_policy ? kFamilyRiafMixed : kFamilyRiafFP64);
    // The mixed Kerr-Schild kernel always carries four channels: the same
    // compiled code traces a ray whatever the other jobs of the batch are.
    if (family == kFamilyRiafMixed) nf_max = KP_MAX_FREQUENCIES;
    std::lock_guard<std::mutex> lock(g_mutex);
    int st = KP_OK;
    DeviceState* dev = device_state(opt.device, &st);
    if (!dev) return st;
    cudaStream_t stream = opt.stream ? static_cast<cudaStream_t>(opt.stream) : dev->stream;
    st = ensure_job_table(dev, njobs);
    if (st != KP_OK) return st;
    void* scratch_base = nullptr;
    if (!opt.outputs_on_device) {
        scratch_base = device_output_buffer(dev, scratch, &st);
        if (!scratch_base) return st;
    }
    // the previous upload from the staging table must be complete before it is rewritten
    cudaEventSynchronize(dev->staging_free);
    std::vector<ImageOutPtrs> dptrs(static_cast<size_t>(njobs));
    long long ray = 0;
    char* carve = static_cast<char*>(scratch_base);
    for (int i = 0; i < njobs; ++i) {
        const kp_riaf_job& jb = jobs[i];
        const int npix = jb.params.camera.nx * jb.params.camera.ny;
        JobDesc& d = dev->h_jobs[i];
        std::memset(&d, 0, sizeof(d));
        d.c = make_consts(&jb.params, &jb.model, jb.frequencies, jb.nfreq, opt.integrator);
        if (nctl > 0) apply_control_riaf(d.c, &jb.params, &jb.model, ctl, nctl);
        double fr[5][4];
        host_camera_frame(d.c, fr);
        for (int mu = 0; mu < 4; ++mu) {
            d.frame.x.v[mu] = fr[0][mu];
            d.frame.e0.v[mu] = fr[1][mu];
            d.frame.e1.v[mu] = fr[2][mu];
            d.frame.e2.v[mu] = fr[3][mu];
            d.frame.e3.v[mu] = fr[4][mu];
        }
        if (opt.outputs_on_device) {
            d.out = from_abi(&jb.out);
        } else {
            d.out = carve_outputs(carve, npix, jb.nfreq);
            carve += carved_bytes(npix, jb.nfreq);
        }
        dptrs[size_t(i)] = d.out;
        d.ray_begin = ray;
        d.npix = npix;
        d.precision = opt.precision;
        ray += npix;
    }
    st = run_wave_jobs(dev, stream, njobs, total, family, nf_max, opt, stats);
    if (st != KP_OK) return st;
    if (stats) stats->device_output_bytes = opt.outputs_on_device ? 0 : scratch;
    if (!opt.outputs_on_device) {
        const auto t1 = std::chrono::steady_clock::now();
        for (int i = 0; i < njobs; ++i) {
            st = copy_outputs_to_host(dptrs[size_t(i)], &jobs[i].out, jobs[i].params.camera.nx * jobs[i].params.camera.ny,
                                      jobs[i].nfreq, stream);
            if (st != KP_OK) return st;
        }
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "device-to-host copy");
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        if (stats) stats->copy_seconds = s;
        if (opt.timing) std::printf("timing image_device_to_host_batch %g s\n", s);
    }
    return KP_OK;
}

int kp_pack_image(const kp_image_out* data, int freq_index, double frequency, int evpa_north,
                  double intensity_to_flux_jy_per_pixel, kp_packed_image* out) {
    if (!data || !out) return set_error(KP_ERR_INVALID, "kp_pack_image: null argument");
    if (freq_index < 0 || freq_index >= data->nfreq)
        return set_error(KP_ERR_INVALID, "frequency index %d outside [0, %d)", freq_index, data->nfreq);
    if (!data->image_i || !data->image_q || !data->image_u || !data->image_v || !data->reason)
        return set_error(KP_ERR_INVALID, "kp_pack_image: image arrays and reason are required");
    const int npix = data->npix;
    const size_t off = size_t(freq_index) * size_t(npix);
    const double sign = evpa_north ? -1.0 : 1.0;
    const double nu3 = frequency * frequency * frequency;
    double sum[4] = {0.0, 0.0, 0.0, 0.0};
    int returned = 0;
    for (int p = 0; p < npix; ++p) {
        const bool reached = data->reason[p] == KP_REASON_REACHED_CAMERA;
        const double i = reached ? data->image_i[off + size_t(p)] : 0.0;
        const double q = reached ? sign * data->image_q[off + size_t(p)] : 0.0;
        const double u = reached ? sign * data->image_u[off + size_t(p)] : 0.0;
        const double v = reached ? data->image_v[off + size_t(p)] : 0.0;
        if (out->i_inv) out->i_inv[p] = i;
        if (out->q_inv) out->q_inv[p] = q;
        if (out->u_inv) out->u_inv[p] = u;
        if (out->v_inv) out->v_inv[p] = v;
        if (out->i_nu) out->i_nu[p] = i * nu3;
        if (out->q_nu) out->q_nu[p] = q * nu3;
        if (out->u_nu) out->u_nu[p] = u * nu3;
        if (out->v_nu) out->v_nu[p] = v * nu3;
        if (out->total_steps && data->pass_a_steps && data->steps)
            out->total_steps[p] = data->pass_a_steps[p] + data->steps[p];
        if (reached) {
            ++returned;
            sum[0] += i;
            sum[1] += q;
            sum[2] += u;
            sum[3] += v;
        }
    }
    out->returned = returned;
    const bool valid = intensity_to_flux_jy_per_pixel > 0.0 && std::isfinite(intensity_to_flux_jy_per_pixel);
    for (int k = 0; k < 4; ++k) {
        out->sum_inv[k] = sum[k];
        out->flux_jy[k] = valid ? sum[k] * frequency * frequency * frequency * intensity_to_flux_jy_per_pixel
                                : std::numeric_limits<double>::quiet_NaN();
    }
    return KP_OK;
}

double kp_flux_scale_jy_per_pixel(double mbh_solar, double dsource_pc, double image_width_x, double image_width_y,
                                  int nx, int ny) {
    const double gnewt = 6.6742e-8, msun = 1.989e33, cl = 2.99792458e10, pc_cgs = 3.085678e18, jy_cgs = 1.0e-23;
    const double l_unit = gnewt * mbh_solar * msun / (cl * cl);
    const double dsource = dsource_pc * pc_cgs;
    if (!(dsource_pc > 0.0 && image_width_x > 0.0 && image_width_y > 0.0 && nx > 0 && ny > 0 && mbh_solar > 0.0))
        return std::numeric_limits<double>::quiet_NaN();
    const double px = image_width_x * l_unit / double(nx);
    const double py = image_width_y * l_unit / double(ny);
    return px * py / (dsource * dsource) / jy_cgs;
}

int kp_autotune_batch(const kp_riaf_job* jobs, int njobs, const kp_run_options* options, kp_tuning* out) {
    if (!out) return set_error(KP_ERR_INVALID, "kp_autotune_batch: null result");
    std::memset(out, 0, sizeof(*out));
    if (njobs < 1 || !jobs) return set_error(KP_ERR_INVALID, "kp_autotune_batch: empty sample");
    kp_run_options opt;
    if (options) {
        opt = *options;
    } else {
        kp_default_run_options(&opt);
    }
    if (opt.blocks_per_sm != 0) return set_error(KP_ERR_INVALID, "blocks_per_sm must be 0: the tuner chooses it");
    if (opt.precision != KP_PRECISION_FP64 && opt.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", opt.precision);
    const bool bl = jobs[0].params.coordinate_system == KP_COORD_BOYER_LINDQUIST;
    const int family = bl ? (opt.precision == KP_PRECISION_MIXED ? kFamilyRiafBLMixed : kFamilyRiafBLFP64)
                          : (opt.precision == KP_PRECISION_MIXED ? kFamilyRiafMixed : kFamilyRiafFP64);
    int nf_max = 1;
    for (int i = 0; i < njobs; ++i)
        if (jobs[i].nfreq > 1) nf_max = KP_MAX_FREQUENCIES;
    if (family == kFamilyRiafMixed) nf_max = KP_MAX_FREQUENCIES;
    int limit[kPhases];
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        int st = KP_OK;
        DeviceState* dev = device_state(opt.device, &st);
        if (!dev) return st;
        for (int phase = 0; phase < kPhases; ++phase) {
            const int th = wave_threads(phase);
            const int occ = family == kFamilyRiafMixed     ? wave_occupancy_mixed(phase, th)
                            : family == kFamilyRiafBLFP64  ? wave_occupancy_bl(phase, nf_max, th)
                            : family == kFamilyRiafBLMixed ? wave_occupancy_bl_mixed(phase, nf_max, th)
                                                           : wave_occupancy_fp64(phase, nf_max, th);
            limit[phase] = occ < 1 ? 1 : (occ > 4 ? 4 : occ);
        }
    }
    auto set_table = [&](const int per_sm[kPhases], int cycles) {
        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceState& dev = g_dev[opt.device];
        for (int p = 0; p < kPhases; ++p) dev.tuned_per_sm[family][p] = per_sm[p];
        dev.tuned_cycles[family] = cycles;
    };
    // device time of the sample under a schedule: the better of two runs
    auto time_sample = [&](int schedule, double* seconds) -> int {
        kp_run_options o = opt;
        o.schedule = schedule;
        double best = 0.0;
        for (int rep = 0; rep < 2; ++rep) {
            kp_batch_stats stats;
            const int st = kp_batch_riaf(jobs, njobs, &o, &stats);
            if (st != KP_OK) return st;
            if (rep == 0 || stats.kernel_seconds < best) best = stats.kernel_seconds;
        }
        *seconds = best;
        return KP_OK;
    };
    const int none[kPhases] = {0, 0, 0};
    set_table(none, 0);
    double t_default = 0.0;
    int st = time_sample(KP_SCHEDULE_PERSISTENT, &t_default);
    if (st != KP_OK) return st;
    static const int kCycleChoices[] = {2, 3, 4, 6};
    int best[kPhases] = {0, 0, 0}, best_cycles = 0, n = 0;
    double t_best = 0.0;
    for (int far = 1; far <= limit[kPhaseFar]; ++far)
        for (int na = 1; na <= limit[kPhaseNearA]; ++na)
            for (int nb = 1; nb <= limit[kPhaseNearB]; ++nb)
                for (int cycles : kCycleChoices) {
                    const int cand[kPhases] = {far, na, nb};
                    set_table(cand, cycles);
                    double t = 0.0;
                    st = time_sample(KP_SCHEDULE_GRAPH, &t);
                    if (st != KP_OK) {
                        set_table(none, 0);
                        return st;
                    }
                    ++n;
                    if (n == 1 || t < t_best) {
                        t_best = t;
                        best_cycles = cycles;
                        for (int p = 0; p < kPhases; ++p) best[p] = cand[p];
                    }
                }
    // A candidate replaces the default only by a margin above the sample's
    // run-to-run noise (about 1%): a small sample favours whatever shortens
    // its own tail, which the full workload need not share.
    constexpr double kAdoptMargin = 0.02;
    if (!(t_best < t_default * (1.0 - kAdoptMargin))) {
        for (int p = 0; p < kPhases; ++p) best[p] = 0;
        best_cycles = 0;
        t_best = t_default;
    }
    set_table(best, best_cycles);
    for (int p = 0; p < kPhases; ++p) out->blocks_per_sm[p] = best[p];
    out->graph_cycles = best_cycles;
    out->seconds = t_best;
    out->default_seconds = t_default;
    out->candidates = n;
    return KP_OK;
}


void kp_default_grmhd_model(kp_grmhd_model* m) {
    if (!m) return;
    std::memset(m, 0, sizeof(*m));
    m->spin = 0.5;
    m->gam = 4.0 / 3.0;
    m->dx1 = m->dx2 = m->dx3 = 1.0;
    m->r_in = 1.0;
    m->r_out = 1000.0;
    m->hslope = 0.3;
    m->mks_smooth = 0.5;
    m->poly_alpha = 14.0;
    m->poly_xt = 0.82;
    m->poly_norm = 1.0;
    m->freq_cgs = 230.0e9;
    m->mbh_solar = 6.2e9;
    m->M_unit = 3.0e25;
    m->trat_small = 1.0;
    m->trat_large = 20.0;
    m->beta_crit = 1.0;
    m->sigma_cut = 1.0;
    m->sigma_cut_high = -1.0;
    m->ne_factor = 1.0;
    m->emission_type = KP_FIT_DEXTER;
    m->emission_scale = m->absorption_scale = m->faraday_scale = 1.0;
    m->max_pol_frac = 0.99;
    m->has_derived_scalars = 1;
}

int kp_grid_upload(const kp_grmhd_model* model, const float* prims, int device, kp_grid** out) {
    if (!out) return set_error(KP_ERR_INVALID, "kp_grid_upload: null output handle");
    *out = nullptr;
    int st = validate_grmhd_model(model);
    if (st != KP_OK) return st;
    if (!prims) return set_error(KP_ERR_INVALID, "kp_grid_upload: null primitives");
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState* dev = device_state(device, &st);
    if (!dev) return st;
    auto* g = new kp_grid();
    g->device = device;
    g->model = *model;
    const size_t ncell = size_t(model->n1) * size_t(model->n2) * size_t(model->n3);
    // cell-major device layout (kPrimStride floats, kDerStride doubles per
    // cell), filled from the reference layout through a staging buffer
    float* staging = nullptr;
    cudaError_t e = cudaMalloc(&g->prims, sizeof(float) * kPrimStride * ncell);
    if (e == cudaSuccess) e = cudaMalloc(&staging, sizeof(float) * 8 * ncell);
    if (e == cudaSuccess && model->has_derived_scalars) e = cudaMalloc(&g->derived, sizeof(double) * kDerStride * ncell);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(g->prims);
        cudaFree(g->derived);
        cudaFree(staging);
        delete g;
        return set_error(KP_ERR_OOM, "grid allocation (%zu cells): %s", ncell, cudaGetErrorString(e));
    }
    e = cudaMemcpyAsync(staging, prims, sizeof(float) * 8 * ncell, cudaMemcpyHostToDevice, dev->stream);
    if (e == cudaSuccess) e = launch_grid_to_cells(staging, g->prims, (long long)ncell, dev->sms, dev->stream);
    if (e == cudaSuccess && g->derived) e = launch_grid_derived(grid_consts(g), g->derived, dev->sms, dev->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(dev->stream);
    cudaFree(staging);
    if (e != cudaSuccess) {
        cudaFree(g->prims);
        cudaFree(g->derived);
        delete g;
        return cuda_error(e, "grid upload");
    }
    *out = g;
    return KP_OK;
}

int kp_grid_derived(const kp_grid* g, double* out) {
    if (!g || !out) return set_error(KP_ERR_INVALID, "kp_grid_derived: null argument");
    if (!g->derived) return set_error(KP_ERR_INVALID, "the grid has no derived scalars");
    cudaError_t e = cudaSetDevice(g->device);
    const size_t ncell = size_t(g->model.n1) * size_t(g->model.n2) * size_t(g->model.n3);
    std::vector<double> cells(ncell * kDerStride);
    if (e == cudaSuccess)
        e = cudaMemcpy(cells.data(), g->derived, sizeof(double) * kDerStride * ncell, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "derived scalar copy");
    for (size_t p = 0; p < ncell; ++p)
        for (int v = 0; v < kNumDerived; ++v) out[size_t(v) * ncell + p] = cells[p * kDerStride + size_t(v)];
    return KP_OK;
}

int kp_grid_release(kp_grid* g) {
    if (!g) return KP_OK;
    // a grid that queued or running server jobs still read is freed when
    // the last of them ends (kp::grid_unref)
    g->released.store(true);
    kp::grid_unref(g, 0);
    return KP_OK;
}

}  // extern "C"

namespace {

// Whether two grids hold the same flow geometry, so one stencil serves both
// (can_interpolate_fluid_with, src/model/grmhd_grid.hpp:129-139, plus the
// grid shape this library gathers both snapshots with).
bool same_grid_geometry(const kp_grmhd_model& a, const kp_grmhd_model& b) {
    return a.n1 == b.n1 && a.n2 == b.n2 && a.n3 == b.n3 && a.spin == b.spin && a.startx1 == b.startx1 &&
           a.startx2 == b.startx2 && a.startx3 == b.startx3 && a.dx1 == b.dx1 && a.dx2 == b.dx2 && a.dx3 == b.dx3 &&
           a.r_in == b.r_in && a.r_out == b.r_out && a.hslope == b.hslope && a.mks_smooth == b.mks_smooth &&
           a.poly_alpha == b.poly_alpha && a.poly_xt == b.poly_xt && a.poly_norm == b.poly_norm &&
           a.has_derived_scalars == b.has_derived_scalars;
}

// One GRMHD image, fast light (nsnap == 0: grids[0] alone) or slow light
// (nsnap >= 2 resident snapshots at `times`, fluid read at t_obs + x^0).
int grmhd_image(const kp_pass_a_params* params, const kp_grid* const* grids, const double* times, int nsnap,
                double t_obs, int radiation_substeps, const double* frequencies, int nfreq,
                const kp_run_options* options, kp_image_out* out, const double* ctl = nullptr, int nctl = 0) {
    const kp_grid* grid = grids ? grids[0] : nullptr;
    if (!params || !grid || !out) return set_error(KP_ERR_INVALID, "GRMHD image: null argument");
    kp_run_options opt;
    if (options) {
        opt = *options;
    } else {
        kp_default_run_options(&opt);
    }
    int vst = kp::validate_grmhd(params, grid, frequencies, nfreq, radiation_substeps, opt.device);
    if (vst != KP_OK) return vst;
    if (opt.precision != KP_PRECISION_FP64 && opt.precision != KP_PRECISION_MIXED)
        return set_error(KP_ERR_INVALID, "unknown precision %d", opt.precision);
    if (opt.integrator != KP_INTEGRATOR_STEP_DOUBLING_RK4 && opt.integrator != KP_INTEGRATOR_CASH_KARP)
        return set_error(KP_ERR_INVALID, "unknown integrator %d", opt.integrator);
    const bool slow = nsnap != 0;
    if (slow) {
        if (nsnap < 2) return set_error(KP_ERR_INVALID, "slow-light requires at least two snapshots");
        if (!times) return set_error(KP_ERR_INVALID, "null snapshot time list");
        if (!std::isfinite(t_obs)) return set_error(KP_ERR_INVALID, "observation time must be finite");
        for (int i = 0; i < nsnap; ++i) {
            if (!grids[i]) return set_error(KP_ERR_INVALID, "null snapshot %d", i);
            if (grids[i]->released.load()) return set_error(KP_ERR_INVALID, "snapshot %d has been released", i);
            if (grids[i]->device != opt.device)
                return set_error(KP_ERR_INVALID, "snapshot %d lives on device %d", i, grids[i]->device);
            if (!same_grid_geometry(grid->model, grids[i]->model))
                return set_error(KP_ERR_INVALID,
                                 "slow-light snapshots must share one grid, coordinate map and derived-scalar layout "
                                 "(snapshot %d differs)", i);
            if (!std::isfinite(times[i]) || (i > 0 && !(times[i] > times[i - 1])))
                return set_error(KP_ERR_INVALID, "snapshot times must be finite and strictly increasing");
        }
    }
    const int npix = params->camera.nx * params->camera.ny;
    int st = check_outputs(out, npix, nfreq);
    if (st != KP_OK) return st;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceState* dev = device_state(opt.device, &st);
    if (!dev) return st;
    cudaStream_t stream = opt.stream ? static_cast<cudaStream_t>(opt.stream) : dev->stream;
    st = ensure_job_table(dev, 1);
    if (st != KP_OK) return st;
    ImageOutPtrs dptr;
    if (opt.outputs_on_device) {
        dptr = from_abi(out);
    } else {
        void* buf = device_output_buffer(dev, carved_bytes(npix, nfreq), &st);
        if (!buf) return st;
        dptr = carve_outputs(buf, npix, nfreq);
    }
    cudaEventSynchronize(dev->staging_free);
    JobDesc& d = dev->h_jobs[0];
    std::memset(&d, 0, sizeof(d));
    d.c = make_consts_grmhd(params, grid, frequencies, nfreq, opt.integrator);
    if (slow) {
        // snapshot table then times, in one grow-only device buffer
        const size_t table = sizeof(GridConsts) * size_t(nsnap);
        const size_t bytes = table + sizeof(double) * size_t(nsnap);
        if (bytes > dev->series_bytes) {
            cudaStreamSynchronize(stream);
            cudaFree(dev->d_series);
            dev->d_series = nullptr;
            dev->series_bytes = 0;
            cudaError_t e = cudaMalloc(&dev->d_series, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return set_error(KP_ERR_OOM, "cudaMalloc(slow-light snapshot table): %s", cudaGetErrorString(e));
            }
            dev->series_bytes = bytes;
        }
        std::vector<unsigned char> host(bytes);
        for (int i = 0; i < nsnap; ++i) {
            const GridConsts g = grid_consts(grids[i]);
            std::memcpy(host.data() + sizeof(GridConsts) * size_t(i), &g, sizeof(g));
        }
        std::memcpy(host.data() + table, times, sizeof(double) * size_t(nsnap));
        cudaError_t e = cudaMemcpyAsync(dev->d_series, host.data(), bytes, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "slow-light snapshot table upload");
        d.c.scene = kSceneGrmhdFmksSlowLight;
        d.c.series = static_cast<const GridConsts*>(dev->d_series);
        d.c.series_times = reinterpret_cast<const double*>(static_cast<unsigned char*>(dev->d_series) + table);
        d.c.nseries = nsnap;
        d.c.t_obs = t_obs;
    }
    fmks_camera_frame(d.c.fmks, params->camera.radius, params->camera.inclination, d.frame.x, d.frame.e0,
                      d.frame.e1, d.frame.e2, d.frame.e3);
    d.out = dptr;
    d.ray_begin = 0;
    d.npix = npix;
    d.precision = opt.precision;
    const bool mixed = opt.precision == KP_PRECISION_MIXED;
    if (mixed) grmhd_emission_scale(params, grid->model, d.c);
    if (nctl > 0) grmhd_apply_control(params, grid->model, d.c, ctl, nctl);
    const int family = slow ? (mixed ? kFamilyGrmhdSlowMixed : kFamilyGrmhdSlowFP64)
                            : (mixed ? kFamilyGrmhdMixed : kFamilyGrmhdFP64);
    // mixed kernels are compiled with FMA contraction: one frequency form
    // for all mixed work keeps an image bit-identical here and in the server
    const int nf_form = (mixed || nfreq > 1) ? KP_MAX_FREQUENCIES : 1;
    st = run_wave_jobs(dev, stream, 1, npix, family, nf_form, opt, nullptr);
    if (st != KP_OK) return st;
    if (!opt.outputs_on_device) {
        st = copy_outputs_to_host(dptr, out, npix, nfreq, stream);
        if (st != KP_OK) return st;
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_error(e, "device-to-host copy");
    }
    return KP_OK;
}

}  // namespace

extern "C" {

int kp_image_grmhd(const kp_pass_a_params* params, const kp_grid* grid, int radiation_substeps,
                   const double* frequencies, int nfreq, const kp_run_options* options, kp_image_out* out) {
    const kp_grid* grids[1] = {grid};
    return grmhd_image(params, grids, nullptr, 0, 0.0, radiation_substeps, frequencies, nfreq, options, out);
}

int kp_image_grmhd_step_control(const kp_pass_a_params* params, const kp_grid* grid, int radiation_substeps,
                                const double* frequencies, int nfreq, const double* control_frequencies,
                                int ncontrol, const kp_run_options* options, kp_image_out* out) {
    const int st = validate_control(control_frequencies, ncontrol);
    if (st != KP_OK) return st;
    if (!grid) return set_error(KP_ERR_INVALID, "GRMHD image: null argument");
    if (nfreq > 1 && !frequencies) return set_error(KP_ERR_INVALID, "null frequency list");
    const kp_grid* grids[1] = {grid};
    const bool separate = separate_control(frequencies, nfreq, grid->model.freq_cgs, control_frequencies, ncontrol);
    return grmhd_image(params, grids, nullptr, 0, 0.0, radiation_substeps, frequencies, nfreq, options, out,
                       separate ? control_frequencies : nullptr, separate ? ncontrol : 0);
}

int kp_image_grmhd_slow_light(const kp_pass_a_params* params, const kp_grid* const* snapshots, const double* times,
                              int nsnap, double observation_time, int radiation_substeps, const double* frequencies,
                              int nfreq, const kp_run_options* options, kp_image_out* out) {
    if (!snapshots) return set_error(KP_ERR_INVALID, "kp_image_grmhd_slow_light: null snapshot list");
    if (nsnap < 2) return set_error(KP_ERR_INVALID, "slow-light requires at least two snapshots");
    return grmhd_image(params, snapshots, times, nsnap, observation_time, radiation_substeps, frequencies, nfreq,
                       options, out);
}

}  // extern "C"
