// kp_io.cu -- C ABI of the GRMHD dump readers (host code: iharm and KHARMA
// HDF5 dumps through kpolaris_b200/host/kp_iharm.hpp and kp_kharma.hpp).  Exceptions never cross
// the ABI: reader and format errors become KP_ERR_IO with their message.
#include <exception>
#include <stdexcept>
#include <string>

#include "kp_iharm.hpp"
#include "kp_kharma.hpp"
#include "kpolaris_b200.h"

namespace kp {
int set_error(int code, const char* fmt, ...);
}

namespace {

template <class F>
int guarded(F&& body) {
    try {
        return body();
    } catch (const kph5::FormatError& e) {
        return kp::set_error(KP_ERR_IO, "%s", e.what());
    } catch (const std::bad_alloc&) {
        return kp::set_error(KP_ERR_OOM, "host allocation failed while reading a dump");
    } catch (const std::exception& e) {
        return kp::set_error(KP_ERR_IO, "%s", e.what());
    }
}

}  // namespace

extern "C" {

void kp_default_iharm_options(kp_iharm_options* o) {
    if (!o) return;
    o->freq_cgs = 230.0e9;
    o->M_unit = 3.0e25;
    o->mbh_solar = 6.2e9;
    o->trat_small = 1.0;
    o->trat_large = 20.0;
    o->beta_crit = 1.0;
    o->sigma_cut = 1.0;
    o->sigma_cut_high = -1.0;
    o->emission_type = KP_FIT_DEXTER;
    o->interpolate_derived_scalars = 1;
}

int kp_iharm_read(const char* path, const kp_iharm_options* options, kp_grmhd_model* model, float* prims,
                  size_t capacity) {
    if (!path || !options || !model) return kp::set_error(KP_ERR_INVALID, "kp_iharm_read: null argument");
    return guarded([&] {
        kpb::IharmDump d = kpb::load_iharm_dump(path, *options, prims != nullptr);
        if (prims) {
            if (capacity < d.prims.size())
                return kp::set_error(KP_ERR_INVALID, "kp_iharm_read: primitives need %zu floats, capacity %zu",
                                     d.prims.size(), capacity);
            std::copy(d.prims.begin(), d.prims.end(), prims);
        }
        *model = d.model;
        return int(KP_OK);
    });
}

int kp_grid_load_iharm(const char* path, const kp_iharm_options* options, int device, kp_grmhd_model* model,
                       kp_grid** out) {
    if (!path || !options || !out) return kp::set_error(KP_ERR_INVALID, "kp_grid_load_iharm: null argument");
    *out = nullptr;
    kpb::IharmDump d;
    const int rc = guarded([&] {
        d = kpb::load_iharm_dump(path, *options, true);
        return int(KP_OK);
    });
    if (rc != KP_OK) return rc;
    if (model) *model = d.model;
    return kp_grid_upload(&d.model, d.prims.data(), device, out);
}

int kp_iharm_dump_time(const char* path, double* t) {
    if (!path || !t) return kp::set_error(KP_ERR_INVALID, "kp_iharm_dump_time: null argument");
    return guarded([&] {
        *t = kpb::read_iharm_dump_time(path);
        return int(KP_OK);
    });
}

int kp_kharma_read(const char* path, const kp_iharm_options* options, int reverse_field, kp_grmhd_model* model,
                   float* prims, size_t capacity) {
    if (!path || !options || !model) return kp::set_error(KP_ERR_INVALID, "kp_kharma_read: null argument");
    return guarded([&] {
        kpb::IharmDump d = kpb::load_kharma_dump(path, *options, reverse_field, prims != nullptr);
        if (prims) {
            if (capacity < d.prims.size())
                return kp::set_error(KP_ERR_INVALID, "kp_kharma_read: primitives need %zu floats, capacity %zu",
                                     d.prims.size(), capacity);
            std::copy(d.prims.begin(), d.prims.end(), prims);
        }
        *model = d.model;
        return int(KP_OK);
    });
}

int kp_grid_load_kharma(const char* path, const kp_iharm_options* options, int reverse_field, int device,
                        kp_grmhd_model* model, kp_grid** out) {
    if (!path || !options || !out) return kp::set_error(KP_ERR_INVALID, "kp_grid_load_kharma: null argument");
    *out = nullptr;
    kpb::IharmDump d;
    const int rc = guarded([&] {
        d = kpb::load_kharma_dump(path, *options, reverse_field, true);
        return int(KP_OK);
    });
    if (rc != KP_OK) return rc;
    if (model) *model = d.model;
    return kp_grid_upload(&d.model, d.prims.data(), device, out);
}

int kp_kharma_dump_time(const char* path, double* t) {
    if (!path || !t) return kp::set_error(KP_ERR_INVALID, "kp_kharma_dump_time: null argument");
    return guarded([&] {
        *t = kpb::read_kharma_dump_time(path);
        return int(KP_OK);
    });
}

}  // extern "C"
