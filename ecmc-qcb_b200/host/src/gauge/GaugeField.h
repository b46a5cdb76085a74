// gauge/GaugeField.h -- the reference's GaugeField (src/gauge/GaugeField.h:18-62) backed by a
// device-resident libqcb field.
//
// `links` keeps the reference's host layout -- (site*4 + mu)*9 complex entries over the halo'd
// (L+2)^4 box of GeometryCB, row-major 3x3 -- and is synchronised lazily with the device copy:
// hot-path calls (heatbath, flow, observables, ILDG) upload host edits first and leave the device
// copy authoritative; view_link / view_link_const / links() bring the host copy up to date (halo
// filled periodically).  Writes through `links` directly must be followed by mark_host_modified().
#pragma once
#include <cstdint>
#include <random>
#include <vector>

#include "../../../../include/qcb.h"
#include "../geometry/GeometryCB.h"
#include "../su3/utils.h"

class GaugeField {
   public:
    std::vector<Complex> links;

    explicit GaugeField(const GeometryCB& geo);
    GaugeField(const GaugeField& other);
    GaugeField& operator=(const GaugeField& other);
    ~GaugeField();

    void hot_start(const GeometryCB& geo, std::mt19937_64& rng);
    void cold_start(const GeometryCB& geo);

    SU3Map view_link(size_t site, int mu);
    [[nodiscard]] SU3ConstMap view_link_const(size_t site, int mu) const;

    void projection_su3(size_t site, int mu);
    void project_field_su3(const GeometryCB& geo);
    void compute_staple(const GeometryCB& geo, size_t site, int mu, SU3& staple) const;

    // ---- device plumbing (no counterpart in the reference)
    qcb_field device() const;        // device handle with host edits uploaded
    void mark_device_modified();     // device copy changed: host copy is stale
    void mark_host_modified();       // host copy changed: device copy is stale
    const GeometryCB& geometry() const { return geo_; }
    // Heatbath stream state: Philox key and the next sweep index (the counter-based replacement
    // of the reference's saved std::mt19937_64 states, src/io/io.cpp:139-218).
    uint64_t hb_seed = 0;
    uint32_t hb_sweep = 0;
    bool hb_seeded = false;

    // Adopts an existing device field (used by GradientFlow::field_c); not owned.
    GaugeField(const GeometryCB& geo, qcb_field borrowed);

   private:
    GeometryCB geo_;
    mutable qcb_field h_ = nullptr;
    bool owns_ = true;
    mutable bool host_stale_ = false;
    mutable bool dev_stale_ = false;
    void sync_host() const;
    void upload_if_stale() const;
};

// Throws std::runtime_error with the library's message when a C ABI call fails.
void qcb_check(int status, const char* what);
