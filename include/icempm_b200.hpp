/*
 * icempm_b200.hpp — C++17 host classes over the C ABI of icempm_b200.h, with
 * the reference's class and method names, for a C++ host that drives the
 * step as the reference does:
 *
 *   HostSideSOA          the pinned-buffer SoA of host_side_soa.h (28 rows of
 *                        `capacity` doubles, row k at k * capacity), here a
 *                        std::vector over page-locked memory (mpm_host_alloc)
 *   GPU_Implementation6  gpu_implementation6.h:24-59 for one partition: the
 *                        halo and point-transfer methods do nothing
 *   Model3D              model_3d.h:30-55 / model_3d.cpp:24-112: Reset,
 *                        Prepare, Step (one frame of UpdateEveryNthStep
 *                        substeps through the phase API)
 *
 * A non-zero status of the library throws std::runtime_error carrying the
 * code (and the CUDA message for MPM_ERR_CUDA), where the reference throws on
 * CUDA errors. Header only; link with -licempm_b200.
 */
#ifndef ICEMPM_B200_HPP
#define ICEMPM_B200_HPP

#include <algorithm>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "icempm_b200.h"

namespace icempm {

inline void check(int code, const char* where) {
    if (code == MPM_OK) return;
    std::string msg = std::string(where) + ": status " + std::to_string(code);
    if (code == MPM_ERR_CUDA) msg += std::string(" (") + mpm_last_error_string() + ")";
    throw std::runtime_error(msg);
}

// Page-locked host memory from the library (mpm_host_alloc), as
// HostSideSOA::Allocate takes it with cudaMallocHost (host_side_soa.cpp:70-86).
template <class T>
struct PinnedAllocator {
    using value_type = T;
    PinnedAllocator() = default;
    template <class U>
    PinnedAllocator(const PinnedAllocator<U>&) {}
    T* allocate(std::size_t count) {
        void* p = nullptr;
        check(mpm_host_alloc(count * sizeof(T), &p), "mpm_host_alloc");
        return static_cast<T*>(p);
    }
    void deallocate(T* p, std::size_t) noexcept { mpm_host_free(p); }
    template <class U>
    bool operator==(const PinnedAllocator<U>&) const { return true; }
    template <class U>
    bool operator!=(const PinnedAllocator<U>&) const { return false; }
};

// HostSideSOA (host_side_soa.h): 28 rows of `capacity` doubles.
struct HostSideSOA {
    std::vector<double, PinnedAllocator<double>> host_buffer;
    unsigned capacity = 0;
    unsigned size = 0;

    void Allocate(unsigned cap) {
        capacity = cap;
        size = 0;
        host_buffer.assign((size_t)MPM_N_PTS_ARRAYS * cap, 0.0);
    }
    double* getPointerToLine(int k) { return host_buffer.data() + (size_t)k * capacity; }
};

class Model3D;

class GPU_Implementation6 {
public:
    Model3D* model = nullptr;
    HostSideSOA hssoa;
    double indenter_force[3] = {0, 0, 0};
    std::vector<double> indenter_sensor_total;
    int precision = MPM_PRECISION_FP64;
    int device = 0;

    GPU_Implementation6() = default;
    GPU_Implementation6(const GPU_Implementation6&) = delete;
    GPU_Implementation6& operator=(const GPU_Implementation6&) = delete;
    ~GPU_Implementation6() { mpm_destroy(h_); }

    inline void initialize();
    void allocate_arrays() {}
    void split_hssoa_into_partitions() {}        // one partition
    void enable_peer_access() {}
    void transfer_ponts_to_device() {
        check(mpm_upload_soa(h_, hssoa.host_buffer.data(), hssoa.capacity, hssoa.size), "mpm_upload_soa");
    }
    inline void transfer_from_device();
    void synchronize() { check(mpm_synchronize(h_), "mpm_synchronize"); }
    inline void update_constants();
    void reset_grid() { check(mpm_reset_grid(h_), "mpm_reset_grid"); }
    void reset_indenter_force_accumulator() {
        check(mpm_reset_indenter_force_accumulator(h_), "mpm_reset_indenter_force_accumulator");
    }
    void evaluate_indenter_total_force() {}     // done in transfer_from_device (mpm_sensors)
    void p2g() { check(mpm_p2g(h_), "mpm_p2g"); }
    void receive_halos() {}                     // one partition: no halo
    inline void update_nodes();
    void g2p(const bool recordPQ, const bool /*enablePointTransfer*/) { check(mpm_g2p(h_, recordPQ), "mpm_g2p"); }
    void receive_points() {}                    // one partition: no migration
    void record_timings(const bool /*enablePointTransfer*/) {}

    mpm_handle* handle() { return h_; }

private:
    mpm_handle* h_ = nullptr;
};

class Model3D {
public:
    SimParams3D prms;
    GPU_Implementation6 gpu;

    Model3D() {
        mpm_params_reset(&prms);
        gpu.model = this;
    }
    // model_3d.cpp:122-130
    void Reset() {
        prms.SimulationStep = 0;
        prms.SimulationTime = 0;
    }
    // model_3d.cpp:132-137
    void Prepare() { gpu.update_constants(); }
    // model_3d.cpp:24-112 for one partition: one frame of substeps, then the
    // transfer of the points, the sensors and the frame's indenter force
    bool Step() {
        double simulation_time = prms.SimulationTime;
        int count_unupdated_steps = 0;
        gpu.reset_indenter_force_accumulator();
        do {
            simulation_time += prms.InitialTimeStep;
            prms.indenter_x = prms.indenter_x_initial + simulation_time * prms.IndVelocity;
            gpu.reset_grid();
            gpu.p2g();
            gpu.receive_halos();
            gpu.update_nodes();
            const bool isZeroStep = (prms.SimulationStep + count_unupdated_steps) % prms.UpdateEveryNthStep == 0;
            gpu.g2p(isZeroStep, false);
            gpu.record_timings(false);
            count_unupdated_steps++;
        } while ((prms.SimulationStep + count_unupdated_steps) % prms.UpdateEveryNthStep != 0);
        prms.SimulationTime = simulation_time;
        prms.SimulationStep += count_unupdated_steps;
        gpu.transfer_from_device();
        return prms.SimulationTime < prms.SimulationEndTime;
    }
};

inline void GPU_Implementation6::initialize() {
    mpm_destroy(h_);
    h_ = nullptr;
    int st = 0;
    h_ = mpm_create(&model->prms, precision, std::max(hssoa.capacity, 1u), device, &st);
    if (!h_) check(st ? st : MPM_ERR_CUDA, "mpm_create");
    indenter_sensor_total.assign((size_t)3 * model->prms.IndenterSubdivisions * model->prms.GridZ, 0.0);
}

inline void GPU_Implementation6::update_constants() {
    check(mpm_update_constants(h_, &model->prms), "mpm_update_constants");
}

inline void GPU_Implementation6::update_nodes() {
    check(mpm_update_nodes(h_, model->prms.indenter_x, model->prms.indenter_y), "mpm_update_nodes");
}

inline void GPU_Implementation6::transfer_from_device() {
    unsigned n = 0;
    check(mpm_download_soa(h_, hssoa.host_buffer.data(), hssoa.capacity, &n), "mpm_download_soa");
    hssoa.size = n;
    check(mpm_sensors(h_, indenter_sensor_total.data(), indenter_force), "mpm_sensors");
}

}  // namespace icempm

#endif
