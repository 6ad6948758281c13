// Drives icempm::Model3D (include/icempm_b200.hpp) for a number of frames, as
// the reference's time loop drives its Model3D.
//   model3d_frames <params.bin> <soa.bin> <n> <frames> <precision> <out_soa.bin> <out_forces.bin>
// params.bin holds the raw SimParams3D block; soa.bin 28 rows of n doubles;
// out_soa.bin receives the final 28 x n SoA, out_forces.bin 3 doubles (the
// frame's indenter force) per frame.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <vector>

#include "icempm_b200.hpp"

static bool read_file(const char* path, void* dst, size_t bytes) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    const size_t got = std::fread(dst, 1, bytes, f);
    std::fclose(f);
    return got == bytes;
}

static bool write_file(const char* path, const void* src, size_t bytes) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    const size_t put = std::fwrite(src, 1, bytes, f);
    std::fclose(f);
    return put == bytes;
}

int main(int argc, char** argv) {
    if (argc != 8) {
        std::fprintf(stderr, "usage: %s params.bin soa.bin n frames precision out_soa.bin out_forces.bin\n", argv[0]);
        return 2;
    }
    const unsigned n = (unsigned)std::strtoul(argv[3], nullptr, 10);
    const int frames = std::atoi(argv[4]);
    try {
        icempm::Model3D model;
        if (!read_file(argv[1], &model.prms, sizeof(SimParams3D))) return 3;
        std::vector<double> soa((size_t)MPM_N_PTS_ARRAYS * n);
        if (!read_file(argv[2], soa.data(), sizeof(double) * soa.size())) return 4;
        icempm::GPU_Implementation6& gpu = model.gpu;
        gpu.precision = std::atoi(argv[5]);
        gpu.hssoa.Allocate(n);
        for (int k = 0; k < MPM_N_PTS_ARRAYS; k++)
            std::memcpy(gpu.hssoa.getPointerToLine(k), soa.data() + (size_t)k * n, sizeof(double) * n);
        gpu.hssoa.size = n;
        gpu.initialize();
        gpu.allocate_arrays();
        gpu.split_hssoa_into_partitions();
        gpu.transfer_ponts_to_device();
        model.Prepare();
        std::vector<double> forces;
        for (int f = 0; f < frames; f++) {
            model.Step();
            forces.insert(forces.end(), gpu.indenter_force, gpu.indenter_force + 3);
        }
        gpu.synchronize();
        if (!write_file(argv[6], gpu.hssoa.host_buffer.data(), sizeof(double) * gpu.hssoa.host_buffer.size())) return 5;
        if (!write_file(argv[7], forces.data(), sizeof(double) * forces.size())) return 6;
        std::printf("frames %d, SimulationStep %d, points %u\n", frames, model.prms.SimulationStep, gpu.hssoa.size);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
