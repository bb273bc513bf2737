// snow_host.cpp -- C++ host driver on the reference's own interface.
//
// It plays the part of the reference's host code around the solver without OpenGL:
//   - buffers: one device array per ParticleDeviceData member for the water, snow and
//     boundary sets and the phase-change buffer, and the three CellData, allocated through
//     allocate_array as ParticleSystem::SetupCUDAMemory (ParticleSystem.cpp:148-858) and
//     NeighborSearch::InitializeCUDA (NeighborSearch.cpp:41-86) allocate them; the arrays the
//     reference maps from GL vertex buffers each frame (positions, T; Simulation.cpp:233-289)
//     are plain device arrays here;
//   - set-up: set_sim_params (Simulation.cpp:422), then the boundary's
//     calculate_hash / sort_particles / reorder_data / compute_boundary_volume sequence of
//     Simulation::InitializeBoundaryCudaData (Simulation.cpp:558-592), and, for scenes that
//     start with interlinks, one sort of the snow set and connect_and_record;
//   - stepping: snow_simulation(ParticleSet*, ParticleSet*, ParticleSet*, ParticleDeviceData*,
//     CellData x3, SceneParams&, dt, iterations, flags...) once per substep, with the
//     arguments Simulation::StepCUDA passes (Simulation.cpp:250-273); the set sizes come back
//     through ParticleSet::m_size.
// Every call goes through the declarations of cuda_simulation.cuh, so linked with
// cuda_simulation_b200.cpp (the shim over libsnowb200) this is the reference's host path
// running on this library.
//
// Usage: snow_host <scene.bin> <out.bin> <substeps>
// The scene file (snowsimulation_b200/host_io.py writes and reads it) holds the sizes,
// SimParams, SceneParams, the step settings and every array of the sets, the buffer and the
// cell data; out.bin receives the state after the substeps in the same format.
#include "cuda_simulation.cuh"
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

// defined in the reference's cuda_simulation.cu:4286 (and in the shim), not in its header
void connect_and_record(ParticleSet* dem_particles, CellData dem_cell_data, bool dynamic_max_connections);

namespace {

const char kMagic[8] = {'S', 'N', 'O', 'W', 'H', 'S', 'T', '1'};
const int kFields = 24;   // members of ParticleDeviceData (Particle.h:14-52)

struct Header {
    char magic[8];
    uint32_t n_sph, n_dem, n_b, full, maxc, num_cells, iterations, init_links, flags;
    float dt, temperature_variation;
    SimParams params;
    SceneParams scene;
};
static_assert(sizeof(SimParams) == 46 * 4, "SimParams layout");

// bytes of member k of ParticleDeviceData for n particles with maxc link slots each
size_t field_bytes(int k, size_t n, size_t maxc)
{
    if (k < 6) return n * sizeof(float3);                 // positions .. correction
    if (k < 16) return n * sizeof(float);                 // mass .. mass_scale
    if (k == 18) return sizeof(uint32_t);                 // new_end
    if (k == 19) return n * maxc * sizeof(uint32_t);      // connect_record
    if (k == 21) return n * maxc * sizeof(float);         // connect_length
    return n * sizeof(uint32_t);                          // predicate, scan_index, iter_end, new_index, trackId
}
void** members(ParticleDeviceData& d) { return reinterpret_cast<void**>(&d); }
void** members(CellData& c) { return reinterpret_cast<void**>(&c); }
size_t cell_bytes(int k, size_t n, size_t cells)
{
    if (k < 2) return n * sizeof(uint32_t);              // grid_hash, grid_index
    if (k < 4) return cells * sizeof(uint32_t);          // cell_start, cell_end
    return n * sizeof(float3);                           // sorted_pos
}

[[noreturn]] void die(const std::string& m)
{
    std::fprintf(stderr, "snow_host: %s\n", m.c_str());
    std::exit(2);
}
void cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) die(std::string(what) + ": " + cudaGetErrorString(e));
}

// one set's device arrays, filled from / written back to the file stream
struct DeviceState {
    Header h;
    ParticleSet sph, dem, bnd;
    ParticleDeviceData buf;
    CellData scd, dcd, bcd;

    void alloc_set(ParticleDeviceData& d, size_t n)
    {
        for (int k = 0; k < kFields; ++k) allocate_array(&members(d)[k], field_bytes(k, n, h.maxc));
    }
    void alloc_cells(CellData& c, size_t n)
    {
        for (int k = 0; k < 5; ++k) allocate_array(&members(c)[k], cell_bytes(k, n, h.num_cells));
    }
    template <class F>
    void each_array(F f)
    {
        ParticleDeviceData* sets[4] = {&sph.m_device_data, &dem.m_device_data, &bnd.m_device_data, &buf};
        const size_t ns[4] = {h.full, h.full, h.n_b, h.full};
        for (int s = 0; s < 4; ++s)
            for (int k = 0; k < kFields; ++k) f(members(*sets[s])[k], field_bytes(k, ns[s], h.maxc));
        CellData* cells[3] = {&scd, &dcd, &bcd};
        const size_t nc[3] = {h.full, h.full, h.n_b};
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 5; ++k) f(members(*cells[c])[k], cell_bytes(k, nc[c], h.num_cells));
    }
    void load(const char* path)
    {
        FILE* fp = std::fopen(path, "rb");
        if (!fp) die(std::string("cannot open ") + path);
        if (std::fread(&h, sizeof h, 1, fp) != 1 || std::memcmp(h.magic, kMagic, 8) != 0) die("bad scene header");
        sph.m_size = h.n_sph; sph.m_full_size = h.full;
        dem.m_size = h.n_dem; dem.m_full_size = h.full;
        bnd.m_size = h.n_b; bnd.m_full_size = h.n_b;
        alloc_set(sph.m_device_data, h.full);
        alloc_set(dem.m_device_data, h.full);
        alloc_set(bnd.m_device_data, h.n_b);
        alloc_set(buf, h.full);
        alloc_cells(scd, h.full);
        alloc_cells(dcd, h.full);
        alloc_cells(bcd, h.n_b);
        std::vector<char> tmp;
        each_array([&](void* dst, size_t bytes) {
            tmp.resize(bytes);
            if (bytes && std::fread(tmp.data(), 1, bytes, fp) != bytes) die("scene file too short");
            cuda(cudaMemcpy(dst, tmp.data(), bytes, cudaMemcpyHostToDevice), "upload");
        });
        std::fclose(fp);
    }
    void save(const char* path)
    {
        cuda(cudaDeviceSynchronize(), "synchronize");
        h.n_sph = (uint32_t)sph.m_size;
        h.n_dem = (uint32_t)dem.m_size;
        FILE* fp = std::fopen(path, "wb");
        if (!fp) die(std::string("cannot write ") + path);
        std::fwrite(&h, sizeof h, 1, fp);
        std::vector<char> tmp;
        each_array([&](void* src, size_t bytes) {
            tmp.resize(bytes);
            cuda(cudaMemcpy(tmp.data(), src, bytes, cudaMemcpyDeviceToHost), "download");
            std::fwrite(tmp.data(), 1, bytes, fp);
        });
        std::fclose(fp);
    }
    void release()
    {
        each_array([](void* p, size_t) { cudaFree(p); });
    }
};

bool flag(const Header& h, int bit) { return (h.flags >> bit) & 1u; }

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 4) die("usage: snow_host <scene.bin> <out.bin> <substeps>");
    const int substeps = std::atoi(argv[3]);
    DeviceState st;
    st.load(argv[1]);
    Header& h = st.h;

    set_sim_params(h.params);
    // Simulation::InitializeBoundaryCudaData (Simulation.cpp:558-592)
    ParticleDeviceData& b = st.bnd.m_device_data;
    calculate_hash(st.bcd, b.m_d_positions, h.n_b);
    sort_particles(st.bcd, h.n_b);
    reorder_data(st.bcd, b.m_d_positions, h.n_b, h.num_cells);
    compute_boundary_volume(st.bcd, b.m_d_mass, b.m_d_volume, h.n_b);
    if (h.init_links) {   // interlinks formed at rest: one sort of the snow set, then the link pass
        ParticleDeviceData& d = st.dem.m_device_data;
        calculate_hash(st.dcd, d.m_d_predict_positions, h.n_dem);
        sort_particles(st.dcd, h.n_dem);
        reorder_data(st.dcd, d.m_d_predict_positions, h.n_dem, h.num_cells);
        connect_and_record(&st.dem, st.dcd, flag(h, 9));
    }
    // Simulation::StepCUDA (Simulation.cpp:250-273), once per substep; flag bits follow the
    // argument order of snow_simulation (cuda_simulation.cuh:52-75)
    for (int k = 0; k < substeps; ++k)
        snow_simulation(&st.sph, &st.dem, &st.bnd, &st.buf, st.scd, st.dcd, st.bcd, h.scene, h.dt,
                        (int)h.iterations, flag(h, 0), flag(h, 1), flag(h, 2), flag(h, 3), flag(h, 4), flag(h, 5),
                        flag(h, 6), flag(h, 7), flag(h, 8), flag(h, 9), flag(h, 10), h.temperature_variation);
    st.save(argv[2]);
    st.release();
    std::printf("snow_host: %d substeps, %zu water + %zu snow\n", substeps, st.sph.m_size, st.dem.m_size);
    return 0;
}
