// cuda_simulation_b200.cpp -- the reference's cuda_simulation.cuh entry points
// (cuda_simulation.cuh:13-75, C++ linkage, void returns) and cuda_tool.cuh's fills on top
// of libsnowb200's C ABI.  Compiled with the reference's headers in place of
// cuda_simulation.cu and cuda_tool.cu; errors print the library's message and exit, as the
// reference's checkCudaErrors does.
#include "cuda_simulation.cuh"      // reference header: ParticleSet, CellData, SimParams, SceneParams
#include "cuda_tool.cuh"            // reference header: cuda_tool_fill_uint / _float
#include "snow_b200.h"              // this library
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static_assert(sizeof(ParticleDeviceData) == sizeof(snowb_particle_data), "layout");
static_assert(sizeof(CellData) == sizeof(snowb_cell_data), "layout");
static_assert(sizeof(SimParams) == sizeof(snowb_sim_params), "layout");
static_assert(sizeof(SceneParams) == sizeof(snowb_scene_params), "layout");

static void check(int rc) {
    if (rc != SNOWB_OK) { std::fprintf(stderr, "libsnowb200: %s\n", snowb_last_error_string()); std::exit(1); }
}
static snowb_particle_data* pd(ParticleSet* s) { return reinterpret_cast<snowb_particle_data*>(&s->m_device_data); }
static snowb_cell_data cd(CellData c) { snowb_cell_data r; std::memcpy(&r, &c, sizeof r); return r; }

void allocate_array(void** p, size_t n)                 { check(snowb_allocate_array(p, n)); }
void set_sim_params(SimParams& p)                       { check(snowb_set_sim_params(reinterpret_cast<snowb_sim_params*>(&p))); }
void compute_grid_size(uint n, uint bs, uint& nb, uint& nt) { check(snowb_compute_grid_size(n, bs, &nb, &nt)); }
void calculate_hash(CellData c, float3* pos, uint n)    { check(snowb_calculate_hash(cd(c), reinterpret_cast<snowb_float3*>(pos), n)); }
void sort_particles(CellData c, uint n)                 { check(snowb_sort_particles(cd(c), n)); }
void reorder_data(CellData c, float3* pos, uint n, uint cells) { check(snowb_reorder_data(cd(c), reinterpret_cast<snowb_float3*>(pos), n, cells)); }
void compute_boundary_volume(CellData c, float* m, float* v, uint n) { check(snowb_compute_boundary_volume(cd(c), m, v, n)); }
void integrate_pbd(ParticleSet* s, float dt, uint n, bool cd_on) { check(snowb_integrate_pbd(pd(s), dt, n, cd_on)); }

void snow_simulation(ParticleSet* sph, ParticleSet* dem, ParticleSet* b, ParticleDeviceData* buf,
                     CellData scd, CellData dcd, CellData bcd, SceneParams& sc, float dt, int iterations,
                     bool sph_dem, bool sph_sph, bool friction, bool temperature, bool change_phase,
                     bool freezing, bool melting, bool dem_visc, bool interlink, bool dynamic, bool cd_on,
                     float dT) {
    uint32_t ns = (uint32_t)sph->m_size, nd = (uint32_t)dem->m_size;
    check(snowb_snow_simulation(pd(sph), &ns, pd(dem), &nd, pd(b), (uint32_t)b->m_size,
                                (uint32_t)sph->m_full_size, reinterpret_cast<snowb_particle_data*>(buf),
                                cd(scd), cd(dcd), cd(bcd), reinterpret_cast<snowb_scene_params*>(&sc), dt,
                                iterations, sph_dem, sph_sph, friction, temperature, change_phase, freezing,
                                melting, dem_visc, interlink, dynamic, cd_on, dT));
    sph->setSize(ns);          // the reference's compact_and_clean does this (cuda_simulation.cu:4545-4546)
    dem->setSize(nd);
}

// connect_and_record (cuda_simulation.cu:4286-4292; defined there with C++ linkage, not
// declared in cuda_simulation.cuh): interlink formation over the sorted snow set.
void connect_and_record(ParticleSet* dem, CellData dcd, bool dynamic) {
    check(snowb_connect_and_record(pd(dem), (uint32_t)dem->m_size, cd(dcd), dynamic));
}

// cuda_tool.cu:3-13: d_arr[start, end) = value.  Called by ParticleSystem's set-up only, so
// one synchronous copy of a host buffer, after the library's stream has drained.
template <class T>
static void fill_range(T* d, size_t start, size_t end, T value) {
    if (end <= start) return;
    check(snowb_synchronize());
    std::vector<T> h(end - start, value);
    const cudaError_t e = cudaMemcpy(d + start, h.data(), (end - start) * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { std::fprintf(stderr, "cuda_tool fill: %s\n", cudaGetErrorString(e)); std::exit(1); }
}
void cuda_tool_fill_uint(uint* d_arr, size_t start, size_t end, uint value)    { fill_range(d_arr, start, end, value); }
void cuda_tool_fill_float(float* d_arr, size_t start, size_t end, float value) { fill_range(d_arr, start, end, value); }
