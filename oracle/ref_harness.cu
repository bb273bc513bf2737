// ref_harness.cu -- drives the reference's own solver (cuda_simulation.cu, unmodified)
// from a C ABI so tests can run it on the same seeded scenes as the oracle and the B200
// library.  TEST INFRASTRUCTURE, built by ref_build.sh into oracle/_ref/.
//
// The harness owns plain cudaMalloc'd device buffers in place of the reference's GL
// vertex buffers (Simulation.cpp:233-289) and fills them from host arrays laid out like
// ParticleDeviceData / CellData, then calls the reference's entry points in the order
// Simulation::InitializeBoundaryCudaData (Simulation.cpp:558-592) and StepCUDA use them.
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>
#include "cuda_simulation.cuh"

// The two out-of-line ParticleSet members the solver's types need (Particle.cpp:172-210
// holds the reference's versions, which also size host vectors this harness never uses).
ParticleSet::ParticleSet() : m_size(0), m_full_size(0) {}
ParticleSet::~ParticleSet() {}

// defined in cuda_simulation.cu:4286, not declared in its header
void connect_and_record(ParticleSet* dem_particles, CellData dem_cell_data, bool dynamic_max_connections);

namespace {
struct Layout {
    size_t n, maxc;
};
// byte size of field k of ParticleDeviceData (Particle.h:14-52) for n particles
size_t field_bytes(int k, const Layout& L)
{
    if (k < 6) return L.n * sizeof(float3);          // positions .. correction
    if (k < 16) return L.n * sizeof(float);          // mass .. mass_scale
    if (k == 18) return sizeof(uint32_t);            // new_end
    if (k == 19) return L.n * L.maxc * sizeof(uint32_t);   // connect_record
    if (k == 21) return L.n * L.maxc * sizeof(float);      // connect_length
    return L.n * sizeof(uint32_t);                   // predicate, scan_index, iter_end, new_index, trackId
}
const int kFields = 24;
void** fields(ParticleDeviceData& d) { return reinterpret_cast<void**>(&d); }
void** cfields(CellData& c) { return reinterpret_cast<void**>(&c); }

struct World {
    ParticleSet sph, dem, bnd;
    ParticleDeviceData buf;
    CellData scd, dcd, bcd;
    Layout Lfull, Lb;
    uint32_t ncells;
    SceneParams scene;
};
World* g_w = nullptr;

int alloc_set(ParticleDeviceData& d, const Layout& L)
{
    std::memset(&d, 0, sizeof(d));
    for (int k = 0; k < kFields; ++k)
        if (cudaMalloc(&fields(d)[k], field_bytes(k, L)) != cudaSuccess) return -1;
    return 0;
}
int alloc_cells(CellData& c, size_t n, uint32_t ncells)
{
    if (cudaMalloc(&c.grid_hash, n * 4) || cudaMalloc(&c.grid_index, n * 4) || cudaMalloc(&c.cell_start, ncells * 4) ||
        cudaMalloc(&c.cell_end, ncells * 4) || cudaMalloc(&c.sorted_pos, n * sizeof(float3)))
        return -1;
    return 0;
}
ParticleDeviceData* set_ptr(int s)
{
    switch (s) {
    case 0: return &g_w->sph.m_device_data;
    case 1: return &g_w->dem.m_device_data;
    case 2: return &g_w->bnd.m_device_data;
    default: return &g_w->buf;
    }
}
CellData* cell_ptr(int s) { return s == 0 ? &g_w->scd : s == 1 ? &g_w->dcd : &g_w->bcd; }
}  // namespace

// the reference's functions used by ref_step_until (C++ linkage, defined in cuda_simulation.cu)
__global__ void compute_snow_sph_density_d(float*, float*, float*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_snow_dem_sph_density_d(float*, float*, float*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_snow_boundary_density_d(float*, float*, float*, float*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_snow_sph_lambdas_d(float*, float*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_dem_sph_lambdas_d(float*, float3*, float*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_snow_boundary_lambdas_d(float*, float*, float3*, float*, float*, CellData, CellData, CellData, uint);
__global__ void compute_pbf_sph_correction(ParticleDeviceData, ParticleDeviceData, ParticleDeviceData, CellData, CellData, CellData, uint, float);
__global__ void compute_pbf_new_dem_correction(ParticleDeviceData, ParticleDeviceData, ParticleDeviceData, CellData, CellData, CellData, uint, float);
__global__ void compute_sph_dem_distance_correction(ParticleDeviceData, ParticleDeviceData, CellData, CellData, uint);
__global__ void compute_dem_sph_distance_correction(ParticleDeviceData, ParticleDeviceData, CellData, CellData, uint);
__global__ void compute_sph_sph_distance_correction(ParticleDeviceData, CellData, uint);
__global__ void compute_dem_distance_correction(ParticleDeviceData, ParticleDeviceData, CellData, CellData, uint);
__global__ void apply_correction(ParticleDeviceData, CellData, uint);
__global__ void compute_friction_correction(float3*, float3*, float3*, float*, float*, CellData, CellData, uint);
__global__ void finalize_correction(float3*, float3*, float3*, float3*, uint, float);
void sort_and_reorder(float3*, CellData, uint, uint);
void transfer_heat(ParticleDeviceData, ParticleDeviceData, CellData, CellData, uint, uint, float, uint, uint, uint, uint);
void environmental_heat_transfer(ParticleSet*, ParticleSet*, float, bool, bool);
void phase_change(ParticleSet*, ParticleSet*, ParticleDeviceData, bool, bool);
void adjust_connections(ParticleSet*);
void solve_snow_interlink_constraint(ParticleSet*);
void apply_XSPH_viscosity(ParticleSet*, ParticleSet*, CellData, CellData, uint, uint, bool, bool, bool);


extern "C" {

int ref_create(const SimParams* p, uint32_t full, uint32_t n_sph, uint32_t n_dem, uint32_t n_b, uint32_t maxc)
{
    if (g_w) return -2;
    g_w = new World();
    g_w->Lfull = {full, maxc};
    g_w->Lb = {n_b, maxc};
    g_w->ncells = p->num_cells;
    ParticleSet* sets[3] = {&g_w->sph, &g_w->dem, &g_w->bnd};
    for (int s = 0; s < 3; ++s) {
        ParticleSet* ps = sets[s];
        ps->m_full_size = s == 2 ? n_b : full;
        ps->m_size = s == 0 ? n_sph : s == 1 ? n_dem : n_b;
        ps->m_maximum_connection = maxc;
        if (alloc_set(ps->m_device_data, s == 2 ? g_w->Lb : g_w->Lfull)) return -1;
    }
    if (alloc_set(g_w->buf, g_w->Lfull)) return -1;
    if (alloc_cells(g_w->scd, full, p->num_cells) || alloc_cells(g_w->dcd, full, p->num_cells) ||
        alloc_cells(g_w->bcd, n_b, p->num_cells))
        return -1;
    SimParams q = *p;
    set_sim_params(q);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// host <-> device copies of one particle set (s: 0 water, 1 snow, 2 boundary, 3 buffer) or
// one cell data (s: 0..2); host pointers laid out like the device structs
int ref_copy_set(int s, void* const* host, int to_device)
{
    ParticleDeviceData* d = set_ptr(s);
    const Layout& L = s == 2 ? g_w->Lb : g_w->Lfull;
    for (int k = 0; k < kFields; ++k) {
        if (!host[k]) continue;
        cudaError_t e = to_device ? cudaMemcpy(fields(*d)[k], host[k], field_bytes(k, L), cudaMemcpyHostToDevice)
                                  : cudaMemcpy(host[k], fields(*d)[k], field_bytes(k, L), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return -1;
    }
    return 0;
}
int ref_copy_cells(int s, void* const* host, int to_device)
{
    CellData* c = cell_ptr(s);
    const size_t n = s == 2 ? g_w->Lb.n : g_w->Lfull.n;
    const size_t bytes[5] = {n * 4, n * 4, (size_t)g_w->ncells * 4, (size_t)g_w->ncells * 4, n * sizeof(float3)};
    for (int k = 0; k < 5; ++k) {
        if (!host[k]) continue;
        cudaError_t e = to_device ? cudaMemcpy(cfields(*c)[k], host[k], bytes[k], cudaMemcpyHostToDevice)
                                  : cudaMemcpy(host[k], cfields(*c)[k], bytes[k], cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return -1;
    }
    return 0;
}

// Simulation::InitializeBoundaryCudaData (Simulation.cpp:558-592)
int ref_init_boundary(void)
{
    ParticleSet& b = g_w->bnd;
    const uint32_t n = (uint32_t)b.m_size;
    calculate_hash(g_w->bcd, b.m_device_data.m_d_positions, n);
    sort_particles(g_w->bcd, n);
    reorder_data(g_w->bcd, b.m_device_data.m_d_positions, n, g_w->ncells);
    compute_boundary_volume(g_w->bcd, b.m_device_data.m_d_mass, b.m_device_data.m_d_volume, n);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// initial interlinks at rest: one sort of the snow set and connect_and_record
int ref_init_links(int dynamic)
{
    ParticleSet& d = g_w->dem;
    const uint32_t n = (uint32_t)d.m_size;
    calculate_hash(g_w->dcd, d.m_device_data.m_d_predict_positions, n);
    sort_particles(g_w->dcd, n);
    reorder_data(g_w->dcd, d.m_device_data.m_d_predict_positions, n, g_w->ncells);
    connect_and_record(&d, g_w->dcd, dynamic != 0);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1;
}

// one snow_simulation call (cuda_simulation.cu:4861-5157); flags in argument order
int ref_step(float* scene3, float dt, int iterations, const int* f, float dTe, uint32_t* sizes)
{
    SceneParams& sc = g_w->scene;
    sc.fluid_start_time = scene3[0];
    sc.solid_start_time = scene3[1];
    sc.current_time = scene3[2];
    snow_simulation(&g_w->sph, &g_w->dem, &g_w->bnd, &g_w->buf, g_w->scd, g_w->dcd, g_w->bcd, sc, dt, iterations,
                    f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], dTe);
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    scene3[2] = sc.current_time;
    sizes[0] = (uint32_t)g_w->sph.m_size;
    sizes[1] = (uint32_t)g_w->dem.m_size;
    return 0;
}

// snow_simulation (cuda_simulation.cu:4861-5157) restated as the same sequence of calls to
// the reference's own host functions and kernels, stopping after stage `stop_after`
// (numbering as in the CPU oracle: 1 start sorts, 2 density, 3 heat, 4 phase change,
// 5 sorts, 6 links, 7 integrate, 10*(it+1)+k inside iteration it with k = 0 sorts,
// 1 density, 2 lambda, 3 PBF, 4 contact, 5 interlink, 6 apply, 7 friction, and 90 after
// finalize).  The inline wrappers of the reference (compute_snow_pbf_* and
// compute_snow_distance_correction) are replaced by their kernel launches with the same
// grid shapes.  Used to compare deterministic stages of the reference with the oracle.
namespace {
void grid_of(uint n, uint& blocks, uint& threads)   // compute_grid_size(n, 512) (:348-357)
{
    if (n == 0) { blocks = threads = 0; return; }
    threads = n < 512u ? n : 512u;
    blocks = (n % threads != 0) ? (n / threads + 1) : (n / threads);
}
}  // namespace

int ref_step_until(float* scene3, float dt, int iterations, const int* f, float dTe, int stop_after,
                   uint32_t* sizes)
{
#define STOP(k) do { if (stop_after == (k)) goto done; } while (0)
    {
    World& W = *g_w;
    ParticleSet* sph = &W.sph; ParticleSet* dem = &W.dem; ParticleSet* bnd = &W.bnd;
    SceneParams& sc = W.scene;
    sc.fluid_start_time = scene3[0]; sc.solid_start_time = scene3[1]; sc.current_time = scene3[2];
    const bool correct_dem = f[0], sph_sph = f[1], friction = f[2], temperature = f[3], change = f[4],
               freezing = f[5], melting = f[6], dem_visc = f[7], interlink = f[8], dynamic = f[9], cd_on = f[10];
    const bool step_sph = sc.current_time >= sc.fluid_start_time;
    const bool step_dem = sc.current_time >= sc.solid_start_time;
    uint sb, st, db, dt_;
    grid_of((uint)sph->m_size, sb, st);
    grid_of((uint)dem->m_size, db, dt_);
    auto sorts = [&]() {
        sort_and_reorder(dem->m_device_data.m_d_predict_positions, W.dcd, (uint)dem->m_size, 262144u);
        sort_and_reorder(sph->m_device_data.m_d_predict_positions, W.scd, (uint)sph->m_size, 262144u);
    };
    auto density = [&]() {
        uint a, b, c, d, e, g;
        grid_of((uint)sph->m_size, a, b); grid_of((uint)dem->m_size, c, d); grid_of((uint)bnd->m_size, e, g);
        ParticleDeviceData &S = sph->m_device_data, &D = dem->m_device_data, &B = bnd->m_device_data;
        compute_snow_sph_density_d<<<a, b>>>(S.m_d_density, S.m_d_mass, S.m_d_C, D.m_d_mass, B.m_d_volume, W.scd, W.dcd, W.bcd, (uint)sph->m_size);
        compute_snow_dem_sph_density_d<<<c, d>>>(S.m_d_mass, D.m_d_mass, D.m_d_C, D.m_d_density, B.m_d_volume, W.scd, W.dcd, W.bcd, (uint)dem->m_size);
        compute_snow_boundary_density_d<<<e, g>>>(S.m_d_mass, D.m_d_mass, B.m_d_mass, B.m_d_volume, B.m_d_C, B.m_d_density, W.scd, W.dcd, W.bcd, (uint)bnd->m_size);
    };
    sorts();
    STOP(1);
    density();
    STOP(2);
    if (temperature) {
        transfer_heat(sph->m_device_data, dem->m_device_data, W.scd, W.dcd, (uint)sph->m_size, (uint)dem->m_size, dt, sb, st, db, dt_);
        environmental_heat_transfer(sph, dem, dTe, step_sph, step_dem);
    }
    STOP(3);
    if (change) phase_change(sph, dem, W.buf, freezing, melting);
    STOP(4);
    sorts();
    STOP(5);
    if (interlink) connect_and_record(dem, W.dcd, dynamic);
    if (interlink && dynamic) adjust_connections(dem);
    STOP(6);
    if (step_sph) integrate_pbd(sph, dt, (uint)sph->m_size, cd_on);
    if (step_dem) integrate_pbd(dem, dt, (uint)dem->m_size, cd_on);
    STOP(7);
    for (int it = 0; it < iterations; ++it) {
        const int base = 10 + 10 * it;
        ParticleDeviceData &S = sph->m_device_data, &D = dem->m_device_data, &B = bnd->m_device_data;
        sorts();
        STOP(base + 0);
        density();
        STOP(base + 1);
        {
            uint a, b, c, d, e, g;
            grid_of((uint)sph->m_size, a, b); grid_of((uint)dem->m_size, c, d); grid_of((uint)bnd->m_size, e, g);
            compute_snow_sph_lambdas_d<<<a, b>>>(S.m_d_lambda, S.m_d_C, S.m_d_mass, B.m_d_volume, W.scd, W.dcd, W.bcd, (uint)sph->m_size);
            compute_dem_sph_lambdas_d<<<c, d>>>(D.m_d_lambda, D.m_d_positions, D.m_d_C, D.m_d_mass, B.m_d_volume, W.scd, W.dcd, W.bcd, (uint)dem->m_size);
            compute_snow_boundary_lambdas_d<<<e, g>>>(B.m_d_lambda, B.m_d_volume, B.m_d_positions, B.m_d_C, B.m_d_mass, W.scd, W.dcd, W.bcd, (uint)bnd->m_size);
        }
        STOP(base + 2);
        {
            uint a, b, c, d;
            grid_of((uint)sph->m_size, a, b); grid_of((uint)dem->m_size, c, d);
            compute_pbf_sph_correction<<<a, b>>>(S, D, B, W.scd, W.dcd, W.bcd, (uint)sph->m_size, dt);
            compute_pbf_new_dem_correction<<<c, d>>>(S, D, B, W.scd, W.dcd, W.bcd, (uint)dem->m_size, dt);
        }
        STOP(base + 3);
        {
            uint a, b, c, d;
            grid_of((uint)sph->m_size, a, b); grid_of((uint)dem->m_size, c, d);
            if (correct_dem) {
                compute_sph_dem_distance_correction<<<a, b>>>(S, D, W.scd, W.dcd, (uint)sph->m_size);
                compute_dem_sph_distance_correction<<<c, d>>>(D, S, W.dcd, W.scd, (uint)dem->m_size);
            }
            if (sph_sph) compute_sph_sph_distance_correction<<<a, b>>>(S, W.scd, (uint)sph->m_size);
            compute_dem_distance_correction<<<c, d>>>(D, B, W.dcd, W.bcd, (uint)dem->m_size);
        }
        STOP(base + 4);
        if (interlink) solve_snow_interlink_constraint(dem);
        STOP(base + 5);
        if (step_sph) apply_correction<<<sb, st>>>(S, W.scd, (uint)sph->m_size);
        if (step_dem) apply_correction<<<db, dt_>>>(D, W.dcd, (uint)dem->m_size);
        STOP(base + 6);
        if (friction && step_dem) {
            sorts();
            compute_friction_correction<<<db, dt_>>>(D.m_d_correction, D.m_d_new_positions, D.m_d_positions, D.m_d_massInv,
                                                     B.m_d_massInv, W.dcd, W.bcd, (uint)dem->m_size);
            apply_correction<<<db, dt_>>>(D, W.dcd, (uint)dem->m_size);
        }
        STOP(base + 7);
    }
    if (step_sph)
        finalize_correction<<<sb, st>>>(sph->m_device_data.m_d_positions, sph->m_device_data.m_d_new_positions,
                                       sph->m_device_data.m_d_predict_positions, sph->m_device_data.m_d_velocity,
                                       (uint)sph->m_size, dt);
    if (step_dem)
        finalize_correction<<<db, dt_>>>(dem->m_device_data.m_d_positions, dem->m_device_data.m_d_new_positions,
                                        dem->m_device_data.m_d_predict_positions, dem->m_device_data.m_d_velocity,
                                        (uint)dem->m_size, dt);
    STOP(90);
    apply_XSPH_viscosity(sph, dem, W.scd, W.dcd, (uint)sph->m_size, (uint)dem->m_size, step_sph, step_dem, dem_visc);
    sc.current_time += dt;
    }
done:
#undef STOP
    if (cudaDeviceSynchronize() != cudaSuccess) return -1;
    scene3[2] = g_w->scene.current_time;
    sizes[0] = (uint32_t)g_w->sph.m_size;
    sizes[1] = (uint32_t)g_w->dem.m_size;
    return 0;
}

int ref_destroy(void)
{
    if (!g_w) return 0;
    ParticleDeviceData* ds[4] = {&g_w->sph.m_device_data, &g_w->dem.m_device_data, &g_w->bnd.m_device_data, &g_w->buf};
    for (auto* d : ds)
        for (int k = 0; k < kFields; ++k) cudaFree(fields(*d)[k]);
    CellData* cs[3] = {&g_w->scd, &g_w->dcd, &g_w->bcd};
    for (auto* c : cs)
        for (int k = 0; k < 5; ++k) cudaFree(cfields(*c)[k]);
    delete g_w;
    g_w = nullptr;
    return 0;
}

}  // extern "C"
