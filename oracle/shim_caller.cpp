// Link check of the C++ shim (test infrastructure, built by shim_check.sh): a caller
// compiled against the reference's own declarations (cuda_simulation.cuh:13-75,
// cuda_tool.cuh:12-13) refers to every entry point and is linked with no undefined symbol
// against the shim.  A shim definition whose signature drifted from the declaration would
// be a separate overload and leave this caller's reference unresolved.  Nothing here is
// ever run.
#include "cuda_simulation.cuh"
#include "cuda_tool.cuh"

void snowb_shim_caller(ParticleSet* sph, ParticleSet* dem, ParticleSet* bnd, ParticleDeviceData* buf, CellData c,
                       SimParams& p, SceneParams& sc)
{
    void* ptr = nullptr;
    uint nb = 0, nt = 0;
    allocate_array(&ptr, 16);
    set_sim_params(p);
    integrate_pbd(dem, 0.f, 0u, false);
    compute_grid_size(0u, 256u, nb, nt);
    calculate_hash(c, nullptr, 0u);
    sort_particles(c, 0u);
    reorder_data(c, nullptr, 0u, 0u);
    compute_boundary_volume(c, nullptr, nullptr, 0u);
    snow_simulation(sph, dem, bnd, buf, c, c, c, sc, 0.f, 3, true, false, true, true, true, true, true, false,
                    true, false, true, 0.f);
    cuda_tool_fill_uint(nullptr, 0, 0, 0u);
    cuda_tool_fill_float(nullptr, 0, 0, 0.f);
}
