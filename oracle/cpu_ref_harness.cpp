// cpu_ref_harness.cpp -- C entry points around the reference's own CPU code, used for the
// reported CPU baselines of the measurement (test and measurement infrastructure: only
// tests and the CPU-baseline leg of the benchmark load it; nothing on the product path).
//
// The reference's CPU sources are compiled unmodified where they lie (NeighborSearch.cpp,
// ConstraintSolver.cpp, Constraints.cpp, Particle.cpp, Collider.cpp,
// CollisionDetection.cpp); see cpu_ref_build.sh.  ParticleSystem.cpp is not compiled: it
// holds the OpenGL buffer code.  The three ParticleSystem members that the neighbour
// search needs are defined below with the effect of ParticleSystem.cpp:8-23 and :115-119.
#include <chrono>
#include <cstdint>
#include <memory>
#include <vector>

#include "ConstraintSolver.h"
#include "NeighborSearch.h"

ParticleSystem::ParticleSystem()
    : m_sph_particles(nullptr), m_dem_particles(nullptr), m_boundary_particles(nullptr),
      m_particle_radius(5.f), m_hottest_temperature(10.f), m_coolest_temperature(-10.f)
{
}
ParticleSystem::~ParticleSystem() { m_particle_indices.clear(); }
ParticleSet* ParticleSystem::AllocateSPHParticles(size_t n, float particle_mass)
{
    m_sph_particles = new ParticleSet(n, particle_mass);
    return m_sph_particles;
}

namespace {
double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

// NeighborSearch::SpatialSearch (NeighborSearch.cpp:154-259) over n predicted positions
// (xyz triples) of the water set with radius h.  One untimed call fills the hash table,
// then `calls` timed calls; *pairs = directed neighbour pairs found (|xi - xj|^2 <= h^2,
// i != j), *sec_per_call = mean seconds per call.  The search runs on the 8 OpenMP threads
// the reference hard-wires (NeighborSearch.cpp:210).
int cpuref_spatial_search(const float* pos, uint32_t n, float h, int calls, uint64_t* pairs,
                          double* sec_per_call)
{
    if (!pos || !pairs || !sec_per_call || calls < 1) return -1;
    auto ps = std::make_shared<ParticleSystem>();
    ParticleSet* set = ps->AllocateSPHParticles(n, 1.f);
    for (uint32_t i = 0; i < n; ++i)
        set->m_predict_positions[i] = glm::vec3(pos[3ull * i], pos[3ull * i + 1], pos[3ull * i + 2]);
    uint64_t found = 0;
    {
        NeighborSearch ns(ps, make_uint3(64, 64, 64));
        ns.Initialize();
        ns.SpatialSearch(h);
        const double t0 = now_s();
        for (int c = 0; c < calls; ++c) ns.SpatialSearch(h);
        *sec_per_call = (now_s() - t0) / calls;
        for (uint32_t i = 0; i < n; ++i) found += ns.FetchNeighbors(i).size();
    }
    *pairs = found;
    delete set;
    return 0;
}

// ConstraintSolver::SolveXPBDConstraints (ConstraintSolver.cpp:51-72) over one
// DistanceConstraint (Constraints.cpp) per link pair (a[k], b[k]) with rest length rest[k],
// `iters` solver iterations, on particles of mass `mass` whose new positions start at pos.
// Each of `calls` timed solves restarts from pos (the reset is outside the timing);
// out_pos (n xyz triples, may be null) receives the new positions after the last solve.
int cpuref_xpbd_links(const float* pos, uint32_t n, const uint32_t* a, const uint32_t* b, const float* rest,
                      uint32_t npairs, float mass, float dt, int iters, int calls, double* sec_per_call,
                      float* out_pos)
{
    if (!pos || !a || !b || !rest || !sec_per_call || calls < 1 || iters < 1) return -1;
    for (uint32_t k = 0; k < npairs; ++k)
        if (a[k] >= n || b[k] >= n) return -2;
    std::vector<Particle_Ptr> parts(n);
    for (uint32_t i = 0; i < n; ++i)
        parts[i] = std::make_shared<Particle>(glm::vec3(pos[3ull * i], pos[3ull * i + 1], pos[3ull * i + 2]), mass);
    std::vector<Constraint*> links;
    links.reserve(npairs);
    for (uint32_t k = 0; k < npairs; ++k) links.push_back(new DistanceConstraint(parts[a[k]], parts[b[k]], rest[k]));
    std::vector<Constraint*> none;
    ConstraintSolver solver(PBD_MODE::XPBD);
    solver.setSolverIteration((uint32_t)iters);
    double total = 0.0;
    for (int c = 0; c < calls; ++c) {
        for (uint32_t i = 0; i < n; ++i) parts[i]->m_new_position = parts[i]->m_position;
        const double t0 = now_s();
        solver.SolveConstraints(dt, links, none);
        total += now_s() - t0;
    }
    *sec_per_call = total / calls;
    if (out_pos)
        for (uint32_t i = 0; i < n; ++i) {
            out_pos[3ull * i] = parts[i]->m_new_position.x;
            out_pos[3ull * i + 1] = parts[i]->m_new_position.y;
            out_pos[3ull * i + 2] = parts[i]->m_new_position.z;
        }
    for (Constraint* c : links) delete c;
    return 0;
}

}  // extern "C"
