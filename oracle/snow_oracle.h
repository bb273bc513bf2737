/*
 * snow_oracle.h -- CPU oracle for the SnowSimulation substep (TEST INFRASTRUCTURE).
 *
 * This header and snow_oracle.c are a plain-C restatement of the per-substep
 * solver behind snow_simulation() in the reference (cuda_simulation.cu:4861-5157).
 * They are the checker for the CUDA library, never part of it: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline may load them.
 *
 * The same source builds two libraries:
 *   liboracle32.so  (ORACLE_REAL=float)  -- performs exactly the IEEE FP32
 *                   operations that the CUDA kernels perform (the reference's
 *                   expressions, no fused multiply-add, correctly rounded sqrt/div,
 *                   identical per-cell summation order), so CUDA-vs-oracle parity
 *                   is bit-exact;
 *   liboracle64.so  (ORACLE_REAL=double) -- the FP64 reference run used to
 *                   report the FP32 error.
 *
 * Data layout mirrors the reference ABI: AoS xyz triples per particle,
 * original-index order, sets padded to full_size (Particle.h:14-52,
 * NeighborSearch.h:19-26, SimParams.h:7-62, SceneParams.h:4-9).
 */
#ifndef SNOW_ORACLE_H
#define SNOW_ORACLE_H

#include <stdint.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

typedef struct { real x, y, z; } r3;

/* Same field order as ParticleDeviceData (Particle.h:14-52). */
typedef struct {
    r3 *positions, *predict_positions, *new_positions, *velocity, *force, *correction;
    real *mass, *massInv, *density, *C, *lambda, *volume;
    real *T, *new_T;
    real *contrib;
    real *mass_scale;
    uint32_t *predicate, *scan_index, *new_end;
    uint32_t *connect_record, *iter_end;
    real *connect_length;
    uint32_t *new_index;
    uint32_t *trackId;
} or_particles;

/* CellData (NeighborSearch.h:19-26). */
typedef struct {
    uint32_t *grid_hash, *grid_index, *cell_start, *cell_end;
    r3 *sorted_pos;
} or_cells;

/* SimParams (SimParams.h:7-62); every member is 4 bytes, float3/uint3 are 3 members. */
typedef struct {
    float gravity[3];
    float global_damping, maximum_speed, minimum_speed;
    float epsilon, pbd_epsilon, kernel_epsilon, effective_radius, particle_radius;
    float rest_density, scorr_coeff, scorr_divisor;
    float boundary_damping, static_friction, kinematic_friction;
    float k_stretch;
    float k_water, k_snow, C_water, C_snow, freezing_point;
    float blending_speed;
    float sor_coeff, sph_viscosity, dem_viscosity;
    float world_origin[3];
    float cell_size[3];
    uint32_t grid_size[3];
    uint32_t num_cells;
    float poly6, poly6_G, spiky, spiky_G, viscosity_laplacian;
    uint32_t maximum_connection;
    float T_homogeneous, k_refreezing, break_threshold;
} or_params;

typedef struct { float fluid_start_time, solid_start_time, current_time; } or_scene;

/* Flags of snow_simulation() (cuda_simulation.cuh:52-75), as bits. */
enum {
    OR_SPH_DEM_CORRECTION = 1u << 0,
    OR_SPH_SPH_CORRECTION = 1u << 1,
    OR_DEM_FRICTION       = 1u << 2,
    OR_COMPUTE_TEMPERATURE= 1u << 3,
    OR_CHANGE_PHASE       = 1u << 4,
    OR_SIMULATE_FREEZING  = 1u << 5,
    OR_SIMULATE_MELTING   = 1u << 6,
    OR_DEM_VISCOSITY      = 1u << 7,
    OR_USE_INTERLINK      = 1u << 8,
    OR_DYNAMIC_MAX_CONN   = 1u << 9,
    OR_CD_ON              = 1u << 10
};

/* quirks: 0 = reproduce the reference's deterministic quirks, 1 = intended physics. */
enum { OR_QUIRKS_REFERENCE = 0, OR_QUIRKS_FIXED = 1 };

/* grid / neighbor structure (cuda_simulation.cu:359-420) */
void or_calculate_hash(const or_params* P, or_cells cd, const r3* pos, uint32_t n);
void or_sort_particles(or_cells cd, uint32_t n);
void or_reorder_data(or_cells cd, const r3* pos, uint32_t n, uint32_t num_cells);
void or_compute_boundary_volume(const or_params* P, or_cells cd, const real* mass, real* volume, uint32_t n);

/*
 * One substep.  sizes are in/out (ParticleSet::m_size after the call).
 * stop_after: 0 = whole substep; otherwise return after the numbered stage
 * (see stage numbering in snow_oracle.c).  Returns 0 on success.
 */
int or_snow_simulation(const or_params* P,
                       or_particles* sph, uint32_t* sph_size,
                       or_particles* dem, uint32_t* dem_size,
                       or_particles* bnd, uint32_t b_size,
                       uint32_t full_size,
                       or_particles* buffer,
                       or_cells sph_cd, or_cells dem_cd, or_cells b_cd,
                       or_scene* scene, float dt, int iterations,
                       uint32_t flags, float temperature_variation,
                       int quirks, int stop_after);

/* Link formation pass alone (connect_and_record, cuda_simulation.cu:4286-4292). */
void or_connect_and_record(const or_params* P, or_particles* dem, uint32_t dem_size,
                           or_cells dem_cd, int dynamic_max_connections);

/* FP64 heat energy sum m*C*T and momentum sum m*v over the live particles. */
void or_energy_momentum(const or_params* P, const or_particles* sph, uint32_t n_sph,
                        const or_particles* dem, uint32_t n_dem, double out[4]);

int or_real_size(void);
void or_set_threads(int n);
/* walls at x = x_min, x_max and z = z_min, z_max, floor at y = floor_y (default -1, 1, -1, 1, 0) */
void or_set_domain(float x_min, float x_max, float z_min, float z_max, float floor_y);

#endif
