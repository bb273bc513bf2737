/*
 * snow_b200.h -- C ABI of libsnowb200.so, a B200 (sm_100a) implementation of the
 * SnowSimulation per-substep solver.
 *
 * Every entry point replaces one function of the reference's CUDA host interface
 * (cuda_simulation.cuh:13-75 and the host wrappers in cuda_simulation.cu); the
 * citation is given beside each.  The reference passes C++ objects (ParticleSet*,
 * CellData, SceneParams&); this ABI takes the same data as plain C structs of
 * device pointers whose layout is identical to the reference's structs
 * (ParticleDeviceData, CellData, SimParams, SceneParams), so a caller can pass
 * &particle_set->m_device_data unchanged.  The C++ shim in
 * snowsimulation_b200/shim/cuda_simulation_b200.cpp restores the reference's exact
 * signatures on top of this ABI.
 *
 * Conventions (all entry points):
 *   - buffers are owned by the caller and live in device memory of the current device;
 *   - every function returns SNOWB_OK (0) or a negative SNOWB_ERR_* code and never
 *     calls exit(); snowb_last_error_string() describes the last failure;
 *   - work is issued on the stream set by snowb_set_stream (default: legacy stream 0);
 *   - the library is single-threaded, as the reference's host interface is: its scratch
 *     buffers, graph cache, tape and profiling state are process-wide, so one host thread
 *     calls it at a time (calls from several threads must be serialised by the caller);
 *   - its device state does not survive a cudaDeviceReset; call snowb_release first.
 */
#ifndef SNOW_B200_H
#define SNOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SNOWB_OK 0
#define SNOWB_ERR_INVALID (-1)      /* bad argument (null pointer, size, grid) */
#define SNOWB_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define SNOWB_ERR_NO_PARAMS (-3)    /* snowb_set_sim_params was never called */
#define SNOWB_ERR_DEVICE (-4)       /* a kernel reported an error flag */

typedef struct snowb_float3 { float x, y, z; } snowb_float3;

/* ParticleDeviceData (Particle.h:14-52): per-particle device arrays in original-index
 * order, each sized full_size (connect_record / connect_length: full_size*maximum_connection,
 * new_end: one element). */
typedef struct snowb_particle_data {
    snowb_float3 *positions, *predict_positions, *new_positions, *velocity, *force, *correction;
    float *mass, *massInv, *density, *C, *lambda, *volume;
    float *T, *new_T;
    float *contrib;
    float *mass_scale;
    uint32_t *predicate, *scan_index, *new_end;
    uint32_t *connect_record, *iter_end;
    float *connect_length;
    uint32_t *new_index;
    uint32_t *trackId;
} snowb_particle_data;

/* CellData (NeighborSearch.h:19-26): grid_hash/grid_index/sorted_pos sized to the set,
 * cell_start/cell_end sized num_cells. */
typedef struct snowb_cell_data {
    uint32_t *grid_hash, *grid_index, *cell_start, *cell_end;
    snowb_float3 *sorted_pos;
} snowb_cell_data;

/* SimParams (SimParams.h:7-62), member for member. */
typedef struct snowb_sim_params {
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
} snowb_sim_params;

/* SceneParams (SceneParams.h:4-9). */
typedef struct snowb_scene_params {
    float fluid_start_time, solid_start_time, current_time;
} snowb_scene_params;

/* Quirk modes.  REFERENCE (default) reproduces the reference's deterministic
 * behaviour including its defects (partial cell-table clear, own-cell heat sum x27,
 * SPH index used for new snow particles, stale launch sizes after a phase change,
 * XSPH of the snow set limited to the water launch size, unseeded coupling s_corr
 * taken as 0).  FIXED applies the intended physics for each of those. */
#define SNOWB_QUIRKS_REFERENCE 0
#define SNOWB_QUIRKS_FIXED 1

/* Options of snowb_snow_simulation_ex. */
typedef struct snowb_step_options {
    int quirks;          /* SNOWB_QUIRKS_* */
    int substeps;        /* substeps to run back to back (sizes stay on the device between them); >= 1 */
    int stop_after;      /* debugging: 0 = full substep, else stop after the numbered stage */
    int use_graph;       /* 1: capture the substep in a CUDA graph and replay it for substeps >= 2 */
    int sync;            /* 1: wait for completion and write the new set sizes back (required by
                            the reference contract; 0 leaves *sph_size/*dem_size untouched and
                            the sizes on the device, see snowb_read_sizes) */
} snowb_step_options;

/* ---- reference interface (cuda_simulation.cuh:13-75) ---------------------------------- */

/* allocate_array (cuda_simulation.cu:1410-1413) */
int snowb_allocate_array(void** dev_ptr, size_t size);

/* set_sim_params (cuda_simulation.cu:1415-1419): the constants for all later calls. */
int snowb_set_sim_params(const snowb_sim_params* params);

/* No counterpart in the reference, which fixes the walls at x, z = +-1 and the floor at
 * y = 0 (integrate_pbd_cd_d, cuda_simulation.cu:487-513).  Moves them for all later calls;
 * the defaults (-1, 1, -1, 1, 0) reproduce the reference bit for bit.  With a larger
 * power-of-two grid (snowb_sim_params.grid_size) this holds scenes wider than 2 m. */
int snowb_set_domain(float x_min, float x_max, float z_min, float z_max, float floor_y);

/* compute_grid_size (cuda_simulation.cu:348-357): the reference's 1-D launch shape. */
int snowb_compute_grid_size(uint32_t n, uint32_t block_size, uint32_t* num_blocks, uint32_t* num_threads);

/* calculate_hash (cuda_simulation.cu:359-375 / calcHashD :194-212):
 * grid_hash[i] = cell hash of pos[i], grid_index[i] = i. */
int snowb_calculate_hash(snowb_cell_data cell_data, const snowb_float3* pos, uint32_t num_particles);

/* sort_particles (cuda_simulation.cu:1455-1468): stable sort of (grid_hash, grid_index) by hash. */
int snowb_sort_particles(snowb_cell_data cell_data, uint32_t num_particles);

/* No counterpart in the reference.  The stable sort of snowb_sort_particles for callers
 * that cannot allocate device memory: a render or game loop that forbids allocation after
 * start-up (cudaMalloc may synchronise the device mid-frame), a plugin whose host owns
 * every device allocation, a process under a fixed device-memory budget.  It allocates
 * nothing: its scratch is a static device array of about 6 MB that every GPU loading the
 * library holds until exit.  Limits: at most SNOWB_STATIC_SORT_MAX_PARTICLES particles and
 * SNOWB_STATIC_SORT_MAX_CELLS cells (larger requests fail with SNOWB_ERR_INVALID).  The
 * first call on a device looks up the array's address and should come before any stream
 * capture.  Calls share the array, so calls that overlap on the GPU race; the caller
 * serialises them.  Not usable after a cudaDeviceReset in the same process.  Blocks until
 * done. */
#define SNOWB_STATIC_SORT_MAX_PARTICLES (1u << 18)
#define SNOWB_STATIC_SORT_MAX_CELLS (1u << 18)
int snowb_sort_particles_static(snowb_cell_data cell_data, uint32_t num_particles);

/* reorder_data (cuda_simulation.cu:377-396 / reorderDataAndFindCellStartD :242-301):
 * clears cell_start[0, num_cells), writes cell_start/cell_end of occupied cells and
 * sorted_pos[i] = old_pos[grid_index[i]]. */
int snowb_reorder_data(snowb_cell_data cell_data, const snowb_float3* old_pos, uint32_t num_particles,
                       uint32_t num_cells);

/* compute_boundary_volume (cuda_simulation.cu:422-433 / :303-346): Akinci boundary volume. */
int snowb_compute_boundary_volume(snowb_cell_data cell_data, float* mass, float* volume, uint32_t num_particles);

/* integrate_pbd (cuda_simulation.cu:1422-1453): gravity, walls, speed clamp, prediction. */
int snowb_integrate_pbd(snowb_particle_data* particles, float dt, uint32_t num_particles, int cd_on);

/* connect_and_record (cuda_simulation.cu:4286-4292): interlink formation pass over the
 * snow set; the cell data must come from a sort of the same positions. */
int snowb_connect_and_record(snowb_particle_data* dem, uint32_t dem_size, snowb_cell_data dem_cell_data,
                             int dynamic_max_connections);

/* snow_simulation (cuda_simulation.cu:4861-5157): one substep.  *sph_size / *dem_size are
 * ParticleSet::m_size on entry and receive the sizes after freezing/melting (the reference
 * calls ParticleSet::setSize); scene->current_time advances by dt. */
int snowb_snow_simulation(snowb_particle_data* sph, uint32_t* sph_size,
                          snowb_particle_data* dem, uint32_t* dem_size,
                          snowb_particle_data* boundary, uint32_t boundary_size,
                          uint32_t full_size,
                          snowb_particle_data* phase_change_buffer,
                          snowb_cell_data sph_cell_data, snowb_cell_data dem_cell_data,
                          snowb_cell_data b_cell_data,
                          snowb_scene_params* scene_params,
                          float dt, int iterations,
                          int sph_dem_correction, int sph_sph_correction, int dem_friction,
                          int compute_temperature, int change_phase, int simulate_freezing,
                          int simulate_melting, int dem_viscosity, int use_interlink,
                          int dynamic_max_connections, int cd_on, float temperature_variation);

/* ---- extensions (no reference counterpart) -------------------------------------------- */

/* snow_simulation with options (quirk mode, several substeps per call, CUDA graph replay). */
int snowb_snow_simulation_ex(snowb_particle_data* sph, uint32_t* sph_size,
                             snowb_particle_data* dem, uint32_t* dem_size,
                             snowb_particle_data* boundary, uint32_t boundary_size,
                             uint32_t full_size,
                             snowb_particle_data* phase_change_buffer,
                             snowb_cell_data sph_cell_data, snowb_cell_data dem_cell_data,
                             snowb_cell_data b_cell_data,
                             snowb_scene_params* scene_params,
                             float dt, int iterations,
                             int sph_dem_correction, int sph_sph_correction, int dem_friction,
                             int compute_temperature, int change_phase, int simulate_freezing,
                             int simulate_melting, int dem_viscosity, int use_interlink,
                             int dynamic_max_connections, int cd_on, float temperature_variation,
                             const snowb_step_options* options);

/* ---- batched scenes (no reference counterpart) ------------------------------------------
 * Many independent scenes that share one snowb_sim_params (same grid, origin, cell size,
 * constants) are stepped by one launch sequence.  The sets of all scenes are concatenated
 * into one set per kind (water, snow, boundary); a scene-id array beside each set says
 * which scene each slot belongs to.  Scene s owns its own copy of the reference's cell
 * grid, at block (s % scenes_x, s / scenes_x) of a grid that is scenes_x times wider in x
 * and scenes_z times deeper in z, and wraps inside that block as a lone scene wraps in its
 * grid, so particles of different scenes never see each other.  With SNOWB_QUIRKS_FIXED
 * (required: the reference's quirks depend on whole-set sizes) every scene's particles
 * come out bit for bit as the same scene run alone, in the same relative order.
 * Cell tables of batched sets hold snowb_batch_num_cells() entries. */
typedef struct snowb_batch {
    uint32_t scenes_x, scenes_z;  /* scene blocks along x and z, each a power of two */
    uint32_t* scene_sph;          /* scene id per water slot (full_size); phase changes move the ids */
    uint32_t* scene_dem;          /* scene id per snow slot (full_size) */
    const uint32_t* scene_boundary; /* scene id per boundary particle */
    uint32_t* scene_buffer;       /* scratch, full_size entries */
} snowb_batch;

/* Cells of the batched grid: num_cells x scenes_x x scenes_z. */
int snowb_batch_num_cells(const snowb_batch* batch, uint32_t* num_cells);

/* calculate_hash for a batched set; scene_of[i] is particle i's scene. */
int snowb_batch_calculate_hash(const snowb_batch* batch, snowb_cell_data cell_data, const snowb_float3* pos,
                               const uint32_t* scene_of, uint32_t num_particles);

/* sort_particles over the batched grid. */
int snowb_batch_sort_particles(const snowb_batch* batch, snowb_cell_data cell_data, uint32_t num_particles);

/* reorder_data over the batched grid (clears all snowb_batch_num_cells() cell_start entries). */
int snowb_batch_reorder_data(const snowb_batch* batch, snowb_cell_data cell_data, const snowb_float3* old_pos,
                             uint32_t num_particles);

/* compute_boundary_volume of the batched boundary set (scene ids: batch->scene_boundary). */
int snowb_batch_compute_boundary_volume(const snowb_batch* batch, snowb_cell_data cell_data, float* mass,
                                        float* volume, uint32_t num_particles);

/* connect_and_record of the batched snow set (scene ids: batch->scene_dem). */
int snowb_batch_connect_and_record(const snowb_batch* batch, snowb_particle_data* dem, uint32_t dem_size,
                                   snowb_cell_data dem_cell_data, int dynamic_max_connections);

/* snowb_snow_simulation_ex over all scenes of the batch; options->quirks must be
 * SNOWB_QUIRKS_FIXED.  Sizes are those of the concatenated sets. */
int snowb_batch_snow_simulation(const snowb_batch* batch,
                                snowb_particle_data* sph, uint32_t* sph_size,
                                snowb_particle_data* dem, uint32_t* dem_size,
                                snowb_particle_data* boundary, uint32_t boundary_size,
                                uint32_t full_size,
                                snowb_particle_data* phase_change_buffer,
                                snowb_cell_data sph_cell_data, snowb_cell_data dem_cell_data,
                                snowb_cell_data b_cell_data,
                                snowb_scene_params* scene_params,
                                float dt, int iterations,
                                int sph_dem_correction, int sph_sph_correction, int dem_friction,
                                int compute_temperature, int change_phase, int simulate_freezing,
                                int simulate_melting, int dem_viscosity, int use_interlink,
                                int dynamic_max_connections, int cd_on, float temperature_variation,
                                const snowb_step_options* options);

/* ---- point-sprite rendering (point_sprite_vs.glsl, point_sprite_temperature_vs.glsl,
 * point_sprite_fs.glsl; Renderer.cpp draws with them) --------------------------------------
 * The reference shades its particles with these OpenGL shaders.  The same vertex and
 * fragment arithmetic runs here as CUDA kernels into a device image (RGBA float,
 * width x height, row 0 at the bottom like a GL framebuffer) with a 64-bit depth/id buffer,
 * no graphics API involved.  Depth test LESS in draw order; up to 32 draws (sets) between
 * clears, `draw` numbering them in drawing order. */
typedef struct snowb_camera {
    float view[16];          /* column-major, as the reference's glm matrices */
    float projection[16];
    float camera_pos[3];
    float light_pos[3];      /* view space, like the shaders' light_pos uniform */
    float point_size;        /* sprite side in pixels at distance 1 (Renderer::m_point_size) */
    uint32_t width, height;
} snowb_camera;
typedef struct snowb_point_colour {
    float rgb[3];            /* point_color */
    int use_temperature;     /* 1: the temperature shader (colour from the set's T) */
    float coolest_rgb[3], hottest_rgb[3];
    float coolest_T, hottest_T;
} snowb_point_colour;
/* Clear the image to (0, 0, 0, 0) and the depth buffer to far. */
int snowb_render_clear(const snowb_camera* cam, float* rgba, unsigned long long* zbuf);
/* Draw the first n particles of a set (positions, and T for the temperature colours). */
int snowb_render_points(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam,
                        const snowb_point_colour* colour, uint32_t draw, float* rgba, unsigned long long* zbuf);
/* The same clear with a clear colour (Renderer::ClearBuffer, m_clear_color). */
int snowb_render_clear_colour(const snowb_camera* cam, const float* clear_rgba, float* rgba, unsigned long long* zbuf);

/* ---- screen-space fluid (the reference's default view: Renderer::Render with
 * m_b_render_fluid, Renderer.cpp:92-109, through RenderSceneDepth, RenderFluidDepth,
 * SmoothDepth, RenderThickness and RenderFluid :404-690; shaders point_depth_*.glsl,
 * bilateral_fs.glsl, ssfr_thickness_*.glsl, ssfr_fluid_fs.glsl) ----------------------------
 * The snow is drawn as point sprites into a scene image and as sphere depth; the water as
 * sphere depth (smoothed by a separable bilateral filter) and additive thickness; a
 * full-screen composite refracts the scene through the water surface.  Images are
 * width x height, row 0 at the bottom; depth maps hold the clip depth z/w clamped to 0..1
 * (1 = empty), thickness is 32.32 fixed point (sum of n.z * 0.005 per covered pixel). */
typedef struct snowb_ssfr {
    float sphere_radius;       /* point_depth_fs sphere_radius (the particle radius) */
    float filter_radius;       /* bilateral half-width in texels (SmoothDepth: 10) */
    float blur_scale;          /* SmoothDepth: 0.1 */
    float blur_depth_falloff;  /* bilateral_fs.glsl: 65 */
    float light_color[4];      /* RenderFluid: (1, 1, 1, 0.8) */
    float clear_color[4];      /* Renderer::m_clear_color: (0.15, 0.15, 0.15, 0) */
} snowb_ssfr;
/* Device workspace of snowb_render_fluid for the camera's image size (48 bytes a pixel). */
int snowb_ssfr_workspace_bytes(const snowb_camera* cam, uint64_t* bytes);
/* The whole view into rgba (width x height x 4 floats): n_dem snow particles in
 * snow_colour, n_sph water particles as the fluid surface.  workspace: 16-byte aligned,
 * snowb_ssfr_workspace_bytes long. */
int snowb_render_fluid(const snowb_particle_data* sph, uint32_t n_sph, const snowb_particle_data* dem, uint32_t n_dem,
                       const snowb_camera* cam, const snowb_point_colour* snow_colour, const snowb_ssfr* ssfr,
                       void* workspace, float* rgba);
/* Its stages.  depth := 1 and thick := 0 (either may be NULL). */
int snowb_ssfr_clear(const snowb_camera* cam, float* depth, unsigned long long* thick);
/* Sphere depth of the first n particles of a set (minimum into depth). */
int snowb_ssfr_sphere_depth(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam, const snowb_ssfr* ssfr,
                            float* depth);
/* Thickness of the first n particles (added into thick). */
int snowb_ssfr_thickness(const snowb_particle_data* set, uint32_t n, const snowb_camera* cam, unsigned long long* thick);
/* Bilateral smoothing, along y into tmp, then along x into out. */
int snowb_ssfr_smooth(const snowb_camera* cam, const snowb_ssfr* ssfr, const float* depth, float* tmp, float* out);
/* Full-screen composite of the smoothed water depth, its thickness, the scene image and the
 * scene depth into rgba. */
int snowb_ssfr_compose(const snowb_camera* cam, const snowb_ssfr* ssfr, const float* depth,
                       const unsigned long long* thick, const float* scene_rgba, const float* scene_depth, float* rgba);
/* The matrices the kernels use: projection * view, view, projection, inverse projection,
 * inverse view (5 x 16 floats, column-major). */
int snowb_ssfr_matrices(const snowb_camera* cam, float* out80);

/* ---- frame export (GLFWApp::ExportBgeoFile, GLFWApp.cpp:287-405) -------------------------
 * One Houdini .bgeo file per set and frame with the reference's point attributes: position,
 * Cd (rgb, 3 floats), pscale (1 float) and label (1 int; the reference stores the bit
 * pattern of the float label, float_label = 1, which makes the file identical to its
 * output; 0 stores the integer).  The reference uses colours (0.7, 0.7, 1) for water and
 * (0.85, 0.85, 0.85) for snow, pscale = particle radius, label 0 water and 1 snow. */
int snowb_export_bgeo(const snowb_particle_data* set, uint32_t n, const char* path, const float* rgb, float pscale,
                      int label, int float_label);
/* The same, asynchronous: the positions are copied to pinned memory on the library's
 * stream (ordered after the work already issued) and a host thread writes the file;
 * snowb_export_wait joins all pending exports and reports the first failure. */
int snowb_export_bgeo_async(const snowb_particle_data* set, uint32_t n, const char* path, const float* rgb,
                            float pscale, int label, int float_label);
int snowb_export_wait(void);
/* The writer alone, from host memory (n points of 3 floats); needs no GPU. */
int snowb_write_bgeo_host(const float* positions, uint32_t n, const char* path, const float* rgb, float pscale,
                          int label, int float_label);

/* ---- autotuner (no reference counterpart) ------------------------------------------------
 * Times the tunable kernels of the substep (neighbour passes, link colouring, apply) under
 * nine launch shapes (64/128/256 threads per block x grid caps of 8/16/64 blocks per SM),
 * each over `substeps` graph-replayed substeps timed from CUDA-event nodes, and keeps the
 * fastest shape per kernel and work-size bucket (floor(log2(threads of work))).  The
 * arguments are those of snowb_snow_simulation_ex (batch: NULL for one scene, else the
 * batch of snowb_batch_snow_simulation); the state advances by 9 x (substeps + 1) substeps,
 * so callers snapshot it first if they need it.  Launch shapes never change results. */
int snowb_autotune(snowb_particle_data* sph, uint32_t* sph_size,
                   snowb_particle_data* dem, uint32_t* dem_size,
                   snowb_particle_data* boundary, uint32_t boundary_size,
                   uint32_t full_size,
                   snowb_particle_data* phase_change_buffer,
                   snowb_cell_data sph_cell_data, snowb_cell_data dem_cell_data,
                   snowb_cell_data b_cell_data,
                   snowb_scene_params* scene_params,
                   float dt, int iterations,
                   int sph_dem_correction, int sph_sph_correction, int dem_friction,
                   int compute_temperature, int change_phase, int simulate_freezing,
                   int simulate_melting, int dem_viscosity, int use_interlink,
                   int dynamic_max_connections, int cd_on, float temperature_variation,
                   int quirks, int substeps, const snowb_batch* batch);
/* The table as text, one "kernel bucket threads_per_block grid_cap_per_sm" line per entry. */
int snowb_autotune_table(char* out, size_t cap);
/* Replace the table with one in that format (e.g. saved from an earlier run). */
int snowb_autotune_load(const char* table);
/* Forget all tuned shapes (back to the built-in ones). */
int snowb_autotune_reset(void);

/* ---- adjoint of the substep (no reference counterpart) -------------------------------
 * Reverse-mode derivatives of snowb_snow_simulation_ex substeps in the fixed quirk mode,
 * with the forward pass's discrete decisions held fixed (neighbour sets, interlink
 * topology and breaking, C > 0, friction branch, wall and speed clamps).  Between
 * snowb_adjoint_begin and snowb_adjoint_end every substep is recorded (requirements: fixed
 * quirks, no graph, sph_sph_correction and dynamic links off, scorr_coeff 0, no phase
 * change and contrib 1 while recording; sizes and iterations constant).  The tape holds
 * about (30 + 8 x iterations x maximum_connection) bytes per particle slot per substep;
 * hosts bound it by checkpointing (record a segment, run its backward, re-record the
 * previous segment from a saved state). */
typedef struct snowb_adjoint_io {
    /* device arrays in original index order, in: adjoint of the state after the last
     * recorded substep; out: adjoint of the state before the first */
    float *gx_sph, *gv_sph, *gT_sph;   /* positions (n x 3), velocities (n x 3), temperatures (n) */
    float *gx_dem, *gv_dem, *gT_dem;
    float* gL_dem;   /* interlink rest lengths (connect_length, n_dem x maximum_connection); a
                        length depends on the positions where its link formed, so its
                        adjoint travels back to that substep */
    /* host, accumulated: dL/d k_refreezing (interlink stiffness), k_stretch (water-snow
     * contact), k_water, k_snow (conductivities) */
    double grad_params[4];
} snowb_adjoint_io;

int snowb_adjoint_begin(void);
/* Stop recording; *substeps = number of substeps on the tape. */
int snowb_adjoint_end(uint32_t* substeps);
/* Reverse pass over the recorded substeps (last to first); empties the tape. */
int snowb_adjoint_backward(snowb_adjoint_io* io);
/* Free the tape and the reverse pass's buffers. */
int snowb_adjoint_release(void);

/* Set sizes kept on the device by the last call with options->sync = 0 (blocks). */
int snowb_read_sizes(uint32_t* sph_size, uint32_t* dem_size);

/* Device counters of the last substep, in this order: n_sph, n_dem, n_boundary, sizes at
 * substep start (2), particles freezing, melting, phase-change flag, sizes after compaction
 * (2), device error bits, tail-dirty flag, particles kept by the link prefilter, links added,
 * neighbour lists that overflowed in the substep's density+lambda passes, (index 15 unused),
 * then for the water and the snow set: the pending full-sort flags (2), the last sort
 * decisions (2), and since the call started the sort points that sorted in full (2) and
 * those that kept the previous sort because no particle had left its cell (2).
 * Copies min(n, 24) values into out (blocks). */
int snowb_device_counters(uint32_t* out, int n);

/* Default quirk mode of snowb_snow_simulation (SNOWB_QUIRKS_REFERENCE initially). */
int snowb_set_quirks(int mode);

/* Stream for all later work (a cudaStream_t; NULL = legacy default stream). */
int snowb_set_stream(void* stream);

/* Block until the library's stream is idle. */
int snowb_synchronize(void);

/* FP64 reductions over the live particles: out[0] = sum m*C*T (heat energy, J),
 * out[1..3] = sum m*v (momentum).  Computed on the GPU in double precision. */
int snowb_energy_momentum(const snowb_particle_data* sph, uint32_t sph_size,
                          const snowb_particle_data* dem, uint32_t dem_size, double out[4]);

/* Number of kernels this library has launched since it was loaded. */
int snowb_launch_count(uint64_t* count);

/* Per-kernel timing: between snowb_profile_begin and snowb_profile_end every launch is
 * bracketed by CUDA events on the library's stream; snowb_profile_end waits for the stream
 * and writes one line per kernel, "name launches total_ms", into out (NUL-terminated). */
int snowb_profile_begin(void);
int snowb_profile_end(char* out, size_t cap);
/* While profiling, after a step: the launches of its last substep (the last replay of its
 * graph, or the last substep run directly) as a timeline, one line per launch in launch
 * order, "name start_ms end_ms", times from the start of that substep's first launch
 * (launches on the library's side streams overlap the others).  NUL-terminated. */
int snowb_profile_timeline(char* out, size_t cap);

/* Release the library's internal device buffers (they are re-created on demand). */
int snowb_release(void);

/* Last error code and message of this thread. */
int snowb_last_error(void);
const char* snowb_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif /* SNOW_B200_H */
