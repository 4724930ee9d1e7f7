/* ilc.h -- C ABI of the B200 (sm_100a) backend for illcrawl's volumetric
 * projection path: nn8 particle-grid reconstruction feeding the RKF4(5)
 * line-of-sight integrator that produces gas projections, X-ray band maps and
 * X-ray spectra.
 *
 * Conventions
 *  - Every call returns an ilc_status; ILC_OK is 0. The message of the last
 *    failure on a context is returned by ilc_last_error().
 *  - A context owns one CUDA stream, the device copy of the particle grid, the
 *    Gaunt table and grow-only scratch buffers. Calls on one context must be
 *    serialised by the caller (one context per host thread); every call has
 *    completed on the device when it returns.
 *  - Arrays are caller-allocated. is_device = 0: host pointers (copied in and
 *    out by the call); is_device = 1: device pointers on the context's device.
 *  - Particles are float4 records (x, y, z, q) -- the reference's particle
 *    layout (particle_grid.hpp:43-48).
 *  - Nothing here falls back to the CPU: without a usable CUDA device
 *    ilc_create() returns NULL.
 */
#ifndef ILC_H
#define ILC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ilc_status {
  ILC_OK = 0,
  ILC_ERR_INVALID_ARGUMENT = 1,
  ILC_ERR_CUDA = 2,
  ILC_ERR_OUT_OF_MEMORY = 3,
  ILC_ERR_NO_PARTICLES = 4,    /* query or render before setup_particles */
  ILC_ERR_NO_GAUNT_TABLE = 5,  /* X-ray quantity before ilc_gaunt_load */
  ILC_ERR_STEP_LIMIT = 6,      /* a ray reached the per-ray RKF step cap */
  ILC_ERR_NONFINITE_INPUT = 7, /* NaN or Inf particle coordinates */
  ILC_ERR_GRID_TOO_LARGE = 8,  /* more than 2^32 grid cells or 2^31 particles */
  ILC_ERR_INTERNAL = 9,
  ILC_ERR_NO_ARF_TABLE = 10    /* Chandra quantity before ilc_arf_load */
} ilc_status;

typedef struct ilc_ctx ilc_ctx;

/* camera (camera.hpp:493-593): position of the screen centre, normalised
 * look-at direction, roll angle [rad], screen width, resolution. */
typedef struct ilc_camera {
  double position[3];
  double look_at[3];
  double roll;
  double screen_width;
  int32_t num_pix_x;
  int32_t num_pix_y;
} ilc_camera;

/* integration::tolerance (integration.hpp:37-49) */
typedef struct ilc_tolerance {
  double absolute;
  double relative;
} ilc_tolerance;

/* Step controller of the adaptive integrator. REF32: the reference's fp32
 * controller (integration.cl:49-131). FP64: the same controller evaluated in
 * double over the fp32 state. */
enum { ILC_CONTROLLER_REF32 = 0, ILC_CONTROLLER_FP64 = 1 };

/* effective_line_of_sight_integration_dA of the reconstructed quantity
 * (quantity.hpp:56-57): PIXEL_AREA for fluxes (quantity.hpp:198-202), UNIT for
 * projected density (quantity.hpp:567-572), INVERSE_RANGE for mean
 * quantities (quantity.hpp:482-487). */
enum { ILC_DA_PIXEL_AREA = 0, ILC_DA_UNIT = 1, ILC_DA_INVERSE_RANGE = 2 };

/* Final image scaling of volumetric_integration.cpp:74-87. */
typedef struct ilc_los_scaling {
  double length_conversion; /* unit_converter::length_conversion_factor() */
  double area_conversion;   /* unit_converter::area_conversion_factor() */
  int32_t dA_mode;          /* ILC_DA_* */
} ilc_los_scaling;

typedef struct ilc_grid_desc {
  float min_corner[3];
  float cell_sizes[3];
  int32_t num_cells[3];
  uint64_t total_cells;
  uint64_t num_particles;
} ilc_grid_desc;

typedef struct ilc_render_stats {
  uint64_t steps;          /* RKF steps over all rays (accepted + rejected) */
  uint64_t accepted_steps;
  uint64_t queries;        /* nn8 evaluations (4 per step) */
  uint64_t cells_visited;  /* in-grid cells walked by all queries */
  uint64_t candidates;     /* particles tested by all queries */
  uint64_t max_steps_per_ray;
  uint64_t rays_at_step_limit;
  float kernel_ms;         /* device time of the render kernel (CUDA events) */
} ilc_render_stats;

/* ---- context (replaces qcl::device_context, qcl.hpp:196-890, for this path) */
ilc_ctx* ilc_create(int device);
void ilc_destroy(ilc_ctx* ctx);
const char* ilc_last_error(const ilc_ctx* ctx);
/* Per-ray RKF step cap (default 2^20); reaching it ends the ray and makes the
 * render return ILC_ERR_STEP_LIMIT. */
ilc_status ilc_set_step_limit(ilc_ctx* ctx, int64_t max_steps);
/* The context's cudaStream_t, for callers that time or order work around it. */
void* ilc_get_stream(ilc_ctx* ctx);
/* Schedule of the adaptive render: rays of a thread block advance through
 * z_window-thick slabs together (0 = every ray runs to its end independently).
 * Changes the order of work only, never a result. */
ilc_status ilc_set_z_window(ilc_ctx* ctx, float z_window);
/* Kernel behind ilc_render_adaptive and ilc_project_xray_flux with the FP64
 * controller. GRID: one thread block per 16 x 8 pixel tile, one launch per
 * image (the reference's one-projection-per-call structure). PERSISTENT: the
 * work-queue kernel of ilc_render_batched with this one camera (its
 * schedule: ilc_set_batch_schedule). Both give the same image bit for bit;
 * the REF32 controller, the fixed-step mode and the adjoint's forward pass
 * always use GRID. Default: PERSISTENT. */
enum { ILC_ENGINE_GRID = 0, ILC_ENGINE_PERSISTENT = 1 };
ilc_status ilc_set_render_engine(ilc_ctx* ctx, int32_t engine);

/* Kernel of ilc_nn8_query (and of the consumers that query through it):
 * ILC_QUERY_THREAD (default) walks each query in one thread, as the
 * reference's kernel does; ILC_QUERY_WARP walks each query with a whole warp
 * (the cells of the spiral and the candidates tested 32 at a time, hits
 * collected by ballot and inserted in candidate order). Both give the same
 * results bit for bit. No reference counterpart. */
enum { ILC_QUERY_THREAD = 0, ILC_QUERY_WARP = 1 };
ilc_status ilc_set_query_engine(ilc_ctx* ctx, int32_t engine);

/* Search counters of the last ilc_nn8_query on this context: grid cells
 * visited and candidate particles tested, summed over its queries (the
 * oracle's counters; the traffic model of the walk). Valid until the next
 * call that launches a kernel. No reference counterpart. */
ilc_status ilc_nn8_query_stats(ilc_ctx* ctx, uint64_t* cells_visited, uint64_t* candidates);

/* Occupancy of the adaptive render: 0 = as many blocks per SM as the
 * kernel's registers allow, 3, 4 or 5 = that many 128-thread blocks per SM
 * (registers capped accordingly). Changes the order of work only, never a
 * result. */
ilc_status ilc_set_render_occupancy(ilc_ctx* ctx, int32_t blocks_per_sm);

/* ---- particle grid + nn8 backend ------------------------------------------
 * ilc_nn8_setup_particles replaces reconstruction_backend::setup_particles
 * (reconstruction_backend.hpp:49-50) as implemented by nn8::setup_particles
 * (volumetric_reconstruction_backend_nn8.cpp:47-55), which builds a
 * particle_grid (particle_grid.cpp:25-119): grid over the particles' bounding
 * box +-0.1, cell width cbrt(8 V / N), cells sorted by key. */
ilc_status ilc_nn8_setup_particles(ilc_ctx* ctx, const float* particles, uint64_t n,
                                   int is_device);

/* particle_grid::get_grid_min_corner / get_num_grid_cells /
 * get_grid_cell_sizes / get_num_particles (particle_grid.hpp:62-77). */
ilc_status ilc_grid_describe(ilc_ctx* ctx, ilc_grid_desc* out);

/* Copies the grid out: cells (int2 [begin, end) per cell, total_cells x 2),
 * sorted->original index map (uint32, n) and sorted particles (float4, n).
 * Any pointer may be NULL. particle_grid::get_grid_cells_buffer /
 * get_particle_buffer and generate_sorted_to_unsorted_map
 * (particle_grid.hpp:68-70,102-103). */
ilc_status ilc_grid_export(ilc_ctx* ctx, int32_t* cells, uint32_t* sorted_to_unsorted,
                           float* sorted_particles, int is_device);

/* nn8 reconstruction at n query points (float4, w ignored). Replaces
 * setup_evaluation_points + run + retrieve_results
 * (reconstruction_backend.hpp:43,52-55; volumetric_reconstruction_backend_nn8.cpp:57-84).
 * merge_previous = 0 starts from empty lists (is_first_run); 1 continues the
 * lists the previous call on this context left for the same n, which is how
 * the reference merges particle blocks. out_values: n floats. out_idx8 /
 * out_dist8 (n x 8, may be NULL): the 8 list slots in slot order as original
 * particle indices (-1 = empty) and distances. */
ilc_status ilc_nn8_query(ilc_ctx* ctx, const float* points, uint64_t n, int merge_previous,
                         float* out_values, int32_t* out_idx8, float* out_dist8,
                         int is_device);

/* ---- quantities ------------------------------------------------------------
 * Thermally averaged free-free Gaunt factors, width x height row-major (row =
 * one log(u), column = one log(gamma^2)), origin (x0, y0), spacing (dx, dy):
 * model::gaunt::thermally_averaged_ff (gaunt_factor.cpp:30-41; the reference
 * loads gaunt_factor.dat with x0 = -6, y0 = -16, dx = dy = 0.2). At most
 * 81 x 146 entries. */
ilc_status ilc_gaunt_load(ilc_ctx* ctx, const float* table, int32_t width, int32_t height,
                          float x0, float y0, float dx, float dy);

/* Per-cell band flux [keV/s/kpc^3/m^2]: the xray_flux kernel
 * (quantities.cl:354-385) run by quantity_transformation (quantity.cpp:111-131).
 * rho [M_sun/kpc^3], u [(km/s)^2], xe: n floats each. */
ilc_status ilc_quantity_xray_flux(ilc_ctx* ctx, const float* rho, const float* u,
                                  const float* xe, uint64_t n, float redshift,
                                  float luminosity_distance, float e_min, float e_max,
                                  int32_t num_samples, float* out, int is_device);

/* Per-cell flux in one energy bin: xray_spectral_flux (quantities.cl:400-430). */
ilc_status ilc_quantity_xray_spectral_flux(ilc_ctx* ctx, const float* rho, const float* u,
                                           const float* xe, uint64_t n, float redshift,
                                           float luminosity_distance, float energy,
                                           float energy_bin_width, float* out,
                                           int is_device);

/* Per-cell flux in n_bins energy bins at once, cell-major: out[i * n_bins + b]
 * = xray_spectral_flux (quantities.cl:400-430) at energies[b], widths[b]; the
 * per-bin values of xray_spectrum_quantity_generator (spectrum.cpp:89-109)
 * in the layout ilc_render_batched reads. energies, widths: host arrays. */
ilc_status ilc_quantity_xray_spectrum(ilc_ctx* ctx, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float redshift,
                                      float luminosity_distance, const float* energies,
                                      const float* widths, int32_t n_bins, float* out,
                                      int is_device);

/* Per-cell photon flux [photons/s/kpc^3/cm^2]: the xray_photon_flux kernel
 * (quantities.cl:640-675), i.e. xray_flux's energy integral of the emission
 * divided by the photon energy, times 1e-4 (per m^2 -> per cm^2). */
ilc_status ilc_quantity_xray_photon_flux(ilc_ctx* ctx, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float redshift,
                                         float luminosity_distance, float e_min, float e_max,
                                         int32_t num_samples, float* out, int is_device);

/* Chandra effective area: n samples [cm^2] from energy x_min [keV] in steps
 * of dx, as util::tabulated_function holds chandra::arf (tabulated_function.hpp:
 * 35-103; chandra.cpp, the Cycle 19 ACIS-I ARF: 1024 samples, x_min 0.105322271585,
 * dx 0.010644). The table is the caller's: the reference keeps it in its
 * sources and this library ships none. At most 65536 samples. */
ilc_status ilc_arf_load(ilc_ctx* ctx, const float* table, int32_t n, float x_min, float dx);

/* Per-cell Chandra count rate [counts/s/kpc^3]: chandra_xray_total_count_rate
 * (quantities.cl:510-557), the count rate of every ARF channel k (energy
 * x_min + k dx, width dx) summed in channel order. Needs ilc_gaunt_load and
 * ilc_arf_load. */
ilc_status ilc_quantity_chandra_count_rate(ilc_ctx* ctx, const float* rho, const float* u,
                                           const float* xe, uint64_t n, float redshift,
                                           float luminosity_distance, float* out,
                                           int is_device);

/* Per-cell Chandra count rate in one channel (energy, energy_bin_width [keV]):
 * chandra_xray_spectral_count_rate (quantities.cl:584-622). */
ilc_status ilc_quantity_chandra_spectral_count_rate(ilc_ctx* ctx, const float* rho,
                                                    const float* u, const float* xe,
                                                    uint64_t n, float redshift,
                                                    float luminosity_distance, float energy,
                                                    float energy_bin_width, float* out,
                                                    int is_device);

/* Per-cell Chandra count rate in n_bins channels at once, cell-major
 * out[i * n_bins + b] (the per-frame quantity of
 * chandra_spectrum_quantity_generator, spectrum.cpp:45-65, in the layout
 * ilc_render_batched reads). energies, widths: host arrays. */
ilc_status ilc_quantity_chandra_spectrum(ilc_ctx* ctx, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float redshift,
                                         float luminosity_distance, const float* energies,
                                         const float* widths, int32_t n_bins, float* out,
                                         int is_device);

/* Per-cell temperature [K]: mean_temperature (quantities.cl:268-284). */
ilc_status ilc_quantity_temperature(ilc_ctx* ctx, const float* u, const float* xe, uint64_t n,
                                    float* out, int is_device);

/* ---- camera and line-of-sight integration -----------------------------------
 * The camera plane as the device sees it (camera.cpp:124-155 in double, cast
 * to float as math::to_device_vector4): out13 = look_at(3), basis0(3),
 * basis1(3), screen min corner(3), pixel size. */
ilc_status ilc_camera_plane(const ilc_camera* cam, float* out13);

/* volumetric_integration::create_projection (volumetric_integration.cpp:32-88):
 * one adaptive RKF4(5) integrator per pixel from z = 0 to z_range along
 * look_at, integrand = nn8 reconstruction of the particles' q. image:
 * num_pix_y x num_pix_x floats (row = y). scaling = NULL leaves the raw line
 * integrals; otherwise they are multiplied as volumetric_integration.cpp:74-87.
 * stats may be NULL. */
ilc_status ilc_render_adaptive(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                               ilc_tolerance tol, int32_t controller,
                               const ilc_los_scaling* scaling, float* image, int is_device,
                               ilc_render_stats* stats);

/* Frozen uniform step sequence: num_steps RKF steps of z_range/num_steps, all
 * accepted (I += delta4 of integration.cl:63-79, k1 carried from the previous
 * step). No reference counterpart as an entry point: it is the reference's
 * integrator with the step controller removed. */
ilc_status ilc_render_fixed(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                            int64_t num_steps, const ilc_los_scaling* scaling, float* image,
                            int is_device, ilc_render_stats* stats);

/* Adaptive render that also records every ray's accepted step sizes: ray
 * k = iy * num_pix_x + ix writes n_steps[k] (at most capacity) sizes to
 * step_sizes[k * capacity ...]. A ray with more accepted steps than capacity
 * keeps its first capacity steps and the call returns ILC_ERR_INVALID_ARGUMENT
 * after the render ("capacity too small"). The parity checkpoint of the
 * frozen-sequence replay; no reference counterpart as an entry point.
 * step_sizes / n_steps follow steps_on_device; image follows is_device. */
ilc_status ilc_render_record(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                             ilc_tolerance tol, int32_t controller, float* step_sizes,
                             int32_t* n_steps, int64_t capacity, int steps_on_device,
                             float* image, int is_device, ilc_render_stats* stats);

/* ilc_render_adaptive that also writes each ray's work counters: ray
 * k = iy * num_pix_x + ix gets ray_stats[4k .. 4k+3] = (RKF steps taken,
 * steps accepted, grid cells visited, candidate particles tested), summed
 * over the 4 integrand points of every step as the oracle's search counters
 * count them (volumetric_nn8_reconstruction.cl:157-203 visits a cell and
 * tests every particle in it). They give each ray's algorithmic bytes
 * 8 cells + 16 candidates + 24 steps + 4. Runs the one-block-per-tile kernel;
 * the image equals ilc_render_adaptive's. ray_stats follows is_device. No
 * reference counterpart as an entry point. */
ilc_status ilc_render_ray_stats(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                                ilc_tolerance tol, int32_t controller,
                                const ilc_los_scaling* scaling, float* image,
                                uint64_t* ray_stats, int is_device, ilc_render_stats* stats);

/* Frozen per-ray step sequence: ray k replays step_sizes[k * capacity + i],
 * i < n_steps[k], every step accepted (I += delta4 of integration.cl:63-79,
 * k1 carried), from z = 0. Replaying a recorded adaptive sequence gives the
 * adaptive render's pixels; replaying it in double (the FP64 oracle) bounds
 * the fp32 path's error at a fixed sequence. z_range is the nominal depth,
 * used only by the scaling. No reference counterpart as an entry point. */
ilc_status ilc_render_frozen(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                             const float* step_sizes, const int32_t* n_steps, int64_t capacity,
                             int steps_on_device, const ilc_los_scaling* scaling, float* image,
                             int is_device, ilc_render_stats* stats);

/* ilc_render_frozen with each ray's fp32 step increments summed in double
 * into a double image (num_pix_y x num_pix_x, follows is_device). The fp32
 * walk and increments are the frozen replay's, so two replays that differ
 * only in a few particles' values differ only in the increments those values
 * enter: finite-difference checks of the adjoint read the difference without
 * the fp32 accumulation's rounding. No reference counterpart. */
ilc_status ilc_render_frozen_f64(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                                 const float* step_sizes, const int32_t* n_steps,
                                 int64_t capacity, int steps_on_device,
                                 const ilc_los_scaling* scaling, double* image, int is_device,
                                 ilc_render_stats* stats);

/* The multiplier applied to every pixel by volumetric_integration.cpp:74-87. */
float ilc_los_scale(const ilc_camera* cam, double z_range, const ilc_los_scaling* scaling);

/* The band-map pipeline of `illcrawl_render -t image -q xray_flux` in one call:
 * reconstructing_data_crawler::run's first pass (reconstructing_data_crawler.cpp:157-256:
 * per-cell xray_flux by quantity_transformation, packed into the particles'
 * q, then setup_particles) followed by create_projection. cells: n float4
 * records (x, y, z, unused); rho, u, xe: n floats. The grid built here stays
 * on the context, as the crawler keeps it for later runs. */
ilc_status ilc_project_xray_flux(ilc_ctx* ctx, const float* cells, const float* rho,
                                 const float* u, const float* xe, uint64_t n, float redshift,
                                 float luminosity_distance, float e_min, float e_max,
                                 int32_t num_samples, const ilc_camera* cam, double z_range,
                                 ilc_tolerance tol, int32_t controller,
                                 const ilc_los_scaling* scaling, float* image, int is_device,
                                 ilc_render_stats* stats);

/* ---- volumetric slice ---------------------------------------------------------
 * volumetric_slice::create_slice (volumetric_slice.cpp:31-101): the nn8
 * reconstruction of the particles' q at every pixel of the camera plane,
 * sample 0 at camera::get_pixel_coordinate(x, y) (camera.cpp:49-54),
 * image[y][x] accumulated as the reference does (float pixel += dV * value /
 * samples, each increment in double). dV is the quantity's
 * effective_volume_integration_dV (quantity.hpp:193-197,477-480).
 * additional_samples > 0 adds jittered samples per pixel; the reference
 * draws their offsets from std::random_device, here they come from a hash of
 * (seed, sample, pixel), so a slice is reproducible. image: num_pix_y x
 * num_pix_x floats. */
ilc_status ilc_volumetric_slice(ilc_ctx* ctx, const ilc_camera* cam, double dV,
                                int32_t additional_samples, uint64_t seed, float* image,
                                int is_device);

/* volumetric_tomography::create_tomographic_cube (volumetric_tomography.cpp:
 * 62-101): num_steps slices of ilc_volumetric_slice (one sample per pixel),
 * slice z taken with the camera moved along look_at by (initial_z_step + z)
 * pixel sizes. cube: num_steps x num_pix_y x num_pix_x floats (x fastest, as
 * the reference's cube). */
ilc_status ilc_volumetric_tomography(ilc_ctx* ctx, const ilc_camera* cam, double dV,
                                     int64_t initial_z_step, int64_t num_steps, float* cube,
                                     int is_device);

/* ---- Monte-Carlo radial profiles ------------------------------------------
 * distributed_mc_radial_profile (profile.cpp:26-355) on one device.
 * Shell i of num_radii: radius r_i = i * max_radius / num_radii
 * (get_comoving_profile_radii), spanning [(r_{i-1} + r_i)/2, (r_i + r_{i+1})/2]
 * (shell 0 from 0; profile.cpp:320-355), with n_i = max(1, floor(norm V_i^2))
 * samples, norm = sample_density * sum(V) / sum(V^2) (generate_num_samples,
 * profile.cpp:93-128). */
enum { ILC_DV_VOLUME = 0, ILC_DV_MEAN = 1 };

/* Shell radii and sample counts (host only; either output may be NULL).
 * num_radii in [1, 2^20]; fails when the samples would exceed 2^40. */
ilc_status ilc_mc_profile_shells(double max_radius, int32_t num_radii, double sample_density,
                                 double* radii, uint64_t* counts);

/* Sample points first .. first + count - 1 of that profile (4 floats each,
 * w = 0), made on the host by the same code as the device's: for callers that
 * evaluate the samples elsewhere or split them over processes (the
 * reference's work_partitioner split of profile.cpp:156-177). Host only. */
ilc_status ilc_mc_profile_points(const double center[3], double max_radius, int32_t num_radii,
                                 double sample_density, uint64_t seed, uint64_t first,
                                 uint64_t count, float* points);

/* The profile of the particles' q (ilc_nn8_setup_particles) around center:
 * per shell, the nn8 values at its samples summed in double, times the
 * quantity's effective dV of apply_volume_factor (profile.cpp:236-256) with
 * dV = V_i / n_i: ILC_DV_VOLUME gives dV * volume_conversion (the X-ray
 * quantities, quantity.hpp:193-197), ILC_DV_MEAN (dV * volume_conversion) /
 * (V_i * volume_conversion) (density, temperature; quantity.hpp:477-480,
 * 560-565). Each sample is uniform in its shell (uniform_spherical_shell,
 * random.cpp:28-86) with its draws hashed from (seed, sample index): the
 * reference seeds std::mt19937 from std::random_device, so its samples are
 * never reproducible. profile: num_radii doubles. sample_points (4 floats per
 * sample) and sample_values (1 float per sample) receive every sample in
 * order, shells in order; either may be NULL. All outputs are host memory. */
ilc_status ilc_mc_radial_profile(ilc_ctx* ctx, const double center[3], double max_radius,
                                 int32_t num_radii, double sample_density, uint64_t seed,
                                 int32_t dV_mode, double volume_conversion, double* profile,
                                 float* sample_points, float* sample_values);

/* ---- cell ingestion ---------------------------------------------------------
 * The per-row loop of reconstructing_data_crawler::run
 * (reconstructing_data_crawler.cpp:170-230) on the device: each cell's float
 * coordinates, widened to double, move by one period along every axis where
 * that puts them inside the cutout box center -/+ extent/2 widened by border
 * (coordinate_system::correct_periodicity, coordinate_system.hpp:25-47; the
 * crawler's border is 100 kpc); cells whose corrected position lies in the
 * cutout box (volume_cutout::contains_point, reconstructing_data_crawler.cpp:
 * 49-60) are kept, in input order, as float4 (x, y, z, q) with the corrected
 * coordinates cast to float, q = their value in q (0 if q is NULL), and their
 * input index in out_index (may be NULL). xyz: n x 3 floats; out_xyzq: room
 * for n float4; *n_out: cells kept. The result feeds ilc_nn8_setup_particles
 * directly. All arrays follow is_device. n < 2^32. */
ilc_status ilc_ingest_cells(ilc_ctx* ctx, const float* xyz, const float* q, uint64_t n,
                            const double* center, const double* extent, const double* periodic,
                            double border, float* out_xyzq, uint32_t* out_index,
                            uint64_t* n_out, int is_device);

/* ---- FITS output --------------------------------------------------------------
 * Writes an image (naxis = 2) or cube (naxis = 3; NAXIS1 = x fastest, as the
 * renders and ilc_render_batched's per-job blocks are laid out) of floats as a
 * FITS primary HDU with BITPIX = -32, the structure util::fits::save
 * (fits.hpp:215-258) produces through cfitsio, followed by header keys as
 * util::fits_header::add_entry (fits.hpp:142-200) appends them (a COMMENT card
 * with the key's comment, then the key; keys longer than 8 characters as
 * HIERARCH cards). Host memory only; no GPU needed. */
enum { ILC_FITS_DOUBLE = 0, ILC_FITS_INTEGER = 1, ILC_FITS_STRING = 2, ILC_FITS_LOGICAL = 3 };
typedef struct ilc_fits_card {
  const char* key;
  int32_t type;           /* ILC_FITS_* */
  double number;          /* DOUBLE */
  int64_t integer;        /* INTEGER, LOGICAL (0 / 1) */
  const char* text;       /* STRING */
  const char* comment;    /* may be NULL */
} ilc_fits_card;
ilc_status ilc_fits_write_image(const char* path, const float* data, int32_t naxis,
                                const int64_t* naxes, const ilc_fits_card* cards,
                                int32_t n_cards);

/* ---- batched render ---------------------------------------------------------
 * Many projections in one persistent launch: the (camera, frame) loop of
 * integrated_projection / distributed_animation (animation.cpp:29-100,229-241)
 * and the per-bin loop of multi_quantity_integrated_projection /
 * spectrum_generator (animation.cpp:264-283, spectrum.hpp:81-126) as one
 * work queue of 32-ray tiles over all jobs, with V value channels per cell
 * integrated along each ray together.
 *
 * A job is one camera. Its rays start on the camera plane like
 * ilc_render_adaptive's and run along look_at over [0, z_range], or, when
 * sphere_radius > 0, over the ray's chord of that sphere (widened about its
 * midpoint to at least min_chord, clipped to start at the camera plane).
 * aperture_radius > 0 masks pixels whose centre lies farther than that from
 * the screen centre (their outputs are 0). Each ray's V channels are
 * integrated with one step sequence from a joint FP64 controller: per channel
 * the reference's error ratio (integration.cl:82-131 with the FP64
 * controller), minimum over channels; a step is accepted only if every
 * channel accepts it. With V = 1 and no mask or chord a job equals
 * ilc_render_adaptive with ILC_CONTROLLER_FP64 bit for bit. For V > 1 the
 * channels' step sequence differs from V separate renders (it is at least as
 * fine as each channel's own).
 *
 * values: n x V floats, cell-major, in the order of the particles given to
 * ilc_nn8_setup_particles (which must have been called; their q is not used).
 * images: job k's V x num_pix_y x num_pix_x block (channel-major, row = y) at
 * element out_offset, multiplied by scale. images_len bounds every block.
 * V <= 256. stats may be NULL. */
typedef struct ilc_job {
  ilc_camera camera;
  double z_range;          /* integration depth when sphere_radius <= 0 */
  double aperture_radius;  /* <= 0: no mask */
  double sphere_center[3];
  double sphere_radius;    /* > 0: integrate over the chord of this sphere */
  double min_chord;        /* chords shorter than this are widened to it */
  float scale;             /* output multiplier, e.g. ilc_los_scale(...) */
  int32_t reserved;        /* 0 */
  uint64_t out_offset;     /* element offset of this job's block in images */
} ilc_job;

ilc_status ilc_render_batched(ilc_ctx* ctx, const float* values, int32_t n_channels,
                              int values_on_device, const ilc_job* jobs, int32_t n_jobs,
                              ilc_tolerance tol, float* images, uint64_t images_len,
                              int images_on_device, ilc_render_stats* stats);

/* Schedule of ilc_render_batched: work items are tiles of tile_w x
 * (32 / tile_w) pixels (tile_w in 1, 2, 4, 8, 16, 32), one per warp, or with
 * tile_w = 0 strided items (pixels k, k + T, k + 2T, ... of a job with T items,
 * which spreads the expensive rays of a small region over many warps); 0
 * (register-limited), 3, 4 or 5 blocks per SM; z_window > 0 makes a warp's rays
 * advance in windows of that depth (they query one slab of the grid at a
 * time); cost_order != 0 hands out the tiles in decreasing order of an
 * estimated cost (particles projected into each tile's columns, weighted by
 * their cell's occupancy), so the longest rays start first. Changes the order
 * of work only, never a result. Default: 8, 4, 40, 1. */
ilc_status ilc_set_batch_schedule(ilc_ctx* ctx, int32_t tile_w, int32_t blocks_per_sm,
                                  float z_window, int32_t cost_order);

/* Autotuner of the batched render's schedule: renders the jobs once per
 * (tile_w, occupancy, z_window) candidate (outputs discarded, cost order on),
 * times the kernel with CUDA events, sets the fastest and returns it
 * (times_ms, may be NULL: n_tiles x n_occupancies x n_windows, in that
 * nesting). Callers pass a representative subset of their jobs (e.g. the
 * same cameras at a lower resolution). */
ilc_status ilc_autotune_batched(ilc_ctx* ctx, const float* values, int32_t n_channels,
                                int values_on_device, const ilc_job* jobs, int32_t n_jobs,
                                ilc_tolerance tol, const int32_t* tile_ws, int32_t n_tiles,
                                const int32_t* occupancies, int32_t n_occupancies,
                                const float* windows, int32_t n_windows, int32_t* best_tile_w,
                                int32_t* best_occupancy, float* best_window, float* times_ms);

/* ---- adjoint ------------------------------------------------------------
 * Gradient of L = sum over pixels of (log I - log I_target)^2 for the X-ray
 * band map of ilc_project_xray_flux, with respect to per-cell ln rho and
 * ln T, the neighbour choice fixed and the line-of-sight step sequence frozen
 * from the forward pass. No reference counterpart (the reference has no
 * differentiation). CHECKPOINT stores every ray's accepted step sizes during
 * the forward pass (4 B x (z_range / 0.2 + 2) per ray of device memory) and
 * replays them; the image is processed in bands of pixel rows (multiples of
 * 8) whose checkpoints fit the context's budget (ilc_set_checkpoint_budget,
 * default a quarter of the device's memory), each band forward, seeded and
 * replayed before the next, so
 * any image size fits. RECOMPUTE runs the step controller again instead. Pixels whose
 * value or target is not positive are left out of L. The per-cell factors
 * dq/dln rho and dq/dln T are exact derivatives of the adaptive energy
 * integration of xray_flux. image receives the forward band map. */
enum { ILC_ADJOINT_CHECKPOINT = 0, ILC_ADJOINT_RECOMPUTE = 1 };

typedef struct ilc_adjoint_stats {
  double loss;
  float quantity_ms;   /* per-cell flux + derivatives */
  float forward_ms;    /* forward render kernel (with step recording in CHECKPOINT) */
  float adjoint_ms;    /* adjoint render kernel */
  uint64_t forward_steps;
  uint64_t adjoint_steps;
} ilc_adjoint_stats;

/* Device memory the CHECKPOINT adjoint may use for step checkpoints (bytes;
 * 0 = a quarter of the device's memory, the default; at least one band of 8
 * pixel rows is always used). No reference counterpart. */
ilc_status ilc_set_checkpoint_budget(ilc_ctx* ctx, uint64_t bytes);

ilc_status ilc_adjoint_xray_flux(ilc_ctx* ctx, const float* cells, const float* rho,
                                 const float* u, const float* xe, uint64_t n, float redshift,
                                 float luminosity_distance, float e_min, float e_max,
                                 int32_t num_samples, const ilc_camera* cam, double z_range,
                                 ilc_tolerance tol, int32_t controller,
                                 const ilc_los_scaling* scaling, const float* target, int32_t mode,
                                 float* image, float* dL_dlnrho, float* dL_dlnT, int is_device,
                                 ilc_adjoint_stats* stats);

/* Autotuner of the adaptive render's schedule: renders every sample_stride-th
 * row of 8-pixel tiles of the view once per (z window, occupancy) candidate
 * pair, times the render kernel with CUDA events, sets the fastest pair on the
 * context and returns it (times_ms, may be NULL: n_windows x n_occupancies
 * kernel times, window-major). Needs the particles set up. The result depends
 * on the particle distribution and the view, so callers cache it per workload. */
ilc_status ilc_autotune_render(ilc_ctx* ctx, const ilc_camera* cam, double z_range,
                               ilc_tolerance tol, int32_t controller, const float* windows,
                               int32_t n_windows, const int32_t* occupancies,
                               int32_t n_occupancies, int32_t sample_stride, float* best_window,
                               int32_t* best_occupancy, float* times_ms);

/* Allocation-free grid build, for callers that cannot allocate device memory
 * when they need a grid (for example a real-time loop with a fixed device
 * memory budget, or a host whose own allocator owns every device buffer and
 * forbids allocations behind its back). No counterpart in the reference. It
 * builds the same grid as ilc_nn8_setup_particles into caller-owned device
 * buffers: particles (n float4), sorted_particles (n float4), cells
 * (cells_capacity int2), sorted_to_unsorted (n uint32), all on the current
 * device; desc receives the grid parameters (also when cells_capacity is too
 * small, so the caller can size the cells buffer and call again). It
 * allocates nothing: the sort's scratch is a fixed device array inside the
 * library, sized for at most ILC_NOALLOC_MAX_PARTICLES particles (about
 * 16.5 MiB per GPU that loads the library, held until the process exits);
 * larger n is rejected with ILC_ERR_INVALID_ARGUMENT. The first call on a
 * device looks the array's device address up once, so make that first call
 * before any stream capture. Every call shares the one scratch array: calls
 * whose work overlaps on the GPU (different streams or host threads at the
 * same time) race. Work is issued on `stream` (a cudaStream_t, NULL = default
 * stream); the call waits on that stream twice (for the bounding box, which
 * the grid parameters are computed from on the host, and for the final
 * status), so its work has finished when it returns. */
#define ILC_NOALLOC_MAX_PARTICLES 1048576
ilc_status ilc_grid_build_noalloc(const float* particles, uint64_t n, float* sorted_particles,
                                  int32_t* cells, uint64_t cells_capacity,
                                  uint32_t* sorted_to_unsorted, ilc_grid_desc* desc,
                                  void* stream);

/* Number of kernels this context has launched so far. */
uint64_t ilc_kernel_launches(const ilc_ctx* ctx);

/* ---- device memory ----------------------------------------------------------
 * Device memory on the context's device, for hosts that keep evaluation
 * points and results on the device without linking the CUDA runtime
 * themselves: the role of the cl::Buffer objects the reference's backends own
 * and hand out (reconstruction_backend.hpp:43 retrieve_results,
 * volumetric_reconstruction_backend_nn8.hpp:72-80 _evaluation_points /
 * _results). ilc_device_free waits for the context's stream first.
 * ilc_copy copies `bytes` between any two host or device pointers on the
 * context's stream and waits for the copy. */
ilc_status ilc_device_alloc(ilc_ctx* ctx, uint64_t bytes, void** out);
ilc_status ilc_device_free(ilc_ctx* ctx, void* p);
ilc_status ilc_copy(ilc_ctx* ctx, void* dst, const void* src, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* ILC_H */
