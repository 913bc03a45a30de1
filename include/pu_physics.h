/* pu_physics.h -- C ABI of the B200 implementations of the physics modules
 * that the boundary-layer drivers run beside the dycore every dt_phys
 * (abl_neutral.cpp:93-104 of the reference):
 *
 *   pu_les_apply            modules::LES_Closure::apply          les_closure.h:30-320
 *   pu_sponge_layer         modules::sponge_layer                sponge_layer.h:7-62
 *   pu_geostrophic_forcing  modules::geostrophic_wind_forcing    geostrophic_wind_forcing.h:7-42
 *   pu_surface_fluxes       modules::apply_surface_fluxes        surface_flux.h:9-125
 *   pu_uniform_pg_wind_forcing         modules::uniform_pg_wind_forcing
 *                                      uniform_pg_wind_forcing.h:6-40
 *   pu_uniform_pg_wind_forcing_height  modules::uniform_pg_wind_forcing_height
 *                                      uniform_pg_wind_forcing.h:43-82
 *                                      (city.cpp:130-136, cubes_periodic.cpp:147-152)
 *   pu_time_averager_accumulate        custom_modules::Time_Averager::accumulate
 *                                      experiments/examples/custom_modules/time_averager.h:56-110
 *   pu_edge_sponge_set_column / _apply custom_modules::EdgeSponge::set_column / apply
 *                                      experiments/examples/custom_modules/edge_sponge.h:14-57
 *
 * The reference's modules read their options and the immersed halo arrays
 * from the coupler; here a pu_physics handle holds them (created once, like
 * the arrays the drivers' init registers, sc_init.h:727-768) and each call
 * takes the coupler arrays as a pu_state_view (pu_dycore.h): density_dry,
 * uvel, vvel, wvel, temp and the tracers in coupler order, C-order
 * (nz,ny,nx) doubles, host or device memory.  Arithmetic is FP64 as in the
 * reference.  Every call returns PU_OK or a PU_ERR_* code (pu_last_error()),
 * where the reference aborts.  Calls on one handle are ordered on its stream
 * and are asynchronous for device views; pu_physics_synchronize waits.
 */
#ifndef PU_PHYSICS_H
#define PU_PHYSICS_H

#include "pu_dycore.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pu_physics pu_physics;

typedef struct pu_physics_config {
  int nx, ny, nz;
  double dx, dy, dz;
  int ntracers;                            /* coupler tracers, including TKE */
  int tracer_diffuse[PU_MAX_TRACERS];      /* get_tracer_info(..., diffuse) */
  int idTKE;                               /* index of the "TKE" tracer (mass-weighted TKE), or -1 */
  double R_d, gamma_d, C0, grav;           /* coupler options */
  int enable_gravity;
  double kinematic_viscosity;              /* option "kinematic_viscosity" (default 0) */
  int dns;                                 /* option "dns" (default false) */
  double les_total_mult, les_dissipation_mult, les_shear_prod_mult; /* defaults 1 */
  int bc_x, bc_y, bc_z;                    /* pu_bc */
  int device;
  void *stream;                            /* cudaStream_t, or NULL for the legacy default stream */
} pu_physics_config;

/* Creates a handle.  imm_prop_h, imm_rough_h, imm_temp_h are the
 * immersed_proportion_halos, immersed_roughness_halos and immersed_temp_halos
 * arrays ((nz+2,ny+2,nx+2) doubles with one halo cell per side; mem is
 * PU_MEM_HOST, PU_MEM_DEVICE or PU_MEM_AUTO); the handle keeps a device copy.
 * Replaces the options and DataManager reads of the four modules. */
int pu_physics_create(const pu_physics_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h, int mem, pu_physics **out);
int pu_physics_destroy(pu_physics *h);

/* LES_Closure::apply(coupler, dt) (les_closure.h:30-320): TKE closure,
 * diffusive fluxes of momentum, theta, TKE and diffused tracers, TKE sources;
 * updates uvel, vvel, wvel, temp, TKE and the diffused tracers in place.  The
 * update reads neighbours, so the new values go to a device scratch first and
 * are copied back (pu_les_apply_to avoids the copy). */
int pu_les_apply(pu_physics *h, pu_state_view *v, double dt);
/* The same update from `in` into `out` (device views, distinct arrays; the
 * untouched fields -- density_dry and the non-diffused tracers other than
 * TKE -- are not written). */
int pu_les_apply_to(pu_physics *h, const pu_state_view *in, pu_state_view *out, double dt);

/* sponge_layer(coupler, dt, time_scale, top_prop) (sponge_layer.h:7-62):
 * relaxes u, v, temp toward their level means and w toward 0 in the top
 * top_prop of the domain.  Level means are FP64 sums with Neumaier
 * compensation. */
int pu_sponge_layer(pu_physics *h, pu_state_view *v, double dt, double time_scale, double top_prop);

/* geostrophic_wind_forcing(coupler, dt, lat_g, u_g, v_g)
 * (geostrophic_wind_forcing.h:7-42). */
int pu_geostrophic_forcing(pu_physics *h, pu_state_view *v, double dt, double lat_g, double u_g, double v_g);

/* apply_surface_fluxes(coupler, dt) (surface_flux.h:9-125): log-law drag and
 * heat flux from immersed face neighbours (the ground is the bottom halo). */
int pu_surface_fluxes(pu_physics *h, pu_state_view *v, double dt);

/* What uniform_pg_wind_forcing carries from call to call; the reference keeps
 * it in the coupler options uniform_pg_wind_forcing_counter, _u0, _v0, _u and
 * _v.  Zero-initialise it before the first call. */
typedef struct pu_uniform_pg_state {
  unsigned long long counter;
  double u0, v0; /* domain means of u and v taken at counter 0 */
  double u, v;   /* the latest domain means */
} pu_uniform_pg_state;

/* uniform_pg_wind_forcing(coupler, dt, tau, update_cycles)
 * (uniform_pg_wind_forcing.h:6-40): when counter % update_cycles == 0 the
 * domain means of uvel and vvel are taken into state->u, v (and u0, v0 on the
 * first call); then every cell gets uvel += dt/tau*(u0-u), vvel +=
 * dt/tau*(v0-v), and counter is incremented.  The means are FP64 sums with
 * Neumaier compensation; a call that takes them synchronises the handle's
 * stream.  PU_ERR_INVALID for update_cycles == 0 or tau <= 0 (the reference
 * divides by them). */
int pu_uniform_pg_wind_forcing(pu_physics *h, pu_state_view *v, double dt, double tau,
                               unsigned long long update_cycles, pu_uniform_pg_state *state);

/* uniform_pg_wind_forcing_height(coupler, dt, height, u0, v0, tau)
 * (uniform_pg_wind_forcing.h:43-82): the mean wind at `height`, linear
 * between the level means of the two levels whose centres bracket it, is
 * relaxed toward (u0, v0): every cell gets uvel += dt/tau*(u0-u(height)),
 * likewise v.  Above the top level centre the two lowest levels are
 * extrapolated, as in the reference.  PU_ERR_INVALID when height is below
 * the first level centre (the reference then reads level -1), nz < 2 or
 * tau <= 0.  Asynchronous for device views. */
int pu_uniform_pg_wind_forcing_height(pu_physics *h, pu_state_view *v, double dt, double height, double u0, double v0,
                                      double tau);

/* The running averages of custom_modules::Time_Averager
 * (experiments/examples/custom_modules/time_averager.h:7-111, run after the
 * LES closure in the boundary-layer drivers, abl_neutral.cpp:98-104): the
 * coupler arrays avg_u .. long_avg_w ((nz,ny,nx) doubles in the memory space
 * of the state view) and the option time_averager_etime. */
typedef struct pu_time_averages {
  double *avg_u, *avg_v, *avg_w, *avg_tke;
  double *avg_up_up, *avg_up_vp, *avg_up_wp, *avg_vp_vp, *avg_vp_wp, *avg_wp_wp;
  double *long_avg_u, *long_avg_v, *long_avg_w;
  double etime; /* time_averager_etime: read, then advanced by dt */
} pu_time_averages;

/* Time_Averager::accumulate(coupler, dt) (time_averager.h:56-110): with
 * inertia = etime/(etime+dt) and inertia_long = elapsed_time/(elapsed_time+dt)
 * (the coupler option elapsed_time), long_avg_u/v/w relax toward u, v, w;
 * avg_u/v/w/tke toward u, v, w, TKE and avg_up_up .. avg_wp_wp toward the
 * products of the departures from the new long averages.  FP64 in the
 * reference's order of operations (no contraction into fma), so results
 * match the reference bit for bit.  PU_ERR_INVALID without a TKE tracer. */
int pu_time_averager_accumulate(pu_physics *h, const pu_state_view *v, pu_time_averages *a, double elapsed_time,
                                double dt);

/* custom_modules::EdgeSponge (experiments/examples/custom_modules/
 * edge_sponge.h:8-101; the urban and turbine drivers, city.cpp:97,137).
 * fields: indices into the state view (0..4 = density_dry, uvel, vvel, wvel,
 * temp; 5+t = tracer t; the reference's default set is 0..4).
 * set_column: the horizontal mean of each field per level into column
 * (nfields*nz doubles, host, field-major), FP64 with Neumaier compensation;
 * synchronous.  apply: relaxes the fields toward column within the fractions
 * prop_x1 / prop_x2 / prop_y1 / prop_y2 of the global domain next to its
 * low-x / high-x / low-y / high-y edges, with weight ((p1-p)/p1)^5 (and the
 * mirror at the high edges), applied in that order.  i_beg, j_beg, nx_glob,
 * ny_glob place this tile in the global grid (0, 0, nx, ny on one rank); on
 * several ranks the caller sums the tiles' column means itself. */
int pu_edge_sponge_set_column(pu_physics *h, const pu_state_view *v, const int *fields, int nfields, double *column);
int pu_edge_sponge_apply(pu_physics *h, pu_state_view *v, const int *fields, int nfields, const double *column,
                         double prop_x1, double prop_x2, double prop_y1, double prop_y2, long long i_beg,
                         long long j_beg, long long nx_glob, long long ny_glob);

/* Waits for the handle's work. */
int pu_physics_synchronize(pu_physics *h);

/* Milliseconds of the last pu_les_apply* kernel (CUDA events on the
 * handle's stream; the copy-back of pu_les_apply is not included), for
 * benchmarks.  Synchronises. */
int pu_physics_last_les_ms(pu_physics *h, double *ms);

#ifdef __cplusplus
}
#endif

#endif /* PU_PHYSICS_H */
