/* C interface of the CPU oracles of the physics modules that run beside the
 * dycore in the boundary-layer drivers (TEST INFRASTRUCTURE ONLY):
 *   orc_phys_*  oracle/_build/liboracle.so      -- this project's restatement
 *   ref_phys_*  oracle/_ref/libporturb_ref.so   -- the reference's own module
 *                                                 headers compiled against the
 *                                                 single-rank shim
 * Modules (model/modules/ of the reference):
 *   LES_Closure::apply              les_closure.h:30-320
 *   sponge_layer                    sponge_layer.h:7-62
 *   geostrophic_wind_forcing        geostrophic_wind_forcing.h:7-42
 *   apply_surface_fluxes            surface_flux.h:9-125
 *   uniform_pg_wind_forcing         uniform_pg_wind_forcing.h:6-40
 *   uniform_pg_wind_forcing_height  uniform_pg_wind_forcing.h:43-82
 *   Time_Averager::accumulate       experiments/examples/custom_modules/time_averager.h:56-110
 *   EdgeSponge::set_column / apply  experiments/examples/custom_modules/edge_sponge.h:14-72
 * All arrays are C-order doubles: coupler fields (nz,ny,nx), tracers
 * (ntr,nz,ny,nx) in coupler order, immersed halo arrays (nz+2,ny+2,nx+2) with
 * one halo cell on each side (immersed_proportion_halos,
 * immersed_roughness_halos, immersed_temp_halos of the drivers' init,
 * sc_init.h:727-768).  The calls update the coupler arrays in place.
 * *_uniform_pg carries st = {counter, u0, v0, u, v} (the coupler options
 * uniform_pg_wind_forcing_counter, _u0, _v0, _u, _v) from call to call.
 * *_time_average takes the 13 averages as one [13][nz][ny][nx] block in the
 * order avg_u, avg_v, avg_w, avg_tke, avg_up_up, avg_up_vp, avg_up_wp,
 * avg_vp_vp, avg_vp_wp, avg_wp_wp, long_avg_u, long_avg_v, long_avg_w and the
 * option time_averager_etime in *etime (advanced by dt). */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_phys_config {
  int nx, ny, nz;
  double xlen, ylen, zlen;
  int ntr;
  int tracer_positive[16], tracer_adds_mass[16], tracer_diffuse[16];
  int idWV, idTKE; /* indices of the water_vapor and TKE tracers */
  double R_d, R_v, cp_d, gamma_d, C0, grav, p0;
  int enable_gravity;
  double kinematic_viscosity;
  int dns;
  double les_total_mult, les_dissipation_mult, les_shear_prod_mult;
  int bc_x, bc_y, bc_z; /* ORC_BC_* of oracle_api.h */
} orc_phys_config;

void *orc_phys_create(const orc_phys_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h);
void orc_phys_destroy(void *h);
int orc_phys_les(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt);
int orc_phys_sponge(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                    double time_scale, double top_prop);
int orc_phys_geostrophic(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                         double lat_g, double u_g, double v_g);
int orc_phys_surface_fluxes(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                            double dt);
int orc_phys_uniform_pg(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                        double tau, unsigned long long update_cycles, double *st);
int orc_phys_uniform_pg_height(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               double dt, double height, double u0, double v0, double tau);
int orc_phys_time_average(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                          double *avgs, double *etime, double elapsed_time, double dt);
/* Edge sponge on the five state fields (the reference's default set):
 * column is (5, nz); set_column fills it, apply uses it. */
int orc_phys_edge_sponge_set_column(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                                    double *column);
int orc_phys_edge_sponge_apply(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               const double *column, double px1, double px2, double py1, double py2);

void *ref_phys_create(const orc_phys_config *cfg, const double *imm_prop_h, const double *imm_rough_h,
                      const double *imm_temp_h);
void ref_phys_destroy(void *h);
int ref_phys_les(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt);
int ref_phys_sponge(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                    double time_scale, double top_prop);
int ref_phys_geostrophic(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                         double lat_g, double u_g, double v_g);
int ref_phys_surface_fluxes(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                            double dt);
int ref_phys_uniform_pg(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc, double dt,
                        double tau, unsigned long long update_cycles, double *st);
int ref_phys_uniform_pg_height(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               double dt, double height, double u0, double v0, double tau);
int ref_phys_time_average(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                          double *avgs, double *etime, double elapsed_time, double dt);
int ref_phys_edge_sponge_set_column(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                                    double *column);
int ref_phys_edge_sponge_apply(void *h, double *rho_d, double *u, double *v, double *w, double *T, double *trc,
                               const double *column, double px1, double px2, double py1, double py2);

#ifdef __cplusplus
}
#endif
