/*
 * aeolus_b200_ghost.h -- C ABI of the ghost-cell wall reconstruction on
 * cut-cell surfaces and of the cut-cell wall model.
 *
 * Replaces (Aeolus.jl):
 *   reconstruct_wall_velocity!(field, stencils, geom; wall_value)
 *                                   src/CutCell.jl:1187-1216  -> aeo_ghost_reconstruct (mode 0)
 *   reconstruct_wall_scalar!(field, stencils, geom; wall_value | wall_flux, kappa)
 *                                   src/CutCell.jl:1218-1266  -> aeo_ghost_reconstruct (mode 0 / 1)
 *   wall_shear_stress(u, v, w, stencils, geom, nu)
 *                                   src/CutCell.jl:1268-1336  -> aeo_ghost_wall_stress (law 0)
 *   wall_shear_stress(u, v, w, stencils, geom, law; nu), wall_slip_velocity(...; nu, nu_eff)
 *                                   src/wall_models/cutcell.jl:1-120 -> aeo_ghost_wall_stress (law 1..3)
 *   friction_velocity(law, U, h; nu) for SpaldingLaw, RoughLogLaw, MOSTWallLaw
 *                                   src/wall_models/laws.jl:72-284
 * The stencils themselves (build_ghost_stencils, src/CutCell.jl:996-1172) are
 * set-up work built on the host (aeolus_b200/ghost.py) and uploaded here.
 *
 * Fields are storage-layout arrays (the reference's Field.data: x fastest,
 * halos included) of nx_s * ny_s * nz_s values; a stencil's target and donors
 * are flat indices into them (donor -1: unused).  Status codes are those of
 * aeolus_b200.h.
 */
#ifndef AEOLUS_B200_GHOST_H
#define AEOLUS_B200_GHOST_H

#include <stdint.h>

#include "aeolus_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aeo_ghost aeo_ghost;

/* n stencils: target[n], donors[8n], weights[8n], dn[n] (signed wall distance),
 * probe[n] (image distance), normal[3n] (unit, into the fluid), flags[n]
 * (bit 0: ghost point, bit 1: valid); host arrays, copied to `device`. */
aeo_status aeo_ghost_create(int32_t nx_s, int32_t ny_s, int32_t nz_s, int64_t n, const int64_t* target,
                            const int64_t* donors, const double* weights, const double* dn, const double* probe,
                            const double* normal, const uint8_t* flags, int32_t device, aeo_ghost** out);
aeo_status aeo_ghost_destroy(aeo_ghost* h);

/* The ghost points of a device field (FP64, or FP32 when fp32 = 1), in place
 * on `stream`: mode 0 Dirichlet, f_ghost = value + (dn/probe)(f_image - value);
 * mode 1 Neumann, f_ghost = f_image + (dn - probe) value/kappa (value the
 * flux kappa df/dn into the fluid).  Only valid ghost stencils are written. */
aeo_status aeo_ghost_reconstruct(aeo_ghost* h, void* field, int32_t fp32, int32_t mode, double value, double kappa,
                                 void* stream);
/* the same on a host FP64 field (copied to the device and back) */
aeo_status aeo_ghost_reconstruct_host(aeo_ghost* h, double* field, int32_t mode, double value, double kappa);

/* The wall shear stress at every (CellCenter) stencil from the face
 * velocities u, v, w and apertures ax, ay, az (FP64 storage arrays; the
 * cell-centred velocity is the aperture-weighted mean of each cell's two
 * faces) interpolated to the image point, its wall-normal part removed:
 * law 0 the resolved nu |u_t| / probe; law 1 Spalding (params kappa, B),
 * 2 the rough log law (kappa, z0), 3 Monin-Obukhov (kappa, z0m, L, U_min;
 * L = inf neutral) give u_tau^2 of the law at h = probe.  slip (3n, may be
 * NULL): the slip velocity u_t (1 - tau probe / (nu_eff |u_t|)) along the
 * tangential image velocity (zero for law 0, an invalid stencil or u_t = 0).
 * tau and slip are device arrays in aeo_ghost_wall_stress, host arrays in
 * the _host form (whose inputs are host arrays too). */
aeo_status aeo_ghost_wall_stress(aeo_ghost* h, const double* u, const double* v, const double* w, const double* ax,
                                 const double* ay, const double* az, int32_t law, const double* params, double nu,
                                 double nu_eff, double* tau, double* slip, void* stream);
aeo_status aeo_ghost_wall_stress_host(aeo_ghost* h, const double* u, const double* v, const double* w,
                                      const double* ax, const double* ay, const double* az, int32_t law,
                                      const double* params, double nu, double nu_eff, double* tau, double* slip);
const char* aeo_ghost_last_error(const aeo_ghost* h);

#ifdef __cplusplus
}
#endif
#endif
