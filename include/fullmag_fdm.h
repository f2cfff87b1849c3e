/*
 * fullmag_fdm.h — C ABI of the B200 FDM time-stepper (drop-in seam).
 *
 * This header declares the exact binary interface that the reference's Rust
 * runner binds (crates/fullmag-fdm-sys/src/lib.rs:200-288) and that the
 * reference declares in native/include/fullmag_fdm.h:35-405.  Every name,
 * enum value, struct field, field order and field type is kept identical so
 * that libfullmag_fdm.so.0 built from this repository replaces the
 * reference's library without recompiling its callers.  The implementation
 * behind it (fullmag_b200/csrc) is new: sm_100a kernels with an in-house
 * FFT, fused stencil/LLG stages, device-side reductions.
 *
 * Conventions (unchanged from the reference interface):
 *   - host vector fields are AoS f64/f32: [x0, y0, z0, x1, y1, z1, ...],
 *     flat cell index = x + nx * (y + ny * z);
 *   - snapshots expose SoA payloads: [x0..xN-1, y0..yN-1, z0..zN-1];
 *   - return codes: 0 ok, -1 invalid argument, -2 CUDA failure, -3 internal;
 *   - fullmag_fdm_backend_create returns a handle even when it fails; the
 *     caller checks fullmag_fdm_backend_last_error and then destroys it.
 */
#ifndef FULLMAG_FDM_H
#define FULLMAG_FDM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes (native/include/fullmag_fdm.h:37-40). */
#define FULLMAG_FDM_OK            0
#define FULLMAG_FDM_ERR_INVALID  -1
#define FULLMAG_FDM_ERR_CUDA     -2
#define FULLMAG_FDM_ERR_INTERNAL -3

/* Size of one side of the square inter-region exchange table (fullmag_fdm.h:43). */
#define FULLMAG_FDM_MAX_EXCHANGE_REGIONS 256

/* Arithmetic of the stepper (fullmag_fdm.h:47-50).  SINGLE selects the
 * FP32-mixed path: FP32 state, stencil, FFT and stages; FP64 Newell setup,
 * renormalisation, energies and error norms. */
typedef enum {
    FULLMAG_FDM_PRECISION_SINGLE = 1,
    FULLMAG_FDM_PRECISION_DOUBLE = 2,
} fullmag_fdm_precision;

/* Time integrators (fullmag_fdm.h:52-58).  All five are implemented, in both
 * precisions: HEUN and DP45 (adaptive, FSAL) on the hot path, and ABM3, RK4
 * and RK23 (adaptive) on the same fused stage kernels. */
typedef enum {
    FULLMAG_FDM_INTEGRATOR_HEUN = 1,
    FULLMAG_FDM_INTEGRATOR_DP45 = 2,
    FULLMAG_FDM_INTEGRATOR_ABM3 = 3,
    FULLMAG_FDM_INTEGRATOR_RK4  = 4,
    FULLMAG_FDM_INTEGRATOR_RK23 = 5,
} fullmag_fdm_integrator;

/* Field observables (fullmag_fdm.h:60-66). */
typedef enum {
    FULLMAG_FDM_OBSERVABLE_M        = 1,
    FULLMAG_FDM_OBSERVABLE_H_EX     = 2,
    FULLMAG_FDM_OBSERVABLE_H_DEMAG  = 3,
    FULLMAG_FDM_OBSERVABLE_H_EXT    = 4,
    FULLMAG_FDM_OBSERVABLE_H_EFF    = 5,
} fullmag_fdm_observable;

/* Scalar type of a snapshot payload (fullmag_fdm.h:68-71). */
typedef enum {
    FULLMAG_FDM_SNAPSHOT_SCALAR_F32 = 1,
    FULLMAG_FDM_SNAPSHOT_SCALAR_F64 = 2,
} fullmag_fdm_snapshot_scalar_type;

/* Boundary-correction tier (fullmag_fdm.h:73-77).  All three are implemented:
 * NONE (binary mask), VOLUME (T0 face-link exchange and phi-weighted demag) and
 * FULL (T1 ECB exchange stencil, phi-weighted demag and the sparse demag
 * correction).  A tier whose per-cell arrays are missing or of the wrong length
 * is rejected with ERR_INVALID instead of being skipped. */
typedef enum {
    FULLMAG_FDM_BOUNDARY_NONE   = 0,
    FULLMAG_FDM_BOUNDARY_VOLUME = 1,
    FULLMAG_FDM_BOUNDARY_FULL   = 2,
} fullmag_fdm_boundary_correction;

/* Grid (fullmag_fdm.h:81-88): cell counts and cell edge lengths in metres. */
typedef struct {
    uint32_t nx;
    uint32_t ny;
    uint32_t nz;
    double   dx;
    double   dy;
    double   dz;
} fullmag_fdm_grid_desc;

/* Material (fullmag_fdm.h:90-95). */
typedef struct {
    double saturation_magnetisation;   /* Ms, A/m */
    double exchange_stiffness;         /* A, J/m */
    double damping;                    /* alpha */
    double gyromagnetic_ratio;         /* gamma, m/(A s), Gilbert form */
} fullmag_fdm_material_desc;

/* Executable plan (fullmag_fdm.h:99-198).  All pointers are borrowed for the
 * duration of fullmag_fdm_backend_create only. */
typedef struct {
    fullmag_fdm_grid_desc      grid;
    fullmag_fdm_material_desc  material;
    fullmag_fdm_precision      precision;
    fullmag_fdm_integrator     integrator;
    int                        disable_precession;  /* 1: RHS keeps only the damping term */
    int                        enable_exchange;
    int                        enable_demag;
    int                        has_external_field;
    double                     external_field_am[3]; /* H_ext, A/m */

    /* Newell tensor spectra, interleaved complex f64 [re, im, ...] of length
     * demag_kernel_spectrum_len = 2 * (2nx)(2ny)(2nz), or 2 * (2nx)(2ny) for
     * the nz = 1 thin-film form.  When the length is 0 and demag is enabled
     * the k k^T / k^2 spectral-projection tensor is used instead. */
    const double              *demag_kernel_xx_spectrum;
    const double              *demag_kernel_yy_spectrum;
    const double              *demag_kernel_zz_spectrum;
    const double              *demag_kernel_xy_spectrum;
    const double              *demag_kernel_xz_spectrum;
    const double              *demag_kernel_yz_spectrum;
    uint64_t                   demag_kernel_spectrum_len;

    /* Optional geometry mask, 1 = active, length = cell count. */
    const uint8_t             *active_mask;
    uint64_t                   active_mask_len;

    /* Optional region ids (< 256), length = cell count. */
    const uint32_t            *region_mask;
    uint64_t                   region_mask_len;

    /* Optional 256 x 256 row-major table A_ij [J/m]; default A_ii = A, A_ij = 0. */
    const double              *exchange_lut;
    uint64_t                   exchange_lut_len;

    /* Boundary-correction inputs (T0/T1 tiers); must be NONE / unused here. */
    fullmag_fdm_boundary_correction boundary_correction;
    double                     boundary_phi_floor;
    double                     boundary_delta_min;
    const double              *volume_fraction;
    uint64_t                   volume_fraction_len;
    const double              *face_link_xp;
    const double              *face_link_xm;
    const double              *face_link_yp;
    const double              *face_link_ym;
    const double              *face_link_zp;
    const double              *face_link_zm;
    const double              *delta_xp;
    const double              *delta_xm;
    const double              *delta_yp;
    const double              *delta_ym;
    const double              *delta_zp;
    const double              *delta_zm;
    int                        has_demag_boundary_corr;
    const int32_t             *demag_corr_target_idx;
    const int32_t             *demag_corr_source_idx;
    const double              *demag_corr_tensor;
    uint32_t                   demag_corr_target_count;
    uint32_t                   demag_corr_stencil_size;

    /* Initial magnetisation, AoS f64, length 3 * cell count. */
    const double              *initial_magnetization_xyz;
    uint64_t                   initial_magnetization_len;

    /* DP45 controller; 0 selects the defaults 1e-5, 1e-18, 1e-10, 0.8. */
    double                     adaptive_max_error;
    double                     adaptive_dt_min;
    double                     adaptive_dt_max;
    double                     adaptive_headroom;
} fullmag_fdm_plan_desc;

/* Per-step diagnostics (fullmag_fdm.h:202-215). */
typedef struct {
    uint64_t step;
    double   time_seconds;
    double   dt_seconds;
    double   exchange_energy_joules;
    double   demag_energy_joules;
    double   external_energy_joules;
    double   total_energy_joules;
    double   max_effective_field_amplitude;  /* max |H_eff| */
    double   max_demag_field_amplitude;      /* max |H_demag| */
    double   max_rhs_amplitude;              /* max |dm/dt| */
    double   suggested_next_dt;              /* DP45: controller proposal for the next call */
    uint64_t wall_time_ns;                   /* host wall time of the call */
} fullmag_fdm_step_stats;

/* Device metadata (fullmag_fdm.h:219-225). */
typedef struct {
    char name[128];
    int  compute_capability_major;
    int  compute_capability_minor;
    int  driver_version;
    int  runtime_version;
} fullmag_fdm_device_info;

/* Snapshot payload description (fullmag_fdm.h:227-232). */
typedef struct {
    uint64_t cell_count;
    uint32_t component_count;
    uint32_t scalar_bytes;
    fullmag_fdm_snapshot_scalar_type scalar_type;
} fullmag_fdm_snapshot_desc;

typedef struct fullmag_fdm_backend fullmag_fdm_backend;
typedef struct fullmag_fdm_field_snapshot fullmag_fdm_field_snapshot;

/* 1 when a CUDA device is usable (FULLMAG_FDM_GPU_INDEX /
 * FULLMAG_CUDA_DEVICE_INDEX honoured), else 0.  fullmag_fdm.h:245. */
int fullmag_fdm_is_available(void);

/* Validate the plan, allocate device state, upload inputs and evaluate the
 * initial fields.  fullmag_fdm.h:252 / native/backends/fdm/src/api.cpp:87-310. */
fullmag_fdm_backend *fullmag_fdm_backend_create(const fullmag_fdm_plan_desc *plan);

/* One Heun step of dt, or one accepted DP45 step starting from dt.
 * fullmag_fdm.h:260 / api.cpp:314-376. */
int fullmag_fdm_backend_step(fullmag_fdm_backend *handle, double dt_seconds,
                             fullmag_fdm_step_stats *out_stats);

/* Copy an observable to host AoS f64 / f32 (out_len = 3 * cell count).
 * fullmag_fdm.h:269,279 / api.cpp:380-426. */
int fullmag_fdm_backend_copy_field_f64(fullmag_fdm_backend *handle,
                                       fullmag_fdm_observable observable,
                                       double *out_xyz, uint64_t out_len);
int fullmag_fdm_backend_copy_field_f32(fullmag_fdm_backend *handle,
                                       fullmag_fdm_observable observable,
                                       float *out_xyz, uint64_t out_len);

/* Box-averaged preview (fullmag_fdm.h:291,308; context.cu:222-286). */
int fullmag_fdm_backend_copy_field_preview_f64(fullmag_fdm_backend *handle,
                                               fullmag_fdm_observable observable,
                                               uint32_t preview_nx, uint32_t preview_ny,
                                               uint32_t preview_nz, uint32_t z_origin,
                                               uint32_t z_stride, double *out_xyz,
                                               uint64_t out_len);
int fullmag_fdm_backend_copy_field_preview_f32(fullmag_fdm_backend *handle,
                                               fullmag_fdm_observable observable,
                                               uint32_t preview_nx, uint32_t preview_ny,
                                               uint32_t preview_nz, uint32_t z_origin,
                                               uint32_t z_stride, float *out_xyz,
                                               uint64_t out_len);

/* Asynchronous SoA snapshot (fullmag_fdm.h:334-357; context.cu:1071-1258). */
fullmag_fdm_field_snapshot *fullmag_fdm_backend_begin_field_snapshot(
    fullmag_fdm_backend *handle, fullmag_fdm_observable observable);
int fullmag_fdm_field_snapshot_wait(fullmag_fdm_field_snapshot *snapshot,
                                    const void **out_data, uint64_t *out_len_bytes,
                                    fullmag_fdm_snapshot_desc *out_desc);
void fullmag_fdm_field_snapshot_destroy(fullmag_fdm_field_snapshot *snapshot);

/* Replace m from host AoS (inactive cells zeroed; time is not advanced).
 * fullmag_fdm.h:364,375. */
int fullmag_fdm_backend_upload_magnetization_f64(fullmag_fdm_backend *handle,
                                                 const double *m_xyz, uint64_t len);
int fullmag_fdm_backend_upload_magnetization_f32(fullmag_fdm_backend *handle,
                                                 const float *m_xyz, uint64_t len);

/* Recompute H_ex, H_demag and H_eff for the current m.  fullmag_fdm.h:384. */
int fullmag_fdm_backend_refresh_observables(fullmag_fdm_backend *handle);

/* fullmag_fdm.h:390. */
int fullmag_fdm_backend_get_device_info(fullmag_fdm_backend *handle,
                                        fullmag_fdm_device_info *out_info);

/* Last error of this handle or NULL; "null handle" for NULL.  fullmag_fdm.h:397. */
const char *fullmag_fdm_backend_last_error(fullmag_fdm_backend *handle);

/* Free device state; NULL is accepted.  fullmag_fdm.h:403. */
void fullmag_fdm_backend_destroy(fullmag_fdm_backend *handle);

#ifdef __cplusplus
}
#endif

#endif /* FULLMAG_FDM_H */
