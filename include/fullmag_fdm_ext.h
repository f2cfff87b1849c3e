/*
 * fullmag_fdm_ext.h — additive C ABI of the B200 FDM stepper.
 *
 * Everything here is new: the reference has no counterpart for these entry
 * points, and existing callers of fullmag_fdm.h are unaffected by them.
 * They expose the capabilities this library adds on top of the drop-in path:
 *   - per-cell saturation magnetisation and a time-dependent Zeeman term;
 *   - FP64 Newell-tensor spectra computed inside the library from the grid
 *     (for callers that do not ship spectra of their own);
 *   - back-to-back stepping without a host round trip per step;
 *   - per-kernel device timing for roofline reports.
 */
#ifndef FULLMAG_FDM_EXT_H
#define FULLMAG_FDM_EXT_H

#include "fullmag_fdm.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FULLMAG_FDM_EXT_VERSION 1

/* How the demag tensor is obtained when enable_demag is set. */
typedef enum {
    FULLMAG_FDM_EXT_DEMAG_FROM_PLAN = 0,   /* use the plan's spectra (or projection if none) */
    FULLMAG_FDM_EXT_DEMAG_NEWELL    = 1,   /* compute FP64 Newell spectra from the grid */
} fullmag_fdm_ext_demag_source;

typedef struct {
    uint32_t struct_size;       /* sizeof(fullmag_fdm_plan_ext) */
    /* Per-cell Ms [A/m], length = cell count; cells with Ms <= 0 are inactive.
     * NULL keeps the uniform material Ms. */
    const double *ms_map;
    uint64_t      ms_map_len;
    /* Zeeman term H(t) = external_field_am + ac_field_am * sin(2 pi f t),
     * evaluated at each stage time (requires has_external_field = 1). */
    double        ac_field_am[3];
    double        ac_frequency_hz;
    fullmag_fdm_ext_demag_source demag_source;
} fullmag_fdm_plan_ext;

/* create() with the extension block (ext may be NULL). */
fullmag_fdm_backend *fullmag_fdm_backend_create_ext(const fullmag_fdm_plan_desc *plan,
                                                    const fullmag_fdm_plan_ext *ext);

/* Take n_steps steps of dt back to back, reading diagnostics back only after
 * the last one (Heun: fixed dt; DP45: each step starts from the previous
 * step's suggested dt).  Equivalent to n_steps calls of
 * fullmag_fdm_backend_step; out_last receives the last step's stats. */
int fullmag_fdm_backend_step_n(fullmag_fdm_backend *handle, double dt_seconds,
                               uint32_t n_steps, fullmag_fdm_step_stats *out_last);

/* ---- Adjoint of a Heun trajectory (no counterpart in the reference) ----
 *
 * fullmag_fdm_adjoint_forward: from the current state, take n_steps Heun
 * steps of dt exactly like n_steps calls of fullmag_fdm_backend_step, keeping
 * the state every checkpoint_every steps on the device (0: ceil(sqrt(n_steps))).
 * out_last receives the last step's stats.
 *
 * fullmag_fdm_adjoint_backward: with dl_dm = dL/dm at the final state (AoS,
 * len = 3 * cell_count), replay each checkpoint segment and pull the cotangent
 * back through the discrete Heun steps (exchange, demag, Zeeman and LLG).
 * Outputs, each optional (NULL):
 *   dl_dms     [cell_count]   dL/dMs per cell (sum it for a uniform Ms);
 *   dl_dh_ext  [3]            dL/dH_ext, A/m (the static external field);
 *   dl_dh_ac   [3]            dL/dH_ac, A/m (amplitude of H_ac sin(2 pi f t));
 *   dl_dm0     [3 cell_count] dL/dm at the starting state (AoS).
 * The backend is left at the final state.  Requires the Heun integrator and a
 * plan without region exchange tables or boundary tiers; the backward pass
 * must follow the forward pass with no step or upload in between.  Memory:
 * (checkpoints + checkpoint_every + 10) state vectors in the plan's precision
 * plus 7 FP64 vectors, allocated by the forward pass. */
int fullmag_fdm_adjoint_forward(fullmag_fdm_backend *handle, double dt_seconds, uint32_t n_steps,
                                uint32_t checkpoint_every, fullmag_fdm_step_stats *out_last);
int fullmag_fdm_adjoint_backward(fullmag_fdm_backend *handle, const double *dl_dm, uint64_t len,
                                 double *dl_dms, double *dl_dh_ext, double *dl_dh_ac, double *dl_dm0);

/* ---- Batched ensemble (no counterpart in the reference) ----
 *
 * Many independent uniform-material problems (own grid, cell size, Ms, A,
 * alpha, gamma, static field and m0) stepped together with Heun: every stage
 * of a step is one persistent launch over all problems, and a step is one
 * CUDA graph.  Grids up to 512 x 512 x 8 cells; the demag spectra are the
 * library's FP64 Newell tensor (no mask, regions or boundary tiers), for each
 * problem's padding: x and y to the smallest power of two >= 2n, or in FP32
 * the smallest power of two or 3 * 2^k (96, 192, 384, 768) >= 2n; z to a power
 * of two >= 2 nz.  On the
 * first fullmag_fdm_batch_step_n call an autotuner picks each kernel's
 * persistent grid size and the tile shape of the x and y passes (128- or
 * 256-thread blocks); fullmag_fdm_batch_tuning reports the picks (7 grid sizes:
 * x forward, y forward, z convolution, y inverse, x inverse, stage, predictor;
 * with len >= 9 also the x and y passes' threads per block).
 * create returns a handle even on failure, with last_error set (NULL only when
 * the handle itself cannot be allocated). */
typedef struct {
    uint32_t nx, ny, nz;
    double dx, dy, dz;
    double saturation_magnetisation;
    double exchange_stiffness;
    double damping;
    double gyromagnetic_ratio;
    double external_field_am[3];
    const double *initial_magnetization_xyz; /* AoS, 3 nx ny nz; read during create */
} fullmag_fdm_batch_problem;

typedef struct fullmag_fdm_batch fullmag_fdm_batch;

fullmag_fdm_batch *fullmag_fdm_batch_create(const fullmag_fdm_batch_problem *problems, uint32_t count,
                                            fullmag_fdm_precision precision);
int fullmag_fdm_batch_step_n(fullmag_fdm_batch *batch, double dt_seconds, uint32_t n_steps);
int fullmag_fdm_batch_copy_m(fullmag_fdm_batch *batch, uint32_t index, double *out_xyz, uint64_t len);
int fullmag_fdm_batch_tuning(const fullmag_fdm_batch *batch, int32_t *grid_sizes, uint32_t len);
const char *fullmag_fdm_batch_last_error(const fullmag_fdm_batch *batch);
void fullmag_fdm_batch_destroy(fullmag_fdm_batch *batch);
/* The CUDA stream (cudaStream_t) the batch's kernels and graphs run on, for
 * timing with events. */
int fullmag_fdm_batch_get_stream(const fullmag_fdm_batch *batch, void **stream_out);
/* One Heun step of the whole batch with its launches issued one by one (not as
 * the graph) and CUDA events around each: ms_per_kind[k] is the device time of
 * kernel kind k during that step, for the 7 kinds of fullmag_fdm_batch_tuning
 * (each demag kind runs twice per step, the stage kernel twice, the predictor
 * kernel not at all).  The batch advances by that step. */
int fullmag_fdm_batch_profile_step(fullmag_fdm_batch *batch, double dt_seconds, float *ms_per_kind,
                                   uint32_t len);

/* Per-kernel device timing with CUDA events on the library's stream. */
int fullmag_fdm_backend_set_profiling(fullmag_fdm_backend *handle, int enable);
int fullmag_fdm_backend_profile_count(fullmag_fdm_backend *handle);
int fullmag_fdm_backend_profile_entry(fullmag_fdm_backend *handle, int index,
                                      const char **out_name, double *out_total_ms,
                                      uint64_t *out_launches);
void fullmag_fdm_backend_profile_reset(fullmag_fdm_backend *handle);

/* Device bytes held by the handle, and the padded FFT extents in use. */
int fullmag_fdm_backend_memory_info(fullmag_fdm_backend *handle, uint64_t *out_device_bytes,
                                    uint32_t *out_fft_dims3);

/* The CUDA stream the handle launches all its work on (a cudaStream_t), so
 * callers can order their own work or record CUDA events around steps. */
int fullmag_fdm_backend_get_stream(fullmag_fdm_backend *handle, void **out_stream);

/* Seeded initial magnetisation as the reference planner draws it
 * (crates/fullmag-plan/src/lib.rs:1928-1957): xorshift64 samples of the cube
 * [-1, 1]^3, normalised; AoS f64 [3 * count]. */
void fullmag_fdm_random_unit_vectors(uint64_t seed, uint64_t count, double *out_xyz);

/* FP64 Newell spectra on the host, in the reference's interleaved complex
 * layout (length 2 * (2nx)(2ny)(2nz), or 2 * (2nx)(2ny) when thin_film_2d and
 * nz == 1): the same arrays the reference runner passes in the plan.
 * Any output pointer may be NULL.  Returns FULLMAG_FDM_OK or ERR_INVALID. */
int fullmag_fdm_newell_spectra(uint32_t nx, uint32_t ny, uint32_t nz, double dx, double dy,
                               double dz, int thin_film_2d, double *xx, double *yy,
                               double *zz, double *xy, double *xz, double *yz);

/* Demag field H = -IFFT(N(k) FFT(Ms m)) without any device allocation.
 *
 * This entry point has no counterpart in the reference.  It serves callers
 * that cannot allocate device memory themselves through this library: code
 * running inside a host framework that owns the whole device-memory budget
 * (every allocation must go through that framework's allocator), and
 * latency-critical loops that must avoid the implicit device synchronisation
 * of cudaMalloc / cudaFree.  The caller passes device pointers for the inputs
 * and the output; the library allocates nothing.
 *
 *   octant : FP64 Newell octant [6][KZ][nx+1][ny+1] (components xx, yy, zz,
 *            xy, xz, yz; KZ = nz + 1, or 1 for the thin-film form): the real
 *            parts of the spectra fullmag_fdm_newell_spectra returns, at
 *            kz <= nz (kz = 0 when thin), kx <= nx, ky <= ny;
 *   m      : SoA [x[N], y[N], z[N]] FP64 unit vectors, every cell active;
 *   ms     : uniform saturation magnetisation (A/m);
 *   h      : SoA [3N] FP64 output;
 *   stream : cudaStream_t to launch on (NULL = legacy default stream);
 *   error_out / error_out_len : optional buffer for a failure message.
 *
 * Limits: 2nx and 2ny powers of two <= 1024, and 2nz <= 16 unless nz = 1 and
 * thin_film_2d is set; the FFT work arrays must fit the library's fixed 32 MiB
 * scratch array (every GPU that loads the library holds it until the process
 * exits).  Larger grids are rejected with FULLMAG_FDM_ERR_INVALID and a message
 * giving the bytes needed.
 *
 * The first call on a device resolves the scratch array's device address,
 * fills the twiddle constants and synchronises the device once; make that
 * first call outside any CUDA stream capture.  The constants are not refilled
 * after cudaDeviceReset (or any new primary context) on that device, so do not
 * use this entry point across a device reset.  All calls share the one scratch
 * array: calls that overlap on the GPU (different streams or threads without
 * ordering) race.  Each call writes every scratch element it reads, so nothing
 * has to start at zero. */
int fullmag_fdm_demag_field_f64_noalloc(uint32_t nx, uint32_t ny, uint32_t nz,
                                        int thin_film_2d, const double *octant,
                                        const double *m, double ms, double *h,
                                        void *stream, char *error_out,
                                        uint64_t error_out_len);

#ifdef __cplusplus
}
#endif

#endif /* FULLMAG_FDM_EXT_H */
