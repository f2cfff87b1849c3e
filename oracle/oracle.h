/*
 * oracle.h — C interface of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a C++ restatement of the reference's CPU engine for the
 * single-grid Exchange + Demag + Zeeman + LLG FDM path:
 *   crates/fullmag-engine/src/lib.rs        (fields, Heun, DP45, RK4, RK23, ABM3, energies, FFT driver)
 *   crates/fullmag-engine/src/vector.rs     (normalisation and vector helpers)
 *   crates/fullmag-fdm-demag/src/newell.rs  (Newell tensor, real space)
 *   crates/fullmag-plan/src/lib.rs:1928-1957 (seeded random unit vectors)
 * plus, where the CPU engine has no counterpart, the semantics of the
 * reference's CUDA backend (region exchange LUT, exchange pair energy:
 * native/backends/fdm/src/exchange_fp64.cu, reductions_fp64.cu).
 *
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * may load this library.  The product library never links it.
 *
 * The reference's FFT is the third-party crate rustfft 6.4.1, which is not
 * vendored with the reference; this oracle uses its own FP64 FFT (mixed radix,
 * direct DFT for prime factors).  FFT results therefore agree with the
 * reference to rounding only; the FFT is checked against numpy.fft and the
 * Newell tensor against the reference's own golden values.
 */
#ifndef FULLMAG_ORACLE_H
#define FULLMAG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_problem oracle_problem;

enum {  /* values of fullmag_fdm_integrator (native/include/fullmag_fdm.h:52-58) */
    ORACLE_HEUN = 1,
    ORACLE_DP45 = 2,
    ORACLE_ABM3 = 3,
    ORACLE_RK4 = 4,
    ORACLE_RK23 = 5,
};

typedef struct {
    uint32_t nx, ny, nz;
    double dx, dy, dz;
    double ms, aex, alpha, gamma;
    int integrator;           /* ORACLE_HEUN / _DP45 / _ABM3 / _RK4 / _RK23 */
    int precession_enabled;   /* 0 = pure damping */
    int enable_exchange;
    int enable_demag;
    int has_external_field;
    double h_ext[3];          /* A/m */
    const uint8_t *active_mask;   /* NULL = all active */
    const uint32_t *region_mask;  /* NULL = no regions */
    const double *exchange_lut;   /* 256*256, NULL = default (A_ii = A) when regions present */
    const double *ms_map;         /* optional per-cell Ms (extension); NULL = uniform ms */
    double max_error, dt_min, dt_max, headroom; /* adaptive (0 -> defaults) */
    /* extension: time-dependent Zeeman  H(t) = h_ext + h_ac * sin(2 pi f t) */
    double h_ac[3];
    double ac_freq;
    int thin_film_2d;         /* demag through the 2-D (nz = 1) spectra, like the GPU runner path */
    /* 1: convolve with the exactly even/odd part of the Newell spectra (real
     * octant mirrored with parity; the form the CUDA library stores) instead of
     * the reference's spectra, which carry rounding noise on the symmetry planes. */
    int symmetric_kernel;
    /* Boundary tiers (native/include/fullmag_fdm.h:151-187): 0 none, 1 T0 (face-link
     * exchange + phi-weighted demag), 2 T1 (ECB exchange + phi-weighted demag).
     * Arrays are [N] doubles, directions in the order xp, xm, yp, ym, zp, zm. */
    int boundary_tier;
    double phi_floor, delta_min;   /* 0 -> 0.05 and 0.1 min(dx, dy, dz) */
    const double *volume_fraction;
    const double *face_link[6];
    const double *delta[6];
    /* sparse demag correction: targets [T], sources [T x S], tensors [T x S x 6]
     * (xx, xy, xz, yy, yz, zz); negative indices are skipped */
    const int32_t *corr_target;
    const int32_t *corr_source;
    const double *corr_tensor;
    uint32_t corr_targets, corr_stencil;
} oracle_desc;

typedef struct {
    double time_seconds, dt_used;
    double e_ex_field;   /* -1/2 mu0 Ms V sum m.H_ex (CPU engine form) */
    double e_ex_pair;    /* forward-pair form (CUDA backend form) */
    double e_demag, e_ext, e_total;
    double max_h_eff, max_h_demag, max_rhs;
    double suggested_next_dt;
    int rejected_attempts;
} oracle_report;

/* Problem lifecycle. m0 is AoS [3N]; it is normalised and masked like
 * ExchangeLlgProblem::new_state (crates/fullmag-engine/src/lib.rs:983-994). */
oracle_problem *oracle_create(const oracle_desc *desc, const double *m0_aos);
void oracle_destroy(oracle_problem *p);
int oracle_step(oracle_problem *p, double dt, oracle_report *out);
void oracle_get_m(const oracle_problem *p, double *out_aos);
void oracle_set_m(oracle_problem *p, const double *m_aos);
double oracle_time(const oracle_problem *p);
void oracle_set_threads(int n);

/* Observables at the current state: fields AoS [3N] (any may be NULL). */
void oracle_observe(oracle_problem *p, double *h_ex, double *h_demag, double *h_ext,
                    double *h_eff, double *rhs, oracle_report *out);

/* Real-space Newell tensor on the (2nx,2ny,2nz) padded grid: 6 arrays of P
 * doubles in order xx, yy, zz, xy, xz, yz (newell.rs:254-519). */
void oracle_newell_kernels(uint32_t nx, uint32_t ny, uint32_t nz,
                           double dx, double dy, double dz, double *out6);
/* Newell spectra, interleaved complex [2P] each, like
 * compute_newell_kernel_spectra (lib.rs:511-540) and the thin-film variant
 * (lib.rs:542-610, P = 4 nx ny). */
void oracle_newell_spectra(uint32_t nx, uint32_t ny, uint32_t nz,
                           double dx, double dy, double dz, int thin_film_2d,
                           double *xx, double *yy, double *zz,
                           double *xy, double *xz, double *yz);
double oracle_newell_f(double x, double y, double z);
double oracle_newell_g(double x, double y, double z);

/* Unnormalised complex FFT of length n (interleaved), sign -1 forward. */
void oracle_fft(double *data, uint64_t n, int inverse);

/* generate_random_unit_vectors (crates/fullmag-plan/src/lib.rs:1928-1957). */
void oracle_random_unit_vectors(uint64_t seed, uint64_t count, double *out_aos);

#ifdef __cplusplus
}
#endif
#endif
