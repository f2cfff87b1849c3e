// backend_impl.hpp — internal entry points shared by api.cu and backend.cu.
#pragma once

#include <vector>

#include "backend.hpp"

namespace fm {

// Asynchronous SoA snapshot owned by the caller until destroyed.
struct Snapshot {
    int device = 0;
    size_t scalar = 8;
    uint64_t cell_count = 0;
    size_t bytes = 0;
    void *dev = nullptr;
    void *host = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ready = nullptr, done = nullptr;
    bool pending = false;
};

bool cuda_ok(Backend &b, cudaError_t e, const char *what);
bool make_line_plan(int L, LinePlan &p);
bool backend_alloc(Backend &b);
bool backend_configure(Backend &b);
bool backend_upload_tables(Backend &b, const std::vector<double> (&spec)[6]);
bool backend_upload_m_f64(Backend &b, const double *m, uint64_t len);
bool backend_upload_m_f32(Backend &b, const float *m, uint64_t len);
bool backend_refresh(Backend &b);
bool backend_step(Backend &b, double dt, fullmag_fdm_step_stats *st);
bool backend_step_n(Backend &b, double dt, uint32_t nsteps, fullmag_fdm_step_stats *st);
bool backend_download_f64(Backend &b, fullmag_fdm_observable o, double *out, uint64_t len);
bool backend_download_f32(Backend &b, fullmag_fdm_observable o, float *out, uint64_t len);
bool backend_preview_f64(Backend &b, fullmag_fdm_observable o, uint32_t pnx, uint32_t pny,
                         uint32_t pnz, uint32_t z_origin, uint32_t z_stride, double *out,
                         uint64_t len);
bool backend_preview_f32(Backend &b, fullmag_fdm_observable o, uint32_t pnx, uint32_t pny,
                         uint32_t pnz, uint32_t z_origin, uint32_t z_stride, float *out,
                         uint64_t len);
bool backend_snapshot_begin(Backend &b, fullmag_fdm_observable obs, Snapshot &s);
void snapshot_free(Snapshot &s);
void backend_free(Backend &b);
bool backend_adjoint_forward(Backend &b, double dt, uint32_t n, uint32_t K, fullmag_fdm_step_stats *st);
bool backend_adjoint_backward(Backend &b, const double *lam_soa, double *gms, double *ghext, double *ghac,
                              double *lam0_soa);
void prof_collect(Backend &b);

}  // namespace fm
