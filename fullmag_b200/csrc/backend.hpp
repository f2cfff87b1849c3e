// backend.hpp — per-handle state of the B200 FDM stepper (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "fullmag_fdm.h"
#include "fullmag_fdm_ext.h"
#include "fft.cuh"

namespace fm {

// Device buffers are typed by the stepper precision (float or double); they
// are kept as void* here and cast in the templated implementation.
struct Backend {
    // ---- configuration (copied from the plan) ----
    int nx = 0, ny = 0, nz = 0;
    long long n = 0;
    double dx = 0, dy = 0, dz = 0;
    double ms = 0, aex = 0, alpha = 0, gamma = 0;
    int precision = FULLMAG_FDM_PRECISION_DOUBLE;
    int integrator = FULLMAG_FDM_INTEGRATOR_HEUN;
    bool precession = true, enable_exchange = true, enable_demag = false, has_ext = false;
    double hext[3] = {0, 0, 0};
    double hac[3] = {0, 0, 0};
    double ac_freq = 0.0;
    bool has_mask = false, has_regions = false, has_ms_map = false;
    std::vector<uint8_t> mask_host;
    std::vector<double> ms_map_host;
    // boundary tiers (fullmag_fdm.h:151-187): tier as given; ex_tier the
    // exchange actually used (1 needs the face links, 2 the distances, as the
    // reference's launch conditions); phi-weighted demag whenever tier > 0
    int boundary_tier = 0, ex_tier = 0;
    double phi_floor = 0.05, delta_min = 0.0;
    std::vector<double> vf_host, face_host, delta_host;  // [N], [6][N], [6][N] (xp, xm, yp, ym, zp, zm)
    std::vector<int32_t> corr_tgt_host, corr_src_host;
    std::vector<double> corr_ten_host;
    uint32_t corr_targets = 0, corr_stencil = 0;
    double *d_vf = nullptr, *d_face = nullptr, *d_delta = nullptr, *d_corr_ten = nullptr;
    int32_t *d_corr_tgt = nullptr, *d_corr_src = nullptr;
    long long active_count = 0;
    double max_error = 1e-5, dt_min = 1e-18, dt_max = 1e-10, headroom = 0.8;

    // ---- dynamic state ----
    uint64_t step_count = 0;
    double time = 0.0;
    bool k1_valid = false;    // k[0] == RHS(m, time)
    bool obs_valid = false;   // hex / heff hold H_ex(m), H_eff(m)

    // ---- device resources ----
    int device = 0;
    cudaStream_t stream = nullptr;
    void *arena = nullptr;
    size_t arena_bytes = 0;
    size_t scalar = 8;        // bytes per state scalar
    void *m = nullptr, *mstage = nullptr, *hd = nullptr;
    void *k[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // adjoint of a Heun trajectory (fullmag_fdm_adjoint_forward / _backward)
    void *adj_mem = nullptr;      // one device block: checkpoints, segment, work buffers
    size_t adj_bytes = 0;
    uint32_t adj_n = 0, adj_K = 0, adj_nck = 0;
    double adj_dt = 0.0;
    std::vector<double> adj_ck_time;   // b.time at each checkpoint
    std::vector<uint64_t> adj_ck_step; // step_count at each checkpoint
    double adj_t_final = 0.0;
    uint64_t adj_step_final = 0;
    bool adj_ready = false;
    bool pred_valid = false;      // mstage holds normalize(m + k1 pred_dt) (Heun's next predictor)
    double pred_dt = 0.0;
    int abm_startup = 0;          // ABM3 start-up steps done (0..3)
    double abm_last_dt = 0.0;     // dt of the last ABM3 step
    void *hex = nullptr, *heff = nullptr;
    void *staging = nullptr;  // device AoS staging (>= 3 n doubles)
    uint8_t *d_mask = nullptr;
    uint32_t *d_region = nullptr;
    double *d_lut = nullptr;
    double *d_msmap = nullptr;

    // ---- demag ----
    bool thin = false;        // 2-D (nz = 1) spectra path
    bool projection = false;  // no spectra supplied: k k^T / k^2 tensor
    int Lx = 0, Ly = 0, Lz = 0, nkx = 0, KZ = 0, KY = 0;
    LinePlan px{}, py{}, pz{};
    void *twx = nullptr, *twy = nullptr, *twz = nullptr;
    void *twxT = nullptr, *twyT = nullptr;  // 4-step twiddle tables (fftreg.cuh fill_tw4 order)
    void *s1 = nullptr, *s2 = nullptr, *spec = nullptr;
    int lines_x = 1, lines_y = 1, kt_z = 1, kb_y = 1;
    size_t smem_xf = 0, smem_yf = 0, smem_z = 0, smem_yc = 0;
    // register-FFT path (power-of-two lengths): block sizes and shared memory
    bool use_reg = false;
    bool force_stockham = false;  // FULLMAG_FDM_FFT=stockham selects the shared-memory FFT
    int thr_x = 0, thr_y = 0, thr_yc = 0;
    bool use_xpipe = false;       // uniform material: cp.async-pipelined x forward
    size_t rsm_xpipe = 0;
    int grid_xpipe = 0, groups_x = 0;
    bool stage_plain = false;     // uniform material: z-marching stage kernel
    bool stage_ring = false;      // ... fed by the cp.async plane ring (FULLMAG_FDM_STAGE=plain: register prefetch)
    bool stage_vec = false;       // stage kernels on 16-byte cell groups (stage_vec.cuh; FULLMAG_FDM_STAGE=ring/plain/cell: off)
    bool stage_vec_mk = false;    // ... in the form with a mask and / or an Ms map
    int stage_zb = 1;             // z planes per thread of that kernel
    bool use_yz = false;          // fused y-z cluster pass (3-D, register FFT)
    bool want_yz = false;         // FULLMAG_FDM_YZ=fused selects it (default: three y/z kernels)
    int yz_P = 0, thr_yz = 0;     // cluster size (ky residues per kx), threads
    int yz_min_P = 1;             // FULLMAG_FDM_YZ_P: smallest cluster size tried
    size_t rsm_yz = 0;
    size_t rsm_x = 0, rsm_y = 0, rsm_yc = 0;
    size_t rsm_xi = 0;            // x inverse: line regions + twiddle table
    bool xi_pair = false;         // x inverse gathers row pairs (ny even)
    bool zdirect = false;         // 3-D, nz <= 8 (FP32: nz <= 16): z convolution by direct summation (k_zd, k_zdw)
    bool use_yzy = false;         // y forward + direct z + y inverse fused per kx plane (k_yzy)
    int yzy_P = 0;                // its cluster size (CTAs per plane)
    int grid_zd = 0;              // its persistent grid (resident blocks x SMs)
    size_t rsm_zd = 0;
    bool use_zdw = false;         // FP32, 8 < nz <= 16: the direct z sum split by output half (k_zdw)
    bool zdw_win = false;         // ... in its window form: z table rows padded to zdw_kyp values
    int zdw_kyp = 0;
    int grid_zdw = 0;
    size_t rsm_zdw = 0;
    // fused x inverse / stage / x forward row pass (Heun, uniform material)
    bool use_row = false;
    int row_rb = 0;               // rows per slab
    size_t rsm_row = 0;
    int s1_state = 0;             // S1 holds: 0 nothing usable, 1 the x transform of Ms m_stage (the predictor)
    bool hd_stale = false;        // hd does not hold H_d(m) (fused Heun steps never write it)

    // ---- reductions ----
    int red_blocks = 0;
    double *partials = nullptr;
    double *d_out = nullptr;      // device address of h_out (mapped pinned memory)
    unsigned *counter = nullptr;  // blocks finished in the reducing stage kernel
    double *h_out = nullptr;  // pinned, NQ doubles

    // ---- per-kernel timing (extension API) ----
    bool profiling = false;
    std::vector<std::string> prof_names;
    std::vector<double> prof_ms;
    std::vector<uint64_t> prof_count;
    std::vector<cudaEvent_t> prof_events;  // pool
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;

    fullmag_fdm_device_info info{};
    bool info_valid = false;
    std::string last_error;
    std::string err_buf;
};

}  // namespace fm
