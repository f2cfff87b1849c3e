// batch.cu — the batched ensemble: many independent uniform-material problems
// of different grids and materials stepped together with Heun, one persistent
// launch per stage for the whole batch (batch.cuh), one CUDA graph per step.
// No counterpart in the reference; exported through include/fullmag_fdm_ext.h.
//
// Per problem: padded lengths are the powers of two >= 2n per axis (any such
// length gives the reference's field, see newell_octant_spectra_padded); a
// film (nz = 1) takes the 3-D pipeline with Lz = 2, the CPU engine's form.
// The autotuner times each stage kernel at persistent grid sizes of 1..16
// blocks per SM on the first call and keeps the fastest.  The z convolution is
// summed directly over the unpadded z (a table of nz planes per problem, built
// from its octant at its Lz), or by z FFTs with FULLMAG_FDM_BATCH_ZCONV=fft.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "fullmag_fdm.h"
#include "fullmag_fdm_ext.h"
#include "newell_host.hpp"

struct fullmag_fdm_batch {
    int device = 0;
    int precision = FULLMAG_FDM_PRECISION_SINGLE;
    cudaStream_t stream = nullptr;
    std::string last_error;
    void *impl = nullptr;  // BatchImpl<T>
    void (*free_impl)(void *) = nullptr;
};

namespace fm {
namespace {

bool batch_ok(fullmag_fdm_batch &B, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    B.last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

int pow2_at_least(int v) {
    int p = 2;
    while (p < v) p *= 2;
    return p;
}

// Padded in-plane length >= v, at least 16: in FP32 the smallest power of two
// or 3 * 2^k in 96..768 (lengths fft4step takes with a radix-3 first level), in
// FP64 a power of two (its batched FFT kernels already use all 255 registers; a
// radix-3 level would spill more).  FULLMAG_FDM_BATCH_PAD=pow2 keeps powers of
// two in FP32 too.  Measured on the 256-problem C4 draw (FP32, one process):
// 4.98 ms per step with powers of two, 4.44 ms with 3 * 2^k from 192 and 4.08 ms
// (another run) from 96.
int batch_length(int v, bool dbl) {
    int L = std::max(16, pow2_at_least(v));
    const char *e = std::getenv("FULLMAG_FDM_BATCH_PAD");
    if (dbl || (e && std::strcmp(e, "pow2") == 0)) return L;
    for (int c : {96, 192, 384, 768})
        if (c >= v && c < L) L = c;
    return L;
}

constexpr int l2_of(int L) { return l2_for(L); }

// kernel kinds tuned and launched per step
enum { KX_FWD = 0, KY_FWD, KZ, KY_INV, KX_INV, KSTAGE, KCOMB, NKINDS };

template <typename T>
struct BatchImpl {
    using C = cx<T>;
    struct Prob {
        fullmag_fdm_batch_problem d{};
        long long n = 0;
        int Lx = 0, Ly = 0, Lz = 0, nkx = 0, KY = 0, KZ = 0;
        size_t off_m = 0, off_ms = 0, off_hd = 0, off_k1 = 0, off_s1 = 0, off_s2 = 0, off_spec = 0;
    };
    std::vector<Prob> probs;
    void *arena = nullptr;
    std::vector<std::pair<int, size_t>> tw_off;   // (L, offset) of shared twiddle tables
    std::vector<std::pair<int, size_t>> tw4_off;  // (L, offset) of the 4-step tables (host_tw4)
    // device argument tables and work lists
    DemagArgs<T> *dA_m = nullptr, *dA_s = nullptr;  // demag of m / of m_stage
    StageArgs<T> *dS_eval = nullptr, *dS_corr = nullptr;
    CombineArgs<T> *dC = nullptr;
    int *d_zb = nullptr;
    int4 *dW[NKINDS] = {};
    int nW[NKINDS] = {};
    size_t smem_x = 0, smem_y = 0;   // for 256-thread x / y blocks (the larger tile)
    // tile shape of the x and y passes, chosen by the autotuner: threads per block
    // (128 or 256), so a block holds tpb / L2 lines of each problem
    int tpb_x = 256, tpb_y = 256;
    int capW[NKINDS] = {};           // work-list capacity (the 128-thread lists are the longest)
    int grid[NKINDS] = {};
    bool tuned = false, k1_valid = false;
    // z convolution: direct sums over the unpadded z with each problem's table
    // (octant_to_z_direct at its Lz), or FULLMAG_FDM_BATCH_ZCONV=fft: z FFTs
    bool zdirect = true;
    int zmax = 1;                    // the largest nz of the batch
    double args_dt = -1.0;
    double time = 0.0;
    uint64_t steps = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<DemagArgs<T>> hA_m, hA_s;
    std::vector<StageArgs<T>> hS_eval, hS_corr;
    std::vector<CombineArgs<T>> hC;

    ~BatchImpl() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (arena) cudaFree(arena);
    }

    char *base() { return (char *)arena; }

    bool create(fullmag_fdm_batch &B, const fullmag_fdm_batch_problem *ps, uint32_t count) {
        const size_t s = sizeof(T), cs = 2 * sizeof(T);
        {
            const char *z = std::getenv("FULLMAG_FDM_BATCH_ZCONV");
            zdirect = !(z && std::strcmp(z, "fft") == 0);
        }
        size_t off = 0;
        auto take = [&](size_t bytes) {
            const size_t o = off;
            off += (bytes + 255) / 256 * 256;
            return o;
        };
        probs.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            Prob &p = probs[i];
            p.d = ps[i];
            const auto &d = p.d;
            if (d.nx == 0 || d.ny == 0 || d.nz == 0) { B.last_error = "problem " + std::to_string(i) + ": empty grid"; return false; }
            if (!(d.dx > 0 && d.dy > 0 && d.dz > 0)) { B.last_error = "problem " + std::to_string(i) + ": cell sizes must be positive"; return false; }
            if (!(d.saturation_magnetisation > 0)) { B.last_error = "problem " + std::to_string(i) + ": saturation_magnetisation must be positive"; return false; }
            if (!d.initial_magnetization_xyz) { B.last_error = "problem " + std::to_string(i) + ": initial_magnetization_xyz is null"; return false; }
            p.n = (long long)d.nx * d.ny * d.nz;
            zmax = std::max(zmax, (int)d.nz);
            // in-plane lengths of at least 16 (the smallest the batched x / y kernels take)
            p.Lx = batch_length(2 * (int)d.nx, sizeof(T) == 8);
            p.Ly = batch_length(2 * (int)d.ny, sizeof(T) == 8);
            p.Lz = pow2_at_least(2 * (int)d.nz);
            if (p.Lx > 1024 || p.Ly > 1024 || p.Lz > 16) {
                B.last_error = "problem " + std::to_string(i) + ": grid too large for the batch (nx, ny <= 512, nz <= 8)";
                return false;
            }
            p.nkx = p.Lx / 2 + 1;
            p.KY = p.Ly / 2 + 1;
            p.KZ = p.Lz / 2 + 1;
            const size_t v = 3 * (size_t)p.n * s;
            p.off_m = take(v);
            p.off_ms = take(v);
            p.off_hd = take(v);
            p.off_k1 = take(v);
            p.off_s1 = take((size_t)3 * d.nz * p.nkx * d.ny * cs);
            p.off_s2 = take((size_t)3 * d.nz * p.nkx * p.Ly * cs);
            p.off_spec = take((size_t)6 * p.KZ * p.nkx * p.KY * s);
            const int Ls[3] = {p.Lx, p.Ly, p.Lz};
            for (int L : Ls) {
                bool have = false;
                for (auto &t : tw_off) have = have || t.first == L;
                if (!have) {
                    tw_off.push_back({L, take((size_t)L * cs)});
                    tw4_off.push_back({L, take((size_t)L * cs)});
                }
            }
        }
        // FP64 sums of nz > 4 hold more registers than a thread has: z FFTs there
        if (sizeof(T) == 8 && zmax > 4) zdirect = false;
        // work lists (x and y: for 128-thread blocks, the longest; rebuilt per tile shape)
        std::vector<int4> W[NKINDS];
        xy_lists(128, 128, W);
        for (uint32_t i = 0; i < count; ++i) {
            const Prob &p = probs[i];
            const int nx = p.d.nx, ny = p.d.ny;
            const int P = (!zdirect && p.Lz > 8) ? 2 : 1;
            const long long tasks = (long long)p.nkx * p.Ly * P;
            for (long long ch = 0; ch < (tasks + 127) / 128; ++ch) W[KZ].push_back(make_int4((int)i, (int)ch, 0, 0));
            for (int bz = 0; bz < 1; ++bz)
                for (int by = 0; by < (ny + kStagePlainBY - 1) / kStagePlainBY; ++by)
                    for (int bx = 0; bx < (nx + 31) / 32; ++bx) W[KSTAGE].push_back(make_int4((int)i, bx, by, bz));
            for (long long ch = 0; ch < (p.n + 255) / 256; ++ch) W[KCOMB].push_back(make_int4((int)i, (int)ch, 0, 0));
        }
        const size_t off_tables = take(0);
        size_t o_A_m = take(count * sizeof(DemagArgs<T>)), o_A_s = take(count * sizeof(DemagArgs<T>));
        size_t o_S_e = take(count * sizeof(StageArgs<T>)), o_S_c = take(count * sizeof(StageArgs<T>));
        size_t o_C = take(count * sizeof(CombineArgs<T>)), o_zb = take(count * sizeof(int));
        size_t o_W[NKINDS];
        for (int k = 0; k < NKINDS; ++k) {
            nW[k] = capW[k] = (int)W[k].size();
            o_W[k] = take(W[k].size() * sizeof(int4));
        }
        (void)off_tables;
        if (!batch_ok(B, cudaMalloc(&arena, off), "cudaMalloc(batch arena)")) return false;
        // legacy-stream memset: ordered before the synchronous uploads below
        if (!batch_ok(B, cudaMemset(arena, 0, off), "batch memset")) return false;
        dA_m = (DemagArgs<T> *)(base() + o_A_m);
        dA_s = (DemagArgs<T> *)(base() + o_A_s);
        dS_eval = (StageArgs<T> *)(base() + o_S_e);
        dS_corr = (StageArgs<T> *)(base() + o_S_c);
        dC = (CombineArgs<T> *)(base() + o_C);
        d_zb = (int *)(base() + o_zb);
        for (int k = 0; k < NKINDS; ++k) {
            dW[k] = (int4 *)(base() + o_W[k]);
            if (nW[k] && !batch_ok(B, cudaMemcpy(dW[k], W[k].data(), W[k].size() * sizeof(int4), cudaMemcpyHostToDevice), "upload work list"))
                return false;
        }
        // twiddles exp(-2 pi i k / L), computed in FP64
        for (auto &t : tw_off) {
            std::vector<C> tw(t.first);
            for (int k = 0; k < t.first; ++k) {
                const double a = 2.0 * kPi * (double)k / (double)t.first;
                tw[k] = mk<T>((T)std::cos(a), (T)(-std::sin(a)));
            }
            if (!batch_ok(B, cudaMemcpy(base() + t.second, tw.data(), tw.size() * sizeof(C), cudaMemcpyHostToDevice), "upload twiddles"))
                return false;
        }
        for (auto &t : tw4_off) {
            const std::vector<C> tw = host_tw4<T>(t.first);
            if (!batch_ok(B, cudaMemcpy(base() + t.second, tw.data(), tw.size() * sizeof(C), cudaMemcpyHostToDevice), "upload 4-step twiddles"))
                return false;
        }
        // per problem: octant spectra, m0, shared-memory needs
        std::vector<int> zb(count);
        for (uint32_t i = 0; i < count; ++i) {
            Prob &p = probs[i];
            const auto &d = p.d;
            std::vector<double> spec[6], zt[6];
            newell_octant_spectra_padded(d.nx, d.ny, d.nz, d.dx, d.dy, d.dz, false, p.Lx, p.Ly, p.Lz, spec);
            // the direct table has nz planes per component (nz <= Lz / 2 < KZ: it
            // fits the octant's allocation)
            if (zdirect) octant_to_z_direct(p.nkx, p.KY, (int)d.nz, spec, zt, p.Lz / 2);
            const auto &src = zdirect ? zt : spec;
            const size_t plane = (size_t)(zdirect ? (int)d.nz : p.KZ) * p.nkx * p.KY;
            std::vector<T> host(6 * plane);
            for (int c = 0; c < 6; ++c)
                for (size_t o = 0; o < plane; ++o) host[c * plane + o] = (T)src[c][o];
            if (!batch_ok(B, cudaMemcpy(base() + p.off_spec, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "upload spectra"))
                return false;
            std::vector<T> m(3 * (size_t)p.n);
            for (long long c = 0; c < p.n; ++c)
                for (int k = 0; k < 3; ++k) m[k * p.n + c] = (T)d.initial_magnetization_xyz[3 * c + k];
            if (!batch_ok(B, cudaMemcpy(base() + p.off_m, m.data(), m.size() * sizeof(T), cudaMemcpyHostToDevice), "upload m0"))
                return false;
            zb[i] = (int)d.nz;
            const int lx2 = l2_of(p.Lx), ly2 = l2_of(p.Ly);
            const size_t TEx = (size_t)std::max(lx2 == 1 ? 0 : (p.Lx / lx2) * (lx2 + 1), p.Lx) + 1;
            smem_x = std::max(smem_x, ((size_t)(256 / lx2) * TEx) * cs);
            const size_t TEy = ly2 == 1 ? 0 : (size_t)(p.Ly / ly2) * (ly2 + 1);
            smem_y = std::max(smem_y, ((size_t)(256 / ly2) * TEy) * cs);
        }
        if (!batch_ok(B, cudaMemcpy(d_zb, zb.data(), count * sizeof(int), cudaMemcpyHostToDevice), "upload zb")) return false;
        if (smem_x > 227 * 1024 || smem_y > 227 * 1024) { B.last_error = "batch FFT tiles exceed shared memory"; return false; }
        bool ok = batch_ok(B, cudaFuncSetAttribute(k_batch_x<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x), "attr x") &&
                  batch_ok(B, cudaFuncSetAttribute(k_batch_x<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_x), "attr x") &&
                  batch_ok(B, cudaFuncSetAttribute(k_batch_y<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_y), "attr y") &&
                  batch_ok(B, cudaFuncSetAttribute(k_batch_y<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_y), "attr y");
        if (!ok) return false;
        return set_tiles(B, 256, 256) && upload_args(B, 1e-13);
    }

    // x / y work lists for tx- and ty-thread blocks: x item (problem, row block of
    // 2 tx / L2 rows, z, component), y item (problem, block of ty / L2 lines)
    void xy_lists(int tx, int ty, std::vector<int4> (&W)[NKINDS]) const {
        for (int k : {KX_FWD, KX_INV, KY_FWD, KY_INV}) W[k].clear();
        for (size_t i = 0; i < probs.size(); ++i) {
            const Prob &p = probs[i];
            const int ny = p.d.ny, nz = p.d.nz;
            const int RB = 2 * std::max(1, tx / l2_of(p.Lx));
            for (int c = 0; c < 3; ++c)
                for (int z = 0; z < nz; ++z)
                    for (int bx = 0; bx < (ny + RB - 1) / RB; ++bx) {
                        W[KX_FWD].push_back(make_int4((int)i, bx, z, c));
                        W[KX_INV].push_back(make_int4((int)i, bx, z, c));
                    }
            const int ly = std::max(1, ty / l2_of(p.Ly));
            const long long lines = 3LL * nz * p.nkx;
            for (long long bx = 0; bx < (lines + ly - 1) / ly; ++bx) {
                W[KY_FWD].push_back(make_int4((int)i, (int)bx, 0, 0));
                W[KY_INV].push_back(make_int4((int)i, (int)bx, 0, 0));
            }
        }
    }

    // Switch the x / y tile shape: work lists and the lines per block in the
    // argument tables (uploaded with the next upload_args).
    bool set_tiles(fullmag_fdm_batch &B, int tx, int ty) {
        std::vector<int4> W[NKINDS];
        xy_lists(tx, ty, W);
        for (int k : {KX_FWD, KX_INV, KY_FWD, KY_INV}) {
            if ((int)W[k].size() > capW[k]) { B.last_error = "batch work list overflow"; return false; }
            nW[k] = (int)W[k].size();
            if (nW[k] && !batch_ok(B, cudaMemcpy(dW[k], W[k].data(), W[k].size() * sizeof(int4), cudaMemcpyHostToDevice), "upload work list"))
                return false;
        }
        tpb_x = tx;
        tpb_y = ty;
        return true;
    }

    const C *tw(int L) {
        for (auto &t : tw_off)
            if (t.first == L) return (const C *)(base() + t.second);
        return nullptr;
    }

    const C *tw4(int L) {
        for (auto &t : tw4_off)
            if (t.first == L) return (const C *)(base() + t.second);
        return nullptr;
    }

    // argument tables for step size dt (the predictor and corrector use it)
    bool upload_args(fullmag_fdm_batch &B, double dt) {
        const size_t P = probs.size();
        hA_m.assign(P, DemagArgs<T>{});
        hA_s.assign(P, DemagArgs<T>{});
        hS_eval.assign(P, StageArgs<T>{});
        hS_corr.assign(P, StageArgs<T>{});
        hC.assign(P, CombineArgs<T>{});
        for (size_t i = 0; i < P; ++i) {
            Prob &p = probs[i];
            const auto &d = p.d;
            T *m = (T *)(base() + p.off_m), *ms = (T *)(base() + p.off_ms);
            T *hd = (T *)(base() + p.off_hd), *k1 = (T *)(base() + p.off_k1);
            DemagArgs<T> a{};
            a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.n = p.n;
            a.Lx = p.Lx; a.Ly = p.Ly; a.Lz = p.Lz; a.nkx = p.nkx; a.KZ = p.KZ; a.KY = p.KY;
            a.twx = tw(p.Lx); a.twy = tw(p.Ly); a.twz = tw(p.Lz);
            a.twxT = tw4(p.Lx); a.twyT = tw4(p.Ly);
            a.s1 = (C *)(base() + p.off_s1);
            a.s2 = (C *)(base() + p.off_s2);
            a.spec = (const T *)(base() + p.off_spec);
            a.ms = d.saturation_magnetisation;
            a.hd = hd;
            a.norm = 1.0 / ((double)p.Lx * (double)p.Ly * (double)p.Lz);
            a.lines_x = std::max(1, tpb_x / l2_of(p.Lx));
            a.lines_y = std::max(1, tpb_y / l2_of(p.Ly));
            a.m = m;
            hA_m[i] = a;
            a.m = ms;
            hA_s[i] = a;
            StageArgs<T> s{};
            s.nx = d.nx; s.ny = d.ny; s.nz = d.nz; s.n = p.n;
            s.idx2 = (T)(1.0 / (d.dx * d.dx)); s.idy2 = (T)(1.0 / (d.dy * d.dy)); s.idz2 = (T)(1.0 / (d.dz * d.dz));
            s.dinv[0] = 1.0 / (d.dx * d.dx); s.dinv[1] = 1.0 / (d.dy * d.dy); s.dinv[2] = 1.0 / (d.dz * d.dz);
            s.aex = d.exchange_stiffness; s.ms = d.saturation_magnetisation;
            s.ex_pref = 2.0 * d.exchange_stiffness / (kMu0 * d.saturation_magnetisation);
            s.enable_exchange = 1; s.enable_demag = 1; s.has_ext = 1;
            for (int c = 0; c < 3; ++c) s.hext[c] = d.external_field_am[c];
            s.gamma_bar = d.gyromagnetic_ratio / (1.0 + d.damping * d.damping);
            s.alpha = d.damping;
            s.precession = 1;
            s.vol = d.dx * d.dy * d.dz;
            s.hd = hd;
            s.m = m;
            s.kout = k1;
            s.pred_out = ms;  // the next step's predictor, written by the RHS kernel
            s.pred_dt = dt;
            hS_eval[i] = s;
            s.pred_out = nullptr;
            s.m = ms;
            s.kout = nullptr;
            s.m0 = m;
            s.k1 = k1;
            s.half_dt = 0.5 * dt;
            hS_corr[i] = s;
            CombineArgs<T> cb{};
            cb.n = p.n; cb.m0 = m; cb.k[0] = k1; cb.c[0] = dt; cb.dt = dt; cb.form = 0; cb.out = ms;
            hC[i] = cb;
        }
        args_dt = dt;
        return batch_ok(B, cudaMemcpy(dA_m, hA_m.data(), P * sizeof(DemagArgs<T>), cudaMemcpyHostToDevice), "upload args") &&
               batch_ok(B, cudaMemcpy(dA_s, hA_s.data(), P * sizeof(DemagArgs<T>), cudaMemcpyHostToDevice), "upload args") &&
               batch_ok(B, cudaMemcpy(dS_eval, hS_eval.data(), P * sizeof(StageArgs<T>), cudaMemcpyHostToDevice), "upload args") &&
               batch_ok(B, cudaMemcpy(dS_corr, hS_corr.data(), P * sizeof(StageArgs<T>), cudaMemcpyHostToDevice), "upload args") &&
               batch_ok(B, cudaMemcpy(dC, hC.data(), P * sizeof(CombineArgs<T>), cudaMemcpyHostToDevice), "upload args");
    }

    int g(int kind, int G) const { return std::max(1, std::min(G, nW[kind])); }

    void launch(cudaStream_t st, int kind, bool staged, int G) {
        const DemagArgs<T> *A = staged ? dA_s : dA_m;
        switch (kind) {
            case KX_FWD: k_batch_x<T, false><<<g(kind, G), tpb_x, smem_x * tpb_x / 256, st>>>(A, dW[kind], nW[kind]); break;
            case KY_FWD: k_batch_y<T, false><<<g(kind, G), tpb_y, smem_y * tpb_y / 256, st>>>(A, dW[kind], nW[kind]); break;
            case KZ:
                if (zdirect && zmax <= 4) k_batch_z<T, true, 4><<<g(kind, G), 128, 0, st>>>(A, dW[kind], nW[kind]);
                else if (zdirect) {
                    if constexpr (sizeof(T) == 4) k_batch_z<T, true, 8><<<g(kind, G), 128, 0, st>>>(A, dW[kind], nW[kind]);
                } else k_batch_z<T, false><<<g(kind, G), 128, 0, st>>>(A, dW[kind], nW[kind]);
                break;
            case KY_INV: k_batch_y<T, true><<<g(kind, G), tpb_y, smem_y * tpb_y / 256, st>>>(A, dW[kind], nW[kind]); break;
            case KX_INV: k_batch_x<T, true><<<g(kind, G), tpb_x, smem_x * tpb_x / 256, st>>>(A, dW[kind], nW[kind]); break;
            case KSTAGE:
                if (staged)
                    k_batch_stage<T, MODE_HEUN_CORR><<<g(kind, G), dim3(32, kStagePlainBY), 0, st>>>(dS_corr, d_zb, dW[kind], nW[kind]);
                else
                    k_batch_stage<T, MODE_EVAL><<<g(kind, G), dim3(32, kStagePlainBY), 0, st>>>(dS_eval, d_zb, dW[kind], nW[kind]);
                break;
            case KCOMB: k_batch_combine<T><<<g(kind, G), 256, 0, st>>>(dC, dW[kind], nW[kind]); break;
        }
    }

    void demag(cudaStream_t st, bool staged) {
        const int kinds[5] = {KX_FWD, KY_FWD, KZ, KY_INV, KX_INV};
        for (int k : kinds) launch(st, k, staged, grid[k]);
    }

    // Autotuner: for the x and y passes the tile shape (128- or 256-thread blocks,
    // so tpb / L2 lines of a problem per block) together with the persistent grid
    // size; for the other kernels the grid size; grid sizes from {1, 2, 4, 8, 16}
    // blocks per SM; by CUDA-event time of two launches each (after one warm-up).
    // The stage kernel is tuned in its RHS form, which writes only k1.
    bool tune(fullmag_fdm_batch &B) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.device);
        cudaEvent_t e0, e1;
        if (!batch_ok(B, cudaEventCreate(&e0), "event") || !batch_ok(B, cudaEventCreate(&e1), "event")) return false;
        auto tune_kind = [&](int k, float &best, int &best_g) -> bool {
            best = 1e30f;
            best_g = sms;
            const int pers[5] = {1, 2, 4, 8, 16};
            for (int per : pers) {
                const int G = sms * per;
                launch(B.stream, k, false, G);
                cudaEventRecord(e0, B.stream);
                launch(B.stream, k, false, G);
                launch(B.stream, k, false, G);
                cudaEventRecord(e1, B.stream);
                if (!batch_ok(B, cudaEventSynchronize(e1), "autotune")) return false;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; best_g = G; }
                if (G >= nW[k]) break;
            }
            return true;
        };
        int tx = 256, ty = 256, gx[2] = {sms, sms}, gy[2] = {sms, sms};
        float bx = 1e30f, by = 1e30f;
        for (int t : {256, 128}) {
            if (!set_tiles(B, t, t) || !upload_args(B, args_dt)) return false;
            float f[4];
            int g4[4];
            const int kinds[4] = {KX_FWD, KX_INV, KY_FWD, KY_INV};
            for (int i = 0; i < 4; ++i)
                if (!tune_kind(kinds[i], f[i], g4[i])) return false;
            if (f[0] + f[1] < bx) { bx = f[0] + f[1]; tx = t; gx[0] = g4[0]; gx[1] = g4[1]; }
            if (f[2] + f[3] < by) { by = f[2] + f[3]; ty = t; gy[0] = g4[2]; gy[1] = g4[3]; }
        }
        if (!set_tiles(B, tx, ty) || !upload_args(B, args_dt)) return false;
        grid[KX_FWD] = gx[0]; grid[KX_INV] = gx[1];
        grid[KY_FWD] = gy[0]; grid[KY_INV] = gy[1];
        for (int k : {KZ, KSTAGE, KCOMB}) {
            float f;
            if (!tune_kind(k, f, grid[k])) return false;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        tuned = true;
        return batch_ok(B, cudaGetLastError(), "autotune launches");
    }

    // one Heun step: demag(m_p), corrector, demag(m), RHS (next k1 and the next
    // predictor m_p; the first one comes from the initial RHS launch)
    void step_launches(cudaStream_t st) {
        demag(st, true);
        launch(st, KSTAGE, true, grid[KSTAGE]);
        demag(st, false);
        launch(st, KSTAGE, false, grid[KSTAGE]);
    }

    bool step_n(fullmag_fdm_batch &B, double dt, uint32_t n) {
        if (dt != args_dt) {
            if (!upload_args(B, dt)) return false;
            if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
            if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
            k1_valid = false;  // the stored predictor used the previous dt
        }
        if (!tuned && !tune(B)) return false;
        if (!k1_valid) {
            demag(B.stream, false);
            launch(B.stream, KSTAGE, false, grid[KSTAGE]);
            if (!batch_ok(B, cudaGetLastError(), "initial RHS")) return false;
            k1_valid = true;
        }
        if (!exec) {
            if (!batch_ok(B, cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return false;
            step_launches(B.stream);
            if (!batch_ok(B, cudaStreamEndCapture(B.stream, &graph), "end capture")) return false;
            if (!batch_ok(B, cudaGraphInstantiate(&exec, graph, 0), "graph instantiate")) return false;
        }
        for (uint32_t s = 0; s < n; ++s)
            if (!batch_ok(B, cudaGraphLaunch(exec, B.stream), "graph launch")) return false;
        time += dt * n;
        steps += n;
        return batch_ok(B, cudaStreamSynchronize(B.stream), "batch step sync");
    }

    // One step with every launch issued directly and timed by kind.
    bool profile_step(fullmag_fdm_batch &B, double dt, float *ms) {
        if (dt != args_dt) {
            if (!upload_args(B, dt)) return false;
            if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
            if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
            k1_valid = false;
        }
        if (!tuned && !tune(B)) return false;
        if (!k1_valid) {
            demag(B.stream, false);
            launch(B.stream, KSTAGE, false, grid[KSTAGE]);
            if (!batch_ok(B, cudaGetLastError(), "initial RHS")) return false;
            k1_valid = true;
        }
        const int kinds[5] = {KX_FWD, KY_FWD, KZ, KY_INV, KX_INV};
        std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev;
        auto timed = [&](int kind, bool staged) {
            cudaEvent_t e0, e1;
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, B.stream);
            launch(B.stream, kind, staged, grid[kind]);
            cudaEventRecord(e1, B.stream);
            ev.push_back({kind, {e0, e1}});
        };
        for (bool staged : {true, false}) {
            for (int k : kinds) timed(k, staged);
            timed(KSTAGE, staged);
        }
        bool ok = batch_ok(B, cudaGetLastError(), "profiled step") && batch_ok(B, cudaStreamSynchronize(B.stream), "profiled step sync");
        for (int k = 0; k < NKINDS; ++k) ms[k] = 0.f;
        for (auto &e : ev) {
            float t = 0.f;
            if (ok) cudaEventElapsedTime(&t, e.second.first, e.second.second);
            ms[e.first] += t;
            cudaEventDestroy(e.second.first);
            cudaEventDestroy(e.second.second);
        }
        time += dt;
        steps += 1;
        return ok;
    }

    bool copy_m(fullmag_fdm_batch &B, uint32_t index, double *out) {
        const Prob &p = probs[index];
        std::vector<T> h(3 * (size_t)p.n);
        if (!batch_ok(B, cudaMemcpyAsync(h.data(), base() + p.off_m, h.size() * sizeof(T), cudaMemcpyDeviceToHost, B.stream), "copy m") ||
            !batch_ok(B, cudaStreamSynchronize(B.stream), "copy m sync"))
            return false;
        for (long long c = 0; c < p.n; ++c)
            for (int k = 0; k < 3; ++k) out[3 * c + k] = (double)h[k * p.n + c];
        return true;
    }
};

// This translation unit's copy of the W_64 table (fftreg.cuh).
bool batch_upload_tw64(fullmag_fdm_batch &B) {
    double2 d[64];
    float2 f[64];
    for (int k = 0; k < 64; ++k) {
        const double a = 2.0 * kPi * (double)k / 64.0;
        d[k] = make_double2(std::cos(a), -std::sin(a));
        f[k] = make_float2((float)d[k].x, (float)d[k].y);
    }
    double2 d3[192];
    float2 f3[192];
    host_tw192(d3, f3);
    // legacy-stream uploads from pageable memory, then a device synchronisation:
    // the batch's stream is non-blocking
    return batch_ok(B, cudaMemcpyToSymbol(c_tw64d, d, sizeof(d)), "twiddle64 d (batch)") &&
           batch_ok(B, cudaMemcpyToSymbol(c_tw64f, f, sizeof(f)), "twiddle64 f (batch)") &&
           batch_ok(B, cudaMemcpyToSymbol(c_tw192d, d3, sizeof(d3)), "twiddle192 d (batch)") &&
           batch_ok(B, cudaMemcpyToSymbol(c_tw192f, f3, sizeof(f3)), "twiddle192 f (batch)") &&
           batch_ok(B, cudaDeviceSynchronize(), "twiddle (batch) sync");
}

template <typename T>
void free_impl(void *p) { delete (BatchImpl<T> *)p; }

}  // namespace
}  // namespace fm

using fm::BatchImpl;

extern "C" {

fullmag_fdm_batch *fullmag_fdm_batch_create(const fullmag_fdm_batch_problem *problems, uint32_t count,
                                            fullmag_fdm_precision precision) {
    auto *B = new (std::nothrow) fullmag_fdm_batch();
    if (!B) return nullptr;
    if (!problems || count == 0) { B->last_error = "no problems"; return B; }
    if (precision != FULLMAG_FDM_PRECISION_SINGLE && precision != FULLMAG_FDM_PRECISION_DOUBLE) {
        B->last_error = "unknown precision";
        return B;
    }
    B->precision = precision;
    const char *s = std::getenv("FULLMAG_FDM_GPU_INDEX");
    if (!s || !*s) s = std::getenv("FULLMAG_CUDA_DEVICE_INDEX");
    if (s && *s) {
        if (!fm::batch_ok(*B, cudaSetDevice(std::atoi(s)), "cudaSetDevice")) return B;
    }
    if (!fm::batch_ok(*B, cudaGetDevice(&B->device), "cudaGetDevice")) return B;
    if (!fm::batch_ok(*B, cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking), "cudaStreamCreate")) return B;
    if (!fm::batch_upload_tw64(*B)) return B;
    bool ok;
    if (precision == FULLMAG_FDM_PRECISION_DOUBLE) {
        auto *impl = new BatchImpl<double>();
        B->impl = impl;
        B->free_impl = fm::free_impl<double>;
        ok = impl->create(*B, problems, count);
    } else {
        auto *impl = new BatchImpl<float>();
        B->impl = impl;
        B->free_impl = fm::free_impl<float>;
        ok = impl->create(*B, problems, count);
    }
    if (ok) fm::batch_ok(*B, cudaStreamSynchronize(B->stream), "batch create sync");
    return B;
}

int fullmag_fdm_batch_step_n(fullmag_fdm_batch *B, double dt, uint32_t n_steps) {
    if (!B || n_steps == 0) return FULLMAG_FDM_ERR_INVALID;
    if (!B->impl || !B->last_error.empty()) {
        if (B->last_error.empty()) B->last_error = "batch was not created successfully";
        return FULLMAG_FDM_ERR_INVALID;
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) { B->last_error = "dt must be positive and finite"; return FULLMAG_FDM_ERR_INVALID; }
    if (!fm::batch_ok(*B, cudaSetDevice(B->device), "cudaSetDevice")) return FULLMAG_FDM_ERR_CUDA;
    const bool ok = B->precision == FULLMAG_FDM_PRECISION_DOUBLE ? ((BatchImpl<double> *)B->impl)->step_n(*B, dt, n_steps)
                                                                 : ((BatchImpl<float> *)B->impl)->step_n(*B, dt, n_steps);
    return ok ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_batch_copy_m(fullmag_fdm_batch *B, uint32_t index, double *out_xyz, uint64_t len) {
    if (!B || !out_xyz) return FULLMAG_FDM_ERR_INVALID;
    if (!B->impl || !B->last_error.empty()) {
        if (B->last_error.empty()) B->last_error = "batch was not created successfully";
        return FULLMAG_FDM_ERR_INVALID;
    }
    const auto size_of = [&](uint32_t i) -> long long {
        return B->precision == FULLMAG_FDM_PRECISION_DOUBLE ? (i < ((BatchImpl<double> *)B->impl)->probs.size() ? ((BatchImpl<double> *)B->impl)->probs[i].n : -1)
                                                            : (i < ((BatchImpl<float> *)B->impl)->probs.size() ? ((BatchImpl<float> *)B->impl)->probs[i].n : -1);
    };
    const long long n = size_of(index);
    if (n < 0) { B->last_error = "problem index out of range"; return FULLMAG_FDM_ERR_INVALID; }
    if (len != 3 * (uint64_t)n) { B->last_error = "out_len mismatch"; return FULLMAG_FDM_ERR_INVALID; }
    if (!fm::batch_ok(*B, cudaSetDevice(B->device), "cudaSetDevice")) return FULLMAG_FDM_ERR_CUDA;
    const bool ok = B->precision == FULLMAG_FDM_PRECISION_DOUBLE ? ((BatchImpl<double> *)B->impl)->copy_m(*B, index, out_xyz)
                                                                 : ((BatchImpl<float> *)B->impl)->copy_m(*B, index, out_xyz);
    return ok ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

int fullmag_fdm_batch_tuning(const fullmag_fdm_batch *B, int32_t *grid_sizes, uint32_t len) {
    if (!B || !grid_sizes || len < fm::NKINDS || !B->impl) return FULLMAG_FDM_ERR_INVALID;
    const bool dbl = B->precision == FULLMAG_FDM_PRECISION_DOUBLE;
    const int *g = dbl ? ((BatchImpl<double> *)B->impl)->grid : ((BatchImpl<float> *)B->impl)->grid;
    for (int k = 0; k < fm::NKINDS; ++k) grid_sizes[k] = g[k];
    if (len >= fm::NKINDS + 2) {  // the tile shape: threads per block of the x and y passes
        grid_sizes[fm::NKINDS] = dbl ? ((BatchImpl<double> *)B->impl)->tpb_x : ((BatchImpl<float> *)B->impl)->tpb_x;
        grid_sizes[fm::NKINDS + 1] = dbl ? ((BatchImpl<double> *)B->impl)->tpb_y : ((BatchImpl<float> *)B->impl)->tpb_y;
    }
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_batch_get_stream(const fullmag_fdm_batch *B, void **stream_out) {
    if (!B || !stream_out) return FULLMAG_FDM_ERR_INVALID;
    *stream_out = (void *)B->stream;
    return FULLMAG_FDM_OK;
}

int fullmag_fdm_batch_profile_step(fullmag_fdm_batch *B, double dt, float *ms_per_kind, uint32_t len) {
    if (!B || !ms_per_kind || len < fm::NKINDS) return FULLMAG_FDM_ERR_INVALID;
    if (!B->impl || !B->last_error.empty()) {
        if (B->last_error.empty()) B->last_error = "batch was not created successfully";
        return FULLMAG_FDM_ERR_INVALID;
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) { B->last_error = "dt must be positive and finite"; return FULLMAG_FDM_ERR_INVALID; }
    if (!fm::batch_ok(*B, cudaSetDevice(B->device), "cudaSetDevice")) return FULLMAG_FDM_ERR_CUDA;
    const bool ok = B->precision == FULLMAG_FDM_PRECISION_DOUBLE
                        ? ((BatchImpl<double> *)B->impl)->profile_step(*B, dt, ms_per_kind)
                        : ((BatchImpl<float> *)B->impl)->profile_step(*B, dt, ms_per_kind);
    return ok ? FULLMAG_FDM_OK : FULLMAG_FDM_ERR_CUDA;
}

const char *fullmag_fdm_batch_last_error(const fullmag_fdm_batch *B) {
    if (!B) return "null handle";
    return B->last_error.empty() ? nullptr : B->last_error.c_str();
}

void fullmag_fdm_batch_destroy(fullmag_fdm_batch *B) {
    if (!B) return;
    cudaSetDevice(B->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (B->impl && B->free_impl) B->free_impl(B->impl);
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
}

}  // extern "C"
