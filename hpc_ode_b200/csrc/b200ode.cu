// b200ode: kernels and C ABI (include/b200ode.h).
//
// Execution model (sm_100a):
//   * one warp integrates one cell with the CVODE-semantics BDF of bdf_warp.cuh;
//   * persistent form: a grid sized to the SM count x resident CTAs, every warp
//     pulls cell indices from a device work queue (one 64-bit atomic per cell)
//     and refills itself until the queue is empty, so cells of very different
//     stiffness (a few vs hundreds of steps) never leave lanes idle;
//   * one-launch-per-step form (the plain FP64 comparison form): every launch
//     advances each unfinished cell by one BDF step, state kept in HBM between
//     launches (k_bdf with per-cell records);
//   * state in HBM is structure-of-arrays with the cell index innermost.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/b200ode.h"
#include "b200ode_internal.h"
#include "bdf_warp.cuh"
#include "mech/gri30_mech.h"
#include "mech/h2o2_mech.h"
#include "mech/nDodecane_Reitz_mech.h"
#include "mech/h2_li_2004_mech.h"
#include "mech/ESTiMatE-Mech_04042022_mech.h"

using namespace b200;

namespace {

thread_local std::string g_last_error;
std::mutex g_tables_mu;
std::map<std::pair<int, int>, unsigned char*> g_tables;   // (device, mechanism) -> tables

// Host-side NVTX range for profilers (Nsight Systems): one per entry point and
// per phase it enqueues.  Header-only NVTX: no cost when no tool is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

b200ode_status fail(b200ode_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(B200ODE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GEN_TABLES(tag, PFX)                                                                         \
    GenTables{#tag, PFX##_NSP, PFX##_NRXN, PFX##_MAXP, PFX##_NTB, PFX##_NU_DEN, PFX##_NPLOGLEV,       \
              PFX##_NPLOGTERM, tag##_species_names, tag##_mw,                                         \
              tag##_tmid, tag##_nasa_lo, tag##_nasa_hi, tag##_rxn_type, tag##_rxn_rev, tag##_rxn_A,   \
              tag##_rxn_logA, tag##_rxn_b, tag##_rxn_EaR, tag##_rxn_A0, tag##_rxn_logA0, tag##_rxn_b0, \
              tag##_rxn_EaR0, tag##_rxn_troe, tag##_rxn_troe_T2, tag##_rxn_reac_sp,                   \
              tag##_rxn_reac_nu, tag##_rxn_prod_sp, tag##_rxn_prod_nu, tag##_rxn_tb_off, tag##_tb_sp,  \
              tag##_tb_alpha, tag##_plog_off, tag##_plog_lnP, tag##_plog_term_off, tag##_plog_A,      \
              tag##_plog_logA, tag##_plog_b, tag##_plog_EaR}

enum MechId { MECH_GRI30 = 0, MECH_H2O2 = 1, MECH_NDODECANE = 2, MECH_H2LI = 3, MECH_ESTIMATE = 4 };

// Traits of each compiled mechanism, per formulation (CV = 1: constant volume).
#define MECH_TRAITS(PFX, ID) MechT<PFX##_NSP, PFX##_NRXN, ID, PFX##_NU_DEN, PFX##_NUNITS, PFX##_NPLOG, CV>
template <int CV> using GriF = MECH_TRAITS(MECH_GRI30, MECH_GRI30);
template <int CV> using H2F = MECH_TRAITS(MECH_H2O2, MECH_H2O2);
template <int CV> using NdF = MECH_TRAITS(MECH_NDODECANE_REITZ, MECH_NDODECANE);
template <int CV> using H2LiF = MECH_TRAITS(MECH_H2_LI_2004, MECH_H2LI);
// kerosene (214 species): mixed precision only -- one warp's FP32 Newton
// matrix (214 x 215 x 4 B = 184 KB) fills an SM's shared memory; the FP64
// matrix would not fit
template <int CV> using EstF = MECH_TRAITS(MECH_ESTIMATE_MECH_04042022, MECH_ESTIMATE);
using GriT = GriF<0>;
using H2T = H2F<0>;
using NdT = NdF<0>;
using H2LiT = H2LiF<0>;
using EstT = EstF<0>;
static_assert(MECH_ESTIMATE + 1 == kNumMech, "one descriptor per mechanism");

int mech_from_name(const char* name) {
    if (!name) return -1;
    std::string s(name);
    if (s.size() > 5 && s.substr(s.size() - 5) == ".yaml") s = s.substr(0, s.size() - 5);
    if (s.size() > 4 && s.substr(s.size() - 4) == ".xml") s = s.substr(0, s.size() - 4);
    if (s == "gri30") return MECH_GRI30;
    if (s == "h2o2") return MECH_H2O2;
    if (s == "nDodecane_Reitz") return MECH_NDODECANE;
    if (s == "h2_li_2004") return MECH_H2LI;
    if (s == "ESTiMatE-Mech_04042022") return MECH_ESTIMATE;
    return -1;
}

int dispatch_units(int mech) {
    switch (mech) {
        case MECH_GRI30: return GriT::NUNITMAX;
        case MECH_H2O2: return H2T::NUNITMAX;
        case MECH_NDODECANE: return NdT::NUNITMAX;
        case MECH_H2LI: return H2LiT::NUNITMAX;
        case MECH_ESTIMATE: return EstT::NUNITMAX;
        default: return 0;
    }
}

}  // namespace

// ---------------------------------------------------------------- kernels
struct KParams {
    long long ncells;
    long long pitch;                  // row stride of Y in cells (>= ncells; a chunk of a larger batch)
    const double* P;
    double P_scalar;
    double* T;
    double* Y;
    int32_t* status;
    int32_t* cnt[7];                  // per-cell counters (each may be null)
    unsigned long long* queue;        // persistent form: work-queue head
    unsigned long long* totals;       // [8] call totals
    unsigned long long* prof;         // [5] per-phase cycle totals, or null
    void* wglobal;                    // WarpGlobal per resident warp (persistent) or per cell (step form)
    unsigned char* records;           // step form: per-cell state records; null = persistent form
    unsigned long long* done_count;   // step form: cells finished
    double t0, t1, rtol, atol;
    int max_steps, max_order, refine, steps;
    int chunk;                        // persistent form: cells a warp claims per queue access
    int helpers;                      // widest mechanisms: helper warps may serve warp 0
    long long helper_join_cycles;     // helper hand-off wait limits (0 = defaults, see HelperCtl)
    long long helper_drain_cycles;
    long long helper_idle_cycles;
};

template <class MT>
__device__ __forceinline__ void load_cell(const KParams& p, long long cell, int lane, double (&y0)[MT::NS]) {
    constexpr int N = MT::N;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + MT::G * s;
        if (i < N - 1) y0[s] = p.Y[(long long)i * p.pitch + cell];
        else if (i == N - 1) y0[s] = p.T[cell];
        else y0[s] = 0.0;
    }
}

// Density P W / (R T) of a cell's state at pressure P; y in internal order
// [Y_0 .. Y_{N-2}, T].  In the constant-volume form the kernels carry rho in
// the pressure slot (the chemistry then takes it as fixed, see species_phase).
template <class MT>
__device__ __forceinline__ double cell_density(double P, const double (&y)[MT::NS], int lane) {
    constexpr int N = MT::N;
    const DevMech& M = mech<MT>();
    double sy = 0.0, sw = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + MT::G * s;
        if (i < N - 1) {
            sy += y[s];
            sw += y[s] * __ldg(M.inv_mw + i);
        }
    }
    sy = group_sum<MT::G>(sy);
    sw = group_sum<MT::G>(sw) + (1.0 - sy) * __ldg(M.inv_mw + N - 1);
    const double T = group_shfl<MT::G>(y[(N - 1) / MT::G], (N - 1) % MT::G);
    return ode_div(P, kRU * T * sw);
}

// The value the chemistry takes in its pressure slot: P (constant pressure) or
// the density of the state at P (constant volume: the density the cell keeps).
template <class MT>
__device__ __forceinline__ double pressure_slot(const KParams& p, long long cell, const double (&y)[MT::NS],
                                                int lane) {
    const double P = p.P ? p.P[cell] : p.P_scalar;
    if constexpr (MT::CONV) return cell_density<MT>(P, y, lane);
    else return P;
}

template <class MT>
__device__ __forceinline__ void store_cell(const KParams& p, long long cell, int lane, const double (&yo)[MT::NS]) {
    constexpr int N = MT::N;
    double part = 0.0;
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + MT::G * s;
        if (i < N - 1) part += yo[s];
    }
    const double yN = 1.0 - group_sum<MT::G>(part);
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + MT::G * s;
        if (i < N - 1) p.Y[(long long)i * p.pitch + cell] = yo[s];
        else if (i == N - 1) {
            p.T[cell] = yo[s];
            p.Y[(long long)(N - 1) * p.pitch + cell] = yN;
        }
    }
}

// The BDF kernel, both forms:
//   persistent (records == null): a grid of resident warps; each warp pulls
//     cell indices from the device work queue and integrates each cell to t1;
//   one launch per step (records != null): warp w owns cell w and advances it by
//     at most `steps` BDF steps, its full state kept in HBM between launches.
// The step code is inlined once, so both forms execute the same instructions
// and give the same bits.
// MINB: minimum resident 128-thread blocks per SM the register allocation must
// allow (1 -> up to 255 registers, 3 -> at most 168, 4 -> at most 128: the last
// only for the mechanisms below kMinb4MaxN unknowns); the host picks the variant
// that keeps the most CTAs resident, or the options name it.
// Helper warp of a CTA that integrates one cell of a widest mechanism: runs the
// shares warp 0 posts until it posts kCmdExit (or, bounded, stops posting).
template <class MT, class LinT>
__device__ __noinline__ void helper_loop(int wib, int lane) {
    HelperCtl* h = &g_helper_ctl;
    unsigned seen = 0;
#pragma unroll 1
    for (;;) {
        const long long t0 = clock64();
        const long long idle_limit = h->idle_cycles;
        unsigned cur;
        bool idle_out = false;
        while ((cur = ld_volatile(&h->seq)) == seen) {
            if (clock64() - t0 > idle_limit) { idle_out = true; break; }
            __nanosleep(32);
        }
        __syncwarp();
        if (__any_sync(kFull, idle_out)) {
            if (lane == 0) h->err = 1;
            return;
        }
        __threadfence_block();
        seen = cur;
        const int cmd = *(const volatile int*)&h->cmd;
        if (cmd == kCmdExit) return;
        if (cmd == kCmdRhs)
            rhs_groups<MT>(h->rc, h->C_off, h->G_off, h->q_off, wib, kHelperWarps + 1, lane);
        else if (cmd == kCmdLu)
            lu_trailing<MT, LinT>(smem_at<LinT>(h->A_off), h->k0, h->kend, lane, wib, kHelperWarps + 1);
        __threadfence_block();
        __syncwarp();
        if (lane == 0) atomicAdd(&h->done, 1u);
    }
}

template <class MT, class LinT, int MINB>
__global__ void __launch_bounds__(128, MINB) k_bdf(const __grid_constant__ KParams p) {
    using R = StepRecord<MT, LinT>;
    constexpr int G = MT::G;                 // lanes per cell
    const int lane = threadIdx.x % G;        // lane within the cell's group
    const int wib = threadIdx.x / G;         // the cell's slot in the CTA
    long long cells_per_block = blockDim.x / G;
    if constexpr (MT::N >= kWideN) {
        // one cell per CTA: warp 0 integrates, warps 1-3 serve it (see HelperCtl)
        HelperCtl* hc = &g_helper_ctl;
        const bool serve = p.helpers && blockDim.x == 32 * (kHelperWarps + 1);
        if (threadIdx.x == 0) {
            hc->seq = 0;
            hc->done = 0;
            hc->posted = 0;
            hc->cmd = 0;
            hc->err = 0;
            hc->poisoned = 0;
            hc->exit_posted = serve ? 0 : 1;
            hc->nhelpers = serve ? kHelperWarps : 0;
            hc->join_cycles = p.helper_join_cycles > 0 ? p.helper_join_cycles : kJoinCycles;
            hc->drain_cycles = p.helper_drain_cycles > 0 ? p.helper_drain_cycles : kDrainCycles;
            hc->idle_cycles = p.helper_idle_cycles > 0 ? p.helper_idle_cycles : kHelperIdleCycles;
        }
        __syncthreads();
        if (serve) {
            if (wib != 0) {
                helper_loop<MT, LinT>(wib, lane);
                return;
            }
            cells_per_block = 1;
        }
    }
    auto* w = reinterpret_cast<WarpSmem<MT, LinT>*>(dyn_smem()) + wib;
    const unsigned off = smem_off(w);
    BdfState& S = w->st;
    const long long gw = (long long)blockIdx.x * cells_per_block + wib;
    const bool step_form = p.records != nullptr;
    auto* wglob = reinterpret_cast<WarpGlobal<MT, LinT>*>(p.wglobal);
    const int profiling = (p.prof != nullptr && !step_form) ? 1 : 0;
    if (profiling && lane < 8) wglob[gw].prof[lane] = 0;
    __syncwarp(gmask<G>());
    const long long t_start = profiling ? clock64() : 0;
    unsigned long long tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long cell = gw;
    unsigned long long next = 0;   // persistent form: next claimed cell and how many remain
    int left = 0;
#pragma unroll 1
    for (int iter = 0;; ++iter) {
        if (step_form) {
            if (iter > 0 || cell >= p.ncells) break;
        } else {
            if (left == 0) {
                unsigned long long c = 0;
                if (lane == 0) c = atomicAdd(p.queue, (unsigned long long)p.chunk);
                next = group_shfl<G>(c, 0);
                left = p.chunk;
            }
            if (next >= (unsigned long long)p.ncells) break;
            cell = (long long)next;
            ++next;
            --left;
        }
        WarpGlobal<MT, LinT>* wg = wglob + (step_form ? cell : gw);
        unsigned char* rec = step_form ? p.records + cell * (long long)R::kBytes : nullptr;
        const int phase = step_form ? *reinterpret_cast<const int*>(rec + R::kPhaseOff) : 0;
        if (phase == 2) continue;
        if (phase != 0) bdf_load<MT, LinT>(off, rec, lane);
        S.rtol = p.rtol;
        S.atol = p.atol;
        S.max_steps = p.max_steps;
        S.qmax = p.max_order;
        S.refine = p.refine;
        S.profiling = profiling;
        S.prof = wg->prof;
        S.lu_dirty = 0;
        int status = 0;
        bool done = false;
        bool ill = false;   // cell left as given: pressure not > 0 (or NaN, CVODE's CV_ILL_INPUT),
                            // or claimed by a poisoned CTA (CV_ERR_FAILURE, see HelperCtl)
        if constexpr (MT::N >= kWideN) {
            if (g_helper_ctl.poisoned) {
                ill = done = true;
                status = cv::CV_ERR_FAILURE;
                for (int i = 0; i < 7; ++i) S.cnt[i] = 0;
            }
        }
        if (!done && phase == 0) {
            Vec<MT::NS> y0;
            load_cell<MT>(p, cell, lane, y0.v);
            const double P0 = p.P ? p.P[cell] : p.P_scalar;
            if (!(P0 > 0.0)) {
                ill = done = true;
                status = cv::CV_ILL_INPUT;
                for (int i = 0; i < 7; ++i) S.cnt[i] = 0;
            } else {
                S.P = pressure_slot<MT>(p, cell, y0.v, lane);
                status = bdf_begin<MT, LinT>(off, y0, p.t0, p.t1, lane);
                done = (status != 0);
            }
        }
        if (!done) status = bdf_advance<MT, LinT>(off, wg, p.t1, p.steps, done, lane);
        if constexpr (MT::N >= kWideN) {
            // the CTA was poisoned during this cell: late helper writes may have
            // reached its rates or factors
            if (g_helper_ctl.poisoned && !ill) {
                status = cv::CV_ERR_FAILURE;
                done = true;
            }
        }
        if (done) {
            if (!ill) {
                const Vec<MT::NS> yo = bdf_finish<MT, LinT>(off, status, p.t1, lane);
                store_cell<MT>(p, cell, lane, yo.v);
            }
            if (lane == 0) {
                if (p.status) p.status[cell] = status;
                for (int i = 0; i < 7; ++i)
                    if (p.cnt[i]) p.cnt[i][cell] = S.cnt[i];
                if (step_form) atomicAdd(p.done_count, 1ULL);
            }
            for (int i = 0; i < 7; ++i) tot[i] += (unsigned long long)S.cnt[i];
            tot[7] += (status != 0);
        }
        if (step_form) bdf_save<MT, LinT>(off, rec, done ? 2 : 1, lane);
    }
    if constexpr (MT::N >= kWideN) {
        if (!g_helper_ctl.exit_posted) helpers_post(&g_helper_ctl, kCmdExit, lane);
    }
    if (lane == 0)
        for (int i = 0; i < 8; ++i)
            if (tot[i]) atomicAdd(p.totals + i, tot[i]);
    if (profiling && lane == 0) {
        long long* pr = wglob[gw].prof;
        pr[PH_TOTAL] = clock64() - t_start;
        for (int i = 0; i < 5; ++i) atomicAdd(p.prof + i, (unsigned long long)pr[i]);
    }
}

// Batched chemistry alone (one warp per cell): the counterparts of the
// reference's dydt_cvode_GPU / kernel_dydt and jacobian_cvode_GPU /
// kernel_eval_jacob (src/Integrators/Drivers/CVodeGPUDriver.cu:28-106), with
// outputs in the reference's layout.
template <class MT, class LinT>
__global__ void __launch_bounds__(128) k_eval_rhs(const __grid_constant__ KParams p, double* dTdt, double* dYdt) {
    const int lane = threadIdx.x % MT::G, wib = threadIdx.x / MT::G;
    if constexpr (MT::N >= kWideN) {   // no helper warps here
        if (threadIdx.x == 0) g_helper_ctl.nhelpers = 0;
        __syncthreads();
    }
    const long long cell = (long long)blockIdx.x * (blockDim.x / MT::G) + wib;
    if (cell >= p.ncells) return;
    auto* sm = reinterpret_cast<WarpSmem<MT, LinT>*>(dyn_smem()) + wib;
    Vec<MT::NS> y;
    load_cell<MT>(p, cell, lane, y.v);
    const double P = pressure_slot<MT>(p, cell, y.v, lane);
    const Vec<MT::NS> f = warp_rhs<MT>(P, y, smem_off(&sm->chem), lane);
#pragma unroll
    for (int s = 0; s < MT::NS; ++s) {
        const int i = lane + MT::G * s;
        if (i < MT::N - 1) dYdt[(long long)i * p.ncells + cell] = f.v[s];
        else if (i == MT::N - 1) dTdt[cell] = f.v[s];
    }
}

// jac: per cell N*N column-major, reference order [T, Y_0 .. Y_{N-2}].
template <class MT, class LinT>
__global__ void __launch_bounds__(128) k_eval_jac(const __grid_constant__ KParams p, double* jac) {
    const int lane = threadIdx.x % MT::G, wib = threadIdx.x / MT::G;
    if constexpr (MT::N >= kWideN) {   // no helper warps here
        if (threadIdx.x == 0) g_helper_ctl.nhelpers = 0;
        __syncthreads();
    }
    const long long cell = (long long)blockIdx.x * (blockDim.x / MT::G) + wib;
    if (cell >= p.ncells) return;
    auto* sm = reinterpret_cast<WarpSmem<MT, LinT>*>(dyn_smem()) + wib;
    auto* wg = reinterpret_cast<WarpGlobal<MT, LinT>*>(p.wglobal) + cell;
    Vec<MT::NS> y;
    load_cell<MT>(p, cell, lane, y.v);
    const double P = pressure_slot<MT>(p, cell, y.v, lane);
    warp_jac<MT, LinT>(P, y, smem_off(sm->A), smem_off(&sm->chem), &wg->js, wg->savedJ, lane);
    constexpr int N = MT::N;
    double* out = jac + cell * (long long)(N * N);
    for (int i = 0; i < N; ++i)
        for (int j = lane; j < N; j += MT::G) {   // internal row i, column j
            const int ri = (i == N - 1) ? 0 : i + 1, rj = (j == N - 1) ? 0 : j + 1;
            out[ri + N * rj] = (double)sm->A[i * MT::LDA + j];
        }
}

// Mixture specific enthalpy h = sum_k Y_k h_k(T) / W_k [J/kg] of each cell,
// one thread per cell (the reads of Y[k][c] are coalesced across the warp).
// The NASA-7 enthalpy polynomial is the one the RHS uses.
template <class MT>
__global__ void __launch_bounds__(256) k_enthalpy(long long n, const double* T, const double* Y, double* hmass) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const DevMech& M = mech<MT>();
    const double t = T[c];
    const double invT = 1.0 / t;
    double acc = 0.0;
#pragma unroll 1
    for (int k = 0; k < MT::N; ++k) {
        const double* a = M.nasa + 14 * k + ((t <= __ldg(M.tmid + k)) ? 0 : 7);
        const double hRT = __ldg(a + 0) + t * (__ldg(a + 1) * 0.5 + t * (__ldg(a + 2) * (1.0 / 3.0) +
                           t * (__ldg(a + 3) * 0.25 + __ldg(a + 4) * 0.2 * t))) + __ldg(a + 5) * invT;
        acc += Y[(long long)k * n + c] * hRT * __ldg(M.inv_mw + k);
    }
    hmass[c] = acc * kRU * t;
}

// FP64 FMA throughput probe: independent DFMA chains per thread.
__global__ void k_fp64_peak(double* out, int iters) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9, a4 = a0 + 4e-9,
           a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
    const double m = 0.999999, c = 1e-9;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
            a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
        }
    }
    const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.0) out[0] = r;   // keep the chains live
}

// FP32 FMA throughput probe: independent FFMA chains per thread (the Newton
// matrix, its LU and the triangular solves run on this pipe in mixed precision).
__global__ void k_fp32_peak(float* out, int iters) {
    float a0 = threadIdx.x * 1e-9f, a1 = a0 + 1e-9f, a2 = a0 + 2e-9f, a3 = a0 + 3e-9f, a4 = a0 + 4e-9f,
          a5 = a0 + 5e-9f, a6 = a0 + 6e-9f, a7 = a0 + 7e-9f;
    const float m = 0.999999f, c = 1e-9f;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.0f) out[0] = r;   // keep the chains live
}

// ------------------------------------------------------------------ handle
// struct b200ode_handle: b200ode_internal.h

namespace {

// Shared memory of one warp: the per-cell WarpSmem of each of its 32 / G cells.
template <class MT, class LinT>
size_t warp_smem_bytes() { return sizeof(WarpSmem<MT, LinT>) * (32 / MT::G); }

// Cells a CTA of wpb warps integrates at once (one per warp, or 32 / G per warp
// for the mechanisms that put several cells in a warp; with helper warps the
// CTA is launched as wpb = 1 and holds one cell).
template <class MT>
long long cells_per_block(int wpb) { return (long long)wpb * (32 / MT::G); }

b200ode_status ensure_wg(b200ode_handle* h, size_t bytes) {
    if (bytes <= h->wg_bytes) return B200ODE_OK;
    if (h->d_wg) cudaFree(h->d_wg);
    h->d_wg = nullptr;
    h->wg_bytes = 0;
    CUDA_TRY(cudaMalloc(&h->d_wg, bytes));
    h->wg_bytes = bytes;
    return B200ODE_OK;
}

// Threads per CTA of the BDF kernel for wpb cells per CTA: one 128-thread CTA
// per cell when a widest mechanism's helper warps serve (wpb = 1).
template <class MT>
int bdf_threads(const b200ode_handle* h, int wpb) {
    if (MT::N >= kWideN && wpb == 1 && h->opt.cta_helpers) return 32 * (kHelperWarps + 1);
    return wpb * 32;
}

// Resident CTAs per SM of the BDF kernel's register variant MINB (launch
// bounds of 1 or 3 CTAs per SM) at wpb warps per CTA; 0 if it does not fit.
template <class MT, class LinT, int MINB>
int bdf_occupancy(const b200ode_handle* h, int wpb) {
    const size_t smem = warp_smem_bytes<MT, LinT>() * wpb;
    auto k = k_bdf<MT, LinT, MINB>;
    int bps = 0;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, bdf_threads<MT>(h, wpb), smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return bps;
}

// The 128-register variant (4 CTAs per SM) is built only below this many
// unknowns: the H2 kernels fit it with few spills and gain a fourth CTA (16
// warps per SM: +9 % mixed, +14 % FP64 on 32,768 cells), while larger cells are
// held to 3 CTAs or fewer by shared memory, where it would only add spills.
constexpr int kMinb4MaxN = 32;

// Register variant MINB's resident CTAs for wpb warps per CTA (0 for a variant
// this mechanism does not build).
template <class MT, class LinT>
int bdf_variant_occupancy(const b200ode_handle* h, int wpb, int minb) {
    if (minb == 4) {
        if constexpr (MT::N < kMinb4MaxN) return bdf_occupancy<MT, LinT, 4>(h, wpb);
        return 0;
    }
    return minb == 3 ? bdf_occupancy<MT, LinT, 3>(h, wpb) : bdf_occupancy<MT, LinT, 1>(h, wpb);
}

// The register variant (1, 3 or 4) that keeps the most CTAs of wpb warps
// resident; ties keep the one with more registers a thread.
template <class MT, class LinT>
int best_variant(const b200ode_handle* h, int wpb, int* ctas) {
    int best = 1, occ = bdf_variant_occupancy<MT, LinT>(h, wpb, 1);
    for (int v : {3, 4}) {
        const int o = bdf_variant_occupancy<MT, LinT>(h, wpb, v);
        if (o > occ) {
            occ = o;
            best = v;
        }
    }
    if (ctas) *ctas = occ;
    return best;
}

// Warps per CTA: the option when set, else the shape (4, 2 or 1 warps per CTA,
// any register variant) that keeps the most warps resident per SM for this
// mechanism and precision (shared memory per warp and registers decide), ties
// to the larger CTA.  Computed once per handle.
template <class MT, class LinT>
int pick_wpb(b200ode_handle* h) {
    if (h->opt.warps_per_block > 0) return std::min(h->opt.warps_per_block, 4);
    if (h->auto_wpb > 0) return h->auto_wpb;
    int best = 4, best_warps = -1;
    for (int wpb : {4, 2, 1}) {
        int bps = 0;
        best_variant<MT, LinT>(h, wpb, &bps);
        if (bps * wpb > best_warps) {
            best_warps = bps * wpb;
            best = wpb;
        }
    }
    h->auto_wpb = best;
    return best;
}

// The BDF kernel's register variant for wpb warps per CTA: with
// options.blocks_per_sm set, the variant whose launch bounds allow that many
// CTAs (4 x 4 / wpb or more: 128 registers where built; 3 x 4 / wpb or more:
// 168), else the one that keeps the most CTAs resident (decided once per
// handle and CTA shape).
template <class MT, class LinT>
auto bdf_kernel(b200ode_handle* h, int wpb) -> void (*)(KParams) {
    int v;
    if (h->opt.blocks_per_sm > 0) {
        v = h->opt.blocks_per_sm >= 3 * (4 / wpb) ? 3 : 1;
        if (MT::N < kMinb4MaxN && h->opt.blocks_per_sm >= 4 * (4 / wpb)) v = 4;
    } else {
        const int key = wpb * 1024 + bdf_threads<MT>(h, wpb);
        auto it = h->auto_minb.find(key);
        if (it == h->auto_minb.end()) it = h->auto_minb.emplace(key, best_variant<MT, LinT>(h, wpb, nullptr)).first;
        v = it->second;
    }
    if constexpr (MT::N < kMinb4MaxN) {
        if (v == 4) return k_bdf<MT, LinT, 4>;
    }
    return v == 3 ? k_bdf<MT, LinT, 3> : k_bdf<MT, LinT, 1>;
}

template <class MT, class LinT>
b200ode_status launch_bdf(b200ode_handle* h, KParams& p, cudaStream_t st, int* launches) {
    using R = StepRecord<MT, LinT>;
    const int wpb = pick_wpb<MT, LinT>(h);
    const size_t smem = warp_smem_bytes<MT, LinT>() * wpb;
    auto kern = bdf_kernel<MT, LinT>(h, wpb);
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t n = (size_t)p.ncells;
    CUDA_TRY(cudaMemsetAsync(h->d_ctl, 0, 16 * sizeof(unsigned long long), st));
    p.queue = h->d_ctl;
    p.totals = h->d_ctl + 1;
    p.done_count = h->d_ctl + 9;
    if (h->opt.persistent) {
        int bps = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, bdf_threads<MT>(h, wpb), smem));
        if (bps < 1) return fail(B200ODE_ERR_CUDA, "kernel does not fit on an SM");
        if (h->opt.blocks_per_sm > 0) bps = std::min(bps, h->opt.blocks_per_sm);
        h->last_blocks_per_sm = bps;
        const long long cpb = cells_per_block<MT>(wpb);
        long long blocks = (long long)bps * h->num_sms;
        blocks = std::max(1LL, std::min(blocks, ((long long)n + cpb - 1) / cpb));
        b200ode_status rc = ensure_wg(h, (size_t)(blocks * cpb) * sizeof(WarpGlobal<MT, LinT>));
        if (rc != B200ODE_OK) return rc;
        p.wglobal = h->d_wg;
        p.records = nullptr;
        p.steps = 0x7fffffff;
        kern<<<(unsigned)blocks, bdf_threads<MT>(h, wpb), smem, st>>>(p);
        CUDA_TRY(cudaGetLastError());
        *launches += 1;
        return B200ODE_OK;
    }
    // one launch per BDF step: per-cell scratch and state records in HBM
    b200ode_status rc = ensure_wg(h, n * sizeof(WarpGlobal<MT, LinT>));
    if (rc != B200ODE_OK) return rc;
    const size_t rb = n * R::kBytes;
    if (rb > h->rec_bytes) {
        if (h->d_rec) cudaFree(h->d_rec);
        h->d_rec = nullptr;
        h->rec_bytes = 0;
        CUDA_TRY(cudaMalloc(&h->d_rec, rb));
        h->rec_bytes = rb;
    }
    if (!h->h_done) CUDA_TRY(cudaMallocHost(&h->h_done, sizeof(unsigned long long)));
    CUDA_TRY(cudaMemsetAsync(h->d_rec, 0, rb, st));
    p.wglobal = h->d_wg;
    p.records = h->d_rec;
    p.steps = 1;
    const long long cpb = cells_per_block<MT>(wpb);
    const unsigned blocks = (unsigned)(((long long)n + cpb - 1) / cpb);
    const int per_check = h->opt.use_graph ? 16 : 1;
    cudaGraphExec_t gexec = nullptr;
    if (h->opt.use_graph) {
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < per_check; ++i) kern<<<blocks, bdf_threads<MT>(h, wpb), smem, st>>>(p);
        CUDA_TRY(cudaStreamEndCapture(st, &g));
        cudaError_t e = cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(B200ODE_ERR_CUDA, "cudaGraphInstantiate");
    }
    // every launch finishes a cell or advances it one step: at most max_steps + 2 launches
    const long long max_launch = (long long)h->opt.max_steps + 2;
    rc = B200ODE_OK;
    for (long long it = 0; it < max_launch; it += per_check) {
        if (gexec) {
            if (cudaGraphLaunch(gexec, st) != cudaSuccess) { rc = fail(B200ODE_ERR_CUDA, "cudaGraphLaunch"); break; }
        } else {
            kern<<<blocks, bdf_threads<MT>(h, wpb), smem, st>>>(p);
        }
        *launches += per_check;
        if (cudaMemcpyAsync(h->h_done, p.done_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = fail(B200ODE_ERR_CUDA, std::string("step-form launch: ") + cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (*h->h_done >= n) break;
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    return rc;
}

template <int CV, class F>
b200ode_status dispatch_form(const b200ode_handle* h, F&& f) {
    const bool fp64 = h->opt.precision == B200ODE_FP64;
    if (h->mech == MECH_GRI30) return fp64 ? f(GriF<CV>{}, double{}) : f(GriF<CV>{}, float{});
    if (h->mech == MECH_NDODECANE) return fp64 ? f(NdF<CV>{}, double{}) : f(NdF<CV>{}, float{});
    if (h->mech == MECH_ESTIMATE) return f(EstF<CV>{}, float{});   // FP64 refused at creation
    if (h->mech == MECH_H2LI) return fp64 ? f(H2LiF<CV>{}, double{}) : f(H2LiF<CV>{}, float{});
    return fp64 ? f(H2F<CV>{}, double{}) : f(H2F<CV>{}, float{});
}

// Calls f(MT{}, LinT{}) with the handle's mechanism, formulation and
// Newton-matrix precision.
template <class F>
b200ode_status dispatch_mech(const b200ode_handle* h, F&& f) {
    if (h->opt.formulation == B200ODE_CONV) return dispatch_form<1>(h, f);
    return dispatch_form<0>(h, f);
}

b200ode_status run(b200ode_handle* h, KParams& p, cudaStream_t st, int* launches) {
    return dispatch_mech(h, [&](auto mt, auto lt) {
        return launch_bdf<decltype(mt), decltype(lt)>(h, p, st, launches);
    });
}

// Launch shape of the persistent form: the same choice launch_bdf makes.
template <class MT, class LinT>
b200ode_status persistent_shape(b200ode_handle* h, long long n, void (**kern)(KParams), long long* blocks,
                                int* wpb_out, size_t* smem_out) {
    const int wpb = pick_wpb<MT, LinT>(h);
    const size_t smem = warp_smem_bytes<MT, LinT>() * wpb;
    auto k = bdf_kernel<MT, LinT>(h, wpb);
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int bps = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, bdf_threads<MT>(h, wpb), smem));
    if (bps < 1) return fail(B200ODE_ERR_CUDA, "kernel does not fit on an SM");
    if (h->opt.blocks_per_sm > 0) bps = std::min(bps, h->opt.blocks_per_sm);
    const long long cpb = cells_per_block<MT>(wpb);
    long long b = (long long)bps * h->num_sms;
    b = std::max(1LL, std::min(b, (n + cpb - 1) / cpb));
    *kern = k;
    *blocks = b;
    *wpb_out = wpb;
    *smem_out = smem;
    return B200ODE_OK;
}

template <class MT, class LinT>
b200ode_status launch_eval(b200ode_handle* h, KParams& p, double* d_dT, double* d_dY, double* d_jac,
                           cudaStream_t st) {
    const int wpb = pick_wpb<MT, LinT>(h);   // shared memory per warp decides (4 for GRI, 1-2 for larger)
    const size_t smem = warp_smem_bytes<MT, LinT>() * wpb;
    const long long cpb = cells_per_block<MT>(wpb);
    const unsigned blocks = (unsigned)((p.ncells + cpb - 1) / cpb);
    if (d_jac) {
        b200ode_status rc = ensure_wg(h, (size_t)p.ncells * sizeof(WarpGlobal<MT, LinT>));
        if (rc != B200ODE_OK) return rc;
        p.wglobal = h->d_wg;
        auto k = k_eval_jac<MT, LinT>;
        CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<blocks, wpb * 32, smem, st>>>(p, d_jac);
    } else {
        auto k = k_eval_rhs<MT, LinT>;
        CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<blocks, wpb * 32, smem, st>>>(p, d_dT, d_dY);
    }
    CUDA_TRY(cudaGetLastError());
    return B200ODE_OK;
}

b200ode_status ensure_cap(b200ode_handle* h, size_t n) {
    if (n <= h->cap) return B200ODE_OK;
    cudaFree(h->d_T); cudaFree(h->d_Y); cudaFree(h->d_P); cudaFree(h->d_status); cudaFree(h->d_cnt);
    h->d_T = h->d_Y = h->d_P = nullptr; h->d_status = h->d_cnt = nullptr; h->cap = 0;
    const size_t nsp = h->hm.nsp;
    CUDA_TRY(cudaMalloc(&h->d_T, n * sizeof(double)));
    CUDA_TRY(cudaMalloc(&h->d_Y, n * nsp * sizeof(double)));
    CUDA_TRY(cudaMalloc(&h->d_P, n * sizeof(double)));
    CUDA_TRY(cudaMalloc(&h->d_status, n * sizeof(int32_t)));
    CUDA_TRY(cudaMalloc(&h->d_cnt, 7 * n * sizeof(int32_t)));
    h->cap = n;
    return B200ODE_OK;
}

b200ode_status check_args(const b200ode_handle* h, int64_t n, double t0, double t1) {
    if (!h) return fail(B200ODE_ERR_INVALID, "null handle");
    if (n < 0) return fail(B200ODE_ERR_INVALID, "n_cells < 0");
    if (!(t1 == t1) || !(t0 == t0)) return fail(B200ODE_ERR_INVALID, "t0/t1 not finite");
    return B200ODE_OK;
}

void fill_params(b200ode_handle* h, KParams& p, int64_t n, const double* dP, double Ps, double* dT,
                 double* dY, int32_t* dstat, int32_t* const* dcnt, double t0, double t1) {
    std::memset(&p, 0, sizeof(p));
    p.ncells = n;
    p.pitch = n;
    p.P = dP;
    p.P_scalar = Ps;
    p.T = dT;
    p.Y = dY;
    p.status = dstat;
    for (int i = 0; i < 7; ++i) p.cnt[i] = dcnt ? dcnt[i] : nullptr;
    p.queue = h->d_ctl;
    p.totals = h->d_ctl + 1;
    p.done_count = h->d_ctl + 9;
    p.prof = h->opt.profile_phases ? h->d_ctl + 10 : nullptr;
    p.t0 = t0;
    p.t1 = t1;
    p.rtol = h->opt.reltol;
    p.atol = h->opt.abstol;
    p.max_steps = h->opt.max_steps;
    p.max_order = h->opt.max_order;
    p.refine = h->opt.refine;
    p.chunk = std::max(1, std::min(h->opt.queue_chunk, 64));
    p.helpers = h->opt.cta_helpers != 0;
    p.helper_join_cycles = h->opt.helper_join_cycles;
    p.helper_drain_cycles = h->opt.helper_drain_cycles;
    p.helper_idle_cycles = h->opt.helper_idle_cycles;
}

// Device bytes per cell a launch of this handle needs beyond the caller's
// buffers: the one-launch-per-step form keeps a state record and a
// WarpGlobal per cell; the persistent form only per resident warp.
size_t step_form_bytes_per_cell(const b200ode_handle* h) {
    if (h->opt.persistent) return 0;
    size_t b = 0;
    dispatch_mech(h, [&](auto mt, auto lt) {
        using MT = decltype(mt);
        using LinT = decltype(lt);
        b = StepRecord<MT, LinT>::kBytes + sizeof(WarpGlobal<MT, LinT>);
        return B200ODE_OK;
    });
    return b;
}

// Cells per launch: the whole batch when it fits, else memory-sized chunks
// (the reference's calc_gpu_points, src/Integrators/Drivers/CVodeGPUDriver.cu:108-130,
// takes 80 % of the free memory over its per-cell footprint the same way).
// io_bytes_per_cell: the handle's own I/O buffers (host-buffer entry point) or
// 0 (caller's device buffers).  `held` = bytes the handle already holds for
// these buffers (freed and re-allocated when they grow).
int64_t cells_per_launch(const b200ode_handle* h, int64_t n, size_t io_bytes_per_cell) {
    if (n <= 0) return 1;
    int64_t limit = n;
    if (h->opt.max_cells_per_launch > 0) limit = std::min<int64_t>(limit, h->opt.max_cells_per_launch);
    const size_t per_cell = step_form_bytes_per_cell(h) + io_bytes_per_cell;
    if (per_cell > 0) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const size_t held = h->rec_bytes + (h->opt.persistent ? 0 : h->wg_bytes) +
                                h->cap * io_bytes_per_cell;
            const double avail = 0.8 * (double)(free_b + held);
            int64_t fit = (int64_t)(avail / (double)per_cell);
            if (fit >= 64) fit -= fit % 32;
            limit = std::min<int64_t>(limit, std::max<int64_t>(fit, 1));
        } else {
            cudaGetLastError();
        }
    }
    return std::max<int64_t>(limit, 1);
}

// Adds one launch's call totals (read from the control block) into *s.
b200ode_status add_totals(b200ode_handle* h, const unsigned long long* ctl, b200ode_stats* s, cudaStream_t st) {
    unsigned long long t[15];
    CUDA_TRY(cudaMemcpyAsync(t, ctl + 1, sizeof(t), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < 5; ++i) s->phase_cycles[i] += h->opt.profile_phases ? (int64_t)t[9 + i] : 0;
    s->total_nst += (int64_t)t[0]; s->total_nfe += (int64_t)t[1]; s->total_nje += (int64_t)t[2];
    s->total_nsetups += (int64_t)t[3]; s->total_nni += (int64_t)t[4]; s->total_ncfn += (int64_t)t[5];
    s->total_netf += (int64_t)t[6]; s->n_failed += (int64_t)t[7];
    return B200ODE_OK;
}

// Zeroes the totals and timings of *s, keeping its per-cell counter pointers.
void clear_totals(b200ode_stats* s) {
    int32_t* keep[7] = {s->nst, s->nfe, s->nje, s->nsetups, s->nni, s->ncfn, s->netf};
    std::memset(s, 0, sizeof(*s));
    s->nst = keep[0]; s->nfe = keep[1]; s->nje = keep[2]; s->nsetups = keep[3];
    s->nni = keep[4]; s->ncfn = keep[5]; s->netf = keep[6];
}

}  // namespace

// ------------------------------------------------- internal API (b200ode_internal.h)
namespace b200 {

b200ode_status set_error(b200ode_status st, const std::string& msg) { return fail(st, msg); }

size_t persistent_scratch_bytes(b200ode_handle* h, int64_t n) {
    size_t bytes = 0;
    dispatch_mech(h, [&](auto mt, auto lt) {
        using MT = decltype(mt);
        using LinT = decltype(lt);
        void (*k)(KParams) = nullptr;
        long long blocks = 0;
        int wpb = 0;
        size_t smem = 0;
        b200ode_status rc = persistent_shape<MT, LinT>(h, std::max<long long>(n, 1), &k, &blocks, &wpb, &smem);
        if (rc == B200ODE_OK) bytes = (size_t)(blocks * cells_per_block<MT>(wpb)) * sizeof(WarpGlobal<MT, LinT>);
        return rc;
    });
    return bytes;
}

b200ode_status launch_persistent(b200ode_handle* h, int64_t n, const double* dP, double Ps, double* dT,
                                 double* dY, int32_t* dstat, double t0, double t1, unsigned long long* ctl,
                                 void* wg, cudaStream_t st) {
    if (n <= 0) return B200ODE_OK;
    KParams p;
    fill_params(h, p, n, dP, Ps, dT, dY, dstat, nullptr, t0, t1);
    p.queue = ctl;
    p.totals = ctl + 1;
    p.done_count = ctl + 9;
    p.prof = h->opt.profile_phases ? ctl + 10 : nullptr;
    p.wglobal = wg;
    p.records = nullptr;
    p.steps = 0x7fffffff;
    return dispatch_mech(h, [&](auto mt, auto lt) {
        using MT = decltype(mt);
        using LinT = decltype(lt);
        void (*k)(KParams) = nullptr;
        long long blocks = 0;
        int wpb = 0;
        size_t smem = 0;
        b200ode_status rc = persistent_shape<MT, LinT>(h, n, &k, &blocks, &wpb, &smem);
        if (rc != B200ODE_OK) return rc;
        CUDA_TRY(cudaMemsetAsync(ctl, 0, kCtlWords * sizeof(unsigned long long), st));
        k<<<(unsigned)blocks, bdf_threads<MT>(h, wpb), smem, st>>>(p);
        CUDA_TRY(cudaGetLastError());
        return B200ODE_OK;
    });
}

}  // namespace b200

// ------------------------------------------------------------------- C ABI
extern "C" {

void b200ode_default_options(b200ode_options* o) {
    if (!o) return;
    o->reltol = 1.0e-6;
    o->abstol = 1.0e-10;
    o->max_steps = 10000;
    o->max_order = 5;
    o->precision = B200ODE_MIXED;
    o->refine = 0;
    o->persistent = 1;
    o->warps_per_block = 0;
    o->blocks_per_sm = 0;
    o->queue_chunk = 1;
    o->use_graph = 0;
    o->device = -1;
    o->profile_phases = 0;
    o->formulation = B200ODE_CONP;
    o->cta_helpers = 1;
    o->helper_join_cycles = 0;
    o->helper_drain_cycles = 0;
    o->helper_idle_cycles = 0;
    o->max_cells_per_launch = 0;
}

const char* b200ode_last_error(void) { return g_last_error.c_str(); }

const char* b200ode_version(void) { return "b200ode 0.1 (sm_100a)"; }

int32_t b200ode_num_species(const b200ode_handle* h) { return h ? h->hm.nsp : -1; }

int32_t b200ode_mechanism_species(const char* mech_name) {
    switch (mech_from_name(mech_name)) {
        case MECH_GRI30: return MECH_GRI30_NSP;
        case MECH_H2O2: return MECH_H2O2_NSP;
        case MECH_NDODECANE: return MECH_NDODECANE_REITZ_NSP;
        case MECH_H2LI: return MECH_H2_LI_2004_NSP;
        case MECH_ESTIMATE: return MECH_ESTIMATE_MECH_04042022_NSP;
        default: return -1;
    }
}

b200ode_status b200ode_create(const char* mech_name, const b200ode_options* opts, b200ode_handle** out) {
    if (!out) return fail(B200ODE_ERR_INVALID, "null output pointer");
    *out = nullptr;
    const int mech = mech_from_name(mech_name);
    if (mech < 0)
        return fail(B200ODE_ERR_MECHANISM,
                    std::string("unknown mechanism '") + (mech_name ? mech_name : "(null)") +
                        "' (available: gri30.yaml, h2o2.yaml, nDodecane_Reitz.yaml, h2_li_2004.xml, "
                        "ESTiMatE-Mech_04042022.xml)");
    b200ode_options o;
    b200ode_default_options(&o);
    if (opts) o = *opts;
    if (!(o.reltol >= 0.0) || !(o.abstol > 0.0))
        return fail(B200ODE_ERR_INVALID, "reltol must be >= 0 and abstol > 0");
    if (o.max_steps <= 0) o.max_steps = 500;
    if (o.max_order < 1 || o.max_order > 5) o.max_order = 5;
    if (o.precision != B200ODE_FP64 && o.precision != B200ODE_MIXED)
        return fail(B200ODE_ERR_INVALID, "precision must be B200ODE_FP64 or B200ODE_MIXED");
    if (o.formulation != B200ODE_CONP && o.formulation != B200ODE_CONV)
        return fail(B200ODE_ERR_INVALID, "formulation must be B200ODE_CONP or B200ODE_CONV");
    if (mech == MECH_ESTIMATE && o.precision == B200ODE_FP64)
        return fail(B200ODE_ERR_INVALID,
                    "ESTiMatE-Mech_04042022 (214 unknowns) runs in B200ODE_MIXED only: its FP64 Newton "
                    "matrix (" + std::to_string(sizeof(WarpSmem<EstT, double>)) +
                        " bytes of shared memory per cell) exceeds an SM's shared memory");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(B200ODE_ERR_NO_DEVICE, "no CUDA device available");
    }
    auto* h = new b200ode_handle();
    h->mech = mech;
    h->opt = o;
    std::string err;
    h->hm = pack_mechanism(mech == MECH_GRI30  ? GEN_TABLES(gri30, MECH_GRI30)
                           : mech == MECH_H2O2 ? GEN_TABLES(h2o2, MECH_H2O2)
                           : mech == MECH_H2LI ? GEN_TABLES(h2_li_2004, MECH_H2_LI_2004)
                           : mech == MECH_ESTIMATE ? GEN_TABLES(estimate_mech_04042022, MECH_ESTIMATE_MECH_04042022)
                                               : GEN_TABLES(ndodecane_reitz, MECH_NDODECANE_REITZ),
                           &err);
    if (h->hm.nsp == 0) {
        delete h;
        return fail(B200ODE_ERR_MECHANISM, "mechanism packing failed: " + err);
    }
    // the per-warp gather scratch is sized at compile time from the generated unit count
    const int units_max = dispatch_units(mech);
    if (h->hm.nunit > units_max) {
        delete h;
        return fail(B200ODE_ERR_MECHANISM, "mechanism packing: " + std::to_string(h->hm.nunit) +
                                               " gather units, the kernels hold " + std::to_string(units_max));
    }
    auto cleanup = [&](b200ode_status st) { b200ode_destroy(h); return st; };
    if (o.device >= 0) {
        if (cudaSetDevice(o.device) != cudaSuccess) return cleanup(fail(B200ODE_ERR_CUDA, "cudaSetDevice failed"));
    }
    if (cudaGetDevice(&h->device) != cudaSuccess) return cleanup(fail(B200ODE_ERR_CUDA, "cudaGetDevice failed"));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess)
        return cleanup(fail(B200ODE_ERR_CUDA, "cudaGetDeviceProperties failed"));
    if (prop.major < 10)
        return cleanup(fail(B200ODE_ERR_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100 class"));
    h->num_sms = prop.multiProcessorCount;
    {
        // mechanism tables: one device copy per (device, mechanism) for the
        // process lifetime, published through the __constant__ descriptor
        std::lock_guard<std::mutex> lk(g_tables_mu);
        auto key = std::make_pair(h->device, mech);
        auto it = g_tables.find(key);
        if (it == g_tables.end()) {
            unsigned char* blob = nullptr;
            if (cudaMalloc(&blob, h->hm.blob.size()) != cudaSuccess)
                return cleanup(fail(B200ODE_ERR_ALLOC, "cudaMalloc mechanism tables"));
            if (cudaMemcpy(blob, h->hm.blob.data(), h->hm.blob.size(), cudaMemcpyHostToDevice) != cudaSuccess)
                return cleanup(fail(B200ODE_ERR_CUDA, "copy mechanism tables"));
            const DevMech dm = h->hm.bind(blob);
            if (cudaMemcpyToSymbol(c_mech, &dm, sizeof(DevMech), mech * sizeof(DevMech)) != cudaSuccess)
                return cleanup(fail(B200ODE_ERR_CUDA, "publish mechanism descriptor"));
            it = g_tables.emplace(key, blob).first;
        }
        h->d_blob = it->second;
        h->dm = h->hm.bind(h->d_blob);
    }
    if (cudaMalloc(&h->d_ctl, 16 * sizeof(unsigned long long)) != cudaSuccess)
        return cleanup(fail(B200ODE_ERR_ALLOC, "cudaMalloc control block"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(fail(B200ODE_ERR_CUDA, "cudaStreamCreate"));
    for (auto& e : h->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return cleanup(fail(B200ODE_ERR_CUDA, "cudaEventCreate"));
    *out = h;
    return B200ODE_OK;
}

void b200ode_destroy(b200ode_handle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_T); cudaFree(h->d_Y); cudaFree(h->d_P);
    cudaFree(h->d_status); cudaFree(h->d_cnt); cudaFree(h->d_ctl); cudaFree(h->d_wg);
    cudaFree(h->d_rec);
    if (h->h_done) cudaFreeHost(h->h_done);
    for (auto& e : h->ev) if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

b200ode_status b200ode_integrate_device(b200ode_handle* h, int64_t n, const double* dP, double Ps,
                                        double* dT, double* dY, double t0, double t1, int32_t* dstat,
                                        b200ode_stats* stats, void* stream) {
    NvtxRange range("b200ode_integrate_device");
    b200ode_status rc = check_args(h, n, t0, t1);
    if (rc != B200ODE_OK) return rc;
    if (stats) clear_totals(stats);
    if (n == 0) return B200ODE_OK;
    if (!dT || !dY) return fail(B200ODE_ERR_INVALID, "null T or Y");
    cudaStream_t st = (cudaStream_t)stream;
    int32_t* cnt[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (stats) {
        int32_t* src[7] = {stats->nst, stats->nfe, stats->nje, stats->nsetups, stats->nni, stats->ncfn, stats->netf};
        for (int i = 0; i < 7; ++i) cnt[i] = src[i];
    }
    // memory-sized chunks (one launch sequence each; the step form's per-cell
    // records would otherwise outgrow the device for very large batches)
    const int64_t chunk = cells_per_launch(h, n, 0);
    int launches = 0;
    float kernel_ms = 0.f;
    for (int64_t a = 0; a < n; a += chunk) {
        const int64_t m = std::min(chunk, n - a);
        int32_t* dcnt[7];
        for (int i = 0; i < 7; ++i) dcnt[i] = cnt[i] ? cnt[i] + a : nullptr;
        KParams p;
        fill_params(h, p, m, dP ? dP + a : nullptr, Ps, dT + a, dY + a, dstat ? dstat + a : nullptr, dcnt, t0, t1);
        p.pitch = n;
        CUDA_TRY(cudaEventRecord(h->ev[1], st));
        rc = run(h, p, st, &launches);
        if (rc != B200ODE_OK) return rc;
        CUDA_TRY(cudaEventRecord(h->ev[2], st));
        if (stats) {
            rc = add_totals(h, h->d_ctl, stats, st);
            if (rc != B200ODE_OK) return rc;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]);
            kernel_ms += ms;
        }
    }
    if (stats) {
        stats->kernel_ms = kernel_ms;
        stats->h2d_ms = stats->d2h_ms = 0.0;
        stats->gpu_launches = launches;
    }
    return B200ODE_OK;
}

b200ode_status b200ode_integrate(b200ode_handle* h, int64_t n, const double* P, double Ps, double* T,
                                 double* Y, double t0, double t1, int32_t* cell_status,
                                 b200ode_stats* stats) {
    NvtxRange range("b200ode_integrate");
    b200ode_status rc = check_args(h, n, t0, t1);
    if (rc != B200ODE_OK) return rc;
    if (stats) clear_totals(stats);
    if (n == 0) return B200ODE_OK;
    if (!T || !Y) return fail(B200ODE_ERR_INVALID, "null T or Y");
    if (!P && !(Ps > 0.0)) return fail(B200ODE_ERR_INVALID, "pressure must be > 0");
    const size_t nsp = h->hm.nsp;
    // the handle's device buffers hold one chunk: the whole batch when it fits
    // in device memory, else memory-sized chunks copied in and out in turn
    const size_t io_per_cell = (nsp + 2) * sizeof(double) + 8 * sizeof(int32_t);
    const int64_t chunk = cells_per_launch(h, n, io_per_cell);
    rc = ensure_cap(h, (size_t)chunk);
    if (rc != B200ODE_OK) return rc;
    cudaStream_t st = h->stream;
    const bool want_cnt = stats && (stats->nst || stats->nfe || stats->nje || stats->nsetups ||
                                    stats->nni || stats->ncfn || stats->netf);
    int32_t* dst[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (want_cnt) {
        int32_t* d[7] = {stats->nst, stats->nfe, stats->nje, stats->nsetups, stats->nni, stats->ncfn, stats->netf};
        for (int i = 0; i < 7; ++i) dst[i] = d[i];
    }
    int launches = 0;
    float t_h2d = 0.f, t_kernel = 0.f, t_d2h = 0.f;
    for (int64_t a = 0; a < n; a += chunk) {
        const int64_t m = std::min(chunk, n - a);
        {
            NvtxRange h2d_range("h2d");
            CUDA_TRY(cudaEventRecord(h->ev[0], st));
            CUDA_TRY(cudaMemcpyAsync(h->d_T, T + a, m * sizeof(double), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpy2DAsync(h->d_Y, m * sizeof(double), Y + a, n * sizeof(double), m * sizeof(double),
                                       nsp, cudaMemcpyHostToDevice, st));
            if (P) CUDA_TRY(cudaMemcpyAsync(h->d_P, P + a, m * sizeof(double), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaEventRecord(h->ev[1], st));
        }
        int32_t* dcnt[7];
        for (int i = 0; i < 7; ++i) dcnt[i] = want_cnt ? h->d_cnt + (size_t)i * m : nullptr;
        KParams p;
        fill_params(h, p, m, P ? h->d_P : nullptr, Ps, h->d_T, h->d_Y, h->d_status, dcnt, t0, t1);
        rc = run(h, p, st, &launches);
        if (rc != B200ODE_OK) return rc;
        CUDA_TRY(cudaEventRecord(h->ev[2], st));
        CUDA_TRY(cudaMemcpyAsync(T + a, h->d_T, m * sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpy2DAsync(Y + a, n * sizeof(double), h->d_Y, m * sizeof(double), m * sizeof(double), nsp,
                                   cudaMemcpyDeviceToHost, st));
        if (cell_status)
            CUDA_TRY(cudaMemcpyAsync(cell_status + a, h->d_status, m * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        for (int i = 0; i < 7; ++i)
            if (dst[i])
                CUDA_TRY(cudaMemcpyAsync(dst[i] + a, h->d_cnt + (size_t)i * m, m * sizeof(int32_t),
                                         cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaEventRecord(h->ev[3], st));
        {
            NvtxRange wait("device (copies + BDF kernel)");
            CUDA_TRY(cudaStreamSynchronize(st));
        }
        if (stats) {
            rc = add_totals(h, h->d_ctl, stats, st);
            if (rc != B200ODE_OK) return rc;
            float x = 0.f, y = 0.f, z = 0.f;
            cudaEventElapsedTime(&x, h->ev[0], h->ev[1]);
            cudaEventElapsedTime(&y, h->ev[1], h->ev[2]);
            cudaEventElapsedTime(&z, h->ev[2], h->ev[3]);
            t_h2d += x;
            t_kernel += y;
            t_d2h += z;
        }
    }
    if (stats) {
        stats->h2d_ms = t_h2d;
        stats->kernel_ms = t_kernel;
        stats->d2h_ms = t_d2h;
        stats->gpu_launches = launches;
    }
    return B200ODE_OK;
}

static b200ode_status eval_chem(b200ode_handle* h, int64_t n, const double* P, double Ps, const double* T,
                                const double* Y, double* dTdt, double* dYdt, double* jac) {
    b200ode_status rc = check_args(h, n, 0.0, 0.0);
    if (rc != B200ODE_OK) return rc;
    if (n == 0) return B200ODE_OK;
    if (!T || !Y || (!jac && (!dTdt || !dYdt))) return fail(B200ODE_ERR_INVALID, "null buffer");
    if (!P && !(Ps > 0.0)) return fail(B200ODE_ERR_INVALID, "pressure must be > 0");
    rc = ensure_cap(h, (size_t)n);
    if (rc != B200ODE_OK) return rc;
    cudaStream_t st = h->stream;
    const size_t N = h->hm.nsp;
    CUDA_TRY(cudaMemcpyAsync(h->d_T, T, n * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(h->d_Y, Y, n * N * sizeof(double), cudaMemcpyHostToDevice, st));
    if (P) CUDA_TRY(cudaMemcpyAsync(h->d_P, P, n * sizeof(double), cudaMemcpyHostToDevice, st));
    KParams p;
    fill_params(h, p, n, P ? h->d_P : nullptr, Ps, h->d_T, h->d_Y, nullptr, nullptr, 0.0, 0.0);
    double* d_out = nullptr;
    const size_t out_elems = jac ? (size_t)n * N * N : (size_t)n * (N - 1) + n;
    CUDA_TRY(cudaMallocAsync(&d_out, out_elems * sizeof(double), st));
    double* d_dT = jac ? nullptr : d_out;
    double* d_dY = jac ? nullptr : d_out + n;
    double* d_jac = jac ? d_out : nullptr;
    rc = dispatch_mech(h, [&](auto mt, auto lt) {
        return launch_eval<decltype(mt), decltype(lt)>(h, p, d_dT, d_dY, d_jac, st);
    });
    if (rc == B200ODE_OK) {
        if (jac) {
            CUDA_TRY(cudaMemcpyAsync(jac, d_out, out_elems * sizeof(double), cudaMemcpyDeviceToHost, st));
        } else {
            CUDA_TRY(cudaMemcpyAsync(dTdt, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(cudaMemcpyAsync(dYdt, d_out + n, n * (N - 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
    }
    cudaFreeAsync(d_out, st);
    CUDA_TRY(cudaStreamSynchronize(st));
    return rc;
}

b200ode_status b200ode_eval_enthalpy_device(b200ode_handle* h, int64_t n, const double* dT, const double* dY,
                                            double* dh, void* stream) {
    b200ode_status rc = check_args(h, n, 0.0, 0.0);
    if (rc != B200ODE_OK) return rc;
    if (n == 0) return B200ODE_OK;
    if (!dT || !dY || !dh) return fail(B200ODE_ERR_INVALID, "null buffer");
    NvtxRange range("b200ode_eval_enthalpy");
    const unsigned blocks = (unsigned)((n + 255) / 256);
    cudaStream_t st = (cudaStream_t)stream;
    dispatch_mech(h, [&](auto mt, auto) {
        k_enthalpy<decltype(mt)><<<blocks, 256, 0, st>>>(n, dT, dY, dh);
        return B200ODE_OK;
    });
    CUDA_TRY(cudaGetLastError());
    return B200ODE_OK;
}

b200ode_status b200ode_eval_enthalpy(b200ode_handle* h, int64_t n, const double* T, const double* Y, double* hmass) {
    b200ode_status rc = check_args(h, n, 0.0, 0.0);
    if (rc != B200ODE_OK) return rc;
    if (n == 0) return B200ODE_OK;
    if (!T || !Y || !hmass) return fail(B200ODE_ERR_INVALID, "null buffer");
    rc = ensure_cap(h, (size_t)n);
    if (rc != B200ODE_OK) return rc;
    cudaStream_t st = h->stream;
    const size_t nsp = h->hm.nsp;
    CUDA_TRY(cudaMemcpyAsync(h->d_T, T, n * sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(h->d_Y, Y, n * nsp * sizeof(double), cudaMemcpyHostToDevice, st));
    rc = b200ode_eval_enthalpy_device(h, n, h->d_T, h->d_Y, h->d_P, st);   // d_P as the output scratch
    if (rc != B200ODE_OK) return rc;
    CUDA_TRY(cudaMemcpyAsync(hmass, h->d_P, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return B200ODE_OK;
}

b200ode_status b200ode_eval_rhs(b200ode_handle* h, int64_t n, const double* P, double Ps, const double* T,
                                const double* Y, double* dTdt, double* dYdt) {
    return eval_chem(h, n, P, Ps, T, Y, dTdt, dYdt, nullptr);
}

b200ode_status b200ode_eval_jacobian(b200ode_handle* h, int64_t n, const double* P, double Ps,
                                     const double* T, const double* Y, double* jac) {
    if (!jac) return fail(B200ODE_ERR_INVALID, "null jac");
    return eval_chem(h, n, P, Ps, T, Y, nullptr, nullptr, jac);
}

b200ode_status b200ode_autotune(b200ode_handle* h, int64_t n, const double* dP, double Ps, const double* dT,
                                const double* dY, double t0, double t1, int32_t* wpb_out, int32_t* bps_out) {
    b200ode_status rc = check_args(h, n, t0, t1);
    if (rc != B200ODE_OK) return rc;
    if (n <= 0 || !dT || !dY) return fail(B200ODE_ERR_INVALID, "autotune needs cells (device T and Y)");
    if (!dP && !(Ps > 0.0)) return fail(B200ODE_ERR_INVALID, "pressure must be > 0");
    const bool wide_mech = (h->mech == MECH_ESTIMATE);   // one cell per SM: helper warps on or off
    // the sample: the first m cells -- 192 per SM, about 16 per resident warp, so
    // that the timing reflects the work queue's steady state rather than its
    // tail (two per SM for the widest mechanism, whose cells take seconds) --
    // copied so the caller's buffers stay untouched
    const int64_t m = std::min<int64_t>(n, (wide_mech ? 2 : 192) * (int64_t)h->num_sms);
    const size_t nsp = h->hm.nsp;
    rc = ensure_cap(h, (size_t)m);
    if (rc != B200ODE_OK) return rc;
    cudaStream_t st = h->stream;
    int smem_optin = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    double *sT = nullptr, *sY = nullptr;
    CUDA_TRY(cudaMallocAsync(&sT, m * sizeof(double), st));
    CUDA_TRY(cudaMallocAsync(&sY, m * nsp * sizeof(double), st));
    CUDA_TRY(cudaMemcpyAsync(sT, dT, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CUDA_TRY(cudaMemcpy2DAsync(sY, m * sizeof(double), dY, n * sizeof(double), m * sizeof(double), nsp,
                               cudaMemcpyDeviceToDevice, st));
    if (dP) CUDA_TRY(cudaMemcpyAsync(h->d_P, dP, m * sizeof(double), cudaMemcpyDeviceToDevice, st));
    const b200ode_options saved = h->opt;
    h->opt.persistent = 1;
    // best of two timed persistent runs of the sample under the handle's current options
    auto time_opts = [&](float* out_ms) -> b200ode_status {
        float ms_c = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            if (cudaMemcpyAsync(h->d_T, sT, m * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(h->d_Y, sY, m * nsp * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return fail(B200ODE_ERR_CUDA, "autotune: sample copy");
            KParams p;
            fill_params(h, p, m, dP ? h->d_P : nullptr, Ps, h->d_T, h->d_Y, h->d_status, nullptr, t0, t1);
            int launches = 0;
            if (cudaEventRecord(h->ev[1], st) != cudaSuccess) return fail(B200ODE_ERR_CUDA, "event");
            b200ode_status r = run(h, p, st, &launches);
            if (r != B200ODE_OK) return r;
            cudaEventRecord(h->ev[2], st);
            if (cudaEventSynchronize(h->ev[2]) != cudaSuccess) return fail(B200ODE_ERR_CUDA, "autotune run");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]);
            ms_c = std::min(ms_c, ms);
        }
        *out_ms = ms_c;
        return B200ODE_OK;
    };
    // stage 1, the launch shape: warps per CTA (4, 2, 1) x register variant
    // (blocks_per_sm = 0: the variant that keeps the most CTAs resident;
    // blocks_per_sm = 3 * 4 / wpb: the 168-register one, which trades spills
    // for resident warps) x threads per cell for the widest
    // mechanism (a 4-warp CTA per cell with helper warps, or one warp); shapes
    // whose shared memory exceeds a CTA's are skipped
    struct Cand { int wpb, bps, helpers, chunk; };
    std::vector<Cand> shapes;
    for (int wpb : {4, 2, 1})
        for (int v = 0; v < 2; ++v)
            for (int helpers : {1, 0}) {
                if (helpers == 0 && !(wide_mech && wpb == 1)) continue;
                shapes.push_back({wpb, v ? 3 * (4 / wpb) : 0, helpers, 1});
            }
    float best_ms = 0.f;
    Cand best{0, 0, 0, 0};
    bool have = false;
    for (const Cand& c : shapes) {
        if (rc != B200ODE_OK) break;
        h->opt.warps_per_block = c.wpb;
        h->opt.blocks_per_sm = c.bps;
        h->opt.cta_helpers = c.helpers;
        h->opt.queue_chunk = 1;
        size_t warp_smem = 0;
        dispatch_mech(h, [&](auto mt, auto lt) {
            warp_smem = warp_smem_bytes<decltype(mt), decltype(lt)>();
            return B200ODE_OK;
        });
        if ((size_t)c.wpb * warp_smem > (size_t)smem_optin) continue;
        float ms = 0.f;
        rc = time_opts(&ms);
        if (rc == B200ODE_OK && (!have || ms < best_ms)) {
            best_ms = ms;
            best = c;
            have = true;
        }
    }
    // stage 2, the work-queue chunk (cells a warp claims per queue access) on
    // the chosen shape
    if (rc == B200ODE_OK && have) {
        h->opt.warps_per_block = best.wpb;
        h->opt.blocks_per_sm = best.bps;
        h->opt.cta_helpers = best.helpers;
        for (int chunk : {2, 8}) {
            h->opt.queue_chunk = chunk;
            float ms = 0.f;
            rc = time_opts(&ms);
            if (rc != B200ODE_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best.chunk = chunk;
            }
        }
    }
    cudaFreeAsync(sT, st);
    cudaFreeAsync(sY, st);
    cudaStreamSynchronize(st);
    h->opt = saved;
    if (rc != B200ODE_OK) return rc;
    if (!have) return fail(B200ODE_ERR_CUDA, "autotune: no launch shape fits this device");
    h->opt.warps_per_block = best.wpb;
    h->opt.blocks_per_sm = best.bps;
    h->opt.cta_helpers = best.helpers;
    h->opt.queue_chunk = best.chunk;
    if (wpb_out) *wpb_out = best.wpb;
    if (bps_out) *bps_out = best.bps;
    return B200ODE_OK;
}

b200ode_status b200ode_get_options(const b200ode_handle* h, b200ode_options* out) {
    if (!h || !out) return fail(B200ODE_ERR_INVALID, "null handle or output");
    *out = h->opt;
    return B200ODE_OK;
}

b200ode_status b200ode_fp32_peak(int32_t device, double* gflops) {
    if (!gflops) return fail(B200ODE_ERR_INVALID, "null output");
    if (device >= 0) CUDA_TRY(cudaSetDevice(device));
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    float* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(float)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int iters = 4096, threads = 256, blocks = sms * 8;
    k_fp32_peak<<<blocks, threads>>>(d, 16);
    cudaEventRecord(a);
    k_fp32_peak<<<blocks, threads>>>(d, iters);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return fail(B200ODE_ERR_CUDA, cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    *gflops = flops / (ms * 1e-3) / 1e9;
    return B200ODE_OK;
}

b200ode_status b200ode_fp64_peak(int32_t device, double* gflops) {
    if (!gflops) return fail(B200ODE_ERR_INVALID, "null output");
    if (device >= 0) CUDA_TRY(cudaSetDevice(device));
    int dev = 0, sms = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double* d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(double)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int iters = 2048, threads = 256, blocks = sms * 8;
    k_fp64_peak<<<blocks, threads>>>(d, 16);
    cudaEventRecord(a);
    k_fp64_peak<<<blocks, threads>>>(d, iters);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return fail(B200ODE_ERR_CUDA, cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    *gflops = flops / (ms * 1e-3) / 1e9;
    return B200ODE_OK;
}

}  // extern "C"

// ------------------------------------------- no-allocation entry point
// b200ode_integrate_device_noalloc runs the persistent BDF kernel with all of
// its device scratch in one file-scope array instead of the handle's cudaMalloc'd
// buffers.  It serves callers that must not allocate device memory while they
// integrate: a flow solver whose own pool has taken the whole device at start-up,
// or one that cannot accept the device-wide synchronization of cudaFree (which
// b200ode_integrate_device issues when a larger launch outgrows the handle's
// scratch) in the middle of its time step.
//
// Layout of the array: bytes [0, 256) are the control block (work-queue head,
// 8 call totals, 5 phase-cycle totals), which every call clears before its
// launch; from byte 256 on, one WarpGlobal (saved Newton Jacobian and Jacobian
// rate scratch) per resident warp, which the kernel writes before it reads, so
// the previous call's contents there do no harm.  The array exists once per
// device that loads this library and stays reserved until the process exits.
// Every call on a device uses the same array: calls that overlap on the GPU
// (different streams, handles or host threads without ordering) race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[B200ODE_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr size_t kNoAllocCtlBytes = 256;
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on `device`, which must be current.  The
// host-side name g_noalloc_scratch is only a handle for the runtime; the address
// is looked up once per device (the first call there) and kept.
b200ode_status noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices)
        return fail(B200ODE_ERR_INVALID, "b200ode_integrate_device_noalloc: device ordinal " +
                                             std::to_string(device) + " out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(B200ODE_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                              cudaGetErrorString(e));
        g_noalloc_ptr[device] = static_cast<unsigned char*>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return B200ODE_OK;
}

// Makes `device` current for the lifetime of the guard, then restores the
// caller's device.
struct NoAllocDeviceGuard {
    int prev = -1;
    cudaError_t enter(int device) {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) { prev = -1; return e; }
        if (prev == device) { prev = -1; return cudaSuccess; }
        return cudaSetDevice(device);
    }
    ~NoAllocDeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// Same launch shape as the persistent branch of launch_bdf -- CTA size from
// bdf_threads (one 128-thread CTA per cell when the widest mechanisms' helper
// warps serve), blocks from occupancy -- so both entry points run identical
// grids, with queue, totals and per-warp scratch in the array.  With helper
// warps the per-cell scratch index is the CTA index (one cell per CTA), so the
// scratch stays blocks x wpb WarpGlobals.
template <class MT, class LinT>
b200ode_status launch_bdf_noalloc(b200ode_handle* h, KParams& p, unsigned char* scratch, cudaStream_t st,
                                  int* launches) {
    using WG = WarpGlobal<MT, LinT>;
    const int wpb = pick_wpb<MT, LinT>(h);
    const size_t smem = warp_smem_bytes<MT, LinT>() * wpb;
    auto kern = bdf_kernel<MT, LinT>(h, wpb);
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int threads = bdf_threads<MT>(h, wpb);
    int bps = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, smem));
    if (bps < 1) return fail(B200ODE_ERR_CUDA, "kernel does not fit on an SM");
    if (h->opt.blocks_per_sm > 0) bps = std::min(bps, h->opt.blocks_per_sm);
    const size_t n = (size_t)p.ncells;
    const long long cpb = cells_per_block<MT>(wpb);
    long long blocks = (long long)bps * h->num_sms;
    blocks = std::max(1LL, std::min(blocks, ((long long)n + cpb - 1) / cpb));
    const size_t need = kNoAllocCtlBytes + (size_t)(blocks * cpb) * sizeof(WG);
    if (need > (size_t)B200ODE_NOALLOC_SCRATCH_BYTES)
        return fail(B200ODE_ERR_INVALID,
                    "b200ode_integrate_device_noalloc: this launch needs " + std::to_string(need) +
                        " bytes of scratch (" + std::to_string(blocks) + " blocks x " + std::to_string(cpb) +
                        " cells x " + std::to_string(sizeof(WG)) + " bytes + 256) but the static scratch holds " +
                        std::to_string((size_t)B200ODE_NOALLOC_SCRATCH_BYTES) +
                        " bytes; lower options.blocks_per_sm or options.warps_per_block");
    h->last_blocks_per_sm = bps;
    auto* ctl = reinterpret_cast<unsigned long long*>(scratch);
    CUDA_TRY(cudaMemsetAsync(ctl, 0, kNoAllocCtlBytes, st));
    p.queue = ctl;
    p.totals = ctl + 1;
    p.done_count = ctl + 9;
    p.prof = h->opt.profile_phases ? ctl + 10 : nullptr;
    p.wglobal = scratch + kNoAllocCtlBytes;
    p.records = nullptr;
    p.steps = 0x7fffffff;
    kern<<<(unsigned)blocks, threads, smem, st>>>(p);
    CUDA_TRY(cudaGetLastError());
    *launches += 1;
    return B200ODE_OK;
}

}  // namespace

extern "C" b200ode_status b200ode_integrate_device_noalloc(b200ode_handle* h, int64_t n, const double* dP,
                                                           double Ps, double* dT, double* dY, double t0,
                                                           double t1, int32_t* dstat, b200ode_stats* stats,
                                                           void* stream) {
    b200ode_status rc = check_args(h, n, t0, t1);
    if (rc != B200ODE_OK) return rc;
    int32_t* dcnt[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (stats) {
        int32_t* keep[7] = {stats->nst, stats->nfe, stats->nje, stats->nsetups, stats->nni, stats->ncfn, stats->netf};
        std::memset(stats, 0, sizeof(*stats));
        stats->nst = keep[0]; stats->nfe = keep[1]; stats->nje = keep[2]; stats->nsetups = keep[3];
        stats->nni = keep[4]; stats->ncfn = keep[5]; stats->netf = keep[6];
        for (int i = 0; i < 7; ++i) dcnt[i] = keep[i];
    }
    if (n == 0) return B200ODE_OK;
    if (!dT || !dY) return fail(B200ODE_ERR_INVALID, "null T or Y");
    if (!dP && !(Ps > 0.0)) return fail(B200ODE_ERR_INVALID, "pressure must be > 0");
    NoAllocDeviceGuard guard;
    CUDA_TRY(guard.enter(h->device));
    unsigned char* scratch = nullptr;
    rc = noalloc_scratch(h->device, &scratch);
    if (rc != B200ODE_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    KParams p;
    fill_params(h, p, n, dP, Ps, dT, dY, dstat, dcnt, t0, t1);
    int launches = 0;
    CUDA_TRY(cudaEventRecord(h->ev[1], st));
    rc = dispatch_mech(h, [&](auto mt, auto lt) {
        return launch_bdf_noalloc<decltype(mt), decltype(lt)>(h, p, scratch, st, &launches);
    });
    if (rc != B200ODE_OK) return rc;
    CUDA_TRY(cudaEventRecord(h->ev[2], st));
    if (stats) {
        unsigned long long t[15];
        CUDA_TRY(cudaMemcpyAsync(t, scratch + sizeof(unsigned long long), sizeof(t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < 5; ++i) stats->phase_cycles[i] = h->opt.profile_phases ? (int64_t)t[9 + i] : 0;
        stats->total_nst = (int64_t)t[0]; stats->total_nfe = (int64_t)t[1]; stats->total_nje = (int64_t)t[2];
        stats->total_nsetups = (int64_t)t[3]; stats->total_nni = (int64_t)t[4]; stats->total_ncfn = (int64_t)t[5];
        stats->total_netf = (int64_t)t[6]; stats->n_failed = (int64_t)t[7];
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev[1], h->ev[2]);
        stats->kernel_ms = ms;
        stats->gpu_launches = launches;
    }
    return B200ODE_OK;
}
