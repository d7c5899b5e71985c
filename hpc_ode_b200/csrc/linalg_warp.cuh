// Warp-per-cell dense LU with partial pivoting and triangular solves for the
// Newton matrix M = I - gamma*J of one cell (N x N, N = 53 for GRI-Mech 3.0).
//
// Replaces, for one cell, MAGMA's batched getrf/getrs behind SUNDIALS'
// SUNLinSol_MagmaDense (ext/magma-2.6.2/src/dgetrf_batched.cpp:82-230,
// dgetrs_batched.cpp:87-190; used at src/Integrators/CVodeIntegratorGPU.cpp:86-90)
// and SUNDIALS' serial dense getrf/getrs on the CPU path
// (SUNLinSol_Dense, CVodeIntegrator.cpp:127-131).  Same factorization: row
// interchanges chosen as the first index of the largest |a_ik| in column k,
// multipliers scaled by the reciprocal of the pivot, unit-lower L and upper U
// stored in place.
//
// Layout: A row-major in shared memory with an odd leading dimension, so
// that 32 lanes reading one column (different rows) or one row (different
// columns) hit 32 distinct banks.  The matrix type LinT is float in the
// mixed-precision form and double in the FP64 form; right-hand sides arrive
// and leave in FP64.
#pragma once

#include "chem_warp.cuh"

namespace b200 {

template <class T>
__device__ __forceinline__ T absT(T v) { return v < T(0) ? -v : v; }

// Trailing update A22 -= L21 U12 of the blocked LU after panel [k0, kend) for
// the columns j = lane + 32 s of the slots s with s % nw == w (nw warps share
// the columns; nw = 1: all).  The block rows' entries u are read from A (row
// k0 as the panel left it, rows k0+1.. as U12 stored them); rows go in batches
// of kRows whose multipliers and entries are loaded before any store.  Each
// element receives the same fused multiply-adds in the same order whichever
// warp updates it, so splitting the columns does not change the factors.
template <class MT, class LinT>
__device__ __forceinline__ void lu_trailing(LinT* A, int k0, int kend, int lane, int w, int nw) {
    static_assert(MT::G == 32, "the blocked LU serves one cell per warp");
    constexpr int N = MT::N, LDA = MT::LDA, NS = MT::NS;
    constexpr int kPanel = 4;
    constexpr int kRows = sizeof(LinT) == 4 ? 8 : 4;
    LinT u[kPanel][NS];
    bool on[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int j = lane + 32 * s;
        const bool mine = j >= kend && j < N && (s % nw) == w;
        bool nz = false;
#pragma unroll
        for (int r = 0; r < kPanel; ++r) {
            u[r][s] = (mine && k0 + r < kend) ? A[(k0 + r) * LDA + j] : LinT(0);
            nz = nz || (u[r][s] != LinT(0));
        }
        on[s] = mine && nz;   // columns with a zero U12 block need no update
    }
#pragma unroll 1
    for (int i0 = kend; i0 < N; i0 += kRows) {
        const int nr = min(kRows, N - i0);
        LinT l[kRows][kPanel];
#pragma unroll
        for (int rr = 0; rr < kRows; ++rr)
#pragma unroll
            for (int q = 0; q < kPanel; ++q)
                l[rr][q] = (rr < nr && k0 + q < kend) ? A[(i0 + rr) * LDA + k0 + q] : LinT(0);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            if (on[s]) {
                const int j = lane + 32 * s;
                LinT a[kRows];
#pragma unroll
                for (int rr = 0; rr < kRows; ++rr)
                    if (rr < nr) a[rr] = A[(i0 + rr) * LDA + j];
#pragma unroll
                for (int q = 0; q < kPanel; ++q) {
                    if (u[q][s] != LinT(0)) {
#pragma unroll
                        for (int rr = 0; rr < kRows; ++rr) a[rr] = a[rr] - l[rr][q] * u[q][s];
                    }
                }
#pragma unroll
                for (int rr = 0; rr < kRows; ++rr)
                    if (rr < nr) A[(i0 + rr) * LDA + j] = a[rr];
            }
        }
    }
}

// The trailing update run by warp 0, with the CTA's helper warps taking their
// share of the columns when they serve it (mechanisms of kWideN+ unknowns).
template <class MT, class LinT>
__device__ __forceinline__ void lu_trailing_forked(unsigned A_off, int k0, int kend, int lane) {
    LinT* A = smem_at<LinT>(A_off);
    if constexpr (MT::N >= kWideN) {
        HelperCtl* h = &g_helper_ctl;
        if (h->nhelpers == kHelperWarps) {
            if (lane == 0) {
                h->A_off = A_off;
                h->k0 = k0;
                h->kend = kend;
            }
            helpers_post(h, kCmdLu, lane);
            lu_trailing<MT, LinT>(A, k0, kend, lane, 0, kHelperWarps + 1);
            helpers_join(h, lane);
            return;
        }
    }
    lu_trailing<MT, LinT>(A, k0, kend, lane, 0, 1);
}

// LU factorization in place (both forms below give the same factors).  perm =
// the composed row permutation ((P b)[i] = b[perm[i]]); the diagonal holds
// 1 / U_kk (no step reads U_kk once its column's multipliers are formed).
// Returns 0, or k+1 if U_kk == 0 (singular).  All 32 lanes call it.
//
// Blocked form, in LAPACK's getrf order: a panel of kPanel columns is factored with
// partial pivoting (full rows swapped), then the panel's block rows right of
// it are eliminated (U12 = L11^-1 A12) and the trailing matrix gets one
// rank-kPanel update.  Every element receives the same fused multiply-adds in
// the same order as in the unblocked right-looking factorization, so the
// factors are the same; the rank-kPanel update loads and stores each trailing
// element once per panel instead of once per column.
//
// Every loop that stores into A first loads all it needs (registers), then
// stores: the compiler may not move a load above a store to the same array,
// so load-store-load chains would wait out the full shared-memory latency
// once per element (with one warp per SM for the largest mechanisms, nothing
// else hides it).
template <class MT, class LinT>
__device__ __forceinline__ int warp_lu_blocked(unsigned A_off, unsigned perm_off, int lane) {
    static_assert(MT::G == 32, "the blocked LU serves one cell per warp");
    constexpr int N = MT::N, LDA = MT::LDA, NS = MT::NS;
    constexpr int kPanel = 4;                               // panel width
    constexpr int kRows = sizeof(LinT) == 4 ? 8 : 4;        // rows per trailing-update batch
    static_assert(N <= 256, "perm holds bytes");
    LinT* A = smem_at<LinT>(A_off);
    unsigned char* perm = smem_at<unsigned char>(perm_off);
    int sing = 0;
    int pv[NS];   // lane tracks perm[i] for i = lane + 32 s
#pragma unroll
    for (int s = 0; s < NS; ++s) pv[s] = lane + 32 * s;
#pragma unroll 1
    for (int k0 = 0; k0 < N; k0 += kPanel) {
        const int kend = min(k0 + kPanel, N);
        // ---- 1. panel: columns [k0, kend), rows >= k
#pragma unroll 1
        for (int k = k0; k < kend; ++k) {
            // pivot: first index of the max |a_ik|, i >= k
            LinT best = LinT(-1);
            int bi = N;
            for (int i = k + lane; i < N; i += 32) {
                const LinT v = absT(A[i * LDA + k]);
                if (v > best) { best = v; bi = i; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const LinT ov = __shfl_xor_sync(kFull, best, o);
                const int oi = __shfl_xor_sync(kFull, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (!(best > LinT(0))) { sing = k + 1; break; }   // zero (or NaN) pivot
            if (bi != k) {   // swap the full rows k and bi
                LinT rk[NS], rb[NS];
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const int j = lane + 32 * s;
                    if (j < N) { rk[s] = A[k * LDA + j]; rb[s] = A[bi * LDA + j]; }
                }
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const int j = lane + 32 * s;
                    if (j < N) { A[k * LDA + j] = rb[s]; A[bi * LDA + j] = rk[s]; }
                }
                // compose the permutation: swap entries k and bi
                const int ok = __shfl_sync(kFull, pick<NS>(pv, k >> 5), k & 31);
                const int ob = __shfl_sync(kFull, pick<NS>(pv, bi >> 5), bi & 31);
                if (lane == (k & 31)) place<NS>(pv, k >> 5, ob);
                if (lane == (bi & 31)) place<NS>(pv, bi >> 5, ok);
                __syncwarp();
            }
            const LinT inv = LinT(1) / A[k * LDA + k];
            // multipliers (column k below the diagonal), then the panel's
            // columns right of k; lane owns rows i = k + 1 + lane + 32 t
            LinT ukj[kPanel - 1];
#pragma unroll
            for (int q = 0; q < kPanel - 1; ++q)
                ukj[q] = (k + 1 + q < kend) ? A[k * LDA + k + 1 + q] : LinT(0);
#pragma unroll
            for (int t = 0; t < NS; ++t) {
                const int i = k + 1 + lane + 32 * t;
                if (i < N) {
                    const LinT lik = A[i * LDA + k] * inv;
                    LinT a[kPanel - 1];
#pragma unroll
                    for (int q = 0; q < kPanel - 1; ++q)
                        if (k + 1 + q < kend) a[q] = A[i * LDA + k + 1 + q];
                    A[i * LDA + k] = lik;
#pragma unroll
                    for (int q = 0; q < kPanel - 1; ++q)
                        if (k + 1 + q < kend && ukj[q] != LinT(0)) A[i * LDA + k + 1 + q] = a[q] - lik * ukj[q];
                }
            }
            __syncwarp();   // every lane has read U_kk
            if (lane == 0) A[k * LDA + k] = inv;
        }
        if (sing || kend >= N) break;
        // ---- 2. block rows right of the panel: U12 = L11^-1 A12 (lane owns
        // columns j = lane + 32 s >= kend; rows in registers)
        LinT u[kPanel][NS];
        bool on[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = lane + 32 * s;
            on[s] = j >= kend && j < N;
#pragma unroll
            for (int r = 0; r < kPanel; ++r) u[r][s] = (on[s] && k0 + r < kend) ? A[(k0 + r) * LDA + j] : LinT(0);
        }
#pragma unroll
        for (int r = 1; r < kPanel; ++r) {
            if (k0 + r < kend) {
#pragma unroll
                for (int q = 0; q < r; ++q) {
                    const LinT lrq = A[(k0 + r) * LDA + k0 + q];
#pragma unroll
                    for (int s = 0; s < NS; ++s)
                        if (u[q][s] != LinT(0)) u[r][s] = u[r][s] - lrq * u[q][s];
                }
            }
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int j = lane + 32 * s;
            if (on[s]) {
#pragma unroll
                for (int r = 1; r < kPanel; ++r)
                    if (k0 + r < kend) A[(k0 + r) * LDA + j] = u[r][s];
            }
        }
        __syncwarp();
        // ---- 3. trailing update A22 -= L21 U12 (split over the CTA's helper warps
        // when they serve this warp, see lu_trailing)
        lu_trailing_forked<MT, LinT>(A_off, k0, kend, lane);
        __syncwarp();
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if (lane + 32 * s < N) perm[lane + 32 * s] = pv[s];
    __syncwarp();
    return sing;
}

// Matrices from this size up take the batched rank-1 update in the compact form.
constexpr int kBatchedUpdateMinN = 32;

// The unblocked right-looking form of the same factorization (row by row,
// one rank-1 update per column): the smallest code.  With several warps per
// SM the latency it exposes is hidden by the other warps, and the kernels of
// the small mechanisms are bound by instruction fetch, where the blocked
// form's larger code costs more than it saves.
template <class MT, class LinT>
__device__ __forceinline__ int warp_lu_compact(unsigned A_off, unsigned perm_off, int lane) {
    constexpr int N = MT::N, LDA = MT::LDA, NS = MT::NS, G = MT::G;
    const unsigned gm = gmask<G>();
    static_assert(N <= 256, "perm holds bytes");
    LinT* A = smem_at<LinT>(A_off);
    unsigned char* perm = smem_at<unsigned char>(perm_off);
    int sing = 0;
    int pv[NS];   // lane tracks perm[i] for i = lane + G s
#pragma unroll
    for (int s = 0; s < NS; ++s) pv[s] = lane + G * s;
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
        LinT best = LinT(-1);
        int bi = N;
        for (int i = k + lane; i < N; i += G) {
            const LinT v = absT(A[i * LDA + k]);
            if (v > best) { best = v; bi = i; }
        }
        if constexpr (sizeof(LinT) == 4) {
            // FP32: two warp reductions instead of a shuffle tree.  The bits of
            // a non-negative float order as the floats do (the sign bit cleared:
            // M holds -0.0 wherever gamma scaled a zero of J); key 0 = no
            // candidate on this lane (none, or only NaN), so a key <= 1 means no
            // pivot > 0.
            const unsigned key = (best >= LinT(0)) ? __float_as_uint(fabsf((float)best)) + 1u : 0u;
            const unsigned kmax = __reduce_max_sync(gm, key);
            if (kmax <= 1u) { sing = k + 1; break; }   // zero (or NaN) pivot
            // first index of the maximum: the smallest row among the lanes holding it
            bi = (int)__reduce_min_sync(gm, key == kmax ? (unsigned)bi : (unsigned)N);
        } else {
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                const LinT ov = __shfl_xor_sync(gm, best, o, G);
                const int oi = __shfl_xor_sync(gm, bi, o, G);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (!(best > LinT(0))) { sing = k + 1; break; }   // zero (or NaN) pivot
        }
        if (bi != k) {
#pragma unroll 1
            for (int j = lane; j < N; j += G) {
                const LinT t = A[k * LDA + j];
                A[k * LDA + j] = A[bi * LDA + j];
                A[bi * LDA + j] = t;
            }
            const int ok = group_shfl<G>(pick<NS>(pv, k / G), k % G);
            const int ob = group_shfl<G>(pick<NS>(pv, bi / G), bi % G);
            if (lane == (k % G)) place<NS>(pv, k / G, ob);
            if (lane == (bi % G)) place<NS>(pv, bi / G, ok);
            __syncwarp(gm);
        }
        const LinT inv = LinT(1) / A[k * LDA + k];
        for (int i = k + 1 + lane; i < N; i += G) A[i * LDA + k] *= inv;
        __syncwarp(gm);   // every lane has read U_kk
        if (lane == 0) A[k * LDA + k] = inv;
        // rank-1 update of the trailing block; lane owns columns j = lane + G s > k.
        if constexpr (N >= kBatchedUpdateMinN) {
            // rows in batches of kRows whose multipliers and entries are all
            // loaded before any store (a load may not pass a store to the same
            // array, so element-by-element updates would each wait out the full
            // shared-memory latency); every element gets the same single fused
            // multiply-add as in the element-wise form below
            constexpr int kRows = 8;
            LinT u[NS];
            bool on[NS];
            bool any = false;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int j = lane + G * s;
                u[s] = (j > k && j < N) ? A[k * LDA + j] : LinT(0);
                on[s] = u[s] != LinT(0);
                any = any || on[s];
            }
            if (__any_sync(gm, any)) {
#pragma unroll 1
                for (int i0 = k + 1; i0 < N; i0 += kRows) {
                    LinT l[kRows];
#pragma unroll
                    for (int r = 0; r < kRows; ++r) l[r] = (i0 + r < N) ? A[(i0 + r) * LDA + k] : LinT(0);
#pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        if (on[s]) {
                            const int j = lane + G * s;
                            LinT a[kRows];
#pragma unroll
                            for (int r = 0; r < kRows; ++r)
                                if (i0 + r < N) a[r] = A[(i0 + r) * LDA + j];
#pragma unroll
                            for (int r = 0; r < kRows; ++r)
                                if (i0 + r < N) A[(i0 + r) * LDA + j] = a[r] - l[r] * u[s];
                        }
                    }
                }
            }
        } else {
            // the smallest matrices: the short element-wise form (the batched one
            // takes registers that cost these kernels resident warps)
            for (int j = k + 1 + lane; j < N; j += G) {
                const LinT ukj = A[k * LDA + j];
                if (ukj != LinT(0)) {
#pragma unroll 4
                    for (int i = k + 1; i < N; ++i) A[i * LDA + j] -= A[i * LDA + k] * ukj;
                }
            }
        }
        __syncwarp(gm);
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
        if (lane + G * s < N) perm[lane + G * s] = pv[s];
    __syncwarp(gm);
    return sing;
}

// Matrices from this size up (one to four warps per SM) take the blocked form.
constexpr int kBlockedLuMinN = 96;

template <class MT, class LinT>
__device__ __noinline__ int warp_lu(unsigned A_off, unsigned perm_off, int lane) {
    if constexpr (MT::N >= kBlockedLuMinN) return warp_lu_blocked<MT, LinT>(A_off, perm_off, lane);
    else return warp_lu_compact<MT, LinT>(A_off, perm_off, lane);
}

// Matrices from this size up take the blocked triangular sweeps.
constexpr int kBlockedSolveMinN = 64;

// Solve (L U) x = P b.  b: lane elements (FP64, element i = lane + G s) in,
// solution out.  Arithmetic in LinT.
template <class MT, class LinT>
__device__ __noinline__ Vec<MT::NS> warp_lu_solve(unsigned A_off, unsigned perm_off,
                                                  const Vec<MT::NS> bv, int lane) {
    constexpr int N = MT::N, LDA = MT::LDA, NS = MT::NS, G = MT::G;
    const LinT* A = smem_at<LinT>(A_off);
    const unsigned char* perm = smem_at<unsigned char>(perm_off);
    const double (&b)[NS] = bv.v;
    Vec<NS> out;
    LinT x[NS];
    // gather: x[i] = b[perm[i]]
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int i = lane + G * s;
        const int src = (i < N) ? perm[i] : i;
        double v = 0.0;
#pragma unroll
        for (int s2 = 0; s2 < NS; ++s2) {
            const double t = group_shfl<G>(b[s2], src % G);
            if ((src / G) == s2) v = t;
        }
        x[s] = (i < N) ? (LinT)v : LinT(0);
    }
    // Sweeps of the larger matrices (kBlockedSolveMinN unknowns up) go in
    // blocks of kB rows: every lane takes the block's kB partial values (one
    // shuffle latency for the block instead of one per row), solves the block's
    // kB x kB triangle itself, and applies the block's columns to its own rows
    // in column order -- each element gets the same fused multiply-adds in the
    // same order as in the one-column-at-a-time sweep below, so both give the
    // same bits.  The smaller matrices take the one-column sweep: rolled and
    // short (this runs every Newton iteration and must stay small in the
    // instruction cache, and its registers cost the small kernels resident warps).
    if constexpr (N >= kBlockedSolveMinN) {
        constexpr int kB = 4;
        // forward: unit lower
#pragma unroll 1
        for (int k0 = 0; k0 < N - 1; k0 += kB) {
            LinT y[kB];
#pragma unroll
            for (int r = 0; r < kB; ++r) {
                const int k = k0 + r;
                y[r] = (k < N) ? group_shfl<G>(pick<NS>(x, k / G), k % G) : LinT(0);
            }
#pragma unroll
            for (int r = 1; r < kB; ++r) {
                if (k0 + r < N) {
#pragma unroll
                    for (int q = 0; q < r; ++q) y[r] -= A[(k0 + r) * LDA + k0 + q] * y[q];
                }
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int i = lane + G * s;
                if (i >= k0 + kB && i < N) {
#pragma unroll
                    for (int q = 0; q < kB; ++q) x[s] -= A[i * LDA + k0 + q] * y[q];
                }
#pragma unroll
                for (int r = 1; r < kB; ++r)
                    if (i == k0 + r && i < N) x[s] = y[r];
            }
        }
        // backward: upper (the diagonal holds 1 / U_kk)
#pragma unroll 1
        for (int k1 = N - 1; k1 >= 0; k1 -= kB) {
            LinT y[kB];
#pragma unroll
            for (int r = 0; r < kB; ++r) {
                const int k = k1 - r;
                y[r] = (k >= 0) ? group_shfl<G>(pick<NS>(x, k / G), k % G) : LinT(0);
            }
#pragma unroll
            for (int r = 0; r < kB; ++r) {
                const int k = k1 - r;
                if (k >= 0) {
#pragma unroll
                    for (int q = 0; q < r; ++q) y[r] -= A[k * LDA + k1 - q] * y[q];
                    y[r] = y[r] * A[k * LDA + k];
                }
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int i = lane + G * s;
                if (i <= k1 - kB) {
#pragma unroll
                    for (int q = 0; q < kB; ++q) x[s] -= A[i * LDA + k1 - q] * y[q];
                }
#pragma unroll
                for (int r = 0; r < kB; ++r)
                    if (i == k1 - r) x[s] = y[r];
            }
        }
    } else {
        // forward: unit lower (rolled: this runs every Newton iteration and must
        // stay small in the instruction cache)
#pragma unroll 1
        for (int k = 0; k < N - 1; ++k) {
            const LinT xk = group_shfl<G>(pick<NS>(x, k / G), k % G);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int i = lane + G * s;
                if (i > k && i < N) x[s] -= A[i * LDA + k] * xk;
            }
        }
        // backward: upper (the diagonal holds 1 / U_kk)
#pragma unroll 1
        for (int k = N - 1; k >= 0; --k) {
            const LinT xk = group_shfl<G>(pick<NS>(x, k / G), k % G) * A[k * LDA + k];
            if (lane == (k % G)) place<NS>(x, k / G, xk);
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int i = lane + G * s;
                if (i < k) x[s] -= A[i * LDA + k] * xk;
            }
        }
    }
    // A species no reaction changes has a zero row in J, so its row of M is
    // the identity row and its solution component is exactly its right-hand
    // side; taking b itself keeps such species (inert colliders such as Ar,
    // He) free of the round-off the pivoted LinT solve would give them.
    const DevMech& M = mech<MT>();
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const int i = lane + G * s;
        out.v[s] = (i < N - 1 && __ldg(M.inert + i)) ? b[s] : (double)x[s];
    }
    return out;
}

}  // namespace b200
