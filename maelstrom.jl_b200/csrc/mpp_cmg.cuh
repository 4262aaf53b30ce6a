// The V-cycle's small levels, resident in a thread-block cluster's shared memory.
//
// Below the fine level the V-cycle's levels shrink 8x each, and from about 64^3 down a
// pass over one of them is a few microseconds of launch, drain and memory latency for a
// fraction of a microsecond of work. Here levels ls .. lb-1 live, for one half of vcycle!
// (src/flip.jl:992-1014), in the shared memory of one cluster of CS CTAs: CTA r holds planes
// [r P, (r + 1) P) of each level, a z-slab in the level's own row-split layout (so loading
// and storing it is a flat copy), and reads the planes of its neighbours in z through
// distributed shared memory (mapa'd generic addresses). Passes are separated by the
// cluster's hardware barrier (release/acquire at cluster scope, about a third of a
// microsecond). Each slab keeps the list of its rows that hold a LIQUID cell; a pass runs
// over the (row, cell) items of those rows, flattened over the CTA's threads, RB items a
// thread at a time with all their loads issued before any result is computed.
//   down (k_cmg<Pr, 0>): load each slab's codes and diagonals and level ls's b; per level
//        start, the down colours, residual, restriction into the next level's slab (into
//        the one-CTA bottom levels' input in global memory after the last); store each
//        level's x and b for the up half.
//   up (k_cmg<Pr, 1>): load the slabs again; per level from lb-1 to ls, prolongation from
//        the level below (the bottom level's x in global memory first), the up colours;
//        store level ls's x.
// Each pass computes what the per-level kernel computes for the same cell, in the same
// order (rbgs, residual, restriction's 64 terms, prolongation's 8; terms outside the grid
// are zeros and are left out, which rounds the same: a sum that starts at +0 is never -0),
// so the results are bit for bit those of the per-level launches. Every thread of every CTA
// runs the same barrier sequence (loop bounds are kernel arguments), and a last barrier
// keeps each CTA's shared memory alive until no other CTA reads it.
#pragma once

#include "mpp_tiles.cuh"

namespace mpp {

constexpr int CMG_MAXLEV = 6;
#ifndef MPP_CMG_THREADS
#define MPP_CMG_THREADS 512
#endif
constexpr int CMG_THREADS = MPP_CMG_THREADS, CMG_WARPS = CMG_THREADS / 32;
constexpr unsigned CMG_HEADER = 64;  // bytes: the levels' active-row counts
#ifndef MPP_CMG_RB
#define MPP_CMG_RB 2
#endif
constexpr int CMG_RB = MPP_CMG_RB;  // items a thread has in flight

__device__ __forceinline__ void cluster_barrier() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n"
        "barrier.cluster.wait.acquire.aligned;\n" ::
            : "memory");
}

// One level's slab: geometry, division constants and the byte offsets of its arrays in
// every CTA's shared memory (the same layout in each, so a neighbour's copy is at the same
// offset). t / d for t, d < 2^16 is __umulhi(t, floor((2^32 - 1) / d) + 1).
struct CmgSlab {
    int n1, n2, n3, P, H;  // P planes per CTA; H = n1 / 2
    unsigned mH, mN, mP;   // division by H, n1, P (P = 1 needs none)
    unsigned ox, ob, orr, ocode, odg, odi, orows;  // x, b, r, code, diagonal, 1/diagonal (16-bit
                                                  // forms), active rows (uint32: kk << 16 | j)
};

template <class M>
struct CmgArgs {
    Lev<M> g[CMG_MAXLEV + 1];  // the levels' global arrays; g[nl] is the bottom level lb
    CmgSlab s[CMG_MAXLEV];
    int nl, sweeps;
    void* botb;                // the bottom levels' right-hand side (C, natural order)
};

extern __shared__ __align__(128) unsigned char cmg_sm[];

template <class T>
__device__ __forceinline__ T* cmg_ptr(unsigned off) {
    return reinterpret_cast<T*>(cmg_sm + off);
}
__device__ __forceinline__ int& cmg_count(int q) { return reinterpret_cast<int*>(cmg_sm)[q]; }
__device__ __forceinline__ int cmg_div(int t, unsigned m) { return (int)__umulhi((unsigned)t, m); }

// The generic address of the same shared-memory location in CTA r of the cluster.
template <class T>
__device__ __forceinline__ const T* cmg_map(const T* p, int r) {
    uint64_t o;
    asm("mapa.u64 %0, %1, %2;" : "=l"(o) : "l"(reinterpret_cast<uint64_t>(p)), "r"(r));
    return reinterpret_cast<const T*>(o);
}

// Plane k (0 <= k < n3) of array `off` of slab S, as a generic pointer (this CTA's or another's).
template <class T>
__device__ __forceinline__ const T* cmg_plane(const CmgSlab& S, unsigned off, int k, int me) {
    const int r = S.P == 1 ? k : cmg_div(k, S.mP);
    const T* p = cmg_ptr<T>(off) + (k - r * S.P) * S.n1 * S.n2;
    return r == me ? p : cmg_map<T>(p, r);
}

// The item's row: plane kk of the slab, row j.
__device__ __forceinline__ void cmg_row(const uint32_t* rows, int ri, int& kk, int& j) {
    const uint32_t w = rows[ri];
    kk = (int)(w >> 16);
    j = (int)(w & 0xffffu);
}

// Copy between a slab array and its level's global rows [me P n2 n1, (me + 1) P n2 n1),
// 16 bytes a load when both sides and the size allow it.
template <class T, bool TO_SMEM>
__device__ __forceinline__ void cmg_copy(T* sm, T* gl, int n) {
    const size_t bytes = (size_t)n * sizeof(T);
    if (((reinterpret_cast<uintptr_t>(gl) | reinterpret_cast<uintptr_t>(sm) | bytes) & 15) == 0) {
        uint4* s = reinterpret_cast<uint4*>(sm);
        uint4* g = reinterpret_cast<uint4*>(gl);
        const int n16 = (int)(bytes / 16);
        for (int u = (int)threadIdx.x; u < n16; u += 4 * CMG_THREADS) {
            uint4 v[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (u + q * CMG_THREADS < n16) v[q] = TO_SMEM ? g[u + q * CMG_THREADS] : s[u + q * CMG_THREADS];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (u + q * CMG_THREADS < n16) (TO_SMEM ? s : g)[u + q * CMG_THREADS] = v[q];
        }
    } else {
        for (int u = (int)threadIdx.x; u < n; u += 4 * CMG_THREADS) {
            T v[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (u + q * CMG_THREADS < n) v[q] = TO_SMEM ? gl[u + q * CMG_THREADS] : sm[u + q * CMG_THREADS];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (u + q * CMG_THREADS < n) (TO_SMEM ? sm : gl)[u + q * CMG_THREADS] = v[q];
        }
    }
}
// Zero a slab array (its size rounded up to 16 bytes, which the layout reserves).
__device__ __forceinline__ void cmg_zero(unsigned off, size_t bytes) {
    uint4* s = cmg_ptr<uint4>(off);
    const int n16 = (int)((bytes + 15) / 16);
    for (int u = (int)threadIdx.x; u < n16; u += CMG_THREADS) s[u] = make_uint4(0, 0, 0, 0);
}

// Fill slab q from its level's global arrays (b: 1 loaded, 0 zeros, -1 left alone; x loaded
// or zeros; r zeros when asked).
template <class Pr>
__device__ __forceinline__ void cmg_load(const CmgSlab& S, const Lev<typename Pr::M>& G, int me, int ldb, bool ldx,
                                         bool clr) {
    using M = typename Pr::M;
    const int n = S.P * S.n2 * S.n1;
    const int64_t g0 = (int64_t)me * n;
    cmg_copy<uint8_t, true>(cmg_ptr<uint8_t>(S.ocode), G.code + g0, n);
    cmg_copy<M, true>(cmg_ptr<M>(S.odg), G.dg + g0, n);
    if (Pr::scaled) cmg_copy<M, true>(cmg_ptr<M>(S.odi), G.di + g0, n);
    if (ldb > 0) cmg_copy<M, true>(cmg_ptr<M>(S.ob), G.b + g0, n);
    else if (ldb == 0) cmg_zero(S.ob, sizeof(M) * n);
    if (ldx) cmg_copy<M, true>(cmg_ptr<M>(S.ox), G.x + g0, n);
    else cmg_zero(S.ox, sizeof(M) * n);
    if (clr) cmg_zero(S.orr, sizeof(M) * n);
}
// List slab q's rows that hold a LIQUID cell (after its codes are in and a block barrier).
__device__ __forceinline__ void cmg_rows(const CmgSlab& S, int q) {
    const int nrow = S.P * S.n2, lane = (int)threadIdx.x & 31;
    const uint8_t* code = cmg_ptr<uint8_t>(S.ocode);
    uint32_t* rows = cmg_ptr<uint32_t>(S.orows);
    for (int row = (int)threadIdx.x >> 5; row < nrow; row += CMG_WARPS) {
        bool any = false;
        for (int i = lane; i < S.n1; i += 32) any |= (code[row * S.n1 + i] & SELF) != 0;
        if (__any_sync(0xffffffffu, any) && lane == 0) {
            const int kk = row / S.n2, j = row - kk * S.n2;
            rows[atomicAdd(&cmg_count(q), 1)] = (uint32_t)(kk << 16) | (uint32_t)j;
        }
    }
}
template <class Pr>
__device__ __forceinline__ void cmg_store(const CmgSlab& S, const Lev<typename Pr::M>& G, int me, bool stb) {
    using M = typename Pr::M;
    const int n = S.P * S.n2 * S.n1;
    const int64_t g0 = (int64_t)me * n;
    cmg_copy<M, false>(cmg_ptr<M>(S.ox), G.x + g0, n);
    if (stb) cmg_copy<M, false>(cmg_ptr<M>(S.ob), G.b + g0, n);
}

// A cell's six neighbour values (+x,-x,+y,-y,+z,-z) from the other colour's half-row at o
// (its position h in that half; ci the cell's offset 2h + ci in the row). Reads at the
// slab's and the grid's edges are redirected to the cell's own half-row (those neighbours
// are not LIQUID, and liquidsum skips them); +-z beyond the slab come from the
// neighbouring CTAs (xa, xb: their slabs' first element), or from this one's own slab
// where there is no such CTA (again not LIQUID).
template <class M>
struct CmgNb {
    M v[6];
};
template <class M>
__device__ __forceinline__ void cmg_nb(CmgNb<M>& r, const M* x, const M* xa, const M* xb, const CmgSlab& S, int o,
                                       int h, int ci, int j, int kk) {
    const int sz = S.n1 * S.n2;
    r.v[0] = x[h + ci < S.H ? o + ci : o];
    r.v[1] = x[h + ci > 0 ? o + ci - 1 : o];
    r.v[2] = x[j + 1 < S.n2 ? o + S.n1 : o];
    r.v[3] = x[j > 0 ? o - S.n1 : o];
    r.v[4] = kk + 1 < S.P ? x[o + sz] : xa[o - kk * sz];
    r.v[5] = kk > 0 ? x[o - sz] : xb[o - kk * sz + (S.P - 1) * sz];
}
template <class C, class M>
__device__ __forceinline__ C cmg_sum(const CmgNb<M>& r, uint8_t cd) {
    C v[6];
#pragma unroll
    for (int m = 0; m < 6; m++) v[m] = ld<C>(&r.v[m]);
    return sum6<C>(v, cd);
}
template <class M>
__device__ __forceinline__ void cmg_faces(const CmgSlab& S, int me, int cs, const M*& xa, const M*& xb) {
    const M* x = cmg_ptr<M>(S.ox);
    xa = me + 1 < cs ? cmg_map<M>(x, me + 1) : x;
    xb = me > 0 ? cmg_map<M>(x, me - 1) : x;
}

// start (the first colour's first sweep from x = 0): x = b / diag on colour 0, 0 elsewhere.
template <class Pr>
__device__ __forceinline__ void cmg_start(const CmgSlab& S, int q) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    M* x = cmg_ptr<M>(S.ox);
    const M* b = cmg_ptr<M>(S.ob);
    const uint8_t* code = cmg_ptr<uint8_t>(S.ocode);
    const M* dd = cmg_ptr<M>(Pr::scaled ? S.odi : S.odg);
    const uint32_t* rows = cmg_ptr<uint32_t>(S.orows);
    const int T = cmg_count(q) * S.n1;
    for (int t = (int)threadIdx.x; t < T; t += CMG_THREADS) {
        const int ri = cmg_div(t, S.mN), p = t - ri * S.n1;
        int kk, j;
        cmg_row(rows, ri, kk, j);
        const int e = (kk * S.n2 + j) * S.n1 + p;
        C v = (C)0;
        if (p < S.H && (code[e] & SELF)) {
            const C d = ld<C>(dd + e);
            if constexpr (Pr::scaled) v = ld<C>(b + e) * d;
            else v = d > (C)0 ? ld<C>(b + e) / d : (C)0;
        }
        st(x + e, v);
    }
}

// One colour of red-black Gauss-Seidel (rbgs_kernel!, src/flip.jl:859-880).
template <class Pr>
__device__ __forceinline__ void cmg_rbgs(const CmgSlab& S, int q, int colour, int me, int cs) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    M* x = cmg_ptr<M>(S.ox);
    const M* b = cmg_ptr<M>(S.ob);
    const uint8_t* code = cmg_ptr<uint8_t>(S.ocode);
    const M* dd = cmg_ptr<M>(Pr::scaled ? S.odi : S.odg);
    const uint32_t* rows = cmg_ptr<uint32_t>(S.orows);
    const M *xa, *xb;
    cmg_faces<M>(S, me, cs, xa, xb);
    const int T = cmg_count(q) * S.H;
    for (int t0 = (int)threadIdx.x; t0 < T; t0 += CMG_RB * CMG_THREADS) {
        int e[CMG_RB];
        uint8_t cd[CMG_RB];
        M bv[CMG_RB], dv[CMG_RB];
        CmgNb<M> nb[CMG_RB];
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            const int t = t0 + u * CMG_THREADS;
            cd[u] = 0;
            e[u] = 0;
            if (t < T) {
                const int ri = cmg_div(t, S.mH), h = t - ri * S.H;
                int kk, j;
                cmg_row(rows, ri, kk, j);
                const int k = me * S.P + kk, ci = (colour + j + k + 1) & 1;
                const int sb = (kk * S.n2 + j) * S.n1, o = sb + (1 - colour) * S.H + h;
                e[u] = sb + colour * S.H + h;
                cd[u] = code[e[u]];
                bv[u] = b[e[u]];
                dv[u] = dd[e[u]];
                cmg_nb<M>(nb[u], x, xa, xb, S, o, h, ci, j, kk);
            }
        }
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            if (!(cd[u] & SELF)) continue;
            const C s = cmg_sum<C, M>(nb[u], cd[u]);
            const C d = ld<C>(&dv[u]);
            C v;
            if constexpr (Pr::scaled) v = (ld<C>(&bv[u]) + s) * d;
            else v = d > (C)0 ? (ld<C>(&bv[u]) + s) / d : (C)0;
            st(x + e[u], v);
        }
    }
}

// residual_kernel! (src/flip.jl:882-898): r = b - A x on the LIQUID cells, 0 elsewhere.
template <class Pr>
__device__ __forceinline__ void cmg_residual(const CmgSlab& S, int q, int me, int cs) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    const M* x = cmg_ptr<M>(S.ox);
    const M* b = cmg_ptr<M>(S.ob);
    M* r = cmg_ptr<M>(S.orr);
    const uint8_t* code = cmg_ptr<uint8_t>(S.ocode);
    const M* dg = cmg_ptr<M>(S.odg);
    const uint32_t* rows = cmg_ptr<uint32_t>(S.orows);
    const M *xa, *xb;
    cmg_faces<M>(S, me, cs, xa, xb);
    const int T = cmg_count(q) * S.n1;
    for (int t0 = (int)threadIdx.x; t0 < T; t0 += CMG_RB * CMG_THREADS) {
        int e[CMG_RB];
        uint8_t cd[CMG_RB];
        M bv[CMG_RB], dv[CMG_RB], xv[CMG_RB];
        CmgNb<M> nb[CMG_RB];
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            const int t = t0 + u * CMG_THREADS;
            cd[u] = 0;
            e[u] = -1;
            if (t < T) {
                const int ri = cmg_div(t, S.mN), p = t - ri * S.n1;
                int kk, j;
                cmg_row(rows, ri, kk, j);
                const int c = p >= S.H ? 1 : 0, h = p - c * S.H;
                const int k = me * S.P + kk, ci = (c + j + k + 1) & 1;
                const int sb = (kk * S.n2 + j) * S.n1, o = sb + (1 - c) * S.H + h;
                e[u] = sb + p;
                cd[u] = code[e[u]];
                bv[u] = b[e[u]];
                dv[u] = dg[e[u]];
                xv[u] = x[e[u]];
                cmg_nb<M>(nb[u], x, xa, xb, S, o, h, ci, j, kk);
            }
        }
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            if (e[u] < 0) continue;
            C v = (C)0;
            if (cd[u] & SELF)
                v = ld<C>(&bv[u]) - (ld<C>(&dv[u]) * ld<C>(&xv[u]) - cmg_sum<C, M>(nb[u], cd[u]));
            st(r + e[u], v);
        }
    }
}

// restrict_kernel! value of coarse cell (I, J, K) from fine slab F's r: the 64 terms
// 16 c + 4 b + a in the reference's order, those outside the grid (zeros) left out. Fine
// row (jf, kf) holds x = 2I-1+a at its colour (jf+kf)&1 half, position I-1, I, I, I+1 for
// a = 0..3, alternating halves. Each term as macc<FUSE> rounds it.
template <bool FUSE, class C, class M>
__device__ __forceinline__ C cmg_restrict_cell(const CmgSlab& F, int I, int J, int K, int me) {
    C s = (C)0;
    const M* r0 = cmg_ptr<M>(F.orr);
#pragma unroll
    for (int c3 = 0; c3 < 4; c3++) {
        const int kf = 2 * K - 1 + c3;
        const bool kok = kf >= 0 && kf < F.n3;
        const M* pl = kok ? cmg_plane<M>(F, F.orr, kf, me) : r0;
#pragma unroll
        for (int b3 = 0; b3 < 4; b3++) {
            const int jf = 2 * J - 1 + b3;
            const bool ok = kok && jf >= 0 && jf < F.n2;
            const int par = (jf + kf) & 1;
            const M* row = pl + (ok ? jf : 0) * F.n1;
            const M* A = row + par * F.H;
            const M* B = row + (1 - par) * F.H;
            M t[4];
            t[0] = A[I > 0 ? I - 1 : 0];
            t[1] = B[I];
            t[2] = A[I];
            t[3] = B[I + 1 < F.H ? I + 1 : I];
            if (!ok) continue;
#pragma unroll
            for (int a3 = 0; a3 < 4; a3++) {
                if (a3 == 0 && I == 0) continue;
                if (a3 == 3 && I + 1 >= F.H) continue;
                s = macc<FUSE>(s, rw<C>(16 * c3 + 4 * b3 + a3), ld<C>(&t[a3]));
            }
        }
    }
    return s;
}

// restrict_kernel! into the coarse slab Cs's active rows (b of its other rows stays 0).
template <class Pr>
__device__ __forceinline__ void cmg_restrict(const CmgSlab& F, const CmgSlab& Cs, int qc, int me) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    const uint8_t* code = cmg_ptr<uint8_t>(Cs.ocode);
    M* b = cmg_ptr<M>(Cs.ob);
    const uint32_t* rows = cmg_ptr<uint32_t>(Cs.orows);
    const int T = cmg_count(qc) * Cs.n1;
    for (int t = (int)threadIdx.x; t < T; t += CMG_THREADS) {
        const int ri = cmg_div(t, Cs.mN), p = t - ri * Cs.n1;
        int kk, J;
        cmg_row(rows, ri, kk, J);
        const int K = me * Cs.P + kk, c = p >= Cs.H ? 1 : 0, h = p - c * Cs.H;
        const int I = 2 * h + ((c + J + K + 1) & 1), e = (kk * Cs.n2 + J) * Cs.n1 + p;
        C v = (C)0;
        if (code[e] & SELF) {
            const C s = cmg_restrict_cell<Pr::scaled, C, M>(F, I, J, K, me);
            v = Pr::scaled ? s : (C)4 * s;
        }
        st(b + e, v);
    }
}

// restrict_kernel! into the bottom levels' input (global, natural order): the bottom level's
// cells spread over the whole cluster.
template <class Pr>
__device__ __forceinline__ void cmg_restrict_bottom(const CmgSlab& F, const Lev<typename Pr::M>& B,
                                                    typename Pr::C* out, int me, int cs) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    const int n = B.n1 * B.n2 * B.n3;
    for (int e = me * CMG_THREADS + (int)threadIdx.x; e < n; e += cs * CMG_THREADS) {
        C v = (C)0;
        if (B.code[e] & SELF) {
            const int I = e % B.n1, JK = e / B.n1, J = JK % B.n2, K = JK / B.n2;
            const C s = cmg_restrict_cell<Pr::scaled, C, M>(F, I, J, K, me);
            v = Pr::scaled ? s : (C)4 * s;
        }
        out[e] = v;
    }
}

// prolong_kernel! (src/flip.jl:914-929) into slab F's LIQUID cells from slab Cs, or from the
// bottom level in global memory (natural order, `G`).
template <class Pr>
__device__ __forceinline__ void cmg_prolong(const CmgSlab& F, int qf, const CmgSlab& Cs,
                                            const Lev<typename Pr::M>& G, bool from_global, int me) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    M* x = cmg_ptr<M>(F.ox);
    const uint8_t* code = cmg_ptr<uint8_t>(F.ocode);
    const uint32_t* rows = cmg_ptr<uint32_t>(F.orows);
    const int cn1 = from_global ? G.n1 : Cs.n1, cn2 = from_global ? G.n2 : Cs.n2, cn3 = from_global ? G.n3 : Cs.n3;
    const int T = cmg_count(qf) * F.n1;
    for (int t0 = (int)threadIdx.x; t0 < T; t0 += CMG_RB * CMG_THREADS) {
        int e[CMG_RB], ci[CMG_RB][3];  // the cell and its coordinates (i, j, k)
        bool live[CMG_RB];
        M xv[CMG_RB], cv[CMG_RB][8];
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            const int t = t0 + u * CMG_THREADS;
            live[u] = false;
            e[u] = 0;
            if (t >= T) continue;
            const int ri = cmg_div(t, F.mN), p = t - ri * F.n1;
            int kk, j;
            cmg_row(rows, ri, kk, j);
            const int k = me * F.P + kk, c = p >= F.H ? 1 : 0, h = p - c * F.H;
            const int i = 2 * h + ((c + j + k + 1) & 1);
            ci[u][0] = i;
            ci[u][1] = j;
            ci[u][2] = k;
            e[u] = (kk * F.n2 + j) * F.n1 + p;
            live[u] = (code[e[u]] & SELF) != 0;
            xv[u] = x[e[u]];
            // the coarse cells of prolongweights along each axis (the weights are formed again
            // below); those outside the grid are read at index 0 and left out
            int a0, a1, b0, b1, k0, k1;
            C wd;
            pweights<C>(i, a0, wd, a1, wd);
            pweights<C>(j, b0, wd, b1, wd);
            pweights<C>(k, k0, wd, k1, wd);
            const bool k0ok = k0 >= 0 && k0 < cn3, k1ok = k1 >= 0 && k1 < cn3;
            const M *pl0 = nullptr, *pl1 = nullptr;
            if (!from_global) {
                pl0 = cmg_plane<M>(Cs, Cs.ox, k0ok ? k0 : 0, me);
                pl1 = cmg_plane<M>(Cs, Cs.ox, k1ok ? k1 : 0, me);
            }
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int A = (m & 1) ? a1 : a0, B = (m & 2) ? b1 : b0, Kc = (m & 4) ? k1 : k0;
                const bool ok = A >= 0 && A < cn1 && B >= 0 && B < cn2 && ((m & 4) ? k1ok : k0ok);
                const int As = ok ? A : 0, Bs = ok ? B : 0, Ks = ok ? Kc : 0;
                if (from_global) cv[u][m] = G.x[As + cn1 * (Bs + cn2 * Ks)];
                else cv[u][m] = ((m & 4) ? pl1 : pl0)[Bs * cn1 + ((As + Bs + Ks + 1) & 1) * Cs.H + (As >> 1)];
            }
        }
#pragma unroll
        for (int u = 0; u < CMG_RB; u++) {
            if (!live[u]) continue;
            int a0, a1, b0, b1, c0, c1;
            C wa0, wa1, wb0, wb1, wc0, wc1;
            pweights<C>(ci[u][0], a0, wa0, a1, wa1);
            pweights<C>(ci[u][1], b0, wb0, b1, wb1);
            pweights<C>(ci[u][2], c0, wc0, c1, wc1);
            C s = (C)0;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int A = (m & 1) ? a1 : a0, B = (m & 2) ? b1 : b0, Kc = (m & 4) ? c1 : c0;
                if (A < 0 || A >= cn1 || B < 0 || B >= cn2 || Kc < 0 || Kc >= cn3) continue;  // a zero term
                const C wa = (m & 1) ? wa1 : wa0, wb = (m & 2) ? wb1 : wb0, wc = (m & 4) ? wc1 : wc0;
                s = macc<Pr::scaled>(s, wa * wb * wc, ld<C>(&cv[u][m]));
            }
            st(x + e[u], ld<C>(&xv[u]) + (Pr::scaled ? (C)4 * s : s));
        }
    }
}

template <class Pr, int UP>
__device__ __forceinline__ void cmg_dev(const CmgArgs<typename Pr::M>& a) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    const int me = (int)blockIdx.x, cs = (int)gridDim.x, nl = a.nl;
    // Loaded before the programmatic-dependent-launch wait: what the preceding kernel does
    // not write. Down follows the restriction into level ls (its b, loaded after the wait);
    // up follows the bottom solve (the bottom level's x, read by the first prolongation).
    if (threadIdx.x < CMG_MAXLEV) cmg_count((int)threadIdx.x) = 0;
    for (int q = 0; q < nl; q++) cmg_load<Pr>(a.s[q], a.g[q], me, UP ? 1 : (q == 0 ? -1 : 0), UP, !UP);
    pdl_wait();
    pdl_trigger();
    if (!UP) {
        const CmgSlab& S = a.s[0];
        const int n = S.P * S.n2 * S.n1;
        cmg_copy<M, true>(cmg_ptr<M>(S.ob), a.g[0].b + (int64_t)me * n, n);
    }
    __syncthreads();
    for (int q = 0; q < nl; q++) cmg_rows(a.s[q], q);
    cluster_barrier();
    if (!UP) {
        for (int q = 0; q < nl; q++) {
            const CmgSlab& S = a.s[q];
            cmg_start<Pr>(S, q);
            cluster_barrier();
            for (int i = 0; i < 2 * a.sweeps - 1; i++) {  // down colours [1, 0, 1, ...]
                cmg_rbgs<Pr>(S, q, (i + 1) & 1, me, cs);
                cluster_barrier();
            }
            cmg_residual<Pr>(S, q, me, cs);
            cluster_barrier();
            if (q + 1 < nl) cmg_restrict<Pr>(S, a.s[q + 1], q + 1, me);
            else cmg_restrict_bottom<Pr>(S, a.g[nl], static_cast<C*>(a.botb), me, cs);
            cluster_barrier();
        }
        for (int q = 0; q < nl; q++) cmg_store<Pr>(a.s[q], a.g[q], me, q > 0);
    } else {
        for (int q = nl - 1; q >= 0; q--) {
            const CmgSlab& S = a.s[q];
            cmg_prolong<Pr>(S, q, q + 1 < nl ? a.s[q + 1] : S, a.g[q + 1], q + 1 == nl, me);
            for (int i = 0; i < 2 * a.sweeps; i++) {  // up colours [1, 0, 1, 0, ...]
                cluster_barrier();
                cmg_rbgs<Pr>(S, q, (i & 1) ? 0 : 1, me, cs);
            }
            cluster_barrier();
        }
        cmg_store<Pr>(a.s[0], a.g[0], me, false);
    }
    // (every CTA passed the last barrier after its last read of another CTA's memory)
}
template <class Pr, int UP>
__global__ void __launch_bounds__(CMG_THREADS, 1) k_cmg(const __grid_constant__ CmgArgs<typename Pr::M> a) {
    cmg_dev<Pr, UP>(a);
}

}  // namespace mpp
