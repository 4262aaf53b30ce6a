// The sparse two-resolution basin's pressure projection (sm_100a): fine 16^3 blocks of cells
// dx wide where the surface is, over a dense coarse grid of cells 4 dx wide, solved at once
// (src/sflip.jl:1059-2018 of the reference; src/fgmres.jl for the fallback).
//
// Layout (the reference's own, so a caller's arrays are used in place):
//   * the block table: slot[bi + nb0 (bj + nb1 bk)] = the block's 1-based slot in the fine
//     pools, 0 for a coarse-only block; where[3 (s-1) + a] = slot s's block coordinates, -1s
//     for a free slot (src/sflip.jl:78-84);
//   * fine cell pools: 4096 cells a slot, i + 16 (j + 16 k); fine face pools: 17*256 faces a
//     slot and axis (faceindex, :106-110); level 1's pools the same at 8^3 (512 cells, 9*64
//     faces);
//   * the coarse grid and its halvings: column-major, face arrays one longer along their axis.
// Kernels: the stencil passes of the two composite levels (Jacobi sweeps, residuals, A x)
// run a CTA per fine block, the block and a one-cell halo staged in shared memory (level 0's
// couplings packed in a 16-bit code a cell, level 1's read from its aggregated face arrays,
// each cell's whole diagonal precomputed once per operator); the CG's vector passes take a
// slot's cells in 16-byte pieces; the coarse grid, the dense levels and the set-up passes run
// a thread per cell or face, consecutive threads on consecutive grid indices. The fine and
// coarse parts of a level pass are one launch (the first `gf` CTAs on the fine blocks, the
// rest on the coarse cells): both read the pass's source and write its destination, so they
// are independent.
//
// Arithmetic: every value is computed in the reference kernel's Float32 operation order
// (the library is built with -fmad=false), so the operator, the coefficients, the
// hierarchy, the smoothers, the transfers and the whole V-cycle are bit-identical with
// the oracle; the CG's dot products are FP64 sums (deterministic, grid_sum) rounded to
// Float32, so whole solves agree to rounding, not bit for bit.
#pragma once

#include "mpp.h"
#include "mpp_common.cuh"

namespace mpp {
namespace sp {

constexpr int BLOCK = 16, RATIO = 4, BCELLS = 4096, BFACES = 17 * 256, BCELLS1 = 512, BFACES1 = 9 * 64;
constexpr float FINE_FINE = 1.0f, FINE_COARSE = 0.4f, COARSE_COARSE = 4.0f;
constexpr float OMEGA = 6.0f / 7.0f;  // Jacobi's damping (src/sflip.jl:1074), rounded to Float32 as there
constexpr int SPT = 256;              // threads a block

// The grid and the block table as the kernels see them.
struct Topo {
    const int32_t* slot;
    const int32_t* where;
    int nslots;
    int nb[3], nc[3];
    float lo[3], dx, radius, floor_z;
};

__device__ __forceinline__ int64_t lin(const int* n, int i, int j, int k) {
    return (int64_t)i + (int64_t)n[0] * ((int64_t)j + (int64_t)n[1] * (int64_t)k);
}
__device__ __forceinline__ int64_t lin3(int n0, int n1, int i, int j, int k) {
    return (int64_t)i + (int64_t)n0 * ((int64_t)j + (int64_t)n1 * (int64_t)k);
}
__device__ __forceinline__ bool inblocks(const Topo& t, int bi, int bj, int bk) {
    return bi >= 0 && bi < t.nb[0] && bj >= 0 && bj < t.nb[1] && bk >= 0 && bk < t.nb[2];
}
__device__ __forceinline__ int blockslot(const Topo& t, int bi, int bj, int bk) {
    return __ldg(t.slot + (bi + t.nb[0] * (bj + t.nb[1] * bk)));
}
// cellslot (src/sflip.jl:92-97)
__device__ __forceinline__ int cellslot(const Topo& t, int I, int J, int K) {
    const int bi = I >> 4, bj = J >> 4, bk = K >> 4;
    return inblocks(t, bi, bj, bk) ? blockslot(t, bi, bj, bk) : 0;
}
// covered (src/sflip.jl:128): a coarse cell lies in a fine block
__device__ __forceinline__ bool covered(const Topo& t, int I, int J, int K) {
    return cellslot(t, I * RATIO, J * RATIO, K * RATIO) != 0;
}
__device__ __forceinline__ void where_of(const Topo& t, int sl, int w[3]) {
    const int32_t* p = t.where + 3 * (sl - 1);
    w[0] = __ldg(p);
    w[1] = __ldg(p + 1);
    w[2] = __ldg(p + 2);
}
__device__ __forceinline__ bool slot_used(const Topo& t, int sl) { return __ldg(t.where + 3 * (sl - 1)) >= 0; }

// A level's fine part (N = 16: level 0; N = 8: level 1): 1-based pool indices, 0 = none, as
// cellidx / faceidx / cellat / faceat (src/sflip.jl:1080-1111).
template <int N>
struct Lv {
    static constexpr int SH = N == 16 ? 4 : 3, M = N - 1, CELLS = N * N * N, FACES = (N + 1) * N * N;
    __device__ static __forceinline__ int64_t cell(int sl, int i, int j, int k) {
        return (int64_t)(sl - 1) * CELLS + i + N * (j + N * k) + 1;
    }
    __device__ static __forceinline__ int64_t face(int sl, int a, int i, int j, int k) {
        const int f = a == 1 ? i + (N + 1) * (j + N * k) : (a == 2 ? i + N * (j + (N + 1) * k) : i + N * (j + N * k));
        return (int64_t)(sl - 1) * FACES + f + 1;
    }
    __device__ static __forceinline__ int64_t cellat(const Topo& t, int I, int J, int K) {
        const int bi = I >> SH, bj = J >> SH, bk = K >> SH;
        if (!inblocks(t, bi, bj, bk)) return 0;
        const int sl = blockslot(t, bi, bj, bk);
        return sl == 0 ? 0 : cell(sl, I & M, J & M, K & M);
    }
    __device__ static __forceinline__ int64_t faceat(const Topo& t, int a, int I, int J, int K) {
        const int bi = I >> SH, bj = J >> SH, bk = K >> SH;
        if (inblocks(t, bi, bj, bk)) {
            const int sl = blockslot(t, bi, bj, bk);
            if (sl != 0) return face(sl, a, I & M, J & M, K & M);
        }
        const int Im = I - (a == 1), Jm = J - (a == 2), Km = K - (a == 3);
        if (!((Im >> SH) != bi || (Jm >> SH) != bj || (Km >> SH) != bk)) return 0;
        if (!inblocks(t, Im >> SH, Jm >> SH, Km >> SH)) return 0;
        const int sl = blockslot(t, Im >> SH, Jm >> SH, Km >> SH);
        if (sl == 0) return 0;
        return face(sl, a, a == 1 ? N : (Im & M), a == 2 ? N : (Jm & M), a == 3 ? N : (Km & M));
    }
};
using L16 = Lv<16>;
using L8 = Lv<8>;
__device__ __forceinline__ int64_t fineat(const Topo& t, int I, int J, int K) { return L16::cellat(t, I, J, K); }
// finefaceat (src/sflip.jl:116-126) is level 0's faceat
__device__ __forceinline__ int64_t finefaceat(const Topo& t, int a, int I, int J, int K) {
    return L16::faceat(t, a, I, J, K);
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int64_t coarse_clamped(const Topo& t, int ci, int cj, int ck) {
    return lin(t.nc, clampi(ci, 0, t.nc[0] - 1), clampi(cj, 0, t.nc[1] - 1), clampi(ck, 0, t.nc[2] - 1));
}

// issolid at a fine or coarse cell centre (src/sflip.jl:59-65), Float32 as the reference
__device__ __forceinline__ bool issolid_p(const Topo& t, float px, float py, float pz) {
    return px * px + py * py > t.radius * t.radius || pz < t.floor_z;
}
__device__ __forceinline__ bool issolid_fine(const Topo& t, int I, int J, int K) {
    return issolid_p(t, t.lo[0] + ((float)I + 0.5f) * t.dx, t.lo[1] + ((float)J + 0.5f) * t.dx,
                     t.lo[2] + ((float)K + 0.5f) * t.dx);
}
__device__ __forceinline__ bool issolid_coarse(const Topo& t, int I, int J, int K) {
    const float h = (float)RATIO * t.dx;
    return issolid_p(t, t.lo[0] + ((float)I + 0.5f) * h, t.lo[1] + ((float)J + 0.5f) * h,
                     t.lo[2] + ((float)K + 0.5f) * h);
}

// celltype (src/sflip.jl:1335-1342): a fine cell's class and whether a fine block holds it
__device__ __forceinline__ uint8_t celltype(const Topo& t, const uint8_t* tf, const uint8_t* tc, int I, int J, int K,
                                            bool& fine) {
    const int64_t idx = fineat(t, I, J, K);
    if (idx > 0) {
        fine = true;
        return tf[idx - 1];
    }
    fine = false;
    const int ci = I >> 2, cj = J >> 2, ck = K >> 2;
    if (!(ci >= 0 && ci < t.nc[0] && cj >= 0 && cj < t.nc[1] && ck >= 0 && ck < t.nc[2])) return SOLID;
    return tc[lin(t.nc, ci, cj, ck)];
}
// neighbourφ (src/sflip.jl:883-888) and pressureat (:1909-1914): a fine-cell value, the
// coarse cell's where no fine block holds it
__device__ __forceinline__ float fine_or_coarse(const Topo& t, const float* f, const float* c, int I, int J, int K) {
    const int64_t idx = fineat(t, I, J, K);
    return idx > 0 ? f[idx - 1] : c[coarse_clamped(t, I >> 2, J >> 2, K >> 2)];
}

// The arrays of one composite level (level 0 or 1): its fine part's couplings, Dirichlet
// diagonal and activity, and the coarse grid's (shared by both levels).
struct Comp {
    const float *cfx, *cfy, *cfz, *dDf;
    const uint8_t* actf;
    const float *ccx, *ccy, *ccz, *dDc;
    const uint8_t* actc;
    // the coarse cells the composite passes update (LIQUID, no fine block over them; actc is
    // set on exactly these outside fine blocks), listed once per operator: the passes walk
    // the list, and every other coarse cell of their outputs stays at the zero it was cleared to
    const int* clist;
    const int* nclist;
};

// Where a level-0 pass reads x: the stored values (SrcX), or values formed on the fly, with
// the same Float32 operations, from what a pass that the fused one replaces would have
// stored. SrcZS: the first sweep of smooth! from zeros, elementwise (x = 0 makes off = 0).
// SrcPro: z after prolong10fine_kernel! / prolongcoarse_kernel! (z plus boost times the
// level-1 cell's value, on LIQUID fine cells and on the coarse unknowns).
struct SrcX {
    const float* xf;
    const float* xc;
    __device__ __forceinline__ float4 fine4(int64_t n) const { return *reinterpret_cast<const float4*>(xf + n); }
    __device__ __forceinline__ float fine(int64_t n) const { return xf[n]; }
    __device__ __forceinline__ float coarse(int64_t c) const { return xc[c]; }
};
struct SrcZS {
    const uint16_t* code0;
    const float* dg0;
    const float* bf;
    const uint8_t* cmask;  // the coarse unknowns: the cells the coarse part of a sweep writes
    const float* dgc;      // their whole diagonals, coarserow's sums
    const float* bc;
    __device__ __forceinline__ static float sweep0(bool act, float diag, float b) {
        const float x0 = 0.0f, off = 0.0f;
        return act && diag > 0.0f ? x0 + OMEGA * (b - (diag * x0 - off)) / diag : 0.0f;
    }
    __device__ __forceinline__ float4 fine4(int64_t n) const {
        const ushort4 cd = *reinterpret_cast<const ushort4*>(code0 + n);
        const float4 d = *reinterpret_cast<const float4*>(dg0 + n), b = *reinterpret_cast<const float4*>(bf + n);
        return make_float4(sweep0(cd.x & 0x1000u, d.x, b.x), sweep0(cd.y & 0x1000u, d.y, b.y),
                           sweep0(cd.z & 0x1000u, d.z, b.z), sweep0(cd.w & 0x1000u, d.w, b.w));
    }
    __device__ __forceinline__ float fine(int64_t n) const { return sweep0(code0[n] & 0x1000u, dg0[n], bf[n]); }
    __device__ __forceinline__ float coarse(int64_t c) const { return sweep0(cmask[c] != 0, dgc[c], bc[c]); }
};
struct SrcPro {
    const float* zf;
    const float* zc;
    const uint16_t* code0;
    const float* x1f;
    const float* x1c;
    const uint8_t* cmask;
    float boost;
    // the level-1 cell of fine pool cell n
    __device__ __forceinline__ static int64_t parent(int64_t n) {
        const int c = (int)(n & (BCELLS - 1)), i = c & 15, j = (c >> 4) & 15, k = c >> 8;
        return (n >> 12) * BCELLS1 + (i >> 1) + 8 * ((j >> 1) + 8 * (k >> 1));
    }
    __device__ __forceinline__ float4 fine4(int64_t n) const {
        float4 z = *reinterpret_cast<const float4*>(zf + n);
        const ushort4 cd = *reinterpret_cast<const ushort4*>(code0 + n);
        const int64_t b1 = parent(n);
        const float xa = x1f[b1], xb = x1f[b1 + 1];
        if (cd.x & 0x2000u) z.x += boost * xa;
        if (cd.y & 0x2000u) z.y += boost * xa;
        if (cd.z & 0x2000u) z.z += boost * xb;
        if (cd.w & 0x2000u) z.w += boost * xb;
        return z;
    }
    __device__ __forceinline__ float fine(int64_t n) const {
        float v = zf[n];
        if (code0[n] & 0x2000u) v += boost * x1f[parent(n)];
        return v;
    }
    __device__ __forceinline__ float coarse(int64_t c) const {
        float v = zc[c];
        if (cmask[c] != 0) v += boost * x1c[c];
        return v;
    }
};

// coarserow (src/sflip.jl:1176-1217): a coarse cell outside fine blocks, its coarse
// neighbours through coarse faces, a fine block's cells through the block's R^2 sub-faces.
template <int N, bool ZS, class Src>
__device__ __forceinline__ void coarserow_s(const Topo& t, const Comp& L, const Src& src, int I, int J, int K,
                                            float& diag, float& off) {
    using V = Lv<N>;
    constexpr int R = N / 4;
    const int n1 = t.nc[0], n2 = t.nc[1], n3 = t.nc[2];
    diag = L.dDc[lin(t.nc, I, J, K)];
    off = 0.0f;
#pragma unroll
    for (int a = 1; a <= 3; a++) {
        const int e0 = a == 1, e1 = a == 2, e2 = a == 3;
        const float* Cc = a == 1 ? L.ccx : (a == 2 ? L.ccy : L.ccz);
        const float* Cf = a == 1 ? L.cfx : (a == 2 ? L.cfy : L.cfz);
        const int f0 = n1 + e0, f1 = n2 + e1;
#pragma unroll
        for (int sg = -1; sg <= 1; sg += 2) {
            const int In = I + sg * e0, Jn = J + sg * e1, Kn = K + sg * e2;
            if (!(0 <= In && In < n1 && 0 <= Jn && Jn < n2 && 0 <= Kn && Kn < n3)) continue;
            // the neighbouring coarse cell's block: covered when it has a slot
            const int s2 = cellslot(t, In * RATIO, Jn * RATIO, Kn * RATIO);
            if (s2 != 0) {
                // Its R^2 cells across the plane lie in block s2; each couples through its own
                // sub-face, which is in s2 too: the cell's low face (sg > 0), or s2's high plane
                // (sg < 0; the face's upper cell is this uncovered coarse cell's, faceat takes
                // the lower block's copy). This is faceat / cellat with the block looked up once.
#pragma unroll
                for (int q = 0; q < R; q++)
#pragma unroll
                    for (int p = 0; p < R; p++) {
                        const int FI = a == 1 ? (sg > 0 ? R * In : R * I - 1) : R * I + p;
                        const int FJ = a == 2 ? (sg > 0 ? R * Jn : R * J - 1) : R * J + (a == 1 ? p : q);
                        const int FK = a == 3 ? (sg > 0 ? R * Kn : R * K - 1) : R * K + q;
                        constexpr int M = N - 1;
                        const int64_t fidx = sg > 0 ? V::face(s2, a, FI & M, FJ & M, FK & M)
                                                    : V::face(s2, a, a == 1 ? N : (FI & M), a == 2 ? N : (FJ & M),
                                                              a == 3 ? N : (FK & M));
                        const int64_t cidx = V::cell(s2, FI & M, FJ & M, FK & M);
                        const float c = Cf[fidx - 1];
                        diag += c;
                        off += c * (ZS ? 0.0f : src.fine(cidx - 1));
                    }
            } else {
                const float c = sg < 0 ? Cc[lin3(f0, f1, I, J, K)] : Cc[lin3(f0, f1, I + e0, J + e1, K + e2)];
                if (c > 0.0f) {
                    diag += c;
                    off += c * (ZS ? 0.0f : src.coarse(lin(t.nc, In, Jn, Kn)));
                }
            }
        }
    }
}

template <int N, bool ZS>
__device__ __forceinline__ void coarserow(const Topo& t, const Comp& L, const float* xf, const float* xc, int I,
                                          int J, int K, float& diag, float& off) {
    coarserow_s<N, ZS>(t, L, SrcX{xf, xc}, I, J, K, diag, off);
}

// The fine pool cell of thread index n: slot (1-based), local (i, j, k).
template <int N>
__device__ __forceinline__ void pool_cell(int64_t n, int& sl, int& i, int& j, int& k) {
    constexpr int S = Lv<N>::SH;
    sl = (int)(n >> (3 * S)) + 1;
    const int c = (int)(n & (N * N * N - 1));
    i = c & (N - 1);
    j = (c >> S) & (N - 1);
    k = c >> (2 * S);
}
// (i, j, k) of linear index o over n0 x n1 (x n2): 32-bit arithmetic (the library keeps every
// grid and face array below 2^31 elements)
__device__ __forceinline__ void split3(int64_t o, int n0, int n1, int& i, int& j, int& k) {
    const int v = (int)o, r = v / n0;
    i = v - r * n0;
    k = r / n1;
    j = r - k * n1;
}
__device__ __forceinline__ void coarse_cell(const Topo& t, int64_t c, int& I, int& J, int& K) {
    split3(c, t.nc[0], t.nc[1], I, J, K);
}

// A fused launch's CTAs: the coarse part first (CTAs [0, gridDim - gf), dispatched first, so
// its slower cells next to fine blocks overlap the fine part instead of trailing it), the
// fine part the last gf (a CTA per slot in the block kernels, a grid-stride range otherwise).
__device__ __forceinline__ bool sp_is_fine(int gf) { return (int)blockIdx.x >= (int)gridDim.x - gf; }
__device__ __forceinline__ int sp_slot(int gf) { return (int)blockIdx.x - ((int)gridDim.x - gf) + 1; }
#define SP_FINE_LOOP(n, total, gf)                                                                        \
    for (int64_t n = (int64_t)((int)blockIdx.x - ((int)gridDim.x - (gf))) * blockDim.x + threadIdx.x; n < (total); \
         n += (int64_t)(gf) * blockDim.x)
// The coarse part's walk over the operator's list of coarse unknowns (the coarse CTAs of a
// fused launch, [0, gridDim - gf), as SP_COARSE_LOOP).
#define SP_ACTIVE_LOOP(c, L, gf)                                                                   \
    for (int64_t e_ = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, ne_ = *(L).nclist; e_ < ne_; \
         e_ += (int64_t)(gridDim.x - (gf)) * blockDim.x)                                           \
        if (const int64_t c = (L).clist[e_]; true)
#define SP_COARSE_LOOP(c, total, gf)                                                               \
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < (total);                  \
         c += (int64_t)(gridDim.x - (gf)) * blockDim.x)

// ---- coefficients, level 0 (src/sflip.jl:1315-1451) ----
// finecoef_kernel! (:1324-1333), the three axes (blockIdx.y)
__global__ void __launch_bounds__(SPT) k_sp_finecoef(Topo t, float* cu, float* cv, float* cw, const uint8_t* tf,
                                                     const uint8_t* tc) {
    pdl_wait();
    pdl_trigger();
    const int a = (int)blockIdx.y + 1;
    float* c = a == 1 ? cu : (a == 2 ? cv : cw);
    const int64_t nf = (int64_t)t.nslots * BFACES;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += (int64_t)gridDim.x * blockDim.x) {
        const int sl = (int)n / BFACES + 1, f = (int)n - (sl - 1) * BFACES;
        int w[3];
        where_of(t, sl, w);
        if (w[0] < 0) continue;
        int i, j, k;
        if (a == 1) { i = f % 17; const int r = f / 17; j = r & 15; k = r >> 4; }
        else if (a == 2) { i = f & 15; const int r = f >> 4; j = r % 17; k = r / 17; }
        else { i = f & 15; j = (f >> 4) & 15; k = f >> 8; }
        const int I = w[0] * BLOCK + i, J = w[1] * BLOCK + j, K = w[2] * BLOCK + k;
        bool fp, fm;
        const uint8_t tp = celltype(t, tf, tc, I, J, K, fp);
        const uint8_t tm = celltype(t, tf, tc, I - (a == 1), J - (a == 2), K - (a == 3), fm);
        c[n] = (tp == LIQUID && tm == LIQUID) ? (fp && fm ? FINE_FINE : FINE_COARSE) : 0.0f;
    }
}
// coarsecoef_kernel! (:1344-1354), the three axes
__global__ void __launch_bounds__(SPT) k_sp_coarsecoef(Topo t, float* cu, float* cv, float* cw, const uint8_t* tc) {
    pdl_wait();
    pdl_trigger();
    const int a = (int)blockIdx.y + 1, e0 = a == 1, e1 = a == 2, e2 = a == 3;
    float* c = a == 1 ? cu : (a == 2 ? cv : cw);
    const int f0 = t.nc[0] + e0, f1 = t.nc[1] + e1, f2 = t.nc[2] + e2;
    const int64_t nfc = (int64_t)f0 * f1 * f2;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nfc; o += (int64_t)gridDim.x * blockDim.x) {
        int I, J, K;
            split3(o, f0, f1, I, J, K);
        const int Im = I - e0, Jm = J - e1, Km = K - e2;
        const bool ok = 0 <= Im && 0 <= Jm && 0 <= Km && I < t.nc[0] && J < t.nc[1] && K < t.nc[2];
        c[o] = (ok && !covered(t, I, J, K) && !covered(t, Im, Jm, Km) && tc[lin(t.nc, I, J, K)] == LIQUID &&
                tc[lin(t.nc, Im, Jm, Km)] == LIQUID)
                   ? COARSE_COARSE
                   : 0.0f;
    }
}
// finedirichlet_kernel! (:1356-1374) + coarsedirichlet_kernel! (:1376-1407) +
// activecoarse_kernel! (:1315-1319), one launch (fine part first)
//
// The fine part also packs each cell's six couplings for the block kernels (code0: 2 bits a
// face in finerow's order -x, +x, -y, +y, -z, +z: 0 none, 1 FINE_COARSE, 2 FINE_FINE; bit 12
// active (not SOLID), bit 13 LIQUID) and its whole diagonal dg0 = dD + the positive
// couplings, added in finerow's order (the same Float32 sums finerow forms every sweep); the
// coarse part marks the coarse unknowns (LIQUID, no fine block over them) for the dots.
__device__ __forceinline__ unsigned ccode(float c) { return c == FINE_FINE ? 2u : (c == FINE_COARSE ? 1u : 0u); }
__global__ void __launch_bounds__(SPT) k_sp_dirichlet(Topo t, float* dDf, float* dDc, uint8_t* actc, const uint8_t* tf,
                                                      const uint8_t* tc, const float* phif, const float* phic,
                                                      const float* cfx, const float* cfy, const float* cfz,
                                                      uint16_t* code0, float* dg0, uint8_t* cmask, int* clist,
                                                      int* nclist, int gf) {
    pdl_wait();
    pdl_trigger();
    if (sp_is_fine(gf)) {
        const int64_t nf = (int64_t)t.nslots * BCELLS;
        SP_FINE_LOOP(n, nf, gf) {
            int sl, i, j, k;
            pool_cell<16>(n, sl, i, j, k);
            int w[3];
            where_of(t, sl, w);
            if (w[0] < 0) continue;
            float d = 0.0f;
            if (tf[n] == LIQUID) {
                const int I = w[0] * BLOCK + i, J = w[1] * BLOCK + j, K = w[2] * BLOCK + k;
                const float pc = phif[n];
                // neighbour (src/flip.jl:84-92): +x, -x, +y, -y, +z, -z
#pragma unroll
                for (int m = 0; m < 6; m++) {
                    const int a = I + (m == 0) - (m == 1), b = J + (m == 2) - (m == 3), cc = K + (m == 4) - (m == 5);
                    bool fine;
                    const uint8_t ty = celltype(t, tf, tc, a, b, cc, fine);
                    if (ty == AIR) d += (fine ? FINE_FINE : FINE_COARSE) / theta<float>(pc, fine_or_coarse(t, phif, phic, a, b, cc));
                }
            }
            dDf[n] = d;
            const float c6[6] = {cfx[L16::face(sl, 1, i, j, k) - 1], cfx[L16::face(sl, 1, i + 1, j, k) - 1],
                                 cfy[L16::face(sl, 2, i, j, k) - 1], cfy[L16::face(sl, 2, i, j + 1, k) - 1],
                                 cfz[L16::face(sl, 3, i, j, k) - 1], cfz[L16::face(sl, 3, i, j, k + 1) - 1]};
            float dg = d;
            unsigned code = (tf[n] != SOLID ? 1u << 12 : 0u) | (tf[n] == LIQUID ? 1u << 13 : 0u);
#pragma unroll
            for (int m = 0; m < 6; m++) {
                if (c6[m] > 0.0f) dg += c6[m];
                code |= ccode(c6[m]) << (2 * m);
            }
            code0[n] = (uint16_t)code;
            dg0[n] = dg;
        }
    } else {
        const int64_t nc = (int64_t)t.nc[0] * t.nc[1] * t.nc[2];
        const int n1 = t.nc[0], n2 = t.nc[1], n3 = t.nc[2];
        SP_COARSE_LOOP(c, nc, gf) {
            int I, J, K;
            coarse_cell(t, c, I, J, K);
            const bool cov = covered(t, I, J, K);
            float d = 0.0f;
            if (tc[c] == LIQUID && !cov) {
                const float pc = phic[c];
                for (int a = 1; a <= 3; a++) {
                    const int e0 = a == 1, e1 = a == 2, e2 = a == 3;
                    for (int sg = -1; sg <= 1; sg += 2) {
                        const int In = I + sg * e0, Jn = J + sg * e1, Kn = K + sg * e2;
                        if (!(0 <= In && In < n1 && 0 <= Jn && Jn < n2 && 0 <= Kn && Kn < n3)) continue;
                        if (covered(t, In, Jn, Kn)) {
                            for (int q = 0; q < 4; q++)
                                for (int p = 0; p < 4; p++) {
                                    const int FI = a == 1 ? (sg > 0 ? RATIO * In : RATIO * I - 1) : RATIO * I + p;
                                    const int FJ = a == 2 ? (sg > 0 ? RATIO * Jn : RATIO * J - 1) : RATIO * J + (a == 1 ? p : q);
                                    const int FK = a == 3 ? (sg > 0 ? RATIO * Kn : RATIO * K - 1) : RATIO * K + q;
                                    const int64_t idx = fineat(t, FI, FJ, FK);
                                    if (idx > 0 && tf[idx - 1] == AIR) d += FINE_COARSE / theta<float>(pc, phif[idx - 1]);
                                }
                        } else if (tc[lin(t.nc, In, Jn, Kn)] == AIR) {
                            d += COARSE_COARSE / theta<float>(pc, phic[lin(t.nc, In, Jn, Kn)]);
                        }
                    }
                }
            }
            dDc[c] = d;
            actc[c] = (tc[c] == LIQUID && !cov) ? 1 : 0;
            cmask[c] = actc[c];
            if (actc[c]) clist[atomicAdd(nclist, 1)] = (int)c;
        }
    }
}

// ---- the hierarchy (src/sflip.jl:1453-1586) ----
// coef1_kernel! (:1453-1465): level 1's faces, the sums of the four level-0 faces they cover
__global__ void __launch_bounds__(SPT) k_sp_coef1(Topo t, float* c1x, float* c1y, float* c1z, const float* c0x,
                                                  const float* c0y, const float* c0z) {
    pdl_wait();
    pdl_trigger();
    const int a = (int)blockIdx.y + 1;
    const float* c0 = a == 1 ? c0x : (a == 2 ? c0y : c0z);
    float* c1 = a == 1 ? c1x : (a == 2 ? c1y : c1z);
    const int64_t nf = (int64_t)t.nslots * BFACES1;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nf; n += (int64_t)gridDim.x * blockDim.x) {
        const int sl = (int)n / BFACES1 + 1, f = (int)n - (sl - 1) * BFACES1;
        if (!slot_used(t, sl)) continue;
        int i, j, k;
        if (a == 1) { i = f % 9; const int r = f / 9; j = r % 8; k = r / 8; }
        else if (a == 2) { i = f % 8; const int r = f / 8; j = r % 9; k = r / 9; }
        else { i = f % 8; const int r = f / 8; j = r % 8; k = r / 8; }
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < 2; q++)
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const int ii = a == 1 ? 2 * i : 2 * i + p;
                const int jj = a == 2 ? 2 * j : 2 * j + (a == 1 ? p : q);
                const int kk = a == 3 ? 2 * k : 2 * k + q;
                acc += c0[L16::face(sl, a, ii, jj, kk) - 1];
            }
        c1[n] = acc;
    }
}
// cells1_kernel! (:1467-1479)
// and each level-1 cell's whole diagonal dg1 = dD1 + its positive couplings in finerow's
// order (the block kernels of level 1 read it; the same Float32 sums finerow forms).
__global__ void __launch_bounds__(SPT) k_sp_cells1(Topo t, float* dD1, uint8_t* act1, const float* dD0,
                                                   const uint8_t* tf, const float* c1x, const float* c1y,
                                                   const float* c1z, float* dg1) {
    pdl_wait();
    pdl_trigger();
    const int64_t n1 = (int64_t)t.nslots * BCELLS1;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < n1; n += (int64_t)gridDim.x * blockDim.x) {
        int sl, i, j, k;
        pool_cell<8>(n, sl, i, j, k);
        if (!slot_used(t, sl)) continue;
        float d = 0.0f;
        uint8_t act = 0;
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int a = 0; a < 2; a++) {
                    const int64_t m = L16::cell(sl, 2 * i + a, 2 * j + b, 2 * k + c) - 1;
                    d += dD0[m];
                    if (tf[m] == LIQUID) act = 1;
                }
        dD1[n] = d;
        act1[n] = act;
        const float c6[6] = {c1x[L8::face(sl, 1, i, j, k) - 1], c1x[L8::face(sl, 1, i + 1, j, k) - 1],
                             c1y[L8::face(sl, 2, i, j, k) - 1], c1y[L8::face(sl, 2, i, j + 1, k) - 1],
                             c1z[L8::face(sl, 3, i, j, k) - 1], c1z[L8::face(sl, 3, i, j, k + 1) - 1]};
#pragma unroll
        for (int m = 0; m < 6; m++)
            if (c6[m] > 0.0f) d += c6[m];
        dg1[n] = d;
    }
}
// coef2_kernel! (:1485-1507), the three axes, and cells2_kernel! (:1509-1523) as blockIdx.y == 3
__global__ void __launch_bounds__(SPT) k_sp_level2(Topo t, float* c2x, float* c2y, float* c2z, const float* c0x,
                                                   const float* c0y, const float* c0z, const float* c1x,
                                                   const float* c1y, const float* c1z, float* dD2, uint8_t* act2,
                                                   const float* dD0c, const float* dD1, const uint8_t* act1) {
    pdl_wait();
    pdl_trigger();
    const int a = (int)blockIdx.y + 1;
    if (a <= 3) {
        const int e0 = a == 1, e1 = a == 2, e2 = a == 3;
        const float* c0 = a == 1 ? c0x : (a == 2 ? c0y : c0z);
        const float* c1 = a == 1 ? c1x : (a == 2 ? c1y : c1z);
        float* c2 = a == 1 ? c2x : (a == 2 ? c2y : c2z);
        const int f0 = t.nc[0] + e0, f1 = t.nc[1] + e1, f2 = t.nc[2] + e2;
        const int64_t nfc = (int64_t)f0 * f1 * f2;
        for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nfc; o += (int64_t)gridDim.x * blockDim.x) {
            int I, J, K;
            split3(o, f0, f1, I, J, K);
            if (covered(t, I, J, K) || covered(t, I - e0, J - e1, K - e2)) {
                float acc = 0.0f;
#pragma unroll
                for (int q = 0; q < 2; q++)
#pragma unroll
                    for (int p = 0; p < 2; p++) {
                        const int FI = a == 1 ? 2 * I : 2 * I + p;
                        const int FJ = a == 2 ? 2 * J : 2 * J + (a == 1 ? p : q);
                        const int FK = a == 3 ? 2 * K : 2 * K + q;
                        const int64_t idx = L8::faceat(t, a, FI, FJ, FK);
                        if (idx > 0) acc += c1[idx - 1];
                    }
                c2[o] = acc;
            } else {
                c2[o] = c0[o];
            }
        }
    } else {
        const int64_t nc = (int64_t)t.nc[0] * t.nc[1] * t.nc[2];
        for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nc; o += (int64_t)gridDim.x * blockDim.x) {
            int I, J, K;
            coarse_cell(t, o, I, J, K);
            if (covered(t, I, J, K)) {
                float d = 0.0f;
                uint8_t act = 0;
#pragma unroll
                for (int c = 0; c < 2; c++)
#pragma unroll
                    for (int b = 0; b < 2; b++)
#pragma unroll
                        for (int aa = 0; aa < 2; aa++) {
                            const int64_t m = L8::cellat(t, 2 * I + aa, 2 * J + b, 2 * K + c) - 1;
                            d += dD1[m];
                            if (act1[m] != 0) act = 1;
                        }
                dD2[o] = d;
                act2[o] = act;
            } else {
                dD2[o] = dD0c[o];
            }
        }
    }
}

// A dense level of the hierarchy.
struct DL {
    int n[3];
    float *x, *b, *r, *t, *cx, *cy, *cz, *dD;
    uint8_t* act;
};
// coefdense_kernel! (:1525-1535), the three axes, and cellsdense_kernel! (:1537-1546) as blockIdx.y == 3
__global__ void __launch_bounds__(SPT) k_sp_dense_level(DL F, DL C) {
    pdl_wait();
    pdl_trigger();
    const int a = (int)blockIdx.y + 1;
    if (a <= 3) {
        const int e0 = a == 1, e1 = a == 2, e2 = a == 3;
        const float* cf = a == 1 ? F.cx : (a == 2 ? F.cy : F.cz);
        float* cc = a == 1 ? C.cx : (a == 2 ? C.cy : C.cz);
        const int g0 = F.n[0] + e0, g1 = F.n[1] + e1;
        const int f0 = C.n[0] + e0, f1 = C.n[1] + e1, f2 = C.n[2] + e2;
        const int64_t nfc = (int64_t)f0 * f1 * f2;
        for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nfc; o += (int64_t)gridDim.x * blockDim.x) {
            int I, J, K;
            split3(o, f0, f1, I, J, K);
            float acc = 0.0f;
#pragma unroll
            for (int q = 0; q < 2; q++)
#pragma unroll
                for (int p = 0; p < 2; p++) {
                    const int FI = a == 1 ? 2 * I : 2 * I + p;
                    const int FJ = a == 2 ? 2 * J : 2 * J + (a == 1 ? p : q);
                    const int FK = a == 3 ? 2 * K : 2 * K + q;
                    acc += cf[lin3(g0, g1, FI, FJ, FK)];
                }
            cc[o] = acc;
        }
    } else {
        const int64_t nc = (int64_t)C.n[0] * C.n[1] * C.n[2];
        for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nc; o += (int64_t)gridDim.x * blockDim.x) {
            int I, J, K;
            split3(o, C.n[0], C.n[1], I, J, K);
            float d = 0.0f;
            uint8_t act = 0;
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int b = 0; b < 2; b++)
#pragma unroll
                    for (int aa = 0; aa < 2; aa++) {
                        const int64_t m = lin(F.n, 2 * I + aa, 2 * J + b, 2 * K + c);
                        d += F.dD[m];
                        if (F.act[m] != 0) act = 1;
                    }
            C.dD[o] = d;
            C.act[o] = act;
        }
    }
}

// ---- the dense levels (src/sflip.jl:1575-1660) ----
// denserow (:1575-1586)
template <bool ZS>
__device__ __forceinline__ void denserow(const DL& L, const float* x, int i, int j, int k, int64_t c, float& diag,
                                         float& off) {
    const int n1 = L.n[0], n2 = L.n[1], n3 = L.n[2];
    diag = L.dD[c];
    off = 0.0f;
    float v;
    v = L.cx[lin3(n1 + 1, n2, i, j, k)];
    if (v > 0.0f && i > 0) { diag += v; off += v * (ZS ? 0.0f : x[c - 1]); }
    v = L.cx[lin3(n1 + 1, n2, i + 1, j, k)];
    if (v > 0.0f && i < n1 - 1) { diag += v; off += v * (ZS ? 0.0f : x[c + 1]); }
    v = L.cy[lin3(n1, n2 + 1, i, j, k)];
    if (v > 0.0f && j > 0) { diag += v; off += v * (ZS ? 0.0f : x[c - n1]); }
    v = L.cy[lin3(n1, n2 + 1, i, j + 1, k)];
    if (v > 0.0f && j < n2 - 1) { diag += v; off += v * (ZS ? 0.0f : x[c + n1]); }
    v = L.cz[lin3(n1, n2, i, j, k)];
    if (v > 0.0f && k > 0) { diag += v; off += v * (ZS ? 0.0f : x[c - (int64_t)n1 * n2]); }
    v = L.cz[lin3(n1, n2, i, j, k + 1)];
    if (v > 0.0f && k < n3 - 1) { diag += v; off += v * (ZS ? 0.0f : x[c + (int64_t)n1 * n2]); }
}
// jacobidense_kernel! (:1588-1596)
template <bool ZS>
__global__ void __launch_bounds__(SPT) k_sp_djacobi(DL L, float* out, const float* x) {
    pdl_wait();
    pdl_trigger();
    const int64_t nc = (int64_t)L.n[0] * L.n[1] * L.n[2];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        float v = 0.0f;
        if (L.act[c] != 0) {
            int i, j, k;
            split3(c, L.n[0], L.n[1], i, j, k);
            float diag, off;
            denserow<ZS>(L, x, i, j, k, c, diag, off);
            const float x0 = ZS ? 0.0f : x[c];
            v = diag > 0.0f ? x0 + OMEGA * (L.b[c] - (diag * x0 - off)) / diag : 0.0f;
        }
        out[c] = v;
    }
}
// residualdense_kernel! (:1598-1607) + restrictdense_kernel! (:1609-1616) of the level below
// are two launches: the restriction reads the residual's neighbours.
__global__ void __launch_bounds__(SPT) k_sp_dresidual(DL L) {
    pdl_wait();
    pdl_trigger();
    const int64_t nc = (int64_t)L.n[0] * L.n[1] * L.n[2];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        float v = 0.0f;
        if (L.act[c] != 0) {
            int i, j, k;
            split3(c, L.n[0], L.n[1], i, j, k);
            float diag, off;
            denserow<false>(L, L.x, i, j, k, c, diag, off);
            v = L.b[c] - (diag * L.x[c] - off);
        }
        L.r[c] = v;
    }
}
__global__ void __launch_bounds__(SPT) k_sp_drestrict(DL F, DL C) {
    pdl_wait();
    pdl_trigger();
    const int64_t nc = (int64_t)C.n[0] * C.n[1] * C.n[2];
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nc; o += (int64_t)gridDim.x * blockDim.x) {
        int i, j, k;
            split3(o, C.n[0], C.n[1], i, j, k);
        float acc = 0.0f;
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int a = 0; a < 2; a++) acc += F.r[lin(F.n, 2 * i + a, 2 * j + b, 2 * k + c)];
        C.b[o] = acc;
    }
}
// prolongdense_kernel! (:1618-1621)
__global__ void __launch_bounds__(SPT) k_sp_dprolong(DL F, DL C, float boost) {
    pdl_wait();
    pdl_trigger();
    const int64_t nc = (int64_t)F.n[0] * F.n[1] * F.n[2];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        if (F.act[c] == 0) continue;
        int i, j, k;
            split3(c, F.n[0], F.n[1], i, j, k);
        F.x[c] += boost * C.x[lin(C.n, i >> 1, j >> 1, k >> 1)];
    }
}
// coarsest_kernel! (:1627-1660): red-black Gauss-Seidel from zero in one CTA's shared memory,
// `sweeps` sweeps and as many in the reverse colour order. A thread a cell (<= 1024 cells).
__global__ void __launch_bounds__(1024) k_sp_coarsest(DL L, int sweeps) {
    pdl_wait();
    pdl_trigger();
    __shared__ float xs[1024];
    const int t = (int)threadIdx.x, n1 = L.n[0], n2 = L.n[1], n3 = L.n[2], N = n1 * n2 * n3;
    const bool inside = t < N;
    const int i = t % n1, j = (t / n1) % n2, k = t / (n1 * n2);
    const bool act = inside && L.act[t] != 0;
    const int par = (i + j + k + 1) & 1;  // the reference's 1-based (i + j + k) % 2
    float bi = 0.0f, d0 = 0.0f, c[6] = {0, 0, 0, 0, 0, 0};
    if (inside) {
        bi = L.b[t];
        d0 = L.dD[t];
        c[0] = L.cx[lin3(n1 + 1, n2, i, j, k)];
        c[1] = L.cx[lin3(n1 + 1, n2, i + 1, j, k)];
        c[2] = L.cy[lin3(n1, n2 + 1, i, j, k)];
        c[3] = L.cy[lin3(n1, n2 + 1, i, j + 1, k)];
        c[4] = L.cz[lin3(n1, n2, i, j, k)];
        c[5] = L.cz[lin3(n1, n2, i, j, k + 1)];
    }
    xs[t] = 0.0f;
    __syncthreads();
    for (int s = 1; s <= 2 * sweeps; s++)
        for (int half = 0; half <= 1; half++) {
            const int colour = s <= sweeps ? half : 1 - half;
            if (act && par == colour) {
                float diag = d0, acc = bi;
                if (c[0] > 0.0f && i > 0) { diag += c[0]; acc += c[0] * xs[t - 1]; }
                if (c[1] > 0.0f && i < n1 - 1) { diag += c[1]; acc += c[1] * xs[t + 1]; }
                if (c[2] > 0.0f && j > 0) { diag += c[2]; acc += c[2] * xs[t - n1]; }
                if (c[3] > 0.0f && j < n2 - 1) { diag += c[3]; acc += c[3] * xs[t + n1]; }
                if (c[4] > 0.0f && k > 0) { diag += c[4]; acc += c[4] * xs[t - n1 * n2]; }
                if (c[5] > 0.0f && k < n3 - 1) { diag += c[5]; acc += c[5] * xs[t + n1 * n2]; }
                xs[t] = diag > 0.0f ? acc / diag : 0.0f;
            }
            __syncthreads();
        }
    if (inside) L.x[t] = xs[t];
}

// ---- between levels (src/sflip.jl:1662-1705) ----
// restrict01_kernel! (:1662-1672): level 1's fine right-hand side (its coarse part is level
// 0's coarse residual itself)
__global__ void __launch_bounds__(SPT) k_sp_restrict01(Topo t, float* b1f, const float* r0f) {
    pdl_wait();
    pdl_trigger();
    const int64_t n1 = (int64_t)t.nslots * BCELLS1;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < n1; n += (int64_t)gridDim.x * blockDim.x) {
        int sl, i, j, k;
        pool_cell<8>(n, sl, i, j, k);
        if (!slot_used(t, sl)) continue;
        float acc = 0.0f;
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int a = 0; a < 2; a++) acc += r0f[L16::cell(sl, 2 * i + a, 2 * j + b, 2 * k + c) - 1];
        b1f[n] = acc;
    }
}
// restrict12_kernel! (:1674-1686)
__global__ void __launch_bounds__(SPT) k_sp_restrict12(Topo t, float* b2, const float* r1f, const float* r1c) {
    pdl_wait();
    pdl_trigger();
    const int64_t nc = (int64_t)t.nc[0] * t.nc[1] * t.nc[2];
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nc; o += (int64_t)gridDim.x * blockDim.x) {
        int I, J, K;
        coarse_cell(t, o, I, J, K);
        if (covered(t, I, J, K)) {
            float acc = 0.0f;
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int b = 0; b < 2; b++)
#pragma unroll
                    for (int a = 0; a < 2; a++) acc += r1f[L8::cellat(t, 2 * I + a, 2 * J + b, 2 * K + c) - 1];
            b2[o] = acc;
        } else {
            b2[o] = r1c[o];
        }
    }
}
// prolong21fine_kernel! + prolongcoarse_kernel! (:1688-1699) as one launch: level 2's
// correction added to level 1's active fine cells (each from the coarse cell it lies in) and
// to its active coarse cells outside fine blocks.
__global__ void __launch_bounds__(SPT) k_sp_prolong21(Topo t, float* xf, float* xc, const float* x2,
                                                      const uint8_t* act1, const uint8_t* act2, float boost, int gf) {
    pdl_wait();
    pdl_trigger();
    if (sp_is_fine(gf)) {
        const int64_t nf = (int64_t)t.nslots * BCELLS1;
        SP_FINE_LOOP(n, nf, gf) {
            int sl, i, j, k;
            pool_cell<8>(n, sl, i, j, k);
            int w[3];
            where_of(t, sl, w);
            if (w[0] < 0 || act1[n] == 0) continue;
            xf[n] += boost * x2[lin(t.nc, (w[0] * 8 + i) >> 1, (w[1] * 8 + j) >> 1, (w[2] * 8 + k) >> 1)];
        }
    } else {
        const int64_t nc = (int64_t)t.nc[0] * t.nc[1] * t.nc[2];
        SP_COARSE_LOOP(c, nc, gf) {
            int I, J, K;
            coarse_cell(t, c, I, J, K);
            if (act2[c] != 0 && !covered(t, I, J, K)) xc[c] += boost * x2[c];
        }
    }
}

// ---- the CG (src/sflip.jl:1766-1904): device-resident Float32 scalars ----
struct SpState {
    float tol;
    int maxiter;
    float bnorm, target, rnorm, rho, alpha, beta, den;
    int status, it, done;
    float vol, gamma;  // project!'s volume and volume-control divergence
    float volume0;
    int pad;
    double dt, recover;
};

// The inner (src/sflip.jl:1794-1805) masks: LIQUID fine cells of slots in use; LIQUID coarse
// cells outside fine blocks.
__device__ __forceinline__ bool fine_unknown(const Topo& t, const uint8_t* tf, int64_t n) {
    return tf[n] == LIQUID && slot_used(t, (int)(n >> 12) + 1);
}
__device__ __forceinline__ bool coarse_unknown(const Topo& t, const uint8_t* tc, int64_t c) {
    if (tc[c] != LIQUID) return false;
    int I, J, K;
    coarse_cell(t, c, I, J, K);
    return !covered(t, I, J, K);
}
__device__ __forceinline__ float f32sum(double v) { return (float)v; }

// apply! at level 0's coarse part (src/sflip.jl:1837-1847): q = A x on active uncovered
// coarse cells, else 0.
__device__ __forceinline__ float apply_coarse(const Topo& t, const Comp& L, const float* xf, const float* xc, int64_t c,
                                              bool& cov) {
    int I, J, K;
    coarse_cell(t, c, I, J, K);
    cov = covered(t, I, J, K);
    if (L.actc[c] == 0 || cov) return 0.0f;
    float diag, off;
    coarserow<16, false>(t, L, xf, xc, I, J, K, diag, off);
    return diag * xc[c] - off;
}


// ---- level 0's fine part, a CTA per 16^3 block ----
// The level's stencil passes (Jacobi sweeps, the residual, apply!) run one CTA per slot:
// the block's x (4096 cells, 16-byte loads) and its one-cell halo (6 x 256 cells: the
// neighbouring block's boundary plane where that block is fine, else the coarse cell the
// halo cell lies in, as finerow's neighbourvalue) are staged in shared memory; each thread
// then takes four consecutive cells of a row four times, reading their codes (code0: the six
// couplings, 2 bits each, and the active and LIQUID bits), whole diagonals (dg0) and right-
// hand sides as 8- and 16-byte loads and their neighbours from shared memory. Per cell the
// arithmetic is finerow's: off sums c x_n over the positive couplings in the order -x, +x,
// -y, +y, -z, +z, and diag is dg0, the same Float32 sums.
constexpr int PX = 18, PXY = PX * PX, PCELLS = PXY * PX;  // the staged block with its halo
__device__ __forceinline__ int pidx(int i, int j, int k) { return (k + 1) * PXY + (j + 1) * PX + (i + 1); }
__device__ __forceinline__ float cdec(unsigned code, int m) {
    const unsigned v = (code >> (2 * m)) & 3u;
    return v == 2u ? FINE_FINE : (v == 1u ? FINE_COARSE : 0.0f);
}

// Stage slot sl's x and its halo into xs (256 threads).
template <class Src>
__device__ __forceinline__ void stage_block_s(const Topo& t, const Src& src, int sl, const int w[3], float* xs) {
    const int tid = (int)threadIdx.x;
    const int64_t base = (int64_t)(sl - 1) * BCELLS;
    float4 v[4];
#pragma unroll
    for (int m = 0; m < 4; m++) v[m] = src.fine4(base + 4 * (tid + 256 * m));
    const int p = tid & 15, q = tid >> 4;
    float hv[6];
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const int ax = f >> 1, sg = (f & 1) ? 1 : -1;
        const int i = ax == 0 ? (sg < 0 ? -1 : 16) : p;
        const int j = ax == 1 ? (sg < 0 ? -1 : 16) : (ax == 0 ? p : q);
        const int k = ax == 2 ? (sg < 0 ? -1 : 16) : q;
        const int nbi = w[0] + (ax == 0 ? sg : 0), nbj = w[1] + (ax == 1 ? sg : 0), nbk = w[2] + (ax == 2 ? sg : 0);
        const int s2 = inblocks(t, nbi, nbj, nbk) ? blockslot(t, nbi, nbj, nbk) : 0;
        if (s2 > 0) {
            hv[f] = src.fine((int64_t)(s2 - 1) * BCELLS + (i & 15) + 16 * ((j & 15) + 16 * (k & 15)));
        } else {
            const int I = w[0] * BLOCK + i, J = w[1] * BLOCK + j, K = w[2] * BLOCK + k;
            hv[f] = src.coarse(coarse_clamped(t, I >> 2, J >> 2, K >> 2));
        }
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int c = 4 * (tid + 256 * m), i = c & 15, j = (c >> 4) & 15, k = c >> 8;
        float* d = xs + pidx(i, j, k);
        d[0] = v[m].x;
        d[1] = v[m].y;
        d[2] = v[m].z;
        d[3] = v[m].w;
    }
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const int ax = f >> 1, sg = (f & 1) ? 1 : -1;
        const int i = ax == 0 ? (sg < 0 ? -1 : 16) : p;
        const int j = ax == 1 ? (sg < 0 ? -1 : 16) : (ax == 0 ? p : q);
        const int k = ax == 2 ? (sg < 0 ? -1 : 16) : q;
        xs[pidx(i, j, k)] = hv[f];
    }
}

__device__ __forceinline__ void stage_block(const Topo& t, const float* __restrict__ x, const float* __restrict__ xc,
                                            int sl, const int w[3], float* xs) {
    stage_block_s(t, SrcX{x, xc}, sl, w, xs);
}

// off of one cell from the staged block (ZS: x all zeros, off = 0).
template <bool ZS>
__device__ __forceinline__ float block_off(const float* xs, int o, unsigned code) {
    float off = 0.0f;
    if (ZS) return off;
    const int nb[6] = {-1, 1, -PX, PX, -PXY, PXY};
#pragma unroll
    for (int m = 0; m < 6; m++) {
        const float c = cdec(code, m);
        if (c > 0.0f) off += c * xs[o + nb[m]];
    }
    return off;
}

// The block operations: a Jacobi sweep (from x, or from zeros), the residual, and A x.
enum { BOP_JAC = 0, BOP_JAC_ZS = 1, BOP_RES = 2, BOP_APPLY = 3 };

// One slot's cells through `op`; `sink(n, value, x)` receives each cell's result (pool
// index, value, the cell's own x). The caller has staged x into xs (not for BOP_JAC_ZS).
template <int OP, class Sink>
__device__ __forceinline__ void block_cells(const uint16_t* __restrict__ code0, const float* __restrict__ dg0,
                                            const float* __restrict__ b, const float* xs, int sl, Sink&& sink) {
    const int tid = (int)threadIdx.x;
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
        const int q = tid + 256 * m, c = 4 * q, i = c & 15, j = (c >> 4) & 15, k = c >> 8;
        const int64_t n = (int64_t)(sl - 1) * BCELLS + c;
        const ushort4 cd = *reinterpret_cast<const ushort4*>(code0 + n);
        const float4 dg = *reinterpret_cast<const float4*>(dg0 + n);
        float4 bb = make_float4(0.f, 0.f, 0.f, 0.f);
        if (OP != BOP_APPLY) bb = *reinterpret_cast<const float4*>(b + n);
        const unsigned cs[4] = {cd.x, cd.y, cd.z, cd.w};
        const float ds[4] = {dg.x, dg.y, dg.z, dg.w}, bs[4] = {bb.x, bb.y, bb.z, bb.w};
        float out[4], xv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int o = pidx(i + u, j, k);
            const unsigned code = cs[u];
            const float x0 = OP == BOP_JAC_ZS ? 0.0f : xs[o];
            xv[u] = x0;
            const float diag = ds[u];
            float v = 0.0f;
            if (OP == BOP_APPLY) {
                if (code & (1u << 13)) v = diag * x0 - block_off<false>(xs, o, code);
            } else if (code & (1u << 12)) {
                const float off = OP == BOP_JAC_ZS ? block_off<true>(xs, o, code) : block_off<false>(xs, o, code);
                if (OP == BOP_RES) v = bs[u] - (diag * x0 - off);
                else v = diag > 0.0f ? x0 + OMEGA * (bs[u] - (diag * x0 - off)) / diag : 0.0f;
            }
            out[u] = v;
        }
        sink(n, out, xv);
    }
}


// ---- level 1's fine part, a CTA (128 threads) per 8^3 block ----
// As level 0's block kernels: the block's x (512 cells) and its halo (6 x 64 cells: the
// neighbouring block's boundary plane, else the coarse cell the halo cell lies in) staged in
// shared memory, a thread a piece of four cells of a row. The couplings are level 1's
// aggregated face arrays (sums of four level-0 faces, read as floats), the diagonal dg1.
constexpr int T8 = 128, Q = 10, QY = Q * Q, QCELLS = QY * Q;
__device__ __forceinline__ int qidx(int i, int j, int k) { return (k + 1) * QY + (j + 1) * Q + (i + 1); }

__device__ __forceinline__ void stage_block8(const Topo& t, const float* __restrict__ x, const float* __restrict__ xc,
                                             int sl, const int w[3], float* xs) {
    const int tid = (int)threadIdx.x;
    const float4 v = reinterpret_cast<const float4*>(x + (int64_t)(sl - 1) * BCELLS1)[tid];
    float hv[3];
    int hi[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
        const int h = tid + T8 * u, f = h >> 6, pq = h & 63, p = pq & 7, q = pq >> 3;
        const int ax = f >> 1, sg = (f & 1) ? 1 : -1;
        const int i = ax == 0 ? (sg < 0 ? -1 : 8) : p;
        const int j = ax == 1 ? (sg < 0 ? -1 : 8) : (ax == 0 ? p : q);
        const int k = ax == 2 ? (sg < 0 ? -1 : 8) : q;
        const int nbi = w[0] + (ax == 0 ? sg : 0), nbj = w[1] + (ax == 1 ? sg : 0), nbk = w[2] + (ax == 2 ? sg : 0);
        const int s2 = inblocks(t, nbi, nbj, nbk) ? blockslot(t, nbi, nbj, nbk) : 0;
        if (s2 > 0) {
            hv[u] = x[(int64_t)(s2 - 1) * BCELLS1 + (i & 7) + 8 * ((j & 7) + 8 * (k & 7))];
        } else {
            const int I = w[0] * 8 + i, J = w[1] * 8 + j, K = w[2] * 8 + k;
            hv[u] = xc[coarse_clamped(t, I >> 1, J >> 1, K >> 1)];
        }
        hi[u] = qidx(i, j, k);
    }
    const int c = 4 * tid, i = c & 7, j = (c >> 3) & 7, k = c >> 6;
    float* d = xs + qidx(i, j, k);
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
    d[3] = v.w;
#pragma unroll
    for (int u = 0; u < 3; u++) xs[hi[u]] = hv[u];
}

// Level 1's Jacobi sweeps and residual (jacobifine_kernel! / residualfine_kernel! at N = 8,
// with jacobicoarse_kernel! / residualcoarse_kernel! for the coarse part).
template <int OP>
__global__ void __launch_bounds__(T8) k_sp_blk8(Topo t, Comp L, const float* dg1, float* outf, float* outc,
                                                const float* xf, const float* xc, const float* bf, const float* bc,
                                                int gf) {
    __shared__ float xs[QCELLS];
    pdl_wait();
    pdl_trigger();
    constexpr bool ZS = OP == BOP_JAC_ZS;
    if (sp_is_fine(gf)) {
        const int sl = sp_slot(gf);
        int w[3];
        where_of(t, sl, w);
        if (w[0] < 0) return;
        const int tid = (int)threadIdx.x, c = 4 * tid, i0 = c & 7, j = (c >> 3) & 7, k = c >> 6;
        const int64_t n = (int64_t)(sl - 1) * BCELLS1 + c;
        // this piece's own arrays first: they do not depend on the staging
        const float4 dg = *reinterpret_cast<const float4*>(dg1 + n);
        const float4 bb = *reinterpret_cast<const float4*>(bf + n);
        const uchar4 act = *reinterpret_cast<const uchar4*>(L.actf + n);
        float cx[5], cy[4][2], cz[4][2];
#pragma unroll
        for (int u = 0; u <= 4; u++) cx[u] = L.cfx[L8::face(sl, 1, i0 + u, j, k) - 1];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            cy[u][0] = L.cfy[L8::face(sl, 2, i0 + u, j, k) - 1];
            cy[u][1] = L.cfy[L8::face(sl, 2, i0 + u, j + 1, k) - 1];
            cz[u][0] = L.cfz[L8::face(sl, 3, i0 + u, j, k) - 1];
            cz[u][1] = L.cfz[L8::face(sl, 3, i0 + u, j, k + 1) - 1];
        }
        if (!ZS) {
            stage_block8(t, xf, xc, sl, w, xs);
            __syncthreads();
        }
        const float ds[4] = {dg.x, dg.y, dg.z, dg.w}, bs[4] = {bb.x, bb.y, bb.z, bb.w};
        const uint8_t as[4] = {act.x, act.y, act.z, act.w};
        float out[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int o = qidx(i0 + u, j, k);
            const float c6[6] = {cx[u], cx[u + 1], cy[u][0], cy[u][1], cz[u][0], cz[u][1]};
            const int nb[6] = {-1, 1, -Q, Q, -QY, QY};
            float off = 0.0f;
            if (!ZS) {
#pragma unroll
                for (int m = 0; m < 6; m++)
                    if (c6[m] > 0.0f) off += c6[m] * xs[o + nb[m]];
            }
            const float x0 = ZS ? 0.0f : xs[o], diag = ds[u];
            float v = 0.0f;
            if (as[u] != 0) {
                if (OP == BOP_RES) v = bs[u] - (diag * x0 - off);
                else v = diag > 0.0f ? x0 + OMEGA * (bs[u] - (diag * x0 - off)) / diag : 0.0f;
            }
            out[u] = v;
        }
        *reinterpret_cast<float4*>(outf + n) = make_float4(out[0], out[1], out[2], out[3]);
    } else {
        SP_ACTIVE_LOOP(c, L, gf) {
            int I, J, K;
            coarse_cell(t, c, I, J, K);
            float diag, off;
            coarserow<8, ZS>(t, L, xf, xc, I, J, K, diag, off);
            const float x0 = ZS ? 0.0f : xc[c];
            float v;
            if (OP == BOP_RES) v = bc[c] - (diag * x0 - off);
            else v = diag > 0.0f ? x0 + OMEGA * (bc[c] - (diag * x0 - off)) / diag : 0.0f;
            outc[c] = v;
        }
    }
}

}  // namespace sp
}  // namespace mpp
