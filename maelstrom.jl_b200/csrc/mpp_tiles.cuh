// The projection's per-iteration kernels (sm_100a): the V-cycle passes over each level's
// active tiles, the small levels and the coarsest solve in one CTA, and the CG passes.
//
// Work layout. A tile is TH row-split columns (h) x TY rows (j) x TZ planes (k), i.e.
// 2 TH x TY x TZ cells. Tile lists hold packed coordinates (th | tj << 10 | tk << 20). In
// the column kernels a 256-thread block works on TILES_PER_BLOCK tiles at once; each
// thread owns one (h, j) column of its tile and walks its TZ planes (both colours where
// the pass covers both), first loading everything it needs for all planes, then
// computing and storing. Indices are 32-bit.
//
// Arithmetic. Each cell's update is the reference kernel's, in its operation order
// (sums over neighbours in the order +x,-x,+y,-y,+z,-z; restriction terms with a
// innermost; prolongation terms m = 0..7), so the FP32 form rounds as the reference's
// Float32 code does (the library is built with -fmad=false).
#pragma once

#include "mpp_base.cuh"

namespace mpp {

constexpr int COLS = TH * TY;                // threads per tile in the column kernels
constexpr int TILES_PER_BLOCK = TPB / COLS;  // 4
constexpr int BOTTOM_CELLS = 4096;           // levels this small are solved in one CTA (k_bottom)
constexpr int BOTTOM_MAXLEV = 8;

// ---- active-tile lists ----
// One block per level compacts the level's tile flags in tile order (a block-wide scan),
// so the lists, and the reductions over them, are the same on every run.
struct TileTab {
    int nlev;
    int ntiles[16];
    int GH[16], GJ[16];
    uint8_t* flags[16];
    uint32_t* tiles[16];
    int* count[16];
};
__global__ void __launch_bounds__(1024) k_tilelists(TileTab tab) {
    pdl_wait();
    pdl_trigger();
    const int l = blockIdx.x;
    if (l >= tab.nlev) return;
    const int n = tab.ntiles[l], GH = tab.GH[l], GJ = tab.GJ[l];
    const uint8_t* f = tab.flags[l];
    const int chunk = (n + 1023) / 1024;
    const int lo = min(n, (int)threadIdx.x * chunk), hi = min(n, lo + chunk);
    int c = 0;
    for (int t = lo; t < hi; t++) c += f[t] != 0;
    __shared__ int sc[1024];
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int v = threadIdx.x >= (unsigned)o ? sc[threadIdx.x - o] : 0;
        __syncthreads();
        sc[threadIdx.x] += v;
        __syncthreads();
    }
    int w = sc[threadIdx.x] - c;
    for (int t = lo; t < hi; t++)
        if (f[t]) {
            const uint32_t th = (uint32_t)(t % GH), tj = (uint32_t)((t / GH) % GJ), tk = (uint32_t)(t / (GH * GJ));
            tab.tiles[l][w++] = th | (tj << 10) | (tk << 20);
        }
    if (threadIdx.x == 1023) *tab.count[l] = sc[1023];
}

// A thread's column: row-split column h, row j, planes k0 .. k0+kn-1; rb = start of row (j, k0).
struct Col {
    int h, j, k0, kn, rb;
};
template <class M>
__device__ __forceinline__ bool col_of(const Lev<M>& L, uint32_t tile, Col& c) {
    const int lane = threadIdx.x & (COLS - 1);
    c.h = (int)(tile & 1023u) * TH + (lane & (TH - 1));
    c.j = (int)((tile >> 10) & 1023u) * TY + lane / TH;
    c.k0 = (int)(tile >> 20) * TZ;
    c.kn = min(TZ, L.n3 - c.k0);
    c.rb = (c.k0 * L.n2 + c.j) * L.n1;
    return c.h < L.H && c.j < L.n2;
}
// colour-c cell of the column at plane k: i = 2h + ci
__device__ __forceinline__ int ci_of(int c, int j, int k) { return (c + j + k + 1) & 1; }

#define FOR_TILES(L)                                                                                  \
    for (int t_ = blockIdx.x * TILES_PER_BLOCK + (int)(threadIdx.x / COLS), n_ = *(L).count; t_ < n_; \
         t_ += gridDim.x * TILES_PER_BLOCK)

// ---- the V-cycle (src/flip.jl:992-1014) on row-split levels ----

// weightB (src/flip.jl:891): (1, 3, 3, 1) / 8.
template <class C>
__device__ __forceinline__ C wB(int a) {
    return (a == 1 || a == 2) ? (C)0.375f : (C)0.125f;
}

// restrict_kernel! (src/flip.jl:894-906): b_c = 4 sum w_a w_b w_c r_f over the LIQUID fine
// cells of the 4x4x4 block (a fastest); the scaled (16-bit) forms drop the factor 4.
// One block per coarse tile: the tile's fine region (RX x RY x RZ cells) is staged in
// shared memory, non-LIQUID cells as zero, then each thread sums its two coarse cells.
// The region is staged as the fine level stores it: per fine row (j, k) and colour, the
// R_W row-split columns from 2 TH th - 1 on, so a warp's loads are contiguous runs. In
// those terms fine cell (2I-1+a, 2J-1+b, 2K-1+c) of coarse cell (I, J, K) has colour
// (a+b+c) & 1 and column I - 2 TH th + {0,1,1,2}[a].
constexpr int RX = 4 * TH + 2, RY = 2 * TY + 2, RZ = 2 * TZ + 2;
constexpr int R_W = 2 * TH + 2, R_ROWS = 2 * RY * RZ;  // staged columns per row, rows (x2 colours)

// Term t = 16 c + 4 b + a of a coarse cell: weight w_a w_b w_c (exact dyadic constants,
// associated as the reference's (w_a w_b) w_c).
template <class C>
__host__ __device__ constexpr C rw(int t) {
    return (((t & 3) == 1 || (t & 3) == 2) ? (C)0.375f : (C)0.125f) *
           ((((t >> 2) & 3) == 1 || ((t >> 2) & 3) == 2) ? (C)0.375f : (C)0.125f) *
           (((t >> 4) == 1 || (t >> 4) == 2) ? (C)0.375f : (C)0.125f);
}

// 16 bytes of elements of type M.
template <class M>
union Vec16 {
    uint4 u;
    M m[16 / sizeof(M)];
    __device__ Vec16() {}
};

// A tile's coarse cells from its staged region (rows W elements apart, the region's column 0
// at sm): b = the weighted sum, and with `start` the level's x started from it. A thread's
// two cells are the natural columns 2h and 2h + 1 (one of each colour); per fine row (b, c)
// they read three consecutive staged elements of each colour's row (the first cell's
// a = 0, 2 and the second's a = 0, 2 from one; both cells' a = 1, 3 from the other), so
// each staged element is read once a thread, and each cell's 64 terms are summed in the
// reference's order (c outer, a inner), each term as macc rounds it.
// P: where the 8-byte-aligned pairs of S lie: 0 none (element loads), 1 from column 0 (sm
// and W even), 2 from column 1 (sm odd, W even).
template <class Pr, int W, int P, class S>
__device__ __forceinline__ void restrict_cells(const Lev<typename Pr::M>& L, uint32_t tile, const S* sm, int start) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    using S2 = typename std::conditional<sizeof(S) == 4, float2, double2>::type;
    const int lh = slot_h(), lj = slot_j(), lk = slot_k();
    const int th = (int)(tile & 1023u), tj = (int)((tile >> 10) & 1023u), tk = (int)(tile >> 20);
    const int h = th * TH + lh, J = tj * TY + lj, K = tk * TZ + lk;
    if (h >= L.H || J >= L.n2 || K >= L.n3) return;
    const int rb = (K * L.n2 + J) * L.n1;
    C s0 = (C)0, s1 = (C)0;  // the cells at natural columns 2h and 2h + 1
    auto term = [](C& acc, C w, C x) { acc = macc<Pr::scaled>(acc, w, x); };
#pragma unroll
    for (int c = 0; c < 4; c++) {
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const S* ra = sm + (((2 * lk + c) * RY + 2 * lj + b) * 2 + ((b + c) & 1)) * W + 2 * lh;
            const S* rq = sm + (((2 * lk + c) * RY + 2 * lj + b) * 2 + ((b + c + 1) & 1)) * W + 2 * lh;
            C a0, a1, a2, q0, q1, q2;  // ra[0..2], rq[1..3]
            if constexpr (P == 1) {
                const S2 pa = *reinterpret_cast<const S2*>(ra), pq = *reinterpret_cast<const S2*>(rq + 2);
                a0 = (C)pa.x; a1 = (C)pa.y; a2 = ld<C>(ra + 2);
                q0 = ld<C>(rq + 1); q1 = (C)pq.x; q2 = (C)pq.y;
            } else if constexpr (P == 2) {
                const S2 pa = *reinterpret_cast<const S2*>(ra + 1), pq = *reinterpret_cast<const S2*>(rq + 1);
                a0 = ld<C>(ra); a1 = (C)pa.x; a2 = (C)pa.y;
                q0 = (C)pq.x; q1 = (C)pq.y; q2 = ld<C>(rq + 3);
            } else {
                a0 = ld<C>(ra); a1 = ld<C>(ra + 1); a2 = ld<C>(ra + 2);
                q0 = ld<C>(rq + 1); q1 = ld<C>(rq + 2); q2 = ld<C>(rq + 3);
            }
            const int t = 16 * c + 4 * b;
            term(s0, rw<C>(t), a0);
            term(s0, rw<C>(t + 1), q0);
            term(s0, rw<C>(t + 2), a1);
            term(s0, rw<C>(t + 3), q1);
            term(s1, rw<C>(t), a1);
            term(s1, rw<C>(t + 1), q1);
            term(s1, rw<C>(t + 2), a2);
            term(s1, rw<C>(t + 3), q2);
        }
    }
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
        const int p = rb + cc * L.H + h;
        const bool liq = (L.code[p] & SELF) != 0;
        const C sum = ci_of(cc, J, K) ? s1 : s0;
        const C v = liq ? (Pr::scaled ? sum : (C)4 * sum) : (C)0;
        st(L.b + p, v);
        if (start) {
            // start_kernel! on the coarse level, fused: x = b / diag on its colour-0
            // LIQUID cells (b as stored, in the level's element type), 0 elsewhere
            C xv = (C)0;
            if (cc == 0 && liq) {
                M bm;
                st(&bm, v);
                const C bb = ld<C>(&bm), d = ld<C>((Pr::scaled ? L.di : L.dg) + p);
                if constexpr (Pr::scaled) xv = bb * d;
                else xv = d > (C)0 ? bb / d : (C)0;
            }
            st(L.x + p, xv);
        }
    }
}

// The staged region in 16-byte pieces of the fine level's r: per staged row NCH pieces from
// the aligned column below hbase (2 TH th - 1), so element (row, hbase + off) sits at
// row * RWP + CH - 1 + off. A piece lies wholly inside the row [0, H) or wholly outside it.
template <class M>
struct RPieces {
    static constexpr int CH = 16 / (int)sizeof(M), NCH = (R_W + 2 * CH - 2) / CH + 1, RWP = NCH * CH,
                         NV = R_ROWS * NCH, ELEMS = R_ROWS * RWP;
};
// A tile's staging copies (cp.async; pieces outside the level are zero-filled).
template <class M>
__device__ __forceinline__ void restrict_issue(const Lev<M>& F, uint32_t tile, M* stage) {
    using RP = RPieces<M>;
    const int th = (int)(tile & 1023u), tj = (int)((tile >> 10) & 1023u), tk = (int)(tile >> 20);
    const int h8 = 2 * TH * th - RP::CH, j0 = 2 * TY * tj - 1, k0 = 2 * TZ * tk - 1;
#pragma unroll 2
    for (int e0 = 0; e0 < RP::NV; e0 += TPB) {
        const int e = e0 + (int)threadIdx.x;
        if (e < RP::NV) {
            const int r = e / RP::NCH, ch = e - r * RP::NCH;
            const int col = r & 1, jk = r >> 1, j = j0 + jk % RY, k = k0 + jk / RY, h = h8 + ch * RP::CH;
            const bool in = j >= 0 && j < F.n2 && k >= 0 && k < F.n3 && h >= 0 && h < F.H;
            cp_async16_zfill(stage + r * RP::RWP + ch * RP::CH, in ? F.r + (k * F.n2 + j) * F.n1 + col * F.H + h : F.r,
                             in ? 16u : 0u);
        }
    }
}

// Shared memory of k_restrict in bytes: the 4-byte form's two stages of pieces; the 16-bit
// forms' one stage and its copy widened to the arithmetic type; the region in the
// arithmetic type (the 8-byte form, and levels whose rows are not whole pieces).
__host__ __device__ constexpr int restrict_smem_bytes(int msize, int csize) {
    const int region = R_ROWS * R_W * csize;
    if (msize == 8) return region;
    const int stage = R_ROWS * ((R_W + 2 * (16 / msize) - 2) / (16 / msize) + 1) * 16;  // bytes of pieces
    const int piped = msize == csize ? 2 * stage : stage + stage / msize * csize;
    return piped > region ? piped : region;
}

template <class Pr>
__device__ __forceinline__ void restrict_body(Lev<typename Pr::M> F, Lev<typename Pr::M> L, int start) {
    using C = typename Pr::C;
    extern __shared__ __align__(128) unsigned char smraw[];
    C* sm = reinterpret_cast<C*>(smraw);
    using M = typename Pr::M;
    const int n = *L.count;
    const bool vec = F.H % (16 / (int)sizeof(M)) == 0 && F.n1 % (16 / (int)sizeof(M)) == 0 &&
                     (reinterpret_cast<uintptr_t>(F.r) & 15) == 0;
    if constexpr (sizeof(M) <= 4) {
        if (vec) {
            // Pipelined: a block's copies of its next tile's region go out before it sums
            // this one, so the loads stay in flight while it computes.
            using RP = RPieces<M>;
            M* raw = reinterpret_cast<M*>(smraw);
            int t = blockIdx.x;
            if (t < n) restrict_issue(F, L.tiles[t], raw);
            cp_async_commit();
            if constexpr (std::is_same<M, C>::value) {
                // two stages, summed where they land
                for (int i = 0; t < n; t += gridDim.x, i++) {
                    const uint32_t tile = L.tiles[t];
                    if (t + (int)gridDim.x < n) restrict_issue(F, L.tiles[t + gridDim.x], raw + ((i + 1) & 1) * RP::ELEMS);
                    cp_async_commit();
                    cp_async_wait<1>();
                    __syncthreads();
                    restrict_cells<Pr, RP::RWP, 2>(L, tile, raw + (i & 1) * RP::ELEMS + (RP::CH - 1), start);
                    __syncthreads();  // this stage free for the copies after next
                }
            } else {
                // one stage, widened into a copy of the same layout (the sums read each
                // element eight times), after which the next tile's copies reuse the stage
                C* cv = reinterpret_cast<C*>(smraw + RP::ELEMS * sizeof(M));
                for (; t < n; t += gridDim.x) {
                    const uint32_t tile = L.tiles[t];
                    cp_async_wait<0>();
                    __syncthreads();
#pragma unroll 2
                    for (int e0 = 0; e0 < RP::NV; e0 += TPB) {
                        const int e = e0 + (int)threadIdx.x;
                        if (e < RP::NV) {
                            Vec16<M> w;
                            w.u = *reinterpret_cast<const uint4*>(raw + e * RP::CH);
                            C v[RP::CH];
#pragma unroll
                            for (int q = 0; q < RP::CH; q++) v[q] = ld<C>(&w.m[q]);
#pragma unroll
                            for (int q = 0; q < RP::CH; q += 4)
                                *reinterpret_cast<float4*>(cv + e * RP::CH + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
                        }
                    }
                    __syncthreads();
                    if (t + (int)gridDim.x < n) restrict_issue(F, L.tiles[t + gridDim.x], raw);
                    cp_async_commit();
                    restrict_cells<Pr, RP::RWP, 2>(L, tile, cv + (RP::CH - 1), start);
                }
            }
            cp_async_wait<0>();
            return;
        }
    }
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const uint32_t tile = L.tiles[t];
        const int th = (int)(tile & 1023u), tj = (int)((tile >> 10) & 1023u), tk = (int)(tile >> 20);
        const int hbase = 2 * TH * th - 1, j0 = 2 * TY * tj - 1, k0 = 2 * TZ * tk - 1;
        __syncthreads();
        // Every non-LIQUID cell's r is zero (the residual pass writes zeros in active tiles
        // and the set-up clears the array each projection), so r is staged unmasked: all of
        // a thread's loads go out at once, then land in shared memory. (The 2- and 4-byte
        // forms come here only for rows that are not whole pieces.)
        if (sizeof(M) == 8 && vec) {
            // 16-byte pieces: each staged row's columns from the aligned column below hbase,
            // a piece wholly inside the row [0, H) or wholly outside it (read as zeros)
            constexpr int CH = 16 / (int)sizeof(M), NCH = (R_W + 2 * CH - 2) / CH + 1;
            constexpr int NV = R_ROWS * NCH, PERV = (NV + TPB - 1) / TPB;
            const int h8 = hbase + 1 - CH;  // hbase + 1 = 2 TH th is a multiple of CH
            constexpr int VB = 3;  // pieces a thread has in flight
#pragma unroll 1
            for (int u0 = 0; u0 < PERV; u0 += VB) {
                Vec16<M> v[VB];
                int rr[VB], hh[VB];
#pragma unroll
                for (int u = 0; u < VB; u++) {
                    const int e = (int)threadIdx.x + (u0 + u) * TPB;
                    const int r = e / NCH, ch = e - r * NCH;
                    const int col = r & 1, jk = r >> 1, j = j0 + jk % RY, k = k0 + jk / RY, h = h8 + ch * CH;
                    rr[u] = e < NV ? r : -1;
                    hh[u] = h;
                    v[u].u = make_uint4(0u, 0u, 0u, 0u);
                    if (e < NV && j >= 0 && j < F.n2 && k >= 0 && k < F.n3 && h >= 0 && h < F.H)
                        v[u].u = *reinterpret_cast<const uint4*>(F.r + (k * F.n2 + j) * F.n1 + col * F.H + h);
                }
#pragma unroll
                for (int u = 0; u < VB; u++) {
                    if (rr[u] < 0) continue;
#pragma unroll
                    for (int q = 0; q < CH; q++) {
                        const int off = hh[u] + q - hbase;
                        if (off >= 0 && off < R_W) sm[rr[u] * R_W + off] = ld<C>(&v[u].m[q]);
                    }
                }
            }
            __syncthreads();
        } else {
        // in batches of RB loads a thread, so few registers hold them and more blocks fit
        constexpr int NE = R_ROWS * R_W, PER = (NE + TPB - 1) / TPB, RB = 8;
#pragma unroll
        for (int u0 = 0; u0 < PER; u0 += RB) {
            C vals[RB];
#pragma unroll
            for (int q = 0; q < RB; q++) {
                const int e = (int)threadIdx.x + (u0 + q) * TPB;
                const int r = e / R_W, off = e - r * R_W;  // staged row (jk, colour), column
                const int col = r & 1, jk = r >> 1, j = j0 + jk % RY, k = k0 + jk / RY, h = hbase + off;
                vals[q] = (C)0;
                if (u0 + q < PER && e < NE && j >= 0 && j < F.n2 && k >= 0 && k < F.n3 && h >= 0 && h < F.H)
                    vals[q] = ld<C>(F.r + (k * F.n2 + j) * F.n1 + col * F.H + h);
            }
#pragma unroll
            for (int q = 0; q < RB; q++) {
                const int e = (int)threadIdx.x + (u0 + q) * TPB;
                if (u0 + q < PER && e < NE) sm[e] = vals[q];
            }
        }
        __syncthreads();
        }
        restrict_cells<Pr, R_W, 1>(L, tile, sm, start);
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 3) k_restrict(Lev<typename Pr::M> F, Lev<typename Pr::M> L, int start) {
    pdl_wait();
    pdl_trigger();
    restrict_body<Pr>(F, L, start);
}

// prolongweights (src/flip.jl:908-911), 0-based.
template <class C>
__device__ __forceinline__ void pweights(int i, int& c0, C& w0, int& c1, C& w1) {
    const int I = i >> 1;
    if ((i & 1) == 0) { c0 = I - 1; w0 = (C)0.25f; c1 = I; w1 = (C)0.75f; }
    else { c0 = I; w0 = (C)0.75f; c1 = I + 1; w1 = (C)0.25f; }
}

// prolong_kernel! (src/flip.jl:914-929): x_f += sum over the LIQUID coarse cells of the
// trilinear weights times x_c (m = 0..7; x4 in the scaled forms). Each tile's PX x PY x PZ
// coarse cells are staged in shared memory, non-LIQUID as zero. The coarse level is
// row-split, or the bottom level in natural order (`cnat`).
constexpr int PX = TH + 2, PY = TY / 2 + 2, PZ = TZ / 2 + 2;

template <class Pr>
__device__ __forceinline__ void prolong_body(Lev<typename Pr::M> L, Lev<typename Pr::M> Cl, int cnat) {
    using C = typename Pr::C;
    __shared__ C sm[TILES_PER_BLOCK][PZ][PY][PX];
    const int n = *L.count;
    const int sub = threadIdx.x / COLS;
    const int sz = L.n1 * L.n2;
    for (int t0 = blockIdx.x * TILES_PER_BLOCK; t0 < n; t0 += gridDim.x * TILES_PER_BLOCK) {
        __syncthreads();
        // Every non-LIQUID coarse cell's x is zero (start writes zeros over active tiles, the
        // set-up clears the arrays each projection, the bottom solve writes every cell), so
        // x is staged unmasked, all of a thread's loads at once.
        constexpr int NE = TILES_PER_BLOCK * PX * PY * PZ, PER = (NE + TPB - 1) / TPB;
        C vals[PER];
#pragma unroll
        for (int u = 0; u < PER; u++) {
            const int e = (int)threadIdx.x + u * TPB;
            const int s = e / (PX * PY * PZ), r = e % (PX * PY * PZ);
            const int ii = r % PX, jj = (r / PX) % PY, kk = r / (PX * PY);
            vals[u] = (C)0;
            if (e < NE && t0 + s < n) {
                const uint32_t tile = L.tiles[t0 + s];
                const int I = (int)(tile & 1023u) * TH - 1 + ii;
                const int J = (int)((tile >> 10) & 1023u) * (TY / 2) - 1 + jj;
                const int K = (int)(tile >> 20) * (TZ / 2) - 1 + kk;
                if (I >= 0 && I < Cl.n1 && J >= 0 && J < Cl.n2 && K >= 0 && K < Cl.n3)
                    vals[u] = ld<C>(Cl.x + (cnat ? (int)Cl.nat(I, J, K) : (int)Cl.pos(I, J, K)));
            }
        }
#pragma unroll
        for (int u = 0; u < PER; u++) {
            const int e = (int)threadIdx.x + u * TPB;
            if (e < NE) (&sm[0][0][0][0])[e] = vals[u];
        }
        __syncthreads();
        const int t = t0 + sub;
        if (t >= n) continue;
        Col c;
        if (!col_of(L, L.tiles[t], c)) continue;
        const int Ib = (int)(L.tiles[t] & 1023u) * TH - 1;  // coarse origin of the staged region
        const int Jb = c.j - (c.j & (TY - 1));
        int b0, b1;
        C wb0, wb1;
        pweights<C>(c.j, b0, wb0, b1, wb1);
        b0 = b0 - (Jb / 2 - 1);
        b1 = b1 - (Jb / 2 - 1);
        C v[2][TZ];
        bool live[2][TZ];
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            const int k = c.k0 + q;
            int k0, k1;
            C wc0, wc1;
            pweights<C>(k, k0, wc0, k1, wc1);
            k0 -= c.k0 / 2 - 1;
            k1 -= c.k0 / 2 - 1;
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                live[cc][q] = false;
                v[cc][q] = (C)0;
                if (q < c.kn) {
                    const int p = c.rb + q * sz + cc * L.H + c.h;
                    if (L.code[p] & SELF) {
                        live[cc][q] = true;
                        const int i = 2 * c.h + ci_of(cc, c.j, k);
                        int a0, a1;
                        C wa0, wa1;
                        pweights<C>(i, a0, wa0, a1, wa1);
                        a0 -= Ib;
                        a1 -= Ib;
                        C s = (C)0;
#pragma unroll
                        for (int m = 0; m < 8; m++) {
                            const int A = (m & 1) ? a1 : a0, B = (m & 2) ? b1 : b0, Kc = (m & 4) ? k1 : k0;
                            const C wa = (m & 1) ? wa1 : wa0, wb = (m & 2) ? wb1 : wb0, wc = (m & 4) ? wc1 : wc0;
                            s = macc<Pr::scaled>(s, wa * wb * wc, sm[sub][Kc][B][A]);
                        }
                        v[cc][q] = ld<C>(L.x + p) + (Pr::scaled ? (C)4 * s : s);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < TZ; q++)
#pragma unroll
            for (int cc = 0; cc < 2; cc++)
                if (live[cc][q]) st(L.x + c.rb + q * sz + cc * L.H + c.h, v[cc][q]);
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_prolong(Lev<typename Pr::M> L, Lev<typename Pr::M> Cl, int cnat) {
    pdl_wait();
    pdl_trigger();
    prolong_body<Pr>(L, Cl, cnat);
}

// ---- the small levels and the coarsest, in one CTA ----
// Levels lb .. L-1 (each at most a few thousand cells) live in shared memory in natural
// order for the whole of their part of the V-cycle: the restriction into lb from the
// level above (restrict_kernel!), then for each level start, the down sweeps, residual
// and restriction, the coarsest solve (coarse_kernel!, src/flip.jl:935-962: `sweeps`
// red-black sweeps from zero and as many in reverse colour order, the accumulator
// starting at b, the diagonal the count of non-SOLID neighbours), and back up:
// prolongation and the up sweeps. Level lb's correction is written to global memory.
struct BotLev {
    int n1, n2, n3;
    const uint8_t* code;  // stencil codes, natural order, global (k_level)
    const uint8_t* dc;    // non-SOLID neighbour counts, natural order, global (k_level)
    int ox, ob, orr, ocode, odc;  // shared-memory offsets (bytes)
    int olist;            // the level's LIQUID cells by colour (uint16 indices), levels above the coarsest
};
struct BotArgs {
    int nl;  // levels in shared memory, the last one the coarsest
    int sweeps, coarse;
    BotLev lv[BOTTOM_MAXLEV];
};

template <class Pr>
__device__ __forceinline__ void bottom_dev(const typename Pr::C* __restrict__ bin, typename Pr::M* __restrict__ xout,
                                           const BotArgs& a) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    using CC = typename Pr::CC;
    extern __shared__ __align__(128) unsigned char smraw[];
    const int T = blockDim.x, tid = threadIdx.x;
    // codes and non-SOLID neighbour counts of every level, and level lb's right-hand side
    // (restricted from the level above by k_restrict_bottom)
    // per level above the coarsest: its LIQUID cells listed by colour (the red-black passes
    // walk a colour's list; the order within a list does not matter, a colour's cells being
    // independent of each other)
    __shared__ int lcount[BOTTOM_MAXLEV][2];
    if (tid < 2 * BOTTOM_MAXLEV) lcount[tid >> 1][tid & 1] = 0;
    __syncthreads();
    for (int l = 0; l < a.nl; l++) {
        const BotLev& B = a.lv[l];
        const int N = B.n1 * B.n2 * B.n3;
        uint8_t* code = smraw + B.ocode;
        uint8_t* dc = smraw + B.odc;
        for (int c = tid; c < N; c += T) {
            const uint8_t cd = B.code[c];
            code[c] = cd;
            dc[c] = B.dc[c];
            if (l + 1 < a.nl && (cd & SELF)) {
                const int i = c % B.n1, j = (c / B.n1) % B.n2, k = c / (B.n1 * B.n2);
                const int col = (i + j + k + 1) & 1;
                reinterpret_cast<uint16_t*>(smraw + B.olist)[col * N + atomicAdd(&lcount[l][col], 1)] = (uint16_t)c;
            }
        }
    }
    {
        const BotLev& B = a.lv[0];
        const int N = B.n1 * B.n2 * B.n3;
        if (a.nl == 1) {
            CC* b = reinterpret_cast<CC*>(smraw + B.ob);
            for (int c = tid; c < N; c += T) b[c] = (CC)bin[c];
        } else {
            C* b = reinterpret_cast<C*>(smraw + B.ob);
            for (int c = tid; c < N; c += T) b[c] = bin[c];
        }
    }
    __syncthreads();
    // restriction between shared-memory levels
    auto restrict_into = [&](int l, auto* bout, auto getf) {
        const BotLev& B = a.lv[l];
        const int N = B.n1 * B.n2 * B.n3;
        const uint8_t* code = smraw + B.ocode;
        using T2 = typename std::remove_pointer<decltype(bout)>::type;
        for (int c = tid; c < N; c += T) {
            T2 v = (T2)0;
            if (code[c] & SELF) {
                const int I = c % B.n1, J = (c / B.n1) % B.n2, K = c / (B.n1 * B.n2);
                C s = (C)0;
                for (int c3 = 0; c3 < 4; c3++)
                    for (int b3 = 0; b3 < 4; b3++)
#pragma unroll
                        for (int a3 = 0; a3 < 4; a3++)
                            s = macc<Pr::scaled>(s, wB<C>(a3) * wB<C>(b3) * wB<C>(c3),
                                                 getf(2 * I + a3 - 1, 2 * J + b3 - 1, 2 * K + c3 - 1));
                v = (T2)(Pr::scaled ? s : (C)4 * s);
            }
            bout[c] = v;
        }
    };
    // smoothing passes on a shared-memory level
    auto sweep = [&](int l, int colour) {
        const BotLev& B = a.lv[l];
        const int N = B.n1 * B.n2 * B.n3, sy = B.n1, sz = B.n1 * B.n2;
        const uint8_t* code = smraw + B.ocode;
        const uint8_t* dc = smraw + B.odc;
        C* x = reinterpret_cast<C*>(smraw + B.ox);
        const C* b = reinterpret_cast<const C*>(smraw + B.ob);
        const uint16_t* lst = reinterpret_cast<const uint16_t*>(smraw + B.olist) + colour * N;
        const int nl = lcount[l][colour];
        for (int e = tid; e < nl; e += T) {
            const int c = lst[e];
            const uint8_t cd = code[c];
            C s = (C)0;
            if (cd & 1) s += x[c + 1];
            if (cd & 2) s += x[c - 1];
            if (cd & 4) s += x[c + sy];
            if (cd & 8) s += x[c - sy];
            if (cd & 16) s += x[c + sz];
            if (cd & 32) s += x[c - sz];
            const C d = (C)dc[c];
            x[c] = d > (C)0 ? (b[c] + s) / d : (C)0;
        }
        __syncthreads();
    };
    const int sw = a.sweeps;
    for (int l = 0; l + 1 < a.nl; l++) {
        const BotLev& B = a.lv[l];
        const int N = B.n1 * B.n2 * B.n3, sy = B.n1, sz = B.n1 * B.n2;
        const uint8_t* code = smraw + B.ocode;
        const uint8_t* dc = smraw + B.odc;
        C* x = reinterpret_cast<C*>(smraw + B.ox);
        C* b = reinterpret_cast<C*>(smraw + B.ob);
        C* r = reinterpret_cast<C*>(smraw + B.orr);
        // start_kernel!: x = b / diag on colour 0's LIQUID cells, zero elsewhere
        for (int c = tid; c < N; c += T) x[c] = (C)0;
        __syncthreads();
        {
            const uint16_t* lst = reinterpret_cast<const uint16_t*>(smraw + B.olist);
            const int nl = lcount[l][0];
            for (int e = tid; e < nl; e += T) {
                const int c = lst[e];
                const C d = (C)dc[c];
                if (d > (C)0) x[c] = b[c] / d;
            }
        }
        __syncthreads();
        for (int q = 1; q < 2 * sw; q++) sweep(l, q & 1);  // down: colours 1, 0, 1, ...
        // residual_kernel! on the LIQUID cells (the restriction reads r nowhere else)
        for (int e = tid; e < lcount[l][0] + lcount[l][1]; e += T) {
            const int col = e < lcount[l][0] ? 0 : 1;
            const int c = reinterpret_cast<const uint16_t*>(smraw + B.olist)[col * N + (col ? e - lcount[l][0] : e)];
            const uint8_t cd = code[c];
            C v = (C)0;
            {
                C s = (C)0;
                if (cd & 1) s += x[c + 1];
                if (cd & 2) s += x[c - 1];
                if (cd & 4) s += x[c + sy];
                if (cd & 8) s += x[c - sy];
                if (cd & 16) s += x[c + sz];
                if (cd & 32) s += x[c - sz];
                v = b[c] - ((C)dc[c] * x[c] - s);
            }
            r[c] = v;
        }
        __syncthreads();
        const uint8_t* fcode = code;
        auto getL = [&](int i, int j, int k) -> C {
            if (i < 0 || i >= B.n1 || j < 0 || j >= B.n2 || k < 0 || k >= B.n3) return (C)0;
            const int p = i + B.n1 * (j + B.n2 * k);
            return (fcode[p] & SELF) ? r[p] : (C)0;
        };
        if (l + 2 == a.nl) restrict_into(l + 1, reinterpret_cast<CC*>(smraw + a.lv[l + 1].ob), getL);
        else restrict_into(l + 1, reinterpret_cast<C*>(smraw + a.lv[l + 1].ob), getL);
        __syncthreads();
    }
    {  // coarse_kernel!
        const BotLev& B = a.lv[a.nl - 1];
        const int N = B.n1 * B.n2 * B.n3, sy = B.n1, sz = B.n1 * B.n2;
        const uint8_t* code = smraw + B.ocode;
        const uint8_t* dc = smraw + B.odc;
        CC* x = reinterpret_cast<CC*>(smraw + B.ox);
        const CC* b = reinterpret_cast<const CC*>(smraw + B.ob);
        for (int c = tid; c < N; c += T) x[c] = (CC)0;
        __syncthreads();
        // With n1 even a thread owns cells 2t and 2t+1 of one row, one of each colour, and each
        // half-sweep updates the one of that colour (selected without branching); with n1 odd,
        // one cell per thread. Only the threads that own cells meet at each barrier.
        const int per = (B.n1 % 2 == 0) ? 2 : 1;
        const int nthreads = (((N + per - 1) / per + 31) / 32) * 32;
        if (tid < nthreads) {
            uint8_t cd[2] = {0, 0};
            int cell[2] = {0, 0};
            CC bi[2] = {(CC)0, (CC)0}, d[2] = {(CC)0, (CC)0}, rd[2] = {(CC)0, (CC)0};
            int col0 = 0;
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int c = per * tid + u;
                cell[u] = c;
                if (u < per && c < N) {
                    cd[u] = code[c];
                    const int i = c % B.n1, j = (c / B.n1) % B.n2, k = c / sz;
                    if (u == 0) col0 = (i + j + k + 1) & 1;
                    bi[u] = b[c];
                    d[u] = (CC)dc[c];
                    rd[u] = d[u] > (CC)0 ? (CC)1 / d[u] : (CC)0;
                }
            }
            for (int s = 1; s <= 2 * a.coarse; s++)
                for (int half = 0; half <= 1; half++) {
                    const int colour = s <= a.coarse ? half : 1 - half;
                    // this thread's cell of `colour` (per == 1: its only cell, if that colour)
                    const bool second = per == 2 && col0 != colour;
                    const uint8_t cdv = (per == 1 && col0 != colour) ? (uint8_t)0 : (second ? cd[1] : cd[0]);
                    if (cdv & SELF) {
                        const int c = second ? cell[1] : cell[0];
                        CC acc = second ? bi[1] : bi[0];
                        if (cdv & 1) acc += x[c + 1];
                        if (cdv & 2) acc += x[c - 1];
                        if (cdv & 4) acc += x[c + sy];
                        if (cdv & 8) acc += x[c - sy];
                        if (cdv & 16) acc += x[c + sz];
                        if (cdv & 32) acc += x[c - sz];
                        if constexpr (std::is_same<CC, float>::value) {
                            const CC dd = second ? d[1] : d[0];
                            x[c] = dd > (CC)0 ? acc / dd : (CC)0;
                        } else {
                            x[c] = acc * (second ? rd[1] : rd[0]);  // FP64 coarsest of the 16-bit forms
                        }
                    }
                    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
                }
        }
        __syncthreads();
    }
    // back up: prolongation and the up sweeps
    for (int l = a.nl - 2; l >= 0; l--) {
        const BotLev& B = a.lv[l];
        const BotLev& Bc = a.lv[l + 1];
        const int N = B.n1 * B.n2 * B.n3;
        const uint8_t* code = smraw + B.ocode;
        const uint8_t* ccode = smraw + Bc.ocode;
        C* x = reinterpret_cast<C*>(smraw + B.ox);
        const bool coarsest = l + 2 == a.nl;
        (void)code;
        for (int e = tid; e < lcount[l][0] + lcount[l][1]; e += T) {  // the LIQUID cells
            const int col = e < lcount[l][0] ? 0 : 1;
            const int c = reinterpret_cast<const uint16_t*>(smraw + B.olist)[col * N + (col ? e - lcount[l][0] : e)];
            const int i = c % B.n1, j = (c / B.n1) % B.n2, k = c / (B.n1 * B.n2);
            int a0, a1, b0, b1, k0, k1;
            C wa0, wa1, wb0, wb1, wc0, wc1;
            pweights<C>(i, a0, wa0, a1, wa1);
            pweights<C>(j, b0, wb0, b1, wb1);
            pweights<C>(k, k0, wc0, k1, wc1);
            C s = (C)0;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int A = (m & 1) ? a1 : a0, Bj = (m & 2) ? b1 : b0, K = (m & 4) ? k1 : k0;
                const C wa = (m & 1) ? wa1 : wa0, wb = (m & 2) ? wb1 : wb0, wc = (m & 4) ? wc1 : wc0;
                if (A < 0 || A >= Bc.n1 || Bj < 0 || Bj >= Bc.n2 || K < 0 || K >= Bc.n3) continue;
                const int q = A + Bc.n1 * (Bj + Bc.n2 * K);
                if (!(ccode[q] & SELF)) continue;
                const C xc = coarsest ? (C)reinterpret_cast<const CC*>(smraw + Bc.ox)[q]
                                      : reinterpret_cast<const C*>(smraw + Bc.ox)[q];
                s = macc<Pr::scaled>(s, wa * wb * wc, xc);
            }
            x[c] = x[c] + (Pr::scaled ? (C)4 * s : s);
        }
        __syncthreads();
        for (int q = 0; q < 2 * sw; q++) sweep(l, (q & 1) ? 0 : 1);  // up: colours 1, 0, 1, 0, ...
    }
    // level lb's correction out, natural order
    {
        const BotLev& B = a.lv[0];
        const int N = B.n1 * B.n2 * B.n3;
        if (a.nl == 1) {
            const CC* x = reinterpret_cast<const CC*>(smraw + B.ox);
            for (int c = tid; c < N; c += T) st(xout + c, x[c]);
        } else {
            const C* x = reinterpret_cast<const C*>(smraw + B.ox);
            for (int c = tid; c < N; c += T) st(xout + c, x[c]);
        }
    }
}
template <class Pr>
__global__ void __launch_bounds__(1024) k_bottom(const typename Pr::C* __restrict__ bin, typename Pr::M* __restrict__ xout,
                                                 const __grid_constant__ BotArgs a) {
    bottom_dev<Pr>(bin, xout, a);
}

}  // namespace mpp
