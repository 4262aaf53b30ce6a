// The per-iteration kernels that stream a level's active tiles (sm_100a): start, one
// colour of red-black Gauss-Seidel and the residual of the V-cycle, and the CG passes
// (z.r, q = A p, the step, the true residual, A x).
//
// Load pattern. Every load a cell needs is issued at once, whatever its stencil code
// says: the code is only read afterwards, to choose which loaded neighbours enter the
// sums (in the reference's order, skipping the others, so the FP32 form still rounds as
// the reference does). A thread therefore waits for one round trip per plane instead of
// a chain of them (code, then data), and the next tile's id is fetched one step ahead.
// Neighbour reads of level x arrays and the CG direction d may run past the array ends
// at the box faces: those arrays are allocated with a zeroed guard of one plane plus a
// margin on each side. The user's P is read with clamped indices.
#pragma once

#include "mpp_tiles.cuh"

namespace mpp {

// Guard elements on each side of the arrays read at neighbour offsets.
__host__ __device__ constexpr int guard_of(int n1, int n2) { return (n1 * n2 + 64 + 63) / 64 * 64; }

__device__ __forceinline__ int clampi(int p, int N) { return p < 0 ? 0 : (p >= N ? N - 1 : p); }

// Walk this block's share of a level's tile list, the next tile id fetched one step ahead.
#define FOR_TILES_PF(L, tile)                                                                  \
    const int n_ = *(L).count, s_ = gridDim.x * TILES_PER_BLOCK;                                \
    int t_ = blockIdx.x * TILES_PER_BLOCK + (int)(threadIdx.x / COLS);                          \
    uint32_t tile = t_ < n_ ? (L).tiles[t_] : 0u;                                               \
    for (uint32_t next_; t_ < n_; t_ += s_, tile = next_)                                       \
        if ((next_ = (t_ + s_ < n_ ? (L).tiles[t_ + s_] : 0u)), true)

// The six neighbours of a row-split cell in the order +x,-x,+y,-y,+z,-z: positions in the
// other colour's half, o being the cell's own column there.
template <class C, class T>
__device__ __forceinline__ void load6(C (&v)[6], const T* x, int o, int ci, int sy, int sz) {
    v[0] = ld<C>(x + o + ci);
    v[1] = ld<C>(x + o + ci - 1);
    v[2] = ld<C>(x + o + sy);
    v[3] = ld<C>(x + o - sy);
    v[4] = ld<C>(x + o + sz);
    v[5] = ld<C>(x + o - sz);
}
// liquidsum (src/flip.jl:852-857): s = 0, then the LIQUID neighbours in order.
template <class C>
__device__ __forceinline__ C sum6(const C (&v)[6], uint8_t cd) {
    C s = (C)0;
#pragma unroll
    for (int m = 0; m < 6; m++)
        if (cd & (1u << m)) s += v[m];
    return s;
}

// liquidsum (src/flip.jl:849-857) for a cell whose six neighbour values are loaded. Every
// non-LIQUID cell of these arrays holds exactly 0 (start, smoother, prolongation and the
// CG step write only LIQUID cells; the rest is cleared), so adding all six in the same
// order rounds exactly as adding the LIQUID ones. The one exception is a read past the
// row or plane at the level's x/y faces, which lands in a neighbouring row: when a LIQUID
// cell lies there (`edge`), the code's mask is applied.
template <class C>
__device__ __forceinline__ C nsum6(const C (&v)[6], uint8_t cd, bool edge) {
    if (edge) return sum6<C>(v, cd);
    return ((((v[0] + v[1]) + v[2]) + v[3]) + v[4]) + v[5];
}

// ---- the scalar steps of pressure!, run by the last block of each reduction ----
// After z.r (src/flip.jl:1095-1096, 1105-1107): rho_new and beta = rho_new / rho (0 on the
// first pass); the flexible form takes the Polak-Ribiere beta (src/sflip.jl:1896-1897).
template <class Pr>
__device__ __forceinline__ void dot_finish(Scalars* sc, const double (&acc)[2]) {
    State& S = sc->s;
    const double rho_new = rs<Pr>(acc[0]);
    if (!finite_d(rho_new)) {
        S.status = ST_NONFINITE;
        S.done = 1;
        return;
    }
    if constexpr (Pr::flexible) {
        if (!(rho_new > 0.0)) {  // src/sflip.jl:1880,1896
            S.status = ST_INDEFINITE;
            S.done = 1;
            return;
        }
        const double beta = S.it == 0 ? 0.0 : -S.alpha * acc[1] / S.rho;
        S.beta = beta > 0.0 ? beta : 0.0;
    } else {
        S.beta = S.it == 0 ? 0.0 : dv<Pr>(rho_new, S.rho);
    }
    S.rho = rho_new;
}
// After p.q: alpha = rho / p.q (src/flip.jl:1100), or a nonfinite/indefinite status.
template <class Pr>
__device__ __forceinline__ void search_finish(Scalars* sc, const double (&acc)[1]) {
    State& S = sc->s;
    S.pq = rs<Pr>(acc[0]);
    if (!finite_d(S.pq)) {
        S.status = ST_NONFINITE;
        S.done = 1;
    } else if (!(S.pq > 0.0)) {  // src/sflip.jl:1876-1877
        S.status = ST_INDEFINITE;
        S.done = 1;
    } else {
        S.alpha = dv<Pr>(S.rho, S.pq);
    }
}
// After r.r: rnorm and the exit test rnorm <= tol |b| (src/flip.jl:1102-1103), or maxiter;
// sets the graph's loop condition.
template <class Pr>
__device__ __forceinline__ void advance_finish(Scalars* sc, const double (&acc)[1], cudaGraphConditionalHandle cond,
                                               int use_cond) {
    State& S = sc->s;
    S.it += 1;
    S.rnorm = sq<Pr>(acc[0]);
    S.rscale = next_rscale(S.rnorm, S.nliq);
    if (!finite_d(S.rnorm)) {
        S.status = ST_NONFINITE;
        S.done = 1;
    } else if (S.rnorm <= S.target) {
        S.status = ST_OK;
        S.done = 1;
    } else if (S.it >= sc->p.maxiter) {
        S.status = ST_NOT_CONVERGED;
        S.done = 1;
    }
    set_cond(cond, use_cond, !S.done);
}

// ---- the V-cycle (src/flip.jl:992-1014) on row-split levels ----

// start_kernel! (src/flip.jl:965-973): colour-0 LIQUID cells get b/diag, every other cell 0.
template <class Pr>
__device__ __forceinline__ void start_body(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    const int sz = L.n1 * L.n2;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
        uint8_t cd[TZ];
        C dv[TZ], bv[TZ];
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            cd[q] = 0;
            if (q < c.kn) {
                const int p = c.rb + q * sz + c.h;
                cd[q] = L.code[p];
                dv[q] = ld<C>((Pr::scaled ? L.di : L.dg) + p);
                bv[q] = ld<C>(L.b + p);
            }
        }
#pragma unroll
        for (int q = 0; q < TZ; q++)
            if (q < c.kn) {
                const int p = c.rb + q * sz + c.h;
                C v = (C)0;
                // the 16-bit forms multiply by the stored reciprocal (0 where the diagonal is)
                if constexpr (Pr::scaled) {
                    if (cd[q] & SELF) v = bv[q] * dv[q];
                } else {
                    if ((cd[q] & SELF) && dv[q] > (C)0) v = bv[q] / dv[q];
                }
                st(L.x + p, v);
                st(L.x + p + L.H, (C)0);
            }
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_start(Lev<typename Pr::M> L) {
    pdl_wait();
    pdl_trigger();
    start_body<Pr>(L);
}

// rbgs_kernel! (src/flip.jl:870-877): one colour of red-black Gauss-Seidel,
// x = (b + sum_LIQ x_n) / diag on LIQUID cells of that colour.
template <class Pr>
__device__ __forceinline__ void rbgs_body(Lev<typename Pr::M> L, int colour) {
    using C = typename Pr::C;
    const int sy = L.n1, sz = L.n1 * L.n2;
    const int own = colour * L.H, oth = (1 - colour) * L.H;
    const bool edge = *L.edge != 0;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
        uint8_t cd[TZ];
        C nb[TZ][6], dv[TZ], bv[TZ];
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            cd[q] = 0;
            if (q < c.kn) {
                const int rb = c.rb + q * sz;
                cd[q] = L.code[rb + own + c.h];
                dv[q] = ld<C>((Pr::scaled ? L.di : L.dg) + rb + own + c.h);
                bv[q] = ld<C>(L.b + rb + own + c.h);
                load6<C>(nb[q], L.x, rb + oth + c.h, ci_of(colour, c.j, c.k0 + q), sy, sz);
            }
        }
#pragma unroll
        for (int q = 0; q < TZ; q++)
            if (cd[q] & SELF) {
                const C s = nsum6<C>(nb[q], cd[q], edge);
                C v;
                if constexpr (Pr::scaled) v = (bv[q] + s) * dv[q];
                else v = dv[q] > (C)0 ? (bv[q] + s) / dv[q] : (C)0;
                st(L.x + c.rb + q * sz + own + c.h, v);
            }
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs(Lev<typename Pr::M> L, int colour) {
    pdl_wait();
    pdl_trigger();
    rbgs_body<Pr>(L, colour);
}

// ---- vector form: 8 consecutive same-colour cells of a row per lane ----
// A warp takes one tile: lane = (h chunk of 8) x (row j) x (plane k), so with TH = 32 a
// tile is 4 x 4 x 2 lanes. Every array moves in 16-byte pieces (8 elements), which cuts
// the memory instructions per cell by 8; it needs H to be a multiple of 8.
constexpr int V8 = 8;
constexpr int V8_LANES_H = TH / V8;  // 4
static_assert(V8_LANES_H * TY * TZ == 32, "one warp per tile in the vector kernels");

template <class T>
struct Vec8 {
    T v[V8];
};
template <class T>
__device__ __forceinline__ Vec8<T> ld8(const T* p) {  // p 16-byte aligned
    Vec8<T> r;
    constexpr int n = (int)(sizeof(T) * V8 / 16);
#pragma unroll
    for (int q = 0; q < n; q++) reinterpret_cast<uint4*>(r.v)[q] = reinterpret_cast<const uint4*>(p)[q];
    return r;
}
template <class T>
__device__ __forceinline__ void st8(T* p, const Vec8<T>& r) {
    constexpr int n = (int)(sizeof(T) * V8 / 16);
#pragma unroll
    for (int q = 0; q < n; q++) reinterpret_cast<uint4*>(p)[q] = reinterpret_cast<const uint4*>(r.v)[q];
}

// rbgs_kernel! (src/flip.jl:870-877), vector form. Own colour: code (8 bytes), diagonal
// and b in, x out (zero where the cell is not LIQUID, which is what every such cell holds,
// so its old value need not be read); other colour: the same 8 columns of this row (the
// +x/-x neighbours, plus one element on each side) and of the rows at -+y, -+z.
// Software-pipelined: a warp issues the next tile's loads before this tile's arithmetic
// (tile ids two ahead), so its loads stay in flight while it computes; two blocks of 256
// per SM hold both tiles' registers, and the grid is exactly that many blocks. Before its
// programmatic-dependent-launch wait, a warp already loads its first tile's id, code,
// diagonal and b: the preceding kernel (a colour pass, start or prolongation) writes only
// x, and everything older is complete once that kernel has passed its own wait. After a
// restriction that also started the level (b_late), b waits too.
template <class M>
struct RbLd {
    uint2 cdw;
    Vec8<M> dv, bv, xc, yp, ym, zp, zm;
    M xl, xr;
    int p, ci;
    bool ok;
};
// A tile's loads in two parts: what no pass of the smoother writes (the code, diagonal and
// b of the own colour; issued before the kernel waits on its predecessor), then the other
// colour's x.
template <class Pr>
__device__ __forceinline__ void rbgs_fetch_s(const Lev<typename Pr::M>& L, int colour, uint32_t tile, int hq, int lj,
                                             int lk, bool need_code, bool with_b, RbLd<typename Pr::M>& a) {
    const int h = (int)(tile & 1023u) * TH + hq * V8, j = (int)((tile >> 10) & 1023u) * TY + lj,
              k = (int)(tile >> 20) * TZ + lk;
    a.ok = h < L.H && j < L.n2 && k < L.n3;
    if (!a.ok) return;
    const int p = (k * L.n2 + j) * L.n1 + colour * L.H + h;
    a.p = p;
    a.ci = ci_of(colour, j, k);
    if (need_code) a.cdw = *reinterpret_cast<const uint2*>(L.code + p);
    a.dv = ld8((Pr::scaled ? L.di : L.dg) + p);
    if (with_b) a.bv = ld8(L.b + p);
}
template <class Pr>
__device__ __forceinline__ void rbgs_fetch_x(const Lev<typename Pr::M>& L, int colour, bool with_b, RbLd<typename Pr::M>& a) {
    if (!a.ok) return;
    if (with_b) a.bv = ld8(L.b + a.p);
    const int sy = L.n1, sz = L.n1 * L.n2;
    const int o = a.p + (1 - 2 * colour) * L.H;  // the same columns in the other colour's half
    a.xc = ld8(L.x + o);
    a.yp = ld8(L.x + o + sy);
    a.ym = ld8(L.x + o - sy);
    a.zp = ld8(L.x + o + sz);
    a.zm = ld8(L.x + o - sz);
    a.xl = L.x[o - 1];
    a.xr = L.x[o + V8];
}

// by_di: the 16-bit forms on a level with no LIQUID cell on its x/y faces, whose stencil
// codes are not read. There the unmasked neighbour sum needs no code, and a cell is LIQUID
// exactly when its stored reciprocal diagonal is nonzero: the set-up stores 0 off-liquid,
// and a LIQUID cell's diagonal is at most 6 x 100 (theta >= 0.01), so its reciprocal is a
// normal FP16 number. The one exception, a LIQUID cell with no open face (diagonal 0), gets
// +0 where (b + s) * 0 could give -0.
template <class C, class M>
__device__ __forceinline__ Vec8<M> rbgs_tile(const RbLd<M>& cur, bool edge, bool scaled, bool by_di) {
    Vec8<M> out;
#pragma unroll
    for (int q = 0; q < V8; q++) {
        // constant element indices only (selects), so the tile stays in registers
        const C d = ld<C>(&cur.dv.v[q]);
        const uint8_t cd = by_di ? (uint8_t)(d != (C)0 ? SELF : 0)
                                 : (uint8_t)(((q < 4 ? cur.cdw.x : cur.cdw.y) >> (8 * (q & 3))) & 0xffu);
        const M xp = cur.ci ? (q + 1 < V8 ? cur.xc.v[q + 1 < V8 ? q + 1 : 0] : cur.xr) : cur.xc.v[q];
        const M xm = cur.ci ? cur.xc.v[q] : (q > 0 ? cur.xc.v[q > 0 ? q - 1 : 0] : cur.xl);
        const M nb[6] = {xp, xm, cur.yp.v[q], cur.ym.v[q], cur.zp.v[q], cur.zm.v[q]};
        C v = (C)0;
        if (cd & SELF) {
            // liquidsum in the reference's order, each stored neighbour widened inside its add
            C s;
            if (edge) {
                s = (C)0;
#pragma unroll
                for (int m = 0; m < 6; m++)
                    if (cd & (1u << m)) s = addm(nb[m], s);
            } else {
                s = ld<C>(&nb[0]);
#pragma unroll
                for (int m = 1; m < 6; m++) s = addm(nb[m], s);
            }
            // the 16-bit forms multiply by the stored reciprocal (0 where the diagonal is)
            if (scaled) v = addm(cur.bv.v[q], s) * d;
            else v = d > (C)0 ? addm(cur.bv.v[q], s) / d : (C)0;
        }
        st(&out.v[q], v);
    }
    return out;
}
// The kernel's body, PDL wait included: the first tile's static loads go out before it.
// The 16-bit forms keep two tiles in flight; the 4- and 8-byte forms (twice the registers
// a tile) one.
template <class Pr>
__device__ __forceinline__ void rbgs_v8_body(Lev<typename Pr::M> L, int colour, int b_late) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    constexpr bool PIPE = sizeof(M) <= 2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = TPB / 32;
    const int hq = lane % V8_LANES_H, lj = (lane / V8_LANES_H) % TY, lk = lane / (V8_LANES_H * TY);
    const int n = *L.count;  // tile lists and codes date from the set-up
    const bool edge = *L.edge != 0;
    const bool by_di = Pr::scaled && !edge, need_code = !by_di;
    const int stride = gridDim.x * wpb;
    int t = blockIdx.x * wpb + warp;
    RbLd<M> cur;
    uint32_t tile1 = 0u;
    if (t < n) {
        tile1 = t + stride < n ? L.tiles[t + stride] : 0u;
        rbgs_fetch_s<Pr>(L, colour, L.tiles[t], hq, lj, lk, need_code, !b_late, cur);
    }
    pdl_wait();
    pdl_trigger();
    if (t >= n) return;
    rbgs_fetch_x<Pr>(L, colour, b_late != 0, cur);
    for (; t < n; t += stride) {
        const uint32_t tile2 = t + 2 * stride < n ? L.tiles[t + 2 * stride] : 0u;
        if constexpr (PIPE) {
            // the next tile's loads first (a tile's own-colour cells are no other tile's, and
            // the other colour is only read, so they may pass this tile's stores)
            RbLd<M> nxt;
            nxt.ok = false;
            if (t + stride < n) {
                rbgs_fetch_s<Pr>(L, colour, tile1, hq, lj, lk, need_code, true, nxt);
                rbgs_fetch_x<Pr>(L, colour, false, nxt);
            }
            if (cur.ok) st8(L.x + cur.p, rbgs_tile<C, M>(cur, edge, Pr::scaled, by_di));
            cur = nxt;
        } else {
            if (cur.ok) st8(L.x + cur.p, rbgs_tile<C, M>(cur, edge, Pr::scaled, by_di));
            cur.ok = false;
            if (t + stride < n) {
                rbgs_fetch_s<Pr>(L, colour, tile1, hq, lj, lk, need_code, true, cur);
                rbgs_fetch_x<Pr>(L, colour, false, cur);
            }
        }
        tile1 = tile2;
    }
}
// blocks per SM of k_rbgs_v8, and its grid: exactly the blocks that are resident at once
// (two of 256 threads at up to 128 registers a thread)
constexpr int RBGS_V8_BLOCKS = 2;
template <class Pr>
__global__ void __launch_bounds__(TPB, RBGS_V8_BLOCKS) k_rbgs_v8(Lev<typename Pr::M> L, int colour, int b_late) {
    rbgs_v8_body<Pr>(L, colour, b_late);
}

// A lane's 8 columns in a tile (vector kernels): h .. h+7 of row j, plane k.
struct Lane8 {
    int h, j, k, rb;
};
template <class M>
__device__ __forceinline__ bool lane8_of(const Lev<M>& L, uint32_t tile, Lane8& a) {
    const int lane = threadIdx.x & 31;
    a.h = (int)(tile & 1023u) * TH + (lane % V8_LANES_H) * V8;
    a.j = (int)((tile >> 10) & 1023u) * TY + (lane / V8_LANES_H) % TY;
    a.k = (int)(tile >> 20) * TZ + lane / (V8_LANES_H * TY);
    a.rb = (a.k * L.n2 + a.j) * L.n1;
    return a.h < L.H && a.j < L.n2 && a.k < L.n3;
}
// (the next tile's id fetched one step ahead)
#define FOR_TILES_W(L, tile)                                                                              \
    const int n_ = *(L).count, s_ = gridDim.x * (TPB / 32);                                               \
    int t_ = blockIdx.x * (TPB / 32) + (int)(threadIdx.x >> 5);                                           \
    uint32_t tile = t_ < n_ ? (L).tiles[t_] : 0u;                                                         \
    for (uint32_t next_; t_ < n_; t_ += s_, tile = next_)                                                 \
        if ((next_ = (t_ + s_ < n_ ? (L).tiles[t_ + s_] : 0u)), true)

// Walk this warp's share of a level's tile list in units (tile, sub-unit < NU), the loads
// of the next unit issued before the arithmetic of this one and its tile id fetched two
// units ahead (the rbgs_v8 pipeline, for passes whose units do not overlap in what they
// write). fetch_s(tile, sub, Ld&) issues the loads of arrays the preceding kernel does not
// write, fetch_d(Ld&) the rest; the first unit's fetch_s runs before gate() (the
// programmatic-dependent-launch wait; false: the pass has nothing to do), and
// compute(const Ld&) consumes a unit.
template <int NU, class Ld, class FetchS, class FetchD, class Gate, class Compute>
__device__ __forceinline__ void walk_tiles_pipelined(const uint32_t* tiles, int n, FetchS&& fetch_s, FetchD&& fetch_d,
                                                     Gate&& gate, Compute&& compute) {
    const int wpb = TPB / 32, warp = threadIdx.x >> 5;
    const int stride = gridDim.x * wpb, total = n * NU;
    int u = blockIdx.x * wpb + warp;
    uint32_t tile1 = 0u;
    Ld cur;
    if (u < total) {
        tile1 = u + stride < total ? tiles[(u + stride) / NU] : 0u;
        fetch_s(tiles[u / NU], u % NU, cur);
    }
    if (!gate() || u >= total) return;
    fetch_d(cur);
    for (; u < total; u += stride) {
        Ld nxt;
        const uint32_t tile2 = u + 2 * stride < total ? tiles[(u + 2 * stride) / NU] : 0u;
        if (u + stride < total) {
            fetch_s(tile1, (u + stride) % NU, nxt);
            fetch_d(nxt);
        }
        tile1 = tile2;
        compute(cur);
        cur = nxt;
    }
}

// The other colour's values around a lane's 8 cells: the same 8 columns of this row
// (the +x/-x neighbours) with one element on each side, and of the rows at +-y, +-z.
template <class M>
struct Nb8 {
    Vec8<M> c, yp, ym, zp, zm;
    M l, r;
};
template <class M>
__device__ __forceinline__ Nb8<M> ld_nb8(const M* x, int o, int sy, int sz) {
    Nb8<M> a;
    a.c = ld8(x + o);
    a.yp = ld8(x + o + sy);
    a.ym = ld8(x + o - sy);
    a.zp = ld8(x + o + sz);
    a.zm = ld8(x + o - sz);
    a.l = x[o - 1];
    a.r = x[o + V8];
    return a;
}
// neighbour m (+x,-x,+y,-y,+z,-z) of the lane's cell q; ci: its colour offset in the row
// (q is a compile-time constant in the unrolled callers; ci selects between two
// compile-time-indexed values, so nothing is indexed at run time.)
template <class C, class M>
__device__ __forceinline__ void nb6_of(C (&nb)[6], const Nb8<M>& a, int q, int ci) {
    const M xp = ci ? (q + 1 < V8 ? a.c.v[q + 1 < V8 ? q + 1 : 0] : a.r) : a.c.v[q];
    const M xm = ci ? a.c.v[q] : (q >= 1 ? a.c.v[q >= 1 ? q - 1 : 0] : a.l);
    nb[0] = ld<C>(&xp);
    nb[1] = ld<C>(&xm);
    nb[2] = ld<C>(&a.yp.v[q]);
    nb[3] = ld<C>(&a.ym.v[q]);
    nb[4] = ld<C>(&a.zp.v[q]);
    nb[5] = ld<C>(&a.zm.v[q]);
}

template <class M>
struct StartLd {
    uint2 cdw;
    Vec8<M> dv, bv;
    int p;
    bool ok;
};
// start_kernel! (src/flip.jl:965-973), vector form, pipelined: code and diagonal load
// before the programmatic-dependent-launch wait, b (the preceding restriction's or CG
// step's output) after it.
template <class Pr>
__device__ __forceinline__ void start_v8_body(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    walk_tiles_pipelined<1, StartLd<M>>(
        L.tiles, *L.count,
        [&](uint32_t tile, int, StartLd<M>& a) {
            Lane8 l8;
            a.ok = lane8_of(L, tile, l8);
            if (!a.ok) return;
            a.p = l8.rb + l8.h;
            a.cdw = *reinterpret_cast<const uint2*>(L.code + a.p);
            a.dv = ld8((Pr::scaled ? L.di : L.dg) + a.p);
        },
        [&](StartLd<M>& a) {
            if (a.ok) a.bv = ld8(L.b + a.p);
        },
        [&]() {
            pdl_wait();
            pdl_trigger();
            return true;
        },
        [&](const StartLd<M>& a) {
            if (!a.ok) return;
            Vec8<M> x0, x1;
#pragma unroll
            for (int q = 0; q < V8; q++) {
                const uint8_t cd = (uint8_t)(((q < 4 ? a.cdw.x : a.cdw.y) >> (8 * (q & 3))) & 0xffu);
                const C d = ld<C>(&a.dv.v[q]);
                if constexpr (Pr::scaled) st(&x0.v[q], (cd & SELF) ? ld<C>(&a.bv.v[q]) * d : (C)0);
                else st(&x0.v[q], ((cd & SELF) && d > (C)0) ? ld<C>(&a.bv.v[q]) / d : (C)0);
                st(&x1.v[q], (C)0);
            }
            st8(L.x + a.p, x0);
            st8(L.x + a.p + L.H, x1);
        });
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_start_v8(Lev<typename Pr::M> L) {
    start_v8_body<Pr>(L);
}

// residual_kernel! (src/flip.jl:859-863), vector form: one colour of a tile a unit,
// pipelined; code, diagonal and b (older than the preceding colour pass) load before the
// programmatic-dependent-launch wait, x after it.
template <class M>
struct ResLd {
    uint2 cdw;
    Vec8<M> dv, bv, xv;
    Nb8<M> nb;
    int p, o, ci;
    bool ok;
};
template <class Pr>
__device__ __forceinline__ void residual_v8_body(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    const int sy = L.n1, sz = L.n1 * L.n2;
    const bool edge = *L.edge != 0;
    walk_tiles_pipelined<2, ResLd<M>>(
        L.tiles, *L.count,
        [&](uint32_t tile, int cc, ResLd<M>& a) {
            Lane8 l8;
            a.ok = lane8_of(L, tile, l8);
            if (!a.ok) return;
            a.p = l8.rb + cc * L.H + l8.h;
            a.o = l8.rb + (1 - cc) * L.H + l8.h;
            a.ci = ci_of(cc, l8.j, l8.k);
            a.cdw = *reinterpret_cast<const uint2*>(L.code + a.p);
            a.dv = ld8(L.dg + a.p);
            a.bv = ld8(L.b + a.p);
        },
        [&](ResLd<M>& a) {
            if (!a.ok) return;
            a.xv = ld8(L.x + a.p);
            a.nb = ld_nb8(L.x, a.o, sy, sz);
        },
        [&]() {
            pdl_wait();
            pdl_trigger();
            return true;
        },
        [&](const ResLd<M>& a) {
            if (!a.ok) return;
            Vec8<M> out;
#pragma unroll
            for (int q = 0; q < V8; q++) {
                const uint8_t cd = (uint8_t)(((q < 4 ? a.cdw.x : a.cdw.y) >> (8 * (q & 3))) & 0xffu);
                C v = (C)0;
                if (cd & SELF) {
                    // liquidsum (each stored neighbour widened inside its add), then b - (d x - s)
                    const M xp = a.ci ? (q + 1 < V8 ? a.nb.c.v[q + 1 < V8 ? q + 1 : 0] : a.nb.r) : a.nb.c.v[q];
                    const M xm = a.ci ? a.nb.c.v[q] : (q >= 1 ? a.nb.c.v[q >= 1 ? q - 1 : 0] : a.nb.l);
                    const M n6[6] = {xp, xm, a.nb.yp.v[q], a.nb.ym.v[q], a.nb.zp.v[q], a.nb.zm.v[q]};
                    C s;
                    if (edge) {
                        s = (C)0;
#pragma unroll
                        for (int m = 0; m < 6; m++)
                            if (cd & (1u << m)) s = addm(n6[m], s);
                    } else {
                        s = ld<C>(&n6[0]);
#pragma unroll
                        for (int m = 1; m < 6; m++) s = addm(n6[m], s);
                    }
                    v = ld<C>(&a.bv.v[q]) - (ld<C>(&a.dv.v[q]) * ld<C>(&a.xv.v[q]) - s);
                }
                st(&out.v[q], v);
            }
            st8(L.r + a.p, out);
        });
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_residual_v8(Lev<typename Pr::M> L) {
    residual_v8_body<Pr>(L);
}

// inner(s, z, r) and the flexible z.q (see k_dot), vector form: one colour of a tile a
// unit, pipelined.
template <class M, class V, bool FLEX>
struct DotLd {
    uint2 cdw;
    Vec8<M> zv;
    Vec8<V> rv;
    Vec8<V> qq;  // (flexible form only)
    int p;
    bool ok;
};
template <class Pr>
__device__ __forceinline__ void dot_v8_dev(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ r, const typename Pr::V* __restrict__ qv,
             Scalars* sc, double* partials, unsigned* counter) {
    using M = typename Pr::M;
    using V = typename Pr::V;
    using Ld = DotLd<M, V, Pr::flexible>;
    double acc[2] = {0.0, 0.0};
    bool done = false;
    // r and q date from the previous iteration's step and search; z is the V-cycle's last
    // pass's output, loaded after the wait
    walk_tiles_pipelined<2, Ld>(
        L.tiles, *L.count,
        [&](uint32_t tile, int cc, Ld& a) {
            Lane8 l8;
            a.ok = lane8_of(L, tile, l8);
            if (!a.ok) return;
            a.p = l8.rb + cc * L.H + l8.h;
            a.cdw = *reinterpret_cast<const uint2*>(L.code + a.p);
            a.rv = ld8(r + a.p);
            if constexpr (Pr::flexible) a.qq = ld8(qv + a.p);
        },
        [&](Ld& a) {
            if (a.ok) a.zv = ld8(L.x + a.p);
        },
        [&]() {
            pdl_wait();
            pdl_trigger();
            done = sc->s.done != 0;
            return !done;
        },
        [&](const Ld& a) {
            if (!a.ok) return;
#pragma unroll
            for (int q = 0; q < V8; q++) {
                const uint8_t cd = (uint8_t)(((q < 4 ? a.cdw.x : a.cdw.y) >> (8 * (q & 3))) & 0xffu);
                if (cd & SELF) {
                    const double z = ld<double>(&a.zv.v[q]);
                    acc[0] += z * (double)a.rv.v[q];
                    if constexpr (Pr::flexible) acc[1] += z * (double)a.qq.v[q];
                }
            }
        });
    if (done) return;
    if (grid_sum<2>(acc, partials, counter) && threadIdx.x == 0) dot_finish<Pr>(sc, acc);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_dot_v8(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ r, const typename Pr::V* __restrict__ qv,
             Scalars* sc, double* partials, unsigned* counter) {
    dot_v8_dev<Pr>(L, r, qv, sc, partials, counter);
}

// search_kernel! (src/flip.jl:1033-1054), vector form: one colour of a tile a unit. Every
// array it reads dates from before the preceding kernel (z·r, which writes only the
// scalars), so a warp loads its first unit before the programmatic-dependent-launch wait;
// beta is read after it (d is loaded on the first pass too, and not used).
template <class M, class V>
struct SearchLd {
    uint2 cdw;
    Vec8<V> gv, dc;
    Vec8<M> zc;
    Nb8<M> zn;
    Nb8<V> dn;
    int p, ci;
    bool ok;
};
template <class Pr>
__device__ __forceinline__ void search_fetch(const Lev<typename Pr::M>& L, const typename Pr::V* dvec,
                                             const typename Pr::V* diag, uint32_t tile, int cc,
                                             SearchLd<typename Pr::M, typename Pr::V>& a) {
    Lane8 l8;
    a.ok = lane8_of(L, tile, l8);
    if (!a.ok) return;
    const int sy = L.n1, sz = L.n1 * L.n2;
    const int p = l8.rb + cc * L.H + l8.h, o = l8.rb + (1 - cc) * L.H + l8.h;
    a.p = p;
    a.ci = ci_of(cc, l8.j, l8.k);
    a.cdw = *reinterpret_cast<const uint2*>(L.code + p);
    a.gv = ld8(diag + p);
    a.zc = ld8(L.x + p);
    a.zn = ld_nb8(L.x, o, sy, sz);
    a.dc = ld8(dvec + p);
    a.dn = ld_nb8(dvec, o, sy, sz);
}
template <class Pr>
__device__ __forceinline__ void search_v8_dev(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ diag,
                typename Pr::V* __restrict__ qout, Scalars* sc, double* partials, unsigned* counter) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    using V = typename Pr::V;
    const int wpb = TPB / 32, warp = threadIdx.x >> 5;
    const int n = *L.count, total = 2 * n, stride = gridDim.x * wpb;
    int u = blockIdx.x * wpb + warp;
    SearchLd<M, V> a;
    uint32_t tile1 = 0u;
    if (u < total) {
        tile1 = u + stride < total ? L.tiles[(u + stride) >> 1] : 0u;
        search_fetch<Pr>(L, dvec, diag, L.tiles[u >> 1], u & 1, a);
    }
    pdl_wait();
    pdl_trigger();
    if (sc->s.done) return;
    const C beta = (C)sc->s.beta;
    const bool first = sc->s.beta == 0.0;
    const bool edge = *L.edge != 0;
    double acc[1] = {0.0};
    for (; u < total; u += stride) {
        const uint32_t tile2 = u + 2 * stride < total ? L.tiles[(u + 2 * stride) >> 1] : 0u;
        if (a.ok) {
            Vec8<V> out;
#pragma unroll
            for (int q = 0; q < V8; q++) {
                const uint8_t cd = (uint8_t)(((q < 4 ? a.cdw.x : a.cdw.y) >> (8 * (q & 3))) & 0xffu);
                C qv = (C)0;
                if (cd & SELF) {
                    C z6[6], d6[6];
                    nb6_of(z6, a.zn, q, a.ci);
                    if (!first) nb6_of(d6, a.dn, q, a.ci);
                    const C pc = first ? ld<C>(&a.zc.v[q]) : ld<C>(&a.zc.v[q]) + beta * (C)a.dc.v[q];
                    C s = (C)0;  // nsum6 over p = z + beta d, formed term by term
#pragma unroll
                    for (int m = 0; m < 6; m++) {
                        const C pm = first ? z6[m] : z6[m] + beta * d6[m];
                        if (!edge || (cd & (1u << m))) s += pm;
                    }
                    qv = (C)a.gv.v[q] * pc - s;
                    acc[0] += (double)pc * (double)qv;
                }
                st(&out.v[q], qv);
            }
            st8(qout + a.p, out);
        }
        a.ok = false;
        if (u + stride < total) search_fetch<Pr>(L, dvec, diag, tile1, (u + stride) & 1, a);
        tile1 = tile2;
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) search_finish<Pr>(sc, acc);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 2) k_search_v8(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ diag,
                typename Pr::V* __restrict__ qout, Scalars* sc, double* partials, unsigned* counter) {
    search_v8_dev<Pr>(L, dvec, diag, qout, sc, partials, counter);
}

// advance_kernel! (src/flip.jl:1059-1073), vector form. The lane's 16 cells (both colours)
// are 16 consecutive cells of the natural row, so P moves as one 16-element run.
template <class Pr>
__device__ __forceinline__ void advance_v8_dev(Lev<typename Pr::M> L, typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ qv,
                 typename Pr::V* __restrict__ r, typename Pr::V* __restrict__ P, Scalars* sc, double* partials,
                 unsigned* counter, cudaGraphConditionalHandle cond, int use_cond, int start) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    using V = typename Pr::V;
    // the first tile id (the tile lists date from the set-up) before the wait
    const int n_ = *L.count, s_ = gridDim.x * (TPB / 32);
    int t_ = blockIdx.x * (TPB / 32) + (int)(threadIdx.x >> 5);
    uint32_t tile = t_ < n_ ? L.tiles[t_] : 0u;
    pdl_wait();
    pdl_trigger();
    if (sc->s.done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(cond, use_cond, 0);
        return;
    }
    const C beta = (C)sc->s.beta, alpha = (C)sc->s.alpha;
    const bool first = sc->s.beta == 0.0;
    const bool sep_b = (void*)L.b != (void*)r;
    const C rsc = (C)sc->s.rscale;
    double acc[1] = {0.0};
    for (uint32_t next_; t_ < n_; t_ += s_, tile = next_) {
        next_ = t_ + s_ < n_ ? L.tiles[t_ + s_] : 0u;
        Lane8 a;
        if (!lane8_of(L, tile, a)) continue;
        const int pn = a.rb + 2 * a.h;  // natural run of the lane's 16 cells
        Vec8<V> P0 = ld8(P + pn), P1 = ld8(P + pn + V8);
#pragma unroll
        for (int cc = 0; cc < 2; cc++) {
            const int p = a.rb + cc * L.H + a.h;
            const int ci = ci_of(cc, a.j, a.k);
            const uint2 cdw = *reinterpret_cast<const uint2*>(L.code + p);
            const Vec8<M> zv = ld8(L.x + p);
            Vec8<V> dd = ld8(dvec + p), rr = ld8(r + p);
            const Vec8<V> qq = ld8(qv + p);
            const uint8_t* cd = reinterpret_cast<const uint8_t*>(&cdw);
            // the V-cycle's right-hand side is written whole: zero off-liquid, which is what it
            // holds there (the set-up writes zeros, every later writer only LIQUID cells)
            Vec8<M> rbv;
#pragma unroll
            for (int q = 0; q < V8; q++) st(&rbv.v[q], (C)0);
#pragma unroll
            for (int q = 0; q < V8; q++) {
                if (!(cd[q] & SELF)) continue;
                const C pc = first ? ld<C>(&zv.v[q]) : ld<C>(&zv.v[q]) + beta * (C)dd.v[q];
                const C rl = (C)rr.v[q] - alpha * (C)qq.v[q];
                st(&dd.v[q], pc);
                st(&rr.v[q], rl);
                if (sep_b) st(&rbv.v[q], rl * rsc);
                // the cell's place in the natural run: 2q + ci (compile-time index per branch)
                if (ci == 0) {
                    V& Pi = (2 * q < V8) ? P0.v[(2 * q) % V8] : P1.v[(2 * q) % V8];
                    st(&Pi, (C)Pi + alpha * pc);
                } else {
                    V& Pi = (2 * q + 1 < V8) ? P0.v[(2 * q + 1) % V8] : P1.v[(2 * q + 1) % V8];
                    st(&Pi, (C)Pi + alpha * pc);
                }
                acc[0] += (double)rl * (double)rl;
            }
            st8(dvec + p, dd);
            st8(r + p, rr);
            if (sep_b) st8(L.b + p, rbv);
            if (start) {
                // the next V-cycle's start_kernel! (start_v8_body's arithmetic): x = b / diag
                // on the first colour's LIQUID cells, b as this step stores it; 0 elsewhere
                Vec8<M> xs;
                if (cc == 0) {
                    const Vec8<M> dv = ld8((Pr::scaled ? L.di : L.dg) + p);
#pragma unroll
                    for (int q = 0; q < V8; q++) {
                        const C bq = sep_b ? ld<C>(&rbv.v[q]) : (C)rr.v[q];
                        const C d = ld<C>(&dv.v[q]);
                        C xq;
                        if constexpr (Pr::scaled) xq = (cd[q] & SELF) ? bq * d : (C)0;
                        else xq = ((cd[q] & SELF) && d > (C)0) ? bq / d : (C)0;
                        st(&xs.v[q], xq);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < V8; q++) st(&xs.v[q], (C)0);
                }
                st8(L.x + p, xs);
            }
        }
        st8(P + pn, P0);
        st8(P + pn + V8, P1);
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) advance_finish<Pr>(sc, acc, cond, use_cond);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 3) k_advance_v8(Lev<typename Pr::M> L, typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ qv,
                 typename Pr::V* __restrict__ r, typename Pr::V* __restrict__ P, Scalars* sc, double* partials,
                 unsigned* counter, cudaGraphConditionalHandle cond, int use_cond, int start) {
    advance_v8_dev<Pr>(L, dvec, qv, r, P, sc, partials, counter, cond, use_cond, start);
}

// prolong_kernel! (src/flip.jl:914-929), vector form: one warp per fine tile stages the
// tile's PX x PY x PZ coarse cells in its own slice of shared memory (non-LIQUID coarse
// cells hold zero, as in k_prolong), then each lane adds the trilinear correction to its
// 16 fine cells (8 columns, both colours) and writes them back in 16-byte pieces.
template <class Pr>
__device__ __forceinline__ void prolong_v8_body(Lev<typename Pr::M> L, Lev<typename Pr::M> Cl, int cnat) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    constexpr int WPB = TPB / 32, NE = PX * PY * PZ, PER = (NE + 31) / 32;
    __shared__ C smw[WPB][PZ][PY][PX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    C(*S)[PY][PX] = smw[warp];
    const int n = *L.count, stride = gridDim.x * WPB;
    constexpr int CH = 16 / (int)sizeof(M), NCHK = (TH / 2 + 2 * CH) / CH, NV = PY * PZ * 2 * NCHK,
                  NVL = (NV + 31) / 32;
    static_assert((TH / 2) % CH == 0, "pieces aligned to the tile's coarse columns");
    const bool vec = !cnat && Cl.n1 % (2 * CH) == 0 && (reinterpret_cast<uintptr_t>(Cl.x) & 15) == 0;
    // the first tile id before the programmatic-dependent-launch wait (the tile lists date
    // from the set-up; the coarse x is the preceding kernel's output)
    int t = blockIdx.x * WPB + warp;
    uint32_t tile = t < n ? L.tiles[t] : 0u;
    pdl_wait();
    pdl_trigger();
    for (; t < n; t += stride) {
        const uint32_t tile_next = t + stride < n ? L.tiles[t + stride] : 0u;
        const int I0 = (int)(tile & 1023u) * TH - 1, J0 = (int)((tile >> 10) & 1023u) * (TY / 2) - 1,
                  K0 = (int)(tile >> 20) * (TZ / 2) - 1;
        const int ps = (int)(tile & 1023u) * (TH / 2) - CH;  // first piece's position
        C vals[PER];
        Vec16<M> vv[NVL];
        if (vec) {
            // row-split coarse rows in 16-byte pieces: the region's natural columns I0 ..
            // I0 + PX - 1 sit at positions (TH / 2) th - 1 .. (TH / 2)(th + 1) of each colour's
            // half-row, covered by NCHK aligned pieces from (TH / 2) th - CH; a piece lies
            // wholly inside [0, H) or wholly outside it (read as zeros)
#pragma unroll
            for (int u = 0; u < NVL; u++) {
                const int e = lane + 32 * u, rr = e / (2 * NCHK), rem = e - rr * 2 * NCHK;
                const int c = rem / NCHK, ch = rem - c * NCHK;
                const int J = J0 + rr % PY, K = K0 + rr / PY, pos0 = ps + ch * CH;
                vv[u].u = make_uint4(0u, 0u, 0u, 0u);
                if (e < NV && J >= 0 && J < Cl.n2 && K >= 0 && K < Cl.n3 && pos0 >= 0 && pos0 < Cl.H)
                    vv[u].u = *reinterpret_cast<const uint4*>(Cl.x + (K * Cl.n2 + J) * Cl.n1 + c * Cl.H + pos0);
            }
        } else {
#pragma unroll
            for (int u = 0; u < PER; u++) {
                const int e = lane + 32 * u;
                const int ii = e % PX, jj = (e / PX) % PY, kk = e / (PX * PY);
                const int I = I0 + ii, J = J0 + jj, K = K0 + kk;
                vals[u] = (C)0;
                if (e < NE && I >= 0 && I < Cl.n1 && J >= 0 && J < Cl.n2 && K >= 0 && K < Cl.n3)
                    vals[u] = ld<C>(Cl.x + (cnat ? (int)Cl.nat(I, J, K) : (int)Cl.pos(I, J, K)));
            }
        }
        // this lane's fine cells, loaded beside the staging loads
        Lane8 a;
        const bool ok = lane8_of(L, tile, a);
        uint2 cdw[2];
        Vec8<M> xv[2];
        if (ok) {
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = a.rb + cc * L.H + a.h;
                cdw[cc] = *reinterpret_cast<const uint2*>(L.code + p);
                xv[cc] = ld8(L.x + p);
            }
        }
        __syncwarp();
        if (vec) {
#pragma unroll
            for (int u = 0; u < NVL; u++) {
                const int e = lane + 32 * u, rr = e / (2 * NCHK), rem = e - rr * 2 * NCHK;
                const int c = rem / NCHK, ch = rem - c * NCHK;
                const int jj = rr % PY, kk = rr / PY, par = (c + J0 + jj + K0 + kk + 1) & 1;
                if (e >= NV) continue;
#pragma unroll
                for (int q = 0; q < CH; q++) {
                    const int ii = 2 * (ps + ch * CH + q) + par - I0;  // natural column in the region
                    if (ii >= 0 && ii < PX) S[kk][jj][ii] = ld<C>(&vv[u].m[q]);
                }
            }
        } else {
#pragma unroll
            for (int u = 0; u < PER; u++) {
                const int e = lane + 32 * u;
                if (e < NE) (&S[0][0][0])[e] = vals[u];
            }
        }
        __syncwarp();
        tile = tile_next;
        if (!ok) continue;
        int b0, b1, k0, k1;
        C wb0, wb1, wc0, wc1;
        pweights<C>(a.j, b0, wb0, b1, wb1);
        pweights<C>(a.k, k0, wc0, k1, wc1);
        b0 -= J0; b1 -= J0; k0 -= K0; k1 -= K0;
        // prolongweights of i = 2 (h + q) + ci: coarse columns h + q - 1 + ci and the next,
        // weights by the parity ci alone. The lane's cells of parity 0 (e0) and 1 (e1) are
        // summed together, one staged row (B, K) at a time: the row's 10 columns the lane
        // needs are read once into registers, and each cell takes its 8 terms (w_a w_b) w_c
        // x in the reference's order (a fastest, then b, then c), each as macc rounds it.
        C e0[V8], e1[V8];
#pragma unroll
        for (int q = 0; q < V8; q++) e0[q] = e1[q] = (C)0;
        const int lo = a.h - 1 - I0;  // the row's first column the lane reads
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int B = (r & 1) ? b1 : b0, K = (r & 2) ? k1 : k0;
            const C wbc = ((r & 1) ? wb1 : wb0), wc = ((r & 2) ? wc1 : wc0);
            // w_a w_b w_c for a = 0, 1 at parity 0 (w_a 1/4, 3/4) and parity 1 (3/4, 1/4)
            const C wq = (C)0.25f * wbc * wc, w3 = (C)0.75f * wbc * wc;
            const C* row = &S[K][B][lo];
            C v[V8 + 2];
#pragma unroll
            for (int e = 0; e < V8 + 2; e++) v[e] = row[e];
#pragma unroll
            for (int q = 0; q < V8; q++) {
                e0[q] = macc<Pr::scaled>(e0[q], wq, v[q]);
                e0[q] = macc<Pr::scaled>(e0[q], w3, v[q + 1]);
                e1[q] = macc<Pr::scaled>(e1[q], w3, v[q + 1]);
                e1[q] = macc<Pr::scaled>(e1[q], wq, v[q + 2]);
            }
        }
#pragma unroll
        for (int cc = 0; cc < 2; cc++) {
            const int p = a.rb + cc * L.H + a.h;
            const bool odd = ci_of(cc, a.j, a.k) != 0;
#pragma unroll
            for (int q = 0; q < V8; q++) {
                const uint8_t cd = (uint8_t)(((q < 4 ? cdw[cc].x : cdw[cc].y) >> (8 * (q & 3))) & 0xffu);
                if (!(cd & SELF)) continue;
                const C s = odd ? e1[q] : e0[q];
                st(&xv[cc].v[q], addm(xv[cc].v[q], Pr::scaled ? (C)4 * s : s));
            }
            st8(L.x + p, xv[cc]);
        }
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_prolong_v8(Lev<typename Pr::M> L, Lev<typename Pr::M> Cl, int cnat) {
    prolong_v8_body<Pr>(L, Cl, cnat);
}

// residual_kernel! (src/flip.jl:859-863): r = b - (diag x - sum_LIQ x_n) on LIQUID, else 0.
template <class Pr>
__device__ __forceinline__ void residual_body(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    const int sy = L.n1, sz = L.n1 * L.n2;
    const bool edge = *L.edge != 0;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            if (q >= c.kn) break;
            const int rb = c.rb + q * sz;
            uint8_t cd[2];
            C nb[2][6], dv[2], bv[2], xv[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = rb + cc * L.H + c.h;
                cd[cc] = L.code[p];
                dv[cc] = ld<C>(L.dg + p);
                bv[cc] = ld<C>(L.b + p);
                xv[cc] = ld<C>(L.x + p);
                load6<C>(nb[cc], L.x, rb + (1 - cc) * L.H + c.h, ci_of(cc, c.j, c.k0 + q), sy, sz);
            }
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                C v = (C)0;
                if (cd[cc] & SELF) v = bv[cc] - (dv[cc] * xv[cc] - nsum6<C>(nb[cc], cd[cc], edge));
                st(L.r + rb + cc * L.H + c.h, v);
            }
        }
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_residual(Lev<typename Pr::M> L) {
    pdl_wait();
    pdl_trigger();
    residual_body<Pr>(L);
}

// ---- CG (src/flip.jl:1033-1111) over the fine level's active tiles ----

// inner(s, z, r) after the V-cycle (src/flip.jl:1095-1096, 1105-1107): rho_new = z.r, then
// beta = rho_new / rho (0 on the first pass). The flexible form also sums z.q and takes
// the Polak-Ribiere beta = max(0, (rho_new - z.r_old) / rho) of the reference's flexible
// CG (src/sflip.jl:1896-1897); as r = r_old - alpha q, z.r_old = rho_new + alpha z.q, so
// no copy of r_old is kept.
template <class Pr>
__device__ __forceinline__ void dot_dev(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ r, const typename Pr::V* __restrict__ q,
          Scalars* sc, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_trigger();
    if (sc->s.done) return;
    const int sz = L.n1 * L.n2;
    double acc[2] = {0.0, 0.0};
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
        uint8_t cd[TZ][2];
        double zv[TZ][2], rv[TZ][2], qv[TZ][2];
#pragma unroll
        for (int qq = 0; qq < TZ; qq++)
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                cd[qq][cc] = 0;
                if (qq < c.kn) {
                    const int p = c.rb + qq * sz + cc * L.H + c.h;
                    cd[qq][cc] = L.code[p];
                    zv[qq][cc] = ld<double>(L.x + p);
                    rv[qq][cc] = (double)r[p];
                    if constexpr (Pr::flexible) qv[qq][cc] = (double)q[p];
                }
            }
#pragma unroll
        for (int qq = 0; qq < TZ; qq++)
#pragma unroll
            for (int cc = 0; cc < 2; cc++)
                if (cd[qq][cc] & SELF) {
                    acc[0] += zv[qq][cc] * rv[qq][cc];
                    if constexpr (Pr::flexible) acc[1] += zv[qq][cc] * qv[qq][cc];
                }
    }
    if (grid_sum<2>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        const double rho_new = rs<Pr>(acc[0]);
        if (!finite_d(rho_new)) {
            S.status = ST_NONFINITE;
            S.done = 1;
            return;
        }
        if constexpr (Pr::flexible) {
            if (!(rho_new > 0.0)) {  // src/sflip.jl:1880,1896
                S.status = ST_INDEFINITE;
                S.done = 1;
                return;
            }
            const double beta = S.it == 0 ? 0.0 : -S.alpha * acc[1] / S.rho;
            S.beta = beta > 0.0 ? beta : 0.0;
        } else {
            S.beta = S.it == 0 ? 0.0 : dv<Pr>(rho_new, S.rho);
        }
        S.rho = rho_new;
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_dot(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ r, const typename Pr::V* __restrict__ q,
          Scalars* sc, double* partials, unsigned* counter) {
    dot_dev<Pr>(L, r, q, sc, partials, counter);
}

// search_kernel! (src/flip.jl:1033-1054): p = z + beta d made where it is used, q = A p,
// and p.q; then alpha = rho / p.q (src/flip.jl:1100).
template <class Pr>
__device__ __forceinline__ void search_dev(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ diag,
             typename Pr::V* __restrict__ q, Scalars* sc, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    if (sc->s.done) return;
    const C beta = (C)sc->s.beta;
    const bool first = sc->s.beta == 0.0;
    const int sy = L.n1, sz = L.n1 * L.n2;
    double acc[1] = {0.0};
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int qq = 0; qq < TZ; qq++) {
            if (qq >= c.kn) break;
            const int rb = c.rb + qq * sz;
            uint8_t cd[2];
            C zn[2][6], dn[2][6], zc[2], dc[2], gv[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = rb + cc * L.H + c.h, o = rb + (1 - cc) * L.H + c.h, ci = ci_of(cc, c.j, c.k0 + qq);
                cd[cc] = L.code[p];
                gv[cc] = (C)diag[p];
                zc[cc] = ld<C>(L.x + p);
                load6<C>(zn[cc], L.x, o, ci, sy, sz);
                if (!first) {
                    dc[cc] = (C)dvec[p];
                    load6<C>(dn[cc], dvec, o, ci, sy, sz);
                }
            }
            C qv[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                qv[cc] = (C)0;
                if (cd[cc] & SELF) {
                    const C pc = first ? zc[cc] : zc[cc] + beta * dc[cc];
                    C a = (C)0;
#pragma unroll
                    for (int m = 0; m < 6; m++)
                        if (cd[cc] & (1u << m)) a += first ? zn[cc][m] : zn[cc][m] + beta * dn[cc][m];
                    qv[cc] = gv[cc] * pc - a;
                    acc[0] += (double)pc * (double)qv[cc];
                }
            }
            st(q + rb + c.h, qv[0]);
            st(q + rb + L.H + c.h, qv[1]);
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        S.pq = rs<Pr>(acc[0]);
        if (!finite_d(S.pq)) {
            S.status = ST_NONFINITE;
            S.done = 1;
        } else if (!(S.pq > 0.0)) {  // src/sflip.jl:1876-1877
            S.status = ST_INDEFINITE;
            S.done = 1;
        } else {
            S.alpha = dv<Pr>(S.rho, S.pq);
        }
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_search(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ diag,
             typename Pr::V* __restrict__ q, Scalars* sc, double* partials, unsigned* counter) {
    search_dev<Pr>(L, dvec, diag, q, sc, partials, counter);
}

// advance_kernel! (src/flip.jl:1059-1073): d = z + beta d; P += alpha d; r -= alpha q; then
// rnorm = sqrt(r.r) and the exit test rnorm <= tol |b| (src/flip.jl:1102-1103), or maxiter.
// The 16-bit forms also store the (scaled) r in the V-cycle's precision for its next pass.
template <class Pr>
__device__ __forceinline__ void advance_dev(Lev<typename Pr::M> L, typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ q,
              typename Pr::V* __restrict__ r, typename Pr::V* __restrict__ P, Scalars* sc, double* partials,
              unsigned* counter, cudaGraphConditionalHandle cond, int use_cond) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    if (sc->s.done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(cond, use_cond, 0);
        return;
    }
    const C beta = (C)sc->s.beta, alpha = (C)sc->s.alpha;
    const bool first = sc->s.beta == 0.0;
    const bool sep_b = (void*)L.b != (void*)r;
    const C rsc = (C)sc->s.rscale;
    const int sz = L.n1 * L.n2;
    double acc[1] = {0.0};
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int qq = 0; qq < TZ; qq++) {
            if (qq >= c.kn) break;
            const int rb = c.rb + qq * sz;
            uint8_t cd[2];
            C zv[2], dd[2], qv[2], rv[2], pv[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = rb + cc * L.H + c.h;
                const int pn = rb + 2 * c.h + ci_of(cc, c.j, c.k0 + qq);
                cd[cc] = L.code[p];
                zv[cc] = ld<C>(L.x + p);
                dd[cc] = (C)dvec[p];
                qv[cc] = (C)q[p];
                rv[cc] = (C)r[p];
                pv[cc] = (C)P[pn];
            }
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                if (!(cd[cc] & SELF)) continue;
                const int p = rb + cc * L.H + c.h;
                const int pn = rb + 2 * c.h + ci_of(cc, c.j, c.k0 + qq);
                const C pc = first ? zv[cc] : zv[cc] + beta * dd[cc];
                const C rl = rv[cc] - alpha * qv[cc];
                st(dvec + p, pc);
                st(P + pn, pv[cc] + alpha * pc);
                st(r + p, rl);
                if (sep_b) st(L.b + p, rl * rsc);
                acc[0] += (double)rl * (double)rl;
            }
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        S.it += 1;
        S.rnorm = sq<Pr>(acc[0]);
        S.rscale = next_rscale(S.rnorm, S.nliq);
        if (!finite_d(S.rnorm)) {
            S.status = ST_NONFINITE;
            S.done = 1;
        } else if (S.rnorm <= S.target) {
            S.status = ST_OK;
            S.done = 1;
        } else if (S.it >= sc->p.maxiter) {
            S.status = ST_NOT_CONVERGED;
            S.done = 1;
        }
        set_cond(cond, use_cond, !S.done);
    }
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_advance(Lev<typename Pr::M> L, typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ q,
              typename Pr::V* __restrict__ r, typename Pr::V* __restrict__ P, Scalars* sc, double* partials,
              unsigned* counter, cudaGraphConditionalHandle cond, int use_cond) {
    advance_dev<Pr>(L, dvec, q, r, P, sc, partials, counter, cond, use_cond);
}

// |b - A P| over the fine level: the true residual at exit (the reference's sparse
// solver checks it the same way, src/fgmres.jl:101-103). P is the caller's array
// (natural order, no guard), so its neighbour indices are clamped.
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_true_residual(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ b, const typename Pr::V* __restrict__ diag,
                    const typename Pr::V* __restrict__ P, typename Pr::V* __restrict__ rout, Scalars* sc,
                    double* partials, unsigned* counter) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    const int n1 = L.n1, sz = L.n1 * L.n2, N = L.n1 * L.n2 * L.n3;
    double acc[1] = {0.0};
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int qq = 0; qq < TZ; qq++) {
            if (qq >= c.kn) break;
            const int rb = c.rb + qq * sz;
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = rb + cc * L.H + c.h;
                const int pn = rb + 2 * c.h + ci_of(cc, c.j, c.k0 + qq);
                const uint8_t cd = L.code[p];
                const C bv = (C)b[p], gv = (C)diag[p], pc = (C)P[pn];
                C nb[6];
                nb[0] = (C)P[clampi(pn + 1, N)];
                nb[1] = (C)P[clampi(pn - 1, N)];
                nb[2] = (C)P[clampi(pn + n1, N)];
                nb[3] = (C)P[clampi(pn - n1, N)];
                nb[4] = (C)P[clampi(pn + sz, N)];
                nb[5] = (C)P[clampi(pn - sz, N)];
                if (!(cd & SELF)) continue;
                const C rv = bv - (gv * pc - sum6<C>(nb, cd));
                if (rout) st(rout + p, rv);
                acc[0] += (double)rv * (double)rv;
            }
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) sc->s.true_rr = acc[0];
}

// y = A x on the fine level (row-split, every cell of the active tiles; 0 off-liquid).
template <class Pr>
__global__ void __launch_bounds__(TPB) k_apply(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ x,
                                               const typename Pr::V* __restrict__ diag, typename Pr::V* __restrict__ y) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    const int sy = L.n1, sz = L.n1 * L.n2;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int qq = 0; qq < TZ; qq++) {
            if (qq >= c.kn) break;
            const int rb = c.rb + qq * sz;
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = rb + cc * L.H + c.h;
                const uint8_t cd = L.code[p];
                C nb[6];
                load6<C>(nb, x, rb + (1 - cc) * L.H + c.h, ci_of(cc, c.j, c.k0 + qq), sy, sz);
                const C v = (cd & SELF) ? (C)diag[p] * (C)x[p] - sum6<C>(nb, cd) : (C)0;
                st(y + p, v);
            }
        }
    }
}

}  // namespace mpp
