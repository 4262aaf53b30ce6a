// The red-black smoother as a TMA pipeline (sm_100a).
//
// rbgs_kernel! (src/flip.jl:870-877) streams three arrays of its own colour (b, the
// diagonal, the stencil code) and the other colour's x with a one-cell halo. Issued as
// plain loads, each thread waits on a chain of dependent loads (tile id -> codes ->
// data) and HBM stays mostly idle. Here one thread per CTA moves whole tiles into shared
// memory with cp.async.bulk.tensor (into its own CTA only), S tiles ahead of the 256 threads that
// compute, so every SM keeps tens of kilobytes of loads in flight.
//
// Tensor maps view a row-split level array as 4-D (h, colour, j, k) with h innermost.
// Boxes: own colour {TH, 1, TY, TZ} at (TH th, c, TY tj, TZ tk); the other colour's x
// {TH + 2 PAD, 1, TY + 2, TZ + 2} at (TH th - PAD, 1 - c, TY tj - 1, TZ tk - 1), PAD = 16 bytes of
// elements so the innermost coordinate times the element size stays a multiple of 16
// bytes. Coordinates outside the array read as zero; the stencil code (also zero there)
// keeps them out of every sum.
#pragma once

#include <cuda.h>

#include "mpp_stream.cuh"

namespace mpp {

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// A wait that gives up: MBAR_SPINS polls of try_wait (each returns within a bounded,
// hardware-defined time), then false.
constexpr int MBAR_SPINS = 1 << 18;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int it = 0; it < MBAR_SPINS; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// The tensor maps of one row-split level.
struct TmaLev {
    CUtensorMap xh;    // x, box {TH + 2 PAD, 1, TY + 2, TZ + 2}
    CUtensorMap b;     // b, box {TH, 1, TY, TZ}
    CUtensorMap dg;    // smoother diagonal, box {TH, 1, TY, TZ}
    CUtensorMap code;  // stencil codes, box {TH, 1, TY, TZ}
};

template <class M>
struct TmaGeom {
    static constexpr int PAD = 16 / (int)sizeof(M);
    static constexpr int XW = TH + 2 * PAD;
    static constexpr int XB = XW * (TY + 2) * (TZ + 2) * (int)sizeof(M);
    static constexpr int BB = TH * TY * TZ * (int)sizeof(M);
    static constexpr int CB = TH * TY * TZ;
    static constexpr int up(int x) { return (x + 127) / 128 * 128; }
    static constexpr int OXB = 0, OBB = up(XB), ODB = OBB + up(BB), OCB = ODB + up(BB);
    static constexpr int STAGE = OCB + up(CB);
    static constexpr int STAGES = 4;
    static constexpr int SMEM = STAGES * STAGE + 128;  // + room to align the first stage
    static constexpr uint32_t TX = (uint32_t)(XB + 2 * BB + CB);
};

// rbgs_kernel! on one row-split level, tiles streamed by TMA. Grid: persistent, block b
// takes tiles b, b + G, b + 2G, ... of the level's active list. On a wait that times out
// the block records `fault`, waits (bounded) for the copies it still has in flight, and
// returns.
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs_tma(Lev<typename Pr::M> L, int colour, const __grid_constant__ TmaLev tm,
                                                  int* fault) {
    pdl_wait();
    pdl_trigger();
    using C = typename Pr::C;
    using M = typename Pr::M;
    using G = TmaGeom<M>;
    constexpr int S = G::STAGES;
    extern __shared__ __align__(128) unsigned char smraw[];
    // TMA destinations 128-byte aligned whatever the dynamic region's start (SMEM has room)
    unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t full[S];
    __shared__ uint32_t tid_of[S];
    const int n = *L.count;
    const int GB = gridDim.x;
    const int mine = n > (int)blockIdx.x ? (n - 1 - (int)blockIdx.x) / GB + 1 : 0;
    if (mine == 0) return;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int i) {  // thread 0 only
        const int s = i % S;
        const uint32_t tile = L.tiles[blockIdx.x + (size_t)i * GB];
        tid_of[s] = tile;
        const int h0 = (int)(tile & 1023u) * TH, j0 = (int)((tile >> 10) & 1023u) * TY, k0 = (int)(tile >> 20) * TZ;
        unsigned char* stg = sm + s * G::STAGE;
        mbar_expect_tx(&full[s], G::TX);
        tma_load_4d(stg + G::OXB, &tm.xh, &full[s], h0 - G::PAD, 1 - colour, j0 - 1, k0 - 1);
        tma_load_4d(stg + G::OBB, &tm.b, &full[s], h0, colour, j0, k0);
        tma_load_4d(stg + G::ODB, &tm.dg, &full[s], h0, colour, j0, k0);
        tma_load_4d(stg + G::OCB, &tm.code, &full[s], h0, colour, j0, k0);
    };
    int issued = 0;
    if (threadIdx.x == 0)
        for (; issued < S && issued < mine; issued++) issue(issued);
    const int lh = slot_h(), lj = slot_j(), lk = slot_k();
    const int xi = lh + G::PAD;  // this slot's column in the halo box
    const int H = L.H, sz = L.n1 * L.n2;
    int i = 0;
    bool bad = false;
    for (; i < mine; i++) {
        const int s = i % S;
        const bool ok = mbar_wait_bounded(&full[s], (uint32_t)((i / S) & 1));
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        const unsigned char* stg = sm + s * G::STAGE;
        const M* xh = reinterpret_cast<const M*>(stg + G::OXB);
        const M* bb = reinterpret_cast<const M*>(stg + G::OBB);
        const M* dd = reinterpret_cast<const M*>(stg + G::ODB);
        const uint8_t* cc = stg + G::OCB;
        const int own = (lk * TY + lj) * TH + lh;
        const uint8_t cd = cc[own];
        if (cd & SELF) {
            const uint32_t tile = tid_of[s];
            const int h = (int)(tile & 1023u) * TH + lh, j = (int)((tile >> 10) & 1023u) * TY + lj,
                      k = (int)(tile >> 20) * TZ + lk;
            const int ci = ci_of(colour, j, k);
            auto X = [&](int kk, int jj, int ii) { return ld<C>(xh + (kk * (TY + 2) + jj) * G::XW + ii); };
            C s2 = (C)0;
            if (cd & 1) s2 += X(lk + 1, lj + 1, xi + ci);
            if (cd & 2) s2 += X(lk + 1, lj + 1, xi + ci - 1);
            if (cd & 4) s2 += X(lk + 1, lj + 2, xi);
            if (cd & 8) s2 += X(lk + 1, lj, xi);
            if (cd & 16) s2 += X(lk + 2, lj + 1, xi);
            if (cd & 32) s2 += X(lk, lj + 1, xi);
            const C d = ld<C>(dd + own);  // the 16-bit forms' map holds the reciprocal
            C v;
            if constexpr (Pr::scaled) v = (ld<C>(bb + own) + s2) * d;
            else v = d > (C)0 ? (ld<C>(bb + own) + s2) / d : (C)0;
            st(L.x + (k * L.n2 + j) * L.n1 + colour * H + h, v);
        }
        __syncthreads();  // stage s fully read
        if (threadIdx.x == 0 && issued < mine) {
            fence_proxy_async_smem();
            issue(issued);
            issued++;
        }
    }
    if (bad) {
        if (threadIdx.x == 0) {
            atomicExch(fault, 1);
            // copies still in flight: tiles i .. i + S - 1 that were issued
            for (int q = i; q < issued; q++) mbar_wait_bounded(&full[q % S], (uint32_t)((q / S) & 1));
        }
        __syncthreads();
    }
    (void)sz;
}

// ---- the async-copy smoother (16-bit forms): rbgs_kernel! with every load in flight as
// cp.async into shared memory ----
// The vector form holds a tile's loads in registers, two tiles a warp, and at 16 warps an
// SM keeps too few bytes in flight to cover HBM latency. Here a warp streams its tiles
// through a ring of AS_STAGES buffers in its own slice of shared memory with 16-byte
// cp.async copies (no registers held while they fly): the own colour's b and reciprocal
// diagonal (one piece a lane) and the other colour's x around the tile (the 4 x 2 rows of
// the tile, the rows at -+y, the planes at -+z, and one piece each side along x: 96 pieces),
// AS_STAGES - 1 tiles ahead of the one it computes, in slots of exactly those 96 pieces. A lane then reads its 8 cells'
// neighbours from shared memory and updates them with the vector form's arithmetic
// (rbgs_tile), so both forms give the same values. Reads past the level's rows and planes
// land in the x array's zeroed guard, as the vector form's do.
constexpr int AS_STAGES = 4;
constexpr int AS_PIECES = 96;  // x pieces a tile needs
constexpr int AS_STAGE = AS_PIECES * 16 + 2 * 32 * 16;  // + b and 1/diag, a piece a lane
constexpr int AS_SMEM = (TPB / 32) * AS_STAGES * AS_STAGE;

// The e-th of a tile's 96 x pieces (slot e of a stage), as (plane kk, row jj, piece pc)
// around the tile (kk: planes k0-1 .. k0+2, jj: rows j0-1 .. j0+4, pc: pieces -1 .. 4): the
// tile's own rows (e < 32, e = the lane that owns the piece: 16 (kk-1) + 4 (jj-1) + pc-1),
// the rows at -+y, the planes at -+z, the pieces beside the rows along x.
__device__ __forceinline__ void as_piece(int e, int& kk, int& jj, int& pc) {
    if (e < 32) {
        kk = 1 + (e >> 4); jj = 1 + ((e >> 2) & 3); pc = 1 + (e & 3);
    } else if (e < 48) {
        e -= 32; kk = 1 + (e >> 3); jj = ((e >> 2) & 1) ? 5 : 0; pc = 1 + (e & 3);
    } else if (e < 80) {
        e -= 48; kk = (e >> 4) ? 3 : 0; jj = 1 + ((e >> 2) & 3); pc = 1 + (e & 3);
    } else {
        e -= 80; kk = 1 + (e >> 3); jj = 1 + ((e >> 1) & 3); pc = (e & 1) ? 5 : 0;
    }
}

template <class Pr>
__device__ __forceinline__ void rbgs_async_dev(Lev<typename Pr::M> L, int colour) {
    using C = typename Pr::C;
    using M = typename Pr::M;
    static_assert(sizeof(M) == 2, "the async form stages 8 elements a 16-byte piece");
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ uint32_t tid_of[TPB / 32][AS_STAGES];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = TPB / 32;
    const int hq = lane % V8_LANES_H, lj = (lane / V8_LANES_H) % TY, lk = lane / (V8_LANES_H * TY);
    unsigned char* ring = smraw + (size_t)warp * AS_STAGES * AS_STAGE;
    pdl_wait();
    pdl_trigger();
    const int n = *L.count;
    const bool edge = *L.edge != 0;
    const bool by_di = Pr::scaled && !edge, need_code = !by_di;
    const int stride = gridDim.x * wpb, wg = blockIdx.x * wpb + warp;
    const int mine = wg < n ? (n - 1 - wg) / stride + 1 : 0;
    if (mine == 0) return;
    const int H = L.H, n1 = L.n1, n2 = L.n2;
    const int own = colour * H, oth = (1 - colour) * H;
    const M* dsrc = Pr::scaled ? L.di : L.dg;
    // this lane's three x pieces, relative to the tile's corner: the same for every tile
    int pj[3], pk[3], poff[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        int kk, jj, pc;
        as_piece(lane + 32 * q, kk, jj, pc);
        pj[q] = jj - 1;
        pk[q] = kk - 1;
        poff[q] = (pk[q] * n2 + pj[q]) * n1 + (pc - 1) * V8;
    }
    auto issue = [&](int i) {
        const int s = i % AS_STAGES;
        const uint32_t tile = L.tiles[wg + i * stride];
        if (lane == 0) tid_of[warp][s] = tile;
        const int h0 = (int)(tile & 1023u) * TH, j0 = (int)((tile >> 10) & 1023u) * TY, k0 = (int)(tile >> 20) * TZ;
        unsigned char* st = ring + s * AS_STAGE;
        const int h = h0 + hq * V8, j = j0 + lj, k = k0 + lk;
        if (h < H && j < n2 && k < L.n3) {
            const int p = (k * n2 + j) * n1 + own + h;
            cp_async16(st + AS_PIECES * 16 + lane * 16, L.b + p);
            cp_async16(st + AS_PIECES * 16 + 512 + lane * 16, dsrc + p);
        }
        const int tbase = (k0 * n2 + j0) * n1 + oth + h0;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int jr = j0 + pj[q], kr = k0 + pk[q];
            // rows past the level's last (a partial tile's) are read by no cell that updates;
            // skipping them keeps every copy inside the array and its one-plane guard
            if (jr > n2 || (kr == L.n3 && jr >= n2)) continue;
            cp_async16(st + (lane + 32 * q) * 16, L.x + tbase + poff[q]);
        }
    };
#pragma unroll
    for (int i = 0; i < AS_STAGES - 1; i++) {
        if (i < mine) issue(i);
        cp_async_commit();
    }
    for (int i = 0; i < mine; i++) {
        if (i + AS_STAGES - 1 < mine) issue(i + AS_STAGES - 1);
        cp_async_commit();
        cp_async_wait<AS_STAGES - 1>();  // tile i's copies (this lane's) are in
        __syncwarp();                     // and every lane's
        const int s = i % AS_STAGES;
        const unsigned char* st = ring + s * AS_STAGE;
        const uint32_t tile = tid_of[warp][s];
        const int h = (int)(tile & 1023u) * TH + hq * V8, j = (int)((tile >> 10) & 1023u) * TY + lj,
                  k = (int)(tile >> 20) * TZ + lk;
        RbLd<M> a;
        a.ok = h < H && j < n2 && k < L.n3;
        if (a.ok) {
            a.p = (k * n2 + j) * n1 + own + h;
            a.ci = ci_of(colour, j, k);
            if (need_code) a.cdw = *reinterpret_cast<const uint2*>(L.code + a.p);
            auto piece = [&](int e) {
                Vec8<M> v;
                *reinterpret_cast<uint4*>(v.v) = *reinterpret_cast<const uint4*>(st + e * 16);
                return v;
            };
            // the lane's own piece is slot `lane`; its neighbours' are the adjacent lanes'
            // slots inside the tile, the halo slots at its edges
            *reinterpret_cast<uint4*>(a.bv.v) = *reinterpret_cast<const uint4*>(st + AS_PIECES * 16 + lane * 16);
            *reinterpret_cast<uint4*>(a.dv.v) =
                *reinterpret_cast<const uint4*>(st + AS_PIECES * 16 + 512 + lane * 16);
            a.xc = piece(lane);
            a.yp = piece(lj < TY - 1 ? lane + 4 : 32 + 8 * lk + 4 + hq);
            a.ym = piece(lj > 0 ? lane - 4 : 32 + 8 * lk + hq);
            a.zp = piece(lk == 0 ? lane + 16 : 64 + 4 * lj + hq);
            a.zm = piece(lk == 1 ? lane - 16 : 48 + 4 * lj + hq);
            a.xl = reinterpret_cast<const M*>(st + (hq > 0 ? lane - 1 : 80 + 8 * lk + 2 * lj) * 16)[V8 - 1];
            a.xr = reinterpret_cast<const M*>(st + (hq < V8_LANES_H - 1 ? lane + 1 : 81 + 8 * lk + 2 * lj) * 16)[0];
        }
        __syncwarp();  // stage s is read; the next iteration's copies may overwrite it
        if (a.ok) st8(L.x + a.p, rbgs_tile<C, M>(a, edge, Pr::scaled, by_di));
    }
    cp_async_wait<0>();
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs_async(Lev<typename Pr::M> L, int colour) {
    rbgs_async_dev<Pr>(L, colour);
}

}  // namespace mpp
