// Shared device definitions of libmpp: cell classes, the internal layout, precision
// bundles, conversions and deterministic block reductions.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace mpp {

// Cell classes, as the reference's SOLID/LIQUID/AIR (src/flip.jl:24-26).
constexpr uint8_t SOLID = 0, LIQUID = 1, AIR = 2;

// Per-cell stencil code (internal): bit m (m = 0..5 for +x,-x,+y,-y,+z,-z, the order of
// `neighbour`, src/flip.jl:84-92) is set when that neighbour is LIQUID; SELF when the
// cell itself is. A cell whose code lacks SELF is never updated and never read.
constexpr uint8_t SELF = 1u << 6;

// Tiles: 32 (h) x 4 (j) x 2 (k) slots of 2 cells each (one per colour), so a tile is a
// 64 x 4 x 2 block of cells; 256 threads, one slot each; a warp reads one row's 32
// consecutive same-colour values (64-128 bytes).
#ifndef MPP_TILE_H
#define MPP_TILE_H 32
#define MPP_TILE_Y 4
#define MPP_TILE_Z 2
#endif
constexpr int TH = MPP_TILE_H, TY = MPP_TILE_Y, TZ = MPP_TILE_Z, TPB = 256;
static_assert(TY % 2 == 0 && TZ % 2 == 0, "prolongation maps a tile's rows and planes onto whole coarse ones");
static_assert(TH * TY * TZ == TPB, "one thread per tile slot");

// Grid-wide sums: at most MAXK values per block, at most MAXBLOCKS_PER_SM blocks per SM
// (the partial-sum buffer holds MAXK * MAXBLOCKS_PER_SM * SMs doubles).
constexpr int MAXK = 4, MAXBLOCKS_PER_SM = 8;

// Precision bundles. V: the CG vectors and the fine operator; M: the V-cycle's storage;
// C: stencil arithmetic; CC: the coarsest solve.
struct PrecFP32 {
    using V = float; using M = float; using C = float; using CC = float;
    static constexpr bool flexible = false;  // standard PCG, beta = rho_new / rho
    static constexpr bool f32_scalars = true;  // scalars rounded to Float32 like the reference
    static constexpr bool scaled = false;      // coarse levels hold the reference's values
};
struct PrecFP16 {
    using V = float; using M = __half; using C = float; using CC = double;
    static constexpr bool flexible = true;  // Polak-Ribiere flexible PCG
    static constexpr bool f32_scalars = false;
    // 16-bit storage: level l holds 4^-l times the reference's b and x (restriction
    // without its factor 4, prolongation with it; exact power-of-two scalings), and the
    // fine residual handed to the V-cycle is scaled by a power of two, so values stay
    // in FP16's range as the residual falls. CG is invariant to both.
    static constexpr bool scaled = true;
};
struct PrecBF16 {
    using V = float; using M = __nv_bfloat16; using C = float; using CC = double;
    static constexpr bool flexible = true;
    static constexpr bool f32_scalars = false;
    static constexpr bool scaled = true;
};
struct PrecFP64 {
    using V = double; using M = double; using C = double; using CC = double;
    static constexpr bool flexible = false;
    static constexpr bool f32_scalars = false;
    static constexpr bool scaled = false;
};

template <class C, class T>
__device__ __forceinline__ C ld(const T* p) {
    if constexpr (std::is_same<T, __half>::value) return (C)__half2float(*p);
    else if constexpr (std::is_same<T, __nv_bfloat16>::value) return (C)__bfloat162float(*p);
    else return (C)(*p);
}
template <class T, class C>
__device__ __forceinline__ void st(T* p, C v) {
    if constexpr (std::is_same<T, __half>::value) *p = __float2half_rn((float)v);
    else if constexpr (std::is_same<T, __nv_bfloat16>::value) *p = __float2bfloat16_rn((float)v);
    else *p = (T)v;
}

// acc + w x, a term of the V-cycle's transfer sums (restriction, prolongation): FUSE (the
// 16-bit storage forms) rounds once (a fused multiply-add), otherwise the product and the
// sum round separately, as in the reference's Float32 arithmetic. A zero term leaves acc
// unchanged either way, so sums that leave out zero terms agree with ones that add them.
template <bool FUSE, class C>
__device__ __forceinline__ C macc(C acc, C w, C x) {
    if constexpr (FUSE) return fmaf(w, x, acc);
    else return acc + w * x;
}

// c + a for a stored value a and an arithmetic value c: for the 16-bit storage forms one
// mixed-precision add (PTX add.rn.f32.f16 / .bf16: a is widened exactly inside the add,
// which rounds once), the same bits as widening a first and adding in FP32, in one
// instruction instead of two.
template <class C, class T>
__device__ __forceinline__ C addm(T a, C c) {
    if constexpr (std::is_same<T, __half>::value && std::is_same<C, float>::value) {
        float d;
        asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(__half_as_ushort(a)), "f"(c));
        return d;
    } else if constexpr (std::is_same<T, __nv_bfloat16>::value && std::is_same<C, float>::value) {
        float d;
        asm("add.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(__bfloat16_as_ushort(a)), "f"(c));
        return d;
    } else {
        return ld<C>(&a) + c;
    }
}

// theta (src/flip.jl:113): the free surface's fraction of the way from a liquid cell
// centre to an air one, clamp(phi_i / (phi_i - phi_j), 0.01, 1) in Julia's clamp order.
template <class C>
__device__ __forceinline__ C theta(C pi, C pj) {
    C t = pi / (pi - pj);
    return t > (C)1 ? (C)1 : (t < (C)0.01f ? (C)0.01f : t);
}

// Walk an n1 x n2 x n3 box row by row: blocks stride over the rows (j, k), a block's
// threads over i. The row's (j, k) is one 32-bit division per row, not three 64-bit ones
// per cell, and a warp's cells are consecutive.
#define FOR_CELLS(n1, n2, n3, i, j, k, idx)                                                     \
    for (int r_ = (int)blockIdx.x, nr_ = (n2) * (n3); r_ < nr_; r_ += (int)gridDim.x)           \
        for (int i = (int)threadIdx.x, j = r_ % (n2), k = r_ / (n2); i < (n1); i += (int)blockDim.x) \
            if (const int64_t idx = (int64_t)r_ * (n1) + i; true)

// One multigrid level as the kernels see it. Levels other than the coarsest are stored
// row-split: each x-row of n1 cells holds its colour-0 cells (in i order) and then its
// colour-1 cells, so cell (i,j,k) sits at row(j,k) + colour*H + i/2 with
// colour = (i+j+k+1) & 1 (the reference's 1-based (i+j+k) % 2) and H = n1/2. A
// red-black half-sweep then reads and writes only contiguous runs of its own colour.
// The coarsest level is stored in natural order (i + n1*(j + n2*k)).
template <class M>
struct Lev {
    int n1, n2, n3, H;
    int GH, GJ, GK;  // tile grid
    uint8_t* code;   // split
    M* dg;           // diagonal used by the smoother (split)
    M* x;            // correction
    M* b;            // right-hand side
    M* r;            // residual
    uint8_t* types;  // natural order (coarse levels)
    uint8_t* dc;     // non-SOLID neighbour counts (bottom levels, natural order; their code is natural too)
    uint8_t* tflag;  // per-tile "has liquid" flags
    uint32_t* tiles; // active tile list
    int* count;      // its length (device)
    M* di;           // 1/diagonal (0 off-liquid) for the 16-bit forms' smoother, else null (split)
    int* edge;       // nonzero when a LIQUID cell lies on the level's x or y faces (device)

    __device__ __forceinline__ int64_t row(int j, int k) const { return ((int64_t)k * n2 + j) * n1; }
    __device__ __forceinline__ int64_t pos(int i, int j, int k) const {
        return row(j, k) + (int64_t)(((i + j + k + 1) & 1) * H + (i >> 1));
    }
    __device__ __forceinline__ int64_t nat(int i, int j, int k) const {
        return (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k);
    }
    __device__ __forceinline__ int tile_of(int i, int j, int k) const {
        return (i >> 1) / TH + GH * (j / TY + GJ * (k / TZ));
    }
};

// Programmatic dependent launch. Kernels are launched so that the next one may start while
// the previous one drains; pdl_wait() (first thing in every kernel) blocks until the
// previous kernel has completed and its writes are visible, and pdl_trigger() (after a
// block's main work) lets the next kernel's blocks start launching. Both are no-ops in a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Asynchronous 16-byte copies global -> shared (cp.async, L2 only), committed and waited on
// in groups. The zero-filling form copies `bytes` (0 or 16) and fills the rest with zeros.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void* sm, const void* gm) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sm)), "l"(gm) : "memory");
}
__device__ __forceinline__ void cp_async16_zfill(void* sm, const void* gm, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(sm)), "l"(gm), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A thread's slot in a tile (256 threads, one per slot): column h, row j, plane k offsets.
// A warp covers TH consecutive columns of one row.
__device__ __forceinline__ int slot_h() { return (int)threadIdx.x % TH; }
__device__ __forceinline__ int slot_j() { return ((int)threadIdx.x / TH) % TY; }
__device__ __forceinline__ int slot_k() { return (int)threadIdx.x / (TH * TY); }

// ---- deterministic reductions ----
// Block sums of K doubles (256 threads); the result is valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
    __shared__ double ws[K][TPB / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; q++) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) ws[q][w] = a;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) {
            double a = lane < (int)(blockDim.x >> 5) ? ws[q][lane] : 0.0;  // blocks of <= TPB threads
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
            v[q] = a;
        }
    }
    __syncthreads();
}

// Each block stores its K partial sums; the last block to finish adds all partials in
// block order (fixed, so the result does not depend on scheduling), resets the counter
// and returns true with the totals in thread 0's v.
template <int K>
__device__ __forceinline__ bool grid_sum(double (&v)[K], double* partials, unsigned* counter) {
    static_assert(K <= MAXK, "partial-sum buffer holds MAXK values per block");
    block_sum<K>(v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; q++) partials[(size_t)blockIdx.x * K + q] = v[q];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s[K];
#pragma unroll
    for (int q = 0; q < K; q++) s[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < K; q++) s[q] += __ldcg(partials + (size_t)b * K + q);
    }
    block_sum<K>(s);
    if (threadIdx.x == 0) {
        *counter = 0u;
#pragma unroll
        for (int q = 0; q < K; q++) v[q] = s[q];
    }
    return true;
}

}  // namespace mpp
