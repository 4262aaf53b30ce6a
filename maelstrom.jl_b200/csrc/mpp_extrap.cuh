// Velocity extrapolation after the projection: extrapolate! (src/flip.jl:1192-1206), its
// extrapolate_kernel! (:1161-1177) and unreached_kernel! (:1181-1184), and the solidify!
// (:801-806) it ends with. The three face arrays keep the caller's natural column-major
// layout (u (nx+1, ny, nz), v (nx, ny+1, nz), w (nx, ny, nz+1), i fastest), as the
// projection's gradient pass leaves them with their valid flags fu, fv, fw.
//
// The reference ping-pongs every face's value and flag through a scratch copy each layer
// (10 bytes a face a layer). Here a one-byte reach code a face replaces the copies: 0 for a
// face flagged on entry, l for a face first reached by layer l, UNREACHED otherwise. Layer l
// takes a face that is not yet reached and not walled to the mean of its neighbours whose
// code is below l, and writes its value in place: those neighbours' values are final (a
// value is written once, in the layer that reaches its face), and a face written in layer l
// is read by no other face in layer l (its code was UNREACHED and becomes l, neither below
// l). So each layer matches the reference's bit for bit, and moves about a byte a face (the
// codes) plus the values of the faces it reaches. A last pass writes the 0/1 flags and
// zeroes what no layer reached and every walled face. One launch a pass covers all three
// arrays (blockIdx.y is the array); a thread takes 16 consecutive faces of a row.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

constexpr uint8_t UNREACHED = 0xFF;

// walled (src/flip.jl:784-789) for the faces of one row (j, k) of the array along `ax`: the
// grid's own edge, or a SOLID cell on either side (issolidcell, src/flip.jl:64-66, with the
// row's y and z terms computed once: the same Float32 operations in the same order).
struct RowWall {
    bool edge;          // every face of the row is on the grid's edge
    float yyb, zb;      // the cell before the face: py*py and pz
    float yya, za;      // the cell after it
    int bi;             // the cell before is i - bi
};
__device__ __forceinline__ float cc_term(const Geo& g, int a, int i) {
    return g.lo[a] + ((float)i + 0.5f) * g.dx;
}
__device__ __forceinline__ RowWall row_wall(const Geo& g, int ax, int j, int k) {
    RowWall w;
    w.edge = (ax == 1 && (j == 0 || j == g.n[1])) || (ax == 2 && (k == 0 || k == g.n[2]));
    const float pya = cc_term(g, 1, j), pyb = cc_term(g, 1, ax == 1 ? j - 1 : j);
    w.yya = pya * pya;
    w.yyb = pyb * pyb;
    w.za = cc_term(g, 2, k);
    w.zb = cc_term(g, 2, ax == 2 ? k - 1 : k);
    w.bi = ax == 0 ? 1 : 0;
    return w;
}
__device__ __forceinline__ bool solid_in_row(const Geo& g, int i, float yy, float pz) {
    const float px = cc_term(g, 0, i);
    return px * px + yy > g.radius * g.radius || pz < g.floor_z;
}
__device__ __forceinline__ bool walled_in_row(const Geo& g, const RowWall& w, int ax, int i) {
    if (w.edge || (ax == 0 && (i == 0 || i == g.n[0]))) return true;
    return solid_in_row(g, i - w.bi, w.yyb, w.zb) || solid_in_row(g, i, w.yya, w.za);
}

// A field of array `ax` by selects, not by an indexed (local-memory) copy of the parameters.
template <class T>
__device__ __forceinline__ T pick3(int ax, T a, T b, T c) {
    return ax == 0 ? a : (ax == 1 ? b : c);
}

// The codes live in rows padded to a multiple of 16 bytes (pitch P), so a thread reads the
// codes of 16 consecutive faces of a row, and of the same 16 columns in the rows at -+y and
// -+z, as five 16-byte loads (one round trip), and loads values only for the faces it
// reaches. Padding reads as UNREACHED. A conversion pass writes the first codes: 0 for a
// face flagged on entry, WALLED for an unflagged walled face (never reached, so the layers
// skip the geometry), UNREACHED otherwise.
constexpr uint8_t WALLED = 0xFE;
constexpr int EXTRAP_MAX_LAYERS = 253;  // codes 1 .. 253
constexpr int EXT_CHUNK = 16;

struct ExtChunks {
    float* x[3];
    uint8_t* f[3];
    uint8_t* code[3];  // rows of `pitch[a]` bytes
    int d[3][3];
    int pitch[3];
};

struct Chunk {
    int ax, a1, a2, a3, P;
    unsigned r;  // row
    int j, k, i0;
};
__device__ __forceinline__ Chunk chunk_of(const ExtChunks& E, unsigned t) {
    Chunk c;
    c.ax = blockIdx.y;
    c.a1 = pick3(c.ax, E.d[0][0], E.d[1][0], E.d[2][0]);
    c.a2 = pick3(c.ax, E.d[0][1], E.d[1][1], E.d[2][1]);
    c.a3 = pick3(c.ax, E.d[0][2], E.d[1][2], E.d[2][2]);
    c.P = pick3(c.ax, E.pitch[0], E.pitch[1], E.pitch[2]);
    const unsigned cpr = (unsigned)c.P / EXT_CHUNK;
    c.r = t / cpr;
    c.i0 = (int)(t % cpr) * EXT_CHUNK;
    c.j = (int)(c.r % (unsigned)c.a2);
    c.k = (int)(c.r / (unsigned)c.a2);
    return c;
}
__device__ __forceinline__ unsigned chunk_threads(const ExtChunks& E, int ax) {
    const int a2 = pick3(ax, E.d[0][1], E.d[1][1], E.d[2][1]), a3 = pick3(ax, E.d[0][2], E.d[1][2], E.d[2][2]);
    const int P = pick3(ax, E.pitch[0], E.pitch[1], E.pitch[2]);
    return (unsigned)a2 * (unsigned)a3 * (unsigned)(P / EXT_CHUNK);
}
union Code16 {
    uint4 v;
    uint8_t b[16];
};

// The first codes, from the caller's flags.
__global__ void __launch_bounds__(TPB) k_extrap_codes(Geo g, ExtChunks E) {
    pdl_wait();
    pdl_trigger();
    const unsigned n = chunk_threads(E, blockIdx.y);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const Chunk c = chunk_of(E, t);
        const uint8_t* fin = pick3(c.ax, E.f[0], E.f[1], E.f[2]);
        uint8_t* R = pick3(c.ax, E.code[0], E.code[1], E.code[2]);
        const unsigned base = c.r * (unsigned)c.a1;
        uint8_t fl[EXT_CHUNK];
#pragma unroll
        for (int q = 0; q < EXT_CHUNK; q++) fl[q] = c.i0 + q < c.a1 ? fin[base + c.i0 + q] : (uint8_t)0;
        const RowWall w = row_wall(g, c.ax, c.j, c.k);
        Code16 out;
#pragma unroll
        for (int q = 0; q < EXT_CHUNK; q++) {
            const int i = c.i0 + q;
            out.b[q] = i >= c.a1 ? UNREACHED : (fl[q] ? (uint8_t)0 : (walled_in_row(g, w, c.ax, i) ? WALLED : UNREACHED));
        }
        *reinterpret_cast<uint4*>(R + c.r * (unsigned)c.P + c.i0) = out.v;
    }
}

// Layer `layer` (1 .. EXTRAP_MAX_LAYERS) on the codes.
__global__ void __launch_bounds__(TPB, 4) k_extrap_layer(ExtChunks E, int layer) {
    pdl_wait();
    pdl_trigger();
    const unsigned n = chunk_threads(E, blockIdx.y);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const Chunk c = chunk_of(E, t);
        uint8_t* R = pick3(c.ax, E.code[0], E.code[1], E.code[2]);
        float* x = pick3(c.ax, E.x[0], E.x[1], E.x[2]);
        const unsigned rowoff = c.r * (unsigned)c.P + (unsigned)c.i0;
        const unsigned P = (unsigned)c.P, PZ = (unsigned)c.P * (unsigned)c.a2;
        Code16 own, yp, ym, zp, zm;
        const uint4 none = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        own.v = *reinterpret_cast<const uint4*>(R + rowoff);
        yp.v = c.j + 1 < c.a2 ? *reinterpret_cast<const uint4*>(R + rowoff + P) : none;
        ym.v = c.j > 0 ? *reinterpret_cast<const uint4*>(R + rowoff - P) : none;
        zp.v = c.k + 1 < c.a3 ? *reinterpret_cast<const uint4*>(R + rowoff + PZ) : none;
        zm.v = c.k > 0 ? *reinterpret_cast<const uint4*>(R + rowoff - PZ) : none;
        const uint8_t left = c.i0 > 0 ? R[rowoff - 1] : UNREACHED;
        const uint8_t right = c.i0 + EXT_CHUNK < c.a1 ? R[rowoff + EXT_CHUNK] : UNREACHED;
        // the neighbours each face takes (reached before this layer), +x -x +y -y +z -z
        unsigned take[EXT_CHUNK];
        bool any = false;
#pragma unroll
        for (int q = 0; q < EXT_CHUNK; q++) {
            take[q] = 0;
            if (own.b[q] == UNREACHED) {  // padding is UNREACHED too, but has no reached neighbour
                const uint8_t nb[6] = {q + 1 < EXT_CHUNK ? own.b[q + 1] : right, q > 0 ? own.b[q - 1] : left,
                                       yp.b[q], ym.b[q], zp.b[q], zm.b[q]};
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if ((int)nb[e] < layer) take[q] |= 1u << e;
                if (c.i0 + q >= c.a1) take[q] = 0;
                any = any || take[q] != 0;
            }
        }
        if (!any) continue;
        const unsigned s1 = (unsigned)c.a1, s2 = (unsigned)c.a1 * (unsigned)c.a2;
        const unsigned base = c.r * s1 + (unsigned)c.i0;
        // the taken values, eight faces' loads at a time before their stores
#pragma unroll
        for (int h = 0; h < EXT_CHUNK; h += 8) {
            float sum[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const unsigned id = base + h + q;
                const unsigned nbi[6] = {id + 1, id - 1, id + s1, id - s1, id + s2, id - s2};
                sum[q] = 0.f;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (take[h + q] & (1u << e)) sum[q] = __fadd_rn(sum[q], x[nbi[e]]);
            }
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (take[h + q]) {
                    x[base + h + q] = __fdiv_rn(sum[q], (float)__popc(take[h + q]));
                    own.b[h + q] = (uint8_t)layer;
                }
        }
        *reinterpret_cast<uint4*>(R + rowoff) = own.v;
    }
}

// The last pass on the codes: zero every face not reached and every walled one, and write
// the reached flags (unless keep_flags: no layer ran, and the flags stay as they are).
__global__ void __launch_bounds__(TPB) k_extrap_final(Geo g, ExtChunks E, int keep_flags) {
    pdl_wait();
    pdl_trigger();
    const unsigned n = chunk_threads(E, blockIdx.y);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const Chunk c = chunk_of(E, t);
        const uint8_t* R = pick3(c.ax, E.code[0], E.code[1], E.code[2]);
        float* x = pick3(c.ax, E.x[0], E.x[1], E.x[2]);
        uint8_t* f = pick3(c.ax, E.f[0], E.f[1], E.f[2]);
        Code16 own;
        own.v = *reinterpret_cast<const uint4*>(R + c.r * (unsigned)c.P + c.i0);
        const RowWall w = row_wall(g, c.ax, c.j, c.k);
        const unsigned base = c.r * (unsigned)c.a1 + (unsigned)c.i0;
#pragma unroll
        for (int q = 0; q < EXT_CHUNK; q++) {
            const int i = c.i0 + q;
            if (i >= c.a1) continue;
            const uint8_t cd = own.b[q];
            const bool reached = cd < WALLED;
            // only a face flagged on entry (code 0) can be both reached and walled
            if (!reached || (cd == 0 && walled_in_row(g, w, c.ax, i))) x[base + q] = 0.f;
            if (!keep_flags) f[base + q] = reached ? 1 : 0;
        }
    }
}

}  // namespace mpp
