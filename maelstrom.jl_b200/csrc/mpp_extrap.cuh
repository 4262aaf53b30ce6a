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
// zeroes what no layer reached and every walled face. One launch a layer covers all three
// arrays (blockIdx.y is the array); a block takes one row of faces at a time, so a face's
// (j, k) and its row's part of the solid test cost nothing per face.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

constexpr uint8_t UNREACHED = 0xFF;
constexpr int EXTRAP_MAX_LAYERS = 254;  // codes 1 .. 254; 255 is UNREACHED

struct ExtArrays {
    float* x[3];        // the caller's face values, updated in place
    uint8_t* f[3];      // the caller's flags
    uint8_t* reach[3];  // scratch reach codes
    int d[3][3];        // each array's dims
};

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

// Layer `layer` (1 .. EXTRAP_MAX_LAYERS). Layer 1 reads the caller's flags and writes every
// face's code; later layers read the codes and write those of the faces they reach.
__global__ void __launch_bounds__(TPB) k_extrap_layer(Geo g, ExtArrays E, int layer) {
    const int ax = blockIdx.y;
    const int a1 = pick3(ax, E.d[0][0], E.d[1][0], E.d[2][0]), a2 = pick3(ax, E.d[0][1], E.d[1][1], E.d[2][1]),
              a3 = pick3(ax, E.d[0][2], E.d[1][2], E.d[2][2]);
    const unsigned rows = (unsigned)a2 * (unsigned)a3, s1 = (unsigned)a1, s2 = (unsigned)a1 * (unsigned)a2;
    float* x = pick3(ax, E.x[0], E.x[1], E.x[2]);
    const uint8_t* fin = pick3(ax, E.f[0], E.f[1], E.f[2]);
    uint8_t* R = pick3(ax, E.reach[0], E.reach[1], E.reach[2]);
    const bool first = layer == 1;
    pdl_wait();
    pdl_trigger();
    for (unsigned r = blockIdx.x; r < rows; r += gridDim.x) {
        const int j = (int)(r % (unsigned)a2), k = (int)(r / (unsigned)a2);
        const RowWall w = row_wall(g, ax, j, k);
        const unsigned base = r * s1;
        for (int i = threadIdx.x; i < a1; i += blockDim.x) {
            const unsigned id = base + (unsigned)i;
            int rc = first ? (fin[id] ? 0 : UNREACHED) : R[id];
            if (rc == UNREACHED && !walled_in_row(g, w, ax, i)) {
                // the mean of the neighbours reached before this layer, in neighbour order
                // (+x, -x, +y, -y, +z, -z)
                float s = 0.f;
                int m = 0;
                auto take = [&](unsigned n) {
                    if (first ? fin[n] != 0 : (int)R[n] < layer) {
                        s = __fadd_rn(s, x[n]);
                        m++;
                    }
                };
                if (i + 1 < a1) take(id + 1);
                if (i > 0) take(id - 1);
                if (j + 1 < a2) take(id + s1);
                if (j > 0) take(id - s1);
                if (k + 1 < a3) take(id + s2);
                if (k > 0) take(id - s2);
                if (m > 0) {
                    x[id] = __fdiv_rn(s, (float)m);
                    rc = layer;
                }
            }
            if (first || rc == layer) R[id] = (uint8_t)rc;
        }
    }
}

// The last pass: zero every face no layer reached and every walled face, and write the
// reached flags. from_fin (no layer ran): reached means flagged on entry, and the flags stay
// as they are.
__global__ void __launch_bounds__(TPB) k_extrap_final(Geo g, ExtArrays E, int from_fin) {
    const int ax = blockIdx.y;
    const int a1 = pick3(ax, E.d[0][0], E.d[1][0], E.d[2][0]), a2 = pick3(ax, E.d[0][1], E.d[1][1], E.d[2][1]),
              a3 = pick3(ax, E.d[0][2], E.d[1][2], E.d[2][2]);
    const unsigned rows = (unsigned)a2 * (unsigned)a3, s1 = (unsigned)a1;
    float* x = pick3(ax, E.x[0], E.x[1], E.x[2]);
    uint8_t* f = pick3(ax, E.f[0], E.f[1], E.f[2]);
    const uint8_t* R = pick3(ax, E.reach[0], E.reach[1], E.reach[2]);
    pdl_wait();
    pdl_trigger();
    for (unsigned r = blockIdx.x; r < rows; r += gridDim.x) {
        const int j = (int)(r % (unsigned)a2), k = (int)(r / (unsigned)a2);
        const RowWall w = row_wall(g, ax, j, k);
        const unsigned base = r * s1;
        for (int i = threadIdx.x; i < a1; i += blockDim.x) {
            const unsigned id = base + (unsigned)i;
            const bool reached = from_fin ? f[id] != 0 : R[id] != UNREACHED;
            if (!reached || walled_in_row(g, w, ax, i)) x[id] = 0.f;
            if (!from_fin) f[id] = reached ? 1 : 0;
        }
    }
}

}  // namespace mpp
