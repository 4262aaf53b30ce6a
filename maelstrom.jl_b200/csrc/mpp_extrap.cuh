// Velocity extrapolation after the projection: extrapolate! (src/flip.jl:1192-1206), its
// extrapolate_kernel! (:1161-1177) and unreached_kernel! (:1181-1184), and the solidify!
// (:801-806) it ends with. The three face arrays keep the caller's natural column-major
// layout (u (nx+1, ny, nz), v (nx, ny+1, nz), w (nx, ny, nz+1), i fastest), as the
// projection's gradient pass leaves them with their valid flags fu, fv, fw.
//
// The reference ping-pongs every face's value and flag through a scratch copy each layer
// (10 bytes a face a layer). Here the flags are bit masks, 32 faces of a row per word (rows
// padded to whole words): R_l, the faces valid after layer l (R_0: flagged on entry), and
// O, the faces that are not walled (the grid's geometry alone, built once per context). A
// layer is a bit dilation: D_l = (R_{l-1} moved one face along each of the six directions)
// & O & ~R_{l-1} are the faces it reaches, R_l = R_{l-1} | D_l (ping-pong masks). Only the
// faces of D_l load values: each takes the Float32 mean of its neighbours in R_{l-1},
// summed +x, -x, +y, -y, +z, -z, whose values are final (a value is written once, in the
// layer that reaches its face, and no face of D_l is in R_{l-1}). So every layer matches the
// reference's bit for bit, and moves a bit a face (the masks, which stay in L2) plus the
// values on the front. A last pass writes the 0/1 flags and zeroes what no layer reached
// and every walled face. One launch a pass covers all three arrays (blockIdx.y is the
// array); the flags are read and written a warp a mask word (32 faces of a row, coalesced),
// a layer takes a thread a mask word.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

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

constexpr int EXTRAP_MAX_LAYERS = 253;

// The three arrays, their masks (W words a row, rows in the arrays' row order) and dims.
struct ExtBits {
    float* x[3];
    uint8_t* f[3];
    uint32_t* open[3];  // O: in range and not walled
    uint32_t* ra[3];    // R, ping
    uint32_t* rb[3];    // R, pong
    int d[3][3];
    int W[3];
};

// Array ax's dims and masks, by selects.
struct ExtArr {
    int a1, a2, a3, W;
    unsigned nw;  // mask words
};
__device__ __forceinline__ ExtArr ext_arr(const ExtBits& E, int ax) {
    ExtArr a;
    a.a1 = pick3(ax, E.d[0][0], E.d[1][0], E.d[2][0]);
    a.a2 = pick3(ax, E.d[0][1], E.d[1][1], E.d[2][1]);
    a.a3 = pick3(ax, E.d[0][2], E.d[1][2], E.d[2][2]);
    a.W = pick3(ax, E.W[0], E.W[1], E.W[2]);
    a.nw = (unsigned)a.W * (unsigned)a.a2 * (unsigned)a.a3;
    return a;
}

// The open mask O (in range and not walled): the grid's geometry only, once per context.
// A thread a word.
__global__ void __launch_bounds__(TPB) k_extrap_open(Geo g, ExtBits E) {
    pdl_wait();
    pdl_trigger();
    const int ax = blockIdx.y;
    const ExtArr A = ext_arr(E, ax);
    uint32_t* O = pick3(ax, E.open[0], E.open[1], E.open[2]);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < A.nw; t += gridDim.x * blockDim.x) {
        const unsigned r = t / (unsigned)A.W;
        const int wx = (int)(t % (unsigned)A.W);
        const RowWall w = row_wall(g, ax, (int)(r % (unsigned)A.a2), (int)(r / (unsigned)A.a2));
        uint32_t o = 0;
        for (int b = 0; b < 32; b++) {
            const int i = 32 * wx + b;
            if (i < A.a1 && !walled_in_row(g, w, ax, i)) o |= 1u << b;
        }
        O[t] = o;
    }
}

// R_0 from the caller's flags (a face is valid when its flag is not 0): a warp takes EXT_WW
// consecutive words at a time, lane b reading face 32 wx + b of each (a 32-byte piece a word,
// the EXT_WW loads in flight together), each word formed by a ballot.
constexpr int EXT_WW = 8;
__global__ void __launch_bounds__(TPB) k_extrap_flags(ExtBits E) {
    pdl_wait();
    pdl_trigger();
    const int ax = blockIdx.y;
    const ExtArr A = ext_arr(E, ax);
    const uint8_t* fin = pick3(ax, E.f[0], E.f[1], E.f[2]);
    uint32_t* R = pick3(ax, E.ra[0], E.ra[1], E.ra[2]);
    const int lane = threadIdx.x & 31;
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    for (unsigned w0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * EXT_WW; w0 < A.nw;
         w0 += warps * EXT_WW) {
        bool f[EXT_WW];
#pragma unroll
        for (int q = 0; q < EXT_WW; q++) {
            const unsigned w = w0 + q;
            const unsigned r = w / (unsigned)A.W;
            const int i = 32 * (int)(w - r * (unsigned)A.W) + lane;
            f[q] = w < A.nw && i < A.a1 && fin[r * (unsigned)A.a1 + (unsigned)i] != 0;
        }
#pragma unroll
        for (int q = 0; q < EXT_WW; q++) {
            const uint32_t m = __ballot_sync(0xffffffffu, f[q]);
            if (lane == q && w0 + q < A.nw) R[w0 + q] = m;
        }
    }
}

// Layer `layer` (1-based): Rn = R | D, and the values of the faces D reaches. A thread a mask
// word; a word on the front takes its faces eight at a time (their loads before their
// stores). `from_a`: the layer reads ra and writes rb (else the other way round).
__global__ void __launch_bounds__(TPB) k_extrap_layer(ExtBits E, int from_a) {
    pdl_wait();
    pdl_trigger();
    const int ax = blockIdx.y;
    const ExtArr A = ext_arr(E, ax);
    const uint32_t* R = from_a ? pick3(ax, E.ra[0], E.ra[1], E.ra[2]) : pick3(ax, E.rb[0], E.rb[1], E.rb[2]);
    uint32_t* Rn = from_a ? pick3(ax, E.rb[0], E.rb[1], E.rb[2]) : pick3(ax, E.ra[0], E.ra[1], E.ra[2]);
    const uint32_t* O = pick3(ax, E.open[0], E.open[1], E.open[2]);
    float* x = pick3(ax, E.x[0], E.x[1], E.x[2]);
    const unsigned PY = (unsigned)A.W, PZ = (unsigned)A.W * (unsigned)A.a2;
    const unsigned s1 = (unsigned)A.a1, s2 = (unsigned)A.a1 * (unsigned)A.a2;
    for (unsigned w = blockIdx.x * blockDim.x + threadIdx.x; w < A.nw; w += gridDim.x * blockDim.x) {
        const unsigned r = w / (unsigned)A.W;
        const int wx = (int)(w % (unsigned)A.W);
        const int j = (int)(r % (unsigned)A.a2), k = (int)(r / (unsigned)A.a2);
        const uint32_t rc = R[w], o = O[w];
        const uint32_t rl = wx > 0 ? R[w - 1] : 0u, rr = wx + 1 < A.W ? R[w + 1] : 0u;
        const uint32_t ryp = j + 1 < A.a2 ? R[w + PY] : 0u, rym = j > 0 ? R[w - PY] : 0u;
        const uint32_t rzp = k + 1 < A.a3 ? R[w + PZ] : 0u, rzm = k > 0 ? R[w - PZ] : 0u;
        // neighbour validity, bit i of each: the face at +x, -x, +y, -y, +z, -z of face i
        const uint32_t vxp = (rc >> 1) | (rr << 31), vxm = (rc << 1) | (rl >> 31);
        uint32_t d = (vxp | vxm | ryp | rym | rzp | rzm) & o & ~rc;
        Rn[w] = rc | d;
        const unsigned base = r * s1 + 32u * (unsigned)wx;
        while (d) {
            int bits[8];
            int nb = 0;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                bits[q] = d ? __ffs(d) - 1 : -1;
                if (d) {
                    d &= d - 1;
                    nb++;
                }
            }
            float sum[8];
            int cnt[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                sum[q] = 0.f;
                cnt[q] = 0;
                if (q >= nb) continue;
                const int bit = bits[q];
                const unsigned id = base + (unsigned)bit;
                const bool take[6] = {((vxp >> bit) & 1u) != 0, ((vxm >> bit) & 1u) != 0, ((ryp >> bit) & 1u) != 0,
                                      ((rym >> bit) & 1u) != 0, ((rzp >> bit) & 1u) != 0, ((rzm >> bit) & 1u) != 0};
                const unsigned nbi[6] = {id + 1, id - 1, id + s1, id - s1, id + s2, id - s2};
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (take[e]) {
                        sum[q] = __fadd_rn(sum[q], x[nbi[e]]);
                        cnt[q]++;
                    }
            }
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (q < nb) x[base + (unsigned)bits[q]] = __fdiv_rn(sum[q], (float)cnt[q]);
        }
    }
}

// The last pass: zero every face not reached and every walled one, and write the reached
// flags (unless keep_flags: no layer ran, and the flags stay as they are). A warp takes
// EXT_WW consecutive mask words at a time, lane b on face 32 wx + b of each. `in_a`: the last
// layer's mask is ra (else rb).
__global__ void __launch_bounds__(TPB) k_extrap_final(ExtBits E, int in_a, int keep_flags) {
    pdl_wait();
    pdl_trigger();
    const int ax = blockIdx.y;
    const ExtArr A = ext_arr(E, ax);
    const uint32_t* R = in_a ? pick3(ax, E.ra[0], E.ra[1], E.ra[2]) : pick3(ax, E.rb[0], E.rb[1], E.rb[2]);
    const uint32_t* O = pick3(ax, E.open[0], E.open[1], E.open[2]);
    float* x = pick3(ax, E.x[0], E.x[1], E.x[2]);
    uint8_t* f = pick3(ax, E.f[0], E.f[1], E.f[2]);
    const int lane = threadIdx.x & 31;
    const unsigned warps = gridDim.x * (blockDim.x >> 5);
    for (unsigned w0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * EXT_WW; w0 < A.nw;
         w0 += warps * EXT_WW) {
        uint32_t rv[EXT_WW], ov[EXT_WW];
#pragma unroll
        for (int q = 0; q < EXT_WW; q++) {
            const bool in = w0 + q < A.nw;
            rv[q] = in ? R[w0 + q] : 0u;
            ov[q] = in ? O[w0 + q] : 0u;
        }
#pragma unroll
        for (int q = 0; q < EXT_WW; q++) {
            const unsigned w = w0 + q;
            const unsigned r = w / (unsigned)A.W;
            const int i = 32 * (int)(w - r * (unsigned)A.W) + lane;
            if (w >= A.nw || i >= A.a1) continue;
            const bool reached = (rv[q] >> lane) & 1u, open = (ov[q] >> lane) & 1u;
            const unsigned id = r * (unsigned)A.a1 + (unsigned)i;
            // unreached_kernel!, then solidify! (a walled face is zero, reached or not)
            if (!reached || !open) x[id] = 0.f;
            if (!keep_flags) f[id] = reached ? 1 : 0;
        }
    }
}

}  // namespace mpp
