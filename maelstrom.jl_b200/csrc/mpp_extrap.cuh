// Velocity extrapolation after the projection: extrapolate! (src/flip.jl:1192-1206), its
// extrapolate_kernel! (:1161-1177) and unreached_kernel! (:1181-1184), and the solidify!
// (:801-806) it ends with. The three face arrays keep the caller's natural column-major
// layout (u (nx+1, ny, nz), v (nx, ny+1, nz), w (nx, ny, nz+1), i fastest), as the
// projection's gradient pass leaves them with their valid flags fu, fv, fw.
//
// One launch a layer covers all three arrays (blockIdx.y is the array), each ping-ponging
// between the caller's arrays and two scratch copies; the last layer also zeroes what no
// layer reached and every walled face, and writes into the caller's arrays, so the reference's
// copy-back, unreached and solidify passes cost no traffic of their own. A layer reads a
// face's value and flag and writes both (10 bytes a face); the neighbours' flags and values
// come from the same or adjacent rows and planes, through L1 and the 126 MB L2.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

struct ExtArrays {
    const float* src[3];
    const uint8_t* fin[3];
    float* dst[3];
    uint8_t* fout[3];
    int d[3][3];  // each array's dims
};

// walled (src/flip.jl:784-789): face (i, j, k) along `axis` (0-based) is the grid's own
// edge, or has a SOLID cell on either side (the cell before it along the axis, and the cell
// (i, j, k) after it).
__device__ __forceinline__ bool walled_face(const Geo& g, int i, int j, int k, int axis) {
    const int f = axis == 0 ? i : (axis == 1 ? j : k);
    if (f == 0 || f == g.n[axis]) return true;
    return issolidcell(g, i - (axis == 0), j - (axis == 1), k - (axis == 2)) || issolidcell(g, i, j, k);
}

// mode 0: one layer. 1: one layer, then zero where the face is unreached or walled (the last
// layer). 2: only that zeroing (layers = 0; may run in place: a thread reads and writes only
// its own face).
__global__ void __launch_bounds__(TPB) k_extrapolate(Geo g, ExtArrays E, int mode) {
    const int ax = blockIdx.y;
    const unsigned a1 = (unsigned)E.d[ax][0], a2 = (unsigned)E.d[ax][1], a3 = (unsigned)E.d[ax][2];
    const unsigned total = a1 * a2 * a3, s1 = a1, s2 = a1 * a2;
    const float* src = E.src[ax];
    const uint8_t* fin = E.fin[ax];
    float* dst = E.dst[ax];
    uint8_t* fout = E.fout[ax];
    pdl_wait();
    pdl_trigger();
    for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < total; id += gridDim.x * blockDim.x) {
        const unsigned i = id % a1, jk = id / a1, j = jk % a2, k = jk / a2;
        const uint8_t f0 = fin[id];
        float val = src[id];
        uint8_t fl = mode == 2 ? f0 : (f0 ? 1 : 0);  // with no layer the flags stay as they are
        if (mode != 2 && !f0 && !walled_face(g, (int)i, (int)j, (int)k, ax)) {
            // the flagged neighbours' mean, summed in neighbour order (+x, -x, +y, -y, +z, -z)
            float s = 0.f;
            int m = 0;
            if (i + 1 < a1 && fin[id + 1]) { s = __fadd_rn(s, src[id + 1]); m++; }
            if (i > 0 && fin[id - 1]) { s = __fadd_rn(s, src[id - 1]); m++; }
            if (j + 1 < a2 && fin[id + s1]) { s = __fadd_rn(s, src[id + s1]); m++; }
            if (j > 0 && fin[id - s1]) { s = __fadd_rn(s, src[id - s1]); m++; }
            if (k + 1 < a3 && fin[id + s2]) { s = __fadd_rn(s, src[id + s2]); m++; }
            if (k > 0 && fin[id - s2]) { s = __fadd_rn(s, src[id - s2]); m++; }
            if (m > 0) {
                val = __fdiv_rn(s, (float)m);
                fl = 1;
            }
        }
        if (mode != 0 && (!fl || walled_face(g, (int)i, (int)j, (int)k, ax))) val = 0.f;
        dst[id] = val;
        fout[id] = fl;
    }
}

}  // namespace mpp
