// Semi-Lagrangian advection (advect_kernel!, src/flip.jl:357-369; trilinear,
// src/interpolation.jl:4-17; nodepos/indexspace/velocity, src/flip.jl:76-81) and its
// adjoint, for rollouts of advection + projection.
//
// Forward, per sample node of an array (face arrays u, v, w at UOFF/VOFF/WOFF, the level
// set at COFF): p = the node's position; m = clamp(ceil(|V(p)| dt / dx), 1, 32) RK2
// sub-steps of h = dt/m, each p -= h V(p - h/2 V(p)); out = trilinear(src, p). Float32
// throughout in the reference's operation order (the library is built without FMA
// contraction, so results are bit-exact with a C restatement).
//
// Adjoint: the trajectory is recomputed from the step's velocity (the rollout keeps one
// checkpoint per step) and walked back: the cotangent of `out` goes to src's 8 corners
// and, through the trilinear gradient, to the final position; each sub-step passes it to
// the velocity samples' corners and back to the previous position. The sub-step count
// is piecewise constant (no derivative); a clamp passes the derivative on its closed
// range. Corner cotangents are accumulated with FP64 atomics, then rounded once.
#pragma once

#include "mpp_common.cuh"

namespace mpp {

// The three face arrays as velocity sources, and the sampled arrays of one launch.
struct Flow {
    const float* f[3];
    int d[3][3];
    float lo[3], dx;
};
struct AdvArrays {
    float* out[4];
    const float* src[4];
    int d[4][3];
    float off[4][3];
    int64_t n[4];
};

struct Tri {
    int64_t b;         // corner (i, j, k)
    int sy, sz;        // strides of +j, +k
    float fx, fy, fz;  // fractions
    bool in[3];        // coordinate inside the array (derivative passes)
};

__device__ __forceinline__ float clampf(float x, float hi) { return x > hi ? hi : (x < 0.f ? 0.f : x); }

// trilinear(A, q) (src/interpolation.jl:4-17): the corner and fractions of q.
__device__ __forceinline__ Tri tri_at(const int d[3], float qx, float qy, float qz) {
    Tri t;
    const float x = clampf(qx, (float)(d[0] - 1)), y = clampf(qy, (float)(d[1] - 1)), z = clampf(qz, (float)(d[2] - 1));
    int i = (int)x, j = (int)y, k = (int)z;
    i = i > d[0] - 2 ? d[0] - 2 : i;
    j = j > d[1] - 2 ? d[1] - 2 : j;
    k = k > d[2] - 2 ? d[2] - 2 : k;
    t.fx = x - (float)i;
    t.fy = y - (float)j;
    t.fz = z - (float)k;
    t.sy = d[0];
    t.sz = d[0] * d[1];
    t.b = (int64_t)i + (int64_t)d[0] * ((int64_t)j + (int64_t)d[1] * k);
    t.in[0] = qx >= 0.f && qx <= (float)(d[0] - 1);
    t.in[1] = qy >= 0.f && qy <= (float)(d[1] - 1);
    t.in[2] = qz >= 0.f && qz <= (float)(d[2] - 1);
    return t;
}

__device__ __forceinline__ float tri_val(const float* __restrict__ A, const Tri& t) {
    const float* a = A + t.b;
    const float gx = 1.f - t.fx;
    const float c00 = a[0] * gx + a[1] * t.fx;
    const float c10 = a[t.sy] * gx + a[t.sy + 1] * t.fx;
    const float c01 = a[t.sz] * gx + a[t.sz + 1] * t.fx;
    const float c11 = a[t.sz + t.sy] * gx + a[t.sz + t.sy + 1] * t.fx;
    return (c00 * (1.f - t.fy) + c10 * t.fy) * (1.f - t.fz) + (c01 * (1.f - t.fy) + c11 * t.fy) * t.fz;
}

// d trilinear / d q (zero along an axis whose coordinate lies outside the array).
__device__ __forceinline__ void tri_grad(const float* __restrict__ A, const Tri& t, float g[3]) {
    const float* a = A + t.b;
    const float gx = 1.f - t.fx, gy = 1.f - t.fy, gz = 1.f - t.fz;
    const float c00 = a[0] * gx + a[1] * t.fx;
    const float c10 = a[t.sy] * gx + a[t.sy + 1] * t.fx;
    const float c01 = a[t.sz] * gx + a[t.sz + 1] * t.fx;
    const float c11 = a[t.sz + t.sy] * gx + a[t.sz + t.sy + 1] * t.fx;
    const float dx = ((a[1] - a[0]) * gy + (a[t.sy + 1] - a[t.sy]) * t.fy) * gz +
                     ((a[t.sz + 1] - a[t.sz]) * gy + (a[t.sz + t.sy + 1] - a[t.sz + t.sy]) * t.fy) * t.fz;
    const float dy = (c10 - c00) * gz + (c11 - c01) * t.fz;
    const float dz = (c01 * gy + c11 * t.fy) - (c00 * gy + c10 * t.fy);
    g[0] = t.in[0] ? dx : 0.f;
    g[1] = t.in[1] ? dy : 0.f;
    g[2] = t.in[2] ? dz : 0.f;
}

// Add c * (the 8 trilinear weights) into acc at the corners.
__device__ __forceinline__ void tri_scatter(double* __restrict__ acc, const Tri& t, float c) {
    if (c == 0.f) return;
    const float gx = 1.f - t.fx, gy = 1.f - t.fy, gz = 1.f - t.fz;
    double* a = acc + t.b;
    atomicAdd(a, (double)(c * (gx * gy * gz)));
    atomicAdd(a + 1, (double)(c * (t.fx * gy * gz)));
    atomicAdd(a + t.sy, (double)(c * (gx * t.fy * gz)));
    atomicAdd(a + t.sy + 1, (double)(c * (t.fx * t.fy * gz)));
    atomicAdd(a + t.sz, (double)(c * (gx * gy * t.fz)));
    atomicAdd(a + t.sz + 1, (double)(c * (t.fx * gy * t.fz)));
    atomicAdd(a + t.sz + t.sy, (double)(c * (gx * t.fy * t.fz)));
    atomicAdd(a + t.sz + t.sy + 1, (double)(c * (t.fx * t.fy * t.fz)));
}

// indexspace(g, p, off) (src/flip.jl:77) for velocity component c.
__device__ __forceinline__ Tri flow_tri(const Flow& fl, int c, const float p[3]) {
    const float q0 = (p[0] - fl.lo[0]) / fl.dx - (c == 0 ? 0.f : 0.5f);
    const float q1 = (p[1] - fl.lo[1]) / fl.dx - (c == 1 ? 0.f : 0.5f);
    const float q2 = (p[2] - fl.lo[2]) / fl.dx - (c == 2 ? 0.f : 0.5f);
    return tri_at(fl.d[c], q0, q1, q2);
}

// velocity(u, v, w, g, p) (src/flip.jl:80-81).
__device__ __forceinline__ void flow_vel(const Flow& fl, const float p[3], float v[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) v[c] = tri_val(fl.f[c], flow_tri(fl, c, p));
}

// substeps (src/flip.jl:372).
__device__ __forceinline__ int substeps(float cells) {
    const float c = ceilf(cells);
    if (!(c >= 1.f)) return 1;
    return c > 32.f ? 32 : (int)c;
}

__device__ __forceinline__ void node_pos(const AdvArrays& A, int a, int64_t idx, const Flow& fl, float p[3]) {
    const int i = (int)(idx % A.d[a][0]), j = (int)((idx / A.d[a][0]) % A.d[a][1]);
    const int k = (int)(idx / ((int64_t)A.d[a][0] * A.d[a][1]));
    p[0] = fl.lo[0] + ((float)i + A.off[a][0]) * fl.dx;
    p[1] = fl.lo[1] + ((float)j + A.off[a][1]) * fl.dx;
    p[2] = fl.lo[2] + ((float)k + A.off[a][2]) * fl.dx;
}

__device__ __forceinline__ int node_steps(const Flow& fl, const float p[3], float dt) {
    float v[3];
    flow_vel(fl, p, v);
    return substeps(sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * dt / fl.dx);
}

// Forward: blockIdx.y picks the array.
__global__ void __launch_bounds__(TPB) k_advect(Flow fl, AdvArrays A, float dt) {
    pdl_wait();
    pdl_trigger();
    const int a = blockIdx.y;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < A.n[a]; idx += (int64_t)gridDim.x * TPB) {
        float p[3];
        node_pos(A, a, idx, fl, p);
        const int m = node_steps(fl, p, dt);
        const float h = dt / (float)m, hh = 0.5f * h;
        for (int s = 0; s < m; s++) {
            float v1[3], pm[3], v2[3];
            flow_vel(fl, p, v1);
#pragma unroll
            for (int c = 0; c < 3; c++) pm[c] = p[c] - hh * v1[c];
            flow_vel(fl, pm, v2);
#pragma unroll
            for (int c = 0; c < 3; c++) p[c] = p[c] - h * v2[c];
        }
        const Tri t = tri_at(A.d[a], (p[0] - fl.lo[0]) / fl.dx - A.off[a][0], (p[1] - fl.lo[1]) / fl.dx - A.off[a][1],
                             (p[2] - fl.lo[2]) / fl.dx - A.off[a][2]);
        A.out[a][idx] = tri_val(A.src[a], t);
    }
}

// Adjoint: A.out[a] holds the cotangent of array a's output (read), acc_src[a] gets
// d/d src and acc_flow[c] d/d (u, v, w)[c] (FP64 accumulators, zeroed by the caller;
// they may be the same arrays when src is the flow itself).
struct AdvAcc {
    double* src[4];
    double* flow[3];
};
constexpr int ADV_MAXSTEPS = 32;

__global__ void __launch_bounds__(128) k_advect_vjp(Flow fl, AdvArrays A, AdvAcc acc, float dt) {
    pdl_wait();
    pdl_trigger();
    const int a = blockIdx.y;
    for (int64_t idx = (int64_t)blockIdx.x * 128 + threadIdx.x; idx < A.n[a]; idx += (int64_t)gridDim.x * 128) {
        const float go = A.out[a][idx];
        if (go == 0.f) continue;
        float ps[ADV_MAXSTEPS + 1][3], pms[ADV_MAXSTEPS][3];
        node_pos(A, a, idx, fl, ps[0]);
        const int m = node_steps(fl, ps[0], dt);
        const float h = dt / (float)m, hh = 0.5f * h;
        for (int s = 0; s < m; s++) {
            float v1[3], v2[3];
            flow_vel(fl, ps[s], v1);
#pragma unroll
            for (int c = 0; c < 3; c++) pms[s][c] = ps[s][c] - hh * v1[c];
            flow_vel(fl, pms[s], v2);
#pragma unroll
            for (int c = 0; c < 3; c++) ps[s + 1][c] = ps[s][c] - h * v2[c];
        }
        const Tri t = tri_at(A.d[a], (ps[m][0] - fl.lo[0]) / fl.dx - A.off[a][0],
                             (ps[m][1] - fl.lo[1]) / fl.dx - A.off[a][1], (ps[m][2] - fl.lo[2]) / fl.dx - A.off[a][2]);
        tri_scatter(acc.src[a], t, go);
        float pb[3], gq[3];
        tri_grad(A.src[a], t, gq);
#pragma unroll
        for (int c = 0; c < 3; c++) pb[c] = go * gq[c] / fl.dx;
        for (int s = m - 1; s >= 0; s--) {
            // p_{s+1} = p_s - h V(pm_s), pm_s = p_s - hh V(p_s)
            float vb[3], pmb[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int c = 0; c < 3; c++) vb[c] = -h * pb[c];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const Tri tv = flow_tri(fl, c, pms[s]);
                tri_scatter(acc.flow[c], tv, vb[c]);
                float g[3];
                tri_grad(fl.f[c], tv, g);
#pragma unroll
                for (int e = 0; e < 3; e++) pmb[e] += vb[c] * (g[e] / fl.dx);
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                pb[c] += pmb[c];
                vb[c] = -hh * pmb[c];
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const Tri tv = flow_tri(fl, c, ps[s]);
                tri_scatter(acc.flow[c], tv, vb[c]);
                float g[3];
                tri_grad(fl.f[c], tv, g);
#pragma unroll
                for (int e = 0; e < 3; e++) pb[e] += vb[c] * (g[e] / fl.dx);
            }
        }
    }
}

// out = (float) acc (+ base when given).
__global__ void __launch_bounds__(TPB) k_acc_round(float* __restrict__ out, const double* __restrict__ acc,
                                                   const float* __restrict__ base, int64_t n) {
    pdl_wait();
    pdl_trigger();
    for (int64_t i = (int64_t)blockIdx.x * TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TPB)
        out[i] = (float)(acc[i] + (base ? (double)base[i] : 0.0));
}

}  // namespace mpp
