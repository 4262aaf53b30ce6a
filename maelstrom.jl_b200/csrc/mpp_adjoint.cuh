// The adjoint (vector-Jacobian product) of project! with respect to the face velocities.
//
// project! (src/flip.jl:1144-1156) is affine in (u, v, w) for fixed cell classes and level
// set: b = -dx D u + dx^2 gamma on LIQUID cells (rhs_kernel!, src/flip.jl:817-822),
// A P = b, and u_out = u - G P (project_kernel!, src/flip.jl:1113-1130), where G takes
// the face difference of P with the ghost-fluid 1/theta at liquid-air faces. With A
// symmetric, the transpose of d u_out / d u = I + dx G A^-1 D is I + D^T A^-1 (dx G^T),
// so for a cotangent g on the output faces:
//   beta  = dx G^T g            (k_vjp_rhs; on LIQUID cells)
//   A mu  = beta                (the same preconditioned solve as the forward pressure)
//   g_in  = g + D^T mu          (k_vjp_faces; on every face)
// gamma depends on the level set only, so it has no velocity derivative.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

// One face of cell c (natural index ci, LIQUID) seen from c: its neighbour's class and the
// face weight of G (1 towards LIQUID, 1/theta towards AIR, none towards SOLID).
template <class C>
__device__ __forceinline__ C vjp_term(const float* __restrict__ g, int64_t fi, const uint8_t* __restrict__ types,
                                      const float* __restrict__ phi, int n1, int n2, int n3, int64_t ci, int a, int b,
                                      int c) {
    const uint8_t t = typeat(types, n1, n2, n3, a, b, c);
    if (t == SOLID) return (C)0;
    if (t == LIQUID) return (C)g[fi];
    const int64_t cn = (int64_t)a + (int64_t)n1 * ((int64_t)b + (int64_t)n2 * c);
    return (C)g[fi] / theta<C>((C)phi[ci], (C)phi[cn]);
}

// beta_c = sum over c's low faces of w g - sum over its high faces of w g (LIQUID c; 0
// elsewhere), in the order -x, +x, -y, +y, -z, +z. Natural order, one thread per cell;
// C = float, or double for the FP64 form.
template <class C>
__global__ void __launch_bounds__(TPB) k_vjp_rhs(int n1, int n2, int n3, C* __restrict__ beta,
                                                 const float* __restrict__ gu, const float* __restrict__ gv,
                                                 const float* __restrict__ gw, const uint8_t* __restrict__ types,
                                                 const float* __restrict__ phi) {
    pdl_wait();
    pdl_trigger();
    const int m1 = n1 + 1, m2 = n2 + 1;
    FOR_CELLS(n1, n2, n3, i, j, k, idx) {
        C s = (C)0;
        if (types[idx] == LIQUID) {
            const int64_t fu = (int64_t)i + (int64_t)m1 * ((int64_t)j + (int64_t)n2 * k);
            const int64_t fv = (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)m2 * k);
            const int64_t fw = idx;
            s = s + vjp_term<C>(gu, fu, types, phi, n1, n2, n3, idx, i - 1, j, k);
            s = s - vjp_term<C>(gu, fu + 1, types, phi, n1, n2, n3, idx, i + 1, j, k);
            s = s + vjp_term<C>(gv, fv, types, phi, n1, n2, n3, idx, i, j - 1, k);
            s = s - vjp_term<C>(gv, fv + n1, types, phi, n1, n2, n3, idx, i, j + 1, k);
            s = s + vjp_term<C>(gw, fw, types, phi, n1, n2, n3, idx, i, j, k - 1);
            s = s - vjp_term<C>(gw, fw + (int64_t)n1 * n2, types, phi, n1, n2, n3, idx, i, j, k + 1);
        }
        beta[idx] = s;
    }
}

// g_in = g + mu_before [before LIQUID] - mu_after [after LIQUID] on one face, in mu's type.
template <class C>
__device__ __forceinline__ void vjp_face(float* out, const float* g, int64_t fi, const C* __restrict__ mu,
                                         const uint8_t* __restrict__ types, int n1, int n2, int n3, int a, int b,
                                         int c, int i, int j, int k) {
    C r = (C)g[fi];
    if (typeat(types, n1, n2, n3, a, b, c) == LIQUID)
        r = r + mu[(int64_t)a + (int64_t)n1 * ((int64_t)b + (int64_t)n2 * c)];
    if (typeat(types, n1, n2, n3, i, j, k) == LIQUID)
        r = r - mu[(int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k)];
    out[fi] = (float)r;
}

// All three face sets in one launch, one thread per face site of the (n+1)^3 lattice (as
// k_gradient). `out` may be `g` itself: each thread reads and writes only its own faces.
template <class C>
__global__ void __launch_bounds__(TPB) k_vjp_faces(int n1, int n2, int n3, float* ou, float* ov, float* ow,
                                                   const float* gu, const float* gv, const float* gw,
                                                   const C* __restrict__ mu, const uint8_t* __restrict__ types) {
    pdl_wait();
    pdl_trigger();
    const int m1 = n1 + 1, m2 = n2 + 1;
    FOR_CELLS(n1 + 1, n2 + 1, n3 + 1, i, j, k, idx) {
        (void)idx;
        if (j < n2 && k < n3)
            vjp_face(ou, gu, (int64_t)i + (int64_t)m1 * ((int64_t)j + (int64_t)n2 * k), mu, types, n1, n2, n3, i - 1, j,
                     k, i, j, k);
        if (i < n1 && k < n3)
            vjp_face(ov, gv, (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)m2 * k), mu, types, n1, n2, n3, i, j - 1,
                     k, i, j, k);
        if (i < n1 && j < n2)
            vjp_face(ow, gw, (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k), mu, types, n1, n2, n3, i, j,
                     k - 1, i, j, k);
    }
}

}  // namespace mpp
