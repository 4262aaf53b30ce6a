// Vector kernels of the FGMRES fallback (restated from the reference's solver,
// src/fgmres.jl:26-92, for the dense operator). They work over the fine level's active
// tiles in the row-split layout, both colours of each column, and keep every vector zero
// on the non-LIQUID cells of those tiles; cells outside the active tiles are never read
// as LIQUID neighbours. The Arnoldi scalars (Gram-Schmidt coefficients, norms) are FP64
// grid sums left in device memory, so the Gram-Schmidt passes of one column run without
// a host round trip; the small Hessenberg/Givens system is solved on the host in FP64,
// as the reference does.
#pragma once

#include "mpp_stream.cuh"

namespace mpp {

// Visit the LIQUID cells of this thread's column: body(p) with p the row-split position.
#define FG_CELLS(L, p, body)                                                 \
    {                                                                        \
        const int sz_ = (L).n1 * (L).n2;                                     \
        FOR_TILES_PF(L, tile) {                                              \
            Col c_;                                                          \
            if (!col_of(L, tile, c_)) continue;                              \
            _Pragma("unroll") for (int q_ = 0; q_ < TZ; q_++) {              \
                if (q_ >= c_.kn) break;                                      \
                _Pragma("unroll") for (int cc_ = 0; cc_ < 2; cc_++) {        \
                    const int p = c_.rb + q_ * sz_ + cc_ * (L).H + c_.h;     \
                    const bool liquid_ = ((L).code[p] & SELF) != 0;          \
                    body                                                     \
                }                                                            \
            }                                                                \
        }                                                                    \
    }

// out[slot] = a.b over LIQUID cells (FP64, deterministic grid sum).
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_dot(Lev<float> L, const V* __restrict__ a, const V* __restrict__ b,
                                                double* out, int slot, double* partials, unsigned* counter) {
    pdl_wait();
    pdl_trigger();
    double acc[1] = {0.0};
    FG_CELLS(L, p, if (liquid_) acc[0] += (double)a[p] * (double)b[p];)
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) out[slot] = acc[0];
}

// y = alpha x (0 off-liquid).
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_scale(Lev<float> L, V* __restrict__ y, const V* __restrict__ x,
                                                  double alpha) {
    pdl_wait();
    pdl_trigger();
    FG_CELLS(L, p, y[p] = liquid_ ? (V)(alpha * (double)x[p]) : (V)0;)
}

// One modified Gram-Schmidt step: q -= h[slot] v, h left by k_fg_dot.
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_orth(Lev<float> L, V* __restrict__ q, const V* __restrict__ v,
                                                 const double* __restrict__ h, int slot) {
    pdl_wait();
    pdl_trigger();
    const double hv = h[slot];
    FG_CELLS(L, p, if (liquid_) q[p] = (V)((double)q[p] - hv * (double)v[p]);)
}

// v = q / sqrt(nrm2[slot]) (0 when the norm is 0 or not finite: the host stops then).
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_normalize(Lev<float> L, V* __restrict__ v, const V* __restrict__ q,
                                                      const double* __restrict__ nrm2, int slot) {
    pdl_wait();
    pdl_trigger();
    const double n = sqrt(nrm2[slot]);
    const double inv = (n > 0.0 && n < INFINITY) ? 1.0 / n : 0.0;
    FG_CELLS(L, p, v[p] = liquid_ ? (V)(inv * (double)q[p]) : (V)0;)
}

// The V-cycle's input: the fine level's b (type M) = scale * v.
template <class M, class V>
__global__ void __launch_bounds__(TPB) k_fg_to_cycle(Lev<float> L, M* __restrict__ dst, const V* __restrict__ v,
                                                     double scale) {
    pdl_wait();
    pdl_trigger();
    FG_CELLS(L, p, st(dst + p, liquid_ ? scale * (double)v[p] : 0.0);)
}

// z = scale * (the V-cycle's output, type M).
template <class M, class V>
__global__ void __launch_bounds__(TPB) k_fg_from_cycle(Lev<float> L, V* __restrict__ z, const M* __restrict__ x,
                                                       double scale) {
    pdl_wait();
    pdl_trigger();
    FG_CELLS(L, p, z[p] = liquid_ ? (V)(scale * ld<double>(x + p)) : (V)0;)
}

// P (natural order) += y z (row-split) on LIQUID cells: the FGMRES update.
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_update_P(Lev<float> L, V* __restrict__ P, const V* __restrict__ z, double y) {
    pdl_wait();
    pdl_trigger();
    const int sz = L.n1 * L.n2;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            if (q >= c.kn) break;
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = c.rb + q * sz + cc * L.H + c.h;
                if (!(L.code[p] & SELF)) continue;
                const int pn = c.rb + q * sz + 2 * c.h + ci_of(cc, c.j, c.k0 + q);
                P[pn] = (V)((double)P[pn] + y * (double)z[p]);
            }
        }
    }
}

// P = 0 on LIQUID cells (the reference zeroes P before FGMRES when CG diverged).
template <class V>
__global__ void __launch_bounds__(TPB) k_fg_zero_P(Lev<float> L, V* __restrict__ P) {
    pdl_wait();
    pdl_trigger();
    const int sz = L.n1 * L.n2;
    FOR_TILES_PF(L, tile) {
        Col c;
        if (!col_of(L, tile, c)) continue;
#pragma unroll
        for (int q = 0; q < TZ; q++) {
            if (q >= c.kn) break;
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int p = c.rb + q * sz + cc * L.H + c.h;
                if (L.code[p] & SELF) P[c.rb + q * sz + 2 * c.h + ci_of(cc, c.j, c.k0 + q)] = (V)0;
            }
        }
    }
}

}  // namespace mpp
