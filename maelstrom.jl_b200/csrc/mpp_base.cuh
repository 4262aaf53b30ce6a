// The projection's whole-grid kernels (sm_100a): parameters and device state, volume,
// the fine set-up pass, coarsening, the gradient update, layout conversions. Every kernel
// names the reference kernel(s) of
// src/flip.jl it computes; the per-cell arithmetic follows the reference's operation
// order, and the library is built with -fmad=false, so the FP32 form rounds exactly as
// the reference's Float32 code does. Reductions are FP64 and deterministic (mpp_common).
#pragma once

#include "mpp_common.cuh"

namespace mpp {

// ---- per-call parameters and the device-resident solver state ----
struct Params {
    float volume0;   // s.volume0
    float tol;       // relative tolerance
    double dt;       // time step (project!)
    double recover;  // volume recovery time (project!)
    int maxiter;
    int project;     // 1: gamma from the volume loss; 0: no volume term
    float gamma;     // (unused when project = 1)
    int pad;
};

struct State {
    double vol;      // volume(s), m^3
    double bnorm, target, rnorm, rho, alpha, beta, pq, true_rr;
    double nliq;     // LIQUID cells
    double rscale;   // power of two the next V-cycle input is scaled by (16-bit forms)
    float gamma;
    int status;      // MPP_* status
    int it;          // CG iterations done
    int done;        // 1 once the loop must stop
    int fault;       // a bounded device wait gave up (the host reports an error)
    int pad;
};

struct Scalars {
    Params p;
    State s;
};

enum { ST_OK = 0, ST_NOT_CONVERGED = 1, ST_NONFINITE = 2, ST_INDEFINITE = 3, ST_BREAKDOWN = 4 };

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

// Scalars as the reference keeps them: Float32 (f32_scalars) or FP64.
template <class Pr>
__device__ __forceinline__ double rs(double x) {
    if constexpr (Pr::f32_scalars) return (double)(float)x;
    else return x;
}
template <class Pr>
__device__ __forceinline__ double sq(double x) {
    if constexpr (Pr::f32_scalars) return (double)sqrtf((float)x);
    else return sqrt(x);
}
template <class Pr>
__device__ __forceinline__ double dv(double a, double b) {
    if constexpr (Pr::f32_scalars) return (double)((float)a / (float)b);
    else return a / b;
}

// The power of two the next V-cycle input is scaled by in the 16-bit forms: it brings
// the residual's typical entry, |r| / sqrt(liquid cells), to about 1/4, far from both
// ends of FP16's range. (The V-cycle is linear and CG is invariant to a scalar on the
// preconditioner, so the scale changes no iterate.)
__device__ __forceinline__ double next_rscale(double rnorm, double nliq) {
    if (!(rnorm > 0.0) || !isfinite(rnorm) || !(nliq > 0.0)) return 1.0;
    double e = rint(log2(0.25 * sqrt(nliq) / rnorm));
    e = e > 60.0 ? 60.0 : (e < -60.0 ? -60.0 : e);
    return exp2(e);
}

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use, int go) {
    if (use) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// ---- geometry (FlipGrid, src/flip.jl:39-66) ----
struct Geo {
    float lo[3];
    float dx;
    int n[3];
    float radius, floor_z;
};
// issolidcell: the cell centre lies outside the cylinder or under the floor (Float32).
__device__ __forceinline__ bool issolidcell(const Geo& g, int i, int j, int k) {
    float px = g.lo[0] + ((float)i + 0.5f) * g.dx;
    float py = g.lo[1] + ((float)j + 0.5f) * g.dx;
    float pz = g.lo[2] + ((float)k + 0.5f) * g.dx;
    return px * px + py * py > g.radius * g.radius || pz < g.floor_z;
}

__device__ __forceinline__ uint8_t typeat(const uint8_t* __restrict__ t, int n1, int n2, int n3, int i, int j,
                                          int k) {
    return (i >= 0 && i < n1 && j >= 0 && j < n2 && k >= 0 && k < n3)
               ? t[(int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k)]
               : SOLID;
}

// A cell's liquid fraction clamp(0.5 - phi/dx, 0, 1) (src/flip.jl:268). Outside the
// band |phi| < dx/2 it is 0 or 1 without the division: 0.5 dx is exact, correctly rounded
// division is monotone and 0.5 is representable, so phi >= dx/2 gives phi/dx >= 0.5 and
// phi <= -dx/2 gives phi/dx <= -0.5 (NaN takes the division, as before).
__device__ __forceinline__ float liquid_fraction(float ph, float dx) {
    const float h = 0.5f * dx;
    if (ph >= h) return 0.f;
    if (ph <= -h) return 1.f;
    const float x = 0.5f - ph / dx;
    return x > 1.f ? 1.f : (x < 0.f ? 0.f : x);
}

// volume_kernel! + volume + the gamma of project! (src/flip.jl:261-279, 293, 1146-1147):
// liquid volume sum clamp(0.5 - phi/dx, 0, 1) dx^3 over cells whose centre is not solid,
// then gamma = clamp(loss / recover, -0.01/dt, 0.01/dt) with loss the relative volume loss.
__global__ void __launch_bounds__(TPB) k_volume(Geo g, const float* __restrict__ phi, Scalars* sc,
                                                double* partials, unsigned* counter) {
    pdl_wait();
    pdl_trigger();
    double acc[1] = {0.0};
    if (g.n[0] % 8 == 0 && (reinterpret_cast<uintptr_t>(phi) & 15) == 0) {  // 8 cells of a row a thread
        const int nq = g.n[0] / 8, n2 = g.n[1], nch = nq * n2 * g.n[2];
        // the chunk's (q8, j, k) stepped by the grid stride's own with carries
        const int ch0 = (int)(blockIdx.x * TPB + threadIdx.x), step = (int)(gridDim.x * TPB);
        int qi = ch0 % nq, ji = (ch0 / nq) % n2, ki = ch0 / nq / n2;
        const int dq = step % nq, dj = (step / nq) % n2, dk = step / nq / n2;
        for (int ch = ch0; ch < nch; ch += step) {
            const int q8 = qi, j = ji, k = ki, i0 = 8 * q8;
            qi += dq;
            ji += dj;
            ki += dk;
            if (qi >= nq) { qi -= nq; ji++; }
            if (ji >= n2) { ji -= n2; ki++; }
            const float4* p4 = reinterpret_cast<const float4*>(phi + (int64_t)(j + n2 * k) * g.n[0] + i0);
            const float4 a = p4[0], b = p4[1];
            const float ph[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int m = 0; m < 8; m++)
                if (!issolidcell(g, i0 + m, j, k)) acc[0] += (double)liquid_fraction(ph[m], g.dx);
        }
    } else {
        FOR_CELLS(g.n[0], g.n[1], g.n[2], i, j, k, idx) {
            if (!issolidcell(g, i, j, k)) acc[0] += (double)liquid_fraction(phi[idx], g.dx);
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) {
        float vol = (float)acc[0] * (g.dx * g.dx * g.dx);
        sc->s.vol = (double)vol;
        if (sc->p.project) {
            float loss = (sc->p.volume0 - vol) / sc->p.volume0;
            double lo = -0.01 / sc->p.dt, hi = 0.01 / sc->p.dt, x = (double)loss / sc->p.recover;
            sc->s.gamma = (float)(x > hi ? hi : (x < lo ? lo : x));
        } else {
            sc->s.gamma = sc->p.gamma;
        }
    }
}

// Inputs of the fine-level set-up pass.
template <class V>
struct SetupIn {
    const float* u;  // faces, or null when b is given
    const float* v;
    const float* w;
    const float* bnat;  // given rhs (natural), or null
    const double* bnat64;  // given FP64 rhs (natural; the FP64 adjoint), or null
    V* P;               // pressure (natural): warm start in
    const uint8_t* types;
    const float* phi;   // null: no ghost-fluid terms (rhs-only passes)
    float dx;
    int clear_P;   // clearair (src/flip.jl:1132-1135)
    int residual;  // 1: r = b - A P and the norms; 0: operator only
};

// pressure!'s opening (src/flip.jl:1086-1094), by the set-up's last block: |b|, |r| of the
// warm start, the tolerance's target, and the loop's first test.
template <class Pr>
__device__ __forceinline__ void setup_finish(Scalars* sc, const double (&acc)[3], cudaGraphConditionalHandle cond,
                                             int use_cond) {
    State& s = sc->s;
    s.bnorm = sq<Pr>(acc[0]);
    s.target = rs<Pr>((double)sc->p.tol * s.bnorm);
    s.rnorm = sq<Pr>(acc[1]);
    s.nliq = acc[2];
    s.rscale = next_rscale(s.rnorm, s.nliq);
    s.it = 0;
    s.rho = 0.0;
    s.beta = 0.0;
    s.alpha = 0.0;
    s.status = ST_OK;
    s.done = 0;
    if (!finite_d(s.bnorm) || !finite_d(s.rnorm)) {
        s.status = ST_NONFINITE;
        s.done = 1;
    } else if (s.bnorm == 0.0 || s.rnorm <= s.target) {
        s.done = 1;  // pressure! returns 0 (src/flip.jl:1091-1094)
    }
    set_cond(cond, use_cond, !s.done);
}

// The fine level's set-up, one pass over every cell (natural order):
//   diag_kernel! (src/flip.jl:824-836) -> diag (and the smoother's copy),
//   rhs_kernel!  (src/flip.jl:817-822) -> b (unless b is given),
//   clearair_kernel! (src/flip.jl:1132-1135) -> P = 0 off-liquid,
//   residual_kernel! (src/flip.jl:859-863) on the warm start -> r,
//   the stencil codes and the level's tile flags, and |b|^2, |r|^2 for pressure!'s
//   first tests (src/flip.jl:1090-1094).
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_setup(SetupIn<typename Pr::V> a, Lev<typename Pr::M> L, typename Pr::V* __restrict__ diag,
            typename Pr::V* __restrict__ b, typename Pr::V* __restrict__ r, Scalars* sc, double* partials,
            unsigned* counter, cudaGraphConditionalHandle cond, int use_cond) {
    pdl_wait();
    pdl_trigger();
    using V = typename Pr::V;
    using M = typename Pr::M;
    using C = typename Pr::C;
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3;
    const C dx = (C)a.dx;
    const C gamma = (C)(sc->p.project ? sc->s.gamma : sc->p.gamma);
    const bool sep_dg = (void*)L.dg != (void*)diag;
    const bool sep_b = (void*)L.b != (void*)r;
    double acc[3] = {0.0, 0.0, 0.0};
    FOR_CELLS(n1, n2, n3, i, j, k, idx) {
        const uint8_t t = a.types[idx];
        acc[2] += t == LIQUID ? 1.0 : 0.0;
        const int64_t p = L.pos(i, j, k);
        uint8_t code = 0;
        C d = (C)0, bv = (C)0, rv = (C)0;
        if (t == LIQUID) {
            const int di[6] = {1, -1, 0, 0, 0, 0}, dj[6] = {0, 0, 1, -1, 0, 0}, dk[6] = {0, 0, 0, 0, 1, -1};
            const C phc = a.phi ? (C)a.phi[idx] : (C)0;
#pragma unroll
            for (int m = 0; m < 6; m++) {
                const int ii = i + di[m], jj = j + dj[m], kk = k + dk[m];
                const uint8_t tn = typeat(a.types, n1, n2, n3, ii, jj, kk);
                if (tn == LIQUID) {
                    code |= (uint8_t)(1u << m);
                    d += (C)1;
                }
                if (tn == AIR && a.phi)
                    d += (C)1 / theta<C>(phc, (C)a.phi[(int64_t)ii + (int64_t)n1 * ((int64_t)jj + (int64_t)n2 * kk)]);
            }
            code |= SELF;
            if (a.bnat64) {
                bv = (C)a.bnat64[idx];
            } else if (a.bnat) {
                bv = (C)a.bnat[idx];
            } else if (a.u) {
                C div = (C)a.u[(int64_t)(i + 1) + (int64_t)(n1 + 1) * ((int64_t)j + (int64_t)n2 * k)] -
                        (C)a.u[(int64_t)i + (int64_t)(n1 + 1) * ((int64_t)j + (int64_t)n2 * k)];
                div = div + (C)a.v[(int64_t)i + (int64_t)n1 * ((int64_t)(j + 1) + (int64_t)(n2 + 1) * k)];
                div = div - (C)a.v[(int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)(n2 + 1) * k)];
                div = div + (C)a.w[idx + (int64_t)n1 * n2];
                div = div - (C)a.w[idx];
                bv = (-dx) * div + (dx * dx) * gamma;
            }
            if (a.residual) {
                C s = (C)0;
#pragma unroll
                for (int m = 0; m < 6; m++)
                    if (code & (1u << m)) s += (C)a.P[(int64_t)(i + di[m]) + (int64_t)n1 * ((int64_t)(j + dj[m]) + (int64_t)n2 * (k + dk[m]))];
                rv = bv - (d * (C)a.P[idx] - s);
            }
            L.tflag[L.tile_of(i, j, k)] = 1;
            if (i == 0 || i == n1 - 1 || j == 0 || j == n2 - 1) atomicOr(L.edge, 1);
        } else if (a.clear_P) {
            a.P[idx] = (V)0;
        }
        L.code[p] = code;
        st(diag + p, d);
        if (sep_dg) st(L.dg + p, d);
        if (L.di) st(L.di + p, d > (C)0 ? (C)1 / d : (C)0);
        st(b + p, bv);
        if (a.residual) {
            st(r + p, rv);
            if (sep_b) st(L.b + p, rv);
            acc[0] += (double)bv * (double)bv;
            acc[1] += (double)rv * (double)rv;
        }
    }
    if (!a.residual) return;
    if (grid_sum<3>(acc, partials, counter) && threadIdx.x == 0) setup_finish<Pr>(sc, acc, cond, use_cond);
}

// k_setup with 8 consecutive cells of a row per thread (rows a multiple of 8 long): the
// classes, velocities and warm start come in as 8-wide row pieces, and the outputs leave
// as 4-wide pieces of each colour's half of the row-split rows. Same arithmetic, in the
// same order, as k_setup.
template <class T, int W>
struct RowW {
    T v[W];
};
// N-element pieces (aligned to their size) moved as one access of that size, or 16-byte ones.
template <int BYTES>
__device__ __forceinline__ void copy_piece(void* dst, const void* src) {
    if constexpr (BYTES == 2) *reinterpret_cast<uint16_t*>(dst) = *reinterpret_cast<const uint16_t*>(src);
    else if constexpr (BYTES == 4) *reinterpret_cast<uint32_t*>(dst) = *reinterpret_cast<const uint32_t*>(src);
    else if constexpr (BYTES == 8) *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(src);
    else {
        static_assert(BYTES % 16 == 0, "pieces of 2, 4, 8 or a multiple of 16 bytes");
#pragma unroll
        for (int q = 0; q < BYTES / 16; q++)
            reinterpret_cast<uint4*>(dst)[q] = reinterpret_cast<const uint4*>(src)[q];
    }
}
template <int W, class T>
__device__ __forceinline__ RowW<T, W> ld_row(const T* p) {  // W-element aligned
    RowW<T, W> r;
    copy_piece<(int)sizeof(T) * W>(r.v, p);
    return r;
}
template <int N, class T>
__device__ __forceinline__ void st_piece(T* p, const T (&v)[N]) {  // N-element aligned
    copy_piece<(int)sizeof(T) * N>(p, v);
}

// W = 4 or 8 cells of a row a thread; 128-thread blocks (at this kernel's register count
// the finer-grained blocks fill more of each SM).
constexpr int SETUP_V8_TPB = 128, SETUP_W = 4;
template <class Pr, int W>
__global__ void __launch_bounds__(SETUP_V8_TPB, 4)
    k_setup_v8(SetupIn<typename Pr::V> a, Lev<typename Pr::M> L, typename Pr::V* __restrict__ diag,
               typename Pr::V* __restrict__ b, typename Pr::V* __restrict__ r, Scalars* sc, double* partials,
               unsigned* counter, cudaGraphConditionalHandle cond, int use_cond) {
    pdl_wait();
    pdl_trigger();
    using V = typename Pr::V;
    using M = typename Pr::M;
    using C = typename Pr::C;
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3, nq = n1 / W, sz = n1 * n2;
    const C dx = (C)a.dx;
    const C gamma = (C)(sc->p.project ? sc->s.gamma : sc->p.gamma);
    const bool sep_dg = (void*)L.dg != (void*)diag;
    const bool sep_b = (void*)L.b != (void*)r;
    double acc[3] = {0.0, 0.0, 0.0};
    const int nch = nq * n2 * n3;
    // the chunk's (q8, j, k), stepped by the grid stride's own (dq, dj, dk) with carries
    // instead of divided out of the chunk index each step
    const int ch0 = (int)(blockIdx.x * SETUP_V8_TPB + threadIdx.x), step = (int)(gridDim.x * SETUP_V8_TPB);
    int qi = ch0 % nq, ji = (ch0 / nq) % n2, ki = ch0 / nq / n2;
    const int dq = step % nq, dj = (step / nq) % n2, dk = step / nq / n2;
    for (int ch = ch0; ch < nch; ch += step) {
        const int q8 = qi, j = ji, k = ki, i0 = W * q8;
        const int row = (j + n2 * k) * n1, idx0 = row + i0;
        qi += dq;
        ji += dj;
        ki += dk;
        if (qi >= nq) { qi -= nq; ji++; }
        if (ji >= n2) { ji -= n2; ki++; }
        RowW<uint8_t, W> tc = ld_row<W>(a.types + idx0), tym, typ, tzm, tzp;
#pragma unroll
        for (int m = 0; m < W; m++) tym.v[m] = typ.v[m] = tzm.v[m] = tzp.v[m] = SOLID;
        if (j > 0) tym = ld_row<W>(a.types + idx0 - n1);
        if (j + 1 < n2) typ = ld_row<W>(a.types + idx0 + n1);
        if (k > 0) tzm = ld_row<W>(a.types + idx0 - sz);
        if (k + 1 < n3) tzp = ld_row<W>(a.types + idx0 + sz);
        const uint8_t txm = i0 > 0 ? a.types[idx0 - 1] : (uint8_t)SOLID;
        const uint8_t txp = i0 + W < n1 ? a.types[idx0 + W] : (uint8_t)SOLID;
        bool any = false;
#pragma unroll
        for (int m = 0; m < W; m++) any |= tc.v[m] == LIQUID;
        uint8_t code[W];
        C d[W], bv[W], rv[W];
#pragma unroll
        for (int m = 0; m < W; m++) {
            code[m] = 0;
            d[m] = bv[m] = rv[m] = (C)0;
        }
        if (any) {
            // rhs inputs (aligned rows of v and w; u rows are n1 + 1 long: element loads)
            RowW<float, W> vlo, vhi, wlo, whi;
            float ur[W + 1];
            const bool rhs = !a.bnat64 && !a.bnat && a.u;
            if (rhs) {
                const int ub = (n1 + 1) * (j + n2 * k) + i0;
#pragma unroll
                for (int m = 0; m < W + 1; m++) ur[m] = a.u[ub + m];
                vlo = ld_row<W>(a.v + (int64_t)n1 * (j + (n2 + 1) * k) + i0);
                vhi = ld_row<W>(a.v + (int64_t)n1 * (j + 1 + (n2 + 1) * k) + i0);
                wlo = ld_row<W>(a.w + idx0);
                whi = ld_row<W>(a.w + idx0 + sz);
            }
            // the warm start's rows around the chunk (rows past the grid's are SOLID
            // neighbours, never read) and the chunk's own level-set values
            RowW<V, W> pc, pyp, pym, pzp, pzm;
            V pxl = (V)0, pxr = (V)0;
            RowW<float, W> phr;
#pragma unroll
            for (int m = 0; m < W; m++) {
                pc.v[m] = pyp.v[m] = pym.v[m] = pzp.v[m] = pzm.v[m] = (V)0;
                phr.v[m] = 0.f;
            }
            if (a.residual) {
                pc = ld_row<W>(a.P + idx0);
                if (j + 1 < n2) pyp = ld_row<W>(a.P + idx0 + n1);
                if (j > 0) pym = ld_row<W>(a.P + idx0 - n1);
                if (k + 1 < n3) pzp = ld_row<W>(a.P + idx0 + sz);
                if (k > 0) pzm = ld_row<W>(a.P + idx0 - sz);
                if (i0 > 0) pxl = a.P[idx0 - 1];
                if (i0 + W < n1) pxr = a.P[idx0 + W];
            }
            if (a.phi) phr = ld_row<W>(a.phi + idx0);
            bool at_edge = false;
#pragma unroll
            for (int m = 0; m < W; m++) {
                if (tc.v[m] != LIQUID) continue;
                const int i = i0 + m, idx = idx0 + m;
                const uint8_t tn[6] = {m < W - 1 ? tc.v[m < W - 1 ? m + 1 : 0] : txp, m > 0 ? tc.v[m > 0 ? m - 1 : 0] : txm,
                                       typ.v[m], tym.v[m], tzp.v[m], tzm.v[m]};
                const int off[6] = {1, -1, n1, -n1, sz, -sz};
                C dd = (C)0;
                uint8_t cd = 0;
                const C phc = (C)phr.v[m];
#pragma unroll
                for (int n = 0; n < 6; n++) {
                    if (tn[n] == LIQUID) {
                        cd |= (uint8_t)(1u << n);
                        dd += (C)1;
                    }
                    if (tn[n] == AIR && a.phi) dd += (C)1 / theta<C>(phc, (C)a.phi[idx + off[n]]);
                }
                cd |= SELF;
                code[m] = cd;
                d[m] = dd;
                C bb = (C)0;
                if (a.bnat64) {
                    bb = (C)a.bnat64[idx];
                } else if (a.bnat) {
                    bb = (C)a.bnat[idx];
                } else if (rhs) {
                    C div = (C)ur[m + 1] - (C)ur[m];
                    div = div + (C)vhi.v[m];
                    div = div - (C)vlo.v[m];
                    div = div + (C)whi.v[m];
                    div = div - (C)wlo.v[m];
                    bb = (-dx) * div + (dx * dx) * gamma;
                }
                bv[m] = bb;
                if (a.residual) {
                    const V pn[6] = {m < W - 1 ? pc.v[m < W - 1 ? m + 1 : 0] : pxr, m > 0 ? pc.v[m > 0 ? m - 1 : 0] : pxl,
                                     pyp.v[m], pym.v[m], pzp.v[m], pzm.v[m]};
                    C s = (C)0;
#pragma unroll
                    for (int n = 0; n < 6; n++)
                        if (cd & (1u << n)) s += (C)pn[n];
                    rv[m] = bb - (dd * (C)pc.v[m] - s);
                }
                at_edge |= i == 0 || i == n1 - 1 || j == 0 || j == n2 - 1;
                acc[2] += 1.0;
            }
            // the chunk's cells share one tile (a tile row is 2 TH cells, W divides it)
            L.tflag[L.tile_of(i0, j, k)] = 1;
            if (at_edge) atomicOr(L.edge, 1);
        }
        if (a.clear_P) {
#pragma unroll
            for (int m = 0; m < W; m++)
                if (tc.v[m] != LIQUID) a.P[idx0 + m] = (V)0;
        }
        // the two colours' halves: colour c holds the cells m = p, p + 2, p + 4, p + 6
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int p0 = (c + j + k + 1) & 1;
            const int pos = row + c * L.H + i0 / 2;
            uint8_t cq[W / 2];
            V dq[W / 2], bq[W / 2], rq[W / 2];
            M gq[W / 2], iq[W / 2], lq[W / 2];
#pragma unroll
            for (int s2 = 0; s2 < W / 2; s2++) {
                const int m = p0 + 2 * s2;  // p0 is 0 or 1: pick by select, not by index
                const uint8_t cm = p0 ? code[(2 * s2 + 1) & (W - 1)] : code[2 * s2];
                const C dm = p0 ? d[(2 * s2 + 1) & (W - 1)] : d[2 * s2];
                const C bm = p0 ? bv[(2 * s2 + 1) & (W - 1)] : bv[2 * s2];
                const C rm = p0 ? rv[(2 * s2 + 1) & (W - 1)] : rv[2 * s2];
                (void)m;
                cq[s2] = cm;
                st(&dq[s2], dm);
                st(&bq[s2], bm);
                st(&rq[s2], rm);
                st(&gq[s2], dm);
                st(&iq[s2], dm > (C)0 ? (C)1 / dm : (C)0);
                st(&lq[s2], rm);
                if (a.residual && (cm & SELF)) {
                    acc[0] += (double)bm * (double)bm;
                    acc[1] += (double)rm * (double)rm;
                }
            }
            st_piece<W / 2>(L.code + pos, cq);
            st_piece<W / 2>(diag + pos, dq);
            if (sep_dg) st_piece<W / 2>(L.dg + pos, gq);
            if (L.di) st_piece<W / 2>(L.di + pos, iq);
            st_piece<W / 2>(b + pos, bq);
            if (a.residual) {
                st_piece<W / 2>(r + pos, rq);
                if (sep_b) st_piece<W / 2>(L.b + pos, lq);
            }
        }
    }
    if (!a.residual) return;
    if (grid_sum<3>(acc, partials, counter) && threadIdx.x == 0) setup_finish<Pr>(sc, acc, cond, use_cond);
}

// coarsen_kernel! (src/flip.jl:880-889) for level l from level l-1, fused with the coarse
// level's stencil codes, its diagonal (celldiag, src/flip.jl:843-850: the count of
// non-SOLID neighbours) and its tile flags. One thread per coarse cell (natural order);
// the neighbours' classes are coarsened again from their children, which are cached.
__device__ __forceinline__ uint8_t coarsen_at(const uint8_t* __restrict__ tf, int f1, int f2, int f3, int I, int J,
                                              int K) {
    bool air = false, liquid = false;
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int a = 0; a < 2; a++) {
                uint8_t t = typeat(tf, f1, f2, f3, 2 * I + a, 2 * J + b, 2 * K + c);
                air |= t == AIR;
                liquid |= t == LIQUID;
            }
    return air ? AIR : (liquid ? LIQUID : SOLID);
}

template <class Pr>
__global__ void __launch_bounds__(TPB) k_level(const uint8_t* __restrict__ tf, int f1, int f2, int f3,
                                               Lev<typename Pr::M> L, int split) {
    pdl_wait();
    pdl_trigger();
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3;
    const int N = n1 * n2 * n3;  // coarse levels: short rows, so one flat 32-bit index
    for (int idx = (int)(blockIdx.x * TPB + threadIdx.x); idx < N; idx += (int)(gridDim.x * TPB)) {
        const int I = idx % n1, JK = idx / n1, J = JK % n2, K = JK / n2;
        const uint8_t t = coarsen_at(tf, f1, f2, f3, I, J, K);
        L.types[idx] = t;
        uint8_t code = 0;
        float d = 0.f;
        if (t == LIQUID) {
            const int di[6] = {1, -1, 0, 0, 0, 0}, dj[6] = {0, 0, 1, -1, 0, 0}, dk[6] = {0, 0, 0, 0, 1, -1};
#pragma unroll
            for (int m = 0; m < 6; m++) {
                const int ii = I + di[m], jj = J + dj[m], kk = K + dk[m];
                uint8_t tn = SOLID;
                if (ii >= 0 && ii < n1 && jj >= 0 && jj < n2 && kk >= 0 && kk < n3)
                    tn = coarsen_at(tf, f1, f2, f3, ii, jj, kk);
                if (tn != SOLID) d += 1.f;
                if (tn == LIQUID) code |= (uint8_t)(1u << m);
            }
            code |= SELF;
            if (split) L.tflag[L.tile_of(I, J, K)] = 1;
            if (split && (I == 0 || I == n1 - 1 || J == 0 || J == n2 - 1)) atomicOr(L.edge, 1);
        }
        if (split) {
            const int64_t p = L.pos(I, J, K);
            L.code[p] = code;
            st(L.dg + p, d);
            if (L.di) st(L.di + p, d > 0.f ? 1.f / d : 0.f);
        } else {  // a level of the one-CTA bottom solve: natural order
            L.code[idx] = code;
            L.dc[idx] = (uint8_t)d;
        }
    }
}

// restrict_kernel! (src/flip.jl:894-906) into the first level of the one-CTA bottom solve
// (natural order, a few thousand cells), from the row-split level above: one thread per
// coarse cell, its 64 code and residual loads issued together. Values in C precision
// (the scaled forms without the factor 4).
template <class Pr>
__device__ __forceinline__ void restrict_bottom_body(Lev<typename Pr::M> F, Lev<typename Pr::M> L,
                                                         typename Pr::C* __restrict__ bout) {
    using C = typename Pr::C;
    const int N = L.n1 * L.n2 * L.n3;
    for (int c = blockIdx.x * TPB + threadIdx.x; c < N; c += gridDim.x * TPB) {
        C v = (C)0;
        if (L.code[c] & SELF) {
            const int I = c % L.n1, J = (c / L.n1) % L.n2, K = c / (L.n1 * L.n2);
            C s = (C)0;
#pragma unroll
            for (int c3 = 0; c3 < 4; c3++)
#pragma unroll
                for (int b3 = 0; b3 < 4; b3++)
#pragma unroll
                    for (int a3 = 0; a3 < 4; a3++) {
                        const int i = 2 * I + a3 - 1, j = 2 * J + b3 - 1, k = 2 * K + c3 - 1;
                        C rv = (C)0;
                        if (i >= 0 && i < F.n1 && j >= 0 && j < F.n2 && k >= 0 && k < F.n3) {
                            const int p = (int)F.pos(i, j, k);
                            const uint8_t cd = F.code[p];
                            const C r = ld<C>(F.r + p);
                            rv = (cd & SELF) ? r : (C)0;
                        }
                        const C w = (a3 == 1 || a3 == 2 ? (C)0.375f : (C)0.125f) *
                                    (b3 == 1 || b3 == 2 ? (C)0.375f : (C)0.125f) *
                                    (c3 == 1 || c3 == 2 ? (C)0.375f : (C)0.125f);
                        s = macc<Pr::scaled>(s, w, rv);
                    }
            v = Pr::scaled ? s : (C)4 * s;
        }
        bout[c] = v;
    }
}
template <class Pr>
__device__ __forceinline__ void restrict_bottom_dev(Lev<typename Pr::M> F, Lev<typename Pr::M> L,
                                                         typename Pr::C* __restrict__ bout) {
    pdl_wait();
    pdl_trigger();
    restrict_bottom_body<Pr>(F, L, bout);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_restrict_bottom(Lev<typename Pr::M> F, Lev<typename Pr::M> L,
                                                         typename Pr::C* __restrict__ bout) {
    restrict_bottom_dev<Pr>(F, L, bout);
}


// project_kernel! (src/flip.jl:1113-1130) for all three face sets in one launch: a face
// with no SOLID side and a LIQUID one gets u -= delta/dx (ghost fluid at air faces) and
// valid = 1; every other face valid = 0. One thread per face site (i,j,k) of the
// (nx+1, ny+1, nz+1) lattice, handling the u, v and w faces that exist there.
__device__ __forceinline__ void face_update(float* __restrict__ u, uint8_t* __restrict__ f, int64_t fi,
                                            const float* __restrict__ P, const uint8_t* __restrict__ types,
                                            const float* __restrict__ phi, int n1, int n2, int n3, int a, int b,
                                            int c, int i, int j, int k, float dx) {
    const uint8_t t0 = typeat(types, n1, n2, n3, a, b, c), t1 = typeat(types, n1, n2, n3, i, j, k);
    const bool ok = t0 != SOLID && t1 != SOLID && (t0 == LIQUID || t1 == LIQUID);
    if (ok) {
        const int64_t c0 = (int64_t)a + (int64_t)n1 * ((int64_t)b + (int64_t)n2 * c);
        const int64_t c1 = (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k);
        float delta;
        if (t0 == LIQUID && t1 == LIQUID) delta = P[c1] - P[c0];
        else if (t0 == LIQUID) delta = (-P[c0]) / theta<float>(phi[c0], phi[c1]);
        else delta = P[c1] / theta<float>(phi[c1], phi[c0]);
        u[fi] = u[fi] - delta / dx;
    }
    f[fi] = ok ? 1 : 0;
}

__global__ void __launch_bounds__(TPB) k_gradient(int n1, int n2, int n3, float* __restrict__ u, float* __restrict__ v,
                                                  float* __restrict__ w, uint8_t* __restrict__ fu,
                                                  uint8_t* __restrict__ fv, uint8_t* __restrict__ fw,
                                                  const float* __restrict__ P, const uint8_t* __restrict__ types,
                                                  const float* __restrict__ phi, float dx) {
    pdl_wait();
    pdl_trigger();
    const int m1 = n1 + 1, m2 = n2 + 1;
    FOR_CELLS(n1 + 1, n2 + 1, n3 + 1, i, j, k, idx) {
        (void)idx;
        if (j < n2 && k < n3)
            face_update(u, fu, (int64_t)i + (int64_t)m1 * ((int64_t)j + (int64_t)n2 * k), P, types, phi, n1, n2, n3,
                        i - 1, j, k, i, j, k, dx);
        if (i < n1 && k < n3)
            face_update(v, fv, (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)m2 * k), P, types, phi, n1, n2, n3,
                        i, j - 1, k, i, j, k, dx);
        if (i < n1 && j < n2)
            face_update(w, fw, (int64_t)i + (int64_t)n1 * ((int64_t)j + (int64_t)n2 * k), P, types, phi, n1, n2, n3,
                        i, j, k - 1, i, j, k, dx);
    }
}

// One face's update from its two cells' class, pressure and level set (face_update's
// arithmetic; (t0, p0, f0) the cell on the low side).
__device__ __forceinline__ bool face_delta(uint8_t t0, uint8_t t1, float p0, float p1, float f0, float f1, float dx,
                                           float& u) {
    const bool ok = t0 != SOLID && t1 != SOLID && (t0 == LIQUID || t1 == LIQUID);
    if (ok) {
        float delta;
        if (t0 == LIQUID && t1 == LIQUID) delta = p1 - p0;
        else if (t0 == LIQUID) delta = (-p0) / theta<float>(f0, f1);
        else delta = p1 / theta<float>(f1, f0);
        u = u - delta / dx;
    }
    return ok;
}

// k_gradient with 4 consecutive cells of a row per thread (rows a multiple of 4 long, the
// arrays aligned): each thread updates the u, v and w faces on the low side of its cells
// (4-wide loads of the classes, P and phi of its cells and of the rows below in y and z),
// and a second loop clears the flags of the faces on the box's high sides (i = n1, j = n2,
// k = n3), which have a cell outside the grid and so are never valid. A chunk whose cells
// and low neighbours hold no LIQUID cell only writes its flags.
__global__ void __launch_bounds__(TPB) k_gradient_v4(int n1, int n2, int n3, float* __restrict__ u,
                                                     float* __restrict__ v, float* __restrict__ w,
                                                     uint8_t* __restrict__ fu, uint8_t* __restrict__ fv,
                                                     uint8_t* __restrict__ fw, const float* __restrict__ P,
                                                     const uint8_t* __restrict__ types, const float* __restrict__ phi,
                                                     float dx) {
    pdl_wait();
    pdl_trigger();
    const int nq = n1 / 4, sz = n1 * n2, nch = nq * n2 * n3;
    // the chunk's (q4, j, k) stepped by the grid stride's own with carries
    const int ch0 = (int)(blockIdx.x * TPB + threadIdx.x), step = (int)(gridDim.x * TPB);
    int qi = ch0 % nq, ji = (ch0 / nq) % n2, ki = ch0 / nq / n2;
    const int dq = step % nq, dj = (step / nq) % n2, dk = step / nq / n2;
    for (int ch = ch0; ch < nch; ch += step) {
        const int q4 = qi, j = ji, k = ki, i0 = 4 * q4;
        qi += dq;
        ji += dj;
        ki += dk;
        if (qi >= nq) { qi -= nq; ji++; }
        if (ji >= n2) { ji -= n2; ki++; }
        const int c = (j + n2 * k) * n1 + i0;  // the first cell
        const uchar4 tc = *reinterpret_cast<const uchar4*>(types + c);
        const uint8_t t[4] = {tc.x, tc.y, tc.z, tc.w};
        const uint8_t tx = i0 > 0 ? types[c - 1] : (uint8_t)SOLID;
        uint8_t ty[4] = {SOLID, SOLID, SOLID, SOLID}, tz[4] = {SOLID, SOLID, SOLID, SOLID};
        if (j > 0) {
            const uchar4 a = *reinterpret_cast<const uchar4*>(types + c - n1);
            ty[0] = a.x; ty[1] = a.y; ty[2] = a.z; ty[3] = a.w;
        }
        if (k > 0) {
            const uchar4 a = *reinterpret_cast<const uchar4*>(types + c - sz);
            tz[0] = a.x; tz[1] = a.y; tz[2] = a.z; tz[3] = a.w;
        }
        bool any = tx == LIQUID;
#pragma unroll
        for (int m = 0; m < 4; m++) any |= t[m] == LIQUID || ty[m] == LIQUID || tz[m] == LIQUID;
        const int64_t ui = (int64_t)i0 + (int64_t)(n1 + 1) * ((int64_t)j + (int64_t)n2 * k);
        const int64_t vi = (int64_t)i0 + (int64_t)n1 * ((int64_t)j + (int64_t)(n2 + 1) * k);
        const int64_t wi = (int64_t)c;  // i0 + n1 (j + n2 k): w's layout has n3 + 1 planes
        uint8_t ok_u[4] = {0, 0, 0, 0}, ok_v[4] = {0, 0, 0, 0}, ok_w[4] = {0, 0, 0, 0};
        if (any) {
            const float4 p4 = *reinterpret_cast<const float4*>(P + c), f4 = *reinterpret_cast<const float4*>(phi + c);
            const float pc[4] = {p4.x, p4.y, p4.z, p4.w}, fc[4] = {f4.x, f4.y, f4.z, f4.w};
            const float px = i0 > 0 ? P[c - 1] : 0.f, fx = i0 > 0 ? phi[c - 1] : 0.f;
            float py[4] = {0.f, 0.f, 0.f, 0.f}, fy[4] = {0.f, 0.f, 0.f, 0.f};
            float pz[4] = {0.f, 0.f, 0.f, 0.f}, fz[4] = {0.f, 0.f, 0.f, 0.f};
            if (j > 0) {
                const float4 a = *reinterpret_cast<const float4*>(P + c - n1), b = *reinterpret_cast<const float4*>(phi + c - n1);
                py[0] = a.x; py[1] = a.y; py[2] = a.z; py[3] = a.w;
                fy[0] = b.x; fy[1] = b.y; fy[2] = b.z; fy[3] = b.w;
            }
            if (k > 0) {
                const float4 a = *reinterpret_cast<const float4*>(P + c - sz), b = *reinterpret_cast<const float4*>(phi + c - sz);
                pz[0] = a.x; pz[1] = a.y; pz[2] = a.z; pz[3] = a.w;
                fz[0] = b.x; fz[1] = b.y; fz[2] = b.z; fz[3] = b.w;
            }
            float uu[4];
#pragma unroll
            for (int m = 0; m < 4; m++) uu[m] = u[ui + m];
            float4 v4 = *reinterpret_cast<const float4*>(v + vi), w4 = *reinterpret_cast<const float4*>(w + wi);
            float vv[4] = {v4.x, v4.y, v4.z, v4.w}, ww[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const uint8_t tl = m > 0 ? t[m > 0 ? m - 1 : 0] : tx;
                const float pl = m > 0 ? pc[m > 0 ? m - 1 : 0] : px, fl = m > 0 ? fc[m > 0 ? m - 1 : 0] : fx;
                ok_u[m] = face_delta(tl, t[m], pl, pc[m], fl, fc[m], dx, uu[m]);
                ok_v[m] = face_delta(ty[m], t[m], py[m], pc[m], fy[m], fc[m], dx, vv[m]);
                ok_w[m] = face_delta(tz[m], t[m], pz[m], pc[m], fz[m], fc[m], dx, ww[m]);
            }
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (ok_u[m]) u[ui + m] = uu[m];
            *reinterpret_cast<float4*>(v + vi) = make_float4(vv[0], vv[1], vv[2], vv[3]);
            *reinterpret_cast<float4*>(w + wi) = make_float4(ww[0], ww[1], ww[2], ww[3]);
        }
#pragma unroll
        for (int m = 0; m < 4; m++) fu[ui + m] = ok_u[m];
        *reinterpret_cast<uchar4*>(fv + vi) = make_uchar4(ok_v[0], ok_v[1], ok_v[2], ok_v[3]);
        *reinterpret_cast<uchar4*>(fw + wi) = make_uchar4(ok_w[0], ok_w[1], ok_w[2], ok_w[3]);
    }
    // the high-side faces: u at i = n1, v at j = n2, w at k = n3
    const int bu = n2 * n3, bv = n1 * n3, bw = n1 * n2;
    for (int e = (int)(blockIdx.x * TPB + threadIdx.x); e < bu + bv + bw; e += (int)(gridDim.x * TPB)) {
        if (e < bu) {
            fu[(int64_t)n1 + (int64_t)(n1 + 1) * e] = 0;  // e = j + n2 k
        } else if (e < bu + bv) {
            const int f = e - bu, i = f % n1, k = f / n1;
            fv[(int64_t)i + (int64_t)n1 * ((int64_t)n2 + (int64_t)(n2 + 1) * k)] = 0;
        } else {
            fw[(int64_t)(e - bu - bv) + (int64_t)n1 * n2 * n3] = 0;  // i + n1 j on plane n3
        }
    }
}

// ---- layout conversions (natural <-> row-split) for the single-pass entry points ----
template <class T, class S>
__global__ void __launch_bounds__(TPB) k_to_split(Lev<float> L, T* __restrict__ dst, const S* __restrict__ src) {
    pdl_wait();
    pdl_trigger();
    const int64_t N = (int64_t)L.n1 * L.n2 * L.n3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % L.n1), j = (int)((idx / L.n1) % L.n2), k = (int)(idx / ((int64_t)L.n1 * L.n2));
        st(dst + L.pos(i, j, k), ld<double>(src + idx));
    }
}
template <class T, class S>
__global__ void __launch_bounds__(TPB) k_from_split(Lev<float> L, T* __restrict__ dst, const S* __restrict__ src) {
    pdl_wait();
    pdl_trigger();
    const int64_t N = (int64_t)L.n1 * L.n2 * L.n3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % L.n1), j = (int)((idx / L.n1) % L.n2), k = (int)(idx / ((int64_t)L.n1 * L.n2));
        st(dst + idx, ld<double>(src + L.pos(i, j, k)));
    }
}

// P (float, natural) <-> the FP64 solution vector.
__global__ void __launch_bounds__(TPB) k_widen(double* __restrict__ dst, const float* __restrict__ src, int64_t n) {
    pdl_wait();
    pdl_trigger();
    for (int64_t i = (int64_t)blockIdx.x * TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TPB)
        dst[i] = (double)src[i];
}
__global__ void __launch_bounds__(TPB) k_narrow(float* __restrict__ dst, const double* __restrict__ src, int64_t n) {
    pdl_wait();
    pdl_trigger();
    for (int64_t i = (int64_t)blockIdx.x * TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TPB)
        dst[i] = (float)src[i];
}


}  // namespace mpp
