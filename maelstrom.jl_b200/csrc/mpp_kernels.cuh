// The projection's kernels (sm_100a). Every kernel names the reference kernel(s) of
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
    int pad[2];
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

// volume_kernel! + volume + the gamma of project! (src/flip.jl:261-279, 293, 1146-1147):
// liquid volume sum clamp(0.5 - phi/dx, 0, 1) dx^3 over cells whose centre is not solid,
// then gamma = clamp(loss / recover, -0.01/dt, 0.01/dt) with loss the relative volume loss.
__global__ void __launch_bounds__(TPB) k_volume(Geo g, const float* __restrict__ phi, Scalars* sc,
                                                double* partials, unsigned* counter) {
    const int64_t N = (int64_t)g.n[0] * g.n[1] * g.n[2];
    double acc[1] = {0.0};
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        int i = (int)(idx % g.n[0]);
        int j = (int)((idx / g.n[0]) % g.n[1]);
        int k = (int)(idx / ((int64_t)g.n[0] * g.n[1]));
        if (!issolidcell(g, i, j, k)) {
            float x = 0.5f - phi[idx] / g.dx;
            acc[0] += (double)(x > 1.f ? 1.f : (x < 0.f ? 0.f : x));
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
    V* P;               // pressure (natural): warm start in
    const uint8_t* types;
    const float* phi;   // null: no ghost-fluid terms (rhs-only passes)
    float dx;
    int clear_P;   // clearair (src/flip.jl:1132-1135)
    int residual;  // 1: r = b - A P and the norms; 0: operator only
};

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
    using V = typename Pr::V;
    using M = typename Pr::M;
    using C = typename Pr::C;
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3;
    const int64_t N = (int64_t)n1 * n2 * n3;
    const C dx = (C)a.dx;
    const C gamma = (C)(sc->p.project ? sc->s.gamma : sc->p.gamma);
    const bool sep_dg = (void*)L.dg != (void*)diag;
    const bool sep_b = (void*)L.b != (void*)r;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % n1);
        const int j = (int)((idx / n1) % n2);
        const int k = (int)(idx / ((int64_t)n1 * n2));
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
            if (a.bnat) {
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
        } else if (a.clear_P) {
            a.P[idx] = (V)0;
        }
        L.code[p] = code;
        st(diag + p, d);
        if (sep_dg) st(L.dg + p, d);
        st(b + p, bv);
        if (a.residual) {
            st(r + p, rv);
            if (sep_b) st(L.b + p, rv);
            acc[0] += (double)bv * (double)bv;
            acc[1] += (double)rv * (double)rv;
        }
    }
    if (!a.residual) return;
    if (grid_sum<3>(acc, partials, counter) && threadIdx.x == 0) {
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
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3;
    const int64_t N = (int64_t)n1 * n2 * n3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int I = (int)(idx % n1), J = (int)((idx / n1) % n2), K = (int)(idx / ((int64_t)n1 * n2));
        const uint8_t t = coarsen_at(tf, f1, f2, f3, I, J, K);
        L.types[idx] = t;
        if (!split) continue;
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
            L.tflag[L.tile_of(I, J, K)] = 1;
        }
        const int64_t p = L.pos(I, J, K);
        L.code[p] = code;
        st(L.dg + p, d);
    }
}

// The active-tile lists: one block per level compacts that level's tile flags in tile
// order (a block-wide scan), so the lists, and the reductions over them, are the same
// on every run.
struct TileTab {
    int nlev;
    int ntiles[16];
    uint8_t* flags[16];
    uint32_t* tiles[16];
    int* count[16];
};
__global__ void __launch_bounds__(1024) k_tilelists(TileTab tab) {
    const int l = blockIdx.x;
    if (l >= tab.nlev) return;
    const int n = tab.ntiles[l];
    const uint8_t* f = tab.flags[l];
    const int chunk = (n + 1023) / 1024;
    const int lo = min(n, (int)threadIdx.x * chunk), hi = min(n, lo + chunk);
    int c = 0;
    for (int t = lo; t < hi; t++) c += f[t] != 0;
    __shared__ int sc[1024];
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int v = threadIdx.x >= (unsigned)o ? sc[threadIdx.x - o] : 0;
        __syncthreads();
        sc[threadIdx.x] += v;
        __syncthreads();
    }
    int w = sc[threadIdx.x] - c;
    for (int t = lo; t < hi; t++)
        if (f[t]) tab.tiles[l][w++] = (uint32_t)t;
    if (threadIdx.x == 1023) *tab.count[l] = sc[1023];
}

// ---- the V-cycle (src/flip.jl:992-1014), one kernel per pass, over active tiles ----

// start_kernel! (src/flip.jl:965-973): colour-0 LIQUID cells get b/diag, every other cell 0.
template <class Pr>
__global__ void __launch_bounds__(TPB) k_start(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    const int n = *L.count;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
        const int64_t p0 = rb + s.h, p1 = rb + L.H + s.h;
        C v = (C)0;
        if (L.code[p0] & SELF) {
            C d = ld<C>(L.dg + p0);
            if (d > (C)0) v = ld<C>(L.b + p0) / d;
        }
        st(L.x + p0, v);
        st(L.x + p1, (C)0);
    }
}

// rbgs_kernel! (src/flip.jl:870-877): one colour of red-black Gauss-Seidel,
// x = (b + sum_LIQ x_n) / diag on LIQUID cells of that colour.
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs(Lev<typename Pr::M> L, int colour) {
    using C = typename Pr::C;
    const int n = *L.count;
    const int64_t sy = L.n1, sz = (int64_t)L.n1 * L.n2;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
        const int64_t p = rb + (int64_t)colour * L.H + s.h;
        const uint8_t code = L.code[p];
        if (!(code & SELF)) continue;
        const int i = cell_i(s.h, colour, s.j, s.k);
        const C sum = nbsum<C>(L.x, code, rb + (int64_t)(1 - colour) * L.H, i, s.h, sy, sz);
        const C d = ld<C>(L.dg + p);
        st(L.x + p, d > (C)0 ? (ld<C>(L.b + p) + sum) / d : (C)0);
    }
}

// residual_kernel! (src/flip.jl:859-863): r = b - (diag x - sum_LIQ x_n) on LIQUID, else 0.
template <class Pr>
__global__ void __launch_bounds__(TPB) k_residual(Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    const int n = *L.count;
    const int64_t sy = L.n1, sz = (int64_t)L.n1 * L.n2;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            const uint8_t code = L.code[p];
            C v = (C)0;
            if (code & SELF) {
                const int i = cell_i(s.h, c, s.j, s.k);
                const C sum = nbsum<C>(L.x, code, rb + (int64_t)(1 - c) * L.H, i, s.h, sy, sz);
                v = ld<C>(L.b + p) - (ld<C>(L.dg + p) * ld<C>(L.x + p) - sum);
            }
            st(L.r + p, v);
        }
    }
}

// weightB (src/flip.jl:891): (1, 3, 3, 1) / 8.
template <class C>
__device__ __forceinline__ C wB(int a) {
    return (a == 1 || a == 2) ? (C)0.375f : (C)0.125f;
}

// restrict_kernel! (src/flip.jl:894-906) at coarse cell (I,J,K): 4 sum w_a w_b w_c rf over
// the LIQUID fine cells of the 4x4x4 block, a fastest (the reference's loop order). The
// scaled (16-bit) forms drop the factor 4.
template <bool SCALED, class C, class M>
__device__ __forceinline__ C restrict_at(const Lev<M>& F, int I, int J, int K) {
    C s = (C)0;
    for (int c = 0; c < 4; c++) {
        const int k = 2 * K + c - 1;
        if (k < 0 || k >= F.n3) continue;
        for (int b = 0; b < 4; b++) {
            const int j = 2 * J + b - 1;
            if (j < 0 || j >= F.n2) continue;
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int i = 2 * I + a - 1;
                if (i < 0 || i >= F.n1) continue;
                const int64_t p = F.pos(i, j, k);
                if (F.code[p] & SELF) s += wB<C>(a) * wB<C>(b) * wB<C>(c) * ld<C>(F.r + p);
            }
        }
    }
    return SCALED ? s : (C)4 * s;
}

template <class Pr>
__global__ void __launch_bounds__(TPB) k_restrict(Lev<typename Pr::M> F, Lev<typename Pr::M> L) {
    using C = typename Pr::C;
    const int n = *L.count;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            C v = (C)0;
            if (L.code[p] & SELF) v = restrict_at<Pr::scaled, C>(F, cell_i(s.h, c, s.j, s.k), s.j, s.k);
            st(L.b + p, v);
        }
    }
}

// prolongweights (src/flip.jl:908-911), 0-based.
template <class C>
__device__ __forceinline__ void pweights(int i, int& c0, C& w0, int& c1, C& w1) {
    const int I = i >> 1;
    if ((i & 1) == 0) { c0 = I - 1; w0 = (C)0.25f; c1 = I; w1 = (C)0.75f; }
    else { c0 = I; w0 = (C)0.75f; c1 = I + 1; w1 = (C)0.25f; }
}

// prolong_kernel! (src/flip.jl:914-929): xf += sum of the trilinear weights times xc over
// LIQUID coarse cells (m = 0..7, a from bit 0, b bit 1, c bit 2). The coarse level is
// row-split, or the coarsest in natural order (`cnat`).
template <class Pr>
__global__ void __launch_bounds__(TPB) k_prolong(Lev<typename Pr::M> L, Lev<typename Pr::M> Cl, int cnat) {
    using C = typename Pr::C;
    const int n = *L.count;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
        int b0, b1, k0, k1;
        C wb0, wb1, wc0, wc1;
        pweights<C>(s.j, b0, wb0, b1, wb1);
        pweights<C>(s.k, k0, wc0, k1, wc1);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            if (!(L.code[p] & SELF)) continue;
            const int i = cell_i(s.h, c, s.j, s.k);
            int a0, a1;
            C wa0, wa1;
            pweights<C>(i, a0, wa0, a1, wa1);
            C sum = (C)0;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                const int A = (m & 1) ? a1 : a0, B = (m & 2) ? b1 : b0, K = (m & 4) ? k1 : k0;
                const C wa = (m & 1) ? wa1 : wa0, wb = (m & 2) ? wb1 : wb0, wc = (m & 4) ? wc1 : wc0;
                if (A < 0 || A >= Cl.n1 || B < 0 || B >= Cl.n2 || K < 0 || K >= Cl.n3) continue;
                if (cnat) {
                    const int64_t q = Cl.nat(A, B, K);
                    if (Cl.types[q] == LIQUID) sum += wa * wb * wc * ld<C>(Cl.x + q);
                } else {
                    const int64_t q = Cl.pos(A, B, K);
                    if (Cl.code[q] & SELF) sum += wa * wb * wc * ld<C>(Cl.x + q);
                }
            }
            st(L.x + p, ld<C>(L.x + p) + (Pr::scaled ? (C)4 * sum : sum));
        }
    }
}

// The coarsest level (at most 1024 cells) in one block: restrict_kernel! into it from the
// level above (src/flip.jl:1004), then coarse_kernel! (src/flip.jl:935-962): `sweeps`
// red-black sweeps from zero and as many in reverse colour order, in shared memory, the
// diagonal the count of non-SOLID neighbours and the accumulator starting at b.
template <class Pr>
__global__ void __launch_bounds__(1024) k_coarsest(Lev<typename Pr::M> F, Lev<typename Pr::M> L, int sweeps) {
    using C = typename Pr::C;
    using CC = typename Pr::CC;
    __shared__ CC xs[1024];
    const int t = threadIdx.x;
    const int n1 = L.n1, n2 = L.n2, n3 = L.n3, N = n1 * n2 * n3;
    const bool active = t < N;
    const int i = t % n1, j = (t / n1) % n2, k = t / (n1 * n2);
    uint8_t ti = active ? L.types[t] : SOLID;
    CC bi = (CC)0, d = (CC)0;
    int nb[6];
    int nn = 0;
    if (active && ti == LIQUID) {
        bi = (CC)restrict_at<Pr::scaled, C>(F, i, j, k);
        const int di[6] = {1, -1, 0, 0, 0, 0}, dj[6] = {0, 0, 1, -1, 0, 0}, dk[6] = {0, 0, 0, 0, 1, -1};
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const int a = i + di[m], b = j + dj[m], c = k + dk[m];
            const uint8_t tn = typeat(L.types, n1, n2, n3, a, b, c);
            if (tn != SOLID) d += (CC)1;
            if (tn == LIQUID) nb[nn++] = a + n1 * (b + n2 * c);
        }
    }
    const int mycol = (i + j + k + 1) & 1;
    xs[t] = (CC)0;
    __syncthreads();
    for (int s = 1; s <= 2 * sweeps; s++) {
        for (int half = 0; half <= 1; half++) {
            const int colour = s <= sweeps ? half : 1 - half;
            if (active && ti == LIQUID && mycol == colour) {
                CC acc = bi;
                for (int q = 0; q < nn; q++) acc += xs[nb[q]];
                xs[t] = d > (CC)0 ? acc / d : (CC)0;
            }
            __syncthreads();
        }
    }
    if (active) st(L.x + t, xs[t]);
}

// ---- CG (src/flip.jl:1033-1111) over the fine level's active tiles ----

// inner(s, z, r) after the V-cycle (src/flip.jl:1095-1096, 1105-1107): rho_new = z.r, then
// beta = rho_new / rho (beta = 0 on the first pass). The flexible form also sums z.q and
// takes the Polak-Ribiere beta = max(0, (rho_new - z.r_old) / rho) of the reference's
// flexible CG (src/sflip.jl:1896-1897); since r = r_old - alpha q, z.r_old = rho_new +
// alpha z.q, so no copy of r_old is kept.
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_dot(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ r, const typename Pr::V* __restrict__ q,
          Scalars* sc, double* partials, unsigned* counter) {
    using V = typename Pr::V;
    if (sc->s.done) return;
    const int n = *L.count;
    double acc[2] = {0.0, 0.0};
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            if (!(L.code[p] & SELF)) continue;
            const double z = ld<double>(L.x + p);
            acc[0] += z * (double)r[p];
            if constexpr (Pr::flexible) acc[1] += z * (double)q[p];
        }
    }
    if (grid_sum<2>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        const double rho_new = rs<Pr>(acc[0]);
        if (!finite_d(rho_new)) {
            S.status = ST_NONFINITE;
            S.done = 1;
            return;
        }
        if constexpr (Pr::flexible) {
            if (!(rho_new > 0.0)) {  // src/sflip.jl:1880,1896
                S.status = ST_INDEFINITE;
                S.done = 1;
                return;
            }
            double beta = S.it == 0 ? 0.0 : -S.alpha * acc[1] / S.rho;
            S.beta = beta > 0.0 ? beta : 0.0;
        } else {
            S.beta = S.it == 0 ? 0.0 : dv<Pr>(rho_new, S.rho);
        }
        S.rho = rho_new;
    }
}

// search_kernel! (src/flip.jl:1033-1054): p = z + beta d made where it is used, q = A p,
// and p.q; then alpha = rho / p.q (src/flip.jl:1100).
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_search(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ diag,
             typename Pr::V* __restrict__ q, Scalars* sc, double* partials, unsigned* counter) {
    using C = typename Pr::C;
    if (sc->s.done) return;
    const C beta = (C)sc->s.beta;
    const bool first = sc->s.beta == 0.0;
    const int n = *L.count;
    const int64_t sy = L.n1, sz = (int64_t)L.n1 * L.n2;
    double acc[1] = {0.0};
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            const uint8_t code = L.code[p];
            C qv = (C)0;
            if (code & SELF) {
                const int i = cell_i(s.h, c, s.j, s.k);
                const int64_t o = rb + (int64_t)(1 - c) * L.H;
                const C pc = first ? ld<C>(L.x + p) : ld<C>(L.x + p) + beta * (C)dvec[p];
                C a = (C)0;
                int64_t nq[6];
                nq[0] = o + ((i + 1) >> 1); nq[1] = o + ((i - 1) >> 1);
                nq[2] = o + sy + s.h; nq[3] = o - sy + s.h; nq[4] = o + sz + s.h; nq[5] = o - sz + s.h;
#pragma unroll
                for (int m = 0; m < 6; m++)
                    if (code & (1u << m))
                        a += first ? ld<C>(L.x + nq[m]) : ld<C>(L.x + nq[m]) + beta * (C)dvec[nq[m]];
                qv = (C)diag[p] * pc - a;
                acc[0] += (double)pc * (double)qv;
            }
            st(q + p, qv);
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        S.pq = rs<Pr>(acc[0]);
        if (!finite_d(S.pq)) {
            S.status = ST_NONFINITE;
            S.done = 1;
        } else if (!(S.pq > 0.0)) {  // src/sflip.jl:1876-1877
            S.status = ST_INDEFINITE;
            S.done = 1;
        } else {
            S.alpha = dv<Pr>(S.rho, S.pq);
        }
    }
}

// advance_kernel! (src/flip.jl:1059-1073): d = z + beta d; P += alpha d; r -= alpha q; then
// rnorm = sqrt(r.r) and the exit test rnorm <= tol |b| (src/flip.jl:1102-1103), or maxiter.
// The mixed forms also store r in the V-cycle's precision for its next pass.
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_advance(Lev<typename Pr::M> L, typename Pr::V* __restrict__ dvec, const typename Pr::V* __restrict__ q,
              typename Pr::V* __restrict__ r, typename Pr::V* __restrict__ P, Scalars* sc, double* partials,
              unsigned* counter, cudaGraphConditionalHandle cond, int use_cond) {
    using C = typename Pr::C;
    if (sc->s.done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(cond, use_cond, 0);
        return;
    }
    const C beta = (C)sc->s.beta, alpha = (C)sc->s.alpha;
    const bool first = sc->s.beta == 0.0;
    const bool sep_b = (void*)L.b != (void*)r;
    const C rsc = (C)sc->s.rscale;
    const int n = *L.count;
    double acc[1] = {0.0};
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            if (!(L.code[p] & SELF)) continue;
            const int i = cell_i(s.h, c, s.j, s.k);
            const int64_t pn = (int64_t)i + (int64_t)L.n1 * ((int64_t)s.j + (int64_t)L.n2 * s.k);
            const C pc = first ? ld<C>(L.x + p) : ld<C>(L.x + p) + beta * (C)dvec[p];
            st(dvec + p, pc);
            st(P + pn, (C)P[pn] + alpha * pc);
            const C rl = (C)r[p] - alpha * (C)q[p];
            st(r + p, rl);
            if (sep_b) st(L.b + p, rl * rsc);
            acc[0] += (double)rl * (double)rl;
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) {
        State& S = sc->s;
        S.it += 1;
        S.rnorm = sq<Pr>(acc[0]);
        S.rscale = next_rscale(S.rnorm, S.nliq);
        if (!finite_d(S.rnorm)) {
            S.status = ST_NONFINITE;
            S.done = 1;
        } else if (S.rnorm <= S.target) {
            S.status = ST_OK;
            S.done = 1;
        } else if (S.it >= sc->p.maxiter) {
            S.status = ST_NOT_CONVERGED;
            S.done = 1;
        }
        set_cond(cond, use_cond, !S.done);
    }
}

// |b - A P| over the fine level: the true residual at exit (the reference's sparse
// solver checks it the same way, src/fgmres.jl:101-103).
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_true_residual(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ b, const typename Pr::V* __restrict__ diag,
                    const typename Pr::V* __restrict__ P, typename Pr::V* __restrict__ rout, Scalars* sc,
                    double* partials, unsigned* counter) {
    using C = typename Pr::C;
    const int n = *L.count;
    const int n1 = L.n1, n2 = L.n2;
    double acc[1] = {0.0};
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            const uint8_t code = L.code[p];
            if (!(code & SELF)) continue;
            const int i = cell_i(s.h, c, s.j, s.k);
            const int64_t pn = (int64_t)i + (int64_t)n1 * ((int64_t)s.j + (int64_t)n2 * s.k);
            C sum = (C)0;
            if (code & 1) sum += (C)P[pn + 1];
            if (code & 2) sum += (C)P[pn - 1];
            if (code & 4) sum += (C)P[pn + n1];
            if (code & 8) sum += (C)P[pn - n1];
            if (code & 16) sum += (C)P[pn + (int64_t)n1 * n2];
            if (code & 32) sum += (C)P[pn - (int64_t)n1 * n2];
            const C rv = (C)b[p] - ((C)diag[p] * (C)P[pn] - sum);
            if (rout) st(rout + p, rv);
            acc[0] += (double)rv * (double)rv;
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0) sc->s.true_rr = acc[0];
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
    const int m1 = n1 + 1, m2 = n2 + 1, m3 = n3 + 1;
    const int64_t N = (int64_t)m1 * m2 * m3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % m1), j = (int)((idx / m1) % m2), k = (int)(idx / ((int64_t)m1 * m2));
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

// ---- layout conversions (natural <-> row-split) for the single-pass entry points ----
template <class T, class S>
__global__ void __launch_bounds__(TPB) k_to_split(Lev<float> L, T* __restrict__ dst, const S* __restrict__ src) {
    const int64_t N = (int64_t)L.n1 * L.n2 * L.n3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % L.n1), j = (int)((idx / L.n1) % L.n2), k = (int)(idx / ((int64_t)L.n1 * L.n2));
        st(dst + L.pos(i, j, k), ld<double>(src + idx));
    }
}
template <class T, class S>
__global__ void __launch_bounds__(TPB) k_from_split(Lev<float> L, T* __restrict__ dst, const S* __restrict__ src) {
    const int64_t N = (int64_t)L.n1 * L.n2 * L.n3;
    for (int64_t idx = (int64_t)blockIdx.x * TPB + threadIdx.x; idx < N; idx += (int64_t)gridDim.x * TPB) {
        const int i = (int)(idx % L.n1), j = (int)((idx / L.n1) % L.n2), k = (int)(idx / ((int64_t)L.n1 * L.n2));
        st(dst + idx, ld<double>(src + L.pos(i, j, k)));
    }
}

// y = A x on the fine level (row-split, every cell of the active tiles; 0 off-liquid).
template <class Pr>
__global__ void __launch_bounds__(TPB) k_apply(Lev<typename Pr::M> L, const typename Pr::V* __restrict__ x,
                                               const typename Pr::V* __restrict__ diag, typename Pr::V* __restrict__ y) {
    using C = typename Pr::C;
    const int n = *L.count;
    const int64_t sy = L.n1, sz = (int64_t)L.n1 * L.n2;
    for (int t = blockIdx.x; t < n; t += gridDim.x) {
        const Slot s = slot_of(L, L.tiles[t]);
        if (!s.in) continue;
        const int64_t rb = L.row(s.j, s.k);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int64_t p = rb + (int64_t)c * L.H + s.h;
            const uint8_t code = L.code[p];
            C v = (C)0;
            if (code & SELF) {
                const int i = cell_i(s.h, c, s.j, s.k);
                v = (C)diag[p] * (C)x[p] - nbsum<C>(x, code, rb + (int64_t)(1 - c) * L.H, i, s.h, sy, sz);
            }
            st(y + p, v);
        }
    }
}

// P (float, natural) <-> the FP64 solution vector.
__global__ void __launch_bounds__(TPB) k_widen(double* __restrict__ dst, const float* __restrict__ src, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TPB)
        dst[i] = (double)src[i];
}
__global__ void __launch_bounds__(TPB) k_narrow(float* __restrict__ dst, const double* __restrict__ src, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * TPB)
        dst[i] = (float)src[i];
}

}  // namespace mpp
