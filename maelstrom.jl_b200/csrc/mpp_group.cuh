// Batches in groups (sm_100a): the CG loop of many basins that share a grid size and every
// setting that shapes the launch sequence (precision, sweeps, smoother forms, level
// split), run as one launch per pass for the whole group. blockIdx.y is the basin and
// blockIdx.x walks that basin's active tiles exactly as the single-basin launch does (the
// same grid width, the same per-cell arithmetic, the same fixed-order reductions), so a
// basin's result is bit for bit its own solve's. Each launch carries the group's
// per-basin arguments by value (a __grid_constant__ array of at most GRP_MAX entries) and
// every basin's done flag: a basin that has converged skips the remaining passes while the
// others iterate, and the group's loop (one conditional WHILE node) ends when every basin
// is done.
#pragma once

#include "mpp_cmg.cuh"
#include "mpp_tma.cuh"

namespace mpp {

constexpr int GRP_MAX = 16;

template <class T>
struct Grp {
    T a[GRP_MAX];
};

// One basin's arguments for each kind of pass, and its done flag (State::done).
template <class M>
struct GLev {
    Lev<M> L;
    const int* done;
};
template <class M>
struct GLev2 {
    Lev<M> F;  // the finer level (restriction) or the level itself (prolongation)
    Lev<M> C;  // the coarser level
    const int* done;
};
template <class M, class C>
struct GRestrictBottom {
    Lev<M> F, L;
    C* bout;
    const int* done;
};
template <class M>
struct GCmg {
    CmgArgs<M> a;
    const int* done;
};
template <class M, class C>
struct GBottom {
    const C* bin;
    M* xout;
    BotArgs a;
    const int* done;
};
template <class M, class V>
struct GCg {
    Lev<M> L;
    V *r, *q, *d, *P;
    const V* diag;
    Scalars* sc;
    double* partials;
    unsigned* counter;
};

// A basin that is done skips a V-cycle pass (read after the wait: the flag was written by
// an earlier kernel of the sequence, so every block, and every CTA of a cluster, sees the
// same value).
__device__ __forceinline__ bool grp_skip(const int* done) {
    pdl_wait();
    return *done != 0;
}

template <class Pr>
__global__ void __launch_bounds__(TPB) k_start_v8_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    start_v8_body<Pr>(a.L);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_start_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    pdl_trigger();
    start_body<Pr>(a.L);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, RBGS_V8_BLOCKS) k_rbgs_v8_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g,
                                                                 int colour, int b_late) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    rbgs_v8_body<Pr>(a.L, colour, b_late);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g, int colour) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    pdl_trigger();
    rbgs_body<Pr>(a.L, colour);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_rbgs_async_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g, int colour) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    rbgs_async_dev<Pr>(a.L, colour);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_residual_v8_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    residual_v8_body<Pr>(a.L);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_residual_g(const __grid_constant__ Grp<GLev<typename Pr::M>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    pdl_trigger();
    residual_body<Pr>(a.L);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 3) k_restrict_g(const __grid_constant__ Grp<GLev2<typename Pr::M>> g, int start) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    pdl_trigger();
    restrict_body<Pr>(a.F, a.C, start);
}
template <class Pr>
__global__ void __launch_bounds__(TPB)
    k_restrict_bottom_g(const __grid_constant__ Grp<GRestrictBottom<typename Pr::M, typename Pr::C>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    restrict_bottom_dev<Pr>(a.F, a.L, a.bout);
}
template <class Pr, int UP>
__global__ void __launch_bounds__(CMG_THREADS, 1) k_cmg_g(const __grid_constant__ Grp<GCmg<typename Pr::M>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;  // every CTA of the basin's cluster returns together
    cmg_dev<Pr, UP>(a.a);
}
template <class Pr>
__global__ void __launch_bounds__(1024)
    k_bottom_g(const __grid_constant__ Grp<GBottom<typename Pr::M, typename Pr::C>> g) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    bottom_dev<Pr>(a.bin, a.xout, a.a);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_prolong_v8_g(const __grid_constant__ Grp<GLev2<typename Pr::M>> g, int cnat) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    prolong_v8_body<Pr>(a.F, a.C, cnat);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_prolong_g(const __grid_constant__ Grp<GLev2<typename Pr::M>> g, int cnat) {
    const auto& a = g.a[blockIdx.y];
    if (grp_skip(a.done)) return;
    pdl_trigger();
    prolong_body<Pr>(a.F, a.C, cnat);
}
// The CG passes check the flag themselves (after their wait, every block alike).
template <class Pr>
__global__ void __launch_bounds__(TPB) k_dot_v8_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g) {
    const auto& a = g.a[blockIdx.y];
    dot_v8_dev<Pr>(a.L, a.r, a.q, a.sc, a.partials, a.counter);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_dot_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g) {
    const auto& a = g.a[blockIdx.y];
    dot_dev<Pr>(a.L, a.r, a.q, a.sc, a.partials, a.counter);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 2) k_search_v8_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g) {
    const auto& a = g.a[blockIdx.y];
    search_v8_dev<Pr>(a.L, a.d, a.diag, a.q, a.sc, a.partials, a.counter);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_search_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g) {
    const auto& a = g.a[blockIdx.y];
    search_dev<Pr>(a.L, a.d, a.diag, a.q, a.sc, a.partials, a.counter);
}
template <class Pr>
__global__ void __launch_bounds__(TPB, 3) k_advance_v8_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g,
                                                           int start) {
    const auto& a = g.a[blockIdx.y];
    advance_v8_dev<Pr>(a.L, a.d, a.q, a.r, a.P, a.sc, a.partials, a.counter, cudaGraphConditionalHandle{}, 0, start);
}
template <class Pr>
__global__ void __launch_bounds__(TPB) k_advance_g(const __grid_constant__ Grp<GCg<typename Pr::M, typename Pr::V>> g) {
    const auto& a = g.a[blockIdx.y];
    advance_dev<Pr>(a.L, a.d, a.q, a.r, a.P, a.sc, a.partials, a.counter, cudaGraphConditionalHandle{}, 0);
}

// The end of a group's iteration: another while any basin of the group is not done.
__global__ void k_group_cond(const __grid_constant__ Grp<const int*> done, int n, cudaGraphConditionalHandle cond) {
    pdl_wait();
    int any = 0;
    for (int i = 0; i < n; i++) any |= *done.a[i] == 0;
    cudaGraphSetConditional(cond, any ? 1u : 0u);
}

}  // namespace mpp
