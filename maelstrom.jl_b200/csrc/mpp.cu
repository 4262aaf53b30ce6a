// libmpp: host side. The context (workspace of one basin), the launch sequence of a
// projection, its CUDA graph (one launch per projection: the CG loop is a conditional
// WHILE node whose condition the kernels set on the device), and the C ABI of
// include/mpp.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <vector>

#include "mpp.h"
#include <cudaTypedefs.h>

#include "mpp_adjoint.cuh"
#include "mpp_advect.cuh"
#include "mpp_extrap.cuh"
#include "mpp_fgmres.cuh"
#include "mpp_levelset.cuh"
#include "mpp_tma.cuh"
#include "mpp_cmg.cuh"
#include "mpp_group.cuh"

using namespace mpp;

namespace {

thread_local char g_err[512] = "";

void set_err(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

#define CK(call)                                                                             \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return MPP_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

constexpr int MAXLEV = 16;
constexpr int NCOUNTERS = 8;
enum { CNT_VOLUME, CNT_SETUP, CNT_DOT, CNT_SEARCH, CNT_ADVANCE, CNT_TRUE, CNT_FG };
// longest FGMRES restart cycle (Krylov basis vectors kept)
constexpr int FG_MAXR = 64;

int vsize(int prec) { return prec == MPP_PREC_FP64 ? 8 : 4; }
int msize(int prec) {
    return prec == MPP_PREC_FP64 ? 8 : (prec == MPP_PREC_MIXED_FP16 || prec == MPP_PREC_MIXED_BF16) ? 2 : 4;
}

struct LevelBuf {
    int n[3];
    int H, GH, GJ, GK, ntiles;
    bool split;
    uint8_t* code;
    void* dg;
    void* x;
    void* b;
    void* r;
    uint8_t* types;
    uint8_t* dc;
    uint8_t* tflag;
    uint32_t* tiles;
    int* count;
    void* di;   // reciprocal diagonal (16-bit forms)
    int* edge;  // LIQUID cell on an x/y face (device flag, set during set-up)
};

// Kernel families, for the profiler.
enum { F_VOLUME, F_SETUP, F_LEVEL, F_TILES, F_START, F_RBGS, F_RESID, F_RESTRICT, F_BOTTOM, F_PROLONG, F_DOT,
       F_SEARCH, F_ADVANCE, F_TRUE, F_GRADIENT, F_CONVERT, F_CMG, NFAM };
const char* const FAM_NAMES[NFAM] = {"volume",   "setup",    "coarsen", "tilelists", "start",         "rbgs",
                                     "residual", "restrict", "bottom",   "prolong",  "dot",           "search",
                                     "advance",  "true_residual", "gradient", "convert", "cluster"};
constexpr int NGRAPHS = 4;
struct GraphEntry {
    cudaGraphExec_t exec;
    cudaGraph_t graph;
    const void* key[11];
    int kind;
    int g_prologue, g_body, g_epilogue;  // kernel counts in the graph's parts
    uint64_t used;                       // last use (LRU eviction)
};
void drop_graph(GraphEntry& e) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
    memset(&e, 0, sizeof(e));
}

struct ProfRec {
    int fam, level;
    cudaEvent_t a, b;
};
struct ProfAcc {
    int64_t n;
    double ms, bytes;
    int64_t cells;
};

}  // namespace

struct mpp_ctx {
    mpp_grid grid;
    mpp_opts opts;
    int prec;
    int L;
    int dev, nsm;
    LevelBuf lv[MAXLEV];
    // fine-level CG vectors (row-split, type V)
    void *diag, *bvec, *r, *d, *q;
    void* Pd;  // FP64 solution (natural), FP64 contexts only
    uint8_t* tflag_all;
    int* edges;  // the levels' edge flags
    // extrapolation scratch (allocated at the first mpp_extrapolate, whatever its layer
    // count): ext_n mask words, three masks (open, reach ping and pong) per face array
    uint8_t* ext_r;
    int64_t ext_n;
    size_t tflag_bytes;
    Scalars* sc;
    Scalars* sc_host;  // pinned
    double* partials;
    unsigned* counters;
    std::vector<void*> allocs;
    size_t bytes;
    int64_t launches;
    // graph cache: a few captured solves keyed by their arrays (a forward and an adjoint
    // call alternate in a rollout without re-capturing)
    GraphEntry gc[NGRAPHS];
    uint64_t gclock;
    uint64_t gen;  // bumped whenever the captured solves are dropped (options, smoothers)
    cudaStream_t cap;  // stream the graphs are captured on (never the caller's)
    // second stream for the coarse levels' set-up, beside the fine set-up pass, and for the
    // true residual beside the gradient; not used by a batch's contexts (whose graph already
    // runs every basin's solve side by side: measured, the extra branches cost throughput)
    cudaStream_t aux;
    cudaEvent_t ev_fork, ev_join;
    bool in_batch;
    // levels lb .. L-1 are solved in one CTA's shared memory (k_bottom)
    int lb;
    BotArgs bot;
    size_t bot_smem, restrict_smem;
    void* botb;  // level lb's right-hand side (natural order, stencil precision)
    // levels cmg_ls .. lb-1 resident in one cluster of cmg_cs CTAs (k_cmg), when cmg_ls > 0
    int cmg_ls, cmg_cs;
    size_t cmg_smem;
    CmgSlab cmg_slab[CMG_MAXLEV];
    // TMA tensor maps of the row-split levels the smoother streams with cp.async.bulk.tensor
    TmaLev tma[MAXLEV];
    bool tma_ok[MAXLEV];
    int tma_blocks;    // persistent grid of k_rbgs_tma
    int async_blocks;  // resident grid of k_rbgs_async (16-bit forms; 0: not available)
    // smoother form of the fine level and of the coarser row-split levels (MPP_SMOOTHER_*;
    // the environment's MPP_RBGS / MPP_RBGS_COARSE: vector, tma, column); the other passes
    // of a level take the vector forms unless its smoother is the column form
    int form_fine, form_coarse;
    // profiler
    int prof_on;
    std::vector<ProfRec> pending;
    std::vector<cudaEvent_t> evfree, evall;
    ProfAcc prof[NFAM][MAXLEV + 1];
    int active[MAXLEV];
    // FGMRES fallback workspace, allocated on its first use: basis V (fg_restart + 1
    // vectors, row-split, type V), preconditioned vectors Z (guarded), Arnoldi scalars
    void* fV;
    void* fZ[FG_MAXR];
    int fg_restart;
    double* fgd;
    double* fgd_host;  // pinned
    int fg_used, fg_its;
    double fg_residual;
    void* vjp_beta;  // the adjoint solve's right-hand side (natural, V's type), allocated on first use
    double* adv_acc[3];  // FP64 accumulators of the advection adjoint (face shapes), on first use
    // trapped-air fill (mpp_filltrapped), on first use: AIR and reached bit masks, the round
    // loop's state, and the graph of the round loop (a conditional WHILE node)
    uint32_t *trap_air, *trap_reach;
    TrapState* trap_st;
    cudaGraph_t trap_graph;
    cudaGraphExec_t trap_exec;
};

namespace {

int alloc(mpp_ctx* c, void** p, size_t bytes);

// An array read at neighbour offsets past its ends (see mpp_stream.cuh): `guard` zeroed
// elements on each side; *p points at element 0.
int alloc_guarded(mpp_ctx* c, void** p, size_t es, size_t n, size_t guard) {
    void* base = nullptr;
    if (int e = alloc(c, &base, es * (n + 2 * guard))) return e;
    *p = static_cast<char*>(base) + es * guard;
    return MPP_OK;
}

int alloc(mpp_ctx* c, void** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        set_err("cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        return MPP_ERR_NOMEM;
    }
    e = cudaMemset(*p, 0, bytes);
    if (e != cudaSuccess) {
        set_err("cudaMemset failed: %s", cudaGetErrorString(e));
        return MPP_ERR_CUDA;
    }
    c->allocs.push_back(*p);
    c->bytes += bytes;
    return MPP_OK;
}

template <class M>
Lev<M> view(const mpp_ctx* c, int l) {
    const LevelBuf& b = c->lv[l];
    Lev<M> v;
    v.n1 = b.n[0]; v.n2 = b.n[1]; v.n3 = b.n[2];
    v.H = b.H; v.GH = b.GH; v.GJ = b.GJ; v.GK = b.GK;
    v.code = b.code;
    v.dg = (M*)b.dg; v.x = (M*)b.x; v.b = (M*)b.b; v.r = (M*)b.r;
    v.types = b.types; v.dc = b.dc; v.tflag = b.tflag; v.tiles = b.tiles; v.count = b.count;
    v.di = (M*)b.di; v.edge = b.edge;
    return v;
}

int grid_cells(const mpp_ctx* c, int64_t n) {
    int64_t g = (n + TPB - 1) / TPB;
    int64_t cap = (int64_t)c->nsm * MAXBLOCKS_PER_SM;
    return (int)(g < cap ? (g > 0 ? g : 1) : cap);
}
// Column kernels: TILES_PER_BLOCK tiles per block per step of their grid-stride loop.
int grid_tiles(const mpp_ctx* c, int l) {
    int g = (c->lv[l].ntiles + TILES_PER_BLOCK - 1) / TILES_PER_BLOCK;
    int cap = c->nsm * MAXBLOCKS_PER_SM;
    return g < cap ? (g > 0 ? g : 1) : cap;
}

// Kernel launches: programmatic dependent launch (see pdl_wait in mpp_common.cuh), so a
// kernel's blocks can be scheduled while the previous kernel drains.
template <typename... KArgs, typename... Args>
void launch(void (*kern)(KArgs...), dim3 grid, int block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}
// A launch without programmatic dependent launch: the kernel starts after the previous
// one has completed (for a kernel whose loads before its wait read what that one writes).
template <typename... KArgs, typename... Args>
void launch_serial(void (*kern)(KArgs...), dim3 grid, int block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// A launch of one thread-block cluster of `cs` CTAs (k_cmg), with programmatic dependent
// launch like the others.
template <typename... KArgs, typename... Args>
void launch_cluster(void (*kern)(KArgs...), int cs, int block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cs);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = (unsigned)cs;
    at[1].val.clusterDim.y = 1;
    at[1].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

Geo geo_of(const mpp_grid& g) {
    Geo o;
    for (int a = 0; a < 3; a++) { o.lo[a] = g.lo[a]; o.n[a] = g.n[a]; }
    o.dx = g.dx;
    o.radius = g.radius;
    o.floor_z = g.floor_z;
    return o;
}

cudaEvent_t prof_event(mpp_ctx* c) {
    if (!c->evfree.empty()) {
        cudaEvent_t e = c->evfree.back();
        c->evfree.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    c->evall.push_back(e);
    return e;
}

// Algorithmic bytes of one launch of a kernel family: each array element the pass must
// read or write, counted once, over the cells it covers (m, v: the V-cycle's and the CG
// vectors' element sizes; p: the solution's).
void prof_size(const mpp_ctx* c, int fam, int level, double& bytes, int64_t& cells) {
    const double m = msize(c->prec), v = vsize(c->prec), p = c->prec == MPP_PREC_FP64 ? 8 : 4;
    const bool sep = m != v;
    const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    const int64_t tile_cells = 2 * TH * TY * TZ;
    auto lcells = [&](int l) { return (int64_t)c->lv[l].n[0] * c->lv[l].n[1] * c->lv[l].n[2]; };
    auto act = [&](int l) { return (int64_t)c->active[l] * tile_cells; };
    double bpc = 0;
    switch (fam) {
        case F_VOLUME: cells = N; bpc = 4; break;
        case F_SETUP: cells = N; bpc = 1 + 12 + 4 + 8 + 1 + 3 * v + (sep ? 2 * m : 0); break;
        case F_LEVEL: cells = lcells(level); bpc = 8 + 1 + 1 + m; break;
        case F_TILES: {
            cells = 0;
            for (int l = 0; l < c->lb; l++) cells += c->lv[l].ntiles;
            bpc = 1 + 4;
            break;
        }
        case F_START: cells = act(level); bpc = 1 + 2 * m; break;
        case F_RBGS: cells = act(level); bpc = 0.5 + 2 * m; break;
        case F_RESID: cells = act(level); bpc = 1 + 4 * m; break;
        case F_RESTRICT: cells = act(level); bpc = 8 * (1 + m) + 1 + m; break;
        case F_BOTTOM: {  // the restriction into level lb reads the level above; the rest is on chip
            cells = 0;
            for (int l = c->lb; l < c->L; l++) cells += lcells(l);
            bpc = (8.0 * (1 + m) * lcells(c->lb) + m * lcells(c->lb) + cells) / (double)cells;
            break;
        }
        case F_PROLONG: cells = act(level); bpc = 1 + 2 * m + (1 + m) / 8; break;
        case F_DOT: cells = act(level); bpc = 1 + m + v + (sep ? v : 0); break;
        case F_SEARCH: cells = act(level); bpc = 1 + m + 3 * v; break;
        case F_ADVANCE: cells = act(level); bpc = 1 + m + 5 * v + 2 * p + (sep ? m : 0); break;
        case F_TRUE: cells = act(level); bpc = 1 + 2 * v + p; break;
        case F_GRADIENT: cells = N; bpc = 1 + 4 + 4 + 24 + 3; break;
        case F_CONVERT: cells = N; bpc = 12; break;
        case F_CMG: {  // levels cmg_ls .. lb-1 in shared memory: what crosses to global memory
            cells = 0;
            double b = 0;
            for (int l = c->cmg_ls; l < c->lb; l++) {
                const double n = (double)lcells(l);
                cells += lcells(l);
                // down: code, diagonal(s), b of level ls in; x and b of the others out (x of ls);
                // up: code, diagonal(s), x, b in, x of ls out
                const double dgs = (m == 2 ? 2 : 1) * m;
                b += level == 0 ? n * (1 + dgs + (l == c->cmg_ls ? m : 0) + m + (l > c->cmg_ls ? m : 0))
                                : n * (1 + dgs + 2 * m + (l == c->cmg_ls ? m : 0));
            }
            bpc = cells > 0 ? b / (double)cells : 0;
            break;
        }
        default: cells = 0; bpc = 0;
    }
    bytes = bpc * (double)cells;
}

// Fold the finished launches' event pairs into the accumulators (after a sync).
void prof_collect(mpp_ctx* c) {
    if (c->pending.empty()) return;
    for (int l = 0; l < c->lb; l++) cudaMemcpy(&c->active[l], c->lv[l].count, sizeof(int), cudaMemcpyDeviceToHost);
    for (const ProfRec& r : c->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        ProfAcc& a = c->prof[r.fam][r.level < 0 ? MAXLEV : r.level];
        double bytes;
        int64_t cells;
        prof_size(c, r.fam, r.level, bytes, cells);
        a.n += 1;
        a.ms += ms;
        a.bytes += bytes;
        a.cells = cells;
        c->evfree.push_back(r.a);
        c->evfree.push_back(r.b);
    }
    c->pending.clear();
}

// ---- launch sequences (the same code records the graph and runs the host loop) ----
// Every launch goes through beg()/end(): with profiling on they bracket it with CUDA
// events on the launching stream, tagged with its kernel family and level.
template <class Pr>
struct Run {
    using V = typename Pr::V;
    using M = typename Pr::M;
    mpp_ctx* c;
    cudaStream_t s;
    int nk = 0;  // kernels launched
    cudaEvent_t ev0 = nullptr;
    int fam = 0, lvl = 0;

    unsigned* cnt(int i) { return c->counters + i; }
    // vector (8 cells per lane) kernels on level l: rows of whole 8-element chunks
    int form(int l) const { return l == 0 ? c->form_fine : c->form_coarse; }
    bool vec(int l) const { return form(l) != MPP_SMOOTHER_COLUMN && c->lv[l].H % V8 == 0; }
    // a pipelined vector kernel's grid: the blocks resident at once (no second wave), at
    // most one warp per tile
    // Block-per-tile kernels with dynamic shared memory (the restriction): a block a tile, at
    // most the blocks resident at once, so each block streams its tiles through its copies.
    int grid_blk(const void* kern, int l, size_t smem) const {
        static std::mutex mu;
        static std::vector<std::pair<const void*, int>> occ;
        int nb = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto& e : occ)
                if (e.first == kern) nb = e.second;
            if (nb == 0) {
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TPB, smem) != cudaSuccess || nb < 1) nb = 1;
                occ.emplace_back(kern, nb);
            }
        }
        const int cap = c->nsm * nb, g = c->lv[l].ntiles;
        return g < cap ? (g > 0 ? g : 1) : cap;
    }
    int grid_res(const void* kern, int l) const {
        static std::mutex mu;
        static std::vector<std::pair<const void*, int>> occ;
        int nb = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto& e : occ)
                if (e.first == kern) nb = e.second;
            if (nb == 0) {
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TPB, 0) != cudaSuccess || nb < 1) nb = 1;
                if (nb > MAXBLOCKS_PER_SM) nb = MAXBLOCKS_PER_SM;  // the partial-sum buffer's bound
                occ.emplace_back(kern, nb);
            }
        }
        const int wpb = TPB / 32, cap = c->nsm * nb;
        const int g = (c->lv[l].ntiles + wpb - 1) / wpb;
        return g < cap ? (g > 0 ? g : 1) : cap;
    }
    int grid_w(int l) const {
        const int wpb = TPB / 32, cap = c->nsm * MAXBLOCKS_PER_SM;
        const int g = (c->lv[l].ntiles + wpb - 1) / wpb;
        return g < cap ? (g > 0 ? g : 1) : cap;
    }

    void beg(int f, int l) {
        nk++;
        if (!c->prof_on) return;
        fam = f;
        lvl = l;
        ev0 = prof_event(c);
        cudaEventRecord(ev0, s);
    }
    void end() {
        if (!c->prof_on) return;
        cudaEvent_t ev1 = prof_event(c);
        cudaEventRecord(ev1, s);
        c->pending.push_back(ProfRec{fam, lvl, ev0, ev1});
    }

    // volume(s) and gamma (src/flip.jl:1146-1147)
    void volume(const float* phi) {
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        beg(F_VOLUME, -1);
        launch(k_volume, grid_cells(c, N), TPB, 0, s, geo_of(c->grid), phi, c->sc, c->partials, cnt(CNT_VOLUME));
        end();
    }

    // The fine set-up pass, the coarse levels and the tile lists.
    void setup(const SetupIn<V>& in, cudaGraphConditionalHandle cond, int use_cond) {
        cudaMemsetAsync(c->tflag_all, 0, c->tflag_bytes, s);
        cudaMemsetAsync(c->edges, 0, sizeof(int) * MAXLEV, s);
        // Level residuals and coarse corrections start at zero each projection, so every cell
        // outside the active tiles reads as zero in the staged restriction/prolongation.
        const size_t ms = msize(c->prec);
        for (int l = 0; l < c->lb; l++) {
            const size_t Nl = (size_t)c->lv[l].n[0] * c->lv[l].n[1] * c->lv[l].n[2];
            cudaMemsetAsync(c->lv[l].r, 0, ms * Nl, s);
            if (l > 0) cudaMemsetAsync(c->lv[l].x, 0, ms * Nl, s);
        }
        // The coarse levels need only the classes: they are built on a second stream beside
        // the fine set-up pass, joined before the tile lists.
        const cudaStream_t s0 = s;
        const bool fork = !c->in_batch;
        if (fork) {
            cudaEventRecord(c->ev_fork, s);
            cudaStreamWaitEvent(c->aux, c->ev_fork, 0);
            s = c->aux;
        }
        for (int l = 1; l < c->L; l++) {
            const LevelBuf& f = c->lv[l - 1];
            const uint8_t* tf = l == 1 ? in.types : f.types;
            const int64_t Nl = (int64_t)c->lv[l].n[0] * c->lv[l].n[1] * c->lv[l].n[2];
            beg(F_LEVEL, l);
            launch(k_level<Pr>, grid_cells(c, Nl), TPB, 0, s, tf, f.n[0], f.n[1], f.n[2], view<M>(c, l),
                                                           c->lv[l].split ? 1 : 0);
            end();
        }
        if (fork) cudaEventRecord(c->ev_join, c->aux);
        s = s0;
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        beg(F_SETUP, -1);
        auto al = [](const void* q, uintptr_t a) { return (reinterpret_cast<uintptr_t>(q) & (a - 1)) == 0; };
        // SETUP_W cells of a row per thread, with SETUP_W-byte loads of the caller's classes and
        // 16-byte ones of its faces
        if (c->grid.n[0] % SETUP_W == 0 && al(in.types, SETUP_W) && (!in.v || al(in.v, 16)) &&
            (!in.w || al(in.w, 16)) && al(in.P, 16) && (!in.phi || al(in.phi, 16)))
            launch(k_setup_v8<Pr, SETUP_W>, grid_cells(c, (N / SETUP_W) * TPB / SETUP_V8_TPB), SETUP_V8_TPB, 0, s, in,
                   view<M>(c, 0), (V*)c->diag, (V*)c->bvec, (V*)c->r, c->sc, c->partials, cnt(CNT_SETUP), cond,
                   use_cond);
        else
            launch(k_setup<Pr>, grid_cells(c, N), TPB, 0, s, in, view<M>(c, 0), (V*)c->diag, (V*)c->bvec, (V*)c->r,
                   c->sc, c->partials, cnt(CNT_SETUP), cond, use_cond);
        end();
        if (fork) cudaStreamWaitEvent(s, c->ev_join, 0);
        TileTab tab;
        memset(&tab, 0, sizeof(tab));
        tab.nlev = c->lb;
        for (int l = 0; l < c->lb; l++) {
            tab.ntiles[l] = c->lv[l].ntiles;
            tab.GH[l] = c->lv[l].GH;
            tab.GJ[l] = c->lv[l].GJ;
            tab.flags[l] = c->lv[l].tflag;
            tab.tiles[l] = c->lv[l].tiles;
            tab.count[l] = c->lv[l].count;
        }
        beg(F_TILES, -1);
        launch(k_tilelists, tab.nlev, 1024, 0, s, tab);
        end();
    }

    // b_late: the first pass follows a kernel that wrote the level's b (the restriction
    // with the level's start fused in)
    void smooth(int l, const std::vector<int>& colours, bool b_late = false) {
        // the async-copy form exists for 16-bit storage; the others take the vector form
        bool async = false;
        if constexpr (sizeof(M) == 2)
            async = form(l) == MPP_SMOOTHER_ASYNC && c->lv[l].H % V8 == 0 && c->async_blocks > 0;
        for (int col : colours) {
            beg(F_RBGS, l);
            if (form(l) == MPP_SMOOTHER_TMA && c->tma_ok[l]) {
                const int g = c->lv[l].ntiles < c->tma_blocks ? c->lv[l].ntiles : c->tma_blocks;
                launch(k_rbgs_tma<Pr>, g > 0 ? g : 1, TPB, TmaGeom<M>::SMEM, s, view<M>(c, l), col, c->tma[l],
                                                                           &c->sc->s.fault);
            } else if (async) {
                if constexpr (sizeof(M) == 2) {
                    const int wpb = TPB / 32;
                    int g = (c->lv[l].ntiles + wpb - 1) / wpb;
                    g = g < c->async_blocks ? (g > 0 ? g : 1) : c->async_blocks;
                    launch(k_rbgs_async<Pr>, g, TPB, AS_SMEM, s, view<M>(c, l), col);
                }
            } else if (form(l) != MPP_SMOOTHER_COLUMN && c->lv[l].H % V8 == 0) {
                const int wpb = TPB / 32, cap = c->nsm * RBGS_V8_BLOCKS;
                int g = (c->lv[l].ntiles + wpb - 1) / wpb;
                g = g < cap ? (g > 0 ? g : 1) : cap;
                launch(k_rbgs_v8<Pr>, g, TPB, 0, s, view<M>(c, l), col, b_late ? 1 : 0);
                b_late = false;
            } else {
                launch(k_rbgs<Pr>, grid_tiles(c, l), TPB, 0, s, view<M>(c, l), col);
            }
            end();
        }
    }

    // start_kernel! on the fine level (the first colour's first sweep of a V-cycle). serial:
    // it follows the tile lists' build (its tile ids load before its wait).
    void start0(bool serial = false) {
        beg(F_START, 0);
        if (vec(0)) {
            if (serial) launch_serial(k_start_v8<Pr>, grid_res((const void*)k_start_v8<Pr>, 0), TPB, 0, s, view<M>(c, 0));
            else launch(k_start_v8<Pr>, grid_res((const void*)k_start_v8<Pr>, 0), TPB, 0, s, view<M>(c, 0));
        } else {
            launch(k_start<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0));
        }
        end();
    }
    // vcycle! (src/flip.jl:992-1014): z = M^-1 r from zero. with_start = false: the fine
    // level's start already ran (the CG loop's: after the set-up, and in the step).
    void vcycle(bool with_start = true) {
        // sweeps of the fine level and of the coarser ones (the reference's one `sweeps`
        // unless sweeps_coarse is set)
        const int swf = c->opts.sweeps, sw = c->opts.sweeps_coarse > 0 ? c->opts.sweeps_coarse : swf;
        std::vector<int> down, up, down0, up0;
        for (int q = 0; q < sw; q++) { down.push_back(0); down.push_back(1); }
        down.erase(down.begin());  // the start kernel is the first colour's first sweep
        for (int q = 0; q < sw; q++) { up.push_back(1); up.push_back(0); }
        for (int q = 0; q < swf; q++) { down0.push_back(0); down0.push_back(1); }
        down0.erase(down0.begin());
        for (int q = 0; q < swf; q++) { up0.push_back(1); up0.push_back(0); }
        const int lb = c->lb;
        const int ls = c->cmg_ls > 0 ? c->cmg_ls : lb;  // levels ls .. lb-1 in the cluster
        for (int l = 0; l < ls; l++) {
            if (l == 0 && with_start) start0();  // the coarser levels' starts ride on the restriction
            // b of the level's first pass waits for the preceding kernel where that kernel wrote
            // it: the restriction that started a coarse level, the step that started level 0
            smooth(l, l == 0 ? down0 : down, l > 0 || !with_start);
            beg(F_RESID, l);
            if (vec(l)) launch(k_residual_v8<Pr>, grid_res((const void*)k_residual_v8<Pr>, l), TPB, 0, s, view<M>(c, l));
            else launch(k_residual<Pr>, grid_tiles(c, l), TPB, 0, s, view<M>(c, l));
            end();
            if (l + 1 < lb) {
                beg(F_RESTRICT, l + 1);
                launch(k_restrict<Pr>, grid_blk((const void*)k_restrict<Pr>, l + 1, c->restrict_smem), TPB, c->restrict_smem, s, view<M>(c, l), view<M>(c, l + 1),
                       l + 1 < ls ? 1 : 0);
                end();
            }
        }
        BotArgs ba = c->bot;
        ba.sweeps = sw;
        ba.coarse = c->opts.coarse;
        CmgArgs<M> ca;
        if (ls < lb) {
            memset(&ca, 0, sizeof(ca));
            ca.nl = lb - ls;
            ca.sweeps = sw;
            ca.botb = c->botb;
            for (int l = ls; l <= lb; l++) ca.g[l - ls] = view<M>(c, l);
            for (int l = ls; l < lb; l++) ca.s[l - ls] = c->cmg_slab[l - ls];
            beg(F_CMG, 0);
            launch_cluster(k_cmg<Pr, 0>, c->cmg_cs, CMG_THREADS, c->cmg_smem, s, ca);
            end();
        } else {
            const int64_t Nb = (int64_t)c->lv[lb].n[0] * c->lv[lb].n[1] * c->lv[lb].n[2];
            beg(F_RESTRICT, lb);
            launch(k_restrict_bottom<Pr>, grid_cells(c, Nb), TPB, 0, s, view<M>(c, lb - 1), view<M>(c, lb),
                                                                    (typename Pr::C*)c->botb);
            end();
        }
        beg(F_BOTTOM, lb);
        launch(k_bottom<Pr>, 1, 1024, c->bot_smem, s, (const typename Pr::C*)c->botb, (M*)c->lv[lb].x, ba);
        end();
        if (ls < lb) {
            beg(F_CMG, 1);
            launch_cluster(k_cmg<Pr, 1>, c->cmg_cs, CMG_THREADS, c->cmg_smem, s, ca);
            end();
        }
        for (int l = ls - 1; l >= 0; l--) {
            beg(F_PROLONG, l);
            if (vec(l))
                launch(k_prolong_v8<Pr>, grid_w(l), TPB, 0, s, view<M>(c, l), view<M>(c, l + 1), l + 1 == lb ? 1 : 0);
            else
                launch(k_prolong<Pr>, grid_tiles(c, l), TPB, 0, s, view<M>(c, l), view<M>(c, l + 1), l + 1 == lb ? 1 : 0);
            end();
            smooth(l, l == 0 ? up0 : up);
        }
    }

    // One CG iteration, rotated so a loop of them is pressure!'s loop (src/flip.jl:1095-1108):
    // z = M^-1 r, rho/beta, q = A p and alpha, then the step and the exit test.
    // The next V-cycle's fine start is part of the step: the vector step writes it (the b
    // it has just formed, over the stored reciprocal diagonal or diagonal), otherwise the start
    // kernel follows the step; the set-up is followed by one (record_prologue).
    void body(V* P, cudaGraphConditionalHandle cond, int use_cond) {
        vcycle(false);
        const bool v = vec(0);
        beg(F_DOT, 0);
        if (v)
            launch(k_dot_v8<Pr>, grid_res((const void*)k_dot_v8<Pr>, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->r, (const V*)c->q, c->sc, c->partials,
                                                    cnt(CNT_DOT));
        else
            launch(k_dot<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->r, (const V*)c->q, c->sc,
                                                        c->partials, cnt(CNT_DOT));
        end();
        beg(F_SEARCH, 0);
        if (v)
            launch(k_search_v8<Pr>, grid_res((const void*)k_search_v8<Pr>, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->d, (const V*)c->diag, (V*)c->q,
                                                       c->sc, c->partials, cnt(CNT_SEARCH));
        else
            launch(k_search<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->d, (const V*)c->diag, (V*)c->q,
                                                           c->sc, c->partials, cnt(CNT_SEARCH));
        end();
        beg(F_ADVANCE, 0);
        // the vector step moves P in 16-element runs: it needs a 16-byte aligned P
        if (v && (reinterpret_cast<uintptr_t>(P) & 15) == 0)
            launch(k_advance_v8<Pr>, grid_w(0), TPB, 0, s, view<M>(c, 0), (V*)c->d, (const V*)c->q, (V*)c->r, P, c->sc,
                                                        c->partials, cnt(CNT_ADVANCE), cond, use_cond, 1);
        else
            launch(k_advance<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (V*)c->d, (const V*)c->q, (V*)c->r, P,
                                                            c->sc, c->partials, cnt(CNT_ADVANCE), cond, use_cond);
        end();
        if (!(v && (reinterpret_cast<uintptr_t>(P) & 15) == 0)) start0();
    }

    void true_residual(const V* P) {
        beg(F_TRUE, 0);
        launch(k_true_residual<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->bvec, (const V*)c->diag, P,
                                                              nullptr, c->sc, c->partials, cnt(CNT_TRUE));
        end();
    }

    void gradient(float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw, const float* P,
                  const uint8_t* types, const float* phi) {
        const int64_t N = (int64_t)(c->grid.n[0] + 1) * (c->grid.n[1] + 1) * (c->grid.n[2] + 1);
        beg(F_GRADIENT, -1);
        auto al = [](const void* q, uintptr_t a) { return (reinterpret_cast<uintptr_t>(q) & (a - 1)) == 0; };
        if (c->grid.n[0] % 4 == 0 && phi && al(P, 16) && al(phi, 16) && al(v, 16) && al(w, 16) && al(types, 4) &&
            al(fv, 4) && al(fw, 4))
            launch(k_gradient_v4, grid_cells(c, N / 4), TPB, 0, s, c->grid.n[0], c->grid.n[1], c->grid.n[2], u, v, w,
                   fu, fv, fw, P, types, phi, c->grid.dx);
        else
            launch(k_gradient, grid_cells(c, N), TPB, 0, s, c->grid.n[0], c->grid.n[1], c->grid.n[2], u, v, w, fu, fv,
                   fw, P, types, phi, c->grid.dx);
        end();
    }

    void widen(const float* P) {
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        beg(F_CONVERT, -1);
        launch(k_widen, grid_cells(c, N), TPB, 0, s, (double*)c->Pd, P, N);
        end();
    }
    void narrow(float* P) {
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        beg(F_CONVERT, -1);
        launch(k_narrow, grid_cells(c, N), TPB, 0, s, P, (const double*)c->Pd, N);
        end();
    }
};

// A launch of `ny` thread-block clusters of `cs` CTAs side by side (blockIdx.y: the basin of
// a group), with programmatic dependent launch.
template <typename... KArgs, typename... Args>
void launch_clusters(void (*kern)(KArgs...), int cs, int ny, int block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cs, (unsigned)ny);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    at[1].id = cudaLaunchAttributeClusterDimension;
    at[1].val.clusterDim.x = (unsigned)cs;
    at[1].val.clusterDim.y = 1;
    at[1].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// A group's CG loop body: Run<Pr>::body's launch sequence with every launch covering the
// group's basins (grid y), each basin's grid width as its own solve's (run0 computes them for
// the first basin; every basin of a group has the same grid, options and forms).
template <class Pr>
struct GroupRun {
    using V = typename Pr::V;
    using M = typename Pr::M;
    using C = typename Pr::C;
    std::vector<mpp_ctx*> cs;
    std::vector<V*> P;  // each basin's pressure (the caller's array)
    cudaStream_t s;
    int nk = 0;
    Run<Pr> run0;

    GroupRun(const std::vector<mpp_ctx*>& ctxs, const std::vector<V*>& Ps, cudaStream_t st)
        : cs(ctxs), P(Ps), s(st), run0{ctxs[0], st} {}
    int nb() const { return (int)cs.size(); }
    const mpp_ctx* c0() const { return cs[0]; }
    dim3 g2(int gx) const { return dim3((unsigned)gx, (unsigned)nb()); }
    static const int* done_of(const mpp_ctx* c) { return &c->sc->s.done; }

    Grp<GLev<M>> lev(int l) const {
        Grp<GLev<M>> g;
        memset(&g, 0, sizeof(g));
        for (int i = 0; i < nb(); i++) g.a[i] = GLev<M>{view<M>(cs[i], l), done_of(cs[i])};
        return g;
    }
    Grp<GLev2<M>> lev2(int f, int cl) const {
        Grp<GLev2<M>> g;
        memset(&g, 0, sizeof(g));
        for (int i = 0; i < nb(); i++) g.a[i] = GLev2<M>{view<M>(cs[i], f), view<M>(cs[i], cl), done_of(cs[i])};
        return g;
    }
    Grp<GCg<M, V>> cg() const {
        Grp<GCg<M, V>> g;
        memset(&g, 0, sizeof(g));
        for (int i = 0; i < nb(); i++) {
            mpp_ctx* c = cs[i];
            g.a[i] = GCg<M, V>{view<M>(c, 0), (V*)c->r, (V*)c->q, (V*)c->d, P[i], (const V*)c->diag,
                               c->sc, c->partials, c->counters};
        }
        return g;
    }
    // the counters of a CG pass (each basin's own, at the same index as its single solve's)
    Grp<GCg<M, V>> cg_at(int cnt) const {
        Grp<GCg<M, V>> g = cg();
        for (int i = 0; i < nb(); i++) g.a[i].counter = cs[i]->counters + cnt;
        return g;
    }

    void smooth(int l, const std::vector<int>& colours, bool b_late) {
        const mpp_ctx* c = c0();
        bool async = false;
        if constexpr (sizeof(M) == 2)
            async = run0.form(l) == MPP_SMOOTHER_ASYNC && c->lv[l].H % V8 == 0 && c->async_blocks > 0;
        const auto g = lev(l);
        for (int col : colours) {
            nk++;
            if (async) {
                if constexpr (sizeof(M) == 2) {
                    const int wpb = TPB / 32;
                    int gx = (c->lv[l].ntiles + wpb - 1) / wpb;
                    gx = gx < c->async_blocks ? (gx > 0 ? gx : 1) : c->async_blocks;
                    launch(k_rbgs_async_g<Pr>, g2(gx), TPB, AS_SMEM, s, g, col);
                }
            } else if (run0.form(l) != MPP_SMOOTHER_COLUMN && c->lv[l].H % V8 == 0) {
                const int wpb = TPB / 32, cap = c->nsm * RBGS_V8_BLOCKS;
                int gx = (c->lv[l].ntiles + wpb - 1) / wpb;
                gx = gx < cap ? (gx > 0 ? gx : 1) : cap;
                launch(k_rbgs_v8_g<Pr>, g2(gx), TPB, 0, s, g, col, b_late ? 1 : 0);
                b_late = false;
            } else {
                launch(k_rbgs_g<Pr>, g2(grid_tiles(c, l)), TPB, 0, s, g, col);
            }
        }
    }

    void start0() {
        const mpp_ctx* c = c0();
        nk++;
        if (run0.vec(0))
            launch(k_start_v8_g<Pr>, g2(run0.grid_res((const void*)k_start_v8<Pr>, 0)), TPB, 0, s, lev(0));
        else
            launch(k_start_g<Pr>, g2(grid_tiles(c, 0)), TPB, 0, s, lev(0));
    }
    void vcycle(bool with_start = true) {
        const mpp_ctx* c = c0();
        const int swf = c->opts.sweeps, sw = c->opts.sweeps_coarse > 0 ? c->opts.sweeps_coarse : swf;
        std::vector<int> down, up, down0, up0;
        for (int q = 0; q < sw; q++) { down.push_back(0); down.push_back(1); }
        down.erase(down.begin());
        for (int q = 0; q < sw; q++) { up.push_back(1); up.push_back(0); }
        for (int q = 0; q < swf; q++) { down0.push_back(0); down0.push_back(1); }
        down0.erase(down0.begin());
        for (int q = 0; q < swf; q++) { up0.push_back(1); up0.push_back(0); }
        const int lb = c->lb;
        const int ls = c->cmg_ls > 0 ? c->cmg_ls : lb;
        for (int l = 0; l < ls; l++) {
            if (l == 0 && with_start) start0();
            // b of the level's first pass waits for the preceding kernel where that kernel wrote
            // it: the restriction that started a coarse level, the step that started level 0
            smooth(l, l == 0 ? down0 : down, l > 0 || !with_start);
            nk++;
            if (run0.vec(l))
                launch(k_residual_v8_g<Pr>, g2(run0.grid_res((const void*)k_residual_v8<Pr>, l)), TPB, 0, s, lev(l));
            else
                launch(k_residual_g<Pr>, g2(grid_tiles(c, l)), TPB, 0, s, lev(l));
            if (l + 1 < lb) {
                nk++;
                launch(k_restrict_g<Pr>, g2(run0.grid_blk((const void*)k_restrict_g<Pr>, l + 1, c->restrict_smem)), TPB,
                       c->restrict_smem, s, lev2(l, l + 1),
                       l + 1 < ls ? 1 : 0);
            }
        }
        Grp<GCmg<M>> gc;
        memset(&gc, 0, sizeof(gc));
        if (ls < lb) {
            for (int i = 0; i < nb(); i++) {
                mpp_ctx* ci = cs[i];
                CmgArgs<M>& ca = gc.a[i].a;
                ca.nl = lb - ls;
                ca.sweeps = sw;
                ca.botb = ci->botb;
                for (int l = ls; l <= lb; l++) ca.g[l - ls] = view<M>(ci, l);
                for (int l = ls; l < lb; l++) ca.s[l - ls] = ci->cmg_slab[l - ls];
                gc.a[i].done = done_of(ci);
            }
            nk++;
            launch_clusters(k_cmg_g<Pr, 0>, c->cmg_cs, nb(), CMG_THREADS, c->cmg_smem, s, gc);
        } else {
            Grp<GRestrictBottom<M, C>> gr;
            memset(&gr, 0, sizeof(gr));
            for (int i = 0; i < nb(); i++)
                gr.a[i] = GRestrictBottom<M, C>{view<M>(cs[i], lb - 1), view<M>(cs[i], lb), (C*)cs[i]->botb,
                                                done_of(cs[i])};
            const int64_t Nb = (int64_t)c->lv[lb].n[0] * c->lv[lb].n[1] * c->lv[lb].n[2];
            nk++;
            launch(k_restrict_bottom_g<Pr>, g2(grid_cells(c, Nb)), TPB, 0, s, gr);
        }
        Grp<GBottom<M, C>> gb;
        memset(&gb, 0, sizeof(gb));
        for (int i = 0; i < nb(); i++) {
            BotArgs ba = cs[i]->bot;
            ba.sweeps = sw;
            ba.coarse = cs[i]->opts.coarse;
            gb.a[i] = GBottom<M, C>{(const C*)cs[i]->botb, (M*)cs[i]->lv[lb].x, ba, done_of(cs[i])};
        }
        nk++;
        launch(k_bottom_g<Pr>, g2(1), 1024, c->bot_smem, s, gb);
        if (ls < lb) {
            nk++;
            launch_clusters(k_cmg_g<Pr, 1>, c->cmg_cs, nb(), CMG_THREADS, c->cmg_smem, s, gc);
        }
        for (int l = ls - 1; l >= 0; l--) {
            nk++;
            if (run0.vec(l))
                launch(k_prolong_v8_g<Pr>, g2(run0.grid_w(l)), TPB, 0, s, lev2(l, l + 1), l + 1 == lb ? 1 : 0);
            else
                launch(k_prolong_g<Pr>, g2(grid_tiles(c, l)), TPB, 0, s, lev2(l, l + 1), l + 1 == lb ? 1 : 0);
            smooth(l, l == 0 ? up0 : up, false);
        }
    }

    // Run<Pr>::body for the group, then the group's loop condition.
    void body(cudaGraphConditionalHandle cond) {
        const mpp_ctx* c = c0();
        vcycle(false);
        const bool v = run0.vec(0);
        nk += 4;
        if (v) launch(k_dot_v8_g<Pr>, g2(run0.grid_res((const void*)k_dot_v8<Pr>, 0)), TPB, 0, s, cg_at(CNT_DOT));
        else launch(k_dot_g<Pr>, g2(grid_tiles(c, 0)), TPB, 0, s, cg_at(CNT_DOT));
        if (v) launch(k_search_v8_g<Pr>, g2(run0.grid_res((const void*)k_search_v8<Pr>, 0)), TPB, 0, s, cg_at(CNT_SEARCH));
        else launch(k_search_g<Pr>, g2(grid_tiles(c, 0)), TPB, 0, s, cg_at(CNT_SEARCH));
        bool aligned = true;  // the vector step moves P in 16-element runs
        for (V* p : P) aligned = aligned && (reinterpret_cast<uintptr_t>(p) & 15) == 0;
        if (v && aligned) launch(k_advance_v8_g<Pr>, g2(run0.grid_w(0)), TPB, 0, s, cg_at(CNT_ADVANCE), 1);
        else launch(k_advance_g<Pr>, g2(grid_tiles(c, 0)), TPB, 0, s, cg_at(CNT_ADVANCE));
        if (!(v && aligned)) start0();
        Grp<const int*> d;
        memset(&d, 0, sizeof(d));
        for (int i = 0; i < nb(); i++) d.a[i] = done_of(cs[i]);
        launch(k_group_cond, 1, 1, 0, s, d, nb(), cond);
    }
};
static_assert(sizeof(Grp<GCmg<double>>) < 32000, "a group launch's arguments fit the kernel parameter space");

int write_params(mpp_ctx* c, float volume0, double dt, double recover, int project, float gamma, cudaStream_t s) {
    Params& p = c->sc_host->p;
    p.volume0 = volume0;
    p.tol = c->opts.tol;
    p.dt = dt;
    p.recover = recover;
    // with the fallback on, CG gets at most cg_maxiter_with_fallback iterations (src/fgmres.jl:99)
    p.maxiter = c->opts.fallback ? std::min(c->opts.maxiter, c->opts.cg_maxiter_with_fallback) : c->opts.maxiter;
    p.project = project;
    p.gamma = gamma;
    CK(cudaMemcpyAsync(&c->sc->p, &c->sc_host->p, sizeof(Params), cudaMemcpyHostToDevice, s));
    return MPP_OK;
}

int read_state(mpp_ctx* c, cudaStream_t s) {
    CK(cudaMemcpyAsync(&c->sc_host->s, &c->sc->s, sizeof(State), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return MPP_OK;
}

struct Call {
    // project (kind 1) or pressure (kind 0)
    int kind;
    float *u, *v, *w;
    uint8_t *fu, *fv, *fw;
    float* P;
    const float* bnat;
    const uint8_t* types;
    const float* phi;
    const double* bnat64;  // FP64 rhs (the FP64 adjoint), or null
};

template <class Pr>
SetupIn<typename Pr::V> setup_in(mpp_ctx* c, const Call& k) {
    using V = typename Pr::V;
    SetupIn<V> in;
    in.u = k.kind == 1 ? k.u : nullptr;
    in.v = k.kind == 1 ? k.v : nullptr;
    in.w = k.kind == 1 ? k.w : nullptr;
    in.bnat = k.kind == 1 ? nullptr : k.bnat;
    in.bnat64 = k.kind == 1 ? nullptr : k.bnat64;
    in.P = std::is_same<V, double>::value ? (V*)c->Pd : (V*)k.P;
    in.types = k.types;
    in.phi = k.phi;
    in.dx = c->grid.dx;
    in.clear_P = k.kind == 1;
    in.residual = 1;
    return in;
}

// The prologue and epilogue of a solve, recorded on stream s.
template <class Pr>
void record_prologue(Run<Pr>& run, const Call& k, cudaGraphConditionalHandle cond, int use_cond) {
    if (k.kind == 1) run.volume(k.phi);
    if (std::is_same<typename Pr::V, double>::value) run.widen(k.P);
    run.setup(setup_in<Pr>(run.c, k), cond, use_cond);
    run.start0(true);  // the first V-cycle's fine start (the loop's steps write the later ones)
}

template <class Pr>
void record_epilogue(Run<Pr>& run, const Call& k) {
    using V = typename Pr::V;
    mpp_ctx* c = run.c;
    V* P = std::is_same<V, double>::value ? (V*)c->Pd : (V*)k.P;
    // the true residual (read only for the result and the fallback decision) on the second
    // stream, beside the gradient update; both only read the final P
    const cudaStream_t s0 = run.s;
    const bool fork = !c->in_batch;
    if (fork) {
        cudaEventRecord(c->ev_fork, s0);
        cudaStreamWaitEvent(c->aux, c->ev_fork, 0);
        run.s = c->aux;
    }
    run.true_residual(P);
    if (fork) cudaEventRecord(c->ev_join, c->aux);
    run.s = s0;
    if (std::is_same<V, double>::value) run.narrow(k.P);
    // with the fallback on, the gradient waits for the host's fallback decision
    if (k.kind == 1 && !c->opts.fallback) run.gradient(k.u, k.v, k.w, k.fu, k.fv, k.fw, k.P, k.types, k.phi);
    if (fork) cudaStreamWaitEvent(s0, c->ev_join, 0);
}

// ---- the FGMRES fallback (src/fgmres.jl:26-110, restated for the dense operator) ----
Lev<float> fine_layout(mpp_ctx* c);

// The Krylov workspace for `restart`, allocated on first use (outside any capture).
int fg_workspace(mpp_ctx* c, int R) {
    if (c->fg_restart >= R) return MPP_OK;
    if (c->fg_restart > 0) {
        set_err("the fallback's restart length cannot grow after its first use (%d > %d)", R, c->fg_restart);
        return MPP_ERR_INVALID;
    }
    const size_t N = (size_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    const size_t vs = vsize(c->prec), gd = guard_of(c->grid.n[0], c->grid.n[1]);
    if (int e = alloc(c, &c->fV, vs * N * (size_t)(R + 1))) return e;
    for (int j = 0; j < R; j++)
        if (int e = alloc_guarded(c, &c->fZ[j], vs, N, gd)) return e;
    if (int e = alloc(c, (void**)&c->fgd, sizeof(double) * (2 * (FG_MAXR + 1) + 1))) return e;
    CK(cudaMallocHost((void**)&c->fgd_host, sizeof(double) * (2 * (FG_MAXR + 1) + 1)));
    c->fg_restart = R;
    return MPP_OK;
}

// Restarted right-preconditioned flexible GMRES: basis V (FP32, or FP64 in the FP64 form)
// with two passes of modified Gram-Schmidt, z_j = M^-1 v_j by the V-cycle, FP64 Hessenberg
// and Givens rotations on the host, the true residual checked after every cycle. The
// Gram-Schmidt coefficients stay on the device (slot pass*(R+1)+i, the norm in slot
// 2*(R+1)); the host reads a column once, after its last kernel. Sets `status` and `its`.
template <class Pr>
int fgmres(mpp_ctx* c, cudaStream_t s, typename Pr::V* P, int& its, int& status) {
    using V = typename Pr::V;
    using M = typename Pr::M;
    Run<Pr> run{c, s};
    const Lev<float> L = fine_layout(c);
    const size_t N = (size_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    const int R = c->opts.restart, maxit = c->opts.fallback_maxiter;
    const int gtw = grid_tiles(c, 0);
    const int NS = 2 * (FG_MAXR + 1) + 1, SN = 2 * (FG_MAXR + 1);
    auto vec = [&](int i) { return reinterpret_cast<V*>(c->fV) + (size_t)i * N; };
    auto zv = [&](int i) { return reinterpret_cast<V*>(c->fZ[i]); };
    V* q = reinterpret_cast<V*>(c->q);
    V* r = reinterpret_cast<V*>(c->r);
    double residual = 0.0;
    auto finish = [&]() -> int {
        c->fg_residual = residual;
        c->launches += run.nk;
        run.nk = 0;
        CK(cudaGetLastError());
        return MPP_OK;
    };
    auto true_res = [&](double& res) -> int {  // r = b - A P and its norm (src/fgmres.jl:35-40)
        run.nk++;
        launch(k_true_residual<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->bvec, (const V*)c->diag,
               (const V*)P, r, c->sc, c->partials, run.cnt(CNT_TRUE));
        if (int e = read_state(c, s)) return e;
        res = sqrt(c->sc_host->s.true_rr);
        return MPP_OK;
    };
    // the V-cycle's input is scaled so 16-bit storage keeps its precision (M^-1 is linear):
    // a unit vector's entries are ~1/sqrt(n), scaled to ~1/4
    const double nliq = c->sc_host->s.nliq > 0 ? (double)c->sc_host->s.nliq : 1.0;
    const double cyc = Pr::scaled ? exp2(rint(log2(0.25 * sqrt(nliq)))) : 1.0;
    const double bnorm = c->sc_host->s.bnorm;
    its = 0;
    status = MPP_OK;
    if (!std::isfinite(bnorm)) {
        status = MPP_NONFINITE;  // "Nonfinite pressure RHS" (src/fgmres.jl:31)
        return MPP_OK;
    }
    if (bnorm == 0.0) {
        run.nk++;
        launch(k_fg_zero_P<V>, gtw, TPB, 0, s, L, P);
        return finish();
    }
    if (int e = fg_workspace(c, R)) return e;
    const double target = (double)c->opts.tol * bnorm;
    if (int e = true_res(residual)) return e;
    std::vector<double> H((size_t)(R + 1) * R), g(R + 1), cs(R), sn(R), y(R);
    auto Hs = [&](int i, int j) -> double& { return H[(size_t)i * R + j]; };
    while (residual > target && its < maxit) {
        if (!std::isfinite(residual)) {
            status = MPP_NONFINITE;  // "Nonfinite pressure residual" (src/fgmres.jl:46)
            return finish();
        }
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = residual;
        run.nk++;
        launch(k_fg_scale<V>, gtw, TPB, 0, s, L, vec(0), (const V*)r, 1.0 / residual);
        int used = 0;
        for (int j = 0; j < R && its < maxit; j++) {
            run.nk++;
            launch(k_fg_to_cycle<M, V>, gtw, TPB, 0, s, L, (M*)c->lv[0].b, (const V*)vec(j), cyc);
            run.vcycle();
            run.nk += 2;
            launch(k_fg_from_cycle<M, V>, gtw, TPB, 0, s, L, zv(j), (const M*)c->lv[0].x, 1.0 / cyc);
            launch(k_apply<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)zv(j), (const V*)c->diag, q);
            // twice-repeated modified Gram-Schmidt (src/fgmres.jl:59-63)
            for (int pass = 0; pass < 2; pass++)
                for (int i = 0; i <= j; i++) {
                    const int slot = pass * (FG_MAXR + 1) + i;
                    run.nk += 2;
                    launch(k_fg_dot<V>, gtw, TPB, 0, s, L, (const V*)q, (const V*)vec(i), c->fgd, slot, c->partials,
                           run.cnt(CNT_FG));
                    launch(k_fg_orth<V>, gtw, TPB, 0, s, L, q, (const V*)vec(i), (const double*)c->fgd, slot);
                }
            run.nk += 2;
            launch(k_fg_dot<V>, gtw, TPB, 0, s, L, (const V*)q, (const V*)q, c->fgd, SN, c->partials, run.cnt(CNT_FG));
            launch(k_fg_normalize<V>, gtw, TPB, 0, s, L, vec(j + 1), (const V*)q, (const double*)c->fgd, SN);
            CK(cudaMemcpyAsync(c->fgd_host, c->fgd, sizeof(double) * NS, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (int i = 0; i <= j; i++) Hs(i, j) = c->fgd_host[i] + c->fgd_host[FG_MAXR + 1 + i];
            const double hnext = sqrt(c->fgd_host[SN]);
            if (!std::isfinite(hnext)) {
                status = MPP_NONFINITE;  // "Nonfinite pressure Arnoldi vector" (src/fgmres.jl:65)
                return finish();
            }
            Hs(j + 1, j) = hnext;
            for (int i = 0; i < j; i++) {
                const double a = Hs(i, j), b = Hs(i + 1, j);
                Hs(i, j) = cs[i] * a + sn[i] * b;
                Hs(i + 1, j) = -sn[i] * a + cs[i] * b;
            }
            const double a = Hs(j, j), b = Hs(j + 1, j);
            const double hyp = std::hypot(a, b);
            if (!(hyp > 0.0)) {
                status = MPP_BREAKDOWN;  // "Pressure Arnoldi breakdown" (src/fgmres.jl:77)
                return finish();
            }
            cs[j] = a / hyp;
            sn[j] = b / hyp;
            Hs(j, j) = hyp;
            Hs(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            used = j + 1;
            its++;
            if (std::fabs(g[j + 1]) <= target || hnext == 0.0) break;
        }
        for (int i = used - 1; i >= 0; i--) {  // UpperTriangular(H) \ g (src/fgmres.jl:84)
            double t = g[i];
            for (int k = i + 1; k < used; k++) t -= Hs(i, k) * y[k];
            y[i] = t / Hs(i, i);
        }
        for (int j = 0; j < used; j++) {
            run.nk++;
            launch(k_fg_update_P<V>, gtw, TPB, 0, s, L, P, (const V*)zv(j), y[j]);
        }
        if (int e = true_res(residual)) return e;
    }
    status = residual <= target ? MPP_OK : MPP_NOT_CONVERGED;  // src/fgmres.jl:90
    return finish();
}

// After the CG solve with the fallback on (src/fgmres.jl:96-110): keep CG's pressure when its
// true residual meets tol; else zero P if that residual is nonfinite or above 2|b|, run FGMRES,
// and then (project!) the gradient update.
template <class Pr>
int fallback_and_finish(mpp_ctx* c, const Call& k, cudaStream_t s) {
    using V = typename Pr::V;
    State& S = c->sc_host->s;
    c->fg_used = 0;
    c->fg_its = 0;
    const double target = (double)c->opts.tol * S.bnorm;
    const double tres = sqrt(S.true_rr);
    V* P = std::is_same<V, double>::value ? (V*)c->Pd : (V*)k.P;
    const bool cg_ok = S.status == MPP_OK && (S.bnorm == 0.0 || tres <= target);
    if (!cg_ok && std::isfinite(S.bnorm) && S.bnorm > 0.0) {
        const Lev<float> L = fine_layout(c);
        if (!std::isfinite(tres) || tres > 2.0 * S.bnorm) {
            launch(k_fg_zero_P<V>, grid_tiles(c, 0), TPB, 0, s, L, P);
            c->launches++;
        }
        int its = 0, st = 0;
        if (int e = fgmres<Pr>(c, s, P, its, st)) return e;
        c->fg_used = 1;
        c->fg_its = its;
        S.status = st;
        S.true_rr = c->fg_residual * c->fg_residual;
        if (std::is_same<V, double>::value) {
            Run<Pr> run{c, s};
            run.narrow(k.P);
            c->launches += run.nk;
        }
    }
    if (k.kind == 1) {
        Run<Pr> run{c, s};
        run.gradient(k.u, k.v, k.w, k.fu, k.fv, k.fw, k.P, k.types, k.phi);
        c->launches += run.nk;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return MPP_OK;
}

// Record one solve (prologue, the CG loop as a conditional WHILE node, epilogue) into
// graph g as a chain of its own: its first nodes have no dependencies, so the chains of
// several basins recorded into one graph run concurrently. counts = kernels per part.
template <class Pr>
int record_solve(mpp_ctx* c, const Call& k, cudaGraph_t g, int counts[3]) {
    using V = typename Pr::V;
    cudaStream_t s = c->cap;
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    Run<Pr> pro{c, s};
    CK(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    record_prologue<Pr>(pro, k, cond, 1);
    // the prologue's last nodes: the capture's current dependencies
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaStreamCaptureStatus cst;
    const cudaError_t qe = cudaStreamGetCaptureInfo(s, &cst, nullptr, nullptr, &deps, &nd);
    std::vector<cudaGraphNode_t> tail;
    if (qe == cudaSuccess) tail.assign(deps, deps + nd);
    cudaGraph_t gg = g;
    CK(cudaStreamEndCapture(s, &gg));
    CK(qe);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, g, tail.data(), tail.size(), &cp));
    cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
    Run<Pr> bod{c, s};
    CK(cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    V* P = std::is_same<V, double>::value ? (V*)c->Pd : (V*)k.P;
    bod.body(P, cond, 1);
    const cudaError_t le = cudaGetLastError();  // a launch refused during the capture
    CK(cudaStreamEndCapture(s, &bodyg));
    CK(le);
    Run<Pr> epi{c, s};
    CK(cudaStreamBeginCaptureToGraph(s, g, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
    record_epilogue<Pr>(epi, k);
    gg = g;
    CK(cudaStreamEndCapture(s, &gg));
    counts[0] = pro.nk;
    counts[1] = bod.nk;
    counts[2] = epi.nk;
    return MPP_OK;
}

template <class Pr>
int build_graph(mpp_ctx* c, const Call& k, GraphEntry& ge) {
    drop_graph(ge);
    cudaGraph_t g;
    CK(cudaGraphCreate(&g, 0));
    ge.graph = g;
    int counts[3];
    if (int e = record_solve<Pr>(c, k, g, counts)) return e;
    CK(cudaGraphInstantiate(&ge.exec, g, 0));
    ge.g_prologue = counts[0];
    ge.g_body = counts[1];
    ge.g_epilogue = counts[2];
    const void* key[11] = {k.u, k.v, k.w, k.fu, k.fv, k.fw, k.P, k.bnat, k.types, k.phi, k.bnat64};
    memcpy(ge.key, key, sizeof(key));
    ge.kind = k.kind;
    return MPP_OK;
}

// The cached graph of this call, captured on a miss into the least recently used slot.
template <class Pr>
int graph_for(mpp_ctx* c, const Call& k, GraphEntry*& out) {
    const void* key[11] = {k.u, k.v, k.w, k.fu, k.fv, k.fw, k.P, k.bnat, k.types, k.phi, k.bnat64};
    GraphEntry* victim = &c->gc[0];
    for (GraphEntry& e : c->gc) {
        if (e.exec && e.kind == k.kind && memcmp(key, e.key, sizeof(key)) == 0) {
            e.used = ++c->gclock;
            out = &e;
            return MPP_OK;
        }
        if (!e.exec || e.used < victim->used) victim = &e;
    }
    if (int e = build_graph<Pr>(c, k, *victim)) {
        drop_graph(*victim);
        return e;
    }
    victim->used = ++c->gclock;
    out = victim;
    return MPP_OK;
}

void drop_graphs(mpp_ctx* c) {
    for (GraphEntry& e : c->gc) drop_graph(e);
    c->gen++;  // a batch's graph over this context is stale too
}

template <class Pr>
int solve(mpp_ctx* c, const Call& k, cudaStream_t s) {
    using V = typename Pr::V;
    int64_t launched = 0;
    CK(cudaMemsetAsync(&c->sc->s.fault, 0, sizeof(int), s));
    if (c->opts.graph && !c->prof_on) {
        GraphEntry* ge = nullptr;
        if (int e = graph_for<Pr>(c, k, ge)) return e;
        CK(cudaGraphLaunch(ge->exec, s));
        if (int e = read_state(c, s)) return e;
        launched = ge->g_prologue + (int64_t)ge->g_body * c->sc_host->s.it + ge->g_epilogue;
    } else {
        Run<Pr> run{c, s};
        record_prologue<Pr>(run, k, 0, 0);
        if (int e = read_state(c, s)) return e;
        V* P = std::is_same<V, double>::value ? (V*)c->Pd : (V*)k.P;
        while (!c->sc_host->s.done) {
            run.body(P, 0, 0);
            if (int e = read_state(c, s)) return e;
        }
        record_epilogue<Pr>(run, k);
        if (int e = read_state(c, s)) return e;
        launched = run.nk;
        prof_collect(c);
    }
    CK(cudaGetLastError());
    c->launches += launched;
    if (c->sc_host->s.fault) {
        set_err("a bounded device wait (TMA pipeline) gave up; results are not valid");
        return MPP_ERR_CUDA;
    }
    c->fg_used = c->fg_its = 0;
    if (c->opts.fallback) return fallback_and_finish<Pr>(c, k, s);
    return MPP_OK;
}

template <class F>
int dispatch(int prec, F&& f) {
    switch (prec) {
        case MPP_PREC_FP32: return f(PrecFP32{});
        case MPP_PREC_MIXED_FP16: return f(PrecFP16{});
        case MPP_PREC_MIXED_BF16: return f(PrecBF16{});
        case MPP_PREC_FP64: return f(PrecFP64{});
    }
    set_err("unknown precision %d", prec);
    return MPP_ERR_INVALID;
}

void fill_result(mpp_ctx* c, mpp_result* res, int64_t launches) {
    if (!res) return;
    const State& S = c->sc_host->s;
    memset(res, 0, sizeof(*res));
    res->iterations = S.it;
    res->status = S.status;
    res->bnorm = S.bnorm;
    res->rel_residual = S.bnorm > 0 ? S.rnorm / S.bnorm : 0.0;
    res->true_rel_residual = S.bnorm > 0 ? sqrt(S.true_rr) / S.bnorm : 0.0;
    res->volume = S.vol;
    res->gamma = S.gamma;
    res->kernel_launches = launches;
    res->fallback_used = c->fg_used;
    res->fallback_iterations = c->fg_its;
}

int check_ctx(mpp_ctx* c) {
    if (!c) {
        set_err("null context");
        return MPP_ERR_INVALID;
    }
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev != c->dev) {
        set_err("context belongs to device %d, current device is %d", c->dev, dev);
        return MPP_ERR_INVALID;
    }
    return MPP_OK;
}

// Operator-only set-up shared by the single-pass entry points.
template <class Pr>
int operator_setup(mpp_ctx* c, Run<Pr>& run, const uint8_t* types, const float* phi, const float* u,
                   const float* v, const float* w, float gamma) {
    SetupIn<typename Pr::V> in;
    memset(&in, 0, sizeof(in));
    in.u = u;
    in.v = v;
    in.w = w;
    in.types = types;
    in.phi = phi;
    in.dx = c->grid.dx;
    in.clear_P = 0;
    in.residual = 0;
    if (int e = write_params(c, 1.f, 1.0, 1.0, 0, gamma, run.s)) return e;
    run.setup(in, 0, 0);
    return MPP_OK;
}

Lev<float> fine_layout(mpp_ctx* c) { return view<float>(c, 0); }

// ---- TMA tensor maps (cuTensorMapEncodeTiled through the runtime's driver entry point) ----
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// A row-split level array as 4-D (h, colour, j, k), h innermost; box {bx, 1, by, bz}.
bool encode_level(CUtensorMap* m, CUtensorMapDataType dt, void* base, size_t es, const LevelBuf& b, int bx, int by,
                  int bz) {
    auto enc = tma_encoder();
    if (!enc || !base) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)b.H, 2, (cuuint64_t)b.n[1], (cuuint64_t)b.n[2]};
    const cuuint64_t strides[3] = {(cuuint64_t)b.H * es, (cuuint64_t)b.n[0] * es,
                                   (cuuint64_t)b.n[0] * (cuuint64_t)b.n[1] * es};
    const cuuint32_t box[4] = {(cuuint32_t)bx, 1, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, dt, 4, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps for every row-split level whose rows are whole tiles (h extent a multiple of
// 16, so every box start is 16-byte aligned) and whose j and k extents hold a halo box.
// Levels without them, or with MPP_NO_TMA set in the environment, use k_rbgs.
// The cluster-resident small levels: the lowest first level ls >= 1 of at most 32^3 cells
// whose levels ls .. lb-1 fit, as z-slabs, in the shared memory of a cluster of 16 CTAs (8,
// 4 or 2 when 16 does not divide their plane counts or does not run). In the environment
// MPP_CMG=0 keeps the per-level launches, MPP_CMG_MAXCELLS sets the size bound and
// MPP_CMG_CS the largest cluster.
int build_cmg(mpp_ctx* c) {
    c->cmg_ls = 0;
    c->cmg_cs = 0;
    c->cmg_smem = 0;
    const char* env = getenv("MPP_CMG");
    if ((env && !strcmp(env, "0")) || c->lb < 2) return MPP_OK;
    // a level joins the cluster from this many cells down: 16 SMs run a pass over 32^3 cells
    // in well under the latency of one launch over the whole GPU, over 64^3 cells they do not
    int64_t maxcells = 32768;
    if (const char* mc = getenv("MPP_CMG_MAXCELLS")) maxcells = atoll(mc);
    int csmax = 16;
    if (const char* cm = getenv("MPP_CMG_CS")) csmax = atoi(cm);
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    const size_t ms = msize(c->prec);
    const bool half = ms == 2;
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        cudaFuncAttributes fa0, fa1;
        CK(cudaFuncGetAttributes(&fa0, k_cmg<Pr, 0>));
        CK(cudaFuncGetAttributes(&fa1, k_cmg<Pr, 1>));
        const size_t stat = fa0.sharedSizeBytes > fa1.sharedSizeBytes ? fa0.sharedSizeBytes : fa1.sharedSizeBytes;
        for (int ls = 1; ls < c->lb; ls++) {
            if (c->lb - ls > CMG_MAXLEV) continue;
            if ((int64_t)c->lv[ls].n[0] * c->lv[ls].n[1] * c->lv[ls].n[2] > maxcells) continue;
            for (int cs : {16, 8, 4, 2}) {
                if (cs > csmax) continue;
                bool ok = true;
                size_t off = CMG_HEADER;  // the active-row counts
                CmgSlab sl[CMG_MAXLEV];
                auto take = [&](size_t bytes) {
                    const unsigned o = (unsigned)off;
                    off += (bytes + 15) / 16 * 16;
                    return o;
                };
                for (int l = ls; l < c->lb && ok; l++) {
                    const LevelBuf& b = c->lv[l];
                    if (!b.split || b.n[0] % 2 || b.n[0] < 4 || b.n[2] % cs || b.n[1] > 65535) {
                        ok = false;
                        break;
                    }
                    CmgSlab& S = sl[l - ls];
                    S.n1 = b.n[0];
                    S.n2 = b.n[1];
                    S.n3 = b.n[2];
                    S.P = b.n[2] / cs;
                    S.H = S.n1 / 2;
                    auto magic = [](int d) { return d > 1 ? 0xFFFFFFFFu / (unsigned)d + 1u : 0u; };
                    S.mH = magic(S.H);
                    S.mN = magic(S.n1);
                    S.mP = magic(S.P);
                    const size_t n = (size_t)S.P * S.n1 * S.n2;
                    if (n >= 65536) {  // items of a pass are counted in 16 bits
                        ok = false;
                        break;
                    }
                    S.ox = take(ms * n);
                    S.ob = take(ms * n);
                    S.orr = take(ms * n);
                    S.ocode = take(n);
                    S.odg = take(ms * n);
                    S.odi = half ? take(ms * n) : 0;
                    S.orows = take(sizeof(uint32_t) * (size_t)S.P * S.n2);
                }
                if (!ok || off + stat > (size_t)optin) continue;
                for (auto kern : {k_cmg<Pr, 0>, k_cmg<Pr, 1>}) {  // the limit is the function's: the device's
                    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)stat));
                    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
                }
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)cs);
                cfg.blockDim = dim3((unsigned)CMG_THREADS);
                cfg.dynamicSmemBytes = off;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = (unsigned)cs;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                int nc = 0;
                if (cudaOccupancyMaxActiveClusters(&nc, k_cmg<Pr, 0>, &cfg) != cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                if (nc < 1) continue;
                c->cmg_ls = ls;
                c->cmg_cs = cs;
                c->cmg_smem = off;
                for (int l = ls; l < c->lb; l++) c->cmg_slab[l - ls] = sl[l - ls];
                return MPP_OK;
            }
        }
        return MPP_OK;
    });
}

int build_tma(mpp_ctx* c) {
    const size_t ms = msize(c->prec);
    const CUtensorMapDataType dt = c->prec == MPP_PREC_FP64        ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                   : c->prec == MPP_PREC_MIXED_FP16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                   : c->prec == MPP_PREC_MIXED_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const int pad = 16 / (int)ms;
    const bool off = getenv("MPP_NO_TMA") != nullptr;
    const char* mode = getenv("MPP_RBGS");
    auto parse = [](const char* m, int dflt) {
        return !m ? dflt
                  : (!strcmp(m, "tma") ? MPP_SMOOTHER_TMA
                     : !strcmp(m, "column") ? MPP_SMOOTHER_COLUMN
                     : !strcmp(m, "async") ? MPP_SMOOTHER_ASYNC
                                           : MPP_SMOOTHER_VECTOR);
    };
    c->form_fine = parse(mode, MPP_SMOOTHER_VECTOR);
    c->form_coarse = parse(getenv("MPP_RBGS_COARSE"), c->form_fine);
    for (int l = 0; l < MAXLEV; l++) c->tma_ok[l] = false;
    for (int l = 0; l < c->lb; l++) {
        const LevelBuf& b = c->lv[l];
        if (off || b.H % TH != 0 || b.n[1] < TY + 4 || b.n[2] < TZ + 4) continue;
        TmaLev& t = c->tma[l];
        c->tma_ok[l] = encode_level(&t.xh, dt, b.x, ms, b, TH + 2 * pad, TY + 2, TZ + 2) &&
                       encode_level(&t.b, dt, b.b, ms, b, TH, TY, TZ) &&
                       encode_level(&t.dg, dt, ms == 2 ? b.di : b.dg, ms, b, TH, TY, TZ) &&
                       encode_level(&t.code, CU_TENSOR_MAP_DATA_TYPE_UINT8, b.code, 1, b, TH, TY, TZ);
    }
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        using M = typename Pr::M;
        CK(cudaFuncSetAttribute(k_rbgs_tma<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize, TmaGeom<M>::SMEM));
        int nb = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_rbgs_tma<Pr>, TPB, TmaGeom<M>::SMEM));
        c->tma_blocks = (nb > 0 ? nb : 1) * c->nsm;
        c->async_blocks = 0;
        if constexpr (sizeof(M) == 2) {
            CK(cudaFuncSetAttribute(k_rbgs_async<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize, AS_SMEM));
            int na = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&na, k_rbgs_async<Pr>, TPB, AS_SMEM));
            c->async_blocks = na * c->nsm;
        }
        return MPP_OK;
    });
}

}  // namespace

// ======================================================================= C ABI

extern "C" {

void mpp_opts_default(mpp_opts* o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->tol = 1e-4f;
    o->maxiter = 60;
    o->sweeps = 2;
    o->sweeps_coarse = 0;
    o->coarse = 40;
    o->precision = MPP_PREC_FP32;
    o->graph = 0;
    o->fallback = 0;
    o->restart = 8;
    o->fallback_maxiter = 240;
    o->cg_maxiter_with_fallback = 80;
}

int32_t mpp_levels_for(const int32_t n[3]) {
    if (!n || n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return -1;
    for (int levels = 2; levels < MAXLEV; levels++) {
        const int m = 1 << (levels - 1);
        if (n[0] % m || n[1] % m || n[2] % m) return -1;
        if ((int64_t)(n[0] / m) * (n[1] / m) * (n[2] / m) <= 1024) return levels;
    }
    return -1;
}

// The error text of the other translation units of the library (not exported).
__attribute__((visibility("hidden"))) void mpp_internal_error(const char* msg) { set_err("%s", msg); }

const char* mpp_last_error(void) { return g_err; }
const char* mpp_version(void) { return "libmpp 0.1 (sm_100a)"; }

int mpp_ctx_destroy(mpp_ctx* c) {
    if (!c) return MPP_OK;
    drop_graphs(c);
    if (c->trap_exec) cudaGraphExecDestroy(c->trap_exec);
    if (c->trap_graph) cudaGraphDestroy(c->trap_graph);
    for (void* p : c->allocs) cudaFree(p);
    if (c->sc_host) cudaFreeHost(c->sc_host);
    if (c->fgd_host) cudaFreeHost(c->fgd_host);
    if (c->cap) cudaStreamDestroy(c->cap);
    if (c->aux) cudaStreamDestroy(c->aux);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    for (cudaEvent_t e : c->evall) cudaEventDestroy(e);
    delete c;
    return MPP_OK;
}

static int validate(const mpp_grid* g, const mpp_opts* o) {
    if (!g || !o) {
        set_err("null grid or options");
        return MPP_ERR_INVALID;
    }
    if (g->levels < 2 || g->levels >= MAXLEV) {
        set_err("levels must be in [2, %d), got %d", MAXLEV, g->levels);
        return MPP_ERR_INVALID;
    }
    const int m = 1 << (g->levels - 1);
    for (int a = 0; a < 3; a++)
        if (g->n[a] <= 0 || g->n[a] % m) {
            set_err("grid side %d = %d is not a positive multiple of 2^(levels-1) = %d", a, g->n[a], m);
            return MPP_ERR_INVALID;
        }
    if ((int64_t)(g->n[0] / m) * (g->n[1] / m) * (g->n[2] / m) > 1024) {
        set_err("the coarsest level has more than 1024 cells; use more levels");
        return MPP_ERR_INVALID;
    }
    if (!(g->dx > 0.f)) {
        set_err("dx must be positive");
        return MPP_ERR_INVALID;
    }
    if (o->sweeps < 1 || o->sweeps > 16 || o->sweeps_coarse < 0 || o->sweeps_coarse > 16 || o->coarse < 0 ||
        o->maxiter < 0 || !(o->tol >= 0.f)) {
        set_err("bad solver options");
        return MPP_ERR_INVALID;
    }
    if (o->precision < 0 || o->precision > 3) {
        set_err("unknown precision %d", o->precision);
        return MPP_ERR_INVALID;
    }
    if (o->fallback && (o->restart < 1 || o->restart > FG_MAXR || o->fallback_maxiter < 0 ||
                        o->cg_maxiter_with_fallback < 0)) {
        set_err("bad fallback options (restart must be in [1, %d])", FG_MAXR);
        return MPP_ERR_INVALID;
    }
    return MPP_OK;
}

int mpp_ctx_create(mpp_ctx** out, const mpp_grid* g, const mpp_opts* o) {
    if (!out) {
        set_err("null output");
        return MPP_ERR_INVALID;
    }
    *out = nullptr;
    if (int e = validate(g, o)) return e;
    mpp_ctx* c = new mpp_ctx();
    memset(c->lv, 0, sizeof(c->lv));
    c->grid = *g;
    c->opts = *o;
    c->prec = o->precision;
    c->L = g->levels;
    c->diag = c->bvec = c->r = c->d = c->q = c->Pd = nullptr;
    memset(c->gc, 0, sizeof(c->gc));
    c->gclock = 0;
    c->gen = 0;
    c->bytes = 0;
    c->launches = 0;
    c->sc_host = nullptr;
    c->cap = nullptr;
    c->aux = nullptr;
    c->ev_fork = c->ev_join = nullptr;
    c->in_batch = false;
    c->ext_r = nullptr;
    c->ext_n = 0;
    c->prof_on = 0;
    memset(c->prof, 0, sizeof(c->prof));
    memset(c->active, 0, sizeof(c->active));
    c->fV = nullptr;
    memset(c->fZ, 0, sizeof(c->fZ));
    c->fg_restart = 0;
    c->fgd = nullptr;
    c->fgd_host = nullptr;
    c->fg_used = c->fg_its = 0;
    c->fg_residual = 0.0;
    c->vjp_beta = nullptr;
    for (int a = 0; a < 3; a++) c->adv_acc[a] = nullptr;
    c->trap_air = c->trap_reach = nullptr;
    c->trap_st = nullptr;
    c->trap_graph = nullptr;
    c->trap_exec = nullptr;
    auto fail = [&](int e) {
        mpp_ctx_destroy(c);
        return e;
    };
    cudaError_t ce = cudaGetDevice(&c->dev);
    if (ce != cudaSuccess) {
        set_err("cudaGetDevice: %s", cudaGetErrorString(ce));
        return fail(MPP_ERR_CUDA);
    }
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
    const size_t vs = vsize(c->prec), ms = msize(c->prec);
    const bool alias = vs == ms;  // FP32 and FP64: the V-cycle's fine arrays alias the CG's
    const int64_t N = (int64_t)g->n[0] * g->n[1] * g->n[2];
    int e;
    // level geometry
    size_t tflag_total = 0;
    // the first level small enough for the one-CTA bottom solve: 4096 cells, or 512 when the
    // levels above it can run in a thread-block cluster (k_cmg takes a 16^3 level's passes in
    // well under the time one CTA needs); MPP_BOTTOM_CELLS in the environment lowers the bound
    const char* cmg_env = getenv("MPP_CMG");
    int64_t botcells = (cmg_env && !strcmp(cmg_env, "0")) ? BOTTOM_CELLS : BOTTOM_CELLS / 8;
    if (const char* bc = getenv("MPP_BOTTOM_CELLS")) botcells = std::min<int64_t>(BOTTOM_CELLS, atoll(bc));
    c->lb = c->L - 1;
    for (int l = 1; l < c->L; l++) {
        const int64_t Nl = (int64_t)(g->n[0] >> l) * (g->n[1] >> l) * (g->n[2] >> l);
        if (Nl <= botcells) {
            c->lb = l;
            break;
        }
    }
    for (int l = 0; l < c->L; l++) {
        LevelBuf& b = c->lv[l];
        for (int a = 0; a < 3; a++) b.n[a] = g->n[a] >> l;
        b.split = l < c->lb;
        if (b.split) {
            b.H = b.n[0] / 2;
            b.GH = (b.H + TH - 1) / TH;
            b.GJ = (b.n[1] + TY - 1) / TY;
            b.GK = (b.n[2] + TZ - 1) / TZ;
            b.ntiles = b.GH * b.GJ * b.GK;
            tflag_total += (size_t)b.ntiles;
        }
    }
    c->tflag_bytes = tflag_total;
    if ((e = alloc(c, (void**)&c->tflag_all, tflag_total))) return fail(e);
    size_t off = 0;
    for (int l = 0; l < c->L; l++) {
        LevelBuf& b = c->lv[l];
        const int64_t Nl = (int64_t)b.n[0] * b.n[1] * b.n[2];
        if (l > 0 && (e = alloc(c, (void**)&b.types, Nl))) return fail(e);
        if (b.split) {
            b.tflag = c->tflag_all + off;
            off += b.ntiles;
            if ((e = alloc(c, (void**)&b.tiles, sizeof(uint32_t) * b.ntiles))) return fail(e);
            if ((e = alloc(c, (void**)&b.count, sizeof(int)))) return fail(e);
            if ((e = alloc(c, (void**)&b.code, Nl))) return fail(e);
            if ((e = alloc_guarded(c, &b.x, ms, Nl, guard_of(b.n[0], b.n[1])))) return fail(e);
            if ((e = alloc(c, &b.r, ms * Nl))) return fail(e);
            if (l > 0 || !alias) {
                if ((e = alloc(c, &b.dg, ms * Nl))) return fail(e);
                if ((e = alloc(c, &b.b, ms * Nl))) return fail(e);
            }
            if (ms == 2 && (e = alloc(c, &b.di, ms * Nl))) return fail(e);
        } else {  // a level of the one-CTA bottom solve: natural order
            if ((e = alloc(c, &b.x, ms * Nl))) return fail(e);
            if ((e = alloc(c, (void**)&b.code, Nl))) return fail(e);
            if ((e = alloc(c, (void**)&b.dc, Nl))) return fail(e);
        }
    }
    if ((e = alloc(c, (void**)&c->edges, sizeof(int) * MAXLEV))) return fail(e);
    for (int l = 0; l < c->L; l++) c->lv[l].edge = c->edges + l;
    {
        const LevelBuf& b = c->lv[c->lb];
        const size_t cs = c->prec == MPP_PREC_FP64 ? 8 : 4;
        if ((e = alloc(c, &c->botb, cs * (size_t)b.n[0] * b.n[1] * b.n[2]))) return fail(e);
    }
    {  // the bottom solve's shared-memory layout: levels lb .. L-1 in natural order
        const size_t cs = c->prec == MPP_PREC_FP64 ? 8 : 4;   // stencil arithmetic (C)
        const size_t ccs = c->prec == MPP_PREC_FP32 ? 4 : 8;  // coarsest (CC)
        size_t o = 0;
        auto take = [&](size_t bytes) {
            const size_t at = o;
            o += (bytes + 15) & ~(size_t)15;
            return (int)at;
        };
        BotArgs& ba = c->bot;
        memset(&ba, 0, sizeof(ba));
        ba.nl = c->L - c->lb;
        if (ba.nl > BOTTOM_MAXLEV) {
            set_err("%d levels below %lld cells; at most %d are supported", ba.nl, (long long)botcells, BOTTOM_MAXLEV);
            return fail(MPP_ERR_INVALID);
        }
        for (int q = 0; q < ba.nl; q++) {
            const LevelBuf& b = c->lv[c->lb + q];
            const size_t Nl = (size_t)b.n[0] * b.n[1] * b.n[2];
            const bool coarsest = q == ba.nl - 1;
            BotLev& B = ba.lv[q];
            B.n1 = b.n[0];
            B.n2 = b.n[1];
            B.n3 = b.n[2];
            B.code = b.code;
            B.dc = b.dc;
            B.ox = take((coarsest ? ccs : cs) * Nl);
            B.ob = take((coarsest ? ccs : cs) * Nl);
            B.orr = coarsest ? 0 : take(cs * Nl);
            B.ocode = take(Nl);
            B.odc = take(Nl);
            B.olist = coarsest ? 0 : take(2 * sizeof(uint16_t) * Nl);
        }
        c->bot_smem = o;
        c->restrict_smem = (size_t)restrict_smem_bytes((int)msize(c->prec), (int)cs);
        int optin = 0;
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
        if (c->bot_smem + 2 * BOTTOM_MAXLEV * sizeof(int) > (size_t)optin) {  // with the list counts
            set_err("the bottom levels need %zu bytes of shared memory; the device allows %d", c->bot_smem, optin);
            return fail(MPP_ERR_INVALID);
        }
        const int ea = dispatch(c->prec, [&](auto pr) -> int {
            using Pr = decltype(pr);
            // The limit is the function's, shared by every context of the process: raise it
            // to the device's maximum once rather than to this basin's need, which would
            // lower it under a larger basin created earlier.
            cudaFuncAttributes fb;
            CK(cudaFuncGetAttributes(&fb, k_bottom<Pr>));  // its static part (the list counts)
            CK(cudaFuncSetAttribute(k_bottom<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    optin - (int)fb.sharedSizeBytes));
            CK(cudaFuncSetAttribute(k_restrict<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)c->restrict_smem));
            return MPP_OK;
        });
        if (ea) return fail(ea);
    }
    if ((e = alloc(c, &c->diag, vs * N))) return fail(e);
    if ((e = alloc(c, &c->bvec, vs * N))) return fail(e);
    if ((e = alloc(c, &c->r, vs * N))) return fail(e);
    if ((e = alloc_guarded(c, &c->d, vs, N, guard_of(g->n[0], g->n[1])))) return fail(e);
    if ((e = alloc(c, &c->q, vs * N))) return fail(e);
    if (alias) {
        c->lv[0].dg = c->diag;
        c->lv[0].b = c->r;
    }
    if ((e = build_tma(c))) return fail(e);
    if ((e = build_cmg(c))) return fail(e);
    if (c->prec == MPP_PREC_FP64 && (e = alloc(c, &c->Pd, sizeof(double) * N))) return fail(e);
    if ((e = alloc(c, (void**)&c->sc, sizeof(Scalars)))) return fail(e);
    if ((e = alloc(c, (void**)&c->partials, sizeof(double) * MAXK * (size_t)c->nsm * MAXBLOCKS_PER_SM))) return fail(e);
    if ((e = alloc(c, (void**)&c->counters, sizeof(unsigned) * NCOUNTERS))) return fail(e);
    ce = cudaMallocHost((void**)&c->sc_host, sizeof(Scalars));
    if (ce != cudaSuccess) {
        set_err("cudaMallocHost: %s", cudaGetErrorString(ce));
        return fail(MPP_ERR_NOMEM);
    }
    memset(c->sc_host, 0, sizeof(Scalars));
    ce = cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (ce != cudaSuccess) {
        set_err("cudaStreamCreate: %s", cudaGetErrorString(ce));
        return fail(MPP_ERR_CUDA);
    }
    *out = c;
    return MPP_OK;
}

int mpp_ctx_set_opts(mpp_ctx* c, const mpp_opts* o) {
    if (int e = check_ctx(c)) return e;
    if (int e = validate(&c->grid, o)) return e;
    if (o->precision != c->prec) {
        set_err("precision is fixed at context creation");
        return MPP_ERR_INVALID;
    }
    if (o->sweeps != c->opts.sweeps || o->sweeps_coarse != c->opts.sweeps_coarse || o->coarse != c->opts.coarse ||
        o->graph != c->opts.graph ||
        (o->fallback != 0) != (c->opts.fallback != 0)) {
        drop_graphs(c);
    }
    c->opts = *o;
    return MPP_OK;
}

size_t mpp_ctx_bytes(const mpp_ctx* c) { return c ? c->bytes : 0; }

int mpp_profile_enable(mpp_ctx* c, int on) {
    if (int e = check_ctx(c)) return e;
    c->prof_on = on ? 1 : 0;
    if (on) memset(c->prof, 0, sizeof(c->prof));
    return MPP_OK;
}

int mpp_profile_read(mpp_ctx* c, mpp_prof_entry* out, int max) {
    if (int e = check_ctx(c)) return e;
    int n = 0;
    for (int f = 0; f < NFAM; f++)
        for (int l = 0; l <= MAXLEV; l++) {
            const ProfAcc& a = c->prof[f][l];
            if (a.n == 0) continue;
            if (out && n < max) {
                mpp_prof_entry& e = out[n];
                memset(&e, 0, sizeof(e));
                snprintf(e.name, sizeof(e.name), "%s", FAM_NAMES[f]);
                e.level = l == MAXLEV ? -1 : l;
                e.launches = a.n;
                e.ms = a.ms;
                e.bytes = a.bytes;
                e.cells = a.cells;
            }
            n++;
        }
    return n;
}

int mpp_volume(mpp_ctx* c, const float* phi, double* vol, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!phi || !vol) {
        set_err("null argument");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (int e = write_params(c, 1.f, 1.0, 1.0, 0, 0.f, s)) return e;
    Run<PrecFP32> run{c, s};
    run.volume(phi);
    if (int e = read_state(c, s)) return e;
    CK(cudaGetLastError());
    c->launches += run.nk;
    *vol = c->sc_host->s.vol;
    return MPP_OK;
}

int mpp_project(mpp_ctx* c, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw, float* P,
                const uint8_t* types, const float* phi, float volume0, double dt, double recover, mpp_result* res,
                mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!u || !v || !w || !fu || !fv || !fw || !P || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    if (!(dt > 0.0) || !(recover > 0.0) || !(volume0 != 0.f)) {
        set_err("dt and recover must be positive and volume0 nonzero");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (int e = write_params(c, volume0, dt, recover, 1, 0.f, s)) return e;
    Call k{1, u, v, w, fu, fv, fw, P, nullptr, types, phi};
    const int64_t before = c->launches;
    int e = dispatch(c->prec, [&](auto pr) { return solve<decltype(pr)>(c, k, s); });
    if (e < 0) return e;
    fill_result(c, res, c->launches - before);
    return c->sc_host->s.status;
}

int mpp_project_vjp(mpp_ctx* c, const float* gu, const float* gv, const float* gw, float* ou, float* ov, float* ow,
                    float* mu, const uint8_t* types, const float* phi, mpp_result* res, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!gu || !gv || !gw || !ou || !ov || !ow || !mu || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int n1 = c->grid.n[0], n2 = c->grid.n[1], n3 = c->grid.n[2];
    const int64_t N = (int64_t)n1 * n2 * n3, NF = (int64_t)(n1 + 1) * (n2 + 1) * (n3 + 1);
    // the FP64 form keeps beta and mu in FP64 (mu's float copy is the warm start and output)
    const bool f64 = c->prec == MPP_PREC_FP64;
    if (!c->vjp_beta)
        if (int e = alloc(c, &c->vjp_beta, (f64 ? sizeof(double) : sizeof(float)) * (size_t)N)) return e;
    const int64_t before = c->launches;
    if (f64) launch(k_vjp_rhs<double>, grid_cells(c, N), TPB, 0, s, n1, n2, n3, (double*)c->vjp_beta, gu, gv, gw, types, phi);
    else launch(k_vjp_rhs<float>, grid_cells(c, N), TPB, 0, s, n1, n2, n3, (float*)c->vjp_beta, gu, gv, gw, types, phi);
    c->launches++;
    CK(cudaGetLastError());
    if (int e = write_params(c, 1.f, 1.0, 1.0, 0, 0.f, s)) return e;
    Call k{0,  nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, mu, f64 ? nullptr : (const float*)c->vjp_beta,
           types, phi, f64 ? (const double*)c->vjp_beta : nullptr};
    int e = dispatch(c->prec, [&](auto pr) { return solve<decltype(pr)>(c, k, s); });
    if (e < 0) return e;
    if (f64)
        launch(k_vjp_faces<double>, grid_cells(c, NF), TPB, 0, s, n1, n2, n3, ou, ov, ow, gu, gv, gw,
               (const double*)c->Pd, types);
    else
        launch(k_vjp_faces<float>, grid_cells(c, NF), TPB, 0, s, n1, n2, n3, ou, ov, ow, gu, gv, gw, (const float*)mu,
               types);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    fill_result(c, res, c->launches - before);
    return c->sc_host->s.status;
}

// ---- batches: many basins, one graph launch ----
// Each basin keeps its own context (workspace, levels, partial sums); the batch records
// every basin's solve chain into ONE graph, so a projection of all of them is one graph
// launch whose chains the GPU runs concurrently, each with its own device-side
// convergence loop. The graph is cached by the basins' arrays.
struct mpp_batch {
    std::vector<mpp_ctx*> ctx;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key;
    std::vector<int> counts;  // per basin: prologue, body, epilogue kernels
    int dev = -1;
    int grouped = GRP_MAX;        // largest group of basins that share a size and settings (< 2: none)
    std::vector<int> group_of;    // per basin: its group in the recorded graph, -1 alone
    int ngroups = 0;
};

extern "C++" {
namespace {
// Basins that may share a group's launches: the same grid, precision, sweeps, smoother forms
// and level split (so the same launch sequence and grid widths); FP64 and the TMA form keep
// their own chains.
bool groupable(const mpp_ctx* c) {
    return c->prec != MPP_PREC_FP64 && c->form_fine != MPP_SMOOTHER_TMA && c->form_coarse != MPP_SMOOTHER_TMA;
}
bool same_group(const mpp_ctx* a, const mpp_ctx* b) {
    return a->prec == b->prec && a->grid.n[0] == b->grid.n[0] && a->grid.n[1] == b->grid.n[1] &&
           a->grid.n[2] == b->grid.n[2] && a->L == b->L && a->opts.sweeps == b->opts.sweeps &&
           a->opts.sweeps_coarse == b->opts.sweeps_coarse && a->opts.coarse == b->opts.coarse &&
           a->form_fine == b->form_fine && a->form_coarse == b->form_coarse && a->lb == b->lb &&
           a->cmg_ls == b->cmg_ls && a->cmg_cs == b->cmg_cs && a->cmg_smem == b->cmg_smem &&
           a->bot_smem == b->bot_smem && a->async_blocks == b->async_blocks;
}

// The group kernels' shared-memory limits, as their single-basin twins'.
template <class Pr>
int group_attrs(const mpp_ctx* c) {
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    cudaFuncAttributes fb;
    CK(cudaFuncGetAttributes(&fb, k_bottom_g<Pr>));  // its static part (the list counts)
    CK(cudaFuncSetAttribute(k_bottom_g<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fb.sharedSizeBytes));
    CK(cudaFuncSetAttribute(k_restrict_g<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->restrict_smem));
    for (auto kern : {k_cmg_g<Pr, 0>, k_cmg_g<Pr, 1>}) {
        cudaFuncAttributes fa;
        CK(cudaFuncGetAttributes(&fa, kern));
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    if constexpr (sizeof(typename Pr::M) == 2)
        CK(cudaFuncSetAttribute(k_rbgs_async_g<Pr>, cudaFuncAttributeMaxDynamicSharedMemorySize, AS_SMEM));
    return MPP_OK;
}

// Record a group's solves into graph g: each basin's prologue as a chain of its own, one
// conditional WHILE node over the group's loop body (GroupRun) after all of them, then each
// basin's epilogue. counts: per basin, kernels in prologue, body, epilogue.
template <class Pr>
int record_group(const std::vector<mpp_ctx*>& cs, const std::vector<Call>& ks, cudaGraph_t g, int* counts) {
    using V = typename Pr::V;
    if (int e = group_attrs<Pr>(cs[0])) return e;
    cudaStream_t s = cs[0]->cap;
    std::vector<cudaGraphNode_t> tails;
    for (size_t i = 0; i < cs.size(); i++) {
        Run<Pr> pro{cs[i], s};
        CK(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        record_prologue<Pr>(pro, ks[i], 0, 0);
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        cudaStreamCaptureStatus cst;
        const cudaError_t qe = cudaStreamGetCaptureInfo(s, &cst, nullptr, nullptr, &deps, &nd);
        if (qe == cudaSuccess) tails.insert(tails.end(), deps, deps + nd);
        cudaGraph_t gg = g;
        CK(cudaStreamEndCapture(s, &gg));
        CK(qe);
        counts[3 * i] = pro.nk;
    }
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CK(cudaGraphAddNode(&cnode, g, tails.data(), tails.size(), &cp));
    cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
    std::vector<V*> Ps;
    for (const Call& k : ks) Ps.push_back((V*)k.P);
    GroupRun<Pr> gr(cs, Ps, s);
    CK(cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    gr.body(cond);
    const cudaError_t le = cudaGetLastError();  // a launch refused during the capture
    CK(cudaStreamEndCapture(s, &bodyg));
    CK(le);
    for (size_t i = 0; i < cs.size(); i++) {
        Run<Pr> epi{cs[i], s};
        CK(cudaStreamBeginCaptureToGraph(s, g, &cnode, nullptr, 1, cudaStreamCaptureModeThreadLocal));
        record_epilogue<Pr>(epi, ks[i]);
        cudaGraph_t gg = g;
        CK(cudaStreamEndCapture(s, &gg));
        counts[3 * i + 1] = gr.nk;
        counts[3 * i + 2] = epi.nk;
    }
    return MPP_OK;
}
}  // namespace
}  // extern "C++"

static void batch_drop_graph(mpp_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->key.clear();
}

int mpp_batch_create(mpp_batch** out, int count, const mpp_grid* grids, const mpp_opts* opts) {
    if (!out || count <= 0 || !grids) {
        set_err("null output, grids or an empty batch");
        return MPP_ERR_INVALID;
    }
    *out = nullptr;
    mpp_batch* b = new mpp_batch();
    CK(cudaGetDevice(&b->dev));
    for (int i = 0; i < count; i++) {
        mpp_opts o;
        if (opts) o = opts[i];
        else mpp_opts_default(&o);
        mpp_ctx* c = nullptr;
        if (int e = mpp_ctx_create(&c, &grids[i], &o)) {
            for (mpp_ctx* x : b->ctx) mpp_ctx_destroy(x);
            delete b;
            return e;
        }
        c->in_batch = true;
        b->ctx.push_back(c);
    }
    *out = b;
    return MPP_OK;
}

int mpp_batch_destroy(mpp_batch* b) {
    if (!b) return MPP_OK;
    batch_drop_graph(b);
    for (mpp_ctx* c : b->ctx) mpp_ctx_destroy(c);
    delete b;
    return MPP_OK;
}

int mpp_batch_size(const mpp_batch* b) { return b ? (int)b->ctx.size() : 0; }

int mpp_batch_set_grouped(mpp_batch* b, int max_group) {
    if (!b) {
        set_err("null batch");
        return MPP_ERR_INVALID;
    }
    const int g = max_group < 2 ? 0 : (max_group > GRP_MAX ? GRP_MAX : max_group);
    if (b->grouped != g) batch_drop_graph(b);
    b->grouped = g;
    return MPP_OK;
}

int mpp_batch_groups(const mpp_batch* b) { return b ? b->ngroups : 0; }

mpp_ctx* mpp_batch_ctx(mpp_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->ctx.size()) return nullptr;
    batch_drop_graph(b);  // the caller may change the basin's options
    return b->ctx[i];
}

int mpp_batch_project(mpp_batch* b, const mpp_basin_arrays* basins, double dt, double recover, mpp_result* results,
                      mpp_stream stream) {
    if (!b || !basins) {
        set_err("null batch or arrays");
        return MPP_ERR_INVALID;
    }
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev != b->dev) {
        set_err("batch belongs to device %d, current device is %d", b->dev, dev);
        return MPP_ERR_INVALID;
    }
    if (!(dt > 0.0) || !(recover > 0.0)) {
        set_err("dt and recover must be positive");
        return MPP_ERR_INVALID;
    }
    const int n = (int)b->ctx.size();
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<const void*> key;
    for (int i = 0; i < n; i++) {
        const mpp_basin_arrays& a = basins[i];
        if (!a.u || !a.v || !a.w || !a.fu || !a.fv || !a.fw || !a.P || !a.types || !a.phi || !(a.volume0 != 0.f)) {
            set_err("basin %d: null array or zero volume0", i);
            return MPP_ERR_INVALID;
        }
        const void* k[10] = {a.u, a.v, a.w, a.fu, a.fv, a.fw, a.P, a.types, a.phi,
                             reinterpret_cast<const void*>((uintptr_t)b->ctx[i]->gen)};
        key.insert(key.end(), k, k + 10);
    }
    std::vector<int64_t> launches0(n);
    for (int i = 0; i < n; i++) {
        mpp_ctx* c = b->ctx[i];
        launches0[i] = c->launches;
        CK(cudaMemsetAsync(&c->sc->s.fault, 0, sizeof(int), s));
        if (int e = write_params(c, basins[i].volume0, dt, recover, 1, 0.f, s)) return e;
    }
    if (!b->exec || key != b->key) {
        batch_drop_graph(b);
        CK(cudaGraphCreate(&b->graph, 0));
        b->counts.assign(3 * n, 0);
        b->group_of.assign(n, -1);
        b->ngroups = 0;
        auto call_of = [&](int i) {
            const mpp_basin_arrays& a = basins[i];
            return Call{1, a.u, a.v, a.w, a.fu, a.fv, a.fw, a.P, nullptr, a.types, a.phi};
        };
        // groups of basins with the same launch sequence (at most GRP_MAX each), in basin order
        std::vector<std::vector<int>> groups;
        if (b->grouped >= 2)
            for (int i = 0; i < n; i++) {
                mpp_ctx* c = b->ctx[i];
                if (!groupable(c) || b->group_of[i] >= 0) continue;
                std::vector<int> g{i};
                for (int j = i + 1; j < n && (int)g.size() < b->grouped; j++)
                    if (b->group_of[j] < 0 && groupable(b->ctx[j]) && same_group(c, b->ctx[j])) g.push_back(j);
                if (g.size() < 2) continue;
                for (int j : g) b->group_of[j] = (int)groups.size();
                groups.push_back(g);
            }
        b->ngroups = (int)groups.size();
        for (const auto& g : groups) {
            std::vector<mpp_ctx*> cs;
            std::vector<Call> ks;
            for (int j : g) {
                cs.push_back(b->ctx[j]);
                ks.push_back(call_of(j));
            }
            std::vector<int> cnt(3 * g.size());
            int e = dispatch(cs[0]->prec, [&](auto pr) { return record_group<decltype(pr)>(cs, ks, b->graph, cnt.data()); });
            if (e) {
                batch_drop_graph(b);
                return e;
            }
            for (size_t q = 0; q < g.size(); q++)
                for (int r = 0; r < 3; r++) b->counts[3 * g[q] + r] = cnt[3 * q + r];
        }
        for (int i = 0; i < n; i++) {
            if (b->group_of[i] >= 0) continue;
            const Call k = call_of(i);
            mpp_ctx* c = b->ctx[i];
            int e = dispatch(c->prec, [&](auto pr) { return record_solve<decltype(pr)>(c, k, b->graph, &b->counts[3 * i]); });
            if (e) {
                batch_drop_graph(b);
                return e;
            }
        }
        CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->key = key;
    }
    CK(cudaGraphLaunch(b->exec, s));
    for (int i = 0; i < n; i++)
        CK(cudaMemcpyAsync(&b->ctx[i]->sc_host->s, &b->ctx[i]->sc->s, sizeof(State), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    int worst = MPP_OK;
    for (int i = 0; i < n; i++) {
        mpp_ctx* c = b->ctx[i];
        const int* k3 = &b->counts[3 * i];
        c->launches += k3[0] + (int64_t)k3[1] * c->sc_host->s.it + k3[2];
        if (c->sc_host->s.fault) {
            set_err("basin %d: a bounded device wait (TMA pipeline) gave up; results are not valid", i);
            return MPP_ERR_CUDA;
        }
        c->fg_used = c->fg_its = 0;
        if (c->opts.fallback) {
            const mpp_basin_arrays& a = basins[i];
            Call k{1, a.u, a.v, a.w, a.fu, a.fv, a.fw, a.P, nullptr, a.types, a.phi};
            int e = dispatch(c->prec, [&](auto pr) { return fallback_and_finish<decltype(pr)>(c, k, s); });
            if (e) return e;
        }
        if (results) fill_result(c, &results[i], c->launches - launches0[i]);
        const int st = c->sc_host->s.status;
        if (st > worst) worst = st;
    }
    return worst;
}

// ---- the autotuner: smoother form x sweeps, timed on the basin's own solve ----
int mpp_ctx_set_smoothers(mpp_ctx* c, int fine, int coarse) {
    if (int e = check_ctx(c)) return e;
    for (int f : {fine, coarse})
        if (f < MPP_SMOOTHER_VECTOR || f > MPP_SMOOTHER_ASYNC) {
            set_err("unknown smoother form %d", f);
            return MPP_ERR_INVALID;
        }
    c->form_fine = fine;
    c->form_coarse = coarse;
    drop_graphs(c);
    return MPP_OK;
}

int mpp_ctx_set_smoother(mpp_ctx* c, int form) { return mpp_ctx_set_smoothers(c, form, form); }

int mpp_ctx_smoothers(const mpp_ctx* c, int* fine, int* coarse) {
    if (!c) {
        set_err("null context");
        return MPP_ERR_INVALID;
    }
    if (fine) *fine = c->form_fine;
    if (coarse) *coarse = c->form_coarse;
    return MPP_OK;
}

int mpp_autotune(mpp_ctx* c, const float* u, const float* v, const float* w, const uint8_t* types, const float* phi,
                 mpp_tune_entry* table, int capacity, int* chosen, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!u || !v || !w || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    const mpp_opts saved = c->opts;
    const int saved_fine = c->form_fine, saved_coarse = c->form_coarse;
    bool tma0 = c->tma_ok[0], tma1 = false;
    for (int l = 1; l < c->lb; l++) tma1 = tma1 || c->tma_ok[l];
    float *b = nullptr, *P = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<mpp_tune_entry> tried;
    // trial buffers live only for the call
    auto run = [&]() -> int {
        CK(cudaMalloc(&b, sizeof(float) * (size_t)N));
        CK(cudaMalloc(&P, sizeof(float) * (size_t)N));
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        if (int e = mpp_rhs(c, b, u, v, w, types, 0.f, stream)) return e;
        auto trial = [&](int fine, int coarse, int sw, int swc, int csw) -> int {
            mpp_opts o = saved;
            o.sweeps = sw;
            o.sweeps_coarse = swc;
            o.coarse = csw;
            o.graph = 1;
            o.fallback = 0;
            if (int e = mpp_ctx_set_opts(c, &o)) return e;
            if (int e = mpp_ctx_set_smoothers(c, fine, coarse)) return e;
            mpp_tune_entry t{fine, coarse, sw, swc, csw, 0, MPP_OK, 0.f};
            for (int rep = 0; rep < 3; rep++) {  // the first run captures the graph
                CK(cudaMemsetAsync(P, 0, sizeof(float) * (size_t)N, s));
                CK(cudaEventRecord(e0, s));
                mpp_result r;
                const int st = mpp_pressure(c, P, b, types, phi, &r, stream);
                if (st < 0) return st;
                CK(cudaEventRecord(e1, s));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (rep > 0) t.ms += 0.5f * ms;
                t.iterations = r.iterations;
                t.status = st;
            }
            tried.push_back(t);
            return MPP_OK;
        };
        auto best_of = [&](size_t from) {
            int bi = -1;
            for (size_t i = from; i < tried.size(); i++)
                if (tried[i].status == MPP_OK && (bi < 0 || tried[i].ms < tried[bi].ms)) bi = (int)i;
            return bi;
        };
        // 1: the smoother forms, at the context's sweeps
        const int sw0 = saved.sweeps, swc0 = saved.sweeps_coarse, csw0 = saved.coarse;
        const bool async_ok = c->async_blocks > 0;
        for (int fine = MPP_SMOOTHER_VECTOR; fine <= MPP_SMOOTHER_ASYNC; fine++) {
            if (fine == MPP_SMOOTHER_TMA && !tma0) continue;
            if (fine == MPP_SMOOTHER_ASYNC && !async_ok) continue;
            for (int coarse = MPP_SMOOTHER_VECTOR; coarse <= MPP_SMOOTHER_ASYNC; coarse++) {
                if (coarse == MPP_SMOOTHER_TMA && !tma1) continue;
                if (coarse == MPP_SMOOTHER_ASYNC && !async_ok) continue;
                if (c->lb < 2 && coarse != fine) continue;  // no coarse row-split level
                if (int e = trial(fine, coarse, sw0, swc0, csw0)) return e;
            }
        }
        const int bf = best_of(0);
        if (bf < 0) return MPP_OK;
        const int fine = tried[bf].smoother, coarse = tried[bf].coarse_smoother;
        // 2: with those forms, the fine and coarse sweeps and (16-bit forms: the FP32 form
        // keeps the reference's V-cycle) 10 instead of 40 coarsest sweeps
        const bool half = c->prec == MPP_PREC_MIXED_FP16 || c->prec == MPP_PREC_MIXED_BF16;
        for (int sw = 1; sw <= 6; sw++)  // at most 16 + 96 candidates in all
            for (int swc = 1; swc <= 8; swc++)
                for (int csw : {csw0, 10}) {
                    if (csw == 10 && (!half || csw0 == 10)) continue;
                    if (sw == sw0 && swc == (swc0 > 0 ? swc0 : sw0) && csw == csw0) continue;  // tried in 1
                    if (int e = trial(fine, coarse, sw, swc, csw)) return e;
                }
        return MPP_OK;
    };
    const int err = run();
    if (b) cudaFree(b);
    if (P) cudaFree(P);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    int best = -1;
    for (int i = 0; i < (int)tried.size(); i++)
        if (tried[i].status == MPP_OK && (best < 0 || tried[i].ms < tried[best].ms)) best = i;
    // apply the winner, or put the previous settings back
    mpp_opts o = saved;
    int fine = saved_fine, coarse = saved_coarse;
    if (err == MPP_OK && best >= 0) {
        o.sweeps = tried[best].sweeps;
        o.sweeps_coarse = tried[best].sweeps_coarse;
        o.coarse = tried[best].coarse_sweeps;
        fine = tried[best].smoother;
        coarse = tried[best].coarse_smoother;
    }
    if (int e = mpp_ctx_set_opts(c, &o)) return e;
    if (int e = mpp_ctx_set_smoothers(c, fine, coarse)) return e;
    if (err) return err;
    for (int i = 0; i < (int)tried.size() && i < capacity && table; i++) table[i] = tried[i];
    if (chosen) *chosen = best;
    return (int)tried.size();
}

// ---- semi-Lagrangian advection and its adjoint ----
static Flow flow_of(const mpp_ctx* c, const float* u, const float* v, const float* w) {
    Flow fl;
    const float* f[3] = {u, v, w};
    for (int a = 0; a < 3; a++) {
        fl.f[a] = f[a];
        for (int e = 0; e < 3; e++) fl.d[a][e] = c->grid.n[e] + (a == e);
        fl.lo[a] = c->grid.lo[a];
    }
    fl.dx = c->grid.dx;
    return fl;
}

static void adv_slot(const mpp_ctx* c, AdvArrays& A, int slot, float* out, const float* src, int axis) {
    A.out[slot] = out;
    A.src[slot] = src;
    A.n[slot] = 1;
    for (int e = 0; e < 3; e++) {
        A.d[slot][e] = c->grid.n[e] + (axis == e);
        A.off[slot][e] = axis < 0 ? 0.5f : (axis == e ? 0.f : 0.5f);  // COFF, or UOFF/VOFF/WOFF
        A.n[slot] *= A.d[slot][e];
    }
}

static int grid_of(const mpp_ctx* c, const AdvArrays& A, int na) {
    int64_t n = 0;
    for (int a = 0; a < na; a++) n = A.n[a] > n ? A.n[a] : n;
    return grid_cells(c, n);
}

static bool overlaps(const float* a, int64_t na, const float* b, int64_t nb) {
    return a < b + nb && b < a + na;
}

int mpp_advect(mpp_ctx* c, float* ou, float* ov, float* ow, const float* u, const float* v, const float* w, float dt,
               mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!ou || !ov || !ow || !u || !v || !w || !(dt >= 0.f)) {
        set_err("null array or negative dt");
        return MPP_ERR_INVALID;
    }
    AdvArrays A;
    memset(&A, 0, sizeof(A));
    float* outs[3] = {ou, ov, ow};
    const float* ins[3] = {u, v, w};
    for (int a = 0; a < 3; a++) adv_slot(c, A, a, outs[a], ins[a], a);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            if (overlaps(outs[a], A.n[a], ins[b], A.n[b])) {
                set_err("advection output overlaps an input velocity array");
                return MPP_ERR_INVALID;
            }
    cudaStream_t s = (cudaStream_t)stream;
    launch(k_advect, dim3(grid_of(c, A, 3), 3), TPB, 0, s, flow_of(c, u, v, w), A, dt);
    c->launches++;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_extrapolate(mpp_ctx* c, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw, int layers,
                    mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!u || !v || !w || !fu || !fv || !fw) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    if (layers < 0) layers = 0;  // `for _ in 1:layers` runs no layer
    if (layers > EXTRAP_MAX_LAYERS) {
        set_err("at most %d extrapolation layers", EXTRAP_MAX_LAYERS);
        return MPP_ERR_INVALID;
    }
    ExtBits E;
    memset(&E, 0, sizeof(E));
    float* X[3] = {u, v, w};
    uint8_t* Fl[3] = {fu, fv, fw};
    int64_t n[3], words[3], wtot = 0, words_max = 0;
    for (int a = 0; a < 3; a++) {
        n[a] = 1;
        for (int e = 0; e < 3; e++) {
            E.d[a][e] = c->grid.n[e] + (a == e);
            n[a] *= E.d[a][e];
        }
        E.W[a] = (E.d[a][0] + 31) / 32;
        words[a] = (int64_t)E.W[a] * E.d[a][1] * E.d[a][2];
        if (n[a] >= ((int64_t)1 << 31) || 4 * words[a] >= ((int64_t)1 << 31)) {
            set_err("face array of 2^31 or more faces");
            return MPP_ERR_INVALID;
        }
        wtot += words[a];
        words_max = std::max<int64_t>(words_max, words[a]);
    }
    // a layer reads its neighbours' faces while others are written: no two of the six
    // arrays may share memory
    const char* lo[6] = {(const char*)u, (const char*)v, (const char*)w, (const char*)fu, (const char*)fv,
                         (const char*)fw};
    const int64_t by[6] = {4 * n[0], 4 * n[1], 4 * n[2], n[0], n[1], n[2]};
    for (int a = 0; a < 6; a++)
        for (int b = a + 1; b < 6; b++)
            if (lo[a] < lo[b] + by[b] && lo[b] < lo[a] + by[a]) {
                set_err("extrapolation arrays overlap");
                return MPP_ERR_INVALID;
            }
    cudaStream_t s = (cudaStream_t)stream;
    const Geo g = geo_of(c->grid);
    const bool first = c->ext_n == 0;
    if (first) {  // the masks (open, and the two reach masks), on the first call
        if (int e = alloc(c, (void**)&c->ext_r, sizeof(uint32_t) * (size_t)(3 * wtot))) return e;
        c->ext_n = 3 * wtot;
    }
    int64_t o = 0;
    uint32_t* M = reinterpret_cast<uint32_t*>(c->ext_r);
    for (int a = 0; a < 3; a++) {
        E.x[a] = X[a];
        E.f[a] = Fl[a];
        E.open[a] = M + o;
        E.ra[a] = M + o + words[a];
        E.rb[a] = M + o + 2 * words[a];
        o += 3 * words[a];
    }
    if (first) {  // the walls are the grid's geometry: the open mask is built once
        launch(k_extrap_open, dim3(grid_cells(c, words_max), 3), TPB, 0, s, g, E);
        c->launches++;
    }
    // a warp a word for the flags in and out, a thread a word for the layers
    const dim3 gwarp(grid_cells(c, 32 * ((words_max + EXT_WW - 1) / EXT_WW)), 3), gword(grid_cells(c, words_max), 3);
    launch(k_extrap_flags, gwarp, TPB, 0, s, E);
    for (int l = 1; l <= layers; l++) launch(k_extrap_layer, gword, TPB, 0, s, E, l & 1);
    launch(k_extrap_final, gwarp, TPB, 0, s, E, layers % 2 == 0 ? 1 : 0, layers == 0 ? 1 : 0);
    c->launches += layers + 2;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_advect_phi(mpp_ctx* c, float* ophi, const float* phi, const float* u, const float* v, const float* w, float dt,
                   mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!ophi || !phi || !u || !v || !w || !(dt >= 0.f)) {
        set_err("null array or negative dt");
        return MPP_ERR_INVALID;
    }
    AdvArrays A;
    memset(&A, 0, sizeof(A));
    adv_slot(c, A, 0, ophi, phi, -1);
    if (overlaps(ophi, A.n[0], phi, A.n[0])) {
        set_err("advection output overlaps its input");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    launch(k_advect, dim3(grid_of(c, A, 1), 1), TPB, 0, s, flow_of(c, u, v, w), A, dt);
    c->launches++;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_advect_vjp(mpp_ctx* c, const float* gou, const float* gov, const float* gow, const float* u, const float* v,
                   const float* w, float dt, float* du, float* dv, float* dw, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!gou || !gov || !gow || !u || !v || !w || !du || !dv || !dw || !(dt >= 0.f)) {
        set_err("null array or negative dt");
        return MPP_ERR_INVALID;
    }
    AdvArrays A;
    memset(&A, 0, sizeof(A));
    const float* gos[3] = {gou, gov, gow};
    const float* ins[3] = {u, v, w};
    float* outs[3] = {du, dv, dw};
    for (int a = 0; a < 3; a++) adv_slot(c, A, a, const_cast<float*>(gos[a]), ins[a], a);
    cudaStream_t s = (cudaStream_t)stream;
    AdvAcc acc;
    memset(&acc, 0, sizeof(acc));
    for (int a = 0; a < 3; a++) {
        if (!c->adv_acc[a])
            if (int e = alloc(c, (void**)&c->adv_acc[a], sizeof(double) * (size_t)A.n[a])) return e;
        CK(cudaMemsetAsync(c->adv_acc[a], 0, sizeof(double) * (size_t)A.n[a], s));
        acc.src[a] = acc.flow[a] = c->adv_acc[a];
    }
    launch(k_advect_vjp, dim3(grid_of(c, A, 3) * 2, 3), 128, 0, s, flow_of(c, u, v, w), A, acc, dt);
    for (int a = 0; a < 3; a++)
        launch(k_acc_round, grid_cells(c, A.n[a]), TPB, 0, s, outs[a], (const double*)c->adv_acc[a],
               (const float*)nullptr, A.n[a]);
    c->launches += 4;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_vjp_rhs(mpp_ctx* c, float* beta, const float* gu, const float* gv, const float* gw, const uint8_t* types,
                const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!beta || !gu || !gv || !gw || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int n1 = c->grid.n[0], n2 = c->grid.n[1], n3 = c->grid.n[2];
    launch(k_vjp_rhs<float>, grid_cells(c, (int64_t)n1 * n2 * n3), TPB, 0, s, n1, n2, n3, beta, gu, gv, gw, types, phi);
    c->launches++;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_vjp_faces(mpp_ctx* c, float* ou, float* ov, float* ow, const float* gu, const float* gv, const float* gw,
                  const float* mu, const uint8_t* types, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!ou || !ov || !ow || !gu || !gv || !gw || !mu || !types) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int n1 = c->grid.n[0], n2 = c->grid.n[1], n3 = c->grid.n[2];
    launch(k_vjp_faces<float>, grid_cells(c, (int64_t)(n1 + 1) * (n2 + 1) * (n3 + 1)), TPB, 0, s, n1, n2, n3, ou, ov,
           ow, gu, gv, gw, mu, types);
    c->launches++;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_redistance(mpp_ctx* c, float* phi, float* phi0, int iterations, uint8_t* types, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!phi || (iterations > 0 && !phi0) || iterations < 0) {
        set_err("null array or negative iteration count");
        return MPP_ERR_INVALID;
    }
    const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    if (N >= ((int64_t)1 << 31)) {
        set_err("grids of 2^31 or more cells are not supported here");
        return MPP_ERR_INVALID;
    }
    if (iterations > 0 && phi0 < phi + N && phi < phi0 + N) {
        set_err("phi and phi0 overlap");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const Geo g = geo_of(c->grid);
    if (iterations == 0) {
        if (types) {
            launch(k_classify, grid_cells(c, N), TPB, 0, s, g, (const float*)phi, types);
            c->launches++;
        }
        CK(cudaGetLastError());
        return MPP_OK;
    }
    // phimax = Float32((iterations + 1) * dx) (src/flip.jl:674)
    const float phimax = (float)(iterations + 1) * c->grid.dx;
    auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
    const bool v4 = c->grid.n[0] % 4 == 0 && al(phi) && al(phi0) && (!types || (reinterpret_cast<uintptr_t>(types) & 3) == 0);
    float* src = phi;
    float* dst = phi0;
    for (int it = 0; it < iterations; it++) {
        uint8_t* ty = it + 1 == iterations ? types : nullptr;
        if (v4) launch(k_reinit<4>, grid_cells(c, N / 4), TPB, 0, s, g, (const float*)src, dst, phimax, ty);
        else launch(k_reinit<1>, grid_cells(c, N), TPB, 0, s, g, (const float*)src, dst, phimax, ty);
        std::swap(src, dst);
    }
    c->launches += iterations;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_classify(mpp_ctx* c, uint8_t* types, const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    launch(k_classify, grid_cells(c, N), TPB, 0, (cudaStream_t)stream, geo_of(c->grid), phi, types);
    c->launches++;
    CK(cudaGetLastError());
    return MPP_OK;
}

int mpp_filltrapped(mpp_ctx* c, uint8_t* types, float* phi, int maxrounds, int* rounds, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!types || !phi || maxrounds < 0) {
        set_err("null array or negative maxrounds");
        return MPP_ERR_INVALID;
    }
    const int n1 = c->grid.n[0], n2 = c->grid.n[1], n3 = c->grid.n[2];
    const int W1 = (n1 + 31) / 32;
    const int64_t words = (int64_t)W1 * n2 * n3;
    if ((int64_t)n1 * n2 * n3 >= ((int64_t)1 << 31)) {
        set_err("grids of 2^31 or more cells are not supported here");
        return MPP_ERR_INVALID;
    }
    if (!c->trap_air) {  // the masks and the round loop's graph, on the first call
        if (int e = alloc(c, (void**)&c->trap_air, sizeof(uint32_t) * (size_t)words)) return e;
        if (int e = alloc(c, (void**)&c->trap_reach, sizeof(uint32_t) * (size_t)words)) return e;
        if (int e = alloc(c, (void**)&c->trap_st, sizeof(TrapState))) return e;
    }
    TrapMasks T{c->trap_air, c->trap_reach, n1, n2, n3, W1};
    const int64_t rows = (int64_t)n2 * n3;
    const int wpb = TPB / 32;
    auto blocks = [&](int64_t units, int per_block) {
        const int64_t b = (units + per_block - 1) / per_block, cap = (int64_t)c->nsm * MAXBLOCKS_PER_SM;
        return (int)(b < 1 ? 1 : (b < cap ? b : cap));
    };
    if (!c->trap_exec) {
        cudaGraph_t g;
        CK(cudaGraphCreate(&g, 0));
        c->trap_graph = g;
        cudaGraphConditionalHandle cond;
        CK(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CK(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        // one round (src/flip.jl:751-757): sweeps along z, x, y, then the round's end
        CK(cudaStreamBeginCaptureToGraph(c->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        launch(k_trap_sweep_col, blocks((int64_t)W1 * n2, wpb), TPB, 0, c->cap, T, c->trap_st, 2);
        launch(k_trap_sweep_x, blocks(rows, TPB), TPB, 0, c->cap, T, c->trap_st);
        launch(k_trap_sweep_col, blocks((int64_t)W1 * n3, wpb), TPB, 0, c->cap, T, c->trap_st, 1);
        launch(k_trap_round, 1, 1, 0, c->cap, c->trap_st, cond);
        const cudaError_t le = cudaGetLastError();
        CK(cudaStreamEndCapture(c->cap, &body));
        CK(le);
        CK(cudaGraphInstantiate(&c->trap_exec, g, 0));
    }
    cudaStream_t s = (cudaStream_t)stream;
    const bool vec = n1 % 32 == 0 && (reinterpret_cast<uintptr_t>(types) & 15) == 0;
    launch(k_trap_pack, blocks(words, TPB), TPB, 0, s, T, (const uint8_t*)types, c->trap_st, maxrounds, vec ? 1 : 0);
    c->launches++;
    if (maxrounds > 0) {
        CK(cudaGraphLaunch(c->trap_exec, s));
    }
    launch(k_trap_fill, blocks(words, TPB), TPB, 0, s, T, types, phi, 2.0f * c->grid.dx);
    c->launches++;
    CK(cudaGetLastError());
    if (rounds) {
        CK(cudaMemcpyAsync(rounds, &c->trap_st->rounds, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        c->launches += 4 * (int64_t)*rounds;
    }
    return MPP_OK;
}

int mpp_pressure(mpp_ctx* c, float* P, const float* b, const uint8_t* types, const float* phi, mpp_result* res,
                 mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!P || !b || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (int e = write_params(c, 1.f, 1.0, 1.0, 0, 0.f, s)) return e;
    Call k{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, P, b, types, phi};
    const int64_t before = c->launches;
    int e = dispatch(c->prec, [&](auto pr) { return solve<decltype(pr)>(c, k, s); });
    if (e < 0) return e;
    fill_result(c, res, c->launches - before);
    return c->sc_host->s.status;
}

int mpp_rhs(mpp_ctx* c, float* b, const float* u, const float* v, const float* w, const uint8_t* types, float gamma,
            mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!b || !u || !v || !w || !types) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // The rhs does not read phi; the set-up pass then skips the ghost-fluid terms.
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        using V = typename Pr::V;
        Run<Pr> run{c, s};
        SetupIn<V> in;
        memset(&in, 0, sizeof(in));
        in.u = u; in.v = v; in.w = w; in.types = types; in.phi = nullptr; in.dx = c->grid.dx;
        if (int e = write_params(c, 1.f, 1.0, 1.0, 0, gamma, s)) return e;
        run.setup(in, 0, 0);
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        launch(k_from_split<float, V>, grid_cells(c, N), TPB, 0, s, fine_layout(c), b, (const V*)c->bvec);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        c->launches += run.nk + 1;
        return MPP_OK;
    });
}

int mpp_diag(mpp_ctx* c, float* diag, const uint8_t* types, const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!diag || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        using V = typename Pr::V;
        Run<Pr> run{c, s};
        if (int e = operator_setup<Pr>(c, run, types, phi, nullptr, nullptr, nullptr, 0.f)) return e;
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        launch(k_from_split<float, V>, grid_cells(c, N), TPB, 0, s, fine_layout(c), diag, (const V*)c->diag);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        c->launches += run.nk + 1;
        return MPP_OK;
    });
}

int mpp_vcycle(mpp_ctx* c, float* z, const float* r, const uint8_t* types, const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!z || !r || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        using M = typename Pr::M;
        Run<Pr> run{c, s};
        if (int e = operator_setup<Pr>(c, run, types, phi, nullptr, nullptr, nullptr, 0.f)) return e;
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        const size_t ms = msize(c->prec);
        CK(cudaMemsetAsync(c->lv[0].x, 0, ms * N, s));
        launch(k_to_split<M, float>, grid_cells(c, N), TPB, 0, s, fine_layout(c), (M*)c->lv[0].b, r);
        run.vcycle();
        launch(k_from_split<float, M>, grid_cells(c, N), TPB, 0, s, fine_layout(c), z, (const M*)c->lv[0].x);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        c->launches += run.nk + 2;
        return MPP_OK;
    });
}

int mpp_apply(mpp_ctx* c, float* y, const float* x, const uint8_t* types, const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!y || !x || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    return dispatch(c->prec, [&](auto pr) -> int {
        using Pr = decltype(pr);
        using V = typename Pr::V;
        using M = typename Pr::M;
        Run<Pr> run{c, s};
        if (int e = operator_setup<Pr>(c, run, types, phi, nullptr, nullptr, nullptr, 0.f)) return e;
        const int64_t N = (int64_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
        const size_t vs = vsize(c->prec);
        CK(cudaMemsetAsync(c->q, 0, vs * N, s));
        launch(k_to_split<V, float>, grid_cells(c, N), TPB, 0, s, fine_layout(c), (V*)c->d, x);
        launch(k_apply<Pr>, grid_tiles(c, 0), TPB, 0, s, view<M>(c, 0), (const V*)c->d, (const V*)c->diag, (V*)c->q);
        launch(k_from_split<float, V>, grid_cells(c, N), TPB, 0, s, fine_layout(c), y, (const V*)c->q);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        c->launches += run.nk + 3;
        return MPP_OK;
    });
}

int mpp_gradient(mpp_ctx* c, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw, const float* P,
                 const uint8_t* types, const float* phi, mpp_stream stream) {
    if (int e = check_ctx(c)) return e;
    if (!u || !v || !w || !fu || !fv || !fw || !P || !types || !phi) {
        set_err("null array");
        return MPP_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    Run<PrecFP32> run{c, s};
    run.gradient(u, v, w, fu, fv, fw, P, types, phi);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->launches += run.nk;
    return MPP_OK;
}

int mpp_solution_f64(mpp_ctx* c, double* out) {
    if (int e = check_ctx(c)) return e;
    if (c->prec != MPP_PREC_FP64 || !c->Pd || !out) {
        set_err("no FP64 solution on this context");
        return MPP_ERR_INVALID;
    }
    const size_t N = (size_t)c->grid.n[0] * c->grid.n[1] * c->grid.n[2];
    CK(cudaMemcpy(out, c->Pd, sizeof(double) * N, cudaMemcpyDeviceToHost));
    return MPP_OK;
}

}  // extern "C"

// ============================================== liquid volume without any allocation
//
// mpp_volume needs a context, and creating one allocates the whole solver workspace.
// Some callers cannot allocate device memory at the moment they want the volume: a
// render or monitoring callback with a fixed memory budget, code running while another
// library owns the allocator, or a health check between steps that must not disturb the
// memory the solver holds. mpp_volume_noalloc serves them: it runs the same volume
// reduction with its scratch (per-block partial sums and the completion counter) in the
// static device array below, which every GPU that loads this library holds until exit.
//
// Each block sums a fixed run of NOALLOC_BLOCK_CELLS cells, so the scratch bounds the
// grid: at most NOALLOC_MAX_BLOCKS * NOALLOC_BLOCK_CELLS = 16,777,216 cells (256^3).
// Every call shares the array, so calls that overlap on the GPU (on different streams
// at once) race and give wrong results; calls in sequence are fine. Every call looks the
// array's address up on the current device (cudaGetSymbolAddress) rather than keeping it,
// so a device reset between calls, which may move the array, is harmless. A call ends by
// synchronising its stream, so it must not be made while that stream is being captured.
namespace {

constexpr int NOALLOC_BLOCK_CELLS = 4096;  // cells per block: 256 threads x 16
constexpr int NOALLOC_MAX_BLOCKS = 4096;
constexpr int64_t NOALLOC_MAX_CELLS = (int64_t)NOALLOC_BLOCK_CELLS * NOALLOC_MAX_BLOCKS;
constexpr int NOALLOC_HEADER = 256;  // completion counter (offset 0) and the result (offset 8)
constexpr size_t NOALLOC_SCRATCH_BYTES = NOALLOC_HEADER + sizeof(double) * NOALLOC_MAX_BLOCKS;  // 33,024

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// The liquid volume of phi over the non-solid cells, times dx^3 (the sum k_volume forms),
// with the scratch laid out in `scratch`: [counter u32 | result f64 | pad][partials f64 x
// blocks].
__global__ void __launch_bounds__(TPB) k_volume_noalloc(Geo g, const float* __restrict__ phi, unsigned char* scratch) {
    pdl_wait();
    pdl_trigger();
    unsigned* counter = reinterpret_cast<unsigned*>(scratch);
    double* result = reinterpret_cast<double*>(scratch + 8);
    double* partials = reinterpret_cast<double*>(scratch + NOALLOC_HEADER);
    const int64_t N = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const int64_t lo = (int64_t)blockIdx.x * NOALLOC_BLOCK_CELLS;
    const int64_t hi = lo + NOALLOC_BLOCK_CELLS < N ? lo + NOALLOC_BLOCK_CELLS : N;
    double acc[1] = {0.0};
    for (int64_t idx = lo + threadIdx.x; idx < hi; idx += TPB) {
        const int i = (int)(idx % g.n[0]);
        const int j = (int)((idx / g.n[0]) % g.n[1]);
        const int k = (int)(idx / ((int64_t)g.n[0] * g.n[1]));
        if (!issolidcell(g, i, j, k)) {
            float x = 0.5f - phi[idx] / g.dx;
            acc[0] += (double)(x > 1.f ? 1.f : (x < 0.f ? 0.f : x));
        }
    }
    if (grid_sum<1>(acc, partials, counter) && threadIdx.x == 0)
        *result = (double)((float)acc[0] * (g.dx * g.dx * g.dx));
}

}  // namespace

extern "C" int mpp_volume_noalloc(const mpp_grid* grid, const float* phi, double* volume, mpp_stream stream) {
    if (!grid || !phi || !volume) {
        set_err("null argument");
        return MPP_ERR_INVALID;
    }
    if (grid->n[0] <= 0 || grid->n[1] <= 0 || grid->n[2] <= 0 || !(grid->dx > 0.f)) {
        set_err("grid sides and dx must be positive");
        return MPP_ERR_INVALID;
    }
    const int64_t N = (int64_t)grid->n[0] * grid->n[1] * grid->n[2];
    if (N > NOALLOC_MAX_CELLS) {
        set_err("mpp_volume_noalloc handles at most %lld cells (its static scratch holds %d block sums of %d cells); "
                "this grid has %lld: use mpp_volume with a context",
                (long long)NOALLOC_MAX_CELLS, NOALLOC_MAX_BLOCKS, NOALLOC_BLOCK_CELLS, (long long)N);
        return MPP_ERR_INVALID;
    }
    // the array's address on the current device, looked up on every call: a cached address
    // would outlive a device reset that reloads the module
    void* ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    unsigned char* scratch = static_cast<unsigned char*>(ptr);
    cudaStream_t s = (cudaStream_t)stream;
    // The counter must start at zero; an interrupted earlier call could have left it set.
    CK(cudaMemsetAsync(scratch, 0, NOALLOC_HEADER, s));
    const int blocks = (int)((N + NOALLOC_BLOCK_CELLS - 1) / NOALLOC_BLOCK_CELLS);
    launch(k_volume_noalloc, blocks, TPB, 0, s, geo_of(*grid), phi, scratch);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(volume, scratch + 8, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return MPP_OK;
}
