/*
 * libmpp — the dense-MAC pressure projection of Maelstrom.jl's FlipBasin, as
 * hand-written CUDA kernels for sm_100a behind a plain C ABI.
 *
 * The Julia package reaches it with `ccall`: every array is the FlipBasin's own
 * device array, passed as a raw pointer, with the same bytes (Julia column-major,
 * i fastest, 0-based linear index i + nx*(j + ny*k)):
 *   u: (nx+1, ny, nz) float   v: (nx, ny+1, nz) float   w: (nx, ny, nz+1) float
 *   fu, fv, fw: uint8 of the same face shapes
 *   P, phi: (nx, ny, nz) float        types: (nx, ny, nz) uint8 (SOLID 0, LIQUID 1, AIR 2)
 *
 * The library owns its workspace (the CG vectors, the multigrid levels, partial sums,
 * the CUDA graph) inside an opaque context, one per basin. All work is queued on
 * the caller's stream; calls that return an mpp_result synchronise that stream once,
 * at the end. A context is not thread-safe; distinct contexts are independent.
 *
 * Return codes: MPP_OK and the solver statuses are >= 0, API/CUDA errors < 0.
 */
#ifndef MAELSTROM_MPP_H
#define MAELSTROM_MPP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CUDA stream handle (cudaStream_t); NULL is the legacy default stream. */
typedef struct CUstream_st* mpp_stream;

typedef struct mpp_ctx mpp_ctx;

/* Solver statuses (mpp_result.status, and the return value of the solve calls). */
enum {
    MPP_OK = 0,            /* converged to tol */
    MPP_NOT_CONVERGED = 1, /* maxiter reached ("pressure solve did not converge", src/flip.jl:1109) */
    MPP_NONFINITE = 2,     /* a NaN/Inf in a norm or step ("Nonfinite pressure ...", src/sflip.jl:1873-1892) */
    MPP_INDEFINITE = 3,    /* p.Ap <= 0 or z.r <= 0 ("Pressure CG requires a positive ...", src/sflip.jl:1880-1896) */
    MPP_BREAKDOWN = 4,     /* FGMRES Arnoldi breakdown (src/fgmres.jl:77) */
};

/* API errors. */
enum {
    MPP_ERR_INVALID = -1, /* bad argument, size or grid */
    MPP_ERR_CUDA = -2,    /* a CUDA runtime call failed (mpp_last_error() has the text) */
    MPP_ERR_NOMEM = -3,   /* workspace allocation failed */
};

/* Arithmetic of the solve. */
enum {
    MPP_PREC_FP32 = 0,       /* the reference's: FP32 values, standard PCG */
    MPP_PREC_MIXED_FP16 = 1, /* V-cycle stored in FP16, computed in FP32; flexible CG; FP64 reductions and coarsest solve */
    MPP_PREC_MIXED_BF16 = 2, /* as above with BF16 storage */
    MPP_PREC_FP64 = 3,       /* everything in FP64: the accuracy oracle, on the GPU */
};

/* FlipGrid (src/flip.jl:39-46): origin of the low corner, cell size, cells per axis, the
 * cylinder's radius and floor height (cells whose centre lies outside the cylinder or
 * under the floor are solid), and the multigrid's level count. */
typedef struct {
    float lo[3];
    float dx;
    int32_t n[3];
    float radius;
    float floor_z;
    int32_t levels;
} mpp_grid;

/* Solver knobs: pressure!(s; tol, maxiter, sweeps) (src/flip.jl:1082) and vcycle!'s
 * `coarse` (src/flip.jl:992), plus this library's own. */
typedef struct {
    float tol;              /* relative residual target (reference default 1e-4) */
    int32_t maxiter;        /* CG iterations (reference default 60) */
    int32_t sweeps;         /* red-black sweeps down and up per level (default 2) */
    int32_t coarse;         /* sweeps of the coarsest solve, each way (default 40) */
    int32_t precision;      /* MPP_PREC_* */
    int32_t graph;          /* 1: the whole projection is one CUDA graph launch with a
                               device-side convergence test (no host round trips) */
    int32_t fallback;       /* 1: FGMRES when CG fails or misses tol on the true residual */
    int32_t restart;        /* FGMRES restart length (default 8, src/fgmres.jl:26) */
    int32_t fallback_maxiter; /* FGMRES iterations (default 240) */
    int32_t cg_maxiter_with_fallback; /* CG iterations before the fallback (default 80, src/fgmres.jl:99) */
    int32_t sweeps_coarse;  /* sweeps on the levels below the fine one (0: `sweeps`, the reference's) */
} mpp_opts;

typedef struct {
    int32_t iterations;          /* CG iterations (what pressure! returns) */
    int32_t status;              /* MPP_OK, MPP_NOT_CONVERGED, ... */
    int32_t fallback_used;       /* 1 if FGMRES ran */
    int32_t fallback_iterations; /* its iterations */
    double rel_residual;         /* last recursive residual / |b| */
    double true_rel_residual;    /* |b - A P| / |b|, recomputed at exit */
    double bnorm;                /* |b| */
    double volume;               /* liquid volume at entry (m^3), volume(s) */
    float gamma;                 /* the volume-control divergence put into the rhs */
    int64_t kernel_launches;     /* kernels this call ran on the device */
} mpp_result;

/* Defaults: tol 1e-4, maxiter 60, sweeps 2, coarse 40, FP32, no graph, no fallback. */
void mpp_opts_default(mpp_opts* opts);

/* FlipGrid's level rule (src/flip.jl:53-61): the fewest levels (>= 2) whose coarsest
 * grid has at most 1024 cells; -1 if n is not a multiple of the level's 2^(levels-1). */
int32_t mpp_levels_for(const int32_t n[3]);

/* Create a context for one basin: allocates the workspace on the current device.
 * Replaces the workspace half of FlipBasin(...) (src/flip.jl:189-224): levels, b, r,
 * z, d, q, diag, rv, partials. */
int mpp_ctx_create(mpp_ctx** out, const mpp_grid* grid, const mpp_opts* opts);
int mpp_ctx_destroy(mpp_ctx* ctx);
/* Change the knobs of an existing context (precision changes need a new context). */
int mpp_ctx_set_opts(mpp_ctx* ctx, const mpp_opts* opts);
/* Device bytes the context holds. */
size_t mpp_ctx_bytes(const mpp_ctx* ctx);

/* volume(s) (src/flip.jl:293): liquid volume in m^3 from the level set. */
int mpp_volume(mpp_ctx* ctx, const float* phi, double* volume, mpp_stream stream);

/* project!(s, dt; recover) (src/flip.jl:1144-1156): gamma from the volume loss, the
 * rhs, clearair, pressure!, and the gradient update with the valid-face flags.
 * In: u, v, w (after forces!/solidify!), types, phi, P (warm start), volume0.
 * Out: u, v, w, fu, fv, fw, P; `res` (may be NULL). Returns the solve status or an error. */
int mpp_project(mpp_ctx* ctx, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                float* P, const uint8_t* types, const float* phi, float volume0, double dt,
                double recover, mpp_result* res, mpp_stream stream);

/* pressure!(s) (src/flip.jl:1082-1111) for a given right-hand side b: P in = warm start,
 * P out = pressure. Returns the solve status or an error. */
int mpp_pressure(mpp_ctx* ctx, float* P, const float* b, const uint8_t* types, const float* phi,
                 mpp_result* res, mpp_stream stream);

/* ---- single passes, for tests and for callers that split project! ---- */
/* rhs_kernel! (src/flip.jl:817-822): b = -dx div u + dx^2 gamma on LIQUID, else 0. */
int mpp_rhs(mpp_ctx* ctx, float* b, const float* u, const float* v, const float* w,
            const uint8_t* types, float gamma, mpp_stream stream);
/* The adjoint of project! with respect to the face velocities (a vector-Jacobian product;
 * the reference has no adjoint: this one is derived from its forward kernels,
 * src/flip.jl:817-822 and 1113-1130). project! is affine in (u, v, w) for fixed types
 * and phi, u_out = u - G A^-1 (-dx D u + dx^2 gamma), and A is symmetric, so for the
 * cotangent (gu, gv, gw) of the output faces:
 *   beta = dx G^T g on LIQUID cells, A mu = beta (the same solve, options and fallback
 *   as the forward), g_in = g + D^T mu on every face.
 * In: gu, gv, gw (face shapes as u, v, w), types, phi, mu (warm start of the adjoint
 * pressure, natural order, any values). Out: ou, ov, ow = g_in (may be gu, gv, gw
 * themselves), mu. gamma has no velocity derivative. Returns the solve status. */
int mpp_project_vjp(mpp_ctx* ctx, const float* gu, const float* gv, const float* gw, float* ou, float* ov,
                    float* ow, float* mu, const uint8_t* types, const float* phi, mpp_result* res,
                    mpp_stream stream);

/* The two passes of mpp_project_vjp on their own: beta = dx G^T g (natural, 0 off-liquid)
 * and g_in = g + D^T mu. */
int mpp_vjp_rhs(mpp_ctx* ctx, float* beta, const float* gu, const float* gv, const float* gw,
                const uint8_t* types, const float* phi, mpp_stream stream);
int mpp_vjp_faces(mpp_ctx* ctx, float* ou, float* ov, float* ow, const float* gu, const float* gv,
                  const float* gw, const float* mu, const uint8_t* types, mpp_stream stream);

/* advect! of the face velocities through themselves (advect_kernel!, src/flip.jl:357-369,
 * 495-497): ou, ov, ow = u, v, w sampled at the nodes traced back over dt in RK2 sub-steps
 * of at most a cell (at most 32). The outputs must not overlap the inputs. */
int mpp_advect(mpp_ctx* ctx, float* ou, float* ov, float* ow, const float* u, const float* v, const float* w,
               float dt, mpp_stream stream);
/* The same for the cell-centred level set (COFF samples). */
int mpp_advect_phi(mpp_ctx* ctx, float* ophi, const float* phi, const float* u, const float* v, const float* w,
                   float dt, mpp_stream stream);
/* extrapolate! (src/flip.jl:1192-1206), in place, after mpp_project: `layers` layers of
 * extrapolate_kernel! (:1161-1177) carry the velocity out from the faces flagged in fu, fv,
 * fw (an unflagged face that is not walled takes the Float32 mean of its flagged neighbours
 * in the same array, summed +x, -x, +y, -y, +z, -z, and becomes flagged); then every face no
 * layer reached is zeroed (unreached_kernel!, :1181-1184) and every walled face too
 * (solidify!, :801-806). fu, fv, fw end as the reached flags. The six arrays must not
 * overlap; layers <= 0 runs no layer (the zeroing only; the flags stay as they are), and
 * more than 253 layers is refused (MPP_ERR_INVALID). The first call on a context, whatever
 * `layers` is, allocates the context's scratch, three bit masks over the faces of the three
 * arrays (rows padded to 32 faces), and builds the wall mask: make it outside any stream
 * capture. That scratch belongs to the
 * context while each call runs on the caller's stream, so calls on one context must not
 * overlap on the GPU (two streams at once race on it). */
int mpp_extrapolate(mpp_ctx* ctx, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                    int layers, mpp_stream stream);

/* ---- the level-set passes step! runs before the projection (src/flip.jl:1399-1401) ---- */
/* redistance!(s; iterations) (src/flip.jl:673-680): `iterations` Jacobi sweeps of
 * reinit_kernel! (:631-666) with phimax = (iterations + 1) dx, between phi and phi0 as the
 * reference swaps s.phi and s.phi0: sweep 1 reads phi and writes phi0, sweep 2 reads phi0
 * and writes phi, and so on, so the result is in phi0 when `iterations` is odd and in phi
 * when it is even (the caller swaps its two arrays `iterations` times, as redistance!
 * does). `types` (may be NULL) gets classify! of the result (src/flip.jl:682-686), fused
 * into the last sweep (with iterations = 0, classify! of phi). Bit-identical to the
 * reference's Float32 arithmetic. phi and phi0 must not overlap. */
int mpp_redistance(mpp_ctx* ctx, float* phi, float* phi0, int iterations, uint8_t* types, mpp_stream stream);
/* classify!(s) (src/flip.jl:682-686): SOLID where the cell centre is outside the walls, else
 * LIQUID where phi < 0, else AIR. */
int mpp_classify(mpp_ctx* ctx, uint8_t* types, const float* phi, mpp_stream stream);
/* filltrapped!(s; maxrounds) (src/flip.jl:747-760), in place: air is reached from the
 * grid's top layer by rounds of sweeps along z, x and y (each fills every run of air along
 * a line that holds a reached cell) until a round reaches nothing or `maxrounds` rounds
 * have run; the air left becomes LIQUID with phi = min(phi, -2 dx). The round loop runs on
 * the device (a CUDA graph whose condition the last kernel of a round sets): no host round
 * trip. `rounds` (a host pointer, may be NULL) gets the rounds run, which synchronises
 * `stream`. The first call on a context allocates its masks (a bit a cell, twice) and
 * captures the round loop: make it outside any stream capture. Calls on one context must
 * not overlap on the GPU. */
int mpp_filltrapped(mpp_ctx* ctx, uint8_t* types, float* phi, int maxrounds, int* rounds, mpp_stream stream);

/* The adjoint of mpp_advect (no reference counterpart; the reverse of its steps): the
 * cotangent (gou, gov, gow) of its outputs in; du, dv, dw = the cotangent of (u, v, w),
 * through both the sampled arrays and the traced positions. The sub-step count is
 * piecewise constant and has no derivative; a clamp passes the derivative on its closed
 * range. Sums are FP64 atomics rounded once to Float32 (not bitwise reproducible run to
 * run). du, dv, dw may be gou, gov, gow. */
int mpp_advect_vjp(mpp_ctx* ctx, const float* gou, const float* gov, const float* gow, const float* u,
                   const float* v, const float* w, float dt, float* du, float* dv, float* dw, mpp_stream stream);

/* ---- batches: many independent basins in one graph launch ----
 * Each basin keeps its own context (created from grids[i] and opts[i], or the defaults
 * when opts is NULL). mpp_batch_project records every basin's project! (the same
 * sequence as mpp_project, each with its device-side convergence loop) into one CUDA
 * graph, cached by the basins' arrays, and launches it once: the basins' chains run
 * concurrently on the GPU. A basin with the FGMRES fallback on finishes on the host after
 * the launch. No reference counterpart (the reference steps basins one at a time). */
typedef struct mpp_batch mpp_batch;
typedef struct {
    float *u, *v, *w;          /* faces, updated */
    uint8_t *fu, *fv, *fw;     /* valid-face flags, written */
    float* P;                  /* warm start in, pressure out */
    const uint8_t* types;
    const float* phi;
    float volume0;
} mpp_basin_arrays;
int mpp_batch_create(mpp_batch** batch, int count, const mpp_grid* grids, const mpp_opts* opts);
int mpp_batch_destroy(mpp_batch* batch);
int mpp_batch_size(const mpp_batch* batch);
/* Group the batch's basins: groups of at most `max_group` (2 .. 16; the default 16) basins
 * with the same grid, precision, sweeps, smoother forms and level split (not FP64, not the
 * TMA form), or, with max_group < 2, a chain of launches for each basin. Each pass of a
 * group's CG loops is one launch over all of its basins (the basin is the launch's second
 * grid dimension, every basin keeping its own grid width, arithmetic and reductions, so the
 * results are bit-identical either way), converged basins skip the remaining passes, and the
 * group's loop is one conditional node that ends when all are done. Fewer launches, but the
 * basins of a group move through the V-cycle's phases together, where chains overlap one
 * basin's latency-bound small levels with another's bandwidth-bound fine level: which is
 * faster depends on the batch (Batch.autotune in the Python binding times the choices).
 * mpp_batch_groups: groups in the last recorded graph. */
int mpp_batch_set_grouped(mpp_batch* batch, int max_group);
int mpp_batch_groups(const mpp_batch* batch);
/* Basin i's context (options, smoother, autotuning); using it drops the batch's graph. */
mpp_ctx* mpp_batch_ctx(mpp_batch* batch, int i);
/* project! of every basin with one graph launch; results[i] (may be NULL) per basin.
 * Returns the largest solver status of the batch, or an error. */
int mpp_batch_project(mpp_batch* batch, const mpp_basin_arrays* basins, double dt, double recover,
                      mpp_result* results, mpp_stream stream);

/* ---- smoother forms and the autotuner ---- */
enum {
    MPP_SMOOTHER_VECTOR = 0, /* warp per 64x4x2 tile, 8 same-colour cells per lane, 16-byte loads */
    MPP_SMOOTHER_TMA = 1,    /* TMA-staged tiles (cp.async.bulk.tensor), persistent pipeline */
    MPP_SMOOTHER_COLUMN = 2, /* thread per tile column, scalar loads */
    MPP_SMOOTHER_ASYNC = 3,  /* warp per tile as the vector form, its loads staged in shared memory by a
                                pipeline of cp.async copies (16-bit forms; the others take the vector form) */
};
/* The smoother form of the fine level and of the coarser row-split levels (each level's
 * other passes take the vector forms unless its smoother is the column form). */
int mpp_ctx_set_smoothers(mpp_ctx* ctx, int fine, int coarse);
int mpp_ctx_set_smoother(mpp_ctx* ctx, int form); /* both */
int mpp_ctx_smoothers(const mpp_ctx* ctx, int* fine, int* coarse);
typedef struct {
    int32_t smoother;        /* MPP_SMOOTHER_* of the fine level */
    int32_t coarse_smoother; /* MPP_SMOOTHER_* of the coarser row-split levels */
    int32_t sweeps;          /* smoother sweeps of the fine level, each way */
    int32_t sweeps_coarse;   /* of the coarser levels */
    int32_t coarse_sweeps;   /* sweeps of the coarsest solve, each way */
    int32_t iterations; /* CG iterations to tol */
    int32_t status;     /* solver status */
    float ms;           /* time of the solve (CUDA events, graph launch) */
} mpp_tune_entry;
/* Time the basin's own pressure solve (rhs from u, v, w; zero start; the context's tol and
 * precision): first every fine x coarse smoother form at the context's sweeps, then with the
 * fastest forms fine sweeps 1..6 x coarse-level sweeps 1..8 (and, in the 16-bit forms, 10
 * instead of 40 coarsest sweeps); keep the fastest that converges on
 * the context, and return the number of candidates tried (table[0..capacity) gets them,
 * *chosen the winner's index, -1 when none converged). Allocates two trial arrays for
 * the call. */
int mpp_autotune(mpp_ctx* ctx, const float* u, const float* v, const float* w, const uint8_t* types,
                 const float* phi, mpp_tune_entry* table, int capacity, int* chosen, mpp_stream stream);

/* diag_kernel! (src/flip.jl:824-836). */
int mpp_diag(mpp_ctx* ctx, float* diag, const uint8_t* types, const float* phi, mpp_stream stream);
/* vcycle!(s, z, r) (src/flip.jl:992-1014): z = M^-1 r for this types/phi. */
int mpp_vcycle(mpp_ctx* ctx, float* z, const float* r, const uint8_t* types, const float* phi,
               mpp_stream stream);
/* y = A x (residual_kernel!'s operator, src/flip.jl:859-863). */
int mpp_apply(mpp_ctx* ctx, float* y, const float* x, const uint8_t* types, const float* phi,
              mpp_stream stream);
/* project_kernel! for the three face sets (src/flip.jl:1113-1130). */
int mpp_gradient(mpp_ctx* ctx, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                 const float* P, const uint8_t* types, const float* phi, mpp_stream stream);

/* FP64 pressure of the last mpp_pressure/mpp_project on an MPP_PREC_FP64 context. */
int mpp_solution_f64(mpp_ctx* ctx, double* out_host);

/* The liquid volume without allocating anything: the sum over the non-solid cells of
 * clamp(0.5 - phi/dx, 0, 1), times dx^3, in m^3. It has no counterpart in the reference. It
 * is for callers that cannot allocate device memory when they want the volume, such as a
 * monitoring or render callback under a fixed memory budget, where creating a context
 * (which allocates the solver's whole workspace) is not an option. Its scratch is a static
 * device array of 33,024 bytes that every GPU loading this library holds until exit; it
 * handles grids of at most 16,777,216 cells (256^3) and returns MPP_ERR_INVALID beyond.
 * All calls share that array: calls overlapping on the GPU race. Each call looks the
 * array's address up on the current device. It synchronises `stream` before returning, so
 * it must not be called while `stream` is being captured. `volume` is a host pointer. */
int mpp_volume_noalloc(const mpp_grid* grid, const float* phi, double* volume, mpp_stream stream);

/* ---- per-kernel timing (the reference has none: bakeflip only logs @elapsed per
 * frame, src/flip.jl:1992-2010) ----
 * With profiling on, solves run their CG loop from the host (no graph) and bracket
 * every kernel with CUDA events on the caller's stream. Each entry sums one kernel
 * family at one level: launches, device milliseconds, and the algorithmic bytes the
 * launches had to move (the array elements each pass reads or writes once, over the
 * level's active tiles; dense passes over every cell). */
typedef struct {
    char name[24];
    int32_t level;    /* multigrid level (0 = fine), -1 for whole-grid passes */
    int32_t reserved;
    int64_t launches;
    double ms;
    double bytes;
    int64_t cells;    /* cells the last launch covered (active tiles x 512, or the grid) */
} mpp_prof_entry;

/* Turn profiling on (1) or off (0); turning it on clears the accumulators. */
int mpp_profile_enable(mpp_ctx* ctx, int on);
/* Copy up to `max` entries; returns how many exist (may exceed max). */
int mpp_profile_read(mpp_ctx* ctx, mpp_prof_entry* out, int max);

/* Text of the last error on this thread. */
const char* mpp_last_error(void);
/* Library version string. */
const char* mpp_version(void);

/* ==== The sparse two-resolution basin (SparseBasin, src/sflip.jl) ====
 *
 * Fine 16^3 blocks of cells dx wide where the surface is, over a dense coarse grid of
 * cells 4 dx wide (nb blocks a side, 4 nb coarse cells), the pressure solved over both at
 * once: the Losasso-coupled operator (1 between fine cells, 0.4 on each fine sub-face to
 * a coarse cell, 4 between coarse cells, src/sflip.jl:1059-1074), Galerkin aggregation
 * multigrid (fine blocks at 16^3 and 8^3 over the coarse grid, then the coarse grid and
 * its halvings), damped Jacobi smoothing, flexible (Polak-Ribiere) PCG, and with
 * `fallback` the CG -> FGMRES dispatch of src/fgmres.jl:96-110.
 *
 * Arrays are the SparseBasin's own device arrays, in the reference's layout:
 *   slot:  int32 [nb0 nb1 nb2], the block's 1-based slot in the fine pools (0: coarse only)
 *          (Topology.slot, src/sflip.jl:78-84)
 *   where: int32 [3 x nslots], each slot's block (bi, bj, bk), -1s for a free slot
 *   fine cell pools: [nslots x 4096] (cell i + 16 (j + 16 k) of a slot)
 *   fine face pools: [nslots x 17*256] a axis (faceindex, src/sflip.jl:106-110)
 *   coarse cells: column-major (4 nb0, 4 nb1, 4 nb2); coarse faces one longer along
 *   their axis. Types are SOLID 0, LIQUID 1, AIR 2.
 * The context owns the workspace for `capacity` slots (the pools' size); a call uses the
 * first `nslots` of them. Calls on one context must not overlap on the GPU. */
typedef struct mpp_sparse_ctx mpp_sparse_ctx;

/* SparseGrid (src/sflip.jl:38-44) */
typedef struct {
    float lo[3];
    float dx;
    int32_t nb[3];
    float radius;
    float floor_z;
} mpp_sparse_grid;

/* The arrays project! reads and writes (Field.fine / Field.coarse pairs). */
typedef struct {
    const int32_t* slot;
    const int32_t* where;
    int32_t nslots;
    const uint8_t* types_f;
    const uint8_t* types_c;
    const float* phi_f;
    const float* phi_c;
    float* P_f;
    float* P_c;
    float* u_f;
    float* u_c;
    float* v_f;
    float* v_c;
    float* w_f;
    float* w_c;
    uint8_t* fu_f;
    uint8_t* fu_c;
    uint8_t* fv_f;
    uint8_t* fv_c;
    uint8_t* fw_f;
    uint8_t* fw_c;
} mpp_sparse_basin;

/* pressure!(::SparseBasin; tol, maxiter, sweeps, boost) (src/sflip.jl:1867) and the
 * fallback dispatch (src/fgmres.jl:96: tol 5e-4, boost 1.5, maxiter 240). */
typedef struct {
    float tol;        /* relative residual (default 1e-4) */
    int32_t maxiter;  /* CG iterations (default 200) */
    int32_t sweeps;   /* damped Jacobi sweep pairs down and up (default 1) */
    float boost;      /* coarse corrections' scale (default 1) */
    int32_t coarse;   /* coarsest solve's sweeps each way (default 40) */
    int32_t fallback; /* 1: CG capped at 80 iterations, then FGMRES (restart 8) on a missed tol */
    int32_t graph;    /* 1: the CG loop is one CUDA graph launch with a device-side exit test */
    int32_t cg_maxiter; /* with fallback: CG iterations before FGMRES (default 80, src/fgmres.jl:99) */
} mpp_sparse_opts;

typedef struct {
    int32_t iterations;        /* what pressure! returns (CG + FGMRES iterations) */
    int32_t fgmres_iterations;
    int32_t status;            /* MPP_OK, MPP_NOT_CONVERGED, ... */
    float rel_residual;        /* last residual / |b| */
    float volume;              /* volume(s) at entry of project! (m^3) */
    float gamma;               /* the volume-control divergence put into the rhs */
    int64_t kernel_launches;
} mpp_sparse_result;

/* Workspace arrays mpp_sparse_read copies out (tests, debugging). */
enum {
    MPP_SP_CU_F = 0, MPP_SP_CV_F, MPP_SP_CW_F, /* level 0 fine face couplings */
    MPP_SP_CU_C, MPP_SP_CV_C, MPP_SP_CW_C,     /* level 0 coarse face couplings */
    MPP_SP_DD_F, MPP_SP_DD_C,                  /* level 0 Dirichlet diagonals */
    MPP_SP_ACT_C,                              /* the coarse grid's activity (uint8) */
    MPP_SP_C1X, MPP_SP_C1Y, MPP_SP_C1Z, MPP_SP_DD1, MPP_SP_ACT1, /* level 1 (8^3 blocks) */
    MPP_SP_C2X, MPP_SP_C2Y, MPP_SP_C2Z, MPP_SP_DD2,             /* level 2 (the coarse grid) */
    MPP_SP_NARRAYS
};

void mpp_sparse_opts_default(mpp_sparse_opts* opts);
/* The dense levels of the hierarchy (the coarse grid halved while it has more than 1024
 * cells and even sizes, src/sflip.jl:318-326); -1 if it does not halve to 1024 cells. */
int32_t mpp_sparse_dense_levels(const int32_t nb[3]);
/* Create a context with workspace for `capacity` slots (SparseBasin's `blocks`). */
int mpp_sparse_ctx_create(mpp_sparse_ctx** out, const mpp_sparse_grid* grid, int32_t capacity);
int mpp_sparse_ctx_destroy(mpp_sparse_ctx* ctx);
size_t mpp_sparse_ctx_bytes(const mpp_sparse_ctx* ctx);
/* volume(s) (src/sflip.jl:1990-1996), m^3. */
int mpp_sparse_volume(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, double* volume, mpp_stream stream);
/* coefficients! (src/sflip.jl:1437-1451) and hierarchy! (:1548-1573) into the context,
 * from the basin's classes and level set: the operator mpp_sparse_apply and
 * mpp_sparse_vcycle use. */
int mpp_sparse_operator(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, mpp_stream stream);
/* apply! (src/sflip.jl:1849-1855): q = A x with the context's operator. */
int mpp_sparse_apply(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, const float* x_f, const float* x_c,
                     float* q_f, float* q_c, mpp_stream stream);
/* vcycle!(s, z, r; sweeps, coarse, boost) (src/sflip.jl:1722-1764) with the context's operator. */
int mpp_sparse_vcycle(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, const float* r_f, const float* r_c,
                      float* z_f, float* z_c, int32_t sweeps, int32_t coarse, float boost, mpp_stream stream);
/* finerhs_kernel! + coarserhs_kernel! (src/sflip.jl:1409-1435) into b_f, b_c. */
int mpp_sparse_rhs(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, float gamma, float* b_f, float* b_c,
                   mpp_stream stream);
/* pressure!(s) for the right-hand side (b_f, b_c): the operator from the basin's classes
 * and level set, then the solve from the warm start in P (src/sflip.jl:1867-1904, or the
 * fallback dispatch, src/fgmres.jl:96-110). Returns the status or an error. */
int mpp_sparse_pressure(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, const float* b_f, const float* b_c,
                        const mpp_sparse_opts* opts, mpp_sparse_result* res, mpp_stream stream);
/* The velocity update and valid flags from P (projectfine_kernel!, projectcoarse_kernel!,
 * restrict! of the faces and flags, src/sflip.jl:584-612, 1917-1962, 2010-2016). */
int mpp_sparse_gradient(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, mpp_stream stream);
/* project!(s::SparseBasin, dt; recover) (src/sflip.jl:1998-2018). Returns the status or an error. */
int mpp_sparse_project(mpp_sparse_ctx* ctx, const mpp_sparse_basin* b, float volume0, double dt, double recover,
                       const mpp_sparse_opts* opts, mpp_sparse_result* res, mpp_stream stream);
/* Copy workspace array `which` (MPP_SP_*) of the current operator into dst (host or
 * device memory, `bytes` at most); the array's size in bytes, or an error. */
int64_t mpp_sparse_read(mpp_sparse_ctx* ctx, int32_t which, void* dst, size_t bytes, mpp_stream stream);

#ifdef __cplusplus
}
#endif
#endif
