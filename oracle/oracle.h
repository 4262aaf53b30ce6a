/*
 * CPU oracle for the dense-MAC pressure projection of Maelstrom.jl's FlipBasin.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it. Nothing in the
 * product path (libmpp.so, the `mpp` Python package) links, loads or calls it.
 *
 * It is a plain C restatement of the reference's projection, src/flip.jl:809-1156
 * (rhs, diagonal, residual, red-black Gauss-Seidel, coarsening, restriction,
 * prolongation, the single-workgroup coarsest solve, the V-cycle, the fused CG
 * passes, the PCG driver, the gradient update, clearair and project!), with the
 * reductions of src/flip.jl:230-293 restated as per-group FP32 tree sums.
 * Each function names the reference lines it follows.
 *
 * PARITY UNPINNED: the reference is Julia on a Vulkan device (through the
 * un-vendored Mantle 0.1) and cannot run on this machine, and its own test suite
 * (test/runtests.jl:48-57) holds no golden vectors for this path. The oracle is
 * pinned instead by analytic known-answer problems (tests/test_oracle_kat.py) and by
 * algebraic properties (operator symmetry, V-cycle symmetry, exact solves).
 *
 * Arrays are the reference's, byte for byte: Julia column-major with i fastest,
 * 0-based here: cell (i,j,k) at i + nx*(j + ny*k); u is (nx+1,ny,nz), v is
 * (nx,ny+1,nz), w is (nx,ny,nz+1); types are UInt8 SOLID=0, LIQUID=1, AIR=2.
 *
 * Every entry point exists twice: *_f32 is the reference arithmetic (Float32 values,
 * Float32 group partials); *_f64 is the same algorithm in double precision, used as
 * the FP64 accuracy oracle.
 */
#ifndef MAELSTROM_ORACLE_H
#define MAELSTROM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FlipGrid (src/flip.jl:39-46): origin, spacing, cells, cylinder radius, floor, levels. */
typedef struct {
    float lo[3];
    float dx;
    int32_t n[3];
    float radius;
    float floor_z;
    int32_t levels;
} orc_grid;

typedef struct {
    int32_t iterations;    /* value pressure! returns (src/flip.jl:1082-1111) */
    int32_t converged;     /* 1 unless maxiter ran out */
    double rnorm;          /* last recursive residual norm */
    double bnorm;          /* norm of the right-hand side */
    double volume;         /* volume(s) at entry of project! (m^3) */
    float gamma;           /* the volume-control divergence used in the rhs */
} orc_info;

/* ---- single passes (for unit tests) ---- */
double orc_volume_f32(const orc_grid* g, const float* phi);
double orc_volume_f64(const orc_grid* g, const double* phi);
void orc_rhs_f32(const orc_grid* g, float* b, const float* u, const float* v, const float* w,
                 const uint8_t* types, float gamma);
void orc_rhs_f64(const orc_grid* g, double* b, const double* u, const double* v, const double* w,
                 const uint8_t* types, double gamma);
void orc_diag_f32(const orc_grid* g, float* diag, const uint8_t* types, const float* phi);
void orc_diag_f64(const orc_grid* g, double* diag, const uint8_t* types, const double* phi);
void orc_coarsen(const int32_t nf[3], uint8_t* tc, const uint8_t* tf);
/* z = M^-1 r, one V-cycle (src/flip.jl:992-1014). level_types[l] for l=1..L-1 are the
 * coarsened types (level 0 is `types`). Every `sweeps` argument of this file packs the
 * fine level's sweep count in its low byte and, when bits 8-15 are not zero, the coarser
 * levels' count there (ORC_SWEEPS); the reference has the one count for all levels. */
#define ORC_SWEEPS(fine, coarser) ((fine) | ((coarser) << 8))
void orc_vcycle_f32(const orc_grid* g, float* z, const float* r, const uint8_t* types,
                    const float* diag, int sweeps, int coarse);
void orc_vcycle_f64(const orc_grid* g, double* z, const double* r, const uint8_t* types,
                    const double* diag, int sweeps, int coarse);
/* y = A x on LIQUID cells, 0 elsewhere (the operator inside residual_kernel!). */
void orc_apply_f32(const orc_grid* g, float* y, const float* x, const uint8_t* types, const float* diag);
void orc_apply_f64(const orc_grid* g, double* y, const double* x, const uint8_t* types, const double* diag);
void orc_gradient_f32(const orc_grid* g, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv,
                      uint8_t* fw, const float* P, const uint8_t* types, const float* phi);
void orc_gradient_f64(const orc_grid* g, double* u, double* v, double* w, uint8_t* fu, uint8_t* fv,
                      uint8_t* fw, const double* P, const uint8_t* types, const double* phi);

/* ---- the solve and the whole projection ---- */
/* pressure! (src/flip.jl:1082-1111): P is the warm start in, the pressure out; b the rhs. */
int orc_pressure_f32(const orc_grid* g, float* P, const float* b, const uint8_t* types,
                     const float* phi, float tol, int maxiter, int sweeps, int coarse, orc_info* info);
int orc_pressure_f64(const orc_grid* g, double* P, const double* b, const uint8_t* types,
                     const double* phi, double tol, int maxiter, int sweeps, int coarse, orc_info* info);
/* project! (src/flip.jl:1144-1156). */
int orc_project_f32(const orc_grid* g, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv,
                    uint8_t* fw, float* P, const uint8_t* types, const float* phi, float volume0,
                    double dt, double recover, float tol, int maxiter, int sweeps, int coarse,
                    orc_info* info);
int orc_project_f64(const orc_grid* g, double* u, double* v, double* w, uint8_t* fu, uint8_t* fv,
                    uint8_t* fw, double* P, const uint8_t* types, const double* phi, double volume0,
                    double dt, double recover, double tol, int maxiter, int sweeps, int coarse,
                    orc_info* info);

/* The adjoint of project! w.r.t. the face velocities (derived from src/flip.jl:817-822 and
 * 1113-1130; the reference has none): beta = dx G^T g, A mu = beta, g_in = g + D^T mu. */
void orc_vjp_rhs_f32(const orc_grid* g, float* beta, const float* gu, const float* gv, const float* gw,
                     const uint8_t* types, const float* phi);
void orc_vjp_rhs_f64(const orc_grid* g, double* beta, const double* gu, const double* gv, const double* gw,
                     const uint8_t* types, const double* phi);
void orc_vjp_faces_f32(const orc_grid* g, float* ou, float* ov, float* ow, const float* gu, const float* gv,
                       const float* gw, const float* mu, const uint8_t* types);
void orc_vjp_faces_f64(const orc_grid* g, double* ou, double* ov, double* ow, const double* gu, const double* gv,
                       const double* gw, const double* mu, const uint8_t* types);
int orc_project_vjp_f32(const orc_grid* g, float* gu, float* gv, float* gw, float* mu, const uint8_t* types,
                        const float* phi, float tol, int maxiter, int sweeps, int coarse, orc_info* info);
int orc_project_vjp_f64(const orc_grid* g, double* gu, double* gv, double* gw, double* mu, const uint8_t* types,
                        const double* phi, double tol, int maxiter, int sweeps, int coarse, orc_info* info);

/* Semi-Lagrangian advection of one array (dims a, sample offset off) through the face
 * velocities (advect_kernel!, src/flip.jl:357-369) and its adjoint (accumulates into
 * gsrc, gu, gv, gw). */
void orc_advect_f32(const orc_grid* g, float* out, const float* src, const int32_t a[3], const float off[3],
                    const float* u, const float* v, const float* w, float dt);
void orc_advect_f64(const orc_grid* g, double* out, const double* src, const int32_t a[3], const double off[3],
                    const double* u, const double* v, const double* w, double dt);
void orc_advect_vjp_f32(const orc_grid* g, const float* gout, const float* src, const int32_t a[3],
                        const float off[3], const float* u, const float* v, const float* w, float dt, float* gsrc,
                        float* gu, float* gv, float* gw);
void orc_advect_vjp_f64(const orc_grid* g, const double* gout, const double* src, const int32_t a[3],
                        const double off[3], const double* u, const double* v, const double* w, double dt,
                        double* gsrc, double* gu, double* gv, double* gw);

/* extrapolate! (src/flip.jl:1192-1206) in Float32, in place: `layers` layers of
 * extrapolate_kernel! per face array, the unreached faces zeroed, then solidify!. fu, fv,
 * fw (the projection's valid flags on entry) end as the reached flags. */
void orc_extrapolate(const orc_grid* g, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                     int layers);

int orc_num_threads(void);
void orc_set_num_threads(int n);

/* ---- the level-set passes before the projection (levelset.c; src/flip.jl:608-760) ---- */
/* redistance!(s; iterations): `iterations` Jacobi sweeps of reinit_kernel!, result in phi. */
void orc_redistance(const orc_grid* g, float* phi, int iterations);
/* classify!(s): SOLID where the cell centre is solid, else LIQUID where phi < 0, else AIR. */
void orc_classify(const orc_grid* g, uint8_t* types, const float* phi);
/* filltrapped!(s; maxrounds): air not reached from the top layer becomes LIQUID (phi at
 * most -2 dx); returns the sweep rounds run. */
int orc_filltrapped(const orc_grid* g, uint8_t* types, float* phi, int maxrounds);

/* ---- the sparse two-resolution basin (sparse.c; src/sflip.jl:1059-2018, src/fgmres.jl) ----
 * Fine 16^3 blocks over a dense coarse grid of cells 4 dx wide (nb blocks a side, 4 nb coarse
 * cells). slot[bi + nb0 (bj + nb1 bk)] is the block's 1-based slot in the fine pools (0: coarse
 * only); where[3 (s - 1) ..] the slot's block coordinates (-1s: a free slot). Fine cell pools
 * hold 4096 cells a slot (i + 16 (j + 16 k)); fine face pools 17*256 faces a slot a axis
 * (faceindex, src/sflip.jl:106-110). Coarse arrays are column-major over the coarse cells,
 * face arrays one longer along their axis. Float32 throughout, as the reference. */
typedef struct {
    float lo[3];
    float dx;
    int32_t nb[3];
    float radius;
    float floor_z;
} ors_grid;
typedef struct {
    ors_grid g;
    const int32_t* slot;
    const int32_t* where;
    int32_t nslots;
    const uint8_t *tf, *tc;
    const float *phif, *phic;
    float *Pf, *Pc;
    float *uf, *uc, *vf, *vc, *wf, *wc;
    uint8_t *fuf, *fuc, *fvf, *fvc, *fwf, *fwc;
} ors_basin;
typedef struct {
    float tol;      /* pressure!(::SparseBasin) default 1e-4; the fallback dispatch's 5e-4 */
    int32_t maxiter;
    int32_t sweeps; /* damped Jacobi sweep pairs down and up (default 1) */
    float boost;    /* coarse corrections' scale (1; the fallback dispatch's 1.5) */
    int32_t fallback; /* 1: src/fgmres.jl:96-110 (CG capped at cg_maxiter, then FGMRES) */
    int32_t cg_maxiter; /* the dispatch's CG cap (80 in the reference) */
} ors_opts;
enum { ORS_OK = 0, ORS_NOT_CONVERGED = 1, ORS_NONFINITE = 2, ORS_INDEFINITE = 3, ORS_BREAKDOWN = 4 };
typedef struct {
    int32_t iterations;        /* what pressure! returns (CG + FGMRES iterations) */
    int32_t fgmres_iterations;
    int32_t status;            /* ORS_* */
    float rel_residual;        /* last residual / |b| */
    float volume;              /* volume(s) at entry of project! */
    float gamma;
} ors_info;
double ors_volume(const ors_basin* b);
int ors_levels(const ors_basin* b);
int ors_coefficients(const ors_basin* b, float* cuf, float* cvf, float* cwf, float* cuc, float* cvc, float* cwc,
                     float* dDf, float* dDc, uint8_t* actc);
int ors_apply(const ors_basin* b, const float* xf, const float* xc, float* qf, float* qc);
int ors_jacobi(const ors_basin* b, const float* xf, const float* xc, const float* bf, const float* bc, float* of,
               float* oc);
int ors_vcycle(const ors_basin* b, const float* rf, const float* rc, float* zf, float* zc, int sweeps, int coarse,
               float boost);
int ors_rhs(const ors_basin* b, float gamma, float* bf, float* bc);
int ors_pressure(const ors_basin* b, const float* bf, const float* bc, const ors_opts* o, ors_info* info);
int ors_gradient(const ors_basin* b);
int ors_project(const ors_basin* b, float volume0, double dt, double recover, const ors_opts* o, ors_info* info);

#ifdef __cplusplus
}
#endif
#endif
