/*
 * CPU oracle of the sparse two-resolution pressure projection (TEST INFRASTRUCTURE ONLY):
 * project!(s::SparseBasin, dt) of the reference (src/sflip.jl:1998-2018) with everything it
 * calls on the way: the Losasso-coupled operator over fine 16^3 blocks and the dense coarse
 * grid (src/sflip.jl:1059-1313), the coefficients (:1315-1451), Galerkin aggregation into
 * the multigrid hierarchy (:1453-1586), the dense levels and the coarsest solve
 * (:1588-1660), the transfers (:1662-1720), vcycle! (:1722-1764), inner (:1766-1805), the
 * vector updates (:1807-1822), apply! (:1824-1865), the flexible (Polak-Ribiere) PCG
 * pressure! (:1867-1904), the gradient update with its valid flags and the face restriction
 * (:584-612, :1906-1962), the volume (:1964-1996), and the CG -> FGMRES dispatch with the
 * restarted right-preconditioned FGMRES (src/fgmres.jl:1-110).
 *
 * Every function follows its reference kernel's loop order and Float32 operation order
 * (built with -ffp-contract=off, so each a*b+c rounds twice, as Julia's Float32 code).
 * Indices keep the reference's convention where it matters: pool and level indices are
 * 1-based with 0 meaning "none" (fineat, cellat, faceat, finefaceat), so the reference's
 * `idx > 0` tests read the same; arrays are accessed at idx - 1.
 *
 * The reductions: inner's 256-wide FP32 tree per workgroup, then the partials summed in
 * index order (the reference's final `sum` is Mantle's, whose order is not pinned), and the
 * volume's sums in FP64. Parity with the reference itself is unpinned: it runs on Julia and a
 * Vulkan device, neither of which exists here.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SOLID 0
#define LIQUID 1
#define AIR 2

/* src/sflip.jl:23-27 */
#define BLOCK 16
#define RATIO 4
#define BCELLS 4096
#define BFACES (17 * 256)
/* src/sflip.jl:1071-1074 */
#define FINE_FINE 1.0f
#define FINE_COARSE 0.4f
#define COARSE_COARSE 4.0f
#define MAXD 16

static const float OMEGA = 6.0f / 7.0f;

/* ---- the state the solve works on ---- */
typedef struct {
    int n[3];
    float *x, *b, *r, *t, *cx, *cy, *cz, *dD;
    uint8_t* act;
} DLev;

typedef struct {
    const ors_basin* B;
    int nb[3], nc[3];
    int64_t ncc, nsl;
    /* level 0 (src/sflip.jl:1315-1451): the fine faces' couplings, the coarse faces', the
       Dirichlet diagonals */
    float *cuf, *cvf, *cwf, *cuc, *cvc, *cwc, *dDf, *dDc;
    /* level 1: the fine blocks at 8^3 over the coarse grid */
    float *c1x, *c1y, *c1z, *dD1;
    uint8_t* act1;
    float *x1f, *b1f, *r1f, *t1f, *x1c, *b1c, *r1c, *t1c;
    /* the dense levels: D[0] is the coarse grid (level 2), its activity doubling as levels
       0 and 1's coarse activity */
    DLev D[MAXD];
    int nd;
    /* the solver's vectors: fine pool and coarse grid each */
    float *bf, *bc, *rf, *rc, *zf, *zc, *df, *dc, *qf, *qc, *rof, *roc, *tmf, *tmc;
} S;

static inline float theta(float pi, float pj) { /* src/flip.jl:113 */
    float t = pi / (pi - pj);
    return t > 1.0f ? 1.0f : (t < 0.01f ? 0.01f : t);
}
static inline float clampf(float x, float lo, float hi) { return x > hi ? hi : (x < lo ? lo : x); }
static inline int64_t LIN(const int* n, int i, int j, int k) {
    return (int64_t)i + (int64_t)n[0] * ((int64_t)j + (int64_t)n[1] * (int64_t)k);
}
/* the dims of a face array along axis a (1..3) over cells n */
static inline void fdims(const int* n, int a, int* m) {
    m[0] = n[0] + (a == 1);
    m[1] = n[1] + (a == 2);
    m[2] = n[2] + (a == 3);
}
static inline void unitv(int a, int* e) {
    e[0] = a == 1;
    e[1] = a == 2;
    e[2] = a == 3;
}

/* ---- grid and topology (src/sflip.jl:53-66, 90-128) ---- */
static inline int issolid_p(const ors_grid* g, float px, float py, float pz) {
    return px * px + py * py > g->radius * g->radius || pz < g->floor_z;
}
/* finecentre / coarsecentre: lo + (I + 1/2) h */
static inline int issolid_fine(const ors_grid* g, int I, int J, int K) {
    return issolid_p(g, g->lo[0] + ((float)I + 0.5f) * g->dx, g->lo[1] + ((float)J + 0.5f) * g->dx,
                     g->lo[2] + ((float)K + 0.5f) * g->dx);
}
static inline int issolid_coarse(const ors_grid* g, int I, int J, int K) {
    const float h = (float)RATIO * g->dx;
    return issolid_p(g, g->lo[0] + ((float)I + 0.5f) * h, g->lo[1] + ((float)J + 0.5f) * h,
                     g->lo[2] + ((float)K + 0.5f) * h);
}
static inline int inblocks(const S* s, int bi, int bj, int bk) {
    return bi >= 0 && bi < s->nb[0] && bj >= 0 && bj < s->nb[1] && bk >= 0 && bk < s->nb[2];
}
static inline int32_t blockslot(const S* s, int bi, int bj, int bk) {
    return s->B->slot[bi + s->nb[0] * (bj + s->nb[1] * bk)];
}
static inline int32_t cellslot(const S* s, int I, int J, int K) {
    const int bi = I >> 4, bj = J >> 4, bk = K >> 4;
    if (!inblocks(s, bi, bj, bk)) return 0;
    return blockslot(s, bi, bj, bk);
}
static inline int64_t fineindex(int64_t sl, int i, int j, int k) {
    return (sl - 1) * BCELLS + i + BLOCK * (j + BLOCK * k) + 1;
}
static inline int64_t fineat(const S* s, int I, int J, int K) {
    const int32_t sl = cellslot(s, I, J, K);
    return sl == 0 ? 0 : fineindex(sl, I & 15, J & 15, K & 15);
}
static inline int64_t faceindex(int64_t sl, int a, int i, int j, int k) {
    const int64_t f = a == 1 ? i + 17 * (j + BLOCK * k) : (a == 2 ? i + BLOCK * (j + 17 * k) : i + BLOCK * (j + BLOCK * k));
    return (sl - 1) * BFACES + f + 1;
}
static inline int64_t finefaceat(const S* s, int a, int I, int J, int K) {
    const int32_t sl = cellslot(s, I, J, K);
    if (sl != 0) return faceindex(sl, a, I & 15, J & 15, K & 15);
    int e[3];
    unitv(a, e);
    const int Im = I - e[0], Jm = J - e[1], Km = K - e[2];
    const int32_t sm = cellslot(s, Im, Jm, Km);
    if (sm == 0) return 0;
    if (!((Im >> 4) != (I >> 4) || (Jm >> 4) != (J >> 4) || (Km >> 4) != (K >> 4))) return 0;
    return faceindex(sm, a, a == 1 ? BLOCK : (Im & 15), a == 2 ? BLOCK : (Jm & 15), a == 3 ? BLOCK : (Km & 15));
}
static inline int covered(const S* s, int I, int J, int K) { return cellslot(s, I * RATIO, J * RATIO, K * RATIO) != 0; }
static inline const int32_t* whereof(const S* s, int64_t sl) { return s->B->where + 3 * (sl - 1); }

/* ---- a level of the composite operator (src/sflip.jl:1076-1141): N = 16 or 8 ---- */
static inline int log2of(int N) { return N == 16 ? 4 : 3; }
static inline int64_t cellidx(int N, int64_t sl, int i, int j, int k) {
    return (sl - 1) * (int64_t)(N * N * N) + i + N * (j + N * k) + 1;
}
static inline int64_t faceidx(int N, int64_t sl, int a, int i, int j, int k) {
    const int n = N, m = N + 1;
    const int64_t f = a == 1 ? i + m * (j + n * k) : (a == 2 ? i + n * (j + m * k) : i + n * (j + n * k));
    return (sl - 1) * (int64_t)((N + 1) * N * N) + f + 1;
}
static inline int64_t cellat(const S* s, int N, int I, int J, int K) {
    const int sh = log2of(N), m = N - 1;
    const int bi = I >> sh, bj = J >> sh, bk = K >> sh;
    if (!inblocks(s, bi, bj, bk)) return 0;
    const int32_t sl = blockslot(s, bi, bj, bk);
    return sl == 0 ? 0 : cellidx(N, sl, I & m, J & m, K & m);
}
static inline int64_t faceat(const S* s, int N, int a, int I, int J, int K) {
    const int sh = log2of(N), m = N - 1;
    const int bi = I >> sh, bj = J >> sh, bk = K >> sh;
    if (inblocks(s, bi, bj, bk)) {
        const int32_t sl = blockslot(s, bi, bj, bk);
        if (sl != 0) return faceidx(N, sl, a, I & m, J & m, K & m);
    }
    int e[3];
    unitv(a, e);
    const int Im = I - e[0], Jm = J - e[1], Km = K - e[2];
    if (!((Im >> sh) != bi || (Jm >> sh) != bj || (Km >> sh) != bk)) return 0;
    if (!inblocks(s, Im >> sh, Jm >> sh, Km >> sh)) return 0;
    const int32_t sl = blockslot(s, Im >> sh, Jm >> sh, Km >> sh);
    if (sl == 0) return 0;
    return faceidx(N, sl, a, a == 1 ? N : (Im & m), a == 2 ? N : (Jm & m), a == 3 ? N : (Km & m));
}

/* A level's arrays as finerow / coarserow read them. */
typedef struct {
    int N;
    const float *cfx, *cfy, *cfz, *dDf;
    const uint8_t* actf;
    const float *ccx, *ccy, *ccz, *dDc;
    const uint8_t* actc;
} Comp;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* finerow's neighbourvalue: the level's fine cell if a fine block holds it, else the coarse
   cell it lies in (indices clamped to the grid). */
static inline float nv(const S* s, int N, int sh, const float* x, const float* xc, int In, int Jn, int Kn) {
    const int64_t id = cellat(s, N, In, Jn, Kn);
    if (id > 0) return x[id - 1];
    return xc[LIN(s->nc, clampi(In >> sh, 0, s->nc[0] - 1), clampi(Jn >> sh, 0, s->nc[1] - 1),
                  clampi(Kn >> sh, 0, s->nc[2] - 1))];
}
/* finerow (src/sflip.jl:1143-1174): diag and off of A x at a level's fine cell. */
static inline void finerow(const S* s, const Comp* L, const float* x, const float* xc, int64_t sl, int i, int j, int k,
                           const int32_t* w, float* pdiag, float* poff) {
    const int N = L->N, sh = log2of(N) - 2;
    const int I = w[0] * N + i, J = w[1] * N + j, K = w[2] * N + k;
    float diag = L->dDf[cellidx(N, sl, i, j, k) - 1], off = 0.0f;
#define NV(In, Jn, Kn) nv(s, N, sh, x, xc, (In), (Jn), (Kn))
    float c;
    c = L->cfx[faceidx(N, sl, 1, i, j, k) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I - 1, J, K); }
    c = L->cfx[faceidx(N, sl, 1, i + 1, j, k) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I + 1, J, K); }
    c = L->cfy[faceidx(N, sl, 2, i, j, k) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I, J - 1, K); }
    c = L->cfy[faceidx(N, sl, 2, i, j + 1, k) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I, J + 1, K); }
    c = L->cfz[faceidx(N, sl, 3, i, j, k) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I, J, K - 1); }
    c = L->cfz[faceidx(N, sl, 3, i, j, k + 1) - 1];
    if (c > 0.0f) { diag += c; off += c * NV(I, J, K + 1); }
#undef NV
    *pdiag = diag;
    *poff = off;
}

/* coarserow (src/sflip.jl:1176-1217): a coarse cell outside fine blocks; its coarse
   neighbours through the coarse faces, a fine block's cells through the R^2 sub-faces. */
static inline void coarserow(const S* s, const Comp* L, const float* xf, const float* xc, int I, int J, int K,
                             float* pdiag, float* poff) {
    const int N = L->N, R = N / 4;
    const int n1 = s->nc[0], n2 = s->nc[1], n3 = s->nc[2];
    float diag = L->dDc[LIN(s->nc, I, J, K)], off = 0.0f;
    for (int a = 1; a <= 3; a++) {
        int e[3];
        unitv(a, e);
        const float* Cc = a == 1 ? L->ccx : (a == 2 ? L->ccy : L->ccz);
        const float* Cf = a == 1 ? L->cfx : (a == 2 ? L->cfy : L->cfz);
        int fm[3];
        fdims(s->nc, a, fm);
        for (int sg = -1; sg <= 1; sg += 2) {
            const int In = I + sg * e[0], Jn = J + sg * e[1], Kn = K + sg * e[2];
            if (0 <= In && In < n1 && 0 <= Jn && Jn < n2 && 0 <= Kn && Kn < n3) {
                if (covered(s, In, Jn, Kn)) {
                    for (int q = 0; q < R; q++)
                        for (int p = 0; p < R; p++) {
                            const int FI = a == 1 ? (sg > 0 ? R * In : R * I - 1) : R * I + p;
                            const int FJ = a == 2 ? (sg > 0 ? R * Jn : R * J - 1) : R * J + (a == 1 ? p : q);
                            const int FK = a == 3 ? (sg > 0 ? R * Kn : R * K - 1) : R * K + q;
                            const int PI = a == 1 ? (sg > 0 ? FI : FI + 1) : FI;
                            const int PJ = a == 2 ? (sg > 0 ? FJ : FJ + 1) : FJ;
                            const int PK = a == 3 ? (sg > 0 ? FK : FK + 1) : FK;
                            const int64_t fidx = faceat(s, N, a, PI, PJ, PK);
                            const int64_t cidx = cellat(s, N, FI, FJ, FK);
                            if (fidx > 0 && cidx > 0) {
                                const float c = Cf[fidx - 1];
                                diag += c;
                                off += c * xf[cidx - 1];
                            }
                        }
                } else {
                    const float c = sg < 0 ? Cc[LIN(fm, I, J, K)] : Cc[LIN(fm, I + e[0], J + e[1], K + e[2])];
                    if (c > 0.0f) {
                        diag += c;
                        off += c * xc[LIN(s->nc, In, Jn, Kn)];
                    }
                }
            }
        }
    }
    *pdiag = diag;
    *poff = off;
}

/* jacobifine_kernel! / jacobicoarse_kernel! (src/sflip.jl:1219-1243). */
static void jacobi_fine(const S* s, const Comp* L, float* out, const float* x, const float* b, const float* xc) {
    const int N = L->N;
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < N * N * N; c++) {
            const int i = c % N, j = (c / N) % N, k = c / (N * N);
            const int64_t n = (sl - 1) * (int64_t)(N * N * N) + c;
            if (L->actf[n] != 0) {
                float diag, off;
                finerow(s, L, x, xc, sl, i, j, k, w, &diag, &off);
                out[n] = diag > 0.0f ? x[n] + OMEGA * (b[n] - (diag * x[n] - off)) / diag : 0.0f;
            } else {
                out[n] = 0.0f;
            }
        }
    }
}
static void jacobi_coarse(const S* s, const Comp* L, float* out, const float* x, const float* b, const float* xf) {
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                if (L->actc[c] != 0 && !covered(s, I, J, K)) {
                    float diag, off;
                    coarserow(s, L, xf, x, I, J, K, &diag, &off);
                    out[c] = diag > 0.0f ? x[c] + OMEGA * (b[c] - (diag * x[c] - off)) / diag : 0.0f;
                } else {
                    out[c] = 0.0f;
                }
            }
}
/* residualfine_kernel! / residualcoarse_kernel! (src/sflip.jl:1245-1270). */
static void residual_comp(const S* s, const Comp* L, float* rf, float* rc, const float* xf, const float* xc,
                          const float* bf, const float* bc) {
    const int N = L->N;
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < N * N * N; c++) {
            const int i = c % N, j = (c / N) % N, k = c / (N * N);
            const int64_t n = (sl - 1) * (int64_t)(N * N * N) + c;
            if (L->actf[n] != 0) {
                float diag, off;
                finerow(s, L, xf, xc, sl, i, j, k, w, &diag, &off);
                rf[n] = bf[n] - (diag * xf[n] - off);
            } else {
                rf[n] = 0.0f;
            }
        }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                if (L->actc[c] != 0 && !covered(s, I, J, K)) {
                    float diag, off;
                    coarserow(s, L, xf, xc, I, J, K, &diag, &off);
                    rc[c] = bc[c] - (diag * xc[c] - off);
                } else {
                    rc[c] = 0.0f;
                }
            }
}
/* smooth! (src/sflip.jl:1292-1303): `sweeps` pairs of damped Jacobi sweeps x -> t -> x,
   each sweep the fine part then the coarse part, both reading the sweep's source. */
static void smooth_comp(const S* s, const Comp* L, float* xf, float* xc, const float* bf, const float* bc, float* tf,
                        float* tc, int sweeps) {
    for (int q = 0; q < sweeps; q++) {
        jacobi_fine(s, L, tf, xf, bf, xc);
        jacobi_coarse(s, L, tc, xc, bc, xf);
        jacobi_fine(s, L, xf, tf, bf, tc);
        jacobi_coarse(s, L, xc, tc, bc, tf);
    }
}

static Comp level0(const S* s) {
    Comp L = {16, s->cuf, s->cvf, s->cwf, s->dDf, s->B->tf, s->cuc, s->cvc, s->cwc, s->dDc, s->D[0].act};
    return L;
}
static Comp level1(const S* s) {
    Comp L = {8, s->c1x, s->c1y, s->c1z, s->dD1, s->act1, s->cuc, s->cvc, s->cwc, s->dDc, s->D[0].act};
    return L;
}

/* ---- coefficients, level 0 (src/sflip.jl:1315-1451) ---- */
/* celltype (src/sflip.jl:1335-1342) */
static inline uint8_t celltype(const S* s, int I, int J, int K, int* isfine) {
    const int64_t idx = fineat(s, I, J, K);
    if (idx > 0) {
        *isfine = 1;
        return s->B->tf[idx - 1];
    }
    *isfine = 0;
    const int ci = I >> 2, cj = J >> 2, ck = K >> 2;
    if (!(0 <= ci && ci < s->nc[0] && 0 <= cj && cj < s->nc[1] && 0 <= ck && ck < s->nc[2])) return SOLID;
    return s->B->tc[LIN(s->nc, ci, cj, ck)];
}
/* neighbourφ (src/sflip.jl:883-888) */
static inline float nphi(const S* s, int I, int J, int K) {
    const int64_t idx = fineat(s, I, J, K);
    if (idx > 0) return s->B->phif[idx - 1];
    int ci = I >> 2, cj = J >> 2, ck = K >> 2;
    ci = ci < 0 ? 0 : (ci > s->nc[0] - 1 ? s->nc[0] - 1 : ci);
    cj = cj < 0 ? 0 : (cj > s->nc[1] - 1 ? s->nc[1] - 1 : cj);
    ck = ck < 0 ? 0 : (ck > s->nc[2] - 1 ? s->nc[2] - 1 : ck);
    return s->B->phic[LIN(s->nc, ci, cj, ck)];
}
/* The fine face's (slot, local i, j, k) from its offset f in the slot's faces along a (fineface, :365-377). */
static inline void face_local(int a, int f, int* i, int* j, int* k) {
    if (a == 1) {
        *i = f % 17;
        const int r = f / 17;
        *j = r & 15;
        *k = r >> 4;
    } else if (a == 2) {
        *i = f & 15;
        const int r = f >> 4;
        *j = r % 17;
        *k = r / 17;
    } else {
        *i = f & 15;
        *j = (f >> 4) & 15;
        *k = f >> 8;
    }
}
/* finecoef_kernel! (:1324-1333) and coarsecoef_kernel! (:1344-1354) */
static void coefs(S* s) {
    for (int a = 1; a <= 3; a++) {
        float* cf = a == 1 ? s->cuf : (a == 2 ? s->cvf : s->cwf);
        float* cc = a == 1 ? s->cuc : (a == 2 ? s->cvc : s->cwc);
        int e[3], fm[3];
        unitv(a, e);
        fdims(s->nc, a, fm);
        #pragma omp parallel for schedule(static)
        for (int64_t sl = 1; sl <= s->nsl; sl++) {
            const int32_t* w = whereof(s, sl);
            if (w[0] < 0) continue;
            for (int f = 0; f < BFACES; f++) {
                int i, j, k;
                face_local(a, f, &i, &j, &k);
                const int I = w[0] * BLOCK + i, J = w[1] * BLOCK + j, K = w[2] * BLOCK + k;
                int fp, fmn;
                const uint8_t tp = celltype(s, I, J, K, &fp);
                const uint8_t tm = celltype(s, I - e[0], J - e[1], K - e[2], &fmn);
                cf[faceindex(sl, a, i, j, k) - 1] =
                    (tp == LIQUID && tm == LIQUID) ? (fp && fmn ? FINE_FINE : FINE_COARSE) : 0.0f;
            }
        }
        const int n1 = s->nc[0], n2 = s->nc[1], n3 = s->nc[2];
        #pragma omp parallel for schedule(static)
        for (int K = 0; K < fm[2]; K++)
            for (int J = 0; J < fm[1]; J++)
                for (int I = 0; I < fm[0]; I++) {
                    const int Im = I - e[0], Jm = J - e[1], Km = K - e[2];
                    const int ok = 0 <= Im && 0 <= Jm && 0 <= Km && I < n1 && J < n2 && K < n3;
                    cc[LIN(fm, I, J, K)] = (ok && !covered(s, I, J, K) && !covered(s, Im, Jm, Km) &&
                                            s->B->tc[LIN(s->nc, I, J, K)] == LIQUID &&
                                            s->B->tc[LIN(s->nc, Im, Jm, Km)] == LIQUID)
                                               ? COARSE_COARSE
                                               : 0.0f;
                }
    }
}
static const int NB[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
/* finedirichlet_kernel! (:1356-1374) and coarsedirichlet_kernel! (:1376-1407) */
static void dirichlet(S* s) {
    const ors_basin* B = s->B;
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int64_t n = (sl - 1) * BCELLS + c;
            float d = 0.0f;
            if (B->tf[n] == LIQUID) {
                const int I = w[0] * BLOCK + (c & 15), J = w[1] * BLOCK + ((c >> 4) & 15), K = w[2] * BLOCK + (c >> 8);
                const float pc = B->phif[n];
                for (int m = 0; m < 6; m++) {
                    const int a = I + NB[m][0], b = J + NB[m][1], cc = K + NB[m][2];
                    int isfine;
                    const uint8_t ty = celltype(s, a, b, cc, &isfine);
                    if (ty == AIR) d += (isfine ? FINE_FINE : FINE_COARSE) / theta(pc, nphi(s, a, b, cc));
                }
            }
            s->dDf[n] = d;
        }
    }
    const int n1 = s->nc[0], n2 = s->nc[1], n3 = s->nc[2];
    for (int K = 0; K < n3; K++)
        for (int J = 0; J < n2; J++)
            for (int I = 0; I < n1; I++) {
                float d = 0.0f;
                const int64_t ci = LIN(s->nc, I, J, K);
                if (B->tc[ci] == LIQUID && !covered(s, I, J, K)) {
                    const float pc = B->phic[ci];
                    for (int a = 1; a <= 3; a++) {
                        int e[3];
                        unitv(a, e);
                        for (int sg = -1; sg <= 1; sg += 2) {
                            const int In = I + sg * e[0], Jn = J + sg * e[1], Kn = K + sg * e[2];
                            if (0 <= In && In < n1 && 0 <= Jn && Jn < n2 && 0 <= Kn && Kn < n3) {
                                if (covered(s, In, Jn, Kn)) {
                                    for (int q = 0; q < 4; q++)
                                        for (int p = 0; p < 4; p++) {
                                            const int FI = a == 1 ? (sg > 0 ? RATIO * In : RATIO * I - 1) : RATIO * I + p;
                                            const int FJ =
                                                a == 2 ? (sg > 0 ? RATIO * Jn : RATIO * J - 1) : RATIO * J + (a == 1 ? p : q);
                                            const int FK = a == 3 ? (sg > 0 ? RATIO * Kn : RATIO * K - 1) : RATIO * K + q;
                                            const int64_t idx = fineat(s, FI, FJ, FK);
                                            if (idx > 0 && B->tf[idx - 1] == AIR)
                                                d += FINE_COARSE / theta(pc, B->phif[idx - 1]);
                                        }
                                } else if (B->tc[LIN(s->nc, In, Jn, Kn)] == AIR) {
                                    d += COARSE_COARSE / theta(pc, B->phic[LIN(s->nc, In, Jn, Kn)]);
                                }
                            }
                        }
                    }
                }
                s->dDc[ci] = d;
            }
}
/* coefficients! (:1437-1451) with activecoarse_kernel! (:1315-1319) */
static void coefficients(S* s) {
    coefs(s);
    dirichlet(s);
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                s->D[0].act[c] = (s->B->tc[c] == LIQUID && !covered(s, I, J, K)) ? 1 : 0;
            }
}

/* ---- the hierarchy (src/sflip.jl:1453-1586) ---- */
static void hierarchy(S* s) {
    /* coef1_kernel! (:1453-1465) */
    for (int a = 1; a <= 3; a++) {
        const float* c0 = a == 1 ? s->cuf : (a == 2 ? s->cvf : s->cwf);
        float* c1 = a == 1 ? s->c1x : (a == 2 ? s->c1y : s->c1z);
        #pragma omp parallel for schedule(static)
        for (int64_t sl = 1; sl <= s->nsl; sl++) {
            if (whereof(s, sl)[0] < 0) continue;
            for (int f = 0; f < 9 * 64; f++) {
                int i, j, k;
                if (a == 1) { i = f % 9; const int r = f / 9; j = r % 8; k = r / 8; }
                else if (a == 2) { i = f % 8; const int r = f / 8; j = r % 9; k = r / 9; }
                else { i = f % 8; const int r = f / 8; j = r % 8; k = r / 8; }
                float acc = 0.0f;
                for (int q = 0; q < 2; q++)
                    for (int p = 0; p < 2; p++) {
                        const int ii = a == 1 ? 2 * i : 2 * i + p;
                        const int jj = a == 2 ? 2 * j : 2 * j + (a == 1 ? p : q);
                        const int kk = a == 3 ? 2 * k : 2 * k + q;
                        acc += c0[faceidx(16, sl, a, ii, jj, kk) - 1];
                    }
                c1[faceidx(8, sl, a, i, j, k) - 1] = acc;
            }
        }
    }
    /* cells1_kernel! (:1467-1479) */
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        if (whereof(s, sl)[0] < 0) continue;
        for (int c = 0; c < 512; c++) {
            const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
            float d = 0.0f;
            uint8_t act = 0;
            for (int cc = 0; cc < 2; cc++)
                for (int b = 0; b < 2; b++)
                    for (int a = 0; a < 2; a++) {
                        const int64_t m = cellidx(16, sl, 2 * i + a, 2 * j + b, 2 * k + cc) - 1;
                        d += s->dDf[m];
                        if (s->B->tf[m] == LIQUID) act = 1;
                    }
            s->dD1[(sl - 1) * 512 + c] = d;
            s->act1[(sl - 1) * 512 + c] = act;
        }
    }
    /* coef2_kernel! (:1485-1507) and cells2_kernel! (:1509-1523) into D[0] (level 2) */
    DLev* D2 = &s->D[0];
    for (int a = 1; a <= 3; a++) {
        const float* c0c = a == 1 ? s->cuc : (a == 2 ? s->cvc : s->cwc);
        const float* c1 = a == 1 ? s->c1x : (a == 2 ? s->c1y : s->c1z);
        float* c2 = a == 1 ? D2->cx : (a == 2 ? D2->cy : D2->cz);
        int e[3], fm[3];
        unitv(a, e);
        fdims(s->nc, a, fm);
        #pragma omp parallel for schedule(static)
        for (int K = 0; K < fm[2]; K++)
            for (int J = 0; J < fm[1]; J++)
                for (int I = 0; I < fm[0]; I++) {
                    const int64_t o = LIN(fm, I, J, K);
                    if (covered(s, I, J, K) || covered(s, I - e[0], J - e[1], K - e[2])) {
                        float acc = 0.0f;
                        for (int q = 0; q < 2; q++)
                            for (int p = 0; p < 2; p++) {
                                const int FI = a == 1 ? 2 * I : 2 * I + p;
                                const int FJ = a == 2 ? 2 * J : 2 * J + (a == 1 ? p : q);
                                const int FK = a == 3 ? 2 * K : 2 * K + q;
                                const int64_t idx = faceat(s, 8, a, FI, FJ, FK);
                                if (idx > 0) acc += c1[idx - 1];
                            }
                        c2[o] = acc;
                    } else {
                        c2[o] = c0c[o];
                    }
                }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t o = LIN(s->nc, I, J, K);
                if (covered(s, I, J, K)) {
                    float d = 0.0f;
                    uint8_t act = 0;
                    for (int c = 0; c < 2; c++)
                        for (int b = 0; b < 2; b++)
                            for (int a = 0; a < 2; a++) {
                                const int64_t m = cellat(s, 8, 2 * I + a, 2 * J + b, 2 * K + c) - 1;
                                d += s->dD1[m];
                                if (s->act1[m] != 0) act = 1;
                            }
                    D2->dD[o] = d;
                    D2->act[o] = act;
                } else {
                    D2->dD[o] = s->dDc[o];
                }
            }
    /* coefdense_kernel! (:1525-1535) and cellsdense_kernel! (:1537-1546), level by level */
    for (int l = 1; l < s->nd; l++) {
        const DLev* F = &s->D[l - 1];
        DLev* C = &s->D[l];
        for (int a = 1; a <= 3; a++) {
            const float* cf = a == 1 ? F->cx : (a == 2 ? F->cy : F->cz);
            float* cc = a == 1 ? C->cx : (a == 2 ? C->cy : C->cz);
            int fmf[3], fmc[3];
            fdims(F->n, a, fmf);
            fdims(C->n, a, fmc);
            #pragma omp parallel for schedule(static)
            for (int K = 0; K < fmc[2]; K++)
                for (int J = 0; J < fmc[1]; J++)
                    for (int I = 0; I < fmc[0]; I++) {
                        float acc = 0.0f;
                        for (int q = 0; q < 2; q++)
                            for (int p = 0; p < 2; p++) {
                                const int FI = a == 1 ? 2 * I : 2 * I + p;
                                const int FJ = a == 2 ? 2 * J : 2 * J + (a == 1 ? p : q);
                                const int FK = a == 3 ? 2 * K : 2 * K + q;
                                acc += cf[LIN(fmf, FI, FJ, FK)];
                            }
                        cc[LIN(fmc, I, J, K)] = acc;
                    }
        }
        for (int K = 0; K < C->n[2]; K++)
            for (int J = 0; J < C->n[1]; J++)
                for (int I = 0; I < C->n[0]; I++) {
                    float d = 0.0f;
                    uint8_t act = 0;
                    for (int c = 0; c < 2; c++)
                        for (int b = 0; b < 2; b++)
                            for (int a = 0; a < 2; a++) {
                                const int64_t m = LIN(F->n, 2 * I + a, 2 * J + b, 2 * K + c);
                                d += F->dD[m];
                                if (F->act[m] != 0) act = 1;
                            }
                    C->dD[LIN(C->n, I, J, K)] = d;
                    C->act[LIN(C->n, I, J, K)] = act;
                }
    }
}

/* ---- the dense levels (src/sflip.jl:1575-1660) ---- */
/* denserow (:1575-1586) */
static inline void denserow(const DLev* L, const float* x, int i, int j, int k, float* pdiag, float* poff) {
    const int n1 = L->n[0], n2 = L->n[1], n3 = L->n[2];
    int fx[3], fy[3], fz[3];
    fdims(L->n, 1, fx);
    fdims(L->n, 2, fy);
    fdims(L->n, 3, fz);
    float diag = L->dD[LIN(L->n, i, j, k)], off = 0.0f, c;
    c = L->cx[LIN(fx, i, j, k)];
    if (c > 0.0f && i > 0) { diag += c; off += c * x[LIN(L->n, i - 1, j, k)]; }
    c = L->cx[LIN(fx, i + 1, j, k)];
    if (c > 0.0f && i < n1 - 1) { diag += c; off += c * x[LIN(L->n, i + 1, j, k)]; }
    c = L->cy[LIN(fy, i, j, k)];
    if (c > 0.0f && j > 0) { diag += c; off += c * x[LIN(L->n, i, j - 1, k)]; }
    c = L->cy[LIN(fy, i, j + 1, k)];
    if (c > 0.0f && j < n2 - 1) { diag += c; off += c * x[LIN(L->n, i, j + 1, k)]; }
    c = L->cz[LIN(fz, i, j, k)];
    if (c > 0.0f && k > 0) { diag += c; off += c * x[LIN(L->n, i, j, k - 1)]; }
    c = L->cz[LIN(fz, i, j, k + 1)];
    if (c > 0.0f && k < n3 - 1) { diag += c; off += c * x[LIN(L->n, i, j, k + 1)]; }
    *pdiag = diag;
    *poff = off;
}
/* jacobidense_kernel! (:1588-1596) */
static void jacobi_dense(const DLev* L, float* out, const float* x) {
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < L->n[2]; k++)
        for (int j = 0; j < L->n[1]; j++)
            for (int i = 0; i < L->n[0]; i++) {
                const int64_t c = LIN(L->n, i, j, k);
                if (L->act[c] != 0) {
                    float diag, off;
                    denserow(L, x, i, j, k, &diag, &off);
                    out[c] = diag > 0.0f ? x[c] + OMEGA * (L->b[c] - (diag * x[c] - off)) / diag : 0.0f;
                } else {
                    out[c] = 0.0f;
                }
            }
}
/* residualdense_kernel! (:1598-1607) */
static void residual_dense(DLev* L) {
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < L->n[2]; k++)
        for (int j = 0; j < L->n[1]; j++)
            for (int i = 0; i < L->n[0]; i++) {
                const int64_t c = LIN(L->n, i, j, k);
                if (L->act[c] != 0) {
                    float diag, off;
                    denserow(L, L->x, i, j, k, &diag, &off);
                    L->r[c] = L->b[c] - (diag * L->x[c] - off);
                } else {
                    L->r[c] = 0.0f;
                }
            }
}
/* restrictdense_kernel! (:1609-1616) */
static void restrict_dense(const DLev* F, DLev* C) {
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < C->n[2]; k++)
        for (int j = 0; j < C->n[1]; j++)
            for (int i = 0; i < C->n[0]; i++) {
                float acc = 0.0f;
                for (int c = 0; c < 2; c++)
                    for (int b = 0; b < 2; b++)
                        for (int a = 0; a < 2; a++) acc += F->r[LIN(F->n, 2 * i + a, 2 * j + b, 2 * k + c)];
                C->b[LIN(C->n, i, j, k)] = acc;
            }
}
/* prolongdense_kernel! (:1618-1621) */
static void prolong_dense(DLev* F, const DLev* C, float boost) {
    #pragma omp parallel for schedule(static)
    for (int k = 0; k < F->n[2]; k++)
        for (int j = 0; j < F->n[1]; j++)
            for (int i = 0; i < F->n[0]; i++) {
                const int64_t c = LIN(F->n, i, j, k);
                if (F->act[c] != 0) F->x[c] += boost * C->x[LIN(C->n, i >> 1, j >> 1, k >> 1)];
            }
}
/* coarsest_kernel! (:1627-1660): red-black Gauss-Seidel from zero in one workgroup,
   `sweeps` sweeps and as many in the reverse colour order. */
static void coarsest(DLev* L, int sweeps) {
    const int n1 = L->n[0], n2 = L->n[1], n3 = L->n[2], N = n1 * n2 * n3;
    int fx[3], fy[3], fz[3];
    fdims(L->n, 1, fx);
    fdims(L->n, 2, fy);
    fdims(L->n, 3, fz);
    float* xs = (float*)calloc((size_t)N + 1, sizeof(float));
    for (int s = 1; s <= 2 * sweeps; s++)
        for (int half = 0; half <= 1; half++) {
            const int colour = s <= sweeps ? half : 1 - half;
            for (int t = 0; t < N; t++) {
                const int i = t % n1, j = (t / n1) % n2, k = t / (n1 * n2);
                if (L->act[t] == 0 || ((i + j + k + 3) % 2) != colour) continue;
                float diag = L->dD[t], acc = L->b[t], c;
                c = L->cx[LIN(fx, i, j, k)];
                if (c > 0.0f && i > 0) { diag += c; acc += c * xs[t - 1]; }
                c = L->cx[LIN(fx, i + 1, j, k)];
                if (c > 0.0f && i < n1 - 1) { diag += c; acc += c * xs[t + 1]; }
                c = L->cy[LIN(fy, i, j, k)];
                if (c > 0.0f && j > 0) { diag += c; acc += c * xs[t - n1]; }
                c = L->cy[LIN(fy, i, j + 1, k)];
                if (c > 0.0f && j < n2 - 1) { diag += c; acc += c * xs[t + n1]; }
                c = L->cz[LIN(fz, i, j, k)];
                if (c > 0.0f && k > 0) { diag += c; acc += c * xs[t - n1 * n2]; }
                c = L->cz[LIN(fz, i, j, k + 1)];
                if (c > 0.0f && k < n3 - 1) { diag += c; acc += c * xs[t + n1 * n2]; }
                xs[t] = diag > 0.0f ? acc / diag : 0.0f;
            }
        }
    for (int t = 0; t < N; t++) L->x[t] = xs[t];
    free(xs);
}

/* ---- between levels (src/sflip.jl:1662-1705) and vcycle! (:1722-1764) ---- */
static void vcycle(S* s, float* zf, float* zc, const float* rf, const float* rc, int sweeps, int coarse, float boost) {
    const int64_t nf0 = s->nsl * BCELLS, nf1 = s->nsl * 512;
    const Comp L0 = level0(s), L1 = level1(s);
    memset(zf, 0, sizeof(float) * nf0);
    memset(zc, 0, sizeof(float) * s->ncc);
    smooth_comp(s, &L0, zf, zc, rf, rc, s->tmf, s->tmc, sweeps);
    residual_comp(s, &L0, s->qf, s->qc, zf, zc, rf, rc);
    /* restrict01_kernel! (:1662-1672) */
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        if (whereof(s, sl)[0] < 0) continue;
        for (int c = 0; c < 512; c++) {
            const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
            float acc = 0.0f;
            for (int cc = 0; cc < 2; cc++)
                for (int b = 0; b < 2; b++)
                    for (int a = 0; a < 2; a++) acc += s->qf[cellidx(16, sl, 2 * i + a, 2 * j + b, 2 * k + cc) - 1];
            s->b1f[(sl - 1) * 512 + c] = acc;
        }
    }
    memcpy(s->b1c, s->qc, sizeof(float) * s->ncc);
    memset(s->x1f, 0, sizeof(float) * nf1);
    memset(s->x1c, 0, sizeof(float) * s->ncc);
    smooth_comp(s, &L1, s->x1f, s->x1c, s->b1f, s->b1c, s->t1f, s->t1c, sweeps);
    residual_comp(s, &L1, s->r1f, s->r1c, s->x1f, s->x1c, s->b1f, s->b1c);
    /* restrict12_kernel! (:1674-1686) */
    DLev* D = s->D;
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t o = LIN(s->nc, I, J, K);
                if (covered(s, I, J, K)) {
                    float acc = 0.0f;
                    for (int c = 0; c < 2; c++)
                        for (int b = 0; b < 2; b++)
                            for (int a = 0; a < 2; a++) acc += s->r1f[cellat(s, 8, 2 * I + a, 2 * J + b, 2 * K + c) - 1];
                    D[0].b[o] = acc;
                } else {
                    D[0].b[o] = s->r1c[o];
                }
            }
    for (int l = 0; l + 1 < s->nd; l++) {
        DLev* Dl = &D[l];
        const int64_t m = (int64_t)Dl->n[0] * Dl->n[1] * Dl->n[2];
        memset(Dl->x, 0, sizeof(float) * m);
        for (int q = 0; q < sweeps; q++) {
            jacobi_dense(Dl, Dl->t, Dl->x);
            jacobi_dense(Dl, Dl->x, Dl->t);
        }
        residual_dense(Dl);
        restrict_dense(Dl, &D[l + 1]);
    }
    coarsest(&D[s->nd - 1], coarse);
    for (int l = s->nd - 2; l >= 0; l--) {
        DLev* Dl = &D[l];
        prolong_dense(Dl, &D[l + 1], boost);
        for (int q = 0; q < sweeps; q++) {
            jacobi_dense(Dl, Dl->t, Dl->x);
            jacobi_dense(Dl, Dl->x, Dl->t);
        }
    }
    /* prolong21fine_kernel! (:1688-1693) and prolongcoarse_kernel! (:1695-1699) */
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < 512; c++) {
            const int64_t n = (sl - 1) * 512 + c;
            if (s->act1[n] == 0) continue;
            const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
            s->x1f[n] += boost * D[0].x[LIN(s->nc, (w[0] * 8 + i) >> 1, (w[1] * 8 + j) >> 1, (w[2] * 8 + k) >> 1)];
        }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t o = LIN(s->nc, I, J, K);
                if (D[0].act[o] != 0 && !covered(s, I, J, K)) s->x1c[o] += boost * D[0].x[o];
            }
    smooth_comp(s, &L1, s->x1f, s->x1c, s->b1f, s->b1c, s->t1f, s->t1c, sweeps);
    /* prolong10fine_kernel! (:1701-1705) and prolongcoarse_kernel! */
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        if (whereof(s, sl)[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int64_t n = (sl - 1) * BCELLS + c;
            if (s->B->tf[n] != LIQUID) continue;
            const int i = c & 15, j = (c >> 4) & 15, k = c >> 8;
            zf[n] += boost * s->x1f[cellidx(8, sl, i >> 1, j >> 1, k >> 1) - 1];
        }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t o = LIN(s->nc, I, J, K);
                if (D[0].act[o] != 0 && !covered(s, I, J, K)) zc[o] += boost * s->x1c[o];
            }
    smooth_comp(s, &L0, zf, zc, rf, rc, s->tmf, s->tmc, sweeps);
}

/* ---- vectors (src/sflip.jl:1766-1822) ---- */
static inline float tree256(float* v) { /* groupsum! (src/flip.jl:1020-1031) */
    for (int step = 128; step >= 1; step >>= 1)
        for (int t = 0; t < step; t++) v[t] += v[t + step];
    return v[0];
}
/* inner (:1794-1805): FP32 partials of 256 consecutive pool cells (LIQUID cells of slots in
   use), summed, plus the coarse grid's (LIQUID cells outside fine blocks). */
static float inner(const S* s, const float* af, const float* ac, const float* bf, const float* bc) {
    const int64_t nf = s->nsl * BCELLS, gf = (nf + 255) / 256, gc = (s->ncc + 255) / 256;
    float* part = (float*)malloc(sizeof(float) * (size_t)(gf + gc + 1));
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < gf; g++) {
        float v[256];
        for (int t = 0; t < 256; t++) {
            const int64_t i = g * 256 + t;
            v[t] = 0.0f;
            if (i < nf && s->B->tf[i] == LIQUID && whereof(s, i / BCELLS + 1)[0] >= 0) v[t] = af[i] * bf[i];
        }
        part[g] = tree256(v);
    }
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < gc; g++) {
        float v[256];
        for (int t = 0; t < 256; t++) {
            const int64_t i = g * 256 + t;
            v[t] = 0.0f;
            if (i < s->ncc && s->B->tc[i] == LIQUID) {
                const int I = (int)(i % s->nc[0]), J = (int)((i / s->nc[0]) % s->nc[1]), K = (int)(i / ((int64_t)s->nc[0] * s->nc[1]));
                if (!covered(s, I, J, K)) v[t] = ac[i] * bc[i];
            }
        }
        part[gf + g] = tree256(v);
    }
    float acc = 0.0f, acc2 = 0.0f;
    for (int64_t g = 0; g < gf; g++) acc += part[g];
    for (int64_t g = 0; g < gc; g++) acc2 += part[gf + g];
    free(part);
    return acc + acc2;
}
static void axpy(const S* s, float* yf, float* yc, float a, const float* xf, const float* xc) {
    const int64_t nf = s->nsl * BCELLS;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; i++) yf[i] += a * xf[i];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s->ncc; i++) yc[i] += a * xc[i];
}
static void xpby(const S* s, float* yf, float* yc, const float* xf, const float* xc, float b) {
    const int64_t nf = s->nsl * BCELLS;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nf; i++) yf[i] = xf[i] + b * yf[i];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s->ncc; i++) yc[i] = xc[i] + b * yc[i];
}
static void copyv(const S* s, float* yf, float* yc, const float* xf, const float* xc) {
    memcpy(yf, xf, sizeof(float) * s->nsl * BCELLS);
    memcpy(yc, xc, sizeof(float) * s->ncc);
}
/* apply! (:1824-1865): q = A x at level 0 (LIQUID fine cells; active uncovered coarse ones). */
static void apply(const S* s, float* qf, float* qc, const float* xf, const float* xc) {
    const Comp L = level0(s);
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int64_t n = (sl - 1) * BCELLS + c;
            if (s->B->tf[n] == LIQUID) {
                float diag, off;
                finerow(s, &L, xf, xc, sl, c & 15, (c >> 4) & 15, c >> 8, w, &diag, &off);
                qf[n] = diag * xf[n] - off;
            } else {
                qf[n] = 0.0f;
            }
        }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                if (L.actc[c] != 0 && !covered(s, I, J, K)) {
                    float diag, off;
                    coarserow(s, &L, xf, xc, I, J, K, &diag, &off);
                    qc[c] = diag * xc[c] - off;
                } else {
                    qc[c] = 0.0f;
                }
            }
}

/* ---- the solver's workspace ---- */
static void* zal(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }
static int S_init(S* s, const ors_basin* B) {
    memset(s, 0, sizeof(*s));
    s->B = B;
    for (int a = 0; a < 3; a++) {
        s->nb[a] = B->g.nb[a];
        s->nc[a] = B->g.nb[a] * 4;
    }
    s->ncc = (int64_t)s->nc[0] * s->nc[1] * s->nc[2];
    s->nsl = B->nslots;
    const int64_t nf = s->nsl * BCELLS, nff = s->nsl * BFACES, n1 = s->nsl * 512, f1 = s->nsl * 576;
    int fm[3];
    s->cuf = zal(nff, 4); s->cvf = zal(nff, 4); s->cwf = zal(nff, 4);
    fdims(s->nc, 1, fm); s->cuc = zal(LIN(fm, 0, 0, fm[2]), 4);
    fdims(s->nc, 2, fm); s->cvc = zal(LIN(fm, 0, 0, fm[2]), 4);
    fdims(s->nc, 3, fm); s->cwc = zal(LIN(fm, 0, 0, fm[2]), 4);
    s->dDf = zal(nf, 4); s->dDc = zal(s->ncc, 4);
    s->c1x = zal(f1, 4); s->c1y = zal(f1, 4); s->c1z = zal(f1, 4);
    s->dD1 = zal(n1, 4); s->act1 = zal(n1, 1);
    s->x1f = zal(n1, 4); s->b1f = zal(n1, 4); s->r1f = zal(n1, 4); s->t1f = zal(n1, 4);
    s->x1c = zal(s->ncc, 4); s->b1c = zal(s->ncc, 4); s->r1c = zal(s->ncc, 4); s->t1c = zal(s->ncc, 4);
    /* the coarse grid and its halvings, until a workgroup can solve the coarsest (:318-326) */
    int m[3] = {s->nc[0], s->nc[1], s->nc[2]};
    for (;;) {
        if (s->nd == MAXD) return -1;
        DLev* L = &s->D[s->nd++];
        memcpy(L->n, m, sizeof(m));
        const int64_t c = (int64_t)m[0] * m[1] * m[2];
        L->x = zal(c, 4); L->b = zal(c, 4); L->r = zal(c, 4); L->t = zal(c, 4); L->dD = zal(c, 4);
        L->act = zal(c, 1);
        fdims(m, 1, fm); L->cx = zal(LIN(fm, 0, 0, fm[2]), 4);
        fdims(m, 2, fm); L->cy = zal(LIN(fm, 0, 0, fm[2]), 4);
        fdims(m, 3, fm); L->cz = zal(LIN(fm, 0, 0, fm[2]), 4);
        if (c <= 1024 || (m[0] & 1) || (m[1] & 1) || (m[2] & 1)) break;
        m[0] /= 2; m[1] /= 2; m[2] /= 2;
    }
    if ((int64_t)m[0] * m[1] * m[2] > 1024) return -1;
    float** v[] = {&s->bf, &s->rf, &s->zf, &s->df, &s->qf, &s->rof, &s->tmf};
    float** vc[] = {&s->bc, &s->rc, &s->zc, &s->dc, &s->qc, &s->roc, &s->tmc};
    for (int q = 0; q < 7; q++) {
        *v[q] = zal(nf, 4);
        *vc[q] = zal(s->ncc, 4);
    }
    return 0;
}
static void S_free(S* s) {
    void* p[] = {s->cuf, s->cvf, s->cwf, s->cuc, s->cvc, s->cwc, s->dDf, s->dDc, s->c1x, s->c1y, s->c1z, s->dD1,
                 s->act1, s->x1f, s->b1f, s->r1f, s->t1f, s->x1c, s->b1c, s->r1c, s->t1c, s->bf, s->rf, s->zf,
                 s->df, s->qf, s->rof, s->tmf, s->bc, s->rc, s->zc, s->dc, s->qc, s->roc, s->tmc};
    for (size_t q = 0; q < sizeof(p) / sizeof(p[0]); q++) free(p[q]);
    for (int l = 0; l < s->nd; l++) {
        DLev* L = &s->D[l];
        void* d[] = {L->x, L->b, L->r, L->t, L->dD, L->act, L->cx, L->cy, L->cz};
        for (int q = 0; q < 9; q++) free(d[q]);
    }
}

/* ---- pressure! (src/sflip.jl:1867-1904): flexible PCG from the warm start P ---- */
static int pressure_pcg(S* s, float* Pf, float* Pc, float tol, int maxiter, int sweeps, float boost, int* status,
                        float* rel) {
    hierarchy(s);
    apply(s, s->rf, s->rc, Pf, Pc);
    xpby(s, s->rf, s->rc, s->bf, s->bc, -1.0f);
    const float bnorm = sqrtf(inner(s, s->bf, s->bc, s->bf, s->bc));
    *rel = 0.0f;
    if (!isfinite(bnorm)) { *status = ORS_NONFINITE; return 0; }
    if (bnorm == 0.0f) { *status = ORS_OK; return 0; }
    const float target = tol * bnorm;
    float rnorm = sqrtf(inner(s, s->rf, s->rc, s->rf, s->rc));
    *rel = rnorm / bnorm;
    if (rnorm <= target) { *status = ORS_OK; return 0; }
    vcycle(s, s->zf, s->zc, s->rf, s->rc, sweeps, 40, boost);
    copyv(s, s->df, s->dc, s->zf, s->zc);
    float rho = inner(s, s->zf, s->zc, s->rf, s->rc);
    if (!isfinite(rho)) { *status = ORS_NONFINITE; return 0; }
    if (!(rho > 0.0f)) { *status = ORS_INDEFINITE; return 0; }
    for (int it = 1; it <= maxiter; it++) {
        apply(s, s->qf, s->qc, s->df, s->dc);
        const float den = inner(s, s->df, s->dc, s->qf, s->qc);
        if (!(den > 0.0f)) { *status = ORS_INDEFINITE; return it; }
        const float alpha = rho / den;
        if (!isfinite(alpha)) { *status = ORS_NONFINITE; return it; }
        axpy(s, Pf, Pc, alpha, s->df, s->dc);
        copyv(s, s->rof, s->roc, s->rf, s->rc);
        axpy(s, s->rf, s->rc, -alpha, s->qf, s->qc);
        rnorm = sqrtf(inner(s, s->rf, s->rc, s->rf, s->rc));
        *rel = rnorm / bnorm;
        if (rnorm <= target) { *status = ORS_OK; return it; }
        vcycle(s, s->zf, s->zc, s->rf, s->rc, sweeps, 40, boost);
        const float rnew = inner(s, s->zf, s->zc, s->rf, s->rc);
        if (!(rnew > 0.0f)) { *status = ORS_INDEFINITE; return it; }
        float beta = (rnew - inner(s, s->zf, s->zc, s->rof, s->roc)) / rho;
        beta = beta != beta ? beta : (beta > 0.0f ? beta : 0.0f); /* Julia's max(0f0, x): NaN propagates */
        if (!isfinite(beta)) { *status = ORS_NONFINITE; return it; }
        rho = rnew;
        xpby(s, s->df, s->dc, s->zf, s->zc, beta);
    }
    *status = ORS_NOT_CONVERGED;
    return maxiter;
}

/* sparse_diagonal_precondition! (src/fgmres.jl:15-24): one damped Jacobi step from zero. */
static void diagonal_precondition(S* s, float* zf, float* zc, const float* rf, const float* rc) {
    const Comp L = level0(s);
    memset(s->tmf, 0, sizeof(float) * s->nsl * BCELLS);
    memset(s->tmc, 0, sizeof(float) * s->ncc);
    jacobi_fine(s, &L, zf, s->tmf, rf, s->tmc);
    jacobi_coarse(s, &L, zc, s->tmc, rc, s->tmf);
}

/* pressure_fgmres! (src/fgmres.jl:26-92): restarted right-preconditioned FGMRES, FP32 basis
   with two Gram-Schmidt passes, FP64 Hessenberg and Givens rotations. */
#define FGR 8
static int pressure_fgmres(S* s, float* Pf, float* Pc, float tol, int maxiter, int sweeps, float boost, int* status,
                           float* rel) {
    hierarchy(s);
    const int64_t nf = s->nsl * BCELLS, nc = s->ncc;
    float *Vf[FGR + 1], *Vc[FGR + 1], *Zf[FGR], *Zc[FGR];
    for (int j = 0; j <= FGR; j++) { Vf[j] = zal(nf, 4); Vc[j] = zal(nc, 4); }
    for (int j = 0; j < FGR; j++) { Zf[j] = zal(nf, 4); Zc[j] = zal(nc, 4); }
    int its = 0;
    const float bnorm = sqrtf(inner(s, s->bf, s->bc, s->bf, s->bc));
    *status = ORS_OK;
    *rel = 0.0f;
    if (!isfinite(bnorm)) { *status = ORS_NONFINITE; goto done; }
    if (bnorm == 0.0f) {
        memset(Pf, 0, sizeof(float) * nf);
        memset(Pc, 0, sizeof(float) * nc);
        goto done;
    }
    {
        const float target = tol * bnorm;
#define ACTUAL_RESIDUAL()                                                   \
    (apply(s, s->qf, s->qc, Pf, Pc), copyv(s, s->rf, s->rc, s->bf, s->bc), \
     axpy(s, s->rf, s->rc, -1.0f, s->qf, s->qc), sqrtf(inner(s, s->rf, s->rc, s->rf, s->rc)))
        float residual = ACTUAL_RESIDUAL();
        while (residual > target && its < maxiter) {
            if (!isfinite(residual)) { *status = ORS_NONFINITE; goto done; }
            double H[FGR + 1][FGR], g[FGR + 1], cs[FGR], sn[FGR];
            memset(H, 0, sizeof(H));
            memset(g, 0, sizeof(g));
            g[0] = residual;
            memset(Vf[0], 0, sizeof(float) * nf);
            memset(Vc[0], 0, sizeof(float) * nc);
            axpy(s, Vf[0], Vc[0], 1.0f / residual, s->rf, s->rc);
            int used = 0;
            const int jmax = FGR < maxiter - its ? FGR : maxiter - its;
            for (int j = 0; j < jmax; j++) {
                vcycle(s, s->zf, s->zc, Vf[j], Vc[j], sweeps, 40, boost);
                diagonal_precondition(s, Zf[j], Zc[j], Vf[j], Vc[j]);
                axpy(s, Zf[j], Zc[j], 1.0f, s->zf, s->zc);
                apply(s, s->qf, s->qc, Zf[j], Zc[j]);
                for (int pass = 0; pass < 2; pass++)
                    for (int i = 0; i <= j; i++) {
                        const float h = inner(s, s->qf, s->qc, Vf[i], Vc[i]);
                        H[i][j] += (double)h;
                        axpy(s, s->qf, s->qc, -h, Vf[i], Vc[i]);
                    }
                const float hnext = sqrtf(inner(s, s->qf, s->qc, s->qf, s->qc));
                if (!isfinite(hnext)) { *status = ORS_NONFINITE; goto done; }
                H[j + 1][j] = hnext;
                if (hnext > 0.0f) {
                    memset(Vf[j + 1], 0, sizeof(float) * nf);
                    memset(Vc[j + 1], 0, sizeof(float) * nc);
                    axpy(s, Vf[j + 1], Vc[j + 1], 1.0f / hnext, s->qf, s->qc);
                }
                for (int i = 0; i < j; i++) {
                    const double a = H[i][j], b = H[i + 1][j];
                    H[i][j] = cs[i] * a + sn[i] * b;
                    H[i + 1][j] = -sn[i] * a + cs[i] * b;
                }
                const double a = H[j][j], b = H[j + 1][j];
                const double hyp = hypot(a, b);
                if (!(hyp > 0)) { *status = ORS_BREAKDOWN; goto done; }
                cs[j] = a / hyp;
                sn[j] = b / hyp;
                H[j][j] = hyp;
                H[j + 1][j] = 0;
                g[j + 1] = -sn[j] * g[j];
                g[j] = cs[j] * g[j];
                used = j + 1;
                its++;
                if (fabs(g[j + 1]) <= target || hnext == 0.0f) break;
            }
            double y[FGR];
            for (int i = used - 1; i >= 0; i--) {
                double acc = g[i];
                for (int q = i + 1; q < used; q++) acc -= H[i][q] * y[q];
                y[i] = acc / H[i][i];
            }
            for (int j = 0; j < used; j++) axpy(s, Pf, Pc, (float)y[j], Zf[j], Zc[j]);
            residual = ACTUAL_RESIDUAL();
        }
#undef ACTUAL_RESIDUAL
        *rel = residual / bnorm;
        if (!(residual <= target)) *status = ORS_NOT_CONVERGED;
    }
done:
    for (int j = 0; j <= FGR; j++) { free(Vf[j]); free(Vc[j]); }
    for (int j = 0; j < FGR; j++) { free(Zf[j]); free(Zc[j]); }
    return its;
}

/* The pressure solve: the flexible PCG alone (pressure!(::SparseBasin), src/sflip.jl:1867),
   or, with `fallback`, the dispatch of src/fgmres.jl:96-110: CG with at most 80 iterations
   (its errors caught, its iteration count then 0), the true residual checked, P zeroed if
   that residual is nonfinite or above 2|b|, and FGMRES from there. */
static int pressure_dispatch(S* s, float* Pf, float* Pc, const ors_opts* o, ors_info* info) {
    int status = ORS_OK, its = 0;
    float rel = 0.0f;
    info->fgmres_iterations = 0;
    if (!o->fallback) {
        its = pressure_pcg(s, Pf, Pc, o->tol, o->maxiter, o->sweeps, o->boost, &status, &rel);
    } else {
        const int cap = o->maxiter < o->cg_maxiter ? o->maxiter : o->cg_maxiter;
        int st;
        its = pressure_pcg(s, Pf, Pc, o->tol, cap, o->sweeps, o->boost, &st, &rel);
        if (st == ORS_NONFINITE || st == ORS_INDEFINITE) its = 0;
        apply(s, s->qf, s->qc, Pf, Pc);
        copyv(s, s->rf, s->rc, s->bf, s->bc);
        axpy(s, s->rf, s->rc, -1.0f, s->qf, s->qc);
        const float bnorm = sqrtf(inner(s, s->bf, s->bc, s->bf, s->bc));
        const float rnorm = sqrtf(inner(s, s->rf, s->rc, s->rf, s->rc));
        rel = bnorm > 0.0f ? rnorm / bnorm : 0.0f;
        if (!(rnorm <= o->tol * bnorm)) {
            if (!isfinite(rnorm) || rnorm > 2.0f * bnorm) {
                memset(Pf, 0, sizeof(float) * s->nsl * BCELLS);
                memset(Pc, 0, sizeof(float) * s->ncc);
            }
            info->fgmres_iterations = pressure_fgmres(s, Pf, Pc, o->tol, o->maxiter, o->sweeps, o->boost, &status, &rel);
            its += info->fgmres_iterations;
        }
    }
    info->iterations = its;
    info->status = status;
    info->rel_residual = rel;
    return its;
}

/* ---- the right-hand side, clearing, the volume, the gradient ---- */
/* finerhs_kernel! (:1409-1423) and coarserhs_kernel! (:1425-1435) */
static void rhs(S* s, float gamma) {
    const ors_basin* B = s->B;
    const float h = B->g.dx;
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        if (whereof(s, sl)[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int64_t n = (sl - 1) * BCELLS + c;
            const int i = c & 15, j = (c >> 4) & 15, k = c >> 8;
            if (B->tf[n] == LIQUID) {
                float div = B->uf[faceindex(sl, 1, i + 1, j, k) - 1] - B->uf[faceindex(sl, 1, i, j, k) - 1];
                div = div + B->vf[faceindex(sl, 2, i, j + 1, k) - 1];
                div = div - B->vf[faceindex(sl, 2, i, j, k) - 1];
                div = div + B->wf[faceindex(sl, 3, i, j, k + 1) - 1];
                div = div - B->wf[faceindex(sl, 3, i, j, k) - 1];
                s->bf[n] = (-h) * div + (gamma * h) * h;
            } else {
                s->bf[n] = 0.0f;
            }
        }
    }
    int fx[3], fy[3], fz[3];
    fdims(s->nc, 1, fx);
    fdims(s->nc, 2, fy);
    fdims(s->nc, 3, fz);
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                if (B->tc[c] == LIQUID && !covered(s, I, J, K)) {
                    float div = B->uc[LIN(fx, I + 1, J, K)] - B->uc[LIN(fx, I, J, K)];
                    div = div + B->vc[LIN(fy, I, J + 1, K)];
                    div = div - B->vc[LIN(fy, I, J, K)];
                    div = div + B->wc[LIN(fz, I, J, K + 1)];
                    div = div - B->wc[LIN(fz, I, J, K)];
                    s->bc[c] = ((-16.0f) * h) * div + (((64.0f * gamma) * h) * h);
                } else {
                    s->bc[c] = 0.0f;
                }
            }
}
/* clearfine_kernel! / clearcoarse_kernel! (:1964-1974) */
static void clear(S* s) {
    const ors_basin* B = s->B;
    #pragma omp parallel for schedule(static)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        if (whereof(s, sl)[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int64_t n = (sl - 1) * BCELLS + c;
            if (B->tf[n] != LIQUID) B->Pf[n] = 0.0f;
        }
    }
    #pragma omp parallel for schedule(static)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                const int64_t c = LIN(s->nc, I, J, K);
                if (B->tc[c] != LIQUID || covered(s, I, J, K)) B->Pc[c] = 0.0f;
            }
}
/* finevolume_kernel! / coarsevolume_kernel! / volume (:1976-1996): the sums in FP64 here. */
static float volume(const S* s) {
    const ors_basin* B = s->B;
    const float dx = B->g.dx, cdx = (float)RATIO * dx;
    double sf = 0.0, sc = 0.0;
    #pragma omp parallel for schedule(static) reduction(+ : sf)
    for (int64_t sl = 1; sl <= s->nsl; sl++) {
        const int32_t* w = whereof(s, sl);
        if (w[0] < 0) continue;
        for (int c = 0; c < BCELLS; c++) {
            const int I = w[0] * BLOCK + (c & 15), J = w[1] * BLOCK + ((c >> 4) & 15), K = w[2] * BLOCK + (c >> 8);
            if (!issolid_fine(&B->g, I, J, K)) sf += (double)clampf(0.5f - B->phif[(sl - 1) * BCELLS + c] / dx, 0.0f, 1.0f);
        }
    }
    #pragma omp parallel for schedule(static) reduction(+ : sc)
    for (int K = 0; K < s->nc[2]; K++)
        for (int J = 0; J < s->nc[1]; J++)
            for (int I = 0; I < s->nc[0]; I++) {
                if (covered(s, I, J, K) || issolid_coarse(&B->g, I, J, K)) continue;
                sc += (double)(64.0f * clampf(0.5f - B->phic[LIN(s->nc, I, J, K)] / cdx, 0.0f, 1.0f));
            }
    return ((float)sf + (float)sc) * (dx * dx * dx);
}
/* pressureat (:1909-1914) */
static inline float pressureat(const S* s, const float* Pf, const float* Pc, int I, int J, int K) {
    const int64_t idx = fineat(s, I, J, K);
    if (idx > 0) return Pf[idx - 1];
    int ci = I >> 2, cj = J >> 2, ck = K >> 2;
    ci = ci < 0 ? 0 : (ci > s->nc[0] - 1 ? s->nc[0] - 1 : ci);
    cj = cj < 0 ? 0 : (cj > s->nc[1] - 1 ? s->nc[1] - 1 : cj);
    ck = ck < 0 ? 0 : (ck > s->nc[2] - 1 ? s->nc[2] - 1 : ck);
    return Pc[LIN(s->nc, ci, cj, ck)];
}
/* projectfine_kernel! (:1917-1940), projectcoarse_kernel! (:1942-1962) and restrictfaces_kernel!
   (:597-611) for the velocity and its flags, axis by axis as project! runs them (:2010-2016). */
static void gradient(S* s) {
    const ors_basin* B = s->B;
    const float dx = B->g.dx, cdx = (float)RATIO * dx;
    for (int a = 1; a <= 3; a++) {
        float* uf = a == 1 ? B->uf : (a == 2 ? B->vf : B->wf);
        float* uc = a == 1 ? B->uc : (a == 2 ? B->vc : B->wc);
        uint8_t* ff = a == 1 ? B->fuf : (a == 2 ? B->fvf : B->fwf);
        uint8_t* fc = a == 1 ? B->fuc : (a == 2 ? B->fvc : B->fwc);
        int e[3], fm[3];
        unitv(a, e);
        fdims(s->nc, a, fm);
        #pragma omp parallel for schedule(static)
        for (int64_t sl = 1; sl <= s->nsl; sl++) {
            const int32_t* w = whereof(s, sl);
            if (w[0] < 0) continue;
            for (int f = 0; f < BFACES; f++) {
                int i, j, k;
                face_local(a, f, &i, &j, &k);
                const int64_t idx = faceindex(sl, a, i, j, k) - 1;
                const int I = w[0] * BLOCK + i, J = w[1] * BLOCK + j, K = w[2] * BLOCK + k;
                int fp, fmn;
                const uint8_t tp = celltype(s, I, J, K, &fp);
                const uint8_t tm = celltype(s, I - e[0], J - e[1], K - e[2], &fmn);
                const int ok = tp != SOLID && tm != SOLID && (tp == LIQUID || tm == LIQUID);
                if (ok) {
                    const float d = (fp && fmn ? 1.0f : 2.5f) * dx;
                    const float Pp = pressureat(s, B->Pf, B->Pc, I, J, K);
                    const float Pm = pressureat(s, B->Pf, B->Pc, I - e[0], J - e[1], K - e[2]);
                    float D;
                    if (tp == LIQUID && tm == LIQUID) D = Pp - Pm;
                    else if (tm == LIQUID) D = -Pm / theta(nphi(s, I - e[0], J - e[1], K - e[2]), nphi(s, I, J, K));
                    else D = Pp / theta(nphi(s, I, J, K), nphi(s, I - e[0], J - e[1], K - e[2]));
                    uf[idx] -= D / d;
                }
                ff[idx] = ok ? 1 : 0;
            }
        }
        const int n1 = s->nc[0], n2 = s->nc[1], n3 = s->nc[2];
        #pragma omp parallel for schedule(static)
        for (int K = 0; K < fm[2]; K++)
            for (int J = 0; J < fm[1]; J++)
                for (int I = 0; I < fm[0]; I++) {
                    const int Im = I - e[0], Jm = J - e[1], Km = K - e[2];
                    const int inside = 0 <= Im && 0 <= Jm && 0 <= Km && I < n1 && J < n2 && K < n3;
                    const int64_t o = LIN(fm, I, J, K);
                    if (inside && !covered(s, I, J, K) && !covered(s, Im, Jm, Km)) {
                        const uint8_t tp = B->tc[LIN(s->nc, I, J, K)], tm = B->tc[LIN(s->nc, Im, Jm, Km)];
                        const int ok = tp != SOLID && tm != SOLID && (tp == LIQUID || tm == LIQUID);
                        if (ok) {
                            const float Pp = B->Pc[LIN(s->nc, I, J, K)], Pm = B->Pc[LIN(s->nc, Im, Jm, Km)];
                            const float pp = B->phic[LIN(s->nc, I, J, K)], pm = B->phic[LIN(s->nc, Im, Jm, Km)];
                            const float D = (tp == LIQUID && tm == LIQUID) ? Pp - Pm
                                            : (tm == LIQUID ? -Pm / theta(pm, pp) : Pp / theta(pp, pm));
                            uc[o] -= D / cdx;
                        }
                        fc[o] = ok ? 1 : 0;
                    } else if (!inside) {
                        fc[o] = 0;
                    }
                }
        /* restrict!(s, f, a) then restrict!(s, fl, a): the coarse faces fine blocks hold */
        for (int pass = 0; pass < 2; pass++)
            #pragma omp parallel for schedule(static)
            for (int K = 0; K < fm[2]; K++)
                for (int J = 0; J < fm[1]; J++)
                    for (int I = 0; I < fm[0]; I++) {
                        float acc = 0.0f;
                        int found = 0;
                        for (int q = 0; q < 4; q++)
                            for (int p = 0; p < 4; p++) {
                                const int FI = RATIO * I + (a == 1 ? 0 : p);
                                const int FJ = RATIO * J + (a == 1 ? p : (a == 2 ? 0 : q));
                                const int FK = RATIO * K + (a == 3 ? 0 : q);
                                const int64_t idx = finefaceat(s, a, FI, FJ, FK);
                                if (idx > 0) {
                                    acc += pass == 0 ? uf[idx - 1] : (float)ff[idx - 1];
                                    found++;
                                }
                            }
                        if (found == 16) {
                            const int64_t o = LIN(fm, I, J, K);
                            if (pass == 0) uc[o] = acc / 16.0f;
                            else fc[o] = acc >= 16.0f - 0.5f ? 1 : 0;
                        }
                    }
    }
}

/* ---- entry points ---- */
static int S_open(S* s, const ors_basin* B) {
    if (S_init(s, B)) {
        S_free(s);
        return -1;
    }
    return 0;
}

double ors_volume(const ors_basin* B) {
    S s;
    if (S_open(&s, B)) return NAN;
    const float v = volume(&s);
    S_free(&s);
    return (double)v;
}

int ors_coefficients(const ors_basin* B, float* cuf, float* cvf, float* cwf, float* cuc, float* cvc, float* cwc,
                     float* dDf, float* dDc, uint8_t* actc) {
    S s;
    if (S_open(&s, B)) return -1;
    coefficients(&s);
    int fm[3];
    const int64_t nff = s.nsl * BFACES, nf = s.nsl * BCELLS;
    memcpy(cuf, s.cuf, 4 * nff);
    memcpy(cvf, s.cvf, 4 * nff);
    memcpy(cwf, s.cwf, 4 * nff);
    fdims(s.nc, 1, fm); memcpy(cuc, s.cuc, 4 * LIN(fm, 0, 0, fm[2]));
    fdims(s.nc, 2, fm); memcpy(cvc, s.cvc, 4 * LIN(fm, 0, 0, fm[2]));
    fdims(s.nc, 3, fm); memcpy(cwc, s.cwc, 4 * LIN(fm, 0, 0, fm[2]));
    memcpy(dDf, s.dDf, 4 * nf);
    memcpy(dDc, s.dDc, 4 * s.ncc);
    memcpy(actc, s.D[0].act, s.ncc);
    S_free(&s);
    return 0;
}

int ors_levels(const ors_basin* B) {
    S s;
    if (S_open(&s, B)) return -1;
    const int nd = s.nd;
    S_free(&s);
    return nd;
}

int ors_apply(const ors_basin* B, const float* xf, const float* xc, float* qf, float* qc) {
    S s;
    if (S_open(&s, B)) return -1;
    coefficients(&s);
    hierarchy(&s);
    apply(&s, qf, qc, xf, xc);
    S_free(&s);
    return 0;
}

int ors_vcycle(const ors_basin* B, const float* rf, const float* rc, float* zf, float* zc, int sweeps, int coarse,
               float boost) {
    S s;
    if (S_open(&s, B)) return -1;
    coefficients(&s);
    hierarchy(&s);
    vcycle(&s, zf, zc, rf, rc, sweeps, coarse, boost);
    S_free(&s);
    return 0;
}

int ors_jacobi(const ors_basin* B, const float* xf, const float* xc, const float* bf, const float* bc, float* of,
               float* oc) {
    S s;
    if (S_open(&s, B)) return -1;
    coefficients(&s);
    hierarchy(&s);
    const Comp L = level0(&s);
    jacobi_fine(&s, &L, of, xf, bf, xc);
    jacobi_coarse(&s, &L, oc, xc, bc, xf);
    S_free(&s);
    return 0;
}

int ors_rhs(const ors_basin* B, float gamma, float* bf, float* bc) {
    S s;
    if (S_open(&s, B)) return -1;
    rhs(&s, gamma);
    memcpy(bf, s.bf, 4 * s.nsl * BCELLS);
    memcpy(bc, s.bc, 4 * s.ncc);
    S_free(&s);
    return 0;
}

/* pressure! on b: the coefficients from the basin's classes and level set, then the solve
   from the warm start in B's P. */
int ors_pressure(const ors_basin* B, const float* bf, const float* bc, const ors_opts* o, ors_info* info) {
    S s;
    if (S_open(&s, B)) return -1;
    coefficients(&s);
    memcpy(s.bf, bf, 4 * s.nsl * BCELLS);
    memcpy(s.bc, bc, 4 * s.ncc);
    pressure_dispatch(&s, B->Pf, B->Pc, o, info);
    S_free(&s);
    return info->iterations;
}

int ors_gradient(const ors_basin* B) {
    S s;
    if (S_open(&s, B)) return -1;
    gradient(&s);
    S_free(&s);
    return 0;
}

/* project! (src/sflip.jl:1998-2018) */
int ors_project(const ors_basin* B, float volume0, double dt, double recover, const ors_opts* o, ors_info* info) {
    S s;
    if (S_open(&s, B)) return -1;
    const float vol = volume(&s);
    const float loss = (volume0 - vol) / volume0;
    const double x = (double)loss / recover, lo = -0.01 / dt, hi = 0.01 / dt;
    const float gamma = (float)(x > hi ? hi : (x < lo ? lo : x));
    info->volume = vol;
    info->gamma = gamma;
    coefficients(&s);
    rhs(&s, gamma);
    clear(&s);
    pressure_dispatch(&s, B->Pf, B->Pc, o, info);
    gradient(&s);
    S_free(&s);
    return info->iterations;
}
