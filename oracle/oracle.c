/*
 * CPU oracle for the dense-MAC pressure projection (TEST INFRASTRUCTURE ONLY; see
 * oracle.h for what it restates and why its parity is unpinned).
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off). Contraction is off so
 * that every a*b+c rounds twice, as the reference's Julia arithmetic does.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SOLID 0
#define LIQUID 1
#define AIR 2
#define MAXLEV 16

#define ID(n1, n2, i, j, k) ((size_t)(i) + (size_t)(n1) * ((size_t)(j) + (size_t)(n2) * (size_t)(k)))

/* neighbour (src/flip.jl:84-92): +x, -x, +y, -y, +z, -z */
static const int NB[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

/* typeat (src/flip.jl:94): out of range counts as SOLID, so the box edge is a wall. */
static inline uint8_t typeat(const uint8_t* t, int n1, int n2, int n3, int i, int j, int k) {
    return (i >= 0 && i < n1 && j >= 0 && j < n2 && k >= 0 && k < n3) ? t[ID(n1, n2, i, j, k)]
                                                                       : (uint8_t)SOLID;
}

/* cellcentre / issolid / issolidcell (src/flip.jl:64-66), in Float32 as the reference. */
static inline int issolidcell(const orc_grid* g, int i, int j, int k) {
    float px = g->lo[0] + ((float)i + 0.5f) * g->dx;
    float py = g->lo[1] + ((float)j + 0.5f) * g->dx;
    float pz = g->lo[2] + ((float)k + 0.5f) * g->dx;
    return px * px + py * py > g->radius * g->radius || pz < g->floor_z;
}

/* coarsen_kernel! (src/flip.jl:880-889): a coarse cell is AIR if any of its 8 children is,
 * else LIQUID if any is, else SOLID. */
void orc_coarsen(const int32_t nf[3], uint8_t* tc, const uint8_t* tf) {
    const int f1 = nf[0], f2 = nf[1], f3 = nf[2];
    const int n1 = f1 / 2, n2 = f2 / 2, n3 = f3 / 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int K = 0; K < n3; K++)
        for (int J = 0; J < n2; J++)
            for (int I = 0; I < n1; I++) {
                int air = 0, liquid = 0;
                for (int c = 0; c < 2; c++)
                    for (int b = 0; b < 2; b++)
                        for (int a = 0; a < 2; a++) {
                            uint8_t t = typeat(tf, f1, f2, f3, 2 * I + a, 2 * J + b, 2 * K + c);
                            if (t == AIR) air = 1;
                            if (t == LIQUID) liquid = 1;
                        }
                tc[ID(n1, n2, I, J, K)] = air ? AIR : (liquid ? LIQUID : SOLID);
            }
}

/* Length of s.partials: cld(largest face array, 256) (src/flip.jl:219). */
static size_t plen_(const orc_grid* g) {
    size_t n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    size_t a = (n1 + 1) * n2 * n3, b = n1 * (n2 + 1) * n3, c = n1 * n2 * (n3 + 1);
    size_t m = a > b ? a : b;
    m = m > c ? m : c;
    return (m + 255) / 256;
}

#define R float
#define SFX f32
#define SQRT sqrtf
#include "oracle_impl.h"
#undef R
#undef SFX
#undef SQRT

#define R double
#define SFX f64
#define SQRT sqrt
#include "oracle_impl.h"
#undef R
#undef SFX
#undef SQRT

/* walled (src/flip.jl:784-789): face (i, j, k) along axis (0-based face indices) is the
 * grid's own edge, or has a SOLID cell on either side. */
static int walled(const orc_grid* g, int i, int j, int k, int axis) {
    const int f[3] = {i, j, k};
    if (f[axis] == 0 || f[axis] == g->n[axis]) return 1;
    int bi = i, bj = j, bk = k;
    if (axis == 0) bi--;
    else if (axis == 1) bj--;
    else bk--;
    return issolidcell(g, bi, bj, bk) || issolidcell(g, i, j, k);
}

/* extrapolate_kernel! (src/flip.jl:1161-1177), one layer of one face array (dims a): a
 * flagged face keeps its value; an unflagged one that is not walled takes the Float32 mean
 * of its flagged neighbours in the same array, summed in neighbour order, and is flagged
 * if it had any. */
static void extrapolate_layer(const orc_grid* g, float* out, uint8_t* fout, const float* src, const uint8_t* fin,
                              const int32_t a[3], int axis) {
    const int a1 = a[0], a2 = a[1], a3 = a[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < a3; k++)
        for (int j = 0; j < a2; j++)
            for (int i = 0; i < a1; i++) {
                const size_t id = ID(a1, a2, i, j, k);
                if (fin[id]) {
                    out[id] = src[id];
                    fout[id] = 1;
                    continue;
                }
                float s = 0.f;
                int m = 0;
                if (!walled(g, i, j, k, axis))
                    for (int q = 0; q < 6; q++) {
                        const int x = i + NB[q][0], y = j + NB[q][1], z = k + NB[q][2];
                        if (x >= 0 && x < a1 && y >= 0 && y < a2 && z >= 0 && z < a3 && fin[ID(a1, a2, x, y, z)]) {
                            s += src[ID(a1, a2, x, y, z)];
                            m++;
                        }
                    }
                out[id] = m > 0 ? s / (float)m : src[id];
                fout[id] = m > 0 ? 1 : 0;
            }
}

/* extrapolate! (src/flip.jl:1192-1206): per face array, `layers` layers ping-ponged through
 * a scratch copy; the result and its flags back in the caller's arrays; unreached_kernel!
 * (:1181-1184) zeroes what no layer reached; then solidify! (:801-806) zeroes every walled
 * face of the three arrays. fu, fv, fw end as the reached flags. */
void orc_extrapolate(const orc_grid* g, float* u, float* v, float* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                     int layers) {
    float* arrs[3] = {u, v, w};
    uint8_t* flags[3] = {fu, fv, fw};
    for (int axis = 0; axis < 3; axis++) {
        int32_t a[3] = {g->n[0], g->n[1], g->n[2]};
        a[axis]++;
        const size_t n = (size_t)a[0] * a[1] * a[2];
        float* tmp = (float*)malloc(n * sizeof(float));
        uint8_t* ftmp = (uint8_t*)malloc(n);
        float *src = arrs[axis], *dst = tmp;
        uint8_t *fin = flags[axis], *fout = ftmp;
        for (int l = 0; l < layers; l++) {
            extrapolate_layer(g, dst, fout, src, fin, a, axis);
            float* t = src;
            src = dst;
            dst = t;
            uint8_t* ft = fin;
            fin = fout;
            fout = ft;
        }
        if (src != arrs[axis]) memcpy(arrs[axis], src, n * sizeof(float));
        if (fin != flags[axis]) memcpy(flags[axis], fin, n);
        for (size_t q = 0; q < n; q++)
            if (flags[axis][q] == 0) arrs[axis][q] = 0.f;
        free(tmp);
        free(ftmp);
    }
    for (int axis = 0; axis < 3; axis++) {  /* solidify! */
        int32_t a[3] = {g->n[0], g->n[1], g->n[2]};
        a[axis]++;
        float* arr = arrs[axis];
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < a[2]; k++)
            for (int j = 0; j < a[1]; j++)
                for (int i = 0; i < a[0]; i++)
                    if (walled(g, i, j, k, axis)) arr[ID(a[0], a[1], i, j, k)] = 0.f;
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
