/*
 * CPU oracle for the level-set passes step! runs before the projection (TEST
 * INFRASTRUCTURE ONLY, like the rest of this directory): redistance!, classify! and
 * filltrapped! of src/flip.jl:608-760, in Float32, step by step as the reference's
 * kernels do them. Julia's min/max/clamp/abs semantics for Float32 are restated exactly
 * (jmin/jmax below), and the file is built with -ffp-contract=off like oracle.c.
 *
 * The trapped-air sweeps are restated literally (one thread's walk of a line there and
 * back, a carry through runs of air), independently of the library's bit-parallel form.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SOLID 0
#define LIQUID 1
#define AIR 2
#define ID(n1, n2, i, j, k) ((size_t)(i) + (size_t)(n1) * ((size_t)(j) + (size_t)(n2) * (size_t)(k)))

static const int NB[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

/* cellcentre / issolid / issolidcell (src/flip.jl:64-66), Float32. */
static int solidcell(const orc_grid* g, int i, int j, int k) {
    float px = g->lo[0] + ((float)i + 0.5f) * g->dx;
    float py = g->lo[1] + ((float)j + 0.5f) * g->dx;
    float pz = g->lo[2] + ((float)k + 0.5f) * g->dx;
    return px * px + py * py > g->radius * g->radius || pz < g->floor_z;
}

/* Julia's min and max for Float32 (Base: diff = x - y, the argument signbit(diff) picks,
 * NaN when either is NaN), so -0 < +0 as in the reference. */
static float jmin(float x, float y) {
    float diff = x - y;
    if (isnan(x) || isnan(y)) return diff;
    return signbit(diff) ? x : y;
}
static float jmax(float x, float y) {
    float diff = x - y;
    if (isnan(x) || isnan(y)) return diff;
    return signbit(diff) ? y : x;
}
/* clamp(x, lo, hi) = ifelse(x > hi, hi, ifelse(x < lo, lo, x)). */
static float jclamp(float x, float lo, float hi) { return x > hi ? hi : (x < lo ? lo : x); }

/* eikonal (src/flip.jl:611-623): the upwind distance from the three smallest neighbour
 * distances along the axes, Godunov's update, in the reference's operation order. */
static float eikonal(float a, float b, float c, float h) {
    float t0 = jmin(a, b), t1 = jmax(a, b);
    a = t0; b = t1;
    t0 = jmin(b, c); t1 = jmax(b, c);
    b = t0; c = t1;
    t0 = jmin(a, b); t1 = jmax(a, b);
    a = t0; b = t1;
    float d = a + h;
    if (d > b) {
        float ab = a - b;
        d = 0.5f * (a + b + sqrtf(jmax(2.0f * h * h - ab * ab, 0.0f)));
        if (d > c) {
            float t = a + b + c;
            d = (t + sqrtf(jmax(t * t - 3.0f * (a * a + b * b + c * c - h * h), 0.0f))) / 3.0f;
        }
    }
    return d;
}

/* reinit_kernel! (src/flip.jl:631-666): one Jacobi sweep, out from phi. */
static void reinit(const orc_grid* g, float* out, const float* phi, float phimax) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const float h = g->dx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                const size_t id = ID(n1, n2, i, j, k);
                const float c = phi[id];
                if (solidcell(g, i, j, k)) {
                    float lowest = c;
                    int found = 0;
                    for (int m = 0; m < 6; m++) {
                        int a = i + NB[m][0], b = j + NB[m][1], cc = k + NB[m][2];
                        if (a >= 0 && a < n1 && b >= 0 && b < n2 && cc >= 0 && cc < n3 && !solidcell(g, a, b, cc)) {
                            float f = phi[ID(n1, n2, a, b, cc)];
                            lowest = found ? jmin(lowest, f) : f;
                            found = 1;
                        }
                    }
                    out[id] = found ? lowest : jclamp(c, -phimax, phimax);
                } else {
                    const int inside = c < 0.0f;
                    int frozen = 0;
                    float ax = phimax, ay = phimax, az = phimax;
                    for (int m = 0; m < 6; m++) {
                        int a = i + NB[m][0], b = j + NB[m][1], cc = k + NB[m][2];
                        if (a >= 0 && a < n1 && b >= 0 && b < n2 && cc >= 0 && cc < n3 && !solidcell(g, a, b, cc)) {
                            float f = phi[ID(n1, n2, a, b, cc)];
                            if ((f < 0.0f) != inside) frozen = 1;
                            float d = fabsf(f);
                            if (m < 2) ax = jmin(ax, d);
                            else if (m < 4) ay = jmin(ay, d);
                            else az = jmin(az, d);
                        }
                    }
                    if (frozen) {
                        out[id] = c;
                    } else {
                        float d = jmin(eikonal(ax, ay, az, h), phimax);
                        out[id] = inside ? -d : d;
                    }
                }
            }
}

/* redistance!(s; iterations) (src/flip.jl:673-680): phimax = (iterations + 1) dx, then
 * `iterations` Jacobi sweeps; the result is left in phi. */
void orc_redistance(const orc_grid* g, float* phi, int iterations) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2];
    const float phimax = (float)(iterations + 1) * g->dx;
    float* tmp = (float*)malloc(N * sizeof(float));
    float *src = phi, *dst = tmp;
    for (int it = 0; it < iterations; it++) {
        reinit(g, dst, src, phimax);
        float* t = src;
        src = dst;
        dst = t;
    }
    if (src != phi) memcpy(phi, src, N * sizeof(float));
    free(tmp);
}

/* classify_kernel! (src/flip.jl:682-686). */
void orc_classify(const orc_grid* g, uint8_t* types, const float* phi) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                const size_t id = ID(n1, n2, i, j, k);
                types[id] = solidcell(g, i, j, k) ? SOLID : (phi[id] < 0.0f ? LIQUID : AIR);
            }
}

/* sweepair_kernel! (src/flip.jl:710-731) for every line along `axis` (0, 1, 2): a walk
 * there and back, reach carried through runs of air; returns the cells it reached. */
static long sweepair(const int n[3], uint8_t* reach, const uint8_t* types, int axis) {
    const int n1 = n[0], n2 = n[1];
    const int ua = axis == 0 ? 1 : 0, ub = axis == 2 ? 1 : 2;  /* the two other axes */
    long changed = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : changed)
    for (int b = 0; b < n[ub]; b++)
        for (int a = 0; a < n[ua]; a++) {
            const int len = n[axis];
            for (int pass = 0; pass < 2; pass++) {
                int carry = 0;
                for (int m = 0; m < len; m++) {
                    int l = pass == 0 ? m : len - 1 - m;
                    int c[3];
                    c[axis] = l;
                    c[ua] = a;
                    c[ub] = b;
                    size_t id = ID(n1, n2, c[0], c[1], c[2]);
                    if (types[id] == AIR) {
                        if (reach[id] != 0) carry = 1;
                        else if (carry) {
                            reach[id] = 1;
                            changed++;
                        }
                    } else {
                        carry = 0;
                    }
                }
            }
        }
    return changed;
}

/* filltrapped!(s; maxrounds) (src/flip.jl:747-760): air reached from the grid's top layer
 * by rounds of sweeps along z, x, y (until a round reaches nothing, at most maxrounds);
 * the air left becomes LIQUID with phi at most -2 dx. Returns the rounds run. */
int orc_filltrapped(const orc_grid* g, uint8_t* types, float* phi, int maxrounds) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const size_t N = (size_t)n1 * n2 * n3;
    uint8_t* reach = (uint8_t*)calloc(N, 1);
    for (int k = 0; k < n3; k++) /* seedair_kernel! (:706-708) */
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t id = ID(n1, n2, i, j, k);
                reach[id] = (k == n3 - 1 && types[id] == AIR) ? 1 : 0;
            }
    int rounds = 0;
    for (int r = 0; r < maxrounds; r++) {
        long changed = 0;
        changed += sweepair(g->n, reach, types, 2);
        changed += sweepair(g->n, reach, types, 0);
        changed += sweepair(g->n, reach, types, 1);
        rounds++;
        if (changed == 0) break;
    }
    const float depth = 2.0f * g->dx;
    for (size_t i = 0; i < N; i++) /* fillair_kernel! (:734-740) */
        if (types[i] == AIR && reach[i] == 0) {
            types[i] = LIQUID;
            phi[i] = jmin(phi[i], -depth);
        }
    free(reach);
    return rounds;
}
