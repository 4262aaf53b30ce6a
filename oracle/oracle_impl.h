/*
 * Body of the CPU oracle, included twice by oracle.c: once with R=float (the
 * reference arithmetic) and once with R=double (the FP64 accuracy oracle).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Index convention: 0-based (i,j,k); the reference is 1-based, so its colour test
 * (i+j+k) % 2 == colour becomes (i+j+k+1) & 1 == colour here.
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

/* theta (src/flip.jl:113): clamp(phi_i / (phi_i - phi_j), 0.01, 1), Julia's clamp order. */
static inline R FN(theta_)(R pi, R pj) {
    R t = pi / (pi - pj);
    return t > (R)1 ? (R)1 : (t < (R)0.01f ? (R)0.01f : t);
}

/* rhs_kernel! (src/flip.jl:817-822). */
void FN(orc_rhs_)(const orc_grid* g, R* b, const R* u, const R* v, const R* w,
                  const uint8_t* types, R gamma) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const R dx = (R)g->dx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R val = 0;
                if (types[c] == LIQUID) {
                    R div = u[ID(n1 + 1, n2, i + 1, j, k)] - u[ID(n1 + 1, n2, i, j, k)];
                    div = div + v[ID(n1, n2 + 1, i, j + 1, k)];
                    div = div - v[ID(n1, n2 + 1, i, j, k)];
                    div = div + w[ID(n1, n2, i, j, k + 1)];
                    div = div - w[ID(n1, n2, i, j, k)];
                    val = (-dx) * div + (dx * dx) * gamma;
                }
                b[c] = val;
            }
}

/* diag_kernel! (src/flip.jl:824-836): liquid neighbours count 1, air ones 1/theta. */
void FN(orc_diag_)(const orc_grid* g, R* diag, const uint8_t* types, const R* phi) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R d = 0;
                if (types[c] == LIQUID) {
                    for (int m = 0; m < 6; m++) {
                        int a = i + NB[m][0], bb = j + NB[m][1], cc = k + NB[m][2];
                        uint8_t t = typeat(types, n1, n2, n3, a, bb, cc);
                        if (t == LIQUID) d += (R)1;
                        if (t == AIR) d += (R)1 / FN(theta_)(phi[c], phi[ID(n1, n2, a, bb, cc)]);
                    }
                }
                diag[c] = d;
            }
}

/* celldiag (src/flip.jl:840-850): the stored fine diagonal, or a coarse level's
 * count of non-SOLID neighbours. */
static inline R FN(celldiag_)(const R* diag, const uint8_t* t, int n1, int n2, int n3, int i, int j,
                              int k) {
    if (diag) return diag[ID(n1, n2, i, j, k)];
    R d = 0;
    for (int m = 0; m < 6; m++)
        if (typeat(t, n1, n2, n3, i + NB[m][0], j + NB[m][1], k + NB[m][2]) != SOLID) d += (R)1;
    return d;
}

/* liquidsum (src/flip.jl:852-857): s = 0; s += x_n over LIQUID neighbours in order +x,-x,+y,-y,+z,-z. */
static inline R FN(liquidsum_)(const R* x, const uint8_t* t, int n1, int n2, int n3, int i, int j,
                               int k) {
    R s = 0;
    for (int m = 0; m < 6; m++) {
        int a = i + NB[m][0], bb = j + NB[m][1], cc = k + NB[m][2];
        if (typeat(t, n1, n2, n3, a, bb, cc) == LIQUID) s += x[ID(n1, n2, a, bb, cc)];
    }
    return s;
}

/* residual_kernel! (src/flip.jl:859-863). */
static void FN(residual_)(const int n[3], R* r, const R* x, const R* b, const uint8_t* t,
                          const R* diag) {
    const int n1 = n[0], n2 = n[1], n3 = n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R val = 0;
                if (t[c] == LIQUID) {
                    R d = FN(celldiag_)(diag, t, n1, n2, n3, i, j, k);
                    val = b[c] - (d * x[c] - FN(liquidsum_)(x, t, n1, n2, n3, i, j, k));
                }
                r[c] = val;
            }
}

/* The operator alone: y = diag x - sum_LIQ x_n on LIQUID cells (residual_kernel!'s A). */
void FN(orc_apply_)(const orc_grid* g, R* y, const R* x, const uint8_t* types, const R* diag) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R val = 0;
                if (types[c] == LIQUID)
                    val = diag[c] * x[c] - FN(liquidsum_)(x, types, n1, n2, n3, i, j, k);
                y[c] = val;
            }
}

/* rbgs_kernel! (src/flip.jl:870-877): one colour of red-black Gauss-Seidel. Cells of one
 * colour read only the other colour, so the loop order does not matter. */
static void FN(rbgs_)(const int n[3], R* x, const R* b, const uint8_t* t, const R* diag, int colour) {
    const int n1 = n[0], n2 = n[1], n3 = n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = ((colour + j + k + 1) & 1); i < n1; i += 2) {
                size_t c = ID(n1, n2, i, j, k);
                if (t[c] == LIQUID) {
                    R d = FN(celldiag_)(diag, t, n1, n2, n3, i, j, k);
                    x[c] = d > (R)0 ? (b[c] + FN(liquidsum_)(x, t, n1, n2, n3, i, j, k)) / d : (R)0;
                }
            }
}

/* start_kernel! (src/flip.jl:965-973): the first colour from zero, every other cell zero. */
static void FN(start_)(const int n[3], R* x, const R* b, const uint8_t* t, const R* diag) {
    const int n1 = n[0], n2 = n[1], n3 = n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R val = 0;
                if (((i + j + k + 1) & 1) == 0 && t[c] == LIQUID) {
                    R d = FN(celldiag_)(diag, t, n1, n2, n3, i, j, k);
                    if (d > (R)0) val = b[c] / d;
                }
                x[c] = val;
            }
}

/* weightB (src/flip.jl:891): (1,3,3,1)/8. */
static inline R FN(weightB_)(int a) { return (a == 1 || a == 2) ? (R)0.375f : (R)0.125f; }

/* restrict_kernel! (src/flip.jl:894-906): bc = 4 sum w_a w_b w_c rf over LIQUID fine cells. */
static void FN(restrict_)(const int nc[3], R* bc, const R* rf, const uint8_t* tf, const uint8_t* tc) {
    const int n1 = nc[0], n2 = nc[1], n3 = nc[2];
    const int f1 = 2 * n1, f2 = 2 * n2, f3 = 2 * n3;
#pragma omp parallel for collapse(2) schedule(static)
    for (int K = 0; K < n3; K++)
        for (int J = 0; J < n2; J++)
            for (int I = 0; I < n1; I++) {
                R s = 0;
                if (tc[ID(n1, n2, I, J, K)] == LIQUID) {
                    for (int c = 0; c < 4; c++)
                        for (int bb = 0; bb < 4; bb++)
                            for (int a = 0; a < 4; a++) {
                                int i = 2 * I + a - 1, j = 2 * J + bb - 1, k = 2 * K + c - 1;
                                if (typeat(tf, f1, f2, f3, i, j, k) == LIQUID)
                                    s += FN(weightB_)(a) * FN(weightB_)(bb) * FN(weightB_)(c) *
                                         rf[ID(f1, f2, i, j, k)];
                            }
                }
                bc[ID(n1, n2, I, J, K)] = (R)4 * s;
            }
}

/* prolongweights (src/flip.jl:908-911), 0-based: the two coarse cells and their weights. */
static inline void FN(pw_)(int i, int* c0, R* w0, int* c1, R* w1) {
    int I = i >> 1;
    if ((i & 1) == 0) { *c0 = I - 1; *w0 = (R)0.25f; *c1 = I; *w1 = (R)0.75f; }
    else { *c0 = I; *w0 = (R)0.75f; *c1 = I + 1; *w1 = (R)0.25f; }
}

/* prolong_kernel! (src/flip.jl:914-929): xf += trilinear coarse correction over LIQUID coarse cells. */
static void FN(prolong_)(const int nf[3], R* xf, const R* xc, const uint8_t* tf, const uint8_t* tc) {
    const int n1 = nf[0], n2 = nf[1], n3 = nf[2];
    const int c1 = n1 / 2, c2 = n2 / 2, c3 = n3 / 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                if (tf[c] != LIQUID) continue;
                int a0, a1, b0, b1, k0, k1;
                R wa0, wa1, wb0, wb1, wc0, wc1;
                FN(pw_)(i, &a0, &wa0, &a1, &wa1);
                FN(pw_)(j, &b0, &wb0, &b1, &wb1);
                FN(pw_)(k, &k0, &wc0, &k1, &wc1);
                R s = 0;
                for (int m = 0; m < 8; m++) {
                    int a = (m & 1) ? a1 : a0;
                    R wa = (m & 1) ? wa1 : wa0;
                    int bb = (m & 2) ? b1 : b0;
                    R wb = (m & 2) ? wb1 : wb0;
                    int cc = (m & 4) ? k1 : k0;
                    R wc = (m & 4) ? wc1 : wc0;
                    if (typeat(tc, c1, c2, c3, a, bb, cc) == LIQUID) s += wa * wb * wc * xc[ID(c1, c2, a, bb, cc)];
                }
                xf[c] = xf[c] + s;
            }
}

/* coarse_kernel! (src/flip.jl:935-962): `sweeps` red-black sweeps from zero, then as many in
 * reverse colour order; the accumulator starts at b here (acc = b; acc += x_n). */
static void FN(coarsest_)(const int n[3], R* x, const R* b, const uint8_t* t, int sweeps) {
    const int n1 = n[0], n2 = n[1], n3 = n[2];
    const int N = n1 * n2 * n3;
    for (int c = 0; c < N; c++) x[c] = 0;
    for (int s = 1; s <= 2 * sweeps; s++)
        for (int half = 0; half <= 1; half++) {
            int colour = s <= sweeps ? half : 1 - half;
            for (int k = 0; k < n3; k++)
                for (int j = 0; j < n2; j++)
                    for (int i = 0; i < n1; i++) {
                        size_t c = ID(n1, n2, i, j, k);
                        if (t[c] != LIQUID || ((i + j + k + 1) & 1) != colour) continue;
                        R d = 0, acc = b[c];
                        for (int m = 0; m < 6; m++) {
                            int a = i + NB[m][0], bb = j + NB[m][1], cc = k + NB[m][2];
                            uint8_t tn = typeat(t, n1, n2, n3, a, bb, cc);
                            if (tn != SOLID) d += (R)1;
                            if (tn == LIQUID) acc += x[ID(n1, n2, a, bb, cc)];
                        }
                        x[c] = d > (R)0 ? acc / d : (R)0;
                    }
        }
}

typedef struct {
    int L;
    int n[MAXLEV][3];
    uint8_t* t[MAXLEV];
    R *x[MAXLEV], *b[MAXLEV], *r[MAXLEV];
} FN(hier_);

static void FN(hier_init_)(FN(hier_) * h, const orc_grid* g, const uint8_t* types) {
    h->L = g->levels;
    for (int l = 0; l < h->L; l++) {
        for (int a = 0; a < 3; a++) h->n[l][a] = g->n[a] >> l;
        size_t N = (size_t)h->n[l][0] * h->n[l][1] * h->n[l][2];
        h->t[l] = l == 0 ? (uint8_t*)types : (uint8_t*)calloc(N, 1);
        h->x[l] = l == 0 ? NULL : (R*)calloc(N, sizeof(R));
        h->b[l] = l == 0 ? NULL : (R*)calloc(N, sizeof(R));
        h->r[l] = (R*)calloc(N, sizeof(R));
    }
    /* coarsen_kernel! for every level (src/flip.jl:1084-1086) */
    for (int l = 1; l < h->L; l++) orc_coarsen(h->n[l - 1], h->t[l], h->t[l - 1]);
}

static void FN(hier_free_)(FN(hier_) * h) {
    for (int l = 0; l < h->L; l++) {
        if (l > 0) { free(h->t[l]); free(h->x[l]); free(h->b[l]); }
        free(h->r[l]);
    }
}

/* vcycle! (src/flip.jl:992-1014): down [start, 1, 0, 1], residual, restrict; the coarsest
 * solve; up: prolong, [1, 0, 1, 0] (for sweeps = 2). `sweeps` packs two counts: its low byte
 * is the fine level's (the reference's one `sweeps`), and bits 8-15, when not zero, the
 * coarser levels' (ORC_SWEEPS); the same colour schedule runs at each level's count. */
static void FN(vcycle_h_)(FN(hier_) * h, R* z, const R* r, const R* diag, int sweeps, int coarse) {
    const int L = h->L;
    h->x[0] = z;
    h->b[0] = (R*)r;
    const int swf = sweeps & 0xff, swc = (sweeps >> 8) & 0xff ? (sweeps >> 8) & 0xff : swf;
    for (int l = 0; l < L - 1; l++) {
        const R* dg = l == 0 ? diag : NULL;
        const int sw = l == 0 ? swf : swc;
        FN(start_)(h->n[l], h->x[l], h->b[l], h->t[l], dg);
        for (int s = 1; s < 2 * sw; s++) FN(rbgs_)(h->n[l], h->x[l], h->b[l], h->t[l], dg, s & 1);
        FN(residual_)(h->n[l], h->r[l], h->x[l], h->b[l], h->t[l], dg);
        FN(restrict_)(h->n[l + 1], h->b[l + 1], h->r[l], h->t[l], h->t[l + 1]);
    }
    FN(coarsest_)(h->n[L - 1], h->x[L - 1], h->b[L - 1], h->t[L - 1], coarse);
    for (int l = L - 2; l >= 0; l--) {
        const R* dg = l == 0 ? diag : NULL;
        const int sw = l == 0 ? swf : swc;
        FN(prolong_)(h->n[l], h->x[l], h->x[l + 1], h->t[l], h->t[l + 1]);
        for (int s = 0; s < 2 * sw; s++) FN(rbgs_)(h->n[l], h->x[l], h->b[l], h->t[l], dg, 1 - (s & 1));
    }
}

void FN(orc_vcycle_)(const orc_grid* g, R* z, const R* r, const uint8_t* types, const R* diag,
                     int sweeps, int coarse) {
    FN(hier_) h;
    FN(hier_init_)(&h, g, types);
    FN(vcycle_h_)(&h, z, r, diag, sweeps, coarse);
    FN(hier_free_)(&h);
}

/* ---- reductions (src/flip.jl:232-244, 283-287, 1020-1031) ----
 * A workgroup of 256 sums its values by the shared-memory tree (step 128, 64, ..., 1);
 * the partials are then summed. The reference sums the partials with Mantle's `sum`
 * on a device array, whose order is not pinned (Mantle is un-vendored); they are
 * summed in index order here. */
static inline R FN(tree256_)(R* s) {
    for (int step = 128; step >= 1; step >>= 1)
        for (int t = 0; t < step; t++) s[t] += s[t + step];
    return s[0];
}

static R FN(sumseq_)(const R* p, size_t n) {
    R s = 0;
    for (size_t i = 0; i < n; i++) s += p[i];
    return s;
}

/* inner (src/flip.jl:287): dot_kernel! partials over 256-wide linear groups, then the sum. */
static R FN(inner_)(const orc_grid* g, const R* a, const R* b, R* partials) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2], P = plen_(g);
#pragma omp parallel for schedule(static)
    for (size_t gi = 0; gi < P; gi++) {
        R s[256];
        for (int t = 0; t < 256; t++) {
            size_t i = gi * 256 + t;
            s[t] = i < N ? a[i] * b[i] : (R)0;
        }
        partials[gi] = FN(tree256_)(s);
    }
    return FN(sumseq_)(partials, P);
}

/* search_kernel! (src/flip.jl:1033-1054): q = A p for p = z + beta d, partials of p.q per
 * WG3 = (8,8,4) workgroup (cellgroups, src/flip.jl:1057). */
static R FN(search_)(const orc_grid* g, R* q, const R* z, const R* d, const uint8_t* t, const R* diag,
                     R beta, R* cellpartials) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const int G1 = (n1 + 7) / 8, G2 = (n2 + 7) / 8, G3 = (n3 + 3) / 4;
    const size_t NG = (size_t)G1 * G2 * G3;
#pragma omp parallel for schedule(static)
    for (size_t gi = 0; gi < NG; gi++) {
        int gx = (int)(gi % G1), gy = (int)((gi / G1) % G2), gz = (int)(gi / ((size_t)G1 * G2));
        R s[256];
        for (int lz = 0; lz < 4; lz++)
            for (int ly = 0; ly < 8; ly++)
                for (int lx = 0; lx < 8; lx++) {
                    int li = lx + 8 * (ly + 8 * lz);
                    int i = gx * 8 + lx, j = gy * 8 + ly, k = gz * 4 + lz;
                    R val = 0;
                    if (i < n1 && j < n2 && k < n3) {
                        size_t c = ID(n1, n2, i, j, k);
                        R qv = 0;
                        if (t[c] == LIQUID) {
                            R p = z[c] + beta * d[c];
                            R acc = 0;
                            for (int m = 0; m < 6; m++) {
                                int a = i + NB[m][0], bb = j + NB[m][1], cc = k + NB[m][2];
                                if (typeat(t, n1, n2, n3, a, bb, cc) == LIQUID) {
                                    size_t cn = ID(n1, n2, a, bb, cc);
                                    acc += z[cn] + beta * d[cn];
                                }
                            }
                            qv = diag[c] * p - acc;
                            val = p * qv;
                        }
                        q[c] = qv;
                    }
                    s[li] = val;
                }
        cellpartials[gi] = FN(tree256_)(s);
    }
    return FN(sumseq_)(cellpartials, NG);
}

/* advance_kernel! (src/flip.jl:1059-1073): d = z + beta d; x += alpha d; r -= alpha q; partials of r.r. */
static R FN(advance_)(const orc_grid* g, R* x, R* r, R* d, const R* z, const R* q, R alpha, R beta,
                      R* partials) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2], P = plen_(g);
#pragma omp parallel for schedule(static)
    for (size_t gi = 0; gi < P; gi++) {
        R s[256];
        for (int t = 0; t < 256; t++) {
            size_t l = gi * 256 + t;
            R v = 0;
            if (l < N) {
                R p = z[l] + beta * d[l];
                d[l] = p;
                x[l] = x[l] + alpha * p;
                R rl = r[l] - alpha * q[l];
                r[l] = rl;
                v = rl * rl;
            }
            s[t] = v;
        }
        partials[gi] = FN(tree256_)(s);
    }
    return FN(sumseq_)(partials, P);
}

/* pressure! (src/flip.jl:1082-1111): PCG with the V-cycle, from the warm start P. */
int FN(orc_pressure_)(const orc_grid* g, R* P, const R* b, const uint8_t* types, const R* phi, R tol,
                      int maxiter, int sweeps, int coarse, orc_info* info) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2];
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const size_t NGc = (size_t)((n1 + 7) / 8) * ((n2 + 7) / 8) * ((n3 + 3) / 4);
    R* diag = (R*)calloc(N, sizeof(R));
    R* r = (R*)calloc(N, sizeof(R));
    R* z = (R*)calloc(N, sizeof(R));
    R* d = (R*)calloc(N, sizeof(R));
    R* q = (R*)calloc(N, sizeof(R));
    R* partials = (R*)calloc(plen_(g), sizeof(R));
    R* cellpartials = (R*)calloc(NGc, sizeof(R));
    FN(hier_) h;
    FN(hier_init_)(&h, g, types);
    FN(orc_diag_)(g, diag, types, phi);
    FN(residual_)(g->n, r, P, b, types, diag);
    int its = 0, converged = 1;
    R bnorm = SQRT(FN(inner_)(g, b, b, partials));
    R rnorm = 0;
    if (bnorm == (R)0) goto done;
    R target = tol * bnorm;
    rnorm = SQRT(FN(inner_)(g, r, r, partials));
    if (rnorm <= target) goto done;
    FN(vcycle_h_)(&h, z, r, diag, sweeps, coarse);
    R rho = FN(inner_)(g, z, r, partials);
    R beta = 0;
    converged = 0;
    for (int it = 1; it <= maxiter; it++) {
        R pq = FN(search_)(g, q, z, d, types, diag, beta, cellpartials);
        R alpha = rho / pq;
        rnorm = SQRT(FN(advance_)(g, P, r, d, z, q, alpha, beta, partials));
        if (rnorm <= target) { its = it; converged = 1; goto done; }
        FN(vcycle_h_)(&h, z, r, diag, sweeps, coarse);
        R rhonew = FN(inner_)(g, z, r, partials);
        beta = rhonew / rho;
        rho = rhonew;
    }
    its = maxiter;
done:
    if (info) {
        info->iterations = its;
        info->converged = converged;
        info->rnorm = (double)rnorm;
        info->bnorm = (double)bnorm;
    }
    FN(hier_free_)(&h);
    free(diag); free(r); free(z); free(d); free(q); free(partials); free(cellpartials);
    return its;
}

/* project_kernel! (src/flip.jl:1113-1130) for one axis: u -= delta/dx on faces with a LIQUID
 * side and no SOLID side (ghost fluid at air faces); valid flag = 1 exactly there. */
static void FN(gradient_axis_)(const orc_grid* g, R* u, uint8_t* f, const R* P, const uint8_t* t,
                               const R* phi, int axis) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const int e1 = n1 + (axis == 0), e2 = n2 + (axis == 1), e3 = n3 + (axis == 2);
    const R dx = (R)g->dx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < e3; k++)
        for (int j = 0; j < e2; j++)
            for (int i = 0; i < e1; i++) {
                int a = i - (axis == 0), bb = j - (axis == 1), cc = k - (axis == 2);
                uint8_t t0 = typeat(t, n1, n2, n3, a, bb, cc), t1 = typeat(t, n1, n2, n3, i, j, k);
                int ok = t0 != SOLID && t1 != SOLID && (t0 == LIQUID || t1 == LIQUID);
                size_t fidx = ID(e1, e2, i, j, k);
                if (ok) {
                    size_t c0 = ID(n1, n2, a, bb, cc), c1 = ID(n1, n2, i, j, k);
                    R delta;
                    if (t0 == LIQUID && t1 == LIQUID) delta = P[c1] - P[c0];
                    else if (t0 == LIQUID) delta = (-P[c0]) / FN(theta_)(phi[c0], phi[c1]);
                    else delta = P[c1] / FN(theta_)(phi[c1], phi[c0]);
                    u[fidx] = u[fidx] - delta / dx;
                }
                f[fidx] = ok ? 1 : 0;
            }
}

void FN(orc_gradient_)(const orc_grid* g, R* u, R* v, R* w, uint8_t* fu, uint8_t* fv, uint8_t* fw,
                       const R* P, const uint8_t* types, const R* phi) {
    FN(gradient_axis_)(g, u, fu, P, types, phi, 0);
    FN(gradient_axis_)(g, v, fv, P, types, phi, 1);
    FN(gradient_axis_)(g, w, fw, P, types, phi, 2);
}

/* volume_kernel! + volume (src/flip.jl:261-279, 293): sum of clamp(0.5 - phi/dx, 0, 1) over
 * cells whose centre is not solid (geometry, not types), times dx^3. */
double FN(orc_volume_)(const orc_grid* g, const R* phi) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2], P = plen_(g);
    const int n1 = g->n[0], n2 = g->n[1];
    R* partials = (R*)calloc(P, sizeof(R));
    const R dx = (R)g->dx;
#pragma omp parallel for schedule(static)
    for (size_t gi = 0; gi < P; gi++) {
        R s[256];
        for (int t = 0; t < 256; t++) {
            size_t i = gi * 256 + t;
            R v = 0;
            if (i < N) {
                int a = (int)(i % n1), b = (int)((i / n1) % n2), c = (int)(i / ((size_t)n1 * n2));
                if (!issolidcell(g, a, b, c)) {
                    R x = (R)0.5f - phi[i] / dx;
                    v = x > (R)1 ? (R)1 : (x < (R)0 ? (R)0 : x);
                }
            }
            s[t] = v;
        }
        partials[gi] = FN(tree256_)(s);
    }
    R total = FN(sumseq_)(partials, P);
    free(partials);
    return (double)(total * (dx * dx * dx));
}

/* project! (src/flip.jl:1144-1156). */
int FN(orc_project_)(const orc_grid* g, R* u, R* v, R* w, uint8_t* fu, uint8_t* fv, uint8_t* fw, R* P,
                     const uint8_t* types, const R* phi, R volume0, double dt, double recover, R tol,
                     int maxiter, int sweeps, int coarse, orc_info* info) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2];
    R vol = (R)FN(orc_volume_)(g, phi);
    R loss = (volume0 - vol) / volume0;
    double lo = -0.01 / dt, hi = 0.01 / dt, x = (double)loss / recover;
    R gamma = (R)(float)(x > hi ? hi : (x < lo ? lo : x));
    R* b = (R*)calloc(N, sizeof(R));
    FN(orc_rhs_)(g, b, u, v, w, types, gamma);
    /* clearair_kernel! (src/flip.jl:1132-1135) */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; i++)
        if (types[i] != LIQUID) P[i] = 0;
    int its = FN(orc_pressure_)(g, P, b, types, phi, tol, maxiter, sweeps, coarse, info);
    FN(orc_gradient_)(g, u, v, w, fu, fv, fw, P, types, phi);
    if (info) {
        info->volume = (double)vol;
        info->gamma = (float)gamma;
    }
    free(b);
    return its;
}

/* ---- the adjoint of project! w.r.t. the face velocities (not in the reference; derived
 * from its forward kernels rhs_kernel! src/flip.jl:817-822 and project_kernel!
 * src/flip.jl:1113-1130): beta = dx G^T g, A mu = beta, g_in = g + D^T mu. ---- */

/* One face of LIQUID cell c seen from c: w g, w = 1 towards LIQUID, 1/theta towards AIR,
 * the face dropped towards SOLID (project_kernel!'s `ok`). */
static inline R FN(vjp_term_)(const R* gf, size_t fi, const uint8_t* t, const R* phi, int n1, int n2, int n3,
                              size_t c, int a, int b, int cc) {
    uint8_t tn = typeat(t, n1, n2, n3, a, b, cc);
    if (tn == SOLID) return (R)0;
    if (tn == LIQUID) return gf[fi];
    return gf[fi] / FN(theta_)(phi[c], phi[ID(n1, n2, a, b, cc)]);
}

/* beta_c = (low faces) - (high faces) of w g, in the order -x, +x, -y, +y, -z, +z. */
void FN(orc_vjp_rhs_)(const orc_grid* g, R* beta, const R* gu, const R* gv, const R* gw, const uint8_t* types,
                      const R* phi) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; k++)
        for (int j = 0; j < n2; j++)
            for (int i = 0; i < n1; i++) {
                size_t c = ID(n1, n2, i, j, k);
                R s = 0;
                if (types[c] == LIQUID) {
                    size_t fu = ID(n1 + 1, n2, i, j, k), fv = ID(n1, n2 + 1, i, j, k), fw = ID(n1, n2, i, j, k);
                    s = s + FN(vjp_term_)(gu, fu, types, phi, n1, n2, n3, c, i - 1, j, k);
                    s = s - FN(vjp_term_)(gu, ID(n1 + 1, n2, i + 1, j, k), types, phi, n1, n2, n3, c, i + 1, j, k);
                    s = s + FN(vjp_term_)(gv, fv, types, phi, n1, n2, n3, c, i, j - 1, k);
                    s = s - FN(vjp_term_)(gv, ID(n1, n2 + 1, i, j + 1, k), types, phi, n1, n2, n3, c, i, j + 1, k);
                    s = s + FN(vjp_term_)(gw, fw, types, phi, n1, n2, n3, c, i, j, k - 1);
                    s = s - FN(vjp_term_)(gw, ID(n1, n2, i, j, k + 1), types, phi, n1, n2, n3, c, i, j, k + 1);
                }
                beta[c] = s;
            }
}

/* g_in = g + mu_before [before LIQUID] - mu_after [after LIQUID], one axis. */
static void FN(vjp_axis_)(const orc_grid* g, R* out, const R* gf, const R* mu, const uint8_t* t, int axis) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    const int e1 = n1 + (axis == 0), e2 = n2 + (axis == 1), e3 = n3 + (axis == 2);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < e3; k++)
        for (int j = 0; j < e2; j++)
            for (int i = 0; i < e1; i++) {
                int a = i - (axis == 0), bb = j - (axis == 1), cc = k - (axis == 2);
                size_t fi = ID(e1, e2, i, j, k);
                R r = gf[fi];
                if (typeat(t, n1, n2, n3, a, bb, cc) == LIQUID) r = r + mu[ID(n1, n2, a, bb, cc)];
                if (typeat(t, n1, n2, n3, i, j, k) == LIQUID) r = r - mu[ID(n1, n2, i, j, k)];
                out[fi] = r;
            }
}

void FN(orc_vjp_faces_)(const orc_grid* g, R* ou, R* ov, R* ow, const R* gu, const R* gv, const R* gw,
                        const R* mu, const uint8_t* types) {
    FN(vjp_axis_)(g, ou, gu, mu, types, 0);
    FN(vjp_axis_)(g, ov, gv, mu, types, 1);
    FN(vjp_axis_)(g, ow, gw, mu, types, 2);
}

/* The whole adjoint: (gu, gv, gw) in, g_in out in place; mu the warm start in, out. */
int FN(orc_project_vjp_)(const orc_grid* g, R* gu, R* gv, R* gw, R* mu, const uint8_t* types, const R* phi,
                         R tol, int maxiter, int sweeps, int coarse, orc_info* info) {
    const size_t N = (size_t)g->n[0] * g->n[1] * g->n[2];
    R* beta = (R*)calloc(N, sizeof(R));
    FN(orc_vjp_rhs_)(g, beta, gu, gv, gw, types, phi);
    int its = FN(orc_pressure_)(g, mu, beta, types, phi, tol, maxiter, sweeps, coarse, info);
    FN(orc_vjp_faces_)(g, gu, gv, gw, gu, gv, gw, mu, types);
    free(beta);
    return its;
}

/* ---- semi-Lagrangian advection (advect_kernel!, src/flip.jl:357-369; trilinear,
 * src/interpolation.jl:4-17; nodepos/indexspace/velocity, src/flip.jl:76-81) and its
 * adjoint (not in the reference; the reverse of the same steps). ---- */

/* trilinear(A, q) on an a1 x a2 x a3 array (0-based index space, clamped to the array).
 * With wts != NULL it also returns the 8 corner indices and weights and the gradient in
 * q (zero along an axis whose coordinate was clamped). */
static R FN(tri_)(const R* A, int a1, int a2, int a3, R qx, R qy, R qz, size_t* idx, R* wts, R* grad) {
    R x = qx > (R)(a1 - 1) ? (R)(a1 - 1) : (qx < (R)0 ? (R)0 : qx);
    R y = qy > (R)(a2 - 1) ? (R)(a2 - 1) : (qy < (R)0 ? (R)0 : qy);
    R z = qz > (R)(a3 - 1) ? (R)(a3 - 1) : (qz < (R)0 ? (R)0 : qz);
    int i = (int)x, j = (int)y, k = (int)z;
    if (i > a1 - 2) i = a1 - 2;
    if (j > a2 - 2) j = a2 - 2;
    if (k > a3 - 2) k = a3 - 2;
    R fx = x - (R)i, fy = y - (R)j, fz = z - (R)k;
    size_t b000 = ID(a1, a2, i, j, k), sx = 1, sy = (size_t)a1, sz = (size_t)a1 * a2;
    R A000 = A[b000], A100 = A[b000 + sx], A010 = A[b000 + sy], A110 = A[b000 + sx + sy];
    R A001 = A[b000 + sz], A101 = A[b000 + sx + sz], A011 = A[b000 + sy + sz], A111 = A[b000 + sx + sy + sz];
    R c00 = A000 * ((R)1 - fx) + A100 * fx;
    R c10 = A010 * ((R)1 - fx) + A110 * fx;
    R c01 = A001 * ((R)1 - fx) + A101 * fx;
    R c11 = A011 * ((R)1 - fx) + A111 * fx;
    R val = (c00 * ((R)1 - fy) + c10 * fy) * ((R)1 - fz) + (c01 * ((R)1 - fy) + c11 * fy) * fz;
    if (wts) {
        R gx = (R)1 - fx, gy = (R)1 - fy, gz = (R)1 - fz;
        idx[0] = b000; wts[0] = gx * gy * gz;
        idx[1] = b000 + sx; wts[1] = fx * gy * gz;
        idx[2] = b000 + sy; wts[2] = gx * fy * gz;
        idx[3] = b000 + sx + sy; wts[3] = fx * fy * gz;
        idx[4] = b000 + sz; wts[4] = gx * gy * fz;
        idx[5] = b000 + sx + sz; wts[5] = fx * gy * fz;
        idx[6] = b000 + sy + sz; wts[6] = gx * fy * fz;
        idx[7] = b000 + sx + sy + sz; wts[7] = fx * fy * fz;
        /* clamp passes the derivative on its closed range (as ChainRules' and torch's rules) */
        int inx = qx >= (R)0 && qx <= (R)(a1 - 1), iny = qy >= (R)0 && qy <= (R)(a2 - 1);
        int inz = qz >= (R)0 && qz <= (R)(a3 - 1);
        R dx_ = ((A100 - A000) * gy + (A110 - A010) * fy) * gz + ((A101 - A001) * gy + (A111 - A011) * fy) * fz;
        R dy_ = (c10 - c00) * gz + (c11 - c01) * fz;
        R dz_ = (c01 * gy + c11 * fy) - (c00 * gy + c10 * fy);
        grad[0] = inx ? dx_ : (R)0;
        grad[1] = iny ? dy_ : (R)0;
        grad[2] = inz ? dz_ : (R)0;
    }
    return val;
}

typedef struct {
    const R* f[3];  /* u, v, w */
    int d[3][3];    /* their dims */
    R off[3][3];    /* UOFF, VOFF, WOFF */
    R lo[3], dx;
} FN(flow_);

static void FN(flow_init_)(FN(flow_) * fl, const orc_grid* g, const R* u, const R* v, const R* w) {
    const int n1 = g->n[0], n2 = g->n[1], n3 = g->n[2];
    fl->f[0] = u; fl->f[1] = v; fl->f[2] = w;
    for (int c = 0; c < 3; c++) {
        fl->d[c][0] = n1 + (c == 0); fl->d[c][1] = n2 + (c == 1); fl->d[c][2] = n3 + (c == 2);
        for (int a = 0; a < 3; a++) fl->off[c][a] = a == c ? (R)0 : (R)0.5f;
        fl->lo[c] = (R)g->lo[c];
    }
    fl->dx = (R)g->dx;
}

/* velocity(u, v, w, g, p) (src/flip.jl:80-81); with the *_g outputs, each component's
 * corner indices/weights and its gradient in p. */
static void FN(velocity_)(const FN(flow_) * fl, const R p[3], R out[3], size_t (*idx)[8], R (*wts)[8], R (*gp)[3]) {
    for (int c = 0; c < 3; c++) {
        R q[3];
        for (int a = 0; a < 3; a++) q[a] = (p[a] - fl->lo[a]) / fl->dx - fl->off[c][a];
        R gq[3];
        out[c] = FN(tri_)(fl->f[c], fl->d[c][0], fl->d[c][1], fl->d[c][2], q[0], q[1], q[2], idx ? idx[c] : NULL,
                          wts ? wts[c] : NULL, gq);
        if (gp)
            for (int a = 0; a < 3; a++) gp[c][a] = gq[a] / fl->dx;
    }
}

/* substeps (src/flip.jl:372): clamp(trunc(ceil(cells)), 1, 32). */
static int FN(substeps_)(R cells) {
    R c = (R)ceil((double)cells);
    if (!(c >= (R)1)) return 1;
    if (c > (R)32) return 32;
    return (int)c;
}

/* advect_kernel! for one array `src` (dims a[3], sample offset off[3]): out = src traced
 * back through the flow in RK2 sub-steps. */
void FN(orc_advect_)(const orc_grid* g, R* out, const R* src, const int32_t a[3], const R off[3], const R* u,
                     const R* v, const R* w, R dt) {
    FN(flow_) fl;
    FN(flow_init_)(&fl, g, u, v, w);
    const int a1 = a[0], a2 = a[1], a3 = a[2];
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < a3; k++)
        for (int j = 0; j < a2; j++)
            for (int i = 0; i < a1; i++) {
                R p[3] = {fl.lo[0] + ((R)i + off[0]) * fl.dx, fl.lo[1] + ((R)j + off[1]) * fl.dx,
                          fl.lo[2] + ((R)k + off[2]) * fl.dx};
                R vel[3];
                FN(velocity_)(&fl, p, vel, NULL, NULL, NULL);
                int m = FN(substeps_)((R)sqrt((double)(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) * dt / fl.dx);
                R h = dt / (R)m;
                for (int s = 0; s < m; s++) {
                    R v1[3], pm[3], v2[3];
                    FN(velocity_)(&fl, p, v1, NULL, NULL, NULL);
                    R hh = (R)0.5f * h;
                    for (int c = 0; c < 3; c++) pm[c] = p[c] - hh * v1[c];
                    FN(velocity_)(&fl, pm, v2, NULL, NULL, NULL);
                    for (int c = 0; c < 3; c++) p[c] = p[c] - h * v2[c];
                }
                R q[3];
                for (int c = 0; c < 3; c++) q[c] = (p[c] - fl.lo[c]) / fl.dx - off[c];
                out[ID(a1, a2, i, j, k)] = FN(tri_)(src, a1, a2, a3, q[0], q[1], q[2], NULL, NULL, NULL);
            }
}

/* The adjoint of orc_advect_: for the cotangent gout of `out`, adds d/d src into gsrc and
 * d/d (u, v, w) through the traced positions into gu, gv, gw (sequential, so the sums are
 * in a fixed order). The sub-step count is piecewise constant: no derivative. */
void FN(orc_advect_vjp_)(const orc_grid* g, const R* gout, const R* src, const int32_t a[3], const R off[3],
                         const R* u, const R* v, const R* w, R dt, R* gsrc, R* gu, R* gv, R* gw) {
    FN(flow_) fl;
    FN(flow_init_)(&fl, g, u, v, w);
    R* gf[3] = {gu, gv, gw};
    const int a1 = a[0], a2 = a[1], a3 = a[2];
    R ps[33][3], pms[32][3];
    for (int k = 0; k < a3; k++)
        for (int j = 0; j < a2; j++)
            for (int i = 0; i < a1; i++) {
                const R go = gout[ID(a1, a2, i, j, k)];
                R p[3] = {fl.lo[0] + ((R)i + off[0]) * fl.dx, fl.lo[1] + ((R)j + off[1]) * fl.dx,
                          fl.lo[2] + ((R)k + off[2]) * fl.dx};
                R vel[3];
                FN(velocity_)(&fl, p, vel, NULL, NULL, NULL);
                int m = FN(substeps_)((R)sqrt((double)(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) * dt / fl.dx);
                R h = dt / (R)m, hh = (R)0.5f * h;
                for (int c = 0; c < 3; c++) ps[0][c] = p[c];
                for (int s = 0; s < m; s++) {
                    R v1[3], v2[3];
                    FN(velocity_)(&fl, ps[s], v1, NULL, NULL, NULL);
                    for (int c = 0; c < 3; c++) pms[s][c] = ps[s][c] - hh * v1[c];
                    FN(velocity_)(&fl, pms[s], v2, NULL, NULL, NULL);
                    for (int c = 0; c < 3; c++) ps[s + 1][c] = ps[s][c] - h * v2[c];
                }
                /* out = tri(src, q(p_m)) */
                R q[3], gq[3], wt[8], pb[3];
                size_t ix[8];
                for (int c = 0; c < 3; c++) q[c] = (ps[m][c] - fl.lo[c]) / fl.dx - off[c];
                FN(tri_)(src, a1, a2, a3, q[0], q[1], q[2], ix, wt, gq);
                for (int t = 0; t < 8; t++) gsrc[ix[t]] += go * wt[t];
                for (int c = 0; c < 3; c++) pb[c] = go * gq[c] / fl.dx;
                for (int s = m - 1; s >= 0; s--) {
                    /* p_{s+1} = p_s - h V(pm_s), pm_s = p_s - hh V(p_s) */
                    R vv[3], gp[3][3], wv[3][8];
                    size_t iv[3][8];
                    R vb[3], pmb[3];
                    for (int c = 0; c < 3; c++) vb[c] = -h * pb[c];
                    FN(velocity_)(&fl, pms[s], vv, iv, wv, gp);
                    for (int c = 0; c < 3; c++) pmb[c] = (R)0;
                    for (int c = 0; c < 3; c++) {
                        for (int t = 0; t < 8; t++) gf[c][iv[c][t]] += vb[c] * wv[c][t];
                        for (int e = 0; e < 3; e++) pmb[e] += vb[c] * gp[c][e];
                    }
                    for (int c = 0; c < 3; c++) {
                        pb[c] += pmb[c];
                        vb[c] = -hh * pmb[c];
                    }
                    FN(velocity_)(&fl, ps[s], vv, iv, wv, gp);
                    for (int c = 0; c < 3; c++) {
                        for (int t = 0; t < 8; t++) gf[c][iv[c][t]] += vb[c] * wv[c][t];
                        for (int e = 0; e < 3; e++) pb[e] += vb[c] * gp[c][e];
                    }
                }
            }
}

#undef FN
