// The level-set passes step! runs before the projection (sm_100a): redistance! (Jacobi
// sweeps of reinit_kernel!), classify! (fused into the last sweep) and filltrapped! (the
// trapped-air fill), src/flip.jl:608-760.
//
// Redistancing: a thread takes 4 consecutive cells of a row (16-byte loads of the row and
// of the rows at -+y and -+z, one element each side for -+x); the wall test of the cell
// and of its neighbours is the Float32 geometry of issolidcell, with the squares of the
// x positions formed once per thread and shared by the cells. The arithmetic is the
// reference's, in its order, with Julia's min/max (the sign of a zero counts) and clamp;
// the library is built without FMA contraction, so every cell is bit-identical to the
// reference's Float32 code. The last sweep also writes the cell classes (classify!).
//
// Trapped air: the reference reaches air from the grid's top layer by rounds of sweeps of
// one thread per line along z, x and y, until a round reaches nothing (a host read per
// round). A sweep fills every run of air along a line that holds a reached cell (a walk
// there and back with a carry). Here the AIR cells and the reached cells are bit masks,
// 32 cells of a row per word: a sweep along x is a carry through the words of a row with
// a 5-step shift-and-mask fill inside each word; a sweep along y or z moves 32 lines at
// once (one word column) and splits the line over a warp's lanes, each lane filling its
// segment and the carries joined by a warp scan of (generate, propagate) masks. The round
// loop is a conditional WHILE node of a CUDA graph whose last kernel ends it when a round
// reached nothing or maxrounds is done: no host round trip. The masks (a bit a cell each)
// stay in L2 through the rounds.
#pragma once

#include "mpp_base.cuh"

namespace mpp {

// ---- Julia's Float32 min/max/clamp (Base: diff = x - y, its sign bit picks) ----
__device__ __forceinline__ float jmin(float x, float y) {
    const float d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? x : y;
}
__device__ __forceinline__ float jmax(float x, float y) {
    const float d = x - y;
    if (isnan(x) || isnan(y)) return d;
    return signbit(d) ? y : x;
}

// eikonal (src/flip.jl:611-623): Godunov's upwind update from the smallest neighbour
// distance along each axis.
__device__ __forceinline__ float eikonal(float a, float b, float c, float h) {
    float t0 = jmin(a, b), t1 = jmax(a, b);
    a = t0;
    b = t1;
    t0 = jmin(b, c);
    t1 = jmax(b, c);
    b = t0;
    c = t1;
    t0 = jmin(a, b);
    t1 = jmax(a, b);
    a = t0;
    b = t1;
    float d = a + h;
    if (d > b) {
        const float ab = a - b;
        d = 0.5f * (a + b + sqrtf(jmax(2.0f * h * h - ab * ab, 0.0f)));
        if (d > c) {
            const float t = a + b + c;
            d = (t + sqrtf(jmax(t * t - 3.0f * (a * a + b * b + c * c - h * h), 0.0f))) / 3.0f;
        }
    }
    return d;
}

// reinit_kernel! (src/flip.jl:631-666), one Jacobi sweep out <- phi, W cells of a row per
// thread (W = 4: n1 a multiple of 4 and 16-byte aligned arrays; else W = 1). When `types`
// is given the sweep is redistance!'s last and classify_kernel! (src/flip.jl:682-686) runs
// on its output.
template <int W>
__global__ void __launch_bounds__(TPB) k_reinit(Geo g, const float* __restrict__ phi, float* __restrict__ out,
                                                float phimax, uint8_t* __restrict__ types) {
    pdl_wait();
    pdl_trigger();
    const int n1 = g.n[0], n2 = g.n[1], n3 = g.n[2];
    const unsigned rq = (unsigned)(n1 / W);
    const unsigned total = rq * (unsigned)n2 * (unsigned)n3;  // the host checks the grid fits 32 bits
    const float dx = g.dx, h = g.dx, R2 = g.radius * g.radius;
    const unsigned sy = (unsigned)n1, sz = (unsigned)n1 * (unsigned)n2;
    // Far from the surface every neighbour distance is phimax: the update is then the same
    // for every such cell, eikonal(phimax, phimax, phimax, h) (its costliest branch, two
    // square roots and a division), formed once here by the same code.
    const float far = jmin(eikonal(phimax, phimax, phimax, h), phimax);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        // 32-bit index arithmetic: a 64-bit division costs more than the cell's update
        const unsigned row = t / rq;
        const int q = (int)(t - row * rq);
        const unsigned kq = row / (unsigned)n2;
        const int j = (int)(row - kq * (unsigned)n2), k = (int)kq;
        const int i0 = q * W;
        const unsigned base = row * (unsigned)n1 + (unsigned)i0;
        // the wall test (issolidcell, src/flip.jl:64-66) of cells i0-1 .. i0+W and of the
        // rows at -+y, -+z
        float pxx[W + 2];
#pragma unroll
        for (int m = 0; m < W + 2; m++) {
            const float px = g.lo[0] + ((float)(i0 - 1 + m) + 0.5f) * dx;
            pxx[m] = px * px;
        }
        const float py = g.lo[1] + ((float)j + 0.5f) * dx, pyp = g.lo[1] + ((float)(j + 1) + 0.5f) * dx,
                    pym = g.lo[1] + ((float)(j - 1) + 0.5f) * dx;
        const float pyy = py * py, pyyp = pyp * pyp, pyym = pym * pym;
        const float pz = g.lo[2] + ((float)k + 0.5f) * dx, pzp = g.lo[2] + ((float)(k + 1) + 0.5f) * dx,
                    pzm = g.lo[2] + ((float)(k - 1) + 0.5f) * dx;
        const bool zs = pz < g.floor_z, zsp = pzp < g.floor_z, zsm = pzm < g.floor_z;
        // the values: the row's cells, -+x beyond them, the rows at -+y, -+z (read only
        // where the neighbour is in range)
        float c[W], yp[W], ym[W], zp[W], zm[W];
        const bool hy = j + 1 < n2, ly = j > 0, hz = k + 1 < n3, lz = k > 0;
        if constexpr (W == 4) {
            const float4 a = *reinterpret_cast<const float4*>(phi + base);
            c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
            const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 b1 = hy ? *reinterpret_cast<const float4*>(phi + base + sy) : z4;
            const float4 b2 = ly ? *reinterpret_cast<const float4*>(phi + base - sy) : z4;
            const float4 b3 = hz ? *reinterpret_cast<const float4*>(phi + base + sz) : z4;
            const float4 b4 = lz ? *reinterpret_cast<const float4*>(phi + base - sz) : z4;
            yp[0] = b1.x; yp[1] = b1.y; yp[2] = b1.z; yp[3] = b1.w;
            ym[0] = b2.x; ym[1] = b2.y; ym[2] = b2.z; ym[3] = b2.w;
            zp[0] = b3.x; zp[1] = b3.y; zp[2] = b3.z; zp[3] = b3.w;
            zm[0] = b4.x; zm[1] = b4.y; zm[2] = b4.z; zm[3] = b4.w;
        } else {
            c[0] = phi[base];
            yp[0] = hy ? phi[base + sy] : 0.f;
            ym[0] = ly ? phi[base - sy] : 0.f;
            zp[0] = hz ? phi[base + sz] : 0.f;
            zm[0] = lz ? phi[base - sz] : 0.f;
        }
        const float xl = i0 > 0 ? phi[base - 1] : 0.f;
        const float xr = i0 + W < n1 ? phi[base + W] : 0.f;
        float o[W];
        uint8_t ty[W];
#pragma unroll
        for (int m = 0; m < W; m++) {
            const int i = i0 + m;
            const float cm = c[m];
            // neighbours in `neighbour`'s order (src/flip.jl:84-92): +x, -x, +y, -y, +z, -z
            float f[6];
            bool ok[6];
            f[0] = m + 1 < W ? c[m + 1 < W ? m + 1 : 0] : xr;
            f[1] = m > 0 ? c[m > 0 ? m - 1 : 0] : xl;
            f[2] = yp[m];
            f[3] = ym[m];
            f[4] = zp[m];
            f[5] = zm[m];
            ok[0] = i + 1 < n1 && !(pxx[m + 2] + pyy > R2 || zs);
            ok[1] = i > 0 && !(pxx[m] + pyy > R2 || zs);
            ok[2] = hy && !(pxx[m + 1] + pyyp > R2 || zs);
            ok[3] = ly && !(pxx[m + 1] + pyym > R2 || zs);
            ok[4] = hz && !(pxx[m + 1] + pyy > R2 || zsp);
            ok[5] = lz && !(pxx[m + 1] + pyy > R2 || zsm);
            const bool solid = pxx[m + 1] + pyy > R2 || zs;
            float v;
            if (solid) {
                // a wall cell takes the lowest value of the water next to it
                float lowest = cm;
                bool found = false;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (ok[e]) {
                        lowest = found ? jmin(lowest, f[e]) : f[e];
                        found = true;
                    }
                v = found ? lowest : (cm > phimax ? phimax : (cm < -phimax ? -phimax : cm));
            } else {
                const bool inside = cm < 0.0f;
                bool frozen = false;
                float ax = phimax, ay = phimax, az = phimax;
#pragma unroll
                for (int e = 0; e < 6; e++)
                    if (ok[e]) {
                        if ((f[e] < 0.0f) != inside) frozen = true;
                        const float d = fabsf(f[e]);
                        if (e < 2) ax = jmin(ax, d);
                        else if (e < 4) ay = jmin(ay, d);
                        else az = jmin(az, d);
                    }
                if (frozen) {
                    v = cm;
                } else {
                    const float d = (ax == phimax && ay == phimax && az == phimax) ? far
                                                                                  : jmin(eikonal(ax, ay, az, h), phimax);
                    v = inside ? -d : d;
                }
            }
            o[m] = v;
            ty[m] = solid ? SOLID : (v < 0.0f ? LIQUID : AIR);
        }
        if constexpr (W == 4) {
            *reinterpret_cast<float4*>(out + base) = make_float4(o[0], o[1], o[2], o[3]);
            if (types) *reinterpret_cast<uchar4*>(types + base) = make_uchar4(ty[0], ty[1], ty[2], ty[3]);
        } else {
            out[base] = o[0];
            if (types) types[base] = ty[0];
        }
    }
}

// classify_kernel! (src/flip.jl:682-686) on its own (redistance! with no sweep).
__global__ void __launch_bounds__(TPB) k_classify(Geo g, const float* __restrict__ phi, uint8_t* __restrict__ types) {
    pdl_wait();
    pdl_trigger();
    FOR_CELLS(g.n[0], g.n[1], g.n[2], i, j, k, idx) {
        types[idx] = issolidcell(g, i, j, k) ? SOLID : (phi[idx] < 0.0f ? LIQUID : AIR);
    }
}

// ---- trapped air (src/flip.jl:698-760) on bit masks ----
// Word (wx, j, k) of a mask holds cells i = 32 wx .. 32 wx + 31 of row (j, k), bit b for
// i = 32 wx + b; a row has W1 = ceil(n1 / 32) words; bits past n1 are 0 (never AIR).
struct TrapMasks {
    uint32_t* air;    // AIR cells
    uint32_t* reach;  // cells reached from the top layer's air
    int n1, n2, n3, W1;
};
// The round loop's device state.
struct TrapState {
    int changed;    // a sweep of this round reached a new cell
    int rounds;     // rounds run
    int maxrounds;
    int pad;
};

// seedair_kernel! (src/flip.jl:704-708) and the AIR mask: a thread a word.
__global__ void __launch_bounds__(TPB) k_trap_pack(TrapMasks T, const uint8_t* __restrict__ types, TrapState* st,
                                                   int maxrounds, int vec) {
    pdl_wait();
    pdl_trigger();
    const int64_t words = (int64_t)T.W1 * T.n2 * T.n3;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t0 == 0) {
        st->changed = 0;
        st->rounds = 0;
        st->maxrounds = maxrounds;
    }
    for (int64_t t = t0; t < words; t += (int64_t)gridDim.x * blockDim.x) {
        const unsigned row = (unsigned)t / (unsigned)T.W1;  // the host checks the masks fit 32 bits
        const int wx = (int)((unsigned)t - row * (unsigned)T.W1);
        const int k = (int)(row / (unsigned)T.n2);
        const int i0 = wx * 32;
        const uint8_t* p = types + row * T.n1 + i0;
        uint32_t a = 0;
        if (vec) {  // n1 a multiple of 32, types 16-byte aligned: two 16-byte loads
            const uint4 v0 = reinterpret_cast<const uint4*>(p)[0], v1 = reinterpret_cast<const uint4*>(p)[1];
            const uint32_t w[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
#pragma unroll
            for (int q = 0; q < 8; q++)
#pragma unroll
                for (int b = 0; b < 4; b++)
                    if (((w[q] >> (8 * b)) & 0xffu) == AIR) a |= 1u << (4 * q + b);
        } else {
            const int cnt = T.n1 - i0 < 32 ? T.n1 - i0 : 32;
            for (int b = 0; b < cnt; b++)
                if (p[b] == AIR) a |= 1u << b;
        }
        T.air[t] = a;
        T.reach[t] = k == T.n3 - 1 ? a : 0u;  // the top layer's air
    }
}

// Fill toward higher / lower bits from the seeds g through runs of set bits of p (the
// AIR mask): 5 doubling steps of a shift-and-mask carry.
__device__ __forceinline__ uint32_t fill_up(uint32_t g, uint32_t p) {
    g |= p & (g << 1);
    p &= p << 1;
    g |= p & (g << 2);
    p &= p << 2;
    g |= p & (g << 4);
    p &= p << 4;
    g |= p & (g << 8);
    p &= p << 8;
    g |= p & (g << 16);
    return g;
}
__device__ __forceinline__ uint32_t fill_down(uint32_t g, uint32_t p) {
    g |= p & (g >> 1);
    p &= p >> 1;
    g |= p & (g >> 2);
    p &= p >> 2;
    g |= p & (g >> 4);
    p &= p >> 4;
    g |= p & (g >> 8);
    p &= p >> 8;
    g |= p & (g >> 16);
    return g;
}

// sweepair_kernel! along x (src/flip.jl:715-731): a thread a row, there and back through
// its words. A run of air holding a reached cell is reached whole.
__global__ void __launch_bounds__(TPB) k_trap_sweep_x(TrapMasks T, TrapState* st) {
    pdl_wait();
    pdl_trigger();
    const int64_t rows = (int64_t)T.n2 * T.n3;
    bool ch = false;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        uint32_t* R = T.reach + r * T.W1;
        const uint32_t* A = T.air + r * T.W1;
        uint32_t carry = 0;
        for (int w = 0; w < T.W1; w++) {
            const uint32_t a = A[w], r0 = R[w];
            const uint32_t f = fill_up(r0 | (carry & a & 1u), a);
            carry = f >> 31;
            if (f != r0) {
                R[w] = f;
                ch = true;
            }
        }
        carry = 0;
        for (int w = T.W1 - 1; w >= 0; w--) {
            const uint32_t a = A[w], r0 = R[w];
            const uint32_t f = fill_down(r0 | ((carry << 31) & a), a);
            carry = f & 1u;
            if (f != r0) {
                R[w] = f;
                ch = true;
            }
        }
    }
    if (__syncthreads_or(ch) && threadIdx.x == 0) atomicOr(&st->changed, 1);
}

// sweepair_kernel! along y (axis 1) or z (axis 2): a warp takes one word column (32 lines)
// and splits it into 32 segments of S words; each lane fills its segment (a line's fill is
// F_p = A_p & (R_p | F_{p-1})), and the carries into the segments come from a warp scan of
// the segments' (generate, propagate) masks: g = the fill from a zero carry, p = the AND of
// A over the segment, so a carry c leaves the segment as g | (p & c). Lines longer than
// 32 S go chunk by chunk, the carry passed on. Forward over the chunks, then back.
constexpr int TRAP_S = 8;
__global__ void __launch_bounds__(TPB) k_trap_sweep_col(TrapMasks T, TrapState* st, int axis) {
    pdl_wait();
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int64_t ncols = axis == 1 ? (int64_t)T.W1 * T.n3 : (int64_t)T.W1 * T.n2;
    const int len = axis == 1 ? T.n2 : T.n3;
    const int64_t step = axis == 1 ? (int64_t)T.W1 : (int64_t)T.W1 * T.n2;
    const int chunk = 32 * TRAP_S;
    const int nchunks = (len + chunk - 1) / chunk;
    bool ch = false;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t col = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); col < ncols; col += warps) {
        const int wx = (int)(col % T.W1);
        const int64_t other = col / T.W1;  // k (y sweep) or j (z sweep)
        const int64_t base = axis == 1 ? wx + (int64_t)T.W1 * T.n2 * other : wx + (int64_t)T.W1 * other;
        for (int dir = 0; dir < 2; dir++) {  // there (increasing p), then back
            __syncwarp();  // the way back reads what the other lanes wrote on the way there
            uint32_t carry = 0;
            for (int cq = 0; cq < nchunks; cq++) {
                const int cidx = dir == 0 ? cq : nchunks - 1 - cq;
                // this lane's segment of the chunk, in walking order
                const int p0 = cidx * chunk + (dir == 0 ? lane : 31 - lane) * TRAP_S;
                uint32_t a[TRAP_S], r[TRAP_S];
#pragma unroll
                for (int s = 0; s < TRAP_S; s++) {
                    const int p = dir == 0 ? p0 + s : p0 + TRAP_S - 1 - s;
                    const bool in = p < len;
                    a[s] = in ? T.air[base + (int64_t)p * step] : 0u;
                    r[s] = in ? T.reach[base + (int64_t)p * step] : 0u;
                }
                uint32_t gsum = 0, psum = 0xffffffffu;
#pragma unroll
                for (int s = 0; s < TRAP_S; s++) {
                    gsum = a[s] & (r[s] | gsum);
                    psum &= a[s];
                }
                // inclusive scan over the lanes in walking order: (g, p) then (g', p') is
                // (g' | (p' & g), p & p')
                uint32_t G = gsum, P = psum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t go = __shfl_up_sync(0xffffffffu, G, o), po = __shfl_up_sync(0xffffffffu, P, o);
                    if (lane >= o) {
                        G = G | (P & go);
                        P = P & po;
                    }
                }
                uint32_t cin = __shfl_up_sync(0xffffffffu, G, 1);
                uint32_t pin = __shfl_up_sync(0xffffffffu, P, 1);
                // the carry into this lane: from the chunks before, through lanes 0..lane-1
                cin = lane == 0 ? carry : (cin | (pin & carry));
                uint32_t f = cin;
#pragma unroll
                for (int s = 0; s < TRAP_S; s++) {
                    const int p = dir == 0 ? p0 + s : p0 + TRAP_S - 1 - s;
                    f = a[s] & (r[s] | f);
                    if (p < len && f != r[s]) {
                        T.reach[base + (int64_t)p * step] = f;
                        ch = true;
                    }
                }
                // the carry out of the chunk: the last lane's fill
                carry = __shfl_sync(0xffffffffu, f, 31);
            }
        }
    }
    if (__syncthreads_or(ch) && threadIdx.x == 0) atomicOr(&st->changed, 1);
}

// The end of a round (src/flip.jl:751-757): another round while this one reached a cell
// and fewer than maxrounds have run.
__global__ void k_trap_round(TrapState* st, cudaGraphConditionalHandle cond) {
    pdl_wait();
    const int r = st->rounds + 1;
    st->rounds = r;
    const int again = st->changed != 0 && r < st->maxrounds;
    st->changed = 0;
    cudaGraphSetConditional(cond, again ? 1u : 0u);
}

// fillair_kernel! (src/flip.jl:734-740): AIR that no sweep reached becomes LIQUID, with phi
// at most -depth (Julia's min). A thread a word of 32 cells.
__global__ void __launch_bounds__(TPB) k_trap_fill(TrapMasks T, uint8_t* __restrict__ types, float* __restrict__ phi,
                                                   float depth) {
    pdl_wait();
    pdl_trigger();
    const int64_t words = (int64_t)T.W1 * T.n2 * T.n3;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < words; t += (int64_t)gridDim.x * blockDim.x) {
        uint32_t m = T.air[t] & ~T.reach[t];
        if (!m) continue;
        const int wx = (int)(t % T.W1);
        const int64_t at = (t / T.W1) * T.n1 + (int64_t)wx * 32;
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            types[at + b] = LIQUID;
            phi[at + b] = jmin(phi[at + b], -depth);
        }
    }
}

}  // namespace mpp
