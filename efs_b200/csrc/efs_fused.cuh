// efs_fused.cuh — single-pass E+H update (the engine's default core path).
//
// One launch advances E and H of a whole timestep, moving each field value
// through HBM once (read old, write new): 48 B of fields + 4 B of material
// index per cell, against 80 B for separate E and H sweeps.
//
// Layout: NIJK (z fastest).  A block owns a tile of TY rows (y) x 32*CPT
// columns (z) and streams the x-planes of one x-chunk.  At plane x it
//   1. stages H_old(x) of the tile plus a one-cell low halo in shared memory,
//   2. computes E_new(x) on the tile plus a one-cell high halo (an extra warp
//      row for y, an extra cell on lane 31 for z) — the halo is recomputed,
//      never read from a neighbour tile,
//   3. computes H_new(x-1) of the tile from E_new(x-1) (shared memory) and
//      E_new(x) (registers).
// Old and new fields live in separate buffers (as do the UPML flux arrays),
// so recomputed halo cells and neighbouring tiles never race.
//
// H cells whose curl reads an E value that a sparse post-update operation
// rewrites (TFSF, Mur apply, excitation, PBC, series RLC) are flagged in a
// bitmask and left for k_deferred_h, which runs after those operations.  The
// result is the reference's phase order exactly, bit for bit.
#pragma once
#include "efs_kernels.cuh"

namespace efs {

constexpr int PML_MAX_OVERLAP = 4;

struct FusedGrid {
    uint32_t Nx, Ny, Nz, xchunk;
    size_t N, NyNz;
    const float* V0; const float* H0;   // fields at the start of the step
    float* V1; float* H1;               // fields after the step
    const uint32_t* mat; const float* table;
    const float* vv; const float* vi; const float* ii; const float* iv;
    const uint32_t* defer;              // bit per cell: H update deferred (may be null)
};

// UPML chain with separate old/new flux buffers; up to PML_MAX_OVERLAP regions per cell.
template <bool VOLT>
__device__ __forceinline__ float pml_chain_pp(const PmlSet& ps, const PmlSet& pn, uint32_t x, uint32_t y, uint32_t z,
                                              uint32_t n, float vold, bool core, float cv, float ci, float curl, bool write) {
    int reg[PML_MAX_OVERLAP];
    size_t pp[PML_MAX_OVERLAP];
    int cnt = 0;
    for (int r = 0; r < ps.count; ++r)
        if (in_region(ps.r[r], x, y, z) && cnt < PML_MAX_OVERLAP) { reg[cnt] = r; pp[cnt] = region_p(ps.r[r], n, x, y, z); ++cnt; }
    if (cnt == 0) return core ? upd(vold, cv, ci, curl) : vold;
    float fh[PML_MAX_OVERLAP];
    float v = vold;
    for (int k = 0; k < cnt; ++k) {
        const PmlRegion& R = ps.r[reg[k]];
        const float a = VOLT ? R.vv[pp[k]] : R.ii[pp[k]];
        const float b = VOLT ? R.vvfo[pp[k]] : R.iifo[pp[k]];
        const float fo = VOLT ? R.vflux[pp[k]] : R.cflux[pp[k]];
        fh[k] = __fsub_rn(__fmul_rn(a, v), __fmul_rn(b, fo));
        v = fo;
    }
    if (core) v = upd(v, cv, ci, curl);
    for (int k = 0; k < cnt; ++k) {
        const PmlRegion& R = ps.r[reg[k]];
        const float fn = VOLT ? R.vvfn[pp[k]] : R.iifn[pp[k]];
        if (write) {
            float* fl = VOLT ? pn.r[reg[k]].vflux : pn.r[reg[k]].cflux;
            fl[pp[k]] = v;
        }
        v = __fadd_rn(fh[k], __fmul_rn(fn, v));
    }
    return v;
}

template <bool IDX>
__device__ __forceinline__ void coeffs_f(const FusedGrid& g, size_t c, uint32_t m, int base, float out[6]) {
    if (IDX) {
        const float* t = g.table + (size_t)m * 12 + base;
#pragma unroll
        for (int k = 0; k < 6; ++k) out[k] = __ldg(t + k);
    } else {
        const float* a = base == 0 ? g.vv : g.ii;
        const float* b = base == 0 ? g.vi : g.iv;
        out[0] = __ldg(a + c); out[1] = __ldg(a + g.N + c); out[2] = __ldg(a + 2 * g.N + c);
        out[3] = __ldg(b + c); out[4] = __ldg(b + g.N + c); out[5] = __ldg(b + 2 * g.N + c);
    }
}

// A lane's cell k sits at z = z0 + k*32 + lane: every access is coalesced
// across the warp and conflict-free in shared memory.
template <int CPT>
__device__ __forceinline__ void load_cells(const float* __restrict__ p, const bool ok[CPT], float out[CPT]) {
#pragma unroll
    for (int k = 0; k < CPT; ++k) out[k] = ok[k] ? __ldg(p + 32 * k) : 0.f;
}
template <int CPT>
__device__ __forceinline__ void store_cells(float* __restrict__ p, const bool ok[CPT], const float v[CPT]) {
#pragma unroll
    for (int k = 0; k < CPT; ++k) if (ok[k]) p[32 * k] = v[k];
}

template <bool IDX, bool PML, int CPT, int TY>
__global__ void __launch_bounds__(32 * (TY + 1)) k_fused(const FusedGrid g, const PmlSet ps, const PmlSet pn) {
    constexpr int TZ = 32 * CPT;
    constexpr int W = TZ + 2;                    // column j <-> z = z0 - 1 + j
    __shared__ float sH[3][TY + 2][W];           // row r <-> y = y0 - 1 + r
    __shared__ float sE[2][3][TY + 1][W];        // row r <-> y = y0 + r
    const int lane = threadIdx.x, ty = threadIdx.y;
    const uint32_t z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY;
    const uint32_t y = y0 + ty;
    const uint32_t zc = z0 + lane;             // cell k: z = zc + 32*k
    const bool rowIn = y < g.Ny;
    const bool own_row = ty < TY;
    const size_t N = g.N, NyNz = g.NyNz, Nz = g.Nz;
    const uint32_t xs = blockIdx.z * g.xchunk;
    if (xs >= g.Nx) return;                       // whole block idle (uniform)
    const uint32_t xe = min(xs + g.xchunk, g.Nx);
    const uint32_t xl = xe < g.Nx ? xe : g.Nx - 1; // last plane whose E this block computes
    const bool extra = (lane == 31) && (z0 + TZ < g.Nz) && rowIn;
    const uint32_t ze = z0 + TZ;
    bool ok[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) ok[k] = rowIn && (zc + 32 * k < g.Nz);
    const uint32_t ym = y0 > 0 ? y0 - 1 : y0;      // low y halo row (self at y = 0)
    const uint32_t zm = z0 > 0 ? z0 - 1 : z0;      // low z halo column (self at z = 0)

    float hp[CPT][3], hpe[3] = {0.f, 0.f, 0.f};    // H_old(x-1) of my cells (+ halo cell)
    uint32_t matp[CPT];
    if (xs > 0) {
        const size_t b = (size_t)(xs - 1) * NyNz + (size_t)y * Nz + zc;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            float t[CPT];
            load_cells<CPT>(g.H0 + n * N + b, ok, t);
#pragma unroll
            for (int k = 0; k < CPT; ++k) hp[k][n] = t[k];
            if (extra) hpe[n] = __ldg(g.H0 + n * N + (size_t)(xs - 1) * NyNz + (size_t)y * Nz + ze);
        }
    }
#pragma unroll
    for (int k = 0; k < CPT; ++k) matp[k] = 0;

    for (uint32_t x = xs; x <= xl; ++x) {
        const size_t b = (size_t)x * NyNz + (size_t)y * Nz + zc;
        float hc[CPT][3], hce[3] = {0.f, 0.f, 0.f};
        // ---- 1. stage H_old(x)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            float t[CPT];
            load_cells<CPT>(g.H0 + n * N + b, ok, t);
#pragma unroll
            for (int k = 0; k < CPT; ++k) { hc[k][n] = t[k]; sH[n][ty + 1][1 + 32 * k + lane] = t[k]; }
            if (extra) { hce[n] = __ldg(g.H0 + n * N + (size_t)x * NyNz + (size_t)y * Nz + ze); sH[n][ty + 1][TZ + 1] = hce[n]; }
        }
        if (ty == 0) {
            const bool rin = y0 < g.Ny;
            const size_t bm = (size_t)x * NyNz + (size_t)ym * Nz + zc;
            bool okm[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) okm[k] = rin && (zc + 32 * k < g.Nz);
#pragma unroll
            for (int n = 0; n < 3; n += 2) {     // Hx, Hz at y-1
                float t[CPT];
                load_cells<CPT>(g.H0 + n * N + bm, okm, t);
#pragma unroll
                for (int k = 0; k < CPT; ++k) sH[n][0][1 + 32 * k + lane] = t[k];
                if (lane == 31 && rin && ze < g.Nz) sH[n][0][TZ + 1] = __ldg(g.H0 + n * N + (size_t)x * NyNz + (size_t)ym * Nz + ze);
            }
        }
        if (lane == 0 && rowIn) {
            const size_t cz = (size_t)x * NyNz + (size_t)y * Nz + zm;
            sH[0][ty + 1][0] = __ldg(g.H0 + cz);         // Hx at z-1
            sH[1][ty + 1][0] = __ldg(g.H0 + N + cz);     // Hy at z-1
        }
        // ---- 2. E_old(x), material rows
        float eo[CPT][3], eoe[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            float t[CPT];
            load_cells<CPT>(g.V0 + n * N + b, ok, t);
#pragma unroll
            for (int k = 0; k < CPT; ++k) eo[k][n] = t[k];
            if (extra) eoe[n] = __ldg(g.V0 + n * N + (size_t)x * NyNz + (size_t)y * Nz + ze);
        }
        uint32_t matc[CPT], mate = 0;
        if (IDX) {
#pragma unroll
            for (int k = 0; k < CPT; ++k) matc[k] = ok[k] ? __ldg(g.mat + b + 32 * k) : 0u;
            if (extra) mate = __ldg(g.mat + (size_t)x * NyNz + (size_t)y * Nz + ze);
        } else {
#pragma unroll
            for (int k = 0; k < CPT; ++k) matc[k] = 0;
        }
        __syncthreads();
        // ---- 3. E_new(x) on my cells and the halo
        const bool x0self = (x == 0);
        float en[CPT][3];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int j = 1 + 32 * k + lane;
            const uint32_t z = zc + 32 * k;
            if (!ok[k]) { en[k][0] = en[k][1] = en[k][2] = 0.f; }
            else {
                const float hy_xm = x0self ? hc[k][1] : hp[k][1], hz_xm = x0self ? hc[k][2] : hp[k][2];
                const float cx = curl4(hc[k][2], sH[2][ty][j], hc[k][1], sH[1][ty + 1][j - 1]);
                const float cy = curl4(hc[k][0], sH[0][ty + 1][j - 1], hc[k][2], hz_xm);
                const float cz = curl4(hc[k][1], hy_xm, hc[k][0], sH[0][ty][j]);
                float kk[6];
                coeffs_f<IDX>(g, b + 32 * k, matc[k], 0, kk);
                if (PML) {
                    const bool wr = own_row && x < xe;
                    en[k][0] = pml_chain_pp<true>(ps, pn, x, y, z, 0, eo[k][0], true, kk[0], kk[3], cx, wr);
                    en[k][1] = pml_chain_pp<true>(ps, pn, x, y, z, 1, eo[k][1], true, kk[1], kk[4], cy, wr);
                    en[k][2] = pml_chain_pp<true>(ps, pn, x, y, z, 2, eo[k][2], true, kk[2], kk[5], cz, wr);
                } else {
                    en[k][0] = upd(eo[k][0], kk[0], kk[3], cx);
                    en[k][1] = upd(eo[k][1], kk[1], kk[4], cy);
                    en[k][2] = upd(eo[k][2], kk[2], kk[5], cz);
                }
            }
#pragma unroll
            for (int n = 0; n < 3; ++n) sE[x & 1][n][ty][j] = en[k][n];
        }
        if (lane == 31) {
            float ee[3] = {0.f, 0.f, 0.f};
            if (extra) {
                const int j = TZ + 1;
                const float hy_xm = x0self ? hce[1] : hpe[1], hz_xm = x0self ? hce[2] : hpe[2];
                const float cx = curl4(hce[2], sH[2][ty][j], hce[1], sH[1][ty + 1][j - 1]);
                const float cy = curl4(hce[0], sH[0][ty + 1][j - 1], hce[2], hz_xm);
                const float cz = curl4(hce[1], hy_xm, hce[0], sH[0][ty][j]);
                float kk[6];
                const size_t ce = (size_t)x * NyNz + (size_t)y * Nz + ze;
                coeffs_f<IDX>(g, ce, mate, 0, kk);
                if (PML) {
                    ee[0] = pml_chain_pp<true>(ps, pn, x, y, ze, 0, eoe[0], true, kk[0], kk[3], cx, false);
                    ee[1] = pml_chain_pp<true>(ps, pn, x, y, ze, 1, eoe[1], true, kk[1], kk[4], cy, false);
                    ee[2] = pml_chain_pp<true>(ps, pn, x, y, ze, 2, eoe[2], true, kk[2], kk[5], cz, false);
                } else {
                    ee[0] = upd(eoe[0], kk[0], kk[3], cx);
                    ee[1] = upd(eoe[1], kk[1], kk[4], cy);
                    ee[2] = upd(eoe[2], kk[2], kk[5], cz);
                }
            }
#pragma unroll
            for (int n = 0; n < 3; ++n) sE[x & 1][n][ty][TZ + 1] = ee[n];
        }
        if (own_row && x < xe) {
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                float t[CPT];
#pragma unroll
                for (int k = 0; k < CPT; ++k) t[k] = en[k][n];
                store_cells<CPT>(g.V1 + n * N + b, ok, t);
            }
        }
        __syncthreads();
        // ---- 4. H_new(x-1) on my cells
        if (own_row && x > xs) {
            const int pe = (x - 1) & 1;
            const size_t bm1 = b - NyNz;
            float hn[CPT][3];
            bool wr[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int j = 1 + 32 * k + lane;
                const uint32_t z = zc + 32 * k;
                wr[k] = ok[k];
                if (ok[k] && g.defer) {
                    const size_t cm = bm1 + 32 * k;
                    if ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u) wr[k] = false;
                }
                hn[k][0] = hn[k][1] = hn[k][2] = 0.f;
                if (!wr[k]) continue;
                const bool core = (y + 1 < g.Ny) && (z + 1 < g.Nz);
                float cx = 0.f, cy = 0.f, cz = 0.f;
                if (core) {
                    const float ex = sE[pe][0][ty][j], ey = sE[pe][1][ty][j], ez = sE[pe][2][ty][j];
                    cx = curl4(ez, sE[pe][2][ty + 1][j], ey, sE[pe][1][ty][j + 1]);
                    cy = curl4(ex, sE[pe][0][ty][j + 1], ez, en[k][2]);
                    cz = curl4(ey, en[k][1], ex, sE[pe][0][ty + 1][j]);
                }
                float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (core) coeffs_f<IDX>(g, bm1 + 32 * k, matp[k], 6, kk);
                if (PML) {
                    hn[k][0] = pml_chain_pp<false>(ps, pn, x - 1, y, z, 0, hp[k][0], core, kk[0], kk[3], cx, true);
                    hn[k][1] = pml_chain_pp<false>(ps, pn, x - 1, y, z, 1, hp[k][1], core, kk[1], kk[4], cy, true);
                    hn[k][2] = pml_chain_pp<false>(ps, pn, x - 1, y, z, 2, hp[k][2], core, kk[2], kk[5], cz, true);
                } else if (core) {
                    hn[k][0] = upd(hp[k][0], kk[0], kk[3], cx);
                    hn[k][1] = upd(hp[k][1], kk[1], kk[4], cy);
                    hn[k][2] = upd(hp[k][2], kk[2], kk[5], cz);
                } else {
                    hn[k][0] = hp[k][0]; hn[k][1] = hp[k][1]; hn[k][2] = hp[k][2];
                }
            }
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                float t[CPT];
#pragma unroll
                for (int k = 0; k < CPT; ++k) t[k] = hn[k][n];
                store_cells<CPT>(g.H1 + n * N + bm1, wr, t);
            }
        }
        // ---- rotate
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            hp[k][0] = hc[k][0]; hp[k][1] = hc[k][1]; hp[k][2] = hc[k][2];
            matp[k] = matc[k];
        }
        hpe[0] = hce[0]; hpe[1] = hce[1]; hpe[2] = hce[2];
    }
    // ---- H of the last plane x = Nx-1: no core update (loop bounds), UPML / pass-through only
    if (xe == g.Nx && own_row) {
        const size_t bl = (size_t)(g.Nx - 1) * NyNz + (size_t)y * Nz + zc;
        float hn[CPT][3];
        bool wr[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            wr[k] = ok[k];
            if (ok[k] && g.defer) {
                const size_t cm = bl + 32 * k;
                if ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u) wr[k] = false;
            }
#pragma unroll
            for (int n = 0; n < 3; ++n)
                hn[k][n] = (PML && wr[k]) ? pml_chain_pp<false>(ps, pn, g.Nx - 1, y, zc + 32 * k, n, hp[k][n], false, 0.f, 0.f, 0.f, true)
                                          : hp[k][n];
        }
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            float t[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) t[k] = hn[k][n];
            store_cells<CPT>(g.H1 + n * N + bl, wr, t);
        }
    }
}

// H update of the deferred cells, after the E-side sparse operations:
// reads the final E_new, H_old, writes H_new (with UPML), one thread per cell.
template <bool IDX, bool PML>
__global__ void k_deferred_h(const FusedGrid g, const PmlSet ps, const PmlSet pn, const uint32_t* cells, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t c = cells[i];
    const size_t N = g.N, NyNz = g.NyNz, Nz = g.Nz;
    const uint32_t x = (uint32_t)(c / NyNz), y = (uint32_t)((c / Nz) % g.Ny), z = (uint32_t)(c % Nz);
    const bool core = (x + 1 < g.Nx) && (y + 1 < g.Ny) && (z + 1 < g.Nz);
    const float* V = g.V1;
    float cx = 0.f, cy = 0.f, cz = 0.f;
    float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (core) {
        cx = curl4(V[2 * N + c], V[2 * N + c + Nz], V[N + c], V[N + c + 1]);
        cy = curl4(V[c], V[c + 1], V[2 * N + c], V[2 * N + c + NyNz]);
        cz = curl4(V[N + c], V[N + c + NyNz], V[c], V[c + Nz]);
        coeffs_f<IDX>(g, c, IDX ? __ldg(g.mat + c) : 0u, 6, kk);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float ho = g.H0[q * N + c];
        float hn;
        if (PML) hn = pml_chain_pp<false>(ps, pn, x, y, z, q, ho, core, kk[q], kk[3 + q], q == 0 ? cx : (q == 1 ? cy : cz), true);
        else hn = core ? upd(ho, kk[q], kk[3 + q], q == 0 ? cx : (q == 1 ? cy : cz)) : ho;
        g.H1[q * N + c] = hn;
    }
}

}  // namespace efs
