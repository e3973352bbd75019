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
    const uint32_t* defer_rows;         // bit per (x, y) row holding a deferred cell; ceil(Ny/32) words per x
    uint32_t* status;                   // device status word (bit 0: a bounded wait ran out)
};

// UPML chain with separate old/new flux buffers; up to PML_MAX_OVERLAP regions per cell.
template <bool VOLT>
__device__ __forceinline__ float pml_chain_pp(const PmlSet& ps, const PmlSet& pn, uint32_t mask, uint32_t x, uint32_t y,
                                              uint32_t z, uint32_t n, float vold, bool core, float cv, float ci, float curl,
                                              bool write) {
    int reg[PML_MAX_OVERLAP];
    size_t pp[PML_MAX_OVERLAP];
    int cnt = 0;
    for (uint32_t m = mask; m; m &= m - 1) {
        const int r = __ffs(m) - 1;
        if (in_region(ps.r[r], x, y, z) && cnt < PML_MAX_OVERLAP) { reg[cnt] = r; pp[cnt] = region_p(ps.r[r], n, x, y, z); ++cnt; }
    }
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

// UPML chain for a cell whose containing regions are exactly the set bits of
// `cell_mask` (already intersected per axis by the caller).  The single-region
// case (slab interiors) runs in registers; overlaps (corners) use the general chain.
template <bool VOLT>
__device__ __forceinline__ float pml_cell(const PmlSet& ps, const PmlSet& pn, uint32_t cell_mask, uint32_t x, uint32_t y,
                                          uint32_t z, uint32_t n, float vold, bool core, float cv, float ci, float curl,
                                          bool write) {
    if (cell_mask == 0) return core ? upd(vold, cv, ci, curl) : vold;
    if ((cell_mask & (cell_mask - 1)) == 0) {
        const int r = __ffs(cell_mask) - 1;
        const PmlRegion& R = ps.r[r];
        const size_t p = region_p(R, n, x, y, z);
        const float a = VOLT ? R.vv[p] : R.ii[p];
        const float b = VOLT ? R.vvfo[p] : R.iifo[p];
        const float fn = VOLT ? R.vvfn[p] : R.iifn[p];
        const float fo = VOLT ? R.vflux[p] : R.cflux[p];
        const float fh = __fsub_rn(__fmul_rn(a, vold), __fmul_rn(b, fo));
        const float v = core ? upd(fo, cv, ci, curl) : fo;
        if (write) (VOLT ? pn.r[r].vflux : pn.r[r].cflux)[p] = v;
        return __fadd_rn(fh, __fmul_rn(fn, v));
    }
    return pml_chain_pp<VOLT>(ps, pn, cell_mask, x, y, z, n, vold, core, cv, ci, curl, write);
}

// Regions (bit mask) whose extent along `axis` contains coordinate c.
__device__ __forceinline__ uint32_t axis_mask(const PmlSet& ps, uint32_t cand, int axis, uint32_t c) {
    uint32_t m = 0;
    for (uint32_t b = cand; b; b &= b - 1) {
        const int r = __ffs(b) - 1;
        if (c - ps.r[r].s[axis] < ps.r[r].n[axis]) m |= 1u << r;
    }
    return m;
}

template <bool IDX>
__device__ __forceinline__ void coeffs_f(const FusedGrid& g, size_t c, uint32_t m, int base, float out[6]) {
    if (IDX) {
        // a 48-byte row is three float4: [vv0 vv1 vv2 vi0][vi1 vi2 ii0 ii1][ii2 iv0 iv1 iv2]
        const float4* t = reinterpret_cast<const float4*>(g.table) + (size_t)m * 3;
        if (base == 0) {
            const float4 a = __ldg(t), b = __ldg(t + 1);
            out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w; out[4] = b.x; out[5] = b.y;
        } else {
            const float4 b = __ldg(t + 1), d = __ldg(t + 2);
            out[0] = b.z; out[1] = b.w; out[2] = d.x; out[3] = d.y; out[4] = d.z; out[5] = d.w;
        }
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


// cp.async of one float into shared memory; `valid` false zero-fills without reading
__device__ __forceinline__ void cp4(float* smem, const float* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp4u(uint32_t* smem, const uint32_t* gmem, bool valid) {
    cp4(reinterpret_cast<float*>(smem), reinterpret_cast<const float*>(gmem), valid);
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int NW>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NW)); }

template <int CPT, int TY>
struct FusedSmem {
    static constexpr int TZ = 32 * CPT;
    static constexpr int W = TZ + 2;          // column j <-> z = z0 - 1 + j
    float H[2][3][TY + 2][W];                 // H_old of a plane, rows y0-1 .. y0+TY (double-buffered)
    float E[2][3][TY + 1][W];                 // E_old of a plane, rows y0 .. y0+TY
    uint32_t M[2][TY + 1][W];                 // material rows
    float En[2][3][TY + 1][W];                // E_new of planes x-1, x
};

// Stage plane x of the tile (H with low halos, E_old, material) into buffer b.
template <bool IDX, int CPT, int TY>
__device__ __forceinline__ void stage_plane(FusedSmem<CPT, TY>& S, int b, const FusedGrid& g, uint32_t x, uint32_t y0,
                                            uint32_t z0, int lane, int ty) {
    constexpr int TZ = 32 * CPT;
    const size_t N = g.N, NyNz = g.NyNz, Nz = g.Nz;
    const uint32_t y = y0 + ty;
    const bool rowIn = y < g.Ny;
    const size_t base = (size_t)x * NyNz + (size_t)(rowIn ? y : 0) * Nz;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const uint32_t z = z0 + lane + 32 * k;
        const bool ok = rowIn && z < g.Nz;
        const size_t c = base + (ok ? z : 0);
        const int j = 1 + 32 * k + lane;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            cp4(&S.H[b][n][ty + 1][j], g.H0 + n * N + c, ok);
            cp4(&S.E[b][n][ty][j], g.V0 + n * N + c, ok);
        }
        if (IDX) cp4u(&S.M[b][ty][j], g.mat + c, ok);
    }
    const uint32_t ze = z0 + TZ;
    if (lane == 31) {                                   // high z halo cell
        const bool ok = rowIn && ze < g.Nz;
        const size_t c = base + (ok ? ze : 0);
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            cp4(&S.H[b][n][ty + 1][TZ + 1], g.H0 + n * N + c, ok);
            cp4(&S.E[b][n][ty][TZ + 1], g.V0 + n * N + c, ok);
        }
        if (IDX) cp4u(&S.M[b][ty][TZ + 1], g.mat + c, ok);
    }
    if (lane == 0) {                                    // low z halo: Hx, Hy at z-1 (self at z = 0)
        const uint32_t zm = z0 > 0 ? z0 - 1 : z0;
        const size_t c = base + zm;
        cp4(&S.H[b][0][ty + 1][0], g.H0 + c, rowIn);
        cp4(&S.H[b][1][ty + 1][0], g.H0 + N + c, rowIn);
    }
    if (ty == 0) {                                      // low y halo: Hx, Hz at y-1 (self at y = 0)
        const uint32_t ym = y0 > 0 ? y0 - 1 : y0;
        const size_t bm = (size_t)x * NyNz + (size_t)ym * Nz;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const uint32_t z = z0 + lane + 32 * k;
            const bool ok = z < g.Nz;
            const int j = 1 + 32 * k + lane;
            cp4(&S.H[b][0][0][j], g.H0 + bm + (ok ? z : 0), ok);
            cp4(&S.H[b][2][0][j], g.H0 + 2 * N + bm + (ok ? z : 0), ok);
        }
        if (lane == 31) {
            const bool ok = ze < g.Nz;
            cp4(&S.H[b][0][0][TZ + 1], g.H0 + bm + (ok ? ze : 0), ok);
            cp4(&S.H[b][2][0][TZ + 1], g.H0 + 2 * N + bm + (ok ? ze : 0), ok);
        }
    }
}

// E update of one cell at column j of row ty from staged data; hpx = H_old(x-1) (y,z comps).
template <bool IDX, bool PML, int CPT, int TY>
__device__ __forceinline__ void e_cell(const FusedSmem<CPT, TY>& S, int b, int ty, int j, const FusedGrid& g, size_t c,
                                       const PmlSet& ps, const PmlSet& pn, uint32_t pmask, uint32_t x, uint32_t y,
                                       uint32_t z, float hy_xm, float hz_xm, bool write_flux, float en[3]) {
    const float hx = S.H[b][0][ty + 1][j], hy = S.H[b][1][ty + 1][j], hz = S.H[b][2][ty + 1][j];
    const float cx = curl4(hz, S.H[b][2][ty][j], hy, S.H[b][1][ty + 1][j - 1]);
    const float cy = curl4(hx, S.H[b][0][ty + 1][j - 1], hz, hz_xm);
    const float cz = curl4(hy, hy_xm, hx, S.H[b][0][ty][j]);
    float kk[6];
    coeffs_f<IDX>(g, c, IDX ? S.M[b][ty][j] : 0u, 0, kk);
    const float e0 = S.E[b][0][ty][j], e1 = S.E[b][1][ty][j], e2 = S.E[b][2][ty][j];
    if (PML && pmask) {
        en[0] = pml_chain_pp<true>(ps, pn, pmask, x, y, z, 0, e0, true, kk[0], kk[3], cx, write_flux);
        en[1] = pml_chain_pp<true>(ps, pn, pmask, x, y, z, 1, e1, true, kk[1], kk[4], cy, write_flux);
        en[2] = pml_chain_pp<true>(ps, pn, pmask, x, y, z, 2, e2, true, kk[2], kk[5], cz, write_flux);
    } else {
        en[0] = upd(e0, kk[0], kk[3], cx);
        en[1] = upd(e1, kk[1], kk[4], cy);
        en[2] = upd(e2, kk[2], kk[5], cz);
    }
}

template <bool IDX, bool PML, int CPT, int TY>
__global__ void __launch_bounds__(32 * (TY + 1)) k_fused(const FusedGrid g, const PmlSet ps, const PmlSet pn) {
    constexpr int TZ = 32 * CPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FusedSmem<CPT, TY>& S = *reinterpret_cast<FusedSmem<CPT, TY>*>(smem_raw);
    const int lane = threadIdx.x, ty = threadIdx.y;
    const uint32_t z0 = blockIdx.x * TZ, y0 = blockIdx.y * TY;
    const uint32_t y = y0 + ty;
    const bool rowIn = y < g.Ny;
    const bool own_row = ty < TY;
    const size_t N = g.N, NyNz = g.NyNz, Nz = g.Nz;
    const uint32_t xs = blockIdx.z * g.xchunk;
    if (xs >= g.Nx) return;                             // whole block idle (uniform)
    const uint32_t xe = min(xs + g.xchunk, g.Nx);
    const uint32_t xl = xe < g.Nx ? xe : g.Nx - 1;      // last plane whose E this block computes
    const uint32_t ze = z0 + TZ;
    const bool extra = (lane == 31) && rowIn && (ze < g.Nz);
    uint32_t pmask = 0;
    if (PML) {
        const uint32_t lo[3] = {xs, y0, z0};
        const uint32_t hi[3] = {xe, y0 + TY, ze};
        pmask = region_mask(ps, lo, hi);
    }
    bool ok[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) ok[k] = rowIn && (z0 + lane + 32 * k < g.Nz);

    // H_old(x-1) (y and z components are enough for E; all three for H) of my cells
    float hp[CPT][3], hpe[2] = {0.f, 0.f};
    uint32_t matp[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) { hp[k][0] = hp[k][1] = hp[k][2] = 0.f; matp[k] = 0; }
    if (xs > 0) {
        const size_t bb = (size_t)(xs - 1) * NyNz + (size_t)y * Nz;
#pragma unroll
        for (int k = 0; k < CPT; ++k)
            if (ok[k])
#pragma unroll
                for (int n = 0; n < 3; ++n) hp[k][n] = __ldg(g.H0 + n * N + bb + z0 + lane + 32 * k);
        if (extra) { hpe[0] = __ldg(g.H0 + N + bb + ze); hpe[1] = __ldg(g.H0 + 2 * N + bb + ze); }
    }
    stage_plane<IDX, CPT, TY>(S, xs & 1, g, xs, y0, z0, lane, ty);
    cp_commit();

    for (uint32_t x = xs; x <= xl; ++x) {
        const int b = x & 1;
        // prefetch plane x+1 while this one is computed
        if (x < xl) stage_plane<IDX, CPT, TY>(S, b ^ 1, g, x + 1, y0, z0, lane, ty);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const size_t base = (size_t)x * NyNz + (size_t)y * Nz;
        const bool self = (x == 0);
        // ---- E_new(x) of my cells (+ the z halo cell on lane 31)
        float en[CPT][3];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int j = 1 + 32 * k + lane;
            const uint32_t z = z0 + lane + 32 * k;
            if (ok[k]) {
                const float hy_xm = self ? S.H[b][1][ty + 1][j] : hp[k][1];
                const float hz_xm = self ? S.H[b][2][ty + 1][j] : hp[k][2];
                e_cell<IDX, PML, CPT, TY>(S, b, ty, j, g, base + z, ps, pn, pmask, x, y, z, hy_xm, hz_xm,
                                          own_row && x < xe, en[k]);
            } else {
                en[k][0] = en[k][1] = en[k][2] = 0.f;
            }
#pragma unroll
            for (int n = 0; n < 3; ++n) S.En[b][n][ty][j] = en[k][n];
        }
        if (lane == 31) {
            float ee[3] = {0.f, 0.f, 0.f};
            if (extra) {
                const float hy_xm = self ? S.H[b][1][ty + 1][TZ + 1] : hpe[0];
                const float hz_xm = self ? S.H[b][2][ty + 1][TZ + 1] : hpe[1];
                e_cell<IDX, PML, CPT, TY>(S, b, ty, TZ + 1, g, base + ze, ps, pn, pmask, x, y, ze, hy_xm, hz_xm, false, ee);
                hpe[0] = S.H[b][1][ty + 1][TZ + 1];
                hpe[1] = S.H[b][2][ty + 1][TZ + 1];
            }
#pragma unroll
            for (int n = 0; n < 3; ++n) S.En[b][n][ty][TZ + 1] = ee[n];
        }
        if (own_row && x < xe) {
#pragma unroll
            for (int k = 0; k < CPT; ++k)
                if (ok[k])
#pragma unroll
                    for (int n = 0; n < 3; ++n) g.V1[n * N + base + z0 + lane + 32 * k] = en[k][n];
        }
        // H_old(x) and the material rows of my cells, needed for H(x) in the next iteration
        float hc[CPT][3];
        uint32_t matc[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int j = 1 + 32 * k + lane;
#pragma unroll
            for (int n = 0; n < 3; ++n) hc[k][n] = S.H[b][n][ty + 1][j];
            matc[k] = IDX ? S.M[b][ty][j] : 0u;
        }
        __syncthreads();
        // ---- H_new(x-1) of my cells
        if (own_row && x > xs) {
            const int pe = b ^ 1;
            const size_t bm1 = base - NyNz;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                if (!ok[k]) continue;
                const int j = 1 + 32 * k + lane;
                const uint32_t z = z0 + lane + 32 * k;
                const size_t cm = bm1 + z;
                if (g.defer && ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u)) continue;
                const bool core = (y + 1 < g.Ny) && (z + 1 < g.Nz);
                float cx = 0.f, cy = 0.f, cz = 0.f;
                float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (core) {
                    const float ex = S.En[pe][0][ty][j], ey = S.En[pe][1][ty][j], ez = S.En[pe][2][ty][j];
                    cx = curl4(ez, S.En[pe][2][ty + 1][j], ey, S.En[pe][1][ty][j + 1]);
                    cy = curl4(ex, S.En[pe][0][ty][j + 1], ez, en[k][2]);
                    cz = curl4(ey, en[k][1], ex, S.En[pe][0][ty + 1][j]);
                    coeffs_f<IDX>(g, cm, matp[k], 6, kk);
                }
                float hn[3];
                if (PML && pmask) {
#pragma unroll
                    for (int n = 0; n < 3; ++n)
                        hn[n] = pml_chain_pp<false>(ps, pn, pmask, x - 1, y, z, n, hp[k][n], core, kk[n], kk[3 + n],
                                                    n == 0 ? cx : (n == 1 ? cy : cz), true);
                } else if (core) {
                    hn[0] = upd(hp[k][0], kk[0], kk[3], cx);
                    hn[1] = upd(hp[k][1], kk[1], kk[4], cy);
                    hn[2] = upd(hp[k][2], kk[2], kk[5], cz);
                } else {
                    hn[0] = hp[k][0]; hn[1] = hp[k][1]; hn[2] = hp[k][2];
                }
#pragma unroll
                for (int n = 0; n < 3; ++n) g.H1[n * N + cm] = hn[n];
            }
        }
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            hp[k][0] = hc[k][0]; hp[k][1] = hc[k][1]; hp[k][2] = hc[k][2];
            matp[k] = matc[k];
        }
    }
    cp_wait<0>();
    // ---- H of the last plane x = Nx-1: no core update (loop bounds), UPML / pass-through only
    if (xe == g.Nx && own_row) {
        const size_t bl = (size_t)(g.Nx - 1) * NyNz + (size_t)y * Nz;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!ok[k]) continue;
            const uint32_t z = z0 + lane + 32 * k;
            const size_t cm = bl + z;
            if (g.defer && ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u)) continue;
#pragma unroll
            for (int n = 0; n < 3; ++n)
                g.H1[n * N + cm] = (PML && pmask) ? pml_chain_pp<false>(ps, pn, pmask, g.Nx - 1, y, z, n, hp[k][n], false, 0.f, 0.f, 0.f, true)
                                                  : hp[k][n];
        }
    }
}

// ---------------------------------------------------------------------------
// Register-blocked variant (default): no shared memory, no block barriers.
// A warp covers 32 consecutive z (lane l <-> z = z0 + l - 1, z0 = 30*tile):
// lanes 1..30 own their cells, lane 0 only supplies H(z0-1) and lane 31
// computes the E halo at z0+30; z neighbours travel by warp shuffles.  Each
// thread owns RY consecutive y rows, computes E on RY+1 rows (the extra row
// is the y halo) and keeps the previous plane's H_old and E_new in registers
// while it streams x.  Every warp is independent, so the SM keeps many
// planes' loads in flight.
//
// A warp-plane whose rows and lanes all lie inside the grid and which no UPML
// region reaches (most of a large grid) runs a branch-free body; the others
// run the general body with per-cell range checks and the UPML chain.  IT is
// the index type: 32-bit whenever 3*N fits, so that an access costs one
// multiply-add of address arithmetic.
// ---------------------------------------------------------------------------
constexpr int RZ = 30;          // owned z per warp

template <bool B>
struct PlaneKind { static constexpr bool value = B; };

template <bool IDX, bool PML, int RY, typename IT>
__global__ void __launch_bounds__(128) k_fused_reg(const FusedGrid g, const PmlSet ps, const PmlSet pn) {
    static_assert(32 % RY == 0, "the RY rows of a thread share one word of the row summary");
    const int lane = threadIdx.x;
    const uint32_t z0 = blockIdx.x * RZ;
    const int64_t zl = (int64_t)z0 + lane - 1;                  // this lane's z
    const uint32_t z = zl < 0 ? 0u : (uint32_t)zl;              // z = -1 reads z = 0 (self reference)
    const bool zin = zl < (int64_t)g.Nz;
    const bool own_z = lane >= 1 && lane <= RZ && zin;
    const uint32_t y0 = (blockIdx.y * blockDim.y + threadIdx.y) * RY;
    if (y0 >= g.Ny) return;                                      // whole warp idle (uniform per warp)
    const uint32_t xs = blockIdx.z * g.xchunk;
    if (xs >= g.Nx) return;
    const uint32_t xe = min(xs + g.xchunk, g.Nx);
    const uint32_t xl = xe < g.Nx ? xe : g.Nx - 1;
    const IT N = (IT)g.N, NyNz = (IT)g.NyNz, Nz = (IT)g.Nz;
    // rows y0..y0+RY and lanes z0-1..z0+30 all inside the grid, every owned H cell with its full curl
    const bool inner = (y0 + RY < g.Ny) && (z0 + RZ < g.Nz);
    // UPML: candidate regions of this warp's box, then per-axis masks (cell mask = AND)
    uint32_t zmask = 0, ymask[RY + 1];
#pragma unroll
    for (int r = 0; r <= RY; ++r) ymask[r] = 0;
    uint32_t cand = 0, zy = 0;
    if (PML) {
        const uint32_t lo[3] = {xs, y0, z0 > 0 ? z0 - 1 : 0};
        const uint32_t hi[3] = {xe, y0 + RY, z0 + RZ};
        cand = region_mask(ps, lo, hi);
        if (cand) {                                              // uniform per warp
            zmask = axis_mask(ps, cand, 2, z);
            uint32_t yu = 0;
#pragma unroll
            for (int r = 0; r <= RY; ++r) { ymask[r] = axis_mask(ps, cand, 1, y0 + r); yu |= ymask[r]; }
            zy = __reduce_or_sync(0xffffffffu, zmask) & yu;     // regions meeting the warp's (y, z) footprint
        }
    }
    bool rin[RY + 1];
#pragma unroll
    for (int r = 0; r <= RY; ++r) rin[r] = (y0 + r < g.Ny) && zin;
    const uint32_t ym = y0 > 0 ? y0 - 1 : y0;                    // y = -1 reads y = 0 (self reference)
    const IT rowm = (IT)ym * Nz + z;                             // offsets inside a plane: the y-1 halo row
    const IT row0 = (IT)y0 * Nz + z;                             //   and row y0
    const uint32_t rw = (g.Ny + 31) / 32;                        // words per plane of the row summary

    float hp[RY + 1][3];     // H_old(x-1) rows y0..y0+RY
    float ep[RY + 1][3];     // E_new(x-1) rows y0..y0+RY
    uint32_t mp[RY];         // material rows of plane x-1 (owned rows)
#pragma unroll
    for (int r = 0; r <= RY; ++r) { hp[r][0] = hp[r][1] = hp[r][2] = 0.f; ep[r][0] = ep[r][1] = ep[r][2] = 0.f; }
#pragma unroll
    for (int r = 0; r < RY; ++r) mp[r] = 0;
    {   // H_old(xs-1); at xs = 0 the x-1 neighbour is plane 0 itself (self reference)
        const float* H = g.H0 + (IT)(xs > 0 ? xs - 1 : 0) * NyNz;
#pragma unroll
        for (int r = 0; r <= RY; ++r)
            if (rin[r]) {
                const IT c = row0 + (IT)r * Nz;
                hp[r][1] = __ldg(H + (c + N));
                hp[r][2] = __ldg(H + (c + 2 * N));
            }
    }

    // One plane: E_new(x) on rows y0..y0+RY (row RY is the y halo), then H_new(x-1) on the owned rows.
    auto plane = [&](uint32_t x, uint32_t xmask, uint32_t xmask_p, auto kind) {
        constexpr bool FAST = decltype(kind)::value;
        const IT px = (IT)x * NyNz;
        const float* H = g.H0 + px;
        const float* V = g.V0 + px;
        const uint32_t* M = g.mat + px;
        float* V1 = g.V1 + px;
        // ---- loads of plane x: H rows y0-1..y0+RY, E_old and material rows y0..y0+RY
        float h[RY + 2][3], eo[RY + 1][3];
        uint32_t m[RY + 1];
        h[0][0] = (FAST || zin) ? __ldg(H + rowm) : 0.f;
        h[0][1] = 0.f;
        h[0][2] = (FAST || zin) ? __ldg(H + (rowm + 2 * N)) : 0.f;
#pragma unroll
        for (int r = 0; r <= RY; ++r) {
            const IT c = row0 + (IT)r * Nz;
            const bool ok = FAST || rin[r];
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                h[r + 1][n] = ok ? __ldg(H + (c + n * N)) : 0.f;
                eo[r][n] = ok ? __ldg(V + (c + n * N)) : 0.f;
            }
            m[r] = (IDX && ok) ? __ldg(M + c) : 0u;
        }
        // ---- E_new(x)
        float en[RY + 1][3];
        const bool store_e = x < xe;
#pragma unroll
        for (int r = 0; r <= RY; ++r) {
            const IT c = row0 + (IT)r * Nz;
            const float hx = h[r + 1][0], hy = h[r + 1][1], hz = h[r + 1][2];
            const float hy_zm = __shfl_up_sync(0xffffffffu, hy, 1);
            const float hx_zm = __shfl_up_sync(0xffffffffu, hx, 1);
            const float cx = curl4(hz, h[r][2], hy, hy_zm);
            const float cy = curl4(hx, hx_zm, hz, hp[r][2]);
            const float cz = curl4(hy, hp[r][1], hx, h[r][0]);
            en[r][0] = en[r][1] = en[r][2] = 0.f;
            if (FAST || (lane >= 1 && rin[r])) {
                float kk[6];
                coeffs_f<IDX>(g, (size_t)(px + c), m[r], 0, kk);
                const uint32_t cmask = FAST ? 0u : (zmask & ymask[r] & xmask);
                if (PML && cmask) {
                    const bool wr = own_z && r < RY && store_e;
                    en[r][0] = pml_cell<true>(ps, pn, cmask, x, y0 + r, z, 0, eo[r][0], true, kk[0], kk[3], cx, wr);
                    en[r][1] = pml_cell<true>(ps, pn, cmask, x, y0 + r, z, 1, eo[r][1], true, kk[1], kk[4], cy, wr);
                    en[r][2] = pml_cell<true>(ps, pn, cmask, x, y0 + r, z, 2, eo[r][2], true, kk[2], kk[5], cz, wr);
                } else {
                    en[r][0] = upd(eo[r][0], kk[0], kk[3], cx);
                    en[r][1] = upd(eo[r][1], kk[1], kk[4], cy);
                    en[r][2] = upd(eo[r][2], kk[2], kk[5], cz);
                }
                if (own_z && r < RY && store_e) {
                    V1[c] = en[r][0];
                    V1[c + N] = en[r][1];
                    V1[c + 2 * N] = en[r][2];
                }
            }
        }
        // ---- H_new(x-1) on owned rows and lanes
        if (x > xs) {
            const IT pm = px - NyNz;
            float* H1 = g.H1 + pm;
            uint32_t dbits = 0;                                  // rows whose cell is deferred
            if (g.defer_rows) {
                const uint32_t w = __ldg(g.defer_rows + (size_t)(x - 1) * rw + (y0 >> 5));
                const uint32_t rows = (w >> (y0 & 31)) & ((1u << RY) - 1u);
                if (rows && own_z) {
#pragma unroll
                    for (int r = 0; r < RY; ++r)
                        if (((rows >> r) & 1u) && rin[r]) {
                            const IT cm = pm + row0 + (IT)r * Nz;
                            dbits |= ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u) << r;
                        }
                }
            }
#pragma unroll
            for (int r = 0; r < RY; ++r) {
                const IT c = row0 + (IT)r * Nz;
                const float ey_zp = __shfl_down_sync(0xffffffffu, ep[r][1], 1);
                const float ex_zp = __shfl_down_sync(0xffffffffu, ep[r][0], 1);
                if (FAST) {
                    const float cx = curl4(ep[r][2], ep[r + 1][2], ep[r][1], ey_zp);
                    const float cy = curl4(ep[r][0], ex_zp, ep[r][2], en[r][2]);
                    const float cz = curl4(ep[r][1], en[r][1], ep[r][0], ep[r + 1][0]);
                    float kk[6];
                    coeffs_f<IDX>(g, (size_t)(pm + c), mp[r], 6, kk);
                    const float h0 = upd(hp[r][0], kk[0], kk[3], cx);
                    const float h1 = upd(hp[r][1], kk[1], kk[4], cy);
                    const float h2 = upd(hp[r][2], kk[2], kk[5], cz);
                    if (own_z && !((dbits >> r) & 1u)) {
                        H1[c] = h0;
                        H1[c + N] = h1;
                        H1[c + 2 * N] = h2;
                    }
                    continue;
                }
                if (!own_z || !rin[r] || ((dbits >> r) & 1u)) continue;
                const uint32_t y = y0 + r;
                const bool core = (y + 1 < g.Ny) && (z + 1 < g.Nz);
                float cx = 0.f, cy = 0.f, cz = 0.f;
                float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (core) {
                    cx = curl4(ep[r][2], ep[r + 1][2], ep[r][1], ey_zp);
                    cy = curl4(ep[r][0], ex_zp, ep[r][2], en[r][2]);
                    cz = curl4(ep[r][1], en[r][1], ep[r][0], ep[r + 1][0]);
                    coeffs_f<IDX>(g, (size_t)(pm + c), mp[r], 6, kk);
                }
                float hn[3];
                const uint32_t cmask = zmask & ymask[r] & xmask_p;
                if (PML && cmask) {
#pragma unroll
                    for (int n = 0; n < 3; ++n)
                        hn[n] = pml_cell<false>(ps, pn, cmask, x - 1, y, z, n, hp[r][n], core, kk[n], kk[3 + n],
                                                n == 0 ? cx : (n == 1 ? cy : cz), true);
                } else if (core) {
                    hn[0] = upd(hp[r][0], kk[0], kk[3], cx);
                    hn[1] = upd(hp[r][1], kk[1], kk[4], cy);
                    hn[2] = upd(hp[r][2], kk[2], kk[5], cz);
                } else {
                    hn[0] = hp[r][0]; hn[1] = hp[r][1]; hn[2] = hp[r][2];
                }
                H1[c] = hn[0];
                H1[c + N] = hn[1];
                H1[c + 2 * N] = hn[2];
            }
        }
        // ---- rotate
#pragma unroll
        for (int r = 0; r <= RY; ++r) {
            hp[r][0] = h[r + 1][0]; hp[r][1] = h[r + 1][1]; hp[r][2] = h[r + 1][2];
            ep[r][0] = en[r][0]; ep[r][1] = en[r][1]; ep[r][2] = en[r][2];
        }
#pragma unroll
        for (int r = 0; r < RY; ++r) mp[r] = m[r];
    };

    uint32_t xmask_p = 0;    // UPML regions containing plane x-1
    for (uint32_t x = xs; x <= xl; ++x) {
        const uint32_t xmask = cand ? axis_mask(ps, cand, 0, x) : 0u;
        if (inner && !(zy & (xmask | xmask_p))) plane(x, xmask, xmask_p, PlaneKind<true>{});
        else plane(x, xmask, xmask_p, PlaneKind<false>{});
        xmask_p = xmask;
    }
    // ---- H of the last plane x = Nx-1: no core update, UPML / pass-through only
    if (xe == g.Nx && own_z) {
        const IT pl = (IT)(g.Nx - 1) * NyNz;
#pragma unroll
        for (int r = 0; r < RY; ++r) {
            if (!rin[r]) continue;
            const IT cm = pl + row0 + (IT)r * Nz;
            if (g.defer && ((__ldg(g.defer + (cm >> 5)) >> (cm & 31)) & 1u)) continue;
            const uint32_t cmask = zmask & ymask[r] & xmask_p;
#pragma unroll
            for (int n = 0; n < 3; ++n)
                g.H1[cm + n * N] = (PML && cmask) ? pml_cell<false>(ps, pn, cmask, g.Nx - 1, y0 + r, z, n, hp[r][n], false, 0.f, 0.f, 0.f, true)
                                                  : hp[r][n];
        }
    }
}

// H update of the deferred cells, after the E-side sparse operations:
// reads the final E_new, H_old, writes H_new (with UPML), one thread per cell.
template <bool IDX, bool PML>
__device__ __forceinline__ void deferred_h_body(const FusedGrid& g, const PmlSet& ps, const PmlSet& pn, const uint32_t* cells,
                                                uint32_t n, uint32_t i) {
    if (i >= n) return;
    const uint32_t c = cells[i];
    const uint32_t N = (uint32_t)g.N, NyNz = (uint32_t)g.NyNz, Nz = g.Nz;   // 3*N < 2^32
    const uint32_t x = c / NyNz, rem = c - x * NyNz, y = rem / Nz, z = rem - y * Nz;
    const bool core = (x + 1 < g.Nx) && (y + 1 < g.Ny) && (z + 1 < g.Nz);
    const float* V = g.V1;
    float ho[3], ev[9];
    ho[0] = g.H0[c]; ho[1] = g.H0[N + c]; ho[2] = g.H0[2 * N + c];
    uint32_t m = 0;
    if (core) {
        ev[0] = V[c]; ev[1] = V[N + c]; ev[2] = V[2 * N + c];
        ev[3] = V[2 * N + c + Nz]; ev[4] = V[N + c + 1]; ev[5] = V[c + 1];
        ev[6] = V[2 * N + c + NyNz]; ev[7] = V[N + c + NyNz]; ev[8] = V[c + Nz];
        m = IDX ? __ldg(g.mat + c) : 0u;
    }
    float cv[3] = {0.f, 0.f, 0.f};
    float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (core) {
        cv[0] = curl4(ev[2], ev[3], ev[1], ev[4]);
        cv[1] = curl4(ev[0], ev[5], ev[2], ev[6]);
        cv[2] = curl4(ev[1], ev[7], ev[0], ev[8]);
        coeffs_f<IDX>(g, c, m, 6, kk);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        float hn;
        if (PML) hn = pml_chain_pp<false>(ps, pn, ps.count >= 32 ? ~0u : ((1u << ps.count) - 1u), x, y, z, q, ho[q], core,
                                          kk[q], kk[3 + q], cv[q], true);
        else hn = core ? upd(ho[q], kk[q], kk[3 + q], cv[q]) : ho[q];
        g.H1[q * N + c] = hn;
    }
}
template <bool IDX, bool PML>
__global__ void __launch_bounds__(256) k_deferred_h(const FusedGrid g, const PmlSet ps, const PmlSet pn, const uint32_t* cells,
                                                    uint32_t n) {
    deferred_h_body<IDX, PML>(g, ps, pn, cells, n, blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace efs
