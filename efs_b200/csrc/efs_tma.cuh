// efs_tma.cuh — TMA-fed single-pass E+H update (the engine's default core path
// when Nz is a multiple of 4).
//
// A CTA owns a tile of TT_Y rows (y) x TT_Z columns (z) and streams the
// x-planes of one x-chunk through a TT_S-stage shared-memory pipeline: one
// thread issues, per plane, three cp.async.bulk.tensor loads (H with its
// low halos, E_old and the material rows, each a box of the tile plus halos)
// completing on the stage's mbarrier, TT_S-1 planes ahead of the plane being
// computed.  The loads run on the copy engine, so the bytes in flight per SM
// do not depend on how many warps are resident.
//
// At plane x (local index k = x - xs) the CTA
//   1. computes E_new(x) on the tile plus its high halo row and column from
//      the staged H and E_old (H_old(x-1) of its cells it keeps in registers),
//      stores the owned cells and keeps every E_new(x) in plane buffer k % 3,
//   2. one barrier, after which the stage is refilled with plane x+TT_S,
//   3. computes H_new(x-1) of the owned cells from E_new(x-1) (plane buffer
//      (k-1) % 3 and registers) and E_new(x) (registers).
// Three E_new plane buffers make step 3 of plane x and step 1 of plane x+1
// independent, so one barrier per plane suffices.
//
// Boundaries follow the reference's index-0 self reference: the x-1, y-1 and
// z-1 neighbours of index 0 are the cell itself (the TMA zero fill outside
// the grid is never read as a field value).  H cells whose curl reads E values
// rewritten by sparse post-update operations are written here provisionally
// and rewritten afterwards by k_deferred_h, which recomputes them from H_old.
//
// Every mbarrier wait is bounded (about one second of %globaltimer); a wait
// that runs out sets bit 0 of *g.status, the CTA drains its loads in flight
// (bounded again) and returns, and the host reports EFS_ERR_TIMEOUT.
#pragma once
#include "efs_fused.cuh"
#include <cuda.h>

namespace efs {

constexpr int TT_Z = 64;                 // owned z per tile
constexpr int TT_Y = 8;                  // owned y per tile (one warp per row)
constexpr int TT_S = 4;                  // pipeline stages
constexpr int TT_HZ = TT_Z + 8;          // H box: z0-4 .. z0+TT_Z+3 (x coordinate kept 16-byte aligned)
constexpr int TT_HY = TT_Y + 2;          // H box: y0-1 .. y0+TT_Y
constexpr int TT_EZ = TT_Z + 4;          // E_old / material box: z0 .. z0+TT_Z+3
constexpr int TT_EY = TT_Y + 1;          // E_old / material box: y0 .. y0+TT_Y
constexpr int TT_THREADS = 32 * (TT_Y + 1);   // warps 0..TT_Y-1: owned rows; warp TT_Y: halo row + halo column
constexpr uint32_t TT_H_BYTES = 3u * TT_HY * TT_HZ * 4u;
constexpr uint32_t TT_E_BYTES = 3u * TT_EY * TT_EZ * 4u;
constexpr uint32_t TT_M_BYTES = 1u * TT_EY * TT_EZ * 4u;
static_assert(TT_H_BYTES + TT_E_BYTES + TT_M_BYTES < (1u << 20), "mbarrier transaction count");

struct TmaStage {
    alignas(128) float H[3][TT_HY][TT_HZ];
    alignas(128) float E[3][TT_EY][TT_EZ];
    alignas(128) uint32_t M[TT_EY][TT_EZ];
};
struct TmaSmem {
    TmaStage st[TT_S];
    float En[3][3][TT_EY][TT_EZ];        // E_new of planes k % 3, tile + halo row/column
    alignas(8) unsigned long long full[TT_S];
};
constexpr size_t TT_SMEM_BYTES = sizeof(TmaSmem) + 128;   // + slack to align the base to 128 B

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for completion of the phase with the given parity; false after ~limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// Issue the loads of plane x into stage s (one thread).
template <bool IDX>
__device__ __forceinline__ void tt_issue(TmaSmem& S, int s, const CUtensorMap* tmH, const CUtensorMap* tmE,
                                         const CUtensorMap* tmM, int x, int y0, int z0) {
    const uint32_t bar = smem_u32(&S.full[s]);
    const uint32_t bytes = TT_H_BYTES + TT_E_BYTES + (IDX ? TT_M_BYTES : 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic reads of the stage before the refill
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    tma_load_4d(&S.st[s].H[0][0][0], tmH, z0 - 4, y0 - 1, x, 0, bar);
    tma_load_4d(&S.st[s].E[0][0][0], tmE, z0, y0, x, 0, bar);
    if (IDX) tma_load_3d(&S.st[s].M[0][0], tmM, z0, y0, x, bar);
}

template <bool IDX, bool PML>
__global__ void __launch_bounds__(TT_THREADS, 2)
k_fused_tma(const __grid_constant__ CUtensorMap tmH, const __grid_constant__ CUtensorMap tmE,
            const __grid_constant__ CUtensorMap tmM, const FusedGrid g, const PmlSet ps, const PmlSet pn) {
    extern __shared__ unsigned char smem_raw[];
    TmaSmem& S = *reinterpret_cast<TmaSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t z0 = blockIdx.x * TT_Z, y0 = blockIdx.y * TT_Y;
    const uint32_t xs = blockIdx.z * g.xchunk;
    if (xs >= g.Nx) return;                                  // uniform per CTA
    const uint32_t xe = min(xs + g.xchunk, g.Nx);
    const uint32_t xl = xe < g.Nx ? xe : g.Nx - 1;           // last plane whose E this CTA computes
    const int nk = (int)(xl - xs) + 1;                       // planes streamed
    const size_t N = g.N, NyNz = g.NyNz, Nz = g.Nz;
    constexpr uint64_t WAIT_NS = 1000000000ull;

    // ---- E cells of this thread: slots 0, 1 = (row, lane / lane+32); slot 2 = halo column (warp TT_Y, lanes 0..TT_Y)
    const int row = warp;                                    // TT_Y for the halo-row warp
    const bool has2 = (warp == TT_Y) && (lane <= TT_Y);
    int sr[3], sc[3];
    sr[0] = row; sc[0] = lane;
    sr[1] = row; sc[1] = lane + 32;
    sr[2] = has2 ? lane : 0; sc[2] = TT_Z;
    const bool own = warp < TT_Y;                            // slots 0, 1 are owned cells (E stored, H updated)
    uint32_t sy[3], sz[3];
    bool sin[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        sy[s] = y0 + sr[s]; sz[s] = z0 + sc[s];
        sin[s] = sy[s] < g.Ny && sz[s] < g.Nz && (s < 2 || has2);
    }
    // UPML: regions meeting the CTA's box, then the (y, z) part of each cell's mask
    uint32_t cand = 0, yzm[3] = {0u, 0u, 0u};
    if (PML) {
        const uint32_t lo[3] = {xs, y0, z0};
        const uint32_t hi[3] = {xe, y0 + TT_Y, z0 + TT_Z};
        cand = region_mask(ps, lo, hi);
        if (cand)
#pragma unroll
            for (int s = 0; s < 3; ++s) yzm[s] = axis_mask(ps, cand, 1, sy[s]) & axis_mask(ps, cand, 2, sz[s]);
    }

    // ---- pipeline set-up
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < TT_S; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.full[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;                                          // planes issued (thread 0's count)
    if (threadIdx.x == 0)
        for (; issued < TT_S && issued < nk; ++issued)
            tt_issue<IDX>(S, issued, &tmH, &tmE, &tmM, (int)(xs + issued), (int)y0, (int)z0);

    // H_old(xs-1) of the E cells (y, z components); at xs = 0 the x-1 neighbour is plane 0 itself
    float hp[3][3];
    {
        const size_t pb = (size_t)(xs > 0 ? xs - 1 : 0) * NyNz;
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            hp[s][0] = 0.f;
            const size_t c = pb + (size_t)sy[s] * Nz + sz[s];
            hp[s][1] = sin[s] ? __ldg(g.H0 + N + c) : 0.f;
            hp[s][2] = sin[s] ? __ldg(g.H0 + 2 * N + c) : 0.f;
        }
    }
    float ep[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};      // E_new(x-1) of the owned cells
    uint32_t mp[2] = {0u, 0u};                                // material of the owned cells at x-1
    uint32_t xmask_p = 0;
    bool timed_out = false;
    int k = 0;

    for (; k < nk; ++k) {
        const uint32_t x = xs + k;
        const int s = k % TT_S;
        const TmaStage& T = S.st[s];
        const bool ok = mbar_wait_bounded(smem_u32(&S.full[s]), (uint32_t)(k / TT_S) & 1u, WAIT_NS);
        const uint32_t xmask = cand ? axis_mask(ps, cand, 0, x) : 0u;
        float (*En)[TT_EY][TT_EZ] = S.En[k % 3];
        const size_t px = (size_t)x * NyNz;
        float en[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float hc[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        uint32_t mc[2] = {0u, 0u};
        if (ok) {
            // ---- E_new(x) of the thread's cells (cells outside the grid keep E_new = 0)
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q == 2 && !has2) continue;
                const int r = sr[q], c = sc[q];
                if (!sin[q]) {
                    En[0][r][c] = 0.f; En[1][r][c] = 0.f; En[2][r][c] = 0.f;
                    continue;
                }
                const int hr = r + 1, hcol = c + 4;                        // H box indices of the cell
                const int hrm = sy[q] == 0 ? hr : hr - 1;                  // y-1 (self at y = 0)
                const int hcm = sz[q] == 0 ? hcol : hcol - 1;              // z-1 (self at z = 0)
                const float hx = T.H[0][hr][hcol], hy = T.H[1][hr][hcol], hz = T.H[2][hr][hcol];
                const float cx = curl4(hz, T.H[2][hrm][hcol], hy, T.H[1][hr][hcm]);
                const float cy = curl4(hx, T.H[0][hr][hcm], hz, hp[q][2]);
                const float cz = curl4(hy, hp[q][1], hx, T.H[0][hrm][hcol]);
                const uint32_t m = IDX ? T.M[r][c] : 0u;
                if (q < 2) mc[q] = m;
                hc[q][0] = hx; hc[q][1] = hy; hc[q][2] = hz;
                float kk[6];
                coeffs_f<IDX>(g, px + (size_t)sy[q] * Nz + sz[q], m, 0, kk);
                const float e0 = T.E[0][r][c], e1 = T.E[1][r][c], e2 = T.E[2][r][c];
                const uint32_t cmask = PML ? (yzm[q] & xmask) : 0u;
                if (PML && cmask) {
                    const bool wr = own && q < 2 && x < xe;
                    en[q][0] = pml_cell<true>(ps, pn, cmask, x, sy[q], sz[q], 0, e0, true, kk[0], kk[3], cx, wr);
                    en[q][1] = pml_cell<true>(ps, pn, cmask, x, sy[q], sz[q], 1, e1, true, kk[1], kk[4], cy, wr);
                    en[q][2] = pml_cell<true>(ps, pn, cmask, x, sy[q], sz[q], 2, e2, true, kk[2], kk[5], cz, wr);
                } else {
                    en[q][0] = upd(e0, kk[0], kk[3], cx);
                    en[q][1] = upd(e1, kk[1], kk[4], cy);
                    en[q][2] = upd(e2, kk[2], kk[5], cz);
                }
                En[0][r][c] = en[q][0]; En[1][r][c] = en[q][1]; En[2][r][c] = en[q][2];
                if (own && q < 2 && x < xe) {
                    const size_t cell = px + (size_t)sy[q] * Nz + sz[q];
                    g.V1[cell] = en[q][0];
                    g.V1[N + cell] = en[q][1];
                    g.V1[2 * N + cell] = en[q][2];
                }
            }
        }
        // every read of stage s and every write of En[k % 3] done; agree on a timeout
        timed_out = __syncthreads_or(!ok) != 0;
        if (timed_out) break;
        if (threadIdx.x == 0 && issued < nk) {
            tt_issue<IDX>(S, s, &tmH, &tmE, &tmM, (int)(xs + issued), (int)y0, (int)z0);
            ++issued;
        }
        // ---- H_new(x-1) of the owned cells
        if (k > 0 && own) {
            const float (*Ep)[TT_EY][TT_EZ] = S.En[(k + 2) % 3];
            const size_t pm = px - NyNz;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!sin[q]) continue;
                const int r = sr[q], c = sc[q];
                const bool core = (sy[q] + 1 < g.Ny) && (sz[q] + 1 < g.Nz);
                const float ex = ep[q][0], ey = ep[q][1], ez = ep[q][2];
                const float cx = curl4(ez, Ep[2][r + 1][c], ey, Ep[1][r][c + 1]);
                const float cy = curl4(ex, Ep[0][r][c + 1], ez, en[q][2]);
                const float cz = curl4(ey, en[q][1], ex, Ep[0][r + 1][c]);
                const size_t cell = pm + (size_t)sy[q] * Nz + sz[q];
                float kk[6];
                coeffs_f<IDX>(g, cell, mp[q], 6, kk);
                float hn[3];
                const uint32_t cmask = PML ? (yzm[q] & xmask_p) : 0u;
                if (PML && cmask) {
#pragma unroll
                    for (int n = 0; n < 3; ++n)
                        hn[n] = pml_cell<false>(ps, pn, cmask, x - 1, sy[q], sz[q], n, hp[q][n], core, kk[n], kk[3 + n],
                                                n == 0 ? cx : (n == 1 ? cy : cz), true);
                } else {
                    hn[0] = core ? upd(hp[q][0], kk[0], kk[3], cx) : hp[q][0];
                    hn[1] = core ? upd(hp[q][1], kk[1], kk[4], cy) : hp[q][1];
                    hn[2] = core ? upd(hp[q][2], kk[2], kk[5], cz) : hp[q][2];
                }
                g.H1[cell] = hn[0];
                g.H1[N + cell] = hn[1];
                g.H1[2 * N + cell] = hn[2];
            }
        }
        // ---- rotate
#pragma unroll
        for (int q = 0; q < 3; ++q) { hp[q][0] = hc[q][0]; hp[q][1] = hc[q][1]; hp[q][2] = hc[q][2]; }
#pragma unroll
        for (int q = 0; q < 2; ++q) { ep[q][0] = en[q][0]; ep[q][1] = en[q][1]; ep[q][2] = en[q][2]; mp[q] = mc[q]; }
        xmask_p = xmask;
    }

    if (timed_out) {
        if (threadIdx.x == 0) {
            atomicOr(g.status, 1u);
            for (int j = k; j < issued; ++j)                       // drain the loads still in flight
                (void)mbar_wait_bounded(smem_u32(&S.full[j % TT_S]), (uint32_t)(j / TT_S) & 1u, WAIT_NS);
        }
        return;
    }
    // ---- H of the last plane x = Nx-1: no core update, UPML / pass-through only
    if (xe == g.Nx && own) {
        const size_t pl = (size_t)(g.Nx - 1) * NyNz;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!sin[q]) continue;
            const size_t cell = pl + (size_t)sy[q] * Nz + sz[q];
            const uint32_t cmask = PML ? (yzm[q] & xmask_p) : 0u;
#pragma unroll
            for (int n = 0; n < 3; ++n)
                g.H1[n * N + cell] = (PML && cmask)
                    ? pml_cell<false>(ps, pn, cmask, g.Nx - 1, sy[q], sz[q], n, hp[q][n], false, 0.f, 0.f, 0.f, true)
                    : hp[q][n];
        }
    }
}

}  // namespace efs
