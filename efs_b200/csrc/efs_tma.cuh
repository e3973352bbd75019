// efs_tma.cuh — TMA-fed single-pass E+H update (the engine's core path).
//
// A CTA owns a tile of TT_Y rows (y) x TT_Z columns (z) and streams the
// x-planes of one x-chunk through a TT_S-stage shared-memory pipeline: one
// thread issues, per plane, three cp.async.bulk.tensor loads (H with its
// low halos, E_old and the material rows, each a box of the tile plus halos)
// completing on the stage's mbarrier, TT_S-1 planes ahead of the plane being
// computed.  The loads run on the copy engine, so the bytes in flight per SM
// do not depend on how many warps are resident.  The tensor maps span the
// grid's Nz x Ny x Nx cells over the padded device layout (row pitch Pz, a
// multiple of 4 floats, so every global stride is a multiple of 16 bytes):
// box columns at z >= Nz lie outside the map and are zero-filled, so pad
// cells are never loaded.
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
// UPML cells are updated by k_pml_e (E, before this kernel: its E_new is
// staged here in place of E_old and adopted as is) and k_pml_h (H, after it);
// this kernel only needs to know which cells they are.
//
// Boundaries follow the reference's index-0 self reference: the x-1, y-1 and
// z-1 neighbours of index 0 are the cell itself (the TMA zero fill outside
// the grid is never read as a field value).  H cells whose curl reads E values
// rewritten by sparse post-update operations are written here provisionally
// and rewritten afterwards by k_deferred_h, which recomputes them from H_old.
//
// Every mbarrier wait is bounded (g.wait_ns of %globaltimer, about one
// second); a wait that runs out sets bit 0 of *g.status, the CTA drains its
// loads in flight (bounded again) and returns, and the host reports
// EFS_ERR_TIMEOUT.  A diagnostic knob (g.skip_plane) leaves one plane's loads
// unissued so that tests can make a wait run out without any fault.
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
    alignas(128) float D[2][2][TF_DY];   // TFSF face corrections of the plane: [face][Ex, Ey][row]
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

// Issue the loads of plane x into stage s (one thread); dbytes > 0: also the
// plane's TFSF face corrections (rows y0 .. y0+TF_DY-1 of every face).
template <bool IDX>
__device__ __forceinline__ void tt_issue(TmaSmem& S, int s, const CUtensorMap* tmH, const CUtensorMap* tmE,
                                         const CUtensorMap* tmM, const CUtensorMap* tmD, uint32_t dbytes, int x, int y0,
                                         int z0) {
    const uint32_t bar = smem_u32(&S.full[s]);
    const uint32_t bytes = TT_H_BYTES + TT_E_BYTES + (IDX ? TT_M_BYTES : 0u) + dbytes;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic reads of the stage before the refill
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    tma_load_4d(&S.st[s].H[0][0][0], tmH, z0 - 4, y0 - 1, x, 0, bar);
    tma_load_4d(&S.st[s].E[0][0][0], tmE, z0, y0, x, 0, bar);
    if (IDX) tma_load_3d(&S.st[s].M[0][0], tmM, z0, y0, x, bar);
    if (dbytes) tma_load_4d(&S.st[s].D[0][0][0], tmD, y0, x, 0, 0, bar);
}

// The CTA's shared working area: 128-byte aligned, addressed from the shared
// array itself so that every access compiles to a shared-space load or store.
__device__ __forceinline__ TmaSmem& tt_smem() {
    extern __shared__ __align__(128) unsigned char tt_smem_raw[];
    return *reinterpret_cast<TmaSmem*>(tt_smem_raw + ((128u - (smem_u32(tt_smem_raw) & 127u)) & 127u));
}

// mbarrier set-up, once per CTA (all threads call it).
__device__ __forceinline__ void tt_init(TmaSmem& S) {
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < TT_S; ++s) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.full[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// One tile of the streaming update: the x-chunk starting at xs of the tile at
// (y0, z0), called by every thread of the CTA.  K counts the planes the CTA
// consumed before this tile (it selects the stage, the mbarrier phase and the
// E_new buffer, so one CTA can run tiles back to back); every load the tile
// issues is consumed before it returns.  Returns false after a wait ran out.
// TF: the tile may meet a TFSF face corrected here (tested per tile; the single
// engine runs tiles that meet none through the instantiation without that code).
template <bool IDX, bool PML, bool TF>
__device__ __forceinline__ bool tma_tile_body(TmaSmem& S, const CUtensorMap* tmH, const CUtensorMap* tmE, const CUtensorMap* tmM,
                                              const CUtensorMap* tmD, const FusedGrid& g, const PmlSet& ps, uint32_t xs,
                                              uint32_t y0, uint32_t z0, uint32_t& K) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t xe = min(xs + g.xchunk, g.Nx);
    const uint32_t xl = xe < g.Nx ? xe : g.Nx - 1;           // last plane whose E this CTA computes
    const int nk = (int)(xl - xs) + 1;                       // planes streamed
    const uint32_t N = (uint32_t)g.N, NyNz = (uint32_t)g.NyNz, Ny = g.Ny, Nz = g.Nz, Pz = g.Pz;   // 3*N < 2^32
    const uint64_t WAIT_NS = g.wait_ns;
    constexpr int HPL = TT_HY * TT_HZ;                       // one component of a staged H box
    constexpr int EPL = TT_EY * TT_EZ;                       // one component of a staged E box / E_new plane

    // ---- E cells of this thread: slots 0, 1 = (row, lane / lane+32); slot 2 = halo column (warp TT_Y, lanes 0..TT_Y)
    const bool own = warp < TT_Y;                            // slots 0, 1 are owned cells (E stored, H updated)
    const bool has2 = (warp == TT_Y) && (lane <= TT_Y);
    const int sr[3] = {warp, warp, has2 ? lane : 0};
    const int sc[3] = {lane, lane + 32, TT_Z};
    uint32_t sy[3], sz[3], off[3];
    int hi[3], ei[3], dym[3], dzm[3];
    bool sin[3], core[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        sy[q] = y0 + sr[q]; sz[q] = z0 + sc[q];
        sin[q] = sy[q] < Ny && sz[q] < Nz && (q < 2 || has2);
        core[q] = sy[q] + 1 < Ny && sz[q] + 1 < Nz;
        off[q] = sy[q] * Pz + sz[q];                         // offset inside a plane (used when sin)
        hi[q] = (sr[q] + 1) * TT_HZ + sc[q] + 4;             // index in a staged H component
        ei[q] = sr[q] * TT_EZ + sc[q];                       // index in a staged E component / E_new plane
        dym[q] = sy[q] == 0 ? 0 : TT_HZ;                     // y-1 neighbour (self at y = 0)
        dzm[q] = sz[q] == 0 ? 0 : 1;                         // z-1 neighbour (self at z = 0)
    }
    // UPML: regions meeting the CTA's box, then the (y, z) part of each cell's mask
    uint32_t cand = 0, yzm[3] = {0u, 0u, 0u};
    if (PML) {
        const uint32_t lo[3] = {xs, y0, z0};
        const uint32_t hb[3] = {xe, y0 + TT_Y, z0 + TT_Z};
        cand = region_mask(ps, lo, hb);
        if (cand)
#pragma unroll
            for (int q = 0; q < 3; ++q) yzm[q] = axis_mask(ps, cand, 1, sy[q]) & axis_mask(ps, cand, 2, sz[q]);
    }

    bool tf_tile = false;
    if (TF)
        for (uint32_t f = 0; f < g.tf.n; ++f) tf_tile |= g.tf.z[f] >= z0 && g.tf.z[f] <= z0 + TT_Z;
    const uint32_t dbytes = tf_tile ? g.tf.n * 2u * TF_DY * 4u : 0u;
    int tfq[3] = {-1, -1, -1};
    if (tf_tile)
#pragma unroll
        for (int q = 0; q < 3; ++q) tfq[q] = sin[q] ? tf_face(g.tf, sz[q]) : -1;

    // ---- first planes into the pipeline
    int issued = 0;                                          // planes issued (thread 0's count)
    if (threadIdx.x == 0)
        for (; issued < TT_S && issued < nk; ++issued)
            if (xs + issued != g.skip_plane)
                tt_issue<IDX>(S, (int)((K + issued) % TT_S), tmH, tmE, tmM, tmD, dbytes, (int)(xs + issued), (int)y0, (int)z0);

    // H_old(xs-1) of the E cells (y, z components); at xs = 0 the x-1 neighbour is plane 0 itself
    float hp[3][3];
    {
        const float* H = g.H0 + (size_t)(xs > 0 ? xs - 1 : 0) * NyNz;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            hp[q][0] = 0.f;
            hp[q][1] = sin[q] ? __ldg(H + (off[q] + N)) : 0.f;
            hp[q][2] = sin[q] ? __ldg(H + (off[q] + 2 * N)) : 0.f;
        }
    }
    float ep[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};      // E_new(x-1) of the owned cells
    uint32_t mp[2] = {0u, 0u};                                // material of the owned cells at x-1
    uint32_t xmask_p = 0;
    bool timed_out = false;
    int k = 0;

    for (; k < nk; ++k) {
        const uint32_t x = xs + k, kq = K + k;               // plane index within the tile / within the CTA
        const int s = kq % TT_S;
        const bool ok = mbar_wait_bounded(smem_u32(&S.full[s]), (kq / TT_S) & 1u, WAIT_NS);
        const uint32_t xmask = cand ? axis_mask(ps, cand, 0, x) : 0u;
        const float* Hs = &S.st[s].H[0][0][0];
        const float* Es = &S.st[s].E[0][0][0];
        const uint32_t* Ms = &S.st[s].M[0][0];
        float* En = &S.En[kq % 3][0][0][0];
        const uint32_t px = x * NyNz;
        float en[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        float hc[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        uint32_t mc[3] = {0u, 0u, 0u};
        if (ok) {
            // ---- E_new(x): gather every operand of the thread's cells, then update, then store
            float hv[3][7], eo[3][3], kk[3][6];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q == 2 && !has2) continue;
                const int h = hi[q], e = ei[q];
                hv[q][0] = Hs[h]; hv[q][1] = Hs[HPL + h]; hv[q][2] = Hs[2 * HPL + h];
                hv[q][3] = Hs[2 * HPL + h - dym[q]];         // hz(y-1)
                hv[q][4] = Hs[HPL + h - dzm[q]];             // hy(z-1)
                hv[q][5] = Hs[h - dzm[q]];                   // hx(z-1)
                hv[q][6] = Hs[h - dym[q]];                   // hx(y-1)
                eo[q][0] = Es[e]; eo[q][1] = Es[EPL + e]; eo[q][2] = Es[2 * EPL + e];
                mc[q] = IDX ? Ms[e] : 0u;
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q == 2 && !has2) continue;
                if (IDX) coeffs_f<true>(g, 0, mc[q], 0, kk[q]);
                else if (sin[q]) coeffs_f<false>(g, (size_t)px + off[q], 0u, 0, kk[q]);
                else kk[q][0] = kk[q][1] = kk[q][2] = kk[q][3] = kk[q][4] = kk[q][5] = 0.f;
            }
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q == 2 && !has2) continue;
                const float hx = hv[q][0], hy = hv[q][1], hz = hv[q][2];
                const float cx = curl4(hz, hv[q][3], hy, hv[q][4]);
                const float cy = curl4(hx, hv[q][5], hz, hp[q][2]);
                const float cz = curl4(hy, hp[q][1], hx, hv[q][6]);
                hc[q][0] = hx; hc[q][1] = hy; hc[q][2] = hz;
                // a UPML cell's E_new was computed by k_pml_e and staged in place of E_old
                const bool upml = PML && (yzm[q] & xmask);
                en[q][0] = upml ? eo[q][0] : upd(eo[q][0], kk[q][0], kk[q][3], cx);
                en[q][1] = upml ? eo[q][1] : upd(eo[q][1], kk[q][1], kk[q][4], cy);
                en[q][2] = upml ? eo[q][2] : upd(eo[q][2], kk[q][2], kk[q][5], cz);
                if (tf_tile && tfq[q] >= 0) {               // the TFSF point pass's add, here
                    const float* D = &S.st[s].D[tfq[q]][0][0];
                    en[q][0] = __fadd_rn(en[q][0], D[sr[q]]);
                    en[q][1] = __fadd_rn(en[q][1], D[TF_DY + sr[q]]);
                }
            }
            float* V1 = g.V1 + px;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q == 2 && !has2) continue;
                const int e = ei[q];
                En[e] = en[q][0]; En[EPL + e] = en[q][1]; En[2 * EPL + e] = en[q][2];
                if (own && q < 2 && sin[q] && x < xe) {
                    V1[off[q]] = en[q][0];
                    V1[off[q] + N] = en[q][1];
                    V1[off[q] + 2 * N] = en[q][2];
                }
            }
        }
        // every read of stage s and every write of En[k % 3] done; agree on a timeout
        timed_out = __syncthreads_or(!ok) != 0;
        if (timed_out) break;
        if (threadIdx.x == 0 && issued < nk) {
            if (xs + issued != g.skip_plane)   // stage of plane k+TT_S
                tt_issue<IDX>(S, s, tmH, tmE, tmM, tmD, dbytes, (int)(xs + issued), (int)y0, (int)z0);
            ++issued;
        }
        // ---- H_new(x-1) of the owned cells
        if (k > 0 && own) {
            const float* Ep = &S.En[(kq + 2) % 3][0][0][0];
            float nb[2][4], kh[2][6];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int e = ei[q];
                nb[q][0] = Ep[2 * EPL + e + TT_EZ];          // ez(y+1)
                nb[q][1] = Ep[EPL + e + 1];                  // ey(z+1)
                nb[q][2] = Ep[e + 1];                        // ex(z+1)
                nb[q][3] = Ep[e + TT_EZ];                    // ex(y+1)
                if (IDX) coeffs_f<true>(g, 0, mp[q], 6, kh[q]);
                else if (sin[q]) coeffs_f<false>(g, (size_t)(px - NyNz) + off[q], 0u, 6, kh[q]);
                else kh[q][0] = kh[q][1] = kh[q][2] = kh[q][3] = kh[q][4] = kh[q][5] = 0.f;
            }
            float* H1 = g.H1 + (px - NyNz);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const float ex = ep[q][0], ey = ep[q][1], ez = ep[q][2];
                const float cx = curl4(ez, nb[q][0], ey, nb[q][1]);
                const float cy = curl4(ex, nb[q][2], ez, en[q][2]);
                const float cz = curl4(ey, en[q][1], ex, nb[q][3]);
                float hn[3];
                hn[0] = core[q] ? upd(hp[q][0], kh[q][0], kh[q][3], cx) : hp[q][0];
                hn[1] = core[q] ? upd(hp[q][1], kh[q][1], kh[q][4], cy) : hp[q][1];
                hn[2] = core[q] ? upd(hp[q][2], kh[q][2], kh[q][5], cz) : hp[q][2];
                if (sin[q] && !(PML && (yzm[q] & xmask_p))) {     // UPML cells: k_pml_h
                    H1[off[q]] = hn[0];
                    H1[off[q] + N] = hn[1];
                    H1[off[q] + 2 * N] = hn[2];
                }
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
                if (xs + j != g.skip_plane)
                    (void)mbar_wait_bounded(smem_u32(&S.full[(K + j) % TT_S]), ((K + j) / TT_S) & 1u, WAIT_NS);
        }
        return false;
    }
    // ---- H of the last plane x = Nx-1: no core update (pass-through; UPML cells: k_pml_h)
    if (xe == g.Nx && own) {
        float* H1 = g.H1 + (size_t)(g.Nx - 1) * NyNz;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!sin[q] || (PML && (yzm[q] & xmask_p))) continue;
#pragma unroll
            for (int n = 0; n < 3; ++n) H1[off[q] + n * N] = hp[q][n];
        }
    }
    K += nk;
    return true;
}
// A TFSF face corrected in the core update meets the tile's columns (halo column included).
template <bool IDX, bool PML>
__device__ __forceinline__ bool tma_tile(TmaSmem& S, const CUtensorMap* tmH, const CUtensorMap* tmE, const CUtensorMap* tmM,
                                         const CUtensorMap* tmD, const FusedGrid& g, const PmlSet& ps, uint32_t xs,
                                         uint32_t y0, uint32_t z0, uint32_t& K) {
    bool tf = false;
    for (uint32_t f = 0; f < g.tf.n; ++f) tf |= g.tf.z[f] >= z0 && g.tf.z[f] <= z0 + TT_Z;
    return tf ? tma_tile_body<IDX, PML, true>(S, tmH, tmE, tmM, tmD, g, ps, xs, y0, z0, K)
              : tma_tile_body<IDX, PML, false>(S, tmH, tmE, tmM, tmD, g, ps, xs, y0, z0, K);
}

template <bool IDX, bool PML>
__global__ void __launch_bounds__(TT_THREADS, 2)
k_fused_tma(const __grid_constant__ CUtensorMap tmH, const __grid_constant__ CUtensorMap tmE,
            const __grid_constant__ CUtensorMap tmM, const __grid_constant__ CUtensorMap tmD, const FusedGrid g,
            const PmlSet ps) {
    const uint32_t xs = blockIdx.z * g.xchunk;
    if (xs >= g.Nx) return;                                  // uniform per CTA
    TmaSmem& S = tt_smem();
    tt_init(S);
    uint32_t K = 0;
    (void)tma_tile<IDX, PML>(S, &tmH, &tmE, &tmM, &tmD, g, ps, xs, blockIdx.y * TT_Y, blockIdx.x * TT_Z, K);
}

// ---------------------------------------------------------------------------
// UPML cells of the TMA path, outside the streaming kernel.  Their update
// reads per-cell region coefficients and fluxes with dependent loads; run
// inside the plane pipeline those loads stalled every CTA whose tile touches a
// region.  k_pml_e runs before k_fused_tma and k_pml_h after it.  A cell that
// several regions contain is handled once, by the first of them, with the
// chain over all of them in region order.
//
// Both passes are latency-bound (a z-slab region row is 8 cells, 32 bytes,
// long).  A thread takes PML_ZC consecutive z cells of one region row and
// issues every load of them (fields, material index and, for the usual
// single-region cell, the region's flux and compact coefficient row) before
// any arithmetic.  Measured on B200 over PML_ZC in {1, 2, 4} x {2, 3, 4, 6}
// blocks per SM, one cell per thread at 4 blocks per SM (64 registers, no
// spills) is fastest: occupancy hides more latency than per-thread batching.
// ---------------------------------------------------------------------------
#ifndef EFS_PML_ZC
#define EFS_PML_ZC 1
#endif
#ifndef EFS_PML_MINB
#define EFS_PML_MINB 4
#endif
constexpr uint32_t PML_ZC = EFS_PML_ZC;     // z cells per thread
constexpr int PML_MINB = EFS_PML_MINB;      // resident 256-thread blocks per SM the register budget is set for

// Work item i -> region r, row (x, y), first z and cell count (PML_ZC cells
// per item along z, items in region order).
__device__ __forceinline__ bool pml_item(const PmlSet& ps, uint32_t i, int& r, uint32_t& x, uint32_t& y, uint32_t& z,
                                         uint32_t& cnt) {
    for (r = 0; r < ps.count; ++r) {
        const PmlRegion& R = ps.r[r];
        const uint32_t zc = (R.n[2] + PML_ZC - 1) / PML_ZC;
        const uint32_t items = R.n[0] * R.n[1] * zc;
        if (i < items) {
            const uint32_t row = i / zc, zi = i - row * zc;
            x = R.s[0] + row / R.n[1];
            y = R.s[1] + row % R.n[1];
            z = R.s[2] + zi * PML_ZC;
            cnt = min(PML_ZC, R.n[2] - zi * PML_ZC);
            return true;
        }
        i -= items;
    }
    return false;
}

// Every region containing (x, y, z) when region r is the first that does, else 0.
__device__ __forceinline__ uint32_t pml_owner_mask(const PmlSet& ps, int r, uint32_t x, uint32_t y, uint32_t z) {
    for (int q = 0; q < r; ++q)
        if (in_region(ps.r[q], x, y, z)) return 0u;
    uint32_t m = 1u << r;
    for (int q = r + 1; q < ps.count; ++q)
        if (in_region(ps.r[q], x, y, z)) m |= 1u << q;
    return m;
}

// Region coefficients and old flux of one single-region cell (3 components).
// With the compact form the three coefficients come from one table row
// (three float4 loads that hit L1/L2) instead of nine per-cell loads.
template <bool VOLT>
__device__ __forceinline__ void pml_fetch(const PmlRegion& R, uint32_t x, uint32_t y, uint32_t z, float a[3], float b[3],
                                          float fn[3], float fo[3]) {
    const size_t p0 = region_p(R, 0, x, y, z), nreg = (size_t)R.n[0] * R.n[1] * R.n[2];
#pragma unroll
    for (int n = 0; n < 3; ++n) fo[n] = __ldg((VOLT ? R.vflux : R.cflux) + p0 + n * nreg);
    if (R.cidx) {
        const float4* row = R.ctab + 6 * (uint32_t)__ldg(R.cidx + p0) + (VOLT ? 0 : 3);
        const float4 ka = __ldg(row), kb = __ldg(row + 1), kf = __ldg(row + 2);
        a[0] = ka.x; a[1] = ka.y; a[2] = ka.z;
        b[0] = kb.x; b[1] = kb.y; b[2] = kb.z;
        fn[0] = kf.x; fn[1] = kf.y; fn[2] = kf.z;
        return;
    }
#pragma unroll
    for (int n = 0; n < 3; ++n) {
        const size_t p = p0 + n * nreg;
        a[n] = __ldg((VOLT ? R.vv : R.ii) + p);
        b[n] = __ldg((VOLT ? R.vvfo : R.iifo) + p);
        fn[n] = __ldg((VOLT ? R.vvfn : R.iifn) + p);
    }
}

// The single-region chain of pml_cell on prefetched values; writes the new flux.
template <bool VOLT>
__device__ __forceinline__ float pml_one(const PmlRegion& Rn, size_t p, float vold, bool core, float cv, float ci, float curl,
                                         float a, float b, float fn, float fo) {
    const float fh = __fsub_rn(__fmul_rn(a, vold), __fmul_rn(b, fo));
    const float v = core ? upd(fo, cv, ci, curl) : fo;
    (VOLT ? Rn.vflux : Rn.cflux)[p] = v;
    return __fadd_rn(fh, __fmul_rn(fn, v));
}

// E_new of the UPML cells (reads H_old and E_old, the old flux; writes the new
// flux).  E_new is written over E_old in `V0w` (the step's old-E buffer, dead
// after this step's core update), where k_fused_tma stages it.
template <bool IDX>
__device__ __forceinline__ void pml_e_body(const FusedGrid& g, const PmlSet& ps, const PmlSet& pn, float* V0w, uint32_t items,
                                           uint32_t i) {
    if (i >= items) return;
    int r;
    uint32_t x, y, z0, cnt;
    if (!pml_item(ps, i, r, x, y, z0, cnt)) return;
    const uint32_t N = (uint32_t)g.N, NyNz = (uint32_t)g.NyNz, Pz = g.Pz;
    const uint32_t c0 = x * NyNz + y * Pz + z0;
    const uint32_t dx = x > 0 ? NyNz : 0u, dy = y > 0 ? Pz : 0u;      // x-1 / y-1 neighbour (self at index 0)
    const float* H = g.H0;
    const PmlRegion& R = ps.r[r];
    uint32_t mask[PML_ZC], m[PML_ZC];
    float hv[PML_ZC][9], eo[PML_ZC][3], a[PML_ZC][3], b[PML_ZC][3], fn[PML_ZC][3], fo[PML_ZC][3];
    // ---- every load of the item's cells
#pragma unroll
    for (uint32_t j = 0; j < PML_ZC; ++j) {
        mask[j] = j < cnt ? pml_owner_mask(ps, r, x, y, z0 + j) : 0u;
        if (!mask[j]) continue;
        const uint32_t c = c0 + j, dz = (z0 + j) > 0 ? 1u : 0u;
        hv[j][0] = H[c]; hv[j][1] = H[N + c]; hv[j][2] = H[2 * N + c];
        hv[j][3] = H[2 * N + c - dy];      // hz(y-1)
        hv[j][4] = H[N + c - dz];          // hy(z-1)
        hv[j][5] = H[c - dz];              // hx(z-1)
        hv[j][6] = H[2 * N + c - dx];      // hz(x-1)
        hv[j][7] = H[N + c - dx];          // hy(x-1)
        hv[j][8] = H[c - dy];              // hx(y-1)
        eo[j][0] = V0w[c]; eo[j][1] = V0w[N + c]; eo[j][2] = V0w[2 * N + c];
        m[j] = IDX ? __ldg(g.mat + c) : 0u;
        if (mask[j] == (1u << r)) pml_fetch<true>(R, x, y, z0 + j, a[j], b[j], fn[j], fo[j]);
    }
    // ---- update and store
#pragma unroll
    for (uint32_t j = 0; j < PML_ZC; ++j) {
        if (!mask[j]) continue;
        const uint32_t c = c0 + j, z = z0 + j;
        const float cv[3] = {curl4(hv[j][2], hv[j][3], hv[j][1], hv[j][4]),     // backward curl, reference order
                             curl4(hv[j][0], hv[j][5], hv[j][2], hv[j][6]),
                             curl4(hv[j][1], hv[j][7], hv[j][0], hv[j][8])};
        float kk[6];
        coeffs_f<IDX>(g, c, m[j], 0, kk);
        float en[3];
        if (mask[j] == (1u << r)) {
            const size_t p0 = region_p(R, 0, x, y, z), nreg = (size_t)R.n[0] * R.n[1] * R.n[2];
#pragma unroll
            for (int n = 0; n < 3; ++n)
                en[n] = pml_one<true>(pn.r[r], p0 + n * nreg, eo[j][n], true, kk[n], kk[3 + n], cv[n], a[j][n], b[j][n],
                                      fn[j][n], fo[j][n]);
        } else {
#pragma unroll
            for (int n = 0; n < 3; ++n)
                en[n] = pml_chain_pp<true>(ps, pn, mask[j], x, y, z, n, eo[j][n], true, kk[n], kk[3 + n], cv[n], true);
        }
        V0w[c] = en[0]; V0w[N + c] = en[1]; V0w[2 * N + c] = en[2];
    }
}
template <bool IDX>
__global__ void __launch_bounds__(256, PML_MINB) k_pml_e(const FusedGrid g, const PmlSet ps, const PmlSet pn, float* V0w, uint32_t items) {
    pml_e_body<IDX>(g, ps, pn, V0w, items, blockIdx.x * blockDim.x + threadIdx.x);
}

// H_new of the UPML cells from the final E_new: runs after the E-side point
// operations (beside k_deferred_h, which leaves UPML cells to this pass).
template <bool IDX>
__device__ __forceinline__ void pml_h_body(const FusedGrid& g, const PmlSet& ps, const PmlSet& pn, uint32_t items, uint32_t i) {
    if (i >= items) return;
    int r;
    uint32_t x, y, z0, cnt;
    if (!pml_item(ps, i, r, x, y, z0, cnt)) return;
    const uint32_t N = (uint32_t)g.N, NyNz = (uint32_t)g.NyNz, Pz = g.Pz;
    const uint32_t c0 = x * NyNz + y * Pz + z0;
    const float* V = g.V1;
    const PmlRegion& R = ps.r[r];
    uint32_t mask[PML_ZC], m[PML_ZC];
    bool core[PML_ZC];
    float ev[PML_ZC][9], ho[PML_ZC][3], a[PML_ZC][3], b[PML_ZC][3], fn[PML_ZC][3], fo[PML_ZC][3];
    const bool core_xy = (x + 1 < g.Nx) && (y + 1 < g.Ny);
#pragma unroll
    for (uint32_t j = 0; j < PML_ZC; ++j) {
        mask[j] = j < cnt ? pml_owner_mask(ps, r, x, y, z0 + j) : 0u;
        if (!mask[j]) continue;
        const uint32_t c = c0 + j;
        core[j] = core_xy && (z0 + j + 1 < g.Nz);
        if (core[j]) {
            ev[j][0] = V[c]; ev[j][1] = V[N + c]; ev[j][2] = V[2 * N + c];
            ev[j][3] = V[2 * N + c + Pz];      // ez(y+1)
            ev[j][4] = V[N + c + 1];           // ey(z+1)
            ev[j][5] = V[c + 1];               // ex(z+1)
            ev[j][6] = V[2 * N + c + NyNz];    // ez(x+1)
            ev[j][7] = V[N + c + NyNz];        // ey(x+1)
            ev[j][8] = V[c + Pz];              // ex(y+1)
            m[j] = IDX ? __ldg(g.mat + c) : 0u;
        }
        ho[j][0] = g.H0[c]; ho[j][1] = g.H0[N + c]; ho[j][2] = g.H0[2 * N + c];
        if (mask[j] == (1u << r)) pml_fetch<false>(R, x, y, z0 + j, a[j], b[j], fn[j], fo[j]);
    }
#pragma unroll
    for (uint32_t j = 0; j < PML_ZC; ++j) {
        if (!mask[j]) continue;
        const uint32_t c = c0 + j, z = z0 + j;
        float cv[3] = {0.f, 0.f, 0.f};
        float kk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (core[j]) {                        // forward curl, reference order
            cv[0] = curl4(ev[j][2], ev[j][3], ev[j][1], ev[j][4]);
            cv[1] = curl4(ev[j][0], ev[j][5], ev[j][2], ev[j][6]);
            cv[2] = curl4(ev[j][1], ev[j][7], ev[j][0], ev[j][8]);
            coeffs_f<IDX>(g, c, m[j], 6, kk);
        }
        float hn[3];
        if (mask[j] == (1u << r)) {
            const size_t p0 = region_p(R, 0, x, y, z), nreg = (size_t)R.n[0] * R.n[1] * R.n[2];
#pragma unroll
            for (int n = 0; n < 3; ++n)
                hn[n] = pml_one<false>(pn.r[r], p0 + n * nreg, ho[j][n], core[j], kk[n], kk[3 + n], cv[n], a[j][n], b[j][n],
                                       fn[j][n], fo[j][n]);
        } else {
#pragma unroll
            for (int n = 0; n < 3; ++n)
                hn[n] = pml_chain_pp<false>(ps, pn, mask[j], x, y, z, n, ho[j][n], core[j], kk[n], kk[3 + n], cv[n], true);
        }
        g.H1[c] = hn[0]; g.H1[N + c] = hn[1]; g.H1[2 * N + c] = hn[2];
    }
}
template <bool IDX>
__global__ void __launch_bounds__(256, PML_MINB) k_pml_h(const FusedGrid g, const PmlSet ps, const PmlSet pn, uint32_t items) {
    pml_h_body<IDX>(g, ps, pn, items, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// Two independent passes in one launch.  The UPML passes, the deferred H and
// the NF2FF samples are latency-bound (40-56% of DRAM bandwidth alone: their
// items sit one or two per z row); launched as one grid with their blocks
// interleaved, each pass's loads overlap the other's.  Block i: while both
// passes have blocks left, even blocks run A and odd blocks run B; the rest
// run the longer pass.  Every pass uses 256-thread blocks.
// ---------------------------------------------------------------------------
template <bool IDX>
struct PassPmlE {
    FusedGrid g; PmlSet ps, pn; float* V0w; uint32_t items;
    __device__ void run(uint32_t blk) const { pml_e_body<IDX>(g, ps, pn, V0w, items, blk * 256u + threadIdx.x); }
};
template <bool IDX>
struct PassPmlH {
    FusedGrid g; PmlSet ps, pn; uint32_t items;
    __device__ void run(uint32_t blk) const { pml_h_body<IDX>(g, ps, pn, items, blk * 256u + threadIdx.x); }
};
template <bool IDX>
struct PassDeferred {
    FusedGrid g; const uint32_t* cells; uint32_t n;
    __device__ void run(uint32_t blk) const { deferred_h_body<IDX>(g, cells, n, blk * 256u + threadIdx.x); }
};
struct PassNfSample {
    const float* V; const float* C; uint32_t slot; Nf2ffDev d;
    __device__ void run(uint32_t blk) const { nf2ff_sample_body(V, C, slot, d, blk * 256u + threadIdx.x); }
};
template <class A, class B>
__global__ void __launch_bounds__(256, PML_MINB) k_pair(const A a, uint32_t na, const B b, uint32_t nb) {
    const uint32_t i = blockIdx.x, m = min(na, nb);
    if (i < 2 * m) {
        if (i & 1u) b.run(i >> 1);
        else a.run(i >> 1);
    } else if (na > nb) {
        a.run(i - m);
    } else {
        b.run(i - m);
    }
}

}  // namespace efs
