// efs_fused.cuh — definitions shared by the single-pass E+H update
// (efs_tma.cuh), the UPML passes around it and the deferred H update.
//
// One timestep moves each field value through HBM once (read old, write
// new): 48 B of fields + 4 B of material index per cell.  Old and new fields
// live in separate buffers (as do the UPML flux arrays), so recomputed halo
// cells and neighbouring tiles never race.
//
// Device layout: the reference's NIJK order with the z rows padded to a
// pitch Pz (Nz rounded up to a multiple of 4 floats), so that every row and
// plane starts on a 16-byte boundary as the TMA tensor maps require.  The
// field index of (n, x, y, z) is n*N + (x*Ny + y)*Pz + z with N = Nx*Ny*Pz;
// the host translates every index a caller passes (NIJK with pitch Nz) once,
// at configure time.  Pad cells (z >= Nz) are never read as field values.
//
// H cells whose curl reads an E value that a sparse post-update operation
// rewrites (TFSF, Mur apply, excitation, PBC, series RLC, the ADE apply step)
// get a provisional H from the fused kernel and are recomputed by
// k_deferred_h, which runs after those operations (UPML cells among them are
// left to k_pml_h, which runs after them as well).  The result is the
// reference's phase order exactly, bit for bit.
#pragma once
#include "efs_kernels.cuh"

namespace efs {

constexpr int PML_MAX_OVERLAP = 4;

struct FusedGrid {
    uint32_t Nx, Ny, Nz, xchunk;
    uint32_t Pz;                        // z pitch of the device layout (Nz rounded up to a multiple of 4)
    size_t N, NyNz;                     // device component stride Nx*Ny*Pz and plane stride Ny*Pz
    const float* V0; const float* H0;   // fields at the start of the step
    float* V1; float* H1;               // fields after the step
    const uint32_t* mat; const float* table;
    const float* vv; const float* vi; const float* ii; const float* iv;
    uint32_t* status;                   // device status word (bit 0: a bounded wait ran out)
    uint64_t wait_ns;                   // limit of every bounded mbarrier wait (about 1 s)
    uint32_t skip_plane;                // diagnostics: loads of this x-plane are never issued (~0u: none)
    TfsfFace tf;                        // TFSF z faces corrected in the core update (tf.n == 0: none)
};

// Face of z plane z among the TFSF faces the core update corrects, or -1.
__device__ __forceinline__ int tf_face(const TfsfFace& tf, uint32_t z) {
    return tf.n > 0 && z == tf.z[0] ? 0 : (tf.n > 1 && z == tf.z[1]) ? 1 : -1;
}

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

// H update of the deferred cells, after the E-side sparse operations: reads
// the final E_new and H_old, writes H_new, one thread per cell.  No deferred
// cell is a UPML cell (k_pml_h, which runs after the E-side operations too,
// updates those).
template <bool IDX>
__device__ __forceinline__ void deferred_h_body(const FusedGrid& g, const uint32_t* cells, uint32_t n, uint32_t i) {
    if (i >= n) return;
    const uint32_t c = cells[i];
    const uint32_t N = (uint32_t)g.N, NyNz = (uint32_t)g.NyNz, Pz = g.Pz;   // 3*N < 2^32
    const uint32_t x = c / NyNz, rem = c - x * NyNz, y = rem / Pz, z = rem - y * Pz;
    const bool core = (x + 1 < g.Nx) && (y + 1 < g.Ny) && (z + 1 < g.Nz);
    const float* V = g.V1;
    float ho[3], ev[9];
    ho[0] = g.H0[c]; ho[1] = g.H0[N + c]; ho[2] = g.H0[2 * N + c];
    uint32_t m = 0;
    if (core) {
        ev[0] = V[c]; ev[1] = V[N + c]; ev[2] = V[2 * N + c];
        ev[3] = V[2 * N + c + Pz]; ev[4] = V[N + c + 1]; ev[5] = V[c + 1];
        ev[6] = V[2 * N + c + NyNz]; ev[7] = V[N + c + NyNz]; ev[8] = V[c + Pz];
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
    for (int q = 0; q < 3; ++q) g.H1[q * N + c] = core ? upd(ho[q], kk[q], kk[3 + q], cv[q]) : ho[q];
}
template <bool IDX>
__global__ void __launch_bounds__(256) k_deferred_h(const FusedGrid g, const uint32_t* cells, uint32_t n) {
    deferred_h_body<IDX>(g, cells, n, blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace efs
