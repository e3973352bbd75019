// efs_kernels.cuh — device code of the B200 FDTD engine.
//
// Arithmetic: every field update is written with __fmul_rn/__fadd_rn/__fsub_rn
// in the operand order of the reference's update expressions
// (src/webgpu-engine.mjs WGSL, src/webgpu-fdtd.mjs CPU engine), so no FMA
// contraction changes a result: the engine agrees bit for bit with an f32
// restatement of the reference evaluated in the same order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace efs {

constexpr int MAX_PML = 24;     // UPML regions handled by the fused update
struct StepState {              // device-resident, read by every per-step kernel
    uint32_t numTS;
    uint32_t ss_recording;
    uint32_t ss_start;          // numTS at which steady-state recording began
    uint32_t ss_base;           // sample count accumulated before ss_start
};

struct PmlRegion {
    uint32_t s[3], n[3];
    const float* vv; const float* vvfo; const float* vvfn;
    const float* ii; const float* iifo; const float* iifn;
    float* vflux; float* cflux;
    // Optional compact form of the six coefficient arrays (null when a region
    // has more than 65535 distinct cell tuples): per cell a row index, per row
    // six float4 {vv, vvfo, vvfn, ii, iifo, iifn} x 3 components (+ pad).
    const uint16_t* cidx; const float4* ctab;
};
struct PmlSet {
    int count;
    PmlRegion r[MAX_PML];
};

__device__ __forceinline__ float upd(float vold, float cv, float ci, float curl) {
    // V <- (V*vv) + vi*curl, each product rounded (src/webgpu-fdtd.mjs:76-82)
    return __fadd_rn(__fmul_rn(vold, cv), __fmul_rn(ci, curl));
}
__device__ __forceinline__ float curl4(float a, float b, float c, float d) {
    return __fadd_rn(__fsub_rn(__fsub_rn(a, b), c), d);
}

__device__ __forceinline__ bool in_region(const PmlRegion& r, uint32_t x, uint32_t y, uint32_t z) {
    return (x - r.s[0]) < r.n[0] && (y - r.s[1]) < r.n[1] && (z - r.s[2]) < r.n[2];
}

// Regions intersecting the box [lo, hi] (inclusive), as a bit mask.  Blocks
// compute this once so cells of tiles that touch no UPML region skip the
// per-cell membership tests entirely.
__device__ __forceinline__ uint32_t region_mask(const PmlSet& ps, const uint32_t lo[3], const uint32_t hi[3]) {
    uint32_t m = 0;
    for (int r = 0; r < ps.count; ++r) {
        bool hit = true;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            hit = hit && (hi[d] >= ps.r[r].s[d]) && (lo[d] < ps.r[r].s[d] + ps.r[r].n[d]);
        if (hit) m |= 1u << r;
    }
    return m;
}
__device__ __forceinline__ size_t region_p(const PmlRegion& r, uint32_t n, uint32_t x, uint32_t y, uint32_t z) {
    size_t nyz = (size_t)r.n[1] * r.n[2];
    return (size_t)n * r.n[0] * nyz + (size_t)(x - r.s[0]) * nyz + (size_t)(y - r.s[1]) * r.n[2] + (z - r.s[2]);
}

// ---------------------------------------------------------------------------
// sparse per-step operations
// ---------------------------------------------------------------------------

// Additive point sources grouped by target so repeated targets keep the
// reference's sequential order: group g covers entries [off[g], off[g+1]).
// kind 0 = excitation (src/webgpu-fdtd.mjs:161-185, C++ past-end semantics)
// kind 1 = TFSF (src/webgpu-fdtd.mjs:694-733, interpolated, skipped past end)
struct PointSources {
    uint32_t ngroups;
    const uint32_t* target;     // field index per group
    const uint32_t* off;        // ngroups+1
    const uint32_t* delay;      // per entry
    const float* amp;           // per entry
    const float* frac;          // per entry (TFSF)
    const float* signal;
    uint32_t len, period;
};

// Thread bodies below are shared by the single-engine kernels and the
// segmented kernels that advance several engines at once (efs_batch.cuh).
template <int KIND>
__device__ __forceinline__ void point_sources_body(float* __restrict__ F, const StepState* st, uint32_t k, const PointSources& s,
                                                   uint32_t gi) {
    if (gi >= s.ngroups) return;
    const int64_t ts = (int64_t)st->numTS + k;
    const uint32_t t = s.target[gi];
    float v = F[t];
    for (uint32_t e = s.off[gi]; e < s.off[gi + 1]; ++e) {
        if (KIND == 0) {
            int64_t p = s.period > 0 ? (int64_t)s.period : ts + 1;
            int64_t pos = ts - (int64_t)s.delay[e];
            if (pos < 0) pos = 0;
            pos %= p;
            if (pos >= (int64_t)s.len) pos = 0;
            v = __fadd_rn(v, __fmul_rn(s.amp[e], s.signal[pos]));
        } else {
            int64_t d = ts - (int64_t)s.delay[e];
            if (d < 0) continue;
            if (s.period > 0) d %= (int64_t)s.period;
            if (d >= (int64_t)s.len - 1) continue;
            const float delta = s.frac[e];
            const float sig = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, delta), s.signal[d]), __fmul_rn(delta, s.signal[d + 1]));
            v = __fadd_rn(v, __fmul_rn(s.amp[e], sig));
        }
    }
    F[t] = v;
}
template <int KIND>
__global__ void k_point_sources(float* __restrict__ F, const StepState* st, uint32_t k, const PointSources s) {
    point_sources_body<KIND>(F, st, k, s, blockIdx.x * blockDim.x + threadIdx.x);
}

// A field read that the reference makes after the UPML pre-update: for a cell
// inside a region the value there is the region's old flux.  sel 0 = field,
// sel r+1 = flux of region r.
struct ReadLoc { uint32_t sel, idx; };

__device__ __forceinline__ float read_loc(const float* F, const float* const* flux, ReadLoc l) {
    return l.sel == 0 ? F[l.idx] : flux[l.sel - 1][l.idx];
}

// Mur ABC (src/webgpu-fdtd.mjs:992-1023)
struct MurDev {
    uint32_t n, napply;
    const float* coeff;
    const ReadLoc* pre_normal;     // reads after the UPML pre swap
    const ReadLoc* pre_shifted;
    const uint32_t* shifted;
    const uint32_t* apply_target;  // unique normal indices
    const uint32_t* apply_src;     // last entry that writes each target
    float* saved;
    const float* const* vflux;
};
__device__ __forceinline__ void mur_pre_body(const float* __restrict__ V, const MurDev& m, uint32_t i) {
    if (i >= m.n) return;
    float s = read_loc(V, m.vflux, m.pre_shifted[i]);
    float nv = read_loc(V, m.vflux, m.pre_normal[i]);
    m.saved[i] = __fsub_rn(s, __fmul_rn(m.coeff[i], nv));
}
__device__ __forceinline__ void mur_post_body(const float* __restrict__ V, const MurDev& m, uint32_t i) {
    if (i >= m.n) return;
    m.saved[i] = __fadd_rn(m.saved[i], __fmul_rn(m.coeff[i], V[m.shifted[i]]));
}
__device__ __forceinline__ void mur_apply_body(float* __restrict__ V, const MurDev& m, uint32_t i) {
    if (i >= m.napply) return;
    V[m.apply_target[i]] = m.saved[m.apply_src[i]];
}
__global__ void k_mur_pre(const float* __restrict__ V, const MurDev m) { mur_pre_body(V, m, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_mur_post(const float* __restrict__ V, const MurDev m) { mur_post_body(V, m, blockIdx.x * blockDim.x + threadIdx.x); }
__global__ void k_mur_apply(float* __restrict__ V, const MurDev m) { mur_apply_body(V, m, blockIdx.x * blockDim.x + threadIdx.x); }

// Lorentz/Drude ADE state update (src/webgpu-fdtd.mjs:405-454), all orders
// and directions of one field flattened into one list of entries.  The
// per-entry locations and coefficients are stored as runs: the entries
// [run.entry, next run.entry) read consecutive locations from (sel, idx) on
// and share one coefficient tuple, so a sphere row costs one 16-byte run
// instead of 21 bytes per entry.  A thread updates ADE_V consecutive entries
// (one group; state and Lorentz state as 16-byte accesses, so enough bytes are
// in flight per SM).  grp_run[q] names the run of entry q*ADE_V (bit 31: the
// group holds a Lorentz entry), so the state, Lorentz state and run loads
// issue together and the field loads follow; the thread steps forward across
// run starts inside its group.  The run list ends with a sentinel run whose
// entry is n.
constexpr uint32_t ADE_T = 256;                 // threads per block
constexpr uint32_t ADE_V = 4;                   // entries per thread (one group), a multiple of 4: 8 (48
                                                // registers, 5 blocks/SM) measured 2% slower per dispersive step
constexpr uint32_t ADE_BLOCK = ADE_T * ADE_V;   // entries per block
struct AdeRun { uint32_t entry, sel, idx, coef; };   // coef: tuple id, bit 31 set for Lorentz
struct AdeDev {
    uint32_t n;
    const AdeRun* runs;             // + sentinel {n, 0, 0, 0}
    const uint32_t* grp_run;        // per group: run of its first entry, bit 31 if it holds a Lorentz entry
    const float4* coef;             // per tuple: kint, kext, klor, 0
    float* state; float* lor;       // 16-byte aligned
    const float* const* flux;
};
__device__ __forceinline__ float ade_one(float v, float st, float& l, uint32_t cid, const float4& c) {
    if (cid >> 31) {
        l = __fadd_rn(l, __fmul_rn(c.z, st));
        return __fadd_rn(__fmul_rn(c.x, st), __fmul_rn(c.y, __fsub_rn(v, l)));
    }
    return __fadd_rn(__fmul_rn(c.x, st), __fmul_rn(c.y, v));
}
// Group q of one side (thread body shared with the batched form's segmented launch).
__device__ __forceinline__ void ade_body(const float* __restrict__ F, const AdeDev& a, uint32_t q) {
    constexpr uint32_t NQ = ADE_V / 4;
    const uint32_t i0 = q * ADE_V;
    if (i0 >= a.n) return;
    const uint32_t cnt = min(ADE_V, a.n - i0);
    const uint32_t qr = __ldg(a.grp_run + q);
    float4 st[NQ], lr[NQ];
#pragma unroll
    for (uint32_t h = 0; h < NQ; ++h) { st[h] = make_float4(0.f, 0.f, 0.f, 0.f); lr[h] = st[h]; }
    if (cnt == ADE_V) {
#pragma unroll
        for (uint32_t h = 0; h < NQ; ++h) {
            st[h] = *reinterpret_cast<const float4*>(a.state + i0 + 4 * h);
            if (qr >> 31) lr[h] = *reinterpret_cast<const float4*>(a.lor + i0 + 4 * h);
        }
    }
    uint32_t lo = qr & 0x7fffffffu;
    AdeRun r = a.runs[lo];
    uint32_t next = a.runs[lo + 1].entry;
    float v[ADE_V];
    uint32_t cid[ADE_V];
#pragma unroll
    for (uint32_t k = 0; k < ADE_V; ++k) {
        cid[k] = 0;
        v[k] = 0.f;
        if (k < cnt) {
            const uint32_t i = i0 + k;
            while (i >= next) { ++lo; r = a.runs[lo]; next = a.runs[lo + 1].entry; }
            v[k] = read_loc(F, a.flux, ReadLoc{r.sel, r.idx + (i - r.entry)});
            cid[k] = r.coef;
        }
    }
    if (cnt == ADE_V) {
#pragma unroll
        for (uint32_t h = 0; h < NQ; ++h) {
            const uint32_t k = 4 * h;
            st[h].x = ade_one(v[k], st[h].x, lr[h].x, cid[k], a.coef[cid[k] & 0x7fffffffu]);
            st[h].y = ade_one(v[k + 1], st[h].y, lr[h].y, cid[k + 1], a.coef[cid[k + 1] & 0x7fffffffu]);
            st[h].z = ade_one(v[k + 2], st[h].z, lr[h].z, cid[k + 2], a.coef[cid[k + 2] & 0x7fffffffu]);
            st[h].w = ade_one(v[k + 3], st[h].w, lr[h].w, cid[k + 3], a.coef[cid[k + 3] & 0x7fffffffu]);
            *reinterpret_cast<float4*>(a.state + i0 + 4 * h) = st[h];
            if (qr >> 31) *reinterpret_cast<float4*>(a.lor + i0 + 4 * h) = lr[h];
        }
    } else {
        for (uint32_t k = 0; k < cnt; ++k) {
            float l = a.lor[i0 + k];
            a.state[i0 + k] = ade_one(v[k], a.state[i0 + k], l, cid[k], a.coef[cid[k] & 0x7fffffffu]);
            if (cid[k] >> 31) a.lor[i0 + k] = l;
        }
    }
}
__global__ void __launch_bounds__(ADE_T) k_ade(const float* __restrict__ F, const AdeDev a) {
    ade_body(F, a, blockIdx.x * ADE_T + threadIdx.x);
}

// Opt-in ADE apply step (the reference updates the state only; openEMS's
// Apply2Voltages / Apply2Current subtract it): after the apply-to-voltages
// phase (E side) or the post-current phase (H side), F -= state for every
// entry, in configuration order.  When no two entries share a field
// location, the entries are stored as runs over consecutive locations (as
// AdeRun with sel 0) and a thread takes ADE_V entries; otherwise entries are
// grouped by location (ascending) and a thread applies one location's
// entries in configuration order.
struct AdeApplyDev {
    uint32_t n;                     // entries (runs form) or locations (grouped form)
    const AdeRun* runs;             // runs form: + sentinel {n, 0, 0, 0}
    const uint32_t* grp_run;        // runs form: run of entry q*ADE_V
    const uint32_t* target;         // grouped form: location per group
    const uint32_t* off;            // grouped form: entries perm[off[g] .. off[g+1]) of group g
    const uint32_t* perm;
    const float* state;
};
__device__ __forceinline__ void ade_apply_runs_body(float* __restrict__ F, const AdeApplyDev& a, uint32_t q) {
    const uint32_t i0 = q * ADE_V;
    if (i0 >= a.n) return;
    const uint32_t cnt = min(ADE_V, a.n - i0);
    float st[ADE_V];
    if (cnt == ADE_V) {
#pragma unroll
        for (uint32_t h = 0; h < ADE_V / 4; ++h) {
            const float4 v = *reinterpret_cast<const float4*>(a.state + i0 + 4 * h);
            st[4 * h] = v.x; st[4 * h + 1] = v.y; st[4 * h + 2] = v.z; st[4 * h + 3] = v.w;
        }
    } else {
        for (uint32_t k = 0; k < ADE_V; ++k) st[k] = k < cnt ? a.state[i0 + k] : 0.f;
    }
    uint32_t lo = __ldg(a.grp_run + q);
    AdeRun r = a.runs[lo];
    uint32_t next = a.runs[lo + 1].entry;
#pragma unroll
    for (uint32_t k = 0; k < ADE_V; ++k) {
        if (k < cnt) {
            const uint32_t i = i0 + k;
            while (i >= next) { ++lo; r = a.runs[lo]; next = a.runs[lo + 1].entry; }
            const uint32_t t = r.idx + (i - r.entry);
            F[t] = __fsub_rn(F[t], st[k]);
        }
    }
}
__device__ __forceinline__ void ade_apply_grouped_body(float* __restrict__ F, const AdeApplyDev& a, uint32_t g) {
    if (g >= a.n) return;
    const uint32_t t = a.target[g];
    float v = F[t];
    for (uint32_t e = a.off[g]; e < a.off[g + 1]; ++e) v = __fsub_rn(v, a.state[a.perm[e]]);
    F[t] = v;
}
__global__ void __launch_bounds__(ADE_T) k_ade_apply_runs(float* __restrict__ F, const AdeApplyDev a) {
    ade_apply_runs_body(F, a, blockIdx.x * ADE_T + threadIdx.x);
}
__global__ void __launch_bounds__(256) k_ade_apply_grouped(float* __restrict__ F, const AdeApplyDev a) {
    ade_apply_grouped_body(F, a, blockIdx.x * blockDim.x + threadIdx.x);
}

// Lumped RLC (src/webgpu-fdtd.mjs:775-863, CPU order: pre before the core E
// update, apply after Mur apply).  Elements sharing a field cell are grouped.
struct RlcDev {
    uint32_t n, ngroups;
    const uint32_t* gtarget; const uint32_t* goff;  // groups over element ids
    const uint32_t* type;
    const float* p;        // 9 per element: i2v ilv vvd vv2 vj1 vj2 ib0 b1 b2
    float* vdn; float* jn; float* vil;
};
__global__ void k_rlc_pre(const RlcDev r) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.n) return;
    float* V = r.vdn + 3 * (size_t)i;
    V[2] = V[1];
    V[1] = V[0];
    if (r.type[i] == 0) {
        const float* p = r.p + 9 * (size_t)i;
        r.vil[i] = __fadd_rn(r.vil[i], __fmul_rn(__fmul_rn(p[0], p[1]), V[1]));
    }
}
__global__ void k_rlc_apply(float* __restrict__ F, const RlcDev r) {
    uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= r.ngroups) return;
    const uint32_t g = r.gtarget[gi];
    for (uint32_t e = r.goff[gi]; e < r.goff[gi + 1]; ++e) {
        float* V = r.vdn + 3 * (size_t)e;
        float* J = r.jn + 3 * (size_t)e;
        V[0] = F[g];
        J[2] = J[1];
        J[1] = J[0];
        if (r.type[e] == 1) {
            const float* p = r.p + 9 * (size_t)e;  // p: i2v ilv vvd vv2 vj1 vj2 ib0 b1 b2
            float in = __fsub_rn(V[0], r.vil[e]);
            in = __fadd_rn(in, __fmul_rn(p[3], V[2]));
            in = __fadd_rn(in, __fmul_rn(p[4], J[1]));
            in = __fadd_rn(in, __fmul_rn(p[5], J[2]));
            const float v0 = __fmul_rn(p[2], in);
            V[0] = v0;
            float j = __fmul_rn(p[6], __fsub_rn(v0, V[2]));
            j = __fsub_rn(j, __fmul_rn(__fmul_rn(p[7], p[6]), J[1]));
            j = __fsub_rn(j, __fmul_rn(__fmul_rn(p[8], p[6]), J[2]));
            J[0] = j;
            F[g] = v0;
        }
    }
}

// Steady-state energy accumulation (src/webgpu-fdtd.mjs:1054-1070); the
// sample counter is derived from numTS so the kernel needs no atomics.
__global__ void k_steady_state(const float* __restrict__ V, const StepState* st, uint32_t k, const uint32_t* idx,
                               uint32_t n, uint32_t period, float* e1, float* e2) {
    if (!st->ss_recording) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t sample = st->ss_base + (st->numTS + k - st->ss_start);
    const float v = V[idx[i]];
    const float e = __fmul_rn(v, v);
    if (sample < period) e1[i] = __fadd_rn(e1[i], e);
    else e2[i] = __fadd_rn(e2[i], e);
}

// Periodic / Bloch copy (src/webgpu-engine.mjs:519-584), one axis per launch.
struct PbcDev {
    uint32_t axis, volt, src, dst, fs0, fs1, b0, b1;
    uint32_t Nx, Ny, Nz, Pz;     // Pz: z pitch of the device layout
    float cosP, sinP;
    float* imag;       // Bloch imaginary parts of this axis, already offset
};
__global__ void k_pbc(float* __restrict__ F, const PbcDev p) {
    const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i1 = blockIdx.y * blockDim.y + threadIdx.y;
    if (i0 >= p.b0 || i1 >= p.b1) return;
    const uint32_t t0 = (p.axis + 1) % 3, t1 = (p.axis + 2) % 3;
    uint32_t sp[3], dp[3];
    if (p.axis == 0) { sp[0] = p.src; sp[1] = i0; sp[2] = i1; dp[0] = p.dst; dp[1] = i0; dp[2] = i1; }
    else if (p.axis == 1) { sp[0] = i1; sp[1] = p.src; sp[2] = i0; dp[0] = i1; dp[1] = p.dst; dp[2] = i0; }
    else { sp[0] = i0; sp[1] = i1; sp[2] = p.src; dp[0] = i0; dp[1] = i1; dp[2] = p.dst; }
    const size_t N = (size_t)p.Nx * p.Ny * p.Pz, NyNz = (size_t)p.Ny * p.Pz;
    const size_t s = (size_t)sp[0] * NyNz + (size_t)sp[1] * p.Pz + sp[2];
    const size_t d = (size_t)dp[0] * NyNz + (size_t)dp[1] * p.Pz + dp[2];
    const size_t s0 = t0 * N + s, d0 = t0 * N + d, s1 = t1 * N + s, d1 = t1 * N + d;
    if (p.sinP == 0.0f) {
        F[d0] = __fmul_rn(p.cosP, F[s0]);
        F[d1] = __fmul_rn(p.cosP, F[s1]);
    } else {
        const size_t fl = (size_t)i0 * p.fs1 + i1, face = (size_t)p.fs0 * p.fs1;
        float* im = p.imag + (p.volt ? 0 : 2 * face);
        float r0 = F[s0], q0 = im[fl];
        F[d0] = __fsub_rn(__fmul_rn(p.cosP, r0), __fmul_rn(p.sinP, q0));
        im[fl] = __fadd_rn(__fmul_rn(p.sinP, r0), __fmul_rn(p.cosP, q0));
        float r1 = F[s1], q1 = im[face + fl];
        F[d1] = __fsub_rn(__fmul_rn(p.cosP, r1), __fmul_rn(p.sinP, q1));
        im[face + fl] = __fadd_rn(__fmul_rn(p.sinP, r1), __fmul_rn(p.cosP, q1));
    }
}

// Probe gather (src/webgpu-engine.mjs:2593-2606 direct, :2644-2665 ring).
// Ring row = sample index derived from numTS: rows are written at
// (numTS+1) % interval == 0, counted from configure time.
struct RingDev {
    const uint32_t* idx;
    uint32_t G, interval, q0, maxS;
    float* ring;
};
__device__ __forceinline__ void gather_ring_body(const float* __restrict__ V, const float* __restrict__ C, const StepState* st,
                                                 uint32_t k, const RingDev& r, uint32_t i) {
    const uint32_t ts1 = st->numTS + k + 1;
    if (ts1 % r.interval != 0) return;
    const uint32_t q = ts1 / r.interval;
    if (q <= r.q0) return;
    const uint32_t s = q - 1 - r.q0;
    if (s >= r.maxS) return;
    if (i >= r.G) return;
    const uint32_t* idx = r.idx;
    const uint32_t G = r.G;
    float* ring = r.ring;
    const uint32_t t = idx[i];
    float* row = ring + (size_t)s * G * 2;
    row[2 * i] = V[t];
    row[2 * i + 1] = C[t];
}
__global__ void k_gather_ring(const float* __restrict__ V, const float* __restrict__ C, const StepState* st, uint32_t k,
                              const RingDev r) {
    gather_ring_body(V, C, st, k, r, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_gather(const float* __restrict__ V, const float* __restrict__ C, const uint32_t* idx, uint32_t G, float* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    out[2 * i] = V[idx[i]];
    out[2 * i + 1] = C[idx[i]];
}

__global__ void k_advance(StepState* st, uint32_t n) { st->numTS += n; }

// ---------------------------------------------------------------------------
// NF2FF running DFT (src/webgpu-engine.mjs:675-799) for F frequencies.  The
// phase omega*dT*n is formed in f64 and reduced modulo 2*pi before the
// cosine/sine (the reference forms it in f32, :777-782, which loses digits
// as n grows); the accumulation stays f32 in the reference's operand order.
// ---------------------------------------------------------------------------
constexpr int NF_MAX_FREQ = 16;
constexpr uint32_t NF_K = 16;       // steps of surface samples buffered between accumulator passes
// TFSF E corrections of up to two z planes (the box's z faces), applied by the
// fused update as it computes E instead of by the point pass after it: per
// step k_tfsf_face writes, for every TFSF target on those planes that has a
// single entry (Ex or Ey), the value the point pass would add (amplitude x
// interpolated incident signal) into a dense array [face][Ex, Ey][x][y] (row
// pitch ly, a multiple of 4 floats).  Every other cell holds -0.0f, which
// adds as the identity (x + -0 == x for every x, signed zeros included), as
// does an entry outside its signal window.
struct TfsfFace {
    uint32_t n;                     // faces (0: none)
    uint32_t z[2];
};
constexpr int TF_DY = 12;           // staged rows of a face array per plane (>= tile rows + halo, 16-byte inner box)
struct TfsfFaceDev {
    uint32_t n;                     // entries
    const uint32_t* dst;            // index into the face array
    const uint32_t* delay; const float* frac; const float* amp;
    const float* signal; uint32_t len, period;
    float* face;                    // [face][2][Nx][ly]
};
__device__ __forceinline__ void tfsf_face_body(const StepState* st, uint32_t k, const TfsfFaceDev& t, uint32_t i) {
    if (i >= t.n) return;
    const int64_t ts = (int64_t)st->numTS + k;
    float v = -0.0f;                // the identity when the entry adds nothing this step
    int64_t d = ts - (int64_t)t.delay[i];
    if (d >= 0) {
        if (t.period > 0) d %= (int64_t)t.period;
        if (d < (int64_t)t.len - 1) {   // point_sources_body<1>'s value, the same operations
            const float delta = t.frac[i];
            const float sig = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, delta), t.signal[d]), __fmul_rn(delta, t.signal[d + 1]));
            v = __fmul_rn(t.amp[i], sig);
        }
    }
    t.face[t.dst[i]] = v;
}
__global__ void k_tfsf_face(const StepState* st, uint32_t k, const TfsfFaceDev t) {
    tfsf_face_body(st, k, t, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_fill(float* p, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
// Largest element of a uint32 array, folded into *out (atomicMax; *out starts at 0).
__global__ void k_max_u32(const uint32_t* __restrict__ a, size_t n, uint32_t* out) {
    uint32_t m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = max(m, __ldg(a + i));
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

struct Nf2ffDev {
    uint32_t np, nf, maxTS, window;
    uint32_t Nx, Ny, Nz, Pz;        // Pz: z pitch of the device layout
    uint32_t off[6];
    const uint32_t* pts;
    const float* el;
    float* accE; float* accH;       // [f][pid*6+k]
    float* samp;                    // [NF_K][6][np]: buffered E, H samples
    double wdt[NF_MAX_FREQ];        // omega*dT per frequency (f64)
    float dT32, wnorm;
};
// Cell-interpolated E and H at surface point pid (webgpu-engine.mjs:690-761).
__device__ __forceinline__ void nf2ff_fields(const float* __restrict__ V, const float* __restrict__ C, const Nf2ffDev& d,
                                             uint32_t pid, float E[3], float Hh[3]) {
    const uint32_t ix = d.pts[3 * pid], iy = d.pts[3 * pid + 1], iz = d.pts[3 * pid + 2];
    const size_t Ny = d.Ny, Pz = d.Pz, N = (size_t)d.Nx * Ny * Pz, NyNz = Ny * Pz;
    auto fi = [&](uint32_t x, uint32_t y, uint32_t z) { return (size_t)x * NyNz + (size_t)y * Pz + z; };
    const size_t base = fi(ix, iy, iz);
    const bool atB = (ix >= d.Nx - 1) || (iy >= d.Ny - 1) || (iz >= d.Nz - 1);
    E[0] = E[1] = E[2] = 0.f;
    Hh[0] = Hh[1] = Hh[2] = 0.f;
    if (!atB) {
        const float elX = d.el[d.off[0] + ix], elY = d.el[d.off[1] + iy], elZ = d.el[d.off[2] + iz];
        float a = __fadd_rn(__fadd_rn(__fadd_rn(V[base], V[fi(ix, iy + 1, iz)]), V[fi(ix, iy + 1, iz + 1)]), V[fi(ix, iy, iz + 1)]);
        E[0] = __fdiv_rn(a, __fmul_rn(4.0f, elX));
        a = __fadd_rn(__fadd_rn(__fadd_rn(V[N + base], V[N + fi(ix, iy, iz + 1)]), V[N + fi(ix + 1, iy, iz + 1)]), V[N + fi(ix + 1, iy, iz)]);
        E[1] = __fdiv_rn(a, __fmul_rn(4.0f, elY));
        a = __fadd_rn(__fadd_rn(__fadd_rn(V[2 * N + base], V[2 * N + fi(ix + 1, iy, iz)]), V[2 * N + fi(ix + 1, iy + 1, iz)]), V[2 * N + fi(ix, iy + 1, iz)]);
        E[2] = __fdiv_rn(a, __fmul_rn(4.0f, elZ));
    }
    const uint32_t pos[3] = {ix, iy, iz}, lim[3] = {d.Nx, d.Ny, d.Nz};
    const size_t step[3] = {NyNz, Pz, 1};
    for (int n = 0; n < 3; ++n) {
        const float d0 = d.el[d.off[3 + n] + pos[n]];
        if (!(d0 > 0.0f)) continue;
        float h = __fdiv_rn(C[n * N + base], d0);
        if (pos[n] < lim[n] - 1) {
            const float d1 = d.el[d.off[3 + n] + pos[n] + 1];
            const float dr = __fdiv_rn(d0, __fadd_rn(d0, d1));
            const float hu = __fdiv_rn(C[n * N + base + step[n]], d1);
            h = __fadd_rn(__fmul_rn(h, __fsub_rn(1.0f, dr)), __fmul_rn(hu, dr));
        }
        Hh[n] = h;
    }
}

// Every step: the interpolated surface fields of the step into sample slot
// `slot` ([slot][6][np], E then H components).
__device__ __forceinline__ void nf2ff_sample_body(const float* __restrict__ V, const float* __restrict__ C, uint32_t slot,
                                                  const Nf2ffDev& d, uint32_t pid) {
    if (pid >= d.np) return;
    float E[3], Hh[3];
    nf2ff_fields(V, C, d, pid, E, Hh);
    float* s = d.samp + (size_t)slot * 6 * d.np + pid;
#pragma unroll
    for (int n = 0; n < 3; ++n) {
        s[(size_t)n * d.np] = E[n];
        s[(size_t)(3 + n) * d.np] = Hh[n];
    }
}
__global__ void __launch_bounds__(256) k_nf2ff_sample(const float* __restrict__ V, const float* __restrict__ C, uint32_t slot,
                                                      const Nf2ffDev d) {
    nf2ff_sample_body(V, C, slot, d, blockIdx.x * blockDim.x + threadIdx.x);
}

// Running DFT of `cnt` buffered steps (timesteps numTS+k0+1 .. numTS+k0+cnt,
// WebGPUEngine.iterate passes numTS+1, :2484): each accumulator is loaded
// once, takes the steps' terms in step order (the same operations, in the
// same order, as one accumulation per step) and is stored once.  Phase per
// step and frequency in f64 reduced mod 2*pi, then rounded to f32.
constexpr int NF_FG = 4;   // frequencies per register group
// Block body: `blk` is the block's index within this NF2FF set (all threads of a block call it).
__device__ __forceinline__ void nf2ff_flush_block(const StepState* st, uint32_t k0, uint32_t cnt, const Nf2ffDev& d, uint32_t blk) {
    __shared__ float tw[NF_K][NF_MAX_FREQ][4];
    __shared__ float sw[NF_K];
    const uint32_t ts0 = st->numTS + k0 + 1;
    const double two_pi = 6.283185307179586476925286766559;
    for (uint32_t i = threadIdx.x; i < cnt * d.nf; i += blockDim.x) {
        const uint32_t j = i / d.nf, f = i - j * d.nf;
        const double ts = (double)(ts0 + j);
        const double pe = fmod(d.wdt[f] * ts, two_pi);
        const double ph = fmod(d.wdt[f] * (ts + 0.5), two_pi);
        double sn, cs;
        sincos(pe, &sn, &cs);
        tw[j][f][0] = (float)cs; tw[j][f][1] = (float)sn;
        sincos(ph, &sn, &cs);
        tw[j][f][2] = (float)cs; tw[j][f][3] = (float)sn;
    }
    for (uint32_t j = threadIdx.x; j < cnt; j += blockDim.x) {
        float ww = 1.0f;
        if (d.window == 1 && d.maxTS > 1) ww = (float)(0.5 * (1.0 - cos(two_pi * (double)(ts0 + j) / (double)(d.maxTS - 1))));
        sw[j] = __fmul_rn(__fmul_rn(ww, d.wnorm), d.dT32);
    }
    __syncthreads();
    const uint32_t pid = blk * blockDim.x + threadIdx.x;
    if (pid >= d.np) return;
    for (uint32_t f0 = 0; f0 < d.nf; f0 += NF_FG) {
        float aE[NF_FG][6], aH[NF_FG][6];
#pragma unroll
        for (int g = 0; g < NF_FG; ++g) {
            if (f0 + g >= d.nf) break;
            const float* pE = d.accE + ((size_t)(f0 + g) * d.np + pid) * 6;
            const float* pH = d.accH + ((size_t)(f0 + g) * d.np + pid) * 6;
#pragma unroll
            for (int q = 0; q < 6; ++q) { aE[g][q] = pE[q]; aH[g][q] = pH[q]; }
        }
        for (uint32_t j = 0; j < cnt; ++j) {
            const float* s = d.samp + (size_t)j * 6 * d.np + pid;
            float E[3], Hh[3];
#pragma unroll
            for (int n = 0; n < 3; ++n) { E[n] = s[(size_t)n * d.np]; Hh[n] = s[(size_t)(3 + n) * d.np]; }
            const float w = sw[j];
#pragma unroll
            for (int g = 0; g < NF_FG; ++g) {
                if (f0 + g >= d.nf) break;
                const float ce = tw[j][f0 + g][0], se = -tw[j][f0 + g][1], ch = tw[j][f0 + g][2], sh = -tw[j][f0 + g][3];
#pragma unroll
                for (int n = 0; n < 3; ++n) {
                    aE[g][2 * n] = __fadd_rn(aE[g][2 * n], __fmul_rn(__fmul_rn(E[n], ce), w));
                    aE[g][2 * n + 1] = __fadd_rn(aE[g][2 * n + 1], __fmul_rn(__fmul_rn(E[n], se), w));
                    aH[g][2 * n] = __fadd_rn(aH[g][2 * n], __fmul_rn(__fmul_rn(Hh[n], ch), w));
                    aH[g][2 * n + 1] = __fadd_rn(aH[g][2 * n + 1], __fmul_rn(__fmul_rn(Hh[n], sh), w));
                }
            }
        }
#pragma unroll
        for (int g = 0; g < NF_FG; ++g) {
            if (f0 + g >= d.nf) break;
            float* pE = d.accE + ((size_t)(f0 + g) * d.np + pid) * 6;
            float* pH = d.accH + ((size_t)(f0 + g) * d.np + pid) * 6;
#pragma unroll
            for (int q = 0; q < 6; ++q) { pE[q] = aE[g][q]; pH[q] = aH[g][q]; }
        }
    }
}
__global__ void __launch_bounds__(256) k_nf2ff_flush(const StepState* st, uint32_t k0, uint32_t cnt, const Nf2ffDev d) {
    nf2ff_flush_block(st, k0, cnt, d, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Energy: sum over interior cells of volt^2 + curr^2 (src/webgpu-engine.mjs:
// 3071-3145), block-then-warp reduction with f64 block partials.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_energy(const float* __restrict__ V, const float* __restrict__ C, uint32_t Nx,
                                                uint32_t Ny, uint32_t Nz, uint32_t Pz, double* partial) {
    const size_t N = (size_t)Nx * Ny * Pz, inner = (size_t)(Nx - 1) * (Ny - 1) * (Nz - 1);
    const size_t iNz = Nz - 1, iNyNz = (size_t)(Ny - 1) * (Nz - 1);
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < inner; i += (size_t)gridDim.x * blockDim.x) {
        const size_t x = i / iNyNz, r = i - x * iNyNz, y = r / iNz, z = r - y * iNz;
        const size_t c = (x * Ny + y) * Pz + z;
        float s = 0.f;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float v = __ldg(V + n * N + c), h = __ldg(C + n * N + c);
            s = __fadd_rn(__fadd_rn(s, __fmul_rn(v, v)), __fmul_rn(h, h));
        }
        acc += (double)s;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}
__global__ void k_energy_final(const double* partial, uint32_t n, double* out) {
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) *out = v;
    }
}

// Variant of k_energy for the allocation-free entry point: block b sums the
// interior cells [b*cells, (b+1)*cells) (interior index order) into
// partial[b], so the number of partial sums grows with the grid and a fixed
// scratch array bounds the grid it accepts.  Same per-cell f32 arithmetic.
__global__ void __launch_bounds__(256) k_energy_ranges(const float* __restrict__ V, const float* __restrict__ C, uint32_t Nx,
                                                       uint32_t Ny, uint32_t Nz, uint32_t Pz, uint64_t cells,
                                                       double* partial) {
    const size_t N = (size_t)Nx * Ny * Pz, inner = (size_t)(Nx - 1) * (Ny - 1) * (Nz - 1);
    const size_t iNz = Nz - 1, iNyNz = (size_t)(Ny - 1) * (Nz - 1);
    const size_t lo = (size_t)blockIdx.x * cells, hi = min(lo + cells, inner);
    double acc = 0.0;
    for (size_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const size_t x = i / iNyNz, r = i - x * iNyNz, y = r / iNz, z = r - y * iNz;
        const size_t c = (x * Ny + y) * Pz + z;
        float s = 0.f;
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            const float v = __ldg(V + n * N + c), h = __ldg(C + n * N + c);
            s = __fadd_rn(__fadd_rn(s, __fmul_rn(v, v)), __fmul_rn(h, h));
        }
        acc += (double)s;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

// ---------------------------------------------------------------------------
// NF2FF far field (src/webgpu-engine.mjs:830-985): per angle (theta, phi),
//   N = sum_p area_p J_p e^{j k r^.r_p},  L = sum_p area_p M_p e^{j k r^.r_p}
// with the surface currents J = n x H, M = -n x E of each point's face, then
// E_theta, E_phi and the radiated intensity from the theta/phi projections.
//
// k_ff_prep turns every point into a 48-byte record: its position times
// k / 2 pi (the phase comes out in turns) and the two tangential components
// of area*J and area*M (a face with normal axis n carries currents along
// a = n+1 and b = n+2 only), with the points ordered by normal axis (the
// host passes the permutation).  k_ff_angles: a block takes FF_ANG angles; a
// warp holds FF_ANG/8 angles x FF_PL point lanes; the block stages tiles of
// records in shared memory and each thread sums its angle over every
// FF_PL-th point of the tile in f32 (only the two tangential accumulators of
// the segment's normal axis are live), adding the tile's sum into f64
// accumulators; the FF_PL point lanes of an angle are combined with warp
// shuffles and one lane forms the result in f64.  The phase is reduced to
// [-1/2, 1/2] turns before the hardware sine/cosine (error ~2^-21 there).
// ---------------------------------------------------------------------------
constexpr int FF_THREADS = 256;
constexpr int FF_PL = 4;                                  // point lanes per angle (a shuffle group)
constexpr int FF_ANG = FF_THREADS / FF_PL;                // angles per block
constexpr int FF_TILE = 512;                              // records per shared-memory tile
struct FfRecord { float4 pos; float4 j; float4 m; };     // pos: x,y,z in turns (w unused); j, m: a_re a_im b_re b_im
struct FarFieldDev {
    uint32_t np, nth, nph;
    uint32_t seg[4];                                      // records of normal axis n: [seg[n], seg[n+1])
    const FfRecord* rec;
    const float* theta; const float* phi;
    double fre, fim;                                      // k/(4 pi r) e^{-j k r} factor (re, im)
    float* out;                                           // 5 per angle
};
// One record per point, in the order perm (points grouped by normal axis).
__global__ void k_ff_prep(const float* __restrict__ meta, const float* __restrict__ accE, const float* __restrict__ accH,
                          const uint32_t* __restrict__ perm, uint32_t np, float kx, float cx, float cy, float cz,
                          FfRecord* __restrict__ rec) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const uint32_t p = perm[i];
    const float* m = meta + 8 * (size_t)p;
    const float* E = accE + 6 * (size_t)p;
    const float* H = accH + 6 * (size_t)p;
    const int nd = (int)m[3];
    const int ca = (nd + 1) % 3, cb = (nd + 2) % 3;
    const float s = m[4] * m[5];                          // normal sign x area
    FfRecord r;
    r.pos = make_float4((m[0] - cx) * kx, (m[1] - cy) * kx, (m[2] - cz) * kx, 0.f);
    // J_a = -s H_b, J_b = s H_a; M_a = s E_b, M_b = -s E_a  (J = n x H, M = -n x E)
    r.j = make_float4(-s * H[2 * cb], -s * H[2 * cb + 1], s * H[2 * ca], s * H[2 * ca + 1]);
    r.m = make_float4(s * E[2 * cb], s * E[2 * cb + 1], -s * E[2 * ca], -s * E[2 * ca + 1]);
    rec[i] = r;
}
// One (angle, point) pair: the record's tangential currents times e^{j 2 pi phase}
// added into a (N_a, N_b, L_a, L_b as re, im).
__device__ __forceinline__ void ff_pair(const FfRecord& r, float ux, float uy, float uz, float (&a)[8]) {
    float ph = r.pos.x * ux;
    ph = fmaf(r.pos.y, uy, ph);
    ph = fmaf(r.pos.z, uz, ph);
    ph -= rintf(ph);                                       // turns in [-1/2, 1/2]
    float sn, cs;
    __sincosf(6.2831853071795864f * ph, &sn, &cs);
    a[0] = fmaf(r.j.x, cs, fmaf(-r.j.y, sn, a[0])); a[1] = fmaf(r.j.y, cs, fmaf(r.j.x, sn, a[1]));
    a[2] = fmaf(r.j.z, cs, fmaf(-r.j.w, sn, a[2])); a[3] = fmaf(r.j.w, cs, fmaf(r.j.z, sn, a[3]));
    a[4] = fmaf(r.m.x, cs, fmaf(-r.m.y, sn, a[4])); a[5] = fmaf(r.m.y, cs, fmaf(r.m.x, sn, a[5]));
    a[6] = fmaf(r.m.z, cs, fmaf(-r.m.w, sn, a[6])); a[7] = fmaf(r.m.w, cs, fmaf(r.m.z, sn, a[7]));
}
// Records [p0, p1) of normal axis ND for this thread's angle (direction u).
template <int ND>
__device__ __forceinline__ void ff_segment(const FarFieldDev& d, FfRecord* tile, uint32_t p0, uint32_t p1, float ux, float uy,
                                           float uz, int q, bool live, double acc[12]) {
    constexpr int CA = (ND + 1) % 3, CB = (ND + 2) % 3;
    for (uint32_t t0 = p0; t0 < p1; t0 += FF_TILE) {
        const uint32_t nt = min((uint32_t)FF_TILE, p1 - t0);
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < nt; j += FF_THREADS) tile[j] = d.rec[t0 + j];
        __syncthreads();
        if (!live) continue;
        // four points per iteration into two sets of sums: their phases and
        // sines / cosines are independent, so several are in flight per thread
        float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // N_a, N_b, L_a, L_b (re, im)
        float t[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        uint32_t j = q;
        for (; j + 3 * FF_PL < nt; j += 4 * FF_PL) {
            ff_pair(tile[j], ux, uy, uz, s);
            ff_pair(tile[j + FF_PL], ux, uy, uz, t);
            ff_pair(tile[j + 2 * FF_PL], ux, uy, uz, s);
            ff_pair(tile[j + 3 * FF_PL], ux, uy, uz, t);
        }
        for (; j < nt; j += FF_PL) ff_pair(tile[j], ux, uy, uz, s);
#pragma unroll
        for (int i = 0; i < 8; ++i) s[i] += t[i];
        acc[2 * CA] += s[0]; acc[2 * CA + 1] += s[1];
        acc[2 * CB] += s[2]; acc[2 * CB + 1] += s[3];
        acc[6 + 2 * CA] += s[4]; acc[6 + 2 * CA + 1] += s[5];
        acc[6 + 2 * CB] += s[6]; acc[6 + 2 * CB + 1] += s[7];
    }
}
__global__ void __launch_bounds__(FF_THREADS) k_ff_angles(const FarFieldDev d) {
    __shared__ FfRecord tile[FF_TILE];
    const int lane = threadIdx.x & 31, q = lane % FF_PL;
    const uint32_t A = d.nth * d.nph;
    const uint32_t a = blockIdx.x * FF_ANG + threadIdx.x / FF_PL;
    const bool live = a < A;
    float sT = 0.f, cT = 1.f, sP = 0.f, cP = 1.f;
    if (live) {
        sincosf(d.theta[a / d.nph], &sT, &cT);
        sincosf(d.phi[a % d.nph], &sP, &cP);
    }
    const float ux = sT * cP, uy = sT * sP, uz = cT;
    double acc[12];                                      // N_x, N_y, N_z, L_x, L_y, L_z (re, im)
#pragma unroll
    for (int i = 0; i < 12; ++i) acc[i] = 0.0;
    ff_segment<0>(d, tile, d.seg[0], d.seg[1], ux, uy, uz, q, live, acc);
    ff_segment<1>(d, tile, d.seg[1], d.seg[2], ux, uy, uz, q, live, acc);
    ff_segment<2>(d, tile, d.seg[2], d.seg[3], ux, uy, uz, q, live, acc);
    // the FF_PL point lanes of this angle are adjacent lanes of one warp
#pragma unroll
    for (int i = 0; i < 12; ++i)
#pragma unroll
        for (int o = 1; o < FF_PL; o <<= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    if (!live || q != 0) return;
    const double cTcP = (double)cT * cP, cTsP = (double)cT * sP;
    auto proj_t = [&](int b, int c) { return acc[b + c] * cTcP + acc[b + 2 + c] * cTsP - acc[b + 4 + c] * (double)sT; };
    auto proj_p = [&](int b, int c) { return acc[b + 2 + c] * (double)cP - acc[b + c] * (double)sP; };
    const double Ntr = proj_t(0, 0), Nti = proj_t(0, 1), Npr = proj_p(0, 0), Npi = proj_p(0, 1);
    const double Ltr = proj_t(6, 0), Lti = proj_t(6, 1), Lpr = proj_p(6, 0), Lpi = proj_p(6, 1);
    const double Z0 = 376.73031346177066;
    const double ar = Lpr + Z0 * Ntr, ai = Lpi + Z0 * Nti;
    const double Etr = -(d.fre * ar - d.fim * ai), Eti = -(d.fre * ai + d.fim * ar);
    const double br = Ltr - Z0 * Npr, bi = Lti - Z0 * Npi;
    const double Epr = d.fre * br - d.fim * bi, Epi = d.fre * bi + d.fim * br;
    float* o = d.out + 5 * (size_t)a;
    o[0] = (float)((Etr * Etr + Eti * Eti + Epr * Epr + Epi * Epi) / (2 * Z0));
    o[1] = (float)Etr; o[2] = (float)Eti; o[3] = (float)Epr; o[4] = (float)Epi;
}

}  // namespace efs
