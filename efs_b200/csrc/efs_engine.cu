// efs_engine.cu — host side of the B200 FDTD engine behind include/efs.h.
//
// One engine = one grid resident in HBM + one CUDA stream.  A timestep is the
// reference's phase sequence (CPUFDTDEngine.step, src/webgpu-fdtd.mjs:1129-
// 1172, with the PBC and NF2FF/gather passes where WebGPUEngine.iterate puts
// them, src/webgpu-engine.mjs:2448-2499) mapped onto kernels:
//
//   steady-state accumulate | ADE(volt) | Mur pre | RLC pre | ADE(curr)  (sparse)
//   E of UPML cells (k_pml_e)
//   E and H of every other cell in one pass (k_fused_tma)
//   H of UPML cells (k_pml_h)
//   TFSF(volt) | PBC(volt) | Mur post | excitation | Mur apply | RLC apply (sparse)
//   [ADE apply to E]
//   H of cells next to those E writes (k_deferred_h)
//   TFSF(curr) | PBC(curr) | [ADE apply to H]                             (sparse)
//   NF2FF sample/flush | probe ring
//
// Reads that the reference makes between the UPML pre-update and the core
// update (ADE, Mur pre) are redirected to the region's flux array, which is
// what the field holds at that moment, so fusing pre/post into the UPML
// passes keeps the reference's results.  Time-dependent parameters come from
// a device-resident step counter, so `iterate(n)` replays a captured CUDA
// graph of the whole step sequence.
//
// Device layout: NIJK with z rows padded to a multiple of 4 floats (pitch
// Pz; efs_fused.cuh).  Every index a caller passes is in the reference's
// unpadded NIJK order and is translated once, at configure time; field
// transfers (getFields, uploadFields) repack rows with 2D copies.
#include "../../include/efs.h"
#include "efs_kernels.cuh"
#include "efs_fused.cuh"
#include "efs_tma.cuh"
#include "efs_host.h"

#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace efs;

namespace {

thread_local std::string g_create_error = "no error";

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { reset(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct EfsError {
    efs_status code;
    std::string msg;
};

[[noreturn]] void fail(efs_status code, const std::string& msg) { throw EfsError{code, msg}; }

void ck(cudaError_t err, const char* what) {
    if (err != cudaSuccess) fail(err == cudaErrorMemoryAllocation ? EFS_ERR_OOM : EFS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

inline uint32_t blocks(size_t n, uint32_t t) { return (uint32_t)((n + t - 1) / t); }

using efs_host::host_threads;
using efs_host::parallel_chunks;

// An engine's pinned host words: the status word its kernels set through a
// mapped pointer (bit 0: a bounded device wait ran out) and two slots of
// energy results.  They are 32-byte slots of mapped, portable pinned pages
// that live as long as the process and are handed out again after an
// engine's destruction, so creating and destroying engines neither allocates
// nor frees pinned memory (cudaFreeHost of a mapped page has taken up to
// 0.6 s on B200 hosts).
struct HostSlot {
    uint32_t status;
    uint32_t pad0;
    double energy[2];
    uint64_t pad1;
};
static_assert(sizeof(HostSlot) == 32, "host slot layout");
std::mutex g_slot_mu;
std::vector<HostSlot*> g_free_slots;

HostSlot* host_slot_get() {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    if (g_free_slots.empty()) {
        constexpr size_t PAGE = 4096;
        void* p = nullptr;
        ck(cudaHostAlloc(&p, PAGE, cudaHostAllocMapped | cudaHostAllocPortable), "cudaHostAlloc");
        HostSlot* s = static_cast<HostSlot*>(p);
        for (size_t i = PAGE / sizeof(HostSlot); i-- > 0;) g_free_slots.push_back(s + i);
    }
    HostSlot* s = g_free_slots.back();
    g_free_slots.pop_back();
    memset(s, 0, sizeof(*s));
    return s;
}

void host_slot_put(HostSlot* s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(g_slot_mu);
    g_free_slots.push_back(s);
}

}  // namespace

struct efs_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error = "no error";
    size_t dev_bytes = 0;

    bool inited = false;
    uint32_t Nx = 0, Ny = 0, Nz = 0;
    size_t N = 0;               // cells of the caller's grid (component stride of caller indices)
    uint32_t Pz = 0;            // device z pitch: Nz rounded up to a multiple of 4
    size_t Nd = 0;              // device component stride Nx*Ny*Pz
    DevBuf volt, curr;          // fields (parity 0)
    DevBuf volt_b, curr_b;      // second buffers (parity 1): a step reads one parity and writes the other
    int cur = 0;                // parity holding the current fields
    uint32_t xchunk = 32;       // x-planes per CTA of the fused kernel (efs_set_plane_depth)
    uint64_t wait_ns = 1000000000ull;   // limit of the fused kernel's bounded waits
    uint32_t skip_plane = ~0u;          // diagnostics (efs_debug_set_wait): a plane whose loads are never issued
    DevBuf defer_cells;
    uint32_t defer_n = 0;
    std::vector<uint32_t> h_exc_targets, h_tfsf_v_targets, h_mur_apply, h_rlc_series;
    bool indexed = false;
    DevBuf mat, table, vv, vi, ii, iv;
    uint32_t ntable = 0;
    DevBuf state;            // StepState
    uint32_t numTS = 0;      // host mirror
    StepState hstate{};

    // excitation
    bool exc_on = false;
    DevBuf exc_target, exc_off, exc_delay, exc_amp, exc_signal;
    uint32_t exc_groups = 0, exc_len = 0, exc_period = 0;

    // UPML
    struct Region {
        uint32_t s[3], n[3];
        size_t total;
        DevBuf vv, vvfo, vvfn, ii, iifo, iifn, vflux, cflux, vflux_b, cflux_b;
        DevBuf cidx, ctab;      // compact coefficients (empty when the region has too many distinct tuples)
                                // vv..iifn stay empty when the compact table serves every cell (no overlap)
        float* vf(int p) const { return (p && vflux_b.p) ? vflux_b.as<float>() : vflux.as<float>(); }
        float* cf(int p) const { return (p && cflux_b.p) ? cflux_b.as<float>() : cflux.as<float>(); }
    };
    std::vector<std::unique_ptr<Region>> pml;
    DevBuf vflux_ptrs[2], cflux_ptrs[2];

    float* vbuf(int p) const { return p ? volt_b.as<float>() : volt.as<float>(); }
    float* cbuf(int p) const { return p ? curr_b.as<float>() : curr.as<float>(); }
    float* vcur() const { return vbuf(cur); }
    float* ccur() const { return cbuf(cur); }
    static int pnext(int p) { return 1 - p; }

    // Caller index (n*N + x*Ny*Nz + y*Nz + z, the reference's NIJK order) ->
    // device index (n*Nd + (x*Ny + y)*Pz + z).
    // 32-bit arithmetic holds: 3 * Nd < 2^32 (alloc_fields) and N <= Nd.
    uint32_t dev_index(uint32_t f) const {
        if (Pz == Nz) return f;                              // no padding: the layouts coincide
        const uint32_t N32 = (uint32_t)N, nyz = Ny * Nz;
        const uint32_t n = f / N32, cell = f - n * N32;
        const uint32_t x = cell / nyz, r = cell - x * nyz, y = r / Nz, z = r - y * Nz;
        return n * (uint32_t)Nd + (x * Ny + y) * Pz + z;
    }
    size_t dev_cell(uint64_t x, uint64_t y, uint64_t z) const { return (size_t)((x * Ny + y) * Pz + z); }
    // Host array of `comps` components in the caller's layout -> device
    // buffer in the padded layout (pad cells zero).
    void upload_padded(DevBuf& b, const void* src, size_t comps, size_t elem = 4) {
        alloc(b, comps * Nd * elem, Pz != Nz);
        rows_transfer(b.p, const_cast<void*>(src), comps * Nx * Ny, elem, true);
    }
    // Row transfers between the caller's unpadded rows (pitch Nz) in host
    // memory and the padded device rows (pitch Pz).  Equal pitches: one
    // linear copy.  Otherwise each chunk of rows crosses PCIe as one linear
    // copy through a device staging buffer and is repacked by a device-to-
    // device 2D copy (a 2D copy from pageable host memory moves row by row).
    // Synchronous with the host on return.
    void rows_transfer(void* dev, void* host, size_t rows, size_t elem, bool to_device) {
        const size_t w = (size_t)Nz * elem, dp = (size_t)Pz * elem;
        if (Pz == Nz) {
            ck(cudaMemcpyAsync(to_device ? dev : host, to_device ? host : dev, rows * w,
                               to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, stream), "row transfer");
            sync("row transfer");
            return;
        }
        const size_t chunk = std::max<size_t>(1, std::min(rows, ((size_t)64 << 20) / w));
        DevBuf stage;
        alloc(stage, chunk * w, false);
        for (size_t r0 = 0; r0 < rows; r0 += chunk) {
            const size_t n = std::min(chunk, rows - r0);
            uint8_t* d = static_cast<uint8_t*>(dev) + r0 * dp;
            uint8_t* h = static_cast<uint8_t*>(host) + r0 * w;
            if (to_device) {
                ck(cudaMemcpyAsync(stage.p, h, n * w, cudaMemcpyHostToDevice, stream), "row transfer");
                ck(cudaMemcpy2DAsync(d, dp, stage.p, w, w, n, cudaMemcpyDeviceToDevice, stream), "row repack");
            } else {
                ck(cudaMemcpy2DAsync(stage.p, w, d, dp, w, n, cudaMemcpyDeviceToDevice, stream), "row repack");
                ck(cudaMemcpyAsync(h, stage.p, n * w, cudaMemcpyDeviceToHost, stream), "row transfer");
            }
        }
        sync("row transfer");   // the staging buffer is freed on return
    }
    void copy_fields_out(float* dst, const float* dev) {
        rows_transfer(const_cast<float*>(dev), dst, 3 * (size_t)Nx * Ny, 4, false);
    }
    void copy_fields_in(float* dev, const float* src) {
        rows_transfer(dev, const_cast<float*>(src), 3 * (size_t)Nx * Ny, 4, true);
    }

    // Mur (host copies kept to rebuild read redirects)
    bool mur_on = false;
    std::vector<uint32_t> h_mur_normal, h_mur_shifted;
    DevBuf mur_coeff, mur_pre_normal, mur_pre_shifted, mur_shifted, mur_apply_target, mur_apply_src, mur_saved;
    uint32_t mur_n = 0, mur_napply = 0;

    // TFSF
    bool tfsf_on = false;
    DevBuf tfsf_signal;
    uint32_t tfsf_len = 0, tfsf_period = 0;
    struct PointSet { DevBuf target, off, delay, amp, frac; uint32_t groups = 0; };
    PointSet tfsf_v, tfsf_c;

    // ADE
    bool ade_on = false;
    struct AdeSide {
        std::vector<uint32_t> h_field;   // dir*N + pos
        std::vector<uint32_t> h_coef;    // per entry: coefficient tuple id, bit 31 set for Lorentz
        DevBuf runs, grp_run, coef, state, lor;
        uint32_t n = 0;
        // apply step (efs_configure_ade_apply): runs over the field locations
        // when no two entries share one, else entries grouped by location
        bool app_runs = true;
        uint32_t app_n = 0;                          // entries (runs form) or locations (grouped form)
        DevBuf app_run, app_grp, app_target, app_off, app_perm;
        // A side whose coefficients are all zero keeps its state at +0 while
        // the fields stay finite (0*x + 0*y rounds to +0), so its kernel is
        // skipped until a restored state may have put other values there.
        bool zero = false, clean = true;
        bool live() const { return n && !(zero && clean); }
    };
    AdeSide ade_v, ade_c;
    bool ade_apply = false;      // opt-in: subtract the ADE state from E / H after the update (no reference counterpart)

    // RLC
    bool rlc_on = false;
    DevBuf rlc_gtarget, rlc_goff, rlc_type, rlc_p, rlc_vdn, rlc_jn, rlc_vil;
    uint32_t rlc_n = 0, rlc_groups = 0;
    std::vector<uint32_t> rlc_perm;   // device element order -> caller's element order
    std::vector<uint32_t> mur_perm;   // device Mur entry order -> caller's entry order

    // steady state
    bool ss_on = false, ss_recording = false;
    DevBuf ss_idx, ss_e1, ss_e2;
    uint32_t ss_n = 0, ss_period = 0;
    float ss_threshold = 1e-6f;
    uint32_t ss_count_before = 0;   // samples taken before the current recording window

    // PBC
    bool pbc_on = false;
    struct PbcAxis { uint32_t axis; float c, s; size_t imag_off; };
    std::vector<PbcAxis> pbc_axes;
    DevBuf pbc_imag;

    // probes
    DevBuf gd_idx, gd_out;
    uint32_t gd_n = 0;
    bool ring_on = false;
    DevBuf ring_idx, ring;
    std::vector<uint32_t> h_nf_pts;   // host copy of the NF2FF points (plan checks)
    uint32_t ring_n = 0, ring_max = 0, ring_interval = 1, ring_q0 = 0;

    // NF2FF
    bool nf_on = false;
    DevBuf nf_pts, nf_el, nf_E, nf_H, nf_samp;
    Nf2ffDev nf{};
    float ff_ms[2] = {0.f, 0.f};     // device time of the last far-field call: point records, angle sums

    // energy (lagged, double-buffered like computeEnergy :2974-3021)
    DevBuf en_partial, en_result;
    HostSlot* slot = nullptr;        // pinned host words of this engine (status, energy)
    double* en_host = nullptr;       // pinned, 2 slots
    // device status word in mapped pinned host memory: bit 0 = a bounded device wait ran out
    uint32_t* h_status = nullptr;
    uint32_t* d_status = nullptr;
    cudaEvent_t en_event[2] = {nullptr, nullptr};
    int en_idx = 0;
    bool en_pending = false;
    double en_last = 0.0;

    // graphs
    bool plan_dirty = true;
    std::map<uint32_t, cudaGraphExec_t> graphs;

    ~efs_engine() {
        drop_graphs();
        for (auto& ev : en_event) if (ev) cudaEventDestroy(ev);
        host_slot_put(slot);
        if (stream) cudaStreamDestroy(stream);
    }

    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
    void dirty() { plan_dirty = true; drop_graphs(); }

    void alloc(DevBuf& b, size_t bytes, bool zero = true) {
        b.reset();
        if (bytes == 0) bytes = 4;
        ck(cudaMalloc(&b.p, bytes), "cudaMalloc");
        b.bytes = bytes;
        if (zero) ck(cudaMemsetAsync(b.p, 0, bytes, stream), "cudaMemsetAsync");
    }
    template <typename T>
    void upload(DevBuf& b, const T* src, size_t n) {
        alloc(b, n * sizeof(T), false);
        if (n) ck(cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
        sync("upload sync");   // caller may free its buffer on return
    }
    template <typename T>
    void upload(DevBuf& b, const std::vector<T>& v) { upload(b, v.data(), v.size()); }

    // Synchronize the stream and turn a device status report into an error.
    void sync(const char* what) {
        ck(cudaStreamSynchronize(stream), what);
        const uint32_t st = *(volatile uint32_t*)h_status;
        if (st) {
            *(volatile uint32_t*)h_status = 0;
            fail(EFS_ERR_TIMEOUT, std::string(what) + ": a bounded device wait for a TMA plane load ran out");
        }
    }

    void need_init() const { if (!inited) fail(EFS_ERR_STATE, "engine not initialised: call efs_init first"); }
    // stable radix sort of (key, value) pairs by key (efs_host.h)
    static void radix_sort_pairs(std::vector<uint32_t>& key, std::vector<uint32_t>& val) {
        efs_host::radix_sort_pairs(key, val);
    }

    void check_idx3(const uint32_t* p, size_t n, const char* what) const {
        for (size_t i = 0; i < n; ++i)
            if (p[i] >= 3 * N) fail(EFS_ERR_INVALID, std::string(what) + ": index out of range");
    }

    FusedGrid fused_grid(int p) const {
        FusedGrid g;
        g.Nx = Nx; g.Ny = Ny; g.Nz = Nz; g.xchunk = xchunk; g.Pz = Pz;
        g.N = Nd; g.NyNz = (size_t)Ny * Pz;
        g.V0 = vbuf(p); g.H0 = cbuf(p); g.V1 = vbuf(1 - p); g.H1 = cbuf(1 - p);
        g.mat = mat.as<uint32_t>(); g.table = table.as<float>();
        g.vv = vv.as<float>(); g.vi = vi.as<float>(); g.ii = ii.as<float>(); g.iv = iv.as<float>();
        g.status = d_status;
        g.wait_ns = wait_ns;
        g.skip_plane = skip_plane;
        g.tf = tf;
        return g;
    }
    // UPML set whose flux pointers are the parity-p buffers
    PmlSet pml_set(int p = 0) const {
        PmlSet s;
        memset(&s, 0, sizeof(s));
        s.count = (int)pml.size();
        for (size_t r = 0; r < pml.size(); ++r) {
            const Region& R = *pml[r];
            for (int d = 0; d < 3; ++d) { s.r[r].s[d] = R.s[d]; s.r[r].n[d] = R.n[d]; }
            s.r[r].vv = R.vv.as<float>(); s.r[r].vvfo = R.vvfo.as<float>(); s.r[r].vvfn = R.vvfn.as<float>();
            s.r[r].ii = R.ii.as<float>(); s.r[r].iifo = R.iifo.as<float>(); s.r[r].iifn = R.iifn.as<float>();
            s.r[r].vflux = R.vf(p); s.r[r].cflux = R.cf(p);
            s.r[r].cidx = R.cidx.p ? R.cidx.as<uint16_t>() : nullptr;
            s.r[r].ctab = R.cidx.p ? R.ctab.as<float4>() : nullptr;
        }
        return s;
    }

    // Location a read of device field index `field_idx` sees after the UPML
    // pre-update: the flux slot of the last region containing the cell, else
    // the field itself.
    ReadLoc redirect(uint32_t field_idx) const {
        ReadLoc l{0, field_idx};
        if (pml.empty()) return l;
        const uint32_t n = field_idx / (uint32_t)Nd;
        const uint32_t cell = field_idx - n * (uint32_t)Nd;
        const uint32_t row = cell / Pz, z = cell - row * Pz, x = row / Ny, y = row - x * Ny;
        for (size_t r = 0; r < pml.size(); ++r) {
            const Region& R = *pml[r];
            if ((x - R.s[0]) < R.n[0] && (y - R.s[1]) < R.n[1] && (z - R.s[2]) < R.n[2]) {
                size_t nyz = (size_t)R.n[1] * R.n[2];
                size_t p = (size_t)n * R.n[0] * nyz + (size_t)(x - R.s[0]) * nyz + (size_t)(y - R.s[1]) * R.n[2] + (z - R.s[2]);
                l.sel = (uint32_t)r + 1;
                l.idx = (uint32_t)p;
            }
        }
        return l;
    }

    // Rebuild everything that depends on more than one configure call.
    void build_plan() {
        if (!plan_dirty) return;
        nf_pair = nf2ff_clear_of_pml();
        for (int p = 0; p < 2; ++p) {
            std::vector<float*> vp, cp;
            for (auto& r : pml) { vp.push_back(r->vf(p)); cp.push_back(r->cf(p)); }
            if (vp.empty()) { vp.push_back(nullptr); cp.push_back(nullptr); }
            upload(vflux_ptrs[p], vp);
            upload(cflux_ptrs[p], cp);
        }
        plan_tfsf_faces();
        build_deferred();
        if (mur_on) {
            std::vector<ReadLoc> rn(mur_n), rs(mur_n);
            parallel_chunks(mur_n, host_threads(mur_n), [&](unsigned, size_t lo, size_t hi) {
                for (size_t i = lo; i < hi; ++i) { rn[i] = redirect(h_mur_normal[i]); rs[i] = redirect(h_mur_shifted[i]); }
            });
            upload(mur_pre_normal, rn);
            upload(mur_pre_shifted, rs);
        }
        for (AdeSide* s : {&ade_v, &ade_c}) {
            if (!s->n) continue;
            std::vector<AdeRun> runs;
            ReadLoc prev{0, 0};
            for (uint32_t i = 0; i < s->n; ++i) {
                const ReadLoc l = redirect(s->h_field[i]);
                const uint32_t c = s->h_coef[i];
                if (i == 0 || l.sel != prev.sel || l.idx != prev.idx + 1 || c != runs.back().coef)
                    runs.push_back(AdeRun{i, l.sel, l.idx, c});
                prev = l;
            }
            if (runs.size() >= 0x80000000u) fail(EFS_ERR_INVALID, "too many ADE runs");
            const uint32_t nq = (s->n + ADE_V - 1) / ADE_V;   // groups of ADE_V entries
            std::vector<uint32_t> qr(nq);
            size_t r = 0;
            for (uint32_t q = 0; q < nq; ++q) {
                const uint32_t i0 = q * ADE_V, i1 = std::min(s->n, i0 + ADE_V);
                while (r + 1 < runs.size() && runs[r + 1].entry <= i0) ++r;
                uint32_t lor = 0;
                for (size_t k = r; k < runs.size() && runs[k].entry < i1; ++k) lor |= runs[k].coef & 0x80000000u;
                qr[q] = (uint32_t)r | lor;
            }
            runs.push_back(AdeRun{s->n, 0, 0, 0});      // sentinel: ends the last run
            upload(s->runs, runs);
            upload(s->grp_run, qr);
            if (ade_apply) build_ade_apply(*s);
        }
        plan_dirty = false;
    }

    // Apply-step plan of one ADE side: runs over consecutive field locations
    // when every entry has its own location, else groups per location.
    void build_ade_apply(AdeSide& s) {
        std::vector<uint64_t> seen((3 * Nd + 63) / 64, 0);   // one bit per device field location
        s.app_runs = true;
        for (uint32_t f : s.h_field) {
            const uint64_t bit = 1ull << (f & 63);
            if (seen[f >> 6] & bit) { s.app_runs = false; break; }
            seen[f >> 6] |= bit;
        }
        if (s.app_runs) {
            std::vector<AdeRun> runs;
            for (uint32_t i = 0; i < s.n; ++i)
                if (i == 0 || s.h_field[i] != s.h_field[i - 1] + 1) runs.push_back(AdeRun{i, 0, s.h_field[i], 0});
            const uint32_t nq = (s.n + ADE_V - 1) / ADE_V;
            std::vector<uint32_t> qr(nq);
            size_t r = 0;
            for (uint32_t q = 0; q < nq; ++q) {
                while (r + 1 < runs.size() && runs[r + 1].entry <= q * ADE_V) ++r;
                qr[q] = (uint32_t)r;
            }
            runs.push_back(AdeRun{s.n, 0, 0, 0});
            upload(s.app_run, runs);
            upload(s.app_grp, qr);
            s.app_n = s.n;
        } else {
            std::vector<uint32_t> ut, off, perm;
            group_by(s.h_field, ut, off, perm);
            upload(s.app_target, ut);
            upload(s.app_off, off);
            upload(s.app_perm, perm);
            s.app_n = (uint32_t)ut.size();
        }
    }
    AdeApplyDev ade_apply_dev(const AdeSide& s) const {
        return AdeApplyDev{s.app_n, s.app_run.as<AdeRun>(), s.app_grp.as<uint32_t>(), s.app_target.as<uint32_t>(),
                           s.app_off.as<uint32_t>(), s.app_perm.as<uint32_t>(), s.state.as<float>()};
    }
    void launch_ade_apply(const AdeSide& s, float* F) {
        if (s.app_runs) k_ade_apply_runs<<<blocks(s.app_n, ADE_BLOCK), ADE_T, 0, stream>>>(F, ade_apply_dev(s));
        else k_ade_apply_grouped<<<blocks(s.app_n, 256), 256, 0, stream>>>(F, ade_apply_dev(s));
    }

    // H cells whose curl reads an E value rewritten by a sparse post-update
    // operation (TFSF, PBC, Mur apply, excitation, series RLC) are updated
    // after those operations by k_deferred_h.  Targets are device indices.
    // TFSF face corrections applied in the core update (TfsfFace): up to two z
    // planes holding many single-entry Ex/Ey targets (the box's z faces).
    // Their entries leave the point pass, and the deferred set: the H cells
    // next to them see the corrected E inside the core update.
    std::vector<efs_tfsf_point> h_tfsf_v;      // the caller's voltage-side TFSF points
    TfsfFace tf{0, {0, 0}};
    uint32_t tf_n = 0, tf_ly = 0;
    DevBuf tf_face, tf_dst, tf_delay, tf_frac, tf_amp;
    void plan_tfsf_faces();
    TfsfFaceDev tf_dev() const {
        return TfsfFaceDev{tf_n, tf_dst.as<uint32_t>(), tf_delay.as<uint32_t>(), tf_frac.as<float>(), tf_amp.as<float>(),
                           tfsf_signal.as<float>(), tfsf_len, tfsf_period, tf_face.as<float>()};
    }
    // tensor map of the face array: dims y (pitch tf_ly), x, component, face; box TF_DY x 1 x 2 x faces
    CUtensorMap tf_map() const {
        const cuuint64_t dims[4] = {Ny, Nx, 2, tf.n};
        const cuuint64_t strides[3] = {(cuuint64_t)tf_ly * 4, (cuuint64_t)Nx * tf_ly * 4, (cuuint64_t)2 * Nx * tf_ly * 4};
        const uint32_t box[4] = {(uint32_t)TF_DY, 1, 2, tf.n};
        return encode_map(tf_face.p, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, dims, strides, box);
    }

    void build_deferred() {
        defer_n = 0;
        std::vector<uint32_t> mod;   // modified E entries as n*Nd + device cell
        auto add = [&](const std::vector<uint32_t>& v) { mod.insert(mod.end(), v.begin(), v.end()); };
        if (tfsf_on) add(h_tfsf_v_targets);
        if (exc_on) add(h_exc_targets);
        if (mur_on) add(h_mur_apply);
        if (rlc_on) add(h_rlc_series);
        if (ade_apply && ade_v.live()) add(ade_v.h_field);
        const uint32_t nl[3] = {Nx, Ny, Nz};
        if (pbc_on)
            for (auto& a : pbc_axes) {
                uint32_t t0 = (a.axis + 1) % 3, t1 = (a.axis + 2) % 3;
                for (uint32_t i0 = 0; i0 < nl[t0]; ++i0)
                    for (uint32_t i1 = 0; i1 < nl[t1]; ++i1) {
                        uint32_t p[3];
                        p[a.axis] = 0; p[t0] = i0; p[t1] = i1;
                        if (a.axis == 1) { p[0] = i1; p[2] = i0; }   // face_to_grid order of the reference
                        const size_t c = dev_cell(p[0], p[1], p[2]);
                        mod.push_back((uint32_t)(t0 * Nd + c));
                        mod.push_back((uint32_t)(t1 * Nd + c));
                    }
            }
        if (mod.empty()) return;
        // 32-bit cell arithmetic: Nd < 2^32 / 3
        const uint32_t NyPz = Ny * Pz, Nd32 = (uint32_t)Nd;
        std::vector<uint32_t> bits((Nd + 31) / 32, 0);
        auto mark = [&](uint32_t c) { __atomic_fetch_or(&bits[c >> 5], 1u << (c & 31), __ATOMIC_RELAXED); };
        parallel_chunks(mod.size(), host_threads(mod.size()), [&](unsigned, size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i) {
                const uint32_t f = mod[i], n = f / Nd32, cell = f - n * Nd32;
                const uint32_t row = cell / Pz, z = cell - row * Pz, x = row / Ny, y = row - x * Ny;
                // E_n(m) appears in the curls of H at m, m - e_a, m - e_b (a, b != n)
                mark(cell);
                if (n != 0 && x > 0) mark(cell - NyPz);
                if (n != 1 && y > 0) mark(cell - Pz);
                if (n != 2 && z > 0) mark(cell - 1);
            }
        });
        // UPML cells are left to k_pml_h, which runs after the E-side
        // operations: clear each region row's z run [c, c + n_z)
        for (auto& R : pml)
            for (uint32_t x = R->s[0]; x < R->s[0] + R->n[0]; ++x)
                for (uint32_t y = R->s[1]; y < R->s[1] + R->n[1]; ++y) {
                    uint32_t c = (x * Ny + y) * Pz + R->s[2];
                    const uint32_t end = c + R->n[2];
                    while (c < end) {
                        const uint32_t w = c >> 5, b0 = c & 31, b1 = std::min<uint32_t>(32, b0 + (end - c));
                        const uint32_t m = (b1 == 32 ? ~0u : ((1u << b1) - 1)) & ~((1u << b0) - 1);
                        bits[w] &= ~m;
                        c += b1 - b0;
                    }
                }
        // marked cells in ascending order: per-chunk counts, then each chunk
        // writes its cells at its offset
        const size_t W = bits.size();
        const unsigned T = host_threads(W);
        std::vector<size_t> at(T + 1, 0);
        parallel_chunks(W, T, [&](unsigned t, size_t lo, size_t hi) {
            size_t c = 0;
            for (size_t w = lo; w < hi; ++w) c += (size_t)__builtin_popcount(bits[w]);
            at[t + 1] = c;
        });
        for (unsigned t = 0; t < T; ++t) at[t + 1] += at[t];
        std::vector<uint32_t> cells(at[T]);
        parallel_chunks(W, T, [&](unsigned t, size_t lo, size_t hi) {
            size_t o = at[t];
            for (size_t w = lo; w < hi; ++w)
                for (uint32_t b = bits[w]; b; b &= b - 1) cells[o++] = (uint32_t)(w * 32 + __builtin_ctz(b));
        });
        upload(defer_cells, cells);
        defer_n = (uint32_t)cells.size();
    }
    // The NF2FF samples of a step may run beside the next step's UPML E pass
    // when no sample interpolates over a UPML cell (the only cells of its
    // inputs that pass rewrites in place).
    bool nf2ff_clear_of_pml() const {
        if (!nf_on) return false;
        for (size_t i = 0; i + 2 < h_nf_pts.size(); i += 3) {
            const uint32_t x = h_nf_pts[i], y = h_nf_pts[i + 1], z = h_nf_pts[i + 2];   // cells (x..x+1, y..y+1, z..z+1)
            for (auto& R : pml)
                if (x < R->s[0] + R->n[0] && R->s[0] <= x + 1 && y < R->s[1] + R->n[1] && R->s[1] <= y + 1 &&
                    z < R->s[2] + R->n[2] && R->s[2] <= z + 1)
                    return false;
        }
        return true;
    }

    // Enqueue timestep k of a batch (numTS = state.numTS + k); the fields are
    // read from parity p and written to parity 1 - p.
    // `last`: k is the batch's final step (buffered NF2FF samples are flushed).
    // marks: optional EFS_PHASES + 1 events recorded at the phase boundaries
    // (efs_time_phases); null inside captured graphs.
    //
    // Latency-bound passes are paired into one launch (k_pair): the UPML H
    // pass with the deferred H (both after the E-side point operations; no
    // deferred cell is a UPML cell), and, when no NF2FF sample reads a UPML
    // cell (plan flag nf_pair), a step's NF2FF samples with the next step's
    // UPML E pass (k_pml_e rewrites only UPML cells of those inputs, in place);
    // the samples of a batch's last step run on their own.
    void enqueue_step(uint32_t k, int p, bool last, cudaEvent_t* marks = nullptr) {
        auto mark = [&](int i) { if (marks) ck(cudaEventRecord(marks[i], stream), "phase mark"); };
        mark(0);
        const int q = pnext(p);
        StepState* st = state.as<StepState>();
        float* V = vbuf(p);          // E before the core update
        float* C = cbuf(p);          // H before the core update
        float* V1 = vbuf(q);         // E after it
        float* C1 = cbuf(q);         // H after it
        const uint32_t T = 256;
        const float* const* vfl = vflux_ptrs[p].as<const float*>();
        const float* const* cfl = cflux_ptrs[p].as<const float*>();
        const bool split = pml_split();

        // --- pre-voltage ---
        if (ss_on)     // reads the fields before the UPML pre-update
            k_steady_state<<<blocks(ss_n, T), T, 0, stream>>>(V, st, k, ss_idx.as<uint32_t>(), ss_n, ss_period,
                                                              ss_e1.as<float>(), ss_e2.as<float>());
        if (nf_held.on) {            // samples of step k-1 (its fields are this step's inputs) beside the UPML E pass
            const PassNfSample a{V, C, nf_held.j, nf};
            const uint32_t na = blocks(nf.np, T), nb = blocks(pml_items(), T);
            if (indexed) pair(a, na, pml_e_pass<true>(p), nb);
            else pair(a, na, pml_e_pass<false>(p), nb);
            if (nf_held.j == NF_K - 1) k_nf2ff_flush<<<blocks(nf.np, T), T, 0, stream>>>(st, k - 1 - nf_held.j, nf_held.j + 1, nf);
            nf_held.on = false;
        } else if (split) {
            launch_pml_e(p);
        }
        mark(1);
        if (ade_v.live()) k_ade<<<blocks(ade_v.n, ADE_BLOCK), ADE_T, 0, stream>>>(V, ade_dev(ade_v, vfl));
        MurDev md = mur_dev(vfl);
        if (mur_on) k_mur_pre<<<blocks(mur_n, T), T, 0, stream>>>(V, md);
        RlcDev rd = rlc_dev();
        if (rlc_on) k_rlc_pre<<<blocks(rlc_n, T), T, 0, stream>>>(rd);
        // ADE(curr) reads H and the current flux, which the E side never
        // touches: it runs before the fused kernel overwrites the flux.
        if (ade_c.live()) k_ade<<<blocks(ade_c.n, ADE_BLOCK), ADE_T, 0, stream>>>(C, ade_dev(ade_c, cfl));
        if (tf_n) k_tfsf_face<<<blocks(tf_n, T), T, 0, stream>>>(st, k, tf_dev());   // TFSF face values of this step
        mark(2);
        launch_fused_tma(p);
        mark(3);
        // --- post-voltage / apply (on the updated E) ---
        if (tfsf_on && tfsf_v.groups) k_point_sources<1><<<blocks(tfsf_v.groups, T), T, 0, stream>>>(V1, st, k, point_dev(tfsf_v, tfsf_signal, tfsf_len, tfsf_period));
        if (pbc_on) for (auto& a : pbc_axes) launch_pbc(a, true, V1);
        if (mur_on) k_mur_post<<<blocks(mur_n, T), T, 0, stream>>>(V1, md);
        if (exc_on && exc_groups) {
            PointSources s{exc_groups, exc_target.as<uint32_t>(), exc_off.as<uint32_t>(), exc_delay.as<uint32_t>(),
                           exc_amp.as<float>(), nullptr, exc_signal.as<float>(), exc_len, exc_period};
            k_point_sources<0><<<blocks(exc_groups, T), T, 0, stream>>>(V1, st, k, s);
        }
        if (mur_on) k_mur_apply<<<blocks(mur_napply, T), T, 0, stream>>>(V1, md);
        if (rlc_on) k_rlc_apply<<<blocks(rlc_groups, T), T, 0, stream>>>(V1, rd);
        if (ade_apply && ade_v.live()) launch_ade_apply(ade_v, V1);
        mark(4);
        // --- H of the UPML cells and of the cells next to those E writes ---
        if (split && defer_n) {
            const uint32_t na = blocks(pml_items(), T), nb = blocks(defer_n, T);
            if (indexed) pair(pml_h_pass<true>(p), na, deferred_pass<true>(p), nb);
            else pair(pml_h_pass<false>(p), na, deferred_pass<false>(p), nb);
        } else if (split) launch_pml_h(p);
        else if (defer_n) launch_deferred(p);
        mark(5);
        // --- post-current (on the updated H) ---
        if (tfsf_on && tfsf_c.groups) k_point_sources<1><<<blocks(tfsf_c.groups, T), T, 0, stream>>>(C1, st, k, point_dev(tfsf_c, tfsf_signal, tfsf_len, tfsf_period));
        if (pbc_on) for (auto& a : pbc_axes) launch_pbc(a, false, C1);
        if (ade_apply && ade_c.live()) launch_ade_apply(ade_c, C1);
        mark(6);
        // --- after the step ---
        if (nf_on) {
            // surface samples of this step; the accumulators take every NF_K steps
            // and the batch's last step (nothing stays pending between batches)
            const uint32_t j = k % NF_K;
            if (nf_pair && split && !last) {
                nf_held = NfHeld{true, j};           // sampled beside the next step's UPML E pass
            } else {
                k_nf2ff_sample<<<blocks(nf.np, T), T, 0, stream>>>(V1, C1, j, nf);
                if (j == NF_K - 1 || last) k_nf2ff_flush<<<blocks(nf.np, T), T, 0, stream>>>(st, k - j, j + 1, nf);
            }
        }
        if (ring_on) k_gather_ring<<<blocks(ring_n, 64), 64, 0, stream>>>(V1, C1, st, k, ring_dev());
        mark(7);
    }
    struct NfHeld { bool on; uint32_t j; };
    NfHeld nf_held{false, 0};     // capture: NF2FF samples of the previous step not yet issued
    bool nf_pair = false;         // plan: no NF2FF sample reads a UPML cell
    // passes of the paired launches (k_pair, 256-thread blocks)
    template <bool IDX> PassPmlE<IDX> pml_e_pass(int p) const {
        return PassPmlE<IDX>{fused_grid(p), pml_set(p), pml_set(1 - p), vbuf(p), pml_items()};
    }
    template <bool IDX> PassPmlH<IDX> pml_h_pass(int p) const {
        return PassPmlH<IDX>{fused_grid(p), pml_set(p), pml_set(1 - p), pml_items()};
    }
    template <bool IDX> PassDeferred<IDX> deferred_pass(int p) const {
        return PassDeferred<IDX>{fused_grid(p), defer_cells.as<uint32_t>(), defer_n};
    }
    template <class A, class B>
    void pair(const A& a, uint32_t na, const B& b, uint32_t nb) {
        if (na + nb) k_pair<A, B><<<na + nb, 256, 0, stream>>>(a, na, b, nb);
    }
    void launch_deferred(int p) {
        const uint32_t T = 256;
        if (indexed) k_deferred_h<true><<<blocks(defer_n, T), T, 0, stream>>>(fused_grid(p), defer_cells.as<uint32_t>(), defer_n);
        else k_deferred_h<false><<<blocks(defer_n, T), T, 0, stream>>>(fused_grid(p), defer_cells.as<uint32_t>(), defer_n);
    }
    // `steps` timesteps (at most 64) launched one kernel at a time with the
    // phase marks; accumulates device ms per phase into ms[EFS_PHASES].  Same
    // results as iterate(steps).
    void run_marked(uint32_t steps, float* ms) {
        need_init();
        build_plan();
        std::vector<cudaEvent_t> ev((size_t)steps * (EFS_PHASES + 1));
        for (auto& x : ev) ck(cudaEventCreate(&x), "event");
        nf_held.on = false;
        try {
            int q = cur;
            for (uint32_t k = 0; k < steps; ++k) {
                enqueue_step(k, q, k + 1 == steps, ev.data() + (size_t)k * (EFS_PHASES + 1));
                q = pnext(q);
            }
            k_advance<<<1, 1, 0, stream>>>(state.as<StepState>(), steps);
            ck(cudaGetLastError(), "phase run");
            sync("phase run");
            for (uint32_t k = 0; k < steps; ++k)
                for (int i = 0; i < EFS_PHASES; ++i) {
                    float t = 0;
                    const size_t b = (size_t)k * (EFS_PHASES + 1) + i;
                    ck(cudaEventElapsedTime(&t, ev[b], ev[b + 1]), "elapsed");
                    ms[i] += t;
                }
        } catch (...) {
            for (auto& x : ev) cudaEventDestroy(x);
            throw;
        }
        for (auto& x : ev) cudaEventDestroy(x);
        numTS += steps;
        if (steps & 1) cur ^= 1;
    }
    RingDev ring_dev() const { return RingDev{ring_idx.as<uint32_t>(), ring_n, ring_interval, ring_q0, ring_max, ring.as<float>()}; }

    // TMA-fed kernel: tensor maps over this parity's fields and the material
    // rows (the grid's Nz x Ny x Nx cells over the padded layout), boxes of
    // one tile plus halos (efs_tma.cuh)
    CUtensorMap tensor_map(const void* base, CUtensorMapDataType dt, uint32_t rank, const uint32_t box[4]) const {
        const cuuint64_t dims[4] = {Nz, Ny, Nx, 3};
        const cuuint64_t strides[3] = {(cuuint64_t)Pz * 4, (cuuint64_t)Ny * Pz * 4, (cuuint64_t)Nd * 4};
        return encode_map(base, dt, rank, dims, strides, box);
    }
    // dims: innermost first; strides: bytes of dimensions 1.. (multiples of 16)
    static CUtensorMap encode_map(const void* base, CUtensorMapDataType dt, uint32_t rank, const cuuint64_t* dims,
                                  const cuuint64_t* strides, const uint32_t* box) {
        static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
        if (!encode) {
            void* fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q), "cudaGetDriverEntryPoint");
            if (q != cudaDriverEntryPointSuccess || !fn) fail(EFS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        }
        cuuint32_t bx[4] = {1, 1, 1, 1};
        for (uint32_t i = 0; i < rank; ++i) bx[i] = box[i];
        const cuuint32_t es[4] = {1, 1, 1, 1};
        CUtensorMap m;
        const CUresult r = encode(&m, dt, rank, const_cast<void*>(base), dims, strides, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) fail(EFS_ERR_CUDA, "cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
        return m;
    }
    template <bool IDX, bool PML>
    void launch_fused_tma_k(dim3 g, const CUtensorMap& tH, const CUtensorMap& tE, const CUtensorMap& tM, const CUtensorMap& tD,
                            const FusedGrid& fg, const PmlSet& ps) {
        static bool attr_set = false;   // per instantiation; the attribute is per kernel, all devices alike
        if (!attr_set) {
            ck(cudaFuncSetAttribute(k_fused_tma<IDX, PML>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT_SMEM_BYTES),
               "smem attr");
            attr_set = true;
        }
        k_fused_tma<IDX, PML><<<g, TT_THREADS, TT_SMEM_BYTES, stream>>>(tH, tE, tM, tD, fg, ps);
    }
    void launch_fused_tma(int p) {
        const FusedGrid fg = fused_grid(p);
        const PmlSet ps = pml_set(p);
        const uint32_t bh[4] = {TT_HZ, TT_HY, 1, 3}, be[4] = {TT_EZ, TT_EY, 1, 3};
        const CUtensorMap tH = tensor_map(fg.H0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, bh);
        const CUtensorMap tE = tensor_map(fg.V0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, be);
        const CUtensorMap tM = indexed ? tensor_map(fg.mat, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, be) : tE;
        const CUtensorMap tD = tf.n ? tf_map() : tE;   // unused without TFSF faces
        dim3 g(blocks(Nz, TT_Z), blocks(Ny, TT_Y), blocks(Nx, xchunk));
        const bool hp = !pml.empty();
        if (indexed) { if (hp) launch_fused_tma_k<true, true>(g, tH, tE, tM, tD, fg, ps); else launch_fused_tma_k<true, false>(g, tH, tE, tM, tD, fg, ps); }
        else { if (hp) launch_fused_tma_k<false, true>(g, tH, tE, tM, tD, fg, ps); else launch_fused_tma_k<false, false>(g, tH, tE, tM, tD, fg, ps); }
    }
    // UPML cells are updated by k_pml_e / k_pml_h around the fused kernel
    bool pml_split() const { return !pml.empty(); }
    uint32_t pml_items() const {   // work items of k_pml_e / k_pml_h: PML_ZC cells of a region row each
        size_t t = 0;
        for (auto& r : pml) t += (size_t)r->n[0] * r->n[1] * ((r->n[2] + PML_ZC - 1) / PML_ZC);
        return (uint32_t)t;    // at most the regions' cell count, < 2^32 (efs_configure_pml)
    }
    void launch_pml_e(int p) {
        const FusedGrid fg = fused_grid(p);
        const PmlSet ps = pml_set(p), pn = pml_set(1 - p);
        const uint32_t t = pml_items(), T = 256;
        if (indexed) k_pml_e<true><<<blocks(t, T), T, 0, stream>>>(fg, ps, pn, vbuf(p), t);
        else k_pml_e<false><<<blocks(t, T), T, 0, stream>>>(fg, ps, pn, vbuf(p), t);
    }
    void launch_pml_h(int p) {
        const FusedGrid fg = fused_grid(p);
        const PmlSet ps = pml_set(p), pn = pml_set(1 - p);
        const uint32_t t = pml_items(), T = 256;
        if (indexed) k_pml_h<true><<<blocks(t, T), T, 0, stream>>>(fg, ps, pn, t);
        else k_pml_h<false><<<blocks(t, T), T, 0, stream>>>(fg, ps, pn, t);
    }

    PointSources point_dev(const PointSet& p, const DevBuf& sig, uint32_t len, uint32_t period) const {
        return PointSources{p.groups, p.target.as<uint32_t>(), p.off.as<uint32_t>(), p.delay.as<uint32_t>(),
                            p.amp.as<float>(), p.frac.as<float>(), sig.as<float>(), len, period};
    }
    AdeDev ade_dev(const AdeSide& s, const float* const* flux) const {
        return AdeDev{s.n, s.runs.as<AdeRun>(), s.grp_run.as<uint32_t>(), s.coef.as<float4>(), s.state.as<float>(),
                      s.lor.as<float>(), flux};
    }
    MurDev mur_dev(const float* const* vfl) const {
        return MurDev{mur_n, mur_napply, mur_coeff.as<float>(), mur_pre_normal.as<ReadLoc>(), mur_pre_shifted.as<ReadLoc>(),
                      mur_shifted.as<uint32_t>(), mur_apply_target.as<uint32_t>(), mur_apply_src.as<uint32_t>(),
                      mur_saved.as<float>(), vfl};
    }
    RlcDev rlc_dev() const {
        return RlcDev{rlc_n, rlc_groups, rlc_gtarget.as<uint32_t>(), rlc_goff.as<uint32_t>(), rlc_type.as<uint32_t>(),
                      rlc_p.as<float>(), rlc_vdn.as<float>(), rlc_jn.as<float>(), rlc_vil.as<float>()};
    }
    void launch_pbc(const PbcAxis& a, bool isVolt, float* F) {
        const uint32_t nl[3] = {Nx, Ny, Nz};
        PbcDev p;
        p.axis = a.axis; p.volt = isVolt ? 1 : 0;
        uint32_t t0 = (a.axis + 1) % 3, t1 = (a.axis + 2) % 3;
        p.fs0 = nl[t0]; p.fs1 = nl[t1];
        p.b0 = isVolt ? p.fs0 : p.fs0 - 1; p.b1 = isVolt ? p.fs1 : p.fs1 - 1;
        p.src = isVolt ? nl[a.axis] - 2 : 0; p.dst = isVolt ? 0 : nl[a.axis] - 2;
        p.Nx = Nx; p.Ny = Ny; p.Nz = Nz; p.Pz = Pz; p.cosP = a.c; p.sinP = a.s;
        p.imag = pbc_imag.as<float>() + a.imag_off;
        dim3 b(16, 16), gr(blocks(p.b0, 16), blocks(p.b1, 16));
        if (p.b0 && p.b1) k_pbc<<<gr, b, 0, stream>>>(F, p);
    }

    void iterate(uint32_t n) {
        need_init();
        build_plan();
        const uint32_t CH = 64;   // steps per captured graph
        while (n > 0) {
            uint32_t m = std::min(n, CH);
            cudaGraphExec_t ge = graph_for(m, cur);
            ck(cudaGraphLaunch(ge, stream), "cudaGraphLaunch");
            numTS += m;
            if (m & 1) cur ^= 1;
            n -= m;
        }
        ck(cudaGetLastError(), "iterate");
    }

    // graph of m steps starting from parity p (the buffers alternate each step)
    cudaGraphExec_t graph_for(uint32_t m, int p) {
        const uint32_t key = m * 2 + (uint32_t)p;
        auto it = graphs.find(key);
        if (it != graphs.end()) return it->second;
        if (graphs.size() > 12) drop_graphs();
        cudaGraph_t graph;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "BeginCapture");
        nf_held.on = false;
        try {
            int q = p;
            for (uint32_t k = 0; k < m; ++k) { enqueue_step(k, q, k + 1 == m); q = pnext(q); }
            k_advance<<<1, 1, 0, stream>>>(state.as<StepState>(), m);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            throw;
        }
        ck(cudaStreamEndCapture(stream, &graph), "EndCapture");
        cudaGraphExec_t ge;
        cudaError_t err = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        ck(err, "cudaGraphInstantiate");
        graphs[key] = ge;
        return ge;
    }

    void sync_state_to_device() {
        hstate.numTS = numTS;
        ck(cudaMemcpyAsync(state.p, &hstate, sizeof(StepState), cudaMemcpyHostToDevice, stream), "state upload");
        sync("state sync");
    }

    // Entries grouped by target: utarget ascending, group g = entries
    // perm[off[g] .. off[g+1]) in the caller's order (a stable sort by target).
    static void group_by(const std::vector<uint32_t>& tgt, std::vector<uint32_t>& utarget, std::vector<uint32_t>& off,
                         std::vector<uint32_t>& perm) {
        efs_host::group_by(tgt, utarget, off, perm);
    }
};

namespace {

template <typename F>
efs_status guard(efs_engine* e, F&& f) {
    if (!e) return EFS_ERR_INVALID;
    try {
        ck(cudaSetDevice(e->device), "cudaSetDevice");
        f();
        return EFS_OK;
    } catch (const EfsError& err) {
        e->last_error = err.msg;
        return err.code;
    } catch (const std::exception& ex) {
        e->last_error = ex.what();
        return EFS_ERR_OOM;
    }
}

void alloc_fields(efs_engine* e, const uint32_t dims[3]) {
    if (!dims || dims[0] == 0 || dims[1] == 0 || dims[2] == 0) fail(EFS_ERR_INVALID, "grid dimensions must be positive");
    size_t N = (size_t)dims[0] * dims[1] * dims[2];
    const uint32_t Pz = (dims[2] + 3u) & ~3u;
    const size_t Nd = (size_t)dims[0] * dims[1] * Pz;
    if (3 * Nd >= (1ull << 32))
        fail(EFS_ERR_RANGE, "grid too large for 32-bit field indices (3*Nx*Ny*Pz >= 2^32, Pz = Nz rounded up to a multiple of 4)");
    // a fresh init drops every extension; the engine counts as initialised
    // again only when the init call completes (a failed init leaves it unusable)
    e->inited = false;
    e->drop_graphs();
    e->pml.clear();
    e->exc_on = e->mur_on = e->tfsf_on = e->ade_on = e->rlc_on = e->ss_on = e->pbc_on = e->ring_on = e->nf_on = false;
    e->ade_v = efs_engine::AdeSide(); e->ade_c = efs_engine::AdeSide();
    e->ade_apply = false;
    e->gd_n = 0;
    e->Nx = dims[0]; e->Ny = dims[1]; e->Nz = dims[2]; e->N = N; e->Pz = Pz; e->Nd = Nd;
    e->h_exc_targets.clear(); e->h_tfsf_v_targets.clear(); e->h_mur_apply.clear(); e->h_rlc_series.clear();
    e->h_tfsf_v.clear();
    e->tf = TfsfFace{0, {0, 0}};
    e->tf_n = 0;
    e->defer_n = 0;
    // plane depth (x-planes per CTA) of the fused kernel; results do not depend on it
    e->cur = 0;
    e->alloc(e->volt, 3 * Nd * sizeof(float));
    e->alloc(e->curr, 3 * Nd * sizeof(float));
    e->alloc(e->volt_b, 3 * Nd * sizeof(float));
    e->alloc(e->curr_b, 3 * Nd * sizeof(float));
    e->alloc(e->state, sizeof(StepState));
    e->numTS = 0;
    e->hstate = StepState{};
    e->en_pending = false; e->en_last = 0.0; e->en_idx = 0;
    e->en_partial.reset(); e->en_result.reset();
    e->vv.reset(); e->vi.reset(); e->ii.reset(); e->iv.reset(); e->mat.reset(); e->table.reset();
}

// FNV-1a over the 48-byte tuple
struct TupleHash {
    size_t operator()(const std::array<uint32_t, 12>& t) const {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t w : t) { h ^= w; h *= 1099511628211ull; }
        return (size_t)h;
    }
};

}  // namespace

extern "C" {

efs_status efs_create(efs_engine** out, int device) {
    if (!out) return EFS_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    cudaError_t err = cudaGetDeviceCount(&n);
    if (err != cudaSuccess || n == 0) {
        g_create_error = std::string("no CUDA device: ") + (err != cudaSuccess ? cudaGetErrorString(err) : "count 0");
        return EFS_ERR_CUDA;
    }
    if (device < 0 || device >= n) { g_create_error = "device index out of range"; return EFS_ERR_INVALID; }
    auto* e = new efs_engine();
    e->device = device;
    try {
        ck(cudaSetDevice(device), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        e->slot = host_slot_get();
        e->en_host = e->slot->energy;
        e->h_status = &e->slot->status;
        ck(cudaHostGetDevicePointer(&e->d_status, e->h_status, 0), "cudaHostGetDevicePointer");
        for (auto& ev : e->en_event) ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    } catch (const EfsError& ex) {
        g_create_error = ex.msg;
        delete e;
        return ex.code;
    }
    *out = e;
    return EFS_OK;
}

efs_status efs_destroy(efs_engine* e) {
    if (!e) return EFS_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    delete e;
    return EFS_OK;
}

const char* efs_last_error(const efs_engine* e) { return e ? e->last_error.c_str() : g_create_error.c_str(); }

efs_status efs_init(efs_engine* e, const uint32_t dims[3], const float* vv, const float* vi, const float* ii, const float* iv) {
    return guard(e, [&] {
        if (!vv || !vi || !ii || !iv) fail(EFS_ERR_INVALID, "coefficient arrays must be non-null");
        alloc_fields(e, dims);
        const size_t N = e->N;
        // Deduplicate per-cell (vv,vi,ii,iv) x 3 tuples into a material table
        // (material index per cell in the caller's layout; padded on upload).
        std::unordered_map<std::array<uint32_t, 12>, uint32_t, TupleHash> ids;
        std::vector<uint32_t> mat(N);
        std::vector<float> table;
        const size_t limit = std::min<size_t>(1u << 22, std::max<size_t>(4096, N / 4));
        bool ok = true;
        ids.reserve(std::min<size_t>(limit, 1 << 16));
        for (size_t c = 0; c < N && ok; ++c) {
            std::array<uint32_t, 12> t;
            const float* src[4] = {vv, vi, ii, iv};
            for (int a = 0; a < 4; ++a)
                for (int n = 0; n < 3; ++n) memcpy(&t[a * 3 + n], src[a] + n * N + c, 4);
            auto it = ids.find(t);
            if (it == ids.end()) {
                if (ids.size() >= limit) { ok = false; break; }
                uint32_t id = (uint32_t)ids.size();
                ids.emplace(t, id);
                for (int q = 0; q < 12; ++q) { float f; memcpy(&f, &t[q], 4); table.push_back(f); }
                mat[c] = id;
            } else {
                mat[c] = it->second;
            }
        }
        if (ok) {
            e->indexed = true;
            e->ntable = (uint32_t)ids.size();
            e->upload_padded(e->mat, mat.data(), 1);
            e->upload(e->table, table);
        } else {
            e->indexed = false;
            e->upload_padded(e->vv, vv, 3); e->upload_padded(e->vi, vi, 3);
            e->upload_padded(e->ii, ii, 3); e->upload_padded(e->iv, iv, 3);
        }
        e->sync_state_to_device();
        e->inited = true;
        e->dirty();
    });
}

efs_status efs_init_indexed(efs_engine* e, const uint32_t dims[3], const uint32_t* mat, const float* table, uint32_t ntable) {
    return guard(e, [&] {
        if (!mat || !table || ntable == 0) fail(EFS_ERR_INVALID, "mat/table must be non-null and ntable > 0");
        alloc_fields(e, dims);
        // indices are checked on the device after the upload (pad cells hold 0)
        e->upload_padded(e->mat, mat, 1);
        {
            DevBuf mx;
            e->alloc(mx, 4);
            k_max_u32<<<std::min<uint32_t>(blocks(e->Nd, 256), 148 * 8), 256, 0, e->stream>>>(e->mat.as<uint32_t>(), e->Nd,
                                                                                               mx.as<uint32_t>());
            ck(cudaGetLastError(), "material index check");
            uint32_t hmax = 0;
            ck(cudaMemcpyAsync(&hmax, mx.p, 4, cudaMemcpyDeviceToHost, e->stream), "material index check");
            e->sync("material index check");
            if (hmax >= ntable) {
                e->mat.reset();
                fail(EFS_ERR_INVALID, "material index out of range");
            }
        }
        e->indexed = true;
        e->ntable = ntable;
        e->upload(e->table, table, (size_t)ntable * 12);
        e->sync_state_to_device();
        e->inited = true;
        e->dirty();
    });
}

efs_status efs_configure_excitation(efs_engine* e, const float* signal, uint32_t L, const uint32_t* delay, const float* amp,
                                    const uint32_t* dir, const uint32_t* pos, uint32_t count, uint32_t period) {
    return guard(e, [&] {
        e->need_init();
        if (L == 0 || !signal) fail(EFS_ERR_INVALID, "excitation signal must be non-empty");
        if (count && (!delay || !amp || !dir || !pos)) fail(EFS_ERR_INVALID, "excitation arrays must be non-null");
        std::vector<uint32_t> tgt(count);
        for (uint32_t i = 0; i < count; ++i) {
            if (dir[i] > 2 || pos[i] >= e->N) fail(EFS_ERR_INVALID, "excitation dir/pos out of range");
            tgt[i] = e->dev_index(dir[i] * (uint32_t)e->N + pos[i]);
        }
        std::vector<uint32_t> ut, off, perm;
        efs_engine::group_by(tgt, ut, off, perm);
        std::vector<uint32_t> d(count);
        std::vector<float> a(count);
        for (uint32_t i = 0; i < count; ++i) { d[i] = delay[perm[i]]; a[i] = amp[perm[i]]; }
        e->upload(e->exc_target, ut); e->upload(e->exc_off, off);
        e->h_exc_targets = ut;
        e->upload(e->exc_delay, d); e->upload(e->exc_amp, a);
        e->upload(e->exc_signal, signal, L);
        e->exc_groups = (uint32_t)ut.size(); e->exc_len = L; e->exc_period = period;
        e->exc_on = true;
        e->dirty();
    });
}

// The distinct (vv, vvfo, vvfn, ii, iifo, iifn) x 3-component tuples of a
// region's cells as a row table and a 16-bit row index per cell.  A UPML's
// coefficients follow its grading profiles, so a slab has a few thousand
// distinct tuples at most; a region with more keeps only the dense arrays.
struct PmlCompact {
    std::vector<uint16_t> idx;
    std::vector<float> tab;
    bool ok = false;
};
static PmlCompact compact_pml(const efs_engine::Region& R, const efs_pml_region& in) {
    PmlCompact out;
    const size_t nc = R.total / 3;
    const float* src[6] = {in.vv, in.vvfo, in.vvfn, in.ii, in.iifo, in.iifn};
    typedef std::array<uint32_t, 18> Key;
    struct KeyHash {
        size_t operator()(const Key& k) const {
            uint64_t h = 1469598103934665603ull;
            for (uint32_t v : k) { h ^= v; h *= 1099511628211ull; }
            return (size_t)h;
        }
    };
    std::unordered_map<Key, uint32_t, KeyHash> ids;
    std::vector<uint16_t>& idx = out.idx;
    std::vector<float>& tab = out.tab;
    idx.resize(nc);
    // Lookups skip the map when the tuple equals the previous cell's (grading
    // along x or y: constant along a z row) or the previous row's at the same
    // z (grading along z: a z-slab row repeats its tuples).
    const uint32_t nz = R.n[2];
    std::vector<Key> zkey(nz);
    std::vector<uint32_t> zid(nz);
    Key key{}, last{};
    uint32_t last_id = 0;
    for (size_t c = 0; c < nc; ++c) {
        for (int a = 0; a < 6; ++a)
            for (int n = 0; n < 3; ++n) memcpy(&key[a * 3 + n], src[a] + n * nc + c, 4);
        const uint32_t z = (uint32_t)(c % nz);
        if (c > 0 && key == last) {
        } else if (c >= nz && key == zkey[z]) {
            last = key;
            last_id = zid[z];
        } else {
            auto it = ids.find(key);
            if (it == ids.end()) {
                if (ids.size() >= 65535) return PmlCompact{};
                it = ids.emplace(key, (uint32_t)ids.size()).first;
                for (int a = 0; a < 6; ++a) {
                    for (int n = 0; n < 3; ++n) { float f; memcpy(&f, &key[a * 3 + n], 4); tab.push_back(f); }
                    tab.push_back(0.f);
                }
            }
            last = key;
            last_id = it->second;
        }
        zkey[z] = key;
        zid[z] = last_id;
        idx[c] = (uint16_t)last_id;
    }
    out.ok = true;
    return out;
}

efs_status efs_configure_pml(efs_engine* e, uint32_t count, const efs_pml_region* regions) {
    return guard(e, [&] {
        e->need_init();
        if (count > (uint32_t)MAX_PML) fail(EFS_ERR_RANGE, "too many UPML regions (max 24)");
        if (count && !regions) fail(EFS_ERR_INVALID, "regions must be non-null");
        const uint32_t nl[3] = {e->Nx, e->Ny, e->Nz};
        std::vector<std::unique_ptr<efs_engine::Region>> out;
        for (uint32_t r = 0; r < count; ++r) {
            const efs_pml_region& in = regions[r];
            auto R = std::make_unique<efs_engine::Region>();
            for (int d = 0; d < 3; ++d) {
                // wasm-gpu-bridge.mjs:_validatePMLRegion (:206-236)
                if ((uint64_t)in.start[d] + in.num[d] > nl[d]) fail(EFS_ERR_INVALID, "PML region extends beyond grid");
                R->s[d] = in.start[d]; R->n[d] = in.num[d];
            }
            if (!in.vv || !in.vvfo || !in.vvfn || !in.ii || !in.iifo || !in.iifn) fail(EFS_ERR_INVALID, "PML region array missing");
            R->total = 3 * (size_t)R->n[0] * R->n[1] * R->n[2];
            out.push_back(std::move(R));
        }
        // A region's dense coefficient arrays are read only for cells that
        // another region also contains (the multi-region chain) and when its
        // compact table cannot be built: regions that overlap no other upload
        // them only in the second case.
        std::vector<uint8_t> overlaps(count, 0);
        for (uint32_t a = 0; a < count; ++a)
            for (uint32_t b = a + 1; b < count; ++b) {
                bool meet = true;
                for (int d = 0; d < 3; ++d)
                    meet = meet && out[a]->s[d] < out[b]->s[d] + out[b]->n[d] && out[b]->s[d] < out[a]->s[d] + out[a]->n[d];
                if (meet) overlaps[a] = overlaps[b] = 1;
            }
        auto upload_dense = [&](uint32_t r) {
            const efs_pml_region& in = regions[r];
            efs_engine::Region* R = out[r].get();
            e->upload(R->vv, in.vv, R->total); e->upload(R->vvfo, in.vvfo, R->total); e->upload(R->vvfn, in.vvfn, R->total);
            e->upload(R->ii, in.ii, R->total); e->upload(R->iifo, in.iifo, R->total); e->upload(R->iifn, in.iifn, R->total);
        };
        // the regions' coefficient tables are built on host threads (one per
        // region) while this thread uploads what it can already
        std::vector<PmlCompact> comp(count);
        std::vector<std::exception_ptr> errs(count);
        std::vector<std::thread> workers;
        auto join = [&] { for (auto& t : workers) if (t.joinable()) t.join(); };
        try {
            for (uint32_t r = 0; r < count; ++r)
                workers.emplace_back([&, r] {
                    try { comp[r] = compact_pml(*out[r], regions[r]); } catch (...) { errs[r] = std::current_exception(); }
                });
            for (uint32_t r = 0; r < count; ++r) {
                efs_engine::Region* R = out[r].get();
                if (overlaps[r]) upload_dense(r);
                e->alloc(R->vflux, R->total * 4); e->alloc(R->cflux, R->total * 4);
                e->alloc(R->vflux_b, R->total * 4); e->alloc(R->cflux_b, R->total * 4);
            }
        } catch (...) {
            join();
            throw;
        }
        join();
        for (uint32_t r = 0; r < count; ++r) {
            if (errs[r]) std::rethrow_exception(errs[r]);
            if (!comp[r].ok) {
                if (!overlaps[r]) upload_dense(r);
                continue;
            }
            e->upload(out[r]->cidx, comp[r].idx);
            e->upload(out[r]->ctab, comp[r].tab);
        }
        // the per-cell UPML chain keeps at most PML_MAX_OVERLAP regions in registers:
        // test every corner formed by region bounds (the overlap count is maximal at one)
        if (count > (uint32_t)PML_MAX_OVERLAP) {
            std::vector<uint32_t> cx[3];
            for (auto& R : out)
                for (int d = 0; d < 3; ++d) cx[d].push_back(R->s[d]);
            for (uint32_t a : cx[0]) for (uint32_t b : cx[1]) for (uint32_t c : cx[2]) {
                int k = 0;
                for (auto& R : out)
                    k += (a - R->s[0]) < R->n[0] && (b - R->s[1]) < R->n[1] && (c - R->s[2]) < R->n[2];
                if (k > PML_MAX_OVERLAP) fail(EFS_ERR_RANGE, "more than 4 UPML regions overlap at one cell");
            }
        }
        uint64_t cells = 0;   // the UPML passes of the TMA path index region cells with 32 bits
        for (auto& R : out) cells += (uint64_t)R->n[0] * R->n[1] * R->n[2];
        if (cells >= (1ull << 32)) fail(EFS_ERR_RANGE, "UPML regions hold 2^32 cells or more");
        e->pml = std::move(out);
        e->dirty();
    });
}

efs_status efs_configure_mur(efs_engine* e, const float* coeff, const uint32_t* normal, const uint32_t* shifted, uint32_t n) {
    return guard(e, [&] {
        e->need_init();
        if (n && (!coeff || !normal || !shifted)) fail(EFS_ERR_INVALID, "Mur arrays must be non-null");
        e->check_idx3(normal, n, "Mur normal_idx");
        e->check_idx3(shifted, n, "Mur shifted_idx");
        // Entries are kept in field-index order on the device, so neighbouring
        // threads touch neighbouring cells (the caller's face order walks a
        // face across rows).  The pre and post updates are per entry; apply
        // resolves each target to its last writer in the caller's order
        // (sequential loop :1016-1023), which the permutation leaves intact.
        std::vector<uint32_t> perm(n), sn(n);
        for (uint32_t i = 0; i < n; ++i) { perm[i] = i; sn[i] = e->dev_index(normal[i]); }
        efs_engine::radix_sort_pairs(sn, perm);           // stable: equal normals keep the caller's order
        std::vector<uint32_t> ss(n);
        std::vector<float> sc(n);
        for (uint32_t k = 0; k < n; ++k) { ss[k] = e->dev_index(shifted[perm[k]]); sc[k] = coeff[perm[k]]; }
        // apply: per distinct normal (ascending) its last writer in the caller's
        // order, which is the last entry of its run in the sorted order
        std::vector<uint32_t> at, as;
        for (uint32_t k = 0; k < n; ++k)
            if (k + 1 == n || sn[k + 1] != sn[k]) { at.push_back(sn[k]); as.push_back(k); }
        e->h_mur_normal = sn;
        e->h_mur_shifted = ss;
        e->upload(e->mur_coeff, sc);
        e->upload(e->mur_shifted, ss);
        e->upload(e->mur_apply_target, at); e->upload(e->mur_apply_src, as);
        e->mur_perm = perm;
        e->h_mur_apply = at;
        e->alloc(e->mur_saved, (size_t)n * 4);
        e->mur_n = n; e->mur_napply = (uint32_t)at.size();
        e->mur_on = n > 0;
        e->dirty();
    });
}

static void build_points(efs_engine* e, efs_engine::PointSet& ps, const efs_tfsf_point* pts, uint32_t n) {
    std::vector<uint32_t> tgt(n);
    for (uint32_t i = 0; i < n; ++i) tgt[i] = pts[i].field_idx;
    e->check_idx3(tgt.data(), n, "TFSF field_idx");
    for (uint32_t i = 0; i < n; ++i) tgt[i] = e->dev_index(tgt[i]);
    std::vector<uint32_t> ut, off, perm;
    efs_engine::group_by(tgt, ut, off, perm);
    std::vector<uint32_t> d(n);
    std::vector<float> a(n), f(n);
    for (uint32_t i = 0; i < n; ++i) { d[i] = pts[perm[i]].delay_int; a[i] = pts[perm[i]].amp; f[i] = pts[perm[i]].delay_frac; }
    e->upload(ps.target, ut); e->upload(ps.off, off); e->upload(ps.delay, d); e->upload(ps.amp, a); e->upload(ps.frac, f);
    ps.groups = (uint32_t)ut.size();
}

// TFSF faces of the core update: up to two z planes, each holding at least a
// 16th of the voltage-side entries as single-entry Ex/Ey targets (the box's z
// faces); their entries move to the face array, every other entry stays in
// the point pass (in the caller's order per target).
void efs_engine::plan_tfsf_faces() {
    tf = TfsfFace{0, {0, 0}};
    tf_n = 0;
    tf_face.reset(); tf_dst.reset(); tf_delay.reset(); tf_frac.reset(); tf_amp.reset();
    if (!tfsf_on) return;
    const size_t nv = h_tfsf_v.size();
    std::vector<uint32_t> tg(nv);
    for (size_t i = 0; i < nv; ++i) tg[i] = dev_index(h_tfsf_v[i].field_idx);
    // entries in target order (stable: the caller's order per target); the
    // entries whose target no other entry shares are runs of length 1
    std::vector<uint32_t> key(tg), perm(nv);
    for (size_t i = 0; i < nv; ++i) perm[i] = (uint32_t)i;
    radix_sort_pairs(key, perm);
    std::vector<uint8_t> single(nv, 0);
    for (size_t i = 0; i < nv;) {
        size_t j = i + 1;
        while (j < nv && key[j] == key[i]) ++j;
        if (j == i + 1) single[perm[i]] = 1;
        i = j;
    }
    std::vector<uint8_t> cand(nv, 0);
    std::vector<size_t> per_z(Nz, 0);
    for (size_t i = 0; i < nv; ++i) {
        const uint32_t n = tg[i] / (uint32_t)Nd;
        if (n > 1 || !single[i]) continue;
        cand[i] = 1;
        ++per_z[(tg[i] % (uint32_t)Nd) % Pz];
    }
    std::vector<uint32_t> faces;
    if (Ny >= (uint32_t)TF_DY)
        for (int k = 0; k < 2; ++k) {
            uint32_t best = Nz;
            for (uint32_t z = 0; z < Nz; ++z)
                if (per_z[z] * 16 >= nv && per_z[z] > 0 && (best == Nz || per_z[z] > per_z[best]) &&
                    (faces.empty() || z != faces[0]))
                    best = z;
            if (best < Nz) faces.push_back(best);
        }
    const uint32_t ly = (Ny + 3) & ~3u;
    std::vector<uint8_t> on_face(nv, 0);
    std::vector<uint32_t> dst, delay;
    std::vector<float> frac, amp;
    for (size_t i = 0; i < nv; ++i) {
        int f = -1;
        const uint32_t z = (tg[i] % (uint32_t)Nd) % Pz;
        for (size_t q = 0; q < faces.size(); ++q) if (cand[i] && z == faces[q]) f = (int)q;
        if (f < 0) continue;
        on_face[i] = 1;
        const uint32_t n = tg[i] / (uint32_t)Nd, c = tg[i] % (uint32_t)Nd;
        const uint32_t x = c / (Ny * Pz), y = (c / Pz) % Ny;
        dst.push_back(((uint32_t)(f * 2 + n) * Nx + x) * ly + y);
        delay.push_back(h_tfsf_v[i].delay_int); frac.push_back(h_tfsf_v[i].delay_frac); amp.push_back(h_tfsf_v[i].amp);
    }
    // the point pass keeps the other entries, grouped by target in target
    // order (what build_points makes of them: face entries are whole groups)
    {
        std::vector<uint32_t> ut, off(1, 0), d;
        std::vector<float> a, fr;
        for (size_t k = 0; k < nv; ++k) {
            const uint32_t i = perm[k];
            if (on_face[i]) continue;
            if (ut.empty() || key[k] != ut.back()) {
                if (!ut.empty()) off.push_back((uint32_t)d.size());
                ut.push_back(key[k]);
            }
            d.push_back(h_tfsf_v[i].delay_int); a.push_back(h_tfsf_v[i].amp); fr.push_back(h_tfsf_v[i].delay_frac);
        }
        if (!d.empty()) off.push_back((uint32_t)d.size());
        upload(tfsf_v.target, ut); upload(tfsf_v.off, off); upload(tfsf_v.delay, d); upload(tfsf_v.amp, a);
        upload(tfsf_v.frac, fr);
        tfsf_v.groups = (uint32_t)ut.size();
        h_tfsf_v_targets = ut;
    }
    if (faces.empty()) return;
    const size_t nface = faces.size() * 2 * (size_t)Nx * ly;
    alloc(tf_face, nface * 4, false);
    k_fill<<<(unsigned)std::min<size_t>(blocks(nface, 256), 4096), 256, 0, stream>>>(tf_face.as<float>(), nface, -0.0f);
    ck(cudaGetLastError(), "face fill");
    upload(tf_dst, dst); upload(tf_delay, delay); upload(tf_frac, frac); upload(tf_amp, amp);
    tf.n = (uint32_t)faces.size();
    for (size_t q = 0; q < faces.size(); ++q) tf.z[q] = faces[q];
    tf_n = (uint32_t)dst.size();
    tf_ly = ly;
}

efs_status efs_configure_tfsf(efs_engine* e, const float* signal, uint32_t L, uint32_t period, const efs_tfsf_point* vp,
                              uint32_t nv, const efs_tfsf_point* cp, uint32_t nc) {
    return guard(e, [&] {
        e->need_init();
        if (!signal || L == 0) fail(EFS_ERR_INVALID, "TFSF signal must be non-empty");
        if ((nv && !vp) || (nc && !cp)) fail(EFS_ERR_INVALID, "TFSF point arrays must be non-null");
        std::vector<uint32_t> vt(nv);
        for (uint32_t i = 0; i < nv; ++i) vt[i] = vp[i].field_idx;
        e->check_idx3(vt.data(), nv, "TFSF field_idx");
        build_points(e, e->tfsf_c, cp, nc);
        // the voltage side's point set and targets are built by the plan
        // (plan_tfsf_faces), once the core update's z faces are chosen
        e->h_tfsf_v.assign(vp, vp + nv);
        e->h_tfsf_v_targets.clear();
        e->upload(e->tfsf_signal, signal, L);
        e->tfsf_len = L; e->tfsf_period = period;
        e->tfsf_on = true;
        e->dirty();
    });
}

efs_status efs_configure_ade(efs_engine* e, uint32_t count, const efs_ade_order* orders) {
    return guard(e, [&] {
        e->need_init();
        if (count && !orders) fail(EFS_ERR_INVALID, "orders must be non-null");
        for (int side = 0; side < 2; ++side) {
            efs_engine::AdeSide& s = side == 0 ? e->ade_v : e->ade_c;
            s = efs_engine::AdeSide();
            // coefficient tuples (kint, kext, klor bits + Lorentz flag), deduplicated
            std::map<std::array<uint32_t, 4>, uint32_t> ids;
            std::vector<float4> tuples;
            std::array<uint32_t, 4> last{};
            uint32_t last_id = 0;
            auto bits = [](float f) { uint32_t u; memcpy(&u, &f, 4); return u; };
            for (uint32_t o = 0; o < count; ++o) {
                const efs_ade_order& od = orders[o];
                if (od.num_directions && !od.directions) fail(EFS_ERR_INVALID, "ADE directions must be non-null");
                for (uint32_t d = 0; d < od.num_directions; ++d) {
                    const efs_ade_direction& dr = od.directions[d];
                    if (dr.dir > 2 || (od.num_cells && !dr.pos_idx)) fail(EFS_ERR_INVALID, "ADE direction invalid");
                    const float* a = side == 0 ? dr.v_int : dr.i_int;
                    const float* b = side == 0 ? dr.v_ext : dr.i_ext;
                    const float* c = side == 0 ? dr.v_lor : dr.i_lor;
                    for (uint32_t i = 0; i < od.num_cells; ++i) {
                        if (dr.pos_idx[i] >= e->N) fail(EFS_ERR_INVALID, "ADE pos_idx out of range");
                        s.h_field.push_back(e->dev_index(dr.dir * (uint32_t)e->N + dr.pos_idx[i]));
                        const float k0 = a ? a[i] : 0.f, k1 = b ? b[i] : 0.f, k2 = c ? c[i] : 0.f;
                        const std::array<uint32_t, 4> key{bits(k0), bits(k1), bits(k2), od.has_lorentz ? 1u : 0u};
                        if (tuples.empty() || key != last) {
                            auto it = ids.find(key);
                            if (it == ids.end()) {
                                if (tuples.size() >= 0x7fffffffu) fail(EFS_ERR_INVALID, "too many ADE coefficient tuples");
                                it = ids.emplace(key, (uint32_t)tuples.size()).first;
                                tuples.push_back(make_float4(k0, k1, k2, 0.f));
                            }
                            last = key;
                            last_id = it->second | (key[3] << 31);
                        }
                        s.h_coef.push_back(last_id);
                    }
                }
            }
            s.n = (uint32_t)s.h_field.size();
            // all coefficients +0 (bit for bit: a -0 coefficient can make a -0 state)
            s.zero = true;
            for (const auto& kv : ids) s.zero = s.zero && !kv.first[0] && !kv.first[1] && !kv.first[2];
            e->upload(s.coef, tuples);
            e->alloc(s.state, (size_t)s.n * 4); e->alloc(s.lor, (size_t)s.n * 4);
        }
        e->ade_on = count > 0;
        e->dirty();
    });
}

efs_status efs_configure_ade_apply(efs_engine* e, int on) {
    return guard(e, [&] {
        e->need_init();
        e->ade_apply = on != 0;
        e->dirty();
    });
}

efs_status efs_configure_rlc(efs_engine* e, uint32_t n, const efs_rlc_element* el) {
    return guard(e, [&] {
        e->need_init();
        if (n && !el) fail(EFS_ERR_INVALID, "elements must be non-null");
        std::vector<uint32_t> tgt(n), type(n);
        std::vector<float> p(9 * (size_t)n);
        for (uint32_t i = 0; i < n; ++i) {
            if (el[i].direction > 2 || el[i].field_idx >= e->N) fail(EFS_ERR_INVALID, "RLC field_idx/direction out of range");
            tgt[i] = e->dev_index(el[i].direction * (uint32_t)e->N + el[i].field_idx);
            type[i] = el[i].type_flag;
            const float v[9] = {el[i].i2v, el[i].ilv, el[i].vvd, el[i].vv2, el[i].vj1, el[i].vj2, el[i].ib0, el[i].b1, el[i].b2};
            memcpy(&p[9 * (size_t)i], v, sizeof(v));
        }
        std::vector<uint32_t> ut, off, perm;
        efs_engine::group_by(tgt, ut, off, perm);
        // groups hold element ids in original order; state stays per element
        std::vector<uint32_t> goff(off);
        // k_rlc_apply walks e in [goff[g], goff[g+1]) as element ids: permute element data into group order
        std::vector<uint32_t> type2(n);
        std::vector<float> p2(9 * (size_t)n);
        for (uint32_t i = 0; i < n; ++i) { type2[i] = type[perm[i]]; memcpy(&p2[9 * (size_t)i], &p[9 * (size_t)perm[i]], 36); }
        e->upload(e->rlc_gtarget, ut); e->upload(e->rlc_goff, goff);
        e->h_rlc_series.clear();
        for (uint32_t i = 0; i < n; ++i) if (el[i].type_flag == 1) e->h_rlc_series.push_back(tgt[i]);
        e->upload(e->rlc_type, type2); e->upload(e->rlc_p, p2);
        e->alloc(e->rlc_vdn, 3 * (size_t)n * 4); e->alloc(e->rlc_jn, 3 * (size_t)n * 4); e->alloc(e->rlc_vil, (size_t)n * 4);
        e->rlc_n = n; e->rlc_groups = (uint32_t)ut.size();
        e->rlc_on = n > 0;
        // element order on the device is the grouped order; remember it for state reads
        e->rlc_perm = perm;
        e->dirty();
    });
}

efs_status efs_configure_pbc(efs_engine* e, uint32_t count, const uint32_t* axes, const double* phases) {
    return guard(e, [&] {
        e->need_init();
        if (count && !axes) fail(EFS_ERR_INVALID, "axes must be non-null");
        const uint32_t nl[3] = {e->Nx, e->Ny, e->Nz};
        e->pbc_axes.clear();
        size_t off = 0;
        for (uint32_t i = 0; i < count; ++i) {
            if (axes[i] > 2 || nl[axes[i]] < 2) fail(EFS_ERR_INVALID, "PBC axis invalid");
            double ph = phases ? phases[i] : 0.0;
            uint32_t t0 = (axes[i] + 1) % 3, t1 = (axes[i] + 2) % 3;
            size_t fs = (size_t)nl[t0] * nl[t1];
            e->pbc_axes.push_back({axes[i], (float)std::cos(ph), (float)std::sin(ph), ph != 0.0 ? off : 0});
            if (ph != 0.0) off += 4 * fs;
        }
        e->alloc(e->pbc_imag, std::max<size_t>(off, 1) * 4);
        e->pbc_on = count > 0;
        e->dirty();
    });
}

efs_status efs_configure_steady_state(efs_engine* e, const uint32_t* idx, uint32_t n, uint32_t period, float threshold) {
    return guard(e, [&] {
        e->need_init();
        if (n && !idx) fail(EFS_ERR_INVALID, "probe_idx must be non-null");
        e->check_idx3(idx, n, "steady-state probe_idx");
        std::vector<uint32_t> di(n);
        for (uint32_t i = 0; i < n; ++i) di[i] = e->dev_index(idx[i]);
        e->upload(e->ss_idx, di);
        e->alloc(e->ss_e1, (size_t)n * 4); e->alloc(e->ss_e2, (size_t)n * 4);
        e->ss_n = n; e->ss_period = period; e->ss_threshold = threshold > 0 ? threshold : 1e-6f;
        e->ss_on = n > 0; e->ss_recording = false; e->ss_count_before = 0;
        e->hstate.ss_recording = 0; e->hstate.ss_start = e->numTS; e->hstate.ss_base = 0;
        e->sync_state_to_device();
        e->dirty();
    });
}

efs_status efs_set_steady_state_recording(efs_engine* e, int rec) {
    return guard(e, [&] {
        e->need_init();
        if (!e->ss_on) fail(EFS_ERR_STATE, "steady state not configured");
        bool r = rec != 0;
        if (r == e->ss_recording) return;
        if (!r) e->ss_count_before += e->numTS - e->hstate.ss_start;   // close the window
        e->ss_recording = r;
        e->hstate.ss_recording = r ? 1 : 0;
        e->hstate.ss_start = e->numTS;
        e->hstate.ss_base = e->ss_count_before;
        e->sync_state_to_device();
    });
}

efs_status efs_read_steady_state(efs_engine* e, float* e1, float* e2, uint32_t* cur, int* conv) {
    return guard(e, [&] {
        e->need_init();
        if (!e->ss_on) fail(EFS_ERR_STATE, "steady state not configured");
        std::vector<float> a(e->ss_n), b(e->ss_n);
        ck(cudaMemcpyAsync(a.data(), e->ss_e1.p, (size_t)e->ss_n * 4, cudaMemcpyDeviceToHost, e->stream), "read ss");
        ck(cudaMemcpyAsync(b.data(), e->ss_e2.p, (size_t)e->ss_n * 4, cudaMemcpyDeviceToHost, e->stream), "read ss");
        e->sync("sync");
        uint32_t sample = e->ss_count_before + (e->ss_recording ? e->numTS - e->hstate.ss_start : 0);
        if (e1) memcpy(e1, a.data(), a.size() * 4);
        if (e2) memcpy(e2, b.data(), b.size() * 4);
        if (cur) *cur = sample;
        if (conv) {
            // src/webgpu-fdtd.mjs:1076-1092
            int c = 0;
            if (sample >= 2 * e->ss_period) {
                double mr = 0;
                for (uint32_t i = 0; i < e->ss_n; ++i) {
                    double x1 = a[i], x2 = b[i];
                    if (std::fabs(x1) < 1e-30) continue;
                    mr = std::max(mr, std::fabs(x2 - x1) / std::fabs(x1));
                }
                c = mr < e->ss_threshold ? 1 : 0;
            }
            *conv = c;
        }
    });
}

efs_status efs_iterate(efs_engine* e, uint32_t n) { return guard(e, [&] { e->iterate(n); }); }

efs_status efs_num_ts(const efs_engine* e, uint32_t* out) {
    if (!e || !out) return EFS_ERR_INVALID;
    *out = e->numTS;
    return EFS_OK;
}

efs_status efs_sync(efs_engine* e) { return guard(e, [&] { e->sync("cudaStreamSynchronize"); }); }

efs_status efs_get_stream(efs_engine* e, void** s) {
    if (!e || !s) return EFS_ERR_INVALID;
    *s = (void*)e->stream;
    return EFS_OK;
}

efs_status efs_configure_probe_gather(efs_engine* e, const uint32_t* idx, uint32_t n) {
    return guard(e, [&] {
        e->need_init();
        if (n == 0) return;   // the reference returns without configuring (:2578)
        if (!idx) fail(EFS_ERR_INVALID, "indices must be non-null");
        e->check_idx3(idx, n, "probe index");
        std::vector<uint32_t> di(n);
        for (uint32_t i = 0; i < n; ++i) di[i] = e->dev_index(idx[i]);
        e->upload(e->gd_idx, di);
        e->alloc(e->gd_out, 2 * (size_t)n * 4);
        e->gd_n = n;
    });
}

efs_status efs_read_probe_gather(efs_engine* e, float* out, size_t len) {
    return guard(e, [&] {
        e->need_init();
        if (!e->gd_n) fail(EFS_ERR_STATE, "probe gather not configured");
        if (!out || len < 2 * (size_t)e->gd_n) fail(EFS_ERR_INVALID, "output buffer too small");
        k_gather<<<blocks(e->gd_n, 64), 64, 0, e->stream>>>(e->vcur(), e->ccur(), e->gd_idx.as<uint32_t>(),
                                                             e->gd_n, e->gd_out.as<float>());
        ck(cudaGetLastError(), "gather");
        ck(cudaMemcpyAsync(out, e->gd_out.p, 2 * (size_t)e->gd_n * 4, cudaMemcpyDeviceToHost, e->stream), "read gather");
        e->sync("sync");
    });
}

efs_status efs_configure_probe_gather_buffered(efs_engine* e, const uint32_t* idx, uint32_t n, uint32_t maxS, uint32_t interval) {
    return guard(e, [&] {
        e->need_init();
        if (n == 0) return;   // :2624
        if (!idx) fail(EFS_ERR_INVALID, "indices must be non-null");
        if (interval == 0) fail(EFS_ERR_INVALID, "sample_interval must be > 0");
        e->check_idx3(idx, n, "probe index");
        std::vector<uint32_t> di(n);
        for (uint32_t i = 0; i < n; ++i) di[i] = e->dev_index(idx[i]);
        e->upload(e->ring_idx, di);
        e->alloc(e->ring, (size_t)maxS * n * 2 * 4);
        e->ring_n = n; e->ring_max = maxS; e->ring_interval = interval;
        e->ring_q0 = e->numTS / interval;    // multiples already passed at configure time
        e->ring_on = true;
        e->dirty();
    });
}

efs_status efs_read_probe_gather_buffered(efs_engine* e, float* out, size_t len, uint32_t* ns, uint32_t* stride) {
    return guard(e, [&] {
        e->need_init();
        if (!e->ring_on) fail(EFS_ERR_STATE, "buffered probe gather not configured");
        uint32_t q = e->numTS / e->ring_interval;
        uint32_t s = q > e->ring_q0 ? std::min(q - e->ring_q0, e->ring_max) : 0;
        if (ns) *ns = s;
        if (stride) *stride = 2 * e->ring_n;
        if (!out) return;
        size_t need = (size_t)s * e->ring_n * 2;
        if (len < need) fail(EFS_ERR_INVALID, "output buffer too small");
        if (need) ck(cudaMemcpyAsync(out, e->ring.p, need * 4, cudaMemcpyDeviceToHost, e->stream), "read ring");
        e->sync("sync");
    });
}

efs_status efs_configure_nf2ff(efs_engine* e, const uint32_t* pts, uint32_t np, const double* omegas, uint32_t nf, double dT,
                               const float* el, uint32_t maxTS, uint32_t window) {
    return guard(e, [&] {
        e->need_init();
        if (np == 0) return;   // :2732
        if (!pts || !omegas || !el) fail(EFS_ERR_INVALID, "NF2FF arrays must be non-null");
        if (nf == 0 || nf > (uint32_t)NF_MAX_FREQ) fail(EFS_ERR_RANGE, "NF2FF frequency count must be 1..16");
        for (uint32_t i = 0; i < np; ++i)
            if (pts[3 * i] >= e->Nx || pts[3 * i + 1] >= e->Ny || pts[3 * i + 2] >= e->Nz) fail(EFS_ERR_INVALID, "NF2FF point out of grid");
        e->upload(e->nf_pts, pts, 3 * (size_t)np);
        e->h_nf_pts.assign(pts, pts + 3 * (size_t)np);
        size_t nel = 2 * ((size_t)e->Nx + e->Ny + e->Nz);
        e->upload(e->nf_el, el, nel);
        e->alloc(e->nf_E, (size_t)nf * np * 6 * 4);
        e->alloc(e->nf_H, (size_t)nf * np * 6 * 4);
        e->alloc(e->nf_samp, (size_t)NF_K * 6 * np * 4, false);   // written before read each pass
        Nf2ffDev& d = e->nf;
        memset(&d, 0, sizeof(d));
        d.np = np; d.nf = nf; d.maxTS = maxTS; d.window = window;
        d.Nx = e->Nx; d.Ny = e->Ny; d.Nz = e->Nz; d.Pz = e->Pz;
        const uint32_t nl[3] = {e->Nx, e->Ny, e->Nz};
        uint32_t o = 0;
        for (int k = 0; k < 6; ++k) { d.off[k] = o; o += nl[k % 3]; }
        d.pts = e->nf_pts.as<uint32_t>(); d.el = e->nf_el.as<float>();
        d.accE = e->nf_E.as<float>(); d.accH = e->nf_H.as<float>();
        d.samp = e->nf_samp.as<float>();
        for (uint32_t f = 0; f < nf; ++f) d.wdt[f] = omegas[f] * dT;
        d.dT32 = (float)dT;
        double wn = 1.0;
        if (window == 1 && maxTS > 1) {   // windowNorm (:2765-2772)
            double s = 0;
            for (uint32_t n = 0; n < maxTS; ++n) s += 0.5 * (1 - std::cos(2 * M_PI * n / (double)(maxTS - 1)));
            wn = 1.0 / s;
        }
        d.wnorm = (float)wn;
        e->nf_on = true;
        e->dirty();
    });
}

efs_status efs_read_nf2ff(efs_engine* e, float* accE, float* accH, size_t len) {
    return guard(e, [&] {
        e->need_init();
        if (!e->nf_on) fail(EFS_ERR_STATE, "NF2FF not configured");
        size_t n = (size_t)e->nf.nf * e->nf.np * 6;
        if (len < n) fail(EFS_ERR_INVALID, "output buffer too small");
        if (accE) ck(cudaMemcpyAsync(accE, e->nf_E.p, n * 4, cudaMemcpyDeviceToHost, e->stream), "read nf2ff E");
        if (accH) ck(cudaMemcpyAsync(accH, e->nf_H.p, n * 4, cudaMemcpyDeviceToHost, e->stream), "read nf2ff H");
        e->sync("sync");
    });
}

efs_status efs_far_field(efs_engine* e, uint32_t fi, const float* meta, const float* theta, uint32_t nth, const float* phi,
                         uint32_t nph, const double center[3], double freq, double radius, float* out) {
    return guard(e, [&] {
        e->need_init();
        if (!e->nf_on) fail(EFS_ERR_STATE, "NF2FF not configured");
        if (fi >= e->nf.nf) fail(EFS_ERR_INVALID, "frequency index out of range");
        if (!meta || !theta || !phi || !out || !center || nth == 0 || nph == 0) fail(EFS_ERR_INVALID, "far-field arguments invalid");
        const uint32_t np = e->nf.np;
        const uint64_t A64 = (uint64_t)nth * nph;
        if (A64 >= (1ull << 31)) fail(EFS_ERR_RANGE, "too many far-field angles");
        const uint32_t A = (uint32_t)A64;
        // points grouped by the normal axis of their face (counting sort, stable)
        std::vector<uint32_t> perm(np);
        FarFieldDev d;
        memset(&d, 0, sizeof(d));
        {
            uint32_t cnt[4] = {0, 0, 0, 0};
            for (uint32_t p = 0; p < np; ++p) {
                const float nd = meta[8 * (size_t)p + 3];
                if (!(nd == 0.f || nd == 1.f || nd == 2.f)) fail(EFS_ERR_INVALID, "pointMeta normal direction must be 0, 1 or 2");
                ++cnt[(int)nd + 1];
            }
            for (int n = 0; n < 3; ++n) cnt[n + 1] += cnt[n];
            for (int n = 0; n < 4; ++n) d.seg[n] = cnt[n];
            for (uint32_t p = 0; p < np; ++p) perm[cnt[(int)meta[8 * (size_t)p + 3]]++] = p;
        }
        DevBuf dm, dperm, drec, dth, dph, dout;
        e->upload(dm, meta, 8 * (size_t)np);
        e->upload(dperm, perm);
        e->upload(dth, theta, nth);
        e->upload(dph, phi, nph);
        e->alloc(drec, (size_t)np * sizeof(FfRecord), false);
        e->alloc(dout, (size_t)A * 5 * 4, false);
        const double C0 = 299792458.0;
        const double k = 2 * M_PI * freq / C0;
        const double fmag = k / (4 * M_PI * radius), fph = -k * radius;   // (:2880-2884)
        d.np = np; d.nth = nth; d.nph = nph;
        d.rec = drec.as<FfRecord>();
        d.theta = dth.as<float>(); d.phi = dph.as<float>();
        d.fre = fmag * (-std::sin(fph)); d.fim = fmag * std::cos(fph);
        d.out = dout.as<float>();
        cudaEvent_t ev[3];
        for (auto& x : ev) ck(cudaEventCreate(&x), "event");
        ck(cudaEventRecord(ev[0], e->stream), "record");
        k_ff_prep<<<blocks(np, 256), 256, 0, e->stream>>>(dm.as<float>(), e->nf_E.as<float>() + (size_t)fi * np * 6,
                                                          e->nf_H.as<float>() + (size_t)fi * np * 6, dperm.as<uint32_t>(), np,
                                                          (float)(k / (2 * M_PI)), (float)center[0], (float)center[1],
                                                          (float)center[2], drec.as<FfRecord>());
        ck(cudaEventRecord(ev[1], e->stream), "record");
        k_ff_angles<<<blocks(A, FF_ANG), FF_THREADS, 0, e->stream>>>(d);
        ck(cudaEventRecord(ev[2], e->stream), "record");
        ck(cudaGetLastError(), "far field");
        ck(cudaMemcpyAsync(out, dout.p, (size_t)A * 5 * 4, cudaMemcpyDeviceToHost, e->stream), "read far field");
        e->sync("sync");
        cudaEventElapsedTime(&e->ff_ms[0], ev[0], ev[1]);
        cudaEventElapsedTime(&e->ff_ms[1], ev[1], ev[2]);
        for (auto& x : ev) cudaEventDestroy(x);
    });
}

efs_status efs_far_field_time(const efs_engine* e, float* ms) {
    if (!e || !ms) return EFS_ERR_INVALID;
    ms[0] = e->ff_ms[0];
    ms[1] = e->ff_ms[1];
    return EFS_OK;
}

static void energy_launch(efs_engine* e, int slot) {
    if (!e->en_partial.p) {
        e->alloc(e->en_partial, 1024 * sizeof(double));
        e->alloc(e->en_result, sizeof(double));
    }
    double* res = e->en_result.as<double>();
    if (e->Nx < 2 || e->Ny < 2 || e->Nz < 2) {
        ck(cudaMemsetAsync(res, 0, sizeof(double), e->stream), "memset");
    } else {
        k_energy<<<1024, 256, 0, e->stream>>>(e->vcur(), e->ccur(), e->Nx, e->Ny, e->Nz, e->Pz, e->en_partial.as<double>());
        k_energy_final<<<1, 1024, 0, e->stream>>>(e->en_partial.as<double>(), 1024, res);
    }
    ck(cudaGetLastError(), "energy");
    ck(cudaMemcpyAsync(e->en_host + slot, res, sizeof(double), cudaMemcpyDeviceToHost, e->stream), "energy readback");
    ck(cudaEventRecord(e->en_event[slot], e->stream), "event");
}

efs_status efs_energy(efs_engine* e, int lagged, double* out) {
    return guard(e, [&] {
        e->need_init();
        if (!out) fail(EFS_ERR_INVALID, "out must be non-null");
        if (!lagged) {
            energy_launch(e, e->en_idx);
            ck(cudaEventSynchronize(e->en_event[e->en_idx]), "energy wait");
            *out = e->en_host[e->en_idx];
            return;
        }
        // computeEnergy (:2974-3021): queue this value, return the previous one
        const int cur = e->en_idx, prev = 1 - cur;
        energy_launch(e, cur);
        if (e->en_pending) {
            ck(cudaEventSynchronize(e->en_event[prev]), "energy wait");
            e->en_last = e->en_host[prev];
        }
        e->en_pending = true;
        e->en_idx = prev;
        *out = e->en_last;
    });
}

// ---- energy without device allocation ---------------------------------------
// Scratch of efs_energy_noalloc: a fixed array inside this library (every GPU
// that loads it holds one copy until exit).  Slots [0, EN_NA_MAX_PARTIALS)
// take one partial sum per EN_NA_CELLS interior cells, the last slot the
// result.  A call writes every slot it reads before reading it, so nothing
// carries over from the previous call and nothing needs clearing.  All calls
// on a device share it: calls that overlap on the GPU race.
constexpr uint64_t EN_NA_CELLS = 65536;            // interior cells per partial sum
constexpr uint32_t EN_NA_MAX_PARTIALS = 16384;     // => at most 2^30 interior cells
constexpr int EN_NA_MAX_DEVICES = 64;
static __device__ __align__(256) double g_energy_noalloc[EN_NA_MAX_PARTIALS + 1];
static double* g_energy_noalloc_addr[EN_NA_MAX_DEVICES];   // device address per device ordinal
static std::mutex g_energy_noalloc_mu;

// Device address of g_energy_noalloc on `device`, which the caller has made
// current.  Host code cannot use the array's name as a device pointer: the
// first call per device asks the runtime for the address once.
static double* energy_noalloc_scratch(int device) {
    if (device < 0 || device >= EN_NA_MAX_DEVICES) fail(EFS_ERR_RANGE, "efs_energy_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_energy_noalloc_mu);
    if (!g_energy_noalloc_addr[device]) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_energy_noalloc), "efs_energy_noalloc: cudaGetSymbolAddress");
        if (!p) fail(EFS_ERR_CUDA, "efs_energy_noalloc: no device address for the scratch array");
        g_energy_noalloc_addr[device] = static_cast<double*>(p);
    }
    return g_energy_noalloc_addr[device];
}

efs_status efs_energy_noalloc(efs_engine* e, double* out) {
    return guard(e, [&] {
        e->need_init();
        if (!out) fail(EFS_ERR_INVALID, "out must be non-null");
        const uint64_t inner = (e->Nx < 2 || e->Ny < 2 || e->Nz < 2)
                                   ? 0 : (uint64_t)(e->Nx - 1) * (e->Ny - 1) * (e->Nz - 1);
        const uint64_t parts = (inner + EN_NA_CELLS - 1) / EN_NA_CELLS;
        if (parts > EN_NA_MAX_PARTIALS)
            fail(EFS_ERR_RANGE, "efs_energy_noalloc: the grid has " + std::to_string(inner) +
                                    " interior cells; its fixed scratch covers at most 2^30 (16384 partial sums of 65536 cells)");
        double* scratch = energy_noalloc_scratch(e->device);
        if (parts == 0) {
            *out = 0.0;
            return;
        }
        double* result = scratch + EN_NA_MAX_PARTIALS;
        k_energy_ranges<<<(uint32_t)parts, 256, 0, e->stream>>>(e->vcur(), e->ccur(), e->Nx, e->Ny, e->Nz, e->Pz, EN_NA_CELLS,
                                                                scratch);
        k_energy_final<<<1, 1024, 0, e->stream>>>(scratch, (uint32_t)parts, result);
        ck(cudaGetLastError(), "efs_energy_noalloc");
        ck(cudaMemcpyAsync(out, result, sizeof(double), cudaMemcpyDeviceToHost, e->stream), "efs_energy_noalloc readback");
        e->sync("efs_energy_noalloc");
    });
}

efs_status efs_flush_energy(efs_engine* e, double* out) {
    return guard(e, [&] {
        e->need_init();
        if (e->en_pending) {
            const int slot = 1 - e->en_idx;   // the slot written by the last lagged call
            ck(cudaEventSynchronize(e->en_event[slot]), "energy wait");
            e->en_last = e->en_host[slot];
            e->en_pending = false;
        }
        if (out) *out = e->en_last;
    });
}

efs_status efs_get_fields(efs_engine* e, float* v, float* c) {
    return guard(e, [&] {
        e->need_init();
        if (v) e->copy_fields_out(v, e->vcur());
        if (c) e->copy_fields_out(c, e->ccur());
        e->sync("sync");
    });
}

// x-planes [x, x + count) of E and H, packed as (3, count, Ny*Nz) floats
// (unpadded rows) at volt / curr; host or device memory (cudaMemcpyDefault).
static void plane_copies(efs_engine* e, uint32_t x, uint32_t count, float* v, float* c, bool out) {
    if ((uint64_t)x + count > e->Nx) fail(EFS_ERR_INVALID, "plane range beyond the grid");
    const size_t rows = (size_t)count * e->Ny;
    for (int n = 0; n < 3; ++n) {
        const size_t dev_off = (size_t)n * e->Nd + (size_t)x * e->Ny * e->Pz;
        const size_t pk_off = (size_t)n * rows * e->Nz;
        float* bufs[2] = {v, c};
        float* fields[2] = {e->vcur(), e->ccur()};
        for (int k = 0; k < 2; ++k) {
            if (!bufs[k]) continue;
            if (out)
                ck(cudaMemcpy2DAsync(bufs[k] + pk_off, (size_t)e->Nz * 4, fields[k] + dev_off, (size_t)e->Pz * 4,
                                     (size_t)e->Nz * 4, rows, cudaMemcpyDefault, e->stream), "plane copy out");
            else
                ck(cudaMemcpy2DAsync(fields[k] + dev_off, (size_t)e->Pz * 4, bufs[k] + pk_off, (size_t)e->Nz * 4,
                                     (size_t)e->Nz * 4, rows, cudaMemcpyDefault, e->stream), "plane copy in");
        }
    }
    e->sync("plane copy");
}

efs_status efs_get_planes(efs_engine* e, uint32_t x, uint32_t count, float* volt, float* curr) {
    return guard(e, [&] { e->need_init(); plane_copies(e, x, count, volt, curr, true); });
}

efs_status efs_set_planes(efs_engine* e, uint32_t x, uint32_t count, const float* volt, const float* curr) {
    return guard(e, [&] {
        e->need_init();
        plane_copies(e, x, count, const_cast<float*>(volt), const_cast<float*>(curr), false);
    });
}

efs_status efs_set_fields(efs_engine* e, const float* v, const float* c) {
    return guard(e, [&] {
        e->need_init();
        if (v) e->copy_fields_in(e->vcur(), v);
        if (c) e->copy_fields_in(e->ccur(), c);
        e->sync("sync");
    });
}

// state blob: magic, version, numTS, nbuf, then per buffer (bytes, data)
static std::vector<DevBuf*> state_buffers(efs_engine* e) {
    const int p = e->cur;
    std::vector<DevBuf*> b = {p ? &e->volt_b : &e->volt, p ? &e->curr_b : &e->curr};
    for (auto& r : e->pml) { b.push_back(p && r->vflux_b.p ? &r->vflux_b : &r->vflux); b.push_back(p && r->cflux_b.p ? &r->cflux_b : &r->cflux); }
    if (e->mur_on) b.push_back(&e->mur_saved);
    for (auto* s : {&e->ade_v, &e->ade_c}) if (s->n) { b.push_back(&s->state); b.push_back(&s->lor); }
    if (e->rlc_on) { b.push_back(&e->rlc_vdn); b.push_back(&e->rlc_jn); b.push_back(&e->rlc_vil); }
    if (e->ss_on) { b.push_back(&e->ss_e1); b.push_back(&e->ss_e2); }
    if (e->pbc_on) b.push_back(&e->pbc_imag);
    if (e->ring_on) b.push_back(&e->ring);
    if (e->nf_on) { b.push_back(&e->nf_E); b.push_back(&e->nf_H); }
    return b;
}

efs_status efs_get_state(efs_engine* e, void* buf, size_t cap, size_t* size) {
    return guard(e, [&] {
        e->need_init();
        auto bufs = state_buffers(e);
        size_t total = 4 * sizeof(uint64_t);
        for (auto* d : bufs) total += sizeof(uint64_t) + d->bytes;
        if (size) *size = total;
        if (!buf) return;
        if (cap < total) fail(EFS_ERR_INVALID, "state buffer too small");
        uint8_t* p = static_cast<uint8_t*>(buf);
        uint64_t hdr[4] = {0x45465342u /* "EFSB" */, 1, e->numTS, bufs.size()};
        memcpy(p, hdr, sizeof(hdr));
        p += sizeof(hdr);
        for (auto* d : bufs) {
            uint64_t nb = d->bytes;
            memcpy(p, &nb, 8);
            p += 8;
            ck(cudaMemcpyAsync(p, d->p, d->bytes, cudaMemcpyDeviceToHost, e->stream), "state read");
            p += d->bytes;
        }
        e->sync("sync");
    });
}

efs_status efs_set_state(efs_engine* e, const void* buf, size_t size) {
    return guard(e, [&] {
        e->need_init();
        if (!buf || size < 4 * sizeof(uint64_t)) fail(EFS_ERR_INVALID, "state blob too small");
        const uint8_t* p = static_cast<const uint8_t*>(buf);
        uint64_t hdr[4];
        memcpy(hdr, p, sizeof(hdr));
        p += sizeof(hdr);
        auto bufs = state_buffers(e);
        if (hdr[0] != 0x45465342u || hdr[1] != 1 || hdr[3] != bufs.size()) fail(EFS_ERR_INVALID, "state blob does not match this engine's configuration");
        const uint8_t* end = static_cast<const uint8_t*>(buf) + size;
        for (auto* d : bufs) {
            uint64_t nb;
            if (p + 8 > end) fail(EFS_ERR_INVALID, "state blob truncated");
            memcpy(&nb, p, 8);
            p += 8;
            if (nb != d->bytes || p + nb > end) fail(EFS_ERR_INVALID, "state blob buffer size mismatch");
            ck(cudaMemcpyAsync(d->p, p, nb, cudaMemcpyHostToDevice, e->stream), "state write");
            p += nb;
        }
        e->sync("sync");
        e->numTS = (uint32_t)hdr[2];
        e->sync_state_to_device();
        if (e->ade_v.zero || e->ade_c.zero) {   // restored ADE state may be non-zero: run those sides again
            e->ade_v.clean = e->ade_c.clean = false;
            e->dirty();
        }
    });
}

efs_status efs_debug_read(efs_engine* e, const char* name, uint32_t arg, float* out, size_t cap, size_t* count) {
    return guard(e, [&] {
        e->need_init();
        if (!name) fail(EFS_ERR_INVALID, "name must be non-null");
        std::string s(name);
        const DevBuf* b = nullptr;
        size_t n = 0;
        if (s == "tfsf_faces") {   // planned TFSF z faces of the core update (count, then each face's z)
            e->build_plan();
            if (count) *count = 1 + e->tf.n;
            if (!out) return;
            if (cap < 1 + e->tf.n) fail(EFS_ERR_INVALID, "output buffer too small");
            out[0] = (float)e->tf.n;
            for (uint32_t f = 0; f < e->tf.n; ++f) out[1 + f] = (float)e->tf.z[f];
            return;
        }
        if ((s == "pml_volt_flux" || s == "pml_curr_flux") && arg < e->pml.size()) {
            const int p = e->cur;
            auto& R = *e->pml[arg];
            b = s == "pml_volt_flux" ? (p && R.vflux_b.p ? &R.vflux_b : &R.vflux) : (p && R.cflux_b.p ? &R.cflux_b : &R.cflux);
            n = e->pml[arg]->total;
        } else if (s == "mur_saved" && e->mur_on) { b = &e->mur_saved; n = e->mur_n; }
        else if (s == "ade_volt") { b = &e->ade_v.state; n = e->ade_v.n; }
        else if (s == "ade_volt_lor") { b = &e->ade_v.lor; n = e->ade_v.n; }
        else if (s == "ade_curr") { b = &e->ade_c.state; n = e->ade_c.n; }
        else if (s == "ade_curr_lor") { b = &e->ade_c.lor; n = e->ade_c.n; }
        else if (s == "rlc_vdn" && e->rlc_on) { b = &e->rlc_vdn; n = 3 * (size_t)e->rlc_n; }
        else if (s == "rlc_jn" && e->rlc_on) { b = &e->rlc_jn; n = 3 * (size_t)e->rlc_n; }
        else if (s == "rlc_vil" && e->rlc_on) { b = &e->rlc_vil; n = e->rlc_n; }
        else if (s == "pbc_imag" && e->pbc_on) { b = &e->pbc_imag; n = e->pbc_imag.bytes / 4; }
        else fail(EFS_ERR_INVALID, "unknown or unconfigured state name: " + s);
        if (count) *count = n;
        if (!out) return;
        if (cap < n) fail(EFS_ERR_INVALID, "output buffer too small");
        std::vector<float> tmp(n);
        if (n) ck(cudaMemcpyAsync(tmp.data(), b->p, n * 4, cudaMemcpyDeviceToHost, e->stream), "debug read");
        e->sync("sync");
        if (s == "mur_saved") {
            for (size_t k = 0; k < n; ++k) out[e->mur_perm[k]] = tmp[k];   // caller's entry order
        } else if (s.rfind("rlc_", 0) == 0) {
            // device keeps elements grouped by field cell; restore caller order
            const size_t w = (s == "rlc_vil") ? 1 : 3;
            for (size_t i = 0; i < e->rlc_n; ++i)
                for (size_t q = 0; q < w; ++q) out[e->rlc_perm[i] * w + q] = tmp[i * w + q];
        } else {
            memcpy(out, tmp.data(), n * 4);
        }
    });
}

efs_status efs_debug_set_wait(efs_engine* e, uint64_t wait_ns, uint32_t skip_plane) {
    return guard(e, [&] {
        if (wait_ns == 0 || wait_ns > 10000000000ull) fail(EFS_ERR_INVALID, "wait_ns must be in 1 ns .. 10 s");
        e->wait_ns = wait_ns;
        e->skip_plane = skip_plane;
        e->dirty();
    });
}

efs_status efs_set_plane_depth(efs_engine* e, uint32_t xchunk) {
    return guard(e, [&] {
        if (xchunk == 0 || xchunk > 65535) fail(EFS_ERR_INVALID, "plane depth must be in 1 .. 65535");
        e->xchunk = xchunk;
        e->dirty();
    });
}

efs_status efs_time_core(efs_engine* e, uint32_t reps, float* ms) {
    return guard(e, [&] {
        e->need_init();
        if (!ms || reps == 0) fail(EFS_ERR_INVALID, "ms must be non-null and reps > 0");
        e->build_plan();
        // the fused kernel reads parity cur and writes the other one; repeated
        // launches redo the same step, which is what is timed.  ms[0]: the fused
        // kernel; ms[1]: the UPML passes around it
        cudaEvent_t ev[2];
        for (auto& x : ev) ck(cudaEventCreate(&x), "event");
        auto timed = [&](auto launch) {
            ck(cudaEventRecord(ev[0], e->stream), "record");
            for (uint32_t i = 0; i < reps; ++i) launch();
            ck(cudaEventRecord(ev[1], e->stream), "record");
            ck(cudaEventSynchronize(ev[1]), "sync");
            float t = 0;
            cudaEventElapsedTime(&t, ev[0], ev[1]);
            return t / reps;
        };
        const int p = e->cur;
        const float a = timed([&] { e->launch_fused_tma(p); });
        const float b = e->pml_split() ? timed([&] { e->launch_pml_e(p); }) + timed([&] { e->launch_pml_h(p); }) : 0.f;
        ck(cudaGetLastError(), "fused launch");
        for (auto& x : ev) cudaEventDestroy(x);
        e->sync("fused timing");
        ms[0] = a;
        ms[1] = b;
    });
}

efs_status efs_time_phases(efs_engine* e, uint32_t steps, float* ms) {
    return guard(e, [&] {
        if (!ms || steps == 0 || steps > 64) fail(EFS_ERR_INVALID, "ms must be non-null and steps in 1..64");
        for (int i = 0; i < EFS_PHASES; ++i) ms[i] = 0.f;
        e->run_marked(steps, ms);
        for (int i = 0; i < EFS_PHASES; ++i) ms[i] /= (float)steps;
    });
}

efs_status efs_kernels_per_step(efs_engine* e, uint32_t* out) {
    return guard(e, [&] {
        e->need_init();
        if (!out) fail(EFS_ERR_INVALID, "out must be non-null");
        e->build_plan();
        // fused kernel, UPML E pass, UPML H pass and deferred H (one paired launch when both)
        uint32_t k = 1 + e->pml_split() + ((e->defer_n > 0) || e->pml_split());
        k += e->ss_on + e->ade_v.live() + e->ade_c.live() + 3 * e->mur_on + 2 * e->rlc_on;
        if (e->ade_apply) k += e->ade_v.live() + e->ade_c.live();
        k += (e->tfsf_on && e->tfsf_v.groups) + (e->tfsf_on && e->tfsf_c.groups) + (e->exc_on && e->exc_groups > 0);
        k += e->pbc_on ? 2 * (uint32_t)e->pbc_axes.size() : 0;
        k += (e->nf_on && !(e->nf_pair && e->pml_split())) + e->ring_on;   // paired samples ride on the UPML E pass
        *out = k;
    });
}

efs_status efs_device_bytes(const efs_engine* e, size_t* out) {
    if (!e || !out) return EFS_ERR_INVALID;
    size_t t = 0;
    const DevBuf* all[] = {&e->volt, &e->curr, &e->volt_b, &e->curr_b, &e->defer_cells, &e->mat, &e->table, &e->vv, &e->vi, &e->ii, &e->iv};
    for (auto* b : all) t += b->bytes;
    for (auto& r : e->pml) {
        const DevBuf* rb[] = {&r->vv, &r->vvfo, &r->vvfn, &r->ii, &r->iifo, &r->iifn, &r->vflux, &r->cflux, &r->vflux_b, &r->cflux_b};
        for (auto* b : rb) t += b->bytes;
    }
    t += e->nf_E.bytes + e->nf_H.bytes + e->nf_samp.bytes + e->ring.bytes;
    *out = t;
    return EFS_OK;
}

}  // extern "C"

// batched form: several engines advanced together (same translation unit)
#include "efs_batch.cuh"
