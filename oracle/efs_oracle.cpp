// efs_oracle.cpp — CPU restatement of the reference FDTD engine.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
// B200 engine: it is loaded by tests/, by __graft_entry__.smoke() and by the
// cpu_baseline / --impl reference leg of bench.py, and by nothing else.  The
// product path (efs_b200/) never links, loads or calls it.
//
// What it restates (reference paths are relative to the roman01la/efs tree):
//   * CPUFDTDEngine            src/webgpu-fdtd.mjs:13-1202
//       - updateVoltages        :64-106   (backward curl, index-0 self reference)
//       - updateCurrents        :113-155  (forward curl, loops to N-1)
//       - applyExcitation       :161-185  (C++ past-end semantics: signal[0])
//       - UPML pre/post         :239-358
//       - Lorentz/Drude ADE     :381-454 (state update), plus an opt-in
//         apply step the reference lacks: after the apply-to-voltages block
//         (and after the post-current block for H) every ADE entry's state
//         is subtracted from its field, entry by entry in configuration
//         order (openEMS Engine_Ext_Dispersive Apply2Voltages /
//         Apply2Current semantics); off by default, which is the
//         reference's state-only behaviour
//       - TFSF                  :681-733
//       - lumped RLC            :750-863
//       - Mur ABC 3-phase       :941-1023
//       - steady state          :1037-1092
//       - step() phase order    :1129-1172
//   * PBC / Bloch copy          src/webgpu-engine.mjs:475-584 (WGSL; the CPU
//     engine has none, it runs where WebGPUEngine.iterate puts it, :2461,:2480)
//   * buffered probe gather     src/webgpu-engine.mjs:2623-2694, iterate :2491
//   * NF2FF DFT accumulation    src/webgpu-engine.mjs:637-800 (+ multi-frequency)
//   * NF2FF far field           src/webgpu-engine.mjs:802-986, :2871-2967
//   * energy                    src/webgpu-engine.mjs:3071-3145
//
// Arithmetic modes (runtime-selected, one template per mode):
//   MODE_F32 (0): storage f32, every operation rounded to f32 in the same
//                 order as the WGSL shaders, no FMA contraction (this file is
//                 compiled with -ffp-contract=off).  The CUDA kernels issue
//                 __fmul_rn/__fadd_rn in the same order, so they agree with
//                 this mode bit for bit.
//   MODE_JS  (1): storage f32, intermediates in f64, stored to f32 exactly
//                 where the JS CPUFDTDEngine stores to a Float32Array.
//   MODE_F64 (2): storage and arithmetic in f64: the error reference.
//
// NF2FF phase: the reference shader forms omega*n*dT in f32 (:777-782).  The
// oracle offers both that form (phase_mode 0) and the f64 phase that the B200
// engine uses (phase_mode 1, default).

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <vector>
#include <string>
#include <memory>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { MODE_F32 = 0, MODE_JS = 1, MODE_F64 = 2 };

struct PMLRegionIn {
    uint32_t start[3], num[3];
    std::vector<float> vv, vvfo, vvfn, ii, iifo, iifn;
};

struct EngineBase {
    virtual ~EngineBase() {}
    virtual int mode() const = 0;
};

template <typename S, typename C>
struct Engine : EngineBase {
    int mode_;
    uint32_t Nx, Ny, Nz;
    size_t N;
    uint32_t numTS = 0;
    std::vector<S> volt, curr;

    // coefficients: dense (4 arrays of 3N) or indexed (u32 per cell + 12-float rows)
    bool indexed = false;
    std::vector<float> vv, vi, ii, iv;
    std::vector<uint32_t> mat;
    std::vector<float> table;  // row: vv0 vv1 vv2 vi0 vi1 vi2 ii0 ii1 ii2 iv0 iv1 iv2

    // excitation
    bool exc_on = false;
    std::vector<float> exc_signal, exc_amp;
    std::vector<uint32_t> exc_delay, exc_dir, exc_pos;
    uint32_t exc_period = 0;

    // UPML
    struct Region {
        uint32_t start[3], num[3];
        size_t total;  // 3*nx*ny*nz
        std::vector<float> vv, vvfo, vvfn, ii, iifo, iifn;
        std::vector<S> vflux, cflux;
    };
    std::vector<Region> pml;

    // Mur
    bool mur_on = false;
    std::vector<float> mur_coeff;
    std::vector<uint32_t> mur_normal, mur_shifted;
    std::vector<S> mur_saved;

    // TFSF
    bool tfsf_on = false;
    std::vector<float> tfsf_signal;
    uint32_t tfsf_period = 0;
    struct TPt { uint32_t idx, delay_int; float frac, amp; };
    std::vector<TPt> tfsf_v, tfsf_c;

    // ADE
    struct ADEDir {
        uint32_t dir;
        std::vector<uint32_t> pos;
        std::vector<float> v_int, v_ext, v_lor, i_int, i_ext, i_lor;
        std::vector<S> vade, vlor, cade, clor;
    };
    struct ADEOrder { uint32_t numCells; bool lorentz; std::vector<ADEDir> dirs; };
    std::vector<ADEOrder> ade;
    bool ade_apply = false;   // subtract the ADE state from the fields after the core update

    // RLC
    struct RLCElem { uint32_t field_idx, direction, type_flag; float i2v, ilv, vvd, vv2, vj1, vj2, ib0, b1, b2; };
    std::vector<RLCElem> rlc;
    std::vector<S> rlc_vdn, rlc_jn, rlc_vil;

    // steady state
    bool ss_on = false, ss_recording = false;
    std::vector<uint32_t> ss_idx;
    uint32_t ss_period = 0, ss_sample = 0;
    float ss_threshold = 1e-6f;
    std::vector<S> ss_e1, ss_e2;

    // PBC
    struct PBCAxis { uint32_t axis; float cosP, sinP; uint32_t imagOff; };
    std::vector<PBCAxis> pbc;
    std::vector<S> pbc_imag;

    // buffered gather
    bool gather_on = false;
    std::vector<uint32_t> gather_idx;
    uint32_t gather_max = 0, gather_interval = 1, gather_sample = 0;
    std::vector<S> gather_ring;

    // NF2FF accumulation (F frequencies)
    bool nf_on = false;
    uint32_t nf_np = 0, nf_nf = 0, nf_maxTS = 0, nf_window = 0, nf_phase_mode = 1;
    std::vector<uint32_t> nf_pts;
    std::vector<double> nf_omega;
    double nf_dT = 0;
    float nf_dT32 = 0, nf_wnorm = 1.f;
    std::vector<float> nf_el;  // primal x,y,z then dual x,y,z
    uint32_t nf_off[6];
    std::vector<S> nf_E, nf_H;  // [f][pid*6+k]

    Engine(int m, const uint32_t d[3]) : mode_(m), Nx(d[0]), Ny(d[1]), Nz(d[2]) {
        N = (size_t)Nx * Ny * Nz;
        volt.assign(3 * N, S(0));
        curr.assign(3 * N, S(0));
    }
    int mode() const override { return mode_; }

    inline size_t id(uint32_t n, uint32_t x, uint32_t y, uint32_t z) const {
        return (size_t)n * N + (size_t)x * Ny * Nz + (size_t)y * Nz + z;
    }
    inline float cVV(size_t g, uint32_t n, size_t cell) const { return indexed ? table[(size_t)mat[cell] * 12 + n] : vv[g]; }
    inline float cVI(size_t g, uint32_t n, size_t cell) const { return indexed ? table[(size_t)mat[cell] * 12 + 3 + n] : vi[g]; }
    inline float cII(size_t g, uint32_t n, size_t cell) const { return indexed ? table[(size_t)mat[cell] * 12 + 6 + n] : ii[g]; }
    inline float cIV(size_t g, uint32_t n, size_t cell) const { return indexed ? table[(size_t)mat[cell] * 12 + 9 + n] : iv[g]; }

    // V <- S(S(V*vv) + vi*curl): the multiply is stored first in both the JS
    // engine (volt *= vv) and, by rounding, in the f32 WGSL expression.
    static inline S upd(S Vold, float cv, float ci, C curl) {
        S v1 = S(C(Vold) * C(cv));
        return S(C(v1) + C(ci) * curl);
    }

    // src/webgpu-fdtd.mjs:64-106 — E update, backward differences, shift 0 at index 0
    void updateVoltages() {
        const size_t NyNz = (size_t)Ny * Nz;
        #pragma omp parallel for schedule(static)
        for (int64_t xi = 0; xi < (int64_t)Nx; ++xi) {
            uint32_t x = (uint32_t)xi;
            uint32_t sx = x > 0 ? 1 : 0;
            for (uint32_t y = 0; y < Ny; ++y) {
                uint32_t sy = y > 0 ? 1 : 0;
                for (uint32_t z = 0; z < Nz; ++z) {
                    uint32_t sz = z > 0 ? 1 : 0;
                    size_t cell = (size_t)x * NyNz + (size_t)y * Nz + z;
                    size_t ex = cell, ey = N + cell, ez = 2 * N + cell;
                    // Ex: Hz(y) - Hz(y-1) - Hy(z) + Hy(z-1)
                    C cx = ((C(curr[ez]) - C(curr[ez - sy * Nz])) - C(curr[ey])) + C(curr[ey - sz]);
                    volt[ex] = upd(volt[ex], cVV(ex, 0, cell), cVI(ex, 0, cell), cx);
                    // Ey: Hx(z) - Hx(z-1) - Hz(x) + Hz(x-1)
                    C cy = ((C(curr[ex]) - C(curr[ex - sz])) - C(curr[ez])) + C(curr[ez - sx * NyNz]);
                    volt[ey] = upd(volt[ey], cVV(ey, 1, cell), cVI(ey, 1, cell), cy);
                    // Ez: Hy(x) - Hy(x-1) - Hx(y) + Hx(y-1)
                    C cz = ((C(curr[ey]) - C(curr[ey - sx * NyNz])) - C(curr[ex])) + C(curr[ex - sy * Nz]);
                    volt[ez] = upd(volt[ez], cVV(ez, 2, cell), cVI(ez, 2, cell), cz);
                }
            }
        }
    }

    // src/webgpu-fdtd.mjs:113-155 — H update, forward differences over (Nx-1)(Ny-1)(Nz-1)
    void updateCurrents() {
        const size_t NyNz = (size_t)Ny * Nz;
        if (Nx < 2 || Ny < 2 || Nz < 2) return;
        #pragma omp parallel for schedule(static)
        for (int64_t xi = 0; xi < (int64_t)Nx - 1; ++xi) {
            uint32_t x = (uint32_t)xi;
            for (uint32_t y = 0; y + 1 < Ny; ++y) {
                for (uint32_t z = 0; z + 1 < Nz; ++z) {
                    size_t cell = (size_t)x * NyNz + (size_t)y * Nz + z;
                    size_t hx = cell, hy = N + cell, hz = 2 * N + cell;
                    // Hx: Ez(y) - Ez(y+1) - Ey(z) + Ey(z+1)
                    C cx = ((C(volt[hz]) - C(volt[hz + Nz])) - C(volt[hy])) + C(volt[hy + 1]);
                    curr[hx] = upd(curr[hx], cII(hx, 0, cell), cIV(hx, 0, cell), cx);
                    // Hy: Ex(z) - Ex(z+1) - Ez(x) + Ez(x+1)
                    C cy = ((C(volt[hx]) - C(volt[hx + 1])) - C(volt[hz])) + C(volt[hz + NyNz]);
                    curr[hy] = upd(curr[hy], cII(hy, 1, cell), cIV(hy, 1, cell), cy);
                    // Hz: Ey(x) - Ey(x+1) - Ex(y) + Ex(y+1)
                    C cz = ((C(volt[hy]) - C(volt[hy + NyNz])) - C(volt[hx])) + C(volt[hx + Nz]);
                    curr[hz] = upd(curr[hz], cII(hz, 2, cell), cIV(hz, 2, cell), cz);
                }
            }
        }
    }

    // src/webgpu-fdtd.mjs:161-185 (engine_ext_excitation.cpp semantics)
    void applyExcitation() {
        if (!exc_on) return;
        int64_t length = (int64_t)exc_signal.size();
        int64_t p = (int64_t)numTS + 1;
        if (exc_period > 0) p = exc_period;
        for (size_t n = 0; n < exc_amp.size(); ++n) {
            int64_t e = (int64_t)numTS - (int64_t)exc_delay[n];
            e *= (e > 0) ? 1 : 0;
            e %= p;
            e *= (e < length) ? 1 : 0;
            size_t g = (size_t)exc_dir[n] * N + exc_pos[n];
            volt[g] = S(C(volt[g]) + C(exc_amp[n]) * C(exc_signal[(size_t)e]));
        }
    }

    template <bool VOLT, bool PRE>
    void pmlPass() {
        for (auto& r : pml) {
            const uint32_t nx = r.num[0], ny = r.num[1], nz = r.num[2];
            std::vector<S>& F = VOLT ? volt : curr;
            std::vector<S>& flux = VOLT ? r.vflux : r.cflux;
            const float* A = VOLT ? r.vv.data() : r.ii.data();
            const float* B = VOLT ? r.vvfo.data() : r.iifo.data();
            const float* Fn = VOLT ? r.vvfn.data() : r.iifn.data();
            #pragma omp parallel for schedule(static)
            for (int64_t lxi = 0; lxi < (int64_t)nx; ++lxi) {
                uint32_t lx = (uint32_t)lxi;
                for (uint32_t ly = 0; ly < ny; ++ly)
                    for (uint32_t lz = 0; lz < nz; ++lz)
                        for (uint32_t n = 0; n < 3; ++n) {
                            size_t p = (size_t)n * nx * ny * nz + (size_t)lx * ny * nz + (size_t)ly * nz + lz;
                            size_t g = id(n, lx + r.start[0], ly + r.start[1], lz + r.start[2]);
                            if (PRE) {
                                // f_help = vv*V - vvfo*flux; V = flux; flux = f_help  (:239-262)
                                C fh = C(A[p]) * C(F[g]) - C(B[p]) * C(flux[p]);
                                F[g] = flux[p];
                                flux[p] = S(fh);
                            } else {
                                // f_help = flux; flux = V; V = f_help + vvfn*flux  (:271-294)
                                S fh = flux[p];
                                flux[p] = F[g];
                                F[g] = S(C(fh) + C(Fn[p]) * C(flux[p]));
                            }
                        }
            }
        }
    }

    // src/webgpu-fdtd.mjs:405-454
    template <bool VOLT>
    void updateADE() {
        for (auto& o : ade)
            for (auto& d : o.dirs) {
                const std::vector<S>& F = VOLT ? volt : curr;
                std::vector<S>& st = VOLT ? d.vade : d.cade;
                std::vector<S>& lor = VOLT ? d.vlor : d.clor;
                const std::vector<float>& ki = VOLT ? d.v_int : d.i_int;
                const std::vector<float>& ke = VOLT ? d.v_ext : d.i_ext;
                const std::vector<float>& kl = VOLT ? d.v_lor : d.i_lor;
                for (uint32_t i = 0; i < o.numCells; ++i) {
                    S V = F[(size_t)d.dir * N + d.pos[i]];
                    if (o.lorentz) {
                        lor[i] = S(C(lor[i]) + C(kl[i]) * C(st[i]));
                        st[i] = S(C(ki[i]) * C(st[i]) + C(ke[i]) * (C(V) - C(lor[i])));
                    } else {
                        st[i] = S(C(ki[i]) * C(st[i]) + C(ke[i]) * C(V));
                    }
                }
            }
    }

    // Opt-in apply step (no counterpart in the reference engine): F -= state,
    // every (order, direction, cell) entry in configuration order.
    template <bool VOLT>
    void applyADE() {
        for (auto& o : ade)
            for (auto& d : o.dirs) {
                std::vector<S>& F = VOLT ? volt : curr;
                const std::vector<S>& st = VOLT ? d.vade : d.cade;
                for (uint32_t i = 0; i < o.numCells; ++i) {
                    S& f = F[(size_t)d.dir * N + d.pos[i]];
                    f = S(C(f) - C(st[i]));
                }
            }
    }

    // src/webgpu-fdtd.mjs:694-733
    template <bool VOLT>
    void applyTFSF() {
        if (!tfsf_on) return;
        const std::vector<TPt>& pts = VOLT ? tfsf_v : tfsf_c;
        std::vector<S>& F = VOLT ? volt : curr;
        int64_t L = (int64_t)tfsf_signal.size();
        for (const auto& pt : pts) {
            int64_t d = (int64_t)numTS - (int64_t)pt.delay_int;
            if (d < 0) continue;
            if (tfsf_period > 0) d = d % (int64_t)tfsf_period;
            if (d >= L - 1) continue;
            C delta = C(pt.frac);
            C sig = (C(1) - delta) * C(tfsf_signal[(size_t)d]) + delta * C(tfsf_signal[(size_t)d + 1]);
            F[pt.idx] = S(C(F[pt.idx]) + C(pt.amp) * sig);
        }
    }

    // src/webgpu-fdtd.mjs:775-798 (shift form)
    void preVoltageRLC() {
        for (size_t n = 0; n < rlc.size(); ++n) {
            S* V = &rlc_vdn[n * 3];
            V[2] = V[1];
            V[1] = V[0];
            if (rlc[n].type_flag == 0)
                rlc_vil[n] = S(C(rlc_vil[n]) + (C(rlc[n].i2v) * C(rlc[n].ilv)) * C(V[1]));
        }
    }
    // src/webgpu-fdtd.mjs:827-863
    void applyRLC() {
        for (size_t n = 0; n < rlc.size(); ++n) {
            const RLCElem& e = rlc[n];
            size_t g = (size_t)e.direction * N + e.field_idx;
            S* V = &rlc_vdn[n * 3];
            S* J = &rlc_jn[n * 3];
            V[0] = volt[g];
            J[2] = J[1];
            J[1] = J[0];
            if (e.type_flag == 1) {
                C Il = C(rlc_vil[n]);
                C inner = (((C(V[0]) - Il) + C(e.vv2) * C(V[2])) + C(e.vj1) * C(J[1])) + C(e.vj2) * C(J[2]);
                V[0] = S(C(e.vvd) * inner);
                J[0] = S((C(e.ib0) * (C(V[0]) - C(V[2])) - (C(e.b1) * C(e.ib0)) * C(J[1])) - (C(e.b2) * C(e.ib0)) * C(J[2]));
                volt[g] = V[0];
            }
        }
    }

    // src/webgpu-fdtd.mjs:992-1023
    void murPre() {
        if (!mur_on) return;
        for (size_t n = 0; n < mur_coeff.size(); ++n)
            mur_saved[n] = S(C(volt[mur_shifted[n]]) - C(mur_coeff[n]) * C(volt[mur_normal[n]]));
    }
    void murPost() {
        if (!mur_on) return;
        for (size_t n = 0; n < mur_coeff.size(); ++n)
            mur_saved[n] = S(C(mur_saved[n]) + C(mur_coeff[n]) * C(volt[mur_shifted[n]]));
    }
    void murApply() {
        if (!mur_on) return;
        for (size_t n = 0; n < mur_coeff.size(); ++n) volt[mur_normal[n]] = mur_saved[n];
    }

    // src/webgpu-fdtd.mjs:1054-1070
    void accumulateEnergy() {
        if (!ss_on || !ss_recording) return;
        for (size_t n = 0; n < ss_idx.size(); ++n) {
            C v = C(volt[ss_idx[n]]);
            C e = v * v;
            if (ss_sample < ss_period) ss_e1[n] = S(C(ss_e1[n]) + e);
            else ss_e2[n] = S(C(ss_e2[n]) + e);
        }
        ss_sample++;
    }
    // src/webgpu-fdtd.mjs:1076-1092
    int checkConvergence() const {
        if (!ss_on) return 0;
        if (ss_sample < 2 * ss_period) return 0;
        double maxRatio = 0;
        for (size_t n = 0; n < ss_idx.size(); ++n) {
            double e1 = (double)ss_e1[n], e2 = (double)ss_e2[n];
            if (std::fabs(e1) < 1e-30) continue;
            double r = std::fabs(e2 - e1) / std::fabs(e1);
            if (r > maxRatio) maxRatio = r;
        }
        return maxRatio < ss_threshold ? 1 : 0;
    }

    // src/webgpu-engine.mjs:519-584 (pbc_copy), parameters as built at :2041-2120
    template <bool VOLT>
    void pbcCopy() {
        const uint32_t nl[3] = {Nx, Ny, Nz};
        for (const auto& a : pbc) {
            uint32_t t0 = (a.axis + 1) % 3, t1 = (a.axis + 2) % 3;
            uint32_t fs0 = nl[t0], fs1 = nl[t1];
            uint32_t b0 = VOLT ? fs0 : fs0 - 1, b1 = VOLT ? fs1 : fs1 - 1;
            uint32_t src = VOLT ? nl[a.axis] - 2 : 0, dst = VOLT ? 0 : nl[a.axis] - 2;
            std::vector<S>& F = VOLT ? volt : curr;
            for (uint32_t i0 = 0; i0 < b0; ++i0)
                for (uint32_t i1 = 0; i1 < b1; ++i1) {
                    uint32_t sp[3], dp[3];
                    if (a.axis == 0) { sp[0] = src; sp[1] = i0; sp[2] = i1; dp[0] = dst; dp[1] = i0; dp[2] = i1; }
                    else if (a.axis == 1) { sp[0] = i1; sp[1] = src; sp[2] = i0; dp[0] = i1; dp[1] = dst; dp[2] = i0; }
                    else { sp[0] = i0; sp[1] = i1; sp[2] = src; dp[0] = i0; dp[1] = i1; dp[2] = dst; }
                    size_t s0 = id(t0, sp[0], sp[1], sp[2]), d0 = id(t0, dp[0], dp[1], dp[2]);
                    size_t s1 = id(t1, sp[0], sp[1], sp[2]), d1 = id(t1, dp[0], dp[1], dp[2]);
                    size_t fl = (size_t)i0 * fs1 + i1;
                    if (a.sinP == 0.0f) {
                        F[d0] = S(C(a.cosP) * C(F[s0]));
                        F[d1] = S(C(a.cosP) * C(F[s1]));
                    } else {
                        size_t base = a.imagOff + (VOLT ? 0 : 2 * (size_t)fs0 * fs1);
                        size_t im0 = base + fl, im1 = base + (size_t)fs0 * fs1 + fl;
                        C r0 = C(F[s0]), q0 = C(pbc_imag[im0]);
                        F[d0] = S(C(a.cosP) * r0 - C(a.sinP) * q0);
                        pbc_imag[im0] = S(C(a.sinP) * r0 + C(a.cosP) * q0);
                        C r1 = C(F[s1]), q1 = C(pbc_imag[im1]);
                        F[d1] = S(C(a.cosP) * r1 - C(a.sinP) * q1);
                        pbc_imag[im1] = S(C(a.sinP) * r1 + C(a.cosP) * q1);
                    }
                }
        }
    }

    // src/webgpu-engine.mjs:2657-2665 (buffered gather), trigger at :2491
    void gather() {
        if (!gather_on) return;
        if ((numTS + 1) % gather_interval != 0 || gather_sample >= gather_max) return;
        size_t G = gather_idx.size(), base = (size_t)gather_sample * G * 2;
        for (size_t i = 0; i < G; ++i) {
            gather_ring[base + 2 * i] = volt[gather_idx[i]];
            gather_ring[base + 2 * i + 1] = curr[gather_idx[i]];
        }
        gather_sample++;
    }

    // src/webgpu-engine.mjs:675-799, evaluated at ts = numTS+1 (:2484)
    void nf2ffAccumulate(uint32_t ts) {
        if (!nf_on) return;
        const size_t NyNz = (size_t)Ny * Nz;
        auto fi = [&](uint32_t x, uint32_t y, uint32_t z) { return (size_t)x * NyNz + (size_t)y * Nz + z; };
        // per-frequency phase factors (shared by all points)
        std::vector<C> ce(nf_nf), se(nf_nf), ch(nf_nf), sh(nf_nf), wdt(nf_nf);
        C ww = C(1);
        if (nf_window == 1 && nf_maxTS > 1) {
            if (nf_phase_mode == 0) {
                float nf = (float)ts, Nf = (float)(nf_maxTS - 1);
                ww = C(0.5f * (1.0f - std::cos(2.0f * 3.14159265358979f * nf / Nf)));
            } else {
                ww = C((float)(0.5 * (1.0 - std::cos(2.0 * M_PI * (double)ts / (double)(nf_maxTS - 1)))));
            }
        }
        for (uint32_t f = 0; f < nf_nf; ++f) {
            float cef, sef, chf, shf;
            if (nf_phase_mode == 0) {
                float om = (float)nf_omega[f], tsf = (float)ts;
                float pe = om * tsf * nf_dT32;
                float ph = om * (tsf + 0.5f) * nf_dT32;
                cef = std::cos(pe); sef = std::sin(pe); chf = std::cos(ph); shf = std::sin(ph);
            } else {
                // f64 phase reduced modulo 2*pi, the form used by the B200 kernel
                double pe = std::fmod(nf_omega[f] * nf_dT * (double)ts, 2.0 * M_PI);
                double ph = std::fmod(nf_omega[f] * nf_dT * ((double)ts + 0.5), 2.0 * M_PI);
                cef = (float)std::cos(pe); sef = (float)std::sin(pe);
                chf = (float)std::cos(ph); shf = (float)std::sin(ph);
            }
            ce[f] = C(cef); se[f] = C(sef); ch[f] = C(chf); sh[f] = C(shf);
            wdt[f] = C(S(C(S(ww * C(nf_wnorm))) * C(nf_dT32)));
        }
        const float* el = nf_el.data();
        #pragma omp parallel for schedule(static)
        for (int64_t pi = 0; pi < (int64_t)nf_np; ++pi) {
            uint32_t ix = nf_pts[pi * 3], iy = nf_pts[pi * 3 + 1], iz = nf_pts[pi * 3 + 2];
            size_t base = fi(ix, iy, iz);
            bool atB = (ix >= Nx - 1) || (iy >= Ny - 1) || (iz >= Nz - 1);
            C Ex = 0, Ey = 0, Ez = 0, Hx = 0, Hy = 0, Hz = 0;
            if (!atB) {
                C elX = C(el[nf_off[0] + ix]);
                Ex = (((C(volt[base]) + C(volt[fi(ix, iy + 1, iz)])) + C(volt[fi(ix, iy + 1, iz + 1)])) + C(volt[fi(ix, iy, iz + 1)])) / (C(4) * elX);
                C elY = C(el[nf_off[1] + iy]);
                Ey = (((C(volt[N + base]) + C(volt[N + fi(ix, iy, iz + 1)])) + C(volt[N + fi(ix + 1, iy, iz + 1)])) + C(volt[N + fi(ix + 1, iy, iz)])) / (C(4) * elY);
                C elZ = C(el[nf_off[2] + iz]);
                Ez = (((C(volt[2 * N + base]) + C(volt[2 * N + fi(ix + 1, iy, iz)])) + C(volt[2 * N + fi(ix + 1, iy + 1, iz)])) + C(volt[2 * N + fi(ix, iy + 1, iz)])) / (C(4) * elZ);
            }
            auto lerpH = [&](uint32_t comp, uint32_t pos, uint32_t lim, uint32_t off, size_t up) -> C {
                C d0 = C(el[off + pos]);
                if (!(d0 > C(0))) return C(0);
                C h = C(curr[(size_t)comp * N + base]) / d0;
                if (pos < lim - 1) {
                    C d1 = C(el[off + pos + 1]);
                    C dr = d0 / (d0 + d1);
                    C hu = C(curr[(size_t)comp * N + up]) / d1;
                    h = h * (C(1) - dr) + hu * dr;
                }
                return h;
            };
            Hx = lerpH(0, ix, Nx, nf_off[3], fi(ix + 1 < Nx ? ix + 1 : ix, iy, iz));
            Hy = lerpH(1, iy, Ny, nf_off[4], fi(ix, iy + 1 < Ny ? iy + 1 : iy, iz));
            Hz = lerpH(2, iz, Nz, nf_off[5], fi(ix, iy, iz + 1 < Nz ? iz + 1 : iz));
            const C Ev[3] = {Ex, Ey, Ez}, Hv[3] = {Hx, Hy, Hz};
            for (uint32_t f = 0; f < nf_nf; ++f) {
                S* aE = &nf_E[(size_t)f * nf_np * 6 + (size_t)pi * 6];
                S* aH = &nf_H[(size_t)f * nf_np * 6 + (size_t)pi * 6];
                for (int k = 0; k < 3; ++k) {
                    aE[2 * k] = S(C(aE[2 * k]) + C(S(C(S(Ev[k] * ce[f])) * wdt[f])));
                    aE[2 * k + 1] = S(C(aE[2 * k + 1]) + C(S(C(S(Ev[k] * (-se[f]))) * wdt[f])));
                    aH[2 * k] = S(C(aH[2 * k]) + C(S(C(S(Hv[k] * ch[f])) * wdt[f])));
                    aH[2 * k + 1] = S(C(aH[2 * k + 1]) + C(S(C(S(Hv[k] * (-sh[f]))) * wdt[f])));
                }
            }
        }
    }

    void step() {
        // PRE-VOLTAGE
        accumulateEnergy();
        pmlPass<true, true>();
        updateADE<true>();
        murPre();
        preVoltageRLC();
        // CORE
        updateVoltages();
        // POST-VOLTAGE
        pmlPass<true, false>();
        applyTFSF<true>();
        pbcCopy<true>();
        murPost();
        // APPLY
        applyExcitation();
        murApply();
        applyRLC();
        if (ade_apply) applyADE<true>();
        // CURRENT
        pmlPass<false, true>();
        updateADE<false>();
        updateCurrents();
        pmlPass<false, false>();
        applyTFSF<false>();
        pbcCopy<false>();
        if (ade_apply) applyADE<false>();
        // accumulation passes that follow a step (webgpu-engine.mjs:2483-2499)
        nf2ffAccumulate(numTS + 1);
        gather();
        numTS++;
    }

    // src/webgpu-engine.mjs:3090-3103: sum over (Nx-1)(Ny-1)(Nz-1) cells of v^2+c^2
    double energy() const {
        if (Nx < 2 || Ny < 2 || Nz < 2) return 0.0;
        const size_t NyNz = (size_t)Ny * Nz;
        double tot = 0;
        #pragma omp parallel for reduction(+:tot) schedule(static)
        for (int64_t xi = 0; xi < (int64_t)Nx - 1; ++xi) {
            double part = 0;
            for (uint32_t y = 0; y + 1 < Ny; ++y)
                for (uint32_t z = 0; z + 1 < Nz; ++z) {
                    size_t c = (size_t)xi * NyNz + (size_t)y * Nz + z;
                    for (int n = 0; n < 3; ++n) {
                        double v = (double)volt[n * N + c], i = (double)curr[n * N + c];
                        part += v * v + i * i;
                    }
                }
            tot += part;
        }
        return tot;
    }
};

template <typename F>
auto dispatch(EngineBase* b, F&& f) {
    switch (b->mode()) {
    case MODE_F32: return f(static_cast<Engine<float, float>*>(b));
    case MODE_JS: return f(static_cast<Engine<float, double>*>(b));
    default: return f(static_cast<Engine<double, double>*>(b));
    }
}

template <typename E>
std::vector<typename std::remove_reference<decltype(std::declval<E>().volt[0])>::type>* vec_by_name(E* e, const char* name, int a, int b) {
    std::string s(name);
    if (s == "volt") return &e->volt;
    if (s == "curr") return &e->curr;
    if (s == "pml_volt_flux" && a < (int)e->pml.size()) return &e->pml[a].vflux;
    if (s == "pml_curr_flux" && a < (int)e->pml.size()) return &e->pml[a].cflux;
    if (s == "mur_saved") return &e->mur_saved;
    if (a < (int)e->ade.size() && b < (int)e->ade[a].dirs.size()) {
        auto& d = e->ade[a].dirs[b];
        if (s == "ade_volt") return &d.vade;
        if (s == "ade_volt_lor") return &d.vlor;
        if (s == "ade_curr") return &d.cade;
        if (s == "ade_curr_lor") return &d.clor;
    }
    if (s == "rlc_vdn") return &e->rlc_vdn;
    if (s == "rlc_jn") return &e->rlc_jn;
    if (s == "rlc_vil") return &e->rlc_vil;
    if (s == "ss_e1") return &e->ss_e1;
    if (s == "ss_e2") return &e->ss_e2;
    if (s == "gather_ring") return &e->gather_ring;
    if (s == "nf2ff_E") return &e->nf_E;
    if (s == "nf2ff_H") return &e->nf_H;
    if (s == "pbc_imag") return &e->pbc_imag;
    return nullptr;
}

}  // namespace

extern "C" {

void* or_create(int mode, const uint32_t dims[3], const float* vv, const float* vi, const float* ii, const float* iv) {
    EngineBase* b;
    if (mode == MODE_F32) b = new Engine<float, float>(mode, dims);
    else if (mode == MODE_JS) b = new Engine<float, double>(mode, dims);
    else b = new Engine<double, double>(MODE_F64, dims);
    dispatch(b, [&](auto* e) {
        size_t n3 = 3 * e->N;
        e->vv.assign(vv, vv + n3); e->vi.assign(vi, vi + n3);
        e->ii.assign(ii, ii + n3); e->iv.assign(iv, iv + n3);
        return 0;
    });
    return b;
}

void* or_create_indexed(int mode, const uint32_t dims[3], const uint32_t* mat, const float* table, uint32_t ntable) {
    EngineBase* b;
    if (mode == MODE_F32) b = new Engine<float, float>(mode, dims);
    else if (mode == MODE_JS) b = new Engine<float, double>(mode, dims);
    else b = new Engine<double, double>(MODE_F64, dims);
    dispatch(b, [&](auto* e) {
        e->indexed = true;
        e->mat.assign(mat, mat + e->N);
        e->table.assign(table, table + (size_t)ntable * 12);
        return 0;
    });
    return b;
}

void or_destroy(void* h) { delete static_cast<EngineBase*>(h); }

int or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

uint32_t or_num_ts(void* h) { return dispatch(static_cast<EngineBase*>(h), [](auto* e) { return e->numTS; }); }
void or_set_num_ts(void* h, uint32_t t) { dispatch(static_cast<EngineBase*>(h), [&](auto* e) { e->numTS = t; return 0; }); }

void or_configure_excitation(void* h, const float* signal, uint32_t L, const uint32_t* delay, const float* amp,
                             const uint32_t* dir, const uint32_t* pos, uint32_t n, uint32_t period) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->exc_on = true;
        e->exc_signal.assign(signal, signal + L);
        e->exc_delay.assign(delay, delay + n); e->exc_amp.assign(amp, amp + n);
        e->exc_dir.assign(dir, dir + n); e->exc_pos.assign(pos, pos + n);
        e->exc_period = period;
        return 0;
    });
}

// arrays: 6 pointers per region in the order vv, vvfo, vvfn, ii, iifo, iifn
void or_configure_pml(void* h, uint32_t nreg, const uint32_t* start, const uint32_t* num, const float* const* arrays) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->pml.clear();
        for (uint32_t r = 0; r < nreg; ++r) {
            typename std::remove_reference<decltype(*e)>::type::Region R;
            for (int d = 0; d < 3; ++d) { R.start[d] = start[3 * r + d]; R.num[d] = num[3 * r + d]; }
            R.total = 3 * (size_t)R.num[0] * R.num[1] * R.num[2];
            const float* const* a = arrays + 6 * r;
            R.vv.assign(a[0], a[0] + R.total); R.vvfo.assign(a[1], a[1] + R.total); R.vvfn.assign(a[2], a[2] + R.total);
            R.ii.assign(a[3], a[3] + R.total); R.iifo.assign(a[4], a[4] + R.total); R.iifn.assign(a[5], a[5] + R.total);
            R.vflux.assign(R.total, 0); R.cflux.assign(R.total, 0);
            e->pml.push_back(std::move(R));
        }
        return 0;
    });
}

void or_configure_mur(void* h, const float* coeff, const uint32_t* normal, const uint32_t* shifted, uint32_t n) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->mur_on = true;
        e->mur_coeff.assign(coeff, coeff + n);
        e->mur_normal.assign(normal, normal + n); e->mur_shifted.assign(shifted, shifted + n);
        e->mur_saved.assign(n, 0);
        return 0;
    });
}

void or_configure_tfsf(void* h, const float* signal, uint32_t L, uint32_t period,
                       const uint32_t* v_idx, const uint32_t* v_dint, const float* v_frac, const float* v_amp, uint32_t nv,
                       const uint32_t* c_idx, const uint32_t* c_dint, const float* c_frac, const float* c_amp, uint32_t nc) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->tfsf_on = true;
        e->tfsf_signal.assign(signal, signal + L);
        e->tfsf_period = period;
        e->tfsf_v.clear(); e->tfsf_c.clear();
        for (uint32_t i = 0; i < nv; ++i) e->tfsf_v.push_back({v_idx[i], v_dint[i], v_frac[i], v_amp[i]});
        for (uint32_t i = 0; i < nc; ++i) e->tfsf_c.push_back({c_idx[i], c_dint[i], c_frac[i], c_amp[i]});
        return 0;
    });
}

// ADE: one call per (order, direction); coefficient pointers may be null (zeros)
void or_add_ade(void* h, uint32_t order, uint32_t numCells, int lorentz, uint32_t dir, const uint32_t* pos,
                const float* v_int, const float* v_ext, const float* v_lor,
                const float* i_int, const float* i_ext, const float* i_lor) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        while (e->ade.size() <= order) e->ade.push_back({});
        auto& o = e->ade[order];
        o.numCells = numCells; o.lorentz = lorentz != 0;
        typename std::remove_reference<decltype(*e)>::type::ADEDir d;
        d.dir = dir;
        d.pos.assign(pos, pos + numCells);
        auto cp = [&](std::vector<float>& v, const float* p) { if (p) v.assign(p, p + numCells); else v.assign(numCells, 0.f); };
        cp(d.v_int, v_int); cp(d.v_ext, v_ext); cp(d.v_lor, v_lor);
        cp(d.i_int, i_int); cp(d.i_ext, i_ext); cp(d.i_lor, i_lor);
        d.vade.assign(numCells, 0); d.vlor.assign(numCells, 0); d.cade.assign(numCells, 0); d.clor.assign(numCells, 0);
        o.dirs.push_back(std::move(d));
        return 0;
    });
}

// Opt-in ADE apply step (see applyADE)
void or_set_ade_apply(void* h, int on) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->ade_apply = on != 0;
        return 0;
    });
}

// RLC elements as 12 columns: field_idx, direction, type_flag (u32) then
// i2v ilv vvd vv2 vj1 vj2 ib0 b1 b2 (f32)
void or_configure_rlc(void* h, uint32_t n, const uint32_t* field_idx, const uint32_t* direction, const uint32_t* type_flag,
                      const float* params /* n*9 */) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->rlc.clear();
        for (uint32_t i = 0; i < n; ++i) {
            const float* p = params + 9 * (size_t)i;
            e->rlc.push_back({field_idx[i], direction[i], type_flag[i], p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]});
        }
        e->rlc_vdn.assign(3 * (size_t)n, 0); e->rlc_jn.assign(3 * (size_t)n, 0); e->rlc_vil.assign(n, 0);
        return 0;
    });
}

void or_configure_steady_state(void* h, const uint32_t* idx, uint32_t n, uint32_t periodSamples, float threshold) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->ss_on = true; e->ss_recording = false; e->ss_sample = 0;
        e->ss_idx.assign(idx, idx + n);
        e->ss_period = periodSamples; e->ss_threshold = threshold;
        e->ss_e1.assign(n, 0); e->ss_e2.assign(n, 0);
        return 0;
    });
}
void or_set_steady_state(void* h, int recording, uint32_t currentSample) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) { e->ss_recording = recording != 0; e->ss_sample = currentSample; return 0; });
}
uint32_t or_steady_state_sample(void* h) { return dispatch(static_cast<EngineBase*>(h), [](auto* e) { return e->ss_sample; }); }
int or_check_convergence(void* h) { return dispatch(static_cast<EngineBase*>(h), [](auto* e) { return e->checkConvergence(); }); }

// PBC axes: phases in radians (double), as WebGPUEngine.configurePBC (:1976-2123)
void or_configure_pbc(void* h, uint32_t naxes, const uint32_t* axes, const double* phases) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->pbc.clear();
        const uint32_t nl[3] = {e->Nx, e->Ny, e->Nz};
        size_t off = 0;
        for (uint32_t i = 0; i < naxes; ++i) {
            uint32_t ax = axes[i];
            double ph = phases ? phases[i] : 0.0;
            uint32_t t0 = (ax + 1) % 3, t1 = (ax + 2) % 3;
            size_t fs = (size_t)nl[t0] * nl[t1];
            e->pbc.push_back({ax, (float)std::cos(ph), (float)std::sin(ph), (uint32_t)(ph != 0.0 ? off : 0)});
            if (ph != 0.0) off += 4 * fs;
        }
        e->pbc_imag.assign(std::max<size_t>(off, 1), 0);
        return 0;
    });
}

void or_configure_gather(void* h, const uint32_t* idx, uint32_t G, uint32_t maxSamples, uint32_t interval) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->gather_on = G > 0;
        e->gather_idx.assign(idx, idx + G);
        e->gather_max = maxSamples; e->gather_interval = interval ? interval : 1; e->gather_sample = 0;
        e->gather_ring.assign((size_t)maxSamples * G * 2, 0);
        return 0;
    });
}
uint32_t or_gather_samples(void* h) { return dispatch(static_cast<EngineBase*>(h), [](auto* e) { return e->gather_sample; }); }

// NF2FF accumulation: points as (ix,iy,iz) triplets, F angular frequencies,
// edge lengths concatenated primal x,y,z then dual x,y,z (lengths Nx,Ny,Nz each)
void or_configure_nf2ff(void* h, const uint32_t* pts, uint32_t np, const double* omegas, uint32_t nf, double dT,
                        const float* primal_dual, uint32_t maxTS, uint32_t windowType, int phase_mode) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        e->nf_on = np > 0;
        e->nf_np = np; e->nf_nf = nf;
        e->nf_pts.assign(pts, pts + 3 * (size_t)np);
        e->nf_omega.assign(omegas, omegas + nf);
        e->nf_dT = dT; e->nf_dT32 = (float)dT;
        e->nf_maxTS = maxTS; e->nf_window = windowType; e->nf_phase_mode = phase_mode;
        size_t tot = 2 * ((size_t)e->Nx + e->Ny + e->Nz);
        e->nf_el.assign(primal_dual, primal_dual + tot);
        const uint32_t nl[3] = {e->Nx, e->Ny, e->Nz};
        uint32_t o = 0;
        for (int k = 0; k < 6; ++k) { e->nf_off[k] = o; o += nl[k % 3]; }
        double wn = 1.0;
        if (windowType == 1 && maxTS > 1) {
            double s = 0;
            for (uint32_t n = 0; n < maxTS; ++n) s += 0.5 * (1 - std::cos(2 * M_PI * n / (double)(maxTS - 1)));
            wn = 1.0 / s;
        }
        e->nf_wnorm = (float)wn;
        e->nf_E.assign((size_t)nf * np * 6, 0); e->nf_H.assign((size_t)nf * np * 6, 0);
        return 0;
    });
}

void or_step(void* h) { dispatch(static_cast<EngineBase*>(h), [](auto* e) { e->step(); return 0; }); }
void or_iterate(void* h, uint32_t n) {
    dispatch(static_cast<EngineBase*>(h), [&](auto* e) { for (uint32_t i = 0; i < n; ++i) e->step(); return 0; });
}

// Individual phases, for the known-answer tests of single operations.
int or_phase(void* h, const char* name) {
    std::string s(name);
    return dispatch(static_cast<EngineBase*>(h), [&](auto* e) {
        if (s == "updateVoltages") e->updateVoltages();
        else if (s == "updateCurrents") e->updateCurrents();
        else if (s == "applyExcitation") e->applyExcitation();
        else if (s == "preVoltageUpdatePML") e->template pmlPass<true, true>();
        else if (s == "postVoltageUpdatePML") e->template pmlPass<true, false>();
        else if (s == "preCurrentUpdatePML") e->template pmlPass<false, true>();
        else if (s == "postCurrentUpdatePML") e->template pmlPass<false, false>();
        else if (s == "updateVoltADE") e->template updateADE<true>();
        else if (s == "updateCurrADE") e->template updateADE<false>();
        else if (s == "applyVoltADE") e->template applyADE<true>();
        else if (s == "applyCurrADE") e->template applyADE<false>();
        else if (s == "applyTFSFVoltage") e->template applyTFSF<true>();
        else if (s == "applyTFSFCurrent") e->template applyTFSF<false>();
        else if (s == "preVoltageRLC") e->preVoltageRLC();
        else if (s == "applyRLC") e->applyRLC();
        else if (s == "updateRLC") { e->preVoltageRLC(); e->applyRLC(); }
        else if (s == "murPreVoltage") e->murPre();
        else if (s == "murPostVoltage") e->murPost();
        else if (s == "murApply") e->murApply();
        else if (s == "accumulateEnergy") e->accumulateEnergy();
        else if (s == "pbcVoltage") e->template pbcCopy<true>();
        else if (s == "pbcCurrent") e->template pbcCopy<false>();
        else if (s == "step") e->step();
        else return -1;
        return 0;
    });
}

// State access by name, converted through double.  Returns the element count
// (or -1 for an unknown name).  `out` may be null to query the size.
int64_t or_read(void* h, const char* name, int a, int b, double* out, int64_t cap) {
    return dispatch(static_cast<EngineBase*>(h), [&](auto* e) -> int64_t {
        auto* v = vec_by_name(e, name, a, b);
        if (!v) return -1;
        int64_t n = (int64_t)v->size();
        if (out) for (int64_t i = 0; i < std::min(n, cap); ++i) out[i] = (double)(*v)[i];
        return n;
    });
}
int64_t or_write(void* h, const char* name, int a, int b, const double* in, int64_t n) {
    return dispatch(static_cast<EngineBase*>(h), [&](auto* e) -> int64_t {
        auto* v = vec_by_name(e, name, a, b);
        if (!v) return -1;
        using T = typename std::remove_reference<decltype((*v)[0])>::type;
        int64_t m = std::min<int64_t>(n, (int64_t)v->size());
        for (int64_t i = 0; i < m; ++i) (*v)[i] = T(in[i]);
        return m;
    });
}

double or_energy(void* h) { return dispatch(static_cast<EngineBase*>(h), [](auto* e) { return e->energy(); }); }

// NF2FF far field in f64 (restates the math of webgpu-engine.mjs:830-985 and
// the host factor of :2871-2884).  accE/accH: 6 floats per point (re/im of
// x,y,z); meta: 8 floats per point (pos xyz, normalDir, normSign, area, 0, 0).
// out: 5 doubles per angle (P_rad, Et_re, Et_im, Ep_re, Ep_im).
void or_far_field(const float* accE, const float* accH, const float* meta, uint32_t np,
                  const float* theta, uint32_t nth, const float* phi, uint32_t nph,
                  double freq, double radius, const double center[3], double* out) {
    const double C0 = 299792458.0, Z0 = 376.73031346177066;
    const double k = 2 * M_PI * freq / C0;
    const double fac_mag = k / (4 * M_PI * radius), fac_ph = -k * radius;
    const double fre = fac_mag * (-std::sin(fac_ph)), fim = fac_mag * std::cos(fac_ph);
    const int64_t A = (int64_t)nth * nph;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t a = 0; a < A; ++a) {
        double th = theta[a / nph], ph = phi[a % nph];
        double sT = std::sin(th), cT = std::cos(th), sP = std::sin(ph), cP = std::cos(ph);
        double Ntr = 0, Nti = 0, Npr = 0, Npi = 0, Ltr = 0, Lti = 0, Lpr = 0, Lpi = 0;
        for (uint32_t p = 0; p < np; ++p) {
            const float* m = meta + 8 * (size_t)p;
            const float* E = accE + 6 * (size_t)p;
            const float* H = accH + 6 * (size_t)p;
            int nd = (int)m[3];
            double s = m[4], area = m[5];
            double Js[3][2] = {{0, 0}, {0, 0}, {0, 0}}, Ms[3][2] = {{0, 0}, {0, 0}, {0, 0}};
            for (int c = 0; c < 2; ++c) {
                if (nd == 0) {
                    Js[1][c] = -s * H[4 + c]; Js[2][c] = s * H[2 + c];
                    Ms[1][c] = s * E[4 + c];  Ms[2][c] = -s * E[2 + c];
                } else if (nd == 1) {
                    Js[0][c] = s * H[4 + c];  Js[2][c] = -s * H[0 + c];
                    Ms[0][c] = -s * E[4 + c]; Ms[2][c] = s * E[0 + c];
                } else {
                    Js[0][c] = -s * H[2 + c]; Js[1][c] = s * H[0 + c];
                    Ms[0][c] = s * E[2 + c];  Ms[1][c] = -s * E[0 + c];
                }
            }
            double rc = (m[0] - center[0]) * sT * cP + (m[1] - center[1]) * sT * sP + (m[2] - center[2]) * cT;
            double phs = k * rc;
            double ar = area * std::cos(phs), ai = area * std::sin(phs);
            double Jt[2], Jp[2], Mt[2], Mp[2];
            for (int c = 0; c < 2; ++c) {
                Jt[c] = Js[0][c] * cT * cP + Js[1][c] * cT * sP - Js[2][c] * sT;
                Jp[c] = Js[1][c] * cP - Js[0][c] * sP;
                Mt[c] = Ms[0][c] * cT * cP + Ms[1][c] * cT * sP - Ms[2][c] * sT;
                Mp[c] = Ms[1][c] * cP - Ms[0][c] * sP;
            }
            Ntr += ar * Jt[0] - ai * Jt[1]; Nti += ar * Jt[1] + ai * Jt[0];
            Npr += ar * Jp[0] - ai * Jp[1]; Npi += ar * Jp[1] + ai * Jp[0];
            Ltr += ar * Mt[0] - ai * Mt[1]; Lti += ar * Mt[1] + ai * Mt[0];
            Lpr += ar * Mp[0] - ai * Mp[1]; Lpi += ar * Mp[1] + ai * Mp[0];
        }
        double ar_ = Lpr + Z0 * Ntr, ai_ = Lpi + Z0 * Nti;
        double Etr = -(fre * ar_ - fim * ai_), Eti = -(fre * ai_ + fim * ar_);
        double br = Ltr - Z0 * Npr, bi = Lti - Z0 * Npi;
        double Epr = fre * br - fim * bi, Epi = fre * bi + fim * br;
        double P = (Etr * Etr + Eti * Eti + Epr * Epr + Epi * Epi) / (2 * Z0);
        double* o = out + 5 * a;
        o[0] = P; o[1] = Etr; o[2] = Eti; o[3] = Epr; o[4] = Epi;
    }
}

}  // extern "C"
