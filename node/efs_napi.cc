// efs_napi.cc — Node-API addon over libefs.so (include/efs.h).
//
// The JavaScript class in cuda-engine.mjs keeps WebGPUEngine's method names
// and argument objects (src/webgpu-engine.mjs:994-3498 of the reference) and
// calls the functions below; each function checks its arguments, calls one
// or two efs_* entry points and turns a non-zero efs_status into a thrown JS
// Error carrying efs_last_error().  Typed arrays are passed by pointer
// (libefs copies what it keeps before returning), results come back as fresh
// typed arrays.  Readbacks synchronise the engine's CUDA stream on the
// calling thread; iterate only enqueues work (one CUDA graph launch per 64
// timesteps), like WebGPUEngine.iterate encodes and submits without waiting.
//
// Build (node-gyp, binding.gyp beside this file): include_dirs ../include,
// libraries -L../efs_b200 -lefs.
#include <node_api.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "efs.h"

namespace {

// ---- plumbing -----------------------------------------------------------
struct Handle {
    efs_engine* e = nullptr;
};

#define NAPI_OK(call)                                                   \
    do {                                                                \
        if ((call) != napi_ok) {                                        \
            napi_throw_error(env, nullptr, "N-API call failed: " #call); \
            return nullptr;                                             \
        }                                                               \
    } while (0)

napi_value Throw(napi_env env, const std::string& msg) {
    napi_throw_error(env, nullptr, msg.c_str());
    return nullptr;
}

// efs_status -> JS Error (EFS_OK returns true)
bool Check(napi_env env, efs_engine* e, efs_status st, const char* what) {
    if (st == EFS_OK) return true;
    std::string m = std::string(what) + " failed (status " + std::to_string((int)st) + "): " + efs_last_error(e);
    napi_throw_error(env, nullptr, m.c_str());
    return false;
}

struct Args {
    size_t argc = 16;
    napi_value argv[16];
};

bool GetArgs(napi_env env, napi_callback_info info, Args& a, size_t need) {
    if (napi_get_cb_info(env, info, &a.argc, a.argv, nullptr, nullptr) != napi_ok) return false;
    if (a.argc < need) {
        napi_throw_type_error(env, nullptr, ("expected " + std::to_string(need) + " arguments").c_str());
        return false;
    }
    return true;
}

efs_engine* GetEngine(napi_env env, napi_value v) {
    void* p = nullptr;
    if (napi_get_value_external(env, v, &p) != napi_ok || !p || !static_cast<Handle*>(p)->e) {
        napi_throw_error(env, nullptr, "CUDA engine not initialized. Call initGPU() first.");
        return nullptr;
    }
    return static_cast<Handle*>(p)->e;
}

// typed array view (element type checked)
template <typename T>
bool GetTyped(napi_env env, napi_value v, napi_typedarray_type want, const T** data, size_t* len, const char* what) {
    bool is = false;
    napi_is_typedarray(env, v, &is);
    if (!is) {
        napi_throw_type_error(env, nullptr, (std::string(what) + " must be a typed array").c_str());
        return false;
    }
    napi_typedarray_type t;
    void* p = nullptr;
    napi_value ab;
    size_t off = 0;
    napi_get_typedarray_info(env, v, &t, len, &p, &ab, &off);
    if (t != want) {
        napi_throw_type_error(env, nullptr, (std::string(what) + " has the wrong element type").c_str());
        return false;
    }
    *data = static_cast<const T*>(p);
    return true;
}
bool F32(napi_env env, napi_value v, const float** d, size_t* n, const char* w) { return GetTyped(env, v, napi_float32_array, d, n, w); }
bool U32(napi_env env, napi_value v, const uint32_t** d, size_t* n, const char* w) { return GetTyped(env, v, napi_uint32_array, d, n, w); }
bool F64(napi_env env, napi_value v, const double** d, size_t* n, const char* w) { return GetTyped(env, v, napi_float64_array, d, n, w); }
bool U8(napi_env env, napi_value v, const uint8_t** d, size_t* n, const char* w) { return GetTyped(env, v, napi_uint8_array, d, n, w); }

bool GetU32(napi_env env, napi_value v, uint32_t* out) { return napi_get_value_uint32(env, v, out) == napi_ok; }
bool GetF64(napi_env env, napi_value v, double* out) { return napi_get_value_double(env, v, out) == napi_ok; }

napi_value Prop(napi_env env, napi_value obj, const char* name) {
    napi_value v = nullptr;
    napi_get_named_property(env, obj, name, &v);
    return v;
}
bool HasProp(napi_env env, napi_value obj, const char* name) {
    bool has = false;
    napi_has_named_property(env, obj, name, &has);
    if (!has) return false;
    napi_valuetype t;
    napi_typeof(env, Prop(env, obj, name), &t);
    return t != napi_undefined && t != napi_null;
}

napi_value NewF32(napi_env env, const float* src, size_t n) {
    napi_value ab, arr;
    void* p = nullptr;
    napi_create_arraybuffer(env, n * 4, &p, &ab);
    if (n) memcpy(p, src, n * 4);
    napi_create_typedarray(env, napi_float32_array, n, ab, 0, &arr);
    return arr;
}
napi_value Num(napi_env env, double v) {
    napi_value r;
    napi_create_double(env, v, &r);
    return r;
}
napi_value Undefined(napi_env env) {
    napi_value r;
    napi_get_undefined(env, &r);
    return r;
}

// ---- engine lifetime -------------------------------------------------------
void Finalize(napi_env, void* data, void*) {
    auto* h = static_cast<Handle*>(data);
    if (h->e) efs_destroy(h->e);
    delete h;
}

// create(device) -> handle | null (initGPU returns false when no device, :1107-1135)
napi_value Create(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 0)) return nullptr;
    uint32_t dev = 0;
    if (a.argc > 0) GetU32(env, a.argv[0], &dev);
    efs_engine* e = nullptr;
    if (efs_create(&e, (int)dev) != EFS_OK) {
        napi_value n;
        napi_get_null(env, &n);
        return n;
    }
    auto* h = new Handle{e};
    napi_value out;
    NAPI_OK(napi_create_external(env, h, Finalize, nullptr, &out));
    return out;
}

napi_value Destroy(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    void* p = nullptr;
    if (napi_get_value_external(env, a.argv[0], &p) == napi_ok && p) {
        auto* h = static_cast<Handle*>(p);
        if (h->e) efs_destroy(h->e);
        h->e = nullptr;
    }
    return Undefined(env);
}

// init(h, dims: Uint32Array(3), vv, vi, ii, iv: Float32Array(3N))   (:1143-1185)
napi_value Init(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 6)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* dims; size_t nd;
    const float* c[4]; size_t nc[4];
    if (!U32(env, a.argv[1], &dims, &nd, "gridSize") || nd != 3) return Throw(env, "gridSize must hold 3 values");
    const char* names[4] = {"vv", "vi", "ii", "iv"};
    const size_t N3 = 3 * (size_t)dims[0] * dims[1] * dims[2];
    for (int k = 0; k < 4; ++k) {
        if (!F32(env, a.argv[2 + k], &c[k], &nc[k], names[k])) return nullptr;
        if (nc[k] != N3) return Throw(env, std::string(names[k]) + " must hold 3*Nx*Ny*Nz values");
    }
    Check(env, e, efs_init(e, dims, c[0], c[1], c[2], c[3]), "init");
    return Undefined(env);
}

// initIndexed(h, dims, mat: Uint32Array(N), table: Float32Array(12*rows))   (no reference counterpart)
napi_value InitIndexed(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 4)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t *dims, *mat; const float* tab; size_t nd, nm, nt;
    if (!U32(env, a.argv[1], &dims, &nd, "gridSize") || nd != 3) return Throw(env, "gridSize must hold 3 values");
    if (!U32(env, a.argv[2], &mat, &nm, "mat") || !F32(env, a.argv[3], &tab, &nt, "table")) return nullptr;
    if (nm != (size_t)dims[0] * dims[1] * dims[2] || nt % 12 != 0) return Throw(env, "mat/table sizes do not match the grid");
    Check(env, e, efs_init_indexed(e, dims, mat, tab, (uint32_t)(nt / 12)), "initIndexed");
    return Undefined(env);
}

// ---- configure* ----------------------------------------------------------------
// configureExcitation(h, signal, delay, amp, dir, pos, period)   (:1199-1227)
napi_value ConfigureExcitation(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 7)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const float *sig, *amp; const uint32_t *delay, *dir, *pos; size_t ns, na, ndl, ndr, np;
    if (!F32(env, a.argv[1], &sig, &ns, "signal") || !U32(env, a.argv[2], &delay, &ndl, "delay") ||
        !F32(env, a.argv[3], &amp, &na, "amp") || !U32(env, a.argv[4], &dir, &ndr, "dir") || !U32(env, a.argv[5], &pos, &np, "pos"))
        return nullptr;
    if (ndl != na || ndr != na || np != na) return Throw(env, "excitation arrays must have equal lengths");
    uint32_t period = 0;
    GetU32(env, a.argv[6], &period);
    Check(env, e, efs_configure_excitation(e, sig, (uint32_t)ns, delay, amp, dir, pos, (uint32_t)na, period), "configureExcitation");
    return Undefined(env);
}

// configurePML(h, [{startPos, numLines, vv, vvfo, vvfn, ii, iifo, iifn}])   (:1235-1323)
napi_value ConfigurePML(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    NAPI_OK(napi_get_array_length(env, a.argv[1], &n));
    std::vector<efs_pml_region> regs(n);
    const char* keys[6] = {"vv", "vvfo", "vvfn", "ii", "iifo", "iifn"};
    for (uint32_t r = 0; r < n; ++r) {
        napi_value obj;
        NAPI_OK(napi_get_element(env, a.argv[1], r, &obj));
        for (int d = 0; d < 3; ++d) {
            napi_value v;
            napi_get_element(env, Prop(env, obj, "startPos"), d, &v);
            GetU32(env, v, &regs[r].start[d]);
            napi_get_element(env, Prop(env, obj, "numLines"), d, &v);
            GetU32(env, v, &regs[r].num[d]);
        }
        const float* p[6]; size_t len;
        const size_t total = 3 * (size_t)regs[r].num[0] * regs[r].num[1] * regs[r].num[2];
        for (int k = 0; k < 6; ++k) {
            if (!F32(env, Prop(env, obj, keys[k]), &p[k], &len, keys[k])) return nullptr;
            if (len != total) return Throw(env, std::string("PML array ") + keys[k] + " size does not match numLines");
        }
        regs[r].vv = p[0]; regs[r].vvfo = p[1]; regs[r].vvfn = p[2];
        regs[r].ii = p[3]; regs[r].iifo = p[4]; regs[r].iifn = p[5];
    }
    Check(env, e, efs_configure_pml(e, n, regs.data()), "configurePML");
    return Undefined(env);
}

// configureMur(h, coeff: Float32Array, normal_idx, shifted_idx)   (:1822-1918; the dual
// form is concatenated nyP then nyPP by the JS class, as the reference does)
napi_value ConfigureMur(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 4)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const float* c; const uint32_t *nrm, *sh; size_t nc, nn, ns;
    if (!F32(env, a.argv[1], &c, &nc, "coeff") || !U32(env, a.argv[2], &nrm, &nn, "normal_idx") ||
        !U32(env, a.argv[3], &sh, &ns, "shifted_idx"))
        return nullptr;
    if (nc != nn || ns != nn) return Throw(env, "Mur arrays must have equal lengths");
    Check(env, e, efs_configure_mur(e, c, nrm, sh, (uint32_t)nn), "configureMur");
    return Undefined(env);
}

// configureTFSF(h, signal, period, vField, vDelayInt, vDelayFrac, vAmp, cField, cDelayInt, cDelayFrac, cAmp)
// (:1527-1645; the JS class packs the {field_idx, delay_int, delay_frac, amp} objects)
bool Points(napi_env env, napi_value* v, std::vector<efs_tfsf_point>& out) {
    const uint32_t *fi, *di; const float *df, *am; size_t n1, n2, n3, n4;
    if (!U32(env, v[0], &fi, &n1, "field_idx") || !U32(env, v[1], &di, &n2, "delay_int") ||
        !F32(env, v[2], &df, &n3, "delay_frac") || !F32(env, v[3], &am, &n4, "amp"))
        return false;
    if (n2 != n1 || n3 != n1 || n4 != n1) {
        napi_throw_error(env, nullptr, "TFSF point arrays must have equal lengths");
        return false;
    }
    out.resize(n1);
    for (size_t i = 0; i < n1; ++i) out[i] = efs_tfsf_point{fi[i], di[i], df[i], am[i]};
    return true;
}
napi_value ConfigureTFSF(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 11)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const float* sig; size_t ns;
    if (!F32(env, a.argv[1], &sig, &ns, "signal")) return nullptr;
    uint32_t period = 0;
    GetU32(env, a.argv[2], &period);
    std::vector<efs_tfsf_point> vp, cp;
    if (!Points(env, a.argv + 3, vp) || !Points(env, a.argv + 7, cp)) return nullptr;
    Check(env, e, efs_configure_tfsf(e, sig, (uint32_t)ns, period, vp.data(), (uint32_t)vp.size(), cp.data(), (uint32_t)cp.size()),
          "configureTFSF");
    return Undefined(env);
}

// configureADE(h, orders, apply)   (:1358-1475: {numCells, hasLorentz, directions: [{dir, pos_idx,
// v_int_ADE, v_ext_ADE, v_Lor_ADE, i_int_ADE, i_ext_ADE, i_Lor_ADE}]}; `apply` turns on the apply
// step the reference lacks, efs_configure_ade_apply)
napi_value ConfigureADE(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 3)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t no = 0;
    NAPI_OK(napi_get_array_length(env, a.argv[1], &no));
    std::vector<efs_ade_order> orders(no);
    std::vector<std::vector<efs_ade_direction>> dirs(no);
    const char* keys[6] = {"v_int_ADE", "v_ext_ADE", "v_Lor_ADE", "i_int_ADE", "i_ext_ADE", "i_Lor_ADE"};
    for (uint32_t o = 0; o < no; ++o) {
        napi_value od;
        NAPI_OK(napi_get_element(env, a.argv[1], o, &od));
        uint32_t cells = 0;
        GetU32(env, Prop(env, od, "numCells"), &cells);
        bool lor = false;
        napi_get_value_bool(env, Prop(env, od, "hasLorentz"), &lor);
        napi_value dl = Prop(env, od, "directions");
        uint32_t nd = 0;
        NAPI_OK(napi_get_array_length(env, dl, &nd));
        dirs[o].resize(nd);
        for (uint32_t d = 0; d < nd; ++d) {
            napi_value dv;
            NAPI_OK(napi_get_element(env, dl, d, &dv));
            efs_ade_direction& D = dirs[o][d];
            memset(&D, 0, sizeof(D));
            GetU32(env, Prop(env, dv, "dir"), &D.dir);
            size_t len;
            if (!U32(env, Prop(env, dv, "pos_idx"), &D.pos_idx, &len, "pos_idx")) return nullptr;
            if (len != cells) return Throw(env, "pos_idx length must equal numCells");
            const float** dst[6] = {&D.v_int, &D.v_ext, &D.v_lor, &D.i_int, &D.i_ext, &D.i_lor};
            for (int k = 0; k < 6; ++k) {
                if (!HasProp(env, dv, keys[k])) continue;     // absent: zeros (:384-392)
                if (!F32(env, Prop(env, dv, keys[k]), dst[k], &len, keys[k])) return nullptr;
                if (len != cells) return Throw(env, std::string(keys[k]) + " length must equal numCells");
            }
        }
        orders[o] = efs_ade_order{cells, lor ? 1u : 0u, nd, dirs[o].data()};
    }
    if (!Check(env, e, efs_configure_ade(e, no, orders.data()), "configureLorentzADE")) return nullptr;
    bool apply = false;
    napi_get_value_bool(env, a.argv[2], &apply);
    Check(env, e, efs_configure_ade_apply(e, apply ? 1 : 0), "configureLorentzADE (apply)");
    return Undefined(env);
}

// configureRLC(h, u32: Uint32Array(3n) {field_idx, direction, type_flag}, f32: Float32Array(9n)
// {i2v ilv vvd vv2 vj1 vj2 ib0 b1 b2})   (:1722-1808, the reference's 48-byte element packing)
napi_value ConfigureRLC(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 3)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* u; const float* f; size_t nu, nf;
    if (!U32(env, a.argv[1], &u, &nu, "element words") || !F32(env, a.argv[2], &f, &nf, "element values")) return nullptr;
    if (nu % 3 != 0 || nf != 3 * nu) return Throw(env, "RLC element arrays do not match");
    const size_t n = nu / 3;
    std::vector<efs_rlc_element> el(n);
    for (size_t i = 0; i < n; ++i) {
        const float* p = f + 9 * i;
        el[i] = efs_rlc_element{u[3 * i], u[3 * i + 1], u[3 * i + 2], p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8]};
    }
    Check(env, e, efs_configure_rlc(e, (uint32_t)n, el.data()), "configureRLC");
    return Undefined(env);
}

// configurePBC(h, axes: Uint32Array, phases: Float64Array)   (:1976-2155, {axes: [{axis, phase}]})
napi_value ConfigurePBC(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 3)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* ax; const double* ph; size_t na, np;
    if (!U32(env, a.argv[1], &ax, &na, "axes") || !F64(env, a.argv[2], &ph, &np, "phases")) return nullptr;
    if (np != na) return Throw(env, "one phase per PBC axis");
    Check(env, e, efs_configure_pbc(e, (uint32_t)na, ax, ph), "configurePBC");
    return Undefined(env);
}

// configureSteadyState(h, probe_idx, periodSamples, threshold)   (:2170-2216)
napi_value ConfigureSteadyState(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 4)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* idx; size_t n;
    if (!U32(env, a.argv[1], &idx, &n, "probe_idx")) return nullptr;
    uint32_t period = 0;
    double thr = 1e-6;
    GetU32(env, a.argv[2], &period);
    GetF64(env, a.argv[3], &thr);
    Check(env, e, efs_configure_steady_state(e, idx, (uint32_t)n, period, (float)thr), "configureSteadyState");
    return Undefined(env);
}

// setSteadyStateRecording(h, on)
napi_value SetSteadyStateRecording(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    bool on = false;
    napi_get_value_bool(env, a.argv[1], &on);
    Check(env, e, efs_set_steady_state_recording(e, on ? 1 : 0), "steady-state recording");
    return Undefined(env);
}

// readSteadyState(h, numProbes) -> {energy1, energy2, currentSample, converged}
napi_value ReadSteadyState(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    GetU32(env, a.argv[1], &n);
    std::vector<float> e1(n), e2(n);
    uint32_t cur = 0;
    int conv = 0;
    if (!Check(env, e, efs_read_steady_state(e, e1.data(), e2.data(), &cur, &conv), "readSteadyState")) return nullptr;
    napi_value o, b;
    napi_create_object(env, &o);
    napi_set_named_property(env, o, "energy1", NewF32(env, e1.data(), n));
    napi_set_named_property(env, o, "energy2", NewF32(env, e2.data(), n));
    napi_set_named_property(env, o, "currentSample", Num(env, cur));
    napi_get_boolean(env, conv != 0, &b);
    napi_set_named_property(env, o, "converged", b);
    return o;
}

// ---- stepping ----------------------------------------------------------------
// iterate(h, n)   (:2407-2504): enqueues n timesteps
napi_value Iterate(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    if (!GetU32(env, a.argv[1], &n)) return Throw(env, "numSteps must be a non-negative integer");
    Check(env, e, efs_iterate(e, n), "iterate");
    return Undefined(env);
}

napi_value NumTS(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    efs_num_ts(e, &n);
    return Num(env, n);
}

// sync(h): waits for the engine's stream (device.queue.onSubmittedWorkDone in the JS class)
napi_value Sync(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    Check(env, e, efs_sync(e), "sync");
    return Undefined(env);
}

// ---- probes ---------------------------------------------------------------------
napi_value ConfigureProbeGather(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* idx; size_t n;
    if (!U32(env, a.argv[1], &idx, &n, "indices")) return nullptr;
    Check(env, e, efs_configure_probe_gather(e, idx, (uint32_t)n), "configureProbeGather");
    return Undefined(env);
}

// readProbeGather(h, count) -> Float32Array(2*count)   (:2701-2715)
napi_value ReadProbeGather(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    GetU32(env, a.argv[1], &n);
    std::vector<float> out(2 * (size_t)n);
    if (!Check(env, e, efs_read_probe_gather(e, out.data(), out.size()), "readProbeGather")) return nullptr;
    return NewF32(env, out.data(), out.size());
}

napi_value ConfigureProbeGatherBuffered(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 4)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* idx; size_t n;
    if (!U32(env, a.argv[1], &idx, &n, "indices")) return nullptr;
    uint32_t maxS = 0, interval = 1;
    GetU32(env, a.argv[2], &maxS);
    GetU32(env, a.argv[3], &interval);
    Check(env, e, efs_configure_probe_gather_buffered(e, idx, (uint32_t)n, maxS, interval), "configureProbeGatherBuffered");
    return Undefined(env);
}

// readProbeGatherBuffered(h) -> {data, numSamples, stride} | null   (:2689-2695)
napi_value ReadProbeGatherBuffered(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t ns = 0, stride = 0;
    if (!Check(env, e, efs_read_probe_gather_buffered(e, nullptr, 0, &ns, &stride), "readProbeGatherBuffered")) return nullptr;
    if (ns == 0) {
        napi_value n;
        napi_get_null(env, &n);
        return n;
    }
    std::vector<float> data((size_t)ns * stride);
    if (!Check(env, e, efs_read_probe_gather_buffered(e, data.data(), data.size(), &ns, &stride), "readProbeGatherBuffered"))
        return nullptr;
    napi_value o;
    napi_create_object(env, &o);
    napi_set_named_property(env, o, "data", NewF32(env, data.data(), data.size()));
    napi_set_named_property(env, o, "numSamples", Num(env, ns));
    napi_set_named_property(env, o, "stride", Num(env, stride));
    return o;
}

// ---- NF2FF ----------------------------------------------------------------------
// configureNF2FF(h, surfaceIndices, numPoints, omegas: Float64Array, dT, edgeLens: Float32Array
// (primal x y z then dual x y z), maxTS, windowType)   (:2729-2827)
napi_value ConfigureNF2FF(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 8)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint32_t* pts; const double* om; const float* el; size_t n1, no, ne;
    uint32_t np = 0, maxTS = 0, win = 0;
    double dT = 0;
    if (!U32(env, a.argv[1], &pts, &n1, "surfaceIndices") || !F64(env, a.argv[3], &om, &no, "omegas") ||
        !F32(env, a.argv[5], &el, &ne, "edge lengths"))
        return nullptr;
    GetU32(env, a.argv[2], &np);
    GetF64(env, a.argv[4], &dT);
    GetU32(env, a.argv[6], &maxTS);
    GetU32(env, a.argv[7], &win);
    if (n1 < 3 * (size_t)np) return Throw(env, "surfaceIndices must hold 3 values per point");
    Check(env, e, efs_configure_nf2ff(e, pts, np, om, (uint32_t)no, dT, el, maxTS, win), "configureNF2FFAccumulation");
    return Undefined(env);
}

// readNF2FF(h, count) -> {accumE, accumH}, count = numFreq*numPoints*6   (:2844-2855)
napi_value ReadNF2FF(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t n = 0;
    GetU32(env, a.argv[1], &n);
    std::vector<float> E(n), H(n);
    if (!Check(env, e, efs_read_nf2ff(e, E.data(), H.data(), n), "readNF2FFAccumulation")) return nullptr;
    napi_value o;
    napi_create_object(env, &o);
    napi_set_named_property(env, o, "accumE", NewF32(env, E.data(), n));
    napi_set_named_property(env, o, "accumH", NewF32(env, H.data(), n));
    return o;
}

// farField(h, freqIndex, pointMeta, theta, phi, center: Float64Array(3), frequency, radius)
// -> Float32Array(5 * nTheta * nPhi)   (:2871-2967)
napi_value FarField(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 8)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    uint32_t fi = 0;
    GetU32(env, a.argv[1], &fi);
    const float *meta, *th, *ph; const double* c; size_t nm, nt, np, nc;
    if (!F32(env, a.argv[2], &meta, &nm, "pointMeta") || !F32(env, a.argv[3], &th, &nt, "theta") ||
        !F32(env, a.argv[4], &ph, &np, "phi") || !F64(env, a.argv[5], &c, &nc, "center"))
        return nullptr;
    if (nc != 3) return Throw(env, "center must hold 3 values");
    double f = 0, r = 1;
    GetF64(env, a.argv[6], &f);
    GetF64(env, a.argv[7], &r);
    std::vector<float> out(5 * nt * np);
    if (!Check(env, e, efs_far_field(e, fi, meta, th, (uint32_t)nt, ph, (uint32_t)np, c, f, r, out.data()), "computeNF2FFfarField"))
        return nullptr;
    return NewF32(env, out.data(), out.size());
}

// ---- energy -----------------------------------------------------------------------
// energy(h, lagged) -> number   (computeEnergy :2974-3021 with lagged = true)
napi_value Energy(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    bool lagged = true;
    napi_get_value_bool(env, a.argv[1], &lagged);
    double v = 0;
    if (!Check(env, e, efs_energy(e, lagged ? 1 : 0, &v), "computeEnergy")) return nullptr;
    return Num(env, v);
}

napi_value FlushEnergy(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    double v = 0;
    if (!Check(env, e, efs_flush_energy(e, &v), "flushEnergy")) return nullptr;
    return Num(env, v);
}

napi_value EnergyNoAlloc(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    double v = 0;
    if (!Check(env, e, efs_energy_noalloc(e, &v), "energyNoAlloc")) return nullptr;
    return Num(env, v);
}

// ---- state ------------------------------------------------------------------------
// getFields(h, 3N) -> {volt, curr}   (:2533-2561)
napi_value GetFields(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    double n3 = 0;
    GetF64(env, a.argv[1], &n3);
    std::vector<float> v((size_t)n3), c((size_t)n3);
    if (!Check(env, e, efs_get_fields(e, v.data(), c.data()), "getFields")) return nullptr;
    napi_value o;
    napi_create_object(env, &o);
    napi_set_named_property(env, o, "volt", NewF32(env, v.data(), v.size()));
    napi_set_named_property(env, o, "curr", NewF32(env, c.data(), c.size()));
    return o;
}

// setFields(h, volt, curr)   (uploadFields :2568-2571)
napi_value SetFields(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 3)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const float *v, *c; size_t nv, nc;
    if (!F32(env, a.argv[1], &v, &nv, "volt") || !F32(env, a.argv[2], &c, &nc, "curr")) return nullptr;
    if (nv != nc) return Throw(env, "volt and curr must have equal lengths");
    Check(env, e, efs_set_fields(e, v, c), "uploadFields");
    return Undefined(env);
}

// getState(h) -> Uint8Array; setState(h, Uint8Array)   (no reference counterpart)
napi_value GetState(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    size_t size = 0;
    if (!Check(env, e, efs_get_state(e, nullptr, 0, &size), "getState")) return nullptr;
    napi_value ab, arr;
    void* p = nullptr;
    NAPI_OK(napi_create_arraybuffer(env, size, &p, &ab));
    if (!Check(env, e, efs_get_state(e, p, size, &size), "getState")) return nullptr;
    napi_create_typedarray(env, napi_uint8_array, size, ab, 0, &arr);
    return arr;
}
napi_value SetState(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 2)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    const uint8_t* p; size_t n;
    if (!U8(env, a.argv[1], &p, &n, "state")) return nullptr;
    Check(env, e, efs_set_state(e, p, n), "setState");
    return Undefined(env);
}

napi_value DeviceBytes(napi_env env, napi_callback_info info) {
    Args a;
    if (!GetArgs(env, info, a, 1)) return nullptr;
    efs_engine* e = GetEngine(env, a.argv[0]);
    if (!e) return nullptr;
    size_t b = 0;
    efs_device_bytes(e, &b);
    return Num(env, (double)b);
}

// ---- module -----------------------------------------------------------------------
napi_value ModuleInit(napi_env env, napi_value exports) {
    const napi_property_descriptor d[] = {
        {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"destroy", nullptr, Destroy, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"init", nullptr, Init, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"initIndexed", nullptr, InitIndexed, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureExcitation", nullptr, ConfigureExcitation, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configurePML", nullptr, ConfigurePML, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureMur", nullptr, ConfigureMur, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureTFSF", nullptr, ConfigureTFSF, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureADE", nullptr, ConfigureADE, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureRLC", nullptr, ConfigureRLC, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configurePBC", nullptr, ConfigurePBC, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureSteadyState", nullptr, ConfigureSteadyState, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"setSteadyStateRecording", nullptr, SetSteadyStateRecording, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"readSteadyState", nullptr, ReadSteadyState, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"iterate", nullptr, Iterate, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"numTS", nullptr, NumTS, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"sync", nullptr, Sync, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureProbeGather", nullptr, ConfigureProbeGather, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"readProbeGather", nullptr, ReadProbeGather, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureProbeGatherBuffered", nullptr, ConfigureProbeGatherBuffered, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"readProbeGatherBuffered", nullptr, ReadProbeGatherBuffered, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"configureNF2FF", nullptr, ConfigureNF2FF, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"readNF2FF", nullptr, ReadNF2FF, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"farField", nullptr, FarField, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"energy", nullptr, Energy, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"flushEnergy", nullptr, FlushEnergy, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"energyNoAlloc", nullptr, EnergyNoAlloc, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"getFields", nullptr, GetFields, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"setFields", nullptr, SetFields, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"getState", nullptr, GetState, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"setState", nullptr, SetState, nullptr, nullptr, nullptr, napi_default, nullptr},
        {"deviceBytes", nullptr, DeviceBytes, nullptr, nullptr, nullptr, napi_default, nullptr},
    };
    napi_define_properties(env, exports, sizeof(d) / sizeof(d[0]), d);
    return exports;
}

}  // namespace

NAPI_MODULE(NODE_GYP_MODULE_NAME, ModuleInit)
