"""ctypes wrapper of the CPU oracle (oracle/efs_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, never by the product package efs_b200.

`OracleEngine` keeps the method names of the reference's `CPUFDTDEngine`
(src/webgpu-fdtd.mjs:13-1202) so the ported known-answer tests read like the
reference's own tests/test_webgpu.mjs.  Configuration dicts follow the
reference's configure* argument objects; they are normalised here
independently of efs_b200 so a marshalling bug cannot hide on both sides.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libefs_oracle.so")

MODES = {"f32": 0, "js": 1, "f64": 2}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        vp, u32, u32p, f32p, f64p = C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(C.c_double)
        sig = {
            "or_create": (vp, [C.c_int, u32p, f32p, f32p, f32p, f32p]),
            "or_create_indexed": (vp, [C.c_int, u32p, u32p, f32p, u32]),
            "or_destroy": (None, [vp]),
            "or_set_threads": (C.c_int, [C.c_int]),
            "or_num_ts": (u32, [vp]),
            "or_set_num_ts": (None, [vp, u32]),
            "or_configure_excitation": (None, [vp, f32p, u32, u32p, f32p, u32p, u32p, u32, u32]),
            "or_configure_pml": (None, [vp, u32, u32p, u32p, C.POINTER(f32p)]),
            "or_configure_mur": (None, [vp, f32p, u32p, u32p, u32]),
            "or_configure_tfsf": (None, [vp, f32p, u32, u32, u32p, u32p, f32p, f32p, u32, u32p, u32p, f32p, f32p, u32]),
            "or_add_ade": (None, [vp, u32, u32, C.c_int, u32, u32p, f32p, f32p, f32p, f32p, f32p, f32p]),
            "or_set_ade_apply": (None, [vp, C.c_int]),
            "or_configure_rlc": (None, [vp, u32, u32p, u32p, u32p, f32p]),
            "or_configure_steady_state": (None, [vp, u32p, u32, u32, C.c_float]),
            "or_set_steady_state": (None, [vp, C.c_int, u32]),
            "or_steady_state_sample": (u32, [vp]),
            "or_check_convergence": (C.c_int, [vp]),
            "or_configure_pbc": (None, [vp, u32, u32p, f64p]),
            "or_configure_gather": (None, [vp, u32p, u32, u32, u32]),
            "or_gather_samples": (u32, [vp]),
            "or_configure_nf2ff": (None, [vp, u32p, u32, f64p, u32, C.c_double, f32p, u32, u32, C.c_int]),
            "or_step": (None, [vp]),
            "or_iterate": (None, [vp, u32]),
            "or_phase": (C.c_int, [vp, C.c_char_p]),
            "or_read": (C.c_int64, [vp, C.c_char_p, C.c_int, C.c_int, f64p, C.c_int64]),
            "or_write": (C.c_int64, [vp, C.c_char_p, C.c_int, C.c_int, f64p, C.c_int64]),
            "or_energy": (C.c_double, [vp]),
            "or_far_field": (None, [f32p, f32p, f32p, u32, f32p, u32, f32p, u32, C.c_double, C.c_double, f64p, f64p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def set_threads(n):
    return load().or_set_threads(int(n))


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).ravel())


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class OracleEngine:
    """CPU restatement of CPUFDTDEngine; mode 'f32' | 'js' | 'f64'."""

    def __init__(self, numLines=None, coefficients=None, mode="f32"):
        self._lib = load()
        self.mode = mode
        self._h = None
        self._en_prev = None
        self._en_last = 0.0
        if numLines is not None:
            self.init(numLines, coefficients)

    def init(self, numLines, coefficients):
        """Create (or recreate) the engine state; WebGPUEngine.init semantics."""
        if self._h:
            self._lib.or_destroy(self._h)
            self._h = None
        mode = self.mode
        self._en_prev = None
        self._en_last = 0.0
        self.numLines = [int(v) for v in numLines]
        Nx, Ny, Nz = self.numLines
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.totalCells = Nx * Ny * Nz
        dims = _u32(self.numLines)
        if "mat" in coefficients:
            mat = _u32(coefficients["mat"])
            tab = _f32(coefficients["table"])
            self._h = self._lib.or_create_indexed(MODES[mode], _p(dims, C.c_uint32), _p(mat, C.c_uint32),
                                                  _p(tab, C.c_float), tab.size // 12)
        else:
            a = [_f32(coefficients[k]) for k in ("vv", "vi", "ii", "iv")]
            for x in a:
                if x.size != 3 * self.totalCells:
                    raise ValueError("coefficient size mismatch")
            self._h = self._lib.or_create(MODES[mode], _p(dims, C.c_uint32), *[_p(x, C.c_float) for x in a])
        self._nf = None

    def __del__(self):
        try:
            if self._h:
                self._lib.or_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def idx(self, n, x, y, z):
        """ArrayNIJK address (src/webgpu-fdtd.mjs:56-58)."""
        return n * self.totalCells + x * self.Ny * self.Nz + y * self.Nz + z

    # --- state ---------------------------------------------------------
    @property
    def numTS(self):
        return self._lib.or_num_ts(self._h)

    @numTS.setter
    def numTS(self, v):
        self._lib.or_set_num_ts(self._h, int(v))

    def read(self, name, a=0, b=0):
        n = self._lib.or_read(self._h, name.encode(), a, b, None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, np.float64)
        self._lib.or_read(self._h, name.encode(), a, b, _p(out, C.c_double), n)
        return out

    def write(self, name, values, a=0, b=0):
        v = _f64(values)
        if self._lib.or_write(self._h, name.encode(), a, b, _p(v, C.c_double), v.size) < 0:
            raise KeyError(name)

    def set(self, name, index, value, a=0, b=0):
        arr = self.read(name, a, b)
        arr[index] = value
        self.write(name, arr, a, b)

    @property
    def volt(self):
        return self.read("volt")

    @property
    def curr(self):
        return self.read("curr")

    def getFields(self):
        return {"volt": self.read("volt"), "curr": self.read("curr")}

    def uploadFields(self, volt, curr):
        self.write("volt", volt)
        self.write("curr", curr)

    def getPlanes(self, x, count):
        """x-planes [x, x+count) of E and H as (3, count, Ny*Nz) float32 (the
        engine's getPlanes, through whole-field reads: small grids only)."""
        nx, ny, nz = self.numLines
        v = np.asarray(self.read("volt"), np.float32).reshape(3, nx, ny * nz)[:, x:x + count].copy()
        c = np.asarray(self.read("curr"), np.float32).reshape(3, nx, ny * nz)[:, x:x + count].copy()
        return v, c

    def setPlanes(self, x, volt, curr):
        nx, ny, nz = self.numLines
        for name, a in (("volt", volt), ("curr", curr)):
            f = np.asarray(self.read(name), np.float32).reshape(3, nx, ny * nz).copy()
            f[:, x:x + a.shape[1]] = a
            self.write(name, f.reshape(-1))

    # --- configure* (reference argument objects) -------------------------
    def configureExcitation(self, exc):
        sig, amp = _f32(exc["signal"]), _f32(exc["amp"])
        d, di, pos = _u32(exc["delay"]), _u32(exc["dir"]), _u32(exc["pos"])
        self._lib.or_configure_excitation(self._h, _p(sig, C.c_float), sig.size, _p(d, C.c_uint32), _p(amp, C.c_float),
                                          _p(di, C.c_uint32), _p(pos, C.c_uint32), amp.size, int(exc.get("period", 0) or 0))

    def configurePML(self, regions):
        n = len(regions)
        st = _u32([v for r in regions for v in r["startPos"]] or [0])
        nl = _u32([v for r in regions for v in r["numLines"]] or [0])
        keep = []
        ptrs = (C.POINTER(C.c_float) * max(1, 6 * n))()
        for i, r in enumerate(regions):
            for j, k in enumerate(("vv", "vvfo", "vvfn", "ii", "iifo", "iifn")):
                a = _f32(r[k])
                keep.append(a)
                ptrs[6 * i + j] = _p(a, C.c_float)
        self._lib.or_configure_pml(self._h, n, _p(st, C.c_uint32), _p(nl, C.c_uint32), ptrs)

    def configureMur(self, cfg):
        # src/webgpu-fdtd.mjs:941-987: dual form concatenates nyP then nyPP
        if cfg.get("coeff_nyP") is not None:
            coeff = np.concatenate([_f32(cfg["coeff_nyP"]), _f32(cfg["coeff_nyPP"])])
            normal = np.concatenate([_u32(cfg["normal_idx_nyP"]), _u32(cfg["normal_idx_nyPP"])])
            shifted = np.concatenate([_u32(cfg["shifted_idx_nyP"]), _u32(cfg["shifted_idx_nyPP"])])
        else:
            normal, shifted = _u32(cfg["normal_idx"]), _u32(cfg["shifted_idx"])
            c = cfg["coeff"]
            coeff = np.full(normal.size, c, np.float32) if np.isscalar(c) else _f32(c)
        coeff, normal, shifted = _f32(coeff), _u32(normal), _u32(shifted)
        self._lib.or_configure_mur(self._h, _p(coeff, C.c_float), _p(normal, C.c_uint32), _p(shifted, C.c_uint32), normal.size)

    def configureTFSF(self, cfg):
        sig = _f32(cfg["signal"])

        def cols(pts):
            if isinstance(pts, dict):
                return (_u32(pts["field_idx"]), _u32(pts["delay_int"]), _f32(pts["delay_frac"]), _f32(pts["amp"]))
            return (_u32([p["field_idx"] for p in pts] or [0]), _u32([p["delay_int"] for p in pts] or [0]),
                    _f32([p["delay_frac"] for p in pts] or [0]), _f32([p["amp"] for p in pts] or [0]))
        vp, cp = cfg.get("voltagePoints") or [], cfg.get("currentPoints") or []
        v, c = cols(vp), cols(cp)
        vp = v[0] if isinstance(vp, dict) else vp
        cp = c[0] if isinstance(cp, dict) else cp
        self._lib.or_configure_tfsf(self._h, _p(sig, C.c_float), sig.size, int(cfg.get("period", 0) or 0),
                                    _p(v[0], C.c_uint32), _p(v[1], C.c_uint32), _p(v[2], C.c_float), _p(v[3], C.c_float), len(vp),
                                    _p(c[0], C.c_uint32), _p(c[1], C.c_uint32), _p(c[2], C.c_float), _p(c[3], C.c_float), len(cp))

    def configureLorentz(self, cfg):
        for oi, o in enumerate(cfg["orders"]):
            for d in o["directions"]:
                pos = _u32(d["pos_idx"])
                arr = [None if d.get(k) is None else _f32(d[k]) for k in
                       ("v_int_ADE", "v_ext_ADE", "v_Lor_ADE", "i_int_ADE", "i_ext_ADE", "i_Lor_ADE")]
                self._lib.or_add_ade(self._h, oi, int(o["numCells"]), 1 if o.get("hasLorentz") else 0, int(d["dir"]),
                                     _p(pos, C.c_uint32), *[_p(a, C.c_float) for a in arr])
        self._lib.or_set_ade_apply(self._h, 1 if cfg.get("apply") else 0)

    configureLorentzADE = configureLorentz

    def configureRLC(self, cfg):
        els = cfg["elements"]
        fi = _u32([e["field_idx"] for e in els] or [0])
        di = _u32([e["direction"] for e in els] or [0])
        ty = _u32([e["type_flag"] for e in els] or [0])
        pr = _f32([e.get(k, 0.0) for e in els for k in ("i2v", "ilv", "vvd", "vv2", "vj1", "vj2", "ib0", "b1", "b2")] or [0])
        self._lib.or_configure_rlc(self._h, len(els), _p(fi, C.c_uint32), _p(di, C.c_uint32), _p(ty, C.c_uint32), _p(pr, C.c_float))

    def configureSteadyState(self, cfg):
        idx = _u32(cfg["probe_idx"])
        self._lib.or_configure_steady_state(self._h, _p(idx, C.c_uint32), idx.size, int(cfg["periodSamples"]),
                                            float(cfg.get("threshold") or 1e-6))

    def setSteadyState(self, recording, currentSample=None):
        cur = self._lib.or_steady_state_sample(self._h) if currentSample is None else currentSample
        self._lib.or_set_steady_state(self._h, 1 if recording else 0, int(cur))

    def checkConvergence(self):
        return bool(self._lib.or_check_convergence(self._h))

    @property
    def steadyStateSample(self):
        return self._lib.or_steady_state_sample(self._h)

    def configurePBC(self, cfg):
        axes = cfg.get("axes") or []
        ax = _u32([a["axis"] for a in axes] or [0])
        ph = _f64([a.get("phase", 0.0) or 0.0 for a in axes] or [0])
        self._lib.or_configure_pbc(self._h, len(axes), _p(ax, C.c_uint32), _p(ph, C.c_double))

    def configureProbeGatherBuffered(self, indices, maxSamples, sampleInterval):
        idx = _u32(indices)
        self._lib.or_configure_gather(self._h, _p(idx, C.c_uint32), idx.size, int(maxSamples), int(sampleInterval))
        self._G = idx.size

    def readProbeGatherBuffered(self):
        ns = self._lib.or_gather_samples(self._h)
        if ns == 0:
            return None
        ring = self.read("gather_ring")
        return {"data": ring[:ns * self._G * 2], "numSamples": ns, "stride": self._G * 2}

    def configureNF2FFAccumulation(self, cfg, phase_mode=1):
        pts = _u32(cfg["surfaceIndices"])
        om = cfg.get("omegas")
        om = _f64([cfg["omega"]] if om is None else om)
        el = _f32(np.concatenate([_f32(a) for a in list(cfg["primalEdgeLens"]) + list(cfg["dualEdgeLens"])]))
        np_ = int(cfg["numPoints"])
        self._lib.or_configure_nf2ff(self._h, _p(pts, C.c_uint32), np_, _p(om, C.c_double), om.size, float(cfg["dT"]),
                                     _p(el, C.c_float), int(cfg.get("maxTS", 0) or 0), int(cfg.get("windowType", 0) or 0),
                                     int(phase_mode))
        self._nf = (np_, om.size)

    def readNF2FFAccumulation(self, allFrequencies=False):
        np_, nf = self._nf
        e = self.read("nf2ff_E").reshape(nf, np_ * 6)
        h = self.read("nf2ff_H").reshape(nf, np_ * 6)
        if allFrequencies:
            return {"accumE": e, "accumH": h}
        return {"accumE": e[0], "accumH": h[0]}

    # --- stepping ------------------------------------------------------
    def step(self):
        self._lib.or_step(self._h)

    def iterate(self, n):
        self._lib.or_iterate(self._h, int(n))

    def phase(self, name):
        if self._lib.or_phase(self._h, name.encode()) != 0:
            raise KeyError(name)

    def __getattr__(self, name):
        # single-phase methods with the reference's names (updateVoltages, murApply, ...)
        if name in _PHASES:
            return lambda: self.phase(name)
        raise AttributeError(name)

    def energy(self):
        return self._lib.or_energy(self._h)

    def computeEnergy(self, lagged=True):
        """WebGPUEngine.computeEnergy contract: returns the previous call's value (0 first)."""
        cur = self.energy()
        if not lagged:
            return cur
        if self._en_prev is not None:
            self._en_last = self._en_prev
        self._en_prev = cur
        return self._en_last

    def flushEnergy(self):
        if self._en_prev is not None:
            self._en_last = self._en_prev
            self._en_prev = None
        return self._en_last


_PHASES = {"updateVoltages", "updateCurrents", "applyExcitation", "preVoltageUpdatePML", "postVoltageUpdatePML",
           "preCurrentUpdatePML", "postCurrentUpdatePML", "updateVoltADE", "updateCurrADE", "applyTFSFVoltage",
           "applyTFSFCurrent", "preVoltageRLC", "applyRLC", "updateRLC", "murPreVoltage", "murPostVoltage", "murApply",
           "accumulateEnergy", "pbcVoltage", "pbcCurrent"}


def far_field(accE, accH, meta, theta, phi, frequency, radius=1.0, center=(0.0, 0.0, 0.0)):
    """f64 far field of one frequency block -> array (n_angles, 5)."""
    lib = load()
    aE, aH, m = _f32(accE), _f32(accH), _f32(meta)
    th, ph = _f32(theta), _f32(phi)
    cen = _f64(center)
    out = np.zeros(5 * th.size * ph.size, np.float64)
    lib.or_far_field(_p(aE, C.c_float), _p(aH, C.c_float), _p(m, C.c_float), m.size // 8, _p(th, C.c_float), th.size,
                     _p(ph, C.c_float), ph.size, float(frequency), float(radius), _p(cen, C.c_double), _p(out, C.c_double))
    return out.reshape(-1, 5)
