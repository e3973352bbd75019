"""Host-side mirror of the reference's `WebGPUEngine` (src/webgpu-engine.mjs:994-3498).

`CudaEngine` keeps the JavaScript class's method names, argument objects and
error behaviour (an exception on misuse, `initGPU()` returning False when no
device exists) so that a caller written against the reference's engine can
drive the B200 engine unchanged.  Every call goes through the C ABI of
libefs.so (include/efs.h); there is no CPU path.

Inputs that the reference takes as typed arrays are accepted as anything
numpy can convert; they are copied at configure time (the caller keeps its
arrays, as with `_createAndUploadBuffer` :3231-3247).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import EfsError

# Phases of a timestep as efs_time_phases / efs_batch_time_phases report them (EFS_PHASES)
PHASES = ("upml_e", "pre_point_ops", "core", "e_point_ops", "upml_h_deferred_h", "h_point_ops", "outputs")

__all__ = ["CudaEngine", "EfsError"]


def _u32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32).ravel())


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _p(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class CudaEngine:
    """Drop-in for WebGPUEngine.  See include/efs.h for the per-method contract."""

    def __init__(self, device=0):
        self._lib = _lib.load()
        self._device = device
        self._h = None
        self.numLines = None
        self.totalCells = 0
        self._keep = []
        self._nf2ff = None
        self._ring = None
        self._gather_n = 0
        self._ss_n = 0
        self.ssRecording = False

    # --- plumbing -------------------------------------------------------
    def _ck(self, rc):
        if rc != 0:
            msg = self._lib.efs_last_error(self._h).decode()
            raise EfsError(rc, msg)

    def _need_device(self):
        if self._h is None:
            raise RuntimeError("CUDA device not initialized. Call initGPU() first.")

    @property
    def handle(self):
        return self._h

    @property
    def numTS(self):
        if self._h is None:
            return 0
        v = C.c_uint32()
        self._ck(self._lib.efs_num_ts(self._h, C.byref(v)))
        return v.value

    @property
    def stream(self):
        """The engine's cudaStream_t as an integer (for event timing)."""
        s = C.c_void_p()
        self._ck(self._lib.efs_get_stream(self._h, C.byref(s)))
        return s.value or 0

    # --- lifetime -------------------------------------------------------
    def initGPU(self):
        """webgpu-engine.mjs:1107 — False when no CUDA device is usable."""
        h = C.c_void_p()
        rc = self._lib.efs_create(C.byref(h), int(self._device))
        if rc != 0:
            return False
        self._h = h
        return True

    def init(self, gridSize, coefficients):
        """webgpu-engine.mjs:1143 — coefficients {vv,vi,ii,iv} of 3*Nx*Ny*Nz floats,
        or {mat, table} (material index per cell + 12-float rows)."""
        self._need_device()
        dims = _u32(gridSize)
        if dims.size != 3:
            raise ValueError("gridSize must be [Nx, Ny, Nz]")
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        if "mat" in coefficients:
            mat = _u32(coefficients["mat"])
            table = _f32(coefficients["table"]).reshape(-1)
            if mat.size != n or table.size % 12:
                raise ValueError("mat must have Nx*Ny*Nz entries and table rows of 12 floats")
            self._ck(self._lib.efs_init_indexed(self._h, _p(dims, C.c_uint32), _p(mat, C.c_uint32),
                                                _p(table, C.c_float), table.size // 12))
        else:
            arrs = []
            for name in ("vv", "vi", "ii", "iv"):
                if name not in coefficients:
                    raise ValueError("Missing coefficient array: %s" % name)
                a = _f32(coefficients[name])
                if a.size != 3 * n:
                    raise ValueError("Coefficient %s size mismatch: expected %d, got %d" % (name, 3 * n, a.size))
                arrs.append(a)
            self._ck(self._lib.efs_init(self._h, _p(dims, C.c_uint32), *[_p(a, C.c_float) for a in arrs]))
        self.numLines = [int(d) for d in dims]
        self.totalCells = n
        self._nf2ff = None
        self._ring = None

    def destroy(self):
        if self._h is not None:
            self._lib.efs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # --- configure* ---------------------------------------------------
    def configureExcitation(self, excitation):
        """webgpu-engine.mjs:1199 — {signal, delay, amp, dir, pos, period}."""
        self._need_device()
        sig = _f32(excitation["signal"])
        amp = _f32(excitation["amp"])
        d = _u32(excitation["delay"])
        di = _u32(excitation["dir"])
        pos = _u32(excitation["pos"])
        per = int(excitation.get("period", 0) or 0)
        self._ck(self._lib.efs_configure_excitation(self._h, _p(sig, C.c_float), sig.size, _p(d, C.c_uint32),
                                                    _p(amp, C.c_float), _p(di, C.c_uint32), _p(pos, C.c_uint32),
                                                    amp.size, per))

    def configurePML(self, pmlRegions):
        """webgpu-engine.mjs:1235 — list of {startPos, numLines, vv, vvfo, vvfn, ii, iifo, iifn}."""
        self._need_device()
        regs = (_lib.PmlRegion * max(1, len(pmlRegions)))()
        keep = []
        for i, r in enumerate(pmlRegions):
            for field in ("startPos", "numLines", "vv", "vvfo", "vvfn", "ii", "iifo", "iifn"):
                if r.get(field) is None:
                    raise ValueError("PML region %d missing field: %s" % (i, field))
            nl = [int(v) for v in r["numLines"]]
            tot = 3 * nl[0] * nl[1] * nl[2]
            regs[i].start[:] = [int(v) for v in r["startPos"]]
            regs[i].num[:] = nl
            for name in ("vv", "vvfo", "vvfn", "ii", "iifo", "iifn"):
                a = _f32(r[name])
                if a.size != tot:
                    raise ValueError("PML region %d: %s size mismatch: expected %d, got %d" % (i, name, tot, a.size))
                keep.append(a)
                setattr(regs[i], name, _p(a, C.c_float))
        self._ck(self._lib.efs_configure_pml(self._h, len(pmlRegions), regs))

    def configureMur(self, config):
        """webgpu-engine.mjs:1822 — single {coeff, normal_idx, shifted_idx} or dual nyP/nyPP form."""
        self._need_device()
        if config.get("coeff_nyP") is not None:
            coeff = np.concatenate([_f32(config["coeff_nyP"]), _f32(config["coeff_nyPP"])])
            normal = np.concatenate([_u32(config["normal_idx_nyP"]), _u32(config["normal_idx_nyPP"])])
            shifted = np.concatenate([_u32(config["shifted_idx_nyP"]), _u32(config["shifted_idx_nyPP"])])
        else:
            normal = _u32(config["normal_idx"])
            shifted = _u32(config["shifted_idx"])
            c = config["coeff"]
            coeff = np.full(normal.size, c, np.float32) if np.isscalar(c) else _f32(c)
        coeff, normal, shifted = _f32(coeff), _u32(normal), _u32(shifted)
        self._ck(self._lib.efs_configure_mur(self._h, _p(coeff, C.c_float), _p(normal, C.c_uint32),
                                            _p(shifted, C.c_uint32), normal.size))

    @staticmethod
    def _tfsf_points(pts):
        """List of {field_idx, delay_int, delay_frac, amp} objects (the
        reference's form) or one dict of equal-length columns."""
        if isinstance(pts, dict):
            cols = [np.asarray(pts[k]) for k in ("field_idx", "delay_int", "delay_frac", "amp")]
        else:
            cols = [np.asarray([p[k] for p in pts]) for k in ("field_idx", "delay_int", "delay_frac", "amp")]
        n = len(cols[0])
        rec = np.zeros(max(1, n), dtype=[("field_idx", "<u4"), ("delay_int", "<u4"), ("delay_frac", "<f4"), ("amp", "<f4")])
        for name, c in zip(("field_idx", "delay_int", "delay_frac", "amp"), cols):
            rec[name][:n] = c
        return rec, n

    def configureTFSF(self, config):
        """webgpu-engine.mjs:1527 — {signal, period, voltagePoints, currentPoints}."""
        self._need_device()
        sig = _f32(config["signal"])
        (vp, nv), (cp, nc) = (self._tfsf_points(config.get("voltagePoints") or []),
                              self._tfsf_points(config.get("currentPoints") or []))
        tp = C.POINTER(_lib.TfsfPoint)
        self._ck(self._lib.efs_configure_tfsf(self._h, _p(sig, C.c_float), sig.size, int(config.get("period", 0) or 0),
                                             vp.ctypes.data_as(tp), nv, cp.ctypes.data_as(tp), nc))

    def configureLorentzADE(self, config):
        """webgpu-engine.mjs:1358 — {orders: [{numCells, hasLorentz, directions: [...]}], apply}.
        `apply` (default False) turns on the apply step the reference lacks
        (efs_configure_ade_apply): the state is subtracted from E / H."""
        self._need_device()
        orders = config["orders"]
        oarr = (_lib.AdeOrder * max(1, len(orders)))()
        keep = []
        for i, o in enumerate(orders):
            dirs = o["directions"]
            darr = (_lib.AdeDirection * max(1, len(dirs)))()
            for j, d in enumerate(dirs):
                darr[j].dir = int(d["dir"])
                pos = _u32(d["pos_idx"])
                keep.append(pos)
                darr[j].pos_idx = _p(pos, C.c_uint32)
                for name, key in (("v_int", "v_int_ADE"), ("v_ext", "v_ext_ADE"), ("v_lor", "v_Lor_ADE"),
                                  ("i_int", "i_int_ADE"), ("i_ext", "i_ext_ADE"), ("i_lor", "i_Lor_ADE")):
                    if d.get(key) is not None:
                        a = _f32(d[key])
                        keep.append(a)
                        setattr(darr[j], name, _p(a, C.c_float))
            keep.append(darr)
            oarr[i].num_cells = int(o["numCells"])
            oarr[i].has_lorentz = 1 if o.get("hasLorentz") else 0
            oarr[i].num_directions = len(dirs)
            oarr[i].directions = darr
        self._ck(self._lib.efs_configure_ade(self._h, len(orders), oarr))
        # opt-in apply step (no reference counterpart): subtract the state from the fields
        self._ck(self._lib.efs_configure_ade_apply(self._h, 1 if config.get("apply") else 0))

    configureLorentz = configureLorentzADE   # name used by WebGPUFDTD / CPUFDTDEngine

    def configureRLC(self, config):
        """webgpu-engine.mjs:1722 — {elements: [{field_idx, direction, type_flag, i2v, ...}]}."""
        self._need_device()
        els = config["elements"]
        if len(els) == 0:
            return
        arr = (_lib.RlcElement * len(els))()
        for i, e in enumerate(els):
            arr[i].field_idx = int(e["field_idx"])
            arr[i].direction = int(e["direction"])
            arr[i].type_flag = int(e["type_flag"])
            for k in ("i2v", "ilv", "vvd", "vv2", "vj1", "vj2", "ib0", "b1", "b2"):
                setattr(arr[i], k, float(e.get(k, 0.0)))
        self._ck(self._lib.efs_configure_rlc(self._h, len(els), arr))

    def configurePBC(self, config):
        """webgpu-engine.mjs:1976 — {axes: [{axis, phase}]}."""
        self._need_device()
        axes = config.get("axes") or []
        if not axes:
            return
        ax = _u32([a["axis"] for a in axes])
        ph = _f64([a.get("phase", 0.0) or 0.0 for a in axes])
        self._ck(self._lib.efs_configure_pbc(self._h, ax.size, _p(ax, C.c_uint32), _p(ph, C.c_double)))

    def configureSteadyState(self, config):
        """webgpu-engine.mjs:2170 — {probe_idx, periodSamples, threshold}."""
        self._need_device()
        idx = _u32(config["probe_idx"])
        self._ck(self._lib.efs_configure_steady_state(self._h, _p(idx, C.c_uint32), idx.size,
                                                     int(config["periodSamples"]), float(config.get("threshold") or 1e-6)))
        self._ss_n = idx.size
        self.ssRecording = False

    def setSteadyStateRecording(self, recording):
        self._ck(self._lib.efs_set_steady_state_recording(self._h, 1 if recording else 0))
        self.ssRecording = bool(recording)

    def readSteadyState(self):
        e1 = np.zeros(self._ss_n, np.float32)
        e2 = np.zeros(self._ss_n, np.float32)
        cur = C.c_uint32()
        conv = C.c_int()
        self._ck(self._lib.efs_read_steady_state(self._h, _p(e1, C.c_float), _p(e2, C.c_float), C.byref(cur), C.byref(conv)))
        return {"energy_period1": e1, "energy_period2": e2, "currentSample": cur.value, "converged": bool(conv.value)}

    # --- stepping -------------------------------------------------------
    def iterate(self, numSteps):
        """webgpu-engine.mjs:2407 — queue numSteps timesteps (no wait)."""
        self._need_device()
        self._ck(self._lib.efs_iterate(self._h, int(numSteps)))

    def sync(self):
        self._ck(self._lib.efs_sync(self._h))

    # --- probes -------------------------------------------------------
    def configureProbeGather(self, indices):
        idx = _u32(indices)
        if idx.size == 0:
            return
        self._ck(self._lib.efs_configure_probe_gather(self._h, _p(idx, C.c_uint32), idx.size))
        self._gather_n = idx.size

    def readProbeGather(self):
        if not self._gather_n:
            return None
        out = np.zeros(2 * self._gather_n, np.float32)
        self._ck(self._lib.efs_read_probe_gather(self._h, _p(out, C.c_float), out.size))
        return out

    def configureProbeGatherBuffered(self, indices, maxSamples, sampleInterval):
        idx = _u32(indices)
        if idx.size == 0:
            return
        self._ck(self._lib.efs_configure_probe_gather_buffered(self._h, _p(idx, C.c_uint32), idx.size,
                                                               int(maxSamples), int(sampleInterval)))
        self._ring = idx.size

    def readProbeGatherBuffered(self):
        """webgpu-engine.mjs:2689 — {data, numSamples, stride} or None before the first sample."""
        if not self._ring:
            return None
        ns, st = C.c_uint32(), C.c_uint32()
        self._ck(self._lib.efs_read_probe_gather_buffered(self._h, None, 0, C.byref(ns), C.byref(st)))
        if ns.value == 0:
            return None
        out = np.zeros(ns.value * st.value, np.float32)
        self._ck(self._lib.efs_read_probe_gather_buffered(self._h, _p(out, C.c_float), out.size, C.byref(ns), C.byref(st)))
        return {"data": out, "numSamples": ns.value, "stride": st.value}

    def readProbe(self, positions):
        """webgpu-engine.mjs:2512 — [{component, x, y, z}] -> interleaved volt/curr."""
        f = self.getFields()
        Nx, Ny, Nz = self.numLines
        out = np.zeros(2 * len(positions), np.float32)
        for i, p in enumerate(positions):
            li = p["component"] * Nx * Ny * Nz + p["x"] * Ny * Nz + p["y"] * Nz + p["z"]
            out[2 * i] = f["volt"][li]
            out[2 * i + 1] = f["curr"][li]
        return out

    # --- NF2FF ---------------------------------------------------------
    def configureNF2FFAccumulation(self, config):
        """webgpu-engine.mjs:2729 — {surfaceIndices, numPoints, omega | omegas, dT, gridSize,
        primalEdgeLens, dualEdgeLens, maxTS, windowType}."""
        npts = int(config["numPoints"])
        if npts == 0:
            return
        pts = _u32(config["surfaceIndices"])
        om = config.get("omegas")
        om = _f64([config["omega"]] if om is None else om)
        el = np.concatenate([_f32(a) for a in list(config["primalEdgeLens"]) + list(config["dualEdgeLens"])])
        self._ck(self._lib.efs_configure_nf2ff(self._h, _p(pts, C.c_uint32), npts, _p(om, C.c_double), om.size,
                                              float(config["dT"]), _p(el, C.c_float), int(config.get("maxTS", 0) or 0),
                                              int(config.get("windowType", 0) or 0)))
        self._nf2ff = (npts, om.size)

    def readNF2FFAccumulation(self, allFrequencies=False):
        """webgpu-engine.mjs:2844 — {accumE, accumH}; frequency 0 unless allFrequencies."""
        if self._nf2ff is None:
            return None
        npts, nf = self._nf2ff
        e = np.empty(nf * npts * 6, np.float32)       # filled whole by the call
        h = np.empty(nf * npts * 6, np.float32)
        self._ck(self._lib.efs_read_nf2ff(self._h, _p(e, C.c_float), _p(h, C.c_float), e.size))
        if allFrequencies:
            return {"accumE": e.reshape(nf, npts * 6), "accumH": h.reshape(nf, npts * 6)}
        return {"accumE": e[:npts * 6].copy(), "accumH": h[:npts * 6].copy()}

    def farFieldTime(self):
        """Device ms of the last far-field call: [point records, angle sums]."""
        ms = np.zeros(2, np.float32)
        self._ck(self._lib.efs_far_field_time(self._h, _p(ms, C.c_float)))
        return [float(ms[0]), float(ms[1])]

    def computeNF2FFfarField(self, config):
        """webgpu-engine.mjs:2871 — {pointMeta, theta, phi, center, frequency, radius, numPoints[, freqIndex]}
        -> 5 floats per angle (P_rad, Et_re, Et_im, Ep_re, Ep_im)."""
        meta = _f32(config["pointMeta"])
        th = _f32(config["theta"])
        ph = _f32(config["phi"])
        cen = _f64(config.get("center", [0, 0, 0]))
        out = np.zeros(5 * th.size * ph.size, np.float32)
        self._ck(self._lib.efs_far_field(self._h, int(config.get("freqIndex", 0)), _p(meta, C.c_float),
                                        _p(th, C.c_float), th.size, _p(ph, C.c_float), ph.size, _p(cen, C.c_double),
                                        float(config["frequency"]), float(config["radius"]), _p(out, C.c_float)))
        return out

    # --- energy --------------------------------------------------------
    def computeEnergy(self, lagged=True):
        """webgpu-engine.mjs:2974 — lagged by one call like the reference (0 first)."""
        v = C.c_double()
        self._ck(self._lib.efs_energy(self._h, 1 if lagged else 0, C.byref(v)))
        return v.value

    def flushEnergy(self):
        v = C.c_double()
        self._ck(self._lib.efs_flush_energy(self._h, C.byref(v)))
        return v.value

    def energyNoAlloc(self):
        """Current energy (as computeEnergy(lagged=False)) with no device
        allocation: for callers that keep the library from allocating once
        they run (efs_energy_noalloc)."""
        v = C.c_double()
        self._ck(self._lib.efs_energy_noalloc(self._h, C.byref(v)))
        return v.value

    # --- state --------------------------------------------------------
    def getPlanes(self, x, count, out=None):
        """x-planes [x, x+count) of E and H as (3, count, Ny*Nz) float32 arrays
        (efs_get_planes).  `out` may be a pair of torch CUDA tensors of that
        shape: the planes are then copied device to device."""
        Ny, Nz = self.numLines[1], self.numLines[2]
        if out is not None:
            self._ck(self._lib.efs_get_planes(self._h, int(x), int(count), C.c_void_p(out[0].data_ptr()),
                                              C.c_void_p(out[1].data_ptr())))
            return out
        v = np.empty((3, count, Ny * Nz), np.float32)
        c = np.empty((3, count, Ny * Nz), np.float32)
        self._ck(self._lib.efs_get_planes(self._h, int(x), int(count), v.ctypes.data_as(C.c_void_p),
                                          c.ctypes.data_as(C.c_void_p)))
        return v, c

    def setPlanes(self, x, volt, curr):
        """Overwrite x-planes [x, x+count) of E and H (efs_set_planes); numpy
        arrays or torch CUDA tensors of shape (3, count, Ny*Nz)."""
        count = volt.shape[1]
        if hasattr(volt, "data_ptr"):
            self._ck(self._lib.efs_set_planes(self._h, int(x), int(count), C.c_void_p(volt.data_ptr()),
                                              C.c_void_p(curr.data_ptr())))
            return
        v = np.ascontiguousarray(volt, np.float32)
        c = np.ascontiguousarray(curr, np.float32)
        self._ck(self._lib.efs_set_planes(self._h, int(x), int(count), v.ctypes.data_as(C.c_void_p),
                                          c.ctypes.data_as(C.c_void_p)))

    def getFields(self):
        n = 3 * self.totalCells
        v = np.zeros(n, np.float32)
        c = np.zeros(n, np.float32)
        self._ck(self._lib.efs_get_fields(self._h, _p(v, C.c_float), _p(c, C.c_float)))
        return {"volt": v, "curr": c}

    def uploadFields(self, volt, curr):
        v = _f32(volt)
        c = _f32(curr)
        if v.size != 3 * self.totalCells or c.size != 3 * self.totalCells:
            raise ValueError("field arrays must hold 3*Nx*Ny*Nz floats")
        self._ck(self._lib.efs_set_fields(self._h, _p(v, C.c_float), _p(c, C.c_float)))

    def getState(self):
        sz = C.c_size_t()
        self._ck(self._lib.efs_get_state(self._h, None, 0, C.byref(sz)))
        buf = np.zeros(sz.value, np.uint8)
        self._ck(self._lib.efs_get_state(self._h, buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(sz)))
        return buf

    def setState(self, blob):
        b = np.ascontiguousarray(np.asarray(blob, dtype=np.uint8))
        self._ck(self._lib.efs_set_state(self._h, b.ctypes.data_as(C.c_void_p), b.size))

    def deviceBytes(self):
        v = C.c_size_t()
        self._ck(self._lib.efs_device_bytes(self._h, C.byref(v)))
        return v.value

    def debugSetWait(self, wait_ns=1_000_000_000, skip_plane=None):
        """Diagnostics (efs_debug_set_wait): limit of the fused kernel's bounded
        waits, and an x-plane whose loads are never issued (None: none)."""
        self._ck(self._lib.efs_debug_set_wait(self._h, int(wait_ns), 0xFFFFFFFF if skip_plane is None else int(skip_plane)))

    def timePhases(self, steps=16):
        """Diagnostics (efs_time_phases): device ms per timestep of each phase
        of the step over `steps` (<= 64) timesteps launched kernel by kernel
        (advances the engine as iterate does)."""
        ms = (C.c_float * len(PHASES))()
        self._ck(self._lib.efs_time_phases(self._h, int(steps), ms))
        return dict(zip(PHASES, (round(v, 4) for v in ms)))

    def setPlaneDepth(self, xchunk):
        """Tuning (efs_set_plane_depth): x-planes per CTA of the fused kernel
        (default 32); results are bit-identical under every depth."""
        self._ck(self._lib.efs_set_plane_depth(self._h, int(xchunk)))

    def timeCore(self, reps=10):
        """Mean device ms per launch of [the fused kernel, the UPML passes] (advances the fields)."""
        ms = np.zeros(2, np.float32)
        self._ck(self._lib.efs_time_core(self._h, int(reps), _p(ms, C.c_float)))
        return [float(ms[0]), float(ms[1])]

    def kernelsPerStep(self):
        """Kernel launches one timestep enqueues with the current configuration."""
        v = C.c_uint32()
        self._ck(self._lib.efs_kernels_per_step(self._h, C.byref(v)))
        return v.value

    def debugRead(self, name, arg=0):
        cnt = C.c_size_t()
        self._ck(self._lib.efs_debug_read(self._h, name.encode(), int(arg), None, 0, C.byref(cnt)))
        out = np.zeros(cnt.value, np.float32)
        self._ck(self._lib.efs_debug_read(self._h, name.encode(), int(arg), _p(out, C.c_float), out.size, C.byref(cnt)))
        return out


class CudaBatch:
    """Batched form (efs_batch_*): several configured CudaEngine objects of one
    device advanced together by one persistent fused-update launch and one
    launch per sparse phase.  Members keep their own step counters and stay
    usable through their own methods between batch calls."""

    def __init__(self, engines):
        self._lib = _lib.load()
        self.members = list(engines)
        arr = (C.c_void_p * len(self.members))(*[e.handle for e in self.members])
        h = C.c_void_p()
        rc = self._lib.efs_batch_create(C.byref(h), arr, len(self.members))
        if rc != 0:
            raise EfsError(rc, self._lib.efs_batch_last_error(None).decode())
        self._h = h

    def _ck(self, rc):
        if rc != 0:
            raise EfsError(rc, self._lib.efs_batch_last_error(self._h).decode())

    def iterate(self, n):
        self._ck(self._lib.efs_batch_iterate(self._h, int(n)))

    def sync(self):
        self._ck(self._lib.efs_batch_sync(self._h))

    def setShape(self, xchunk, ctas_per_sm=2):
        self._ck(self._lib.efs_batch_set_shape(self._h, int(xchunk), int(ctas_per_sm)))

    def timePhases(self, steps=16):
        """Diagnostics (efs_batch_time_phases): device ms per timestep of each
        phase of a batched step (advances the members by `steps`)."""
        ms = (C.c_float * len(PHASES))()
        self._ck(self._lib.efs_batch_time_phases(self._h, int(steps), ms))
        return dict(zip(PHASES, (round(v, 4) for v in ms)))

    def autotune(self, steps=16):
        """Pick plane depth and CTAs per SM by timing real steps (advances the
        members by 17*steps timesteps; results are the same under every shape)."""
        x, c, ms = C.c_uint32(), C.c_uint32(), C.c_float()
        self._ck(self._lib.efs_batch_autotune(self._h, int(steps), C.byref(x), C.byref(c), C.byref(ms)))
        return {"xchunk": x.value, "ctas_per_sm": c.value, "ms_per_step": ms.value}

    def destroy(self):
        if self._h is not None:
            self._lib.efs_batch_destroy(self._h)
            self._h = None
