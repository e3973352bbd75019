// cuda-engine.mjs — a drop-in for the reference's WebGPUEngine
// (src/webgpu-engine.mjs:994-3498) on libefs.so through the efs_napi addon.
//
// Same method names, argument objects, return shapes and async/sync split as
// WebGPUEngine, so its callers (app/sim-worker.js:730-731,
// scripts/lib/sim-engine.mjs:537-538) change one import.  Every method
// forwards to one addon function (node/efs_napi.cc), which calls the matching
// efs_* entry point of include/efs.h; a failing call throws an Error with
// libefs's message, as WebGPUEngine throws on misuse.
//
// Methods that take a GPUCommandEncoder (stepVoltage, stepPML, ...) are
// WebGPU encoding hooks used inside WebGPUEngine.iterate; the CUDA engine
// runs whole timesteps as captured CUDA graphs, so they throw.  The
// WG_SIZE_3D* workgroup shapes are accepted and ignored.
import { createRequire } from 'node:module';

const require = createRequire(import.meta.url);
const addon = require('./build/Release/efs_napi.node');

const u32 = (a) => (a instanceof Uint32Array ? a : Uint32Array.from(a));
const f32 = (a) => (a instanceof Float32Array ? a : Float32Array.from(a));
const f64 = (a) => (a instanceof Float64Array ? a : Float64Array.from(a));

function encoderHook(name) {
    throw new Error(`${name}(encoder) is a WebGPU command-encoder hook; the CUDA engine runs whole timesteps: use iterate(n)`);
}

export class WebGPUEngine {
    constructor() {
        this._e = null;
        this.numLines = null;
        this.totalCells = 0;
        this._numTS = 0;
        this.device = null;
        this.WG_SIZE_3D = [4, 1, 16];
        this.WG_SIZE_3D_VOLTAGE = null;
        this.WG_SIZE_3D_CURRENT = null;
        this.ssConfigured = false;
        this.ssCurrentSample = 0;
        this._ssRecording = false;
        this._ssNumProbes = 0;
        this._gatherCount = 0;
        this._nf2ffNumPoints = 0;
        this._nf2ffNumFreq = 0;
    }

    _need() {
        if (!this._e) throw new Error('CUDA device not initialized. Call initGPU() first.');
        return this._e;
    }

    // :1107-1135 — false when no CUDA device can be opened
    async initGPU() {
        this._e = addon.create(0);
        if (!this._e) return false;
        const e = this._e;
        // callers wait on device.queue.onSubmittedWorkDone() (app/sim-worker.js:887)
        this.device = { queue: { onSubmittedWorkDone: async () => addon.sync(e) } };
        return true;
    }

    // :1143-1185 — coefficients {vv, vi, ii, iv} (Float32Array 3N each), or
    // {mat, table} (material index per cell + 12-float rows; no reference counterpart)
    async init(gridSize, coefficients) {
        const e = this._need();
        const dims = u32(gridSize);
        if (coefficients.mat) addon.initIndexed(e, dims, u32(coefficients.mat), f32(coefficients.table));
        else addon.init(e, dims, f32(coefficients.vv), f32(coefficients.vi), f32(coefficients.ii), f32(coefficients.iv));
        this.numLines = [dims[0], dims[1], dims[2]];
        this.totalCells = dims[0] * dims[1] * dims[2];
        this._numTS = 0;
    }

    get numTS() { return this._e ? addon.numTS(this._e) : this._numTS; }

    // :1199-1227 — {signal, delay, amp, dir, pos, period}
    configureExcitation(excitation) {
        addon.configureExcitation(this._need(), f32(excitation.signal), u32(excitation.delay), f32(excitation.amp),
            u32(excitation.dir), u32(excitation.pos), excitation.period || 0);
    }

    // :1235-1323 — [{startPos, numLines, vv, vvfo, vvfn, ii, iifo, iifn}]
    configurePML(pmlRegions) {
        addon.configurePML(this._need(), pmlRegions.map((r) => ({
            startPos: Array.from(r.startPos), numLines: Array.from(r.numLines),
            vv: f32(r.vv), vvfo: f32(r.vvfo), vvfn: f32(r.vvfn), ii: f32(r.ii), iifo: f32(r.iifo), iifn: f32(r.iifn),
        })));
    }

    stepPML(encoder, mode) { encoderHook('stepPML'); }

    // :1358-1475 — {orders: [{numCells, hasLorentz, directions: [{dir, pos_idx, v_int_ADE, ...}]}]};
    // `apply: true` turns on the apply step the reference lacks (efs_configure_ade_apply)
    configureLorentzADE(config) {
        const orders = config.orders.map((o) => ({
            numCells: o.numCells, hasLorentz: !!o.hasLorentz,
            directions: o.directions.map((d) => {
                const out = { dir: d.dir, pos_idx: u32(d.pos_idx) };
                for (const k of ['v_int_ADE', 'v_ext_ADE', 'v_Lor_ADE', 'i_int_ADE', 'i_ext_ADE', 'i_Lor_ADE'])
                    if (d[k]) out[k] = f32(d[k]);
                return out;
            }),
        }));
        addon.configureADE(this._need(), orders, !!config.apply);
    }

    stepVoltADE(encoder) { encoderHook('stepVoltADE'); }
    stepCurrADE(encoder) { encoderHook('stepCurrADE'); }

    // :1527-1645 — {signal, period, voltagePoints, currentPoints}, points {field_idx, delay_int, delay_frac, amp}
    configureTFSF(config) {
        const pack = (pts) => {
            const n = pts.length;
            const fi = new Uint32Array(n), di = new Uint32Array(n), df = new Float32Array(n), am = new Float32Array(n);
            for (let i = 0; i < n; i++) {
                fi[i] = pts[i].field_idx; di[i] = pts[i].delay_int; df[i] = pts[i].delay_frac; am[i] = pts[i].amp;
            }
            return [fi, di, df, am];
        };
        addon.configureTFSF(this._need(), f32(config.signal), config.period || 0,
            ...pack(config.voltagePoints || []), ...pack(config.currentPoints || []));
    }

    stepTFSFVoltage(encoder) { encoderHook('stepTFSFVoltage'); }
    stepTFSFCurrent(encoder) { encoderHook('stepTFSFCurrent'); }

    // :1722-1808 — {elements: [{field_idx, direction, type_flag, i2v, ilv, vvd, vv2, vj1, vj2, ib0, b1, b2}]}
    configureRLC(config) {
        const n = config.elements.length;
        if (n === 0) return;
        const w = new Uint32Array(3 * n), v = new Float32Array(9 * n);
        const keys = ['i2v', 'ilv', 'vvd', 'vv2', 'vj1', 'vj2', 'ib0', 'b1', 'b2'];
        config.elements.forEach((el, i) => {
            w[3 * i] = el.field_idx; w[3 * i + 1] = el.direction; w[3 * i + 2] = el.type_flag;
            keys.forEach((k, j) => { v[9 * i + j] = el[k] || 0; });
        });
        addon.configureRLC(this._need(), w, v);
    }

    stepRLC(encoder) { encoderHook('stepRLC'); }

    // :1822-1918 — {coeff, normal_idx, shifted_idx} or the dual form (nyP then nyPP, concatenated as the reference)
    configureMur(config) {
        let coeff, normal, shifted;
        if (config.coeff_nyP) {
            coeff = Float32Array.from([...config.coeff_nyP, ...config.coeff_nyPP]);
            normal = Uint32Array.from([...config.normal_idx_nyP, ...config.normal_idx_nyPP]);
            shifted = Uint32Array.from([...config.shifted_idx_nyP, ...config.shifted_idx_nyPP]);
        } else {
            normal = u32(config.normal_idx);
            shifted = u32(config.shifted_idx);
            coeff = typeof config.coeff === 'number' ? new Float32Array(normal.length).fill(config.coeff) : f32(config.coeff);
        }
        addon.configureMur(this._need(), coeff, normal, shifted);
    }

    stepMurPre(encoder) { encoderHook('stepMurPre'); }
    stepMurPost(encoder) { encoderHook('stepMurPost'); }
    stepMurApply(encoder) { encoderHook('stepMurApply'); }

    // :1976-2155 — {axes: [{axis, phase}]}
    configurePBC(config) {
        const axes = config.axes || [];
        if (axes.length === 0) return;
        addon.configurePBC(this._need(), Uint32Array.from(axes.map((a) => a.axis)),
            Float64Array.from(axes.map((a) => a.phase || 0)));
    }

    stepPBCVoltage(encoder) { encoderHook('stepPBCVoltage'); }
    stepPBCCurrent(encoder) { encoderHook('stepPBCCurrent'); }

    // :2170-2216 — {probe_idx, periodSamples, threshold}; recording is switched by ssRecording
    configureSteadyState(config) {
        addon.configureSteadyState(this._need(), u32(config.probe_idx), config.periodSamples, config.threshold || 1e-6);
        this._ssNumProbes = config.probe_idx.length;
        this.ssConfigured = true;
        this.ssCurrentSample = 0;
        this._ssRecording = false;
    }

    get ssRecording() { return this._ssRecording; }
    set ssRecording(on) {
        if (this.ssConfigured) addon.setSteadyStateRecording(this._need(), !!on);
        this._ssRecording = !!on;
    }

    // steady-state energies of the probes: {energy1, energy2, currentSample, converged}
    async readSteadyState() {
        const r = addon.readSteadyState(this._need(), this._ssNumProbes);
        this.ssCurrentSample = r.currentSample;
        return r;
    }

    stepSteadyState(encoder) { encoderHook('stepSteadyState'); }
    stepVoltage(encoder, options = {}) { encoderHook('stepVoltage'); }
    stepCurrent(encoder, options = {}) { encoderHook('stepCurrent'); }
    applyExcitation(encoder, options = {}) { encoderHook('applyExcitation'); }
    dispatchIfActive(encoder, pipeline, bindGroups, dispatchSize) { encoderHook('dispatchIfActive'); }

    // :2407-2504 — enqueue numSteps timesteps (no wait)
    iterate(numSteps) {
        addon.iterate(this._need(), numSteps);
    }

    // :2512-2527 — [{component, x, y, z}] -> Float32Array(2 * n) of (volt, curr) pairs
    async readProbe(positions) {
        const fields = await this.getFields();
        const [Nx, Ny, Nz] = this.numLines;
        const out = new Float32Array(positions.length * 2);
        positions.forEach(({ component: n, x, y, z }, i) => {
            const idx = n * Nx * Ny * Nz + x * Ny * Nz + y * Nz + z;
            out[2 * i] = fields.volt[idx];
            out[2 * i + 1] = fields.curr[idx];
        });
        return out;
    }

    // :2533-2561 — {volt, curr}
    async getFields() {
        return addon.getFields(this._need(), 3 * this.totalCells);
    }

    // :2568-2571
    uploadFields(volt, curr) {
        addon.setFields(this._need(), f32(volt), f32(curr));
    }

    // :2577-2616
    configureProbeGather(indices) {
        if (indices.length === 0) return;
        addon.configureProbeGather(this._need(), u32(indices));
        this._gatherCount = indices.length;
    }

    // :2623-2681
    configureProbeGatherBuffered(indices, { maxSamples, sampleInterval }) {
        if (indices.length === 0) return;
        addon.configureProbeGatherBuffered(this._need(), u32(indices), maxSamples, sampleInterval);
        this._gatherCount = indices.length;
    }

    // :2689-2695 — {data, numSamples, stride} or null before the first sample
    async readProbeGatherBuffered() {
        return addon.readProbeGatherBuffered(this._need());
    }

    // :2701-2715 — interleaved [volt0, curr0, ...] or null when not configured
    async readProbeGather() {
        if (this._gatherCount === 0) return null;
        return addon.readProbeGather(this._need(), this._gatherCount);
    }

    // :2729-2827 — {surfaceIndices, numPoints, omega (or omegas), dT, gridSize, primalEdgeLens,
    // dualEdgeLens, maxTS, windowType}
    configureNF2FFAccumulation(config) {
        const { surfaceIndices, numPoints, omega, omegas, dT, primalEdgeLens, dualEdgeLens, maxTS = 0, windowType = 0 } = config;
        if (numPoints === 0) return;
        const om = f64(omegas || [omega]);
        const lens = Float32Array.from([...primalEdgeLens[0], ...primalEdgeLens[1], ...primalEdgeLens[2],
            ...dualEdgeLens[0], ...dualEdgeLens[1], ...dualEdgeLens[2]]);
        addon.configureNF2FF(this._need(), u32(surfaceIndices), numPoints, om, dT, lens, maxTS, windowType);
        this._nf2ffNumPoints = numPoints;
        this._nf2ffNumFreq = om.length;
    }

    // :2844-2855 — {accumE, accumH} of the first frequency (all frequencies with allFrequencies)
    async readNF2FFAccumulation(allFrequencies = false) {
        if (this._nf2ffNumPoints === 0) return null;
        const per = this._nf2ffNumPoints * 6;
        const r = addon.readNF2FF(this._need(), per * this._nf2ffNumFreq);
        if (allFrequencies) return r;
        return { accumE: r.accumE.subarray(0, per), accumH: r.accumH.subarray(0, per) };
    }

    // :2871-2967 — {pointMeta, theta, phi, center, frequency, radius, numPoints[, freqIndex]}
    // -> Float32Array(5 per angle: P_rad, Et_re, Et_im, Ep_re, Ep_im)
    async computeNF2FFfarField(config) {
        const { pointMeta, theta, phi, center, frequency, radius, freqIndex = 0 } = config;
        return addon.farField(this._need(), freqIndex, f32(pointMeta), f32(theta), f32(phi), f64(center), frequency, radius);
    }

    // :2974-3021 — lagged by one call (the previous call's value, 0 first)
    async computeEnergy() {
        return addon.energy(this._need(), true);
    }

    // :3027-3037
    async flushEnergy() {
        return addon.flushEnergy(this._need());
    }

    // :3163-3229
    destroy() {
        if (this._e) addon.destroy(this._e);
        this._e = null;
        this.device = null;
    }
}

export { WebGPUEngine as CudaEngine };
export default WebGPUEngine;
