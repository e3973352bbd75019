/*
 * efs.h — C ABI of the B200 FDTD engine (libefs.so).
 *
 * Every entry point replaces one method of the reference's WebGPU engine
 * class `WebGPUEngine` (src/webgpu-engine.mjs, class at :994-3498) so that a
 * thin FFI shim (N-API, ctypes, cffi) can keep that class's JavaScript
 * surface.  Paths below are relative to the roman01la/efs tree.
 *
 * Conventions
 *   - Every function returns efs_status (EFS_OK == 0) and never aborts the
 *     process; efs_last_error() gives the message of the last failure.
 *   - All buffers are caller-owned HOST memory (plain pointers + sizes); the
 *     engine copies inputs into device memory at configure time and copies
 *     results out on read, exactly like the reference's typed-array contract
 *     (_createAndUploadBuffer :3231-3247, _readBuffer :3249-3266).
 *   - Fields use the reference layout NIJK: addr = n*Nx*Ny*Nz + x*Ny*Nz + y*Nz + z
 *     (src/webgpu-engine.mjs:33-43).  Index arguments (excitation pos, Mur,
 *     TFSF, ADE, probe indices) are u32 offsets in that layout.
 *   - One CUDA stream per engine.  An engine is not thread-safe; distinct
 *     engines may be driven from different threads.
 *   - Device-side waits are bounded; a wait that runs out returns
 *     EFS_ERR_TIMEOUT instead of hanging.
 */
#ifndef EFS_H
#define EFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int efs_status;
enum {
    EFS_OK = 0,
    EFS_ERR_INVALID = 1,   /* bad argument (size, index, null pointer)      */
    EFS_ERR_STATE = 2,     /* call out of order (e.g. iterate before init)  */
    EFS_ERR_CUDA = 3,      /* CUDA runtime error                            */
    EFS_ERR_OOM = 4,       /* device allocation failed / over HBM budget    */
    EFS_ERR_TIMEOUT = 5,   /* a bounded device wait ran out                 */
    EFS_ERR_RANGE = 6      /* request exceeds a fixed limit                 */
};

typedef struct efs_engine efs_engine;

/* --- lifetime ---------------------------------------------------------- */

/* WebGPUEngine.initGPU (:1107-1135): bind a device, create the stream.
 * Returns EFS_ERR_CUDA when no device is usable (the reference returns false).
 * Each engine's pinned host words (the status word its kernels report a
 * timed-out wait through, two energy result slots: 32 bytes) come from
 * mapped pinned pages of 4 KB that the library keeps for the life of the
 * process and hands to later engines after efs_destroy. */
efs_status efs_create(efs_engine** out, int device);

/* WebGPUEngine.destroy (:3163-3227): waits for the engine's stream, frees its
 * device memory and graphs.  Safe on NULL. */
efs_status efs_destroy(efs_engine* e);

/* Message of the last failing call on this engine (or of the last failing
 * efs_create when e is NULL). Never NULL. */
const char* efs_last_error(const efs_engine* e);

/* WebGPUEngine.init (:1143-1185): grid [Nx,Ny,Nz] and the four dense
 * operator arrays vv,vi,ii,iv (3*Nx*Ny*Nz floats each, NIJK), as returned by
 * the reference's embind getters (src/embind_api.cpp:230-266, :998-1024).
 * The engine deduplicates the per-cell 12-float coefficient tuples into a
 * material table (bit-identical values) when that shrinks the footprint,
 * else keeps the dense arrays.  Fields start at zero, numTS at 0. */
efs_status efs_init(efs_engine* e, const uint32_t dims[3],
                    const float* vv, const float* vi, const float* ii, const float* iv);

/* Same as efs_init with the coefficients already factored: mat[cell] (Nx*Ny*Nz
 * u32) indexes rows of `table` (ntable rows of 12 floats:
 * vv_x vv_y vv_z vi_x vi_y vi_z ii_x ii_y ii_z iv_x iv_y iv_z).
 * No counterpart in the reference (it always ships dense arrays); used by
 * operator generators that know the material of each cell.  An index >=
 * ntable returns EFS_ERR_INVALID (checked on the device after the upload)
 * and leaves the engine uninitialised. */
efs_status efs_init_indexed(efs_engine* e, const uint32_t dims[3],
                            const uint32_t* mat, const float* table, uint32_t ntable);

/* --- extensions (configure*) ------------------------------------------- */

/* configureExcitation (:1199-1227); semantics of engine_ext_excitation.cpp as
 * restated in src/webgpu-fdtd.mjs:161-185 (past the signal end: signal[0]). */
efs_status efs_configure_excitation(efs_engine* e, const float* signal, uint32_t signal_len,
                                    const uint32_t* delay, const float* amp,
                                    const uint32_t* dir, const uint32_t* pos,
                                    uint32_t count, uint32_t period);

/* One UPML region, as the objects passed to configurePML (:1235-1323) and
 * extracted by getPMLRegion (src/embind_api.cpp:580-623). Each array holds
 * 3*num[0]*num[1]*num[2] floats in NIJK order local to the region. */
typedef struct {
    uint32_t start[3];
    uint32_t num[3];
    const float* vv;
    const float* vvfo;
    const float* vvfn;
    const float* ii;
    const float* iifo;
    const float* iifn;
} efs_pml_region;

efs_status efs_configure_pml(efs_engine* e, uint32_t count, const efs_pml_region* regions);

/* configureMur (:1822-1918), single-component form; the dual form is the
 * concatenation nyP then nyPP (:1827-1842), done by the caller. */
efs_status efs_configure_mur(efs_engine* e, const float* coeff, const uint32_t* normal_idx,
                             const uint32_t* shifted_idx, uint32_t count);

/* TFSF injection point (configureTFSF :1527-1645). */
typedef struct {
    uint32_t field_idx;
    uint32_t delay_int;
    float delay_frac;
    float amp;
} efs_tfsf_point;

efs_status efs_configure_tfsf(efs_engine* e, const float* signal, uint32_t signal_len, uint32_t period,
                              const efs_tfsf_point* volt_points, uint32_t n_volt,
                              const efs_tfsf_point* curr_points, uint32_t n_curr);

/* Lorentz/Drude ADE (configureLorentzADE :1358-1475, state math of
 * src/webgpu-fdtd.mjs:405-454).  Null coefficient pointers mean zeros. */
typedef struct {
    uint32_t dir;
    const uint32_t* pos_idx;
    const float* v_int;
    const float* v_ext;
    const float* v_lor;
    const float* i_int;
    const float* i_ext;
    const float* i_lor;
} efs_ade_direction;

typedef struct {
    uint32_t num_cells;
    uint32_t has_lorentz;
    uint32_t num_directions;
    const efs_ade_direction* directions;
} efs_ade_order;

efs_status efs_configure_ade(efs_engine* e, uint32_t count, const efs_ade_order* orders);

/* Opt-in ADE apply step (on != 0), off by default and after every efs_init.
 * The reference updates the ADE state and never applies it to the fields
 * (src/webgpu-fdtd.mjs:405-454, step order :1129-1172), so dispersion never
 * reaches E or H there.  With the step on, each entry's state is subtracted
 * from its field, in configuration order: E entries after the
 * apply-to-voltages phase (excitation, Mur apply, RLC apply), H entries after
 * the post-current phase (TFSF, PBC) -- openEMS's Apply2Voltages /
 * Apply2Current semantics.  No counterpart in the reference's API; the JS
 * class maps configureLorentzADE({orders, apply: true}) to it. */
efs_status efs_configure_ade_apply(efs_engine* e, int on);

/* Lumped RLC element, same 48-byte packing as configureRLC (:1738-1756). */
typedef struct {
    uint32_t field_idx;
    uint32_t direction;
    uint32_t type_flag;   /* 0 = parallel, 1 = series */
    float i2v, ilv, vvd, vv2, vj1, vj2, ib0, b1, b2;
} efs_rlc_element;

efs_status efs_configure_rlc(efs_engine* e, uint32_t count, const efs_rlc_element* elements);

/* configurePBC (:1976-2123): periodic / Bloch axes, phases in radians. */
efs_status efs_configure_pbc(efs_engine* e, uint32_t count, const uint32_t* axes, const double* phases);

/* configureSteadyState (:2170-2216) and its recording switch (ssRecording). */
efs_status efs_configure_steady_state(efs_engine* e, const uint32_t* probe_idx, uint32_t count,
                                      uint32_t period_samples, float threshold);
efs_status efs_set_steady_state_recording(efs_engine* e, int recording);
/* Reads both period accumulators (count floats each, may be NULL), the sample
 * counter and the convergence test of src/webgpu-fdtd.mjs:1076-1092. */
efs_status efs_read_steady_state(efs_engine* e, float* energy_period1, float* energy_period2,
                                 uint32_t* current_sample, int* converged);

/* --- stepping ---------------------------------------------------------- */

/* WebGPUEngine.iterate (:2407-2504): n full timesteps in the phase order of
 * CPUFDTDEngine.step (src/webgpu-fdtd.mjs:1129-1172), then NF2FF
 * accumulation and the buffered probe gather.  Asynchronous: returns once
 * the work is queued on the engine's stream (as the reference's submit). */
efs_status efs_iterate(efs_engine* e, uint32_t n);

/* numTS (the reference's public field). */
efs_status efs_num_ts(const efs_engine* e, uint32_t* out);

/* Wait for all queued work (the reference's readback await). */
efs_status efs_sync(efs_engine* e);

/* The engine's cudaStream_t, for callers that time or order work around it. */
efs_status efs_get_stream(efs_engine* e, void** stream);

/* --- probes ------------------------------------------------------------ */

/* configureProbeGather (:2577-2621) / readProbeGather (:2701-2715):
 * out[2i] = volt[idx_i], out[2i+1] = curr[idx_i]. */
efs_status efs_configure_probe_gather(efs_engine* e, const uint32_t* indices, uint32_t count);
efs_status efs_read_probe_gather(efs_engine* e, float* out, size_t out_len);

/* configureProbeGatherBuffered (:2623-2681) / readProbeGatherBuffered
 * (:2689-2694): one row of 2*count floats every sample_interval steps, at
 * most max_samples rows.  out may be NULL to query num_samples/stride. */
efs_status efs_configure_probe_gather_buffered(efs_engine* e, const uint32_t* indices, uint32_t count,
                                               uint32_t max_samples, uint32_t sample_interval);
efs_status efs_read_probe_gather_buffered(efs_engine* e, float* out, size_t out_len,
                                          uint32_t* num_samples, uint32_t* stride);

/* --- NF2FF ------------------------------------------------------------- */

/* configureNF2FFAccumulation (:2729-2827) generalised to `num_freq`
 * frequencies.  points: (ix,iy,iz) triplets; edge_lens: primal x,y,z then dual
 * x,y,z (Nx,Ny,Nz floats each, sim-engine.mjs:577-591).  The phase
 * omega*n*dT is formed in f64. */
efs_status efs_configure_nf2ff(efs_engine* e, const uint32_t* points, uint32_t num_points,
                               const double* omegas, uint32_t num_freq, double dT,
                               const float* edge_lens, uint32_t max_ts, uint32_t window_type);

/* readNF2FFAccumulation (:2844-2855): num_freq blocks of num_points*6 floats
 * (re/im of x,y,z) for E and for H. */
efs_status efs_read_nf2ff(efs_engine* e, float* accum_e, float* accum_h, size_t len);

/* computeNF2FFfarField (:2871-2967) for frequency block `freq_index`:
 * point_meta 8 floats per point (pos xyz, normalDir, normSign, area, 0, 0);
 * out 5 floats per (theta,phi): P_rad, Et_re, Et_im, Ep_re, Ep_im. */
efs_status efs_far_field(efs_engine* e, uint32_t freq_index, const float* point_meta,
                         const float* theta, uint32_t n_theta, const float* phi, uint32_t n_phi,
                         const double center[3], double frequency, double radius, float* out);

/* Diagnostics: device time (ms) of the last efs_far_field call's two kernels:
 * ms[0] the per-point records, ms[1] the angle sums.  No counterpart in the
 * reference. */
efs_status efs_far_field_time(const efs_engine* e, float* ms);

/* --- energy ------------------------------------------------------------ */

/* computeEnergy (:2974-3021): sum over the (Nx-1)(Ny-1)(Nz-1) interior
 * cells of volt^2+curr^2.  With lagged != 0 it keeps the reference's
 * double-buffered contract (returns the previous call's value, 0 first);
 * with lagged == 0 it waits and returns the current value. */
efs_status efs_energy(efs_engine* e, int lagged, double* out);
/* flushEnergy (:3027-3037). */
efs_status efs_flush_energy(efs_engine* e, double* out);
/* The current energy (what efs_energy returns with lagged == 0), computed
 * without allocating any device memory.  For callers that cannot let the
 * library call cudaMalloc once they are running: a server that reserves its
 * whole HBM budget for solves up front, or a host runtime that owns every
 * device allocation, where a lazy allocation could fail mid-run or break the
 * caller's accounting (efs_energy allocates its scratch on first use).
 * Scratch is a fixed array inside libefs.so: 16384 partial sums + 1 result
 * (128 KB), held by every GPU that loads the library until the process
 * exits; a grid with more than 2^30 interior cells returns EFS_ERR_RANGE.
 * The first call on each device looks up the array's device address; make
 * that first call before any stream capture.  Devices with ordinals 0..63
 * are served (EFS_ERR_RANGE above).  All calls on a device share
 * the array (each call writes what it reads, so nothing needs clearing):
 * calls that overlap on the GPU, e.g. two engines on one device driven from
 * two threads, race.  Sums in a different order than efs_energy (agrees to
 * ~1e-12 relative).  No counterpart in the reference. */
efs_status efs_energy_noalloc(efs_engine* e, double* out);

/* --- state transfer ---------------------------------------------------- */

/* getFields (:2533-2561) / uploadFields (:2568-2571): 3*Nx*Ny*Nz floats each. */
efs_status efs_get_fields(efs_engine* e, float* volt, float* curr);
efs_status efs_set_fields(efs_engine* e, const float* volt, const float* curr);

/* x-planes [x, x + count) of E (volt) and H (curr), packed as 3 components x
 * count planes x Ny*Nz floats in the reference's NIJK order; either pointer
 * may be NULL; host or device memory (the copy kind is inferred).  The ghost
 * exchange of an x-slab decomposition (efs_b200/slabs.py) moves these planes
 * between the engines of neighbouring slabs.  No counterpart in the
 * reference. */
efs_status efs_get_planes(efs_engine* e, uint32_t x, uint32_t count, float* volt, float* curr);
efs_status efs_set_planes(efs_engine* e, uint32_t x, uint32_t count, const float* volt, const float* curr);

/* Full resident state (fields, UPML flux, Mur, ADE, RLC, steady state, PBC,
 * probe ring, NF2FF accumulators, numTS) as one opaque blob.  buf == NULL
 * queries the size.  Restoring needs an engine with the same configuration.
 * No counterpart in the reference (its getFields covers fields only). */
efs_status efs_get_state(efs_engine* e, void* buf, size_t cap, size_t* size);
efs_status efs_set_state(efs_engine* e, const void* buf, size_t size);

/* Bytes of device memory the engine holds. */
efs_status efs_device_bytes(const efs_engine* e, size_t* out);

/* Diagnostics: copy one internal state array, by name, into `out` (floats).
 * Names: "pml_volt_flux", "pml_curr_flux" (arg = region), "mur_saved",
 * "ade_volt", "ade_volt_lor", "ade_curr", "ade_curr_lor" (all orders and
 * directions concatenated in configuration order), "rlc_vdn", "rlc_jn",
 * "rlc_vil" (caller's element order), "pbc_imag", "tfsf_faces" (the planned
 * TFSF z faces whose E corrections the fused update applies: count, then
 * each face's z).  out == NULL queries the count.  Mirrors the reference tests' direct reads of engine state
 * (tests/test_webgpu.mjs, e.g. :1215, :1946, :2224).  No counterpart in the
 * engine class itself. */
efs_status efs_debug_read(efs_engine* e, const char* name, uint32_t arg, float* out, size_t cap, size_t* count);

/* Diagnostics: launch the engine's core field-update kernels `reps` times
 * on its stream and return the mean device time per launch (CUDA events):
 * ms[0] = the fused E+H kernel, ms[1] = the UPML-cell passes around it (0
 * without UPML regions).  Advances the fields; meant for benchmarks only.
 * No counterpart in the reference. */
efs_status efs_time_core(efs_engine* e, uint32_t reps, float* ms);

/* Diagnostics for failure detection: the limit of every bounded wait in the
 * fused kernel (default 1 s = 1e9 ns; 1 ns .. 10 s accepted) and an x-plane
 * whose loads the kernel never issues (~0u = none, the default).  With a
 * plane skipped, every CTA that streams it gives up after wait_ns, drains
 * its other loads and returns; the next synchronising call returns
 * EFS_ERR_TIMEOUT and the engine's fields are then undefined.  Nothing
 * faults or hangs: the wait gives up.  The reference only logs a lost device
 * (src/webgpu-engine.mjs:1129-1131). */
efs_status efs_debug_set_wait(efs_engine* e, uint64_t wait_ns, uint32_t skip_plane);

/* Tuning: x-planes each CTA of the fused kernel streams (default 32; 1 ..
 * 65535).  Results are bit-identical under every depth; it moves the CTA
 * seams and trades halo re-reads against parallelism.  Kept across init.
 * No counterpart in the reference. */
efs_status efs_set_plane_depth(efs_engine* e, uint32_t xchunk);

/* Diagnostics: device time per timestep of each phase of the step, over
 * `steps` (1..64) timesteps launched kernel by kernel with events between the
 * phases (not as a graph; the engine advances as by efs_iterate and the
 * results are the same).  ms[EFS_PHASES], mean ms per timestep:
 *   0 steady-state accumulation and the UPML E pass (with the previous
 *     step's NF2FF samples in the same launch when they are paired),
 *   1 point operations before the core update (ADE, Mur pre, RLC pre),
 *   2 fused core update, 3 E-side point operations (TFSF, PBC, Mur
 *     post/apply, excitation, RLC, ADE apply), 4 UPML H pass and deferred H
 *     recompute (one launch), 5 H-side point operations, 6 NF2FF samples /
 *     accumulation and probe ring.
 * No counterpart in the reference. */
#define EFS_PHASES 7
efs_status efs_time_phases(efs_engine* e, uint32_t steps, float* ms);

/* Diagnostics: kernel launches one timestep enqueues with the current
 * configuration (a captured batch of n steps adds one counter update and,
 * with NF2FF configured, ceil(n/16) accumulator passes and, when the samples
 * ride on the next step's UPML E pass, one sample pass for its last step). */
efs_status efs_kernels_per_step(efs_engine* e, uint32_t* out);

/* --- batched form ------------------------------------------------------
 * No counterpart in the reference (its sweeps run one solve after another).
 * A batch advances several configured engines of one device together: one
 * persistent fused-update launch over a work-tile list spanning every
 * member, one launch per sparse phase for all members, up to 64 steps per
 * captured CUDA graph.  Each member computes exactly what it computes alone
 * and keeps its own step counter; between batch calls each member stays
 * usable through the per-engine calls (probe reads, energy, fields).  Members
 * need the TMA-fed fused path (Nz a multiple of 4) and may use excitation,
 * Mur, TFSF, Lorentz/Drude ADE, UPML, NF2FF and the probe ring (not steady
 * state, RLC, PBC); members may mix material-index and dense coefficients.  Stepping
 * or reconfiguring a member on its own between batch calls is allowed: the
 * batch re-plans. */
typedef struct efs_batch efs_batch;
efs_status efs_batch_create(efs_batch** out, efs_engine* const* engines, uint32_t count);
efs_status efs_batch_destroy(efs_batch* b);
const char* efs_batch_last_error(const efs_batch* b);
/* Advance every member n timesteps (ordered after and before the members'
 * own stream work; returns without waiting). */
efs_status efs_batch_iterate(efs_batch* b, uint32_t n);
efs_status efs_batch_sync(efs_batch* b);
/* Plane depth (x-planes per work tile) and resident CTAs per SM (1 or 2) of
 * the persistent launch; results do not depend on them. */
efs_status efs_batch_set_shape(efs_batch* b, uint32_t xchunk, uint32_t ctas_per_sm);
/* Autotuner: times `steps` real timesteps for each candidate shape (plane
 * depth 8/16/32/64 x 1-2 CTAs per SM), keeps the fastest and reports it.
 * The timed steps advance the members (bit-identical under every shape):
 * the batch moves forward by 17*steps timesteps in all. */
efs_status efs_batch_autotune(efs_batch* b, uint32_t steps, uint32_t* xchunk, uint32_t* ctas_per_sm, float* ms_per_step);
/* Diagnostics: device ms per timestep of each phase of a batched step, over
 * `steps` (1..64) timesteps launched kernel by kernel (phases as in
 * efs_time_phases, each for all members); the batch advances as by
 * efs_batch_iterate. */
efs_status efs_batch_time_phases(efs_batch* b, uint32_t steps, float* ms);

#ifdef __cplusplus
}
#endif

#endif /* EFS_H */
