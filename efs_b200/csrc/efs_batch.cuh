// efs_batch.cuh — batched form: several engines advanced together.
//
// A batch is a set of configured engines on one device (uneven grids, each
// with its own fields, extensions, step counter and parity).  One timestep of
// the batch is the engines' phase order with every phase issued once for all
// members:
//   * the core update is one persistent launch of k_fused_tma_batch (one per
//     coefficient kind present: material index or dense): every
//     CTA walks a work-tile list spanning all members (tile = member, 64x8
//     tile origin, x-chunk) and runs each tile through the same TMA plane
//     pipeline as the single engine, reading the member's grid, UPML set and
//     tensor maps from a descriptor in global memory;
//   * each sparse phase (Mur, excitation, TFSF, ADE, UPML passes, deferred H,
//     NF2FF, probe ring, step counter) is one segmented launch: block b
//     belongs to member seg[b] and runs the single engine's thread body on
//     that member's arguments.
// Up to 64 such steps are captured in one CUDA graph.  Every member computes
// exactly what it computes alone (same thread bodies, same order per member).
// The plane depth (x-chunk) and CTAs per SM of the persistent launch are
// runtime knobs; efs_batch_autotune picks them by timing real steps, which
// are bit-identical under every setting.
//
// efs_engine.cu includes this file at its end (one translation unit).
#pragma once

namespace efs {

// ---- core update over all members ------------------------------------------
struct BatchMember {            // one member at one step parity (tensor maps first: 64-byte aligned)
    CUtensorMap tmH, tmE, tmM, tmD;
    FusedGrid g;
    PmlSet ps;
};
struct BatchTile { uint32_t m, xs, y0, z0; };

// Persistent: CTA b runs tiles b, b + gridDim.x, ... of a list whose members
// all use material-index (IDX) or all dense coefficients.
template <bool IDX>
__global__ void __launch_bounds__(TT_THREADS, 2)
k_fused_tma_batch(const BatchMember* __restrict__ mem, const BatchTile* __restrict__ tiles, uint32_t ntiles) {
    TmaSmem& S = tt_smem();
    tt_init(S);
    uint32_t K = 0;                                    // planes this CTA has consumed
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile w = tiles[t];
        const BatchMember& M = mem[w.m];
        if (!tma_tile_body<IDX, true, true>(S, &M.tmH, &M.tmE, &M.tmM, &M.tmD, M.g, M.ps, w.xs, w.y0, w.z0, K)) return;
    }
}

// ---- segmented sparse phases ------------------------------------------------
// Block b of a segmented launch runs segment seg[b]'s op with block index
// b - first[seg[b]] inside the segment.  k: step within the captured batch;
// a, b: per-launch arguments of the op.
struct SegMap { const uint32_t* seg; const uint32_t* first; };

template <class Op>
__global__ void __launch_bounds__(256) k_seg(const Op* __restrict__ ops, SegMap sm, uint32_t k, uint32_t a, uint32_t b) {
    const uint32_t s = sm.seg[blockIdx.x];
    ops[s].run(blockIdx.x - sm.first[s], k, a, b);
}

struct OpMurPre {
    const float* V; MurDev m;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const { mur_pre_body(V, m, blk * blockDim.x + threadIdx.x); }
};
struct OpMurPost {
    const float* V; MurDev m;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const { mur_post_body(V, m, blk * blockDim.x + threadIdx.x); }
};
struct OpMurApply {
    float* V; MurDev m;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const { mur_apply_body(V, m, blk * blockDim.x + threadIdx.x); }
};
template <int KIND>
struct OpPoints {
    float* F; const StepState* st; PointSources s;
    __device__ void run(uint32_t blk, uint32_t k, uint32_t, uint32_t) const {
        point_sources_body<KIND>(F, st, k, s, blk * blockDim.x + threadIdx.x);
    }
};
struct OpAde {
    const float* F; AdeDev a;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const { ade_body(F, a, blk * blockDim.x + threadIdx.x); }
};
struct OpTfsfFace {
    const StepState* st; TfsfFaceDev t;
    __device__ void run(uint32_t blk, uint32_t k, uint32_t, uint32_t) const { tfsf_face_body(st, k, t, blk * blockDim.x + threadIdx.x); }
};
struct OpAdeApply {
    float* F; AdeApplyDev a; uint32_t runs;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const {
        if (runs) ade_apply_runs_body(F, a, blk * blockDim.x + threadIdx.x);
        else ade_apply_grouped_body(F, a, blk * blockDim.x + threadIdx.x);
    }
};
struct OpRing {
    const float* V; const float* C; const StepState* st; RingDev r;
    __device__ void run(uint32_t blk, uint32_t k, uint32_t, uint32_t) const {
        gather_ring_body(V, C, st, k, r, blk * blockDim.x + threadIdx.x);
    }
};
struct OpNfSample {
    const float* V; const float* C; Nf2ffDev d;
    __device__ void run(uint32_t blk, uint32_t, uint32_t slot, uint32_t) const {
        nf2ff_sample_body(V, C, slot, d, blk * blockDim.x + threadIdx.x);
    }
};
struct OpNfFlush {
    const StepState* st; Nf2ffDev d;
    __device__ void run(uint32_t blk, uint32_t, uint32_t k0, uint32_t cnt) const { nf2ff_flush_block(st, k0, cnt, d, blk); }
};
template <bool IDX>
struct OpDeferred {
    FusedGrid g; const uint32_t* cells; uint32_t n;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const {
        deferred_h_body<IDX>(g, cells, n, blk * blockDim.x + threadIdx.x);
    }
};
template <bool IDX>
struct OpPmlE {
    FusedGrid g; PmlSet ps, pn; float* V0w; uint32_t items;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const {
        pml_e_body<IDX>(g, ps, pn, V0w, items, blk * blockDim.x + threadIdx.x);
    }
};
template <bool IDX>
struct OpPmlH {
    FusedGrid g; PmlSet ps, pn; uint32_t items;
    __device__ void run(uint32_t blk, uint32_t, uint32_t, uint32_t) const {
        pml_h_body<IDX>(g, ps, pn, items, blk * blockDim.x + threadIdx.x);
    }
};
struct OpAdvance {
    StepState* st;
    __device__ void run(uint32_t blk, uint32_t, uint32_t n, uint32_t) const {
        if (blk == 0 && threadIdx.x == 0) st->numTS += n;
    }
};

}  // namespace efs

// ---- host side ----------------------------------------------------------------
namespace {

constexpr uint32_t SEG_T = 256;   // threads per block of every segmented launch

// One segmented launch: the ops of its members and the block -> member map.
struct SegLaunch {
    DevBuf ops, seg, first;
    uint32_t blocks = 0;
    SegMap map() const { return SegMap{seg.as<uint32_t>(), first.as<uint32_t>()}; }
};

}  // namespace

struct efs_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error = "no error";
    std::vector<efs_engine*> mem;
    std::vector<cudaEvent_t> ev_in;            // member stream -> batch stream
    cudaEvent_t ev_done = nullptr;             // batch stream -> member streams
    uint32_t xchunk = 32, ctas_per_sm = 2, sms = 148;

    // plan, per step phase s (member e at batch step k uses parity cur0[e] ^ s, s = (phase + k) & 1)
    bool planned = false;
    std::vector<int> cur0;
    uint32_t phase = 0;
    DevBuf members[2], tiles[2];               // tiles[1]: material-index members, tiles[0]: dense members
    uint32_t ntiles[2] = {0, 0};
    SegLaunch mur_pre[2], mur_post[2], mur_apply[2], exc[2], tfsf_v[2], tfsf_c[2], ade_v[2], ade_c[2], ade_apply_v[2], ade_apply_c[2],
        ring[2], nf_sample[2], nf_flush[2],
        deferred_i[2], deferred_d[2], pml_e_i[2], pml_e_d[2], pml_h_i[2], pml_h_d[2], tfsf_face[2], advance;   // _i / _d: index / dense members
    bool any_nf = false;
    std::map<uint32_t, cudaGraphExec_t> graphs;

    ~efs_batch() {
        drop_graphs();
        for (auto& ev : ev_in) if (ev) cudaEventDestroy(ev);
        if (ev_done) cudaEventDestroy(ev_done);
        if (stream) cudaStreamDestroy(stream);
    }
    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
    void upload_raw(DevBuf& b, const void* src, size_t bytes) {
        b.reset();
        ck(cudaMalloc(&b.p, bytes ? bytes : 4), "cudaMalloc");
        b.bytes = bytes ? bytes : 4;
        if (bytes) ck(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, stream), "upload");
    }

    // Segmented launch over the members that have this phase (count > 0).
    template <class Op>
    void build_seg(SegLaunch& L, const std::vector<std::pair<uint32_t, Op>>& items) {
        std::vector<Op> ops;
        std::vector<uint32_t> seg, first;
        for (auto& it : items) {
            if (it.first == 0) continue;
            first.push_back((uint32_t)seg.size());
            const uint32_t nb = blocks(it.first, SEG_T);
            for (uint32_t b = 0; b < nb; ++b) seg.push_back((uint32_t)ops.size());
            ops.push_back(it.second);
        }
        L.blocks = (uint32_t)seg.size();
        upload_raw(L.ops, ops.data(), ops.size() * sizeof(Op));
        upload_raw(L.seg, seg.data(), seg.size() * sizeof(uint32_t));
        upload_raw(L.first, first.data(), first.size() * sizeof(uint32_t));
    }
    template <class Op>
    void launch_seg(const SegLaunch& L, uint32_t k, uint32_t a = 0, uint32_t b = 0) {
        if (L.blocks) k_seg<Op><<<L.blocks, SEG_T, 0, stream>>>(L.ops.as<Op>(), L.map(), k, a, b);
    }

    void check_members() {
        for (efs_engine* e : mem) {
            e->need_init();
            if (e->device != device) fail(EFS_ERR_INVALID, "batch members must share one device");
            if (e->ss_on || e->rlc_on || e->pbc_on)
                fail(EFS_ERR_STATE, "batched stepping supports excitation, Mur, TFSF, ADE, UPML, NF2FF and the probe ring "
                                    "(not steady state, RLC or PBC)");
        }
    }

    void plan() {
        check_members();
        drop_graphs();
        const size_t E = mem.size();
        cur0.resize(E);
        for (size_t i = 0; i < E; ++i) { mem[i]->build_plan(); cur0[i] = mem[i]->cur; }
        phase = 0;
        any_nf = false;
        for (int s = 0; s < 2; ++s) {
            std::vector<BatchMember> bm(E);
            std::vector<std::pair<uint32_t, OpMurPre>> mpre;
            std::vector<std::pair<uint32_t, OpMurPost>> mpost;
            std::vector<std::pair<uint32_t, OpMurApply>> mapply;
            std::vector<std::pair<uint32_t, OpPoints<0>>> vexc;
            std::vector<std::pair<uint32_t, OpPoints<1>>> vtv, vtc;
            std::vector<std::pair<uint32_t, OpAde>> vav, vac;
            std::vector<std::pair<uint32_t, OpAdeApply>> vpv, vpc;
            std::vector<std::pair<uint32_t, OpRing>> vring;
            std::vector<std::pair<uint32_t, OpTfsfFace>> vtf;
            std::vector<std::pair<uint32_t, OpNfSample>> vns;
            std::vector<std::pair<uint32_t, OpNfFlush>> vnf;
            std::vector<std::pair<uint32_t, OpDeferred<true>>> vdi;
            std::vector<std::pair<uint32_t, OpDeferred<false>>> vdd;
            std::vector<std::pair<uint32_t, OpPmlE<true>>> vpei;
            std::vector<std::pair<uint32_t, OpPmlE<false>>> vped;
            std::vector<std::pair<uint32_t, OpPmlH<true>>> vphi;
            std::vector<std::pair<uint32_t, OpPmlH<false>>> vphd;
            for (size_t i = 0; i < E; ++i) {
                efs_engine* e = mem[i];
                const int p = cur0[i] ^ s, q = 1 - p;
                const FusedGrid fg = e->fused_grid(p);
                const PmlSet ps = e->pml_set(p), pn = e->pml_set(q);
                // core tile descriptor
                BatchMember& M = bm[i];
                memset(&M, 0, sizeof(M));
                const uint32_t bh[4] = {TT_HZ, TT_HY, 1, 3}, be[4] = {TT_EZ, TT_EY, 1, 3};
                M.tmH = e->tensor_map(fg.H0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, bh);
                M.tmE = e->tensor_map(fg.V0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, be);
                M.tmM = e->indexed ? e->tensor_map(fg.mat, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, be) : M.tmE;
                M.tmD = e->tf.n ? e->tf_map() : M.tmE;
                M.g = fg;
                M.g.xchunk = xchunk;
                M.ps = ps;
                float* V = e->vbuf(p);
                float* V1 = e->vbuf(q);
                float* C1 = e->cbuf(q);
                StepState* st = e->state.as<StepState>();
                const MurDev md = e->mur_dev(e->vflux_ptrs[p].as<const float*>());
                if (e->mur_on) {
                    mpre.push_back({e->mur_n, OpMurPre{V, md}});
                    mpost.push_back({e->mur_n, OpMurPost{V1, md}});
                    mapply.push_back({e->mur_napply, OpMurApply{V1, md}});
                }
                if (e->exc_on && e->exc_groups) {
                    PointSources ps0{e->exc_groups, e->exc_target.as<uint32_t>(), e->exc_off.as<uint32_t>(),
                                     e->exc_delay.as<uint32_t>(), e->exc_amp.as<float>(), nullptr, e->exc_signal.as<float>(),
                                     e->exc_len, e->exc_period};
                    vexc.push_back({e->exc_groups, OpPoints<0>{V1, st, ps0}});
                }
                if (e->tfsf_on && e->tfsf_v.groups)
                    vtv.push_back({e->tfsf_v.groups, OpPoints<1>{V1, st, e->point_dev(e->tfsf_v, e->tfsf_signal, e->tfsf_len, e->tfsf_period)}});
                if (e->tfsf_on && e->tfsf_c.groups)
                    vtc.push_back({e->tfsf_c.groups, OpPoints<1>{C1, st, e->point_dev(e->tfsf_c, e->tfsf_signal, e->tfsf_len, e->tfsf_period)}});
                // ADE: one thread per group of ADE_V entries; reads the pre-update fields and the old flux
                if (e->ade_v.live())
                    vav.push_back({(e->ade_v.n + ADE_V - 1) / ADE_V, OpAde{V, e->ade_dev(e->ade_v, e->vflux_ptrs[p].as<const float*>())}});
                if (e->ade_c.live())
                    vac.push_back({(e->ade_c.n + ADE_V - 1) / ADE_V, OpAde{e->cbuf(p), e->ade_dev(e->ade_c, e->cflux_ptrs[p].as<const float*>())}});
                // ADE apply step: threads of ADE_V entries (runs form) or one per location (grouped form)
                for (int side = 0; side < 2; ++side) {
                    const efs_engine::AdeSide& as = side == 0 ? e->ade_v : e->ade_c;
                    if (!e->ade_apply || !as.live()) continue;
                    const uint32_t thr = as.app_runs ? (as.app_n + ADE_V - 1) / ADE_V : as.app_n;
                    (side == 0 ? vpv : vpc).push_back({thr, OpAdeApply{side == 0 ? V1 : C1, e->ade_apply_dev(as), as.app_runs ? 1u : 0u}});
                }
                if (e->ring_on) vring.push_back({e->ring_n, OpRing{V1, C1, st, e->ring_dev()}});
                if (e->tf_n) vtf.push_back({e->tf_n, OpTfsfFace{st, e->tf_dev()}});
                if (e->nf_on) {
                    vns.push_back({e->nf.np, OpNfSample{V1, C1, e->nf}});
                    vnf.push_back({e->nf.np, OpNfFlush{st, e->nf}});
                    any_nf = true;
                }
                if (e->defer_n) {
                    if (e->indexed) vdi.push_back({e->defer_n, OpDeferred<true>{fg, e->defer_cells.as<uint32_t>(), e->defer_n}});
                    else vdd.push_back({e->defer_n, OpDeferred<false>{fg, e->defer_cells.as<uint32_t>(), e->defer_n}});
                }
                if (e->pml_split()) {
                    const uint32_t it = e->pml_items();
                    if (e->indexed) {
                        vpei.push_back({it, OpPmlE<true>{fg, ps, pn, V, it}});
                        vphi.push_back({it, OpPmlH<true>{fg, ps, pn, it}});
                    } else {
                        vped.push_back({it, OpPmlE<false>{fg, ps, pn, V, it}});
                        vphd.push_back({it, OpPmlH<false>{fg, ps, pn, it}});
                    }
                }
            }
            upload_raw(members[s], bm.data(), bm.size() * sizeof(BatchMember));
            build_seg(mur_pre[s], mpre);
            build_seg(mur_post[s], mpost);
            build_seg(mur_apply[s], mapply);
            build_seg(exc[s], vexc);
            build_seg(tfsf_v[s], vtv);
            build_seg(tfsf_c[s], vtc);
            build_seg(ade_v[s], vav);
            build_seg(ade_c[s], vac);
            build_seg(ade_apply_v[s], vpv);
            build_seg(ade_apply_c[s], vpc);
            build_seg(ring[s], vring);
            build_seg(tfsf_face[s], vtf);
            build_seg(nf_sample[s], vns);
            build_seg(nf_flush[s], vnf);
            build_seg(deferred_i[s], vdi);
            build_seg(deferred_d[s], vdd);
            build_seg(pml_e_i[s], vpei);
            build_seg(pml_e_d[s], vped);
            build_seg(pml_h_i[s], vphi);
            build_seg(pml_h_d[s], vphd);
        }
        std::vector<std::pair<uint32_t, OpAdvance>> adv;
        for (efs_engine* e : mem) adv.push_back({1, OpAdvance{e->state.as<StepState>()}});
        build_seg(advance, adv);
        // work tiles: every member's (z tile, y tile, x chunk), largest members first
        std::vector<size_t> order(E);
        for (size_t i = 0; i < E; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return mem[a]->N > mem[b]->N; });
        std::vector<BatchTile> tl[2];
        for (size_t i : order) {
            const efs_engine* e = mem[i];
            for (uint32_t xs = 0; xs < e->Nx; xs += xchunk)
                for (uint32_t y0 = 0; y0 < e->Ny; y0 += TT_Y)
                    for (uint32_t z0 = 0; z0 < e->Nz; z0 += TT_Z) tl[e->indexed].push_back(BatchTile{(uint32_t)i, xs, y0, z0});
        }
        for (int t = 0; t < 2; ++t) {
            ntiles[t] = (uint32_t)tl[t].size();
            upload_raw(tiles[t], tl[t].data(), tl[t].size() * sizeof(BatchTile));
        }
        ck(cudaStreamSynchronize(stream), "batch plan upload");
        planned = true;
    }

    // Timestep k of a captured batch at step phase s: the single engine's phase order, each phase for all members.
    // marks: optional EFS_PHASES + 1 phase-boundary events (efs_batch_time_phases).
    void enqueue_step(uint32_t k, int s, bool last, cudaEvent_t* marks = nullptr) {
        auto mark = [&](int i) { if (marks) ck(cudaEventRecord(marks[i], stream), "phase mark"); };
        mark(0);
        launch_seg<OpPmlE<true>>(pml_e_i[s], k);  // UPML E (the pre-update reads of UPML cells are redirected
        launch_seg<OpPmlE<false>>(pml_e_d[s], k); // to the old flux, which this pass does not write)
        mark(1);
        launch_seg<OpAde>(ade_v[s], k);          // pre-voltage, as the single engine: ADE(volt), Mur pre
        launch_seg<OpMurPre>(mur_pre[s], k);
        launch_seg<OpAde>(ade_c[s], k);          // ADE(curr) before the core update rewrites H and the flux
        launch_seg<OpTfsfFace>(tfsf_face[s], k); // TFSF face values the core update adds
        mark(2);
        const BatchMember* bm = members[s].as<BatchMember>();
        if (ntiles[1])
            k_fused_tma_batch<true><<<std::min<uint32_t>(ntiles[1], ctas_per_sm * sms), TT_THREADS, TT_SMEM_BYTES, stream>>>(
                bm, tiles[1].as<BatchTile>(), ntiles[1]);
        if (ntiles[0])
            k_fused_tma_batch<false><<<std::min<uint32_t>(ntiles[0], ctas_per_sm * sms), TT_THREADS, TT_SMEM_BYTES, stream>>>(
                bm, tiles[0].as<BatchTile>(), ntiles[0]);
        mark(3);
        launch_seg<OpPoints<1>>(tfsf_v[s], k);
        launch_seg<OpMurPost>(mur_post[s], k);
        launch_seg<OpPoints<0>>(exc[s], k);
        launch_seg<OpMurApply>(mur_apply[s], k);
        launch_seg<OpAdeApply>(ade_apply_v[s], k);
        mark(4);
        launch_seg<OpPmlH<true>>(pml_h_i[s], k);       // UPML H after the E-side operations (no deferred
        launch_seg<OpPmlH<false>>(pml_h_d[s], k);      // cell is a UPML cell)
        launch_seg<OpDeferred<true>>(deferred_i[s], k);
        launch_seg<OpDeferred<false>>(deferred_d[s], k);
        mark(5);
        launch_seg<OpPoints<1>>(tfsf_c[s], k);
        launch_seg<OpAdeApply>(ade_apply_c[s], k);
        mark(6);
        if (any_nf) {
            const uint32_t j = k % NF_K;
            launch_seg<OpNfSample>(nf_sample[s], k, j);
            if (j == NF_K - 1 || last) launch_seg<OpNfFlush>(nf_flush[s], k, k - j, j + 1);
        }
        launch_seg<OpRing>(ring[s], k);
        mark(7);
    }
    // `steps` (<= 64) timesteps launched one kernel at a time with phase marks;
    // accumulates device ms per phase into ms[EFS_PHASES] (same results as iterate).
    void run_marked(uint32_t steps, float* ms) {
        if (stale()) plan();
        for (size_t i = 0; i < mem.size(); ++i) {
            ck(cudaEventRecord(ev_in[i], mem[i]->stream), "event");
            ck(cudaStreamWaitEvent(stream, ev_in[i], 0), "wait");
        }
        std::vector<cudaEvent_t> ev((size_t)steps * (EFS_PHASES + 1));
        for (auto& x : ev) ck(cudaEventCreate(&x), "event");
        try {
            for (uint32_t k = 0; k < steps; ++k)
                enqueue_step(k, (int)((phase + k) & 1), k + 1 == steps, ev.data() + (size_t)k * (EFS_PHASES + 1));
            launch_seg<OpAdvance>(advance, 0, steps);
            ck(cudaGetLastError(), "batch phase run");
            ck(cudaStreamSynchronize(stream), "batch phase run");
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
        for (efs_engine* e : mem) {
            e->numTS += steps;
            if (steps & 1) e->cur ^= 1;
        }
        if (steps & 1) phase ^= 1;
        ck(cudaEventRecord(ev_done, stream), "event");
        for (efs_engine* e : mem) ck(cudaStreamWaitEvent(e->stream, ev_done, 0), "wait");
    }

    cudaGraphExec_t graph_for(uint32_t m) {
        const uint32_t key = m * 2 + phase;
        auto it = graphs.find(key);
        if (it != graphs.end()) return it->second;
        if (graphs.size() > 12) drop_graphs();
        cudaGraph_t graph;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "BeginCapture");
        try {
            for (uint32_t k = 0; k < m; ++k) enqueue_step(k, (int)((phase + k) & 1), k + 1 == m);
            launch_seg<OpAdvance>(advance, 0, m);
        } catch (...) {
            cudaStreamEndCapture(stream, &graph);
            throw;
        }
        ck(cudaStreamEndCapture(stream, &graph), "EndCapture");
        cudaGraphExec_t ge;
        const cudaError_t err = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        ck(err, "cudaGraphInstantiate");
        graphs[key] = ge;
        return ge;
    }

    // Members stepped or reconfigured outside the batch since the plan: re-plan.
    bool stale() const {
        if (!planned) return true;
        for (size_t i = 0; i < mem.size(); ++i)
            if (mem[i]->plan_dirty || mem[i]->cur != (cur0[i] ^ (int)phase)) return true;
        return false;
    }

    void iterate(uint32_t n) {
        if (stale()) plan();
        for (size_t i = 0; i < mem.size(); ++i) {
            ck(cudaEventRecord(ev_in[i], mem[i]->stream), "event");
            ck(cudaStreamWaitEvent(stream, ev_in[i], 0), "wait");
        }
        const uint32_t CH = 64;
        while (n > 0) {
            const uint32_t m = std::min(n, CH);
            ck(cudaGraphLaunch(graph_for(m), stream), "cudaGraphLaunch");
            for (efs_engine* e : mem) {
                e->numTS += m;
                if (m & 1) e->cur ^= 1;
            }
            if (m & 1) phase ^= 1;
            n -= m;
        }
        ck(cudaGetLastError(), "batch iterate");
        ck(cudaEventRecord(ev_done, stream), "event");
        for (efs_engine* e : mem) ck(cudaStreamWaitEvent(e->stream, ev_done, 0), "wait");
    }

    void sync() {
        ck(cudaStreamSynchronize(stream), "batch sync");
        for (efs_engine* e : mem) e->sync("batch member sync");
    }
};

namespace {
template <class F>
efs_status bguard(efs_batch* b, F&& f) {
    if (!b) return EFS_ERR_INVALID;
    try {
        ck(cudaSetDevice(b->device), "cudaSetDevice");
        f();
        return EFS_OK;
    } catch (const EfsError& err) {
        b->last_error = err.msg;
        return err.code;
    } catch (const std::exception& ex) {
        b->last_error = ex.what();
        return EFS_ERR_OOM;
    }
}
}  // namespace

extern "C" {

efs_status efs_batch_create(efs_batch** out, efs_engine* const* engines, uint32_t count) {
    if (!out) return EFS_ERR_INVALID;
    *out = nullptr;
    if (!engines || count == 0) { g_create_error = "a batch needs at least one engine"; return EFS_ERR_INVALID; }
    auto* b = new efs_batch();
    try {
        for (uint32_t i = 0; i < count; ++i) {
            if (!engines[i]) fail(EFS_ERR_INVALID, "null engine in batch");
            for (uint32_t j = 0; j < i; ++j)
                if (engines[j] == engines[i]) fail(EFS_ERR_INVALID, "an engine appears twice in the batch");
            b->mem.push_back(engines[i]);
        }
        b->device = b->mem[0]->device;
        ck(cudaSetDevice(b->device), "cudaSetDevice");
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "SM count");
        b->sms = (uint32_t)sms;
        ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        b->ev_in.resize(count, nullptr);
        for (auto& ev : b->ev_in) ck(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        ck(cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming), "cudaEventCreate");
        static bool attr = false;              // the persistent kernels' dynamic shared memory, once per process
        if (!attr) {
            ck(cudaFuncSetAttribute(k_fused_tma_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT_SMEM_BYTES),
               "smem attr");
            ck(cudaFuncSetAttribute(k_fused_tma_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT_SMEM_BYTES),
               "smem attr");
            attr = true;
        }
        b->check_members();
    } catch (const EfsError& ex) {
        g_create_error = ex.msg;
        delete b;
        return ex.code;
    }
    *out = b;
    return EFS_OK;
}

efs_status efs_batch_destroy(efs_batch* b) {
    if (!b) return EFS_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    return EFS_OK;
}

const char* efs_batch_last_error(const efs_batch* b) { return b ? b->last_error.c_str() : g_create_error.c_str(); }

efs_status efs_batch_iterate(efs_batch* b, uint32_t n) { return bguard(b, [&] { b->iterate(n); }); }

efs_status efs_batch_sync(efs_batch* b) { return bguard(b, [&] { b->sync(); }); }

efs_status efs_batch_set_shape(efs_batch* b, uint32_t xchunk, uint32_t ctas_per_sm) {
    return bguard(b, [&] {
        if (xchunk == 0 || ctas_per_sm == 0 || ctas_per_sm > 2) fail(EFS_ERR_INVALID, "xchunk > 0 and ctas_per_sm in 1..2");
        if (xchunk != b->xchunk) b->planned = false;    // tiles depend on the plane depth
        b->xchunk = xchunk;
        if (ctas_per_sm != b->ctas_per_sm) b->drop_graphs();
        b->ctas_per_sm = ctas_per_sm;
    });
}

efs_status efs_batch_time_phases(efs_batch* b, uint32_t steps, float* ms) {
    return bguard(b, [&] {
        if (!ms || steps == 0 || steps > 64) fail(EFS_ERR_INVALID, "ms must be non-null and steps in 1..64");
        for (int i = 0; i < EFS_PHASES; ++i) ms[i] = 0.f;
        b->run_marked(steps, ms);
        for (int i = 0; i < EFS_PHASES; ++i) ms[i] /= (float)steps;
    });
}

efs_status efs_batch_autotune(efs_batch* b, uint32_t steps, uint32_t* xchunk, uint32_t* ctas_per_sm, float* ms_per_step) {
    return bguard(b, [&] {
        if (steps == 0) fail(EFS_ERR_INVALID, "steps must be > 0");
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        float best = 1e30f;
        uint32_t bx = b->xchunk, bc = b->ctas_per_sm;
        try {
            b->iterate(steps);                           // warm the plan, graphs and caches once
            for (uint32_t c : {2u, 1u})
                for (uint32_t x : {8u, 16u, 32u, 64u}) {
                    if (x != b->xchunk) b->planned = false;
                    if (c != b->ctas_per_sm) b->drop_graphs();
                    b->xchunk = x;
                    b->ctas_per_sm = c;
                    b->iterate(steps);                   // plan + capture outside the timed run
                    ck(cudaEventRecord(e0, b->stream), "record");
                    b->iterate(steps);
                    ck(cudaEventRecord(e1, b->stream), "record");
                    ck(cudaEventSynchronize(e1), "sync");
                    float t = 0;
                    ck(cudaEventElapsedTime(&t, e0, e1), "elapsed");
                    if (t < best) { best = t; bx = x; bc = c; }
                }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (bx != b->xchunk) b->planned = false;
        if (bc != b->ctas_per_sm) b->drop_graphs();
        b->xchunk = bx;
        b->ctas_per_sm = bc;
        if (xchunk) *xchunk = bx;
        if (ctas_per_sm) *ctas_per_sm = bc;
        if (ms_per_step) *ms_per_step = best / steps;
        b->sync();
    });
}

}  // extern "C"
