// Batched CLE over many networks of uneven size (scrna_cle_simulate_batch).
//
// Networks are grouped by register-path kernel variant (warp-per-cell-group kernel with
// its genes-per-lane and regulator class, or block tiles with their quads per thread) and
// by population mode.  Each group runs as ONE persistent launch whose blocks pull
// (network, cell tile, step range) items from a device work queue, largest items first,
// so small and large networks share the GPU without per-network launches.  Groups run on
// their own streams so they overlap.  Population groups advance chunk by chunk (a chunk
// ends at a division check, the division itself happens in the chunk's epilogue); the
// chunk launches of a group are captured once into a CUDA graph and replayed.
// Large dense networks go to the tensor-core path one after another.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <cmath>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "capi_internal.h"

namespace scrna {

namespace {

struct BatchNet {
    int b = 0;
    scrna_net* net = nullptr;
    const scrna_kinetics* kin = nullptr;
    const scrna_population* pop = nullptr;
    scrna_cle_opts o{};
    scrna_state* st = nullptr;
    KernelChoice kc{};
    int64_t n_steps = 0;
    bool tensor = false;
    bool tau = false;
    // this entry's gene tables and kernel arguments: one network handle may appear several
    // times in a batch with other kinetics
    DevBuf genes, ginit, qtel;
    FusedArgs args{};
};

struct GroupKey {
    int tau, warp, gpl, emax, tmax, nwarps, upt, qg, pop, interval;
    int64_t n_steps;
    bool operator<(const GroupKey& r) const {
        return std::tie(tau, warp, gpl, emax, tmax, nwarps, upt, qg, pop, interval, n_steps) <
               std::tie(r.tau, r.warp, r.gpl, r.emax, r.tmax, r.nwarps, r.upt, r.qg, r.pop, r.interval, r.n_steps);
    }
};

struct Group {
    GroupKey key{};
    std::vector<BatchNet*> nets;
    DevBuf args, items, counters;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t graph = nullptr;
    ~Group() {
        if (graph) cudaGraphExecDestroy(graph);
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
    }
};

int64_t cells_per_tile(const BatchNet& bn) {
    if (bn.kc.warp) return warpcell_cells_per_block_host(bn.net->G, bn.kc.gpl, bn.kc.nw1);
    return 32;
}

}  // namespace

int run_batch(scrna_ctx* ctx, std::vector<BatchNet*>& all, const scrna_capture* cap);

int batch_simulate(scrna_ctx* ctx, int32_t B, const scrna_net* const* nets, const scrna_kinetics* kins,
                   int32_t n_kins, const int64_t* cell_nums, const scrna_population* const* pops,
                   const scrna_capture* cap, const scrna_cle_opts* opts, double* const* outs,
                   int32_t* const* counts, bool tau) {
    std::vector<BatchNet> bn(B);
    std::vector<std::unique_ptr<scrna_state, int (*)(scrna_state*)>> owned;
    for (int b = 0; b < B; ++b) {
        BatchNet& x = bn[b];
        x.b = b;
        x.tau = tau;
        x.net = const_cast<scrna_net*>(nets[b]);
        x.kin = &kins[n_kins == 1 ? 0 : b];
        x.pop = pops ? pops[b] : nullptr;
        x.o = *opts;
        x.o.stream = (opts->stream + (uint32_t)b) & 0xFFFFFFu;
        if (!x.pop) {
            if (!cell_nums) return fail(SCRNA_EINVAL, "cell_nums is NULL");
            x.o.cell_num = cell_nums[b];
        }
        if (!x.net) return fail(SCRNA_EINVAL, "network %d is NULL", b);
        if (int r = validate_run(x.net, x.kin, x.pop, cap, &x.o)) return r;
        const int64_t N = x.pop ? x.pop->cell_num : x.o.cell_num;
        if (N <= 0) return fail(SCRNA_EINVAL, "network %d has no cells", b);
        if (x.o.cell_offset < 0 || x.o.cell_offset + N > (1ll << 32)) return fail(SCRNA_EINVAL, "cell indices must fit 32 bits");
        x.n_steps = n_steps_of(&x.o);
        if (x.n_steps >= (1ll << 31)) return fail(SCRNA_EINVAL, "too many steps");
        scrna_state* st = nullptr;
        if (int r = scrna_state_create(ctx, x.net, N, x.o.readout, cap != nullptr, &st)) return r;
        owned.emplace_back(st, scrna_state_destroy);
        x.st = st;
        const NetDev& d = x.net->dev;
        x.tensor = auto_tensor(x.net, tau, N);
        if (!x.tensor) {
            if (int r = state_alloc(st, x.pop != nullptr, false)) return r;
            const int G = x.net->G, nq = (G + 3) / 4;
            std::vector<GeneRec> gr(G);
            std::vector<GeneInit> gi(G);
            std::vector<uint8_t> qt(nq);
            gene_tables_host(x.net, x.kin, x.o.dt, gr.data(), gi.data(), qt.data());
            CU(x.genes.ensure(G * sizeof(GeneRec)));
            CU(x.ginit.ensure(G * sizeof(GeneInit)));
            CU(x.qtel.ensure(nq));
            CU(cudaMemcpy(x.genes.p, gr.data(), G * sizeof(GeneRec), cudaMemcpyHostToDevice));
            CU(cudaMemcpy(x.ginit.p, gi.data(), G * sizeof(GeneInit), cudaMemcpyHostToDevice));
            CU(cudaMemcpy(x.qtel.p, qt.data(), nq, cudaMemcpyHostToDevice));
            ctx->h2d_bytes += (int64_t)(G * (sizeof(GeneRec) + sizeof(GeneInit)) + nq);
            fill_fused_args(x.net, x.kin, x.pop, cap, &x.o, st, &x.args);
            x.args.genes = x.genes.as<GeneRec>();
            x.args.ginit = x.ginit.as<GeneInit>();
            x.args.quad_tel = x.qtel.as<uint8_t>();
            if (tau) {
                fill_tau_args(x.net, x.kin, x.pop, &x.o, &x.args);
                x.kc = choose_kernel(x.net, SCRNA_PATH_BLOCK);
                x.kc.block = tau_plan(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src,
                                      tau_genes_per_unit(d.G, d.n_reg, d.n_in, d.n_na, d.n_na_src, st->N));
                x.kc.smem = x.kc.block.smem;
            } else if (int r = choose_kernel_tuned(ctx, x.net, x.kin, &x.o, st, &x.kc, &x.args, nullptr)) {
                return r;
            }
            x.args.lane_nw1 = x.kc.nw1;
            if (x.kc.smem > kMaxDynamicSmem) return fail(SCRNA_ENOTSUP, "network %d needs too much shared memory", b);
            x.st->have_counts = cap != nullptr;
        }
    }
    std::vector<BatchNet*> ptrs;
    for (auto& x : bn) ptrs.push_back(&x);
    if (int r = run_batch(ctx, ptrs, cap)) return r;
    for (int b = 0; b < B; ++b)
        if (int r = scrna_state_read(ctx, bn[b].st, outs[b], (cap && counts) ? counts[b] : nullptr, nullptr)) return r;
    return SCRNA_OK;
}

int run_batch(scrna_ctx* ctx, std::vector<BatchNet*>& all, const scrna_capture* cap) {
    // tensor-path networks: their tables first (the first preparation of a network waits for
    // the device), so that their runs below overlap the register-path groups
    for (BatchNet* x : all)
        if (x->tensor) {
            if (int r = ensure_gene_tables(x->net, x->kin, x->o.dt, x->pop != nullptr)) return r;
            if (int r = tensor_prepare_net(x->net, 0)) return r;
        }
    // register-path networks: one persistent launch (or one captured chunk sequence) per group
    std::map<GroupKey, std::unique_ptr<Group>> groups;
    for (BatchNet* x : all) {
        if (x->tensor) continue;
        GroupKey k{};
        k.tau = x->tau;
        k.warp = x->kc.warp;
        k.gpl = x->kc.warp ? x->kc.gpl : 0;
        k.emax = x->kc.warp ? x->kc.emax : 0;
        k.tmax = x->kc.warp ? x->kc.tmax : 0;
        k.nwarps = x->kc.warp ? x->kc.nwarps : 0;
        k.upt = x->kc.warp ? 0 : x->kc.block.upt;
        k.qg = x->kc.warp ? 0 : x->kc.block.qg;
        k.pop = x->pop != nullptr;
        k.interval = x->pop ? x->pop->div_check_interval : 0;
        k.n_steps = x->pop ? x->n_steps : 0;
        auto& g = groups[k];
        if (!g) { g.reset(new Group()); g->key = k; }
        g->nets.push_back(x);
    }
    cudaEvent_t start;
    CU(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    CU(cudaEventRecord(start, ctx->stream));
    for (auto& kv : groups) {
        Group& g = *kv.second;
        const GroupKey& k = g.key;
        CU(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        CU(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
        CU(cudaStreamWaitEvent(g.stream, start, 0));
        // kernel arguments of every network of the group, and its work items
        std::vector<FusedArgs> args(g.nets.size());
        std::vector<TileWork> items;
        int nw = 1;
        size_t smem = 0;
        for (size_t i = 0; i < g.nets.size(); ++i) {
            BatchNet* x = g.nets[i];
            args[i] = x->args;
            nw = std::max(nw, x->kc.block.nw);
            smem = std::max(smem, x->kc.smem);
            const int64_t cpt = cells_per_tile(*x);
            const int64_t tiles = (x->st->N + cpt - 1) / cpt;
            for (int64_t t = 0; t < tiles; ++t) {
                TileWork w{};
                w.arg = (int32_t)i;
                w.tile = (int32_t)t;
                w.ctl = TileCtl{1, (int32_t)x->n_steps, 1, 1, 0, 0};
                items.push_back(w);
            }
            if (x->pop)
                for (int q = 0; q < 2; ++q) CU(cudaMemsetAsync(x->st->owner[q].p, 0, (size_t)x->st->N * 8, g.stream));
        }
        // longest items first: cost ~ genes x steps of the item's network
        std::stable_sort(items.begin(), items.end(), [&](const TileWork& a, const TileWork& b) {
            const BatchNet* xa = g.nets[a.arg];
            const BatchNet* xb = g.nets[b.arg];
            return (double)xa->net->G * xa->n_steps > (double)xb->net->G * xb->n_steps;
        });
        CU(g.args.ensure(args.size() * sizeof(FusedArgs)));
        CU(g.items.ensure(items.size() * sizeof(TileWork)));
        CU(cudaMemcpyAsync(g.args.p, args.data(), args.size() * sizeof(FusedArgs), cudaMemcpyHostToDevice, g.stream));
        CU(cudaMemcpyAsync(g.items.p, items.data(), items.size() * sizeof(TileWork), cudaMemcpyHostToDevice, g.stream));
        const int n_items = (int)items.size();
        const int grid = std::max(1, std::min(n_items, ctx->sm_count * (k.warp ? std::max(1, 24 / k.nwarps) : 8)));
        // one seed for the whole call: the lane kernel reads the round keys from its parameters
        KeySchedule ks{};
        bool same_key = !args.empty();
        for (const FusedArgs& fa : args) same_key = same_key && fa.key0 == args[0].key0 && fa.key1 == args[0].key1;
        if (same_key) {
            std::memcpy(ks.rk0, args[0].rk0, sizeof ks.rk0);
            std::memcpy(ks.rk1, args[0].rk1, sizeof ks.rk1);
        }
        auto launch = [&](int* counter, TileCtl ctl, int use_shared) -> cudaError_t {
            if (k.tau)
                return tau_queue_launch(g.args.as<FusedArgs>(), g.items.as<TileWork>(), n_items, counter, k.upt, nw,
                                        smem, k.pop != 0, grid, ctl, use_shared, k.qg, g.stream);
            if (k.warp)
                return warpcell_queue_launch(g.args.as<FusedArgs>(), g.items.as<TileWork>(), n_items, counter, k.gpl,
                                             k.emax, k.tmax, k.pop != 0, smem, grid, k.nwarps, ctl, use_shared,
                                             same_key ? &ks : nullptr, g.stream);
            return fused_queue_launch(g.args.as<FusedArgs>(), g.items.as<TileWork>(), n_items, counter, k.upt, nw,
                                      smem, k.pop != 0, grid, ctl, use_shared, g.stream);
        };
        if (!k.pop) {
            CU(g.counters.ensure(sizeof(int)));
            CU(cudaMemsetAsync(g.counters.p, 0, sizeof(int), g.stream));
            CU(launch(g.counters.as<int>(), TileCtl{}, 0));
            ctx->launches++;
        } else {
            // chunk schedule shared by every network of the group
            std::vector<TileCtl> chunks;
            const int64_t I = k.interval, n_steps = k.n_steps;
            int64_t s0 = 1;
            int epoch = 0;
            bool first = true;
            while (true) {
                const int64_t s1 = n_steps == 0 ? 0 : std::min(n_steps, ((s0 - 1) / I + 1) * I);
                const bool check = s1 >= s0 && (s1 % I == 0);
                const bool final_chunk = s1 >= n_steps;
                chunks.push_back(TileCtl{(int32_t)s0, (int32_t)s1, first ? 1 : 0, (final_chunk && !check) ? 1 : 0,
                                         check ? 1 : 0, epoch});
                first = false;
                if (check) epoch += 1;
                if (final_chunk) {
                    if (check) chunks.push_back(TileCtl{(int32_t)s1 + 1, (int32_t)s1, 0, 1, 0, epoch});
                    break;
                }
                s0 = s1 + 1;
            }
            CU(g.counters.ensure(chunks.size() * sizeof(int)));
            CU(cudaMemsetAsync(g.counters.p, 0, chunks.size() * sizeof(int), g.stream));
            // capture the chunk launches once and replay them as one graph
            cudaGraph_t graph;
            CU(cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeRelaxed));
            cudaError_t le = cudaSuccess;
            for (size_t c = 0; c < chunks.size() && le == cudaSuccess; ++c)
                le = launch(g.counters.as<int>() + c, chunks[c], 1);
            cudaError_t ce = cudaStreamEndCapture(g.stream, &graph);
            if (le != cudaSuccess) { if (ce == cudaSuccess) cudaGraphDestroy(graph); CU(le); }
            CU(ce);
            cudaError_t ie = cudaGraphInstantiate(&g.graph, graph, 0);
            cudaGraphDestroy(graph);
            CU(ie);
            CU(cudaGraphLaunch(g.graph, g.stream));
            ctx->launches += (int64_t)chunks.size();
        }
        CU(cudaEventRecord(g.done, g.stream));
    }
    // tensor-path networks, one after another on the context stream while the groups run
    for (BatchNet* x : all)
        if (x->tensor) {  // the fused tcgen05 kernel (gene-major state); beyond its gene limit the library GEMM
            // the tau-leap and populations: library-GEMM variant only
            const bool fused = !x->tau && !x->pop && x->net->G <= 4096;
            x->st->last_tensor = !fused;
            x->st->last_plain = false;
            x->st->last_pop = x->pop != nullptr;
            x->st->last_tau = x->tau;
            x->st->have_counts = cap != nullptr;
            if (int r = fused ? tc_run(ctx, x->net, x->kin, cap, &x->o, x->st, 0)
                              : tensor_run(ctx, x->net, x->kin, cap, &x->o, x->st, 0, x->tau, x->pop))
                return r;
        }
    for (auto& kv : groups) CU(cudaStreamWaitEvent(ctx->stream, kv.second->done, 0));
    CU(cudaStreamSynchronize(ctx->stream));
    cudaEventDestroy(start);
    return SCRNA_OK;
}

}  // namespace scrna
