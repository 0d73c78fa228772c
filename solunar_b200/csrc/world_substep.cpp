// world_substep.cpp -- World's substeps, solves as CUDA graphs and the whole substep as one graph.
#include "world.h"

namespace slf {

int32_t World::wcsph_substep(float dt, uint32_t& held) {
    Params p = params();
    int a = (cpos + 1) % 3, b = (cpos + 2) % 3;
    int nid = 1 - cid;
    bool whole = whole_substeps();
    SortPlan sp;
    SLF_TRY(plan_sort(sp, whole));
    if (whole) SLF_TRY(substep_graph(dt, p, a, b, nid, sp, whole));
    if (!whole) {
        SLF_TRY(enqueue_sort(a, sp, stream));
        SLF_TRY(reset_status());
        launch_set_consts(consts(dt), d_consts, stream);
        PairLists fl = fluid_lists(), wl = wall_lists();
        timed("density", bytes_per_particle::density_wcsph,
              [&] { density_pass(p, a, fl, wl, rho[nid].p); });
        timed("wcsph_force_advance", bytes_per_particle::wcsph_force,
              [&] { force_pass(p, fl, wl, a, b, nid); });
    }
    SLF_TRY(read_status());
    SLF_TRY(lists_fit());
    SLF_TRY(check_state());
    SLF_TRY(mover_felt(dt, p, a, nid));
    held = h_status->held;
    cpos = b;
    cid = nid;
    lists_pos = a;
    lists_n = n;
    lists_valid = true;
    stats_fresh = true;  // the force pass folded the new state's box and speed
    return SLF_OK;
}

int32_t World::solve(int which, const Params& p, int a, float4* v, int nid, uint32_t& iterations, SolveRec rec) {
    iterations = 0;
    PairLists fl = fluid_lists(), wl = wall_lists();
    // (a graph's loop body needs launches: no particles, no graph)
    if (p.n && graphs_for(rec)) return solve_graph(which, p, a, v, nid, fl, wl, rec, iterations);
    SLF_CUDA(cudaMemsetAsync(&d_status->settled, 0, 4, stream));
    SLF_CUDA(cudaMemsetAsync(&d_status->iterations, 0, 4, stream));
    const char* rate_name = which == 0 ? "rate_divergence" : "rate_density";
    const char* push_name = which == 0 ? "push_divergence" : "push_density";
    double rate_bytes = which == 0 ? bytes_per_particle::rate_divergence : bytes_per_particle::rate_density;
    // warm start: one push at half the stiffness impulse the particle's last solve of this
    // kind applied; the pushes then add theirs to it, for the next substep
    float* applied = nullptr;
    if (warm_on()) {
        applied = reinterpret_cast<float*>(warm[nid].p) + which;
        timed("warm_push", bytes_per_particle::push, [&] {
            launch_warm_kappa(p, d_consts, 0.5f, applied, pos[a].p, stream);
            push_pass(p, fl, wl, a, v);
        });
    }
    size_t first = prof.pending.size();
    std::vector<int> kinds;  // 0 rate, 1 push, in launch order, for the profile
    uint32_t batch = std::max<uint32_t>(expected_iterations[which], 1u);
    uint32_t queued = 0;
    auto rate = [&] {
        timed(rate_name, rate_bytes, [&] { rate_pass(which, p, fl, wl, a, v, nid, rec); });
        kinds.push_back(0);
    };
    // check, then (push, check) pairs: the order of the reference's loop
    rate();
    for (;;) {
        for (uint32_t b = 0; b < batch; ++b) {
            timed(push_name, bytes_per_particle::push, [&] { push_pass(p, fl, wl, a, v, applied); });
            kinds.push_back(1);
            rate();
        }
        queued += batch;
        // profile entries of launches that turned out idle are kept apart
        size_t mark = prof.pending.size();
        SLF_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(Status), cudaMemcpyDeviceToHost, stream));
        SLF_CUDA(cudaStreamSynchronize(stream));
        if (h_status->settled) {
            iterations = h_status->iterations;
            if (prof.on && mark == prof.pending.size()) relabel_idle(first, kinds, iterations);
            SLF_TRY(sync());
            SLF_TRY(lists_fit());
            expected_iterations[which] = std::max<uint32_t>(iterations, 1u);
            return SLF_OK;
        }
        SLF_TRY(lists_fit());
        // the device stops at max_iterations; past that its flag was not written
        if (queued > s.max_iterations + 1) return fail(SLF_ERR_TIMEOUT, "solver stop flag never set");
        batch = std::max<uint32_t>(4u, batch / 2);
    }
}

void World::drop_solve_graphs() {
    for (auto& g : solve_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    solve_graphs.clear();
}

void World::key_lists(std::vector<uint8_t>& k, const PairLists& l) {
    key_add(k, l.cap);
    key_add(k, l.e);
    key_add(k, l.count);
    key_add(k, l.order);
    key_add(k, l.gv);
}

std::vector<uint8_t> World::solve_key(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                                      const PairLists& wl, const SolveRec& rec) {
    static_assert(sizeof(Params) % 4 == 0, "Params holds 4-byte fields only");
    std::vector<uint8_t> k;
    key_add(k, which);
    key_add(k, int32_t(fast()));
    key_add(k, int32_t(rel()));
    key_add(k, int32_t(warm_on()));
    key_add(k, p);
    key_lists(k, fl);
    key_lists(k, wl);
    for (const void* q : {(const void*)pos[a].p, (const void*)v, (const void*)rho[nid].p, (const void*)alpha.p,
                          (const void*)dwalls.p, (const void*)partials.p, (const void*)d_status,
                          (const void*)d_consts, (const void*)(warm_on() ? warm[nid].p : nullptr),
                          (const void*)rec.rate, (const void*)rec.vel})
        key_add(k, q);
    return k;
}

int32_t World::capture_solve(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                             const PairLists& wl, const SolveRec& rec, uint32_t& pre) {
    cudaStream_t cs = cap[0];
    SLF_CUDA(cudaMemsetAsync(&d_status->settled, 0, 4, cs));
    SLF_CUDA(cudaMemsetAsync(&d_status->iterations, 0, 4, cs));
    SLF_CUDA(cudaMemsetAsync(&d_status->bodies, 0, 4, cs));
    SLF_CUDA(cudaMemsetAsync(&d_status->ticket, 0, 4, cs));
    float* applied = nullptr;
    if (warm_on()) {
        applied = reinterpret_cast<float*>(warm[nid].p) + which;
        launch_warm_kappa(p, d_consts, 0.5f, applied, pos[a].p, cs);
        push_pass(p, fl, wl, a, v, nullptr, cs);
        pre += 2;
    }
    cudaStreamCaptureStatus cst;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    SLF_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps));
    cudaGraphConditionalHandle loop;
    SLF_CUDA(cudaGraphConditionalHandleCreate(&loop, graph, 1u, cudaGraphCondAssignDefault));
    rate_pass(which, p, fl, wl, a, v, nid, rec, cs, loop);
    pre += 1;
    SLF_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &graph, &deps, &ndeps));
    // the node parameters are a union without a default constructor: zeroed raw storage
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof raw);
    cudaGraphNodeParams& np = *reinterpret_cast<cudaGraphNodeParams*>(raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = loop;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    SLF_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &np));
    SLF_CUDA(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    SLF_CUDA(cudaStreamBeginCaptureToGraph(cap[1], body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    push_pass(p, fl, wl, a, v, applied, cap[1], loop);
    rate_pass(which, p, fl, wl, a, v, nid, rec, cap[1], loop);
    cudaGraph_t done = nullptr;
    SLF_CUDA(cudaStreamEndCapture(cap[1], &done));
    return SLF_OK;
}

int32_t World::solve_graph(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                           const PairLists& wl, const SolveRec& rec, uint32_t& iterations) {
    std::vector<uint8_t> key = solve_key(which, p, a, v, nid, fl, wl, rec);
    SolveGraph* hit = nullptr;
    for (auto& g : solve_graphs)
        if (g.key == key) hit = &g;
    if (!hit) {
        for (auto& c : cap)
            if (!c) SLF_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
        SolveGraph g;
        g.key = std::move(key);
        uint64_t before = kernel_launches();
        SLF_CUDA(cudaStreamBeginCapture(cap[0], cudaStreamCaptureModeThreadLocal));
        int32_t st = capture_solve(which, p, a, v, nid, fl, wl, rec, g.pre);
        cudaGraph_t graph = nullptr;
        cudaError_t ended = cudaStreamEndCapture(cap[0], &graph);
        // launches recorded into the graph ran nothing yet; they count when it runs
        note_launches(-int64_t(kernel_launches() - before));
        if (st != SLF_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        SLF_CUDA(ended);
        cudaError_t made = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        SLF_CUDA(made);
        if (solve_graphs.size() >= kSolveGraphCache) {
            auto old = std::min_element(solve_graphs.begin(), solve_graphs.end(),
                                        [](const SolveGraph& x, const SolveGraph& y) { return x.used < y.used; });
            cudaGraphExecDestroy(old->exec);
            solve_graphs.erase(old);
        }
        solve_graphs.push_back(std::move(g));
        hit = &solve_graphs.back();
    }
    hit->used = ++graph_clock;
    SLF_CUDA(cudaGraphLaunch(hit->exec, stream));
    note_launches(hit->pre);
    graph_solves |= 1u << which;
    if (!rec.rate) return SLF_OK;
    SLF_TRY(read_status());
    uint32_t its[2] = {0, 0};
    SLF_TRY(finish_graph_solves(its));
    iterations = its[which];
    return SLF_OK;
}

bool World::whole_substeps() const {
    // (the adjoint's recomputed substeps, which redirect the sort and record velocities, launch
    // eagerly)
    return graph_mode >= 2 && !prof.on && s.max_iterations <= kGraphMaxIterations && skip_job < 0 &&
           terrains.empty() && m_pos.empty() && n > 0 && !sort_dest && !vel_pre;
}

void World::drop_substep_graphs() {
    for (auto& g : substep_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    substep_graphs.clear();
    substep_seen.clear();
    unused_graphs = 0;
}

std::vector<uint8_t> World::substep_key(const Params& p, int a, int b, int nid, const SortPlan& sp) {
    static_assert(sizeof(GridDev) == 48, "GridDev has no padding");
    std::vector<uint8_t> k;
    key_add(k, int32_t(s.solver));
    key_add(k, int32_t(fast()));
    key_add(k, int32_t(rel()));
    key_add(k, int32_t(warm_on()));
    key_add(k, p);
    key_add(k, sp.lo);
    key_add(k, sp.span);
    key_add(k, sp.volume);
    key_add(k, sp.keys);
    key_add(k, sp.job_lo);
    key_add(k, sp.job_hi);
    key_add(k, fgrid);
    key_add(k, wgrid);
    key_lists(k, fluid_lists());
    key_lists(k, wall_lists());
    for (const void* q : std::initializer_list<const void*>{
             pos[cpos].p, vel[cpos].p, cells_of(cpos), ids[cid].p, ids[nid].p, rho[cid].p, rho[nid].p,
             pos[a].p, vel[a].p, cells_of(a), pos[b].p, vel[b].p, cells_of(b), warm_in(), warm_out(),
             sort_dest, count.p, tiles.p, lin.p, cslot.p, members.p, worder.p, wkeys.p, wsums.p, press.p,
             scaled.p, alpha.p, dwalls.p, partials.p, d_status, d_consts, vel_pre, h_reset})
        key_add(k, q);
    return k;
}

int32_t World::capture_substep(const Params& p, int a, int b, int nid, const SortPlan& sp, SubstepGraph& g) {
    for (auto& c : cap)
        if (!c) SLF_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    cudaStream_t cs = cap[0];
    uint64_t before = kernel_launches();
    SLF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    auto record = [&]() -> int32_t {
        SLF_TRY(enqueue_sort(a, sp, cs));
        SLF_CUDA(cudaMemcpyAsync(d_status, h_reset, sizeof(Status), cudaMemcpyHostToDevice, cs));
        PairLists fl = fluid_lists(), wl = wall_lists();
        density_pass(p, a, fl, wl, rho[nid].p, cs);
        if (s.solver == SLF_SOLVER_WCSPH) {
            force_pass(p, fl, wl, a, b, nid, cs);
            return SLF_OK;
        }
        uint32_t pre = 0;
        SLF_TRY(capture_solve(0, p, a, vel[a].p, nid, fl, wl, SolveRec{nullptr, nullptr}, pre));
        viscous_pass(p, fl, wl, a, b, nid, cs);
        SLF_TRY(capture_solve(1, p, a, vel[b].p, nid, fl, wl, SolveRec{nullptr, nullptr}, pre));
        advance_pass(p, a, b, vel_pre, cs);
        return SLF_OK;
    };
    int32_t st = record();
    cudaGraph_t graph = nullptr;
    cudaError_t ended = cudaStreamEndCapture(cs, &graph);
    // launches recorded into the graph ran nothing yet; they count when it runs
    int64_t recorded = int64_t(kernel_launches() - before);
    note_launches(-recorded);
    if (st != SLF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    SLF_CUDA(ended);
    cudaError_t made = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    SLF_CUDA(made);
    // each DFSPH solve's loop body (a push and a check) counts per iteration when it runs
    g.outside = uint32_t(recorded - (s.solver == SLF_SOLVER_DFSPH ? 4 : 0));
    return SLF_OK;
}

int32_t World::substep_graph(float dt, const Params& p, int a, int b, int nid, const SortPlan& sp, bool& ran) {
    ran = false;
    std::vector<uint8_t> key = substep_key(p, a, b, nid, sp);
    SubstepGraph* hit = nullptr;
    for (auto& g : substep_graphs)
        if (g.key == key) hit = &g;
    if (!hit) {
        if (unused_graphs >= kUnusedGraphs) {
            auto seen = std::find(substep_seen.begin(), substep_seen.end(), key);
            if (seen == substep_seen.end()) {
                if (substep_seen.size() >= 2 * kGraphCache) substep_seen.erase(substep_seen.begin());
                substep_seen.push_back(std::move(key));
                return SLF_OK;
            }
            substep_seen.erase(seen);
        }
        SubstepGraph g;
        g.key = std::move(key);
        SLF_TRY(capture_substep(p, a, b, nid, sp, g));
        if (substep_graphs.size() >= kGraphCache) {
            auto old = std::min_element(substep_graphs.begin(), substep_graphs.end(),
                                        [](const SubstepGraph& x, const SubstepGraph& y) { return x.used < y.used; });
            if (old->runs <= 1) ++unused_graphs;
            cudaGraphExecDestroy(old->exec);
            substep_graphs.erase(old);
        }
        substep_graphs.push_back(std::move(g));
        hit = &substep_graphs.back();
    }
    hit->used = ++graph_clock;
    ++hit->runs;
    launch_set_consts(consts(dt), d_consts, stream);
    SLF_CUDA(cudaGraphLaunch(hit->exec, stream));
    note_launches(hit->outside);
    graph_solves = s.solver == SLF_SOLVER_DFSPH ? 3u : 0u;
    ++graph_substeps;
    ran = true;
    return SLF_OK;
}

int32_t World::finish_graph_solves(uint32_t its[2]) {
    uint32_t ran = graph_solves;
    graph_solves = 0;
    if (h_status->overrun) return fail(SLF_ERR_TIMEOUT, "solver loop passed max_iterations + 1 bodies");
    SLF_TRY(lists_fit());
    for (int w = 0; w < 2; ++w)
        if (ran & (1u << w)) {
            its[w] = h_status->solved[w];
            note_launches(2 * int64_t(its[w]));
            expected_iterations[w] = std::max<uint32_t>(its[w], 1u);
        }
    return SLF_OK;
}

void World::relabel_idle(size_t first, const std::vector<int>& kinds, uint32_t iterations) {
    uint32_t rates = 0, pushes = 0;
    int idle = prof.kind("solver_idle");
    for (size_t k = 0; k < kinds.size() && first + k < prof.pending.size(); ++k) {
        bool used = kinds[k] == 0 ? rates++ <= iterations : pushes++ < iterations;
        if (!used) {
            prof.pending[first + k].kind = idle;
            prof.pending[first + k].bytes = 0.0;
        }
    }
}

int32_t World::keep_record(uint32_t its, DevBuf<float>& rates, DevBuf<float4>& vels) {
    size_t m = size_t(its) * n;
    if (its > record_room) record_room = its + its / 4 + 4;
    // a record that holds this solve keeps its buffers; one that does not grows to the room
    size_t room = std::max<size_t>(size_t(record_room) * n, 1);
    if (rates.cap < std::max<size_t>(m, 1)) SLF_TRY(rates.ensure(room, 0, stream));
    if (vels.cap < std::max<size_t>(m, 1)) SLF_TRY(vels.ensure(room, 0, stream));
    if (m) {
        SLF_CUDA(cudaMemcpyAsync(rates.p, rec_rate.p, m * 4, cudaMemcpyDeviceToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(vels.p, rec_vel.p, m * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
    }
    return SLF_OK;
}

int32_t World::dfsph_substep(float dt, uint32_t& held, uint32_t& iterations, DfsphRecord* rec) {
    Params p = params();
    int a = (cpos + 1) % 3, b = (cpos + 2) % 3;
    int nid = 1 - cid;
    uint32_t div_it = 0, den_it = 0;
    bool whole = !rec && whole_substeps();
    SortPlan sp;
    SLF_TRY(plan_sort(sp, whole));
    if (whole) SLF_TRY(substep_graph(dt, p, a, b, nid, sp, whole));
    if (!whole) {
        SLF_TRY(enqueue_sort(a, sp, stream));
        if (rec && warm_on()) {  // the impulses the solves start from, which they overwrite
            SLF_TRY(rec->warm.ensure(n, 0, stream));
            SLF_CUDA(cudaMemcpyAsync(rec->warm.p, warm[nid].p, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream));
        }
        SLF_TRY(reset_status());
        graph_solves = 0;
        launch_set_consts(consts(dt), d_consts, stream);
        PairLists fl = fluid_lists(), wl = wall_lists();
        timed("density_alpha", bytes_per_particle::density_dfsph,
              [&] { density_pass(p, a, fl, wl, rho[nid].p); });
        SolveRec sr{nullptr, nullptr};
        if (rec) {
            size_t slots = (size_t(s.max_iterations) + 1) * n;
            SLF_TRY(rec_rate.ensure(slots, 0, stream));
            SLF_TRY(rec_vel.ensure(slots, 0, stream));
            sr = SolveRec{rec_rate.p, rec_vel.p};
        }
        SLF_TRY(solve(0, p, a, vel[a].p, nid, div_it, sr));
        if (rec) {
            SLF_TRY(keep_record(div_it, rec->div_rate, rec->div_vel));
            rec->div_n = div_it;
            SLF_TRY(rec->va.ensure(n, 0, stream));
            SLF_CUDA(
                cudaMemcpyAsync(rec->va.p, vel[a].p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        }
        timed("viscosity", bytes_per_particle::viscosity, [&] { viscous_pass(p, fl, wl, a, b, nid); });
        SLF_TRY(solve(1, p, a, vel[b].p, nid, den_it, sr));
        float4* pre = vel_pre;
        if (rec) {
            SLF_TRY(keep_record(den_it, rec->den_rate, rec->den_vel));
            rec->den_n = den_it;
            SLF_TRY(rec->pre.ensure(n, 0, stream));
            pre = rec->pre.p;
        }
        timed("advance", bytes_per_particle::advance, [&] { advance_pass(p, a, b, pre); });
    }
    SLF_TRY(read_status());
    if (graph_solves) {
        uint32_t its[2] = {div_it, den_it};
        SLF_TRY(finish_graph_solves(its));
        div_it = its[0];
        den_it = its[1];
    }
    SLF_TRY(check_state());
    held = h_status->held;
    iterations = div_it + den_it;
    last_iterations[0] = div_it;
    last_iterations[1] = den_it;
    cpos = b;
    cid = nid;
    lists_pos = a;
    lists_n = n;
    lists_valid = true;
    stats_fresh = true;
    return SLF_OK;
}

int32_t World::step(float dt, slf_report* out) {
    if (!tape.on) return step_untaped(dt, out);
    SLF_TRY(flush());
    if (n != tape.n || has_domain || !flows.empty())
        return fail(SLF_ERR_UNSUPPORTED, "the particles changed while a tape was recording");
    tape.steps.emplace_back();
    tape_step = &tape.steps.back();
    size_t recorded = tape.subs.size(), checkpoints = tape.ckpt_sub.size();
    int32_t st = step_untaped(dt, out);
    tape_step = nullptr;
    if (st != SLF_OK) {  // the failed step's substeps and checkpoints are forgotten
        tape.count -= tape.steps.back().size();
        tape.steps.pop_back();
        tape.ckpt_sub.resize(checkpoints);
        drop_records(recorded);
        return st;
    }
    return SLF_OK;
}

}  // namespace slf
