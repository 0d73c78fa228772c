// world_adjoint.cpp -- World's the tape of slf_tape_begin and the adjoint (slf_step_backward).
#include "world.h"

namespace slf {

auto World::new_record() -> std::unique_ptr<SubRecord> {
    if (spare_records.empty()) return std::make_unique<SubRecord>();
    auto r = std::move(spare_records.back());
    spare_records.pop_back();
    r->kept = false;
    return r;
}

int32_t World::reserve_kept(SubRecord& sub) {
    const size_t slots = PairLists::slots_for(uint32_t(n), list_cap);
    for (auto* b : {&sub.pos, &sub.vel, &sub.spos, &sub.svel, &sub.pre}) SLF_TRY(b->ensure(n, 0, stream));
    for (auto* b : {&sub.rho, &sub.press, &sub.scaled}) SLF_TRY(b->ensure(n, 0, stream));
    for (auto* b : {&sub.ids, &sub.dest, &sub.order, &sub.fcnt, &sub.wcnt}) SLF_TRY(b->ensure(n, 0, stream));
    if (rel()) {
        SLF_TRY(sub.cells.ensure(n, 0, stream));
        SLF_TRY(sub.scells.ensure(n, 0, stream));
    }
    if (!terrains.empty()) SLF_TRY(sub.slope.ensure(n, 0, stream));
    SLF_TRY(sub.fent.ensure(slots, 0, stream));
    SLF_TRY(sub.went.ensure(slots, 0, stream));
    return SLF_OK;
}

int32_t World::keep_wcsph_substep(SubRecord& sub) {
    // the committed substep's sorted slots, as recompute names them
    const int a = (cpos + 2) % 3, nid = cid;
    auto copy = [&](auto& to, const auto* from, size_t count) -> int32_t {
        SLF_TRY(to.ensure(count, 0, stream));
        SLF_CUDA(cudaMemcpyAsync(to.p, from, count * sizeof(*from), cudaMemcpyDeviceToDevice, stream));
        return SLF_OK;
    };
    SLF_TRY(copy(sub.spos, pos[a].p, n));
    SLF_TRY(copy(sub.svel, vel[a].p, n));
    SLF_TRY(copy(sub.rho, rho[nid].p, n));
    SLF_TRY(copy(sub.press, press.p, n));
    SLF_TRY(copy(sub.scaled, scaled.p, n));
    if (rel()) SLF_TRY(copy(sub.scells, cell[a].p, n));
    sub.ordered = walk_order() != nullptr;
    if (sub.ordered) SLF_TRY(copy(sub.order, worder.p, n));
    if (!terrains.empty()) SLF_TRY(copy(sub.slope, gslope.p, n));
    // the body points this substep met, and their cell table
    const MoverDev M = mover_dev();
    sub.mcount = M.count;
    if (M.count) {
        SLF_TRY(copy(sub.mpos, M.pos, M.count));
        SLF_TRY(copy(sub.mvel, M.vel, M.count));
        sub.mgrid = M.grid;
        if (M.grid.mode == 1) {
            size_t cells = size_t(M.grid.sx) * size_t(M.grid.sy) * size_t(M.grid.sz);
            SLF_TRY(copy(sub.mstart, M.grid.start, cells + 1));
            sub.mgrid.start = sub.mstart.p;
        } else if (M.grid.mode == 2) {
            SLF_TRY(copy(sub.mstart, M.grid.start, size_t(M.grid.cells) + 1));
            SLF_TRY(copy(sub.mkeys, M.grid.keys, M.grid.cells));
            sub.mgrid.start = sub.mstart.p;
            sub.mgrid.keys = sub.mkeys.p;
        }
    }
    // the lists change places: the record takes this substep's, the world gets buffers to fill
    sub.cap = list_cap;
    std::swap(fent, sub.fent);
    std::swap(went, sub.went);
    std::swap(fcnt, sub.fcnt);
    std::swap(wcnt, sub.wcnt);
    lists_valid = false;
    SLF_TRY(ensure_work_buffers());
    sub.kept = true;
    return SLF_OK;
}

int32_t World::sync() {
    SLF_CUDA(cudaStreamSynchronize(stream));
    prof.collect();
    return SLF_OK;
}

void World::swap_lists(SubRecord& sub) {
    std::swap(fent, sub.fent);
    std::swap(went, sub.went);
    std::swap(fcnt, sub.fcnt);
    std::swap(wcnt, sub.wcnt);
    std::swap(fgv, sub.fgv);
    std::swap(wgv, sub.wgv);
}

int32_t World::kept_dfsph_substep(float dt, SubRecord& sub) {
    SLF_TRY(sub.dest.ensure(n, 0, stream));
    swap_lists(sub);
    sort_dest = sub.dest.p;
    uint32_t held = 0, its = 0;
    int32_t rs = dfsph_substep(dt, held, its, &sub.rec);
    if (rs == kRetry) rs = dfsph_substep(dt, held, its, &sub.rec);
    if (rs == kRetry) rs = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
    sort_dest = nullptr;
    // the record keeps the lists the substep wrote; the world's own buffers come back, to be
    // refilled by the next substep (a list room grown in the substep grows them too)
    sub.cap = list_cap;
    swap_lists(sub);
    lists_valid = false;
    SLF_TRY(rs);
    SLF_TRY(ensure_work_buffers());
    // the committed substep's sorted slots, as recompute names them
    const int a = (cpos + 2) % 3, nid = cid;
    auto copy = [&](auto& to, const auto* from, size_t count) -> int32_t {
        SLF_TRY(to.ensure(count, 0, stream));
        SLF_CUDA(cudaMemcpyAsync(to.p, from, count * sizeof(*from), cudaMemcpyDeviceToDevice, stream));
        return SLF_OK;
    };
    SLF_TRY(copy(sub.spos, pos[a].p, n));
    SLF_TRY(copy(sub.rho, rho[nid].p, n));
    SLF_TRY(copy(sub.alpha, alpha.p, n));
    sub.ordered = walk_order() != nullptr;
    if (sub.ordered) SLF_TRY(copy(sub.order, worder.p, n));
    sub.kept = true;
    return SLF_OK;
}

int32_t World::tape_begin(uint32_t every) {
    SLF_TRY(flush());
    tape.on = true;
    tape.every = every;
    tape.n = n;
    tape.steps.clear();
    tape.count = 0;
    tape.ckpt_sub.clear();
    drop_records(0);
    tape.keep_segments = false;
    if (every && n) {
        // the records of one checkpoint segment, each with room for its substep's forward, when
        // a segment's worth fits in half the device's free memory (else the backward runs each
        // substep again before its adjoint: WCSPH whole, DFSPH its sort and density pass)
        const size_t slots = PairLists::slots_for(uint32_t(n), list_cap);
        const size_t entry = sizeof(uint2) + (keeps_gradients() ? sizeof(float4) : 0);
        const size_t per = 2 * slots * entry + size_t(n) * (s.solver == SLF_SOLVER_DFSPH ? 112 : 160);
        size_t free = 0, total = 0;
        SLF_CUDA(cudaMemGetInfo(&free, &total));
        tape.keep_segments = size_t(every) * per <= free / 2;
        // (a DFSPH segment's records take their buffers when a backward first keeps one: a
        // short tape replays its segments, and holds none)
        if (tape.keep_segments && s.solver == SLF_SOLVER_WCSPH) {
            while (spare_records.size() < every) spare_records.push_back(std::make_unique<SubRecord>());
            for (size_t k = spare_records.size() - every; k < spare_records.size(); ++k)
                SLF_TRY(reserve_kept(*spare_records[k]));
        }
    }
    return every ? checkpoint() : SLF_OK;
}

void World::drop_records(size_t keep) {
    while (tape.subs.size() > keep) {
        spare_records.push_back(std::move(tape.subs.back()));
        tape.subs.pop_back();
    }
}

int32_t World::record_begin(float dt) {
    auto sub = new_record();
    sub->dt = dt;
    SLF_TRY(sub->pos.ensure(n, 0, stream));
    SLF_TRY(sub->vel.ensure(n, 0, stream));
    SLF_TRY(sub->ids.ensure(n, 0, stream));
    if (rel()) SLF_TRY(sub->cells.ensure(n, 0, stream));
    if (warm_on()) SLF_TRY(sub->warm.ensure(n, 0, stream));
    SLF_TRY(save_state(sub->pos.p, sub->vel.p, sub->ids.p, sub->cells.p, sub->warm.p));
    tape.subs.push_back(std::move(sub));
    return SLF_OK;
}

int32_t World::tape_end() {
    tape.on = false;
    tape.steps.clear();
    tape.count = 0;
    tape.ckpt_sub.clear();
    drop_records(0);
    return sync();
}

int32_t World::checkpoint() {
    size_t c = tape.ckpt_sub.size(), m = n;
    SLF_TRY(tape.cpos.ensure((c + 1) * m, c * m, stream));
    SLF_TRY(tape.cvel.ensure((c + 1) * m, c * m, stream));
    SLF_TRY(tape.cids.ensure((c + 1) * m, c * m, stream));
    if (rel()) SLF_TRY(tape.ccells.ensure((c + 1) * m, c * m, stream));
    if (warm_on()) SLF_TRY(tape.cwarm.ensure((c + 1) * m, c * m, stream));
    SLF_TRY(save_state(tape.cpos.p + c * m, tape.cvel.p + c * m, tape.cids.p + c * m,
                       rel() ? tape.ccells.p + c * m : nullptr, warm_on() ? tape.cwarm.p + c * m : nullptr));
    tape.ckpt_sub.push_back(tape.count);
    return SLF_OK;
}

int32_t World::tape_substep(float dt) {
    if (!tape_step) return SLF_OK;
    if (tape.every && tape.count > 0 && tape.count % tape.every == 0) SLF_TRY(checkpoint());
    tape_step->push_back(dt);
    ++tape.count;
    return SLF_OK;
}

int32_t World::save_state(float4* p, float4* v, uint32_t* id, int4* c, float2* w) {
    if (!n) return SLF_OK;
    if (w && warm_on())
        SLF_CUDA(cudaMemcpyAsync(w, warm[cid].p, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(p, pos[cpos].p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(v, vel[cpos].p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(id, ids[cid].p, n * 4, cudaMemcpyDeviceToDevice, stream));
    if (rel()) SLF_CUDA(cudaMemcpyAsync(c, cell[cpos].p, n * sizeof(int4), cudaMemcpyDeviceToDevice, stream));
    return SLF_OK;
}

int32_t World::load_state(const float4* p, const float4* v, const uint32_t* id, const int4* c, const float2* w) {
    if (n && w && warm_on())
        SLF_CUDA(cudaMemcpyAsync(warm[cid].p, w, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream));
    if (n) {
        SLF_CUDA(cudaMemcpyAsync(pos[cpos].p, p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(vel[cpos].p, v, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(ids[cid].p, id, n * 4, cudaMemcpyDeviceToDevice, stream));
        if (rel()) SLF_CUDA(cudaMemcpyAsync(cell[cpos].p, c, n * sizeof(int4), cudaMemcpyDeviceToDevice, stream));
    }
    stats_fresh = false;
    lists_valid = false;
    return refresh_stats();
}

int32_t World::substep_retrying(float dt) {
    uint32_t held = 0, its = 0;
    auto once = [&] { return s.solver == SLF_SOLVER_WCSPH ? wcsph_substep(dt, held) : dfsph_substep(dt, held, its); };
    int32_t st = once();
    if (st == kRetry) st = once();
    if (st == kRetry) st = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
    return st;
}

int32_t World::dfsph_replay(float dt, int& a, int& nid) {
    Params p = params();
    a = (cpos + 1) % 3;
    nid = 1 - cid;
    for (int attempt = 0;; ++attempt) {
        if (attempt > 0) {  // the committed state's box again
            stats_fresh = false;
            SLF_TRY(refresh_stats());
        }
        SLF_TRY(sort_into(a));
        SLF_TRY(reset_status());
        launch_set_consts(consts(dt), d_consts, stream);
        density_pass(p, a, fluid_lists(), wall_lists(), rho[nid].p);
        SLF_TRY(read_status());
        int32_t st = lists_fit();
        if (st == SLF_OK) return SLF_OK;
        if (st != kRetry || attempt > 0) return st == kRetry ? fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice") : st;
    }
}

int32_t World::step_backward(const float* dpos, const float* dvel, uint64_t k, float* dpos0, float* dvel0,
                             slf_param_grads* out) {
    if (!tape.on || tape.steps.empty()) return fail(SLF_ERR_OUT_OF_RANGE, "no steps recorded");
    SLF_TRY(flush());
    if (k != n || n != tape.n) return fail(SLF_ERR_INVALID_ARGUMENT, "n must equal slf_len()");
    prepare_adjoint_grids();
    slf_param_grads pg{};
    if (n == 0) {
        if (out) *out = pg;
        return SLF_OK;
    }
    // the committed state, to put back at the end, and the pass's scratch (kept for the next
    // call, like the tape's records)
    BackScratch& B = back;
    DevBuf<float4> &spos = B.spos, &svel = B.svel, &xo = B.xo, &vo = B.vo, &xp = B.xp, &vp = B.vp,
                   &ab = B.ab, &xb = B.xb, &vb = B.vb, &pre = B.pre, &gt = B.gt, &kw = B.kw, &vr = B.vr;
    DevBuf<uint32_t> &sids = B.sids, &dest = B.dest;
    DevBuf<int4>& scells = B.scells;
    DevBuf<float> &srho = B.srho, &rb = B.rb, &abar = B.abar, &zeros = B.zeros;
    DevBuf<double>& grads = B.grads;
    int32_t st = SLF_OK;
    auto run = [&]() -> int32_t {
        for (auto* b : {&spos, &svel, &xo, &vo, &xp, &vp, &ab, &xb, &vb, &pre, &gt, &kw, &vr})
            SLF_TRY(b->ensure(n, 0, stream));
        for (auto* b : {&srho, &rb, &abar, &zeros}) SLF_TRY(b->ensure(n, 0, stream));
        SLF_CUDA(cudaMemsetAsync(zeros.p, 0, n * 4, stream));
        SLF_TRY(sids.ensure(n, 0, stream));
        SLF_TRY(dest.ensure(n, 0, stream));
        SLF_TRY(grads.ensure(kGradSlots, 0, stream));
        if (rel()) SLF_TRY(scells.ensure(n, 0, stream));
        if (warm_on()) {
            for (auto* b : {&B.swarm, &B.appbar, &B.appbar_out}) SLF_TRY(b->ensure(n, 0, stream));
            // the impulses the last substep's solves leave reach no output
            SLF_CUDA(cudaMemsetAsync(B.appbar.p, 0, n * sizeof(float2), stream));
        }
        SLF_TRY(save_state(spos.p, svel.p, sids.p, scells.p, B.swarm.p));
        SLF_CUDA(cudaMemcpyAsync(srho.p, rho[cid].p, n * 4, cudaMemcpyDeviceToDevice, stream));
        SLF_TRY(write_vec(xo, dpos, n));
        SLF_TRY(write_vec(vo, dvel, n));
        // the adjoint of the substep whose forward state sits in slots a (sorted positions)
        // and nid (densities), its constants in d_consts: (xo, vo) after it -> (xp, vp) before
        // (kept: a WCSPH substep's forward as a segment's replay kept it, in place of the world's)
        auto adjoint_substep = [&](float dt, int a, int nid, const DfsphRecord& rec,
                                   const SubRecord* kept = nullptr) -> int32_t {
            Params p = params();
            SLF_CUDA(cudaMemsetAsync(grads.p, 0, kGradSlots * sizeof(double), stream));
            PairLists fl = fluid_lists(), wl = wall_lists();
            const int form = !fast() ? 1 : (rel() ? 2 : 0);  // the lists' form (launch.h)
            if (s.solver == SLF_SOLVER_WCSPH && kept) {
                // the stiffness and constants at the sound speed the step ran at (a fast body may
                // have raised it)
                {
                    const float configured = s.sound_speed;
                    if (kept->sound > 0.0f) s.sound_speed = kept->sound;
                    p = params();
                    launch_set_consts(consts(dt), d_consts, stream);
                    s.sound_speed = configured;
                }
                const uint32_t* order = kept->ordered ? kept->order.p : nullptr;
                PairLists kf{kept->cap, kept->fent.p, kept->fcnt.p, order, nullptr};
                PairLists kw_{kept->cap, kept->went.p, kept->wcnt.p, order, nullptr};
                MoverDev km{};
                if (kept->mcount) {
                    km.count = kept->mcount;
                    km.grid = kept->mgrid;
                    km.pos = kept->mpos.p;
                    km.vel = kept->mvel.p;
                }
                timed("adj_wcsph", 0.0, [&] {
                    launch_adjoint_wcsph(p, d_consts, kf, kw_, form, kept->spos.p, kept->svel.p, kept->rho.p,
                                         kept->press.p, kept->scaled.p, dwalls.p, kept->pre.p, kept->dest.p, xo.p,
                                         vo.p, ab.p, xb.p, vb.p, rb.p, xp.p, vp.p, grads.p, tdev,
                                         terrains.empty() ? nullptr : kept->slope.p, km, stream);
                });
            } else if (s.solver == SLF_SOLVER_WCSPH) {
                timed("adj_wcsph", 0.0, [&] {
                    launch_adjoint_wcsph(p, d_consts, fl, wl, form, pos[a].p, vel[a].p, rho[nid].p, press.p,
                                         scaled.p, dwalls.p, pre.p, dest.p, xo.p, vo.p, ab.p, xb.p, vb.p, rb.p, xp.p,
                                         vp.p, grads.p, tdev, terrains.empty() ? nullptr : gslope.p, MoverDev{},
                                         stream);
                });
            } else {
                // the substep's sorted positions, densities, factors, sort destinations, lists
                // and starting impulses: the world's after the replay of its sort and densities,
                // or those a segment's replay kept
                const float4* spx = pos[a].p;
                const float *srh = rho[nid].p, *sal = alpha.p;
                const uint32_t* sdest = dest.p;
                const float2* applied = warm_on() ? warm[nid].p : nullptr;
                if (kept) {
                    spx = kept->spos.p;
                    srh = kept->rho.p;
                    sal = kept->alpha.p;
                    sdest = kept->dest.p;
                    if (applied) applied = kept->rec.warm.p;
                    const uint32_t* order = kept->ordered ? kept->order.p : nullptr;
                    fl = PairLists{kept->cap, kept->fent.p, kept->fcnt.p, order,
                                   keeps_gradients() ? kept->fgv.p : nullptr};
                    wl = PairLists{kept->cap, kept->went.p, kept->wcnt.p, order,
                                   keeps_gradients() ? kept->wgv.p : nullptr};
                    launch_set_consts(consts(dt), d_consts, stream);
                }
                // advance, density solve, viscosity, divergence solve, factors, densities,
                // sort: the substep's steps backwards
                timed("adj_advance", 0.0, [&] {
                    launch_adj_advance_dfsph(p, d_consts, rec.pre.p, xo.p, vo.p, xb.p, vb.p, stream);
                });
                SLF_CUDA(cudaMemsetAsync(rb.p, 0, n * 4, stream));
                SLF_CUDA(cudaMemsetAsync(abar.p, 0, n * 4, stream));
                // warm starts: the adjoint of the impulses after the substep
                const float2* apb = warm_on() ? B.appbar.p : nullptr;
                // each solve's warm push ran before its first check: its adjoint after the
                // last iteration's (share: the forward's half of the last impulse)
                auto warm_push = [&](int which) {
                    if (!applied) return;
                    timed(which == 1 ? "adj_warm_density" : "adj_warm_divergence", 0.0, [&] {
                        launch_adj_warm(which, p, d_consts, fl, wl, form, spx, dwalls.p, vb.p, applied, apb,
                                        0.5f, kw.p, vr.p, B.appbar_out.p, vp.p, xb.p, stream);
                    });
                    std::swap(vb, vp);
                };
                for (uint32_t it = rec.den_n; it-- > 0;) {
                    for (int part = 1; part <= 2; ++part)
                        timed(part == 1 ? "adj_kappa_density" : "adj_push_density", 0.0, [&] {
                            launch_adj_iteration(1, p, d_consts, fl, wl, form, spx, dwalls.p, vb.p,
                                                 rec.den_rate.p + size_t(it) * n, sal, srh,
                                                 rec.den_vel.p + size_t(it) * n, kw.p, vr.p, abar.p, rb.p,
                                                 vp.p, xb.p, stream, part, apb);
                        });
                    std::swap(vb, vp);
                }
                warm_push(1);
                timed("adj_viscosity", 0.0, [&] {
                    launch_adj_viscosity(p, d_consts, fl, wl, form, spx, rec.va.p, srh, zeros.p,
                                         dwalls.p, vb.p, ab.p, xb.p, rb.p, grads.p, stream);
                });
                for (uint32_t it = rec.div_n; it-- > 0;) {
                    for (int part = 1; part <= 2; ++part)
                        timed(part == 1 ? "adj_kappa_divergence" : "adj_push_divergence", 0.0, [&] {
                            launch_adj_iteration(0, p, d_consts, fl, wl, form, spx, dwalls.p, vb.p,
                                                 rec.div_rate.p + size_t(it) * n, sal, srh,
                                                 rec.div_vel.p + size_t(it) * n, kw.p, vr.p, abar.p, rb.p,
                                                 vp.p, xb.p, stream, part, apb);
                        });
                    std::swap(vb, vp);
                }
                warm_push(0);
                timed("adj_factors_density", 0.0, [&] {
                    launch_adj_factors_density(p, fl, wl, form, spx, dwalls.p, sal, abar.p, gt.p,
                                               rb.p, xb.p, stream);
                });
                timed("adj_unsort", 0.0, [&] {
                    launch_adj_unsort(uint32_t(n), sdest, xb.p, vb.p, xp.p, vp.p, stream,
                                      warm_on() ? B.appbar_out.p : nullptr, B.appbar.p);
                });
            }
            double g[kGradSlots];
            SLF_CUDA(cudaMemcpyAsync(g, grads.p, sizeof(g), cudaMemcpyDeviceToHost, stream));
            SLF_TRY(sync());
            if (kept) accumulate_param_grads(dt, g, pg, kept->sound, kept->raised);
            else accumulate_param_grads(dt, g, pg);
            std::swap(xo, xp);
            std::swap(vo, vp);
            return SLF_OK;
        };
        // substep q again from its state, recording what its adjoint reads; the state's slots
        // come back in a and nid
        auto recompute = [&](float dt, DfsphRecord& rec, int& a, int& nid) -> int32_t {
            sort_dest = dest.p;
            vel_pre = pre.p;
            int32_t rs;
            uint32_t held = 0, its = 0;
            if (s.solver == SLF_SOLVER_WCSPH) {
                rs = wcsph_substep(dt, held);
                if (rs == kRetry) rs = wcsph_substep(dt, held);
            } else {
                rs = dfsph_substep(dt, held, its, &rec);
                if (rs == kRetry) rs = dfsph_substep(dt, held, its, &rec);
            }
            if (rs == kRetry) rs = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
            sort_dest = nullptr;
            vel_pre = nullptr;
            a = (cpos + 2) % 3;  // the committed substep's sorted positions
            nid = cid;
            return rs;
        };

        // backward through recorded substeps subs[0, count): each one's sort and densities
        // again (WCSPH: the whole substep, one pass), then its adjoint
        auto backward_through = [&](std::vector<std::unique_ptr<SubRecord>>& subs, size_t count) -> int32_t {
            for (size_t q = count; q-- > 0;) {
                SubRecord& sub = *subs[q];
                if (sub.kept) {  // nothing to run again: its forward is in the record
                    SLF_TRY(adjoint_substep(sub.dt, 0, 0, sub.rec, &sub));
                    continue;
                }
                SLF_TRY(load_state(sub.pos.p, sub.vel.p, sub.ids.p, sub.cells.p, sub.warm.p));
                int a = 0, nid = 0;
                if (s.solver == SLF_SOLVER_WCSPH) {
                    SLF_TRY(recompute(sub.dt, sub.rec, a, nid));
                } else {
                    sort_dest = dest.p;
                    int32_t rs = dfsph_replay(sub.dt, a, nid);
                    sort_dest = nullptr;
                    SLF_TRY(rs);
                }
                SLF_TRY(adjoint_substep(sub.dt, a, nid, sub.rec));
            }
            return SLF_OK;
        };

        // every substep was recorded as it ran
        auto recorded = [&]() -> int32_t { return backward_through(tape.subs, tape.subs.size()); };

        // checkpoints: each segment runs forward again from its checkpoint, recording its
        // substeps (states and solver records), then backward through them
        std::vector<std::unique_ptr<SubRecord>> segsubs;
        auto rel2 = [&] {
            for (auto& r : segsubs) spare_records.push_back(std::move(r));
            segsubs.clear();
        };
        auto segs = [&]() -> int32_t {
            const bool keep_dfsph = tape.keep_segments && (!graphs_for(SolveRec{nullptr, nullptr}) ||
                                                           tape.ckpt_sub.size() >= kKeepMinSegments);
            std::vector<float> all;  // every recorded substep's length, in order
            for (const auto& st : tape.steps) all.insert(all.end(), st.begin(), st.end());
            for (size_t c = tape.ckpt_sub.size(); c-- > 0;) {
                size_t b = tape.ckpt_sub[c];
                size_t e = c + 1 < tape.ckpt_sub.size() ? tape.ckpt_sub[c + 1] : all.size();
                if (b >= e) continue;
                std::vector<float> dts(all.begin() + b, all.begin() + e);
                while (segsubs.size() < dts.size()) segsubs.push_back(new_record());
                SLF_TRY(load_state(tape.cpos.p + c * n, tape.cvel.p + c * n, tape.cids.p + c * n,
                                   rel() ? tape.ccells.p + c * n : nullptr, warm_on() ? tape.cwarm.p + c * n : nullptr));
                for (size_t q = 0; q < dts.size(); ++q) {
                    SubRecord& sub = *segsubs[q];
                    sub.dt = dts[q];
                    SLF_TRY(sub.pos.ensure(n, 0, stream));
                    SLF_TRY(sub.vel.ensure(n, 0, stream));
                    SLF_TRY(sub.ids.ensure(n, 0, stream));
                    if (rel()) SLF_TRY(sub.cells.ensure(n, 0, stream));
                    if (warm_on()) SLF_TRY(sub.warm.ensure(n, 0, stream));
                    SLF_TRY(save_state(sub.pos.p, sub.vel.p, sub.ids.p, sub.cells.p, sub.warm.p));
                    uint32_t held = 0, its = 0;
                    int32_t rs;
                    if (s.solver == SLF_SOLVER_WCSPH && !tape.keep_segments) {
                        rs = wcsph_substep(dts[q], held);
                        if (rs == kRetry) rs = wcsph_substep(dts[q], held);
                    } else if (s.solver == SLF_SOLVER_WCSPH) {
                        // the sort's destinations and the pre-clamp velocities go into the record
                        SLF_TRY(sub.dest.ensure(n, 0, stream));
                        SLF_TRY(sub.pre.ensure(n, 0, stream));
                        sort_dest = sub.dest.p;
                        vel_pre = sub.pre.p;
                        rs = wcsph_substep(dts[q], held);
                        if (rs == kRetry) rs = wcsph_substep(dts[q], held);
                        sort_dest = nullptr;
                        vel_pre = nullptr;
                        if (rs == SLF_OK) rs = keep_wcsph_substep(sub);
                    } else if (keep_dfsph) {
                        rs = kept_dfsph_substep(dts[q], sub);
                    } else {
                        rs = dfsph_substep(dts[q], held, its, &sub.rec);
                        if (rs == kRetry) rs = dfsph_substep(dts[q], held, its, &sub.rec);
                    }
                    if (rs == kRetry) rs = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
                    SLF_TRY(rs);
                }
                SLF_TRY(backward_through(segsubs, dts.size()));
            }
            return SLF_OK;
        };
        int32_t r = tape.every == 0 ? recorded() : segs();
        rel2();
        SLF_TRY(r);
        if (dpos0) SLF_TRY(read_vec(xo, dpos0, n));
        if (dvel0) SLF_TRY(read_vec(vo, dvel0, n));
        // the state as it was
        SLF_TRY(load_state(spos.p, svel.p, sids.p, scells.p, B.swarm.p));
        SLF_CUDA(cudaMemcpyAsync(rho[cid].p, srho.p, n * 4, cudaMemcpyDeviceToDevice, stream));
        return sync();
    };
    st = run();
    sync();
    if (st == SLF_OK && out) *out = pg;
    return st;
}

void World::accumulate_param_grads(float dt, const double* g, slf_param_grads& pg, float sound, bool raised) const {
    // sound: the speed the substep ran at; raised: a fast body set it, so the settings' sound
    // speed did not reach the substep
    double r = radius, c = sound > 0.0f ? sound : s.sound_speed, visc = s.viscosity;
    double dc = raised ? 0.0 : 1.0;
    bool nu_free = double(s.viscosity) * c * r < 0.05 * r * r / dt;
    bool nuw_free = c * r < 0.25 * r * r / dt;
    if (nu_free) {
        pg.viscosity += g[kGradViscosity] * c * r;
        pg.sound_speed += dc * g[kGradViscosity] * visc * r;
    }
    if (nuw_free) pg.sound_speed += dc * g[kGradWallViscosity] * r;
    pg.sound_speed += dc * g[kGradStiffness] * 2.0 * double(s.rest_density) * c / 7.0;
    for (int a = 0; a < 3; ++a) pg.gravity[a] += g[kGradGravity + a];
}

int32_t World::step_untaped(float dt, slf_report* out) {
    slf_report r{};
    if (out) *out = r;
    if (!std::isfinite(dt) || dt < 0.0f) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid step");
    if (dt == 0.0f) return SLF_OK;
    SLF_TRY(flush());
    SLF_TRY(upload_walls());
    SLF_TRY(upload_terrain());
    if (n > 0) {
        SLF_TRY(ensure_work_buffers());
        SLF_TRY(refresh_stats());
        if (s.solver == SLF_SOLVER_WCSPH) {
            // wcsph (step.rs:102-142): the step's sound speed follows the fastest coupled body
            // near the water, its points sweep on through the substeps
            float configured = s.sound_speed, mover = 0.0f;
            SLF_TRY(fastest_near_water(dt, configured / 4.0f, mover));
            struct Restore {
                float& to;
                float value;
                ~Restore() { to = value; }
            } restore{s.sound_speed, configured};
            s.sound_speed = rmax(configured, 4.0f * mover);
            r.sound_speed = s.sound_speed;
            float fast = rmax(fastest(), mover);
            float largest = s.courant * radius / (s.sound_speed + fast);
            float wanted = rmax(std::ceil(dt / largest), 1.0f);
            float cap = float(s.max_substeps);
            uint32_t substeps = uint32_t(rmin(wanted, cap));
            r.capped = wanted > cap;
            float small = dt / float(substeps);
            for (uint32_t i = 0; i < substeps; ++i) {
                uint32_t held = 0;
                SLF_TRY(tape_substep(small));
                if (tape_step && tape.every == 0) SLF_TRY(record_begin(small));
                if (!coupled.empty()) SLF_TRY(carry_movers(small * float(i), small * float(substeps - 1)));
                // with coupled bodies a recording tape keeps each substep's forward as it runs:
                // the body points' order follows their history, so the backward cannot run it again
                SubRecord* keep = tape_step && tape.every == 0 && !coupled.empty() ? tape.subs.back().get() : nullptr;
                if (keep) {
                    SLF_TRY(keep->dest.ensure(n, 0, stream));
                    SLF_TRY(keep->pre.ensure(n, 0, stream));
                    sort_dest = keep->dest.p;
                    vel_pre = keep->pre.p;
                }
                int32_t st = wcsph_substep(small, held);
                if (st == kRetry) st = wcsph_substep(small, held);
                if (st == kRetry) st = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
                if (keep) {
                    sort_dest = nullptr;
                    vel_pre = nullptr;
                    if (st == SLF_OK) st = keep_wcsph_substep(*keep);
                    keep->sound = s.sound_speed;
                    keep->raised = s.sound_speed != configured;
                }
                SLF_TRY(st);
                r.held_back += held;
            }
            r.substeps = substeps;
        } else {
            // dfsph.rs:52-55: ground pushes through the weakly compressible solver's pressure only
            if (!terrains.empty()) return fail(SLF_ERR_INVALID_SETTINGS, "DFSPH takes no terrain");
            // dfsph (dfsph.rs:46-77)
            float spacing = s.spacing, courant = s.courant;
            float pull = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] +
                                   s.gravity[2] * s.gravity[2]);
            float left = dt;
            while (left > 0.0f) {
                float small = courant * spacing / rmax(fastest(), 1e-6f);
                if (pull > 0.0f) small = rmin(small, std::sqrt(2.0f * courant * spacing / pull));
                if (r.substeps + 1 >= s.max_substeps && small < left) {
                    r.capped = 1;
                    small = left;
                }
                small = rmin(small, left);
                uint32_t held = 0, its = 0;
                SLF_TRY(tape_substep(small));
                DfsphRecord* rec = nullptr;
                if (tape_step && tape.every == 0) {
                    SLF_TRY(record_begin(small));
                    rec = &tape.subs.back()->rec;
                }
                int32_t st = dfsph_substep(small, held, its, rec);
                if (st == kRetry) st = dfsph_substep(small, held, its, rec);
                if (st == kRetry) st = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
                SLF_TRY(st);
                r.iterations += its;
                r.held_back += held;
                r.substeps += 1;
                left -= small;
            }
        }
    }
    // the last substep's status holds the committed state's fastest speed (its advance) and
    // largest compression (its density pass): the report's maxima unless flows or the domain
    // change the particles next
    bool settled_report = n > 0 && r.substeps > 0 && flows.empty() && !has_domain && stats_fresh;
    // run_flows (step.rs:76-81), then keep_in_domain (mod.rs:451-486)
    SLF_TRY(run_flows(r.emitted, r.drained));
    SLF_TRY(keep_in_domain(r.lost));
    // max_speed and max_compression of what is left (step.rs:83-88)
    if (settled_report) {
        std::memcpy(&r.max_speed, &h_status->vmax_bits, 4);
        std::memcpy(&r.max_compression, &h_status->maxcomp_bits, 4);
    } else if (n > 0) {
        SLF_TRY(reset_status());
        Params p = params();
        timed("stats", bytes_per_particle::stats, [&] {
            stats_pass(p);
            launch_max_compression(p, rho[cid].p, d_status, stream);
        });
        SLF_TRY(read_status());
        stats_fresh = true;
        std::memcpy(&r.max_speed, &h_status->vmax_bits, 4);
        std::memcpy(&r.max_compression, &h_status->maxcomp_bits, 4);
    }
    if (out) *out = r;
    return SLF_OK;
}

int32_t World::keep_where(F3 low, F3 high, int drain, uint32_t& removed) {
    removed = 0;
    if (n == 0) return SLF_OK;
    Params p = params();
    SLF_TRY(keep.ensure(n + 1, 0, stream));
    SLF_TRY(members.ensure(n + 1, 0, stream));
    SLF_TRY(tiles.ensure(scan_tiles(uint32_t(n)) + 1, 0, stream));
    launch_domain_flags(p, pos[cpos].p, cells_of(cpos), make_float3(low.x, low.y, low.z),
                        make_float3(high.x, high.y, high.z), drain, keep.p, stream);
    SLF_CUDA(cudaMemcpyAsync(members.p, keep.p, n * 4, cudaMemcpyDeviceToDevice, stream));
    launch_exclusive_scan(members.p, uint32_t(n), tiles.p, stream);
    uint32_t kept = 0;
    SLF_CUDA(cudaMemcpyAsync(&kept, members.p + n, 4, cudaMemcpyDeviceToHost, stream));
    SLF_CUDA(cudaStreamSynchronize(stream));
    if (kept == n) return SLF_OK;
    int to = (cpos + 1) % 3;
    if (to == lists_pos) to = (cpos + 2) % 3;
    launch_compact(uint32_t(n), keep.p, members.p, ids[cid].p, pos[cpos].p, vel[cpos].p, rho[cid].p,
                   cells_of(cpos), ids[1 - cid].p, pos[to].p, vel[to].p, rho[1 - cid].p, cells_of(to), warm_in(),
                   warm_out(), stream);
    SLF_CUDA(cudaStreamSynchronize(stream));
    removed = uint32_t(n - kept);
    n = kept;
    cpos = to;
    cid = 1 - cid;
    lists_valid = false;
    stats_fresh = false;
    return SLF_OK;
}

int32_t World::keep_in_domain(uint32_t& lost) {
    lost = 0;
    if (!has_domain) return SLF_OK;
    return keep_where(dlow, dhigh, 0, lost);
}

}  // namespace slf
