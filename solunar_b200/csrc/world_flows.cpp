// world_flows.cpp -- World's emitters and drains (src/fluid/flow.rs).
#include "world.h"

namespace slf {

int32_t World::add_flow(const float* low, const float* high, bool emitter, const float* velocity, uint32_t* out) {
    if (emitter && !finite3(velocity)) return fail(SLF_ERR_NON_FINITE, "non finite value in emitter velocity");
    if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in flow box");
    if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
        return fail(SLF_ERR_OUT_OF_RANGE, "inside out flow box");
    if (flow_next == UINT32_MAX) return fail(SLF_ERR_FLUID_FULL, "no flow ids left");
    FlowBox f{flow_next++, F3{low[0], low[1], low[2]}, F3{high[0], high[1], high[2]}, emitter, F3{0, 0, 0}};
    if (emitter) f.velocity = F3{velocity[0], velocity[1], velocity[2]};
    flows.push_back(f);
    if (out) *out = f.id;
    return SLF_OK;
}

bool World::remove_flow(uint32_t id) {
    size_t before = flows.size();
    flows.erase(std::remove_if(flows.begin(), flows.end(), [&](const FlowBox& f) { return f.id == id; }),
                flows.end());
    return flows.size() != before;
}

int64_t World::as_i64(float v) {
    if (std::isnan(v)) return 0;
    if (v >= 9.2233720e18f) return INT64_MAX;
    if (v <= -9.2233720e18f) return INT64_MIN;
    return int64_t(v);
}

int32_t World::run_flows(uint32_t& emitted, uint32_t& drained) {
    emitted = drained = 0;
    if (flows.empty()) return SLF_OK;
    std::vector<FlowBox> list = flows;
    for (const FlowBox& f : list) {
        if (f.emitter) continue;
        uint32_t gone = 0;
        SLF_TRY(keep_where(f.low, f.high, 1, gone));
        drained += gone;
    }
    const float spacing = s.spacing;
    for (const FlowBox& f : list) {
        if (!f.emitter) continue;
        auto count = [&](float extent) -> int64_t {
            return std::min<int64_t>(std::max<int64_t>(as_i64(std::floor(extent / spacing)), 0), int64_t(1) << 12);
        };
        int64_t cx = count(f.high.x - f.low.x), cy = count(f.high.y - f.low.y), cz = count(f.high.z - f.low.z);
        int64_t total = cx * cy * cz;
        if (total == 0) continue;
        if (total > (int64_t(1) << 30)) return fail(SLF_ERR_OUT_OF_RANGE, "emitter box holds more than 2^30 slots");
        float share = 0.9f * spacing;
        float clear = share * share;
        uint32_t slots = uint32_t(total);
        SLF_TRY(etaken.ensure(size_t(slots) + 1, 0, stream));
        SLF_TRY(etiles.ensure(scan_tiles(slots) + 1, 0, stream));
        SLF_CUDA(cudaMemsetAsync(etaken.p, 0, (size_t(slots) + 1) * 4, stream));
        Params p = params();
        float3 low3 = make_float3(f.low.x, f.low.y, f.low.z);
        int3 cnt = make_int3(int(cx), int(cy), int(cz));
        launch_emitter_taken(p, pos[cpos].p, cells_of(cpos), low3, cnt, spacing, clear, etaken.p, stream);
        launch_exclusive_scan(etaken.p, slots, etiles.p, stream);
        uint32_t taken = 0;
        SLF_CUDA(cudaMemcpyAsync(&taken, etaken.p + slots, 4, cudaMemcpyDeviceToHost, stream));
        SLF_CUDA(cudaStreamSynchronize(stream));
        uint64_t free_slots = uint64_t(slots) - taken;
        // add_particle's room (mod.rs:416-418): the particle cap and the ids left
        uint64_t room = s.max_particles > n ? s.max_particles - n : 0;
        room = std::min<uint64_t>(room, uint64_t(UINT32_MAX - next_id));
        room = std::min<uint64_t>(room, index_limit() > n ? index_limit() - n : 0);
        uint64_t k = std::min<uint64_t>(free_slots, room);
        if (k) {
            uint64_t m = n + k;
            for (int i = 0; i < 3; ++i) {
                SLF_TRY(pos[i].ensure(m, i == cpos ? n : 0, stream));
                SLF_TRY(vel[i].ensure(m, i == cpos ? n : 0, stream));
                if (rel()) SLF_TRY(cell[i].ensure(m, i == cpos ? n : 0, stream));
            }
            for (int i = 0; i < 2; ++i) {
                SLF_TRY(ids[i].ensure(m, i == cid ? n : 0, stream));
                SLF_TRY(rho[i].ensure(m, i == cid ? n : 0, stream));
                if (warm_on()) SLF_TRY(warm[i].ensure(m, i == cid ? n : 0, stream));
            }
            float4* out = pos[cpos].p + n;
            if (rel()) {
                SLF_TRY(estage.ensure(k, 0, stream));
                out = estage.p;
            }
            launch_emit(slots, etaken.p, cnt, low3, spacing, make_float3(f.velocity.x, f.velocity.y, f.velocity.z),
                        uint32_t(k), next_id, out, vel[cpos].p + n, ids[cid].p + n, rho[cid].p + n, stream);
            if (warm_on()) SLF_CUDA(cudaMemsetAsync(warm[cid].p + n, 0, k * sizeof(float2), stream));
            if (rel()) launch_to_relative(p, uint32_t(k), nullptr, estage.p, pos[cpos].p + n, cell[cpos].p + n, stream);
            n = m;
            next_id += uint32_t(k);
            emitted += uint32_t(k);
            lists_valid = false;
            stats_fresh = false;
        }
        if (k < free_slots) return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    }
    return SLF_OK;
}

}  // namespace slf
