// world_bodies.cpp -- World's coupled bodies (src/fluid/couple.rs, lift.rs).
#include "world.h"

namespace slf {

MoverDev World::mover_dev() const {
    MoverDev M{};
    if (m_pos.empty()) return M;
    M.count = uint32_t(m_pos.size());
    M.grid = mgrid;
    M.pos = dmpos.p;
    M.vel = mdevice ? dmcur_vel.p : dmvel.p;
    return M;
}

int32_t World::shape_points(int kind, const float dims[3], float spacing, float reach, uint64_t limit,
                            std::vector<F3>& out) {
    out.clear();
    F3 half;
    float a = dims[0], b = dims[1], c = dims[2];
    if (kind == SLF_SHAPE_CUBOID) {
        half = F3{a, b, c};
    } else if (kind == SLF_SHAPE_SPHERE) {
        half = F3{a, a, a};
    } else if (kind == SLF_SHAPE_CAPSULE) {
        if (!(b >= 0.0f)) return fail(SLF_ERR_INVALID_SHAPE, "invalid shape");
        half = F3{a, b + a, a};
    } else {
        return fail(SLF_ERR_INVALID_SHAPE, "invalid shape");
    }
    bool finite = std::isfinite(half.x) && std::isfinite(half.y) && std::isfinite(half.z);
    if (!finite || rmin(rmin(half.x, half.y), half.z) <= 0.0f) return fail(SLF_ERR_INVALID_SHAPE, "invalid shape");
    auto depth = [&](F3 at) -> float {
        if (kind == SLF_SHAPE_CUBOID) {
            F3 room = half - F3{std::fabs(at.x), std::fabs(at.y), std::fabs(at.z)};
            return rmin(rmin(room.x, room.y), room.z);
        }
        if (kind == SLF_SHAPE_SPHERE) return a - length(at);
        float y = rmin(rmax(at.y, -b), b);
        return a - length(at - F3{0.0f, y, 0.0f});
    };
    auto count = [&](float extent) -> int64_t {
        float v = std::floor(2.0f * extent / spacing);
        return std::isnan(v) ? 0 : (v >= 4096.0f ? 4096 : (v <= 0.0f ? 0 : int64_t(v)));
    };
    int64_t cx = count(half.x), cy = count(half.y), cz = count(half.z);
    if (uint64_t(cx * cy * cz) > limit) return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    auto start = [&](int64_t cells) { return -(float(cells) - 1.0f) * spacing / 2.0f; };
    F3 origin{start(cx), start(cy), start(cz)};
    for (int64_t y = 0; y < cy; ++y)
        for (int64_t z = 0; z < cz; ++z)
            for (int64_t x = 0; x < cx; ++x) {
                F3 at = origin + F3{float(x), float(y), float(z)} * spacing;
                float inside = depth(at);
                if (inside >= 0.0f && inside <= reach) out.push_back(at);
            }
    return SLF_OK;
}

uint64_t World::coupled_points() const {
    uint64_t k = 0;
    for (auto& c : coupled) k += c.points.size();
    return k;
}

int32_t World::couple(uint64_t body, int32_t kind, const float dims[3]) {
    std::vector<F3> points, probes;
    SLF_TRY(shape_points(kind, dims, s.spacing, radius, s.max_particles, points));
    if (points.empty()) return fail(SLF_ERR_INVALID_SHAPE, "invalid shape");
    uint64_t used = coupled_points();
    uint64_t room = s.max_particles > used ? s.max_particles - used : 0;
    if (points.size() > room) return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    // coarser probes for a big body, each standing for its share of the volume
    float probe_spacing = s.spacing;
    for (;;) {
        int32_t st = shape_points(kind, dims, probe_spacing, INFINITY, kMaxProbes, probes);
        if (st == SLF_ERR_FLUID_FULL) {
            probe_spacing = probe_spacing * 1.25f;
            continue;
        }
        SLF_TRY(st);
        if (probes.empty()) {
            probe_spacing = s.spacing;
            probes = points;
        }
        break;
    }
    uncouple(body);
    Coupled c;
    c.body = body;
    c.points = std::move(points);
    c.probes = std::move(probes);
    c.probe_spacing = probe_spacing;
    coupled.push_back(std::move(c));
    std::stable_sort(coupled.begin(), coupled.end(),
                     [](const Coupled& x, const Coupled& y) { return x.body < y.body; });
    return SLF_OK;
}

bool World::uncouple(uint64_t body) {
    size_t before = coupled.size();
    coupled.erase(std::remove_if(coupled.begin(), coupled.end(), [&](const Coupled& c) { return c.body == body; }),
                  coupled.end());
    return coupled.size() != before;
}

const slf_body_pose* World::pose_of(const slf_body_pose* poses, uint64_t n, uint64_t body) {
    for (uint64_t k = 0; k < n; ++k)
        if (poses[k].body == body) return &poses[k];
    return nullptr;
}

void World::place_movers_at(const slf_body_pose* poses, uint64_t npose) {
    coupled.erase(std::remove_if(coupled.begin(), coupled.end(),
                                 [&](const Coupled& c) { return !pose_of(poses, npose, c.body); }),
                  coupled.end());
    m_start.clear();
    m_vel.clear();
    m_own.clear();
    for (size_t owner = 0; owner < coupled.size(); ++owner) {
        Coupled& known = coupled[owner];
        const slf_body_pose& state = *pose_of(poses, npose, known.body);
        F3 center = center_of(state), lin = f3v(state.linear_velocity), ang = f3v(state.angular_velocity);
        known.center = center;
        known.velocity = lin;
        known.impulse = known.angular = F3{0, 0, 0};
        for (const F3& local : known.points) {
            F3 arm = rotate(state.rotation, local);
            m_start.push_back(center + arm);
            m_vel.push_back(lin + cross(ang, arm));
            m_own.push_back(uint32_t(owner));
        }
    }
    m_pos = m_start;
}

int32_t World::plan_movers(float last) {
    size_t k = m_start.size();
    mdevice = false;
    if (!k) return SLF_OK;
    Key3 lo = cell_of(m_start[0]), hi = lo;
    for (size_t i = 0; i < k; ++i)
        for (float e : {0.0f, last}) {
            Key3 c = cell_of(m_start[i] + m_vel[i] * e);
            lo = Key3{std::min(lo.x, c.x), std::min(lo.y, c.y), std::min(lo.z, c.z)};
            hi = Key3{std::max(hi.x, c.x), std::max(hi.y, c.y), std::max(hi.z, c.z)};
        }
    // one cell more on every side, and well inside the i32 range
    const int64_t lim = int64_t(1) << 30;
    for (int64_t v : {int64_t(lo.x), int64_t(lo.y), int64_t(lo.z), int64_t(hi.x), int64_t(hi.y), int64_t(hi.z)})
        if (v <= -lim || v >= lim) return SLF_OK;
    int64_t sx = int64_t(hi.x) - lo.x + 3, sy = int64_t(hi.y) - lo.y + 3, sz = int64_t(hi.z) - lo.z + 3;
    int64_t volume = sx * sy * sz;
    if (volume > int64_t(64) * int64_t(k) + 4096 || volume >= (int64_t(1) << 24)) return SLF_OK;
    mlow = make_int3(lo.x - 1, lo.y - 1, lo.z - 1);
    mspan = make_int3(int(sx), int(sy), int(sz));
    mvolume = uint32_t(volume);
    std::vector<float4> hs(k), hv(k);
    for (size_t i = 0; i < k; ++i) {
        uint32_t bits = m_own[i];
        float w;
        std::memcpy(&w, &bits, 4);
        hs[i] = make_float4(m_start[i].x, m_start[i].y, m_start[i].z, w);
        hv[i] = make_float4(m_vel[i].x, m_vel[i].y, m_vel[i].z, 0.0f);
    }
    for (auto* b : {&dmcur_start, &dmcur_vel, &dmnext_start, &dmnext_vel, &dmpos}) SLF_TRY(b->ensure(k, 0, stream));
    for (auto* b : {&dmlin, &dmslot, &dmmembers}) SLF_TRY(b->ensure(k, 0, stream));
    SLF_TRY(dmtable.ensure(size_t(mvolume) + 1, 0, stream));
    SLF_TRY(dmtable_tiles.ensure(scan_tiles(mvolume) + 1, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(dmcur_start.p, hs.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(dmcur_vel.p, hv.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaStreamSynchronize(stream));  // the staging vectors are pageable and freed next
    mdevice = true;
    return SLF_OK;
}

int32_t World::carry_movers(float elapsed, float last) {
    if (elapsed == 0.0f) SLF_TRY(plan_movers(last));
    size_t k = m_start.size();
    if (k && mdevice) {
        for (auto& known : coupled) known.moved = known.velocity * elapsed;
        launch_carry_movers(params(), uint32_t(k), dmcur_start.p, dmcur_vel.p, elapsed, mlow, mspan, mvolume, dmlin.p,
                            dmslot.p, dmtable.p, dmtable_tiles.p, dmmembers.p, dmnext_start.p, dmnext_vel.p, dmpos.p,
                            stream);
        std::swap(dmcur_start, dmnext_start);
        std::swap(dmcur_vel, dmnext_vel);
        // the sorted velocities: dmcur_vel now; the grid: the dense table over the step's box
        mgrid = GridDev{};
        mgrid.mode = 1;
        mgrid.lx = mlow.x;
        mgrid.ly = mlow.y;
        mgrid.lz = mlow.z;
        mgrid.sx = mspan.x;
        mgrid.sy = mspan.y;
        mgrid.sz = mspan.z;
        mgrid.start = dmtable.p;
        return SLF_OK;
    }
    struct MK {
        Key3 cell;
        uint32_t owner;
        size_t index;
    };
    std::vector<MK> order(k);
    for (size_t i = 0; i < k; ++i) {
        F3 at = m_start[i] + m_vel[i] * elapsed;
        m_pos[i] = at;
        order[i] = MK{cell_of(at), m_own[i], i};
    }
    std::sort(order.begin(), order.end(), [](const MK& a, const MK& b) {
        return std::tie(a.cell.x, a.cell.y, a.cell.z, a.owner, a.index) <
               std::tie(b.cell.x, b.cell.y, b.cell.z, b.owner, b.index);
    });
    std::vector<F3> st(k), ps(k), vs(k);
    std::vector<uint32_t> ow(k);
    std::vector<Key3> keys(k);
    for (size_t i = 0; i < k; ++i) {
        size_t j = order[i].index;
        st[i] = m_start[j];
        ps[i] = m_pos[j];
        vs[i] = m_vel[j];
        ow[i] = m_own[j];
        keys[i] = order[i].cell;
    }
    m_start = std::move(st);
    m_pos = std::move(ps);
    m_vel = std::move(vs);
    m_own = std::move(ow);
    for (auto& known : coupled) known.moved = known.velocity * elapsed;
    if (!k) {
        mgrid = GridDev{};
        return SLF_OK;
    }
    std::vector<float4> hp(k), hv(k);
    for (size_t i = 0; i < k; ++i) {
        uint32_t bits = m_own[i];
        float w;
        std::memcpy(&w, &bits, 4);
        hp[i] = make_float4(m_pos[i].x, m_pos[i].y, m_pos[i].z, w);
        hv[i] = make_float4(m_vel[i].x, m_vel[i].y, m_vel[i].z, 0.0f);
    }
    SLF_TRY(dmpos.ensure(k, 0, stream));
    SLF_TRY(dmvel.ensure(k, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(dmpos.p, hp.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(dmvel.p, hv.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_TRY(grid_from_keys(keys, mgrid, dmstart, dmkeys));  // waits for the copies
    return SLF_OK;
}

int32_t World::fastest_near_water(float dt, float slow, float& most) {
    most = 0.0f;
    size_t count = coupled.size();
    if (!count || m_pos.empty()) return SLF_OK;
    std::vector<float> fastest_of(count, 0.0f);
    std::vector<F3> lows(count, F3{FLT_MAX, FLT_MAX, FLT_MAX}), highs(count, F3{-FLT_MAX, -FLT_MAX, -FLT_MAX});
    for (size_t i = 0; i < m_pos.size(); ++i) {
        size_t owner = m_own[i];
        fastest_of[owner] = rmax(fastest_of[owner], length(m_vel[i]));
        lows[owner] = vmin(lows[owner], m_pos[i]);
        highs[owner] = vmax(highs[owner], m_pos[i]);
    }
    float water = fastest();
    for (size_t b = 0; b < count; ++b) {
        float speed = fastest_of[b];
        if (speed <= most) continue;
        if (speed <= slow) {
            most = speed;
            continue;
        }
        float reach = radius + (speed + water) * dt;
        Key3 lo = cell_of(lows[b] - F3{reach, reach, reach}), hi = cell_of(highs[b] + F3{reach, reach, reach});
        // before the first sort there is no table to ask, any water counts
        bool wet = fgrid.mode == 0 && n > 0;
        if (!wet && fgrid.mode != 0) {
            SLF_TRY(dwet.ensure(1, 0, stream));
            SLF_CUDA(cudaMemsetAsync(dwet.p, 0, 4, stream));
            launch_cells_wet(fgrid, make_int3(lo.x, lo.y, lo.z), make_int3(hi.x, hi.y, hi.z), dwet.p, stream);
            uint32_t flag = 0;
            SLF_CUDA(cudaMemcpyAsync(&flag, dwet.p, 4, cudaMemcpyDeviceToHost, stream));
            SLF_TRY(sync());
            wet = flag != 0;
        }
        if (wet) most = speed;
    }
    return SLF_OK;
}

int32_t World::mover_felt(float dt, const Params& p, int a, int nid) {
    if (coupled.empty() || m_pos.empty() || n == 0) return SLF_OK;
    size_t bodies = coupled.size(), chunks = (n + 511) / 512;
    std::vector<float4> centres(bodies);
    for (size_t b = 0; b < bodies; ++b) {
        F3 o = coupled[b].center + coupled[b].moved;
        centres[b] = make_float4(o.x, o.y, o.z, 0.0f);
    }
    SLF_TRY(dcentre.ensure(bodies, 0, stream));
    SLF_TRY(dfelt.ensure(2 * chunks * bodies, 0, stream));
    SLF_TRY(dmcount.ensure(n + 1, 0, stream));
    SLF_TRY(dmtiles.ensure(scan_tiles(uint32_t(n)) + 1, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(dcentre.p, centres.data(), bodies * sizeof(float4), cudaMemcpyHostToDevice, stream));
    launch_mover_count(p, d_consts, mover_dev(), pos[a].p, vel[a].p, rho[nid].p, press.p, scaled.p, dmcount.p,
                       stream);
    launch_exclusive_scan(dmcount.p, uint32_t(n), dmtiles.p, stream);
    uint32_t total = 0;
    SLF_CUDA(cudaMemcpyAsync(&total, dmcount.p + n, 4, cudaMemcpyDeviceToHost, stream));
    SLF_TRY(sync());
    SLF_TRY(dmpair.ensure(2 * size_t(std::max<uint32_t>(total, 1)), 0, stream));
    launch_mover_felt(p, d_consts, mover_dev(), pos[a].p, vel[a].p, rho[nid].p, press.p, scaled.p, dcentre.p,
                      uint32_t(bodies), dmcount.p, dmpair.p, dfelt.p, stream);
    // folded on the device into the step's impulses, read once when the step ends
    launch_mover_fold(uint32_t(n), uint32_t(bodies), dfelt.p, dt, dimpulse.p, stream);
    return SLF_OK;
}

void World::lift_region(const Coupled& known, const slf_body_pose& state, std::vector<std::pair<F3, F3>>& probes,
                        F3& low, F3& high) const {
    float reach = 3.0f * radius;
    F3 center = center_of(state), lin = f3v(state.linear_velocity), ang = f3v(state.angular_velocity);
    probes.clear();
    for (const F3& local : known.probes) {
        F3 arm = rotate(state.rotation, local);
        probes.push_back({arm, lin + cross(ang, arm)});
    }
    low = F3{FLT_MAX, FLT_MAX, FLT_MAX};
    high = F3{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (auto& pr : probes) {
        low = vmin(low, center + pr.first);
        high = vmax(high, center + pr.first);
    }
    low = low - F3{reach, reach, reach};
    high = high + F3{reach, reach, reach};
}

int32_t World::read_lift_water(const std::vector<float3>& boxes, std::vector<uint32_t>& index, std::vector<F3>& P,
                               std::vector<F3>& V) {
    index.clear();
    P.clear();
    V.clear();
    if (!n || boxes.empty()) return SLF_OK;
    const uint32_t m = uint32_t(n);
    SLF_TRY(lboxes.ensure(boxes.size(), 0, stream));
    SLF_TRY(lkeep.ensure(m, 0, stream));
    SLF_TRY(lat.ensure(size_t(m) + 1, 0, stream));
    SLF_TRY(ltiles.ensure(scan_tiles(m) + 1, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(lboxes.p, boxes.data(), boxes.size() * sizeof(float3), cudaMemcpyHostToDevice, stream));
    launch_in_boxes(m, pos[cpos].p, lboxes.p, uint32_t(boxes.size() / 2), lkeep.p, stream);
    SLF_CUDA(cudaMemcpyAsync(lat.p, lkeep.p, size_t(m) * 4, cudaMemcpyDeviceToDevice, stream));
    launch_exclusive_scan(lat.p, m, ltiles.p, stream);
    uint32_t kept = 0;
    SLF_CUDA(cudaMemcpyAsync(&kept, lat.p + m, 4, cudaMemcpyDeviceToHost, stream));
    SLF_TRY(sync());
    if (!kept) return SLF_OK;
    SLF_TRY(lidx.ensure(kept, 0, stream));
    SLF_TRY(lpv.ensure(size_t(6) * kept, 0, stream));
    launch_gather_kept(m, lkeep.p, lat.p, pos[cpos].p, vel[cpos].p, lidx.p, lpv.p, stream);
    index.resize(kept);
    std::vector<float> pv(size_t(6) * kept);
    SLF_CUDA(cudaMemcpyAsync(index.data(), lidx.p, size_t(kept) * 4, cudaMemcpyDeviceToHost, stream));
    SLF_CUDA(cudaMemcpyAsync(pv.data(), lpv.p, pv.size() * 4, cudaMemcpyDeviceToHost, stream));
    SLF_TRY(sync());
    P.resize(kept);
    V.resize(kept);
    for (uint32_t k = 0; k < kept; ++k) {
        const float* o = pv.data() + 6 * size_t(k);
        P[k] = F3{o[0], o[1], o[2]};
        V[k] = F3{o[3], o[4], o[5]};
    }
    return SLF_OK;
}

int32_t World::write_lift_velocities(const std::vector<F3>& V) {
    if (V.empty()) return SLF_OK;
    std::vector<float> v3(3 * V.size());
    for (size_t k = 0; k < V.size(); ++k) {
        v3[3 * k] = V[k].x;
        v3[3 * k + 1] = V[k].y;
        v3[3 * k + 2] = V[k].z;
    }
    SLF_CUDA(cudaMemcpyAsync(lpv.p, v3.data(), v3.size() * 4, cudaMemcpyHostToDevice, stream));
    launch_scatter_velocities(uint32_t(V.size()), lidx.p, lpv.p, vel[cpos].p, stream);
    return sync();
}

auto World::lifts(float dt, const slf_body_pose* poses, uint64_t npose, const std::vector<F3>& P,
                  const std::vector<F3>& V) const -> std::vector<Lift> {
    F3 g{s.gravity[0], s.gravity[1], s.gravity[2]};
    float grav = length(g);
    F3 up = grav > 0.0f ? (-g) / grav : F3{0.0f, 1.0f, 0.0f};
    float column = radius;
    std::vector<Lift> out;
    std::vector<std::pair<F3, F3>> probes;
    for (size_t owner = 0; owner < coupled.size(); ++owner) {
        const Coupled& known = coupled[owner];
        const slf_body_pose* state = pose_of(poses, npose, known.body);
        if (!state) continue;
        F3 center = center_of(*state);
        F3 low, high;
        lift_region(known, *state, probes, low, high);
        std::vector<uint32_t> near;
        for (size_t i = 0; i < P.size(); ++i)
            if (vmin(vmax(P[i], low), high) == P[i]) near.push_back(uint32_t(i));
        if (near.empty()) continue;
        // the level is the middle of the columns' tops
        struct Top {
            int32_t kx, kz;
            float h;
        };
        std::vector<Top> tops;
        for (uint32_t i : near)
            tops.push_back(Top{sat_i32(std::floor(P[i].x / column)), sat_i32(std::floor(P[i].z / column)),
                               dot(P[i], up)});
        std::sort(tops.begin(), tops.end(), [](const Top& a, const Top& b) {
            if (a.kx != b.kx) return a.kx < b.kx;
            if (a.kz != b.kz) return a.kz < b.kz;
            return total_less(b.h, a.h);
        });
        std::vector<float> heights;
        for (size_t k = 0; k < tops.size(); ++k)
            if (k == 0 || tops[k].kx != tops[k - 1].kx || tops[k].kz != tops[k - 1].kz) heights.push_back(tops[k].h);
        std::sort(heights.begin(), heights.end(), total_less);
        size_t quarter = heights.size() / 4;
        float sum = 0.0f;
        for (size_t k = quarter; k < heights.size() - quarter; ++k) sum += heights[k];
        float level = sum / float(heights.size() - 2 * quarter) + s.spacing / 2.0f;
        F3 flow{0, 0, 0};
        uint32_t wet = 0;
        for (uint32_t i : near)
            if (dot(P[i], up) <= level) {
                flow = flow + V[i];
                ++wet;
            }
        flow = flow / float(std::max<uint32_t>(wet, 1));
        float spacing = known.probe_spacing;
        struct Under {
            F3 arm, velocity;
            float share;
        };
        std::vector<Under> under;
        for (auto& pr : probes) {
            float depth = level - dot(center + pr.first, up);
            float share = rmin(rmax(depth / spacing + 0.5f, 0.0f), 1.0f);
            if (share > 0.0f) under.push_back(Under{pr.first, pr.second, share});
        }
        float wetted = 0.0f;
        for (auto& u : under) wetted += u.share;
        if (wetted <= 0.0f) continue;
        float volume = wetted * (spacing * spacing * spacing);
        float density = s.rest_density;
        F3 middle{0, 0, 0};
        for (auto& u : under) middle = middle + u.arm * u.share;
        middle = middle / wetted;
        F3 force{0, 0, 0}, torque{0, 0, 0};
        F3 buoyancy = up * (density * grav * volume);
        force = force + buoyancy;
        torque = torque + cross(middle, buoyancy);
        float area = std::pow(volume, 2.0f / 3.0f) / wetted;
        for (auto& u : under) {
            F3 past = flow - u.velocity;
            F3 drag = past * (0.5f * 1.0f * density * area * u.share * length(past));
            force = force + drag;
            torque = torque + cross(u.arm, drag);
        }
        size_t nline = 0;
        for (auto& u : under) nline += u.share < 1.0f ? 1 : 0;
        float plane = float(nline) * spacing * spacing;
        float waves = density * plane * std::sqrt(grav * std::sqrt(plane));
        float share = waves / float(std::max<size_t>(nline, 1));
        for (auto& u : under) {
            if (!(u.share < 1.0f)) continue;
            F3 calm = up * (share * dot(flow - u.velocity, up));
            force = force + calm;
            torque = torque + cross(u.arm, calm);
        }
        out.push_back(Lift{owner, force * dt, torque * dt, std::move(near)});
    }
    return out;
}

int32_t World::step_with_bodies(float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out,
                                std::vector<slf_body_push>& pushes) {
    pushes.clear();
    if (s.solver != SLF_SOLVER_WCSPH && !coupled.empty())
        return fail(SLF_ERR_INVALID_SETTINGS, "the divergence free solver does not couple yet");
    if (!coupled.empty() && fast()) return fail(SLF_ERR_UNSUPPORTED, "coupled bodies run with EXACT arithmetic only");
    if (tape.on && !coupled.empty()) {
        // the adjoint takes bodies on the paths the caller gives, substep by substep as recorded
        if (tape.every != 0)
            return fail(SLF_ERR_UNSUPPORTED, "a tape with coupled bodies records every substep (checkpoint_every 0)");
        for (const Coupled& known : coupled) {
            const slf_body_pose* state = pose_of(poses, npose, known.body);
            if (state && state->dynamic)
                return fail(SLF_ERR_UNSUPPORTED,
                            "the adjoint takes no dynamic body: its lift gives momentum back to the water");
        }
    }
    place_movers_at(poses, npose);
    if (!coupled.empty()) {
        SLF_TRY(dimpulse.ensure(2 * coupled.size(), 0, stream));
        SLF_CUDA(cudaMemsetAsync(dimpulse.p, 0, 2 * coupled.size() * sizeof(float4), stream));
    }
    int32_t st = step(dt, out);
    if (st == SLF_OK && !coupled.empty()) {  // the damping the bodies took, as the substeps folded it
        std::vector<float4> imp(2 * coupled.size());
        SLF_CUDA(cudaMemcpyAsync(imp.data(), dimpulse.p, imp.size() * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        SLF_TRY(sync());
        for (size_t b = 0; b < coupled.size(); ++b) {
            coupled[b].impulse = F3{imp[2 * b].x, imp[2 * b].y, imp[2 * b].z};
            coupled[b].angular = F3{imp[2 * b + 1].x, imp[2 * b + 1].y, imp[2 * b + 1].z};
        }
    }
    // the points are gone for the next step
    m_start.clear();
    m_pos.clear();
    m_vel.clear();
    m_own.clear();
    mgrid = GridDev{};
    SLF_TRY(st);
    for (auto& known : coupled) {
        slf_body_push p{};
        p.body = known.body;
        pushes.push_back(p);
    }
    if (!(dt > 0.0f) || coupled.empty()) return SLF_OK;
    // the water the lifts read: the particles inside the bodies' regions, in index order
    std::vector<float3> boxes;
    std::vector<std::pair<F3, F3>> probes;
    for (const Coupled& known : coupled) {
        const slf_body_pose* state = pose_of(poses, npose, known.body);
        if (!state) continue;
        F3 low, high;
        lift_region(known, *state, probes, low, high);
        boxes.push_back(make_float3(low.x, low.y, low.z));
        boxes.push_back(make_float3(high.x, high.y, high.z));
    }
    std::vector<uint32_t> index;
    std::vector<F3> P, V;
    SLF_TRY(read_lift_water(boxes, index, P, V));
    auto put = [](float* d, F3 v) {
        d[0] = v.x;
        d[1] = v.y;
        d[2] = v.z;
    };
    bool gave = false;
    for (const Lift& lift : lifts(dt, poses, npose, P, V)) {
        slf_body_push& p = pushes[lift.owner];
        put(p.lift, lift.impulse);
        put(p.lift_angular, lift.angular);
        if (pose_of(poses, npose, coupled[lift.owner].body)->dynamic) {
            // lift.rs:160-166: the water read for the lift loses what the body got
            F3 change = lift.impulse / (mass * float(lift.near.size()));
            for (uint32_t i : lift.near) V[i] = V[i] - change;
            p.lifted = 1;
            gave = true;
        }
    }
    for (size_t b = 0; b < coupled.size(); ++b) {
        put(pushes[b].damping, coupled[b].impulse);
        put(pushes[b].damping_angular, coupled[b].angular);
        coupled[b].impulse = coupled[b].angular = F3{0, 0, 0};
    }
    if (gave) {
        SLF_TRY(write_lift_velocities(V));
        stats_fresh = false;
    }
    return SLF_OK;
}

}  // namespace slf
