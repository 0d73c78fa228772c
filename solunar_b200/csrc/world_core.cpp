// world_core.cpp -- World's settings, particles, status, the spatial hash and read-outs of the world.
#include "world.h"

namespace slf {

bool World::valid(const slf_settings& s) {
    auto positive = [](float v) { return std::isfinite(v) && v > 0.0f; };
    bool support = s.support >= 1.5f && s.support <= 4.0f;
    return (s.solver == SLF_SOLVER_WCSPH || s.solver == SLF_SOLVER_DFSPH) && positive(s.spacing) &&
           positive(s.rest_density) && support && s.max_particles > 0 && positive(s.sound_speed) &&
           std::isfinite(s.viscosity) && s.viscosity >= 0.0f && finite3(s.gravity) && s.courant > 0.0f &&
           s.courant <= 1.0f && s.max_substeps > 0 && s.min_iterations <= s.max_iterations &&
           std::isfinite(s.divergence_tolerance) && std::isfinite(s.density_tolerance);
}

float World::rest_mass() const {
    HostKernel k(radius);
    int reach = int(std::ceil(s.support));
    float sum = 0.0f;
    for (int z = -reach; z <= reach; ++z)
        for (int y = -reach; y <= reach; ++y)
            for (int x = -reach; x <= reach; ++x) {
                float ox = float(x) * s.spacing, oy = float(y) * s.spacing, oz = float(z) * s.spacing;
                sum += k.value(std::sqrt(ox * ox + oy * oy + oz * oz));
            }
    return s.rest_density / sum;
}

int32_t World::init(const slf_settings& settings) {
    s = settings;
    radius = s.spacing * s.support;
    HostKernel k(radius);
    scale = k.scale;
    mass = rest_mass();
    // lists hold half again the neighbours of a rest lattice, plus slack; a longer one makes
    // the substep run again with more room
    double expected = 4.0 / 3.0 * 3.14159265358979 * double(s.support) * s.support * s.support;
    list_cap = (uint32_t(expected * 1.5 + 16.0) + 7u) & ~7u;
    SLF_CUDA(cudaSetDevice(s.device));
    // device memory freed on the world's stream stays in this process's default pool for the
    // next allocation (tapes, list growth) instead of going back at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s.device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    SLF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SLF_CUDA(cudaMalloc(&d_status, sizeof(Status)));
    SLF_CUDA(cudaMalloc(&d_consts, sizeof(StepConsts)));
    SLF_CUDA(cudaMallocHost(&h_status, sizeof(Status)));
    std::memset(h_status, 0, sizeof(Status));
    SLF_CUDA(cudaMallocHost(&h_reset, sizeof(Status)));
    *h_reset = fresh_status();
    SLF_CUDA(cudaMemsetAsync(d_status, 0, sizeof(Status), stream));
    build_ground_sites();
    return SLF_OK;
}

void World::build_ground_sites() {
    HostKernel k(radius);
    const float spacing = s.spacing;
    int reach = int(std::ceil(radius / spacing));
    site_host.clear();
    far_host.clear();
    for (int z = -reach; z <= reach; ++z)
        for (int y = -reach; y <= reach; ++y)
            for (int x = -reach; x <= reach; ++x) {
                float ox = float(x) * spacing, oy = float(y) * spacing, oz = float(z) * spacing;
                float far = std::sqrt(ox * ox + oy * oy + oz * oz);
                if (far < radius) {
                    site_host.push_back(make_float4(ox, oy, oz, mass * k.value(far)));
                    far_host.push_back(far);
                }
            }
    ground_low = -spacing / 2.0f;
    ground_step = (radius - ground_low) / float(kGroundSamples - 1);
    float soften = 0.01f * radius * radius;
    int across_reach = reach + 1;
    damping_host.assign(kGroundSamples, 0.0f);
    for (int sample = 0; sample < kGroundSamples; ++sample) {
        float distance = ground_low + ground_step * float(sample);
        float weight = 0.0f;
        for (int layer = 0;; ++layer) {
            float depth = distance + spacing * (float(layer) + 0.5f);
            if (depth >= radius) break;
            for (int a = -across_reach; a <= across_reach; ++a)
                for (int b = -across_reach; b <= across_reach; ++b) {
                    float across = float(a * a + b * b) * spacing * spacing;
                    float squared = across + depth * depth;
                    float far = std::sqrt(squared);
                    if (far >= radius || far <= 0.0f) continue;
                    weight += mass * depth * depth * -k.slope(far) / (far * (squared + soften));
                }
        }
        damping_host[sample] = weight;
    }
    ground_reach = radius + spacing / 2.0f;
}

int32_t World::upload_terrain() {
    if (!terrain_dirty) return SLF_OK;
    tdev = TerrainDev{};
    terrain_dirty = false;
    if (terrains.empty()) return SLF_OK;
    std::vector<TerrainRegion> regions;
    std::vector<float> dist;
    for (const TerrainHost& t : terrains) {
        TerrainRegion r{};
        r.lx = t.low.x;
        r.ly = t.low.y;
        r.lz = t.low.z;
        r.step = t.step;
        r.nx = t.nx;
        r.ny = t.ny;
        r.nz = t.nz;
        r.offset = dist.size();
        regions.push_back(r);
        dist.insert(dist.end(), t.distances.begin(), t.distances.end());
    }
    SLF_TRY(dregions.ensure(regions.size(), 0, stream));
    SLF_TRY(ddist.ensure(dist.size(), 0, stream));
    SLF_TRY(dsites.ensure(site_host.size(), 0, stream));
    SLF_TRY(dfar.ensure(far_host.size(), 0, stream));
    SLF_TRY(ddamping.ensure(kGroundSamples, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(dregions.p, regions.data(), regions.size() * sizeof(TerrainRegion),
                             cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(ddist.p, dist.data(), dist.size() * 4, cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(dsites.p, site_host.data(), site_host.size() * sizeof(float4), cudaMemcpyHostToDevice,
                             stream));
    SLF_CUDA(cudaMemcpyAsync(dfar.p, far_host.data(), far_host.size() * 4, cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(ddamping.p, damping_host.data(), kGroundSamples * 4, cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaStreamSynchronize(stream));  // the host vectors are pageable and local
    tdev.regions = uint32_t(regions.size());
    tdev.sites = uint32_t(site_host.size());
    tdev.region = dregions.p;
    tdev.dist = ddist.p;
    tdev.site = dsites.p;
    tdev.far = dfar.p;
    tdev.damping = ddamping.p;
    tdev.spacing = s.spacing;
    tdev.reach = ground_reach;
    tdev.low = ground_low;
    tdev.step = ground_step;
    return SLF_OK;
}

float4* World::ground_slopes() {
    if (terrains.empty()) return nullptr;
    if (gslope.ensure(std::max<uint64_t>(n, 1), 0, stream) != SLF_OK) return nullptr;
    return gslope.p;
}

int32_t World::terrain_nodes(const float* low, const float* high, uint64_t nodes[3]) const {
    if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in terrain box");
    if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
        return fail(SLF_ERR_OUT_OF_RANGE, "inside out terrain box");
    float step = s.spacing / 2.0f;
    for (int a = 0; a < 3; ++a) nodes[a] = uint64_t(rmin(std::ceil((high[a] - low[a]) / step), 1e7f)) + 1;
    unsigned __int128 total = (unsigned __int128)nodes[0] * nodes[1] * nodes[2];
    if (total > kMaxTerrainNodes) return fail(SLF_ERR_FLUID_FULL, "terrain region holds too many nodes");
    return SLF_OK;
}

int32_t World::add_terrain(const float* low, const float* high, const float* distances, uint64_t count, uint32_t* out) {
    if (fast()) return fail(SLF_ERR_UNSUPPORTED, "terrain runs with EXACT arithmetic only");
    if (tape.on) return fail(SLF_ERR_UNSUPPORTED, "terrain is added before a tape begins, not while it records");
    uint64_t nodes[3];
    SLF_TRY(terrain_nodes(low, high, nodes));
    if (count != nodes[0] * nodes[1] * nodes[2])
        return fail(SLF_ERR_INVALID_ARGUMENT, "distances must hold one value per terrain node");
    for (uint64_t i = 0; i < count; ++i)
        if (!std::isfinite(distances[i])) return fail(SLF_ERR_NON_FINITE, "non finite terrain distance");
    TerrainHost t;
    t.low = F3{low[0], low[1], low[2]};
    t.nx = uint32_t(nodes[0]);
    t.ny = uint32_t(nodes[1]);
    t.nz = uint32_t(nodes[2]);
    t.step = s.spacing / 2.0f;
    t.distances.assign(distances, distances + count);
    t.owner = add_wall_points({});
    terrains.push_back(std::move(t));
    terrain_dirty = true;
    lists_valid = false;
    if (out) *out = terrains.back().owner;
    return SLF_OK;
}

Params World::params() const {
    Params p{};
    p.spacing = s.spacing;
    p.radius = radius;
    p.reach = radius * radius;
    p.scale = scale;
    p.mass = mass;
    p.rest = s.rest_density;
    p.rest_sq = s.rest_density * s.rest_density;
    p.stiffness = s.rest_density * (s.sound_speed * s.sound_speed) / 7.0f;
    p.soften = 0.01f * radius * radius;
    p.gravity = make_float3(s.gravity[0], s.gravity[1], s.gravity[2]);
    p.has_bounds = has_bounds ? 1 : 0;
    float half = s.spacing / 2.0f;
    p.low = make_float3(blow.x, blow.y, blow.z);
    p.high = make_float3(bhigh.x, bhigh.y, bhigh.z);
    p.low_in = make_float3(blow.x + half, blow.y + half, blow.z + half);
    p.high_in = make_float3(bhigh.x - half, bhigh.y - half, bhigh.z - half);
    p.n = uint32_t(n);
    p.solver = s.solver;
    p.div_tol = s.divergence_tolerance;
    p.den_tol = s.density_tolerance;
    p.min_iter = s.min_iterations;
    p.max_iter = s.max_iterations;
    p.inv_radius = 1.0f / radius;
    p.grad_scale = scale * -20.0f / (radius * radius);
    p.inv_rest = 1.0f / s.rest_density;
    p.inv_rest_sq = 1.0f / (s.rest_density * s.rest_density);
    p.settles = std::sqrt(s.gravity[0] * s.gravity[0] + s.gravity[1] * s.gravity[1] + s.gravity[2] * s.gravity[2]) *
                s.spacing;
    return p;
}

StepConsts World::consts(float dt) const {
    StepConsts c{};
    c.dt = dt;
    c.viscosity = rmin(s.viscosity * s.sound_speed * radius, 0.05f * radius * radius / dt);
    float stable = radius * radius / dt;
    c.wall_viscosity = rmin(1.0f * s.sound_speed * radius, 0.25f * stable);
    c.dt_sq = dt * dt;
    c.mover_damping = rmin(1.0f * s.sound_speed * radius, 0.25f * radius * radius / dt);
    return c;
}

int32_t World::add(uint64_t k, const float* p, const float* v, uint32_t* ids_out) {
    for (uint64_t i = 0; i < k; ++i)
        if (!finite3(p + 3 * i) || !finite3(v + 3 * i)) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid particle");
    if (total() + k > s.max_particles || uint64_t(next_id) + k > uint64_t(UINT32_MAX) ||
        total() + k > index_limit())
        return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    for (uint64_t i = 0; i < k; ++i) {
        pend_pos.push_back(make_float4(p[3 * i], p[3 * i + 1], p[3 * i + 2], 0.0f));
        pend_vel.push_back(make_float4(v[3 * i], v[3 * i + 1], v[3 * i + 2], 0.0f));
        if (ids_out) ids_out[i] = next_id;
        pend_ids.push_back(next_id++);
    }
    return SLF_OK;
}

int32_t World::fill_box(const float* low, const float* high, uint64_t* count_out) {
    if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid box");
    if (high[0] < low[0] || high[1] < low[1] || high[2] < low[2])
        return fail(SLF_ERR_OUT_OF_RANGE, "inside out fluid box");
    float spacing = s.spacing;
    auto count = [&](float extent) -> uint64_t {
        float c = rmin(std::floor(extent / spacing), 4294967295.0f);
        if (std::isnan(c) || c <= 0.0f) return 0;
        return uint64_t(c);
    };
    float sx = high[0] - low[0], sy = high[1] - low[1], sz = high[2] - low[2];
    uint64_t nx = count(sx), ny = count(sy), nz = count(sz);
    auto sat_mul = [](uint64_t a, uint64_t b) -> uint64_t {
        unsigned __int128 q = (unsigned __int128)a * b;
        return q > UINT64_MAX ? UINT64_MAX : uint64_t(q);
    };
    uint64_t tot = sat_mul(sat_mul(nx, ny), nz);
    uint64_t room = s.max_particles > total() ? s.max_particles - total() : 0;
    uint64_t ids_left = uint64_t(UINT32_MAX - next_id);
    if (index_limit() > total()) room = std::min<uint64_t>(room, index_limit() - total());
    else room = 0;
    if (tot > room || tot > ids_left) return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    float half = spacing * 0.5f;
    float st[3] = {low[0] + half, low[1] + half, low[2] + half};
    std::vector<float> pts;
    pts.reserve(size_t(tot) * 3);
    for (uint64_t y = 0; y < ny; ++y)
        for (uint64_t z = 0; z < nz; ++z)
            for (uint64_t x = 0; x < nx; ++x) {
                pts.push_back(st[0] + float(x) * spacing);
                pts.push_back(st[1] + float(y) * spacing);
                pts.push_back(st[2] + float(z) * spacing);
            }
    std::vector<float> zeros(pts.size(), 0.0f);
    SLF_TRY(add(tot, pts.data(), zeros.data(), nullptr));
    if (count_out) *count_out = tot;
    return SLF_OK;
}

int32_t World::flush() {
    if (pend_ids.empty()) return SLF_OK;
    uint64_t k = pend_ids.size();
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
    if (rel()) {
        // absolute positions land in a free slot, then become offsets and cells
        float4* tmp = pos[(cpos + 1) % 3].p;
        SLF_CUDA(cudaMemcpyAsync(tmp, pend_pos.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
        launch_to_relative(params(), uint32_t(k), nullptr, tmp, pos[cpos].p + n, cell[cpos].p + n, stream);
    } else {
        SLF_CUDA(cudaMemcpyAsync(pos[cpos].p + n, pend_pos.data(), k * sizeof(float4), cudaMemcpyHostToDevice,
                                 stream));
    }
    SLF_CUDA(cudaMemcpyAsync(vel[cpos].p + n, pend_vel.data(), k * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(ids[cid].p + n, pend_ids.data(), k * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemsetAsync(rho[cid].p + n, 0, k * sizeof(float), stream));
    if (warm_on()) SLF_CUDA(cudaMemsetAsync(warm[cid].p + n, 0, k * sizeof(float2), stream));
    SLF_CUDA(cudaStreamSynchronize(stream));  // the staging vectors are pageable and freed next
    pend_pos.clear();
    pend_vel.clear();
    pend_ids.clear();
    n = m;
    lists_valid = false;
    stats_fresh = false;
    return SLF_OK;
}

int32_t World::ensure_work_buffers() {
    prepare_solver_grids();
    if (fast()) prepare_fast_grids();
    SLF_TRY(press.ensure(n, 0, stream));
    SLF_TRY(scaled.ensure(n, 0, stream));
    SLF_TRY(alpha.ensure(n, 0, stream));
    size_t slots = PairLists::slots_for(uint32_t(n), list_cap);
    SLF_TRY(fent.ensure(slots, 0, stream));
    SLF_TRY(went.ensure(slots, 0, stream));
    if (keeps_gradients()) {
        SLF_TRY(fgv.ensure(slots, 0, stream));
        SLF_TRY(wgv.ensure(slots, 0, stream));
    }
    SLF_TRY(fcnt.ensure(n, 0, stream));
    SLF_TRY(wcnt.ensure(n, 0, stream));
    SLF_TRY(lin.ensure(n, 0, stream));
    SLF_TRY(cslot.ensure(n, 0, stream));
    SLF_TRY(members.ensure(n, 0, stream));
    SLF_TRY(partials.ensure(rate_partial_bytes(uint32_t(n)), 0, stream));
    return SLF_OK;
}

void World::density_pass(const Params& p, int a, const PairLists& fl, const PairLists& wl, float* rh, cudaStream_t on) {
    if (!on) on = stream;
    if (fast())
        launch_density_fast(p, fgrid, wgrid, pos[a].p, cells_of(a), dwalls.p, fl, wl, rh, press.p, scaled.p,
                            alpha.p, d_status, on);
    else
        launch_density(p, fgrid, wgrid, pos[a].p, dwalls.p, fl, wl, rh, press.p, scaled.p, alpha.p, d_status,
                       tdev, ground_slopes(), on, mover_dev());
}

void World::force_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid, cudaStream_t on) {
    if (!on) on = stream;
    if (fast())
        launch_wcsph_force_fast(p, d_consts, fl, wl, pos[a].p, cells_of(a), vel[a].p, rho[nid].p, press.p,
                                scaled.p, dwalls.p, pos[b].p, cells_of(b), vel[b].p, d_status, vel_pre, on);
    else
        launch_wcsph_force(p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, press.p, scaled.p, dwalls.p,
                           pos[b].p, vel[b].p, d_status, vel_pre, tdev, terrains.empty() ? nullptr : gslope.p,
                           on, mover_dev());
}

void World::rate_pass(int which, const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v, int nid,
                      SolveRec rec, cudaStream_t cs, unsigned long long loop) {
    cudaStream_t on = cs ? cs : stream;
    if (fast())
        launch_rate_fast(which, rel(), p, d_consts, fl, wl, pos[a].p, v, rho[nid].p, alpha.p, dwalls.p,
                         partials.p, d_status, rec, on, loop);
    else
        launch_rate(which, p, d_consts, fl, wl, pos[a].p, v, rho[nid].p, alpha.p, dwalls.p, partials.p, d_status,
                    rec, on, loop);
}

void World::push_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v, float* applied,
                      cudaStream_t cs, unsigned long long loop) {
    cudaStream_t on = cs ? cs : stream;
    if (fast()) launch_push_fast(rel(), p, d_consts, fl, wl, pos[a].p, v, dwalls.p, d_status, applied, on, loop);
    else launch_push(p, d_consts, fl, wl, pos[a].p, v, dwalls.p, d_status, applied, on, loop);
}

void World::advance_pass(const Params& p, int a, int b, float4* pre, cudaStream_t on) {
    if (!on) on = stream;
    if (rel()) launch_advance_rel(p, d_consts, pos[a].p, cell[a].p, pos[b].p, cell[b].p, vel[b].p, d_status, pre,
                                  on);
    else launch_advance(p, d_consts, pos[a].p, pos[b].p, vel[b].p, d_status, pre, on);
}

void World::viscous_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid,
                         cudaStream_t on) {
    if (!on) on = stream;
    if (fast())
        launch_viscous_fast(rel(), p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, dwalls.p, vel[b].p,
                            on);
    else
        launch_viscous(p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, dwalls.p, vel[b].p, on);
}

int32_t World::lists_fit() {
    if (h_status->list_max <= list_cap) return SLF_OK;
    list_cap = (uint32_t(h_status->list_max) + h_status->list_max / 4 + 15u) & ~7u;
    SLF_TRY(ensure_work_buffers());
    stats_fresh = false;
    SLF_TRY(refresh_stats());
    return kRetry;
}

Status World::fresh_status() {
    Status z{};
    z.cell_lo[0] = z.cell_lo[1] = z.cell_lo[2] = INT32_MAX;
    z.cell_hi[0] = z.cell_hi[1] = z.cell_hi[2] = INT32_MIN;
    return z;
}

int32_t World::reset_status() {
    *h_status = fresh_status();
    SLF_CUDA(cudaMemcpyAsync(d_status, h_status, sizeof(Status), cudaMemcpyHostToDevice, stream));
    return SLF_OK;
}

int32_t World::refresh_stats() {
    if (stats_fresh) return SLF_OK;
    SLF_TRY(reset_status());
    Params p = params();
    timed("stats", bytes_per_particle::stats, [&] { stats_pass(p); });
    SLF_TRY(read_status());
    stats_fresh = true;
    return SLF_OK;
}

int32_t World::sort_into(int to) {
    if (n == 0) return SLF_OK;
    SortPlan sp;
    SLF_TRY(plan_sort(sp, false));
    return enqueue_sort(to, sp, stream);
}

int32_t World::plan_sort(SortPlan& sp, bool stable) {
    int64_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = h_status->cell_lo[a];
        hi[a] = h_status->cell_hi[a];
        if (hi[a] < lo[a]) return fail(SLF_ERR_CUDA, "empty cell box before a sort");
    }
    auto volume_of = [](const int64_t* l, const int64_t* h) {
        __int128 v = 1;
        for (int a = 0; a < 3; ++a) v *= __int128(h[a] - l[a] + 1);
        return v;
    };
    // a dense count table over the box; a scene spread too thin for it is not supported yet
    const __int128 limit = (__int128)64 * (__int128)n + (1 << 22);
    auto fits = [&](__int128 v) { return v <= limit && v < (__int128)(1u << 31); };
    if (stable && has_bounds) {
        Key3 cl = cell_of(blow), ch = cell_of(bhigh);
        int64_t wl[3] = {std::min<int64_t>(lo[0], cl.x), std::min<int64_t>(lo[1], cl.y),
                         std::min<int64_t>(lo[2], cl.z)};
        int64_t wh[3] = {std::max<int64_t>(hi[0], ch.x), std::max<int64_t>(hi[1], ch.y),
                         std::max<int64_t>(hi[2], ch.z)};
        if (fits(volume_of(wl, wh)))
            for (int a = 0; a < 3; ++a) {
                lo[a] = wl[a];
                hi[a] = wh[a];
            }
    }
    __int128 vol = volume_of(lo, hi);
    if (!fits(vol))
        return fail(SLF_ERR_UNSUPPORTED, "particles spread over too many cells for the dense cell table");
    sp.volume = uint32_t(vol);
    sp.lo = make_int3(int(lo[0]), int(lo[1]), int(lo[2]));
    sp.span = make_int3(int(hi[0] - lo[0] + 1), int(hi[1] - lo[1] + 1), int(hi[2] - lo[2] + 1));
    sp.job_lo = sp.job_hi = 0;
    if (skip_job >= 0) {
        sp.job_lo = uint32_t(skip_job) * 512u;
        sp.job_hi = sp.job_lo + 512u;
        skip_job = -1;
    }
    SLF_TRY(ensure_work_buffers());
    SLF_TRY(count.ensure(size_t(sp.volume) + 1, 0, stream));
    SLF_TRY(tiles.ensure(scan_tiles(sp.volume) + 1, 0, stream));
    // the walk order of this sort's lists (identity where its key space would not fit 32 bits,
    // and where every pass over the lists runs a warp a particle)
    size_t keys = walk_order_keys(sp.span);
    sp.keys = 0;
    bool warp_passes = !fast() && s.solver == SLF_SOLVER_WCSPH && warp_rows(uint32_t(n), radius, s.spacing) &&
                       terrains.empty() && m_pos.empty();
    if (keys < (size_t(1) << 31) && !warp_passes) {
        SLF_TRY(worder.ensure(n, 0, stream));
        SLF_TRY(wkeys.ensure(keys + 1, 0, stream));
        SLF_TRY(wsums.ensure(scan_tiles(uint32_t(keys)) + 1, 0, stream));
        sp.keys = keys;
    }
    worder_valid = sp.keys != 0;
    fgrid = GridDev{};
    fgrid.mode = 1;
    fgrid.lx = sp.lo.x;
    fgrid.ly = sp.lo.y;
    fgrid.lz = sp.lo.z;
    fgrid.sx = sp.span.x;
    fgrid.sy = sp.span.y;
    fgrid.sz = sp.span.z;
    fgrid.start = count.p;
    return SLF_OK;
}

int32_t World::enqueue_sort(int to, const SortPlan& sp, cudaStream_t on) {
    Params p = params();
    SLF_CUDA(cudaMemsetAsync(count.p, 0, (size_t(sp.volume) + 1) * 4, on));
    timed("hash_count", bytes_per_particle::count_cells, [&] {
        launch_count_cells(p, pos[cpos].p, cells_of(cpos), sp.lo, sp.span, count.p, lin.p, cslot.p, on);
    });
    timed("hash_scan", bytes_per_particle::scan,
          [&] { launch_exclusive_scan(count.p, sp.volume, tiles.p, on); });
    timed("hash_scatter", bytes_per_particle::scatter, [&] {
        launch_scatter_members(uint32_t(n), lin.p, cslot.p, count.p, ids[cid].p, members.p, on);
    });
    timed("hash_reorder", bytes_per_particle::reorder, [&] {
        launch_rank_reorder(uint32_t(n), lin.p, count.p, members.p, ids[cid].p, pos[cpos].p, vel[cpos].p,
                            rho[cid].p, cells_of(cpos), ids[1 - cid].p, pos[to].p, vel[to].p, rho[1 - cid].p,
                            cells_of(to), warm_in(), warm_out(), sp.job_lo, sp.job_hi, d_status, sort_dest, on);
    });
    if (sp.keys)
        timed("walk_order", bytes_per_particle::walk_order,
              [&] { launch_walk_order(sp.volume, sp.span, count.p, wkeys.p, wsums.p, worder.p, on); });
    return SLF_OK;
}

int32_t World::update_neighbors() {
    SLF_TRY(flush());
    SLF_TRY(upload_walls());
    SLF_TRY(upload_terrain());
    if (n == 0) {
        lists_valid = true;
        lists_n = 0;
        return SLF_OK;
    }
    SLF_TRY(refresh_stats());
    int to = (cpos + 1) % 3;
    h_status->processed = 0;
    SLF_CUDA(cudaMemsetAsync(&d_status->processed, 0, 4, stream));
    SLF_TRY(sort_into(to));
    SLF_TRY(read_status());
    if (h_status->processed != n) {
        lists_valid = false;
        return fail(SLF_ERR_DISPATCH_INCOMPLETE, "dispatcher did not run every job");
    }
    cpos = to;
    cid = 1 - cid;
    lists_pos = to;
    lists_n = n;
    lists_valid = true;
    stats_fresh = false;
    return SLF_OK;
}

int32_t World::compute_densities() {
    SLF_TRY(flush());
    if (!lists_valid || lists_n != n) return fail(SLF_ERR_OUT_OF_RANGE, "neighbour lists are stale");
    if (n == 0) return SLF_OK;
    SLF_TRY(ensure_work_buffers());
    SLF_TRY(upload_walls());
    SLF_TRY(upload_terrain());
    Params p = params();
    for (;;) {
        SLF_TRY(reset_status());
        density_pass(p, cpos, fluid_lists(), wall_lists(), rho[cid].p);
        SLF_TRY(read_status());
        int32_t st = lists_fit();
        if (st == SLF_OK) return SLF_OK;
        if (st != kRetry) return st;
    }
}

int32_t World::read_vec(const DevBuf<float4>& b, float* out, uint64_t k) {
    if (!k) return SLF_OK;
    SLF_TRY(stage.ensure(3 * k, 0, stream));
    launch_pack3(uint32_t(k), b.p, stage.p, stream);
    SLF_CUDA(cudaMemcpyAsync(out, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
    return sync();
}

int32_t World::read_positions(float* out, uint64_t k) {
    if (!rel()) return read_vec(pos[cpos], out, k);
    if (!k) return SLF_OK;
    SLF_TRY(stage.ensure(3 * k, 0, stream));
    launch_from_relative(params(), uint32_t(k), pos[cpos].p, cell[cpos].p, stage.p, stream);
    SLF_CUDA(cudaMemcpyAsync(out, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
    return sync();
}

int32_t World::write_vec(DevBuf<float4>& b, const float* in, uint64_t k) {
    if (!k) return SLF_OK;
    SLF_TRY(stage.ensure(3 * k, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(stage.p, in, k * 12, cudaMemcpyHostToDevice, stream));
    launch_unpack3(uint32_t(k), stage.p, b.p, stream);
    return SLF_OK;
}

int32_t World::write_state(const float* p, const float* v, uint64_t k) {
    SLF_TRY(flush());
    if (k != n) return fail(SLF_ERR_INVALID_ARGUMENT, "n must equal slf_len()");
    if (!k) return SLF_OK;
    int t = (cpos + 1) % 3;
    SLF_TRY(stage.ensure(6 * k, 0, stream));
    SLF_TRY(reset_status());
    uint32_t* bad = &d_status->nonfinite;
    SLF_CUDA(cudaMemcpyAsync(stage.p, p, k * 12, cudaMemcpyHostToDevice, stream));
    SLF_CUDA(cudaMemcpyAsync(stage.p + 3 * k, v, k * 12, cudaMemcpyHostToDevice, stream));
    Params pr = params();
    if (rel()) launch_to_relative(pr, uint32_t(k), stage.p, nullptr, pos[t].p, cell[t].p, stream, bad);
    else launch_unpack3(uint32_t(k), stage.p, pos[t].p, stream, bad);
    launch_unpack3(uint32_t(k), stage.p + 3 * k, vel[t].p, stream, bad);
    if (rel()) launch_state_stats_rel(pr, cell[t].p, vel[t].p, d_status, stream);
    else launch_state_stats(pr, pos[t].p, vel[t].p, d_status, stream);
    SLF_TRY(read_status());
    lists_valid = false;
    if (h_status->nonfinite) {
        stats_fresh = false;
        return fail(SLF_ERR_NON_FINITE, "non finite value in fluid particle");
    }
    cpos = t;
    stats_fresh = true;
    return SLF_OK;
}

int32_t World::read_state(float* p, float* v, uint64_t k) {
    if (!k) return SLF_OK;
    SLF_TRY(stage.ensure(6 * k, 0, stream));
    if (rel()) launch_from_relative(params(), uint32_t(k), pos[cpos].p, cell[cpos].p, stage.p, stream);
    else launch_pack3(uint32_t(k), pos[cpos].p, stage.p, stream);
    launch_pack3(uint32_t(k), vel[cpos].p, stage.p + 3 * k, stream);
    SLF_CUDA(cudaMemcpyAsync(p, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
    SLF_CUDA(cudaMemcpyAsync(v, stage.p + 3 * k, k * 12, cudaMemcpyDeviceToHost, stream));
    return sync();
}

int32_t World::lists(bool walls, uint32_t* start, uint64_t start_len, uint32_t* items, uint64_t cap, uint64_t* len) {
    SLF_TRY(flush());
    if (!lists_valid || lists_n != n) return fail(SLF_ERR_OUT_OF_RANGE, "neighbour lists are stale");
    if (start && start_len != n + 1) return fail(SLF_ERR_INVALID_ARGUMENT, "start must hold len + 1 entries");
    SLF_TRY(upload_walls());
    SLF_TRY(upload_terrain());
    if (n == 0) {
        if (start) start[0] = 0;
        if (len) *len = 0;
        return SLF_OK;
    }
    Params p = params();
    DevBuf<uint32_t> cnt, tl, it;
    SLF_TRY(cnt.ensure(n + 1, 0, stream));
    SLF_TRY(tl.ensure(scan_tiles(uint32_t(n)) + 1, 0, stream));
    const GridDev& g = walls ? wgrid : fgrid;
    const float4* pts = walls ? dwalls.p : pos[lists_pos].p;
    if (rel()) launch_list_rel(p, g, pos[lists_pos].p, cell[lists_pos].p, pts, nullptr, cnt.p, stream);
    else launch_list_count(p, g, pos[lists_pos].p, pts, cnt.p, stream);
    launch_exclusive_scan(cnt.p, uint32_t(n), tl.p, stream);
    uint32_t total_items = 0;
    SLF_CUDA(cudaMemcpyAsync(&total_items, cnt.p + n, 4, cudaMemcpyDeviceToHost, stream));
    SLF_CUDA(cudaStreamSynchronize(stream));
    if (len) *len = total_items;
    int32_t st = SLF_OK;
    if (start) st = read_plain(cnt, start, n + 1);
    if (st == SLF_OK && items) {
        if (cap < total_items) {
            st = fail(SLF_ERR_INVALID_ARGUMENT, "items buffer too small");
        } else if (total_items) {
            st = it.ensure(total_items, 0, stream);
            if (st == SLF_OK) {
                if (rel())
                    launch_list_rel(p, g, pos[lists_pos].p, cell[lists_pos].p, pts, cnt.p, it.p, stream);
                else
                    launch_list_fill(p, g, pos[lists_pos].p, pts, cnt.p, it.p, stream);
                st = read_plain(it, items, total_items);
            }
        }
    }
    cnt.release(stream);
    tl.release(stream);
    it.release(stream);
    cudaStreamSynchronize(stream);
    return st;
}

uint64_t World::state_hash_host(const std::vector<uint32_t>& id, const std::vector<float>& p,
                                const std::vector<float>& v) const {
    std::vector<size_t> order(id.size());
    std::iota(order.begin(), order.end(), size_t(0));
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return id[a] < id[b]; });
    uint64_t h = 0xcbf29ce484222325ull;
    auto put = [&](uint32_t w) {
        for (int k = 0; k < 4; ++k) {
            h ^= uint64_t((w >> (8 * k)) & 0xffu);
            h *= 0x00000100000001b3ull;
        }
    };
    for (size_t i : order) {
        put(id[i]);
        for (int k = 0; k < 3; ++k) put(fbits(p[3 * i + k]));
        for (int k = 0; k < 3; ++k) put(fbits(v[3 * i + k]));
    }
    return h;
}


void set_last_error(const std::string& message) { g_error = message; }

}  // namespace slf
