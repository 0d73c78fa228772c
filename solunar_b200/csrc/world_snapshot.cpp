// world_snapshot.cpp -- World's snapshots (src/fluid/save.rs).
#include "world.h"

namespace slf {

int32_t World::save_snapshot(std::vector<uint8_t>& out) {
    SLF_TRY(flush());
    std::vector<uint32_t> id(n);
    std::vector<float> p(3 * n), v(3 * n);
    SLF_TRY(read_plain(ids[cid], id.data(), n));
    SLF_TRY(read_positions(p.data(), n));
    SLF_TRY(read_vec(vel[cpos], v.data(), n));
    SnapWriter w;
    w.data.reserve(64 + n * 28 + wpos.size() * 16);
    w.bytes("SLFL", 4);
    w.u32(kSnapshotVersion);
    w.u8(s.solver == SLF_SOLVER_DFSPH ? 1 : 0);
    for (float x : {s.spacing, s.rest_density, s.support, s.sound_speed, s.viscosity, s.courant}) w.f32(x);
    w.u64(s.max_particles);
    w.vec3(s.gravity[0], s.gravity[1], s.gravity[2]);
    w.u32(s.max_substeps);
    w.len(n);
    for (uint64_t i = 0; i < n; ++i) {
        w.u32(id[i]);
        w.vec3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
        w.vec3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    }
    w.u32(next_id);
    // Walls::save (boundary.rs:182-195)
    w.len(wpos.size());
    for (size_t k = 0; k < wpos.size(); ++k) {
        w.vec3(wpos[k].x, wpos[k].y, wpos[k].z);
        w.u32(wown[k]);
    }
    w.u32(wall_next);
    w.len(containers.size());
    for (const ContainerBox& c : containers) {
        w.u32(c.id);
        w.vec3(c.low.x, c.low.y, c.low.z);
        w.vec3(c.high.x, c.high.y, c.high.z);
    }
    // Flows::save (flow.rs:36-51)
    w.len(flows.size());
    for (const FlowBox& f : flows) {
        w.u32(f.id);
        w.vec3(f.low.x, f.low.y, f.low.z);
        w.vec3(f.high.x, f.high.y, f.high.z);
        if (f.emitter) {
            w.u8(0);
            w.vec3(f.velocity.x, f.velocity.y, f.velocity.z);
        } else {
            w.u8(1);
        }
    }
    w.u32(flow_next);
    // Coupled::save (couple.rs:50-55)
    w.len(coupled.size());
    for (const Coupled& c : coupled) {
        w.u32(uint32_t(c.body >> 32));
        w.u32(uint32_t(c.body & 0xffffffffu));
        w.len(c.points.size());
        for (const F3& q : c.points) w.vec3(q.x, q.y, q.z);
        w.f32(c.probe_spacing);
        w.len(c.probes.size());
        for (const F3& q : c.probes) w.vec3(q.x, q.y, q.z);
    }
    // TerrainField::save (terrain.rs:44-55)
    w.len(terrains.size());
    for (const TerrainHost& t : terrains) {
        w.u32(t.owner);
        w.vec3(t.low.x, t.low.y, t.low.z);
        w.len(t.nx);
        w.len(t.ny);
        w.len(t.nz);
        w.f32(t.step);
        w.len(t.distances.size());
        for (float d : t.distances) w.f32(d);
    }
    if (has_domain) {
        w.u8(1);
        w.vec3(dlow.x, dlow.y, dlow.z);
        w.vec3(dhigh.x, dhigh.y, dhigh.z);
    } else {
        w.u8(0);
    }
    w.u64(fnv1a64(w.data.data(), w.data.size()));
    out = std::move(w.data);
    return SLF_OK;
}

int32_t World::load_snapshot(const uint8_t* data, size_t size, const slf_settings& lib) {
    auto bad = [&](const std::string& m) { return fail(SLF_ERR_SNAPSHOT, m); };
    if (size > kMaxSnapshotBytes) return bad("snapshot over limit");
    if (size < 4 + 4 + 8) return bad("snapshot truncated");
    if (std::memcmp(data, "SLFL", 4) != 0) return bad("not a snapshot");
    const size_t body = size - 8;
    SnapReader ck{data + body, 8, 0, {}};
    uint64_t stored = 0;
    ck.u64(stored);
    if (stored != fnv1a64(data, body)) return bad("snapshot checksum mismatch");
    SnapReader r{data, body, 4, {}};
    auto rd = [&](bool ok) { return ok ? SLF_OK : bad(r.error); };
    uint32_t version = 0;
    SLF_TRY(rd(r.u32(version)));
    if (version < 1 || version > kSnapshotVersion)
        return bad("unsupported snapshot version " + std::to_string(version));
    uint8_t solver = 0;
    SLF_TRY(rd(r.u8(solver)));
    if (solver > 1) return bad("invalid snapshot: fluid solver");
    float f[6];
    for (float& x : f) SLF_TRY(rd(r.f32(x)));
    uint64_t max_particles = 0;
    SLF_TRY(rd(r.u64(max_particles)));
    F3 grav{};
    SLF_TRY(rd(r.vec3(grav)));
    uint32_t max_substeps = 0;
    SLF_TRY(rd(r.u32(max_substeps)));
    slf_settings st = lib;
    st.solver = solver;
    st.spacing = f[0];
    st.rest_density = f[1];
    st.support = f[2];
    st.sound_speed = f[3];
    st.viscosity = f[4];
    st.courant = f[5];
    st.max_particles = max_particles;
    st.gravity[0] = grav.x;
    st.gravity[1] = grav.y;
    st.gravity[2] = grav.z;
    st.max_substeps = max_substeps;
    if (!valid(st)) return bad("invalid snapshot: fluid settings");
    size_t count = 0;
    SLF_TRY(rd(r.count(28, size_t(std::min<uint64_t>(max_particles, SIZE_MAX)), count)));
    std::vector<uint32_t> lid(count);
    std::vector<float4> lpos(count), lvel(count);
    for (size_t i = 0; i < count; ++i) {
        F3 at{}, v{};
        SLF_TRY(rd(r.u32(lid[i]) && r.vec3(at) && r.vec3(v)));
        if (!finite3f(at) || !finite3f(v)) return bad("invalid snapshot: fluid particle");
        lpos[i] = make_float4(at.x, at.y, at.z, 0.0f);
        lvel[i] = make_float4(v.x, v.y, v.z, 0.0f);
    }
    uint32_t nid = 0;
    SLF_TRY(rd(r.u32(nid)));
    std::vector<uint32_t> seen = lid;
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end() || (!seen.empty() && seen.back() >= nid))
        return bad("invalid snapshot: fluid particle id");
    // Walls::load (boundary.rs:202-227)
    size_t nw = 0;
    SLF_TRY(rd(r.count(16, size_t(std::min<uint64_t>(max_particles, SIZE_MAX)), nw)));
    std::vector<F3> lw(nw);
    std::vector<uint32_t> lo(nw);
    for (size_t k = 0; k < nw; ++k) {
        SLF_TRY(rd(r.vec3(lw[k])));
        if (!finite3f(lw[k])) return bad("invalid snapshot: fluid wall");
        SLF_TRY(rd(r.u32(lo[k])));
    }
    uint32_t wnext = 0;
    SLF_TRY(rd(r.u32(wnext)));
    size_t nc = 0;
    SLF_TRY(rd(r.count(28, size_t(std::min<uint64_t>(max_particles, SIZE_MAX)), nc)));
    std::vector<ContainerBox> lc(nc);
    for (auto& c : lc) {
        SLF_TRY(rd(r.u32(c.id) && r.vec3(c.low) && r.vec3(c.high)));
        bool ok = finite3f(c.low) && finite3f(c.high) && c.high.x > c.low.x && c.high.y > c.low.y &&
                  c.high.z > c.low.z;
        if (!ok || c.id >= wnext) return bad("invalid snapshot: fluid container");
    }
    for (uint32_t o : lo)
        if (o >= wnext) return bad("invalid snapshot: fluid wall owner");
    // Flows::load (flow.rs:53-83)
    size_t nf = 0;
    SLF_TRY(rd(r.count(29, kMaxSnapshotParts, nf)));
    std::vector<FlowBox> lf(nf);
    for (auto& fl : lf) {
        uint8_t kind = 0;
        SLF_TRY(rd(r.u32(fl.id) && r.vec3(fl.low) && r.vec3(fl.high) && r.u8(kind)));
        fl.velocity = F3{0, 0, 0};
        if (kind == 0) {
            fl.emitter = true;
            SLF_TRY(rd(r.vec3(fl.velocity)));
        } else if (kind == 1) {
            fl.emitter = false;
        } else {
            return bad("invalid snapshot: fluid flow kind");
        }
        bool inside_out = fl.high.x <= fl.low.x || fl.high.y <= fl.low.y || fl.high.z <= fl.low.z;
        if (!(finite3f(fl.low) && finite3f(fl.high) && finite3f(fl.velocity)) || inside_out)
            return bad("invalid snapshot: fluid flow");
    }
    uint32_t fnext = 0;
    SLF_TRY(rd(r.u32(fnext)));
    for (auto& fl : lf)
        if (fl.id >= fnext) return bad("invalid snapshot: fluid flow id");
    size_t ncoupled = 0, nterrain = 0;
    SLF_TRY(rd(r.count(12, kMaxSnapshotParts, ncoupled)));
    // Coupled::load (couple.rs:58-75), load_points (couple.rs:435-451)
    std::vector<Coupled> lcoupled;
    uint64_t room = st.max_particles;
    auto points = [&](uint64_t max, std::vector<F3>& out) -> int32_t {
        size_t count = 0;
        SLF_TRY(rd(r.count(12, size_t(std::min<uint64_t>(max, SIZE_MAX)), count)));
        for (size_t k = 0; k < count; ++k) {
            F3 q;
            SLF_TRY(rd(r.vec3(q)));
            if (!finite3f(q)) return bad("invalid snapshot: fluid body point");
            out.push_back(q);
        }
        if (out.empty()) return bad("invalid snapshot: fluid body");
        return SLF_OK;
    };
    for (size_t k = 0; k < ncoupled; ++k) {
        Coupled c;
        uint32_t index = 0, generation = 0;
        SLF_TRY(rd(r.u32(index) && r.u32(generation)));
        c.body = (uint64_t(index) << 32) | generation;
        SLF_TRY(points(room, c.points));
        if (version >= 3) {
            float ps = 0.0f;
            SLF_TRY(rd(r.f32(ps)));
            if (!std::isfinite(ps) || ps <= 0.0f) return bad("invalid snapshot: fluid body probes");
            c.probe_spacing = ps;
            SLF_TRY(points(kMaxProbes, c.probes));
        } else {
            c.probe_spacing = st.spacing;
            c.probes = c.points;
        }
        room -= c.points.size();
        lcoupled.push_back(std::move(c));
    }
    for (size_t k = 1; k < lcoupled.size(); ++k)
        if (lcoupled[k - 1].body >= lcoupled[k].body) return bad("invalid snapshot: fluid body order");
    SLF_TRY(rd(r.count(32, kMaxSnapshotParts, nterrain)));
    // TerrainField::load (terrain.rs:57-97)
    std::vector<TerrainHost> lt(nterrain);
    for (TerrainHost& t : lt) {
        size_t nd = 0;
        SLF_TRY(rd(r.u32(t.owner) && r.vec3(t.low) && r.u32(t.nx) && r.u32(t.ny) && r.u32(t.nz) && r.f32(t.step) &&
                   r.count(4, kMaxTerrainNodes, nd)));
        unsigned __int128 total = (unsigned __int128)t.nx * t.ny * t.nz;
        if (!finite3f(t.low) || !std::isfinite(t.step) || t.step <= 0.0f || t.nx < 2 || t.ny < 2 || t.nz < 2 ||
            total != nd)
            return bad("invalid snapshot: fluid terrain");
        t.distances.resize(nd);
        for (float& d : t.distances) {
            SLF_TRY(rd(r.f32(d)));
            if (!std::isfinite(d)) return bad("invalid snapshot: fluid terrain distance");
        }
        if (t.owner >= wnext) return bad("invalid snapshot: fluid terrain owner");
    }
    bool dom = false;
    F3 dl{}, dh{};
    if (version >= 2) {
        uint8_t flag = 0;
        SLF_TRY(rd(r.u8(flag)));
        if (flag > 1) return bad("invalid snapshot: fluid domain flag");
        if (flag == 1) {
            SLF_TRY(rd(r.vec3(dl) && r.vec3(dh)));
            bool ok = finite3f(dl) && finite3f(dh) && dh.x > dl.x && dh.y > dl.y && dh.z > dl.z;
            if (!ok) return bad("invalid snapshot: fluid domain");
            dom = true;
        }
    }
    if (r.at != body) return bad("invalid snapshot: trailing bytes");
    if (count > index_limit_of(st)) return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    SLF_TRY(init(st));
    pend_pos = std::move(lpos);
    pend_vel = std::move(lvel);
    pend_ids = std::move(lid);
    next_id = nid;
    SLF_TRY(flush());
    if (n) {  // densities of a loaded world: rest density (save.rs:144)
        std::vector<float> rest(n, s.rest_density);
        SLF_CUDA(cudaMemcpyAsync(rho[cid].p, rest.data(), n * 4, cudaMemcpyHostToDevice, stream));
        SLF_TRY(sync());
    }
    wpos = std::move(lw);
    wown = std::move(lo);
    wall_next = wnext;
    containers = std::move(lc);
    update_bounds();
    settle_walls();
    flows = std::move(lf);
    flow_next = fnext;
    if (!lt.empty() && fast()) return fail(SLF_ERR_UNSUPPORTED, "terrain runs with EXACT arithmetic only");
    terrains = std::move(lt);
    terrain_dirty = true;
    coupled = std::move(lcoupled);
    has_domain = dom;
    dlow = dl;
    dhigh = dh;
    return SLF_OK;
}

}  // namespace slf
