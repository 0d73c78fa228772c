// world_walls.cpp -- World's static walls (src/fluid/boundary.rs).
#include "world.h"

namespace slf {

int32_t World::check_box(const float* low, const float* high) {
    if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid box");
    if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
        return fail(SLF_ERR_OUT_OF_RANGE, "inside out fluid box");
    return SLF_OK;
}

void World::cells_in(const float* low, const float* high, int64_t out[3]) const {
    for (int a = 0; a < 3; ++a) {
        float c = rmin(std::round((high[a] - low[a]) / s.spacing), 1e9f);
        out[a] = int64_t(c);
    }
}

int32_t World::check_room(int64_t count) const {
    uint64_t room = s.max_particles > wpos.size() ? s.max_particles - wpos.size() : 0;
    if (index_limit() < UINT64_MAX) room = std::min<uint64_t>(room, index_limit() > wpos.size() ? index_limit() - wpos.size() : 0);
    if (count < 0 || uint64_t(count) > room || wall_next == UINT32_MAX)
        return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
    return SLF_OK;
}

uint32_t World::add_wall_points(const std::vector<F3>& pts) {
    uint32_t id = wall_next++;
    for (auto& p : pts) {
        wpos.push_back(p);
        wown.push_back(id);
    }
    settle_walls();
    return id;
}

int32_t World::add_box_container(const float* low, const float* high, uint32_t* out) {
    SLF_TRY(check_box(low, high));
    int64_t c[3];
    cells_in(low, high, c);
    int64_t layers = int64_t(std::ceil(s.support));
    int64_t shell = (c[0] + 2 * layers) * (c[1] + 2 * layers) * (c[2] + 2 * layers) - c[0] * c[1] * c[2];
    SLF_TRY(check_room(shell));
    std::vector<F3> pts;
    pts.reserve(size_t(shell));
    for (int64_t y = -layers; y < c[1] + layers; ++y)
        for (int64_t z = -layers; z < c[2] + layers; ++z)
            for (int64_t x = -layers; x < c[0] + layers; ++x) {
                bool inside = x >= 0 && x < c[0] && y >= 0 && y < c[1] && z >= 0 && z < c[2];
                if (inside) continue;
                pts.push_back(F3{low[0] + (float(x) + 0.5f) * s.spacing, low[1] + (float(y) + 0.5f) * s.spacing,
                                 low[2] + (float(z) + 0.5f) * s.spacing});
            }
    uint32_t id = add_wall_points(pts);
    containers.push_back(ContainerBox{id, F3{low[0], low[1], low[2]}, F3{high[0], high[1], high[2]}});
    update_bounds();
    if (out) *out = id;
    return SLF_OK;
}

int32_t World::add_wall(const float* low, const float* high, uint32_t* out) {
    SLF_TRY(check_box(low, high));
    int64_t c[3];
    cells_in(low, high, c);
    for (auto& v : c) v = std::max<int64_t>(v, 1);
    int64_t count = c[0] * c[1] * c[2];
    SLF_TRY(check_room(count));
    std::vector<F3> pts;
    pts.reserve(size_t(count));
    for (int64_t y = 0; y < c[1]; ++y)
        for (int64_t z = 0; z < c[2]; ++z)
            for (int64_t x = 0; x < c[0]; ++x)
                pts.push_back(F3{low[0] + (float(x) + 0.5f) * s.spacing, low[1] + (float(y) + 0.5f) * s.spacing,
                                 low[2] + (float(z) + 0.5f) * s.spacing});
    uint32_t id = add_wall_points(pts);
    if (out) *out = id;
    return SLF_OK;
}

bool World::remove_boundary(uint32_t id) {
    size_t before = wpos.size();
    size_t kept = 0;
    for (size_t i = 0; i < wpos.size(); ++i)
        if (wown[i] != id) {
            wpos[kept] = wpos[i];
            wown[kept] = wown[i];
            ++kept;
        }
    wpos.resize(kept);
    wown.resize(kept);
    bool had = false;
    std::vector<ContainerBox> rest;
    for (auto& c : containers) {
        if (c.id == id) had = true;
        else rest.push_back(c);
    }
    containers = rest;
    update_bounds();
    size_t regions = terrains.size();
    terrains.erase(std::remove_if(terrains.begin(), terrains.end(), [&](const TerrainHost& t) { return t.owner == id; }),
                   terrains.end());
    if (terrains.size() != regions) terrain_dirty = true;
    bool gone = wpos.size() != before || had || terrains.size() != regions;
    if (gone) settle_walls();
    return gone;
}

void World::update_bounds() {
    has_bounds = false;
    for (auto& c : containers) {
        if (!has_bounds) {
            blow = c.low;
            bhigh = c.high;
            has_bounds = true;
        } else {
            blow = F3{rmin(blow.x, c.low.x), rmin(blow.y, c.low.y), rmin(blow.z, c.low.z)};
            bhigh = F3{rmax(bhigh.x, c.high.x), rmax(bhigh.y, c.high.y), rmax(bhigh.z, c.high.z)};
        }
    }
}

uint32_t World::fbits(float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
}

void World::settle_walls() {
    size_t m = wpos.size();
    struct WK {
        Key3 cell;
        uint32_t owner, bx, by, bz;
        size_t index;
    };
    std::vector<WK> order(m);
    for (size_t i = 0; i < m; ++i)
        order[i] = WK{cell_of(wpos[i]), wown[i], fbits(wpos[i].x), fbits(wpos[i].y), fbits(wpos[i].z), i};
    std::sort(order.begin(), order.end(), [](const WK& a, const WK& b) {
        return std::tie(a.cell.x, a.cell.y, a.cell.z, a.owner, a.bx, a.by, a.bz, a.index) <
               std::tie(b.cell.x, b.cell.y, b.cell.z, b.owner, b.bx, b.by, b.bz, b.index);
    });
    std::vector<F3> np(m);
    std::vector<uint32_t> no(m);
    for (size_t i = 0; i < m; ++i) {
        np[i] = wpos[order[i].index];
        no[i] = order[i].owner;
    }
    wpos = std::move(np);
    wown = std::move(no);
    walls_dirty = true;
}

int32_t World::grid_from_keys(const std::vector<Key3>& keys, GridDev& g, DevBuf<uint32_t>& dstart, DevBuf<int4>& dkeys) {
    g = GridDev{};
    size_t m = keys.size();
    if (m == 0) return SLF_OK;
    std::vector<Key3> cells;
    std::vector<uint32_t> starts;
    for (size_t i = 0; i < m; ++i)
        if (i == 0 || !(keys[i] == keys[i - 1])) {
            cells.push_back(keys[i]);
            starts.push_back(uint32_t(i));
        }
    starts.push_back(uint32_t(m));
    Key3 lo = cells[0], hi = cells[0];
    for (auto& c : cells) {
        lo = Key3{std::min(lo.x, c.x), std::min(lo.y, c.y), std::min(lo.z, c.z)};
        hi = Key3{std::max(hi.x, c.x), std::max(hi.y, c.y), std::max(hi.z, c.z)};
    }
    int64_t sx = int64_t(hi.x) - lo.x + 1, sy = int64_t(hi.y) - lo.y + 1, sz = int64_t(hi.z) - lo.z + 1;
    __int128 vol = (__int128)sx * sy * sz;
    if (vol <= (__int128)64 * (__int128)cells.size() + 4096 && vol < (__int128)(1u << 30)) {
        size_t volume = size_t(vol);
        std::vector<uint32_t> start(volume + 1, 0);
        // cells are in key order, which is the dense table's x-major order
        size_t c = 0;
        for (size_t at = 0; at < volume; ++at) {
            start[at] = c < cells.size() ? starts[c] : uint32_t(m);
            if (c < cells.size()) {
                const Key3& k = cells[c];
                size_t lin = size_t(((int64_t(k.x) - lo.x) * sy + (int64_t(k.y) - lo.y)) * sz + (int64_t(k.z) - lo.z));
                if (lin == at) ++c;
            }
        }
        start[volume] = uint32_t(m);
        SLF_TRY(dstart.ensure(volume + 1, 0, stream));
        SLF_CUDA(cudaMemcpyAsync(dstart.p, start.data(), (volume + 1) * 4, cudaMemcpyHostToDevice, stream));
        g.mode = 1;
        g.lx = lo.x;
        g.ly = lo.y;
        g.lz = lo.z;
        g.sx = int(sx);
        g.sy = int(sy);
        g.sz = int(sz);
        g.start = dstart.p;
        SLF_CUDA(cudaStreamSynchronize(stream));
    } else {
        std::vector<int4> k4(cells.size());
        for (size_t i = 0; i < cells.size(); ++i) k4[i] = make_int4(cells[i].x, cells[i].y, cells[i].z, 0);
        SLF_TRY(dkeys.ensure(cells.size(), 0, stream));
        SLF_TRY(dstart.ensure(starts.size(), 0, stream));
        SLF_CUDA(cudaMemcpyAsync(dkeys.p, k4.data(), k4.size() * sizeof(int4), cudaMemcpyHostToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(dstart.p, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice, stream));
        SLF_CUDA(cudaStreamSynchronize(stream));
        g.mode = 2;
        g.cells = uint32_t(cells.size());
        g.keys = dkeys.p;
        g.start = dstart.p;
    }
    return SLF_OK;
}

int32_t World::upload_walls() {
    if (!walls_dirty) return SLF_OK;
    size_t m = wpos.size();
    wgrid = GridDev{};
    if (m == 0) {
        walls_dirty = false;
        return SLF_OK;
    }
    std::vector<float4> w(m);
    std::vector<Key3> keys(m);
    for (size_t i = 0; i < m; ++i) {
        keys[i] = cell_of(wpos[i]);
        if (rel()) {  // offset from the corner of the wall point's cell
            const double r = radius;
            w[i] = make_float4(float(double(wpos[i].x) - double(keys[i].x) * r),
                               float(double(wpos[i].y) - double(keys[i].y) * r),
                               float(double(wpos[i].z) - double(keys[i].z) * r), 0.0f);
        } else {
            w[i] = make_float4(wpos[i].x, wpos[i].y, wpos[i].z, 0.0f);
        }
    }
    SLF_TRY(dwalls.ensure(m, 0, stream));
    SLF_CUDA(cudaMemcpyAsync(dwalls.p, w.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SLF_TRY(grid_from_keys(keys, wgrid, dwstart, dwkeys));
    walls_dirty = false;
    return SLF_OK;
}

}  // namespace slf
