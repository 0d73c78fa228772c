// capi.cpp -- the C ABI of include/solunar_fluid.h over World (world.h).
#include "world.h"


// ---- C ABI ---------------------------------------------------------------------------------

using slf::World;
using slf::fail;

struct slf_world {
    World w;
};

#define SLF_NEED(ptr)                                                                \
    do {                                                                             \
        if (!(ptr)) return fail(SLF_ERR_INVALID_ARGUMENT, "null argument: " #ptr);  \
    } while (0)

// Every call on a world runs on that world's device.
#define SLF_WORLD(world)                                                                          \
    do {                                                                                          \
        SLF_NEED(world);                                                                          \
        cudaError_t e_ = cudaSetDevice((world)->w.s.device);                                      \
        if (e_ != cudaSuccess) return fail(SLF_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

int32_t slf_settings_default(slf_settings* out) {
    SLF_NEED(out);
    slf_settings s{};
    s.solver = SLF_SOLVER_WCSPH;
    s.spacing = 0.05f;
    s.rest_density = 1000.0f;
    s.support = 2.0f;
    s.max_particles = uint64_t(1) << 22;
    s.sound_speed = 20.0f;
    s.viscosity = 0.15f;
    s.gravity[0] = 0.0f;
    s.gravity[1] = -9.81f;
    s.gravity[2] = 0.0f;
    s.courant = 0.4f;
    s.max_substeps = 2000;
    s.positions = SLF_POSITIONS_ABSOLUTE;
    s.arithmetic = SLF_ARITHMETIC_EXACT;
    s.warm_start = 0;
    s.divergence_tolerance = 1e-3f;
    s.density_tolerance = 5e-4f;
    s.min_iterations = 2;
    s.max_iterations = 100;
    s.device = 0;
    *out = s;
    return SLF_OK;
}

int32_t slf_create(const slf_settings* settings, slf_world** out) {
    SLF_NEED(settings);
    SLF_NEED(out);
    *out = nullptr;
    if (!World::valid(*settings)) return fail(SLF_ERR_INVALID_SETTINGS, "invalid settings");
    if (settings->arithmetic != SLF_ARITHMETIC_EXACT && settings->arithmetic != SLF_ARITHMETIC_FAST)
        return fail(SLF_ERR_INVALID_SETTINGS, "unknown arithmetic");
    if (settings->positions != SLF_POSITIONS_ABSOLUTE && settings->positions != SLF_POSITIONS_CELL_RELATIVE)
        return fail(SLF_ERR_INVALID_SETTINGS, "unknown positions");
    if (settings->positions == SLF_POSITIONS_CELL_RELATIVE && settings->arithmetic != SLF_ARITHMETIC_FAST)
        return fail(SLF_ERR_UNSUPPORTED, "cell-relative positions run with FAST arithmetic only");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
        return fail(SLF_ERR_CUDA, "no CUDA device");
    if (settings->device < 0 || settings->device >= devices)
        return fail(SLF_ERR_INVALID_SETTINGS, "no such CUDA device");
    auto h = std::make_unique<slf_world>();
    int32_t st = h->w.init(*settings);
    if (st != SLF_OK) return st;
    *out = h.release();
    return SLF_OK;
}

void slf_destroy(slf_world* world) {
    if (!world) return;
    cudaSetDevice(world->w.s.device);
    delete world;
}

int32_t slf_get_settings(const slf_world* world, slf_settings* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    *out = world->w.s;
    return SLF_OK;
}

int32_t slf_particle_mass(const slf_world* world, float* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    *out = world->w.mass;
    return SLF_OK;
}

int32_t slf_kernel(const slf_world* world, float* radius, float* scale) {
    SLF_WORLD(world);
    if (radius) *radius = world->w.radius;
    if (scale) *scale = world->w.scale;
    return SLF_OK;
}

int32_t slf_len(const slf_world* world, uint64_t* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    *out = world->w.total();
    return SLF_OK;
}

int32_t slf_add_particle(slf_world* world, const float position[3], const float velocity[3], uint32_t* id_out) {
    SLF_WORLD(world);
    SLF_NEED(position);
    SLF_NEED(velocity);
    return world->w.add(1, position, velocity, id_out);
}

int32_t slf_add_particles(slf_world* world, uint64_t n, const float* positions, const float* velocities,
                          uint32_t* ids_out) {
    SLF_WORLD(world);
    if (n == 0) return SLF_OK;
    SLF_NEED(positions);
    SLF_NEED(velocities);
    return world->w.add(n, positions, velocities, ids_out);
}

int32_t slf_fill_box(slf_world* world, const float low[3], const float high[3], uint64_t* count_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    return world->w.fill_box(low, high, count_out);
}

int32_t slf_set_domain(slf_world* world, const float* low, const float* high) {
    SLF_WORLD(world);
    World& w = world->w;
    if (!low && !high) {
        w.has_domain = false;
        return SLF_OK;
    }
    SLF_NEED(low);
    SLF_NEED(high);
    if (!slf::finite3(low) || !slf::finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid domain");
    if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
        return fail(SLF_ERR_OUT_OF_RANGE, "inside out fluid domain");
    w.has_domain = true;
    w.dlow = slf::F3{low[0], low[1], low[2]};
    w.dhigh = slf::F3{high[0], high[1], high[2]};
    return SLF_OK;
}

int32_t slf_add_box_container(slf_world* world, const float low[3], const float high[3], uint32_t* boundary_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    return world->w.add_box_container(low, high, boundary_out);
}

int32_t slf_add_wall(slf_world* world, const float low[3], const float high[3], uint32_t* boundary_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    return world->w.add_wall(low, high, boundary_out);
}

int32_t slf_remove_boundary(slf_world* world, uint32_t boundary, int32_t* removed) {
    SLF_WORLD(world);
    bool gone = world->w.remove_boundary(boundary);
    if (removed) *removed = gone ? 1 : 0;
    return SLF_OK;
}

int32_t slf_save_snapshot(slf_world* world, uint8_t* out, uint64_t capacity, uint64_t* size) {
    SLF_WORLD(world);
    SLF_NEED(size);
    std::vector<uint8_t> bytes;
    SLF_TRY(world->w.save_snapshot(bytes));
    *size = bytes.size();
    if (!out) return SLF_OK;
    if (capacity < bytes.size()) return fail(SLF_ERR_INVALID_ARGUMENT, "snapshot buffer too small");
    std::memcpy(out, bytes.data(), bytes.size());
    return SLF_OK;
}

int32_t slf_load_snapshot(const uint8_t* data, uint64_t size, const slf_settings* library, slf_world** out) {
    SLF_NEED(out);
    *out = nullptr;
    if (size) SLF_NEED(data);
    slf_settings lib;
    slf_settings_default(&lib);
    if (library) lib = *library;
    if (lib.arithmetic != SLF_ARITHMETIC_EXACT && lib.arithmetic != SLF_ARITHMETIC_FAST)
        return fail(SLF_ERR_INVALID_SETTINGS, "unknown arithmetic");
    if (lib.positions != SLF_POSITIONS_ABSOLUTE && lib.positions != SLF_POSITIONS_CELL_RELATIVE)
        return fail(SLF_ERR_INVALID_SETTINGS, "unknown positions");
    if (lib.positions == SLF_POSITIONS_CELL_RELATIVE && lib.arithmetic != SLF_ARITHMETIC_FAST)
        return fail(SLF_ERR_UNSUPPORTED, "cell-relative positions run with FAST arithmetic only");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail(SLF_ERR_CUDA, "no CUDA device");
    if (lib.device < 0 || lib.device >= devices) return fail(SLF_ERR_INVALID_SETTINGS, "no such CUDA device");
    if (cudaSetDevice(lib.device) != cudaSuccess) return fail(SLF_ERR_CUDA, "cannot select the CUDA device");
    auto h = std::make_unique<slf_world>();
    int32_t st = h->w.load_snapshot(data, size_t(size), lib);
    if (st != SLF_OK) return st;
    *out = h.release();
    return SLF_OK;
}

int32_t slf_terrain_nodes(const slf_world* world, const float low[3], const float high[3], uint64_t nodes[3]) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    SLF_NEED(nodes);
    return world->w.terrain_nodes(low, high, nodes);
}

int32_t slf_add_terrain(slf_world* world, const float low[3], const float high[3], const float* distances,
                        uint64_t count, uint32_t* boundary_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    if (count) SLF_NEED(distances);
    return world->w.add_terrain(low, high, distances, count, boundary_out);
}

int32_t slf_add_emitter(slf_world* world, const float low[3], const float high[3], const float velocity[3],
                        uint32_t* flow_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    SLF_NEED(velocity);
    return world->w.add_flow(low, high, true, velocity, flow_out);
}

int32_t slf_add_drain(slf_world* world, const float low[3], const float high[3], uint32_t* flow_out) {
    SLF_WORLD(world);
    SLF_NEED(low);
    SLF_NEED(high);
    return world->w.add_flow(low, high, false, nullptr, flow_out);
}

int32_t slf_remove_flow(slf_world* world, uint32_t flow, int32_t* removed) {
    SLF_WORLD(world);
    bool r = world->w.remove_flow(flow);
    if (removed) *removed = r ? 1 : 0;
    return SLF_OK;
}

int32_t slf_couple(slf_world* world, uint64_t body, int32_t shape, const float dims[3]) {
    SLF_WORLD(world);
    SLF_NEED(dims);
    return world->w.couple(body, shape, dims);
}

int32_t slf_uncouple(slf_world* world, uint64_t body, int32_t* removed) {
    SLF_WORLD(world);
    bool r = world->w.uncouple(body);
    if (removed) *removed = r ? 1 : 0;
    return SLF_OK;
}

int32_t slf_coupled(const slf_world* world, uint64_t* bodies, uint32_t* points, uint32_t* probes, uint64_t capacity,
                    uint64_t* count) {
    SLF_WORLD(world);
    const auto& c = world->w.coupled;
    if (count) *count = c.size();
    for (size_t k = 0; k < c.size() && k < capacity; ++k) {
        if (bodies) bodies[k] = c[k].body;
        if (points) points[k] = uint32_t(c[k].points.size());
        if (probes) probes[k] = uint32_t(c[k].probes.size());
    }
    return SLF_OK;
}

int32_t slf_step_with_bodies(slf_world* world, float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out,
                             slf_body_push* pushes, uint64_t capacity, uint64_t* count) {
    SLF_WORLD(world);
    if (npose) SLF_NEED(poses);
    std::vector<slf_body_push> got;
    int32_t st = world->w.step_with_bodies(dt, poses, npose, out, got);
    if (count) *count = got.size();
    for (size_t k = 0; k < got.size() && k < capacity && pushes; ++k) pushes[k] = got[k];
    return st;
}

int32_t slf_wall_count(const slf_world* world, uint64_t* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    *out = world->w.wpos.size();
    return SLF_OK;
}

int32_t slf_read_wall_positions(const slf_world* world, float* out, uint64_t n) {
    SLF_WORLD(world);
    const World& w = world->w;
    if (n != w.wpos.size()) return fail(SLF_ERR_INVALID_ARGUMENT, "n must equal the wall count");
    if (n) SLF_NEED(out);
    for (uint64_t i = 0; i < n; ++i) {
        out[3 * i] = w.wpos[i].x;
        out[3 * i + 1] = w.wpos[i].y;
        out[3 * i + 2] = w.wpos[i].z;
    }
    return SLF_OK;
}

int32_t slf_step(slf_world* world, float dt, slf_report* out) {
    SLF_WORLD(world);
    return world->w.step(dt, out);
}

int32_t slf_update_neighbors(slf_world* world) {
    SLF_WORLD(world);
    return world->w.update_neighbors();
}

int32_t slf_compute_densities(slf_world* world) {
    SLF_WORLD(world);
    return world->w.compute_densities();
}

static int32_t prep_read(const slf_world* world, uint64_t n) {
    World& w = const_cast<World&>(world->w);
    int32_t st = w.flush();
    if (st != SLF_OK) return st;
    if (n != w.n) return fail(SLF_ERR_INVALID_ARGUMENT, "n must equal slf_len()");
    return SLF_OK;
}

int32_t slf_read_ids(const slf_world* world, uint32_t* out, uint64_t n) {
    SLF_WORLD(world);
    SLF_TRY(prep_read(world, n));
    if (n) SLF_NEED(out);
    World& w = const_cast<World&>(world->w);
    return w.read_plain(w.ids[w.cid], out, n);
}

int32_t slf_read_positions(const slf_world* world, float* out, uint64_t n) {
    SLF_WORLD(world);
    SLF_TRY(prep_read(world, n));
    if (n) SLF_NEED(out);
    World& w = const_cast<World&>(world->w);
    return w.read_positions(out, n);
}

int32_t slf_read_state(const slf_world* world, float* positions, float* velocities, uint64_t n) {
    SLF_WORLD(world);
    SLF_TRY(prep_read(world, n));
    if (n) {
        SLF_NEED(positions);
        SLF_NEED(velocities);
    }
    World& w = const_cast<World&>(world->w);
    return w.read_state(positions, velocities, n);
}

int32_t slf_read_velocities(const slf_world* world, float* out, uint64_t n) {
    SLF_WORLD(world);
    SLF_TRY(prep_read(world, n));
    if (n) SLF_NEED(out);
    World& w = const_cast<World&>(world->w);
    return w.read_vec(w.vel[w.cpos], out, n);
}

int32_t slf_read_densities(const slf_world* world, float* out, uint64_t n) {
    SLF_WORLD(world);
    SLF_TRY(prep_read(world, n));
    if (n) SLF_NEED(out);
    World& w = const_cast<World&>(world->w);
    return w.read_plain(w.rho[w.cid], out, n);
}

int32_t slf_neighbor_lists(slf_world* world, uint32_t* start, uint64_t start_len, uint32_t* items,
                           uint64_t items_capacity, uint64_t* items_len) {
    SLF_WORLD(world);
    return world->w.lists(false, start, start_len, items, items_capacity, items_len);
}

int32_t slf_wall_neighbor_lists(slf_world* world, uint32_t* start, uint64_t start_len, uint32_t* items,
                                uint64_t items_capacity, uint64_t* items_len) {
    SLF_WORLD(world);
    return world->w.lists(true, start, start_len, items, items_capacity, items_len);
}

int32_t slf_state_hash(const slf_world* world, uint64_t* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    World& w = const_cast<World&>(world->w);
    SLF_TRY(w.flush());
    uint64_t n = w.n;
    std::vector<uint32_t> id(n);
    std::vector<float> p(3 * n), v(3 * n);
    SLF_TRY(w.read_plain(w.ids[w.cid], id.data(), n));
    SLF_TRY(w.read_positions(p.data(), n));
    SLF_TRY(w.read_vec(w.vel[w.cpos], v.data(), n));
    *out = w.state_hash_host(id, p, v);
    return SLF_OK;
}

const char* slf_last_error(void) { return slf::g_error.c_str(); }

int32_t slf_write_state(slf_world* world, const float* positions, const float* velocities, uint64_t n) {
    SLF_WORLD(world);
    if (n) {
        SLF_NEED(positions);
        SLF_NEED(velocities);
    }
    return world->w.write_state(positions, velocities, n);
}

int32_t slf_get_stream(const slf_world* world, void** stream) {
    SLF_WORLD(world);
    SLF_NEED(stream);
    *stream = world->w.stream;
    return SLF_OK;
}

int32_t slf_tape_begin(slf_world* world, uint32_t checkpoint_every) {
    SLF_WORLD(world);
    return world->w.tape_begin(checkpoint_every);
}

int32_t slf_tape_end(slf_world* world) {
    SLF_WORLD(world);
    return world->w.tape_end();
}

int32_t slf_step_backward(slf_world* world, const float* dpositions, const float* dvelocities, uint64_t n,
                          float* dpositions0, float* dvelocities0, slf_param_grads* out) {
    SLF_WORLD(world);
    if (n) {
        SLF_NEED(dpositions);
        SLF_NEED(dvelocities);
    }
    return world->w.step_backward(dpositions, dvelocities, n, dpositions0, dvelocities0, out);
}

int32_t slf_solver_graphs(slf_world* world, int32_t on) {
    SLF_WORLD(world);
    if (on < 0 || on > 2) return fail(SLF_ERR_INVALID_SETTINGS, "graph mode is 0, 1 or 2");
    world->w.graph_mode = on;
    return SLF_OK;
}

int32_t slf_profile_enable(slf_world* world, int32_t on) {
    SLF_WORLD(world);
    World& w = world->w;
    SLF_CUDA(cudaStreamSynchronize(w.stream));
    w.prof.collect();
    w.prof.on = on != 0;
    return SLF_OK;
}

int32_t slf_profile_read(slf_world* world, slf_profile_entry* out, uint32_t capacity, uint32_t* count) {
    SLF_WORLD(world);
    World& w = world->w;
    SLF_CUDA(cudaStreamSynchronize(w.stream));
    w.prof.collect();
    if (count) *count = uint32_t(w.prof.names.size());
    for (uint32_t i = 0; i < capacity && i < w.prof.names.size(); ++i) {
        slf_profile_entry e{};
        std::snprintf(e.name, sizeof(e.name), "%s", w.prof.names[i].c_str());
        e.launches = w.prof.launches[i];
        e.milliseconds = w.prof.ms[i];
        e.algorithmic_bytes = w.prof.bytes[i];
        out[i] = e;
    }
    return SLF_OK;
}

int32_t slf_profile_reset(slf_world* world) {
    SLF_WORLD(world);
    World& w = world->w;
    SLF_CUDA(cudaStreamSynchronize(w.stream));
    w.prof.collect();
    w.prof.reset();
    return SLF_OK;
}

int32_t slf_kernel_launches(uint64_t* out) {
    SLF_NEED(out);
    *out = slf::kernel_launches();
    return SLF_OK;
}

int32_t slf_debug_skip_job(slf_world* world, int64_t job) {
    SLF_WORLD(world);
    world->w.skip_job = job;
    return SLF_OK;
}

int32_t slf_debug_list_room(slf_world* world, uint32_t room) {
    SLF_WORLD(world);
    World& w = world->w;
    SLF_TRY(w.flush());
    w.list_cap = std::max<uint32_t>(8u, room & ~7u);
    w.lists_valid = false;
    return w.n ? w.ensure_work_buffers() : SLF_OK;
}

int32_t slf_last_iterations(const slf_world* world, uint32_t* divergence, uint32_t* density) {
    SLF_WORLD(world);
    if (divergence) *divergence = world->w.last_iterations[0];
    if (density) *density = world->w.last_iterations[1];
    return SLF_OK;
}

int32_t slf_graph_substeps(const slf_world* world, uint64_t* out) {
    SLF_WORLD(world);
    SLF_NEED(out);
    *out = world->w.graph_substeps;
    return SLF_OK;
}

}  // extern "C"
