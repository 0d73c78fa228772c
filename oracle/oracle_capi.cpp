// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points over the CPU restatement in fluid_oracle.hpp, loaded with ctypes by the tests
// and by bench.py's CPU baseline.  The names mirror include/solunar_fluid.h with an `orc_`
// prefix; a handle holds either the float (parity) or the double (precision) restatement.
// Vectors come in as f32 (the library's input type) and go out as f64, which holds either
// precision exactly.
#include <vector>
#include <string>
#include <cstdint>
#include <cstring>
#include <memory>

#include "../include/solunar_fluid.h"
#include "fluid_oracle.hpp"

using namespace oracle;

namespace {

struct Handle {
    int precision = 32;
    World<float> f;
    World<double> d;
};

Settings from_c(const slf_settings* s, int residual_sum) {
    Settings o;
    o.solver = s->solver;
    o.spacing = s->spacing;
    o.rest_density = s->rest_density;
    o.support = s->support;
    o.max_particles = s->max_particles;
    o.sound_speed = s->sound_speed;
    o.viscosity = s->viscosity;
    o.gravity[0] = s->gravity[0];
    o.gravity[1] = s->gravity[1];
    o.gravity[2] = s->gravity[2];
    o.courant = s->courant;
    o.max_substeps = s->max_substeps;
    o.divergence_tolerance = s->divergence_tolerance;
    o.density_tolerance = s->density_tolerance;
    o.min_iterations = s->min_iterations;
    o.max_iterations = s->max_iterations;
    o.residual_sum = residual_sum;
    o.warm_start = s->warm_start;
    return o;
}

template <class R> V3<R> v3(const float* p) { return V3<R>(R(p[0]), R(p[1]), R(p[2])); }

void to_report(const Report& r, slf_report* out) {
    if (!out) return;
    out->substeps = r.substeps;
    out->capped = r.capped;
    out->max_compression = r.max_compression;
    out->max_speed = r.max_speed;
    out->held_back = r.held_back;
    out->iterations = r.iterations;
    out->emitted = r.emitted;
    out->drained = r.drained;
    out->lost = r.lost;
    out->sound_speed = r.sound_speed;
}

template <class R> int32_t read_lists(const Lists& l, uint32_t* start, uint64_t start_len, uint32_t* items,
                                      uint64_t cap, uint64_t* len) {
    if (len) *len = l.items.size();
    if (start) {
        if (start_len != l.start.size()) return INVALID_ARGUMENT;
        std::memcpy(start, l.start.data(), l.start.size() * 4);
    }
    if (items) {
        if (cap < l.items.size()) return INVALID_ARGUMENT;
        std::memcpy(items, l.items.data(), l.items.size() * 4);
    }
    return OK;
}

}  // namespace

// the settings conversion, for the forward-mode runs of oracle_tangent.cpp
Settings settings_from_c(const slf_settings* s, int residual_sum) { return from_c(s, residual_sum); }

#define ORC_DISPATCH(h, ...)                \
    do {                                    \
        if ((h)->precision == 32) {         \
            auto& w = (h)->f;               \
            using R = float;                \
            (void)sizeof(R);                \
            __VA_ARGS__;                    \
        } else {                            \
            auto& w = (h)->d;               \
            using R = double;               \
            (void)sizeof(R);                \
            __VA_ARGS__;                    \
        }                                   \
    } while (0)

template <class W>
int32_t step_bodies(W& w, float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out, slf_body_push* pushes,
                    uint64_t cap, uint64_t* count) {
    using Wd = typename std::decay<W>::type;
    using R = decltype(w.mass);
    std::vector<typename Wd::Pose> ps(npose);
    for (uint64_t k = 0; k < npose; ++k) {
        auto& q = ps[k];
        q.body = poses[k].body;
        for (int a = 0; a < 3; ++a) {
            q.position[a] = poses[k].position[a];
            q.linear[a] = poses[k].linear_velocity[a];
            q.angular[a] = poses[k].angular_velocity[a];
        }
        for (int a = 0; a < 4; ++a) q.rotation[a] = poses[k].rotation[a];
        q.dynamic = poses[k].dynamic;
    }
    Report r;
    std::vector<typename Wd::Push> got;
    int32_t st = w.step_with_bodies(R(dt), ps.data(), ps.size(), r, got);
    to_report(r, out);
    if (count) *count = got.size();
    for (size_t k = 0; k < got.size() && k < cap && pushes; ++k) {
        slf_body_push& o = pushes[k];
        o.body = got[k].body;
        auto put = [](float* d, const auto& v) {
            d[0] = float(v.x);
            d[1] = float(v.y);
            d[2] = float(v.z);
        };
        put(o.lift, got[k].lift);
        put(o.lift_angular, got[k].lift_angular);
        put(o.damping, got[k].damping);
        put(o.damping_angular, got[k].damping_angular);
        o.lifted = got[k].lifted;
    }
    return st;
}

extern "C" {

int32_t orc_create(const slf_settings* s, int32_t precision, int32_t residual_sum, void** out) {
    if (!s || !out) return INVALID_ARGUMENT;
    auto h = std::make_unique<Handle>();
    h->precision = precision == 64 ? 64 : 32;
    Settings o = from_c(s, residual_sum);
    Status st = h->precision == 32 ? World<float>::create(o, h->f) : World<double>::create(o, h->d);
    if (st != OK) return st;
    *out = h.release();
    return OK;
}

void orc_destroy(void* p) { delete static_cast<Handle*>(p); }

int32_t orc_set_threads(void* p, int32_t threads) {
    auto* h = static_cast<Handle*>(p);
    h->f.threads = threads;
    h->d.threads = threads;
    return OK;
}

int32_t orc_len(void* p, uint64_t* out) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *out = w.len());
    return OK;
}

int32_t orc_particle_mass(void* p, double* out) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *out = double(w.mass));
    return OK;
}

int32_t orc_kernel(void* p, double* radius, double* scale) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, (*radius = double(w.kernel.radius), *scale = double(w.kernel.scale)));
    return OK;
}

int32_t orc_add_particles(void* p, uint64_t n, const float* pos, const float* vel, uint32_t* ids) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        for (uint64_t i = 0; i < n && st == OK; ++i)
            st = w.add_particle(v3<R>(pos + 3 * i), v3<R>(vel + 3 * i), ids ? ids + i : nullptr);
    });
    return st;
}

int32_t orc_fill_box(void* p, const float* low, const float* high, uint64_t* count) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.fill_box(v3<R>(low), v3<R>(high), count));
    return st;
}

int32_t orc_set_domain(void* p, const float* low, const float* high) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        if (low && high) {
            auto a = v3<R>(low), b = v3<R>(high);
            st = w.set_domain(&a, &b);
        } else {
            st = w.set_domain(nullptr, nullptr);
        }
    });
    return st;
}

int32_t orc_add_box_container(void* p, const float* low, const float* high, uint32_t* id) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.add_box_container(v3<R>(low), v3<R>(high), id));
    return st;
}

int32_t orc_add_wall(void* p, const float* low, const float* high, uint32_t* id) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.add_wall(v3<R>(low), v3<R>(high), id));
    return st;
}

int32_t orc_remove_boundary(void* p, uint32_t id, int32_t* removed) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *removed = w.remove_boundary(id) ? 1 : 0);
    return OK;
}

int32_t orc_add_emitter(void* p, const float* low, const float* high, const float* velocity, uint32_t* id) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.add_emitter(v3<R>(low), v3<R>(high), v3<R>(velocity), id));
    return st;
}

int32_t orc_add_drain(void* p, const float* low, const float* high, uint32_t* id) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.add_drain(v3<R>(low), v3<R>(high), id));
    return st;
}

int32_t orc_remove_flow(void* p, uint32_t id, int32_t* removed) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *removed = w.remove_flow(id) ? 1 : 0);
    return OK;
}

int32_t orc_run_flows(void* p, uint32_t* emitted, uint32_t* drained) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.run_flows(*emitted, *drained));
    return st;
}

int32_t orc_terrain_nodes(void* p, const float* low, const float* high, uint64_t* nodes) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    size_t nd[3] = {0, 0, 0};
    ORC_DISPATCH(h, st = w.terrain_nodes(v3<R>(low), v3<R>(high), nd));
    for (int a = 0; a < 3; ++a) nodes[a] = nd[a];
    return st;
}

int32_t orc_add_terrain(void* p, const float* low, const float* high, const float* distances, uint64_t count,
                        uint32_t* id) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.add_terrain(v3<R>(low), v3<R>(high), distances, size_t(count), id));
    return st;
}

// Probes of one terrain region (the reference's unit tests read them): the field's distance and
// way out at a point, and the ground a particle there sees.  *inside = 0 outside the region.
int32_t orc_terrain_probe(void* p, uint32_t region, const float* point, double* distance, double* normal,
                          double* density, double* gradient, int32_t* inside) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        if (region >= w.terrains.size()) {
            st = INVALID_ARGUMENT;
        } else {
            R d, rho;
            V3<R> n, g;
            bool in = w.terrain_ground(w.terrains[region], v3<R>(point), d, n, rho, g);
            *inside = in ? 1 : 0;
            if (in) {
                *distance = double(d);
                normal[0] = double(n.x), normal[1] = double(n.y), normal[2] = double(n.z);
                *density = double(rho);
                gradient[0] = double(g.x), gradient[1] = double(g.y), gradient[2] = double(g.z);
            }
        }
    });
    return st;
}

static std::string g_snapshot_message;

int32_t orc_save_snapshot(void* p, uint8_t* out, uint64_t capacity, uint64_t* size) {
    auto* h = static_cast<Handle*>(p);
    std::vector<uint8_t> bytes;
    ORC_DISPATCH(h, bytes = w.save_snapshot());
    *size = bytes.size();
    if (!out) return OK;
    if (capacity < bytes.size()) return INVALID_ARGUMENT;
    std::memcpy(out, bytes.data(), bytes.size());
    return OK;
}

int32_t orc_load_snapshot(const uint8_t* data, uint64_t size, const slf_settings* s, int32_t precision,
                          int32_t residual_sum, void** out) {
    if (!s || !out) return INVALID_ARGUMENT;
    auto h = std::make_unique<Handle>();
    h->precision = precision == 64 ? 64 : 32;
    Settings base = from_c(s, residual_sum);
    g_snapshot_message.clear();
    Status st = h->precision == 32 ? World<float>::load_snapshot(data, size, base, h->f, g_snapshot_message)
                                   : World<double>::load_snapshot(data, size, base, h->d, g_snapshot_message);
    if (st != OK) return st;
    *out = h.release();
    return OK;
}

const char* orc_snapshot_message() { return g_snapshot_message.c_str(); }

int32_t orc_wall_count(void* p, uint64_t* out) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *out = w.walls.positions.size());
    return OK;
}

int32_t orc_read_wall_positions(void* p, double* out, uint64_t n) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        if (n != w.walls.positions.size()) {
            st = INVALID_ARGUMENT;
        } else {
            for (uint64_t i = 0; i < n; ++i) {
                out[3 * i] = double(w.walls.positions[i].x);
                out[3 * i + 1] = double(w.walls.positions[i].y);
                out[3 * i + 2] = double(w.walls.positions[i].z);
            }
        }
    });
    return st;
}

int32_t orc_step(void* p, float dt, slf_report* out) {
    auto* h = static_cast<Handle*>(p);
    Report r;
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.step(R(dt), r));
    to_report(r, out);
    return st;
}

int32_t orc_couple(void* p, uint64_t body, int32_t shape, const float* dims) {
    auto* h = static_cast<Handle*>(p);
    if (!dims) return INVALID_ARGUMENT;
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.couple(body, shape, dims));
    return st;
}

int32_t orc_uncouple(void* p, uint64_t body, int32_t* removed) {
    auto* h = static_cast<Handle*>(p);
    bool r = false;
    ORC_DISPATCH(h, r = w.uncouple(body));
    if (removed) *removed = r ? 1 : 0;
    return OK;
}

int32_t orc_coupled(void* p, uint64_t* bodies, uint32_t* points, uint32_t* probes, uint64_t cap, uint64_t* count) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, {
        if (count) *count = w.coupled.size();
        for (size_t k = 0; k < w.coupled.size() && k < cap; ++k) {
            if (bodies) bodies[k] = w.coupled[k].body;
            if (points) points[k] = uint32_t(w.coupled[k].points.size());
            if (probes) probes[k] = uint32_t(w.coupled[k].probes.size());
        }
    });
    return OK;
}

int32_t orc_step_with_bodies(void* p, float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out,
                             slf_body_push* pushes, uint64_t cap, uint64_t* count) {
    auto* h = static_cast<Handle*>(p);
    if (npose && !poses) return INVALID_ARGUMENT;
    int32_t st = OK;
    ORC_DISPATCH(h, st = step_bodies(w, dt, poses, npose, out, pushes, cap, count));
    return st;
}

int32_t orc_update_neighbors(void* p) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, w.update_neighbors());
    return OK;
}

int32_t orc_compute_densities(void* p) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = w.compute_densities());
    return st;
}

int32_t orc_read_ids(void* p, uint32_t* out, uint64_t n) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        if (n != w.len()) st = INVALID_ARGUMENT;
        else std::memcpy(out, w.ids.data(), n * 4);
    });
    return st;
}

static int32_t read_vecs(Handle* h, int which, double* out, uint64_t n) {
    int32_t st = OK;
    ORC_DISPATCH(h, {
        const auto& src = which == 0 ? w.positions : w.velocities;
        if (n != src.size()) {
            st = INVALID_ARGUMENT;
        } else {
            for (uint64_t i = 0; i < n; ++i) {
                out[3 * i] = double(src[i].x);
                out[3 * i + 1] = double(src[i].y);
                out[3 * i + 2] = double(src[i].z);
            }
        }
    });
    return st;
}

int32_t orc_read_positions(void* p, double* out, uint64_t n) { return read_vecs(static_cast<Handle*>(p), 0, out, n); }
int32_t orc_read_velocities(void* p, double* out, uint64_t n) { return read_vecs(static_cast<Handle*>(p), 1, out, n); }

int32_t orc_read_densities(void* p, double* out, uint64_t n) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, {
        if (n != w.len()) st = INVALID_ARGUMENT;
        else
            for (uint64_t i = 0; i < n; ++i) out[i] = double(w.densities[i]);
    });
    return st;
}

int32_t orc_neighbor_lists(void* p, uint32_t* start, uint64_t start_len, uint32_t* items, uint64_t cap,
                           uint64_t* len) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = read_lists<R>(w.neighbors, start, start_len, items, cap, len));
    return st;
}

int32_t orc_wall_neighbor_lists(void* p, uint32_t* start, uint64_t start_len, uint32_t* items, uint64_t cap,
                                uint64_t* len) {
    auto* h = static_cast<Handle*>(p);
    int32_t st = OK;
    ORC_DISPATCH(h, st = read_lists<R>(w.wall_neighbors, start, start_len, items, cap, len));
    return st;
}

int32_t orc_state_hash(void* p, uint64_t* out) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, *out = w.state_hash());
    return OK;
}

int32_t orc_last_iterations(void* p, uint32_t* out) {
    auto* h = static_cast<Handle*>(p);
    ORC_DISPATCH(h, (out[0] = w.last_iterations[0], out[1] = w.last_iterations[1]));
    return OK;
}

// Kernel::value / slope / gradient of a kernel with this radius (mod.rs:125-165), float.
int32_t orc_kernel_eval_f32(float radius, uint64_t n, const float* offsets, float* value, float* slope,
                            float* gradient) {
    Kernel<float> k(radius);
    for (uint64_t i = 0; i < n; ++i) {
        V3<float> o(offsets[3 * i], offsets[3 * i + 1], offsets[3 * i + 2]);
        float d = length(o);
        value[i] = k.value(d);
        slope[i] = k.slope(d);
        V3<float> g = k.gradient(o);
        gradient[3 * i] = g.x;
        gradient[3 * i + 1] = g.y;
        gradient[3 * i + 2] = g.z;
    }
    return OK;
}

// Grid::build over sorted keys, then Grid::range for each query (mod.rs:169-247).
// out[2*i], out[2*i+1] = range, or UINT32_MAX twice when the cell is absent.  force_search
// drops the dense table.  *dense_out tells whether a dense table was built.
int32_t orc_grid_ranges(const int32_t* keys, uint64_t n, const int32_t* queries, uint64_t nq, int32_t force_search,
                        uint32_t* out, int32_t* dense_out) {
    std::vector<Key> k(n);
    for (uint64_t i = 0; i < n; ++i) k[i] = Key{keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]};
    Grid g = Grid::build(k);
    if (dense_out) *dense_out = g.dense.empty() ? 0 : 1;
    if (force_search) g.dense.clear();
    for (uint64_t i = 0; i < nq; ++i) {
        Range r;
        if (g.range(Key{queries[3 * i], queries[3 * i + 1], queries[3 * i + 2]}, r)) {
            out[2 * i] = r.begin;
            out[2 * i + 1] = r.end;
        } else {
            out[2 * i] = UINT32_MAX;
            out[2 * i + 1] = UINT32_MAX;
        }
    }
    return OK;
}

}  // extern "C"
